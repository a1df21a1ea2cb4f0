// Per-grain sequential routines (one thread runs one grain).  Each follows a
// reference routine operation for operation so the FP64 form reproduces the
// reference's arithmetic; the cited file:line is the routine it restates.
#pragma once

#include <math.h>

#include "gg_device.cuh"

namespace gg {
namespace {  // internal linkage: each form's translation unit has its own copy


constexpr double kPi = 3.14159265358979323846;  // PI, src/ggLS.h:26

// ---------------------------------------------------------------------------
// Marching squares (src/marchingSquares.cpp:28-301)
// ---------------------------------------------------------------------------
enum : int { MS_UP = 0, MS_DOWN = 1, MS_LEFT = 2, MS_RIGHT = 3, MS_NONE = 4 };
enum : int { C_TL = 1, C_TR = 2, C_BL = 4, C_BR = 8 };

template <typename R>
struct Field {
    const R* v;  // row-major values of box b
    Box b;
    // isInside (src/marchingSquares.cpp:189-196)
    __device__ __forceinline__ bool inside(int row, int col) const {
        if (row < b.y0 || row >= b.y1 || col < b.x0 || col >= b.x1) return false;
        return (double)v[(row - b.y0) * (b.x1 - b.x0) + (col - b.x0)] >= 0;
    }
    __device__ __forceinline__ double at(int row, int col) const {
        return (double)v[(row - b.y0) * (b.x1 - b.x0) + (col - b.x0)];
    }
};

struct ContourOut {
    CPoint* pts;
    int cap;
    int n;
    Junction* js;
    int jcap;
    int jn;
    uint32_t status;
};

__device__ __forceinline__ void ms_insert(ContourOut& o, double x, double y) {
    // insertPoint (src/marchingSquares.cpp:197-203)
    if (o.n == 0 || x != o.pts[o.n - 1].x || y != o.pts[o.n - 1].y) {
        if (o.n >= o.cap) {
            o.status |= S_CONTOUR_OVERFLOW;
            return;
        }
        o.pts[o.n].x = x;
        o.pts[o.n].y = y;
        o.pts[o.n].energy = -1.0;  // SPoint result(-1,-1,-1,-1)
        o.pts[o.n].mob = -1.0;
        o.n++;
    }
}

// generatePoint (src/marchingSquares.cpp:204-265)
template <typename R>
__device__ __forceinline__ void ms_point(const Field<R>& f, int dir, int top, int bottom, int left, int right,
                                         double* px, double* py) {
    double delta, position;
    switch (dir) {
        case MS_LEFT:
            *px = left;
            if (top < f.b.y0) {
                *py = bottom;
            } else {
                delta = f.at(bottom, left) - f.at(top, left);
                position = bottom - f.at(bottom, left) / delta;
                *py = position;
            }
            break;
        case MS_RIGHT:
            *px = right;
            if (bottom >= f.b.y1) {
                *py = top;
            } else {
                delta = f.at(top, right) - f.at(bottom, right);
                position = top + f.at(top, right) / delta;
                *py = position;
            }
            break;
        case MS_UP:
            *py = top;
            if (right >= f.b.x1) {
                *px = left;
            } else {
                delta = f.at(top, left) - f.at(top, right);
                position = left + f.at(top, left) / delta;
                *px = position;
            }
            break;
        default:  // MS_DOWN
            *py = bottom;
            if (left < f.b.x0) {
                *px = right;
            } else {
                delta = f.at(bottom, right) - f.at(bottom, left);
                position = right - f.at(bottom, right) / delta;
                *px = position;
            }
            break;
    }
}

__device__ __forceinline__ void insert_distinct(uint32_t v, uint32_t* arr, int& cnt) {
    // insertDistinctInteger (src/marchingSquares.cpp:303-318)
    bool found = false;
    for (int i = 0; i < cnt; i++) {
        if (arr[i] == v) {
            found = true;
            break;
        }
    }
    if (!found) {
        arr[cnt] = v;
        cnt++;
    }
}

// generateJunction (src/marchingSquares.cpp:266-301); idl is the IDLocal
// buffer over the same box as the field.
template <typename R>
__device__ __forceinline__ void ms_junction(const Field<R>& f, const uint32_t* idl, uint32_t own, int mask, int top,
                                            int bottom, int left, int right, ContourOut& o) {
    const Box& b = f.b;
    if (bottom < b.y0 || bottom >= b.y1 || top < b.y0 || top >= b.y1 || left < b.x0 || left >= b.x1 ||
        right < b.x0 || right >= b.x1)
        return;
    const int w = b.x1 - b.x0;
    uint32_t boxes[4] = {0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu};
    int order = 0;
    insert_distinct((mask & C_BL) ? own : idl[(bottom - b.y0) * w + (left - b.x0)], boxes, order);
    insert_distinct((mask & C_TL) ? own : idl[(top - b.y0) * w + (left - b.x0)], boxes, order);
    insert_distinct((mask & C_BR) ? own : idl[(bottom - b.y0) * w + (right - b.x0)], boxes, order);
    insert_distinct((mask & C_TR) ? own : idl[(top - b.y0) * w + (right - b.x0)], boxes, order);
    if (order > 2) {
        if (o.jn >= o.jcap) {
            o.status |= S_JUNCTION_OVERFLOW;
            return;
        }
        Junction& j = o.js[o.jn++];
        j.type = order;
        for (int q = 0; q < 4; ++q) j.grains[q] = q < order ? boxes[q] : 0xFFFFFFFFu;
        j.segment = -1;
        j.lambda = 0;
        j.x = left + 0.5;
        j.y = top + 0.5;
    }
}

// MarchingSquaresAlgorithm::generateContour (src/marchingSquares.cpp:28-188).
// Returns false when no pixel of the box has phi >= 0.  The walk is bounded
// by 4 (w+2)(h+2) + 16 moves (the reference's loop has no bound).
template <typename R>
__device__ bool ms_contour(const Field<R>& f, const uint32_t* idl, uint32_t own, ContourOut& o) {
    o.n = 0;
    o.jn = 0;
    int startX = -1, startY = -1;
    for (int i = f.b.y0; i < f.b.y1 && startX < 0; i++) {
        for (int j = f.b.x0; j < f.b.x1; j++) {
            if (f.inside(i, j)) {
                startX = j;
                startY = i;
                break;
            }
        }
    }
    if (startX == startY && startX == -1) return false;

    int left = startX - 1, right = startX, top = startY - 1, bottom = startY;
    int next = MS_NONE, prev = MS_NONE;
    const long limit = 4L * (box_w(f.b) + 2) * (box_h(f.b) + 2) + 16;
    long it = 0;
    do {
        int mask = 0;
        if (f.inside(top, left)) mask |= C_TL;
        if (f.inside(top, right)) mask |= C_TR;
        if (f.inside(bottom, left)) mask |= C_BL;
        if (f.inside(bottom, right)) mask |= C_BR;
        bool emit = true;
        switch (mask) {
            case C_TL: next = MS_UP; break;
            case C_TR: next = MS_RIGHT; break;
            case C_TL | C_TR: next = MS_RIGHT; break;
            case C_BL: next = MS_LEFT; break;
            case C_BL | C_TL: next = MS_UP; break;
            case C_BL | C_TR:
                next = (prev == MS_UP) ? MS_RIGHT : MS_LEFT;
                emit = false;
                break;
            case C_BL | C_TR | C_TL: next = MS_RIGHT; break;
            case C_BR: next = MS_DOWN; break;
            case C_BR | C_TL:
                next = (prev == MS_RIGHT) ? MS_DOWN : MS_UP;
                emit = false;
                break;
            case C_BR | C_TR: next = MS_DOWN; break;
            case C_BR | C_TR | C_TL: next = MS_DOWN; break;
            case C_BR | C_BL: next = MS_LEFT; break;
            case C_BR | C_BL | C_TL: next = MS_UP; break;
            case C_BR | C_BL | C_TR: next = MS_LEFT; break;
            default: emit = false; break;  // 0 or 15: direction unchanged
        }
        if (emit) {
            double px, py;
            ms_point(f, next, top, bottom, left, right, &px, &py);
            ms_insert(o, px, py);
        }
        ms_junction(f, idl, own, mask, top, bottom, left, right, o);
        switch (next) {
            case MS_UP: top--; bottom--; break;
            case MS_DOWN: top++; bottom++; break;
            case MS_LEFT: left--; right--; break;
            case MS_RIGHT: left++; right++; break;
            default: break;
        }
        prev = next;
        if (++it > limit) {
            o.status |= S_WALK_LIMIT;
            break;
        }
    } while (left != startX - 1 || bottom != startY);

    if (o.n > 0) {
        if (o.pts[0].x != o.pts[o.n - 1].x || o.pts[0].y != o.pts[o.n - 1].y) {
            if (o.n >= o.cap) {
                o.status |= S_CONTOUR_OVERFLOW;
            } else {
                o.pts[o.n] = o.pts[0];
                o.n++;
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Contour geometry (src/grainBoundary.cpp)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double len_sqr(double x, double y) { return x * x + y * y; }

// PERIODIC(x) of src/grainBoundary.cpp:26 (size_t arithmetic modulo size-1).
// The walks only pass x in [-(size-1), 2(size-1)), where a conditional add or
// subtract gives the same value as the unsigned 64-bit remainder.
__device__ __forceinline__ int periodic(int x, int size) {
    const int m = size - 1;
    if (x >= -m && x < 2 * m) {
        if (x < 0) return x + m;
        if (x >= m) return x - m;
        return x;
    }
    const unsigned long long mm = (unsigned long long)m;
    return (int)(((unsigned long long)(long long)x + mm) % mm);
}

// (j + 1 + real) % real and (j - 1 + real) % real for j in [0, real).
__device__ __forceinline__ int wrap_next(int j, int real) { return j + 1 >= real ? j + 1 - real : j + 1; }
__device__ __forceinline__ int wrap_prev(int j, int real) { return j - 1 < 0 ? j - 1 + real : j - 1; }

// Second half of ExplicitGrainBoundary::projectToGrainBondary
// (src/grainBoundary.cpp:383-420): given the nearest vertex, the closer of
// its two adjacent segments (the following one first, strict <) and the
// clamped lambda on it.  *out_lambda keeps its value if no segment is closer
// than 1e6 (as the reference's out_lambda).
__device__ __forceinline__ int segment_of_vertex(const CPoint* P, int asize, double px, double py, int nearest,
                                                 double* out_lambda) {
    double lam_out = *out_lambda;
    int minimal_segment = nearest;
    double minDist = 1000000.0, dist;
    int next = nearest + 1;
    double ux = P[next].x - P[nearest].x, uy = P[next].y - P[nearest].y;
    double lambda = (px - P[nearest].x) * ux + (py - P[nearest].y) * uy;
    lambda /= (ux * ux + uy * uy);
    if (lambda < 0)
        dist = len_sqr(px - P[nearest].x, py - P[nearest].y);
    else if (lambda > 1)
        dist = len_sqr(P[next].x - px, P[next].y - py);
    else
        dist = len_sqr(px - (P[nearest].x + ux * lambda), py - (P[nearest].y + uy * lambda));
    if (dist < minDist) {
        minimal_segment = nearest;
        minDist = dist;
        lam_out = lambda;
    }
    if (nearest == 0) nearest = asize - 1;
    int previous = nearest - 1;
    ux = P[nearest].x - P[previous].x;
    uy = P[nearest].y - P[previous].y;
    lambda = (px - P[previous].x) * ux + (py - P[previous].y) * uy;
    lambda /= (ux * ux + uy * uy);
    if (lambda < 0)
        dist = len_sqr(px - P[previous].x, py - P[previous].y);
    else if (lambda > 1)
        dist = len_sqr(P[nearest].x - px, P[nearest].y - py);
    else
        dist = len_sqr(px - (P[previous].x + ux * lambda), py - (P[previous].y + uy * lambda));
    if (dist < minDist) {
        minimal_segment = previous;
        minDist = dist;
        lam_out = lambda;
    }
    if (lam_out > 1) lam_out = 1;
    if (lam_out < 0) lam_out = 0;
    *out_lambda = lam_out;
    return minimal_segment;
}

// ExplicitGrainBoundary::projectToGrainBondary (src/grainBoundary.cpp:365-447):
// the first vertex at the smallest squared distance (strict <), then
// segment_of_vertex.
__device__ int project_to_boundary(const CPoint* P, int asize, double px, double py, double* out_lambda) {
    double minDist = 1000000.0;
    double dist = 0;
    int nearest = -1;
    for (int k = 0; k < asize - 1; k++) {
        dist = len_sqr(px - P[k].x, py - P[k].y);
        if (dist < minDist) {
            nearest = k;
            minDist = dist;
        }
    }
    if (nearest < 0) return 0;  // fewer than two contour points: nothing to project on
    return segment_of_vertex(P, asize, px, py, nearest, out_lambda);
}

// Junction projection of extractBoundaryAndJunctions (src/grainBoundary.cpp:51-61)
__device__ void project_junctions(const CPoint* P, int n, Junction* js, int jn) {
    if (n < 2) return;
    double lambda = 0.0;  // one variable for all junctions, as in the reference
    for (int i = 0; i < jn; ++i) {
        int seg = project_to_boundary(P, n, js[i].x, js[i].y, &lambda);
        const int nx = periodic(seg + 1, n);
        js[i].x = P[seg].x + (P[nx].x - P[seg].x) * lambda;
        js[i].y = P[seg].y + (P[nx].y - P[seg].y) * lambda;
        js[i].segment = seg;
        js[i].lambda = lambda;
    }
}

// computeVolume (src/grainBoundary.cpp:201-213)
__device__ __forceinline__ double contour_volume(const CPoint* P, int n, double h) {
    double v = 0;
    for (int i = 0; i < n - 1; i++) v += (P[i].y + P[i + 1].y) * (P[i].x - P[i + 1].x);
    return fabs(v) * h * h * 0.5;
}

// computePerimeter (src/grainBoundary.cpp:224-231)
__device__ __forceinline__ double contour_perimeter(const CPoint* P, int n, double h) {
    double p = 0;
    for (int i = 0; i < n - 1; i++) {
        const double dx = P[i].x - P[i + 1].x, dy = P[i].y - P[i + 1].y;
        p += sqrt(dx * dx + dy * dy) * h;
    }
    return p;
}

// computeEnergy (src/grainBoundary.cpp:215-222)
__device__ __forceinline__ double contour_energy(const CPoint* P, int n, double h) {
    double e = 0;
    for (int i = 0; i < n - 1; i++) {
        const double dx = P[i].x - P[i + 1].x, dy = P[i].y - P[i + 1].y;
        e += sqrt(dx * dx + dy * dy) * P[i].energy * h;
    }
    return e;
}

// LSbox::isMotionRegular (src/box.cpp:1155-1190); *flag_irregular is set in
// the grey zone where the reference clears m_isMotionRegular.
__device__ __forceinline__ bool motion_regular(int old_contour, int new_contour, double old_volume, double new_volume,
                                               double dt, int* flag_irregular) {
    double mullins = (new_volume - old_volume) / dt * (3 / kPi);
    double contourRatio = ((double)new_contour) / old_contour;
    double volumeRatio = new_volume / old_volume;
    if (mullins > -6.0) return true;
    if (volumeRatio < 0.10) return false;
    if (contourRatio < 0.35) return false;
    if (contourRatio > 0.7) return true;
    *flag_irregular = 1;
    return true;
}

// DimensionalBuffer::resizeToSquare (src/dimensionalBuffer.h:123-160)
__device__ __forceinline__ Box resize_to_square(Box r, int maximumLength) {
    int grid_size = maximumLength - 1;
    unsigned int height = r.y1 - r.y0;
    unsigned int width = r.x1 - r.x0;
    if (width == height) return r;
    if (width > height) {
        int diff = width - height;
        r.y0 -= diff / 2;
        r.y1 += diff / 2 + diff % 2;
    } else {
        int diff = height - width;
        r.x0 -= diff / 2;
        r.x1 += diff / 2 + diff % 2;
    }
    if (r.x0 < 0) {
        int d = -r.x0;
        r.x1 += d;
        r.x0 += d;
    } else if (r.x1 > grid_size) {
        int d = grid_size - r.x1;
        r.x1 += d;
        r.x0 += d;
    }
    if (r.y0 < 0) {
        int d = -r.y0;
        r.y1 += d;
        r.y0 += d;
    } else if (r.y1 > grid_size) {
        int d = grid_size - r.y1;
        r.y1 += d;
        r.y0 += d;
    }
    return r;
}

// ---------------------------------------------------------------------------
// Physics (src/box.cpp:1766-1865, src/Quaternion.cpp:58-70, 309-367)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double misorientation_cubic(const double* p, const double* q) {
    // misorientationCubicQxQ: r = inverse(p) * q, then the largest |component|
    // over the 24 cubic symmetry variants (six fundamental quaternions).
    const double a0 = p[0], a1 = -p[1], a2 = -p[2], a3 = -p[3];
    const double b0 = q[0], b1 = q[1], b2 = q[2], b3 = q[3];
    const double a = +a0 * b0 - a1 * b1 - a2 * b2 - a3 * b3;
    const double b = +a1 * b0 + a0 * b1 - a3 * b2 + a2 * b3;
    const double c = +a2 * b0 + a3 * b1 + a0 * b2 - a1 * b3;
    const double d = +a3 * b0 - a2 * b1 + a1 * b2 + a0 * b3;
    const double fac = 1.0 / sqrt(2.0);
    double r[24] = {(a + b) * fac,           (a - b) * fac,           (c + d) * fac,           (c - d) * fac,
                    (a + c) * fac,           (a - c) * fac,           (b + d) * fac,           (b - d) * fac,
                    (a + d) * fac,           (a - d) * fac,           (b + c) * fac,           (b - c) * fac,
                    (a + b + c + d) * 0.5,   (a + b - c - d) * 0.5,   (a - b + c - d) * 0.5,   (a - b - c + d) * 0.5,
                    (a + b + c - d) * 0.5,   (a + b - c + d) * 0.5,   (a - b + c + d) * 0.5,   (a - b - c - d) * 0.5,
                    a,                       b,                       c,                       d};
    double omega = 0.0;
    for (int i = 0; i < 24; i++)
        if (fabs(r[i]) > omega) omega = fabs(r[i]);
    if (omega > 1.0) omega = (double)(int)omega;
    return 2 * acos(omega);
}

// LSbox::computeMisorientation (src/box.cpp:1766-1783): floored at 1 degree.
__device__ __forceinline__ double grain_misorientation(const double* p, const double* q) {
    double r = misorientation_cubic(p, q);
    if (r > 1 * kPi / 180.0) return r;
    return 1 * kPi / 180.0;
}

// LSbox::GBEnergyReadShockley (src/box.cpp:1785-1823), ResearchMode 0.
__device__ __forceinline__ double read_shockley(double theta, const NetConst& C) {
    if (C.isotropic) return 1.0;
    const double gamma_hagb = C.gamma_hagb;
    const double theta_ref = C.theta_ref;
    double gamma;
    if (theta > theta_ref) {
        gamma = gamma_hagb;
    } else {
        if (theta < 1.0 * kPi / 180.0) theta = 1.0 * kPi / 180.0;
        gamma = gamma_hagb * (theta / theta_ref) * (1.0 - log(theta / theta_ref));
        if (gamma != gamma) gamma = 0.01;
    }
    return gamma;
}

// LSbox::GBmobilityModel (src/box.cpp:1825-1865), models 0 and 1, no twins.
__device__ __forceinline__ double mobility_model(double theta, const NetConst& C) {
    if (C.use_mobility_model == 0 || C.isotropic) return 1.0;
    // model 1: 1 - 0.99 exp(-5 (theta / theta_ref)^9), scaled by m_HAGB
    const double m = 1 - (0.99 * exp(-5.0 * (pow(theta / C.theta_ref, 9.0))));
    return C.m_hagb * m;
}

}  // namespace
}  // namespace gg
