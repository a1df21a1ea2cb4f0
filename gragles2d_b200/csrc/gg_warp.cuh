// Warp-per-grain versions of the per-grain sequential stages (level set,
// volume/energy/neighbours, second-order lists).  The parts of each
// reference routine that are independent per pixel, per contour point or per
// list entry run across the 32 lanes; every order-dependent part (the
// marching-squares walk, list construction, sums) runs on lane 0 in the
// reference's order, so the FP64 form stays bit-identical.
#pragma once

#include "gg_grain.cuh"
#include "gg_kernels.cuh"

namespace gg {
namespace {  // internal linkage: each form's translation unit has its own copy

constexpr int kGrainsPerBlock = 4;  // warps (grains) per CTA of the warp kernels

__device__ __forceinline__ int warp_min_i(int v) {
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// First pixel of the box (row-major) with phi >= 0, as the scan of
// generateContour (src/marchingSquares.cpp:32-42); -1 if none.
template <typename R>
__device__ int first_inside_warp(const Field<R>& f, int lane) {
    const int w = box_w(f.b), h = box_h(f.b);
    for (int r = 0; r < h; ++r) {
        int best = 0x7fffffff;
        for (int c = lane; c < w; c += 32)
            if ((double)f.v[r * w + c] >= 0) {
                best = c;
                break;
            }
        best = warp_min_i(best);
        if (best != 0x7fffffff) return r * w + best;
    }
    return -1;
}

// Marching-squares walk from a known start pixel (src/marchingSquares.cpp:44-187).
// The four corner values of the current square are kept in registers and
// only the two corners a move uncovers are loaded; the last emitted point
// is kept in registers for insertPoint's duplicate test; junction corners
// are only read where a junction is possible (at most two inside corners).
template <typename R>
__device__ void ms_walk(const Field<R>& f, const uint32_t* idl, uint32_t own, int startX, int startY,
                        ContourOut& o, double2* xy) {
    o.n = 0;
    o.jn = 0;
    const Box b = f.b;
    const int w = b.x1 - b.x0;
    auto val = [&](int row, int col, double* v) -> bool {  // value and isInside
        if (row < b.y0 || row >= b.y1 || col < b.x0 || col >= b.x1) {
            *v = -1.0;
            return false;
        }
        *v = (double)f.v[(row - b.y0) * w + (col - b.x0)];
        return *v >= 0;
    };
    int left = startX - 1, right = startX, top = startY - 1, bottom = startY;
    double vTL, vTR, vBL, vBR;
    bool iTL = val(top, left, &vTL), iTR = val(top, right, &vTR);
    bool iBL = val(bottom, left, &vBL), iBR = val(bottom, right, &vBR);
    int next = MS_NONE, prev = MS_NONE;
    double lastx = 0, lasty = 0, firstx = 0, firsty = 0;
    const long limit = 4L * (w + 2) * (box_h(b) + 2) + 16;
    long it = 0;
    do {
        int mask = 0;
        if (iTL) mask |= C_TL;
        if (iTR) mask |= C_TR;
        if (iBL) mask |= C_BL;
        if (iBR) mask |= C_BR;
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
            default: emit = false; break;
        }
        if (emit) {  // generatePoint (src/marchingSquares.cpp:204-265) on the cached corners
            double px, py, delta, position;
            switch (next) {
                case MS_LEFT:
                    px = left;
                    if (top < b.y0) {
                        py = bottom;
                    } else {
                        delta = vBL - vTL;
                        position = bottom - vBL / delta;
                        py = position;
                    }
                    break;
                case MS_RIGHT:
                    px = right;
                    if (bottom >= b.y1) {
                        py = top;
                    } else {
                        delta = vTR - vBR;
                        position = top + vTR / delta;
                        py = position;
                    }
                    break;
                case MS_UP:
                    py = top;
                    if (right >= b.x1) {
                        px = left;
                    } else {
                        delta = vTL - vTR;
                        position = left + vTL / delta;
                        px = position;
                    }
                    break;
                default:
                    py = bottom;
                    if (left < b.x0) {
                        px = right;
                    } else {
                        delta = vBR - vBL;
                        position = right - vBR / delta;
                        px = position;
                    }
                    break;
            }
            if (o.n == 0 || px != lastx || py != lasty) {  // insertPoint
                if (o.n >= o.cap) {
                    o.status |= S_CONTOUR_OVERFLOW;
                } else {
                    if (xy) {
                        xy[o.n] = make_double2(px, py);
                    } else {
                        CPoint& q = o.pts[o.n];
                        q.x = px;
                        q.y = py;
                        q.energy = -1.0;
                        q.mob = -1.0;
                    }
                    if (o.n == 0) {
                        firstx = px;
                        firsty = py;
                    }
                    o.n++;
                    lastx = px;
                    lasty = py;
                }
            }
        }
        if (__popc(mask) < 3) ms_junction(f, idl, own, mask, top, bottom, left, right, o);
        switch (next) {
            case MS_UP:
                top--;
                bottom--;
                vBL = vTL;
                vBR = vTR;
                iBL = iTL;
                iBR = iTR;
                iTL = val(top, left, &vTL);
                iTR = val(top, right, &vTR);
                break;
            case MS_DOWN:
                top++;
                bottom++;
                vTL = vBL;
                vTR = vBR;
                iTL = iBL;
                iTR = iBR;
                iBL = val(bottom, left, &vBL);
                iBR = val(bottom, right, &vBR);
                break;
            case MS_LEFT:
                left--;
                right--;
                vTR = vTL;
                vBR = vBL;
                iTR = iTL;
                iBR = iBL;
                iTL = val(top, left, &vTL);
                iBL = val(bottom, left, &vBL);
                break;
            case MS_RIGHT:
                left++;
                right++;
                vTL = vTR;
                vBL = vBR;
                iTL = iTR;
                iBL = iBR;
                iTR = val(top, right, &vTR);
                iBR = val(bottom, right, &vBR);
                break;
            default: break;
        }
        prev = next;
        if (++it > limit) {
            o.status |= S_WALK_LIMIT;
            break;
        }
    } while (left != startX - 1 || bottom != startY);
    if (o.n > 0 && (firstx != lastx || firsty != lasty)) {
        if (o.n >= o.cap) {
            o.status |= S_CONTOUR_OVERFLOW;
        } else {
            if (xy)
                xy[o.n] = make_double2(firstx, firsty);
            else
                o.pts[o.n] = o.pts[0];
            o.n++;
        }
    }
}

// Contour routines over a shared-memory (x, y) buffer: the same operations
// as project_to_boundary, contour_volume, contour_perimeter and
// clear_contour_area on CPoint arrays (src/grainBoundary.cpp:201-231, 365-447,
// src/box.cpp:1888-1906).
__device__ int project_xy(const double2* P, int asize, double px, double py, double* out_lambda) {
    double minDist = 1000000.0;
    int minimal_segment = 0;
    double dist = 0;
    int nearest = -1;
    for (int k = 0; k < asize - 1; k++) {
        dist = len_sqr(px - P[k].x, py - P[k].y);
        if (dist < minDist) {
            nearest = k;
            minDist = dist;
            minimal_segment = k;
        }
    }
    double lam_out = *out_lambda;
    if (nearest < 0) return 0;
    minDist = 1000000.0;
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

// ExplicitGrainBoundary::computeVolume / computePerimeter
// (src/grainBoundary.cpp:201-213, 224-231) by the whole warp: lanes evaluate
// the per-segment terms side by side, then the terms are added one after the
// other in contour order (every lane holds the same sum, rounded exactly as
// the reference's loop).
__device__ __forceinline__ double volume_xy(const double2* P, int n, double h) {
    const int lane = threadIdx.x & 31;
    double v = 0;
    for (int i0 = 0; i0 < n - 1; i0 += 32) {
        const int i = i0 + lane;
        double t = 0;
        if (i < n - 1) t = (P[i].y + P[i + 1].y) * (P[i].x - P[i + 1].x);
        const int m = n - 1 - i0 < 32 ? n - 1 - i0 : 32;
        for (int q = 0; q < m; ++q) v += __shfl_sync(0xffffffffu, t, q);
    }
    return fabs(v) * h * h * 0.5;
}

__device__ __forceinline__ double perimeter_xy(const double2* P, int n, double h) {
    const int lane = threadIdx.x & 31;
    double p = 0;
    for (int i0 = 0; i0 < n - 1; i0 += 32) {
        const int i = i0 + lane;
        double t = 0;
        if (i < n - 1) {
            const double dx = P[i].x - P[i + 1].x, dy = P[i].y - P[i + 1].y;
            t = sqrt(dx * dx + dy * dy) * h;
        }
        const int m = n - 1 - i0 < 32 ? n - 1 - i0 : 32;
        for (int q = 0; q < m; ++q) p += __shfl_sync(0xffffffffu, t, q);
    }
    return p;
}

// The same two sums for the batched form, whose areas and perimeters need
// not round as the reference's loop does: each lane adds its own terms, then
// a tree to lane 0, broadcast (every lane holds the same bits).
__device__ __forceinline__ double warp_sum_to_all(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}

__device__ __forceinline__ double volume_xy_tree(const double2* P, int n, double h) {
    double v = 0;
    for (int i = threadIdx.x & 31; i < n - 1; i += 32) v += (P[i].y + P[i + 1].y) * (P[i].x - P[i + 1].x);
    return fabs(warp_sum_to_all(v)) * h * h * 0.5;
}

__device__ __forceinline__ double perimeter_xy_tree(const double2* P, int n, double h) {
    double p = 0;
    for (int i = threadIdx.x & 31; i < n - 1; i += 32) {
        const double dx = P[i].x - P[i + 1].x, dy = P[i].y - P[i + 1].y;
        p += sqrt(dx * dx + dy * dy) * h;
    }
    return warp_sum_to_all(p);
}

// The level set's sums in the form's rounding: the reference's order in
// FP64 (plain), the tree in the batched form.
template <typename R>
__device__ __forceinline__ double form_volume(const double2* P, int n, double h) {
    if constexpr (sizeof(R) == 4) return volume_xy_tree(P, n, h);
    else return volume_xy(P, n, h);
}
template <typename R>
__device__ __forceinline__ double form_perimeter(const double2* P, int n, double h) {
    if constexpr (sizeof(R) == 4) return perimeter_xy_tree(P, n, h);
    else return perimeter_xy(P, n, h);
}

template <typename R>
__device__ bool clear_area_xy(R* phi, const Box& b, const double2* P, int n, double h) {
    if (n == 0) return true;
    double minx = P[0].x, maxx = P[0].x, miny = P[0].y, maxy = P[0].y;
    for (int i = 0; i < n; i++) {
        minx = fmin(minx, P[i].x);
        maxx = fmax(maxx, P[i].x);
        miny = fmin(miny, P[i].y);
        maxy = fmax(maxy, P[i].y);
    }
    bool ok = true;
    for (int i = (int)(miny - 1); i < maxy + 1; i++)
        for (int j = (int)(minx - 1); j < maxx + 1; j++) {
            uint32_t k;
            if (!buf_index(b, i, j, &k)) {
                ok = false;
                continue;
            }
            if ((double)phi[k] >= 0) phi[k] = (R)(-h);
        }
    return ok;
}

constexpr int kWalkPts = 448;  // shared-memory contour buffer per warp
struct WalkShared;
template <typename R>
__device__ int extract_bitmap_warp(const Field<R>& f, const uint32_t* idl, uint32_t own, ContourOut& o, int lane,
                                   double2* xy, WalkShared& ws);

// Contour + junctions of one grain by one warp; returns false if no pixel
// has phi >= 0.  The walk writes into the warp's shared buffer xy (or, for a
// contour longer than the buffer, directly into the global contour);
// junctions are projected one lane per junction.  On return *in_shared says
// where the points are.
template <typename R>
__device__ bool extract_warp(const Field<R>& f, const uint32_t* idl, uint32_t own, ContourOut& o, int lane,
                             double2* xy, bool* in_shared, WalkShared* ws) {
    if (ws) {
        const uint32_t st0 = o.status;
        const int r = extract_bitmap_warp(f, idl, own, o, lane, xy, *ws);
        if (r >= 0) {
            *in_shared = true;
            return r == 1;
        }
        o.status = st0;  // does not fit the shared buffers: walk in global memory
        o.jn = 0;
    }
    const int start = first_inside_warp(f, lane);
    if (start < 0) {
        o.n = 0;
        o.jn = 0;
        return false;
    }
    const int w = box_w(f.b);
    const int gcap = o.cap;
    bool shared = true;
    if (lane == 0) {
        o.cap = gcap < kWalkPts ? gcap : kWalkPts;
        ms_walk(f, idl, own, f.b.x0 + start % w, f.b.y0 + start / w, o, xy);
        if ((o.status & S_CONTOUR_OVERFLOW) && gcap > kWalkPts) {  // long contour: walk again into global memory
            o.status &= ~S_CONTOUR_OVERFLOW;
            o.cap = gcap;
            ms_walk(f, idl, own, f.b.x0 + start % w, f.b.y0 + start / w, o, (double2*)nullptr);
            shared = false;
        }
        o.cap = gcap;
    }
    shared = __shfl_sync(0xffffffffu, shared, 0);
    o.n = __shfl_sync(0xffffffffu, o.n, 0);
    o.jn = __shfl_sync(0xffffffffu, o.jn, 0);
    o.status = __shfl_sync(0xffffffffu, o.status, 0);
    __syncwarp();
    if (o.n >= 2) {
        for (int j = lane; j < o.jn; j += 32) {
            double lambda = 0.0;
            const int nx_n = o.n;
            int seg;
            double sx, sy, tx, ty;
            if (shared) {
                seg = project_xy(xy, o.n, o.js[j].x, o.js[j].y, &lambda);
                const int nx = periodic(seg + 1, nx_n);
                sx = xy[seg].x;
                sy = xy[seg].y;
                tx = xy[nx].x;
                ty = xy[nx].y;
            } else {
                seg = project_to_boundary(o.pts, o.n, o.js[j].x, o.js[j].y, &lambda);
                const int nx = periodic(seg + 1, nx_n);
                sx = o.pts[seg].x;
                sy = o.pts[seg].y;
                tx = o.pts[nx].x;
                ty = o.pts[nx].y;
            }
            o.js[j].x = sx + (tx - sx) * lambda;
            o.js[j].y = sy + (ty - sy) * lambda;
            o.js[j].segment = seg;
            o.js[j].lambda = lambda;
        }
    }
    __syncwarp();
    *in_shared = shared;
    return true;
}

constexpr int kBitmapCap = 400;  // words of the padded bitmap (boxes up to about 94 x 94)
constexpr int kTrace = 768;      // walk steps recorded per warp

struct WalkShared {
    uint32_t bm[kBitmapCap];
    uint16_t trace[kTrace];
};

// Corner mask of the marching-squares cell whose top-left pixel is at padded
// row tr, padded column lc (C_TL | C_TR from row tr, C_BL | C_BR from tr + 1).
__device__ __forceinline__ int cell_mask(const uint32_t* bm, int wpr, int tr, int lc) {
    const uint32_t* rt = bm + tr * wpr + (lc >> 5);
    const int sh = lc & 31;
    const uint32_t top2 = __funnelshift_r(rt[0], rt[1], sh);
    const uint32_t bot2 = __funnelshift_r(rt[wpr], rt[wpr + 1], sh);
    return (int)((top2 & 3u) | ((bot2 & 3u) << 2));
}

// Next direction of generateContour's switch for each corner mask
// (src/marchingSquares.cpp:64-154), two bits per mask; the saddles 6 and 9
// and the empty / full masks 0 and 15 are decided separately.
constexpr uint32_t ms_next_bits() {
    const int dir[16] = {0, MS_UP, MS_RIGHT, MS_RIGHT, MS_LEFT, MS_UP, 0, MS_RIGHT,
                         MS_DOWN, 0, MS_DOWN, MS_DOWN, MS_LEFT, MS_UP, MS_LEFT, 0};
    uint32_t t = 0;
    for (int m = 0; m < 16; ++m) t |= (uint32_t)dir[m] << (2 * m);
    return t;
}
constexpr uint32_t kMsNext = ms_next_bits();
// masks whose case generates a point (all but 0, 6, 9, 15)
constexpr uint32_t kMsEmit = 0xFFFFu & ~((1u << 0) | (1u << 6) | (1u << 9) | (1u << 15));

// Marching squares with the inside/outside decisions taken from a bitmap of
// the box in shared memory (built with one ballot per 32 pixels, with a
// zero border of one pixel all round so the walk needs no bounds tests), the
// walk recorded as a trace by lane 0 (one 4-bit corner mask per step from two
// funnel shifts), and the points, junctions and duplicate removal evaluated
// across the lanes in walk order.  Returns 0 if no pixel is inside, 1 on
// success, -1 if the box or the walk does not fit the shared buffers (the
// caller then walks in global memory).
template <typename R>
__device__ int extract_bitmap_warp(const Field<R>& f, const uint32_t* idl, uint32_t own, ContourOut& o, int lane,
                                   double2* xy, WalkShared& ws) {
    const Box b = f.b;
    const int w = box_w(b), hgt = box_h(b);
    // padded bitmap: row r + 1, bit c + 1 hold pixel (r, c) of the box
    const int wpr = (w + 2 + 31) >> 5;
    if (w + 2 > 1024 || (hgt + 2) * wpr + 1 > kBitmapCap) return -1;
    bool nonfinite = false;  // a NaN or infinity anywhere in the field
    for (int r0 = 0; r0 < hgt + 2; r0 += 8)  // eight rows of two words: 16 loads in flight
        for (int q0 = 0; q0 < wpr; q0 += 2) {
            bool in[2][8];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int c = (q0 + k) * 32 + lane - 1;
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int r = r0 + u - 1;
                    const bool pix = q0 + k < wpr && r >= 0 && r < hgt && c >= 0 && c < w;
                    const R v = pix ? f.v[r * w + c] : (R)0;  // tested in the field's own type
                    nonfinite |= !isfinite(v);
                    in[k][u] = pix && v >= (R)0;
                }
            }
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const uint32_t word = __ballot_sync(0xffffffffu, in[k][u]);
                    if (lane == 0 && r0 + u < hgt + 2 && q0 + k < wpr) ws.bm[(r0 + u) * wpr + q0 + k] = word;
                }
        }
    if (lane == 0) ws.bm[(hgt + 2) * wpr] = 0u;
    if (__any_sync(0xffffffffu, nonfinite) && lane == 0) o.status |= S_NAN;
    __syncwarp();
    // first inside pixel in row-major order
    int start = -1;
    for (int q0 = 0; q0 < hgt * wpr; q0 += 32) {
        const int q = q0 + lane;
        const uint32_t word = q < hgt * wpr ? ws.bm[wpr + q] : 0u;
        const uint32_t any = __ballot_sync(0xffffffffu, word != 0u);
        if (any) {
            const int src = __ffs(any) - 1;
            const uint32_t wd = __shfl_sync(0xffffffffu, word, src);
            const int qq = q0 + src;
            start = (qq / wpr) * w + (qq % wpr) * 32 + (__ffs(wd) - 1) - 1;
            break;
        }
    }
    if (start < 0) {
        o.n = 0;
        o.jn = 0;
        return 0;
    }
    const int startX = b.x0 + start % w, startY = b.y0 + start / w;
    // lane 0: the walk of generateContour (src/marchingSquares.cpp:44-187) on
    // the bitmap, in padded coordinates lc = left - x0 + 1, tr = top - y0 + 1,
    // recording the cell index tr * (w + 1) + lc of every step (the step's
    // direction is recovered later from the next recorded cell).  The switch
    // of the reference is evaluated as selects, so a step has no branch.
    const int cw = w + 1;
    if ((hgt + 1) * cw > 65535) return -1;
    int nsteps = 0;
    uint32_t st = 0;
    if (lane == 0) {
        const int lc_end = startX - b.x0, tr_end = startY - b.y0;
        int lc = lc_end, tr = tr_end;
        int next = MS_NONE, prev = MS_NONE;
        const int limit = 4 * (w + 2) * (hgt + 2) + 16;
        do {
            const int mask = cell_mask(ws.bm, wpr, tr, lc);
            const int tab = (int)((kMsNext >> (2 * mask)) & 3u);
            const int s6 = (prev == MS_UP) ? MS_RIGHT : MS_LEFT;
            const int s9 = (prev == MS_RIGHT) ? MS_DOWN : MS_UP;
            next = mask == (C_BL | C_TR) ? s6 : mask == (C_BR | C_TL) ? s9 : (mask == 0 || mask == 15) ? next : tab;
            ws.trace[nsteps] = (uint16_t)(tr * cw + lc);
            ++nsteps;
            lc += (next == MS_RIGHT) - (next == MS_LEFT);
            tr += (next == MS_DOWN) - (next == MS_UP);
            prev = next;
            if (nsteps >= kTrace || nsteps > limit) break;
        } while (lc != lc_end || tr != tr_end);
        if (lc != lc_end || tr != tr_end) {
            if (nsteps >= kTrace)
                nsteps = -1;  // longer than the trace buffer: walk again in global memory
            else
                st |= S_WALK_LIMIT;
        }
    }
    nsteps = __shfl_sync(0xffffffffu, nsteps, 0);
    if (nsteps < 0) return -1;
    o.status |= __shfl_sync(0xffffffffu, st, 0);
    __syncwarp();
    // points and junctions of every step, in walk order.  Two 32-step
    // chunks per pass: each lane first issues the field and IDLocal loads of
    // both its steps (generatePoint's two values, generateJunction's corners),
    // then evaluates the steps in order.
    const unsigned lt = (1u << lane) - 1u;
    int ne = 0;
    int jn = 0;
    bool point_overflow = false;
    for (int t0 = 0; t0 < nsteps; t0 += 64) {
        int mask[2], next[2], left[2], top[2];
        bool emit[2], pv[2], jv[2];
        R va[2], vc[2];
        uint32_t id4[2][4];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int t = t0 + 32 * k + lane;
            mask[k] = 0;
            next[k] = MS_UP;
            left[k] = 0;
            top[k] = 0;
            emit[k] = pv[k] = jv[k] = false;
            va[k] = vc[k] = (R)0;
            id4[k][0] = id4[k][1] = id4[k][2] = id4[k][3] = own;
            if (t < nsteps) {
                // the step's direction is the move to the next recorded cell
                const int c = ws.trace[t], cn = ws.trace[t + 1 < nsteps ? t + 1 : 0];
                const int tr = c / cw, lc = c - tr * cw;
                left[k] = lc - 1 + b.x0;
                top[k] = tr - 1 + b.y0;
                const int m = cell_mask(ws.bm, wpr, tr, lc);
                mask[k] = m;
                const int dcell = cn - c;
                const int nx = dcell == -cw ? MS_UP : dcell == cw ? MS_DOWN : dcell == -1 ? MS_LEFT : MS_RIGHT;
                next[k] = nx;
                emit[k] = (kMsEmit >> m) & 1u;
                const int lf = left[k], tp = top[k], right = lf + 1, bottom = tp + 1;
                // generatePoint's values: a then c, delta = a - c (ms_point)
                const int ra = nx == MS_RIGHT || nx == MS_UP ? tp : bottom;
                const int ca = nx == MS_LEFT || nx == MS_UP ? lf : right;
                const int rc = nx == MS_LEFT ? tp : nx == MS_RIGHT ? bottom : ra;
                const int cc = nx == MS_UP ? right : nx == MS_DOWN ? lf : ca;
                pv[k] = nx == MS_LEFT ? tp >= b.y0 : nx == MS_RIGHT ? bottom < b.y1 : nx == MS_UP ? right < b.x1 : lf >= b.x0;
                if (emit[k] && pv[k]) {
                    va[k] = f.v[(ra - b.y0) * w + (ca - b.x0)];
                    vc[k] = f.v[(rc - b.y0) * w + (cc - b.x0)];
                }
                jv[k] = __popc(m) < 3 && bottom >= b.y0 && bottom < b.y1 && tp >= b.y0 && tp < b.y1 && lf >= b.x0 &&
                        lf < b.x1 && right >= b.x0 && right < b.x1;
                if (jv[k]) {  // generateJunction's corners, in its order
                    if (!(m & C_BL)) id4[k][0] = idl[(bottom - b.y0) * w + (lf - b.x0)];
                    if (!(m & C_TL)) id4[k][1] = idl[(tp - b.y0) * w + (lf - b.x0)];
                    if (!(m & C_BR)) id4[k][2] = idl[(bottom - b.y0) * w + (right - b.x0)];
                    if (!(m & C_TR)) id4[k][3] = idl[(tp - b.y0) * w + (right - b.x0)];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int lf = left[k], tp = top[k], right = lf + 1, bottom = tp + 1;
            double px = 0, py = 0;
            if (emit[k]) {  // generatePoint (ms_point) on the loaded values
                const int nx = next[k];
                if (nx == MS_LEFT) {
                    px = lf;
                    py = pv[k] ? bottom - (double)va[k] / ((double)va[k] - (double)vc[k]) : (double)bottom;
                } else if (nx == MS_RIGHT) {
                    px = right;
                    py = pv[k] ? top[k] + (double)va[k] / ((double)va[k] - (double)vc[k]) : (double)tp;
                } else if (nx == MS_UP) {
                    py = tp;
                    px = pv[k] ? lf + (double)va[k] / ((double)va[k] - (double)vc[k]) : (double)lf;
                } else {
                    py = bottom;
                    px = pv[k] ? right - (double)va[k] / ((double)va[k] - (double)vc[k]) : (double)right;
                }
            }
            uint32_t boxes[4] = {0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu};
            int order = 0;
            bool junc = false;
            if (jv[k]) {
                insert_distinct(id4[k][0], boxes, order);
                insert_distinct(id4[k][1], boxes, order);
                insert_distinct(id4[k][2], boxes, order);
                insert_distinct(id4[k][3], boxes, order);
                junc = order > 2;
            }
            const uint32_t eb = __ballot_sync(0xffffffffu, emit[k]);
            if (emit[k]) {
                const int pos = ne + __popc(eb & lt);
                if (pos < kWalkPts)
                    xy[pos] = make_double2(px, py);
                else
                    point_overflow = true;
            }
            ne += __popc(eb);
            const uint32_t jb = __ballot_sync(0xffffffffu, junc);
            if (junc) {
                const int pos = jn + __popc(jb & lt);
                if (pos < o.jcap) {
                    Junction& j = o.js[pos];
                    j.type = order;
                    for (int q = 0; q < 4; ++q) j.grains[q] = q < order ? boxes[q] : 0xFFFFFFFFu;
                    j.segment = -1;
                    j.lambda = 0;
                    j.x = lf + 0.5;
                    j.y = tp + 0.5;
                } else {
                    o.status |= S_JUNCTION_OVERFLOW;
                }
            }
            jn += __popc(jb);
        }
    }
    if (__any_sync(0xffffffffu, point_overflow)) return -1;
    o.jn = jn < o.jcap ? jn : o.jcap;
    __syncwarp();
    // insertPoint's duplicate test: a candidate equal to its predecessor is dropped
    int n = 0;
    for (int i0 = 0; i0 < ne; i0 += 32) {
        const int i = i0 + lane;
        double2 pnt = make_double2(0, 0);
        bool keep = false;
        if (i < ne) {
            pnt = xy[i];
            keep = i == 0 || pnt.x != xy[i - 1].x || pnt.y != xy[i - 1].y;
        }
        __syncwarp();
        const uint32_t kb = __ballot_sync(0xffffffffu, keep);
        if (keep) xy[n + __popc(kb & lt)] = pnt;
        n += __popc(kb);
        __syncwarp();
    }
    const int cap = o.cap < kWalkPts ? o.cap : kWalkPts;
    if (n > 0 && (xy[0].x != xy[n - 1].x || xy[0].y != xy[n - 1].y)) {  // close the loop
        if (lane == 0 && n < kWalkPts) xy[n] = xy[0];
        n++;
    }
    if (n > cap) {
        o.status |= S_CONTOUR_OVERFLOW;
        n = cap;
    }
    o.n = n;
    __syncwarp();
    // junctions projected onto the contour (extractBoundaryAndJunctions, src/grainBoundary.cpp:51-61)
    if (n >= 2) {
        for (int j = lane; j < o.jn; j += 32) {
            double lambda = 0.0;
            const int seg = project_xy(xy, n, o.js[j].x, o.js[j].y, &lambda);
            const int nx = periodic(seg + 1, n);
            o.js[j].x = xy[seg].x + (xy[nx].x - xy[seg].x) * lambda;
            o.js[j].y = xy[seg].y + (xy[nx].y - xy[seg].y) * lambda;
            o.js[j].segment = seg;
            o.js[j].lambda = lambda;
        }
    }
    __syncwarp();
    return 1;
}

// grainhdl::level_set -> LSbox::extractContour (src/grainhdl.cpp:830-848,
// src/box.cpp:1089-1153), one warp per grain.
template <typename R>
__global__ void __launch_bounds__(32 * kGrainsPerBlock, 5) k_levelset_w(NetConst C, NetState* S) {
    __shared__ double2 s_xy[kGrainsPerBlock][kWalkPts];
    __shared__ WalkShared s_walk[kGrainsPerBlock];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int slot = blockIdx.x * kGrainsPerBlock + wid;
    const int g = slot < C.N ? grain_at(S, slot) : C.N + 1;
    if (g > C.N || halted(S)) return;
    const int st = C.state[g];
    const Box bc = S->box_cur[g];
    if (st != G_EXISTS) {
        if (lane == 0) {
            if (st == G_VANISHED) {
                C.state[g] = G_GONE;
                C.gone_loop[g] = S->loop;
            }
            S->box_new[g] = bc;
            S->cn_cur[g] = 0;
            S->jn_cur[g] = 0;
        }
        return;
    }
    double2* xy = s_xy[wid];
    const int old_len = S->cn_prev[g];
    R* phi = phiA_of<R>(S) + S->off_cur[g];
    Field<R> f{phi, bc};
    const uint32_t* idl = S->idCur + S->off_cur[g];
    ContourOut o{S->contCur + S->coff_cur[g], S->ccap_cur[g], 0, S->jCur + (int64_t)g * C.jmax, C.jmax, 0, 0};
    bool shared = true;
    bool ok = extract_warp(f, idl, (uint32_t)g, o, lane, xy, &shared, &s_walk[wid]);
    int irregular = 0;
    if (ok) {
        double newVolume = 0;
        bool regular_motion = true;
        if (shared) newVolume = form_volume<R>(xy, o.n, C.h);
        if (lane == 0) {
            if (!shared) newVolume = contour_volume(o.pts, o.n, C.h);
            regular_motion = motion_regular(old_len, o.n, C.volume[g], newVolume, C.dt, &irregular);
        }
        regular_motion = __shfl_sync(0xffffffffu, regular_motion, 0);
        int tries = 0;
        while (!regular_motion) {  // clear the grain area and extract again (src/box.cpp:1099-1114)
            if (lane == 0) {
                const bool in_range = shared ? clear_area_xy(phi, bc, xy, o.n, C.h)
                                             : clear_contour_area(phi, bc, o.pts, o.n, C.h);
                if (!in_range) o.status |= S_INDEX;
            }
            __syncwarp();
            ok = extract_warp(f, idl, (uint32_t)g, o, lane, xy, &shared, &s_walk[wid]);
            if (!ok) break;
            if (shared) newVolume = form_volume<R>(xy, o.n, C.h);
            if (lane == 0) {
                if (!shared) newVolume = contour_volume(o.pts, o.n, C.h);
                regular_motion = motion_regular(old_len, o.n, C.volume[g], newVolume, C.dt, &irregular);
                if (++tries > 64) {
                    o.status |= S_RETRY_LIMIT;
                    regular_motion = true;
                }
            }
            regular_motion = __shfl_sync(0xffffffffu, regular_motion, 0);
        }
        if (lane == 0 && ok && !isfinite(newVolume)) o.status |= S_NAN;
    }
    if (ok && shared) {  // publish the contour (energy and mobility still unset, as generatePoint leaves them)
        for (int i = lane; i < o.n; i += 32) {
            CPoint q;
            q.x = xy[i].x;
            q.y = xy[i].y;
            q.energy = -1.0;
            q.mob = -1.0;
            o.pts[i] = q;
        }
    }
    double perim = 0;
    if (ok && shared) perim = form_perimeter<R>(xy, o.n, C.h);
    if (ok && !shared && lane == 0) perim = contour_perimeter(o.pts, o.n, C.h);
    if (lane != 0) return;
    if (o.status) set_status(S, o.status);
    C.regular[g] = 1;
    if (!ok) {
        C.state[g] = G_VANISHED;
        S->box_new[g] = bc;
        S->cn_cur[g] = 0;
        S->jn_cur[g] = 0;
        return;
    }
    if (irregular) C.regular[g] = 0;
    int* nb = C.newbb + 4 * (int64_t)g;
    Box nbx = bc;
    if (!C.decouple) {
        if (nb[0] < 0) nb[0] = 0;
        if (nb[2] < 0) nb[2] = 0;
        if (nb[1] > C.m) nb[1] = C.m;
        if (nb[3] > C.m) nb[3] = C.m;
        nbx = resize_to_square(Box{nb[0], nb[1], nb[2], nb[3]}, C.m);
    }
    S->box_new[g] = nbx;
    C.perimeter[g] = perim;
    S->cn_cur[g] = o.n;
    S->jn_cur[g] = o.jn;
}

// Initial contours of a voxelized network (distanceInitialisation ->
// LSbox::extractContour on the initial distance field, as k_init_contour
// does one thread per grain): one warp per grain with the level set's
// warp-parallel extraction (bitmap walk, points, junctions and their
// projection across the lanes), into the previous-step roles the first
// corrector reads.
template <typename R>
__global__ void __launch_bounds__(32 * kGrainsPerBlock, 5) k_init_contour_w(NetConst C, NetState* S) {
    __shared__ double2 s_xy[kGrainsPerBlock][kWalkPts];
    __shared__ WalkShared s_walk[kGrainsPerBlock];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int g = blockIdx.x * kGrainsPerBlock + wid + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    double2* xy = s_xy[wid];
    Field<R> f{phiA_of<R>(S) + S->off_cur[g], S->box_cur[g]};
    const uint32_t* idl = S->idPrev + S->off_prev[g];
    ContourOut o{S->contPrev + S->coff_prev[g], S->ccap_prev[g], 0, S->jPrev + (int64_t)g * C.jmax, C.jmax, 0, 0};
    bool shared = true;
    const bool ok = extract_warp(f, idl, (uint32_t)g, o, lane, xy, &shared, &s_walk[wid]);
    double vol = 0;
    if (ok && shared) {
        for (int i = lane; i < o.n; i += 32) {
            CPoint q;
            q.x = xy[i].x;
            q.y = xy[i].y;
            q.energy = -1.0;
            q.mob = -1.0;
            o.pts[i] = q;
        }
        vol = form_volume<R>(xy, o.n, C.h);
    }
    if (lane != 0) return;
    if (o.status) set_status(S, o.status);
    if (!ok) {
        C.state[g] = G_VANISHED;
        S->cn_prev[g] = 0;
        S->jn_prev[g] = 0;
        C.volume[g] = 0;
        return;
    }
    if (!shared) vol = contour_volume(o.pts, o.n, C.h);
    S->cn_prev[g] = o.n;
    S->jn_prev[g] = o.jn;
    C.volume[g] = vol;
}

// Per contour point result of the neighbour probe of buildDirectNeighbours.
struct PointInfo {
    int32_t cid;
    int32_t pad;
    double theta;
    double len;
};

constexpr int kNbPts = 512;  // per-warp shared buffers of the neighbour build

// LSbox::computeVolumeAndEnergy + ExplicitGrainBoundary::buildDirectNeighbours
// (src/box.cpp:1201-1228, src/grainBoundary.cpp:85-199), one warp per grain:
// lanes probe contour points, evaluate the per-pair physics and the terms of
// the area and energy sums into shared memory; lane 0 builds the neighbour
// list and adds the terms in contour order (the reference's order; the
// batched form sums by trees instead).
template <typename R>
__global__ void __launch_bounds__(32 * kGrainsPerBlock) k_neighbours_w(NetConst C, NetState* S, PointInfo* scratch) {
    __shared__ int s_cid[kGrainsPerBlock][kNbPts];
    __shared__ double s_len[kGrainsPerBlock][kNbPts];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int slot = blockIdx.x * kGrainsPerBlock + wid;
    const int g = slot < C.N ? grain_at(S, slot) : C.N + 1;
    if (g > C.N || C.state[g] != G_EXISTS || C.regular[g] == 0 || halted(S)) return;
    const int loop = S->loop;
    CPoint* P = S->contCur + S->coff_cur[g];
    PointInfo* info = scratch + S->coff_cur[g];
    const int n = S->cn_cur[g];
    const double h = C.h;
    const Box bc = S->box_cur[g];
    const R* phi = phiA_of<R>(S) + S->off_cur[g];
    const uint32_t* idl = S->idCur + S->off_cur[g];
    const double* qg = C.quat + 4 * (int64_t)g;
    const bool sh = n - 1 <= kNbPts;
    auto CID = [&](int q) -> int& { return sh ? s_cid[wid][q] : info[q].cid; };
    auto LEN = [&](int q) -> double& { return sh ? s_len[wid][q] : info[q].len; };
    // area (computeVolume, src/grainBoundary.cpp:201-213): terms side by side,
    // added in contour order (plain) or by a tree (batched, as the sums below)
    constexpr bool kTree = sizeof(R) == sizeof(float);
    double v = 0;
    if constexpr (kTree) {
        for (int i = lane; i < n - 1; i += 32) v += (P[i].y + P[i + 1].y) * (P[i].x - P[i + 1].x);
        v = warp_sum_to_all(v);
    } else {
        for (int i0 = 0; i0 < n - 1; i0 += 32) {
            const int i = i0 + lane;
            double t = 0;
            if (i < n - 1) t = (P[i].y + P[i + 1].y) * (P[i].x - P[i + 1].x);
            const int m = n - 1 - i0 < 32 ? n - 1 - i0 : 32;
            for (int q = 0; q < m; ++q) v += __shfl_sync(FULL, t, q);
        }
    }
    const double newVolume = fabs(fabs(v) * h * h * 0.5);
    // probes; the first failing point ends the reference's loop
    int first_bad = 0x7fffffff;
    for (int i = lane; i < n - 1; i += 32) {
        const double px = P[i].x, py = P[i].y;
        int pxGrid = (int)px, pyGrid = (int)py;
        uint32_t k;
        bool bad = false;
        if (!buf_index(bc, pyGrid, pxGrid, &k)) bad = true;
        if (!bad && (double)phi[k] > 0) {
            pxGrid = (int)(px + 1);
            if (!buf_index(bc, pyGrid, pxGrid, &k)) bad = true;
            if (!bad && (double)phi[k] > 0) {
                pyGrid = (int)(py + 1);
                if (!buf_index(bc, pyGrid, pxGrid, &k)) bad = true;
                if (!bad && (double)phi[k] > 0) pxGrid = (int)px;
            }
        }
        if (!bad && (pyGrid < 0 || pyGrid >= bc.y1 || pxGrid < 0 || pxGrid >= bc.x1)) bad = true;
        if (!bad && !buf_index(bc, pyGrid, pxGrid, &k)) bad = true;
        uint32_t cid = 0;
        if (!bad) {
            cid = idl[k];
            if (cid != 0 && (cid > (uint32_t)C.N || C.state[cid] == G_GONE)) bad = true;
        }
        CID(i) = bad ? -1 : (int)cid;
        if (bad) first_bad = min(first_bad, i);
    }
    first_bad = warp_min_i(first_bad);
    const int upto = first_bad < n - 1 ? first_bad : n - 1;
    __syncwarp();
    // neighbour list in first-occurrence order (one entry per distinct
    // neighbour, at most `cap`; later new neighbours are dropped), then each
    // entry's length summed over its points in contour order
    __shared__ int s_nid[kGrainsPerBlock][48];
    const int cap = C.nbmax < 48 ? C.nbmax : 48;
    int nn = 0;
    bool overflow = false;
    const unsigned lt = (1u << lane) - 1u;
    for (int i0 = 0; i0 < upto; i0 += 32) {
        const int i = i0 + lane;
        const int cid = i < upto ? CID(i) : -2;
        bool fresh = i < upto;
        for (int e = 0; e < nn && fresh; ++e)
            if (s_nid[wid][e] == cid) fresh = false;
        const unsigned same = __match_any_sync(FULL, cid);
        fresh = fresh && (__ffs(same) - 1) == lane;
        const unsigned fb = __ballot_sync(FULL, fresh);
        if (fresh) {
            const int pos = nn + __popc(fb & lt);
            if (pos < cap) s_nid[wid][pos] = cid;
        }
        if (nn + __popc(fb) > cap) overflow = true;
        nn = min(nn + __popc(fb), cap);
        __syncwarp();
    }
    // each listed neighbour's misorientation, energy and mobility, once
    __shared__ double s_nth[kGrainsPerBlock][48], s_nen[kGrainsPerBlock][48], s_nmob[kGrainsPerBlock][48];
    for (int e = lane; e < nn; e += 32) {
        const double theta = grain_misorientation(qg, C.quat + 4 * (int64_t)s_nid[wid][e]);
        s_nth[wid][e] = theta;
        s_nen[wid][e] = read_shockley(theta, C);
        s_nmob[wid][e] = mobility_model(theta, C);
    }
    __syncwarp();
    // physics of the points before the first failure; energy terms of all
    // points, added in contour order (computeEnergy, src/grainBoundary.cpp:215-222)
    double energy_sum = 0;
    for (int i0 = 0; i0 < n - 1; i0 += 32) {
        const int i = i0 + lane;
        double term = 0;
        if (i < n - 1) {
            const double dx = P[i].x - P[i + 1].x, dy = P[i].y - P[i + 1].y;
            const double len = sqrt(dx * dx + dy * dy);
            double energy = -1.0;  // generatePoint's value, kept where the loop never reached
            if (i < upto) {
                // the neighbour's physics, evaluated once per neighbour above
                // (the same calls on the same orientations)
                const int cid = CID(i);
                int e = 0;
                while (e < nn && s_nid[wid][e] != cid) ++e;
                double mob;
                if (e < nn) {
                    mob = s_nmob[wid][e];
                    energy = s_nen[wid][e];
                } else {  // beyond the list's capacity
                    const double theta = grain_misorientation(qg, C.quat + 4 * (int64_t)cid);
                    mob = mobility_model(theta, C);
                    energy = read_shockley(theta, C);
                }
                P[i].mob = mob;
                P[i].energy = energy;
                LEN(i) = len * h;
            }
            term = len * energy * h;
        }
        if constexpr (kTree) {
            energy_sum += term;
        } else {
            const int m = n - 1 - i0 < 32 ? n - 1 - i0 : 32;
            for (int q = 0; q < m; ++q) energy_sum += __shfl_sync(FULL, term, q);
        }
    }
    if constexpr (kTree) energy_sum = warp_sum_to_all(energy_sum);
    __syncwarp();
    Neighbour* nb = C.nb + (int64_t)g * C.nbmax;
    __shared__ double s_nlen[kGrainsPerBlock][48];
    if constexpr (kTree) {  // each neighbour's length by the whole warp
        for (int e = 0; e < nn; ++e) {
            const int cid = s_nid[wid][e];
            double len = 0;
            for (int i = lane; i < upto; i += 32)
                if (CID(i) == cid) len += LEN(i);
            len = warp_sum_to_all(len);
            if (lane == 0) s_nlen[wid][e] = len;
        }
        __syncwarp();
    }
    for (int e = lane; e < nn; e += 32) {
        const int cid = s_nid[wid][e];
        double len = 0;
        if constexpr (kTree) {
            len = s_nlen[wid][e];
        } else {
            for (int i = 0; i < upto; ++i)
                if (CID(i) == cid) len += LEN(i);
        }
        nb[e].id = cid;
        nb[e].length = len;
        nb[e].energy = s_nen[wid][e];
        nb[e].misori = s_nth[wid][e];
        nb[e].mobility = s_nmob[wid][e];
    }
    if (lane != 0) return;
    C.nb_n[g] = nn;
    if (overflow) set_status(S, S_NEIGHBOUR_OVERFLOW);
    if (first_bad < n - 1) {
        C.regular[g] = 0;  // markAsInvalidMotion (src/box.cpp:1939-1945)
    } else if (n > 0) {
        P[n - 1].energy = P[0].energy;
        P[n - 1].mob = P[0].mob;
    }
    C.energy[g] = energy_sum;
    double dA = newVolume - C.volume[g];
    dA = dA / C.dt;
    dA = dA * (3 / kPi);
    const unsigned int lp = (unsigned int)loop;
    if ((unsigned long)(lp - 1u) % (unsigned long)C.analysis_timestep == 0 || lp == 0) C.meanda[g] = 0;
    C.meanda[g] += dA;
    C.volume[g] = newVolume;
}

// LSbox::computeSecondOrderNeighbours (src/box.cpp:1027-1068), one warp per
// grain: candidates of each member's list are tested across lanes and the
// accepted ones appended in list order.
__global__ void __launch_bounds__(32 * kGrainsPerBlock) k_second_order_w(NetConst C, NetState* S) {
    constexpr int kL = 128;
    __shared__ int s_list[kGrainsPerBlock][kL];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int slot = blockIdx.x * kGrainsPerBlock + wid;
    const int g = slot < C.N ? grain_at(S, slot) : C.N + 1;
    if (g > C.N || C.state[g] != G_EXISTS) return;
    const int K = C.kmax < kL ? C.kmax : kL;
    const int* sec = C.sec_ids + (int64_t)g * C.kmax;
    const int ns = C.sec_n[g];
    int* list = s_list[wid];
    const unsigned lt = (1u << lane) - 1u;
    int nc = 0;
    bool overflow = false;
    for (int a0 = 0; a0 < ns; a0 += 32) {  // existing members, in order
        const int a = a0 + lane;
        const bool take = a < ns && C.state[sec[a]] == G_EXISTS;
        const unsigned bal = __ballot_sync(0xffffffffu, take);
        if (take) {
            const int pos = nc + __popc(bal & lt);
            if (pos < K) list[pos] = sec[a]; else overflow = true;
        }
        nc += __popc(bal);
        if (nc > K) nc = K;
    }
    __syncwarp();
    const Box mine = S->box_cur[g];
    for (int a = 0; a < ns; ++a) {
        const int id = sec[a];
        const int* s2 = C.sec_ids + (int64_t)id * C.kmax;
        const int n2 = C.sec_n[id];
        for (int q0 = 0; q0 < n2; q0 += 32) {
            const int q = q0 + lane;
            bool take = false;
            int c = 0;
            if (q < n2) {
                c = s2[q];
                take = C.state[c] == G_EXISTS && c != g && c != 0 && boxes_intersect(mine, S->box_cur[c]);
                if (take)
                    for (int e = 0; e < nc; ++e)
                        if (list[e] == c) {
                            take = false;
                            break;
                        }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, take);
            if (take) {
                const int pos = nc + __popc(bal & lt);
                if (pos < K) list[pos] = c; else overflow = true;
            }
            nc += __popc(bal);
            if (nc > K) nc = K;
            __syncwarp();
        }
    }
    int* cmp = C.cmp_ids + (int64_t)g * C.kmax;
    for (int e = lane; e < nc; e += 32) cmp[e] = list[e];
    if (lane == 0) {
        C.cmp_n[g] = nc;
        if (overflow || C.kmax > kL) set_status(S, overflow ? S_LIST_OVERFLOW : 0u);
    }
}

// LSbox::executeRedistancing (src/box.cpp:1259-1399): one CTA of 64 threads
// per grain.  The output box is built in shared memory when it fits (16 KB,
// small enough for many grains per SM), so the four sweeps (threads over
// columns for y, over rows for x; each column / row a sequential recurrence
// with the running value carried in a register) never re-read global stores;
// the input box is read through L1; the result is clamped to +-delta and
// written back coalesced.
constexpr int kRedistThreads = 64;
constexpr int kRedistSmemBytes = 24 * 1024;

// The four directional sweeps of LSbox::executeRedistancing
// (src/box.cpp:1259-1399) over the new box bo.  The input is read through
// IN(i, j) = in[(i - in_y0) * si + (j - in_x0)] and is only touched inside
// the intersection of bi and bo; the output through OUT(i, j) =
// out[(i - bo.y0) * so + (j - bo.x0)].  One thread per column (y sweeps) or
// row (x sweeps), carrying the running value in a register.
template <typename R>
__device__ void redistance_sweeps_indexed(const R* __restrict__ in, int in_x0, int in_y0, int si, const Box bi,
                                  R* __restrict__ out, int so, const Box bo, R h) {
    const int ixmin = (bi.x0 < bo.x0) ? bo.x0 : bi.x0;
    const int iymin = (bi.y0 < bo.y0) ? bo.y0 : bi.y0;
    const int ixmax = (bi.x1 < bo.x1) ? bi.x1 : bo.x1;
    const int iymax = (bi.y1 < bo.y1) ? bi.y1 : bo.y1;
#define GG_IN(i, j) in[(int64_t)((i) - in_y0) * si + ((j) - in_x0)]
#define GG_OUT(i, j) out[(int64_t)((i) - bo.y0) * so + ((j) - bo.x0)]
    // Each recurrence carries its running value in a register; the loads of
    // the next step (which no store of the current step touches) are issued
    // one step ahead so their latency overlaps the current step.
    for (int j = ixmin + (int)threadIdx.x; j < bo.x1; j += blockDim.x) {
        const bool col_in = j < ixmax;
        if (iymin < bo.y1 - 1) {  // y forward
            R cur = GG_OUT(iymin, j);
            R nxt = GG_OUT(iymin + 1, j);
            R a = (R)0, c = (R)0;
            if (col_in && iymin < iymax - 1) {
                a = GG_IN(iymin, j);
                c = GG_IN(iymin + 1, j);
            }
            for (int i = iymin; i < bo.y1 - 1; i++) {
                const R nxt_n = i + 2 < bo.y1 ? GG_OUT(i + 2, j) : (R)0;
                const R c_n = (col_in && i + 1 < iymax - 1) ? GG_IN(i + 2, j) : (R)0;
                R cand;
                if (col_in && i < iymax - 1) {
                    if (a * c <= (R)0.0) {
                        const R slope = (c - a) / h;
                        const R dz = -a / slope;
                        if (fabs(cur) > fabs(dz)) {
                            cur = -dz * (R)sgn(slope);
                            GG_OUT(i, j) = cur;
                        }
                    }
                    cand = cur + ((R)sgn(c) * h);
                } else {
                    cand = cur + ((R)sgn(nxt) * h);
                }
                if (fabs(cand) < fabs(nxt)) {
                    nxt = cand;
                    GG_OUT(i + 1, j) = nxt;
                }
                cur = nxt;
                nxt = nxt_n;
                a = c;
                c = c_n;
            }
        }
        if (iymax - 1 > bo.y0) {  // y backward
            R cur = GG_OUT(iymax - 1, j);
            R prv = GG_OUT(iymax - 2, j);
            R ip = (col_in && iymax - 1 > iymin) ? GG_IN(iymax - 2, j) : (R)0;
            for (int i = iymax - 1; i > bo.y0; i--) {
                const R prv_n = i - 2 >= bo.y0 ? GG_OUT(i - 2, j) : (R)0;
                const R ip_n = (col_in && i - 1 > iymin) ? GG_IN(i - 2, j) : (R)0;
                R cand;
                if (col_in && i > iymin)
                    cand = cur + ((R)sgn(ip) * h);
                else
                    cand = cur + ((R)sgn(prv) * h);
                if (fabs(cand) < fabs(prv)) {
                    prv = cand;
                    GG_OUT(i - 1, j) = prv;
                }
                cur = prv;
                prv = prv_n;
                ip = ip_n;
            }
        }
    }
    __syncthreads();
    for (int i = iymin + (int)threadIdx.x; i < bo.y1; i += blockDim.x) {
        const bool row_in = i < iymax;
        if (ixmin < bo.x1 - 1) {  // x forward
            R cur = GG_OUT(i, ixmin);
            R nxt = GG_OUT(i, ixmin + 1);
            R a = (R)0, c = (R)0;
            if (row_in && ixmin < ixmax - 1) {
                a = GG_IN(i, ixmin);
                c = GG_IN(i, ixmin + 1);
            }
            for (int j = ixmin; j < bo.x1 - 1; j++) {
                const R nxt_n = j + 2 < bo.x1 ? GG_OUT(i, j + 2) : (R)0;
                const R c_n = (row_in && j + 1 < ixmax - 1) ? GG_IN(i, j + 2) : (R)0;
                R cand;
                if (j < ixmax - 1 && row_in) {
                    if (a * c <= (R)0.0) {
                        const R slope = (c - a) / h;
                        const R dz = -a / slope;
                        if (fabs(cur) > fabs(dz)) {
                            cur = -dz * (R)sgn(slope);
                            GG_OUT(i, j) = cur;
                        }
                    }
                    cand = cur + ((R)sgn(c) * h);
                } else {
                    cand = cur + ((R)sgn(nxt) * h);
                }
                if (fabs(cand) < fabs(nxt)) {
                    nxt = cand;
                    GG_OUT(i, j + 1) = nxt;
                }
                cur = nxt;
                nxt = nxt_n;
                a = c;
                c = c_n;
            }
        }
        if (ixmax - 1 > bo.x0) {  // x backward
            R cur = GG_OUT(i, ixmax - 1);
            R prv = GG_OUT(i, ixmax - 2);
            R ip = (ixmax - 1 > ixmin && row_in) ? GG_IN(i, ixmax - 2) : (R)0;
            for (int j = ixmax - 1; j > bo.x0; j--) {
                const R prv_n = j - 2 >= bo.x0 ? GG_OUT(i, j - 2) : (R)0;
                const R ip_n = (j - 1 > ixmin && row_in) ? GG_IN(i, j - 2) : (R)0;
                R cand;
                if (j > ixmin && row_in)
                    cand = cur + ((R)sgn(ip) * h);
                else
                    cand = cur + (R)sgn(prv) * h;
                if (fabs(cand) < fabs(prv)) {
                    prv = cand;
                    GG_OUT(i, j - 1) = prv;
                }
                cur = prv;
                prv = prv_n;
                ip = ip_n;
            }
        }
    }
#undef GG_IN
#undef GG_OUT
    __syncthreads();
}

// The four directional sweeps of LSbox::executeRedistancing
// (src/box.cpp:1259-1399) over the new box bo.  The input is read through
// IN(i, j) = in[(i - in_y0) * si + (j - in_x0)] and is only touched inside
// the intersection of bi and bo; the output through OUT(i, j) =
// out[(i - bo.y0) * so + (j - bo.x0)].  One thread per column (y sweeps) or
// row (x sweeps), carrying the running value in a register.
template <typename R>
__device__ void redistance_sweeps_walk(const R* __restrict__ in, int in_x0, int in_y0, int si, const Box bi,
                                  R* __restrict__ out, int so, const Box bo, R h) {
    const int ixmin = (bi.x0 < bo.x0) ? bo.x0 : bi.x0;
    const int iymin = (bi.y0 < bo.y0) ? bo.y0 : bi.y0;
    const int ixmax = (bi.x1 < bo.x1) ? bi.x1 : bo.x1;
    const int iymax = (bi.y1 < bo.y1) ? bi.y1 : bo.y1;
    // Each recurrence carries its running value in a register and walks the
    // output (and, inside the intersection, the input) with a pointer; the
    // loads of the next step (which no store of the current step touches) are
    // issued one step ahead so their latency overlaps the current step.  Each
    // sweep is split where the input's region ends, so the loop bodies carry
    // no per-step region test.
    // y sweeps: one thread per column, stride so / si between steps
    for (int j = ixmin + (int)threadIdx.x; j < bo.x1; j += blockDim.x) {
        const bool col_in = j < ixmax;
        R* const ocol = out + (j - bo.x0);
        const R* const icol = in + (j - in_x0);
        if (iymin < bo.y1 - 1) {  // y forward
            const int a_end = col_in ? min(iymax - 1, bo.y1 - 1) : iymin;  // steps that see the input
            R* po = ocol + (iymin - bo.y0) * so;
            const R* pi = icol + (iymin - in_y0) * si;
            R cur = po[0];
            R nxt = po[so];
            int i = iymin;
            if (i < a_end) {
                R a = pi[0], c = pi[si];
                for (; i < a_end; i++) {
                    const R nxt_n = i + 2 < bo.y1 ? po[2 * so] : (R)0;
                    const R c_n = i + 1 < iymax - 1 ? pi[2 * si] : (R)0;
                    if (a * c <= (R)0.0) {
                        const R slope = (c - a) / h;
                        const R dz = -a / slope;
                        if (fabs(cur) > fabs(dz)) {
                            cur = -dz * (R)sgn(slope);
                            po[0] = cur;
                        }
                    }
                    const R cand = cur + ((R)sgn(c) * h);
                    if (fabs(cand) < fabs(nxt)) {
                        nxt = cand;
                        po[so] = nxt;
                    }
                    cur = nxt;
                    nxt = nxt_n;
                    a = c;
                    c = c_n;
                    po += so;
                    pi += si;
                }
            }
            for (; i < bo.y1 - 1; i++) {
                const R nxt_n = i + 2 < bo.y1 ? po[2 * so] : (R)0;
                const R cand = cur + ((R)sgn(nxt) * h);
                if (fabs(cand) < fabs(nxt)) {
                    nxt = cand;
                    po[so] = nxt;
                }
                cur = nxt;
                nxt = nxt_n;
                po += so;
            }
        }
        if (iymax - 1 > bo.y0) {  // y backward
            const int a_end = col_in ? iymin : iymax - 1;  // steps i > a_end see the input
            R* po = ocol + (iymax - 1 - bo.y0) * so;
            R cur = po[0];
            R prv = po[-so];
            int i = iymax - 1;
            if (i > a_end) {
                const R* pi = icol + (iymax - 2 - in_y0) * si;  // IN(i - 1)
                R ip = pi[0];
                for (; i > a_end; i--) {
                    const R prv_n = i - 2 >= bo.y0 ? po[-2 * so] : (R)0;
                    const R ip_n = i - 1 > iymin ? pi[-si] : (R)0;
                    const R cand = cur + ((R)sgn(ip) * h);
                    if (fabs(cand) < fabs(prv)) {
                        prv = cand;
                        po[-so] = prv;
                    }
                    cur = prv;
                    prv = prv_n;
                    ip = ip_n;
                    po -= so;
                    pi -= si;
                }
            }
            for (; i > bo.y0; i--) {
                const R prv_n = i - 2 >= bo.y0 ? po[-2 * so] : (R)0;
                const R cand = cur + ((R)sgn(prv) * h);
                if (fabs(cand) < fabs(prv)) {
                    prv = cand;
                    po[-so] = prv;
                }
                cur = prv;
                prv = prv_n;
                po -= so;
            }
        }
    }
    __syncthreads();
    // x sweeps: one thread per row, unit stride between steps
    for (int i = iymin + (int)threadIdx.x; i < bo.y1; i += blockDim.x) {
        const bool row_in = i < iymax;
        R* const orow = out + (int64_t)(i - bo.y0) * so;
        const R* const irow = in + (int64_t)(i - in_y0) * si;
        if (ixmin < bo.x1 - 1) {  // x forward
            const int a_end = row_in ? min(ixmax - 1, bo.x1 - 1) : ixmin;
            R* po = orow + (ixmin - bo.x0);
            const R* pi = irow + (ixmin - in_x0);
            R cur = po[0];
            R nxt = po[1];
            int j = ixmin;
            if (j < a_end) {
                R a = pi[0], c = pi[1];
                for (; j < a_end; j++) {
                    const R nxt_n = j + 2 < bo.x1 ? po[2] : (R)0;
                    const R c_n = j + 1 < ixmax - 1 ? pi[2] : (R)0;
                    if (a * c <= (R)0.0) {
                        const R slope = (c - a) / h;
                        const R dz = -a / slope;
                        if (fabs(cur) > fabs(dz)) {
                            cur = -dz * (R)sgn(slope);
                            po[0] = cur;
                        }
                    }
                    const R cand = cur + ((R)sgn(c) * h);
                    if (fabs(cand) < fabs(nxt)) {
                        nxt = cand;
                        po[1] = nxt;
                    }
                    cur = nxt;
                    nxt = nxt_n;
                    a = c;
                    c = c_n;
                    ++po;
                    ++pi;
                }
            }
            for (; j < bo.x1 - 1; j++) {
                const R nxt_n = j + 2 < bo.x1 ? po[2] : (R)0;
                const R cand = cur + ((R)sgn(nxt) * h);
                if (fabs(cand) < fabs(nxt)) {
                    nxt = cand;
                    po[1] = nxt;
                }
                cur = nxt;
                nxt = nxt_n;
                ++po;
            }
        }
        if (ixmax - 1 > bo.x0) {  // x backward
            const int a_end = row_in ? ixmin : ixmax - 1;
            R* po = orow + (ixmax - 1 - bo.x0);
            R cur = po[0];
            R prv = po[-1];
            int j = ixmax - 1;
            if (j > a_end) {
                const R* pi = irow + (ixmax - 2 - in_x0);  // IN(i, j - 1)
                R ip = pi[0];
                for (; j > a_end; j--) {
                    const R prv_n = j - 2 >= bo.x0 ? po[-2] : (R)0;
                    const R ip_n = j - 1 > ixmin ? pi[-1] : (R)0;
                    const R cand = cur + ((R)sgn(ip) * h);
                    if (fabs(cand) < fabs(prv)) {
                        prv = cand;
                        po[-1] = prv;
                    }
                    cur = prv;
                    prv = prv_n;
                    ip = ip_n;
                    --po;
                    --pi;
                }
            }
            for (; j > bo.x0; j--) {
                const R prv_n = j - 2 >= bo.x0 ? po[-2] : (R)0;
                const R cand = cur + (R)sgn(prv) * h;
                if (fabs(cand) < fabs(prv)) {
                    prv = cand;
                    po[-1] = prv;
                }
                cur = prv;
                prv = prv_n;
                --po;
            }
        }
    }
    __syncthreads();
}

// The FP32 (batched) form walks pointers with each sweep split where the
// input's region ends (fewer instructions: 0.75 -> 0.68 ms on the 20,000-grain
// workload); the FP64 (plain) form keeps indexed accesses with per-step region
// tests, which the compiler schedules better for doubles (1.75 ms against
// 2.33 ms).  Both evaluate the same expressions in the same order.
template <typename R>
__device__ __forceinline__ void redistance_sweeps(const R* __restrict__ in, int in_x0, int in_y0, int si, const Box bi,
                                                  R* __restrict__ out, int so, const Box bo, R h) {
    if constexpr (sizeof(R) == 4)
        redistance_sweeps_walk<R>(in, in_x0, in_y0, si, bi, out, so, bo, h);
    else
        redistance_sweeps_indexed<R>(in, in_x0, in_y0, si, bi, out, so, bo, h);
}

// LSbox::executeRedistancing of grain g by the whole CTA (any block size).
// When both fit in kSmem bytes, the input over the intersection of the old
// and new boxes and the output box are staged in shared memory with odd row
// strides (so the row-wise sweeps hit distinct banks); a larger box keeps
// only its output there, and the largest stay in global memory.
// clearValues(-1) before, clampValues(-delta, delta) after.
template <typename R, int kSmem>
__device__ void redistance_grain_s(const NetConst& C, NetState* S, int g, unsigned char* s_raw) {
    const R* in_g = phiA_of<R>(S) + S->off_cur[g];
    R* out_g = phiB_of<R>(S) + S->off_new[g];
    const Box bi = S->box_cur[g], bo = S->box_new[g];
    const R h = (R)C.h, delta = (R)C.delta;
    const int wi = box_w(bi), wo = box_w(bo), ho = box_h(bo);
    const int64_t ao = box_area(bo);
    const int ixmin = (bi.x0 < bo.x0) ? bo.x0 : bi.x0;
    const int iymin = (bi.y0 < bo.y0) ? bo.y0 : bi.y0;
    const int ixmax = (bi.x1 < bo.x1) ? bi.x1 : bo.x1;
    const int iymax = (bi.y1 < bo.y1) ? bi.y1 : bo.y1;
    const int wI = ixmax > ixmin ? ixmax - ixmin : 0, hI = iymax > iymin ? iymax - iymin : 0;
    const int so = wo | 1, sI = wI | 1;
    const bool fits = (int64_t)sizeof(R) * ((int64_t)so * ho + (int64_t)sI * hI) <= kSmem;
    if (fits) {
        R* out = reinterpret_cast<R*>(s_raw);
        R* in = out + so * ho;
        // row by row, eight loads in flight per thread
        const R* src = in_g + (int64_t)(iymin - bi.y0) * wi + (ixmin - bi.x0);
        for (int r0 = 0; r0 < hI; r0 += 8)
            for (int c = threadIdx.x; c < wI; c += blockDim.x) {
                R v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = r0 + u < hI ? src[(int64_t)(r0 + u) * wi + c] : (R)0;
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (r0 + u < hI) in[(r0 + u) * sI + c] = v[u];
            }
        for (int p = threadIdx.x; p < so * ho; p += blockDim.x) out[p] = (R)-1.0;  // clearValues(-1)
        __syncthreads();
        redistance_sweeps<R>(in, ixmin, iymin, sI, bi, out, so, bo, h);
        for (int r = 0; r < ho; ++r)  // clampValues(-delta, delta)
            for (int c = threadIdx.x; c < wo; c += blockDim.x) {
                R v = out[r * so + c];
                if (v < -delta)
                    v = -delta;
                else if (v > delta)
                    v = delta;
                out_g[(int64_t)r * wo + c] = v;
            }
    } else if ((int64_t)sizeof(R) * so * ho <= kSmem) {  // output staged, input read in place
        R* out = reinterpret_cast<R*>(s_raw);
        for (int p = threadIdx.x; p < so * ho; p += blockDim.x) out[p] = (R)-1.0;
        __syncthreads();
        redistance_sweeps<R>(in_g, bi.x0, bi.y0, wi, bi, out, so, bo, h);
        for (int r = 0; r < ho; ++r)
            for (int c = threadIdx.x; c < wo; c += blockDim.x) {
                R v = out[r * so + c];
                if (v < -delta)
                    v = -delta;
                else if (v > delta)
                    v = delta;
                out_g[(int64_t)r * wo + c] = v;
            }
    } else {
        for (int64_t p = threadIdx.x; p < ao; p += blockDim.x) out_g[p] = (R)-1.0;
        __syncthreads();
        redistance_sweeps<R>(in_g, bi.x0, bi.y0, wi, bi, out_g, wo, bo, h);
        for (int64_t p = threadIdx.x; p < ao; p += blockDim.x) {
            R v = out_g[p];
            if (v < -delta)
                v = -delta;
            else if (v > delta)
                v = delta;
            out_g[p] = v;
        }
    }
}

// Large boxes (batched form, size bin above NetConst::big_edge, 128 unless
// tuned): k_redistance_big takes them with 256 threads and up to 200 KB of
// shared memory, so a 168^2 box is staged whole and a 256^2 one sweeps 4x as
// many columns at a time.  At 128 the bin starts above the largest boxes of a
// uniform-seed Voronoi network (edge <= 98 at 25 cells per grain), so there
// it is an empty launch.
constexpr int kRedistBigThreads = 256;
constexpr int kRedistBigSmemBytes = 200 * 1024;

// One CTA of 64 threads per grain: every grain in the plain form; in the
// batched form those whose box edge is at most C.big_edge.
template <typename R>
__global__ void __launch_bounds__(kRedistThreads) k_redistance_s(NetConst C, NetState* S) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    const int g = grain_at(S, blockIdx.x);
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    if (S->order && box_w(S->box_cur[g]) > C.big_edge) return;  // the large-box bin
    redistance_grain_s<R, kRedistSmemBytes>(C, S, g, s_raw);
}

// The large-box bin of the batched form: a persistent grid walks the work
// queue (largest boxes first) and stops at the first existing grain at or
// below C.big_edge; k_redistance_s follows it on the same stream (run
// side by side, the two measured slower: the 64-thread kernel's blocks take
// the SMs first).
__global__ void __launch_bounds__(kRedistBigThreads) k_redistance_big(NetConst C, NetState* S) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    if (!S->order) return;
    for (int slot = blockIdx.x; slot < C.N; slot += gridDim.x) {
        const int g = S->order[slot];
        // a grain that vanished in this step's level set keeps its place in
        // the queue; existing grains are in descending box edge
        if (C.state[g] != G_EXISTS || halted(S)) continue;
        if (box_w(S->box_cur[g]) <= C.big_edge) return;
        redistance_grain_s<float, kRedistBigSmemBytes>(C, S, g, s_raw);
        __syncthreads();  // the next grain reuses the shared buffers
    }
}

}  // namespace
}  // namespace gg
