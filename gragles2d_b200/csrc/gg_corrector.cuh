// Anisotropic velocity corrector of the convolution stage
// (LSbox::executeConvolution, src/box.cpp:428-531): per grain, contour
// sectors around the previous step's junctions are built by one warp into
// shared memory, then every pixel projects onto the previous contour and
// blends its convolved value with the sector / junction / boundary weight.
#pragma once

#include <cfloat>
#include "gg_grain.cuh"
#include "gg_kernels.cuh"

namespace gg {
namespace {  // internal linkage: each form's translation unit has its own copy


constexpr int kMaxConstSectors = 32;
constexpr int kMaxSectorJunctions = 24;
constexpr int kMaxInterpSectors = 2 * kMaxConstSectors;
constexpr int kSegShared = 512;  // contours up to this length keep their segment lengths in shared memory

struct ConstSector {
    int left, right;  // contour point IDs (-1, -1: whole contour)
    int nj;
    int js[kMaxSectorJunctions];
    double weight;
};

struct InterpSector {
    int left, right;
    int lb, rb;  // left/right boundary constant sector (-1 if none)
    int len0, len1;  // segments summed into length: len0 .. len1 forward (len0 = -1: none)
    double length;
    double left_w, right_w, boundary_w;
};

struct SectorSet {
    int nconst, ninterp;
    uint32_t status;
    ConstSector cs[kMaxConstSectors];
    InterpSector is[kMaxInterpSectors];
};

// Per contour segment: the sector getWeight would pick (first constant
// sector containing it, else first interpolating sector, else none) and, for
// an interpolating sector, the partial sum of segment lengths from the
// sector's right point up to the segment, accumulated in the same order as
// ContourSector::getWeight (src/contourSector.cpp:242-246).
constexpr int kSegTable = 512;
struct SegTable {
    short sector[kSegTable];  // >= 0 constant, <= -2 interpolating (-2 - q), -1 none
    double acc[kSegTable];
};

// characteristics lookup of ExplicitGrainBoundary::getDirectNeighbourCaracteristic
// (src/grainBoundary.cpp:561-571): by grain ID; a removed grain matches
// nothing; absent -> default (energy 1, mobility 1).
__device__ __forceinline__ const Neighbour* find_characteristic(const NetConst& C, int owner, int id) {
    if (id < 0 || id > C.N || (id != 0 && C.state[id] == G_GONE)) return nullptr;
    if (owner == 0) return nullptr;  // the boundary grain keeps no neighbour list
    const Neighbour* nb = C.nb + (int64_t)owner * C.nbmax;
    const int n = C.nb_n[owner];
    for (int e = 0; e < n; ++e)
        if (nb[e].id == id) return &nb[e];
    return nullptr;
}

// LSbox::getGBEnergyTimesGBMobility(LSbox*) (src/box.cpp:554-561)
__device__ __forceinline__ double gb_weight_for(const NetConst& C, int owner, int id) {
    const Neighbour* c = find_characteristic(C, owner, id);
    const double e = c ? c->energy : 1.0, mo = c ? c->mobility : 1.0;
    if (e * mo > 0.01) return e * mo;
    return 0.01;
}

// The owner's direct-neighbour weights (energy x mobility floored at 0.01)
// for the per-pixel default weight; entries of removed grains are dropped
// because a removed grain matches no characteristic.
struct NbTable {
    int n;
    int id[48];
    double w[48];
    double f[48];   // stored-energy driving force (own - neighbour energy) x mobility, when stored energies are on
    double fm[48];  // magnetic driving force, the same with the magnetic energies, when the field is on
};

__device__ void build_nb_table(const NetConst& C, int owner, NbTable& T) {
    const Neighbour* nb = C.nb + (int64_t)owner * C.nbmax;
    const int n = min(C.nb_n[owner], 48);
    if (threadIdx.x == 0) T.n = n;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int id = nb[e].id;
        const bool gone = id < 0 || id > C.N || (id != 0 && C.state[id] == G_GONE);
        T.id[e] = gone ? -2 : id;
        const double v = nb[e].energy * nb[e].mobility;
        T.w[e] = v > 0.01 ? v : 0.01;
        T.f[e] = (C.stored && !gone) ? (C.stored[owner] - C.stored[id]) * nb[e].mobility : 0.0;
        T.fm[e] = (C.magnetic && !gone) ? (C.magnetic[owner] - C.magnetic[id]) * nb[e].mobility : 0.0;
    }
}

// ExplicitGrainBoundary::get_f_StoredElasticEnergy (src/grainBoundary.cpp:
// 607-615) for the grain `id`: the first characteristic with that ID, else -1.
__device__ __forceinline__ double nb_stored_force(const NbTable& T, int id) {
    for (int e = 0; e < T.n; ++e)
        if (T.id[e] == id) return T.f[e];
    return -1.0;
}

// ExplicitGrainBoundary::get_f_magneticEnergy (src/grainBoundary.cpp:623-631).
__device__ __forceinline__ double nb_magnetic_force(const NbTable& T, int id) {
    for (int e = 0; e < T.n; ++e)
        if (T.id[e] == id) return T.fm[e];
    return -1.0;
}

// The driving-force terms the corrector subtracts at (row, col), stored
// energy first, then magnetic (src/box.cpp:511-527): f(IDLocal) dt / TimeSlope.
template <typename R>
__device__ __forceinline__ R subtract_driving_forces(const NetConst& C, const NbTable& T, const uint32_t* idl,
                                                     const Box& ib, int row, int col, R value, uint32_t* status) {
    uint32_t k;
    if (!buf_index(ib, row, col, &k)) {
        *status |= S_INDEX;
        return value;
    }
    const int id = (int)idl[k];
    if (C.stored) value = (R)((double)value - nb_stored_force(T, id) * C.dt / C.time_slope);
    if (C.magnetic) value = (R)((double)value - nb_magnetic_force(T, id) * C.dt / C.time_slope);
    return value;
}

// getGBEnergyTimesGBMobility(i, j) through the table (first match, as the
// reference's linear search).
__device__ __forceinline__ double table_weight_at(const NbTable& T, const uint32_t* idl, const Box& ib, int row,
                                                  int col, uint32_t* status) {
    uint32_t k;
    if (!buf_index(ib, row, col, &k)) {
        *status |= S_INDEX;
        return 1.0;
    }
    const int id = (int)idl[k];
    for (int e = 0; e < T.n; ++e)
        if (T.id[e] == id) return T.w[e];
    return 1.0;
}

// GrainJunction::getWeight (src/junction.cpp:23-192), mode 4, ResearchMode 0,
// ResearchProject 0, no twin identification, for every junction of grain
// `me`: a group of three lanes per junction, ten junctions per warp at once.
// The group's lanes evaluate the three grain pairs (me-n0, n0-n1, me-n1) side
// by side, the second one also finding n1 in n0's characteristics (first
// match); the first lane then combines the terms in the reference's order,
// so each weight is the value the sequential routine computes.
__device__ void junction_weights(const NetConst& C, const Junction* J, int nj, int me, double* jw,
                                 uint32_t* s_status) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int grp = lane / 3, role = lane - 3 * grp;  // lanes 30 and 31 have no junction
    for (int q0 = warp * 10; q0 < nj; q0 += nw * 10) {
        const int q = q0 + grp;
        const bool act = grp < 10 && q < nj;
        int n0 = 0, n1 = 0;
        bool missing = true, bad_index = false;
        if (act) {
            const int type = J[q].type;
            uint32_t nbr[4] = {0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu, 0xFFFFFFu};
            for (int i = 0, j = 0; i < type && i < 4; i++) {
                const uint32_t gi = J[q].grains[i];
                if ((uint32_t)me != gi) {
                    nbr[j] = gi;
                    j++;
                }
            }
            missing = nbr[0] == 0xFFFFFFu || nbr[1] == 0xFFFFFFu;
            if (!missing) {
                n0 = (int)nbr[0];
                n1 = (int)nbr[1];
                bad_index = n0 > C.N || n1 > C.N;
            }
        }
        double mob = 0, gam = 0;
        if (act && !missing && !bad_index) {
            double c01_mob = 1.0;
            if (role == 1 && !(n1 != 0 && C.state[n1] == G_GONE) && n0 != 0) {
                // characteristics of n1 in n0's list (find_characteristic, first match)
                const Neighbour* nb = C.nb + (int64_t)n0 * C.nbmax;
                const int n = C.nb_n[n0];
                for (int e = 0; e < n; ++e)
                    if (nb[e].id == n1) {
                        c01_mob = nb[e].mobility;
                        break;
                    }
            }
            const double* pa = C.quat + 4 * (int64_t)(role == 1 ? n0 : me);
            const double* pb = C.quat + 4 * (int64_t)(role == 0 ? n0 : n1);
            const double theta = grain_misorientation(pa, pb);
            gam = read_shockley(theta, C);
            mob = role == 1 ? c01_mob : mobility_model(theta, C);
        }
        const int l1 = lane + 1 < 32 ? lane + 1 : 31, l2 = lane + 2 < 32 ? lane + 2 : 31;
        const double m1 = __shfl_sync(FULL, mob, l1), m2 = __shfl_sync(FULL, mob, l2);
        const double g1 = __shfl_sync(FULL, gam, l1), g2 = __shfl_sync(FULL, gam, l2);
        if (act && role == 0) {
            if (missing) {
                jw[q] = 1;
            } else if (bad_index) {
                jw[q] = 1;
                atomicOr(s_status, S_INDEX);
            } else {
                if ((n0 != 0 && C.state[n0] == G_GONE) || (n1 != 0 && C.state[n1] == G_GONE))
                    atomicOr(s_status, S_INDEX);
                double averageMobility = 0;
                averageMobility += mob;
                averageMobility += m1;
                averageMobility += m2;
                double sigma = gam - g1 + g2;
                if (!C.isotropic) {
                    if (C.use_mobility_model > 0 && C.tpd > 0) {
                        averageMobility /= 3;
                        const double drag = 1 / ((1 / (C.ds * C.tpd)) + 1 / averageMobility);
                        sigma *= drag;
                    }
                }
                if (sigma < 0.01) sigma = 0.01;
                jw[q] = sigma;
            }
        }
    }
}

__device__ __forceinline__ double seg_len(const CPoint* P, int a, int b) {
    const double dx = P[a].x - P[b].x, dy = P[a].y - P[b].y;
    return sqrt(dx * dx + dy * dy);
}

// ContourSector::isSegmentWithinSector (src/contourSector.cpp:184-198)
__device__ __forceinline__ bool within(int left, int right, int totalP, int segment) {
    if (right == left && left == -1) return true;
    if (right > left) return (segment >= 0 && segment <= left) || (segment >= right && segment < totalP);
    return segment >= right && segment <= left;
}

// Iteration bound of a walk along the contour that stops once it has covered
// `radius`: the reference's loops (which have no bound) end after
// ceil(radius / perimeter) laps; a zero-length contour would never end.
__device__ __forceinline__ long lap_guard(double perimeter, int size, double radius, uint32_t* status) {
    if (!(perimeter > 0)) {
        *status |= S_SECTOR_GUARD;
        return 2L * size + 8;
    }
    const double laps = ceil(radius / perimeter) + 2.0;
    return (long)(laps * (size + 1)) + 8;
}

// Whole laps of a contour walk at once, with the step-by-step result.  A walk
// adds seg[p], seg[p + dir], ... (indices mod n) to dist while dist stays
// below a limit; on a nearly vanished grain (perimeter far below the sector
// radius) that takes millions of steps.  Inside one binade [2^(e-1), 2^e)
// every double is a multiple of u = 2^(e-53), so each rounded addition
// dist + s adds exactly u * rint(s / u), unless s / u ends in exactly one
// half (the rounding would then depend on dist's last bit): a lap adds the
// exact quantum Q, and m laps that stay below the binade's top and the limit
// add m Q with no rounding at all.  Returns the laps taken (0 when the skip
// does not apply); it leaves at least two laps before the limit, so the
// caller's next step still runs, and takes at most `max_laps`.
constexpr long kSkipAfter = 64;  // steps before a walk tries to skip laps

__device__ long skip_laps(double* dist, double limit, const double* seg, int p, int dir, int n, long max_laps) {
    const double d = *dist;
    if (!(d >= DBL_MIN) || !(d < limit) || n <= 0 || max_laps < 1) return 0;
    int e;
    frexp(d, &e);
    const double u = ldexp(1.0, e - 53);
    const double top = ldexp(1.0, e);
    double Q = 0;
    int k = p;
    for (int i = 0; i < n; ++i) {
        const double r = seg[k] / u;  // exact: u is a power of two
        if (r - floor(r) == 0.5) return 0;
        Q += rint(r) * u;
        k += dir;
        if (k >= n) k -= n;
        if (k < 0) k += n;
    }
    if (!(Q > 0)) return 0;
    double mm = floor((fmin(limit, top) - d) / Q) - 2;
    if (mm > (double)max_laps) mm = (double)max_laps;
    if (!(mm >= 1)) return 0;
    const long m = (long)mm;
    *dist = d + (double)m * Q;  // m Q < top - d: a multiple of u, exact
    return m;
}

// ExplicitGrainBoundary::setPointsOnBoundary (src/grainBoundary.cpp:524-559).
// seg[k] = |P[k+1] - P[k]| h, the term the reference recomputes at every step
// of its walks (same expression, so the sums are bit-identical).
__device__ void set_points_on_boundary(const CPoint* P, const double* seg, int size, const Junction& J0, double h,
                                       double csr, long guard, int* left, int* right, uint32_t* status) {
    double dist = 0;
    int l = J0.segment;
    {
        const int nx = periodic(l + 1, size);
        const double dx = (P[nx].x - P[l].x) * (1 - J0.lambda), dy = (P[nx].y - P[l].y) * (1 - J0.lambda);
        dist += sqrt(dx * dx + dy * dy) * h;
    }
    l = periodic(l + 1, size);
    long it = 0;
    const int n = size - 1;
    while (dist < csr) {
        if (it >= kSkipAfter && (it & (kSkipAfter - 1)) == 0)
            it += n * skip_laps(&dist, csr, seg, l, 1, n, (guard - it) / n - 2);
        dist += seg[l];
        l = periodic(l + 1, size);
        if (++it > guard) {
            *status |= S_SECTOR_GUARD;
            break;
        }
    }
    dist = 0;
    int r = J0.segment;
    {
        const int nx = periodic(r + 1, size);
        const double dx = (P[nx].x - P[r].x) * J0.lambda, dy = (P[nx].y - P[r].y) * J0.lambda;
        dist += sqrt(dx * dx + dy * dy) * h;
    }
    r = periodic(r, size);
    it = 0;
    while (dist < csr) {
        if (it >= kSkipAfter && (it & (kSkipAfter - 1)) == 0)
            it += n * skip_laps(&dist, csr, seg, periodic(r - 1, size), -1, n, (guard - it) / n - 2);
        dist += seg[periodic(r - 1, size)];
        r = periodic(r - 1, size);
        if (++it > guard) {
            *status |= S_SECTOR_GUARD;
            break;
        }
    }
    *right = r;
    *left = l;
}

// ExplicitGrainBoundary::buildBoundarySectors (src/grainBoundary.cpp:233-342)
// plus the per-sector weights of ContourSector::getWeight
// (src/contourSector.cpp:200-272) that do not depend on the pixel, run by the
// 32 lanes of the calling warp.  The contour walks of the reference's
// sequential build are independent per junction (setPointsOnBoundary) and per
// pair of neighbouring constant sectors (the interpolating contours), so
// lanes run them side by side; the order-dependent merge of junction sectors
// runs on lane 0 over the walked end points.  Every sector, end point and
// weight is the one the sequential build produces.
__device__ void build_sectors_warp(const NetConst& C, const NbTable& T, const CPoint* P, const double* seg,
                                   double perimeter, int size, const Junction* J, int nj, const uint32_t* idl,
                                   const Box& ib, SectorSet& S, const double* jw, int* jl, int* jr) {
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        S.nconst = 0;
        S.ninterp = 0;
        S.status = 0;
    }
    __syncwarp();
    if (nj == 0) return;
    const double h = C.h;
    const int real = size - 1;
    uint32_t st = 0;
    const long guard = lap_guard(perimeter, size, C.isr > C.csr ? C.isr : C.csr, &st);
    // 1. sector end points of every junction (setPointsOnBoundary)
    for (int q = lane; q < nj; q += 32)
        set_points_on_boundary(P, seg, size, J[q], h, C.csr, guard, &jl[q], &jr[q], &st);
    __syncwarp();
    // 2. merge the junction sectors in junction order
    if (lane == 0) {
        auto push_const = [&](int jidx) -> int {
            if (S.nconst >= kMaxConstSectors) {
                st |= S_JUNCTION_OVERFLOW;
                return -1;
            }
            ConstSector& c = S.cs[S.nconst];
            c.nj = 1;
            c.js[0] = jidx;
            c.left = jl[jidx];
            c.right = jr[jidx];
            return S.nconst++;
        };
        auto merge = [&](ConstSector& c, int jidx) {
            if (c.nj < kMaxSectorJunctions)
                c.js[c.nj++] = jidx;
            else
                st |= S_JUNCTION_OVERFLOW;
        };
        push_const(0);
        int cb = 0;
        for (int i = 1; i < nj; i++) {
            const int cl = jl[i], cr = jr[i];
            if (within(S.cs[cb].left, S.cs[cb].right, real, cr)) {
                merge(S.cs[cb], i);
                S.cs[cb].left = cl;
                if (i == nj - 1) {
                    if (within(S.cs[0].left, S.cs[0].right, real, S.cs[cb].left)) {
                        if (cb == 0) {
                            S.cs[0].left = -1;
                            S.cs[0].right = -1;
                        } else {
                            const int cnt = S.cs[cb].nj;
                            for (int q = 0; q < cnt; q++) merge(S.cs[0], S.cs[cb].js[q]);
                            S.cs[0].right = S.cs[cb].right;
                        }
                    }
                }
            } else {
                if (i == nj - 1 && within(S.cs[0].left, S.cs[0].right, real, cl)) {
                    S.cs[0].right = cr;
                    merge(S.cs[0], i);
                } else {
                    if (push_const(i) >= 0) cb++;
                }
            }
        }
    }
    __syncwarp();
    const int nconst = S.nconst;
    // 3. constant-sector weights: mean of junction weights in list order
    for (int s = lane; s < nconst; s += 32) {
        double w = 0;
        for (int q = 0; q < S.cs[s].nj; ++q) w += jw[S.cs[s].js[q] < 64 ? S.cs[s].js[q] : 63];
        S.cs[s].weight = w / (double)S.cs[s].nj;
    }
    __syncwarp();
    if (nconst > 1 || S.cs[0].left != S.cs[0].right) {
        // 4. interpolating sectors between constant sector i and i + 1
        InterpSector out0, out1;
        int cnt = 0;
        if (nconst > 1 && lane < nconst) {
            const int iR = lane, iL = (lane + 1 + nconst) % nconst;
            const ConstSector& secR = S.cs[iR];
            const ConstSector& secL = S.cs[iL];
            // secR.generateLeftInterpolatingContour (src/contourSector.cpp:103-122)
            InterpSector nr;
            {
                double dist = 0;
                int j = secR.left, last = -1;
                long it = 0;
                for (; dist <= C.isr; j = wrap_next(j, real)) {
                    if (it >= kSkipAfter && (it & (kSkipAfter - 1)) == 0)
                        it += real * skip_laps(&dist, C.isr, seg, j, 1, real, (guard - it) / real - 2);
                    dist += seg[j];
                    last = j;
                    if (++it > guard) {
                        st |= S_SECTOR_GUARD;
                        break;
                    }
                }
                nr.left = wrap_next(j, real);
                nr.right = secR.left;
                nr.lb = -1;
                nr.rb = iR;
                nr.len0 = last < 0 ? -1 : secR.left;
                nr.len1 = last;
                nr.length = dist;
            }
            // secL.generateRightInterpolatingContour (src/contourSector.cpp:145-168)
            InterpSector nl;
            {
                double dist = 0;
                int j = secL.right, last = -1;
                long it = 0;
                for (; dist <= C.isr; j = wrap_prev(j, real)) {
                    if (it >= kSkipAfter && (it & (kSkipAfter - 1)) == 0)
                        it += real * skip_laps(&dist, C.isr, seg, wrap_prev(j, real), -1, real, (guard - it) / real - 2);
                    dist += seg[wrap_prev(j, real)];
                    last = wrap_prev(j, real);
                    if (++it > guard) {
                        st |= S_SECTOR_GUARD;
                        break;
                    }
                }
                nl.left = secL.right;
                nl.right = wrap_prev(j, real);
                nl.lb = iL;
                nl.rb = -1;
                nl.len0 = last;
                nl.len1 = last < 0 ? -1 : wrap_prev(secL.right, real);
                nl.length = dist;
            }
            bool merged = false;
            {
                int it = 0;
                for (int j = nr.right; j != periodic(nr.left + 1, size); j = periodic(j + 1, size)) {
                    if (j == nl.left || j == nl.right) merged = true;
                    if (++it > size + 1) {
                        st |= S_SECTOR_GUARD;
                        break;
                    }
                }
            }
            if (merged) {
                // secL.generateInterpolatingSector(secR) (src/contourSector.cpp:124-143)
                InterpSector r;
                r.left = secL.right;
                r.lb = iL;
                r.right = secR.left;
                r.rb = iR;
                double dist = 0;
                int it = 0, last = -1;
                for (int j = r.right; j != r.left; j = wrap_next(j, real)) {
                    dist += seg[wrap_prev(j, real)];
                    last = wrap_prev(j, real);
                    if (++it > size + 1) {
                        st |= S_SECTOR_GUARD;
                        break;
                    }
                }
                r.len0 = last < 0 ? -1 : wrap_prev(r.right, real);
                r.len1 = last;
                r.length = dist;
                out0 = r;
                cnt = 1;
            } else {
                out0 = nr;
                out1 = nl;
                cnt = 2;
            }
        }
        // sectors in pair order (at most 2 x 32 = kMaxInterpSectors)
        int pos = cnt;
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, pos, d);
            if (lane >= d) pos += v;
        }
        const int total = __shfl_sync(0xffffffffu, pos, 31);
        pos -= cnt;
        if (cnt >= 1) S.is[pos] = out0;
        if (cnt == 2) S.is[pos + 1] = out1;
        if (lane == 0) S.ninterp = total;
        __syncwarp();
        // 5. interpolating-sector end weights (pixel independent)
        for (int s = lane; s < total; s += 32) {
            InterpSector& q = S.is[s];
            if (q.lb >= 0) {
                q.left_w = S.cs[q.lb].weight;
            } else {
                const int sx = (int)P[q.left].x, sy = (int)P[q.left].y;
                q.left_w = table_weight_at(T, idl, ib, sy, sx, &st);
            }
            if (q.rb >= 0) {
                q.right_w = S.cs[q.rb].weight;
            } else {
                const int sx = (int)P[q.right].x, sy = (int)P[q.right].y;
                q.right_w = table_weight_at(T, idl, ib, sy, sx, &st);
            }
            q.boundary_w = 0;
            if (q.lb >= 0 && q.rb >= 0) {
                const CPoint& smp = P[(q.right + 1) % real];
                q.boundary_w = table_weight_at(T, idl, ib, (int)smp.y, (int)smp.x, &st);
            }
        }
    }
    // status bits of all lanes
    for (int d = 16; d > 0; d >>= 1) st |= __shfl_xor_sync(0xffffffffu, st, d);
    __syncwarp();
    if (lane == 0) S.status |= st;
    __syncwarp();
}

// Segment q's entry of the per-segment table (see SegTable).
__device__ __forceinline__ void seg_table_entry(const SectorSet& S, const double* seg, int size, int q, int* sid_out,
                                                double* acc_out) {
    const int real = size - 1;
    int sid = -1;
    for (int c = 0; c < S.nconst; c++)
        if (within(S.cs[c].left, S.cs[c].right, real, q)) {
            sid = c;
            break;
        }
    if (sid < 0)
        for (int c = 0; c < S.ninterp; c++)
            if (within(S.is[c].left, S.is[c].right, real, q)) {
                sid = -2 - c;
                break;
            }
    double acc = 0;
    if (sid <= -2) {
        const int k0 = S.is[-2 - sid].right;
        int it = 0;
        for (int k = k0; k != q; k = wrap_next(k, real)) {
            acc += seg[k];
            if (++it > size) break;
        }
    }
    *sid_out = sid;
    *acc_out = acc;
}

__device__ void build_seg_table(const SectorSet& S, const double* seg, int size, SegTable& T) {
    for (int q = threadIdx.x; q < size - 1; q += blockDim.x) {
        int sid;
        double acc;
        seg_table_entry(S, seg, size, q, &sid, &acc);
        T.sector[q] = (short)sid;
        T.acc[q] = acc;
    }
}

// The sectors of a grain as the batched corrector reads them, built one step
// ahead (k_sectors): the constant sectors' weights and the interpolating
// sectors; the per-segment table lives beside the contour (NetConst::segsec,
// segacc at the contour's offsets).
struct SectorPack {
    int32_t nconst, ninterp;
    uint32_t status, pad;
    double cw[kMaxConstSectors];
    InterpSector is[kMaxInterpSectors];
};

// ExplicitGrainBoundary::getWeight (src/grainBoundary.cpp:344-363) for one pixel.
__device__ __forceinline__ double pixel_weight(const NetConst& C, const NbTable& T, const CPoint* P,
                                               const double* seg, int size, const SectorSet& S,
                                               const SegTable* ST, const uint32_t* idl, const Box& ib, int i, int j,
                                               uint32_t* status) {
    double lambda = 0.0;
    const int segment = project_to_boundary(P, size, (double)j, (double)i, &lambda);
    const int real = size - 1;
    int sid = -1;
    double interpolator = 0;
    if (ST) {
        sid = ST->sector[segment];
        if (sid <= -2) interpolator = ST->acc[segment];
    } else {
        for (int q = 0; q < S.nconst && sid == -1; q++)
            if (within(S.cs[q].left, S.cs[q].right, real, segment)) sid = q;
        for (int q = 0; q < S.ninterp && sid == -1; q++)
            if (within(S.is[q].left, S.is[q].right, real, segment)) sid = -2 - q;
        if (sid <= -2) {
            int it = 0;
            for (int k = S.is[-2 - sid].right; k != segment; k = wrap_next(k, real)) {
                interpolator += seg[k];
                if (++it > size) break;
            }
        }
    }
    if (sid >= 0) return S.cs[sid].weight;
    if (sid == -1) return table_weight_at(T, idl, ib, i, j, status);
    const InterpSector& s = S.is[-2 - sid];
    const int k = segment;
    const int kn = wrap_next(k, real);
    const double ax = (P[kn].x - P[k].x) * lambda, ay = (P[kn].y - P[k].y) * lambda;
    interpolator += sqrt(ax * ax + ay * ay);
    interpolator /= s.length;
    if (interpolator < 0) interpolator = 0;
    if (interpolator > 1) interpolator = 1;
    if (s.lb >= 0 && s.rb >= 0) {
        const double isr = C.isr;
        const double quot = (s.length > 2 * isr ? 2 * isr : s.length);
        const double amplitude =
            (s.boundary_w - (s.left_w + s.right_w) / 2) / (2 * isr) * quot + (s.left_w + s.right_w) / 2;
        const double a0 = 2 * s.right_w;
        const double a1 = -4 * amplitude;
        const double a2 = 2 * s.left_w;
        const double A = a0 + a1 + a2;
        const double B = -(a0 * 1.5 + a1 + a2 * 0.5);
        const double Cc = a0 * 0.5;
        return A * interpolator * interpolator + B * interpolator + Cc;
    }
    return interpolator * s.left_w + (1 - interpolator) * s.right_w;
}

// Per-grain preparation shared by both correctors: segment lengths (into
// the seg scratch, one thread per segment) and the neighbour table, junction
// weights (one warp per junction), perimeter, then the sector build by warp
// 0 (all its lookups in shared memory).  jl, jr: shared scratch of 64 ints.
// The same on explicit roles: the contour P, its IDLocal map idl on box ib
// and its junctions J (nj of them).
__device__ void prepare_sectors_view(const NetConst& C, NetState* S, int g, const CPoint* P, int size, double* seg,
                                     SectorSet& sec, double* jw, uint32_t* s_st, double* s_per, NbTable& T, int* jl,
                                     int* jr, Box ib, const uint32_t* idl, const Junction* J, int nj);

__device__ void prepare_sectors(const NetConst& C, NetState* S, int g, const CPoint* P, int size, double* seg,
                                SectorSet& sec, double* jw, uint32_t* s_st, double* s_per, NbTable& T, int* jl,
                                int* jr) {
    prepare_sectors_view(C, S, g, P, size, seg, sec, jw, s_st, s_per, T, jl, jr, S->box_prev[g],
                         S->idPrev + S->off_prev[g], S->jPrev + (int64_t)g * C.jmax, min(S->jn_prev[g], 64));
}

__device__ void prepare_sectors_view(const NetConst& C, NetState* S, int g, const CPoint* P, int size, double* seg,
                                     SectorSet& sec, double* jw, uint32_t* s_st, double* s_per, NbTable& T, int* jl,
                                     int* jr, Box ib, const uint32_t* idl, const Junction* J, int nj) {
    if (threadIdx.x == 0) *s_st = 0;
    for (int k = threadIdx.x; k < size - 1; k += blockDim.x) {
        const double dx = P[k + 1].x - P[k].x, dy = P[k + 1].y - P[k].y;
        seg[k] = sqrt(dx * dx + dy * dy) * C.h;
    }
    build_nb_table(C, g, T);
    __syncthreads();
    junction_weights(C, J, nj, g, jw, s_st);
    __syncthreads();
    if (threadIdx.x < 32) {
        // the perimeter only bounds the sector walks (lap_guard): a tree sum
        double per = 0;
        for (int k = threadIdx.x; k < size - 1; k += 32) per += seg[k];
        for (int o = 16; o > 0; o >>= 1) per += __shfl_down_sync(0xffffffffu, per, o);
        per = __shfl_sync(0xffffffffu, per, 0);
        if (threadIdx.x == 0) *s_per = per;
        build_sectors_warp(C, T, P, seg, per, size, J, nj, idl, ib, sec, jw, jl, jr);
        if (threadIdx.x == 0 && (sec.status | *s_st)) set_status(S, sec.status | *s_st);
    }
    __syncthreads();
}

template <typename R>
__global__ void __launch_bounds__(128) k_corrector(NetConst C, NetState* S) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || C.regular[g] == 0 || S->loop == 0 || halted(S)) return;
    __shared__ SectorSet sec;
    __shared__ double jw[64];
    __shared__ uint32_t s_st;
    __shared__ double s_per;
    __shared__ NbTable nbt;
    __shared__ double s_seg[kSegShared];
    __shared__ SegTable stab;
    __shared__ int jl[64], jr[64];
    const CPoint* P = S->contPrev + S->coff_prev[g];
    const int size = S->cn_prev[g];
    if (size < 2) return;
    double* seg = size - 1 <= kSegShared ? s_seg : S->segPrev + S->coff_prev[g];
    const Box ib = S->box_prev[g];
    const uint32_t* idl = S->idPrev + S->off_prev[g];
    prepare_sectors(C, S, g, P, size, seg, sec, jw, &s_st, &s_per, nbt, jl, jr);
    const bool tabled = size - 1 <= kSegTable;
    if (tabled) build_seg_table(sec, seg, size, stab);
    __syncthreads();
    const Box bo = S->box_cur[g];
    const int x0 = ib.x0 < bo.x0 ? bo.x0 : ib.x0;
    const int y0 = ib.y0 < bo.y0 ? bo.y0 : ib.y0;
    const int x1 = ib.x1 > bo.x1 ? bo.x1 : ib.x1;
    const int y1 = ib.y1 > bo.y1 ? bo.y1 : ib.y1;
    if (x1 <= x0 || y1 <= y0) return;
    const int w = x1 - x0;
    const int64_t cnt = (int64_t)w * (y1 - y0);
    const R* in = phiA_of<R>(S) + S->off_cur[g];
    R* out = phiB_of<R>(S) + S->off_cur[g];
    const int wo = box_w(bo);
    const R delta = (R)C.delta;
    uint32_t st = 0;
    for (int64_t p = threadIdx.x; p < cnt; p += blockDim.x) {
        const int i = y0 + (int)(p / w), j = x0 + (int)(p % w);
        const int64_t k = (int64_t)(i - bo.y0) * wo + (j - bo.x0);
        const R val = in[k];
        if (val > -delta) {
            const double weight = pixel_weight(C, nbt, P, seg, size, sec, tabled ? &stab : nullptr, idl, ib, i, j, &st);
            out[k] = (R)((double)val + ((double)out[k] - (double)val) * weight * 1.0);
        } else {
            out[k] = -delta;
        }
        if (C.stored || C.magnetic) out[k] = subtract_driving_forces<R>(C, nbt, idl, ib, i, j, out[k], &st);
    }
    if (st) set_status(S, st);
}

}  // namespace
}  // namespace gg
