// Stage kernels of one level-set timestep over all grains, templated on the
// distance-field element type R (double: plain form; float: batched form).
// Each kernel cites the reference stage it implements.
#pragma once

#include <cuda_runtime.h>

#include "gg_device.cuh"
#include "gg_grain.cuh"

namespace gg {
namespace {  // internal linkage: each form's translation unit has its own copy


template <typename R>
__device__ __forceinline__ R* phiA_of(NetState* S) {
    return reinterpret_cast<R*>(S->phiA);
}
template <typename R>
__device__ __forceinline__ R* phiB_of(NetState* S) {
    return reinterpret_cast<R*>(S->phiB);
}

// ---------------------------------------------------------------------------
// Convolution, plain form (src/box.cpp:622-695 with the FFTW transforms
// evaluated as separable direct DFTs in a fixed summation order): one CTA
// per grain, phi_t (arena A) -> convolved field (arena B, same box).
// Row r2c, column DFT and Gaussian multiply, inverse column DFT, row c2r.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_conv_dft(NetConst C, NetState* S, int tk = -1) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    const Box bx = S->box_cur[g];
    const int n = box_w(bx);
    if (n <= 0) return;
    if (n != box_h(bx) || n > C.tmax) {
        if (threadIdx.x == 0) set_status(S, n > C.tmax ? S_TABLE_RANGE : S_INDEX);
        return;
    }
    const int half = n / 2 + 1;
    // tk >= 0: the same (linear) convolution of tangent field tk
    const R* in = (tk < 0 ? phiA_of<R>(S) : reinterpret_cast<R*>(S->dphiA) + tk * S->phi_cap) + S->off_cur[g];
    R* out = (tk < 0 ? phiB_of<R>(S) : reinterpret_cast<R*>(S->dphiB) + tk * S->phi_cap) + S->off_cur[g];
    R* s1 = reinterpret_cast<R*>(S->spec) + S->soff_cur[g];  // n x half complex
    R* s2 = s1 + 2 * (int64_t)n * half;                        // n x half complex
    const double* w = C.tw + 2 * C.tw_off[n];
    const double* G = C.gk + C.gk_off[n];
    const int tot = n * half;

    // rows: T[r][f] = sum_c x[r][c] w^(f c)
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int r = idx / half, f = idx - r * half;
        R re = 0, im = 0;
        const R* xr = in + r * n;
        int k = 0;
        for (int c = 0; c < n; ++c) {
            const R v = xr[c];
            re = re + v * (R)w[2 * k];
            im = im + v * (R)w[2 * k + 1];
            k += f;
            if (k >= n) k -= n;
        }
        s1[2 * idx] = re;
        s1[2 * idx + 1] = im;
    }
    __syncthreads();
    // columns: Y[q][f] = sum_r T[r][f] w^(q r), then * G(f, min(q, n-q))
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int q = idx / half, f = idx - q * half;
        R re = 0, im = 0;
        int k = 0;
        for (int r = 0; r < n; ++r) {
            const R a = s1[2 * (r * half + f)], b = s1[2 * (r * half + f) + 1];
            const R wc = (R)w[2 * k], ws = (R)w[2 * k + 1];
            re = re + (a * wc - b * ws);
            im = im + (a * ws + b * wc);
            k += q;
            if (k >= n) k -= n;
        }
        const int j2 = q < n - q ? q : n - q;
        const R gv = (R)G[f * half + j2];
        s2[2 * idx] = re * gv;
        s2[2 * idx + 1] = im * gv;
    }
    __syncthreads();
    // inverse columns: T[r][f] = sum_q Y[q][f] conj(w)^(q r)
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int r = idx / half, f = idx - r * half;
        R re = 0, im = 0;
        int k = 0;
        for (int q = 0; q < n; ++q) {
            const R a = s2[2 * (q * half + f)], b = s2[2 * (q * half + f) + 1];
            const R wc = (R)w[2 * k], ws = -(R)w[2 * k + 1];
            re = re + (a * wc - b * ws);
            im = im + (a * ws + b * wc);
            k += r;
            if (k >= n) k -= n;
        }
        s1[2 * idx] = re;
        s1[2 * idx + 1] = im;
    }
    __syncthreads();
    // rows c2r: x[r][c] = T0 + 2 sum_f Re(T_f e^{+i..}) (+ Nyquist)
    const int hmax = (n - 1) / 2;
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int r = idx / n, c = idx - r * n;
        const R* t = s1 + 2 * (int64_t)r * half;
        R acc = t[0];
        int k = 0;
        for (int f = 1; f <= hmax; ++f) {
            k += c;
            if (k >= n) k -= n;
            acc = acc + (R)2.0 * (t[2 * f] * (R)w[2 * k] + t[2 * f + 1] * (R)w[2 * k + 1]);
        }
        if ((n & 1) == 0) {
            const R nyq = t[2 * (n / 2)];
            acc = acc + ((c & 1) ? -nyq : nyq);
        }
        out[idx] = acc;
    }
}

// ---------------------------------------------------------------------------
// LSbox::computeSecondOrderNeighbours (src/box.cpp:1027-1068): one thread per
// grain.  New list = existing members of the previous list, in order, then
// members of their lists whose (convolution) boxes intersect ours, first
// occurrence only, excluding ourselves.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool boxes_intersect(const Box& a, const Box& b) {  // checkIntersection, src/box.cpp:881-888
    return !(a.x0 > b.x1 || a.x1 < b.x0 || a.y0 > b.y1 || a.y1 < b.y0);
}

__global__ void k_second_order(NetConst C, NetState* S) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS) return;
    const int K = C.kmax;
    const int* sec = C.sec_ids + (int64_t)g * K;
    const int ns = C.sec_n[g];
    int* cmp = C.cmp_ids + (int64_t)g * K;
    int nc = 0;
    bool overflow = false;
    for (int a = 0; a < ns; ++a) {
        const int id = sec[a];
        if (C.state[id] == G_EXISTS) {
            if (nc < K) cmp[nc++] = id; else overflow = true;
        }
    }
    const Box mine = S->box_cur[g];
    for (int a = 0; a < ns; ++a) {
        const int id = sec[a];
        const int* s2 = C.sec_ids + (int64_t)id * K;
        const int n2 = C.sec_n[id];
        for (int q = 0; q < n2; ++q) {
            const int c = s2[q];
            if (C.state[c] != G_EXISTS) continue;
            if (!boxes_intersect(mine, S->box_cur[c])) continue;
            if (c == g || c == 0) continue;
            bool in = false;
            for (int e = 0; e < nc; ++e)
                if (cmp[e] == c) {
                    in = true;
                    break;
                }
            if (!in) {
                if (nc < K) cmp[nc++] = c; else overflow = true;
            }
        }
    }
    C.cmp_n[g] = nc;
    if (overflow) set_status(S, S_LIST_OVERFLOW);
}

// ---------------------------------------------------------------------------
// LSbox::executeComparison + boundaryCondition + executeSetComparison
// (src/box.cpp:890-943, 945-1025, 838-879), one CTA per grain.  Every pixel
// of the grain's box takes the maximum of its comparison-list neighbours'
// convolved fields (strict '>', first list member wins ties) and the domain
// wall distance, records the winner in IDLocal, then blends with its own
// field inside the 0.7 delta tube; the new bounding box of phi >= 0 is
// reduced over the CTA.  IDLocal is first resized from the previous box with
// the reference's keep-the-prefix semantics.
// ---------------------------------------------------------------------------
constexpr int kListMaxSmem = 128;

template <typename R>
__global__ void __launch_bounds__(256) k_compare(NetConst C, NetState* S) {
    const int g = grain_at(S, blockIdx.x);
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    __shared__ Box s_box[kListMaxSmem];
    __shared__ int64_t s_org[kListMaxSmem];  // arena index of the member's pixel (0, 0)
    __shared__ int s_id[kListMaxSmem];
    __shared__ int s_red[4][8];
    const int K = C.kmax;
    const int nl = C.cmp_n[g] < kListMaxSmem ? C.cmp_n[g] : kListMaxSmem;
    for (int k = threadIdx.x; k < C.cmp_n[g]; k += blockDim.x) {
        const int id = C.cmp_ids[(int64_t)g * K + k];
        C.sec_ids[(int64_t)g * K + k] = id;  // m_secondOrderNeighbours = m_comparisonList
        if (k < kListMaxSmem) {
            const Box bk = S->box_cur[id];
            s_id[k] = id;
            s_box[k] = bk;
            s_org[k] = S->off_cur[id] - ((int64_t)bk.y0 * (bk.x1 - bk.x0) + bk.x0);
        }
    }
    if (threadIdx.x == 0) C.sec_n[g] = C.cmp_n[g];
    __syncthreads();

    const Box bc = S->box_cur[g];
    const int w = box_w(bc);
    const int64_t area = box_area(bc);
    const int b = C.b, m = C.m;
    // BoundaryIntersection (src/box.cpp:945-962): tube = grid_blowup
    const int lo = b + b, hi = m - b - b;
    const bool bnd = !(bc.x0 > lo && bc.x1 < hi && bc.y0 > lo && bc.y1 < hi);
    if (threadIdx.x == 0) C.inter_bnd[g] = bnd ? 1 : 0;

    const R* conv = phiB_of<R>(S);
    const R* self = conv + S->off_cur[g];
    R* cmpo = phiA_of<R>(S) + S->off_cur[g];
    const int64_t prev_area = box_area(S->box_prev[g]);
    const int64_t keep = prev_area < area ? prev_area : area;
    const uint32_t* idp = S->idPrev + S->off_prev[g];
    uint32_t* idc = S->idCur + S->off_cur[g];
    const R tube = (R)(0.7 * C.delta);

    int xmin = bc.x1, xmax = bc.x0, ymin = bc.y1, ymax = bc.y0;
    // Outside the 0.7 delta tube the compared value is the grain's own value
    // whatever its neighbours hold; there the neighbours' maximum only sets
    // IDLocal.  In the batched form without driving-force terms every reader
    // of IDLocal (junction corners of the contour walk, the neighbour probes,
    // the corrector's default weights and sector samples) looks within a few
    // cells of the zero crossing, well inside the tube, so pixels outside it
    // skip the neighbours (their IDLocal keeps its initial value).  The plain
    // form computes IDLocal everywhere, as the reference does.
    const bool skip_outside = sizeof(R) == sizeof(float) && !C.stored && !C.magnetic;
    // one warp per 8 x 4 tile: the warp first picks the list members whose
    // boxes meet the tile, then every lane takes the maximum over those (in
    // list order, strict '>') with four members' loads in flight
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int hgt = box_h(bc);
    const int ntx = (w + 7) >> 3, ntiles = ntx * ((hgt + 3) >> 2);
    int tcol = warp % ntx, trow = warp / ntx;  // tile t = trow * ntx + tcol, advanced without division
    const int dcol = nwarps % ntx, drow = nwarps / ntx;
    for (int t = warp; t < ntiles; t += nwarps) {
        const int tx0 = bc.x0 + tcol * 8, ty0 = bc.y0 + trow * 4;
        tcol += dcol;
        trow += drow;
        if (tcol >= ntx) {
            tcol -= ntx;
            ++trow;
        }
        const int tx1 = min(tx0 + 8, bc.x1), ty1 = min(ty0 + 4, bc.y1);
        const int j = tx0 + (lane & 7), i = ty0 + (lane >> 3);
        const bool inside = j < tx1 && i < ty1;
        const int64_t p = (int64_t)(i - bc.y0) * w + (j - bc.x0);
        uint32_t id = inside && p < keep ? idp[p] : 0u;
        const R in = inside ? self[p] : (R)0;
        R out = (R)-1.0;
        const bool want = inside && !(skip_outside && !(fabs(in) < tube));  // needs the neighbours' maximum
        const int nlt = __any_sync(FULL, want) ? nl : 0;
        for (int k0 = 0; k0 < nlt; k0 += 32) {
            bool hit = false;
            if (k0 + lane < nl) {
                const Box bk = s_box[k0 + lane];
                hit = bk.x0 < tx1 && bk.x1 > tx0 && bk.y0 < ty1 && bk.y1 > ty0;
            }
            unsigned mask = __ballot_sync(FULL, hit);
            while (mask) {
                int ks[4];
                R ds[4];
                bool ok[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    ks[u] = -1;
                    if (mask) {
                        ks[u] = k0 + __ffs(mask) - 1;
                        mask &= mask - 1;
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    ok[u] = false;
                    ds[u] = (R)0;
                    if (ks[u] >= 0 && want) {
                        const Box bk = s_box[ks[u]];
                        if (i >= bk.y0 && i < bk.y1 && j >= bk.x0 && j < bk.x1) {
                            ok[u] = true;
                            ds[u] = conv[s_org[ks[u]] + (int64_t)i * (bk.x1 - bk.x0) + j];
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (ok[u] && ds[u] > out) {
                        out = ds[u];
                        id = (uint32_t)s_id[ks[u]];
                    }
            }
        }
        if (!inside) continue;
        if (bnd) {
            const int dxmin = -(j - b), dymin = -(i - b);
            const int dxmax = (j - (m - b)), dymax = (i - (m - b));
            const int dx = (abs(dxmin) < abs(dxmax)) ? dxmin : dxmax;
            const int dy = (abs(dymin) < abs(dymax)) ? dymin : dymax;
            double dist = 0;
            if (dx > 0 && dy > 0)
                dist = sqrt((double)dx * dx + dy * dy);
            else if (dx < 0 && dy > 0)
                dist = dy;
            else if (dx > 0 && dy < 0)
                dist = dx;
            else if (dx < 0 && dy < 0)
                dist = dx > dy ? dx : dy;
            else if (dx == 0)
                dist = dy > 0 ? dy : 0;
            else  // dy == 0
                dist = dx > 0 ? dx : 0;
            const R wall = (R)(dist * C.h);
            if (wall > out) {
                out = wall;
                id = 0u;
            }
        }
        const R v = (fabs(in) < tube) ? (R)0.5 * (in - out) : in;  // tube = (R)(0.7 delta): same test as in double
        cmpo[p] = v;
        idc[p] = id;
        if (v >= 0) {
            xmin = j < xmin ? j : xmin;
            xmax = j > xmax ? j : xmax;
            ymin = i < ymin ? i : ymin;
            ymax = i > ymax ? i : ymax;
        }
    }
    // CTA reduction of the bounding box
    for (int o = 16; o > 0; o >>= 1) {
        xmin = min(xmin, __shfl_xor_sync(0xffffffffu, xmin, o));
        xmax = max(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
        ymin = min(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
        ymax = max(ymax, __shfl_xor_sync(0xffffffffu, ymax, o));
    }
    if (lane == 0) {
        s_red[0][warp] = xmin;
        s_red[1][warp] = xmax;
        s_red[2][warp] = ymin;
        s_red[3][warp] = ymax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int q = 1; q < nw; ++q) {
            xmin = min(xmin, s_red[0][q]);
            xmax = max(xmax, s_red[1][q]);
            ymin = min(ymin, s_red[2][q]);
            ymax = max(ymax, s_red[3][q]);
        }
        xmin -= b;
        xmax += b;
        ymin -= b;
        ymax += b;
        if (xmin >= xmax || ymin >= ymax) {
            xmin = bc.x0;
            xmax = bc.x1;
            ymin = bc.y0;
            ymax = bc.y1;
        }
        int* nb = C.newbb + 4 * (int64_t)g;
        nb[0] = xmin;
        nb[1] = xmax;
        nb[2] = ymin;
        nb[3] = ymax;
        if (C.cmp_n[g] > kListMaxSmem) set_status(S, S_LIST_OVERFLOW);
    }
}

// ---------------------------------------------------------------------------
// grainhdl::level_set -> LSbox::extractContour (src/grainhdl.cpp:830-848,
// src/box.cpp:1089-1153): one thread per grain.  Removes grains marked as
// vanished, extracts contour and junctions from the compared field, retries
// after clearing on irregular motion, and computes the next (square) box.
// ---------------------------------------------------------------------------
template <typename R>
__device__ bool clear_contour_area(R* phi, const Box& b, const CPoint* P, int n, double h) {
    // LSbox::clearContourGrainArea (src/box.cpp:1888-1906)
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

template <typename R>
__global__ void k_levelset(NetConst C, NetState* S) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (g > C.N || halted(S)) return;
    const int st = C.state[g];
    const Box bc = S->box_cur[g];
    if (st != G_EXISTS) {
        if (st == G_VANISHED) {  // delete grains[id] (src/grainhdl.cpp:840-842)
            C.state[g] = G_GONE;
            C.gone_loop[g] = S->loop;
        }
        S->box_new[g] = bc;
        S->cn_cur[g] = 0;
        S->jn_cur[g] = 0;
        return;
    }
    C.regular[g] = 1;
    const int old_len = S->cn_prev[g];
    R* phi = phiA_of<R>(S) + S->off_cur[g];
    Field<R> f{phi, bc};
    const uint32_t* idl = S->idCur + S->off_cur[g];
    ContourOut o{S->contCur + S->coff_cur[g], S->ccap_cur[g], 0, S->jCur + (int64_t)g * C.jmax, C.jmax, 0, 0};
    int irregular = 0;
    bool ok = ms_contour(f, idl, (uint32_t)g, o);
    if (ok) {
        project_junctions(o.pts, o.n, o.js, o.jn);
        double newVolume = contour_volume(o.pts, o.n, C.h);
        if (!motion_regular(old_len, o.n, C.volume[g], newVolume, C.dt, &irregular)) {
            int tries = 0;
            do {
                if (!clear_contour_area(phi, bc, o.pts, o.n, C.h)) o.status |= S_INDEX;
                ok = ms_contour(f, idl, (uint32_t)g, o);
                if (!ok) break;
                project_junctions(o.pts, o.n, o.js, o.jn);
                newVolume = contour_volume(o.pts, o.n, C.h);
                if (++tries > 64) {
                    o.status |= S_RETRY_LIMIT;
                    break;
                }
            } while (!motion_regular(old_len, o.n, C.volume[g], newVolume, C.dt, &irregular));
        }
    }
    if (o.status) set_status(S, o.status);
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
    C.perimeter[g] = contour_perimeter(o.pts, o.n, C.h);
    S->cn_cur[g] = o.n;
    S->jn_cur[g] = o.jn;
}

// ---------------------------------------------------------------------------
// Arena allocation for the next step: prefix sums of the new boxes' areas
// (distance fields), spectral scratch and contour capacities; one CTA.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_alloc(NetConst C, NetState* S, int spec_per_complex) {
    // Exclusive prefix sums over slots 0..N of the new box areas, spectral
    // scratch sizes and contour capacities of existing grains.  Each warp owns
    // a contiguous run of slots and reads it 32 consecutive slots at a time
    // (coalesced); pass 1 totals each run, warp 0 scans the 32 totals, pass 2
    // scans every 32-slot piece with shuffles and writes the offsets.
    __shared__ int64_t s_tot[32][3];
    __shared__ int64_t s_base[32][3];
    const int N = C.N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int slots = N + 1;
    const int run = ((slots + nw - 1) / nw + 31) & ~31;
    const int r0 = warp * run, r1 = min(slots, r0 + run);
    // sizes of slot g from its state and new box (loaded first: kU slots of
    // 32 per warp have their loads in flight together)
    auto sizes = [&](bool live, const Box& bx, int64_t* a, int64_t* sp, int64_t* c, int* cc, bool* range) {
        *a = 0;
        *sp = 0;
        *c = 0;
        *cc = 0;
        if (live) {
            const int n = box_w(bx);
            *a = box_area(bx);
            *sp = (int64_t)spec_per_complex * 2 * (int64_t)n * (n / 2 + 1);
            *cc = contour_capacity(n);
            *c = *cc;
            if (n > C.tmax) *range = true;
        }
    };
    constexpr int kU = 4;
    auto load = [&](int g, bool* live, Box* bx) {
        const bool in = g >= 1 && g <= N && g < r1;
        *live = in && C.state[g] == G_EXISTS;
        *bx = in ? S->box_new[g] : Box{0, 0, 0, 0};
    };
    bool range = false;
    int64_t ta = 0, ts = 0, tc = 0;
    for (int g0 = r0; g0 < r1; g0 += 32 * kU) {
        bool live[kU];
        Box bx[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) load(g0 + 32 * u + lane, &live[u], &bx[u]);
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            int64_t a, sp, c;
            int cc;
            sizes(live[u], bx[u], &a, &sp, &c, &cc, &range);
            ta += a;
            ts += sp;
            tc += c;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        ta += __shfl_xor_sync(0xffffffffu, ta, o);
        ts += __shfl_xor_sync(0xffffffffu, ts, o);
        tc += __shfl_xor_sync(0xffffffffu, tc, o);
    }
    if (lane == 0) {
        s_tot[warp][0] = ta;
        s_tot[warp][1] = ts;
        s_tot[warp][2] = tc;
    }
    __syncthreads();
    if (warp == 0) {
        int64_t v[3] = {0, 0, 0};
        if (lane < nw)
            for (int q = 0; q < 3; ++q) v[q] = s_tot[lane][q];
        int64_t inc[3] = {v[0], v[1], v[2]};
        for (int o = 1; o < 32; o <<= 1)
            for (int q = 0; q < 3; ++q) {
                const int64_t u = __shfl_up_sync(0xffffffffu, inc[q], o);
                if (lane >= o) inc[q] += u;
            }
        if (lane < nw)
            for (int q = 0; q < 3; ++q) s_base[lane][q] = inc[q] - v[q];
        if (lane == 31) {
            if (inc[0] > S->phi_cap || inc[1] > S->spec_cap || inc[2] > S->cont_cap) set_status(S, S_ARENA_FULL);
            S->phi_used = inc[0];
            S->spec_used = inc[1];
            S->cont_used = inc[2];
        }
    }
    __syncthreads();
    int64_t ba = s_base[warp][0], bs = s_base[warp][1], bc = s_base[warp][2];
    for (int g00 = r0; g00 < r1; g00 += 32 * kU) {
        bool live[kU];
        Box bx[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) load(g00 + 32 * u + lane, &live[u], &bx[u]);
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int g0 = g00 + 32 * u;
            if (g0 >= r1) break;  // uniform over the warp
            const int g = g0 + lane;
            int64_t a, sp, c;
            int cc;
            sizes(live[u], bx[u], &a, &sp, &c, &cc, &range);
            int64_t ia = a, is = sp, ic = c;
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t ua = __shfl_up_sync(0xffffffffu, ia, o), us = __shfl_up_sync(0xffffffffu, is, o),
                              uc = __shfl_up_sync(0xffffffffu, ic, o);
                if (lane >= o) {
                    ia += ua;
                    is += us;
                    ic += uc;
                }
            }
            if (g < r1) {
                S->off_new[g] = ba + ia - a;
                S->soff_new[g] = bs + is - sp;
                S->coff_new[g] = bc + ic - c;
                S->ccap_new[g] = cc;
            }
            ba += __shfl_sync(0xffffffffu, ia, 31);
            bs += __shfl_sync(0xffffffffu, is, 31);
            bc += __shfl_sync(0xffffffffu, ic, 31);
        }
    }
    if (range) set_status(S, S_TABLE_RANGE);
}

// ---------------------------------------------------------------------------
// LSbox::computeVolumeAndEnergy + ExplicitGrainBoundary::buildDirectNeighbours
// (src/box.cpp:1201-1228, src/grainBoundary.cpp:85-199): one thread per grain.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_neighbours(NetConst C, NetState* S) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int loop = S->loop;
    if (g > C.N || C.state[g] != G_EXISTS || C.regular[g] == 0 || halted(S)) return;
    CPoint* P = S->contCur + S->coff_cur[g];
    const int n = S->cn_cur[g];
    const double h = C.h;
    const double newVolume = fabs(contour_volume(P, n, h));
    const Box bc = S->box_cur[g];
    const R* phi = phiA_of<R>(S) + S->off_cur[g];
    const uint32_t* idl = S->idCur + S->off_cur[g];
    Neighbour* nb = C.nb + (int64_t)g * C.nbmax;
    int nn = 0;
    bool invalid = false, overflow = false;
    const double* qg = C.quat + 4 * (int64_t)g;
    for (int i = 0; i < n - 1; i++) {
        const double px = P[i].x, py = P[i].y;
        int pxGrid = (int)px, pyGrid = (int)py;
        uint32_t k;
        if (!buf_index(bc, pyGrid, pxGrid, &k)) { invalid = true; break; }
        if ((double)phi[k] > 0) {
            pxGrid = (int)(px + 1);
            if (!buf_index(bc, pyGrid, pxGrid, &k)) { invalid = true; break; }
            if ((double)phi[k] > 0) {
                pyGrid = (int)(py + 1);
                if (!buf_index(bc, pyGrid, pxGrid, &k)) { invalid = true; break; }
                if ((double)phi[k] > 0) pxGrid = (int)px;
            }
        }
        // LSbox::getNeighbourAt (src/box.cpp:2190-2195)
        if (pyGrid < 0 || pyGrid >= bc.y1 || pxGrid < 0 || pxGrid >= bc.x1) { invalid = true; break; }
        if (!buf_index(bc, pyGrid, pxGrid, &k)) { invalid = true; break; }
        const uint32_t cid = idl[k];
        if (cid != 0 && (cid > (uint32_t)C.N || C.state[cid] == G_GONE)) { invalid = true; break; }
        const double theta = grain_misorientation(qg, C.quat + 4 * (int64_t)cid);
        P[i].mob = mobility_model(theta, C);
        P[i].energy = read_shockley(theta, C);
        const double dx = P[i].x - P[i + 1].x, dy = P[i].y - P[i + 1].y;
        const double line_length = sqrt(dx * dx + dy * dy) * h;
        int e = 0;
        for (; e < nn; ++e)
            if (nb[e].id == (int)cid) break;
        if (e == nn) {
            if (nn >= C.nbmax) {
                overflow = true;
                continue;
            }
            nb[nn].id = (int)cid;
            nb[nn].length = 0;
            nb[nn].energy = P[i].energy;
            nb[nn].misori = theta;
            nb[nn].mobility = P[i].mob;
            nn++;
        }
        nb[e].length += line_length;
    }
    C.nb_n[g] = nn;
    if (overflow) set_status(S, S_NEIGHBOUR_OVERFLOW);
    if (invalid) {
        C.regular[g] = 0;  // markAsInvalidMotion (src/box.cpp:1939-1945)
    } else if (n > 0) {
        P[n - 1].energy = P[0].energy;
        P[n - 1].mob = P[0].mob;
    }
    C.energy[g] = contour_energy(P, n, h);
    double dA = newVolume - C.volume[g];
    dA = dA / C.dt;
    dA = dA * (3 / kPi);
    const unsigned int lp = (unsigned int)loop;
    if ((unsigned long)(lp - 1u) % (unsigned long)C.analysis_timestep == 0 || lp == 0) C.meanda[g] = 0;
    C.meanda[g] += dA;
    C.volume[g] = newVolume;
}

// ---------------------------------------------------------------------------
// LSbox::executeRedistancing (src/box.cpp:1259-1399): one CTA per grain;
// compared field (arena A, box_cur) -> phi_{t+1} (arena B, box_new).
// y sweeps run one thread per column, x sweeps one thread per row.
// ---------------------------------------------------------------------------
template <typename R>
__device__ void redistance_grain(const R* __restrict__ in, const Box bi, R* __restrict__ out, const Box bo, R h,
                                 R delta) {
    const int wi = box_w(bi), wo = box_w(bo);
    const int64_t ao = box_area(bo);
    for (int64_t p = threadIdx.x; p < ao; p += blockDim.x) out[p] = (R)-1.0;
    __syncthreads();
    const int ixmin = (bi.x0 < bo.x0) ? bo.x0 : bi.x0;
    const int iymin = (bi.y0 < bo.y0) ? bo.y0 : bi.y0;
    const int ixmax = (bi.x1 < bo.x1) ? bi.x1 : bo.x1;
    const int iymax = (bi.y1 < bo.y1) ? bi.y1 : bo.y1;
#define GG_IN(i, j) in[(int64_t)((i) - bi.y0) * wi + ((j) - bi.x0)]
#define GG_OUT(i, j) out[(int64_t)((i) - bo.y0) * wo + ((j) - bo.x0)]
    for (int j = ixmin + (int)threadIdx.x; j < bo.x1; j += blockDim.x) {
        for (int i = iymin; i < bo.y1 - 1; i++) {  // y forward
            R cand;
            if (j < ixmax && i < iymax - 1) {
                const R a = GG_IN(i, j), c = GG_IN(i + 1, j);
                if (a * c <= (R)0.0) {
                    const R slope = (c - a) / h;
                    const R dz = -a / slope;
                    if (fabs(GG_OUT(i, j)) > fabs(dz)) GG_OUT(i, j) = -dz * (R)sgn(slope);
                }
                cand = GG_OUT(i, j) + ((R)sgn(c) * h);
            } else {
                cand = GG_OUT(i, j) + ((R)sgn(GG_OUT(i + 1, j)) * h);
            }
            if (fabs(cand) < fabs(GG_OUT(i + 1, j))) GG_OUT(i + 1, j) = cand;
        }
        for (int i = iymax - 1; i > bo.y0; i--) {  // y backward
            R cand;
            if (j < ixmax && i > iymin)
                cand = GG_OUT(i, j) + ((R)sgn(GG_IN(i - 1, j)) * h);
            else
                cand = GG_OUT(i, j) + ((R)sgn(GG_OUT(i - 1, j)) * h);
            if (fabs(cand) < fabs(GG_OUT(i - 1, j))) GG_OUT(i - 1, j) = cand;
        }
    }
    __syncthreads();
    for (int i = iymin + (int)threadIdx.x; i < bo.y1; i += blockDim.x) {
        for (int j = ixmin; j < bo.x1 - 1; j++) {  // x forward
            R cand;
            if (j < ixmax - 1 && i < iymax) {
                const R a = GG_IN(i, j), c = GG_IN(i, j + 1);
                if (a * c <= (R)0.0) {
                    const R slope = (c - a) / h;
                    const R dz = -a / slope;
                    if (fabs(GG_OUT(i, j)) > fabs(dz)) GG_OUT(i, j) = -dz * (R)sgn(slope);
                }
                cand = GG_OUT(i, j) + ((R)sgn(c) * h);
            } else {
                cand = GG_OUT(i, j) + ((R)sgn(GG_OUT(i, j + 1)) * h);
            }
            if (fabs(cand) < fabs(GG_OUT(i, j + 1))) GG_OUT(i, j + 1) = cand;
        }
        for (int j = ixmax - 1; j > bo.x0; j--) {  // x backward
            R cand;
            if (j > ixmin && i < iymax)
                cand = GG_OUT(i, j) + ((R)sgn(GG_IN(i, j - 1)) * h);
            else
                cand = GG_OUT(i, j) + (R)sgn(GG_OUT(i, j - 1)) * h;
            if (fabs(cand) < fabs(GG_OUT(i, j - 1))) GG_OUT(i, j - 1) = cand;
        }
    }
#undef GG_IN
#undef GG_OUT
    __syncthreads();
    for (int64_t p = threadIdx.x; p < ao; p += blockDim.x) {  // clampValues(-delta, delta)
        const R v = out[p];
        if (v < -delta)
            out[p] = -delta;
        else if (v > delta)
            out[p] = delta;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_redistance(NetConst C, NetState* S) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    const R* in = phiA_of<R>(S) + S->off_cur[g];
    R* out = phiB_of<R>(S) + S->off_new[g];
    redistance_grain<R>(in, S->box_cur[g], out, S->box_new[g], (R)C.h, (R)C.delta);
}

// LSbox::resizeGrid (src/box.cpp:1408-1485) of one grain (not removed) per
// block: its distance function on the coarser grid, by bilinear
// interpolation of the old field (box_cur / off_cur of phiA) at the new grid's
// points, into box_new / off_new of phiB (boxes laid out by the host).  A
// point whose interpolation cell reaches the old box's last two rows or
// columns, or lies before its first, takes -delta_old.  The arithmetic is the
// reference's, term for term.
template <typename R>
__global__ void __launch_bounds__(256) k_resample(NetConst C, NetState* S, double h_old, double hn, double delta_old) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] == G_GONE) return;
    const Box ob = S->box_cur[g];
    const Box nb = S->box_new[g];
    const R* src = phiA_of<R>(S) + S->off_cur[g];
    R* dst = phiB_of<R>(S) + S->off_new[g];
    const int ow = ob.x1 - ob.x0, nw = nb.x1 - nb.x0;
    if (nw <= 0 || nb.y1 <= nb.y0) return;
    const int64_t cnt = (int64_t)nw * (nb.y1 - nb.y0);
    for (int64_t p = threadIdx.x; p < cnt; p += blockDim.x) {
        const int i = nb.y0 + (int)(p / nw), j = nb.x0 + (int)(p % nw);
        const double pointx = j * (hn / h_old);
        const double pointy = i * (hn / h_old);
        const double xl = (int)pointx, xr = (int)(pointx + 1), yo = (int)(pointy + 1), yu = (int)pointy;
        if (xr > ob.x1 - 2 || yo > ob.y1 - 2 || yu < ob.y0 || xl < ob.x0) {
            dst[p] = (R)(-delta_old);
            continue;
        }
        auto at = [&](double row, double col) {
            return (double)src[(int64_t)((int)row - ob.y0) * ow + ((int)col - ob.x0)];
        };
        const double ro = 1 / (xr - xl) * ((xr - pointx) * at(yo, xl) + (pointx - xl) * at(yo, xr));
        const double ru = 1 / (xr - xl) * ((xr - pointx) * at(yu, xl) + (pointx - xl) * at(yu, xr));
        const double v = 1 / (yo - yu) * ((yo - pointy) * ru + (pointy - yu) * ro);
        // the reference stops on a NaN here (src/box.cpp:1470-1474); the
        // library records it (GG_S_NAN) and the call reports GG_E_NUMERIC
        if (v != v) set_status(S, S_NAN);
        dst[p] = (R)v;
    }
}

// ---------------------------------------------------------------------------
// End of step: grainhdl::get_biggestGrainVol (src/grainhdl.cpp:1744-1754) and
// the buffer switches; rotates per-step roles in NetState.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_finalize(NetConst C, NetState* S, int rotate) {
    __shared__ int s_cnt[32];
    __shared__ double s_max[32];
    int cnt = 0;
    double mx = 0.0;
    constexpr int kU = 4;  // four grains' state and volume loads in flight
    for (int g0 = threadIdx.x + 1; g0 <= C.N; g0 += kU * blockDim.x) {
        int st[kU];
        double vol[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int g = g0 + u * (int)blockDim.x;
            st[u] = g <= C.N ? C.state[g] : G_GONE;
            vol[u] = g <= C.N ? C.volume[g] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
            if (st[u] != G_GONE) {
                cnt++;
                mx = fmax(mx, vol[u]);
            }
    }
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        s_cnt[threadIdx.x >> 5] = cnt;
        s_max[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int q = 1; q < (int)((blockDim.x + 31) >> 5); ++q) {
        cnt += s_cnt[q];
        mx = fmax(mx, s_max[q]);
    }
    if (rotate) S->updates += (unsigned long long)S->live;  // grains alive at this step's start
    S->live = cnt;
    S->max_volume = mx;
    if (!rotate) return;
    Box* tb = S->box_prev;
    S->box_prev = S->box_cur;
    S->box_cur = S->box_new;
    S->box_new = tb;
    int64_t* to = S->off_prev;
    S->off_prev = S->off_cur;
    S->off_cur = S->off_new;
    S->off_new = to;
    int64_t* ts = S->soff_cur;
    S->soff_cur = S->soff_new;
    S->soff_new = ts;
    void* tp = S->phiA;
    S->phiA = S->phiB;
    S->phiB = tp;
    tp = S->dphiA;
    S->dphiA = S->dphiB;
    S->dphiB = tp;
    uint32_t* ti = S->idPrev;
    S->idPrev = S->idCur;
    S->idCur = ti;
    CPoint* tc = S->contPrev;
    S->contPrev = S->contCur;
    S->contCur = tc;
    double* tdc = S->dcontPrev;
    S->dcontPrev = S->dcontCur;
    S->dcontCur = tdc;
    int64_t* tco = S->coff_prev;
    S->coff_prev = S->coff_cur;
    S->coff_cur = S->coff_new;
    S->coff_new = tco;
    int32_t* tcc = S->ccap_prev;
    S->ccap_prev = S->ccap_cur;
    S->ccap_cur = S->ccap_new;
    S->ccap_new = tcc;
    int32_t* tn = S->cn_prev;
    S->cn_prev = S->cn_cur;
    S->cn_cur = tn;
    Junction* tj = S->jPrev;
    S->jPrev = S->jCur;
    S->jCur = tj;
    int32_t* tjn = S->jn_prev;
    S->jn_prev = S->jn_cur;
    S->jn_cur = tjn;
    S->loop += 1;
}

// The batched form's work queue (NetState::order): existing grains by
// descending box edge, then the rest, by a counting sort in one CTA.  A
// per-grain launch then starts its longest blocks first and the short ones
// fill the last wave.  The order within one edge length is whatever the
// shared-memory atomics give; no result depends on it.  The same pass flags
// and lists the grains whose contour is longer than the main corrector
// stages (NetState::big_flag, big_list).
constexpr int kOrderBins = 256;
static_assert(kOrderBins % 32 == 0, "the bin scan gives each lane kOrderBins / 32 bins");

__global__ void __launch_bounds__(1024) k_order(NetConst C, NetState* S) {
    int32_t* order = S->order;
    if (!order) return;
    __shared__ int s_bin[kOrderBins];
    __shared__ int s_nbig;
    for (int q = threadIdx.x; q < kOrderBins; q += blockDim.x) s_bin[q] = 0;
    if (threadIdx.x == 0) s_nbig = 0;
    __syncthreads();
    auto bin_from = [](int state, int edge) {
        return state != G_EXISTS ? kOrderBins - 1 : kOrderBins - 2 - min(max(edge, 0), kOrderBins - 2);
    };
    // counts per bin, and the large-contour corrector's grains (list order is
    // free); four grains per thread with their loads issued first
    int32_t* big_flag = S->big_flag;
    constexpr int kU = 4;
    for (int g0 = threadIdx.x + 1; g0 <= C.N; g0 += kU * blockDim.x) {
        int st[kU], bw[kU], cn[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int g = g0 + u * (int)blockDim.x;
            st[u] = g <= C.N ? C.state[g] : G_GONE;
            bw[u] = g <= C.N ? box_w(S->box_cur[g]) : 0;
            cn[u] = g <= C.N && big_flag ? S->cn_prev[g] : 0;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int g = g0 + u * (int)blockDim.x;
            if (g > C.N) break;
            atomicAdd(&s_bin[bin_from(st[u], bw[u])], 1);
            if (big_flag) {
                const bool big = st[u] == G_EXISTS && cn[u] > kCorrStagedPts;
                big_flag[g] = big ? 1 : 0;
                if (big) S->big_list[atomicAdd(&s_nbig, 1)] = g;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan of the bins by one warp, 8 per lane
        constexpr int kPer = kOrderBins / 32;
        int c[kPer], t = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            c[k] = s_bin[threadIdx.x * kPer + k];
            t += c[k];
        }
        int incl = t;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if ((int)threadIdx.x >= o) incl += v;
        }
        int run = incl - t;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            s_bin[threadIdx.x * kPer + k] = run;
            run += c[k];
        }
    }
    __syncthreads();
    for (int g0 = threadIdx.x + 1; g0 <= C.N; g0 += kU * blockDim.x) {
        int bin[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int g = g0 + u * (int)blockDim.x;
            bin[u] = g <= C.N ? bin_from(C.state[g], box_w(S->box_cur[g])) : 0;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int g = g0 + u * (int)blockDim.x;
            if (g <= C.N) order[atomicAdd(&s_bin[bin[u]], 1)] = g;
        }
    }
    if (threadIdx.x == 0 && big_flag) S->n_big = s_nbig;
}

// Traffic model: box areas and comparison-list overlaps of existing grains.
__global__ void k_traffic(NetConst C, NetState* S) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS) return;
    const Box a = S->box_cur[g];
    unsigned long long ov = 0;
    const int n = C.cmp_n[g];
    for (int k = 0; k < n; ++k) {
        const Box b = S->box_cur[C.cmp_ids[(int64_t)g * C.kmax + k]];
        const int x0 = max(a.x0, b.x0), x1 = min(a.x1, b.x1), y0 = max(a.y0, b.y0), y1 = min(a.y1, b.y1);
        if (x1 > x0 && y1 > y0) ov += (unsigned long long)(x1 - x0) * (unsigned long long)(y1 - y0);
    }
    atomicAdd(&S->t_area, (unsigned long long)box_area(a));
    atomicAdd(&S->t_overlap, ov);
    atomicAdd(&S->t_exists, 1ull);
}

// ---------------------------------------------------------------------------
// Initialisation for voxelized input (src/box.cpp:322-341): +-h from the ID
// field, then the redistancing kernel, then the contour of the result.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_init_phi(NetConst C, NetState* S, const int32_t* __restrict__ ids) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    const Box bx = S->box_cur[g];
    const int w = box_w(bx);
    const int64_t area = box_area(bx);
    R* phi = phiA_of<R>(S) + S->off_cur[g];
    const int lo = C.b, hi = C.m - C.b - 1;
    const R h = (R)C.h;
    for (int64_t p = threadIdx.x; p < area; p += blockDim.x) {
        const int i = bx.y0 + (int)(p / w), j = bx.x0 + (int)(p % w);
        R v;
        if (i < lo || i > hi || j < lo || j > hi)
            v = -h;
        else
            v = (ids[(int64_t)(i - lo) * C.nn + (j - lo)] == g) ? h : -h;
        phi[p] = v;
    }
}

template <typename R>
__global__ void k_init_contour(NetConst C, NetState* S) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    const Box bx = S->box_cur[g];
    Field<R> f{phiA_of<R>(S) + S->off_cur[g], bx};
    const uint32_t* idl = S->idPrev + S->off_prev[g];
    ContourOut o{S->contPrev + S->coff_prev[g], S->ccap_prev[g], 0, S->jPrev + (int64_t)g * C.jmax, C.jmax, 0, 0};
    const bool ok = ms_contour(f, idl, (uint32_t)g, o);
    if (o.status) set_status(S, o.status);
    if (!ok) {
        C.state[g] = G_VANISHED;
        S->cn_prev[g] = 0;
        S->jn_prev[g] = 0;
        C.volume[g] = 0;
        return;
    }
    project_junctions(o.pts, o.n, o.js, o.jn);
    S->cn_prev[g] = o.n;
    S->jn_prev[g] = o.jn;
    C.volume[g] = contour_volume(o.pts, o.n, C.h);
}

// ---------------------------------------------------------------------------
// Initialisation for contour input (LSbox::calculateDistanceFunction,
// src/box.cpp:342-400): every pixel (i, j) of the grain's box, at domain
// point ((j - b) h, (i - b) h), takes the distance to the nearest edge of the
// loaded polygon (point-to-segment, the end points where the foot falls
// outside), clamped to delta, positive inside by the crossing-number test.
// Both loops run over the edges (p[k-1], p[k]) in order with the reference's
// expressions, so the FP64 result is the reference's bit for bit; a
// zero-length edge gives NaN and leaves the minimum unchanged, as std::min
// does.  One CTA per grain; the polygon is staged in shared memory when it
// fits, else read from the contour arena.  The other field buffer is zeroed:
// the reference's input buffer is never written in this mode.
// ---------------------------------------------------------------------------
constexpr int kPolySmem = 1024;

template <typename R>
__global__ void __launch_bounds__(256) k_polygon_phi(NetConst C, NetState* S) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    __shared__ double s_x[kPolySmem], s_y[kPolySmem];
    const int np = S->cn_prev[g];
    const CPoint* pts = S->contPrev + S->coff_prev[g];
    const bool staged = np <= kPolySmem;
    if (staged)
        for (int k = threadIdx.x; k < np; k += blockDim.x) {
            s_x[k] = pts[k].x;
            s_y[k] = pts[k].y;
        }
    __syncthreads();
    const Box bx = S->box_cur[g];
    const int w = box_w(bx);
    const int64_t area = box_area(bx);
    R* phi = phiA_of<R>(S) + S->off_cur[g];
    R* other = phiB_of<R>(S) + S->off_cur[g];
    const double h = C.h, delta = C.delta;
    const int b = C.b;
    for (int64_t p = threadIdx.x; p < area; p += blockDim.x) {
        const int i = bx.y0 + (int)(p / w), j = bx.x0 + (int)(p % w);
        const double tx = (j - b) * h, ty = (i - b) * h;
        bool inside = false;
        double min_dist = 1000000.0;
        double lx = staged ? s_x[0] : pts[0].x, ly = staged ? s_y[0] : pts[0].y;
        for (int k = 1; k < np; ++k) {
            const double kx = staged ? s_x[k] : pts[k].x, ky = staged ? s_y[k] : pts[k].y;
            if (((ly > ty) != (ky > ty)) && (tx < (kx - lx) * (ty - ly) / (ky - ly) + lx)) inside = !inside;
            const double ux = kx - lx, uy = ky - ly;
            double lambda = (tx - lx) * ux + (ty - ly) * uy;
            lambda /= ux * ux + uy * uy;
            double dist;
            if (lambda <= 0) {
                const double dx = tx - lx, dy = ty - ly;
                dist = sqrt(dx * dx + dy * dy);
            } else if (lambda >= 1) {
                const double dx = kx - tx, dy = ky - ty;
                dist = sqrt(dx * dx + dy * dy);
            } else {
                const double fx = lx + ux * lambda, fy = ly + uy * lambda;
                const double dx = tx - fx, dy = ty - fy;
                dist = sqrt(dx * dx + dy * dy);
            }
            if (dist < min_dist) min_dist = dist;
            lx = kx;
            ly = ky;
        }
        if (min_dist > delta) min_dist = delta;
        phi[p] = (R)(inside ? min_dist : -min_dist);
        other[p] = (R)0;
    }
}

// grainhdl::find_neighbors + LSbox::computeDirectNeighbours
// (src/grainhdl.cpp:1258-1283, src/box.cpp:2220-2237): every other grain whose
// closed box overlaps (RTree::Overlap, src/RTree.h:1092-1105), ascending ID.
// The grains are first binned by the kNeighbourBin x kNeighbourBin cells
// their boxes cover; a warp per grain then tests the grains of its own cells,
// keeping an overlapping pair only in the cell that holds the lower-left
// corner of the two boxes' overlap (so each pair once), and ranks its hits
// into ascending order.  A grain with more than kFindCandidates hits tests
// every grain instead, 32 consecutive IDs at a time.
constexpr int kFindWarps = 4;
constexpr int kFindCandidates = 256;

__device__ __forceinline__ bool boxes_overlap_closed(const Box& a, const Box& b) {
    return !(a.x0 > b.x1 || b.x0 > a.x1 || a.y0 > b.y1 || b.y0 > a.y1);
}

__device__ __forceinline__ int bin_of(int v, int nc) { return min(max(v / kNeighbourBin, 0), nc - 1); }

// Writes grain g's list of ns hits (ids[0 .. min(ns, kmax)), ascending) as
// the reference's find_neighbors leaves it: comparison list, direct
// neighbours with zero characteristics, no comparison members yet.
__device__ void write_neighbour_list(const NetConst& C, NetState* S, int g, const int* ids, int ns, int lane) {
    int* sec = C.sec_ids + (int64_t)g * C.kmax;
    Neighbour* nb = C.nb + (int64_t)g * C.nbmax;
    for (int pos = lane; pos < ns; pos += 32) {
        const int k = ids[pos];
        if (pos < C.kmax) sec[pos] = k;
        if (pos < C.nbmax) {
            nb[pos].id = k;
            nb[pos].length = 0;
            nb[pos].energy = 0;
            nb[pos].misori = 0;
            nb[pos].mobility = 0;
        }
    }
    if (lane == 0) {
        C.sec_n[g] = ns < C.kmax ? ns : C.kmax;
        C.cmp_n[g] = 0;
        C.nb_n[g] = ns < C.nbmax ? ns : C.nbmax;
        if (ns > C.kmax) set_status(S, S_LIST_OVERFLOW);
    }
}

// Every grain tested, in ID order (the fallback).
__device__ void find_neighbors_scan(const NetConst& C, NetState* S, int g, int lane) {
    const Box a = S->box_cur[g];
    int ns = 0;
    bool overflow = false;
    int* sec = C.sec_ids + (int64_t)g * C.kmax;
    Neighbour* nb = C.nb + (int64_t)g * C.nbmax;
    for (int k0 = 1; k0 <= C.N; k0 += 32) {
        const int k = k0 + lane;
        bool hit = false;
        if (k <= C.N && k != g && C.state[k] != G_GONE) hit = boxes_overlap_closed(a, S->box_cur[k]);
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const int pos = ns + __popc(mask & ((1u << lane) - 1u));
            if (pos < C.kmax) sec[pos] = k; else overflow = true;
            if (pos < C.nbmax) {
                nb[pos].id = k;
                nb[pos].length = 0;
                nb[pos].energy = 0;
                nb[pos].misori = 0;
                nb[pos].mobility = 0;
            }
        }
        ns += __popc(mask);
    }
    overflow = __any_sync(0xffffffffu, overflow);
    if (lane == 0) {
        C.sec_n[g] = ns < C.kmax ? ns : C.kmax;
        C.cmp_n[g] = 0;
        C.nb_n[g] = ns < C.nbmax ? ns : C.nbmax;
        if (overflow) set_status(S, S_LIST_OVERFLOW);
    }
}

// Bins: count, then (after the scan) fill, the grains of every cell.
__global__ void k_bin_grains(NetConst C, NetState* S, NeighbourBins B, int fill) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (g > C.N || C.state[g] == G_GONE) return;
    const Box a = S->box_cur[g];
    const int cx0 = bin_of(a.x0, B.nc), cx1 = bin_of(a.x1, B.nc), cy0 = bin_of(a.y0, B.nc), cy1 = bin_of(a.y1, B.nc);
    for (int cy = cy0; cy <= cy1; ++cy)
        for (int cx = cx0; cx <= cx1; ++cx) {
            const int c = cy * B.nc + cx;
            const int pos = atomicAdd(&B.count[c], 1);
            if (fill) B.items[B.start[c] + pos] = g;
        }
}

// Exclusive scan of the cell counts into starts (start[ncell] = total), the
// counts reset for the fill; one CTA.
__global__ void __launch_bounds__(1024) k_bin_scan(NeighbourBins B) {
    __shared__ int s_warp[32];
    __shared__ int s_run;
    const int ncell = B.nc * B.nc;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) s_run = 0;
    __syncthreads();
    for (int base = 0; base < ncell; base += blockDim.x) {
        const int c = base + (int)threadIdx.x;
        const int v = c < ncell ? B.count[c] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        int before = s_run;
        for (int w = 0; w < warp; ++w) before += s_warp[w];
        if (c < ncell) {
            B.start[c] = before + incl - v;
            B.count[c] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < nw; ++w) t += s_warp[w];
            s_run += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        B.start[ncell] = s_run;
        *B.total = s_run;
    }
}

__global__ void __launch_bounds__(32 * kFindWarps) k_find_neighbors(NetConst C, NetState* S, NeighbourBins B) {
    __shared__ int s_hit[kFindWarps][kFindCandidates];
    __shared__ int s_ord[kFindWarps][kFindCandidates];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int g = blockIdx.x * kFindWarps + wid + 1;
    if (g > C.N || C.state[g] == G_GONE) return;
    const Box a = S->box_cur[g];
    const int nc = B.nc;
    const int cx0 = bin_of(a.x0, nc), cx1 = bin_of(a.x1, nc), cy0 = bin_of(a.y0, nc), cy1 = bin_of(a.y1, nc);
    int* hit_ids = s_hit[wid];
    int n = 0;
    for (int cy = cy0; cy <= cy1; ++cy)
        for (int cx = cx0; cx <= cx1; ++cx) {
            const int c = cy * nc + cx;
            const int q1 = B.start[c + 1];
            for (int q0 = B.start[c]; q0 < q1; q0 += 32) {
                const int q = q0 + lane;
                int k = 0;
                bool hit = false;
                if (q < q1) {
                    k = B.items[q];
                    if (k != g) {
                        const Box b = S->box_cur[k];
                        hit = boxes_overlap_closed(a, b) &&
                              bin_of(max(a.y0, b.y0), nc) * nc + bin_of(max(a.x0, b.x0), nc) == c;
                    }
                }
                const unsigned mask = __ballot_sync(0xffffffffu, hit);
                if (hit) {
                    const int pos = n + __popc(mask & ((1u << lane) - 1u));
                    if (pos < kFindCandidates) hit_ids[pos] = k;
                }
                n += __popc(mask);
            }
        }
    __syncwarp();
    if (n > kFindCandidates) {  // uniform over the warp
        find_neighbors_scan(C, S, g, lane);
        return;
    }
    // ascending ID: each hit's rank among the (distinct) hits
    int* ord = s_ord[wid];
    for (int i = lane; i < n; i += 32) {
        const int v = hit_ids[i];
        int r = 0;
        for (int j = 0; j < n; ++j) r += hit_ids[j] < v;
        ord[r] = v;
    }
    __syncwarp();
    write_neighbour_list(C, S, g, ord, n, lane);
}

}  // namespace
}  // namespace gg
