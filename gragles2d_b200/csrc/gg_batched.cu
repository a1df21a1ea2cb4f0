// Batched form: FP32 distance fields and convolution (FP64 contour areas,
// energies and lengths), every stage over all grains, captured per step as
// one CUDA graph by the host.
#include "gg_corrector.cuh"
#include "gg_kernels.cuh"
#include "gg_launch.cuh"
#include "gg_warp.cuh"

namespace gg {

constexpr int kConvSmemEdgeMax = 128;  // largest tunable edge with the intermediate in shared memory
constexpr int kSepStrip = 4;       // outputs per thread along the convolution axis

// Gaussian convolution as a separable circular convolution in real space:
// out = K X K^T with K[r][r'] = k_n[(r - r') mod n], where k_n is the real
// kernel whose DFT is the reference's Gaussian multiplier
// (src/box.cpp:674-687, G(i2, j2) = g(i2) g(j2) / n^2).  One CTA per grain.
// The kernel is laid out once as kx[j] = k_n[(j - (n-1)) mod n], j < 2n-1
// (zero-padded), so output c of a row is sum_c' X[c'] kx[c - c' + n - 1]:
// each thread accumulates strips of 4 consecutive outputs of two rows (or
// columns) while a 4-entry register window slides down kx (one shared-memory
// load of the kernel per 8 FMAs).  Taps farther than R (circularly) from the
// strip are left out: the host sets R so that every dropped k_n entry is
// below 2^-26 k_n[0].

// The (at most two) index ranges of c' within circular distance R of the
// strip [c0, c0 + 4), as [s0, e0) and [s1, e1).
__device__ __forceinline__ void band_ranges(int c0, int n, int R, int* s0, int* e0, int* s1, int* e1) {
    *s1 = 0;
    *e1 = 0;
    if (2 * R + kSepStrip >= n) {
        *s0 = 0;
        *e0 = n;
        return;
    }
    const int lo = c0 - R, hi = c0 + kSepStrip + R;
    if (lo < 0) {
        *s0 = lo + n;
        *e0 = n;
        *e1 = hi;
    } else if (hi > n) {
        *s0 = lo;
        *e0 = n;
        *e1 = hi - n;
    } else {
        *s0 = lo;
        *e0 = hi;
    }
}

// The taps of band_ranges as one walk of the same length for every strip of
// a box, so that the lanes of a warp run one loop together (the row pass,
// whose strips differ within a warp): the walk starts at c' = *first and
// wraps from n - 1 to 0, *taps steps, with the kernel window starting at kx
// index *base.  In a banded box every strip starts at R + n - 1, one period
// of k_n above the first range's index when that range wraps; kx holds k_n
// periodically below index 2n - 1, so every stored output meets the same
// kernel values in the same order as over the two ranges (the window's
// extra entries past the row end feed only the unstored outputs of a last,
// partial strip).
__device__ __forceinline__ void band_walk(int c0, int n, int R, int* first, int* taps, int* base) {
    if (2 * R + kSepStrip >= n) {
        *first = 0;
        *taps = n;
        *base = c0 + n - 1;
        return;
    }
    const int lo = c0 - R;
    *first = lo < 0 ? lo + n : lo;
    *taps = 2 * R + kSepStrip;
    *base = R + n - 1;
}

// rows: two rows per thread share each kernel window load
__device__ __forceinline__ void sep_pass_rows(const float* __restrict__ X, float* __restrict__ T,
                                              const float* __restrict__ kx, int n, int R) {
    const int nb = (n + kSepStrip - 1) / kSepStrip;
    const int npair = (n + 1) >> 1;
    for (int t = threadIdx.x; t < npair * nb; t += blockDim.x) {
        const int rp = t / nb, c0 = (t - rp * nb) * kSepStrip;
        const int r = 2 * rp;
        const bool two = r + 1 < n;
        const float* xa = X + r * n;
        const float* xb = two ? xa + n : xa;
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, b0 = 0.f, b1 = 0.f, b2 = 0.f, b3 = 0.f;
        int cp, taps, base;
        band_walk(c0, n, R, &cp, &taps, &base);
        float w0 = kx[base], w1 = kx[base + 1], w2 = kx[base + 2], w3 = kx[base + 3];
#pragma unroll 4
        for (int k = 0; k < taps; ++k) {
            const float x = xa[cp], y = xb[cp];
            a0 = fmaf(x, w0, a0);
            a1 = fmaf(x, w1, a1);
            a2 = fmaf(x, w2, a2);
            a3 = fmaf(x, w3, a3);
            b0 = fmaf(y, w0, b0);
            b1 = fmaf(y, w1, b1);
            b2 = fmaf(y, w2, b2);
            b3 = fmaf(y, w3, b3);
            cp = cp + 1 == n ? 0 : cp + 1;
            --base;
            w3 = w2;
            w2 = w1;
            w1 = w0;
            w0 = kx[base];
        }
        float* ta = T + r * n + c0;
        ta[0] = a0;
        if (c0 + 1 < n) ta[1] = a1;
        if (c0 + 2 < n) ta[2] = a2;
        if (c0 + 3 < n) ta[3] = a3;
        if (two) {
            float* tb = ta + n;
            tb[0] = b0;
            if (c0 + 1 < n) tb[1] = b1;
            if (c0 + 2 < n) tb[2] = b2;
            if (c0 + 3 < n) tb[3] = b3;
        }
    }
}

// columns: columns c and c + ceil(n/2) per thread share each kernel window load
__device__ __forceinline__ void sep_pass_cols(const float* __restrict__ T, float* __restrict__ out,
                                              const float* __restrict__ kx, int n, int R) {
    const int nb = (n + kSepStrip - 1) / kSepStrip;
    const int half = (n + 1) >> 1;
    for (int t = threadIdx.x; t < half * nb; t += blockDim.x) {
        const int rb = t / half, c = t - rb * half, r0 = rb * kSepStrip;
        const bool two = c + half < n;
        const int c2 = two ? c + half : c;
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, b0 = 0.f, b1 = 0.f, b2 = 0.f, b3 = 0.f;
        int rs[2], re[2];
        band_ranges(r0, n, R, &rs[0], &re[0], &rs[1], &re[1]);
        for (int q = 0; q < 2; ++q) {
            int base = r0 + n - 1 - rs[q];
            float w0 = kx[base], w1 = kx[base + 1], w2 = kx[base + 2], w3 = kx[base + 3];
#pragma unroll 4
            for (int rp = rs[q]; rp < re[q]; ++rp) {
                const float x = T[rp * n + c], y = T[rp * n + c2];
                a0 = fmaf(w0, x, a0);
                a1 = fmaf(w1, x, a1);
                a2 = fmaf(w2, x, a2);
                a3 = fmaf(w3, x, a3);
                b0 = fmaf(w0, y, b0);
                b1 = fmaf(w1, y, b1);
                b2 = fmaf(w2, y, b2);
                b3 = fmaf(w3, y, b3);
                --base;
                w3 = w2;
                w2 = w1;
                w1 = w0;
                w0 = kx[base];
            }
        }
        out[r0 * n + c] = a0;
        if (r0 + 1 < n) out[(r0 + 1) * n + c] = a1;
        if (r0 + 2 < n) out[(r0 + 2) * n + c] = a2;
        if (r0 + 3 < n) out[(r0 + 3) * n + c] = a3;
        if (two) {
            out[r0 * n + c2] = b0;
            if (r0 + 1 < n) out[(r0 + 1) * n + c2] = b1;
            if (r0 + 2 < n) out[(r0 + 2) * n + c2] = b2;
            if (r0 + 3 < n) out[(r0 + 3) * n + c2] = b3;
        }
    }
}

// Extended kernel length: 2n-1 entries plus the window's look-ahead, and one
// guard entry below index 0 (the window reads kx[-1] after its last step).
__device__ __forceinline__ int kx_len(int n) { return 2 * n + kSepStrip + 1; }

__global__ void __launch_bounds__(128) k_conv_sep(NetConst C, NetState* S) {
    extern __shared__ float sm[];
    const int g = grain_at(S, blockIdx.x);
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    const Box bx = S->box_cur[g];
    const int n = box_w(bx);
    if (n <= 0) return;
    if (n != box_h(bx) || n > C.tmax) {
        if (threadIdx.x == 0) set_status(S, n > C.tmax ? S_TABLE_RANGE : S_INDEX);
        return;
    }
    const float* in = reinterpret_cast<const float*>(S->phiA) + S->off_cur[g];
    float* out = reinterpret_cast<float*>(S->phiB) + S->off_cur[g];
    const float* kg = C.ck + C.ck_off[n];
    const bool fits = n <= C.conv_smem_edge;
    float* kx = sm + 1;  // sm[0] is the guard entry kx[-1]
    const int kl = kx_len(n);
    float* T = fits ? sm + 1 + kl : reinterpret_cast<float*>(S->spec) + S->soff_cur[g];
    for (int j = threadIdx.x; j < kl; j += blockDim.x) {
        int m = j - (n - 1);
        m %= n;
        if (m < 0) m += n;
        kx[j] = j < 2 * n - 1 ? kg[m] : 0.f;
    }
    if (threadIdx.x == 0) sm[0] = 0.f;
    __syncthreads();
    const int R = (int)kg[n];  // band radius stored after the n kernel entries
    sep_pass_rows(in, T, kx, n, R);
    __syncthreads();
    sep_pass_cols(T, out, kx, n, R);
}

size_t conv_sep_smem(int tmax, int edge) {
    // the row-pass intermediate of a box (edge up to `edge`) with its
    // extended kernel, or the extended kernel alone of the largest box (whose
    // intermediate goes to the grain's scratch in device memory)
    const int n = tmax < edge ? tmax : edge;
    const size_t staged = (size_t)n * n + 2 * (size_t)n + kSepStrip + 2;
    const size_t kernel_only = 2 * (size_t)tmax + kSepStrip + 2;
    return sizeof(float) * (staged > kernel_only ? staged : kernel_only);
}

// Batched-form corrector: same sectors as k_corrector (built by one warp),
// with the previous contour staged in shared memory (FP32 box-local
// coordinates) and the per-pixel work in FP32, except the discrete decisions
// of the projection, which follow the reference's FP64 arithmetic.  Each
// warp takes one 8 x 4 tile of the box at a time.  The main kernel stages
// contours up to kCorrStagedPts points; the large-contour kernel, persistent
// over NetState::big_list, up to kCorrBigPts; longer ones are read from
// device memory in FP64.
constexpr int kCorrBigPts = 1024;

// Packed FP32 pairs (sm_100 f32x2 arithmetic).
__device__ __forceinline__ unsigned long long f2_pack(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}

// Nearest contour vertex of projectToGrainBondary (src/grainBoundary.cpp:
// 365-381) through a uniform grid of cells over the previous box: the
// vertices are bucketed by cell (counting sort in shared memory), and a pixel
// measures, in FP64 from the contour itself, the vertices of the 3 x 3 cells
// around its own.  Every vertex within `cell` of the pixel lies in that
// window, so when the smallest distance found is at most (cell - 1e-3)^2 (the
// margin covers the cell index of a vertex on a cell edge) it is the smallest
// over the whole contour; ties go to the lowest index, as the reference's
// strict < over ascending k.  Otherwise the pixel scans every vertex.
constexpr int kCellMax = 24;          // cells per side
template <int kPts>  // vertices bucketed (the staged contours)
struct VertexBuckets {
    int ncx, ncy, cell;
    int end[kCellMax * kCellMax + 1];  // after the fill: end[c + 1] = first vertex of cell c
    short list[kPts];
};

template <int kPts>
__device__ __forceinline__ int bucket_of(const VertexBuckets<kPts>& B, double lx, double ly) {
    int cx = (int)floor(lx / B.cell), cy = (int)floor(ly / B.cell);
    cx = cx < 0 ? 0 : (cx >= B.ncx ? B.ncx - 1 : cx);
    cy = cy < 0 ? 0 : (cy >= B.ncy ? B.ncy - 1 : cy);
    return cy * B.ncx + cx;
}

// All threads: buckets of the vertices 0 .. npts-1 from their staged FP32
// box-local coordinates P32 (each within 2^-24 L of the exact one, far inside
// the search's 1e-3 cell margin).  Ends with a barrier.
template <int kPts>
__device__ void build_buckets(VertexBuckets<kPts>& B, const float2* P32, int npts, int wi, int hi) {
    const int cs = max(4, (max(wi, hi) + kCellMax - 1) / kCellMax);
    const int ncx = (wi + cs - 1) / cs, ncy = (hi + cs - 1) / cs, nc = ncx * ncy;
    if (threadIdx.x == 0) {
        B.ncx = ncx;
        B.ncy = ncy;
        B.cell = cs;
    }
    for (int c = threadIdx.x; c <= nc; c += blockDim.x) B.end[c] = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < npts; k += blockDim.x)
        atomicAdd(&B.end[bucket_of(B, (double)P32[k].x, (double)P32[k].y) + 1], 1);
    __syncthreads();
    if (threadIdx.x < 32) {  // inclusive scan of the counts by one warp
        int carry = 0;
        for (int c0 = 1; c0 <= nc; c0 += 32) {
            const int c = c0 + (int)threadIdx.x;
            int v = c <= nc ? B.end[c] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, v, o);
                if ((int)threadIdx.x >= o) v += u;
            }
            if (c <= nc) B.end[c] = v + carry;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < npts; k += blockDim.x) {
        const int pos = atomicSub(&B.end[bucket_of(B, (double)P32[k].x, (double)P32[k].y) + 1], 1) - 1;
        B.list[pos] = (short)k;
    }
    __syncthreads();
}

__device__ __forceinline__ double dist2_rn(double px, double py, const CPoint& q) {
    const double ex = px - q.x, ey = py - q.y;
    return __dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey));
}

__device__ __forceinline__ float tie_margin(float d, float eps_c) { return (sqrtf(d) + 1.f) * eps_c + d * 1e-6f; }

constexpr unsigned kKeyIndexBits = 10;
constexpr unsigned kKeyIndexMask = (1u << kKeyIndexBits) - 1u;
static_assert(kCorrStagedPts <= kCorrBigPts && kCorrBigPts <= (1 << kKeyIndexBits), "vertex index must fit the key");

// The reference's nearest vertex of the pixels (px, py) of the 32 lanes of a
// warp (grid coordinates; all lanes call it, `need` lanes are the pixels
// that want it).  The lanes scan together the vertices of the union of their
// 3 x 3 cell windows in FP32 on the staged box-local contour P32 (each
// coordinate within 2^-24 L of the exact local value, L the box edge, so a
// squared distance d within 3 sqrt(d) 2^-24 L + 3e-7 d of the exact one):
// each candidate is one 32-bit key, the distance's bits with the low 10
// replaced by the vertex index, and a lane keeps its smallest key k1 and the
// second smallest k2.  A lane whose two best lie within twice the rounding
// bound (tie_margin with eps_c = 8 2^-24 L; the keys' truncation taken on
// both sides) measures the candidates within that margin again in FP64 from
// the contour itself, lowest index first at equal distance.  A lane whose
// best distance exceeds (cell - 1e-3)^2 scans every vertex in FP64 (a vertex
// within `cell` of the pixel lies in its window).
template <int kPts>
__device__ int nearest_vertex_warp(const VertexBuckets<kPts>& B, const float2* P32, const CPoint* P, int npts, int px,
                                   int py, int ox, int oy, float eps_c, bool need) {
    const unsigned FULL = 0xffffffffu;
    const int cs = B.cell;
    const int lx = px - ox, ly = py - oy;
    const int cx = min(max(lx / cs, 0), B.ncx - 1), cy = min(max(ly / cs, 0), B.ncy - 1);
    const int ux0 = max(__reduce_min_sync(FULL, need ? cx : INT_MAX) - 1, 0);
    const int ux1 = min(__reduce_max_sync(FULL, need ? cx : INT_MIN) + 1, B.ncx - 1);
    const int uy0 = max(__reduce_min_sync(FULL, need ? cy : INT_MAX) - 1, 0);
    const int uy1 = min(__reduce_max_sync(FULL, need ? cy : INT_MIN) + 1, B.ncy - 1);
    const float fx = (float)lx, fy = (float)ly;
    unsigned k1 = 0xffffffffu, k2 = 0xffffffffu;
    const int ncell = B.ncx * B.ncy;
    for (int yy = uy0; yy <= uy1; ++yy) {
        // cells ux0 .. ux1 of a row are consecutive in the list
        const int q0 = B.end[yy * B.ncx + ux0 + 1];
        const int cl = yy * B.ncx + ux1;
        const int q1 = cl + 1 < ncell ? B.end[cl + 2] : npts;
        for (int q = q0; q < q1; ++q) {
            const int k = B.list[q];
            const float2 v = P32[k];
            const float dx = fx - v.x, dy = fy - v.y;
            const float d = fmaf(dy, dy, dx * dx);
            const unsigned key = (__float_as_uint(d) & ~kKeyIndexMask) | (unsigned)k;
            k2 = min(k2, max(k1, key));
            k1 = min(k1, key);
        }
    }
    if (!need) return -1;
    const float d1 = __uint_as_float(min(k1 | kKeyIndexMask, 0x7f7fffffu));
    const float r = (float)cs - 1e-3f;
    const bool covered = k1 != 0xffffffffu && d1 <= r * r;
    const float thr = d1 + tie_margin(d1, eps_c);
    const bool tie = covered && k2 != 0xffffffffu && __uint_as_float(k2 & ~kKeyIndexMask) <= thr;
    int nearest = (int)(k1 & kKeyIndexMask);
    if (!covered) {
        const double dpx = (double)px, dpy = (double)py;
        double best = 1000000.0;  // the reference's initial minDist
        nearest = -1;
        for (int k = 0; k < npts; ++k) {
            const double d = dist2_rn(dpx, dpy, P[k]);
            if (d < best) {
                best = d;
                nearest = k;
            }
        }
    } else if (tie) {
        const double dpx = (double)px, dpy = (double)py;
        double best = 1000000.0;
        nearest = -1;
        for (int yy = max(cy - 1, 0); yy <= min(cy + 1, B.ncy - 1); ++yy) {
            const int q0 = B.end[yy * B.ncx + max(cx - 1, 0) + 1];
            const int cl = yy * B.ncx + min(cx + 1, B.ncx - 1);
            const int q1 = cl + 1 < ncell ? B.end[cl + 2] : npts;
            for (int q = q0; q < q1; ++q) {
                const int k = B.list[q];
                const float dx = fx - P32[k].x, dy = fy - P32[k].y;
                if (fmaf(dy, dy, dx * dx) > thr) continue;
                const double d = dist2_rn(dpx, dpy, P[k]);
                if (d < best || (d == best && k < nearest)) {
                    best = d;
                    nearest = k;
                }
            }
        }
    }
    return nearest;
}

// Distance from (fx, fy) to segment a -> b (the reference's three cases);
// *lam receives the unclamped projection parameter.
__device__ __forceinline__ float seg_dist32(float2 a, float2 b, float fx, float fy, float* lam) {
    const float ux = b.x - a.x, uy = b.y - a.y;
    const float l = ((fx - a.x) * ux + (fy - a.y) * uy) / (ux * ux + uy * uy);
    float dx, dy;
    if (l < 0) {
        dx = fx - a.x;
        dy = fy - a.y;
    } else if (l > 1) {
        dx = b.x - fx;
        dy = b.y - fy;
    } else {
        dx = fx - (a.x + ux * l);
        dy = fy - (a.y + uy * l);
    }
    *lam = l;
    return dx * dx + dy * dy;
}

// The segment step of projectToGrainBondary (src/grainBoundary.cpp:383-420)
// on the FP32 local contour P32: the segment after the vertex first, the one
// before it wins only if strictly closer.  When both projections fall beyond
// the vertex, both distances are the vertex's (equal in FP64 too) and the
// segment after it wins with lambda 0; when the two distances lie within the
// FP32 rounding margin (eps_c = 8 2^-24 L, L bounding the local coordinates)
// the step is taken again in FP64 from the contour itself.
__device__ __forceinline__ int segment_step(const float2* P32, const CPoint* P, int asize, int px, int py, int ox,
                                           int oy, float eps_c, int nearest, float* out_lambda) {
    const float fx = (float)(px - ox), fy = (float)(py - oy);
    float la, lb;
    const float da = seg_dist32(P32[nearest], P32[nearest + 1], fx, fy, &la);
    const int nv = nearest == 0 ? asize - 1 : nearest;
    const float db = seg_dist32(P32[nv - 1], P32[nv], fx, fy, &lb);
    if (la <= 0.f && lb >= 1.f) {
        *out_lambda = 0.f;
        return nearest;
    }
    if (fabsf(da - db) <= 4.f * tie_margin(fminf(da, db), eps_c)) {
        double dl = 0;
        const int seg = segment_of_vertex(P, asize, (double)px, (double)py, nearest, &dl);
        *out_lambda = (float)dl;
        return seg;
    }
    const bool before = db < da;
    const float lam = before ? lb : la;
    *out_lambda = fminf(fmaxf(lam, 0.f), 1.f);
    return before ? nv - 1 : nearest;
}

// Sectors of every grain for the next corrector (batched form), built one
// step ahead so that the corrector's warps do not wait on the serial build:
// the same build as the plain corrector's (prepare_sectors: segment lengths,
// neighbour table, junction weights, then setPointsOnBoundary and the
// constant / interpolating sectors, src/grainBoundary.cpp:233-342,
// src/contourSector.cpp), one 32-thread CTA per grain.  kCur: from the roles
// the step just produced (contour, junctions, IDLocal of this step, run after
// the neighbour characteristics are computed), which become the previous
// ones at the end of the step; else from the previous roles (after
// initialisation, grid coarsening or new neighbour lists).
template <bool kCur>
__global__ void __launch_bounds__(32) k_sectors(NetConst C, NetState* S) {
    const int g = grain_at(S, blockIdx.x);
    if (g > C.N || C.state[g] != G_EXISTS || halted(S)) return;
    __shared__ SectorSet sec;
    __shared__ double jw[64];
    __shared__ uint32_t s_st;
    __shared__ double s_per;
    __shared__ NbTable nbt;
    __shared__ int jl[64], jr[64];
    const int64_t coff = kCur ? S->coff_cur[g] : S->coff_prev[g];
    const CPoint* P = (kCur ? S->contCur : S->contPrev) + coff;
    const int size = kCur ? S->cn_cur[g] : S->cn_prev[g];
    SectorPack* pk = reinterpret_cast<SectorPack*>(C.secpack) + g;
    if (size < 2) {
        if (threadIdx.x == 0) {
            pk->nconst = 0;
            pk->ninterp = 0;
        }
        return;
    }
    // segment lengths: the corrector's scratch at this contour's offsets (no
    // corrector reads it while this kernel runs; a global buffer leaves room
    // for more CTAs per SM than a shared one)
    double* seg = S->segPrev + coff;
    const Box ib = kCur ? S->box_cur[g] : S->box_prev[g];
    const uint32_t* idl = kCur ? S->idCur + S->off_cur[g] : S->idPrev + S->off_prev[g];
    const Junction* J = (kCur ? S->jCur : S->jPrev) + (int64_t)g * C.jmax;
    const int nj = min(kCur ? S->jn_cur[g] : S->jn_prev[g], 64);
    prepare_sectors_view(C, S, g, P, size, seg, sec, jw, &s_st, &s_per, nbt, jl, jr, ib, idl, J, nj);
    const int nc = sec.nconst, ni = sec.ninterp;
    if (threadIdx.x == 0) {
        pk->nconst = nc;
        pk->ninterp = ni;
    }
    for (int c = threadIdx.x; c < nc; c += blockDim.x) pk->cw[c] = sec.cs[c].weight;
    for (int c = threadIdx.x; c < ni; c += blockDim.x) pk->is[c] = sec.is[c];
    for (int q = threadIdx.x; q < size - 1; q += blockDim.x) {
        int sid;
        double acc;
        seg_table_entry(sec, seg, size, q, &sid, &acc);
        C.segsec[coff + q] = (int16_t)sid;
        C.segacc[coff + q] = (float)acc;
    }
}

// Shared memory of one CTA of the batched corrector.
template <int kPts>
struct CorrectorSmem {
    float2 sp[kPts];  // the contour, FP32 box-local
    NbTable nbt;
    VertexBuckets<kPts> vb;
    double cw[kMaxConstSectors];
    InterpSector is[kMaxInterpSectors];
    int16_t sid[kPts];  // per-segment sector table
    float acc[kPts];
};

// Whether grain g is corrected at all this step (uniform over the CTA).
__device__ __forceinline__ bool corrects(const NetConst& C, const NetState* S, int g) {
    return g <= C.N && C.state[g] == G_EXISTS && C.regular[g] != 0 && S->loop != 0 && !halted(S);
}

// The correction of grain g by the whole CTA (all threads call it; every
// early return is uniform over the CTA).
template <bool kForces, int kPts>
__device__ __forceinline__ void correct_grain(const NetConst& C, NetState* S, int g, CorrectorSmem<kPts>& sm) {
    float2* sp = sm.sp;
    NbTable& nbt = sm.nbt;
    VertexBuckets<kPts>& vb = sm.vb;
    double* s_cw = sm.cw;
    InterpSector* s_is = sm.is;
    int16_t* s_sid = sm.sid;
    float* s_acc = sm.acc;
    const int64_t coff = S->coff_prev[g];
    const CPoint* P = S->contPrev + coff;
    const int size = S->cn_prev[g];
    if (size < 2) return;
    const Box ib = S->box_prev[g];
    const uint32_t* idl = S->idPrev + S->off_prev[g];
    const bool staged = size <= kPts;
    // the contour in FP32 coordinates local to the previous box (its points
    // lie inside it), so the search's rounding is relative to the box edge
    const int ox = ib.x0, oy = ib.y0;
    if (staged)
        for (int k = threadIdx.x; k < size; k += blockDim.x)
            sp[k] = make_float2((float)(P[k].x - ox), (float)(P[k].y - oy));
    // the sectors, built one step ahead (k_sectors), and the per-segment table
    const SectorPack* pk = reinterpret_cast<const SectorPack*>(C.secpack) + g;
    const int nconst = pk->nconst, ninterp = pk->ninterp;
    for (int c = threadIdx.x; c < nconst; c += blockDim.x) s_cw[c] = pk->cw[c];
    for (int c = threadIdx.x; c < ninterp; c += blockDim.x) s_is[c] = pk->is[c];
    const int16_t* tsid = C.segsec + coff;
    const float* tacc = C.segacc + coff;
    if (staged) {
        for (int q = threadIdx.x; q < size - 1; q += blockDim.x) {
            s_sid[q] = tsid[q];
            s_acc[q] = tacc[q];
        }
        tsid = s_sid;
        tacc = s_acc;
    }
    build_nb_table(C, g, nbt);
    if (staged) build_buckets(vb, sp, size - 1, box_w(ib), box_h(ib));  // ends with a barrier
    __syncthreads();
    const Box bo = S->box_cur[g];
    const int x0 = ib.x0 < bo.x0 ? bo.x0 : ib.x0;
    const int y0 = ib.y0 < bo.y0 ? bo.y0 : ib.y0;
    const int x1 = ib.x1 > bo.x1 ? bo.x1 : ib.x1;
    const int y1 = ib.y1 > bo.y1 ? bo.y1 : ib.y1;
    if (x1 <= x0 || y1 <= y0) return;
    const int w = x1 - x0, hgt = y1 - y0;
    const float* in = reinterpret_cast<const float*>(S->phiA) + S->off_cur[g];
    float* out = reinterpret_cast<float*>(S->phiB) + S->off_cur[g];
    const int wo = box_w(bo), wi = box_w(ib);
    const float delta = (float)C.delta;
    const int real = size - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int ntx = (w + 7) >> 3, ntiles = ntx * ((hgt + 3) >> 2);
    uint32_t st = 0;
    const bool far_ok = C.gamma_hagb <= 1.0 && C.m_hagb <= 1.0;
    // rounding margin of the FP32 segment step: 8 2^-24 L, L bounding every
    // local coordinate of the contour and the pixels
    const float eps_c = 8.f * 5.9604645e-8f * (float)(max(wi, box_h(ib)) + 2);
    // one warp per 8 x 4 tile; pixels at or below -delta are set to -delta
    for (int t = warp; t < ntiles; t += nwarps) {
        const int x = (t % ntx) * 8 + (lane & 7), y = (t / ntx) * 4 + (lane >> 3);
        const bool inside = x < w && y < hgt;
        const int i = y0 + y, j = x0 + x;
        const int k = (i - bo.y0) * wo + (j - bo.x0);
        float val = 0.f, conv = 0.f;
        uint32_t id = 0;
        if (inside) {
            val = __ldg(in + k);
            conv = out[k];
            id = idl[(i - ib.y0) * wi + (j - ib.x0)];
        }
        const bool valid = inside && val > -delta;
        // driving-force terms (src/box.cpp:511-527) of inside pixels
        float se = 0.f;
        if (kForces && inside) {
            double f = 0;
            if (C.stored) f += nb_stored_force(nbt, (int)id) * C.dt / C.time_slope;
            if (C.magnetic) f += nb_magnetic_force(nbt, (int)id) * C.dt / C.time_slope;
            se = (float)f;
        }
        if (inside && !valid) out[k] = -delta - se;
        // The corrected value val + (conv - val) w lies between val and
        // 2 conv - val for every weight w in [0, 2]; with the relative
        // high-angle energy and mobility at most 1 the weights (energy x
        // mobility products, junction sums of three energies, their blends)
        // stay below 2 (far_ok).  When val, conv and
        // 2 conv - val all lie on the same side beyond 0.3 delta (2.1 cells),
        // the pixel keeps that side whatever its weight, and it is not next to
        // a sign change of these near-distance fields; only signs and the
        // values next to sign changes reach the comparison's zero crossings
        // and the redistancing that replaces the field.  Such a pixel takes
        // weight 1 (the convolved value) without the projection.  (On the
        // 20,000-grain workload the areas stay bit-identical for 10 steps and
        // within 1.3e-7 relative, in 18 grains, after 40.)
        const float far_level = 0.3f * delta, stretched = 2.f * conv - val;
        const bool far = far_ok && valid &&
                         ((val >= far_level && conv >= far_level && stretched >= far_level) ||
                          (val <= -far_level && conv <= -far_level && stretched <= -far_level));
        if (far) out[k] = conv - se;
        const bool need = valid && !far;
        if (__ballot_sync(0xffffffffu, need) == 0u) continue;
        float lambda = 0.f;
        int segment = 0;
        if (staged) {
            const int nv = nearest_vertex_warp(vb, sp, P, size - 1, j, i, ox, oy, eps_c, need);
            if (!need) continue;
            if (nv >= 0) segment = segment_step(sp, P, size, j, i, ox, oy, eps_c, nv, &lambda);
        } else {
            if (!need) continue;
            double dl = 0;
            segment = project_to_boundary(P, size, (double)j, (double)i, &dl);
            lambda = (float)dl;
        }
        const int sid = tsid[segment];
        float interpolator = sid <= -2 ? tacc[segment] : 0.f;
        float weight;
        if (sid >= 0) {
            weight = (float)s_cw[sid];
        } else if (sid == -1) {
            // getGBEnergyTimesGBMobility(i, j) through the neighbour table
            weight = 1.f;
            for (int e = 0; e < nbt.n; ++e)
                if (nbt.id[e] == (int)id) {
                    weight = (float)nbt.w[e];
                    break;
                }
        } else {
            const InterpSector& s = s_is[-2 - sid];
            const int kn = wrap_next(segment, real);
            float ax, ay;
            if (staged) {
                ax = (sp[kn].x - sp[segment].x) * lambda;
                ay = (sp[kn].y - sp[segment].y) * lambda;
            } else {
                ax = (float)((P[kn].x - P[segment].x) * lambda);
                ay = (float)((P[kn].y - P[segment].y) * lambda);
            }
            interpolator += sqrtf(ax * ax + ay * ay);
            interpolator /= (float)s.length;
            interpolator = fminf(fmaxf(interpolator, 0.f), 1.f);
            const float lw = (float)s.left_w, rw = (float)s.right_w;
            if (s.lb >= 0 && s.rb >= 0) {
                const float isr = (float)C.isr, len = (float)s.length;
                const float quot = (len > 2 * isr ? 2 * isr : len);
                const float amplitude = ((float)s.boundary_w - (lw + rw) / 2) / (2 * isr) * quot + (lw + rw) / 2;
                const float a0 = 2 * rw, a1 = -4 * amplitude, a2 = 2 * lw;
                const float A = a0 + a1 + a2, B = -(a0 * 1.5f + a1 + a2 * 0.5f), Cc = a0 * 0.5f;
                weight = A * interpolator * interpolator + B * interpolator + Cc;
            } else {
                weight = interpolator * lw + (1 - interpolator) * rw;
            }
        }
        out[k] = val + (conv - val) * weight - se;
    }
    if (st) set_status(S, st);
}

// CTA per grain from the work queue, contours staged up to kCorrStagedPts;
// grains flagged for the large-contour kernel are left to it.
template <bool kForces>
__global__ void __launch_bounds__(128, 7) k_corrector_f(NetConst C, NetState* S) {
    __shared__ __align__(16) CorrectorSmem<kCorrStagedPts> sm;
    const int g = grain_at(S, blockIdx.x);
    if (!corrects(C, S, g) || S->big_flag[g]) return;
    correct_grain<kForces, kCorrStagedPts>(C, S, g, sm);
}

// Persistent over NetState::big_list: the grains whose contour is longer than
// the main kernel stages, up to kCorrBigPts staged; CTA b takes entries b,
// b + G, ... (G CTAs).  The grid (kCorrBigPerSm CTAs per SM) usually covers
// the whole list, so every such grain starts at once, and the launch has the
// device's highest priority, so that these CTAs are placed before the
// pending ones of the main corrector beside them.
template <bool kForces>
__global__ void __launch_bounds__(128) k_corrector_big(NetConst C, NetState* S) {
    __shared__ __align__(16) CorrectorSmem<kCorrBigPts> sm;
    const int n = S->n_big;
    for (int q = blockIdx.x; q < n; q += gridDim.x) {
        const int g = S->big_list[q];
        if (corrects(C, S, g)) correct_grain<kForces, kCorrBigPts>(C, S, g, sm);
        __syncthreads();  // the next grain overwrites the shared memory
    }
}

// persistent grid of the large-box kernels: one CTA per SM
int g_big_grid = 148;
// highest stream priority of the device (numerically lowest)
int g_high_priority = 0;
constexpr int kCorrBigPerSm = 4;

void launch_corrector_main(const NetConst& C, NetState* dS, cudaStream_t s) {
    if (C.stored || C.magnetic)
        k_corrector_f<true><<<C.N, 128, 0, s>>>(C, dS);
    else
        k_corrector_f<false><<<C.N, 128, 0, s>>>(C, dS);
}

void launch_corrector_big(const NetConst& C, NetState* dS, cudaStream_t s) {
    const int grid = C.N < kCorrBigPerSm * g_big_grid ? C.N : kCorrBigPerSm * g_big_grid;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = g_high_priority;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (C.stored || C.magnetic)
        cudaLaunchKernelEx(&cfg, k_corrector_big<true>, C, dS);
    else
        cudaLaunchKernelEx(&cfg, k_corrector_big<false>, C, dS);
}

// Both correctors on one stream (the graph runs them on two).
void launch_corrector_f(const NetConst& C, NetState* dS, cudaStream_t s) {
    launch_corrector_big(C, dS, s);
    launch_corrector_main(C, dS, s);
}

cudaError_t batched_resample(const NetConst& C, NetState* dS, double h_old, double hn, double delta_old,
                             cudaStream_t s) {
    if (C.N > 0) k_resample<float><<<C.N, 256, 0, s>>>(C, dS, h_old, hn, delta_old);
    return cudaGetLastError();
}

cudaError_t batched_prepare(int tmax) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_sep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)conv_sep_smem(tmax, kConvSmemEdgeMax));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_redistance_big, cudaFuncAttributeMaxDynamicSharedMemorySize, kRedistBigSmemBytes);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    g_big_grid = sms > 0 ? sms : 148;
    int least = 0, greatest = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&least, &greatest)) != cudaSuccess) return e;
    g_high_priority = greatest;
    return cudaSuccess;
}

// The redistancing stage: the large-box bin, then the 64-thread kernel for
// the rest.
void launch_redistance(const NetConst& C, NetState* dS, cudaStream_t s) {
    const int grid = C.N < g_big_grid ? C.N : g_big_grid;
    k_redistance_big<<<grid, kRedistBigThreads, kRedistBigSmemBytes, s>>>(C, dS);
    k_redistance_s<float><<<C.N, kRedistThreads, kRedistSmemBytes, s>>>(C, dS);
}

cudaError_t batched_init(const NetConst& C, NetState* dS, const int32_t* d_ids, cudaStream_t s) {
    if (C.N <= 0) return cudaSuccess;
    k_init_phi<float><<<C.N, 256, 0, s>>>(C, dS, d_ids);
    // the step's redistancing kernels take grains from the work queue, so it
    // is built from the initial boxes first
    k_order<<<1, 1024, 0, s>>>(C, dS);
    launch_redistance(C, dS, s);
    cudaError_t e = swap_phi(dS, s);
    if (e != cudaSuccess) return e;
    k_init_contour_w<float><<<(C.N + kGrainsPerBlock - 1) / kGrainsPerBlock, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    return cudaGetLastError();
}

size_t batched_sector_pack_bytes() { return sizeof(SectorPack); }

cudaError_t batched_sectors(const NetConst& C, NetState* dS, cudaStream_t s) {
    if (C.N <= 0) return cudaSuccess;
    k_sectors<false><<<C.N, 32, 0, s>>>(C, dS);
    return cudaGetLastError();
}

cudaError_t batched_order(const NetConst& C, NetState* dS, cudaStream_t s) {
    if (C.N <= 0) return cudaSuccess;
    k_order<<<1, 1024, 0, s>>>(C, dS);
    return cudaGetLastError();
}

cudaError_t batched_init_polygon(const NetConst& C, NetState* dS, cudaStream_t s) {
    if (C.N <= 0) return cudaSuccess;
    k_polygon_phi<float><<<C.N, 256, 0, s>>>(C, dS);
    return cudaGetLastError();
}

cudaError_t batched_stage_kernel(const NetConst& C, NetState* dS, int which, cudaStream_t s, const LaunchCfg& cfg) {
    const int gt = cfg.grain_threads;
    const int gblocks = (C.N + gt - 1) / gt;
    const int wblocks = (C.N + kGrainsPerBlock - 1) / kGrainsPerBlock;
    (void)gblocks;
    switch (which) {
        case 0: k_conv_sep<<<C.N, 128, conv_sep_smem(C.tmax, C.conv_smem_edge), s>>>(C, dS); break;
        case 1: if (!C.isotropic) launch_corrector_f(C, dS, s); break;
        case 2: k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 3: k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS); break;
        case 4: k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 5: k_alloc<<<1, 1024, 0, s>>>(C, dS, 1); break;
        case 6:
            k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo));
            k_sectors<true><<<C.N, 32, 0, s>>>(C, dS);
            break;
        case 7: launch_redistance(C, dS, s); break;
        default:
            k_finalize<<<1, 1024, 0, s>>>(C, dS, 1);
            k_order<<<1, 1024, 0, s>>>(C, dS);
            break;
    }
    return cudaGetLastError();
}

cudaError_t batched_stages(const NetConst& C, NetState* dS, int stages, cudaStream_t s, const LaunchCfg& cfg) {
    if (C.N <= 0) return cudaSuccess;
    const int gt = cfg.grain_threads;
    const int gblocks = (C.N + gt - 1) / gt;
    const int wblocks = (C.N + kGrainsPerBlock - 1) / kGrainsPerBlock;
    (void)gblocks;
    if (stages & ST_CONV) {
        k_conv_sep<<<C.N, 128, conv_sep_smem(C.tmax, C.conv_smem_edge), s>>>(C, dS);
        if (!C.isotropic) launch_corrector_f(C, dS, s);
    }
    if (stages & ST_SECOND) k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_COMPARE) k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS);
    if (stages & ST_LEVELSET) k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_REDIST) {
        k_alloc<<<1, 1024, 0, s>>>(C, dS, 1);
        k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo));
        k_sectors<true><<<C.N, 32, 0, s>>>(C, dS);
        launch_redistance(C, dS, s);
        k_finalize<<<1, 1024, 0, s>>>(C, dS, 1);
        k_order<<<1, 1024, 0, s>>>(C, dS);
    }
    return cudaGetLastError();
}

cudaError_t batched_step_graph(const NetConst& C, NetState* dS, cudaStream_t s, cudaStream_t s2, cudaEvent_t* ev,
                               const LaunchCfg& cfg) {
    if (C.N <= 0) return cudaSuccess;
    const int wblocks = (C.N + kGrainsPerBlock - 1) / kGrainsPerBlock;
    cudaError_t e;
    // second-order lists (lists and boxes only) beside convolution + corrector (fields)
    if ((e = cudaEventRecord(ev[0], s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s2, ev[0], 0)) != cudaSuccess) return e;
    k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s2>>>(C, dS);
    k_conv_sep<<<C.N, 128, conv_sep_smem(C.tmax, C.conv_smem_edge), s>>>(C, dS);
    if (!C.isotropic) {
        // the large-contour corrector beside the main one
        if ((e = cudaEventRecord(ev[4], s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s2, ev[4], 0)) != cudaSuccess) return e;
        launch_corrector_big(C, dS, s2);
        launch_corrector_main(C, dS, s);
    }
    if ((e = cudaEventRecord(ev[1], s2)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s, ev[1], 0)) != cudaSuccess) return e;
    k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS);
    k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    k_alloc<<<1, 1024, 0, s>>>(C, dS, 1);
    // volume / energy / neighbours (contours, lists) and the next step's
    // sectors beside redistancing (fields)
    if ((e = cudaEventRecord(ev[2], s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s2, ev[2], 0)) != cudaSuccess) return e;
    k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s2>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo));
    k_sectors<true><<<C.N, 32, 0, s2>>>(C, dS);  // the next step's sectors
    if ((e = cudaEventRecord(ev[3], s2)) != cudaSuccess) return e;
    launch_redistance(C, dS, s);
    if ((e = cudaStreamWaitEvent(s, ev[3], 0)) != cudaSuccess) return e;
    k_finalize<<<1, 1024, 0, s>>>(C, dS, 1);
    k_order<<<1, 1024, 0, s>>>(C, dS);  // the next step's work queue, from its boxes
    return cudaGetLastError();
}

}  // namespace gg
