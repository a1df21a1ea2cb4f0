// Batched form: FP32 distance fields and convolution (FP64 contour areas,
// energies and lengths), every stage over all grains, captured per step as
// one CUDA graph by the host.
#include "gg_corrector.cuh"
#include "gg_kernels.cuh"
#include "gg_launch.cuh"
#include "gg_warp.cuh"

namespace gg {

constexpr int kSepSmemMaxN = 64;  // intermediate in shared memory up to this edge
constexpr int kSepStrip = 4;       // outputs per thread along the convolution axis

// Gaussian convolution as a separable circular convolution in real space:
// out = K X K^T with K[r][r'] = k_n[(r - r') mod n], where k_n is the real
// kernel whose DFT is the reference's Gaussian multiplier
// (src/box.cpp:674-687, G(i2, j2) = g(i2) g(j2) / n^2).  One CTA per grain.
// The kernel is laid out once as kx[j] = k_n[(j - (n-1)) mod n], j < 2n-1
// (zero-padded), so output c of a row is sum_c' X[c'] kx[c - c' + n - 1]:
// each thread accumulates a strip of 4 consecutive outputs while a 4-entry
// register window slides down kx (one shared-memory load per 4 FMAs).  Taps
// farther than R (circularly) from the strip are left out: the host sets R
// so that every dropped k_n entry is below 2^-26 k_n[0].

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
        int rs[2], re[2];
        band_ranges(c0, n, R, &rs[0], &re[0], &rs[1], &re[1]);
        for (int q = 0; q < 2; ++q) {
            int base = c0 + n - 1 - rs[q];  // kx index of (c0 - c') at c' = rs[q]
            float w0 = kx[base], w1 = kx[base + 1], w2 = kx[base + 2], w3 = kx[base + 3];
#pragma unroll 4
            for (int cp = rs[q]; cp < re[q]; ++cp) {
                const float x = xa[cp], y = xb[cp];
                a0 = fmaf(x, w0, a0);
                a1 = fmaf(x, w1, a1);
                a2 = fmaf(x, w2, a2);
                a3 = fmaf(x, w3, a3);
                b0 = fmaf(y, w0, b0);
                b1 = fmaf(y, w1, b1);
                b2 = fmaf(y, w2, b2);
                b3 = fmaf(y, w3, b3);
                --base;
                w3 = w2;
                w2 = w1;
                w1 = w0;
                w0 = kx[base];
            }
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

__device__ __forceinline__ void sep_pass_cols(const float* __restrict__ T, float* __restrict__ out,
                                              const float* __restrict__ kx, int n, int R) {
    const int nb = (n + kSepStrip - 1) / kSepStrip;
    for (int t = threadIdx.x; t < n * nb; t += blockDim.x) {
        const int rb = t / n, c = t - rb * n, r0 = rb * kSepStrip;
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
        int rs[2], re[2];
        band_ranges(r0, n, R, &rs[0], &re[0], &rs[1], &re[1]);
        for (int q = 0; q < 2; ++q) {
            int base = r0 + n - 1 - rs[q];
            float w0 = kx[base], w1 = kx[base + 1], w2 = kx[base + 2], w3 = kx[base + 3];
#pragma unroll 4
            for (int rp = rs[q]; rp < re[q]; ++rp) {
                const float x = T[rp * n + c];
                a0 = fmaf(w0, x, a0);
                a1 = fmaf(w1, x, a1);
                a2 = fmaf(w2, x, a2);
                a3 = fmaf(w3, x, a3);
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
    const bool fits = n <= kSepSmemMaxN;
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

size_t conv_sep_smem(int tmax) {
    // the row-pass intermediate of a box (edge up to kSepSmemMaxN) with its
    // extended kernel, or the extended kernel alone of the largest box (whose
    // intermediate goes to the grain's scratch in device memory)
    const int n = tmax < kSepSmemMaxN ? tmax : kSepSmemMaxN;
    const size_t staged = (size_t)n * n + 2 * (size_t)n + kSepStrip + 2;
    const size_t kernel_only = 2 * (size_t)tmax + kSepStrip + 2;
    return sizeof(float) * (staged > kernel_only ? staged : kernel_only);
}

// Batched-form corrector: same sectors as k_corrector (built by one warp),
// with the previous contour staged in shared memory (FP32 coordinates) and
// the per-pixel work in FP32.  Each warp takes one 8 x 4 tile of the box at a
// time, so its 32 pixels lie close together and the warp prunes the
// nearest-vertex search as one: chunks of 8 contour points whose bounding box
// is farther from the tile than every lane's best point so far are skipped
// by all lanes together.
constexpr int kCorrMaxPts = 512;

constexpr int kChunk = 8;  // contour points per bounding box of the nearest-vertex search

// Slack on the chunk bound so that a box distance which rounds a little
// above an equal point distance does not drop the chunk (ties matter).
constexpr float kBoundSlack = 1.0000005f;

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two contour points per
// instruction in the nearest-vertex scan.
__device__ __forceinline__ unsigned long long f2_pack(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// projectToGrainBondary (src/grainBoundary.cpp:365-447) for the pixels
// (px, py) of the 32 lanes of a warp (all lanes call it; `valid` lanes are
// the warp's real pixels, the others only follow along), with the reference's
// FP64 decisions.  The search runs in FP32 on the contour staged in box-local
// coordinates (P32, origin (ox, oy), two points per float4; coordinates up to
// L = the box edge, so each is within 2^-24 L of the exact local value):
//   pass 1: each lane's smallest FP32 squared distance dmin, chunks of 8
//           points skipped by all lanes together when their bounding box is
//           farther from the warp's pixels than every lane's best so far;
//   pass 2: every vertex whose FP32 distance is within the rounding margin of
//           dmin (|d32 - d| <= 3 sqrt(d) 2^-24 L + 3e-7 d, taken twice with
//           room to spare: eps_c = 8 2^-24 L) is measured again in FP64 from
//           the contour itself (P), in ascending index order with strict <:
//           the reference's first vertex at the smallest distance.
// The segment and lambda then follow in FP64 (segment_of_vertex).  A vertex
// outside the margin is farther than the FP32 minimum's vertex in exact
// arithmetic, so the FP64 choice is the one the reference makes on this
// contour.  *wseed: the chunk that held the nearest vertex of the warp's
// previous tile, searched first.
constexpr float kFarD = 3.0e38f;

__device__ __forceinline__ int project_warp(const float2* P32, const CPoint* P, const float4* cbb, int asize, int px,
                                            int py, int ox, int oy, float eps_c, bool valid, double* out_lambda,
                                            int* wseed) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const float fx = (float)(px - ox), fy = (float)(py - oy);
    const unsigned long long FX = f2_pack(fx, fx), FY = f2_pack(fy, fy);
    const int npts = asize - 1;
    const int nch = (npts + kChunk - 1) / kChunk;
    const float4* P2 = reinterpret_cast<const float4*>(P32);
    float dmin = kFarD;
    auto scan = [&](int ch) {
        const int k0 = ch * kChunk, k1 = min(k0 + kChunk, npts);
        for (int k = k0; k < k1; k += 2) {
            const float4 v = P2[k >> 1];
            const unsigned long long DX = f2_sub(FX, f2_pack(v.x, v.z)), DY = f2_sub(FY, f2_pack(v.y, v.w));
            float d0, d1;
            f2_unpack(f2_fma(DY, DY, f2_mul(DX, DX)), d0, d1);
            dmin = fminf(dmin, d0);
            if (k + 1 < k1) dmin = fminf(dmin, d1);
        }
    };
    const int sc = *wseed < nch ? *wseed : 0;
    scan(sc);
    const int bx0 = __reduce_min_sync(FULL, valid ? px - ox : INT_MAX);
    const int bx1 = __reduce_max_sync(FULL, valid ? px - ox : INT_MIN);
    const int by0 = __reduce_min_sync(FULL, valid ? py - oy : INT_MAX);
    const int by1 = __reduce_max_sync(FULL, valid ? py - oy : INT_MIN);
    // squared distance from the warp's pixels to chunk ch's bounding box (a
    // lower bound of every lane's distance to its points)
    auto lower = [&](int ch) {
        const float4 b = cbb[ch];
        const float gx = fmaxf(fmaxf(b.x - (float)bx1, (float)bx0 - b.y), 0.f);
        const float gy = fmaxf(fmaxf(b.z - (float)by1, (float)by0 - b.w), 0.f);
        return gx * gx + gy * gy;
    };
    // an upper bound of the valid lanes' values v (non-negative floats)
    auto wmax = [&](float v) { return __uint_as_float(__reduce_max_sync(FULL, valid ? __float_as_uint(v) : 0u)); };
    float U = wmax(dmin);
    for (int c0 = 0; c0 < nch; c0 += 32) {
        const int ch = c0 + lane;
        const float lb = ch < nch ? lower(ch) : kFarD;
        unsigned mask = __ballot_sync(FULL, ch < nch && ch != sc && lb <= U * kBoundSlack);
        while (mask) {
            const int bit = __ffs(mask) - 1;
            mask &= mask - 1;
            const float lbc = __shfl_sync(FULL, lb, bit);
            if (lbc > U * kBoundSlack) continue;
            scan(c0 + bit);
            U = wmax(dmin);
        }
    }
    // pass 2: the candidates within the margin, in FP64 and index order
    const float thr = dmin + (sqrtf(dmin) + 1.f) * eps_c + (dmin + 1.f) * 2e-6f;
    const float T = wmax(thr) * kBoundSlack;
    const double dpx = (double)px, dpy = (double)py;
    double best = 1000000.0;  // the reference's initial minDist
    int nearest = -1;
    for (int c0 = 0; c0 < nch; c0 += 32) {
        const int ch = c0 + lane;
        unsigned mask = __ballot_sync(FULL, ch < nch && lower(ch) <= T);
        while (mask) {
            const int bit = __ffs(mask) - 1;
            mask &= mask - 1;
            const int k0 = (c0 + bit) * kChunk, k1 = min(k0 + kChunk, npts);
            for (int k = k0; k < k1; k += 2) {
                const float4 v = P2[k >> 1];
                const unsigned long long DX = f2_sub(FX, f2_pack(v.x, v.z)), DY = f2_sub(FY, f2_pack(v.y, v.w));
                float d0, d1;
                f2_unpack(f2_fma(DY, DY, f2_mul(DX, DX)), d0, d1);
                if (valid && d0 <= thr) {
                    const double ex = dpx - P[k].x, ey = dpy - P[k].y;
                    const double d = __dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey));
                    if (d < best) {
                        best = d;
                        nearest = k;
                    }
                }
                if (valid && k + 1 < k1 && d1 <= thr) {
                    const double ex = dpx - P[k + 1].x, ey = dpy - P[k + 1].y;
                    const double d = __dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey));
                    if (d < best) {
                        best = d;
                        nearest = k + 1;
                    }
                }
            }
        }
    }
    {
        const int src = __ffs(__ballot_sync(FULL, valid && nearest >= 0)) - 1;
        const int sn = __shfl_sync(FULL, nearest, src < 0 ? 0 : src);
        if (src >= 0) *wseed = sn / kChunk;
    }
    if (!valid || nearest < 0) return 0;
    return segment_of_vertex(P, asize, dpx, dpy, nearest, out_lambda);
}

// kForces: with the stored-energy and / or magnetic driving-force terms.
template <bool kForces>
__global__ void __launch_bounds__(128, 8) k_corrector_f(NetConst C, NetState* S) {
    const int g = grain_at(S, blockIdx.x);
    if (g > C.N || C.state[g] != G_EXISTS || C.regular[g] == 0 || S->loop == 0 || halted(S)) return;
    __shared__ SectorSet sec;
    __shared__ __align__(16) float2 sp[kCorrMaxPts];
    __shared__ double jw[64];
    __shared__ uint32_t s_st;
    __shared__ double s_per;
    __shared__ NbTable nbt;
    __shared__ float4 cbb[kCorrMaxPts / kChunk];
    __shared__ double s_seg[kSegShared];
    __shared__ SegTable stab;
    __shared__ int jl[64], jr[64];
    const CPoint* P = S->contPrev + S->coff_prev[g];
    const int size = S->cn_prev[g];
    if (size < 2) return;
    double* seg = size - 1 <= kSegShared ? s_seg : S->segPrev + S->coff_prev[g];
    const Box ib = S->box_prev[g];
    const uint32_t* idl = S->idPrev + S->off_prev[g];
    const bool staged = size <= kCorrMaxPts;
    // the contour in FP32 coordinates local to the previous box (its points
    // lie inside it), so the search's rounding is relative to the box edge
    const int ox = ib.x0, oy = ib.y0;
    if (staged)
        for (int k = threadIdx.x; k < size; k += blockDim.x)
            sp[k] = make_float2((float)(P[k].x - ox), (float)(P[k].y - oy));
    __syncthreads();
    if (staged) {
        const int npts = size - 1, nch = (npts + kChunk - 1) / kChunk;
        for (int ch = threadIdx.x; ch < nch; ch += blockDim.x) {
            float4 b = make_float4(3.0e38f, -3.0e38f, 3.0e38f, -3.0e38f);
            for (int k = ch * kChunk; k < min(ch * kChunk + kChunk, npts); ++k) {
                b.x = fminf(b.x, sp[k].x);
                b.y = fmaxf(b.y, sp[k].x);
                b.z = fminf(b.z, sp[k].y);
                b.w = fmaxf(b.w, sp[k].y);
            }
            cbb[ch] = b;
        }
    }
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
    const int w = x1 - x0, hgt = y1 - y0;
    const float* in = reinterpret_cast<const float*>(S->phiA) + S->off_cur[g];
    float* out = reinterpret_cast<float*>(S->phiB) + S->off_cur[g];
    const int wo = box_w(bo), wi = box_w(ib);
    const float delta = (float)C.delta;
    const int real = size - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int ntx = (w + 7) >> 3, ntiles = ntx * ((hgt + 3) >> 2);
    uint32_t st = 0;
    int wseed = 0;
    const bool far_ok = C.gamma_hagb <= 1.0 && C.m_hagb <= 1.0;
    // rounding margin of the FP32 search (project_warp): 8 2^-24 L, L bounding
    // every local coordinate of the contour and the pixels
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
        double dl = 0;
        int segment;
        if (staged)
            segment = project_warp(sp, P, cbb, size, j, i, ox, oy, eps_c, need, &dl, &wseed);
        else
            segment = project_to_boundary(P, size, (double)j, (double)i, &dl);
        const float lambda = (float)dl;
        if (!need) continue;
        int sid = -1;
        float interpolator = 0.f;
        if (tabled) {
            sid = stab.sector[segment];
            if (sid <= -2) interpolator = (float)stab.acc[segment];
        } else {
            for (int c = 0; c < sec.nconst && sid == -1; c++)
                if (within(sec.cs[c].left, sec.cs[c].right, real, segment)) sid = c;
            for (int c = 0; c < sec.ninterp && sid == -1; c++)
                if (within(sec.is[c].left, sec.is[c].right, real, segment)) sid = -2 - c;
            if (sid <= -2) {
                int it = 0;
                for (int kk = sec.is[-2 - sid].right; kk != segment; kk = wrap_next(kk, real)) {
                    interpolator += (float)seg[kk];
                    if (++it > size) break;
                }
            }
        }
        float weight;
        if (sid >= 0) {
            weight = (float)sec.cs[sid].weight;
        } else if (sid == -1) {
            // getGBEnergyTimesGBMobility(i, j) through the neighbour table
            weight = 1.f;
            for (int e = 0; e < nbt.n; ++e)
                if (nbt.id[e] == (int)id) {
                    weight = (float)nbt.w[e];
                    break;
                }
        } else {
            const InterpSector& s = sec.is[-2 - sid];
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


void launch_corrector_f(const NetConst& C, NetState* dS, cudaStream_t s) {
    if (C.stored || C.magnetic)
        k_corrector_f<true><<<C.N, 128, 0, s>>>(C, dS);
    else
        k_corrector_f<false><<<C.N, 128, 0, s>>>(C, dS);
}

cudaError_t batched_resample(const NetConst& C, NetState* dS, double h_old, double hn, double delta_old,
                             cudaStream_t s) {
    if (C.N > 0) k_resample<float><<<C.N, 256, 0, s>>>(C, dS, h_old, hn, delta_old);
    return cudaGetLastError();
}

// persistent grid of the large-box redistancing bin: one CTA per SM
int g_big_grid = 148;

cudaError_t batched_prepare(int tmax) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_sep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)conv_sep_smem(tmax));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_redistance_big, cudaFuncAttributeMaxDynamicSharedMemorySize, kRedistBigSmemBytes);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    g_big_grid = sms > 0 ? sms : 148;
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
    k_redistance<float><<<C.N, 256, 0, s>>>(C, dS);
    cudaError_t e = swap_phi(dS, s);
    if (e != cudaSuccess) return e;
    const int gt = 64;
    k_init_contour<float><<<(C.N + gt - 1) / gt, gt, 0, s>>>(C, dS);
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
        case 0: k_conv_sep<<<C.N, 128, conv_sep_smem(C.tmax), s>>>(C, dS); break;
        case 1: if (!C.isotropic) launch_corrector_f(C, dS, s); break;
        case 2: k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 3: k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS); break;
        case 4: k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 5: k_alloc<<<1, 1024, 0, s>>>(C, dS, 1); break;
        case 6: k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo)); break;
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
        k_conv_sep<<<C.N, 128, conv_sep_smem(C.tmax), s>>>(C, dS);
        if (!C.isotropic) launch_corrector_f(C, dS, s);
    }
    if (stages & ST_SECOND) k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_COMPARE) k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS);
    if (stages & ST_LEVELSET) k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_REDIST) {
        k_alloc<<<1, 1024, 0, s>>>(C, dS, 1);
        k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo));
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
    if ((e = cudaEventRecord(ev[1], s2)) != cudaSuccess) return e;
    k_conv_sep<<<C.N, 128, conv_sep_smem(C.tmax), s>>>(C, dS);
    if (!C.isotropic) launch_corrector_f(C, dS, s);
    if ((e = cudaStreamWaitEvent(s, ev[1], 0)) != cudaSuccess) return e;
    k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS);
    k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    k_alloc<<<1, 1024, 0, s>>>(C, dS, 1);
    // volume / energy / neighbours (contours, lists) beside redistancing (fields)
    if ((e = cudaEventRecord(ev[2], s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s2, ev[2], 0)) != cudaSuccess) return e;
    k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s2>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo));
    if ((e = cudaEventRecord(ev[3], s2)) != cudaSuccess) return e;
    launch_redistance(C, dS, s);
    if ((e = cudaStreamWaitEvent(s, ev[3], 0)) != cudaSuccess) return e;
    k_finalize<<<1, 1024, 0, s>>>(C, dS, 1);
    k_order<<<1, 1024, 0, s>>>(C, dS);  // the next step's work queue, from its boxes
    return cudaGetLastError();
}

}  // namespace gg
