// Batched form: FP32 distance fields and convolution (FP64 contour areas,
// energies and lengths), every stage over all grains, captured per step as
// one CUDA graph by the host.
#include "gg_corrector.cuh"
#include "gg_kernels.cuh"
#include "gg_launch.cuh"
#include "gg_warp.cuh"

namespace gg {

constexpr int kSepSmemMaxN = 64;  // box + intermediate in shared memory up to this edge
constexpr int kSepStrip = 4;       // outputs per thread along the convolution axis

// Gaussian convolution as a separable circular convolution in real space:
// out = K X K^T with K[r][r'] = k_n[(r - r') mod n], where k_n is the real
// kernel whose DFT is the reference's Gaussian multiplier
// (src/box.cpp:674-687, G(i2, j2) = g(i2) g(j2) / n^2).  One CTA per grain.
// The kernel is laid out once as kx[j] = k_n[(j - (n-1)) mod n], j < 2n-1
// (zero-padded), so output c of a row is sum_c' X[c'] kx[c - c' + n - 1]:
// each thread accumulates a strip of 4 consecutive outputs while a 4-entry
// register window slides down kx (one shared-memory load per 4 FMAs).
__device__ __forceinline__ void sep_pass_rows(const float* __restrict__ X, float* __restrict__ T,
                                              const float* __restrict__ kx, int n) {
    const int nb = (n + kSepStrip - 1) / kSepStrip;
    for (int t = threadIdx.x; t < n * nb; t += blockDim.x) {
        const int r = t / nb, c0 = (t - r * nb) * kSepStrip;
        const float* xr = X + r * n;
        int base = c0 + n - 1;  // kx index of (c0 - c') at c' = 0
        float w0 = kx[base], w1 = kx[base + 1], w2 = kx[base + 2], w3 = kx[base + 3];
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll 4
        for (int cp = 0; cp < n; ++cp) {
            const float x = xr[cp];
            a0 = fmaf(x, w0, a0);
            a1 = fmaf(x, w1, a1);
            a2 = fmaf(x, w2, a2);
            a3 = fmaf(x, w3, a3);
            --base;
            w3 = w2;
            w2 = w1;
            w1 = w0;
            w0 = kx[base];
        }
        float* tr = T + r * n + c0;
        tr[0] = a0;
        if (c0 + 1 < n) tr[1] = a1;
        if (c0 + 2 < n) tr[2] = a2;
        if (c0 + 3 < n) tr[3] = a3;
    }
}

__device__ __forceinline__ void sep_pass_cols(const float* __restrict__ T, float* __restrict__ out,
                                              const float* __restrict__ kx, int n) {
    const int nb = (n + kSepStrip - 1) / kSepStrip;
    for (int t = threadIdx.x; t < n * nb; t += blockDim.x) {
        const int rb = t / n, c = t - rb * n, r0 = rb * kSepStrip;
        int base = r0 + n - 1;
        float w0 = kx[base], w1 = kx[base + 1], w2 = kx[base + 2], w3 = kx[base + 3];
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll 4
        for (int rp = 0; rp < n; ++rp) {
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
    const int g = blockIdx.x + 1;
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
    const int nn2 = n * n;
    const bool fits = n <= kSepSmemMaxN;
    float* kx = sm + 1;  // sm[0] is the guard entry kx[-1]
    const int kl = kx_len(n);
    float* X = sm + 1 + kl;
    float* T = fits ? X + nn2 : reinterpret_cast<float*>(S->spec) + S->soff_cur[g];
    for (int j = threadIdx.x; j < kl; j += blockDim.x) {
        int m = j - (n - 1);
        m %= n;
        if (m < 0) m += n;
        kx[j] = j < 2 * n - 1 ? kg[m] : 0.f;
    }
    if (threadIdx.x == 0) sm[0] = 0.f;
    if (fits)
        for (int i = threadIdx.x; i < nn2; i += blockDim.x) X[i] = in[i];
    __syncthreads();
    sep_pass_rows(fits ? X : in, T, kx, n);
    __syncthreads();
    sep_pass_cols(T, out, kx, n);
}

size_t conv_sep_smem(int tmax) {
    const int n = tmax < kSepSmemMaxN ? tmax : kSepSmemMaxN;
    return sizeof(float) * (size_t)(2 * n * n + 2 * kSepSmemMaxN + kSepStrip + 2);
}

// Batched-form corrector: same sectors and weights as k_corrector, with the
// previous contour staged in shared memory (FP32 coordinates), junction
// weights computed one thread per junction, and the per-pixel projection in
// FP32.
constexpr int kCorrMaxPts = 1024;
constexpr int kCorrMaxPix = 4096;  // compacted pixel list (boxes up to 64 x 64)

constexpr int kChunk = 8;  // contour points per bounding box of the nearest-vertex search

// projectToGrainBondary (src/grainBoundary.cpp:365-447) in FP32 over the
// staged contour.  The nearest-vertex scan skips every run of 8 consecutive
// points whose bounding box is farther than the best point found so far
// (runs are visited in index order, so ties still go to the first point).
__device__ __forceinline__ int project_f(const float2* P, const float4* cbb, int asize, float px, float py,
                                         float* out_lambda) {
    float minDist = 3.0e38f;
    int nearest = -1;
    const int npts = asize - 1;
    const int nch = (npts + kChunk - 1) / kChunk;
    for (int ch = 0; ch < nch; ++ch) {
        const float4 b = cbb[ch];
        const float bx = fmaxf(fmaxf(b.x - px, px - b.y), 0.f);
        const float by = fmaxf(fmaxf(b.z - py, py - b.w), 0.f);
        if (bx * bx + by * by > minDist) continue;
        const int k1 = min(ch * kChunk + kChunk, npts);
        for (int k = ch * kChunk; k < k1; k++) {
            const float dx = px - P[k].x, dy = py - P[k].y;
            const float d = dx * dx + dy * dy;
            if (d < minDist) {
                nearest = k;
                minDist = d;
            }
        }
    }
    if (nearest < 0) return 0;
    float lam_out = 0.f;
    int seg = nearest;
    minDist = 1e30f;
    {
        const int next = nearest + 1;
        const float ux = P[next].x - P[nearest].x, uy = P[next].y - P[nearest].y;
        float lambda = ((px - P[nearest].x) * ux + (py - P[nearest].y) * uy) / (ux * ux + uy * uy);
        float d;
        if (lambda < 0) {
            const float dx = px - P[nearest].x, dy = py - P[nearest].y;
            d = dx * dx + dy * dy;
        } else if (lambda > 1) {
            const float dx = P[next].x - px, dy = P[next].y - py;
            d = dx * dx + dy * dy;
        } else {
            const float dx = px - (P[nearest].x + ux * lambda), dy = py - (P[nearest].y + uy * lambda);
            d = dx * dx + dy * dy;
        }
        if (d < minDist) {
            seg = nearest;
            minDist = d;
            lam_out = lambda;
        }
    }
    int nb = nearest == 0 ? asize - 1 : nearest;
    {
        const int prev = nb - 1;
        const float ux = P[nb].x - P[prev].x, uy = P[nb].y - P[prev].y;
        float lambda = ((px - P[prev].x) * ux + (py - P[prev].y) * uy) / (ux * ux + uy * uy);
        float d;
        if (lambda < 0) {
            const float dx = px - P[prev].x, dy = py - P[prev].y;
            d = dx * dx + dy * dy;
        } else if (lambda > 1) {
            const float dx = P[nb].x - px, dy = P[nb].y - py;
            d = dx * dx + dy * dy;
        } else {
            const float dx = px - (P[prev].x + ux * lambda), dy = py - (P[prev].y + uy * lambda);
            d = dx * dx + dy * dy;
        }
        if (d < minDist) {
            seg = prev;
            lam_out = lambda;
        }
    }
    *out_lambda = fminf(fmaxf(lam_out, 0.f), 1.f);
    return seg;
}

__global__ void __launch_bounds__(128, 6) k_corrector_f(NetConst C, NetState* S) {
    const int g = blockIdx.x + 1;
    if (g > C.N || C.state[g] != G_EXISTS || C.regular[g] == 0 || S->loop == 0 || halted(S)) return;
    __shared__ SectorSet sec;
    __shared__ float2 sp[kCorrMaxPts];
    __shared__ double jw[64];
    __shared__ uint32_t s_st;
    __shared__ double s_per;
    __shared__ NbTable nbt;
    __shared__ float4 cbb[kCorrMaxPts / kChunk];
    __shared__ unsigned short plist[kCorrMaxPix];
    __shared__ int pcount;
    __shared__ double s_seg[kSegShared];
    __shared__ SegTable stab;
    const CPoint* P = S->contPrev + S->coff_prev[g];
    const int size = S->cn_prev[g];
    if (size < 2) return;
    double* seg = size - 1 <= kSegShared ? s_seg : S->segPrev + S->coff_prev[g];
    const Box ib = S->box_prev[g];
    const uint32_t* idl = S->idPrev + S->off_prev[g];
    const bool staged = size <= kCorrMaxPts;
    if (staged)
        for (int k = threadIdx.x; k < size; k += blockDim.x) sp[k] = make_float2((float)P[k].x, (float)P[k].y);
    if (threadIdx.x == 0) pcount = 0;
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
    prepare_sectors(C, S, g, P, size, seg, sec, jw, &s_st, &s_per, nbt);
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
    const int cnt = w * (y1 - y0);
    const float* in = reinterpret_cast<const float*>(S->phiA) + S->off_cur[g];
    float* out = reinterpret_cast<float*>(S->phiB) + S->off_cur[g];
    const int wo = box_w(bo);
    const float delta = (float)C.delta;
    const int real = size - 1;
    uint32_t st = 0;
    // pixels at or below -delta are set to -delta; the others are compacted
    // into a list so every lane of a warp projects a pixel
    const bool compact = cnt <= kCorrMaxPix;
    for (int p0 = 0; p0 < cnt; p0 += blockDim.x) {
        const int p = p0 + threadIdx.x;
        bool active = false;
        if (p < cnt) {
            const int i = y0 + p / w, j = x0 + p % w;
            const int k = (i - bo.y0) * wo + (j - bo.x0);
            active = in[k] > -delta;
            if (!active) out[k] = -delta;
        }
        if (compact) {
            const int lane = threadIdx.x & 31;
            const unsigned bal = __ballot_sync(0xffffffffu, active);
            int base = 0;
            if (lane == 0 && bal) base = atomicAdd(&pcount, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (active) plist[base + __popc(bal & ((1u << lane) - 1u))] = (unsigned short)p;
        }
    }
    __syncthreads();
    const int total = compact ? pcount : cnt;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const int p = compact ? (int)plist[q] : q;
        const int i = y0 + p / w, j = x0 + p % w;
        const int k = (i - bo.y0) * wo + (j - bo.x0);
        const float val = in[k];
        if (!compact && !(val > -delta)) continue;
        float lambda = 0.f;
        int segment;
        if (staged) {
            segment = project_f(sp, cbb, size, (float)j, (float)i, &lambda);
        } else {
            double dl = 0;
            segment = project_to_boundary(P, size, (double)j, (double)i, &dl);
            lambda = (float)dl;
        }
        int sid = -1;
        double interpolator = 0;
        if (tabled) {
            sid = stab.sector[segment];
            if (sid <= -2) interpolator = stab.acc[segment];
        } else {
            for (int q = 0; q < sec.nconst && sid == -1; q++)
                if (within(sec.cs[q].left, sec.cs[q].right, real, segment)) sid = q;
            for (int q = 0; q < sec.ninterp && sid == -1; q++)
                if (within(sec.is[q].left, sec.is[q].right, real, segment)) sid = -2 - q;
            if (sid <= -2) {
                int it = 0;
                for (int kk = sec.is[-2 - sid].right; kk != segment; kk = wrap_next(kk, real)) {
                    interpolator += seg[kk];
                    if (++it > size) break;
                }
            }
        }
        double weight;
        if (sid >= 0) {
            weight = sec.cs[sid].weight;
        } else if (sid == -1) {
            weight = table_weight_at(nbt, idl, ib, i, j, &st);
        } else {
            const InterpSector& s = sec.is[-2 - sid];
            const int kn = wrap_next(segment, real);
            const double ax = (P[kn].x - P[segment].x) * lambda, ay = (P[kn].y - P[segment].y) * lambda;
            interpolator += sqrt(ax * ax + ay * ay);
            interpolator /= s.length;
            interpolator = fmin(fmax(interpolator, 0.0), 1.0);
            if (s.lb >= 0 && s.rb >= 0) {
                const double isr = C.isr;
                const double quot = (s.length > 2 * isr ? 2 * isr : s.length);
                const double amplitude =
                    (s.boundary_w - (s.left_w + s.right_w) / 2) / (2 * isr) * quot + (s.left_w + s.right_w) / 2;
                const double a0 = 2 * s.right_w, a1 = -4 * amplitude, a2 = 2 * s.left_w;
                const double A = a0 + a1 + a2, B = -(a0 * 1.5 + a1 + a2 * 0.5), Cc = a0 * 0.5;
                weight = A * interpolator * interpolator + B * interpolator + Cc;
            } else {
                weight = interpolator * s.left_w + (1 - interpolator) * s.right_w;
            }
        }
        out[k] = val + (out[k] - val) * (float)weight;
    }
    if (st) set_status(S, st);
}


cudaError_t batched_prepare(int tmax) {
    return cudaFuncSetAttribute(k_conv_sep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)conv_sep_smem(tmax));
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

cudaError_t batched_stage_kernel(const NetConst& C, NetState* dS, int which, cudaStream_t s, const LaunchCfg& cfg) {
    const int gt = cfg.grain_threads;
    const int gblocks = (C.N + gt - 1) / gt;
    const int wblocks = (C.N + kGrainsPerBlock - 1) / kGrainsPerBlock;
    (void)gblocks;
    switch (which) {
        case 0: k_conv_sep<<<C.N, 128, conv_sep_smem(C.tmax), s>>>(C, dS); break;
        case 1: if (!C.isotropic) k_corrector_f<<<C.N, 128, 0, s>>>(C, dS); break;
        case 2: k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 3: k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS); break;
        case 4: k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 5: k_alloc<<<1, 1024, 0, s>>>(C, dS, 1); break;
        case 6: k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo)); break;
        case 7: k_redistance_s<float><<<C.N, kRedistThreads, kRedistSmemBytes, s>>>(C, dS); break;
        default: k_finalize<<<1, 1024, 0, s>>>(C, dS, 1); break;
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
        if (!C.isotropic) k_corrector_f<<<C.N, 128, 0, s>>>(C, dS);
    }
    if (stages & ST_SECOND) k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_COMPARE) k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS);
    if (stages & ST_LEVELSET) k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_REDIST) {
        k_alloc<<<1, 1024, 0, s>>>(C, dS, 1);
        k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo));
        k_redistance_s<float><<<C.N, kRedistThreads, kRedistSmemBytes, s>>>(C, dS);
        k_finalize<<<1, 1024, 0, s>>>(C, dS, 1);
    }
    return cudaGetLastError();
}

}  // namespace gg
