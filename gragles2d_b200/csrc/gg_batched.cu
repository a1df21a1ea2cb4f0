// Batched form: FP32 distance fields and convolution (FP64 contour areas,
// energies and lengths), every stage over all grains, captured per step as
// one CUDA graph by the host.
#include "gg_corrector.cuh"
#include "gg_kernels.cuh"
#include "gg_launch.cuh"
#include "gg_warp.cuh"

namespace gg {

constexpr int kSepSmemMaxN = 64;  // 2 n^2 + n floats of shared memory (larger boxes stage in global scratch)

// Gaussian convolution as a separable circular convolution in real space:
// out = K X K^T with K[r][r'] = k_n[(r - r') mod n], where k_n is the real
// kernel whose DFT is the reference's Gaussian multiplier
// (src/box.cpp:674-687, G(i2, j2) = g(i2) g(j2) / n^2).  One CTA per grain;
// the box and the intermediate stay in shared memory when n <= 64.
__global__ void __launch_bounds__(256) k_conv_sep(NetConst C, NetState* S) {
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
    float* kk = sm;
    float* X = sm + n;
    float* T = fits ? X + nn2 : reinterpret_cast<float*>(S->spec) + S->soff_cur[g];
    const float* Xr = fits ? X : in;
    for (int i = threadIdx.x; i < n; i += blockDim.x) kk[i] = kg[i];
    if (fits)
        for (int i = threadIdx.x; i < nn2; i += blockDim.x) X[i] = in[i];
    __syncthreads();
    for (int idx = threadIdx.x; idx < nn2; idx += blockDim.x) {
        const int r = idx / n, c = idx - r * n;
        const float* xr = Xr + r * n;
        float acc = 0.f;
        int m = c;  // (c - c') mod n, c' = 0
        for (int cp = 0; cp < n; ++cp) {
            acc = fmaf(xr[cp], kk[m], acc);
            m = (m == 0) ? n - 1 : m - 1;
        }
        T[idx] = acc;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nn2; idx += blockDim.x) {
        const int r = idx / n, c = idx - r * n;
        float acc = 0.f;
        int m = r;
        for (int rp = 0; rp < n; ++rp) {
            acc = fmaf(kk[m], T[rp * n + c], acc);
            m = (m == 0) ? n - 1 : m - 1;
        }
        out[idx] = acc;
    }
}

// Batched-form corrector: same sectors and weights as k_corrector, with the
// previous contour staged in shared memory (FP32 coordinates), junction
// weights computed one thread per junction, and the per-pixel projection in
// FP32.
constexpr int kCorrMaxPts = 1024;

__device__ __forceinline__ int project_f(const float2* P, int asize, float px, float py, float* out_lambda) {
    float minDist = 1e30f;
    int nearest = -1;
    for (int k = 0; k < asize - 1; k++) {
        const float dx = px - P[k].x, dy = py - P[k].y;
        const float d = dx * dx + dy * dy;
        if (d < minDist) {
            nearest = k;
            minDist = d;
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
    const CPoint* P = S->contPrev + S->coff_prev[g];
    const int size = S->cn_prev[g];
    if (size < 2) return;
    double* seg = S->segPrev + S->coff_prev[g];
    const Box ib = S->box_prev[g];
    const uint32_t* idl = S->idPrev + S->off_prev[g];
    const bool staged = size <= kCorrMaxPts;
    if (staged)
        for (int k = threadIdx.x; k < size; k += blockDim.x) sp[k] = make_float2((float)P[k].x, (float)P[k].y);
    prepare_sectors(C, S, g, P, size, seg, sec, jw, &s_st, &s_per, nbt);
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
    for (int p = threadIdx.x; p < cnt; p += blockDim.x) {
        const int i = y0 + p / w, j = x0 + p % w;
        const int k = (i - bo.y0) * wo + (j - bo.x0);
        const float val = in[k];
        if (!(val > -delta)) {
            out[k] = -delta;
            continue;
        }
        float lambda = 0.f;
        int segment;
        if (staged) {
            segment = project_f(sp, size, (float)j, (float)i, &lambda);
        } else {
            double dl = 0;
            segment = project_to_boundary(P, size, (double)j, (double)i, &dl);
            lambda = (float)dl;
        }
        double weight = 0;
        bool found = false;
        for (int q = 0; q < sec.nconst && !found; q++)
            if (within(sec.cs[q].left, sec.cs[q].right, real, segment)) {
                weight = sec.cs[q].weight;
                found = true;
            }
        for (int q = 0; q < sec.ninterp && !found; q++) {
            const InterpSector& s = sec.is[q];
            if (!within(s.left, s.right, real, segment)) continue;
            double interpolator = 0;
            int kk = s.right, it = 0;
            for (; kk != segment; kk = (kk + 1 + real) % real) {
                interpolator += seg[kk];
                if (++it > size) break;
            }
            const int kn = (kk + 1 + real) % real;
            const double ax = (P[kn].x - P[kk].x) * lambda, ay = (P[kn].y - P[kk].y) * lambda;
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
            found = true;
        }
        if (!found) weight = table_weight_at(nbt, idl, ib, i, j, &st);
        out[k] = val + (out[k] - val) * (float)weight;
    }
    if (st) set_status(S, st);
}

size_t conv_sep_smem(int tmax) {
    const int n = tmax < kSepSmemMaxN ? tmax : kSepSmemMaxN;
    return sizeof(float) * (size_t)(2 * n * n + n);
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
        case 0: k_conv_sep<<<C.N, cfg.conv_threads, conv_sep_smem(C.tmax), s>>>(C, dS); break;
        case 1: if (!C.isotropic) k_corrector_f<<<C.N, 128, 0, s>>>(C, dS); break;
        case 2: k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 3: k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS); break;
        case 4: k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 5: k_alloc<<<1, 1024, 0, s>>>(C, dS, 1); break;
        case 6: k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo)); break;
        case 7: k_redistance<float><<<C.N, cfg.redist_threads, 0, s>>>(C, dS); break;
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
        k_conv_sep<<<C.N, cfg.conv_threads, conv_sep_smem(C.tmax), s>>>(C, dS);
        if (!C.isotropic) k_corrector_f<<<C.N, 128, 0, s>>>(C, dS);
    }
    if (stages & ST_SECOND) k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_COMPARE) k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS);
    if (stages & ST_LEVELSET) k_levelset_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_REDIST) {
        k_alloc<<<1, 1024, 0, s>>>(C, dS, 1);
        k_neighbours_w<float><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo));
        k_redistance<float><<<C.N, cfg.redist_threads, 0, s>>>(C, dS);
        k_finalize<<<1, 1024, 0, s>>>(C, dS, 1);
    }
    return cudaGetLastError();
}

}  // namespace gg
