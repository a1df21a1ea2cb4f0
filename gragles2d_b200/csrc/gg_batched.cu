// Batched form: FP32 distance fields and convolution (FP64 contour areas,
// energies and lengths), every stage over all grains, captured per step as
// one CUDA graph by the host.
#include "gg_corrector.cuh"
#include "gg_kernels.cuh"
#include "gg_launch.cuh"

namespace gg {

constexpr int kSepSmemMaxN = 110;  // 2 n^2 + n floats of shared memory

// Gaussian convolution as a separable circular convolution in real space:
// out = K X K^T with K[r][r'] = k_n[(r - r') mod n], where k_n is the real
// kernel whose DFT is the reference's Gaussian multiplier
// (src/box.cpp:674-687, G(i2, j2) = g(i2) g(j2) / n^2).  One CTA per grain;
// the box and the intermediate stay in shared memory when n <= 110.
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
    switch (which) {
        case 0: k_conv_sep<<<C.N, cfg.conv_threads, conv_sep_smem(C.tmax), s>>>(C, dS); break;
        case 1: if (!C.isotropic) k_corrector<float><<<C.N, 256, 0, s>>>(C, dS); break;
        case 2: k_second_order<<<gblocks, gt, 0, s>>>(C, dS); break;
        case 3: k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS); break;
        case 4: k_levelset<float><<<gblocks, gt, 0, s>>>(C, dS); break;
        case 5: k_alloc<<<1, 1024, 0, s>>>(C, dS, 1); break;
        case 6: k_neighbours<float><<<gblocks, gt, 0, s>>>(C, dS); break;
        case 7: k_redistance<float><<<C.N, cfg.redist_threads, 0, s>>>(C, dS); break;
        default: k_finalize<<<1, 1024, 0, s>>>(C, dS, 1); break;
    }
    return cudaGetLastError();
}

cudaError_t batched_stages(const NetConst& C, NetState* dS, int stages, cudaStream_t s, const LaunchCfg& cfg) {
    if (C.N <= 0) return cudaSuccess;
    const int gt = cfg.grain_threads;
    const int gblocks = (C.N + gt - 1) / gt;
    if (stages & ST_CONV) {
        k_conv_sep<<<C.N, cfg.conv_threads, conv_sep_smem(C.tmax), s>>>(C, dS);
        if (!C.isotropic) k_corrector<float><<<C.N, 256, 0, s>>>(C, dS);
    }
    if (stages & ST_SECOND) k_second_order<<<gblocks, gt, 0, s>>>(C, dS);
    if (stages & ST_COMPARE) k_compare<float><<<C.N, cfg.compare_threads, 0, s>>>(C, dS);
    if (stages & ST_LEVELSET) k_levelset<float><<<gblocks, gt, 0, s>>>(C, dS);
    if (stages & ST_REDIST) {
        k_alloc<<<1, 1024, 0, s>>>(C, dS, 1);
        k_neighbours<float><<<gblocks, gt, 0, s>>>(C, dS);
        k_redistance<float><<<C.N, cfg.redist_threads, 0, s>>>(C, dS);
        k_finalize<<<1, 1024, 0, s>>>(C, dS, 1);
    }
    return cudaGetLastError();
}

}  // namespace gg
