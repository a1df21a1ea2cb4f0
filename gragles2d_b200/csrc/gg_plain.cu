// Plain form: FP64 kernels compiled without FMA contraction (--fmad=false),
// so every sum, product and quotient rounds exactly as the reference's
// host arithmetic does.
#include "gg_corrector.cuh"
#include "gg_kernels.cuh"
#include "gg_launch.cuh"
#include "gg_tangent.cuh"
#include "gg_warp.cuh"

namespace gg {

__global__ void k_swap_phi(NetState* S) {
    void* t = S->phiA;
    S->phiA = S->phiB;
    S->phiB = t;
    t = S->dphiA;
    S->dphiA = S->dphiB;
    S->dphiB = t;
}

cudaError_t swap_phi(NetState* dS, cudaStream_t s) {
    k_swap_phi<<<1, 1, 0, s>>>(dS);
    return cudaGetLastError();
}

cudaError_t plain_resample(const NetConst& C, NetState* dS, double h_old, double hn, double delta_old,
                           cudaStream_t s) {
    if (C.N > 0) k_resample<double><<<C.N, 256, 0, s>>>(C, dS, h_old, hn, delta_old);
    return cudaGetLastError();
}

// The per-grain statistics of gg_read_grain_stats, gathered into one array.
__global__ void k_pack_stats(NetConst C, const NetState* S, gg_grain_stats* out) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (g > C.N) return;
    gg_grain_stats s;
    s.id = g;
    s.state = C.state[g];
    s.motion_regular = C.regular[g];
    s.intersects_boundary = C.inter_bnd[g];
    s.n_neighbours = C.nb_n[g];
    s.contour_points = S->cn_prev[g];
    const Box b = S->box_cur[g];
    s.box[0] = b.x0;
    s.box[1] = b.x1;
    s.box[2] = b.y0;
    s.box[3] = b.y1;
    s.area = C.volume[g];
    s.energy = C.energy[g];
    s.perimeter = C.perimeter[g];
    s.mean_da = C.meanda[g];
    out[g - 1] = s;
}

cudaError_t pack_stats(const NetConst& C, const NetState* dS, gg_grain_stats* out, cudaStream_t s) {
    if (C.N > 0) k_pack_stats<<<(C.N + 255) / 256, 256, 0, s>>>(C, dS, out);
    return cudaGetLastError();
}

cudaError_t finalize_only(const NetConst& C, NetState* dS, int rotate, cudaStream_t s) {
    k_finalize<<<1, 1024, 0, s>>>(C, dS, rotate);
    return cudaGetLastError();
}

cudaError_t neighbour_bins_count(const NetConst& C, NetState* dS, const NeighbourBins& B, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(B.count, 0, sizeof(int) * (size_t)B.nc * B.nc, s);
    if (e != cudaSuccess) return e;
    if (C.N > 0) k_bin_grains<<<(C.N + 255) / 256, 256, 0, s>>>(C, dS, B, 0);
    k_bin_scan<<<1, 1024, 0, s>>>(B);
    return cudaGetLastError();
}

cudaError_t find_neighbors_launch(const NetConst& C, NetState* dS, const NeighbourBins& B, cudaStream_t s) {
    if (C.N <= 0) return cudaSuccess;
    k_bin_grains<<<(C.N + 255) / 256, 256, 0, s>>>(C, dS, B, 1);
    k_find_neighbors<<<(C.N + kFindWarps - 1) / kFindWarps, 32 * kFindWarps, 0, s>>>(C, dS, B);
    return cudaGetLastError();
}

cudaError_t plain_init(const NetConst& C, NetState* dS, const int32_t* d_ids, cudaStream_t s) {
    if (C.N <= 0) return cudaSuccess;
    k_init_phi<double><<<C.N, 256, 0, s>>>(C, dS, d_ids);
    k_redistance<double><<<C.N, 256, 0, s>>>(C, dS);
    k_swap_phi<<<1, 1, 0, s>>>(dS);
    const int gt = 64;
    k_init_contour<double><<<(C.N + gt - 1) / gt, gt, 0, s>>>(C, dS);
    return cudaGetLastError();
}

cudaError_t plain_init_polygon(const NetConst& C, NetState* dS, cudaStream_t s) {
    if (C.N <= 0) return cudaSuccess;
    k_polygon_phi<double><<<C.N, 256, 0, s>>>(C, dS);
    return cudaGetLastError();
}

cudaError_t traffic_launch(const NetConst& C, NetState* dS, cudaStream_t s) {
    const int gt = 128;
    k_traffic<<<(C.N + gt - 1) / gt, gt, 0, s>>>(C, dS);
    return cudaGetLastError();
}

cudaError_t plain_stage_kernel(const NetConst& C, NetState* dS, int which, cudaStream_t s, const LaunchCfg& cfg) {
    const int gt = cfg.grain_threads;
    const int gblocks = (C.N + gt - 1) / gt;
    const int wblocks = (C.N + kGrainsPerBlock - 1) / kGrainsPerBlock;
    (void)gblocks;
    switch (which) {
        case 0: k_conv_dft<double><<<C.N, cfg.conv_threads, 0, s>>>(C, dS); break;
        case 1: if (!C.isotropic) k_corrector<double><<<C.N, 128, 0, s>>>(C, dS); break;
        case 2: k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 3: k_compare<double><<<C.N, cfg.compare_threads, 0, s>>>(C, dS); break;
        case 4: k_levelset_w<double><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS); break;
        case 5: k_alloc<<<1, 1024, 0, s>>>(C, dS, 2); break;
        case 6: k_neighbours_w<double><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo)); break;
        case 7: k_redistance_s<double><<<C.N, kRedistThreads, kRedistSmemBytes, s>>>(C, dS); break;
        default: k_finalize<<<1, 1024, 0, s>>>(C, dS, 1); break;
    }
    return cudaGetLastError();
}

cudaError_t plain_corrector(const NetConst& C, NetState* dS, cudaStream_t s) {
    k_corrector<double><<<C.N, 128, 0, s>>>(C, dS);
    return cudaGetLastError();
}

cudaError_t plain_stages(const NetConst& C, NetState* dS, int stages, cudaStream_t s, const LaunchCfg& cfg) {
    if (C.N <= 0) return cudaSuccess;
    const int gt = cfg.grain_threads;
    const int gblocks = (C.N + gt - 1) / gt;
    const int wblocks = (C.N + kGrainsPerBlock - 1) / kGrainsPerBlock;
    (void)gblocks;
    // tangent mode (C.dvol set): the tangent kernels of gg_tangent.cuh follow
    // their stages; the corrector's tangent reads the uncorrected convolution,
    // so it runs first
    const bool tan = C.dvol != nullptr;
    if (stages & ST_CONV) {
        k_conv_dft<double><<<C.N, cfg.conv_threads, 0, s>>>(C, dS);
        if (tan)
            for (int tk = 0; tk < kNP; ++tk) k_conv_dft<double><<<C.N, cfg.conv_threads, 0, s>>>(C, dS, tk);
        if (!C.isotropic) {
            if (tan) k_corrector_t<<<C.N, 128, 0, s>>>(C, dS);
            cudaError_t e = plain_corrector(C, dS, s);
            if (e != cudaSuccess) return e;
        }
    }
    if (stages & ST_SECOND) k_second_order_w<<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
    if (stages & ST_COMPARE) {
        k_compare<double><<<C.N, cfg.compare_threads, 0, s>>>(C, dS);
        if (tan) k_compare_t<<<C.N, 256, 0, s>>>(C, dS);
    }
    if (stages & ST_LEVELSET) {
        k_levelset_w<double><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS);
        if (tan) k_area_t<<<(C.N + 127) / 128, 128, 0, s>>>(C, dS);
    }
    if (stages & ST_REDIST) {
        k_alloc<<<1, 1024, 0, s>>>(C, dS, 2);
        k_neighbours_w<double><<<wblocks, 32 * kGrainsPerBlock, 0, s>>>(C, dS, reinterpret_cast<PointInfo*>(C.ptinfo));
        if (tan)
            k_redistance_t<<<C.N, 64, 0, s>>>(C, dS);
        else
            k_redistance_s<double><<<C.N, kRedistThreads, kRedistSmemBytes, s>>>(C, dS);
        k_finalize<<<1, 1024, 0, s>>>(C, dS, 1);
    }
    return cudaGetLastError();
}

}  // namespace gg
