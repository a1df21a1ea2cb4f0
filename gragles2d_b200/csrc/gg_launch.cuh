// Launch sequences of the stages, shared by the plain (double) and batched
// (float) translation units.  Included once per TU with GG_REAL and
// GG_FORM defined.
#pragma once

#include <cuda_runtime.h>

#include "../../include/gg_step.h"
#include "gg_device.cuh"

namespace gg {

// Stage selectors for launch_stages().
enum : int {
    ST_CONV = 1 << 0,
    ST_SECOND = 1 << 1,
    ST_COMPARE = 1 << 2,
    ST_LEVELSET = 1 << 3,
    ST_REDIST = 1 << 4,  // alloc + neighbours + redistancing + end of step
    ST_ALL = 0x1f
};

struct LaunchCfg {
    int conv_threads;
    int compare_threads;
    int redist_threads;
    int grain_threads;  // one-thread-per-grain kernels
};

// Declared per form; defined in gg_plain.cu / gg_batched.cu.
cudaError_t plain_stages(const NetConst& C, NetState* dS, int stages, cudaStream_t s, const LaunchCfg& cfg);
cudaError_t plain_init(const NetConst& C, NetState* dS, const int32_t* d_ids, cudaStream_t s);
// distance initialisation from the loaded polygons (contour input)
cudaError_t plain_init_polygon(const NetConst& C, NetState* dS, cudaStream_t s);
cudaError_t plain_corrector(const NetConst& C, NetState* dS, cudaStream_t s);
cudaError_t batched_stages(const NetConst& C, NetState* dS, int stages, cudaStream_t s, const LaunchCfg& cfg);
// The whole batched step for graph capture on s, with the independent stages
// (second-order lists beside convolution + corrector, volume / energy /
// neighbours beside redistancing) forked onto s2 through the events ev[0..3].
cudaError_t batched_step_graph(const NetConst& C, NetState* dS, cudaStream_t s, cudaStream_t s2, cudaEvent_t* ev,
                               const LaunchCfg& cfg);
size_t conv_sep_smem(int tmax, int edge);
cudaError_t batched_prepare(int tmax);
cudaError_t batched_init(const NetConst& C, NetState* dS, const int32_t* d_ids, cudaStream_t s);
cudaError_t batched_init_polygon(const NetConst& C, NetState* dS, cudaStream_t s);
// rebuilds the batched form's work queue (NetState::order) from the current boxes
cudaError_t batched_order(const NetConst& C, NetState* dS, cudaStream_t s);
// the sectors of the next corrector from the previous roles (after set-up,
// grid coarsening or new neighbour lists); the step builds them itself
cudaError_t batched_sectors(const NetConst& C, NetState* dS, cudaStream_t s);
size_t batched_sector_pack_bytes();
cudaError_t finalize_only(const NetConst& C, NetState* dS, int rotate, cudaStream_t s);
// Every grain's gg_grain_stats into out[0 .. N-1] (device memory).
cudaError_t pack_stats(const NetConst& C, const NetState* dS, gg_grain_stats* out, cudaStream_t s);
// Grid coarsening: every grain's field resampled onto the coarser grid.
cudaError_t plain_resample(const NetConst& C, NetState* dS, double h_old, double hn, double delta_old,
                           cudaStream_t s);
cudaError_t batched_resample(const NetConst& C, NetState* dS, double h_old, double hn, double delta_old,
                             cudaStream_t s);
cudaError_t swap_phi(NetState* dS, cudaStream_t s);
// Counts and scans the bins (stream-ordered; *B.total set on the device).
cudaError_t neighbour_bins_count(const NetConst& C, NetState* dS, const NeighbourBins& B, cudaStream_t s);
// Fills the bins (B.items sized for the total) and runs the search.
cudaError_t find_neighbors_launch(const NetConst& C, NetState* dS, const NeighbourBins& B, cudaStream_t s);
cudaError_t traffic_launch(const NetConst& C, NetState* dS, cudaStream_t s);
// One launch of a single stage kernel (index 0..8 as in GG_NSTAGES order).
cudaError_t plain_stage_kernel(const NetConst& C, NetState* dS, int which, cudaStream_t s, const LaunchCfg& cfg);
cudaError_t batched_stage_kernel(const NetConst& C, NetState* dS, int which, cudaStream_t s, const LaunchCfg& cfg);

}  // namespace gg
