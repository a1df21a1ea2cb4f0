// Host side of the C ABI (include/gg_step.h): settings, voxelized input,
// host-computed tables, device arenas, the stage sequence of the reference
// time loop and the state dump.  Host arithmetic that the FP64 form must
// reproduce (dt, h, delta, Gaussian multipliers, twiddles) is written with
// the reference's expressions and compiled without FMA contraction.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <system_error>
#include <thread>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/gg_step.h"
#include "gg_device.cuh"
#include "gg_launch.cuh"

using namespace gg;

namespace {

constexpr double kPiH = 3.14159265358979323846;  // PI, src/ggLS.h:26

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// Page-locked host buffers kept by the process for its next contexts, as the
// device memory pool keeps device memory: page-locking costs milliseconds, so
// a context takes the smallest free buffer that is large enough (else
// allocates one, portable to every device) and gives it back when destroyed.
std::mutex g_pinned_mutex;
std::vector<DevBuf> g_pinned_free;

cudaError_t pinned_take(void** out, size_t bytes) {
    {
        std::lock_guard<std::mutex> lock(g_pinned_mutex);
        int best = -1;
        for (int i = 0; i < (int)g_pinned_free.size(); ++i)
            if (g_pinned_free[i].bytes >= bytes && (best < 0 || g_pinned_free[i].bytes < g_pinned_free[best].bytes))
                best = i;
        if (best >= 0) {
            *out = g_pinned_free[best].p;
            g_pinned_free.erase(g_pinned_free.begin() + best);
            return cudaSuccess;
        }
    }
    return cudaHostAlloc(out, bytes, cudaHostAllocPortable);
}

void pinned_give(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    g_pinned_free.push_back(DevBuf{p, bytes});
}

}  // namespace

struct gg_ctx {
    gg_params P{};
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;

    // derived settings (grainhdl::setSimulationParameter, src/grainhdl.cpp:56-136)
    int N = 0, nn = 0, m = 0, b = 0, ppg = 0;
    double h = 0, dt = 0, delta = 0, ds = 0;
    bool loaded = false, initialised = false;
    bool tangents = false;  // carry d phi / d p_k (plain form; set before distance initialisation)
    double energy_delta_max = 0;  // grainhdl::m_Energy_deltaMAX (time-step bound of the driving forces)
    int ngrains_ref = 0;          // grainhdl::ngrains: the grain count the coarsening trigger compares with
    std::vector<std::pair<int, double>> dt_from;  // (first loop, dt) after every change of the time step

    size_t d_ids_count = 0;       // elements of d_ids
    std::vector<double> euler;    // 3 per grain
    std::vector<int32_t> bbox;    // 5 per grain
    std::vector<double> stored;   // .uds stored energy per grain (empty: none given)
    std::vector<double> stored_scaled;  // UseStoredElasticEnergy: scaled values, slot 0 = boundary
    std::vector<double> magnetic;       // UseMagneticField: magnetic energies, slot 0 = boundary
    bool contour_input = false;         // MicrostructureGenMode 0: grains loaded as polygons
    std::vector<int32_t> poly_off;      // contour input: point range of grain k at [k-1, k]
    std::vector<double> poly_xy;        // contour input: points in domain coordinates
    std::vector<double> poly_quat;      // contour input: 4 per grain, as given
    std::vector<double> quat;           // orientation quaternion per grain, slot 0 = boundary

    NetConst C{};
    NetState hS{};               // host copy of the device NetState (pointers)
    NetState* dS = nullptr;
    int32_t* d_ids = nullptr;     // ID field of the loaded microstructure (device)
    std::vector<void*> allocs;
    // bins of the initial neighbour search (from the pool, kept for later calls)
    int* nbin_count = nullptr;
    int* nbin_start = nullptr;
    int* nbin_total = nullptr;
    int* nbin_items = nullptr;
    int nbin_nc = 0;
    int64_t nbin_items_cap = 0;
    gg_grain_stats* d_stats = nullptr;  // packed statistics (device) and their pinned host copy
    gg_grain_stats* h_stats = nullptr;
    size_t h_stats_bytes = 0;
    // statistics prefetch: once a caller has read the statistics, every
    // gg_step gathers them and copies them, with the status word, into
    // pinned memory after its timed region; a read with nothing changed since
    // takes them from there
    bool stats_wanted = false;
    bool stats_fresh = false;
    uint32_t* h_status = nullptr;
    cudaEvent_t ev_done = nullptr;
    LaunchCfg cfg{256, 256, 128, 64};

    cudaGraphExec_t graph = nullptr;
    bool sectors_stale = false;    // batched form: the corrector's sectors need a rebuild before the next step
    int32_t graph_kernels = 0;     // kernel nodes of the captured step graph
    int64_t kernel_launches = 0;   // graph_kernels per replay, summed
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t stream2 = nullptr;  // second branch of the captured batched step
    cudaEvent_t fork[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double last_ms = 0;

    ~gg_ctx() {
        if (graph) cudaGraphExecDestroy(graph);
        if (stream) {
            for (void* p : allocs) cudaFreeAsync(p, stream);  // back to the library's pool
            cudaStreamSynchronize(stream);
        }
        pinned_give(h_stats, h_stats_bytes);  // to the process's pinned buffers
        pinned_give(h_status, sizeof(uint32_t));
        if (ev_done) cudaEventDestroy(ev_done);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (cudaEvent_t e : fork)
            if (e) cudaEventDestroy(e);
        if (stream2) cudaStreamDestroy(stream2);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int fail(gg_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(gg_ctx* c, cudaError_t e, const char* where) {
    // consume the runtime's last error as well, so that a failure reported
    // here is not reported again by a later, unrelated call of this thread
    (void)cudaGetLastError();
    return fail(c, GG_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define GG_CUDA(ctx, call)                                           \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);   \
    } while (0)

// Device memory of the contexts comes from a stream-ordered pool of the
// library's own, one per device, which keeps the memory a destroyed context
// gave back for the next context of the process: creating and destroying a
// network then maps and unmaps no memory after the first (cudaMalloc and
// cudaFree of the arenas took 30-110 ms and up to 1 s on the 20,000-grain
// workload).  The pool holds at most what the largest set of contexts alive
// together used, until the process exits.
int library_pool(gg_ctx* c, cudaMemPool_t* out) {
    constexpr int kMaxDevices = 64;
    static std::mutex mutex;
    static cudaMemPool_t pools[kMaxDevices] = {};
    const int dev = c->device;
    if (dev < 0 || dev >= kMaxDevices) return fail(c, GG_E_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lock(mutex);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        GG_CUDA(c, cudaMemPoolCreate(&pool, &props));
        uint64_t keep = UINT64_MAX;
        GG_CUDA(c, cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[dev] = pool;
    }
    *out = pools[dev];
    return GG_OK;
}

// Device memory from the library's pool, zero-filled unless `zero` is false
// (arenas whose every read is of a value a kernel wrote before: fields read
// inside the boxes they were written for, contour data up to the written
// counts).
template <typename T>
int dalloc(gg_ctx* c, T** out, size_t count, bool zero = true) {
    void* p = nullptr;
    const size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    cudaMemPool_t pool = nullptr;
    int rc = library_pool(c, &pool);
    if (rc) return rc;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMallocFromPoolAsync");
    e = zero ? cudaMemsetAsync(p, 0, bytes, c->stream) : cudaSuccess;
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMemset");
    c->allocs.push_back(p);
    *out = reinterpret_cast<T*>(p);
    return GG_OK;
}

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

bool xml_tag(const std::string& doc, const char* tag, std::string* val) {
    const std::string open = std::string("<") + tag + ">";
    const std::string close = std::string("</") + tag + ">";
    size_t a = doc.find(open);
    if (a == std::string::npos) return false;
    a += open.size();
    size_t b = doc.find(close, a);
    if (b == std::string::npos) return false;
    *val = doc.substr(a, b - a);
    return true;
}

// Euler (Bunge ZXZ) to quaternion: Quaternion::euler2quaternion (src/Quaternion.cpp:168-192)
void euler2quaternion(const double* e, double* q) {
    const double p1 = e[0], t = e[1], p2 = e[2];
    const double co1 = cos(t / 2);
    const double s1 = sin(t / 2);
    q[0] = co1 * cos((p1 + p2) / 2);
    q[1] = s1 * cos((p1 - p2) / 2);
    q[2] = s1 * sin((p1 - p2) / 2);
    q[3] = co1 * sin((p1 + p2) / 2);
}

// Quaternion to Euler (Bunge ZXZ, Diebel's (3,1,3) case), with the branch for
// sin(PHI) = 0 where phi1 + phi2 alone is defined and phi2 is set to 0:
// Quaternion::quaternion2EulerConst (src/Quaternion.cpp:242-289).  Angles in
// [0, 2 pi).
void quaternion2euler(const double* q, double* e) {
    const double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
    double cosPHI = q3 * q3 - q2 * q2 - q1 * q1 + q0 * q0;
    const double y0 = 2 * q1 * q3 - 2 * q0 * q2;
    const double x0 = 2 * q2 * q3 + 2 * q0 * q1;
    const double y1 = 2 * q1 * q3 + 2 * q0 * q2;
    const double x1 = -2 * q2 * q3 + 2 * q0 * q1;
    if (cosPHI > 1.) cosPHI = 1.;
    const double one_minus = 1. - cosPHI;
    const double PHI = one_minus * one_minus <= 1e-20 ? 0. : acos(cosPHI);  // QUAT2EUL_ETA, src/mymath.h:31
    const double sP = sin(PHI);
    double phi1, phi2;
    if (sP != 0) {
        phi2 = atan2(y0 / sP, x0 / sP);
        phi1 = atan2(y1 / sP, x1 / sP);
    } else {
        phi1 = atan2((2 * q1 * q2 + 2 * q0 * q3), q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3);
        phi2 = 0.;
    }
    if (phi1 < 0.0) phi1 += 2 * kPiH;
    if (phi2 < 0.0) phi2 += 2 * kPiH;
    e[0] = phi1;
    e[1] = PHI;
    e[2] = phi2;
}

// LSbox::calculateMagneticEnergy (src/box.cpp:2238-2292): the grain's c axis
// (the sample normal rotated by its Bunge angles) against the field direction,
// 1/2 mu0 dchi B^2 cos^2, normalised by HAGB_Energy and the domain size.
double magnetic_energy(const double* q, const gg_params& P) {
    double e[3];
    quaternion2euler(q, e);
    const double p1 = e[0], t = e[1];
    // row 3 of the rotation matrix (the rotated normal), each entry summed
    // onto zero as the reference's matrix-vector loop does
    const double axis[3] = {0.0 + sin(p1) * sin(t), 0.0 + -cos(p1) * sin(t), 0.0 + cos(t)};
    double cosine = (P.magnetic_vector[0] * axis[0]) + (P.magnetic_vector[1] * axis[1]) +
                    (P.magnetic_vector[2] * axis[2]);
    if (cosine > 1) cosine = 1.0;
    double energy = 0.5 * P.vacuum_permeability * P.delta_mag_sys * P.magnetic_force_field * P.magnetic_force_field *
                    cosine * cosine;
    energy = energy / P.hagb_energy * P.physical_domain_size;
    return energy;
}

// DimensionalBuffer::resizeToSquare (src/dimensionalBuffer.h:123-160)
Box host_resize_to_square(Box r, int maximumLength) {
    int grid_size = maximumLength - 1;
    unsigned int height = r.y1 - r.y0;
    unsigned int width = r.x1 - r.x0;
    if (width == height) return r;
    if (width > height) {
        int diff = width - height;
        r.y0 -= diff / 2;
        r.y1 += diff / 2 + diff % 2;
    } else {
        int diff = height - width;
        r.x0 -= diff / 2;
        r.x1 += diff / 2 + diff % 2;
    }
    if (r.x0 < 0) {
        int d = -r.x0;
        r.x1 += d;
        r.x0 += d;
    } else if (r.x1 > grid_size) {
        int d = grid_size - r.x1;
        r.x1 += d;
        r.x0 += d;
    }
    if (r.y0 < 0) {
        int d = -r.y0;
        r.y1 += d;
        r.y0 += d;
    } else if (r.y1 > grid_size) {
        int d = grid_size - r.y1;
        r.y1 += d;
        r.y0 += d;
    }
    return r;
}

// Twiddle exp(-2 pi i k / n) from libm (same expression as the oracle's FFT).
void twiddle(int n, int k, double* re, double* im) {
    double ang = (2.0 * kPiH * (double)k) / (double)n;
    *re = cos(ang);
    *im = -sin(ang);
}

// Gaussian multiplier of LSbox::convolutionGeneratorFFTW (src/box.cpp:674-687).
double gaussian_multiplier(int n, int i2, int j2, double dt, int nn) {
    double nsq = nn * nn;
    double n_nsq = n * n;
    return exp(-sqrt(2 / kPiH) * (i2 * i2 + j2 * j2) * 4.0 * dt * nsq / n_nsq * kPiH * kPiH) / n_nsq;
}

int status_error(gg_ctx* c, uint32_t st) {
    // Capacity overflows invalidate the state and are errors.  The remaining
    // bits mark inputs on which the reference itself would fault or never
    // return (see GG_S_* in gg_step.h); they are kept in the status word for
    // gg_status() and do not stop the run.
    if (st & (S_ARENA_FULL | S_LIST_OVERFLOW | S_CONTOUR_OVERFLOW | S_JUNCTION_OVERFLOW | S_TABLE_RANGE |
              S_NEIGHBOUR_OVERFLOW)) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "device capacity exceeded (status 0x%x)", st);
        return fail(c, GG_E_CAPACITY, buf);
    }
    if (st & S_NAN) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "non-finite distance value or area on the device (status 0x%x)", st);
        return fail(c, GG_E_NUMERIC, buf);
    }
    return GG_OK;
}

int check_status(gg_ctx* c) {
    uint32_t st = 0;
    GG_CUDA(c, cudaMemcpyAsync(&st, &c->dS->status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    return status_error(c, st);
}

int refresh_state(gg_ctx* c) {
    GG_CUDA(c, cudaMemcpyAsync(&c->hS, c->dS, sizeof(NetState), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    return GG_OK;
}

int set_loop(gg_ctx* c, int loop) {
    GG_CUDA(c, cudaMemcpyAsync(&c->dS->loop, &loop, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    return GG_OK;
}

// grainhdl::gridCoarsement (src/grainhdl.cpp:1396-1478), checked at the start
// of step `loop`: when the grains present have fallen below
// GridCoarsementGradient of the count at the last coarsening, every grain's
// field is resampled onto a grid of sqrt(count) x NumberOfPointsPerGrain
// points, the grid constants and the time step are recomputed, IDLocal is
// rebuilt by a comparison of the resampled fields and the contours are
// extracted from them; the step then runs on the new grid.  Returns whether
// the grid changed in *changed.
int launch_stages(gg_ctx* c, int stages);
void conv_tables(const gg_ctx* c, int tmax, const std::vector<int64_t>& gk_off, const std::vector<int64_t>& ck_off,
                 std::vector<double>& gk, std::vector<float>& ck);

int coarsen_if_due(gg_ctx* c, int loop, bool* changed) {
    *changed = false;
    const gg_params& P = c->P;
    if (!P.grid_coarsement || loop == 0) return GG_OK;
    int rc = refresh_state(c);
    if (rc) return rc;
    NetState& S = c->hS;
    NetConst& C = c->C;
    const int current = S.live;
    if (!((double)current / (double)c->ngrains_ref < P.grid_coarsement_gradient)) return GG_OK;
    const int N = c->N;
    const int new_size = (int)(std::sqrt((double)current) * (double)c->ppg);
    if (new_size < 1) return fail(c, GG_E_INVALID, "grid coarsening to an empty grid");
    const int m_new = new_size + 2 * c->b;
    const double h_old = c->h, hn = 1.0 / (double)new_size, delta_old = c->delta;
    std::vector<Box> bcur(N + 1), bnew(N + 1, Box{0, 0, 0, 0});
    std::vector<int32_t> state(N + 1), newbb(4 * (size_t)(N + 1), 0);
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    };
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
    };
    GG_CUDA(c, d2h(bcur.data(), S.box_cur, sizeof(Box) * (N + 1)));
    GG_CUDA(c, d2h(state.data(), C.state, 4 * (N + 1)));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    // LSbox::resizeGrid (src/box.cpp:1408-1436): the old box scaled by h / hn
    // (kept unsquared as m_newXMin ..), the input box made square on the new grid
    std::vector<int64_t> off(N + 1, 0), coff(N + 1, 0);
    std::vector<int32_t> ccap(N + 1, 0);
    int64_t a = 0, cc = 0;
    for (int g = 1; g <= N; ++g) {
        off[g] = a;
        coff[g] = cc;
        if (state[g] == G_GONE) continue;
        const Box& o = bcur[g];
        const int x0 = o.x0 * (h_old / hn) + 0.5, x1 = o.x1 * (h_old / hn) + 0.5;
        const int y0 = o.y0 * (h_old / hn) + 0.5, y1 = o.y1 * (h_old / hn) + 0.5;
        newbb[4 * (size_t)g] = x0;
        newbb[4 * (size_t)g + 1] = x1;
        newbb[4 * (size_t)g + 2] = y0;
        newbb[4 * (size_t)g + 3] = y1;
        bnew[g] = host_resize_to_square(Box{x0, x1, y0, y1}, m_new);
        a += box_area(bnew[g]);
        ccap[g] = contour_capacity(box_w(bnew[g]));
        cc += ccap[g];
    }
    if (a > S.phi_cap || cc > S.cont_cap) return fail(c, GG_E_CAPACITY, "coarsened grid does not fit the arenas");
    GG_CUDA(c, h2d(S.box_new, bnew.data(), sizeof(Box) * (N + 1)));
    GG_CUDA(c, h2d(S.off_new, off.data(), sizeof(int64_t) * (N + 1)));
    cudaError_t e = P.precision == GG_PRECISION_PLAIN ? plain_resample(C, c->dS, h_old, hn, delta_old, c->stream)
                                                      : batched_resample(C, c->dS, h_old, hn, delta_old, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "resample");
    // new grid constants and time step (src/grainhdl.cpp:1414-1451)
    c->nn = new_size;
    c->m = m_new;
    c->delta = (unsigned long)P.domain_border_size * 1 / double(new_size);
    c->h = 1.0 / new_size;
    const unsigned long ppg_used =
        P.decouple_grains == 1 ? (unsigned long)P.number_of_points_per_grain : (unsigned long)c->ppg;
    c->dt = 0.8 / double(new_size * new_size) * ppg_used / 2 / 5.0;
    double correction = 0.5 / new_size / c->energy_delta_max / c->dt;
    if (correction > 1.0) correction = 1.0;
    c->dt *= correction;
    c->ngrains_ref = current;
    c->dt_from.emplace_back(loop, c->dt);
    C.m = c->m;
    C.nn = c->nn;
    C.h = c->h;
    C.delta = c->delta;
    C.dt = c->dt;
    {
        const int tmax = C.tmax;
        std::vector<int64_t> gk_off(tmax + 1, 0), ck_off(tmax + 1, 0);
        int64_t gkn = 0, ckn = 0;
        for (int n = 1; n <= tmax; ++n) {
            gk_off[n] = gkn;
            gkn += (int64_t)(n / 2 + 1) * (n / 2 + 1);
            ck_off[n] = ckn;
            ckn += n + 1;
        }
        const bool plain = P.precision == GG_PRECISION_PLAIN;
        std::vector<double> gk(plain ? gkn : 1);
        std::vector<float> ck(plain ? 1 : ckn);
        conv_tables(c, tmax, gk_off, ck_off, gk, ck);
        if (plain)
            GG_CUDA(c, h2d(const_cast<double*>(C.gk), gk.data(), sizeof(double) * gk.size()));
        else
            GG_CUDA(c, h2d(const_cast<float*>(C.ck), ck.data(), sizeof(float) * ck.size()));
        GG_CUDA(c, cudaStreamSynchronize(c->stream));  // host tables leave scope
    }
    // LSbox::recalculateIDLocal (src/box.cpp:1487-1495): a comparison of the
    // resampled fields (read where the convolution would be: phiB at the new
    // offsets) into the new IDLocal; the old IDLocal stays in idPrev for the
    // buffer-keeping resize
    std::swap(S.box_cur, S.box_new);
    std::swap(S.off_cur, S.off_new);
    GG_CUDA(c, h2d(c->dS, &S, sizeof(NetState)));
    e = P.precision == GG_PRECISION_PLAIN ? plain_stage_kernel(C, c->dS, 3, c->stream, c->cfg)
                                          : batched_stage_kernel(C, c->dS, 3, c->stream, c->cfg);
    if (e != cudaSuccess) return cuda_fail(c, e, "coarsening comparison");
    // LSbox::extractContour (src/box.cpp:1089-1153) of the resampled fields
    // (phiA), with the scaled boxes as m_newXMin .. (not the set comparison's)
    GG_CUDA(c, h2d(C.newbb, newbb.data(), sizeof(int32_t) * newbb.size()));
    std::swap(S.phiA, S.phiB);
    GG_CUDA(c, h2d(c->dS, &S, sizeof(NetState)));
    e = P.precision == GG_PRECISION_PLAIN ? plain_stage_kernel(C, c->dS, 4, c->stream, c->cfg)
                                          : batched_stage_kernel(C, c->dS, 4, c->stream, c->cfg);
    if (e != cudaSuccess) return cuda_fail(c, e, "coarsening contours");
    // the contour extraction does not delete grains that had vanished before
    for (int g = 1; g <= N; ++g)
        if (state[g] == G_VANISHED) {
            const int32_t vanished = G_VANISHED, none = -1;
            GG_CUDA(c, h2d(C.state + g, &vanished, 4));
            GG_CUDA(c, h2d(C.gone_loop + g, &none, 4));
        }
    // the step then starts from the resampled field (phiA, box_cur), the new
    // IDLocal and contour as the previous ones, and fresh contour slots
    std::swap(S.idPrev, S.idCur);
    GG_CUDA(c, cudaMemcpyAsync(S.box_prev, S.box_cur, sizeof(Box) * (N + 1), cudaMemcpyDeviceToDevice, c->stream));
    GG_CUDA(c, cudaMemcpyAsync(S.off_prev, S.off_cur, sizeof(int64_t) * (N + 1), cudaMemcpyDeviceToDevice, c->stream));
    std::swap(S.contPrev, S.contCur);
    std::swap(S.coff_prev, S.coff_cur);
    std::swap(S.ccap_prev, S.ccap_cur);
    std::swap(S.cn_prev, S.cn_cur);
    std::swap(S.jPrev, S.jCur);
    std::swap(S.jn_prev, S.jn_cur);
    GG_CUDA(c, h2d(S.coff_cur, coff.data(), sizeof(int64_t) * (N + 1)));
    GG_CUDA(c, h2d(S.ccap_cur, ccap.data(), sizeof(int32_t) * (N + 1)));
    GG_CUDA(c, h2d(c->dS, &S, sizeof(NetState)));
    if (P.precision != GG_PRECISION_PLAIN) GG_CUDA(c, batched_order(C, c->dS, c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    c->sectors_stale = true;  // new contours
    if (c->graph) {  // the captured step holds the old constants
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    *changed = true;
    return check_status(c);
}

int launch_stages(gg_ctx* c, int stages) {
    if (c->P.precision != GG_PRECISION_PLAIN && (stages & ST_CONV) && c->sectors_stale) {
        GG_CUDA(c, batched_sectors(c->C, c->dS, c->stream));
        c->sectors_stale = false;
    }
    cudaError_t e = c->P.precision == GG_PRECISION_PLAIN ? plain_stages(c->C, c->dS, stages, c->stream, c->cfg)
                                                         : batched_stages(c->C, c->dS, stages, c->stream, c->cfg);
    if (e != cudaSuccess) return cuda_fail(c, e, "stage launch");
    return GG_OK;
}

// The tables of one box edge depend only on (form, edge, dt, grid size);
// every context of the process computes each such table once.
struct TableKey {
    int plain, n;
    uint64_t dt_bits;
    int nn;
    bool operator<(const TableKey& o) const {
        return std::tie(plain, n, dt_bits, nn) < std::tie(o.plain, o.n, o.dt_bits, o.nn);
    }
};
std::mutex g_table_mutex;
std::map<TableKey, std::vector<double>> g_gk_cache;
std::map<TableKey, std::vector<float>> g_ck_cache;

TableKey table_key(const gg_ctx* c, int n) {
    uint64_t bits;
    std::memcpy(&bits, &c->dt, sizeof bits);
    return TableKey{c->P.precision == GG_PRECISION_PLAIN ? 1 : 0, n, bits, c->nn};
}

// Gaussian multipliers (plain form) or separable real-space kernels with their
// band radius (batched form) of every box edge up to tmax, for the context's
// current dt and grid size (both change when the grid is coarsened).
void conv_tables_compute(const gg_ctx* c, int tmax, const std::vector<int64_t>& gk_off,
                         const std::vector<int64_t>& ck_off, std::vector<double>& gk, std::vector<float>& ck,
                         int nlo);

void conv_tables(const gg_ctx* c, int tmax, const std::vector<int64_t>& gk_off, const std::vector<int64_t>& ck_off,
                 std::vector<double>& gk, std::vector<float>& ck) {
    const bool plain = c->P.precision == GG_PRECISION_PLAIN;
    for (int n = 1; n <= tmax; ++n) {
        const TableKey key = table_key(c, n);
        {
            std::lock_guard<std::mutex> lock(g_table_mutex);
            if (plain) {
                const auto it = g_gk_cache.find(key);
                if (it != g_gk_cache.end()) {
                    std::copy(it->second.begin(), it->second.end(), gk.begin() + gk_off[n]);
                    continue;
                }
            } else {
                const auto it = g_ck_cache.find(key);
                if (it != g_ck_cache.end()) {
                    std::copy(it->second.begin(), it->second.end(), ck.begin() + ck_off[n]);
                    continue;
                }
            }
        }
        conv_tables_compute(c, n, gk_off, ck_off, gk, ck, n);
        std::lock_guard<std::mutex> lock(g_table_mutex);
        if (plain) {
            const int64_t len = (int64_t)(n / 2 + 1) * (n / 2 + 1);
            g_gk_cache[key].assign(gk.begin() + gk_off[n], gk.begin() + gk_off[n] + len);
        } else {
            g_ck_cache[key].assign(ck.begin() + ck_off[n], ck.begin() + ck_off[n] + n + 1);
        }
    }
}

// Edges nlo .. tmax.
void conv_tables_compute(const gg_ctx* c, int tmax, const std::vector<int64_t>& gk_off,
                         const std::vector<int64_t>& ck_off, std::vector<double>& gk, std::vector<float>& ck,
                         int nlo) {
    if (c->P.precision == GG_PRECISION_PLAIN) {
        for (int n = nlo; n <= tmax; ++n) {
            const int half = n / 2 + 1;
            for (int i2 = 0; i2 < half; ++i2)
                for (int j2 = i2; j2 < half; ++j2)  // G(i2, j2) = G(j2, i2): i2^2 + j2^2 is the argument
                    gk[gk_off[n] + i2 * half + j2] = gk[gk_off[n] + j2 * half + i2] =
                        gaussian_multiplier(n, i2, j2, c->dt, c->nn);
        }
        return;
    }
        // k_n[r] = (1/n) sum_f g(min(f, n-f)) cos(2 pi f r / n), g(f) = exp(-kappa f^2),
        // kappa = sqrt(2/pi) 4 dt nn^2 / n^2 pi^2 (the 1/n^2 of G split over both axes)
        std::vector<double> gf, cs;
        for (int n = nlo; n <= tmax; ++n) {
            const double kappa = sqrt(2 / kPiH) * 4.0 * c->dt * (double)c->nn * (double)c->nn / ((double)n * n) *
                                 kPiH * kPiH;
            gf.assign(n, 0.0);
            for (int f = 0; f < n; ++f) {
                const int f2 = std::min(f, n - f);
                gf[f] = exp(-kappa * (double)f2 * f2);
            }
            // cos(2 pi k / n) once per k (the same expression the sum would
            // evaluate for k = f r mod n)
            cs.resize(n);
            for (int k = 0; k < n; ++k) cs[k] = cos(2.0 * kPiH * (double)k / n);
            for (int r = 0; r < n; ++r) {
                double acc = 0;
                for (int f = 0, k = 0; f < n; ++f) {  // k = f r mod n
                    acc += gf[f] * cs[k];
                    k += r;
                    if (k >= n) k -= n;
                }
                ck[ck_off[n] + r] = (float)(acc / n);
            }
            // band radius: every entry at circular distance > R is below 2^-26 k_n[0]
            // (under half an FP32 ulp of the centre tap; the dropped tail is the
            // flat aliasing floor of the truncated Gaussian, ~7e-9 k_n[0])
            int R = 0;
            const double tiny = std::ldexp(std::fabs((double)ck[ck_off[n]]), -26);
            for (int r = 1; r < n; ++r)
                if (std::fabs((double)ck[ck_off[n] + r]) > tiny) R = std::max(R, std::min(r, n - r));
            ck[ck_off[n] + n] = (float)R;
        }
}

}  // namespace

extern "C" {

int gg_params_default(gg_params* p) {
    if (!p) return GG_E_INVALID;
    std::memset(p, 0, sizeof(*p));
    p->struct_size = (int32_t)sizeof(gg_params);
    p->precision = GG_PRECISION_PLAIN;
    p->analysis_timestep = 1;
    p->grid_coarsement_gradient = 0.95;
    p->domain_border_size = 7;
    p->microstructure_gen_mode = 4;
    p->convolution_mode = 2;
    p->hagb_energy = 1.0;
    p->hagb_mobility = 1.0;
    p->time_slope = 0.8359;
    p->theta_ref_deg = 15.0;
    p->gamma_hagb = 1.0;
    p->m_hagb = 1.0;
    return GG_OK;
}

int gg_params_from_xml(const char* path, gg_params* p) {
    if (!path || !p) return GG_E_INVALID;
    std::ifstream f(path);
    if (!f) return GG_E_IO;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string doc = ss.str();
    if (doc.find("<Parameters>") == std::string::npos) return GG_E_IO;
    std::string v;
    auto geti = [&](const char* tag, int32_t* dst) {
        if (xml_tag(doc, tag, &v)) *dst = (int32_t)std::stol(trim(v));
    };
    auto getd = [&](const char* tag, double* dst) {
        if (xml_tag(doc, tag, &v)) *dst = std::stod(trim(v));
    };
    auto gets = [&](const char* tag, char* dst, size_t cap) {
        if (xml_tag(doc, tag, &v)) {
            std::string t = trim(v);
            std::strncpy(dst, t.c_str(), cap - 1);
            dst[cap - 1] = 0;
        }
    };
    try {
        geti("StartTime", &p->start_time);
        geti("NumberOfParticles", &p->number_of_particles);
        geti("NumberOfPointsPerGrain", &p->number_of_points_per_grain);
        geti("AnalysisTimestep", &p->analysis_timestep);
        geti("DiscreteSamplingRate", &p->discrete_sampling_rate);
        geti("NumberOfTimesteps", &p->number_of_timesteps);
        geti("BreakupNumber", &p->breakup_number);
        geti("DomainBorderSize", &p->domain_border_size);
        geti("MicrostructureGenMode", &p->microstructure_gen_mode);
        gets("ReadFromFilename", p->read_from_filename, sizeof p->read_from_filename);
        gets("AdditionalFilename", p->additional_filename, sizeof p->additional_filename);
        geti("LatticeType", &p->lattice_type);
        getd("HAGB_Energy", &p->hagb_energy);
        getd("HAGB_Mobility", &p->hagb_mobility);
        getd("Physical_Domain_Size", &p->physical_domain_size);
        getd("TriplePointDrag", &p->triple_point_drag);
        geti("UseMobilityModel", &p->use_mobility_model);
        geti("IdentifyTwins", &p->identify_twins);
        geti("UseMagneticField", &p->use_magnetic_field);
        geti("IsIsotropicNetwork", &p->is_isotropic_network);
        geti("GridCoarsement", &p->grid_coarsement);
        geti("ConvolutionMode", &p->convolution_mode);
        geti("ResearchMode", &p->research_mode);
        geti("ResearchProject", &p->research_project);
        getd("ConstantSectorRadius", &p->constant_sector_radius);
        getd("InterpolatingSectorRadius", &p->interpolating_sector_radius);
        geti("UseStoredElasticEnergy", &p->use_stored_elastic_energy);
        geti("DecoupleGrains", &p->decouple_grains);
        getd("GaussianKernelUserDefTimeSlope", &p->time_slope);
        getd("ThetaRefDegrees", &p->theta_ref_deg);
        getd("HAGB_RelativeEnergy", &p->gamma_hagb);
        getd("HAGB_RelativeMobility", &p->m_hagb);
        getd("DislocEnPerM", &p->dislocation_energy_per_m);
        getd("BoxDefaultStoredElasticEnergy", &p->box_default_stored_elastic_energy);
        geti("Precision", &p->precision);
        geti("PlotInterval", &p->plot_interval);
        geti("UseTexture", &p->use_texture);
        geti("ExecuteInParallel", &p->execute_in_parallel);
        geti("MaximumNumberOfThreads", &p->maximum_number_of_threads);
        geti("NeighbourTracking", &p->neighbour_tracking);
        geti("GrainScheduler", &p->grain_scheduler);
        getd("GridCoarsementGradient", &p->grid_coarsement_gradient);
        // magnetic field parameters from the file MagneticParams names
        // (Settings::readMagneticFieldParams, src/Settings.cpp:291-347); a
        // relative name is looked up beside the parameters file first
        if (p->use_magnetic_field == 1) {
            std::string name;
            if (!xml_tag(doc, "MagneticParams", &name)) return GG_E_IO;
            name = trim(name);
            std::ifstream mf;
            if (!name.empty() && name[0] != '/') {
                std::string dir(path);
                const size_t slash = dir.rfind('/');
                dir = slash == std::string::npos ? std::string() : dir.substr(0, slash + 1);
                mf.open(dir + name);
            }
            if (!mf) mf.open(name);
            if (!mf) return GG_E_IO;
            std::stringstream ms;
            ms << mf.rdbuf();
            const std::string mdoc = ms.str();
            if (mdoc.find("<Parameters>") == std::string::npos) return GG_E_IO;
            auto getm = [&](const char* tag, double* dst) {
                if (xml_tag(mdoc, tag, &v)) *dst = std::stod(trim(v));
            };
            getm("VacuumPermeability", &p->vacuum_permeability);
            getm("MagneticVector_x", &p->magnetic_vector[0]);
            getm("MagneticVector_y", &p->magnetic_vector[1]);
            getm("MagneticVector_z", &p->magnetic_vector[2]);
            getm("deltaMagSys", &p->delta_mag_sys);
            getm("MagneticForceField", &p->magnetic_force_field);
        }
    } catch (...) {
        return GG_E_IO;
    }
    return GG_OK;
}

int gg_create(const gg_params* p, int device, gg_ctx** out) {
    if (!p || !out) return GG_E_INVALID;
    *out = nullptr;
    if (p->struct_size != (int32_t)sizeof(gg_params)) return GG_E_INVALID;
    gg_ctx* c = new gg_ctx();
    c->P = *p;
    c->device = device;
    auto bad = [&](const char* msg) {
        c->err = msg;
        *out = c;
        return GG_E_INVALID;
    };
    if (p->microstructure_gen_mode != 0 && p->microstructure_gen_mode != 4)
        return bad("only MicrostructureGenMode 0 (contour file) and 4 (voxelized) are supported");
    if (p->convolution_mode != 2) return bad("only ConvolutionMode 2 (Gaussian) is supported");
    if (p->lattice_type != 0) return bad("only LatticeType 0 (cubic) is supported");
    if (p->research_mode != 0) return bad("only ResearchMode 0 is supported");
    if (p->grid_coarsement < 0 || p->grid_coarsement > 1) return bad("GridCoarsement must be 0 or 1");
    if (p->grid_coarsement && p->decouple_grains == 1) return bad("GridCoarsement with DecoupleGrains is not supported");
    if (p->use_magnetic_field < 0 || p->use_magnetic_field > 1) return bad("UseMagneticField must be 0 or 1");
    if (p->use_stored_elastic_energy < 0 || p->use_stored_elastic_energy > 1)
        return bad("UseStoredElasticEnergy must be 0 or 1");
    if (p->identify_twins != 0) return bad("IdentifyTwins is not supported");
    if (p->use_mobility_model < 0 || p->use_mobility_model > 1) return bad("UseMobilityModel must be 0 or 1");
    if (p->precision != GG_PRECISION_PLAIN && p->precision != GG_PRECISION_BATCHED) return bad("bad precision");
    if (p->domain_border_size < 1) return bad("DomainBorderSize must be >= 1");
    if (p->analysis_timestep <= 0) return bad("AnalysisTimestep must be > 0");
    if (p->discrete_sampling_rate < 0) return bad("DiscreteSamplingRate must be >= 0");
    if (p->list_capacity < 0 || p->list_capacity > 128) return bad("list_capacity must be 0 or 1..128");
    if (!(p->arena_factor == 0 || p->arena_factor >= 1)) return bad("arena_factor must be 0 or >= 1");
    {
        const double vals[] = {p->triple_point_drag, p->constant_sector_radius, p->interpolating_sector_radius,
                               p->hagb_energy, p->hagb_mobility, p->physical_domain_size, p->time_slope,
                               p->theta_ref_deg, p->gamma_hagb, p->m_hagb, p->dislocation_energy_per_m,
                               p->box_default_stored_elastic_energy, p->vacuum_permeability, p->magnetic_vector[0],
                               p->magnetic_vector[1], p->magnetic_vector[2], p->delta_mag_sys,
                               p->magnetic_force_field, p->grid_coarsement_gradient, p->arena_factor};
        for (double v : vals)
            if (!std::isfinite(v)) {
                c->err = "non-finite parameter value";
                *out = c;
                return GG_E_NUMERIC;
            }
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        c->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
        *out = c;
        return GG_E_CUDA;
    }
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
    for (int k = 0; k < 5 && e == cudaSuccess; ++k) e = cudaEventCreateWithFlags(&c->fork[k], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        c->err = std::string("stream/event: ") + cudaGetErrorString(e);
        *out = c;
        return GG_E_CUDA;
    }
    *out = c;
    return GG_OK;
}

void gg_destroy(gg_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

const char* gg_last_error(const gg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// Non-finite input values are refused before anything reaches the device:
// boxes, pixel indices and contour walks are derived from them there.
static bool all_finite(const double* v, size_t n) {
    for (size_t q = 0; q < n; ++q)
        if (!std::isfinite(v[q])) return false;
    return true;
}

int gg_load_voxels(gg_ctx* c, int32_t nn, const int32_t* ids, int32_t n_grains, const double* euler,
                   const int32_t* bbox) {
    if (!c || !ids || !euler || !bbox || nn <= 0 || n_grains <= 0) return fail(c, GG_E_INVALID, "bad voxel input");
    if (c->initialised) return fail(c, GG_E_STATE, "network already initialised");
    if (!all_finite(euler, 3 * (size_t)n_grains)) return fail(c, GG_E_NUMERIC, "non-finite Euler angle");
    c->nn = nn;
    c->N = n_grains;
    // the ID field goes straight to the device (it is read only by the
    // distance initialisation)
    GG_CUDA(c, cudaSetDevice(c->device));
    if (c->d_ids_count != (size_t)nn * nn) {
        int rc;
        if ((rc = dalloc(c, &c->d_ids, (size_t)nn * nn)) != GG_OK) return rc;
        c->d_ids_count = (size_t)nn * nn;
    }
    GG_CUDA(c, cudaMemcpyAsync(c->d_ids, ids, sizeof(int32_t) * (size_t)nn * nn, cudaMemcpyHostToDevice, c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    c->euler.assign(euler, euler + 3 * (size_t)n_grains);
    c->bbox.assign(bbox, bbox + 5 * (size_t)n_grains);
    c->stored.clear();
    c->contour_input = false;
    c->loaded = true;
    return GG_OK;
}

int gg_load_contours(gg_ctx* c, int32_t n_grains, const int32_t* offsets, const double* xy, const double* quat) {
    if (!c || !offsets || !quat || n_grains <= 0) return fail(c, GG_E_INVALID, "bad contour input");
    if (c->initialised) return fail(c, GG_E_STATE, "network already initialised");
    if (offsets[0] != 0) return fail(c, GG_E_INVALID, "contour offsets must start at 0");
    for (int k = 0; k < n_grains; ++k) {
        const int32_t np = offsets[k + 1] - offsets[k];
        if (np < 0) return fail(c, GG_E_INVALID, "contour offsets must not decrease");
        if (np > 0 && np < 3) return fail(c, GG_E_INVALID, "a present grain needs a polygon of 3 or more points");
    }
    if (offsets[n_grains] > 0 && !xy) return fail(c, GG_E_INVALID, "no contour points");
    if (offsets[n_grains] > 0 && !all_finite(xy, 2 * (size_t)offsets[n_grains]))
        return fail(c, GG_E_NUMERIC, "non-finite contour coordinate");
    if (!all_finite(quat, 4 * (size_t)n_grains)) return fail(c, GG_E_NUMERIC, "non-finite quaternion");
    c->N = n_grains;
    c->poly_off.assign(offsets, offsets + n_grains + 1);
    c->poly_xy.resize(2 * (size_t)offsets[n_grains]);
    // grainhdl::readMicrostructure clamps every point to the unit square
    // (src/grainhdl.cpp:639-646)
    for (size_t q = 0; q < c->poly_xy.size(); ++q) {
        double v = xy[q];
        if (v < 0) v = 0;
        if (v > 1) v = 1;
        c->poly_xy[q] = v;
    }
    c->poly_quat.assign(quat, quat + 4 * (size_t)n_grains);
    c->euler.clear();
    c->bbox.clear();
    c->stored.clear();
    c->contour_input = true;
    c->loaded = true;
    return GG_OK;
}

int gg_load_contour_file(gg_ctx* c, const char* base_dir) {
    if (!c) return GG_E_INVALID;
    std::string path(c->P.read_from_filename);
    if (!path.empty() && path[0] != '/' && base_dir && base_dir[0]) path = std::string(base_dir) + "/" + path;
    std::ifstream f(path);
    if (!f) return fail(c, GG_E_IO, "cannot open " + path);
    // grainhdl::readMicrostructure (src/grainhdl.cpp:605-654): records in file
    // order become grains 1, 2, ...; a record ID at least the grain count
    // raises the count, and the loop reads that many records
    int ngrains = c->P.number_of_particles;
    if (ngrains <= 0) return fail(c, GG_E_INVALID, "NumberOfParticles must be > 0");
    std::vector<int32_t> off(1, 0);
    std::vector<double> xy, quat;
    for (int k = 1; k <= ngrains; ++k) {
        long id = 0, nv = 0;
        double q[4];
        if (!(f >> id)) break;  // fewer records than grains: the rest are absent
        if (id >= ngrains) ngrains = (int)id;
        if (!(f >> nv >> q[0] >> q[1] >> q[2] >> q[3]) || nv < 0)
            return fail(c, GG_E_IO, "truncated contour record in " + path);
        for (long v = 0; v < 2 * nv; ++v) {
            double t;
            if (!(f >> t)) return fail(c, GG_E_IO, "truncated contour points in " + path);
            xy.push_back(t);
        }
        off.push_back(off.back() + (int32_t)nv);
        quat.insert(quat.end(), q, q + 4);
    }
    while ((int)off.size() < ngrains + 1) {
        off.push_back(off.back());
        quat.insert(quat.end(), {1.0, 0.0, 0.0, 0.0});
    }
    return gg_load_contours(c, ngrains, off.data(), xy.data(), quat.data());
}

int gg_load_stored_energy(gg_ctx* c, const double* stored, int32_t n_grains) {
    if (!c || !stored) return GG_E_INVALID;
    if (!c->loaded) return fail(c, GG_E_STATE, "no microstructure loaded");
    if (c->initialised) return fail(c, GG_E_STATE, "network already initialised");
    if (n_grains != c->N) return fail(c, GG_E_INVALID, "one stored energy per grain");
    if (!all_finite(stored, (size_t)n_grains)) return fail(c, GG_E_NUMERIC, "non-finite stored energy");
    c->stored.assign(stored, stored + n_grains);
    return GG_OK;
}

int gg_load_voxel_files(gg_ctx* c, const char* base_dir) {
    if (!c) return GG_E_INVALID;
    auto join = [&](const char* name) {
        std::string s(name);
        if (!s.empty() && s[0] != '/' && base_dir && base_dir[0]) s = std::string(base_dir) + "/" + s;
        return s;
    };
    // read_voxelized_microstructure (src/grainhdl.cpp:336-511): 8 header lines
    FILE* f = std::fopen(join(c->P.additional_filename).c_str(), "r");
    if (!f) return fail(c, GG_E_IO, std::string("cannot open ") + join(c->P.additional_filename));
    char line[4096];
    int id_offset = 1, NX = 0, NY = 0, grains = 0;
    for (int i = 1; i <= 8; ++i) {
        if (!std::fgets(line, sizeof line, f)) {
            std::fclose(f);
            return fail(c, GG_E_IO, "truncated .uds header");
        }
        char name[256];
        int val = 0;
        if (i >= 2 && i <= 7 && std::sscanf(line, "%255s %d", name, &val) == 2) {
            if (i == 2) id_offset = val;
            if (i == 5) NX = val;
            if (i == 6) NY = val;
            if (i == 7) grains = val;
        }
    }
    if (NX <= 0 || NX != NY || grains <= 0) {
        std::fclose(f);
        return fail(c, GG_E_IO, "bad .uds header (need NX == NY > 0 and a grain count)");
    }
    std::vector<double> eul(3 * (size_t)grains), stored(grains);
    std::vector<int32_t> bb(5 * (size_t)grains);
    for (int k = 0; k < grains; ++k) {
        int id, xmin, xmax, ymin, ymax, cnt;
        double x, y, e0, e1, e2, se;
        if (std::fscanf(f, "%d %lf %lf %lf %lf %lf %d %d %d %d %d %lf", &id, &x, &y, &e0, &e1, &e2, &xmin, &xmax,
                        &ymin, &ymax, &cnt, &se) != 12) {
            std::fclose(f);
            return fail(c, GG_E_IO, "truncated .uds grain table");
        }
        if (id - (id_offset - 1) != k + 1) {
            std::fclose(f);
            return fail(c, GG_E_IO, "grain IDs in the .uds must be consecutive from the ID offset");
        }
        eul[3 * k] = e0;
        eul[3 * k + 1] = e1;
        eul[3 * k + 2] = e2;
        bb[5 * k] = xmin;
        bb[5 * k + 1] = xmax;
        bb[5 * k + 2] = ymin;
        bb[5 * k + 3] = ymax;
        bb[5 * k + 4] = cnt;
        stored[k] = se;
    }
    std::fclose(f);
    FILE* fb = std::fopen(join(c->P.read_from_filename).c_str(), "rb");
    if (!fb) return fail(c, GG_E_IO, std::string("cannot open ") + join(c->P.read_from_filename));
    std::vector<int32_t> ids((size_t)NX * NX);
    const size_t got = std::fread(ids.data(), sizeof(int32_t), ids.size(), fb);
    std::fclose(fb);
    if (got != ids.size()) return fail(c, GG_E_IO, "truncated .bin ID field");
    for (auto& v : ids) {
        v = v - (id_offset - 1);
        if (v < 0) v = 0;
    }
    int rc = gg_load_voxels(c, NX, ids.data(), grains, eul.data(), bb.data());
    if (rc == GG_OK && c->P.use_stored_elastic_energy) rc = gg_load_stored_energy(c, stored.data(), grains);
    return rc;
}

// Launch bins chosen by gg_autotune, kept for the process per (largest box
// edge, grain count): a later context of the same network size starts with
// them.
struct TunedBins {
    int compare_threads, big_edge, conv_smem_edge;
};
std::mutex g_tune_mutex;
std::map<std::pair<int, int>, TunedBins> g_tuned;

void apply_cached_tuning(gg_ctx* c) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    const auto it = g_tuned.find({c->C.tmax, c->N});
    if (it == g_tuned.end()) return;
    c->cfg.compare_threads = it->second.compare_threads;
    c->C.big_edge = it->second.big_edge;
    c->C.conv_smem_edge = it->second.conv_smem_edge;
}

int gg_distance_initialisation(gg_ctx* c) {
    if (!c) return GG_E_INVALID;
    c->stats_fresh = false;
    if (!c->loaded) return fail(c, GG_E_STATE, "no microstructure loaded");
    if (c->initialised) return fail(c, GG_E_STATE, "already initialised");
    GG_CUDA(c, cudaSetDevice(c->device));
    const gg_params& P = c->P;
    const bool poly = c->contour_input;
    if (poly) {
        // grainhdl::setSimulationParameter for file input (src/grainhdl.cpp:74-78):
        // the grid follows the parameters, not the loaded grains
        c->nn = (int)(std::sqrt((double)(unsigned)P.number_of_particles) * (double)P.number_of_points_per_grain);
        if (c->nn <= 0) return fail(c, GG_E_INVALID, "NumberOfParticles and NumberOfPointsPerGrain give no grid");
        c->ppg = P.number_of_points_per_grain;
    } else {
        // grainhdl::read_HeaderCPG / setSimulationParameter (src/grainhdl.cpp:56-136, 275-334)
        c->ppg = (int)(c->nn / sqrt(c->N));
    }
    const int realDomainSize = c->nn;
    // orientation quaternions, slot 0 the boundary (Euler (0,0,0),
    // src/grainhdl.cpp:137): converted from the Euler angles of a voxelized
    // input (src/box.cpp:156-217), used as given for contour input
    // (src/box.cpp:112)
    c->quat.assign(4 * (size_t)(c->N + 1), 0.0);
    c->quat[0] = 1.0;
    auto convert = [c, poly](int g0, int g1) {
        for (int g = g0; g < g1; ++g) {
            double* q = &c->quat[4 * (size_t)g];
            if (poly)
                for (int k = 0; k < 4; ++k) q[k] = c->poly_quat[4 * (size_t)(g - 1) + k];
            else
                euler2quaternion(&c->euler[3 * (size_t)(g - 1)], q);
        }
    };
    // each grain's conversion is independent (six trigonometric calls): large
    // inputs are split over up to 8 host threads, the same calls per grain
    const int nthreads =
        c->N >= 4096 ? (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    bool converted = false;
    if (nthreads > 1) {
        std::vector<std::thread> workers;
        try {
            const int per = (c->N + nthreads - 1) / nthreads;
            for (int t = 0; t < nthreads; ++t) {
                const int g0 = 1 + t * per, g1 = std::min(c->N + 1, g0 + per);
                if (g0 < g1) workers.emplace_back(convert, g0, g1);
            }
            converted = true;
        } catch (const std::system_error&) {
            converted = false;  // no threads: the rest below, on this one
        }
        for (std::thread& w : workers) w.join();
        if (!converted) convert(1, c->N + 1);
        converted = true;
    }
    if (!converted) convert(1, c->N + 1);
    auto present = [&](int g) {
        return poly ? c->poly_off[g] > c->poly_off[g - 1] : c->bbox[5 * (size_t)(g - 1) + 4] != 0;
    };
    const double csr_raw = P.constant_sector_radius, isr_raw = P.interpolating_sector_radius;
    c->ds = (csr_raw * 2 + isr_raw * 2) / double(realDomainSize);
    const unsigned long ppg_used =
        P.decouple_grains == 1 ? (unsigned long)P.number_of_points_per_grain : (unsigned long)c->ppg;
    c->dt = 0.8 / double(realDomainSize * realDomainSize) * ppg_used / 2 / 5.0;
    c->h = 1.0 / double(realDomainSize);
    // Stored elastic energies: each grain's value scaled as LSbox's voxel
    // constructor scales it (src/box.cpp:163-175), the domain boundary's
    // default value (src/box.cpp:35-43), and the time step shortened so that
    // the largest stored-energy difference moves a boundary by at most half a
    // grid spacing per step (grainhdl::read_HeaderCPG, src/grainhdl.cpp:404-460;
    // grainhdl::find_correctTimestepSize, 250-274).  Slot 0 is the boundary.
    std::vector<double>& stored_scaled = c->stored_scaled;
    stored_scaled.clear();
    double energy_delta_max = 0;  // grainhdl::m_Energy_deltaMAX
    bool correct_dt = false;
    if (P.use_stored_elastic_energy && poly) {
        // the contour constructor sets every grain's stored energy to 0
        // (src/box.cpp:115); the boundary keeps its default, and
        // m_Energy_deltaMAX is not computed for this input (it stays 0)
        const double D = P.dislocation_energy_per_m, H = P.hagb_energy, L = P.physical_domain_size;
        stored_scaled.assign((size_t)c->N + 1, 0.0);
        stored_scaled[0] = P.box_default_stored_elastic_energy;
        stored_scaled[0] *= D / H * L;
        correct_dt = true;
    } else if (P.use_stored_elastic_energy) {
        if (c->stored.size() != (size_t)c->N) return fail(c, GG_E_STATE, "no stored energies loaded");
        const double D = P.dislocation_energy_per_m, H = P.hagb_energy, L = P.physical_domain_size;
        stored_scaled.assign((size_t)c->N + 1, 0.0);
        stored_scaled[0] = P.box_default_stored_elastic_energy;
        stored_scaled[0] *= D / H * L;
        double lo = 1e20, hi = 0;
        for (int g = 1; g <= c->N; ++g) {
            const double v = c->stored[g - 1];
            if (std::fabs(v) < lo) lo = std::fabs(v);
            if (std::fabs(v) > hi) hi = std::fabs(v);
            stored_scaled[g] = v;
            stored_scaled[g] *= D / H * L;
        }
        if (std::fabs(stored_scaled[0]) / D * H / L < lo) lo = std::fabs(stored_scaled[0]) / D * H / L;
        if (std::fabs(stored_scaled[0]) / D * H / L > hi) hi = std::fabs(stored_scaled[0]) / D * H / L;
        if (c->N == 1) lo = 0.0;
        energy_delta_max = D * (hi - lo) / H * L;
        correct_dt = true;
    }
    // Magnetic energies (UseMagneticField): per grain from its orientation,
    // slot 0 the boundary's (identity orientation, src/box.cpp:35-49); their
    // range over grains 1 .. N-1 present (the reference's loop bound) replaces
    // the stored-energy difference (find_correctTimestepSize,
    // src/grainhdl.cpp:250-265).
    std::vector<double>& magnetic = c->magnetic;
    magnetic.clear();
    if (P.use_magnetic_field) {
        magnetic.assign((size_t)c->N + 1, 0.0);
        const double identity[4] = {1.0, 0.0, 0.0, 0.0};
        magnetic[0] = magnetic_energy(identity, P);
        for (int g = 1; g <= c->N; ++g) magnetic[g] = magnetic_energy(&c->quat[4 * (size_t)g], P);
        double lo = 1000000, hi = 0;
        for (int g = 1; g < c->N; ++g) {
            if (!present(g)) continue;  // absent grain (no LSbox)
            if (magnetic[g] < lo) lo = magnetic[g];
            if (magnetic[g] > hi) hi = magnetic[g];
        }
        if (c->N == 1) lo = 0.0;
        energy_delta_max = hi - lo;
        correct_dt = true;
    }
    c->energy_delta_max = energy_delta_max;
    c->ngrains_ref = c->N;
    if (correct_dt) {
        const double vmax = energy_delta_max * c->dt;
        double correction = 0.5 / (vmax / c->h);
        if (correction > 1.0) correction = 1.0;
        c->dt *= correction;
    }
    c->delta = (unsigned long)P.domain_border_size * 1 / double(realDomainSize);
    c->b = P.domain_border_size;
    c->m = realDomainSize + 2 * c->b;
    const int N = c->N, m = c->m, b = c->b;

    // boxes of the voxel constructor (src/box.cpp:156-217) or of the contour
    // constructor (src/box.cpp:108-159)
    std::vector<Box> box0(N + 1, Box{0, 0, 0, 0});
    std::vector<int32_t> state(N + 1, G_GONE);
    int maxn = 1;
    for (int g = 1; g <= N; ++g) {
        if (!present(g)) continue;  // zero-pixel grains and missing contours are skipped
        if (poly) {
            const double h = c->h;
            int xmax = 0, xmin = m, ymax = 0, ymin = xmin;
            for (int32_t k = c->poly_off[g - 1]; k < c->poly_off[g]; ++k) {
                const double x = c->poly_xy[2 * (size_t)k], y = c->poly_xy[2 * (size_t)k + 1];
                if (y / h < ymin) ymin = (int)(y / h);
                if (y / h > ymax) ymax = (int)(y / h);
                if (x / h < xmin) xmin = (int)(x / h);
                if (x / h > xmax) xmax = (int)(x / h);
            }
            xmax += 2 * b;
            ymax += 2 * b;
            if (ymax > m) ymax = m;
            if (xmax > m) xmax = m;
            box0[g] = host_resize_to_square(Box{xmin, xmax, ymin, ymax}, m);
            state[g] = G_EXISTS;
            maxn = std::max(maxn, box_w(box0[g]));
            continue;
        }
        const int32_t* q = &c->bbox[5 * (size_t)(g - 1)];
        int xmin = m, xmax = 0, ymin = m, ymax = 0;
        const int vx[4] = {q[0], q[0], q[1], q[1]}, vy[4] = {q[2], q[3], q[2], q[3]};
        for (int k = 0; k < 4; ++k) {
            if (vy[k] < ymin) ymin = vy[k];
            if (vy[k] > ymax) ymax = vy[k];
            if (vx[k] < xmin) xmin = vx[k];
            if (vx[k] > xmax) xmax = vx[k];
        }
        xmax += 2 * b;
        ymax += 2 * b;
        if (ymax > m) ymax = m;
        if (xmax > m) xmax = m;
        if (ymin < 0) ymin = 0;
        if (xmin < 0) xmin = 0;
        box0[g] = host_resize_to_square(Box{xmin, xmax, ymin, ymax}, m);
        state[g] = G_EXISTS;
        maxn = std::max(maxn, box_w(box0[g]));
    }
    const int tmax = std::min(m, std::max(160, 2 * maxn + 32));

    // offsets of the initial layout
    std::vector<int64_t> off(N + 1, 0), soff(N + 1, 0), coff(N + 1, 0);
    std::vector<int32_t> ccap(N + 1, 0);
    const int spc = P.precision == GG_PRECISION_PLAIN ? 2 : 1;
    int64_t a = 0, sp = 0, cc = 0;
    for (int g = 0; g <= N; ++g) {
        off[g] = a;
        soff[g] = sp;
        coff[g] = cc;
        if (g >= 1 && state[g] == G_EXISTS) {
            const int n = box_w(box0[g]);
            a += box_area(box0[g]);
            sp += (int64_t)spc * 2 * (int64_t)n * (n / 2 + 1);
            ccap[g] = contour_capacity(n);
            if (poly) ccap[g] = std::max(ccap[g], c->poly_off[g] - c->poly_off[g - 1]);
            cc += ccap[g];
        }
    }
    // arenas: twice the initial totals (and room for 2^20 more values), or
    // exactly arena_factor times them
    const double af = P.arena_factor;
    auto cap = [&](int64_t total, int64_t slack) {
        return af > 0 ? std::max<int64_t>(total, (int64_t)std::ceil(af * (double)total))
                      : std::max<int64_t>(2 * total, total + slack);
    };
    const int64_t phi_cap = cap(a, 1 << 20);
    const int64_t spec_cap = cap(sp, 1 << 20);
    const int64_t cont_cap = cap(cc, 1 << 16);
    const size_t rsz = P.precision == GG_PRECISION_PLAIN ? sizeof(double) : sizeof(float);

    // constant settings
    NetConst& C = c->C;
    C.N = N;
    C.m = m;
    C.b = b;
    C.nn = c->nn;
    C.kmax = P.list_capacity > 0 ? P.list_capacity : 96;
    C.nbmax = 48;
    C.jmax = 48;
    C.tmax = tmax;
    C.big_edge = 128;
    C.conv_smem_edge = 64;
    C.isotropic = P.is_isotropic_network ? 1 : 0;
    C.use_mobility_model = P.use_mobility_model;
    C.analysis_timestep = P.analysis_timestep;
    C.decouple = P.decouple_grains == 1 ? 1 : 0;
    C.h = c->h;
    C.delta = c->delta;
    C.dt = c->dt;
    C.csr = csr_raw * c->h;
    C.isr = isr_raw * c->h;
    C.ds = c->ds;
    C.tpd = P.triple_point_drag;
    C.theta_ref = P.theta_ref_deg * kPiH / 180.0;
    C.gamma_hagb = P.gamma_hagb;
    C.m_hagb = P.m_hagb;

    int rc;
#define ALLOC(ptr, cnt) \
    if ((rc = dalloc(c, &(ptr), (cnt))) != GG_OK) return rc
#define ALLOC_UNZEROED(ptr, cnt) \
    if ((rc = dalloc(c, &(ptr), (cnt), false)) != GG_OK) return rc
    ALLOC(C.state, N + 1);
    ALLOC(C.regular, N + 1);
    ALLOC(C.inter_bnd, N + 1);
    ALLOC(C.newbb, 4 * (size_t)(N + 1));
    ALLOC(C.volume, N + 1);
    ALLOC(C.energy, N + 1);
    ALLOC(C.perimeter, N + 1);
    ALLOC(C.meanda, N + 1);
    ALLOC(C.quat, 4 * (size_t)(N + 1));
    ALLOC(C.cmp_n, N + 1);
    ALLOC(C.cmp_ids, (size_t)C.kmax * (N + 1));
    ALLOC(C.sec_n, N + 1);
    ALLOC(C.sec_ids, (size_t)C.kmax * (N + 1));
    ALLOC(C.nb_n, N + 1);
    ALLOC(C.nb, (size_t)C.nbmax * (N + 1));
    ALLOC(C.gone_loop, N + 1);
    C.time_slope = P.time_slope;
    if (P.use_stored_elastic_energy) ALLOC(C.stored, N + 1);
    if (P.use_magnetic_field) ALLOC(C.magnetic, N + 1);
    GG_CUDA(c, cudaMemsetAsync(C.gone_loop, 0xff, sizeof(int32_t) * (N + 1), c->stream));

    // tables: twiddles and Gaussian multipliers (plain), separable kernels (batched)
    std::vector<int64_t> tw_off(tmax + 1, 0), gk_off(tmax + 1, 0), ck_off(tmax + 1, 0);
    int64_t twn = 0, gkn = 0, ckn = 0;
    for (int n = 1; n <= tmax; ++n) {
        tw_off[n] = twn;
        twn += n;
        gk_off[n] = gkn;
        gkn += (int64_t)(n / 2 + 1) * (n / 2 + 1);
        ck_off[n] = ckn;
        ckn += n + 1;  // k_n, then its band radius
    }
    const bool plain = P.precision == GG_PRECISION_PLAIN;
    std::vector<double> tw(plain ? 2 * twn : 2), gk(plain ? gkn : 1);
    std::vector<float> ck(plain ? 1 : ckn);
    if (plain)
        for (int n = 1; n <= tmax; ++n)
            for (int k = 0; k < n; ++k) twiddle(n, k, &tw[2 * (tw_off[n] + k)], &tw[2 * (tw_off[n] + k) + 1]);
    conv_tables(c, tmax, gk_off, ck_off, gk, ck);
    double* d_tw;
    double* d_gk;
    float* d_ck;
    int64_t *d_twoff, *d_gkoff, *d_ckoff;
    ALLOC(d_tw, tw.size());
    ALLOC(d_gk, gk.size());
    ALLOC(d_ck, ck.size());
    ALLOC(d_twoff, tmax + 1);
    ALLOC(d_gkoff, tmax + 1);
    ALLOC(d_ckoff, tmax + 1);
    GG_CUDA(c, cudaMemcpyAsync(d_tw, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice, c->stream));
    GG_CUDA(c, cudaMemcpyAsync(d_gk, gk.data(), sizeof(double) * gk.size(), cudaMemcpyHostToDevice, c->stream));
    GG_CUDA(c, cudaMemcpyAsync(d_ck, ck.data(), sizeof(float) * ck.size(), cudaMemcpyHostToDevice, c->stream));
    GG_CUDA(c, cudaMemcpyAsync(d_twoff, tw_off.data(), sizeof(int64_t) * (tmax + 1), cudaMemcpyHostToDevice,
                               c->stream));
    GG_CUDA(c, cudaMemcpyAsync(d_gkoff, gk_off.data(), sizeof(int64_t) * (tmax + 1), cudaMemcpyHostToDevice,
                               c->stream));
    GG_CUDA(c, cudaMemcpyAsync(d_ckoff, ck_off.data(), sizeof(int64_t) * (tmax + 1), cudaMemcpyHostToDevice,
                               c->stream));
    C.tw = d_tw;
    C.gk = d_gk;
    C.ck = d_ck;
    C.tw_off = d_twoff;
    C.gk_off = d_gkoff;
    C.ck_off = d_ckoff;

    // rotating state
    NetState& S = c->hS;
    std::memset(&S, 0, sizeof S);
    Box* boxes[3];
    int64_t* offs[3];
    int64_t* soffs[2];
    int64_t* coffs[3];
    int32_t* ccaps[3];
    for (int k = 0; k < 3; ++k) {
        ALLOC(boxes[k], N + 1);
        ALLOC(offs[k], N + 1);
        ALLOC(coffs[k], N + 1);
        ALLOC(ccaps[k], N + 1);
    }
    for (int k = 0; k < 2; ++k) ALLOC(soffs[k], N + 1);
    S.box_prev = boxes[0];
    S.box_cur = boxes[1];
    S.box_new = boxes[2];
    S.off_prev = offs[0];
    S.off_cur = offs[1];
    S.off_new = offs[2];
    S.soff_cur = soffs[0];
    S.soff_new = soffs[1];
    S.coff_prev = coffs[0];
    S.coff_cur = coffs[1];
    S.coff_new = coffs[2];
    S.ccap_prev = ccaps[0];
    S.ccap_cur = ccaps[1];
    S.ccap_new = ccaps[2];
    if (plain) {
        double *pa, *pb, *sp_;
        ALLOC(pa, phi_cap);
        ALLOC(pb, phi_cap);
        ALLOC(sp_, spec_cap);
        S.phiA = pa;
        S.phiB = pb;
        S.spec = sp_;
        if (c->tangents) {  // zero tangents: the initial field does not depend on the parameters
            double *da, *db;
            ALLOC(da, 4 * (size_t)phi_cap);
            ALLOC(db, 4 * (size_t)phi_cap);
            S.dphiA = da;
            S.dphiB = db;
            ALLOC(C.dvol, 4 * (size_t)(N + 1));
            ALLOC(S.dcontPrev, 8 * (size_t)cont_cap);
            ALLOC(S.dcontCur, 8 * (size_t)cont_cap);
            ALLOC(C.dseg, 4 * (size_t)cont_cap);
        }
    } else {
        float *pa, *pb, *sp_;
        ALLOC_UNZEROED(pa, phi_cap);  // fields and the convolution's scratch: read only inside written boxes
        ALLOC_UNZEROED(pb, phi_cap);
        ALLOC_UNZEROED(sp_, spec_cap);
        S.phiA = pa;
        S.phiB = pb;
        S.spec = sp_;
        // sectors built one step ahead for the corrector
        char* pk;
        ALLOC(pk, batched_sector_pack_bytes() * (size_t)(N + 1));
        C.secpack = pk;
        ALLOC(C.segsec, cont_cap);
        ALLOC(C.segacc, cont_cap);
        c->sectors_stale = true;
    }
    (void)rsz;
    ALLOC(S.idPrev, phi_cap);
    ALLOC(S.idCur, phi_cap);
    ALLOC_UNZEROED(S.contPrev, cont_cap);  // contour data: read up to the written counts
    ALLOC_UNZEROED(S.contCur, cont_cap);
    ALLOC_UNZEROED(S.segPrev, cont_cap);
    {
        double* pt;
        ALLOC_UNZEROED(pt, 4 * (size_t)cont_cap);  // PointInfo: 32 bytes per contour point
        C.ptinfo = pt;
    }
    ALLOC(S.cn_prev, N + 1);
    ALLOC(S.cn_cur, N + 1);
    ALLOC(S.jPrev, (size_t)C.jmax * (N + 1));
    ALLOC(S.jCur, (size_t)C.jmax * (N + 1));
    ALLOC(S.jn_prev, N + 1);
    ALLOC(S.jn_cur, N + 1);
    S.phi_cap = phi_cap;
    S.spec_cap = spec_cap;
    S.cont_cap = cont_cap;
    S.loop = P.start_time;
    if (!plain) ALLOC(S.order, N + 1);  // the batched step's work queue
    if (!plain) ALLOC(S.big_flag, N + 1);  // grains for the large-contour corrector
    if (!plain) ALLOC(S.big_list, N + 1);
    ALLOC(c->dS, 1);

#undef ALLOC
#undef ALLOC_UNZEROED

    // initial per-grain data
    const std::vector<double>& quat = c->quat;
    std::vector<int32_t> ones(N + 1, 1);
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
    };
    for (int k = 0; k < 3; ++k) {
        GG_CUDA(c, h2d(boxes[k], box0.data(), sizeof(Box) * (N + 1)));
        GG_CUDA(c, h2d(offs[k], off.data(), sizeof(int64_t) * (N + 1)));
        GG_CUDA(c, h2d(coffs[k], coff.data(), sizeof(int64_t) * (N + 1)));
        GG_CUDA(c, h2d(ccaps[k], ccap.data(), sizeof(int32_t) * (N + 1)));
    }
    GG_CUDA(c, h2d(soffs[0], soff.data(), sizeof(int64_t) * (N + 1)));
    GG_CUDA(c, h2d(C.state, state.data(), sizeof(int32_t) * (N + 1)));
    GG_CUDA(c, h2d(C.regular, ones.data(), sizeof(int32_t) * (N + 1)));
    GG_CUDA(c, h2d(C.quat, quat.data(), sizeof(double) * quat.size()));
    if (C.stored) GG_CUDA(c, h2d(C.stored, stored_scaled.data(), sizeof(double) * stored_scaled.size()));
    if (C.magnetic) GG_CUDA(c, h2d(C.magnetic, magnetic.data(), sizeof(double) * magnetic.size()));

    S.phi_used = a;
    S.spec_used = sp;
    S.cont_used = cc;
    GG_CUDA(c, h2d(c->dS, &S, sizeof(NetState)));

    if (!plain) GG_CUDA(c, batched_prepare(tmax));
    if (poly) {
        // the loaded polygon is the grain's contour until the first level-set
        // stage (energy and mobility 0, no junctions); its area is
        // computeVolume / h^2 (src/box.cpp:396-397, src/grainBoundary.cpp:201-213)
        std::vector<CPoint> pts((size_t)std::max<int64_t>(cc, 1), CPoint{0, 0, 0, 0});
        std::vector<int32_t> cn(N + 1, 0);
        std::vector<double> vol(N + 1, 0.0);
        for (int g = 1; g <= N; ++g) {
            if (state[g] != G_EXISTS) continue;
            const int32_t k0 = c->poly_off[g - 1], np = c->poly_off[g] - k0;
            for (int32_t k = 0; k < np; ++k)
                pts[coff[g] + k] = CPoint{c->poly_xy[2 * (size_t)(k0 + k)], c->poly_xy[2 * (size_t)(k0 + k) + 1], 0, 0};
            cn[g] = np;
            double v = 0;
            for (int32_t k = 0; k + 1 < np; ++k) {
                const CPoint& p0 = pts[coff[g] + k];
                const CPoint& p1 = pts[coff[g] + k + 1];
                v += (p0.y + p1.y) * (p0.x - p1.x);
            }
            v = std::fabs(v) * c->h * c->h * 0.5;
            vol[g] = v / (c->h * c->h);
        }
        GG_CUDA(c, h2d(S.contPrev, pts.data(), sizeof(CPoint) * (size_t)cc));
        GG_CUDA(c, h2d(S.cn_prev, cn.data(), sizeof(int32_t) * (N + 1)));
        GG_CUDA(c, h2d(C.volume, vol.data(), sizeof(double) * (N + 1)));
        GG_CUDA(c, plain ? plain_init_polygon(C, c->dS, c->stream) : batched_init_polygon(C, c->dS, c->stream));
    } else {
        GG_CUDA(c, plain ? plain_init(C, c->dS, c->d_ids, c->stream) : batched_init(C, c->dS, c->d_ids, c->stream));
    }
    GG_CUDA(c, finalize_only(C, c->dS, 0, c->stream));
    if (!plain) GG_CUDA(c, batched_order(C, c->dS, c->stream));
    if (!plain) apply_cached_tuning(c);
    rc = check_status(c);
    if (rc != GG_OK) return rc;
    c->initialised = true;
    c->dt_from.assign(1, std::make_pair((int)P.start_time, c->dt));
    return refresh_state(c);
}

int gg_find_neighbors(gg_ctx* c) {
    if (!c) return GG_E_INVALID;
    c->stats_fresh = false;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    c->sectors_stale = c->P.precision != GG_PRECISION_PLAIN;  // junction weights read the neighbour lists
    // the grains binned by the cells their boxes cover: counts and starts,
    // then the binned IDs, sized by the count read back
    const int nc = c->C.m / kNeighbourBin + 1;
    int rc;
    if (nc > c->nbin_nc) {
        if ((rc = dalloc(c, &c->nbin_count, (size_t)nc * nc)) != GG_OK) return rc;
        if ((rc = dalloc(c, &c->nbin_start, (size_t)nc * nc + 1)) != GG_OK) return rc;
        if ((rc = dalloc(c, &c->nbin_total, 1)) != GG_OK) return rc;
        c->nbin_nc = nc;
    }
    NeighbourBins B{nc, c->nbin_count, c->nbin_start, c->nbin_items, c->nbin_total};
    GG_CUDA(c, neighbour_bins_count(c->C, c->dS, B, c->stream));
    int total = 0;
    GG_CUDA(c, cudaMemcpyAsync(&total, c->nbin_total, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (total > c->nbin_items_cap || !c->nbin_items) {
        if ((rc = dalloc(c, &c->nbin_items, (size_t)std::max(total, 1))) != GG_OK) return rc;
        c->nbin_items_cap = std::max(total, 1);
    }
    B.items = c->nbin_items;
    GG_CUDA(c, find_neighbors_launch(c->C, c->dS, B, c->stream));
    return check_status(c);
}

int gg_set_neighbours(gg_ctx* c, const int32_t* offsets, const int32_t* ids) {
    if (!c || !offsets || !ids) return GG_E_INVALID;
    c->stats_fresh = false;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    const int N = c->N, K = c->C.kmax;
    c->sectors_stale = c->P.precision != GG_PRECISION_PLAIN;
    std::vector<int32_t> sec((size_t)K * (N + 1), 0), n(N + 1, 0), zero(N + 1, 0);
    std::vector<Neighbour> nb((size_t)c->C.nbmax * (N + 1));
    std::vector<int32_t> nbn(N + 1, 0);
    for (int g = 1; g <= N; ++g) {
        const int a = offsets[g - 1], e = offsets[g];
        if (e - a > K) return fail(c, GG_E_CAPACITY, "neighbour list longer than the list capacity");
        for (int k = a; k < e; ++k) {
            if (ids[k] < 1 || ids[k] > N) return fail(c, GG_E_INVALID, "neighbour ID out of range");
            sec[(size_t)g * K + (k - a)] = ids[k];
            if (k - a < c->C.nbmax) {
                Neighbour& q = nb[(size_t)g * c->C.nbmax + (k - a)];
                q.id = ids[k];
                q.length = q.energy = q.misori = q.mobility = 0;
                nbn[g]++;
            }
        }
        n[g] = e - a;
    }
    GG_CUDA(c, cudaMemcpyAsync(c->C.sec_ids, sec.data(), sizeof(int32_t) * sec.size(), cudaMemcpyHostToDevice,
                               c->stream));
    GG_CUDA(c, cudaMemcpyAsync(c->C.sec_n, n.data(), sizeof(int32_t) * n.size(), cudaMemcpyHostToDevice, c->stream));
    GG_CUDA(c, cudaMemcpyAsync(c->C.cmp_n, zero.data(), sizeof(int32_t) * zero.size(), cudaMemcpyHostToDevice,
                               c->stream));
    GG_CUDA(c, cudaMemcpyAsync(c->C.nb, nb.data(), sizeof(Neighbour) * nb.size(), cudaMemcpyHostToDevice,
                               c->stream));
    GG_CUDA(c, cudaMemcpyAsync(c->C.nb_n, nbn.data(), sizeof(int32_t) * nbn.size(), cudaMemcpyHostToDevice,
                               c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    return GG_OK;
}

namespace {
int run_stage(gg_ctx* c, int stages, bool setloop, int loop) {
    if (!c) return GG_E_INVALID;
    c->stats_fresh = false;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    if (setloop) {
        int r = set_loop(c, loop);
        if (r) return r;
    }
    int r = launch_stages(c, stages);
    if (r) return r;
    return check_status(c);
}
}  // namespace

int gg_convolution(gg_ctx* c, int32_t loop) {
    if (!c) return GG_E_INVALID;
    c->stats_fresh = false;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    bool coarsened = false;
    const int rc = coarsen_if_due(c, loop, &coarsened);  // the first stage of a loop (src/grainhdl.cpp:1053)
    if (rc) return rc;
    return run_stage(c, ST_CONV, true, loop);
}
int gg_update_second_order_neighbors(gg_ctx* c) { return run_stage(c, ST_SECOND, false, 0); }
int gg_comparison(gg_ctx* c) { return run_stage(c, ST_COMPARE, false, 0); }
int gg_level_set(gg_ctx* c, int32_t loop) { return run_stage(c, ST_LEVELSET, true, loop); }
int gg_redistancing(gg_ctx* c, int32_t loop) { return run_stage(c, ST_REDIST, true, loop); }

int gg_grain_count(gg_ctx* c, int32_t* current, double* max_volume) {
    if (!c) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    int rc = refresh_state(c);
    if (rc) return rc;
    if (current) *current = c->hS.live;
    if (max_volume) *max_volume = c->hS.max_volume;
    return GG_OK;
}

int gg_step(gg_ctx* c, int32_t loop, int32_t nsteps);

int gg_autotune(gg_ctx* c, int32_t loop, int32_t steps_per_candidate, gg_tuning* out) {
    if (!c || !out) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    std::memset(out, 0, sizeof *out);
    if (c->P.precision == GG_PRECISION_PLAIN) {  // the plain form has no bins to tune
        out->compare_threads = c->cfg.compare_threads;
        return GG_OK;
    }
    const int k = steps_per_candidate > 0 ? steps_per_candidate : 2;
    int steps = 0;
    // device ms per step of the current bins over k steps (a fresh graph
    // for every candidate; capture is outside the timed region)
    auto measure = [&](double* ms) -> int {
        if (c->graph) {
            cudaGraphExecDestroy(c->graph);
            c->graph = nullptr;
        }
        double total = 0;
        for (int s = 0; s < k; ++s) {
            const int rc = gg_step(c, loop + steps, 1);
            if (rc) return rc;
            total += c->last_ms;
            ++steps;
        }
        *ms = total / k;
        return GG_OK;
    };
    double best = 0;
    int rc = measure(&best);
    if (rc) return rc;
    out->ms_default = best;
    // one knob at a time; a candidate replaces the current value only when
    // it is faster by more than 1% (the network changes a little between the
    // steps the candidates run on)
    auto tune = [&](int* knob, std::initializer_list<int> cands) -> int {
        const int keep = *knob;
        int chosen = keep;
        for (int v : cands) {
            if (v == keep) continue;
            *knob = v;
            double ms = 0;
            const int r = measure(&ms);
            if (r) return r;
            if (ms < 0.99 * best) {
                best = ms;
                chosen = v;
            }
        }
        *knob = chosen;
        return GG_OK;
    };
    if ((rc = tune(&c->C.big_edge, {64, 96, 128, 192, 1 << 20})) != GG_OK) return rc;
    if ((rc = tune(&c->cfg.compare_threads, {128, 256})) != GG_OK) return rc;  // k_compare: at most 256
    if ((rc = tune(&c->C.conv_smem_edge, {48, 64, 96, 128})) != GG_OK) return rc;
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[{c->C.tmax, c->N}] = TunedBins{c->cfg.compare_threads, c->C.big_edge, c->C.conv_smem_edge};
    }
    out->compare_threads = c->cfg.compare_threads;
    out->big_edge = c->C.big_edge;
    out->conv_smem_edge = c->C.conv_smem_edge;
    out->steps_run = steps;
    out->ms_tuned = best;
    return GG_OK;
}

int gg_step(gg_ctx* c, int32_t loop, int32_t nsteps) {
    if (!c) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    if (nsteps <= 0) return GG_OK;
    c->stats_fresh = false;
    if (c->P.grid_coarsement && nsteps > 1) {
        // the coarsening test needs the grain count between steps
        double total = 0;
        for (int s = 0; s < nsteps; ++s) {
            const int rs = gg_step(c, loop + s, 1);
            if (rs) return rs;
            total += c->last_ms;
        }
        c->last_ms = total;
        return GG_OK;
    }
    bool coarsened = false;
    int rc = coarsen_if_due(c, loop, &coarsened);
    if (rc) return rc;
    rc = set_loop(c, loop);
    if (rc) return rc;
    if (c->P.precision == GG_PRECISION_BATCHED) {
        if (!c->graph) {
            cudaGraph_t gr;
            GG_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = batched_step_graph(c->C, c->dS, c->stream, c->stream2, c->fork, c->cfg);
            cudaError_t e2 = cudaStreamEndCapture(c->stream, &gr);
            if (e != cudaSuccess) return cuda_fail(c, e, "capture");
            if (e2 != cudaSuccess) return cuda_fail(c, e2, "end capture");
            size_t nn = 0;
            e = cudaGraphGetNodes(gr, nullptr, &nn);
            std::vector<cudaGraphNode_t> nodes(nn);
            if (e == cudaSuccess && nn) e = cudaGraphGetNodes(gr, nodes.data(), &nn);
            int32_t kn = 0;
            for (size_t q = 0; q < nn && e == cudaSuccess; ++q) {
                cudaGraphNodeType t;
                e = cudaGraphNodeGetType(nodes[q], &t);
                if (t == cudaGraphNodeTypeKernel) ++kn;
            }
            // per-node priorities: the large-contour corrector's CTAs go first
            if (e == cudaSuccess) e = cudaGraphInstantiate(&c->graph, gr, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(gr);
            if (e != cudaSuccess) return cuda_fail(c, e, "graph instantiate");
            c->graph_kernels = kn;
        }
        if (c->sectors_stale) {
            GG_CUDA(c, batched_sectors(c->C, c->dS, c->stream));
            c->sectors_stale = false;
        }
        GG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
        for (int s = 0; s < nsteps; ++s) GG_CUDA(c, cudaGraphLaunch(c->graph, c->stream));
        GG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
        c->kernel_launches += (int64_t)nsteps * c->graph_kernels;
    } else {
        GG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
        for (int s = 0; s < nsteps; ++s) {
            rc = launch_stages(c, ST_ALL);
            if (rc) return rc;
        }
        GG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    }
    if (c->stats_wanted && c->d_stats && c->h_stats) {
        // after the timed region: the statistics and the status word in one
        // pinned copy each, then one wait for all of it
        if (!c->h_status) GG_CUDA(c, pinned_take(reinterpret_cast<void**>(&c->h_status), sizeof(uint32_t)));
        if (!c->ev_done) GG_CUDA(c, cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming));
        GG_CUDA(c, pack_stats(c->C, c->dS, c->d_stats, c->stream));
        GG_CUDA(c, cudaMemcpyAsync(c->h_stats, c->d_stats, sizeof(gg_grain_stats) * (size_t)c->N,
                                   cudaMemcpyDeviceToHost, c->stream));
        GG_CUDA(c, cudaMemcpyAsync(c->h_status, &c->dS->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        GG_CUDA(c, cudaEventRecord(c->ev_done, c->stream));
        GG_CUDA(c, cudaEventSynchronize(c->ev_done));
        float ms = 0;
        GG_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        c->last_ms = ms;
        const int rc2 = status_error(c, *c->h_status);
        if (rc2 == GG_OK) c->stats_fresh = true;
        return rc2;
    }
    GG_CUDA(c, cudaEventSynchronize(c->ev1));
    float ms = 0;
    GG_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms = ms;
    return check_status(c);
}

int gg_status(gg_ctx* c, uint32_t* status, int32_t clear) {
    if (!c || !status) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    GG_CUDA(c, cudaMemcpyAsync(status, &c->dS->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (clear) GG_CUDA(c, cudaMemsetAsync(&c->dS->status, 0, sizeof(uint32_t), c->stream));
    return GG_OK;
}

int gg_grain_updates(gg_ctx* c, int64_t* updates) {
    if (!c || !updates) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    int rc = refresh_state(c);
    if (rc) return rc;
    *updates = (int64_t)c->hS.updates;
    return GG_OK;
}

int gg_profile_steps(gg_ctx* c, int32_t loop, int32_t nsteps, double* stage_ms) {
    if (!c || !stage_ms) return GG_E_INVALID;
    c->stats_fresh = false;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    if (c->tangents) return fail(c, GG_E_STATE, "stage profiling runs without tangents");
    int rc = set_loop(c, loop);
    if (rc) return rc;
    const bool plain = c->P.precision == GG_PRECISION_PLAIN;
    if (!plain && c->sectors_stale) {
        GG_CUDA(c, batched_sectors(c->C, c->dS, c->stream));
        c->sectors_stale = false;
    }
    cudaEvent_t ev[GG_NSTAGES + 1];
    for (int k = 0; k <= GG_NSTAGES; ++k) GG_CUDA(c, cudaEventCreate(&ev[k]));
    for (int s = 0; s < nsteps; ++s) {
        GG_CUDA(c, cudaEventRecord(ev[0], c->stream));
        for (int k = 0; k < GG_NSTAGES; ++k) {
            GG_CUDA(c, plain ? plain_stage_kernel(c->C, c->dS, k, c->stream, c->cfg)
                             : batched_stage_kernel(c->C, c->dS, k, c->stream, c->cfg));
            GG_CUDA(c, cudaEventRecord(ev[k + 1], c->stream));
        }
        GG_CUDA(c, cudaEventSynchronize(ev[GG_NSTAGES]));
        for (int k = 0; k < GG_NSTAGES; ++k) {
            float ms = 0;
            GG_CUDA(c, cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            stage_ms[k] += ms;
        }
    }
    for (int k = 0; k <= GG_NSTAGES; ++k) cudaEventDestroy(ev[k]);
    return check_status(c);
}

int gg_traffic(gg_ctx* c, int64_t* sum_area, int64_t* sum_overlap, int32_t* n_exists) {
    if (!c) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    unsigned long long z[3] = {0, 0, 0};
    GG_CUDA(c, cudaMemcpyAsync(&c->dS->t_area, z, sizeof z, cudaMemcpyHostToDevice, c->stream));
    GG_CUDA(c, traffic_launch(c->C, c->dS, c->stream));
    int rc = refresh_state(c);
    if (rc) return rc;
    if (sum_area) *sum_area = (int64_t)c->hS.t_area;
    if (sum_overlap) *sum_overlap = (int64_t)c->hS.t_overlap;
    if (n_exists) *n_exists = (int32_t)c->hS.t_exists;
    return GG_OK;
}

int gg_kernel_launches(gg_ctx* c, int64_t* total, int32_t* per_step) {
    if (!c || !total) return GG_E_INVALID;
    *total = c->kernel_launches;
    if (per_step) *per_step = c->graph_kernels;
    return GG_OK;
}

int gg_last_step_ms(gg_ctx* c, double* ms) {
    if (!c || !ms) return GG_E_INVALID;
    *ms = c->last_ms;
    return GG_OK;
}

int gg_dims(gg_ctx* c, int32_t* n_grains, int32_t* ngridpoints, double* h, double* delta, double* dt) {
    if (!c) return GG_E_INVALID;
    if (n_grains) *n_grains = c->N;
    if (ngridpoints) *ngridpoints = c->m;
    if (h) *h = c->h;
    if (delta) *delta = c->delta;
    if (dt) *dt = c->dt;
    return GG_OK;
}

int gg_tangent_enable(gg_ctx* c, int32_t enable) {
    if (!c) return GG_E_INVALID;
    if (c->initialised) return fail(c, GG_E_STATE, "tangents must be enabled before gg_distance_initialisation");
    if (enable && c->P.precision != GG_PRECISION_PLAIN)
        return fail(c, GG_E_INVALID, "tangents need the plain (FP64) form");
    if (enable && (c->P.use_stored_elastic_energy || c->P.use_magnetic_field))
        return fail(c, GG_E_INVALID, "tangents do not cover the stored-energy or magnetic driving force");
    if (enable && c->P.grid_coarsement) return fail(c, GG_E_INVALID, "tangents do not cover grid coarsening");
    c->tangents = enable != 0;
    return GG_OK;
}

int gg_read_area_tangents(gg_ctx* c, double* out, int32_t capacity) {
    if (!c || !out) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    if (!c->tangents || !c->C.dvol) return fail(c, GG_E_STATE, "tangents not enabled");
    const int N = c->N;
    if (capacity < 4 * N) return fail(c, GG_E_INVALID, "capacity smaller than 4 x grain count");
    std::vector<double> dv(4 * (size_t)(N + 1));
    GG_CUDA(c, cudaMemcpyAsync(dv.data(), c->C.dvol, sizeof(double) * dv.size(), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    const double per_degree = kPiH / 180.0;  // the kernels differentiate in radians
    for (int g = 1; g <= N; ++g) {
        out[4 * (g - 1) + 0] = dv[4 * (size_t)g + 0] * per_degree;
        for (int k = 1; k < 4; ++k) out[4 * (g - 1) + k] = dv[4 * (size_t)g + k];
    }
    return GG_OK;
}

int gg_write_analysis(gg_ctx* c, const char* directory, int32_t loop) {
    if (!c || !directory) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    int rc = refresh_state(c);
    if (rc) return rc;
    if (loop < c->P.start_time || c->hS.loop != loop + 1)
        return fail(c, GG_E_STATE, "loop is not the last completed step");
    const int N = c->N;
    const bool aniso = c->P.is_isotropic_network == 0;
    const NetConst& C = c->C;
    std::vector<int32_t> state(N + 1), reg(N + 1), bnd(N + 1), nbn(N + 1), gone(N + 1);
    std::vector<double> vol(N + 1), en(N + 1), per(N + 1), mda(N + 1);
    std::vector<Neighbour> nb;
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    };
    GG_CUDA(c, d2h(state.data(), C.state, 4 * (N + 1)));
    GG_CUDA(c, d2h(reg.data(), C.regular, 4 * (N + 1)));
    GG_CUDA(c, d2h(bnd.data(), C.inter_bnd, 4 * (N + 1)));
    GG_CUDA(c, d2h(nbn.data(), C.nb_n, 4 * (N + 1)));
    GG_CUDA(c, d2h(gone.data(), C.gone_loop, 4 * (N + 1)));
    GG_CUDA(c, d2h(vol.data(), C.volume, 8 * (N + 1)));
    GG_CUDA(c, d2h(en.data(), C.energy, 8 * (N + 1)));
    GG_CUDA(c, d2h(per.data(), C.perimeter, 8 * (N + 1)));
    GG_CUDA(c, d2h(mda.data(), C.meanda, 8 * (N + 1)));
    if (c->P.discrete_sampling_rate > 0) {
        nb.resize((size_t)C.nbmax * (N + 1));
        GG_CUDA(c, d2h(nb.data(), C.nb, sizeof(Neighbour) * nb.size()));
    }
    GG_CUDA(c, cudaStreamSynchronize(c->stream));

    const std::string dir(directory);
    const std::string tex_path = dir + "/Texture_" + std::to_string(loop) + ".ori";
    const std::string modf_path = dir + "/MODF_" + std::to_string(loop) + ".txt";
    const std::string stats_path = dir + "/NrGrains&EnergyStatistics.txt";
    std::ofstream tex(tex_path);
    if (!tex) return fail(c, GG_E_IO, "cannot write " + tex_path);
    // save_Texture (src/grainhdl.cpp:871-1023): one line per existing grain
    // with regular motion; the MODF takes half of each boundary length in the
    // bin of its misorientation and is renormalised to unit sum after every
    // grain.
    const int nbins = c->P.discrete_sampling_rate;
    const double dh = 62.8 / (double)nbins;  // LatticeType 0
    std::vector<double> modf(nbins, 0.0);
    double total_energy = 0.0;
    for (int g = 1; g <= N; ++g) {
        if (state[g] != G_EXISTS || reg[g] == 0) continue;
        total_energy += en[g];
        double eul[3];
        quaternion2euler(&c->quat[4 * (size_t)g], eul);
        if (nbins > 0) {
            // ExplicitGrainBoundary::calculateDiscreteEnergyDistribution
            // (src/grainBoundary.cpp:578-598): lengths summed per bin in
            // neighbour order, bins visited in ascending order
            std::vector<std::pair<int, double>> local;
            const Neighbour* L = nb.data() + (size_t)g * C.nbmax;
            for (int e = 0; e < nbn[g]; ++e) {
                const int key = (int)((L[e].misori * 180 / kPiH) / dh - 0.5);
                auto it = std::find_if(local.begin(), local.end(), [&](const auto& kv) { return kv.first == key; });
                if (it == local.end()) local.emplace_back(key, L[e].length);
                else it->second += L[e].length;
            }
            std::sort(local.begin(), local.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            for (const auto& kv : local)
                if (kv.first >= 0 && kv.first < nbins) modf[kv.first] += kv.second / 2;
        }
        tex << g << '\t' << nbn[g] << '\t' << (bnd[g] != 0) << '\t' << vol[g] << '\t'
            << mda[g] / (double)c->P.analysis_timestep << '\t' << per[g] << '\t' << en[g] << '\t'
            << (!c->magnetic.empty() ? c->magnetic[g] : c->stored_scaled.empty() ? 0.0 : c->stored_scaled[g])
            << '\t' << eul[0] << '\t' << eul[1] << '\t' << eul[2] << std::endl;
        double sum = 0.0;
        for (int i = 0; i < nbins; ++i) sum += modf[i];
        for (int i = 0; i < nbins; ++i)
            if (modf[i] > 0) modf[i] = modf[i] / sum;
    }
    tex.close();
    FILE* mf = std::fopen(modf_path.c_str(), "w");
    if (!mf) return fail(c, GG_E_IO, "cannot write " + modf_path);
    if (aniso)
        for (int i = 0; i < nbins; ++i) std::fprintf(mf, "%lf\t%lf\n", (float)(dh * (i + 1)), (float)modf[i]);
    std::fclose(mf);

    // save_NrGrainsStats (src/grainhdl.cpp:1225-1241): simulated time before
    // this step's increment (src/grainhdl.cpp:1115-1117), grains present when
    // the step began (get_biggestGrainVol of the previous step,
    // src/grainhdl.cpp:1744-1754: vanished grains count until the next level
    // set deletes them), total energy, grid size
    int nr = 0;
    for (int g = 1; g <= N; ++g) nr += (state[g] != G_GONE || gone[g] == loop) ? 1 : 0;
    // each step adds the increment of its own time step (which a coarsening changes)
    double realtime = 0.0;
    for (int l = c->P.start_time; l < loop; ++l) {
        double dt = c->dt_from.front().second;
        for (const auto& seg : c->dt_from)
            if (seg.first <= l) dt = seg.second;
        realtime += (dt * (c->P.physical_domain_size * c->P.physical_domain_size) /
                     (c->P.time_slope * c->P.hagb_energy * c->P.hagb_mobility));
    }
    std::ofstream st(stats_path, loop == 0 ? std::ios::out : std::ios::app);
    if (!st) return fail(c, GG_E_IO, "cannot write " + stats_path);
    st << realtime << "\t" << nr << "\t" << 0.5 * total_energy << "\t" << c->nn << std::endl;
    return GG_OK;
}

int gg_write_restart(gg_ctx* c, const char* directory, int32_t loop) {
    if (!c || !directory) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    int rc = refresh_state(c);
    if (rc) return rc;
    if (loop < c->P.start_time || c->hS.loop != loop + 1)
        return fail(c, GG_E_STATE, "loop is not the last completed step");
    const int N = c->N;
    const NetState& S = c->hS;
    std::vector<int32_t> state(N + 1), gone(N + 1), cn(N + 1);
    std::vector<int64_t> coff(N + 1);
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    };
    GG_CUDA(c, d2h(state.data(), c->C.state, 4 * (N + 1)));
    GG_CUDA(c, d2h(gone.data(), c->C.gone_loop, 4 * (N + 1)));
    GG_CUDA(c, d2h(cn.data(), S.cn_prev, 4 * (N + 1)));
    GG_CUDA(c, d2h(coff.data(), S.coff_prev, 8 * (N + 1)));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    // the latest contours (rotated into the previous-contour arena at the end
    // of the step), copied as one range
    int64_t lo = INT64_MAX, hi = 0;
    for (int g = 1; g <= N; ++g)
        if (state[g] == G_EXISTS && cn[g] > 0) {
            lo = std::min(lo, coff[g]);
            hi = std::max(hi, coff[g] + cn[g]);
        }
    std::vector<CPoint> pts(hi > lo ? (size_t)(hi - lo) : 0);
    if (!pts.empty()) {
        GG_CUDA(c, d2h(pts.data(), S.contPrev + lo, sizeof(CPoint) * pts.size()));
        GG_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    int nr = 0;  // grains present when the step began (as in gg_write_analysis)
    for (int g = 1; g <= N; ++g) nr += (state[g] != G_GONE || gone[g] == loop) ? 1 : 0;
    const std::string tail = "_TIMESTEP_" + std::to_string(loop) + "_GRAINS_" + std::to_string(nr);
    const std::string dat_name = "NETWORK_NONAME" + tail + ".dat";
    const std::string dir(directory);
    // LSbox::plot_full_grain (src/box.cpp:1552-1596): domain coordinates,
    // except after step 0 of a contour input, where the reference prints the
    // grid coordinates as they are (src/grainhdl.cpp:1194-1198)
    std::ofstream dat(dir + "/" + dat_name);
    if (!dat) return fail(c, GG_E_IO, "cannot write " + dir + "/" + dat_name);
    const double h = c->h;
    const int blowup = c->b;
    const bool absolute = loop != 0 || !c->contour_input;
    for (int g = 1; g <= N; ++g) {
        if (state[g] != G_EXISTS) continue;
        const double* q = &c->quat[4 * (size_t)g];
        dat << g << "\t" << cn[g] << "\t" << q[0] << "\t" << q[1] << "\t" << q[2] << "\t" << q[3] << std::endl;
        for (int k = 0; k < cn[g]; ++k) {
            const CPoint& p = pts[(size_t)(coff[g] - lo + k)];
            if (absolute)
                dat << (p.x - blowup) * h << "\t" << (p.y - blowup) * h << std::endl;
            else
                dat << p.x << "\t" << p.y << std::endl;
        }
        dat << std::endl;
    }
    dat.close();
    // Settings::generateXMLParametersNode (src/Settings.cpp:363-400), printed
    // as rapidxml prints a document: one tab-indented element per line
    const gg_params& P = c->P;
    std::ostringstream x;
    auto tag = [&](const char* name, const auto& value) { x << "\t<" << name << ">" << value << "</" << name << ">\n"; };
    auto flag = [](int v) { return v != 0 ? 1 : 0; };
    x << "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n<Parameters>\n";
    tag("StartTime", loop);
    tag("NumberOfParticles", nr);
    tag("NumberOfPointsPerGrain", c->ppg);  // from the grid in mode 4 (src/grainhdl.cpp:331), else as given
    tag("AnalysisTimestep", P.analysis_timestep);
    tag("PlotInterval", P.plot_interval);
    tag("NumberOfTimesteps", P.number_of_timesteps);
    tag("BreakupNumber", P.breakup_number);
    tag("DiscreteSamplingRate", P.discrete_sampling_rate);
    tag("DomainBorderSize", P.domain_border_size);
    tag("MicrostructureGenMode", 0);
    tag("ReadFromFilename", dat_name);
    tag("HAGB_Energy", P.hagb_energy);
    tag("HAGB_Mobility", P.hagb_mobility);
    tag("Physical_Domain_Size", P.physical_domain_size);
    tag("TriplePointDrag", P.triple_point_drag);
    tag("UseMobilityModel", P.use_mobility_model);
    tag("IdentifyTwins", flag(P.identify_twins));
    tag("IsIsotropicNetwork", flag(P.is_isotropic_network));
    tag("UseTexture", flag(P.use_texture));
    tag("ExecuteInParallel", flag(P.execute_in_parallel));
    tag("MaximumNumberOfThreads", P.maximum_number_of_threads);
    tag("GridCoarsement", flag(P.grid_coarsement));
    tag("GridCoarsementGradient", P.grid_coarsement_gradient);
    tag("ConvolutionMode", P.convolution_mode);
    tag("ResearchMode", flag(P.research_mode));
    tag("ResearchProject", P.research_project);
    // scaled by h at set-up (src/grainhdl.cpp:130-131), not again when the grid is coarsened
    tag("ConstantSectorRadius", c->C.csr);
    tag("InterpolatingSectorRadius", c->C.isr);
    tag("NeighbourTracking", P.neighbour_tracking);
    tag("UseStoredElasticEnergy", flag(P.use_stored_elastic_energy));
    tag("GrainScheduler", P.grain_scheduler);
    x << "</Parameters>\n\n";
    const std::string xml_name = dir + "/PARAMETERS_SIM_NONAME" + tail + ".xml";
    std::ofstream xf(xml_name);
    if (!xf) return fail(c, GG_E_IO, "cannot write " + xml_name);
    xf << x.str();
    return GG_OK;
}

int gg_read_grain_stats(gg_ctx* c, gg_grain_stats* out, int32_t capacity) {
    if (!c || !out) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    if (capacity < c->N) return fail(c, GG_E_INVALID, "capacity smaller than the grain count");
    const int N = c->N;
    c->stats_wanted = true;
    if (c->stats_fresh) {  // gathered and copied by the step that just ran
        std::memcpy(out, c->h_stats, sizeof(gg_grain_stats) * (size_t)N);
        return GG_OK;
    }
    // gathered on the device, one copy through a pinned buffer
    if (!c->d_stats) {
        int rc = dalloc(c, &c->d_stats, (size_t)N);
        if (rc) return rc;
    }
    if (!c->h_stats) {
        c->h_stats_bytes = sizeof(gg_grain_stats) * (size_t)(N > 0 ? N : 1);
        GG_CUDA(c, pinned_take(reinterpret_cast<void**>(&c->h_stats), c->h_stats_bytes));
    }
    GG_CUDA(c, pack_stats(c->C, c->dS, c->d_stats, c->stream));
    GG_CUDA(c, cudaMemcpyAsync(c->h_stats, c->d_stats, sizeof(gg_grain_stats) * (size_t)N, cudaMemcpyDeviceToHost,
                               c->stream));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));
    std::memcpy(out, c->h_stats, sizeof(gg_grain_stats) * (size_t)N);
    return GG_OK;
}

int gg_dump(gg_ctx* c, const char* path, int32_t steps_done, int32_t append) {
    if (!c || !path) return GG_E_INVALID;
    if (!c->initialised) return fail(c, GG_E_STATE, "not initialised");
    int rc = refresh_state(c);
    if (rc) return rc;
    const int N = c->N;
    const NetState& S = c->hS;
    const NetConst& C = c->C;
    const bool plain = c->P.precision == GG_PRECISION_PLAIN;
    const size_t rsz = plain ? 8 : 4;
    std::vector<int32_t> state(N + 1), reg(N + 1), bnd(N + 1), cmpn(N + 1), secn(N + 1), nbn(N + 1), cn(N + 1),
        jn(N + 1), newbb(4 * (N + 1));
    std::vector<int32_t> cmp((size_t)C.kmax * (N + 1)), sec((size_t)C.kmax * (N + 1));
    std::vector<double> vol(N + 1), en(N + 1), per(N + 1), mda(N + 1);
    std::vector<Box> bcur(N + 1), bprev(N + 1);
    std::vector<int64_t> ocur(N + 1), oprev(N + 1), coff(N + 1);
    std::vector<Neighbour> nb((size_t)C.nbmax * (N + 1));
    std::vector<Junction> js((size_t)C.jmax * (N + 1));
    std::vector<char> phi((size_t)S.phi_cap * rsz);
    std::vector<uint32_t> idl((size_t)S.phi_cap);
    std::vector<CPoint> cont((size_t)S.cont_cap);
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    };
    GG_CUDA(c, d2h(state.data(), C.state, 4 * (N + 1)));
    GG_CUDA(c, d2h(reg.data(), C.regular, 4 * (N + 1)));
    GG_CUDA(c, d2h(bnd.data(), C.inter_bnd, 4 * (N + 1)));
    GG_CUDA(c, d2h(cmpn.data(), C.cmp_n, 4 * (N + 1)));
    GG_CUDA(c, d2h(secn.data(), C.sec_n, 4 * (N + 1)));
    GG_CUDA(c, d2h(nbn.data(), C.nb_n, 4 * (N + 1)));
    GG_CUDA(c, d2h(newbb.data(), C.newbb, 16 * (N + 1)));
    GG_CUDA(c, d2h(cmp.data(), C.cmp_ids, 4 * cmp.size()));
    GG_CUDA(c, d2h(sec.data(), C.sec_ids, 4 * sec.size()));
    GG_CUDA(c, d2h(vol.data(), C.volume, 8 * (N + 1)));
    GG_CUDA(c, d2h(en.data(), C.energy, 8 * (N + 1)));
    GG_CUDA(c, d2h(per.data(), C.perimeter, 8 * (N + 1)));
    GG_CUDA(c, d2h(mda.data(), C.meanda, 8 * (N + 1)));
    GG_CUDA(c, d2h(nb.data(), C.nb, sizeof(Neighbour) * nb.size()));
    GG_CUDA(c, d2h(bcur.data(), S.box_cur, sizeof(Box) * (N + 1)));
    GG_CUDA(c, d2h(bprev.data(), S.box_prev, sizeof(Box) * (N + 1)));
    GG_CUDA(c, d2h(ocur.data(), S.off_cur, 8 * (N + 1)));
    GG_CUDA(c, d2h(oprev.data(), S.off_prev, 8 * (N + 1)));
    GG_CUDA(c, d2h(coff.data(), S.coff_prev, 8 * (N + 1)));
    GG_CUDA(c, d2h(cn.data(), S.cn_prev, 4 * (N + 1)));
    GG_CUDA(c, d2h(jn.data(), S.jn_prev, 4 * (N + 1)));
    GG_CUDA(c, d2h(js.data(), S.jPrev, sizeof(Junction) * js.size()));
    GG_CUDA(c, d2h(phi.data(), S.phiA, phi.size()));
    GG_CUDA(c, d2h(idl.data(), S.idPrev, 4 * idl.size()));
    GG_CUDA(c, d2h(cont.data(), S.contPrev, sizeof(CPoint) * cont.size()));
    GG_CUDA(c, cudaStreamSynchronize(c->stream));

    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) return fail(c, GG_E_IO, std::string("cannot open ") + path);
    auto wi = [&](int32_t v) { std::fwrite(&v, 4, 1, f); };
    auto wu = [&](uint32_t v) { std::fwrite(&v, 4, 1, f); };
    auto wd = [&](double v) { std::fwrite(&v, 8, 1, f); };
    if (!append) {
        std::fwrite("GGD1", 1, 4, f);
        wi(1);
        wi(N);
        wi(c->m);
        wi(c->nn);
        wd(c->h);
        wd(c->delta);
        wd(c->dt);
    }
    wi(0x52454344);
    wi(steps_done);
    wi(S.live);
    for (int g = 1; g <= N; ++g) {
        wi(g);
        if (state[g] == G_GONE) {
            wi(0);
            continue;
        }
        wi(state[g] == G_EXISTS ? 1 : 2);
        wi(reg[g]);
        wi(bnd[g]);
        wd(vol[g]);
        wd(en[g]);
        wd(per[g]);
        wd(mda[g]);
        const Box bx = bcur[g];
        wi(bx.x0);
        wi(bx.x1);
        wi(bx.y0);
        wi(bx.y1);
        const int64_t area = box_area(bx);
        for (int64_t k = 0; k < area; ++k) {
            double v = 0;
            if (state[g] == G_EXISTS) {
                if (plain)
                    v = reinterpret_cast<const double*>(phi.data())[ocur[g] + k];
                else
                    v = reinterpret_cast<const float*>(phi.data())[ocur[g] + k];
            }
            wd(v);
        }
        const Box ib = bprev[g];
        wi(ib.x0);
        wi(ib.x1);
        wi(ib.y0);
        wi(ib.y1);
        const int64_t ia = box_area(ib);
        for (int64_t k = 0; k < ia; ++k) wu(state[g] == G_EXISTS ? idl[oprev[g] + k] : 0xFFFFFFFFu);
        wi(cmpn[g]);
        for (int k = 0; k < cmpn[g]; ++k) wi(cmp[(size_t)g * C.kmax + k]);
        wi(secn[g]);
        for (int k = 0; k < secn[g]; ++k) wi(sec[(size_t)g * C.kmax + k]);
        wi(cn[g]);
        for (int k = 0; k < cn[g]; ++k) {
            const CPoint& p = cont[coff[g] + k];
            wd(p.x);
            wd(p.y);
            wd(p.energy);
            wd(p.mob);
        }
        wi(jn[g]);
        for (int k = 0; k < jn[g]; ++k) {
            const Junction& j = js[(size_t)g * C.jmax + k];
            wi(j.type);
            for (int q = 0; q < 4; ++q) wu(j.grains[q]);
            wi(j.segment);
            wd(j.lambda);
            wd(j.x);
            wd(j.y);
        }
        wi(nbn[g]);
        for (int k = 0; k < nbn[g]; ++k) {
            const Neighbour& q = nb[(size_t)g * C.nbmax + k];
            wi(q.id);
            wd(q.length);
            wd(q.energy);
            wd(q.misori);
            wd(q.mobility);
        }
        for (int q = 0; q < 4; ++q) wi(newbb[4 * g + q]);
    }
    std::fclose(f);
    return GG_OK;
}

}  // extern "C"
