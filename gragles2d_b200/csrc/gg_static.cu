// Allocation-free box convolution (gg_convolve_box_static in gg_step.h).
//
// Some callers cannot allocate device memory: an application that hands this
// library device buffers from its own memory pool and does not let plug-ins
// allocate (to keep its pool the only owner of device memory and avoid
// fragmentation or out-of-memory failures in the middle of a run).  For them
// this file convolves one n x n distance-field box with the Gaussian kernel
// of the convolution stage, using only device memory compiled into the
// library: a file-scope scratch array of fixed size, which every GPU that
// loads the library holds until the process exits.  The caller passes the
// input and output boxes; nothing here calls cudaMalloc, cudaFree or any
// allocating library routine.
//
// The arithmetic is the plain form's (separable direct DFTs in a fixed order,
// host-computed twiddles and Gaussian multipliers, no FMA contraction), so
// the result is bit-identical to the convolution stage of a plain context.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/gg_step.h"

namespace {

constexpr int kMaxN = GG_STATIC_CONV_MAX_N;
constexpr int kMaxHalf = kMaxN / 2 + 1;
// Layout of the scratch (doubles): two spectra of n x (n/2+1) complex values,
// the twiddles exp(-2 pi i k / n) for k < n, the multipliers G(i2, j2).
constexpr size_t kSpecDoubles = 2 * 2 * (size_t)kMaxN * kMaxHalf;
constexpr size_t kTwDoubles = 2 * (size_t)kMaxN;
constexpr size_t kGDoubles = (size_t)kMaxHalf * kMaxHalf;
constexpr size_t kScratchDoubles = kSpecDoubles + kTwDoubles + kGDoubles;

// The fixed device scratch.  In host code this name is only a host-side
// stand-in for the symbol, not a device address: the address used by kernels
// comes from cudaGetSymbolAddress on each device (see scratch_on_device).
static __device__ __align__(256) double g_conv_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

constexpr double kPiS = 3.14159265358979323846;

// A failed runtime call: consume the runtime's last error as well, so that
// this failure is not reported again by a later, unrelated call.
int cuda_error() {
    (void)cudaGetLastError();
    return GG_E_CUDA;
}

// Same expressions as the context's table builder, so the tables match bit
// for bit.
void twiddle(int n, int k, double* re, double* im) {
    double ang = (2.0 * kPiS * (double)k) / (double)n;
    *re = cos(ang);
    *im = -sin(ang);
}

double gaussian_multiplier(int n, int i2, int j2, double dt, int nn) {
    double nsq = nn * nn;
    double n_nsq = n * n;
    return exp(-sqrt(2 / kPiS) * (i2 * i2 + j2 * j2) * 4.0 * dt * nsq / n_nsq * kPiS * kPiS) / n_nsq;
}

// Device address of the scratch on the current device, looked up once per
// device (the first call on a device does this set-up).
int scratch_on_device(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return cuda_error();
    if (dev < 0 || dev >= kMaxDevices) return GG_E_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_conv_scratch);
        if (e != cudaSuccess) return cuda_error();
        if (!p) return GG_E_CUDA;
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return GG_OK;
}

// One CTA: rows r2c, columns DFT times G, inverse columns, rows c2r; the same
// sums in the same order as the plain convolution stage.
__global__ void __launch_bounds__(256) k_conv_box_static(const double* __restrict__ in, double* __restrict__ out,
                                                         int n, double* __restrict__ scratch) {
    const int half = n / 2 + 1;
    double* s1 = scratch;
    double* s2 = scratch + 2 * (size_t)n * half;
    const double* w = scratch + kSpecDoubles;
    const double* G = w + kTwDoubles;
    const int tot = n * half;
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int r = idx / half, f = idx - r * half;
        double re = 0, im = 0;
        const double* xr = in + (size_t)r * n;
        int k = 0;
        for (int c = 0; c < n; ++c) {
            const double v = xr[c];
            re = re + v * w[2 * k];
            im = im + v * w[2 * k + 1];
            k += f;
            if (k >= n) k -= n;
        }
        s1[2 * idx] = re;
        s1[2 * idx + 1] = im;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int q = idx / half, f = idx - q * half;
        double re = 0, im = 0;
        int k = 0;
        for (int r = 0; r < n; ++r) {
            const double a = s1[2 * (r * half + f)], b = s1[2 * (r * half + f) + 1];
            const double wc = w[2 * k], ws = w[2 * k + 1];
            re = re + (a * wc - b * ws);
            im = im + (a * ws + b * wc);
            k += q;
            if (k >= n) k -= n;
        }
        const int j2 = q < n - q ? q : n - q;
        const double gv = G[f * half + j2];
        s2[2 * idx] = re * gv;
        s2[2 * idx + 1] = im * gv;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int r = idx / half, f = idx - r * half;
        double re = 0, im = 0;
        int k = 0;
        for (int q = 0; q < n; ++q) {
            const double a = s2[2 * (q * half + f)], b = s2[2 * (q * half + f) + 1];
            const double wc = w[2 * k], ws = -w[2 * k + 1];
            re = re + (a * wc - b * ws);
            im = im + (a * ws + b * wc);
            k += r;
            if (k >= n) k -= n;
        }
        s1[2 * idx] = re;
        s1[2 * idx + 1] = im;
    }
    __syncthreads();
    const int hmax = (n - 1) / 2;
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int r = idx / n, c = idx - r * n;
        const double* t = s1 + 2 * (size_t)r * half;
        double acc = t[0];
        int k = 0;
        for (int f = 1; f <= hmax; ++f) {
            k += c;
            if (k >= n) k -= n;
            acc = acc + 2.0 * (t[2 * f] * w[2 * k] + t[2 * f + 1] * w[2 * k + 1]);
        }
        if ((n & 1) == 0) {
            const double nyq = t[2 * (n / 2)];
            acc = acc + ((c & 1) ? -nyq : nyq);
        }
        out[idx] = acc;
    }
}

}  // namespace

extern "C" int gg_convolve_box_static(const double* d_in, double* d_out, int32_t n, double dt,
                                      int32_t real_domain_size, void* stream) {
    if (n < 1 || n > kMaxN) return GG_E_INVALID;
    if (!d_in || !d_out || real_domain_size < 1 || !(dt > 0)) return GG_E_INVALID;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // A call copies its tables from this stack frame and waits for the
    // stream, neither of which a stream capture admits: a capturing stream
    // is refused before anything is issued on it, so the capture stays valid.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return cuda_error();
    if (cap != cudaStreamCaptureStatusNone) return GG_E_INVALID;
    double* scratch = nullptr;
    const int rc = scratch_on_device(&scratch);
    if (rc != GG_OK) return rc;
    // Tables for this n, built on the host stack (no heap allocation) and
    // copied into the scratch; every value the kernel reads is rewritten by
    // this call, so nothing has to be cleared between calls.
    double tables[kTwDoubles + kGDoubles];
    const int half = n / 2 + 1;
    for (int k = 0; k < n; ++k) twiddle(n, k, &tables[2 * k], &tables[2 * k + 1]);
    double* G = tables + kTwDoubles;
    for (int i2 = 0; i2 < half; ++i2)
        for (int j2 = 0; j2 < half; ++j2) G[i2 * half + j2] = gaussian_multiplier(n, i2, j2, dt, real_domain_size);
    cudaError_t e = cudaMemcpyAsync(scratch + kSpecDoubles, tables, sizeof(tables), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_error();
    k_conv_box_static<<<1, 256, 0, s>>>(d_in, d_out, n, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error();
    // The host table buffer lives on this stack frame: wait for the copy.
    e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? GG_OK : cuda_error();
}
