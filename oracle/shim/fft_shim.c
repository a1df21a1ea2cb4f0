/*
 * Test-infrastructure FFT (oracle only; never linked into the product).
 *
 * GraGLeS2D links FFTW3 (src/CMakeLists.txt:67-68, no version pinned) for
 * its per-box Gaussian convolution (src/box.cpp:622-695).  FFTW3 is not
 * under the reference tree and not installed, so this file restates the
 * transform FFTW documents for fftw_plan_dft_r2c_2d / fftw_plan_dft_c2r_2d:
 *
 *   r2c:  Y[k0][k1] = sum_{r,c} x[r][c] exp(-2 pi i (k0 r / n0 + k1 c / n1)),
 *         k1 in [0, n1/2], output row-major n0 x (n1/2 + 1), unnormalised;
 *   c2r:  x[r][c]   = sum_{k0,k1} Y[k0][k1] exp(+2 pi i (...)), with the
 *         missing half taken from Hermitian symmetry, unnormalised; the
 *         imaginary parts of the k1 = 0 and k1 = n1/2 columns are ignored.
 *
 * Both are evaluated as separable direct DFTs (rows, then columns; columns,
 * then rows for the inverse) with a twiddle table exp(-2 pi i k / n) built
 * from libm cos/sin, summing each output in index order.  The sm_100a
 * plain-form kernels evaluate the identical sums in the identical order,
 * so the FP64 convolution agrees bit for bit (both sides compiled without
 * FMA contraction).  Any n >= 1 is accepted, primes included.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define GG_SHIM_PI 3.14159265358979323846

void gg_shim_twiddle(int n, int k, double* re, double* im) {
    double ang = (2.0 * GG_SHIM_PI * (double)k) / (double)n;
    *re = cos(ang);
    *im = -sin(ang);
}

enum { SHIM_R2C = 1, SHIM_C2R = 2 };

struct gg_shim_plan_s {
    int kind;
    int single;
    int n0, n1;
    void* in;
    void* out;
    double* w0; /* 2*n0: re, im interleaved */
    double* w1; /* 2*n1 */
};

static double* make_table(int n) {
    double* w = (double*)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < n; ++k) gg_shim_twiddle(n, k, &w[2 * k], &w[2 * k + 1]);
    return w;
}

static struct gg_shim_plan_s* make_plan(int kind, int single, int n0, int n1, void* in, void* out) {
    struct gg_shim_plan_s* p = (struct gg_shim_plan_s*)calloc(1, sizeof(*p));
    p->kind = kind;
    p->single = single;
    p->n0 = n0;
    p->n1 = n1;
    p->in = in;
    p->out = out;
    p->w0 = make_table(n0);
    p->w1 = make_table(n1);
    return p;
}

/* ---- double precision ---------------------------------------------------- */

static void r2c_d(const struct gg_shim_plan_s* p) {
    const int n0 = p->n0, n1 = p->n1, half = n1 / 2 + 1;
    const double* x = (const double*)p->in;
    double* y = (double*)p->out; /* interleaved complex, n0 x half */
    double* t = (double*)malloc(sizeof(double) * 2 * (size_t)n0 * half);
    for (int r = 0; r < n0; ++r) {
        for (int f = 0; f < half; ++f) {
            double re = 0.0, im = 0.0;
            for (int c = 0; c < n1; ++c) {
                int k = (int)(((long)f * c) % n1);
                double v = x[(size_t)r * n1 + c];
                re = re + v * p->w1[2 * k];
                im = im + v * p->w1[2 * k + 1];
            }
            t[2 * ((size_t)r * half + f)] = re;
            t[2 * ((size_t)r * half + f) + 1] = im;
        }
    }
    for (int f = 0; f < half; ++f) {
        for (int q = 0; q < n0; ++q) {
            double re = 0.0, im = 0.0;
            for (int r = 0; r < n0; ++r) {
                int k = (int)(((long)q * r) % n0);
                double a = t[2 * ((size_t)r * half + f)];
                double b = t[2 * ((size_t)r * half + f) + 1];
                double wc = p->w0[2 * k], ws = p->w0[2 * k + 1];
                re = re + (a * wc - b * ws);
                im = im + (a * ws + b * wc);
            }
            y[2 * ((size_t)q * half + f)] = re;
            y[2 * ((size_t)q * half + f) + 1] = im;
        }
    }
    free(t);
}

static void c2r_d(const struct gg_shim_plan_s* p) {
    const int n0 = p->n0, n1 = p->n1, half = n1 / 2 + 1;
    const double* y = (const double*)p->in;
    double* x = (double*)p->out;
    double* t = (double*)malloc(sizeof(double) * 2 * (size_t)n0 * half);
    for (int f = 0; f < half; ++f) {
        for (int r = 0; r < n0; ++r) {
            double re = 0.0, im = 0.0;
            for (int q = 0; q < n0; ++q) {
                int k = (int)(((long)q * r) % n0);
                double a = y[2 * ((size_t)q * half + f)];
                double b = y[2 * ((size_t)q * half + f) + 1];
                double wc = p->w0[2 * k], ws = -p->w0[2 * k + 1];
                re = re + (a * wc - b * ws);
                im = im + (a * ws + b * wc);
            }
            t[2 * ((size_t)r * half + f)] = re;
            t[2 * ((size_t)r * half + f) + 1] = im;
        }
    }
    const int hmax = (n1 - 1) / 2;
    for (int r = 0; r < n0; ++r) {
        for (int c = 0; c < n1; ++c) {
            double acc = t[2 * ((size_t)r * half)];
            for (int f = 1; f <= hmax; ++f) {
                int k = (int)(((long)f * c) % n1);
                double a = t[2 * ((size_t)r * half + f)];
                double b = t[2 * ((size_t)r * half + f) + 1];
                acc = acc + 2.0 * (a * p->w1[2 * k] + b * p->w1[2 * k + 1]);
            }
            if ((n1 & 1) == 0) {
                double nyq = t[2 * ((size_t)r * half + n1 / 2)];
                acc = acc + ((c & 1) ? -nyq : nyq);
            }
            x[(size_t)r * n1 + c] = acc;
        }
    }
    free(t);
}

/* ---- single precision (same sums, float storage, double twiddles rounded) - */

static void r2c_f(const struct gg_shim_plan_s* p) {
    const int n0 = p->n0, n1 = p->n1, half = n1 / 2 + 1;
    const float* x = (const float*)p->in;
    float* y = (float*)p->out;
    float* t = (float*)malloc(sizeof(float) * 2 * (size_t)n0 * half);
    for (int r = 0; r < n0; ++r)
        for (int f = 0; f < half; ++f) {
            float re = 0.0f, im = 0.0f;
            for (int c = 0; c < n1; ++c) {
                int k = (int)(((long)f * c) % n1);
                float v = x[(size_t)r * n1 + c];
                re = re + v * (float)p->w1[2 * k];
                im = im + v * (float)p->w1[2 * k + 1];
            }
            t[2 * ((size_t)r * half + f)] = re;
            t[2 * ((size_t)r * half + f) + 1] = im;
        }
    for (int f = 0; f < half; ++f)
        for (int q = 0; q < n0; ++q) {
            float re = 0.0f, im = 0.0f;
            for (int r = 0; r < n0; ++r) {
                int k = (int)(((long)q * r) % n0);
                float a = t[2 * ((size_t)r * half + f)], b = t[2 * ((size_t)r * half + f) + 1];
                float wc = (float)p->w0[2 * k], ws = (float)p->w0[2 * k + 1];
                re = re + (a * wc - b * ws);
                im = im + (a * ws + b * wc);
            }
            y[2 * ((size_t)q * half + f)] = re;
            y[2 * ((size_t)q * half + f) + 1] = im;
        }
    free(t);
}

static void c2r_f(const struct gg_shim_plan_s* p) {
    const int n0 = p->n0, n1 = p->n1, half = n1 / 2 + 1;
    const float* y = (const float*)p->in;
    float* x = (float*)p->out;
    float* t = (float*)malloc(sizeof(float) * 2 * (size_t)n0 * half);
    for (int f = 0; f < half; ++f)
        for (int r = 0; r < n0; ++r) {
            float re = 0.0f, im = 0.0f;
            for (int q = 0; q < n0; ++q) {
                int k = (int)(((long)q * r) % n0);
                float a = y[2 * ((size_t)q * half + f)], b = y[2 * ((size_t)q * half + f) + 1];
                float wc = (float)p->w0[2 * k], ws = -(float)p->w0[2 * k + 1];
                re = re + (a * wc - b * ws);
                im = im + (a * ws + b * wc);
            }
            t[2 * ((size_t)r * half + f)] = re;
            t[2 * ((size_t)r * half + f) + 1] = im;
        }
    const int hmax = (n1 - 1) / 2;
    for (int r = 0; r < n0; ++r)
        for (int c = 0; c < n1; ++c) {
            float acc = t[2 * ((size_t)r * half)];
            for (int f = 1; f <= hmax; ++f) {
                int k = (int)(((long)f * c) % n1);
                float a = t[2 * ((size_t)r * half + f)], b = t[2 * ((size_t)r * half + f) + 1];
                acc = acc + 2.0f * (a * (float)p->w1[2 * k] + b * (float)p->w1[2 * k + 1]);
            }
            if ((n1 & 1) == 0) {
                float nyq = t[2 * ((size_t)r * half + n1 / 2)];
                acc = acc + ((c & 1) ? -nyq : nyq);
            }
            x[(size_t)r * n1 + c] = acc;
        }
    free(t);
}

/* ---- FFTW-compatible entry points ---------------------------------------- */

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags) {
    (void)flags;
    return (fftw_plan)make_plan(SHIM_R2C, 0, n0, n1, in, out);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags) {
    (void)flags;
    return (fftw_plan)make_plan(SHIM_C2R, 0, n0, n1, in, out);
}
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned flags) {
    (void)flags;
    return (fftwf_plan)make_plan(SHIM_R2C, 1, n0, n1, in, out);
}
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned flags) {
    (void)flags;
    return (fftwf_plan)make_plan(SHIM_C2R, 1, n0, n1, in, out);
}

static void execute(const struct gg_shim_plan_s* p) {
    if (!p || p->n0 <= 0 || p->n1 <= 0) return;
    if (p->single) {
        if (p->kind == SHIM_R2C) r2c_f(p); else c2r_f(p);
    } else {
        if (p->kind == SHIM_R2C) r2c_d(p); else c2r_d(p);
    }
}

void fftw_execute(const fftw_plan p) { execute((const struct gg_shim_plan_s*)p); }
void fftwf_execute(const fftwf_plan p) { execute((const struct gg_shim_plan_s*)p); }

static void destroy(struct gg_shim_plan_s* p) {
    if (!p) return;
    free(p->w0);
    free(p->w1);
    free(p);
}
void fftw_destroy_plan(fftw_plan p) { destroy((struct gg_shim_plan_s*)p); }
void fftwf_destroy_plan(fftwf_plan p) { destroy((struct gg_shim_plan_s*)p); }

void* fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void* p) { free(p); }
void* fftwf_malloc(size_t n) { return malloc(n); }
void fftwf_free(void* p) { free(p); }
