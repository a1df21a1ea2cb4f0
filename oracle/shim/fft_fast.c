/*
 * Test-infrastructure FFT for timing (oracle only; never linked into the
 * product).  Same API and transform as fft_shim.c (FFTW3's unnormalised
 * 2-D r2c / c2r, fftw_plan_dft_r2c_2d / fftw_plan_dft_c2r_2d, as
 * GraGLeS2D calls them at src/box.cpp:580-600, 812-818), evaluated in
 * O(n^2 log n) per 2-D transform instead of fft_shim.c's O(n^3) direct
 * DFT, so that the reference's CPU path is timed with an FFT of the kind
 * FFTW3 provides:
 *
 *   - 1-D complex transforms of any length n by recursive mixed-radix
 *     decimation in time (Cooley-Tukey) over the prime factors of n, each
 *     combine step a p-point DFT of twiddled sub-transform outputs;
 *   - lengths with a prime factor above 13 by Bluestein's chirp-z
 *     algorithm (L. Bluestein, 1970): X_k = c_k sum_j (x_j c_j) conj(c_{k-j}),
 *     c_k = exp(-pi i k^2 / n), the sum as a circular convolution of length
 *     M = the power of two >= 2n - 1 through two radix-2 FFTs;
 *   - 2-D r2c: rows (real input as complex), keeping columns 0 .. n1/2, then
 *     columns; c2r: columns, then each row from its Hermitian half (the
 *     imaginary parts of columns 0 and n1/2 drop out of the real part).
 *
 * Results agree with the direct DFT to rounding (about 1e-15 relative),
 * not bit for bit: parity runs use fft_shim.c.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define GG_PI 3.14159265358979323846

typedef struct {
    double re, im;
} cpx;

static inline cpx cmul(cpx a, cpx b) {
    cpx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}

typedef struct fft1 {
    int n;
    int nf;
    int fac[40];
    cpx* tw;  /* exp(-2 pi i k / n), k < n */
    cpx* tmp;  /* n scratch values */
    cpx* obuf; /* n: output of the recursion */
    /* Bluestein */
    int m;
    cpx* chirp; /* c_k, k < n */
    cpx* bhat;  /* FFT_m of conj(c) wrapped */
    cpx* work;  /* m */
    struct fft1* sub;
} fft1;

static void factorise(fft1* f, int n) {
    f->nf = 0;
    while (n % 4 == 0) {
        f->fac[f->nf++] = 4;
        n /= 4;
    }
    for (int p = 2; p * p <= n; ++p)
        while (n % p == 0) {
            f->fac[f->nf++] = p;
            n /= p;
        }
    if (n > 1) f->fac[f->nf++] = n;
}

static fft1* fft1_new(int n);
static void fft1_run(fft1* f, cpx* x);

static int largest_factor(const fft1* f) {
    int m = 1;
    for (int k = 0; k < f->nf; ++k)
        if (f->fac[k] > m) m = f->fac[k];
    return m;
}

static fft1* fft1_new(int n) {
    fft1* f = (fft1*)calloc(1, sizeof(fft1));
    f->n = n;
    factorise(f, n);
    f->tw = (cpx*)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < n; ++k) {
        const double a = -2.0 * GG_PI * (double)k / (double)n;
        f->tw[k].re = cos(a);
        f->tw[k].im = sin(a);
    }
    f->tmp = (cpx*)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
    f->obuf = (cpx*)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
    if (n > 1 && largest_factor(f) > 13) {
        int m = 1;
        while (m < 2 * n - 1) m <<= 1;
        f->m = m;
        f->sub = fft1_new(m);
        f->chirp = (cpx*)malloc(sizeof(cpx) * (size_t)n);
        f->bhat = (cpx*)calloc((size_t)m, sizeof(cpx));
        f->work = (cpx*)malloc(sizeof(cpx) * (size_t)m);
        for (int k = 0; k < n; ++k) {
            const long long k2 = ((long long)k * k) % (2LL * n);
            const double a = -GG_PI * (double)k2 / (double)n;
            f->chirp[k].re = cos(a);
            f->chirp[k].im = sin(a);
        }
        for (int k = 0; k < n; ++k) {
            const cpx c = {f->chirp[k].re, -f->chirp[k].im};
            f->bhat[k] = c;
            if (k) f->bhat[m - k] = c;
        }
        fft1_run(f->sub, f->bhat);
    }
    return f;
}

static void fft1_free(fft1* f) {
    if (!f) return;
    free(f->tw);
    free(f->tmp);
    free(f->obuf);
    free(f->chirp);
    free(f->bhat);
    free(f->work);
    fft1_free(f->sub);
    free(f);
}

/* out[0 .. n) = DFT of in[0], in[s], in[2s], ... (n values); level `lev` of
 * the factor list, tstep = N / n for the top-level twiddle table. */
static void rec(const fft1* f, const cpx* in, int s, cpx* out, int n, int lev, int tstep, cpx* tmp) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int p = f->fac[lev], m = n / p;
    for (int q = 0; q < p; ++q) rec(f, in + (size_t)q * s, s * p, out + (size_t)q * m, m, lev + 1, tstep * p, tmp);
    const int N = f->n;
    for (int k = 0; k < m; ++k) {
        /* twiddled inputs t_q = sub_q[k] w_n^{qk} */
        for (int q = 0; q < p; ++q) {
            const cpx v = out[(size_t)q * m + k];
            tmp[q] = q ? cmul(v, f->tw[((long long)q * k * tstep) % N]) : v;
        }
        if (p == 2) {
            const cpx a = tmp[0], b = tmp[1];
            out[k].re = a.re + b.re;
            out[k].im = a.im + b.im;
            out[k + m].re = a.re - b.re;
            out[k + m].im = a.im - b.im;
        } else if (p == 4) {
            const cpx a = tmp[0], b = tmp[1], c = tmp[2], d = tmp[3];
            const cpx s0 = {a.re + c.re, a.im + c.im}, s1 = {a.re - c.re, a.im - c.im};
            const cpx s2 = {b.re + d.re, b.im + d.im}, s3 = {b.re - d.re, b.im - d.im};
            out[k].re = s0.re + s2.re;
            out[k].im = s0.im + s2.im;
            out[k + 2 * m].re = s0.re - s2.re;
            out[k + 2 * m].im = s0.im - s2.im;
            /* -i s3 and +i s3 */
            out[k + m].re = s1.re + s3.im;
            out[k + m].im = s1.im - s3.re;
            out[k + 3 * m].re = s1.re - s3.im;
            out[k + 3 * m].im = s1.im + s3.re;
        } else {
            /* p-point DFT: X_u = sum_q t_q w_p^{qu}, w_p = w_N^{N/p} */
            const int wstep = N / p;
            for (int u = 0; u < p; ++u) {
                cpx acc = tmp[0];
                for (int q = 1; q < p; ++q) {
                    const cpx w = f->tw[((long long)q * u % p) * wstep];
                    const cpx t = cmul(tmp[q], w);
                    acc.re += t.re;
                    acc.im += t.im;
                }
                out[(size_t)u * m + k] = acc;
            }
        }
    }
}

/* In-place forward DFT of x[0 .. n). */
static void fft1_run(fft1* f, cpx* x) {
    const int n = f->n;
    if (n <= 1) return;
    if (f->sub) {
        const int m = f->m;
        cpx* w = f->work;
        for (int k = 0; k < n; ++k) w[k] = cmul(x[k], f->chirp[k]);
        for (int k = n; k < m; ++k) w[k].re = w[k].im = 0.0;
        fft1_run(f->sub, w);
        for (int k = 0; k < m; ++k) w[k] = cmul(w[k], f->bhat[k]);
        /* inverse FFT of length m via conjugation */
        for (int k = 0; k < m; ++k) w[k].im = -w[k].im;
        fft1_run(f->sub, w);
        const double inv = 1.0 / (double)m;
        for (int k = 0; k < n; ++k) {
            const cpx v = {w[k].re * inv, -w[k].im * inv};
            x[k] = cmul(v, f->chirp[k]);
        }
        return;
    }
    cpx tmpbuf[64];
    cpx* tmp = largest_factor(f) <= 64 ? tmpbuf : f->tmp;
    rec(f, x, 1, f->obuf, n, 0, 1, tmp);
    memcpy(x, f->obuf, sizeof(cpx) * (size_t)n);
}

/* In-place unnormalised inverse DFT (exp(+2 pi i ...)). */
static void ifft1_run(fft1* f, cpx* x) {
    for (int k = 0; k < f->n; ++k) x[k].im = -x[k].im;
    fft1_run(f, x);
    for (int k = 0; k < f->n; ++k) x[k].im = -x[k].im;
}

enum { FAST_R2C = 1, FAST_C2R = 2 };

struct fast_plan {
    int kind, single, n0, n1;
    void* in;
    void* out;
    fft1* f0;
    fft1* f1;
    cpx* t;   /* n0 x (n1/2 + 1) */
    cpx* row; /* max(n0, n1) */
};

static struct fast_plan* make_plan(int kind, int single, int n0, int n1, void* in, void* out) {
    struct fast_plan* p = (struct fast_plan*)calloc(1, sizeof(*p));
    p->kind = kind;
    p->single = single;
    p->n0 = n0;
    p->n1 = n1;
    p->in = in;
    p->out = out;
    p->f0 = fft1_new(n0);
    p->f1 = n1 == n0 ? NULL : fft1_new(n1);
    p->t = (cpx*)malloc(sizeof(cpx) * (size_t)n0 * (size_t)(n1 / 2 + 1));
    p->row = (cpx*)malloc(sizeof(cpx) * (size_t)(n0 > n1 ? n0 : n1));
    return p;
}

static void free_plan(struct fast_plan* p) {
    if (!p) return;
    fft1_free(p->f0);
    fft1_free(p->f1);
    free(p->t);
    free(p->row);
    free(p);
}

static double get_in(const struct fast_plan* p, size_t i) {
    return p->single ? (double)((const float*)p->in)[i] : ((const double*)p->in)[i];
}

static void exec(struct fast_plan* p) {
    const int n0 = p->n0, n1 = p->n1, half = n1 / 2 + 1;
    fft1* f1 = p->f1 ? p->f1 : p->f0;
    cpx* row = p->row;
    cpx* t = p->t;
    if (p->kind == FAST_R2C) {
        for (int r = 0; r < n0; ++r) {
            for (int c = 0; c < n1; ++c) {
                row[c].re = get_in(p, (size_t)r * n1 + c);
                row[c].im = 0.0;
            }
            fft1_run(f1, row);
            memcpy(t + (size_t)r * half, row, sizeof(cpx) * (size_t)half);
        }
        for (int f = 0; f < half; ++f) {
            for (int r = 0; r < n0; ++r) row[r] = t[(size_t)r * half + f];
            fft1_run(p->f0, row);
            for (int r = 0; r < n0; ++r) {
                const size_t o = 2 * ((size_t)r * half + f);
                if (p->single) {
                    ((float*)p->out)[o] = (float)row[r].re;
                    ((float*)p->out)[o + 1] = (float)row[r].im;
                } else {
                    ((double*)p->out)[o] = row[r].re;
                    ((double*)p->out)[o + 1] = row[r].im;
                }
            }
        }
    } else {
        for (int f = 0; f < half; ++f) {
            for (int r = 0; r < n0; ++r) {
                const size_t o = 2 * ((size_t)r * half + f);
                if (p->single) {
                    row[r].re = ((const float*)p->in)[o];
                    row[r].im = ((const float*)p->in)[o + 1];
                } else {
                    row[r].re = ((const double*)p->in)[o];
                    row[r].im = ((const double*)p->in)[o + 1];
                }
            }
            ifft1_run(p->f0, row);
            for (int r = 0; r < n0; ++r) t[(size_t)r * half + f] = row[r];
        }
        for (int r = 0; r < n0; ++r) {
            const cpx* z = t + (size_t)r * half;
            for (int f = 0; f < half; ++f) row[f] = z[f];
            for (int f = half; f < n1; ++f) {
                row[f].re = z[n1 - f].re;
                row[f].im = -z[n1 - f].im;
            }
            ifft1_run(f1, row);
            for (int c = 0; c < n1; ++c) {
                if (p->single)
                    ((float*)p->out)[(size_t)r * n1 + c] = (float)row[c].re;
                else
                    ((double*)p->out)[(size_t)r * n1 + c] = row[c].re;
            }
        }
    }
}

void gg_shim_twiddle(int n, int k, double* re, double* im) {
    const double a = (2.0 * GG_PI * (double)k) / (double)n;
    *re = cos(a);
    *im = -sin(a);
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags) {
    (void)flags;
    return (fftw_plan)make_plan(FAST_R2C, 0, n0, n1, in, out);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags) {
    (void)flags;
    return (fftw_plan)make_plan(FAST_C2R, 0, n0, n1, in, out);
}
void fftw_execute(const fftw_plan p) { exec((struct fast_plan*)p); }
void fftw_destroy_plan(fftw_plan p) { free_plan((struct fast_plan*)p); }
void* fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void* p) { free(p); }

fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned flags) {
    (void)flags;
    return (fftwf_plan)make_plan(FAST_R2C, 1, n0, n1, in, out);
}
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned flags) {
    (void)flags;
    return (fftwf_plan)make_plan(FAST_C2R, 1, n0, n1, in, out);
}
void fftwf_execute(const fftwf_plan p) { exec((struct fast_plan*)p); }
void fftwf_destroy_plan(fftwf_plan p) { free_plan((struct fast_plan*)p); }
void* fftwf_malloc(size_t n) { return malloc(n); }
void fftwf_free(void* p) { free(p); }
