/*
 * Test-infrastructure shim (oracle only; never linked into the product).
 *
 * Declares the subset of the FFTW3 API that GraGLeS2D calls
 * (src/box.cpp:580-600 plans, src/box.cpp:812-818 execute,
 * src/box.cpp:524-529 destroy) so the reference's own sources compile
 * here without FFTW3 (not installed, no network).  The arithmetic behind
 * it lives in fft_shim.c and restates FFTW's published definition of the
 * unnormalised real-to-complex / complex-to-real 2-D DFT.
 */
#ifndef GG_ORACLE_FFTW3_SHIM_H
#define GG_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef float fftwf_complex[2];

typedef struct fftw_plan_s* fftw_plan;
typedef struct fftwf_plan_s* fftwf_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void* fftw_malloc(size_t n);
void fftw_free(void* p);

fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
void* fftwf_malloc(size_t n);
void fftwf_free(void* p);

/* Twiddle used by every transform: w_n^k = exp(-2 pi i k / n). */
void gg_shim_twiddle(int n, int k, double* re, double* im);

#ifdef __cplusplus
}
#endif

#endif
