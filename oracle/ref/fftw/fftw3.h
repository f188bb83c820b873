/* Minimal stand-in for the FFTW 3 interface (FFTW 3.3, www.fftw.org) that the reference's FDft
 * (Src/Utils/FDft.hpp:245-350) binds: complex, real-to-complex and complex-to-real DFTs of any rank, in
 * double and single precision.  FFTW itself is not in this image; the definitions in fftw_dft.cpp compute
 * the same transforms FFTW documents -- unnormalised, out[k] = sum_j in[j] exp(sign 2 pi i j.k / n),
 * row-major multi-dimensional, r2c/c2r keeping n_last/2+1 entries of the last dimension -- by direct
 * summation.  Test infrastructure only: it lets the reference's Lagrange (uniform) kernel, whose M2L
 * runs in Fourier space, be compiled and run as the checker. */
#ifndef ORACLE_FFTW3_STANDIN_H
#define ORACLE_FFTW3_STANDIN_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct oracle_dft_plan_d *fftw_plan;   /* distinct types, as in FFTW: overloads tell them apart */
typedef struct oracle_dft_plan_f *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_UNALIGNED (1U << 1)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft(int rank, const int *n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c(int rank, const int *n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r(int rank, const int *n, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
fftwf_plan fftwf_plan_dft(int rank, const int *n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c(int rank, const int *n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r(int rank, const int *n, fftwf_complex *in, float *out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif
#endif
