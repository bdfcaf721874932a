/*
 * Test infrastructure (oracle side only; never linked into the product).
 *
 * A minimal FFTW3-float API declaration, written for this project, covering
 * exactly the symbols MEGADOCK's CPU path uses (src/fft_process.cpp:188-202,
 * 386-388, 822-823 and src/fft_process.h:159-161):
 *   fftwf_complex, fftwf_plan, FFTW_FORWARD, FFTW_BACKWARD, FFTW_ESTIMATE,
 *   fftwf_plan_dft_3d, fftwf_execute, fftwf_destroy_plan,
 *   fftwf_malloc, fftwf_free, fftwf_cleanup.
 *
 * libfftw3f is not installed on this image, so the reference's CPU sources are
 * linked against fftw_shim.cpp instead: an unnormalised complex DFT with FFTW's
 * sign convention (FORWARD = exp(-2*pi*i*jk/n), BACKWARD = exp(+2*pi*i*jk/n)).
 * The arithmetic precision is chosen at run time by MD_SHIM_FFT=fp32|fp64
 * (default fp32: float data and float arithmetic with double-computed twiddles,
 * the stand-in for FFTW's float path; fp64: float in/out, double internally).
 */
#ifndef MD_ORACLE_FFTW3_SHIM_H
#define MD_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex *in,
                             fftwf_complex *out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
void fftwf_cleanup(void);

#ifdef __cplusplus
}
#endif

#endif
