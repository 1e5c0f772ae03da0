/* fftw3.h — the part of FFTW 3's public interface that the reference's
 * Interp_function.cpp uses, so that file compiles here, where FFTW is not installed.
 * The plans run the DFT of oracle/orc_fft.c (fftw_shim.c).  TEST INFRASTRUCTURE ONLY.
 * Names, argument lists and the sign/flag values follow FFTW 3's documented API. */
#ifndef ORACLE_FFTW3_API_H
#define ORACLE_FFTW3_API_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct orc_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

#ifdef __cplusplus
}
#endif

#endif
