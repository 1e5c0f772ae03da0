/* orc_fft.h — discrete Fourier transforms for the CPU oracle (TEST INFRASTRUCTURE ONLY;
 * never linked into the product).
 *
 * The reference's F-K interpolation (Interp_function.cpp:127-244) calls FFTW 3
 * (fftw_plan_dft_1d / fftw_plan_dft_2d with FFTW_ESTIMATE, double precision).  FFTW is not
 * part of the reference checkout and not installed here; this file restates the transform
 * FFTW documents for those plans:
 *     out[k] = sum_j in[j] * exp(sign * 2*pi*i * j*k / n),  sign = -1 forward, +1 backward,
 * unnormalised, and for 2-D plans over a row-major [n0][n1] array the same along both axes.
 * The algorithm is a mixed-radix Cooley-Tukey recursion on the smallest prime factor (a
 * direct sum for prime lengths), in double precision with a cos/sin twiddle table. */
#ifndef ORC_FFT_H
#define ORC_FFT_H

#ifdef __cplusplus
extern "C" {
#endif

/* In-place transform of n complex values (interleaved re, im) spaced `stride` complex
 * elements apart.  Returns 0, or -1 when memory runs out. */
int orc_dft_1d(double *x, int n, long stride, int sign);

/* In-place 2-D transform of a row-major [n0][n1] complex array. */
int orc_dft_2d(double *x, int n0, int n1, int sign);

#ifdef __cplusplus
}
#endif

#endif
