/* fftw_shim.c — FFTW 3 plans (fftw_api/fftw3.h) executed by the oracle's DFT, for building
 * the reference's Interp_function.cpp from its own source.  TEST INFRASTRUCTURE ONLY. */
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"
#include "../orc_fft.h"

struct orc_fftw_plan_s {
    int n0, n1;   /* n0 = 1 for 1-D plans */
    double *in, *out;
    int sign;
};

static fftw_plan make(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign)
{
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    if (!p) abort();
    p->n0 = n0;
    p->n1 = n1;
    p->in = (double *)in;
    p->out = (double *)out;
    p->sign = sign;
    return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
    (void)flags;
    return make(1, n, in, out, sign);
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
    (void)flags;
    return make(n0, n1, in, out, sign);
}

void fftw_execute(const fftw_plan p)
{
    size_t n = (size_t)p->n0 * p->n1;
    if (p->out != p->in) memcpy(p->out, p->in, sizeof(double) * 2 * n);
    if ((p->n0 == 1 ? orc_dft_1d(p->out, p->n1, 1, p->sign) : orc_dft_2d(p->out, p->n0, p->n1, p->sign)) != 0)
        abort();
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }
