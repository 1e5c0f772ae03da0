/* orc_fft.c — mixed-radix DFT for the CPU oracle (TEST INFRASTRUCTURE ONLY).  The
 * transform definition it restates is in orc_fft.h. */
#include "orc_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int smallest_factor(int n)
{
    int p;
    if (n % 2 == 0) return 2;
    for (p = 3; (long)p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

/* out[k] = sum_j in[j*s] * W^(j*k*step), W = exp(sign*2*pi*i/N) (tw holds W^e, e < N),
 * for a transform of length n = N/step.  out is contiguous; tmp holds 4*n doubles. */
static void rec(const double *in, long s, double *out, int n, const double *tw, long N, long step, double *tmp)
{
    int p, m, r, q, k;
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    p = smallest_factor(n);
    m = n / p;
    /* sub-transforms Y_r (length m) of the samples r, r+p, r+2p, ... into out[r*m ...] */
    for (r = 0; r < p; r++) rec(in + 2 * r * s, s * p, out + 2 * (long)r * m, m, tw, N, step * p, tmp);
    /* X[k + q*m] = sum_r W_n^(r*(k + q*m)) Y_r[k] */
    for (k = 0; k < m; k++) {
        double *t = tmp, *u = tmp + 2 * p;
        for (r = 0; r < p; r++) {
            long e = ((long)r * k % n) * step;
            double wr = tw[2 * e], wi = tw[2 * e + 1];
            double yr = out[2 * ((long)r * m + k)], yi = out[2 * ((long)r * m + k) + 1];
            t[2 * r] = yr * wr - yi * wi;
            t[2 * r + 1] = yr * wi + yi * wr;
        }
        for (q = 0; q < p; q++) {
            double sr = 0.0, si = 0.0;
            for (r = 0; r < p; r++) {
                long e = ((long)r * q % p) * m * step;
                double wr = tw[2 * e], wi = tw[2 * e + 1];
                sr += t[2 * r] * wr - t[2 * r + 1] * wi;
                si += t[2 * r] * wi + t[2 * r + 1] * wr;
            }
            u[2 * q] = sr;
            u[2 * q + 1] = si;
        }
        for (q = 0; q < p; q++) {
            out[2 * (k + (long)q * m)] = u[2 * q];
            out[2 * (k + (long)q * m) + 1] = u[2 * q + 1];
        }
    }
    (void)N;
}

int orc_dft_1d(double *x, int n, long stride, int sign)
{
    double *tw, *out, *tmp;
    long j;
    if (n <= 1) return 0;
    tw = (double *)malloc(sizeof(double) * 2 * n);
    out = (double *)malloc(sizeof(double) * 2 * n);
    tmp = (double *)malloc(sizeof(double) * 4 * n);
    if (!tw || !out || !tmp) {
        free(tw); free(out); free(tmp);
        return -1;
    }
    for (j = 0; j < n; j++) {
        double a = 2.0 * 3.14159265358979323846 * (double)j / (double)n;
        tw[2 * j] = cos(a);
        tw[2 * j + 1] = sign < 0 ? -sin(a) : sin(a);
    }
    rec(x, stride, out, n, tw, n, 1, tmp);
    for (j = 0; j < n; j++) {
        x[2 * j * stride] = out[2 * j];
        x[2 * j * stride + 1] = out[2 * j + 1];
    }
    free(tw); free(out); free(tmp);
    return 0;
}

int orc_dft_2d(double *x, int n0, int n1, int sign)
{
    int i, rc = 0;
#pragma omp parallel for schedule(static) reduction(| : rc)
    for (i = 0; i < n0; i++) rc |= orc_dft_1d(x + 2 * (long)i * n1, n1, 1, sign);
    if (rc) return -1;
#pragma omp parallel for schedule(static) reduction(| : rc)
    for (i = 0; i < n1; i++) rc |= orc_dft_1d(x + 2 * (long)i, n0, n1, sign);
    return rc ? -1 : 0;
}
