/* orc_interp.c — CPU restatement of the reference's seismic interpolation, used by the
 * real-data path (TEST INFRASTRUCTURE ONLY; never linked into the product):
 *   orc_kaiser          Kaiser window            Interp_function.cpp:10-43
 *   orc_sinc_interp     windowed-sinc resampling  Interp_function.cpp:44-115 (Sinc, sum_ABC,
 *                                                 Sincinterp)
 *   orc_fk_interp       general F-K interpolation Interp_function.cpp:116-244
 *   orc_interp_gather   Interpseis2d              Interp_function.cpp:245-264
 * Float and double evaluation follow the reference expression by expression (its FFTs are
 * FFTW's double-precision DFT, restated in orc_fft.c).  Where the reference's behaviour is
 * undefined the restatement defines it; each case is stated at the function.
 * Parity: pinned to the reference's own Interp_function.cpp, compiled from its sources
 * against an FFTW-interface shim (oracle/ref), and to fixtures made from it. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "orc_fft.h"
#include "rtm_oracle.h"

#define ORC_PI_D 3.1415926535897932   /* the reference's `pi` (common.h:11), a double */

/* modZeroBessel, Interp_function.cpp:10-24: 20-term series of I0 in double. */
static double bessel_i0(double x)
{
    double x_2 = x / 2, num = 1, fact = 1, result = 1;
    int i;
    for (i = 1; i < 20; i++) {
        num *= x_2 * x_2;
        fact *= i;
        result += num / (fact * fact);
    }
    return result;
}

void orc_kaiser(float *w, int n, double beta)
{
    double m_2 = (double)(n - 1) / 2.0, denom = bessel_i0(beta);
    int k;
    for (k = 0; k < n; k++) {
        double v = ((k) - m_2) / m_2;
        v = 1 - (v * v);
        w[k] = (float)(bessel_i0(beta * sqrt(v)) / denom);
    }
}

/* Sinc, Interp_function.cpp:44-52: sin(pi x)/(pi x) in double, returned as float. */
static float sinc_f(float x)
{
    if (x == 0.0f) return (float)cos((double)x);
    return (float)(sin(ORC_PI_D * x) / (ORC_PI_D * x));
}

/* Sincinterp: seisin [nt0][ld_in] (columns 0..nx-1 used) -> seisout [nt][nx].  21-tap
 * Kaiser (beta 2) window around input sample it0 = (int)((it+1)*dt/dt0), sinc centred on
 * t = it*dt; at the start the window is shifted to stay aligned, at the end it is cut from
 * its first tap (the reference's inwstart rule); products and sum in float, left to right. */
void orc_sinc_interp(const float *seisin, int ld_in, float *seisout, int nx, int nt, int nt0, float dt, float dt0)
{
    const float nw = 21;
    const int halfnw = (int)((nw - 1) / 2);
    float wk[21];
    int ix;
    orc_kaiser(wk, (int)nw, 2.0);
#pragma omp parallel for schedule(static)
    for (ix = 0; ix < nx; ix++) {
        int it;
        for (it = 0; it < nt; it++) {
            int it0 = (int)((float)(it + 1) * dt / dt0);
            int itstart = it0 - halfnw > 0 ? it0 - halfnw : 0;
            int itend = nt0 - 1 < it0 + halfnw ? nt0 - 1 : it0 + halfnw;
            int lenit = itend - itstart + 1;
            int inwstart = (int)((float)((itstart > halfnw) * 0) + (float)(itstart <= halfnw) * (nw - (float)lenit));
            float t = (float)it * dt, sum = 0.0f;
            int ik;
            for (ik = 0; ik < lenit; ik++) {
                float tn = (float)(ik + itstart) * dt0;
                float a = seisin[(size_t)(ik + itstart) * ld_in + ix];
                float b = sinc_f((t - tn) / dt0);
                float c = wk[ik + inwstart];
                float abc = a * b;
                abc = abc * c;
                sum = sum + abc;
            }
            seisout[(size_t)it * nx + ix] = sum;
        }
    }
}

/* GeneralFKinterp: seisin [nt0][nx0] -> seisout [nt0][nx], lx-fold in x.
 *  1. K = 2-D DFT of the input as [nx0][nt0]; C = K repeated lx times along x.
 *  2. S = 2-D DFT of the input zero-padded to [lx*nx0][lx*nt0]; Z = the lx aliased copies
 *     of S along x summed and divided by lx, repeated lx times; Z += max|Z| * 1e-5 (real
 *     part); H = S/Z on the first nf = 1 + nt0/2 frequencies, |H| > lx^2 -> H = lx.
 *  3. G1 = H*C per frequency, inverse DFT along x; negative frequencies from the conjugate
 *     of G1 at it1 = (nt0+1)/2, (nt0+1)/2 - 1, ... (mirror = 0, the reference's indexing,
 *     one row off the Hermitian partner nt0-it) or at nt0-it (mirror = 1); inverse DFT
 *     along t; the real part of the first nx columns is the output.
 * |z| is sqrtf of the float-rounded double re^2+im^2 (common.h:25-26).  Undefined in the
 * reference and defined here: for odd nt0 with mirror 0 the first mirrored row lies one
 * past G1 and reads as zero; nx > lx*nx0 is refused (-2).  Returns 0, -1 out of memory. */
int orc_fk_interp(const float *seisin, float *seisout, int nx, int nx0, int nt0, int lx, int mirror)
{
    const int nf = 1 + nt0 / 2, Nx = lx * nx0, Nt = lx * nt0;
    double *K, *S, *Z, *G1, *G;
    float zmax = 0.0f;
    long ix, it, il;
    int rc = 0;
    if (lx < 1 || nx > Nx || nx < 1 || nx0 < 1 || nt0 < 1) return -2;
    K = (double *)calloc((size_t)2 * nx0 * nt0, sizeof(double));
    S = (double *)calloc((size_t)2 * Nx * Nt, sizeof(double));
    Z = (double *)calloc((size_t)2 * nx0 * Nt, sizeof(double));
    G1 = (double *)calloc((size_t)2 * nf * Nx, sizeof(double));
    G = (double *)calloc((size_t)2 * nx * nt0, sizeof(double));
    if (!K || !S || !Z || !G1 || !G) {
        rc = -1;
        goto out;
    }
    for (ix = 0; ix < nx0; ix++)
        for (it = 0; it < nt0; it++) {
            double v = seisin[(size_t)it * nx0 + ix];
            K[2 * (ix * nt0 + it)] = v;
            S[2 * (ix * Nt + it)] = v;
        }
    if (orc_dft_2d(K, nx0, nt0, -1) || orc_dft_2d(S, Nx, Nt, -1)) {
        rc = -1;
        goto out;
    }
    /* aliased sum (one period; the lx copies are identical) */
    for (ix = 0; ix < nx0; ix++)
        for (it = 0; it < Nt; it++) {
            double zr = 0.0, zi = 0.0;
            for (il = 0; il < lx; il++) {
                zr = zr + S[2 * ((ix + il * nx0) * Nt + it)];
                zi = zi + S[2 * ((ix + il * nx0) * Nt + it) + 1];
            }
            zr = zr / lx;
            zi = zi / lx;
            Z[2 * (ix * Nt + it)] = zr;
            Z[2 * (ix * Nt + it) + 1] = zi;
            {
                float m = sqrtf((float)(zr * zr + zi * zi));
                zmax = zmax > m ? zmax : m;
            }
        }
    for (ix = 0; ix < nx0 * (long)Nt; ix++) Z[2 * ix] = Z[2 * ix] + zmax * 0.00001;
    /* H, G1 = H*C (G1 stored [nf][Nx]) */
    for (ix = 0; ix < Nx; ix++)
        for (it = 0; it < nf; it++) {
            const double *s = S + 2 * (ix * Nt + it), *z = Z + 2 * ((ix % nx0) * Nt + it);
            const double *c = K + 2 * ((ix % nx0) * nt0 + it);
            double den = z[0] * z[0] + z[1] * z[1];
            double h0 = (s[0] * z[0] + s[1] * z[1]) / den, h1 = (s[1] * z[0] - s[0] * z[1]) / den;
            if (sqrtf((float)(h0 * h0 + h1 * h1)) > lx * lx) {
                h0 = (float)(lx);
                h1 = 0.0;
            }
            G1[2 * (it * Nx + ix)] = h0 * c[0] - h1 * c[1];
            G1[2 * (it * Nx + ix) + 1] = h0 * c[1] + h1 * c[0];
        }
    for (it = 0; it < nf; it++)
        if (orc_dft_1d(G1 + 2 * it * Nx, Nx, 1, +1)) {
            rc = -1;
            goto out;
        }
    for (ix = 0; ix < nx; ix++) {
        long it1 = (nt0 + 1) / 2;
        for (it = 0; it < nt0; it++) {
            double gr = 0.0, gi = 0.0;
            if (it < nf) {
                gr = G1[2 * (it * Nx + ix)];
                gi = G1[2 * (it * Nx + ix) + 1];
            } else {
                long src = mirror ? nt0 - it : it1;
                if (src < nf) {
                    gr = G1[2 * (src * Nx + ix)];
                    gi = -G1[2 * (src * Nx + ix) + 1];
                }
                it1--;
            }
            G[2 * (ix * nt0 + it)] = gr;
            G[2 * (ix * nt0 + it) + 1] = gi;
        }
        if (orc_dft_1d(G + 2 * ix * nt0, nt0, 1, +1)) {
            rc = -1;
            goto out;
        }
    }
    for (it = 0; it < nt0; it++)
        for (ix = 0; ix < nx; ix++) seisout[(size_t)it * nx + ix] = (float)G[2 * (ix * nt0 + it)];
out:
    free(K); free(S); free(Z); free(G1); free(G);
    return rc;
}

/* Interpseis2d: seisobs [nt0][nx0] (traces at the data spacing, dt0) -> seiscal [nt][nx]
 * (model spacing, dt).  lx = (nx-1)/(nx0-1).  x and t: F-K then sinc; x only: F-K; t only:
 * sinc on the first nx traces.  Defined here where the reference is not: with neither
 * (nx <= nx0, nt <= nt0) the reference leaves seiscal unwritten (it assigns the pointer
 * only) and this copies the first nt samples of the first nx traces; in the x-only branch
 * with nt < nt0 the reference writes nt0 rows into nt and this keeps the first nt; nx > nx0
 * with nx0 < 2 (a division by zero there) is refused (-2).  Returns 0, -1, -2. */
int orc_interp_gather(const float *seisobs, int nx0, int nt0, float *seiscal, int nx, int nt, float dt, float dt0,
                      int mirror)
{
    int rc = 0;
    if (nx > nx0) {
        int lx;
        float *tmp;
        if (nx0 < 2) return -2;
        lx = (nx - 1) / (nx0 - 1);
        tmp = (float *)malloc(sizeof(float) * (size_t)nt0 * nx);
        if (!tmp) return -1;
        rc = orc_fk_interp(seisobs, tmp, nx, nx0, nt0, lx, mirror);
        if (!rc) {
            if (nt > nt0) orc_sinc_interp(tmp, nx, seiscal, nx, nt, nt0, dt, dt0);
            else memcpy(seiscal, tmp, sizeof(float) * (size_t)nt * nx);
        }
        free(tmp);
        return rc;
    }
    if (nt > nt0) {
        orc_sinc_interp(seisobs, nx0, seiscal, nx, nt, nt0, dt, dt0);
        return 0;
    }
    {
        int it;
        for (it = 0; it < nt; it++) memcpy(seiscal + (size_t)it * nx, seisobs + (size_t)it * nx0, sizeof(float) * nx);
    }
    return 0;
}
