/*
 * rtm_oracle.c — CPU restatement of the reference's RTM hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see rtm_oracle.h).  Built with -ffp-contract=off so the float
 * build evaluates each expression exactly as written, independent of the host CPU.
 */
#include "rtm_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.1415926535897932 /* common.h:11 */

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Liu-Yang optimised staggered-grid coefficients, half-orders 1..10
 * (FD_function.cpp:73-165); table layout c[(h-1)*10 + i-1] as built at
 * RTM_GPU_velstr.cpp:184-196.  These are the reference's published constants. */
void orc_coef_table(float *c)
{
    static const float t[10][10] = {
        {1.0f},
        {0.1129042e+1f, -0.4301412e-1f},
        {0.1185991e+1f, -0.7249965e-1f, 0.6301572e-2f},
        {0.1217990e+1f, -0.9382142e-1f, 0.1507536e-1f, -0.1700324e-2f},
        {0.1236607e+1f, -0.1082265e+0f, 0.2343440e-1f, -0.5033546e-2f, 0.6817483e-3f},
        {0.1247662e+1f, -0.1175538e+0f, 0.2997970e-1f, -0.8719078e-2f, 0.2215897e-2f,
         -0.3462075e-3f},
        {0.1254799e+1f, -0.1238928e+0f, 0.3494371e-1f, -0.1208897e-1f, 0.4132531e-2f,
         -0.1197110e-2f, 0.2122227e-3f},
        {0.1259312e+1f, -0.1280347e+0f, 0.3841945e-1f, -0.1473229e-1f, 0.5924913e-2f,
         -0.2248618e-2f, 0.7179226e-3f, -0.1400855e-3f},
        {0.1262502e+1f, -0.1310244e+0f, 0.4103928e-1f, -0.1686807e-1f, 0.7530520e-2f,
         -0.3345071e-2f, 0.1380367e-2f, -0.4808410e-3f, 0.1023759e-3f},
        {0.1264748e+1f, -0.1331606e+0f, 0.4296909e-1f, -0.1851897e-1f, 0.8861071e-2f,
         -0.4347073e-2f, 0.2076101e-2f, -0.9164925e-3f, 0.3437446e-3f, -0.7874250e-4f},
    };
    int h, i;
    for (h = 0; h < 10; h++)
        for (i = 0; i < 10; i++) c[h * 10 + i] = t[h][i];
}

/* Ricker wavelet as generated on the device, kernel.cu:13-22:
 * temp = (float)(pi*fdom*|it*dt - 1/fdom|); temp *= temp; w = (1 - 2*temp)*expf(-temp). */
void orc_ricker_device(float *w, float fdom, float dt, int nt)
{
    int it;
    for (it = 0; it < nt; it++) {
        float itdt = (float)it * dt;
        float temp = (float)(ORC_PI * fdom * fabs((double)itdt - 1.0 / fdom));
        temp *= temp;
        w[it] = (float)((1.0 - 2.0 * temp) * expf(-temp));
    }
}

/* Host Ricker (FD_function.cpp:7-24); computed by the reference's main but unused by the
 * migration itself. */
void orc_ricker_host(float *w, float fdom, int nt, float dt)
{
    int i;
    float t0 = (float)(1.0 / fdom);
    for (i = 0; i < nt; i++) {
        float i1 = (float)i;
        float t = (float)(ORC_PI * fdom * (i1 * dt - t0));
        w[i] = (float)((1.0 - 2.0 * powf(t, 2.0f)) * expf(-powf(t, 2.0f)));
    }
}

/* PML damping profiles, kernel.cu:174-269, called at rtm_model.cu:257-260 with
 * (nxpad, nzpad, nxpad-1, nzpad-1). */
static void pml_profile(float *d, float vpmax, float h, int npml, int n, double shift)
{
    float R = 1.0e-10f;
    float dd = npml * h;
    float d0 = (float)(1.5 * vpmax * logf(1 / R) / dd);
    int idx;
    for (idx = 0; idx < n; idx++) {
        float temp;
        if (idx < npml) {
            temp = (shift == 0.0) ? (float)(npml - idx) : (float)((float)(npml - idx) - shift);
            temp = temp / npml;
            temp = temp * temp;
            d[idx] = d0 * temp;
        } else if (idx < n - npml) {
            d[idx] = 0.0f;
        } else {
            temp = (shift == 0.0) ? (float)(idx - n + npml + 1)
                                  : (float)((float)(idx - n + npml + 1) - shift);
            temp = temp / npml;
            temp = temp * temp;
            d[idx] = d0 * temp;
        }
    }
}

void orc_pml_profiles(float *ddx, float *ddz, float *ddxvx, float *ddzvz, float vpmax, float dx,
                      float dz, int npml, int X, int Z)
{
    pml_profile(ddx, vpmax, dx, npml, X, 0.0);
    pml_profile(ddz, vpmax, dz, npml, Z, 0.0);
    pml_profile(ddxvx, vpmax, dx, npml, X - 1, 0.5);
    pml_profile(ddzvz, vpmax, dz, npml, Z - 1, 0.5);
}

static int imin(int a, int b) { return a < b ? a : b; }

/* Local FD order maps, kernel.cu:271-317: norder on the p grid (entries on the outer
 * edge stay 0, as after the cudaMemset at rtm_model.cu:253), norderx on the X-1 vx
 * columns, norderz on the Z-1 vz rows. */
void orc_norder(int *norder, int *norderx, int *norderz, int X, int Z)
{
    const int h = ORC_NORDER / 2;
    int iz, ix;
    memset(norder, 0, sizeof(int) * (size_t)X * Z);
    for (iz = 0; iz < Z; iz++)
        for (ix = 0; ix < X; ix++) {
            int v = -1;
            int inx = (ix >= 1 && ix < X - 1), inz = (iz >= 1 && iz < Z - 1);
            if (!inx || !inz) continue;
            if (iz < h) {
                if (ix < h) v = 2 * imin(ix, iz);
                else if (ix < X - h) v = 2 * iz;
                else v = 2 * imin(iz, X - ix - 1);
            } else if (iz < Z - h) {
                if (ix < h) v = 2 * ix;
                else if (ix < X - h) v = ORC_NORDER;
                else v = 2 * (X - ix - 1);
            } else {
                if (ix < h) v = 2 * imin(ix, Z - iz - 1);
                else if (ix < X - h) v = 2 * (Z - iz - 1);
                else v = 2 * imin(Z - iz - 1, X - ix - 1);
            }
            norder[(size_t)iz * X + ix] = v;
        }
    for (ix = 0; ix < X - 1; ix++) {
        int n = X - 1;
        norderx[ix] = (ix < h) ? 2 * (ix + 1) : (ix < n - h ? ORC_NORDER : 2 * (n - ix));
    }
    for (iz = 0; iz < Z - 1; iz++) {
        int n = Z - 1;
        norderz[iz] = (iz < h) ? 2 * (iz + 1) : (iz < n - h ? ORC_NORDER : 2 * (n - iz));
    }
}

/* Gaussian source, kernel.cu:23-35: src = amp*expf(-alp*alp*dist), dist in m^2 (float). */
void orc_source(float *src, int X, int Z, int nsx, int nsz, float amp, float alp, float dx2,
                float dz2)
{
    int ix, iz;
    for (iz = 0; iz < Z; iz++)
        for (ix = 0; ix < X; ix++) {
            float a = (float)((ix - nsx) * (ix - nsx)) * dx2;
            float b = (float)((iz - nsz) * (iz - nsz)) * dz2;
            float dist = a + b;
            src[(size_t)iz * X + ix] = amp * expf(-alp * alp * dist);
        }
}

/* Direct-wave mute, kernel.cu:96-121 (layout 1/2), :122-147 (layout 3), :148-173 (layout 4).
 * The receiver of trace ix sits at padded column rx0+ix on row rz. */
void orc_mute(float *gather, const float *vp2, int X, int nsx, int nsz, int nt, int rz, int rx0,
              int nrec, int nw, int tlength, float dx2, float dz2, float rdt)
{
    int ix, it;
    for (ix = 0; ix < nrec; ix++) {
        float vtemp = (float)(0.482 * (1.0 / sqrtf(vp2[(size_t)rz * X + rx0 + ix]) +
                                       1.0 / sqrtf(vp2[(size_t)nsz * X + nsx])));
        float a = (float)((rx0 + ix - nsx) * (rx0 + ix - nsx)) * dx2;
        float b = (float)((rz - nsz) * (rz - nsz)) * dz2;
        float dist = sqrtf(a + b);
        int temp = tlength < nt ? tlength : nt;
        int t0 = (int)(dist * vtemp * rdt) + nw;
        int cut = t0 < nt ? t0 : nt;
        cut = cut > temp ? cut : temp;
        cut = cut < nt ? cut : nt;
        for (it = 0; it < nt && it <= cut; it++) gather[(size_t)it * nrec + ix] = 0.0f;
    }
}

/* Lateral taper profile, kernel.cu:1591-1604 (one row; identical for every depth). */
void orc_taper(float *taper, int nxlen, int nwin, float alpha)
{
    int ix;
    for (ix = 0; ix < nxlen; ix++) {
        float v = 1.0f;
        if (ix < nwin) v = expf(-alpha * alpha * (float)(nwin - ix) * (float)(nwin - ix));
        if (ix >= nxlen - nwin)
            v = expf(-alpha * alpha * (float)(ix - nxlen + nwin + 1) * (float)(ix - nxlen + nwin + 1));
        if (ix >= nwin && ix < nxlen - nwin) v = 1.0f;
        taper[ix] = v;
    }
}

int orc_taper_nwin(int nxlength)
{
    int nwin = 50;                   /* rtm_model.cu:70 */
    while (2 * nwin >= nxlength) nwin -= 3;
    return nwin;
}

/* Shot geometry per acquisition layout: 1 bilateral (rtm_model.cu:122-154), 2 full array
 * (:626-650), 3 unilateral right (:1122-1158), 4 unilateral left (:1629-1665). */
int orc_geometry(orc_geom *g, int layout, int ishot, int nx, int nz, int nt, float dx, float dz,
                 float dt, int npml, float spx0, float spz0, float dspx, float offset,
                 float offsetmax)
{
    float spx = 0, spz;
    int NX, sp1, np, nr, is;
    memset(g, 0, sizeof(*g));
    g->noffset = 0;
    if (layout == 2) {
        g->nx1 = 0;
        g->nx2 = nx - 1;
        g->nxlength = g->nx2 - g->nx1 + 1;
        spx = spx0 + (ishot - 1) * dspx;
    } else if (layout == 1 || layout == 3 || layout == 4) {
        NX = (int)(offsetmax / dx + 1);
        sp1 = (int)(spx0 / dx);
        np = (int)(dspx / dx);
        is = sp1 + (ishot - 1) * np;
        if (layout == 1) {
            nr = (NX - 1) / 2;
            g->nx1 = is - nr > 0 ? is - nr : 0;
            g->nx2 = is + nr < nx - 1 ? is + nr : nx - 1;
        } else {
            nr = NX - 1;
            g->noffset = (int)(offset / dx);
            if (layout == 3) {
                g->nx1 = is > 0 ? is : 0;
                g->nx2 = is + nr < nx - 1 ? is + nr : nx - 1;
            } else {
                g->nx1 = is - nr > 0 ? is - nr : 0;
                g->nx2 = is < nx - 1 ? is : nx - 1;
            }
        }
        g->nxlength = g->nx2 - g->nx1 + 1;
        spx = (is - g->nx1) * dx;
    } else {
        return -1;
    }
    spz = spz0;
    if (layout == 1 || layout == 2) {
        g->iTraceAll = (ishot - 1) * g->nxlength + 1;
        g->Offset = (int)(g->nx1 * dx - spx);
        g->gx = (int)(g->nx1 * dx);
        g->Ntrace = g->nxlength;
    } else {
        g->iTraceAll = (ishot - 1) * (g->nxlength - g->noffset) + 1;
        g->Offset = (int)(offset);
        g->gx = (int)(offset + g->nx1 * dx);
        g->Ntrace = g->nxlength - g->noffset;
    }
    g->iTrace = 1;
    g->sx = (int)(spx);
    g->Nt = (unsigned short)(nt);
    g->Dt = (unsigned short)(dt * 1000000);
    g->Dx = dx;
    spx = spx + npml * dx;
    spz = spz + npml * dz;
    g->nxpad = g->nxlength + 2 * npml;
    g->nzpad = nz + 2 * npml;
    g->nsx = (int)(spx / dx);
    g->nsz = (int)(spz / dz);
    g->rx0 = npml + (layout == 3 ? g->noffset : 0);
    g->nrec = g->nxlength - g->noffset;
    return 0;
}

/* ---- model preparation, Velocity_function.cpp ---- */

/* extractvel1 (:2051-2062, square = 1) and extractrho1 (:2063-2073, square = 0). */
void orc_extractvel1(float *out, const float *v, int nx, int nz, int nx1, int nx2, int square)
{
    int ix, iz, nxl = nx2 - nx1 + 1;
    for (iz = 0; iz < nz; iz++)
        for (ix = nx1; ix <= nx2; ix++) {
            float a = v[(size_t)iz * nx + ix];
            out[(size_t)iz * nxl + ix - nx1] = square ? a * a : a;
        }
}

/* extendvel1 (:2011-2030): edge-replicate padding by npml on every side. */
void orc_extendvel1(float *vp, const float *vp0, int nx, int nz, int npml)
{
    int ix, iz, nxpad = nx + 2 * npml, nzpad = nz + 2 * npml;
    for (iz = 0; iz < nz; iz++)
        for (ix = 0; ix < nx; ix++) vp[(size_t)(iz + npml) * nxpad + ix + npml] = vp0[(size_t)iz * nx + ix];
    for (iz = npml; iz < nzpad - npml; iz++)
        for (ix = 0; ix < npml; ix++) {
            vp[(size_t)iz * nxpad + ix] = vp[(size_t)iz * nxpad + npml];
            vp[(size_t)iz * nxpad + nxpad - 1 - ix] = vp[(size_t)iz * nxpad + nxpad - npml - 1];
        }
    for (ix = 0; ix < nxpad; ix++)
        for (iz = 0; iz < npml; iz++) {
            vp[(size_t)iz * nxpad + ix] = vp[(size_t)npml * nxpad + ix];
            vp[(size_t)(nzpad - 1 - iz) * nxpad + ix] = vp[(size_t)(nzpad - 1 - npml) * nxpad + ix];
        }
}

/* pmlvelsmooth1d (:9-103): mirror the interior into the PML, then in-place 4-neighbour
 * averaging of the PML band until the relative change is <= 5e-4 (at most 1001 sweeps). */
void orc_pmlvelsmooth1d(float *vp, int nx, int nz, int npml)
{
    int ix, iz;
    float *w = (float *)malloc(sizeof(float) * (size_t)nx * nz);
#define V(z, x) w[(size_t)(z) * nx + (x)]
    for (ix = 0; ix < npml; ix++)
        for (iz = 1; iz < nz - 1; iz++) {
            vp[(size_t)iz * nx + ix] = vp[(size_t)iz * nx + 2 * npml - ix - 1];
            vp[(size_t)iz * nx + nx - npml + ix] = vp[(size_t)iz * nx + nx - npml - ix - 1];
        }
    for (iz = 0; iz < npml; iz++)
        for (ix = 1; ix < nx - 1; ix++) {
            vp[(size_t)iz * nx + ix] = vp[(size_t)(2 * npml - iz - 1) * nx + ix];
            vp[(size_t)(nz - npml + iz) * nx + ix] = vp[(size_t)(nz - npml - iz - 1) * nx + ix];
        }
    {
        float Error = 1.0f;
        int Num = 0;
        float MaxIter = 1000;
        memcpy(w, vp, sizeof(float) * (size_t)nx * nz);
        while (Num <= MaxIter && Error > 0.0005) {
            for (ix = 1; ix < npml; ix++)
                for (iz = 1; iz < nz - 1; iz++) {
                    V(iz, ix) = (float)(0.25 * (V(iz, ix + 1) + V(iz, ix - 1) + V(iz + 1, ix) + V(iz - 1, ix)));
                    V(iz, ix + nx - npml - 1) =
                        (float)(0.25 * (V(iz, ix + nx - npml) + V(iz, ix + nx - npml - 2) +
                                        V(iz + 1, ix + nx - npml - 1) + V(iz - 1, ix + nx - npml - 1)));
                }
            for (ix = 1; ix < nx - 1; ix++)
                for (iz = 1; iz < npml; iz++) {
                    V(iz, ix) = (float)(0.25 * (V(iz, ix + 1) + V(iz, ix - 1) + V(iz + 1, ix) + V(iz - 1, ix)));
                    V(iz + nz - npml - 1, ix) =
                        (float)(0.25 * (V(iz + nz - npml - 1, ix + 1) + V(iz + nz - npml - 1, ix - 1) +
                                        V(iz + nz - npml, ix) + V(iz + nz - npml - 2, ix)));
                }
            for (iz = 1; iz < nz - 1; iz++) {
                V(iz, 0) = (float)(0.25 * (V(iz, 0) + V(iz, 1) + V(iz + 1, 0) + V(iz - 1, 0)));
                V(iz, nx - 1) = (float)(0.25 * (V(iz, nx - 1) + V(iz, nx - 2) + V(iz + 1, nx - 1) + V(iz - 1, nx - 1)));
            }
            for (ix = 1; ix < nx - 1; ix++) {
                V(0, ix) = (float)(0.25 * (V(0, ix) + V(1, ix) + V(0, ix - 1) + V(0, ix + 1)));
                V(nz - 1, ix) = (float)(0.25 * (V(nz - 1, ix) + V(nz - 2, ix) + V(nz - 1, ix - 1) + V(nz - 1, ix + 1)));
            }
            V(0, 0) = (float)(0.25 * (V(0, 0) + V(1, 0) + V(0, 1) + V(1, 1)));
            V(nz - 1, 0) = (float)(0.25 * (V(nz - 1, 0) + V(nz - 2, 0) + V(nz - 1, 1) + V(nz - 2, 1)));
            V(0, nx - 1) = (float)(0.25 * (V(0, nx - 1) + V(0, nx - 2) + V(1, nx - 1) + V(1, nx - 2)));
            V(nz - 1, nx - 1) = (float)(0.25 * (V(nz - 1, nx - 1) + V(nz - 2, nx - 1) + V(nz - 1, nx - 2) + V(nz - 2, nx - 2)));
            {
                float maxvel = -1.0e+5f;
                size_t i, n = (size_t)nx * nz;
                for (i = 0; i < n; i++) {
                    double r = fabs((double)(vp[i] - w[i])) / fabs((double)vp[i]);
                    maxvel = (float)(r > maxvel ? r : maxvel);
                }
                Error = maxvel;
                memcpy(vp, w, sizeof(float) * n);
            }
            Num = Num + 1;
        }
    }
#undef V
    free(w);
}

/* velsmooth1d (:199-313): Gaussian smoothing, half-window nsp, sigma = nsp/3, edge
 * replicated, weights and sums in double. */
void orc_velsmooth1d(float *vp, int n1, int n2, int nsp)
{
    int n1e = n1 + 2 * nsp, n2e = n2 + 2 * nsp, i1, i2, i11, i22;
    float *b = (float *)calloc((size_t)n1e * n2e, sizeof(float));
    float *a = (float *)calloc((size_t)n1 * n2, sizeof(float));
    double a1, b1;
#define B(i, j) b[(size_t)(i) * n2e + (j)]
    for (i1 = 0; i1 < n1; i1++)
        for (i2 = 0; i2 < n2; i2++) B(i1 + nsp, i2 + nsp) = vp[(size_t)i1 * n2 + i2];
    for (i1 = 0; i1 < n1; i1++)
        for (i2 = 0; i2 < nsp; i2++) {
            B(i1 + nsp, i2) = vp[(size_t)i1 * n2];
            B(i1 + nsp, i2 + n2 + nsp) = vp[(size_t)i1 * n2 + n2 - 1];
        }
    for (i1 = 0; i1 < nsp; i1++)
        for (i2 = 0; i2 < n2; i2++) {
            B(i1, i2 + nsp) = vp[i2];
            B(nsp + n1 + i1, i2 + nsp) = vp[(size_t)(n1 - 1) * n2 + i2];
        }
    for (i1 = 0; i1 < nsp; i1++)
        for (i2 = 0; i2 < nsp; i2++) {
            B(i1, i2) = vp[0];
            B(i1, nsp + n2 + i2) = vp[n2 - 1];
            B(i1 + nsp + n1, i2) = vp[(size_t)(n1 - 1) * n2];
            B(i1 + nsp + n1, i2 + nsp + n2) = vp[(size_t)(n1 - 1) * n2 + n2 - 1];
        }
    {
        double *wt = (double *)malloc(sizeof(double) * (size_t)(2 * nsp + 1) * (2 * nsp + 1));
        for (i11 = -nsp; i11 <= nsp; i11++)
            for (i22 = -nsp; i22 <= nsp; i22++) {
                double d1 = i11, d2 = i22;
                wt[(size_t)(i11 + nsp) * (2 * nsp + 1) + i22 + nsp] =
                    exp(-(d1 * d1 + d2 * d2) / (2.0 * nsp / 3.0 * nsp / 3.0));
            }
#pragma omp parallel for private(i2, i11, i22, a1) schedule(static)
        for (i1 = nsp; i1 < n1 + nsp; i1++)
            for (i2 = nsp; i2 < n2 + nsp; i2++) {
                a1 = 0;
                for (i11 = i1 - nsp; i11 <= i1 + nsp; i11++)
                    for (i22 = i2 - nsp; i22 <= i2 + nsp; i22++)
                        a1 += wt[(size_t)(i11 - i1 + nsp) * (2 * nsp + 1) + i22 - i2 + nsp] * B(i11, i22);
                a[(size_t)(i1 - nsp) * n2 + i2 - nsp] = (float)a1;
            }
        free(wt);
    }
    a1 = 0;
    for (i11 = 0; i11 <= 2.0 * nsp; i11++)
        for (i22 = 0; i22 <= 2.0 * nsp; i22++) {
            double d1 = i11 - nsp, d2 = i22 - nsp;
            b1 = exp(-(d1 * d1 + d2 * d2) / (2.0 * nsp / 3.0 * nsp / 3.0));
            a1 += b1;
        }
    for (i1 = 0; i1 < n1; i1++)
        for (i2 = 0; i2 < n2; i2++) vp[(size_t)i1 * n2 + i2] = (float)(a[(size_t)i1 * n2 + i2] / a1);
#undef B
    free(a);
    free(b);
}

/* interpvel1 (:1946-1975): bilinear refinement by integer factors lx, lz. */
void orc_interpvel1(const float *vp0, float *vp, int nx0, int nz0, int nx, int nz, int lx, int lz)
{
    int ix, iz, il;
    float *vel = (float *)malloc(sizeof(float) * (size_t)nx * nz0);
    (void)nz;
    for (iz = 0; iz < nz0; iz++) {
        for (ix = 0; ix < nx0 - 1; ix++)
            for (il = 0; il < lx; il++)
                vel[(size_t)iz * nx + ix * lx + il] =
                    ((lx - il) * vp0[(size_t)iz * nx0 + ix] + il * vp0[(size_t)iz * nx0 + ix + 1]) / lx;
        vel[(size_t)iz * nx + (nx0 - 1) * lx] = vp0[(size_t)iz * nx0 + nx0 - 1];
    }
    for (ix = 0; ix < nx; ix++) {
        for (iz = 0; iz < nz0 - 1; iz++)
            for (il = 0; il < lz; il++)
                vp[(size_t)(iz * lz + il) * nx + ix] =
                    ((lz - il) * vel[(size_t)iz * nx + ix] + il * vel[(size_t)(iz + 1) * nx + ix]) / lz;
        vp[(size_t)(nz0 - 1) * lz * nx + ix] = vel[(size_t)(nz0 - 1) * nx + ix];
    }
    free(vel);
}

/* laplacefd1d (image_function.cpp:44-79): 5-point Laplacian with integer dx, dz; the
 * second differences are formed in double, the border is zeroed. */
void orc_laplacefd1d(int nx, int nz, int dx, int dz, float *image)
{
    int ix, iz;
    float *c = (float *)malloc(sizeof(float) * (size_t)nx * nz);
    memcpy(c, image, sizeof(float) * (size_t)nx * nz);
    for (ix = 1; ix < nx - 1; ix++)
        for (iz = 1; iz < nz - 1; iz++) {
            const float *r = &c[(size_t)iz * nx + ix];
            float t1 = (float)((r[1] + r[-1] - 2.0 * r[0]) / (dx * dx));
            float t2 = (float)((r[nx] + r[-nx] - 2.0 * r[0]) / (dz * dz));
            image[(size_t)iz * nx + ix] = t1 + t2;
        }
    for (ix = 0; ix < nx; ix++) { image[ix] = 0.0f; image[(size_t)(nz - 1) * nx + ix] = 0.0f; }
    for (iz = 0; iz < nz; iz++) { image[(size_t)iz * nx] = 0.0f; image[(size_t)iz * nx + nx - 1] = 0.0f; }
    free(c);
}

/* scaleimage1d (image_function.cpp:11-20): grad /= illum + 1e-4*max|illum|. */
void orc_scaleimage1d(const float *illum, float *grad, int n)
{
    int i;
    float m = fabsf(illum[0]);
    for (i = 0; i < n; i++) m = fabsf(illum[i]) > m ? fabsf(illum[i]) : m;
    {
        float maxillum = (float)(0.0001 * m);
        for (i = 0; i < n; i++) grad[i] /= illum[i] + maxillum;
    }
}

/* get_constant (RTM_GPU_velstr.cpp:319-362): dispersion regrid and CFL check. */
void orc_get_constant(const float *vp, float fdom, float dx0, float dz0, int nx0, int nz0, int nt0,
                      float dt0, float *dx, float *dz, int *nx, int *nz, int *nt, float *dt, int *lx,
                      int *lz, float *vpmin, float *vpmax)
{
    int i;
    float coef[100], s = 0, hmin, dx_max, dz_max, dt_max, t;
    *dx = dx0; *dz = dz0; *nx = nx0; *nz = nz0; *nt = nt0; *dt = dt0; *lx = 1; *lz = 1;
    *vpmax = vp[0]; *vpmin = vp[0];
    for (i = 0; i < nx0 * nz0; i++) {
        *vpmax = vp[i] > *vpmax ? vp[i] : *vpmax;
        *vpmin = vp[i] < *vpmin ? vp[i] : *vpmin;
    }
    dx_max = (float)((double)(*vpmin / fdom) / 7.25);
    dz_max = dx_max;
    while (dx_max < *dx) { *dx = *dx / 2; *lx = (*lx) * 2; *nx = (*nx - 1) * 2 + 1; }
    while (dz_max < *dz) { *dz = *dz / 2; *lz = (*lz) * 2; *nz = (*nz - 1) * 2 + 1; }
    hmin = (*dx < *dz) ? *dx : *dz;
    orc_coef_table(coef);
    for (i = 0; i < 10; i++) s = (float)(s + fabs((double)coef[90 + i]));
    dt_max = hmin / (float)(sqrtf(2.0f) * s * (*vpmax));
    t = nt0 * dt0;
    if (dt_max < dt0) {
        *dt = (float)((int)(dt_max * 10000.0) * 0.0001);
        *nt = (int)(t / (*dt));
    }
}

/* ---- per-shot finalisation ---- */
void orc_finalize_f32(float *g1, float *illum, int nxlen, int nz, int nx, int nx1, float *image1,
                      float *image2s, float *illum_total)
{
    int ix, iz;
    float *taper = (float *)malloc(sizeof(float) * nxlen);
    orc_taper(taper, nxlen, orc_taper_nwin(nxlen), 0.06f);
    for (iz = 0; iz < nz; iz++)
        for (ix = 0; ix < nxlen; ix++) {
            size_t ip = (size_t)iz * nxlen + ix, jf = (size_t)iz * nx + ix + nx1;
            g1[ip] *= taper[ix];
            illum[ip] *= taper[ix];
            image2s[jf] = (float)(image2s[jf] + g1[ip] / (illum[ip] + 1.0e-6));
            image1[jf] += g1[ip];
            illum_total[jf] += illum[ip];
        }
    free(taper);
}

void orc_finalize_f64(double *g1, double *illum, int nxlen, int nz, int nx, int nx1,
                      double *image1, double *image2s, double *illum_total)
{
    int ix, iz;
    float *taper = (float *)malloc(sizeof(float) * nxlen);
    orc_taper(taper, nxlen, orc_taper_nwin(nxlen), 0.06f);
    for (iz = 0; iz < nz; iz++)
        for (ix = 0; ix < nxlen; ix++) {
            size_t ip = (size_t)iz * nxlen + ix, jf = (size_t)iz * nx + ix + nx1;
            g1[ip] *= taper[ix];
            illum[ip] *= taper[ix];
            image2s[jf] += g1[ip] / (illum[ip] + 1.0e-6);
            image1[jf] += g1[ip];
            illum_total[jf] += illum[ip];
        }
    free(taper);
}

#define FIN_EXTRA(T, NAME)                                                                              \
    void NAME(T *g2, T *g3, T *g4, T *g3t, const T *illum, int nxlen, int nz, int nx, int nx1, T *image3s,     \
              T *image4s, T *image5s, T *image3m, T *image4m, T *image5m, T *imagetrue)                     \
    {                                                                                                          \
        int ix, iz;                                                                                            \
        float *taper = (float *)malloc(sizeof(float) * nxlen);                                                 \
        orc_taper(taper, nxlen, orc_taper_nwin(nxlen), 0.06f);                                                 \
        for (iz = 0; iz < nz; iz++)                                                                            \
            for (ix = 0; ix < nxlen; ix++) {                                                                   \
                size_t ip = (size_t)iz * nxlen + ix, jf = (size_t)iz * nx + ix + nx1;                          \
                g2[ip] *= taper[ix];                                                                           \
                g3[ip] *= taper[ix];                                                                           \
                g4[ip] *= taper[ix];                                                                           \
                g3t[ip] *= taper[ix];                                                                          \
                image3s[jf] = (T)(image3s[jf] + g2[ip] / (illum[ip] + 1.0e-6));                                \
                image4s[jf] = (T)(image4s[jf] + g3[ip] / (illum[ip] + 1.0e-6));                                \
                image5s[jf] = (T)(image5s[jf] + g4[ip] / (illum[ip] + 1.0e-6));                                \
                image3m[jf] += g2[ip];                                                                         \
                image4m[jf] += g3[ip];                                                                         \
                image5m[jf] += g4[ip];                                                                         \
                imagetrue[jf] += g3t[ip];                                                                      \
            }                                                                                                  \
        free(taper);                                                                                           \
    }
/* cuda_taper_image + cuda_applyics / cuda_applyic for the extra images (kernel.cu:1556-1604) */
FIN_EXTRA(float, orc_finalize_extra_f32)
FIN_EXTRA(double, orc_finalize_extra_f64)
#undef FIN_EXTRA

/* ---- precision-templated hot path ---- */
#define R float
#define SFX(x) x##_f32
#include "rtm_oracle_impl.h"
#undef R
#undef SFX

#define R double
#define SFX(x) x##_f64
#include "rtm_oracle_impl.h"
#undef R
#undef SFX
