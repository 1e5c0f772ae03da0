/*
 * rtm_oracle_impl.h — precision-templated body of the oracle (TEST INFRASTRUCTURE ONLY).
 * Included twice by rtm_oracle.c with R = float / double and SFX(x) = x##_f32 / x##_f64.
 *
 * The loops restate the reference kernels (gubingluo kernel.cu) cell by cell, in the
 * reference's launch order within one time step (rtm_model.cu:326-336, 413-455).
 * Region boundaries follow the reference at npml == 32 and generalise to any npml >= 10.
 */

typedef struct {
    R *p, *vx, *vz;
    R *pl1, *pl2, *pr1, *pr2;   /* [Z][npml]         kernel.cu:714-841 */
    R *pt1, *pt2, *pb1, *pb2;   /* [npml][X-2*npml]  kernel.cu:842-963 */
} SFX(wave);

typedef struct {
    int X, Z, npml;
    R dt, dtx, dtz;
    R coef[100];
    const R *vp2, *rho;          /* current model (v^2 and density), padded */
    R *ddx, *ddz, *ddxvx, *ddzvz;
    int *norder, *norderx, *norderz;
} SFX(ctx);

static void SFX(wave_alloc)(SFX(wave) *w, int X, int Z, int npml)
{
    size_t nxi = (size_t)(X - 2 * npml);
    w->p = (R *)calloc((size_t)X * Z, sizeof(R));
    w->vx = (R *)calloc((size_t)(X - 1) * Z, sizeof(R));
    w->vz = (R *)calloc((size_t)X * (Z - 1), sizeof(R));
    w->pl1 = (R *)calloc((size_t)npml * Z, sizeof(R));
    w->pl2 = (R *)calloc((size_t)npml * Z, sizeof(R));
    w->pr1 = (R *)calloc((size_t)npml * Z, sizeof(R));
    w->pr2 = (R *)calloc((size_t)npml * Z, sizeof(R));
    w->pt1 = (R *)calloc((size_t)npml * nxi, sizeof(R));
    w->pt2 = (R *)calloc((size_t)npml * nxi, sizeof(R));
    w->pb1 = (R *)calloc((size_t)npml * nxi, sizeof(R));
    w->pb2 = (R *)calloc((size_t)npml * nxi, sizeof(R));
}

static void SFX(wave_free)(SFX(wave) *w)
{
    free(w->p); free(w->vx); free(w->vz);
    free(w->pl1); free(w->pl2); free(w->pr1); free(w->pr2);
    free(w->pt1); free(w->pt2); free(w->pb1); free(w->pb2);
}

/* Velocity update of one wavefield, whole padded grid.
 * vx: kernel.cu:430-465 (interior columns, full order) and kernel.cu:542-630 (PML columns,
 * local order norderx, damped with ddxVx).  vz: kernel.cu:466-500 and kernel.cu:631-713. */
static void SFX(fwd_v)(SFX(wave) *w, const SFX(ctx) *c)
{
    const int X = c->X, Z = c->Z, npml = c->npml;
    const R *p = w->p;
    int iz;
#pragma omp parallel for schedule(static)
    for (iz = 0; iz < Z; iz++) {
        int ix, i;
        for (ix = 0; ix < X - 1; ix++) {
            int interior = (ix >= npml && ix <= X - npml - 2);
            int r = interior ? ORC_RADIUS : c->norderx[ix] / 2;
            const R *cf = &c->coef[(r - 1) * ORC_RADIUS];
            const R *pr = &p[(size_t)iz * X + ix];
            R d = 0;
            for (i = 1; i <= r; i++) d += cf[i - 1] * (pr[i] - pr[-i + 1]);
            d = d * c->dtx / c->rho[(size_t)iz * X + ix];
            R *v = &w->vx[(size_t)iz * (X - 1) + ix];
            if (interior) {
                *v -= d;
            } else {
                R c1 = (R)(1.0 - 0.5 * c->dt * c->ddxvx[ix]);
                R c2 = (R)(2.0 - c1);
                *v = (c1 * *v - d) / c2;
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (iz = 0; iz < Z - 1; iz++) {
        int ix, i;
        int interior = (iz >= npml && iz <= Z - npml - 2);
        int r = interior ? ORC_RADIUS : c->norderz[iz] / 2;
        const R *cf = &c->coef[(r - 1) * ORC_RADIUS];
        R c1 = 1, c2 = 1;
        if (!interior) {
            c1 = (R)(1.0 - 0.5 * c->dt * c->ddzvz[iz]);
            c2 = (R)(2.0 - c1);
        }
        for (ix = 0; ix < X; ix++) {
            const R *pc = &p[(size_t)iz * X + ix];
            R d = 0;
            for (i = 1; i <= r; i++) d += cf[i - 1] * (pc[(size_t)i * X] - pc[-(ptrdiff_t)(i - 1) * X]);
            d = d * c->dtz / c->rho[(size_t)iz * X + ix];
            R *v = &w->vz[(size_t)iz * X + ix];
            if (interior) *v -= d;
            else *v = (c1 * *v - d) / c2;
        }
    }
}

/* Pressure update of one wavefield, whole padded grid: interior kernel.cu:501-541,
 * left/right strips kernel.cu:714-841, top/bottom kernel.cu:842-963, corners
 * kernel.cu:964-1185.  Row 0, row Z-1, column 0 and column X-1 are never updated. */
static void SFX(fwd_p)(SFX(wave) *w, const SFX(ctx) *c)
{
    const int X = c->X, Z = c->Z, npml = c->npml;
    const int nxi = X - 2 * npml;
    int iz;
#pragma omp parallel for schedule(static)
    for (iz = 1; iz < Z - 1; iz++) {
        int ix, i;
        int zb = (iz < npml) ? -1 : (iz >= Z - npml ? 1 : 0);
        for (ix = 1; ix < X - 1; ix++) {
            int xb = (ix < npml) ? -1 : (ix >= X - npml ? 1 : 0);
            int r = (xb == 0 && zb == 0) ? ORC_RADIUS : c->norder[(size_t)iz * X + ix] / 2;
            const R *cf = &c->coef[(r - 1) * ORC_RADIUS];
            const R *vxr = &w->vx[(size_t)iz * (X - 1) + ix];
            const R *vzc = &w->vz[(size_t)iz * X + ix];
            R dxs = 0, dzs = 0;
            for (i = 1; i <= r; i++) {
                dxs += cf[i - 1] * (vxr[i - 1] - vxr[-i]);
                dzs += cf[i - 1] * (vzc[(ptrdiff_t)(i - 1) * X] - vzc[-(ptrdiff_t)i * X]);
            }
            size_t id = (size_t)iz * X + ix;
            dxs = dxs * c->dtx * c->rho[id] * c->vp2[id];
            dzs = dzs * c->dtz * c->rho[id] * c->vp2[id];
            if (xb == 0 && zb == 0) {
                w->p[id] -= dxs + dzs;
                continue;
            }
            R c1x = 1, c2x = 1, c1z = 1, c2z = 1;
            if (xb != 0) { c1x = (R)(1.0 - 0.5 * c->dt * c->ddx[ix]); c2x = (R)(2.0 - c1x); }
            if (zb != 0) { c1z = (R)(1.0 - 0.5 * c->dt * c->ddz[iz]); c2z = (R)(2.0 - c1z); }
            R *s1, *s2;
            if (xb != 0) {            /* left/right strips and the four corners */
                size_t k = (size_t)iz * npml + (xb < 0 ? ix : ix - (X - npml));
                s1 = (xb < 0 ? w->pl1 : w->pr1) + k;
                s2 = (xb < 0 ? w->pl2 : w->pr2) + k;
            } else {                  /* top/bottom strips */
                size_t k = (size_t)(zb < 0 ? iz : iz - (Z - npml)) * nxi + (ix - npml);
                s1 = (zb < 0 ? w->pt1 : w->pb1) + k;
                s2 = (zb < 0 ? w->pt2 : w->pb2) + k;
            }
            *s1 = (c1x * *s1 - dxs) / c2x;
            *s2 = (c1z * *s2 - dzs) / c2z;
            w->p[id] = *s1 + *s2;
        }
    }
}

/* p += dt*src*w[it] over the whole grid (add = +1) or p -= ... (add = -1); kernel.cu:36-47 */
static void SFX(add_source)(R *p, const R *src, R dt, R wit, size_t n, int add)
{
    size_t i;
    for (i = 0; i < n; i++) {
        if (src[i] == 0) continue;  /* adding an exact zero leaves p unchanged */
        if (add > 0) p[i] += dt * src[i] * wit;
        else p[i] -= dt * src[i] * wit;
    }
}

/* Boundary strips (effective-boundary storage), kernel.cu:1186-1400.
 * Per step: vx [2][nzi][10], vz [2][10][nxi], p lr [2][nzi][10], p tb [2][10][nxi]. */
static void SFX(strips_io)(SFX(wave) *w, int X, int Z, int npml, R *svx, R *svz, R *splr,
                           R *sptb, int save, int which /* 1 = v, 2 = p */)
{
    const int nzi = Z - 2 * npml, nxi = X - 2 * npml;
    int iz, ix, k;
    for (iz = 0; iz < nzi; iz++)
        for (k = 0; k < ORC_RADIUS; k++) {
            size_t a = (size_t)iz * ORC_RADIUS + k, b = a + (size_t)ORC_RADIUS * nzi;
            if (which == 1) {
                R *L = &w->vx[(size_t)(iz + npml) * (X - 1) + npml - ORC_RADIUS + k];
                R *Rr = &w->vx[(size_t)(iz + npml) * (X - 1) + X - npml - 1 + k];
                if (save) { svx[a] = *L; svx[b] = *Rr; } else { *L = svx[a]; *Rr = svx[b]; }
            } else {
                R *L = &w->p[(size_t)(iz + npml) * X + npml - ORC_RADIUS + k];
                R *Rr = &w->p[(size_t)(iz + npml) * X + X - npml + k];
                if (save) { splr[a] = *L; splr[b] = *Rr; } else { *L = splr[a]; *Rr = splr[b]; }
            }
        }
    for (k = 0; k < ORC_RADIUS; k++)
        for (ix = 0; ix < nxi; ix++) {
            size_t a = (size_t)k * nxi + ix, b = a + (size_t)ORC_RADIUS * nxi;
            if (which == 1) {
                R *T = &w->vz[(size_t)(npml - ORC_RADIUS + k) * X + ix + npml];
                R *B = &w->vz[(size_t)(Z - npml - 1 + k) * X + ix + npml];
                if (save) { svz[a] = *T; svz[b] = *B; } else { *T = svz[a]; *B = svz[b]; }
            } else {
                R *T = &w->p[(size_t)(npml - ORC_RADIUS + k) * X + ix + npml];
                R *B = &w->p[(size_t)(Z - npml + k) * X + ix + npml];
                if (save) { sptb[a] = *T; sptb[b] = *B; } else { *T = sptb[a]; *B = sptb[b]; }
            }
        }
}

/* Source-wavefield reconstruction, interior only (kernel.cu:318-429):
 * v += (dt/h)/rho * D(ps) then p += dt*rho*v^2 * D(v). */
static void SFX(bwd_v)(SFX(wave) *w, const SFX(ctx) *c)
{
    const int X = c->X, Z = c->Z, npml = c->npml;
    const R *cf = &c->coef[(ORC_RADIUS - 1) * ORC_RADIUS];
    int iz;
#pragma omp parallel for schedule(static)
    for (iz = npml; iz < Z - npml; iz++) {
        int ix, i;
        for (ix = npml; ix <= X - npml - 2; ix++) {
            const R *pr = &w->p[(size_t)iz * X + ix];
            R d = 0;
            for (i = 1; i <= ORC_RADIUS; i++) d += cf[i - 1] * (pr[i] - pr[-i + 1]);
            d = d * c->dtx / c->rho[(size_t)iz * X + ix];
            w->vx[(size_t)iz * (X - 1) + ix] += d;
        }
    }
#pragma omp parallel for schedule(static)
    for (iz = npml; iz <= Z - npml - 2; iz++) {
        int ix, i;
        for (ix = npml; ix < X - npml; ix++) {
            const R *pc = &w->p[(size_t)iz * X + ix];
            R d = 0;
            for (i = 1; i <= ORC_RADIUS; i++) d += cf[i - 1] * (pc[(size_t)i * X] - pc[-(ptrdiff_t)(i - 1) * X]);
            d = d * c->dtz / c->rho[(size_t)iz * X + ix];
            w->vz[(size_t)iz * X + ix] += d;
        }
    }
}

static void SFX(bwd_p)(SFX(wave) *w, const SFX(ctx) *c)
{
    const int X = c->X, Z = c->Z, npml = c->npml;
    const R *cf = &c->coef[(ORC_RADIUS - 1) * ORC_RADIUS];
    int iz;
#pragma omp parallel for schedule(static)
    for (iz = npml; iz < Z - npml; iz++) {
        int ix, i;
        for (ix = npml; ix < X - npml; ix++) {
            const R *vxr = &w->vx[(size_t)iz * (X - 1) + ix];
            const R *vzc = &w->vz[(size_t)iz * X + ix];
            R dxs = 0, dzs = 0;
            for (i = 1; i <= ORC_RADIUS; i++) {
                dxs += cf[i - 1] * (vxr[i - 1] - vxr[-i]);
                dzs += cf[i - 1] * (vzc[(ptrdiff_t)(i - 1) * X] - vzc[-(ptrdiff_t)i * X]);
            }
            size_t id = (size_t)iz * X + ix;
            dxs = dxs * c->dtx * c->rho[id] * c->vp2[id];
            dzs = dzs * c->dtz * c->rho[id] * c->vp2[id];
            w->p[id] += dxs + dzs;
        }
    }
}

static void SFX(ctx_init)(SFX(ctx) *c, const orc_shot *s, const float *coef)
{
    int i;
    c->X = s->X; c->Z = s->Z; c->npml = s->npml;
    c->dt = (R)s->dt;
    {
        float dtx = s->dt / s->dx, dtz = s->dt / s->dz;  /* rtm_model.cu:73-74 */
        c->dtx = (R)dtx; c->dtz = (R)dtz;
        if (sizeof(R) == sizeof(double)) {
            c->dtx = (R)((double)s->dt / (double)s->dx);
            c->dtz = (R)((double)s->dt / (double)s->dz);
        }
    }
    for (i = 0; i < 100; i++) c->coef[i] = (R)coef[i];
    {
        float *ddx = (float *)calloc(s->X, sizeof(float)), *ddz = (float *)calloc(s->Z, sizeof(float));
        float *ddxvx = (float *)calloc(s->X - 1, sizeof(float)), *ddzvz = (float *)calloc(s->Z - 1, sizeof(float));
        orc_pml_profiles(ddx, ddz, ddxvx, ddzvz, s->vpmax, s->dx, s->dz, s->npml, s->X, s->Z);
        c->ddx = (R *)malloc(sizeof(R) * s->X); c->ddz = (R *)malloc(sizeof(R) * s->Z);
        c->ddxvx = (R *)malloc(sizeof(R) * (s->X - 1)); c->ddzvz = (R *)malloc(sizeof(R) * (s->Z - 1));
        for (i = 0; i < s->X; i++) c->ddx[i] = (R)ddx[i];
        for (i = 0; i < s->Z; i++) c->ddz[i] = (R)ddz[i];
        for (i = 0; i < s->X - 1; i++) c->ddxvx[i] = (R)ddxvx[i];
        for (i = 0; i < s->Z - 1; i++) c->ddzvz[i] = (R)ddzvz[i];
        free(ddx); free(ddz); free(ddxvx); free(ddzvz);
    }
    c->norder = (int *)calloc((size_t)s->X * s->Z, sizeof(int));
    c->norderx = (int *)calloc(s->X - 1, sizeof(int));
    c->norderz = (int *)calloc(s->Z - 1, sizeof(int));
    orc_norder(c->norder, c->norderx, c->norderz, s->X, s->Z);
}

static void SFX(ctx_free)(SFX(ctx) *c)
{
    free(c->ddx); free(c->ddz); free(c->ddxvx); free(c->ddzvz);
    free(c->norder); free(c->norderx); free(c->norderz);
}

static R *SFX(promote)(const float *a, size_t n)
{
    R *b = (R *)malloc(sizeof(R) * n);
    size_t i;
    for (i = 0; i < n; i++) b[i] = (R)a[i];
    return b;
}

/* Source field: the f32 build uses the reference's float formula; the f64 build evaluates
 * the same Gaussian in double. */
static R *SFX(make_source)(const orc_shot *s)
{
    size_t n = (size_t)s->X * s->Z, i;
    R *src = (R *)malloc(sizeof(R) * n);
    if (sizeof(R) == sizeof(float)) {
        float *f = (float *)malloc(sizeof(float) * n);
        orc_source(f, s->X, s->Z, s->nsx, s->nsz, s->amp, s->alp, s->dx * s->dx, s->dz * s->dz);
        for (i = 0; i < n; i++) src[i] = (R)f[i];
        free(f);
    } else {
        int ix, iz;
        double dx2 = (double)s->dx * s->dx, dz2 = (double)s->dz * s->dz, a = s->alp;
        for (iz = 0; iz < s->Z; iz++)
            for (ix = 0; ix < s->X; ix++) {
                double d = (double)(ix - s->nsx) * (ix - s->nsx) * dx2 + (double)(iz - s->nsz) * (iz - s->nsz) * dz2;
                double v = (double)s->amp * exp(-a * a * d);
                /* keep the reference's support: cells where the float source underflows
                 * to zero stay zero */
                float fd = (float)((ix - s->nsx) * (ix - s->nsx)) * (s->dx * s->dx) +
                           (float)((iz - s->nsz) * (iz - s->nsz)) * (s->dz * s->dz);
                src[(size_t)iz * s->X + ix] = (s->amp * expf(-s->alp * s->alp * fd) == 0.0f) ? 0 : (R)v;
            }
    }
    return src;
}

static R *SFX(make_wavelet)(const orc_shot *s, const float *wavelet)
{
    R *w = (R *)malloc(sizeof(R) * s->nt);
    int it;
    if (wavelet) {
        for (it = 0; it < s->nt; it++) w[it] = (R)wavelet[it];
    } else if (sizeof(R) == sizeof(float)) {
        float *f = (float *)malloc(sizeof(float) * s->nt);
        orc_ricker_device(f, s->fdom, s->dt, s->nt);
        for (it = 0; it < s->nt; it++) w[it] = (R)f[it];
        free(f);
    } else {
        for (it = 0; it < s->nt; it++) {
            double t = 3.1415926535897932 * (double)s->fdom * fabs((double)it * s->dt - 1.0 / s->fdom);
            t *= t;
            w[it] = (R)((1.0 - 2.0 * t) * exp(-t));
        }
    }
    return w;
}

/* Single-precision math in the float build (the reference's CUDA kernels call sqrtf, acosf,
 * cosf and sinf), double precision in the double build. */
static R SFX(m_sqrt)(R x) { return sizeof(R) == 4 ? (R)sqrtf((float)x) : (R)sqrt((double)x); }
static R SFX(m_acos)(R x) { return sizeof(R) == 4 ? (R)acosf((float)x) : (R)acos((double)x); }
static R SFX(m_cos)(R x) { return sizeof(R) == 4 ? (R)cosf((float)x) : (R)cos((double)x); }
static R SFX(m_sin)(R x) { return sizeof(R) == 4 ? (R)sinf((float)x) : (R)sin((double)x); }

/* The extra imaging conditions of one backward step, on the interior, after the receiver
 * update (rtm_model.cu:450-455):
 *   g2  wavefield decomposition (cuda_wavefield_decomposition, kernel.cu:1417-1451): the
 *       up-down, down-up, left-right and right-left products; the reference keeps four
 *       arrays and adds them after the last step (cuda_stack_udlr, :1523-1533), here they
 *       go into one;
 *   g3  Poynting-vector angle weighting ps p cos(theta) (cuda_poynting, :1452-1485); the
 *       reference bins it by whole degrees of theta in 61 arrays and adds the bins after the
 *       last step (cuda_stack_theta, :1534-1545), here it goes straight into the sum;
 *   g3t its "true amplitude" variant ps p 16 pi v / sin(theta);
 *   g4  energy norm (cuda_energynorm, :1486-1522): -(dps)(dp)/(dt^2 v^2) + grad ps . grad p
 *       with the change over the step and centred first differences.
 * extra == 2 reads vx as the reference does: at the pressure cell's flat index z*X + x on
 * the (X-1)-wide vx arrays, and with the receiver's vz in the source term of the Poynting
 * vector.  extra == 1 reads vx at its own cell (z, x) and the source's vz.  The operand
 * types follow the reference's expressions (float values, double literals). */
static void SFX(extra_imaging)(const SFX(wave) *ws, const SFX(wave) *w, const R *ps_pre, const R *p_pre,
                               const R *vp2, int X, int Z, int npml, float dx, float dz, float dt, int extra,
                               R *g2, R *g3, R *g3t, R *g4)
{
    const int nzi = Z - 2 * npml, nxi = X - 2 * npml;
    int iz;
#pragma omp parallel for schedule(static)
    for (iz = 0; iz < nzi; iz++) {
        int ix;
        for (ix = 0; ix < nxi; ix++) {
            const int idz = iz + npml, idx = ix + npml;
            const size_t id = (size_t)idz * X + idx, im = (size_t)iz * nxi + ix;
            const size_t ivx = extra == 2 ? id : (size_t)idz * (X - 1) + idx;
            const R ps = ws->p[id], p = w->p[id];
            const R vxs = ws->vx[ivx], vx = w->vx[ivx], vzs = ws->vz[id], vz = w->vz[id];
            /* decomposition */
            const R vectxs = -ps * vxs, vectzs = -ps * vzs, vectxr = -p * vx, vectzr = -p * vz;
            const R psu = vectzs < 0 ? ps : 0, psd = vectzs > 0 ? ps : 0;
            const R psl = vectxs < 0 ? ps : 0, psr = vectxs > 0 ? ps : 0;
            const R pu = vectzr < 0 ? p : 0, pd = vectzr > 0 ? p : 0;
            const R pl = vectxr < 0 ? p : 0, pr = vectxr > 0 ? p : 0;
            g2[im] += psu * pd + psd * pu + psl * pr + psr * pl;
            /* Poynting angle */
            {
                const R ksx = ps * vxs, ksz = ps * (extra == 2 ? vz : vzs), krx = p * vx, krz = p * vz;
                const R q = (ksx * ksx + ksz * ksz) * (krx * krx + krz * krz);
                const double den = SFX(m_sqrt)(q) > 0 ? (double)SFX(m_sqrt)(q) : 1.0e-6;
                R wt = (R)((double)(ksx * krx + ksz * krz) / den);
                if (wt >= -1.0 && wt <= 1.0) {
                    wt = (R)(0.5 * (double)SFX(m_acos)(wt));
                    wt = (R)(ORC_PI / 2.0 - (double)wt);
                    if (wt > 0 && wt <= ORC_PI / 3.0) {
                        g3[im] += ps * p * SFX(m_cos)(wt);
                        g3t[im] = (R)((double)g3t[im] + (double)(ps * p) * 16.0 * ORC_PI *
                                                           (double)SFX(m_sqrt)(vp2[id]) / (double)SFX(m_sin)(wt));
                    }
                }
            }
            /* energy norm */
            {
                const R psx = (R)(0.5 * (double)(ws->p[id + 1] - ws->p[id - 1]) / dx);
                const R psz = (R)(0.5 * (double)(ws->p[id + X] - ws->p[id - X]) / dz);
                const R px = (R)(0.5 * (double)(w->p[id + 1] - w->p[id - 1]) / dx);
                const R pz = (R)(0.5 * (double)(w->p[id + X] - w->p[id - X]) / dz);
                const R rdt = (R)dt;
                g4[im] += -(ps - ps_pre[id]) * (p - p_pre[id]) / (rdt * rdt * vp2[id]) + psx * px + psz * pz;
            }
        }
    }
}

int SFX(orc_forward)(const orc_shot *s, const float *vp2, const float *rho, const float *coef,
                     const float *wavelet, int nsteps, R *p, R *vx, R *vz, R *gather)
{
    SFX(ctx) c;
    SFX(wave) w;
    size_t n = (size_t)s->X * s->Z;
    int it, j;
    R *m_vp2 = SFX(promote)(vp2, n), *m_rho = SFX(promote)(rho, n);
    R *src = SFX(make_source)(s), *wl = SFX(make_wavelet)(s, wavelet);
    SFX(ctx_init)(&c, s, coef);
    c.vp2 = m_vp2; c.rho = m_rho;
    SFX(wave_alloc)(&w, s->X, s->Z, s->npml);
    for (it = 0; it < nsteps; it++) {
        SFX(fwd_v)(&w, &c);
        SFX(fwd_p)(&w, &c);
        SFX(add_source)(w.p, src, c.dt, wl[it], n, 1);
        if (gather)
            for (j = 0; j < s->nrec; j++)
                gather[(size_t)it * s->nrec + j] = w.p[(size_t)s->rz * s->X + s->rx0 + j];
    }
    if (p) memcpy(p, w.p, sizeof(R) * n);
    if (vx) memcpy(vx, w.vx, sizeof(R) * (size_t)(s->X - 1) * s->Z);
    if (vz) memcpy(vz, w.vz, sizeof(R) * (size_t)s->X * (s->Z - 1));
    SFX(wave_free)(&w);
    SFX(ctx_free)(&c);
    free(m_vp2); free(m_rho); free(src); free(wl);
    return 0;
}

int SFX(orc_shot_ex)(const orc_shot *s, const float *vp2f, const float *rhof, const float *vp2b,
                     const float *rhob, const float *coef, const float *wavelet, int mode,
                     float *gather, int mute, int nw, int tlength, R *g1, R *illum, R *ps_out,
                     R *p_out, int extra, R *g2, R *g3, R *g3t, R *g4)
{
    const int X = s->X, Z = s->Z, npml = s->npml, nt = s->nt;
    const int nzi = Z - 2 * npml, nxi = X - 2 * npml;
    const size_t n = (size_t)X * Z;
    const size_t lv = (size_t)ORC_RADIUS * 2 * nzi, lh = (size_t)ORC_RADIUS * 2 * nxi;
    SFX(ctx) c;
    SFX(wave) w, ws;
    int it, j;
    size_t i;
    R *m_vp2f = SFX(promote)(vp2f, n), *m_rhof = SFX(promote)(rhof, n);
    R *m_vp2b = SFX(promote)(vp2b, n), *m_rhob = SFX(promote)(rhob, n);
    R *src = SFX(make_source)(s), *wl = SFX(make_wavelet)(s, wavelet);
    R *svx = (R *)malloc(sizeof(R) * lv * nt), *splr = (R *)malloc(sizeof(R) * lv * nt);
    R *svz = (R *)malloc(sizeof(R) * lh * nt), *sptb = (R *)malloc(sizeof(R) * lh * nt);
    R *rec = (R *)malloc(sizeof(R) * (size_t)nt * s->nrec);
    float *mig = (float *)malloc(sizeof(float) * (size_t)nt * s->nrec);
    R *ps_pre = extra ? (R *)malloc(sizeof(R) * n) : NULL, *p_pre = extra ? (R *)malloc(sizeof(R) * n) : NULL;
    if (!svx || !splr || !svz || !sptb || !rec || !mig || (extra && (!ps_pre || !p_pre || !g2 || !g3 || !g3t || !g4)))
        return -1;

    SFX(ctx_init)(&c, s, coef);
    SFX(wave_alloc)(&w, X, Z, npml);

    /* Source pass (rtm_model.cu:322-346): forward steps with the source added, strips
     * saved after every step.  In mode 0 the reference first runs a separate modelling
     * pass (rtm_model.cu:266-290) that is the same computation in the same model, so the
     * gather is recorded here from the identical wavefield. */
    c.vp2 = m_vp2f; c.rho = m_rhof;
    for (it = 0; it < nt; it++) {
        SFX(fwd_v)(&w, &c);
        SFX(fwd_p)(&w, &c);
        SFX(add_source)(w.p, src, c.dt, wl[it], n, 1);
        if (mode == 0)
            for (j = 0; j < s->nrec; j++)
                gather[(size_t)it * s->nrec + j] = (float)w.p[(size_t)s->rz * X + s->rx0 + j];
        SFX(strips_io)(&w, X, Z, npml, svx + lv * it, svz + lh * it, NULL, NULL, 1, 1);
        SFX(strips_io)(&w, X, Z, npml, NULL, NULL, splr + lv * it, sptb + lh * it, 1, 2);
    }
    memcpy(mig, gather, sizeof(float) * (size_t)nt * s->nrec);
    if (mute) {
        float dx2 = s->dx * s->dx, dz2 = s->dz * s->dz;
        float rdt = (float)(1.0 / s->dt);  /* rtm_model.cu:75 */
        orc_mute(mig, mute == 2 ? vp2b : vp2f, X, s->nsx, s->nsz, nt, s->rz, s->rx0, s->nrec, nw, tlength, dx2, dz2,
                 rdt);
    }
    for (i = 0; i < (size_t)nt * s->nrec; i++) rec[i] = (R)mig[i];

    /* Backward loop (rtm_model.cu:348-456).  Source side: ps = final forward p, vxs = vzs = 0
     * (the reconstruction restarts the particle velocities from zero). */
    SFX(wave_alloc)(&ws, X, Z, npml);
    memcpy(ws.p, w.p, sizeof(R) * n);
    SFX(wave_free)(&w);
    SFX(wave_alloc)(&w, X, Z, npml);
    for (i = 0; i < (size_t)nzi * nxi; i++) { g1[i] = 0; illum[i] = 0; }
    if (extra)
        for (i = 0; i < (size_t)nzi * nxi; i++) { g2[i] = 0; g3[i] = 0; g3t[i] = 0; g4[i] = 0; }
    c.vp2 = m_vp2b; c.rho = m_rhob;
    for (j = 0; j < s->nrec; j++)                               /* kernel.cu:72-79 */
        w.p[(size_t)s->rz * X + s->rx0 + j] = c.dt * rec[(size_t)(nt - 1) * s->nrec + j];
    for (it = nt - 2; it >= 0; it--) {
        if (extra) {   /* the pressures before this step, for the energy norm (rtm_model.cu:419-420) */
            memcpy(ps_pre, ws.p, sizeof(R) * n);
            memcpy(p_pre, w.p, sizeof(R) * n);
        }
        SFX(strips_io)(&ws, X, Z, npml, svx + lv * (it + 1), svz + lh * (it + 1), NULL, NULL, 0, 1);
        SFX(bwd_v)(&ws, &c);
        SFX(strips_io)(&ws, X, Z, npml, NULL, NULL, splr + lv * it, sptb + lh * it, 0, 2);
        SFX(bwd_p)(&ws, &c);
        SFX(add_source)(ws.p, src, c.dt, wl[it], n, -1);
        SFX(fwd_v)(&w, &c);
        SFX(fwd_p)(&w, &c);
        for (j = 0; j < s->nrec; j++)
            w.p[(size_t)s->rz * X + s->rx0 + j] = c.dt * rec[(size_t)it * s->nrec + j];
        {
            int iz;
#pragma omp parallel for schedule(static)
            for (iz = 0; iz < nzi; iz++) {                      /* kernel.cu:1401-1416 */
                int ix;
                for (ix = 0; ix < nxi; ix++) {
                    size_t id = (size_t)(iz + npml) * X + ix + npml;
                    size_t im = (size_t)iz * nxi + ix;
                    g1[im] += ws.p[id] * w.p[id];
                    illum[im] += ws.p[id] * ws.p[id];
                }
            }
        }
        if (extra)
            SFX(extra_imaging)(&ws, &w, ps_pre, p_pre, m_vp2b, X, Z, npml, s->dx, s->dz, s->dt, extra, g2, g3, g3t,
                               g4);
    }
    if (ps_out) memcpy(ps_out, ws.p, sizeof(R) * n);
    if (p_out) memcpy(p_out, w.p, sizeof(R) * n);

    SFX(wave_free)(&w);
    SFX(wave_free)(&ws);
    SFX(ctx_free)(&c);
    free(m_vp2f); free(m_rhof); free(m_vp2b); free(m_rhob);
    free(src); free(wl); free(svx); free(splr); free(svz); free(sptb); free(rec); free(mig);
    free(ps_pre); free(p_pre);
    return 0;
}

int SFX(orc_shot)(const orc_shot *s, const float *vp2f, const float *rhof, const float *vp2b,
                  const float *rhob, const float *coef, const float *wavelet, int mode,
                  float *gather, int mute, int nw, int tlength, R *g1, R *illum, R *ps_out,
                  R *p_out)
{
    return SFX(orc_shot_ex)(s, vp2f, rhof, vp2b, rhob, coef, wavelet, mode, gather, mute, nw, tlength, g1, illum,
                            ps_out, p_out, 0, NULL, NULL, NULL, NULL);
}
