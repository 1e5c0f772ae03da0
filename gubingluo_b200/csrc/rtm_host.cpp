// rtm_host.cpp — host-side pieces of the RTM path: shot geometry, model preparation,
// coefficient table, SU/SEG-Y/image files and the parameter file.  Each function states
// the reference routine whose behaviour (including its float/double evaluation order and
// integer truncations) it reproduces.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rtm_b200.h"
#include "rtm_internal.h"

namespace rtm {

// ---- errors --------------------------------------------------------------------------
static thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}
void clear_error() { g_last_error.clear(); }
const char *last_error() { return g_last_error.c_str(); }

// ---- coefficients --------------------------------------------------------------------
// Liu-Yang optimised staggered coefficients for half-orders 1..10 (FD_function.cpp:73-165),
// laid out c[(h-1)*10 + i-1] with zeros beyond each order (RTM_GPU_velstr.cpp:184-196).
void coef_table(float *c)
{
    static const float t[10][10] = {
        {1.0f},
        {0.1129042e+1f, -0.4301412e-1f},
        {0.1185991e+1f, -0.7249965e-1f, 0.6301572e-2f},
        {0.1217990e+1f, -0.9382142e-1f, 0.1507536e-1f, -0.1700324e-2f},
        {0.1236607e+1f, -0.1082265e+0f, 0.2343440e-1f, -0.5033546e-2f, 0.6817483e-3f},
        {0.1247662e+1f, -0.1175538e+0f, 0.2997970e-1f, -0.8719078e-2f, 0.2215897e-2f, -0.3462075e-3f},
        {0.1254799e+1f, -0.1238928e+0f, 0.3494371e-1f, -0.1208897e-1f, 0.4132531e-2f, -0.1197110e-2f,
         0.2122227e-3f},
        {0.1259312e+1f, -0.1280347e+0f, 0.3841945e-1f, -0.1473229e-1f, 0.5924913e-2f, -0.2248618e-2f,
         0.7179226e-3f, -0.1400855e-3f},
        {0.1262502e+1f, -0.1310244e+0f, 0.4103928e-1f, -0.1686807e-1f, 0.7530520e-2f, -0.3345071e-2f,
         0.1380367e-2f, -0.4808410e-3f, 0.1023759e-3f},
        {0.1264748e+1f, -0.1331606e+0f, 0.4296909e-1f, -0.1851897e-1f, 0.8861071e-2f, -0.4347073e-2f,
         0.2076101e-2f, -0.9164925e-3f, 0.3437446e-3f, -0.7874250e-4f},
    };
    for (int h = 0; h < 10; h++)
        for (int i = 0; i < 10; i++) c[h * 10 + i] = t[h][i];
}

// ---- geometry ------------------------------------------------------------------------
// Shot window, source node and first-trace header keys for each acquisition layout:
// 1 bilateral (rtm_model.cu:122-154), 2 full array (:626-650), 3 unilateral right
// (:1122-1158), 4 unilateral left (:1629-1665).  Receivers: row npml + receiver_depth;
// layout 3 skips the first noffset columns (kernel.cu:56-63), layout 4 the last noffset.
int shot_geometry(const rtm_survey &s, int ishot, rtm_geometry &g)
{
    std::memset(&g, 0, sizeof(g));
    const float dx = s.dx, dz = s.dz;
    float spx;
    if (s.layout == 2) {
        g.nx1 = 0;
        g.nx2 = s.nx - 1;
        spx = s.spx0 + (ishot - 1) * s.dspx;
    } else if (s.layout == 1 || s.layout == 3 || s.layout == 4) {
        int NX = (int)(s.offsetmax / dx + 1);
        int sp1 = (int)(s.spx0 / dx);
        int np = (int)(s.dspx / dx);
        int is = sp1 + (ishot - 1) * np;
        if (s.layout == 1) {
            int nr = (NX - 1) / 2;
            g.nx1 = std::max(0, is - nr);
            g.nx2 = std::min(s.nx - 1, is + nr);
        } else {
            int nr = NX - 1;
            g.noffset = (int)(s.offset / dx);
            if (s.layout == 3) {
                g.nx1 = std::max(0, is);
                g.nx2 = std::min(s.nx - 1, is + nr);
            } else {
                g.nx1 = std::max(0, is - nr);
                g.nx2 = std::min(s.nx - 1, is);
            }
        }
        spx = (is - g.nx1) * dx;
    } else {
        return fail(RTM_ERR_ARG, "layout must be 1, 2, 3 or 4");
    }
    g.nxlength = g.nx2 - g.nx1 + 1;
    if (g.nxlength < 2) return fail(RTM_ERR_ARG, "shot " + std::to_string(ishot) + " has an empty window");
    if (s.layout == 1 || s.layout == 2) {
        g.iTraceAll = (ishot - 1) * g.nxlength + 1;
        g.Offset = (int)(g.nx1 * dx - spx);
        g.gx = (int)(g.nx1 * dx);
        g.Ntrace = g.nxlength;
    } else {
        g.iTraceAll = (ishot - 1) * (g.nxlength - g.noffset) + 1;
        g.Offset = (int)(s.offset);
        g.gx = (int)(s.offset + g.nx1 * dx);
        g.Ntrace = g.nxlength - g.noffset;
    }
    g.iTrace = 1;
    g.sx = (int)(spx);
    g.Nt = (unsigned short)(s.nt);
    g.Dt = (unsigned short)(s.dt * 1000000);
    g.Dx = dx;
    float spxp = spx + s.npml * dx;
    float spzp = s.spz0 + s.npml * dz;
    g.nxpad = g.nxlength + 2 * s.npml;
    g.nzpad = s.nz + 2 * s.npml;
    g.nsx = (int)(spxp / dx);
    g.nsz = (int)(spzp / dz);
    g.rz = s.npml + s.receiver_depth;
    g.rx0 = s.npml + (s.layout == 3 ? g.noffset : 0);
    g.nrec = g.nxlength - g.noffset;
    if (g.nrec < 1) return fail(RTM_ERR_ARG, "offset leaves no receivers");
    if (g.nsx < 0 || g.nsx >= g.nxpad || g.nsz < 0 || g.nsz >= g.nzpad)
        return fail(RTM_ERR_ARG, "shot " + std::to_string(ishot) + " source lies outside its grid");
    if (g.rz >= g.nzpad - s.npml) return fail(RTM_ERR_ARG, "receiver depth below the model");
    return RTM_OK;
}

// ---- model preparation -----------------------------------------------------------------
// extractvel1 / extractrho1 (Velocity_function.cpp:2051-2073) then extendvel1 (:2011-2030).
void extract_extend(const float *v, int nx, int nz, int nx1, int nx2, int npml, bool square, float *pad)
{
    const int nxl = nx2 - nx1 + 1, nxpad = nxl + 2 * npml, nzpad = nz + 2 * npml;
    for (int iz = 0; iz < nz; iz++)
        for (int ix = 0; ix < nxl; ix++) {
            float a = v[(size_t)iz * nx + ix + nx1];
            pad[(size_t)(iz + npml) * nxpad + ix + npml] = square ? a * a : a;
        }
    for (int iz = npml; iz < nzpad - npml; iz++)
        for (int ix = 0; ix < npml; ix++) {
            pad[(size_t)iz * nxpad + ix] = pad[(size_t)iz * nxpad + npml];
            pad[(size_t)iz * nxpad + nxpad - 1 - ix] = pad[(size_t)iz * nxpad + nxpad - npml - 1];
        }
    for (int ix = 0; ix < nxpad; ix++)
        for (int iz = 0; iz < npml; iz++) {
            pad[(size_t)iz * nxpad + ix] = pad[(size_t)npml * nxpad + ix];
            pad[(size_t)(nzpad - 1 - iz) * nxpad + ix] = pad[(size_t)(nzpad - 1 - npml) * nxpad + ix];
        }
}

// pmlvelsmooth1d (Velocity_function.cpp:9-103): mirror the interior into the PML zone, then
// Gauss-Seidel 4-neighbour averaging of the zone until the largest relative change is at
// most 5e-4 (or 1001 sweeps).
void pml_smooth(float *vp, int nx, int nz, int npml)
{
    for (int ix = 0; ix < npml; ix++)
        for (int iz = 1; iz < nz - 1; iz++) {
            vp[(size_t)iz * nx + ix] = vp[(size_t)iz * nx + 2 * npml - ix - 1];
            vp[(size_t)iz * nx + nx - npml + ix] = vp[(size_t)iz * nx + nx - npml - ix - 1];
        }
    for (int iz = 0; iz < npml; iz++)
        for (int ix = 1; ix < nx - 1; ix++) {
            vp[(size_t)iz * nx + ix] = vp[(size_t)(2 * npml - iz - 1) * nx + ix];
            vp[(size_t)(nz - npml + iz) * nx + ix] = vp[(size_t)(nz - npml - iz - 1) * nx + ix];
        }
    std::vector<float> w(vp, vp + (size_t)nx * nz);
    auto V = [&](int z, int x) -> float & { return w[(size_t)z * nx + x]; };
    auto avg = [](float a, float b, float c, float d) { return (float)(0.25 * (a + b + c + d)); };
    float err = 1.0f;
    int num = 0;
    const float max_iter = 1000;
    while (num <= max_iter && err > 0.0005) {
        for (int ix = 1; ix < npml; ix++)
            for (int iz = 1; iz < nz - 1; iz++) {
                V(iz, ix) = avg(V(iz, ix + 1), V(iz, ix - 1), V(iz + 1, ix), V(iz - 1, ix));
                int xr = ix + nx - npml - 1;
                V(iz, xr) = avg(V(iz, xr + 1), V(iz, xr - 1), V(iz + 1, xr), V(iz - 1, xr));
            }
        for (int ix = 1; ix < nx - 1; ix++)
            for (int iz = 1; iz < npml; iz++) {
                V(iz, ix) = avg(V(iz, ix + 1), V(iz, ix - 1), V(iz + 1, ix), V(iz - 1, ix));
                int zb = iz + nz - npml - 1;
                V(zb, ix) = avg(V(zb, ix + 1), V(zb, ix - 1), V(zb + 1, ix), V(zb - 1, ix));
            }
        for (int iz = 1; iz < nz - 1; iz++) {
            V(iz, 0) = avg(V(iz, 0), V(iz, 1), V(iz + 1, 0), V(iz - 1, 0));
            V(iz, nx - 1) = avg(V(iz, nx - 1), V(iz, nx - 2), V(iz + 1, nx - 1), V(iz - 1, nx - 1));
        }
        for (int ix = 1; ix < nx - 1; ix++) {
            V(0, ix) = avg(V(0, ix), V(1, ix), V(0, ix - 1), V(0, ix + 1));
            V(nz - 1, ix) = avg(V(nz - 1, ix), V(nz - 2, ix), V(nz - 1, ix - 1), V(nz - 1, ix + 1));
        }
        V(0, 0) = avg(V(0, 0), V(1, 0), V(0, 1), V(1, 1));
        V(nz - 1, 0) = avg(V(nz - 1, 0), V(nz - 2, 0), V(nz - 1, 1), V(nz - 2, 1));
        V(0, nx - 1) = avg(V(0, nx - 1), V(0, nx - 2), V(1, nx - 1), V(1, nx - 2));
        V(nz - 1, nx - 1) = avg(V(nz - 1, nx - 1), V(nz - 2, nx - 1), V(nz - 1, nx - 2), V(nz - 2, nx - 2));
        float maxrel = -1.0e+5f;
        const size_t n = (size_t)nx * nz;
        for (size_t i = 0; i < n; i++) {
            double r = std::fabs((double)(vp[i] - w[i])) / std::fabs((double)vp[i]);
            maxrel = (float)(r > maxrel ? r : maxrel);
        }
        err = maxrel;
        std::memcpy(vp, w.data(), sizeof(float) * n);
        num++;
    }
}

// velsmooth1d (Velocity_function.cpp:199-313): 2-D Gaussian of half-width nsp and
// sigma = nsp/3 over an edge-replicated extension; weights and sums in double, each
// output cell summed in the reference's (row, column) order.
void gauss_smooth(float *vp, int n1, int n2, int nsp)
{
    if (nsp <= 0) return;
    const int n1e = n1 + 2 * nsp, n2e = n2 + 2 * nsp, w = 2 * nsp + 1;
    std::vector<float> b((size_t)n1e * n2e);
    auto clampi = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
    for (int i1 = 0; i1 < n1e; i1++)
        for (int i2 = 0; i2 < n2e; i2++)
            b[(size_t)i1 * n2e + i2] = vp[(size_t)clampi(i1 - nsp, 0, n1 - 1) * n2 + clampi(i2 - nsp, 0, n2 - 1)];
    std::vector<double> wt((size_t)w * w);
    for (int a = -nsp; a <= nsp; a++)
        for (int c = -nsp; c <= nsp; c++) {
            double d1 = a, d2 = c;
            wt[(size_t)(a + nsp) * w + c + nsp] = std::exp(-(d1 * d1 + d2 * d2) / (2.0 * nsp / 3.0 * nsp / 3.0));
        }
    double norm = 0;
    for (int a = 0; a <= 2.0 * nsp; a++)
        for (int c = 0; c <= 2.0 * nsp; c++) {
            double d1 = a - nsp, d2 = c - nsp;
            norm += std::exp(-(d1 * d1 + d2 * d2) / (2.0 * nsp / 3.0 * nsp / 3.0));
        }
    std::vector<float> out((size_t)n1 * n2);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i1 = 0; i1 < n1; i1++)
        for (int i2 = 0; i2 < n2; i2++) {
            double acc = 0;
            for (int a = 0; a < w; a++) {
                const float *br = &b[(size_t)(i1 + a) * n2e + i2];
                const double *wr = &wt[(size_t)a * w];
                for (int c = 0; c < w; c++) acc += wr[c] * br[c];
            }
            out[(size_t)i1 * n2 + i2] = (float)acc;
        }
    for (size_t i = 0; i < out.size(); i++) vp[i] = (float)(out[i] / norm);
}

// interpvel1 (Velocity_function.cpp:1946-1975).
void interp_model(const float *vp0, float *vp, int nx0, int nz0, int nx, int lx, int lz)
{
    std::vector<float> vel((size_t)nx * nz0);
    for (int iz = 0; iz < nz0; iz++) {
        for (int ix = 0; ix < nx0 - 1; ix++)
            for (int il = 0; il < lx; il++)
                vel[(size_t)iz * nx + ix * lx + il] =
                    ((lx - il) * vp0[(size_t)iz * nx0 + ix] + il * vp0[(size_t)iz * nx0 + ix + 1]) / lx;
        vel[(size_t)iz * nx + (nx0 - 1) * lx] = vp0[(size_t)iz * nx0 + nx0 - 1];
    }
    for (int ix = 0; ix < nx; ix++) {
        for (int iz = 0; iz < nz0 - 1; iz++)
            for (int il = 0; il < lz; il++)
                vp[(size_t)(iz * lz + il) * nx + ix] =
                    ((lz - il) * vel[(size_t)iz * nx + ix] + il * vel[(size_t)(iz + 1) * nx + ix]) / lz;
        vp[(size_t)(nz0 - 1) * lz * nx + ix] = vel[(size_t)(nz0 - 1) * nx + ix];
    }
}

// get_constant (RTM_GPU_velstr.cpp:319-362).
void get_constant(const float *vp, float fdom, float dx0, float dz0, int nx0, int nz0, int nt0, float dt0,
                  float *dx, float *dz, int *nx, int *nz, int *nt, float *dt, int *lx, int *lz, float *vpmin,
                  float *vpmax)
{
    *dx = dx0; *dz = dz0; *nx = nx0; *nz = nz0; *nt = nt0; *dt = dt0; *lx = 1; *lz = 1;
    float mx = vp[0], mn = vp[0];
    for (long i = 0; i < (long)nx0 * nz0; i++) { mx = vp[i] > mx ? vp[i] : mx; mn = vp[i] < mn ? vp[i] : mn; }
    *vpmax = mx; *vpmin = mn;
    float dx_max = (float)((double)(*vpmin / fdom) / 7.25);
    float dz_max = dx_max;
    while (dx_max < *dx) { *dx = *dx / 2; *lx = *lx * 2; *nx = (*nx - 1) * 2 + 1; }
    while (dz_max < *dz) { *dz = *dz / 2; *lz = *lz * 2; *nz = (*nz - 1) * 2 + 1; }
    float hmin = (*dx < *dz) ? *dx : *dz;
    float c[100];
    coef_table(c);
    float s = 0;
    for (int i = 0; i < 10; i++) s = (float)(s + std::fabs((double)c[90 + i]));
    float dt_max = hmin / (sqrtf(2.0f) * s * (*vpmax));
    float t = nt0 * dt0;
    if (dt_max < dt0) {
        *dt = (float)((int)(dt_max * 10000.0) * 0.0001);
        *nt = (int)(t / (*dt));
    }
}

// laplacefd1d (image_function.cpp:44-79).
void laplace_image(float *image, int nx, int nz, int dx, int dz)
{
    std::vector<float> c(image, image + (size_t)nx * nz);
    for (int ix = 1; ix < nx - 1; ix++)
        for (int iz = 1; iz < nz - 1; iz++) {
            const float *r = &c[(size_t)iz * nx + ix];
            float t1 = (float)((r[1] + r[-1] - 2.0 * r[0]) / (dx * dx));
            float t2 = (float)((r[nx] + r[-nx] - 2.0 * r[0]) / (dz * dz));
            image[(size_t)iz * nx + ix] = t1 + t2;
        }
    for (int ix = 0; ix < nx; ix++) { image[ix] = 0.0f; image[(size_t)(nz - 1) * nx + ix] = 0.0f; }
    for (int iz = 0; iz < nz; iz++) { image[(size_t)iz * nx] = 0.0f; image[(size_t)iz * nx + nx - 1] = 0.0f; }
}

// scaleimage1d (image_function.cpp:11-20).
void scale_image(const float *illum, float *grad, int n)
{
    float m = std::fabs(illum[0]);
    for (int i = 0; i < n; i++) m = (float)std::max((double)m, std::fabs((double)illum[i]));
    float maxillum = (float)(0.0001 * m);
    for (int i = 0; i < n; i++) grad[i] /= illum[i] + maxillum;
}

// ---- files ---------------------------------------------------------------------------
static void swap2(void *p)
{
    unsigned char *b = (unsigned char *)p;
    std::swap(b[0], b[1]);
}
static void swap4(void *p)
{
    unsigned char *b = (unsigned char *)p;
    std::swap(b[0], b[3]);
    std::swap(b[1], b[2]);
}

// ReadVelMod (IO_function.cpp:9-35): nx traces, each a 240-byte header and nz native floats.
int read_velocity(const char *path, int nx, int nz, float *vp)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(RTM_ERR_IO, std::string("cannot open velocity file ") + path);
    std::vector<float> tr(nz);
    for (int ix = 0; ix < nx; ix++) {
        if (std::fseek(f, 240L, SEEK_CUR) != 0 || std::fread(tr.data(), sizeof(float), nz, f) != (size_t)nz) {
            std::fclose(f);
            return fail(RTM_ERR_IO, std::string("velocity file too short: ") + path);
        }
        for (int iz = 0; iz < nz; iz++) vp[(size_t)iz * nx + ix] = tr[iz];
    }
    std::fclose(f);
    return RTM_OK;
}

// Output1d (IO_function.cpp:366-422): per column a 120-short header with [0] = trace
// number, [57] = (short)nt, [58] = (short)(d*1e6), [104] = (short)nx, then nt floats.
// The (short) conversions wrap the way x86 truncates through a 32-bit integer.
int write_image_su(const char *path, const float *image, int nz, int nx, float d)
{
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(RTM_ERR_IO, std::string("cannot create ") + path);
    short h[120];
    std::memset(h, 0, sizeof(h));
    h[57] = (short)nz;
    h[58] = (short)(int)(d * 1000000.0);
    h[104] = (short)nx;
    std::vector<float> tr(nz);
    for (int ix = 0; ix < nx; ix++) {
        h[0] = (short)(ix + 1);
        std::fwrite(h, 2, 120, f);
        for (int iz = 0; iz < nz; iz++) tr[iz] = image[(size_t)iz * nx + ix];
        std::fwrite(tr.data(), sizeof(float), nz, f);
    }
    std::fclose(f);
    return RTM_OK;
}

// 240-byte SU/SEG-Y trace header (sgyhead.h:4-89) with the nine keys the reference
// writes (sgyhead_function.cpp:351-383): tracl@0, tracf@12, offset@36, sx@72, gx@80,
// ns@114, dt@116, d2@188, ntr@204.
static void make_trace_header(unsigned char *h, int tracl, int tracf, int offset, int sx, int gx, short ns,
                              short dt, float d2, int ntr, int endian)
{
    std::memset(h, 0, 240);
    auto put4 = [&](int off, const void *v) {
        std::memcpy(h + off, v, 4);
        if (endian) swap4(h + off);
    };
    auto put2 = [&](int off, short v) {
        std::memcpy(h + off, &v, 2);
        if (endian) swap2(h + off);
    };
    put4(0, &tracl);
    put4(12, &tracf);
    put4(36, &offset);
    put4(72, &sx);
    put4(80, &gx);
    put2(114, ns);
    put2(116, dt);
    put4(188, &d2);
    put4(204, &ntr);
}

// Outseisfile1d (IO_function.cpp:131-183) with outflag 0: gather [nt][ntr]; optional
// 3600-byte zero volume header (sgyflag); big-endian samples and headers (endianflag).
int write_gather_su(const char *path, const float *gather, const rtm_geometry &g, int nt, int sgyflag,
                    int endianflag)
{
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(RTM_ERR_IO, std::string("cannot create ") + path);
    if (sgyflag) {
        std::vector<char> vol(3600, 0);
        std::fwrite(vol.data(), 1, 3600, f);
    }
    const short ns = (short)g.Nt;
    const int ntr = g.Ntrace;
    unsigned char h[240];
    std::vector<float> tr(ns > 0 ? ns : 0);
    for (int ix = 0; ix < ntr; ix++) {
        make_trace_header(h, g.iTraceAll + ix, g.iTrace + ix, g.Offset + (int)(ix * g.Dx), g.sx,
                          g.gx + (int)(ix * g.Dx), ns, (short)g.Dt, g.Dx, ntr, endianflag);
        std::fwrite(h, 1, 240, f);
        for (int it = 0; it < ns; it++) {
            float v = it < nt ? gather[(size_t)it * ntr + ix] : 0.0f;
            if (endianflag) swap4(&v);
            tr[it] = v;
        }
        std::fwrite(tr.data(), sizeof(float), ns, f);
    }
    std::fclose(f);
    return RTM_OK;
}

// get_parameter + Inseisfile1d (IO_function.cpp:226-324): detect the byte order from the
// first header's ns/dt (swap when either is <= 0 as little-endian), count traces, read the
// first header's keys and all samples into gather [nt][ntr].
int read_gather_su(const char *path, int sgyflag, float *gather, int *nt_out, int *ntr_out, rtm_geometry *keys)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(RTM_ERR_IO, std::string("cannot open gather ") + path);
    std::fseek(f, 0, SEEK_END);
    long size = std::ftell(f);
    long start = sgyflag ? 3600 : 0;
    if (size < start + 240) {
        std::fclose(f);
        return fail(RTM_ERR_IO, std::string("gather file too short: ") + path);
    }
    unsigned char h[240];
    std::fseek(f, start, SEEK_SET);
    if (std::fread(h, 1, 240, f) != 240) {
        std::fclose(f);
        return fail(RTM_ERR_IO, std::string("cannot read header of ") + path);
    }
    short ns, dt;
    std::memcpy(&ns, h + 114, 2);
    std::memcpy(&dt, h + 116, 2);
    int endian = 0;
    if (dt <= 0 || ns <= 0) {
        short ns2 = ns, dt2 = dt;
        swap2(&ns2);
        swap2(&dt2);
        if (dt2 > 0 && ns2 > 0) { endian = 1; ns = ns2; dt = dt2; }
    }
    if (ns <= 0) {
        std::fclose(f);
        return fail(RTM_ERR_IO, std::string("bad sample count in ") + path);
    }
    long tracebytes = 240 + (long)ns * 4;
    int ntr = (int)((size - start) / tracebytes);
    if (ntr < 1 || (size - start) % tracebytes != 0) {
        std::fclose(f);
        return fail(RTM_ERR_IO, std::string("gather file is not a whole number of traces: ") + path);
    }
    auto get4 = [&](int off) {
        int v;
        std::memcpy(&v, h + off, 4);
        if (endian) swap4(&v);
        return v;
    };
    if (keys) {
        std::memset(keys, 0, sizeof(*keys));
        keys->iTraceAll = get4(0);
        keys->iTrace = get4(12);
        keys->Offset = get4(36);
        keys->sx = get4(72);
        keys->gx = get4(80);
        keys->Nt = ns;
        keys->Dt = dt;
        float d2;
        std::memcpy(&d2, h + 188, 4);
        if (endian) swap4(&d2);
        keys->Dx = d2;
        keys->Ntrace = ntr;
    }
    if (nt_out) *nt_out = ns;
    if (ntr_out) *ntr_out = ntr;
    if (gather) {
        std::vector<float> tr(ns);
        std::fseek(f, start, SEEK_SET);
        for (int ix = 0; ix < ntr; ix++) {
            std::fseek(f, 240L, SEEK_CUR);
            if (std::fread(tr.data(), 4, ns, f) != (size_t)ns) {
                std::fclose(f);
                return fail(RTM_ERR_IO, std::string("short read in ") + path);
            }
            for (int it = 0; it < ns; it++) {
                float v = tr[it];
                if (endian) swap4(&v);
                gather[(size_t)it * ntr + ix] = v;
            }
        }
    }
    std::fclose(f);
    return RTM_OK;
}

// Parameter file (RTM_GPU_velstr.cpp:60-120): ./input/cmd.in names the parameter file on
// its second line; the parameter file alternates one comment line and one value line.
// ---- real-data path: multi-shot SU / SEG-Y files ----------------------------------------
// scanshotgather (RTM_GPU_velstr.cpp:363-454).  Byte order from the first trace header: read
// as little-endian, swapped when its ns or dt is <= 0 (and refused when neither order gives
// positive values).  Every trace is assumed to hold the first header's ns samples.  One pass
// over the headers; a shot starts wherever sx changes.  profile is [4][max_shots]: rows sx,
// trace count, number of the shot's first trace in the file (from 1), offset of that trace.
// The scan stops at the first incomplete trace or at a header with ns or dt <= 0.  Two
// outcomes of the reference are not kept: for a byte-swapped file its end-of-file read swaps
// the last header's keys back, which opens a trailing shot of zero traces (written one entry
// past the shots, beyond a table sized to the shot count); and its trace count includes the
// trace whose header ended the scan.
int scan_shotgather(const char *path, int sgyflag, int *endianflag, int *profile, int max_shots, int *nshots)
{
    if (!path || !profile || max_shots < 1) return fail(RTM_ERR_ARG, "scan_shotgather: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(RTM_ERR_IO, std::string("cannot open shot gather file ") + path);
    std::fseek(f, 0, SEEK_END);
    const long long size = std::ftell(f);
    const long long start = sgyflag ? 3600 : 0;
    unsigned char h[240];
    std::fseek(f, (long)start, SEEK_SET);
    if (size < start + 240 || std::fread(h, 1, 240, f) != 240) {
        std::fclose(f);
        return fail(RTM_ERR_IO, std::string("shot gather file too short: ") + path);
    }
    short ns, dt;
    std::memcpy(&ns, h + 114, 2);
    std::memcpy(&dt, h + 116, 2);
    int endian = 0;
    if (dt <= 0 || ns <= 0) {
        swap2(&ns);
        swap2(&dt);
        if (dt <= 0 || ns <= 0) {
            std::fclose(f);
            return fail(RTM_ERR_IO, std::string("no byte order gives positive ns and dt in ") + path);
        }
        endian = 1;
    }
    auto key4 = [&](int off) {
        int v;
        std::memcpy(&v, h + off, 4);
        if (endian) swap4(&v);
        return v;
    };
    auto key2 = [&](int off) {
        short v;
        std::memcpy(&v, h + off, 2);
        if (endian) swap2(&v);
        return v;
    };
    const long long tb = 240 + (long long)ns * 4;
    int n = 0;
    for (long long k = 0; start + (k + 1) * tb <= size; k++) {
        std::fseek(f, (long)(start + k * tb), SEEK_SET);
        if (std::fread(h, 1, 240, f) != 240) break;
        if (key2(114) <= 0 || key2(116) <= 0) break;
        const int sx = key4(72);
        if (n == 0 || profile[n - 1] != sx) {
            if (n == max_shots) {
                std::fclose(f);
                return fail(RTM_ERR_ARG, std::string("more than ") + std::to_string(max_shots) + " shots in " + path);
            }
            profile[n] = sx;
            profile[max_shots + n] = 0;
            profile[2 * max_shots + n] = (int)(k + 1);
            profile[3 * max_shots + n] = key4(36);
            n++;
        }
        profile[max_shots + n - 1]++;
    }
    std::fclose(f);
    if (endianflag) *endianflag = endian;
    if (nshots) *nshots = n;
    return RTM_OK;
}

// Shot window and source/receiver nodes of one recorded shot (rtm_real.cu:134-157): the
// receivers lie to the right of the source from `offset` on, every dx0 (the data spacing),
// so the spread ends at offsetmax = offset + (ntrace-1)*dx0; the window spans source to last
// receiver on the model grid (dx).  ncols0 = the spread's width on the data grid, the number
// of columns the recorded traces are read into before interpolation.  Refused where the
// reference reads outside the model: a window starting left of x = 0 or ending beyond nx-1.
int real_geometry(const rtm_survey &s, int sx, int offset, int ntrace, float dx0, rtm_geometry &g, int *ncols0)
{
    std::memset(&g, 0, sizeof(g));
    if (ntrace < 1 || !(dx0 > 0.0f)) return fail(RTM_ERR_ARG, "real_geometry: ntrace and dx0 must be positive");
    const float dx = s.dx, dz = s.dz;
    const float offsetmax = (float)(offset + (ntrace - 1) * dx0);
    const float off = (float)offset;
    float spx = (float)sx;
    float spz = s.spz0;
    const int noffset0 = (int)(off / dx0);
    const int nx10 = (int)(spx / dx0);
    const int nx20 = (int)((spx + offsetmax) / dx0);
    g.noffset = (int)(off / dx);
    g.nx1 = (int)(spx / dx);
    g.nx2 = (int)((spx + offsetmax) / dx);
    g.nxlength = g.nx2 - g.nx1 + 1;
    if (sx < 0 || g.nx1 < 0 || g.nx2 > s.nx - 1)
        return fail(RTM_ERR_ARG, "shot at sx = " + std::to_string(sx) + " spreads beyond the model (columns " +
                                     std::to_string(g.nx1) + ".." + std::to_string(g.nx2) + " of " +
                                     std::to_string(s.nx) + ")");
    spx = spx - g.nx1 * dx;
    spx = spx + s.npml * dx;
    spz = spz + s.npml * dz;
    g.nxpad = g.nxlength + 2 * s.npml;
    g.nzpad = s.nz + 2 * s.npml;
    g.nsx = (int)(spx / dx);
    g.nsz = (int)(spz / dz);
    g.rz = s.npml + s.receiver_depth;
    g.rx0 = s.npml + g.noffset;
    g.nrec = g.nxlength - g.noffset;
    g.iTraceAll = 1;
    g.iTrace = 1;
    g.Offset = offset;
    g.sx = sx;
    g.gx = sx + offset;
    g.Nt = (unsigned short)s.nt;
    g.Dt = (unsigned short)(s.dt * 1000000);
    g.Dx = dx;
    g.Ntrace = g.nrec;
    const int nc0 = nx20 - nx10 + 1 - noffset0;
    if (ncols0) *ncols0 = nc0;
    if (g.nxlength < 2 || g.nrec < 1 || nc0 < 1)
        return fail(RTM_ERR_ARG, "shot at sx = " + std::to_string(sx) + " has no receivers on the grid");
    if (g.nsx < 0 || g.nsx >= g.nxpad || g.nsz < 0 || g.nsz >= g.nzpad)
        return fail(RTM_ERR_ARG, "shot at sx = " + std::to_string(sx) + ": source outside its grid");
    if (g.rz >= g.nzpad - s.npml) return fail(RTM_ERR_ARG, "receiver depth below the model");
    return RTM_OK;
}

// The trace-reading loop of rtm_real.cu:379-394: ntrace traces from trace number itrace_all
// on (240-byte header skipped, nt0 floats, byte-swapped when endianflag) into column ix of
// seisobs [nt0][ncols].  Columns from ntrace on are zero (the reference leaves them
// unwritten); traces beyond ncols are not stored (the reference writes past its array).
// Refused: a file too short for the traces, or a first header whose ns is not nt0.
int read_shot_traces(const char *path, int sgyflag, int endianflag, int nt0, long long itrace_all, int ntrace,
                     int ncols, float *seisobs)
{
    if (!path || !seisobs || nt0 < 1 || ncols < 1 || ntrace < 1 || itrace_all < 1)
        return fail(RTM_ERR_ARG, "read_shot_traces: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(RTM_ERR_IO, std::string("cannot open shot gather file ") + path);
    std::fseek(f, 0, SEEK_END);
    const long long size = std::ftell(f);
    const long long tb = 240 + (long long)nt0 * 4;
    const long long first = (itrace_all - 1) * tb + 3600LL * (sgyflag ? 1 : 0);
    if (first + ntrace * tb > size) {
        std::fclose(f);
        return fail(RTM_ERR_IO, std::string("shot gather file ends before trace ") +
                                    std::to_string(itrace_all + ntrace - 1) + ": " + path);
    }
    std::memset(seisobs, 0, sizeof(float) * (size_t)nt0 * ncols);
    std::vector<float> tr(nt0);
    unsigned char h[240];
    int rc = RTM_OK;
    for (int ix = 0; ix < ntrace && ix < ncols && !rc; ix++) {
        std::fseek(f, (long)(first + ix * tb), SEEK_SET);
        if (std::fread(h, 1, 240, f) != 240 || std::fread(tr.data(), sizeof(float), nt0, f) != (size_t)nt0) {
            rc = fail(RTM_ERR_IO, std::string("cannot read trace of ") + path);
            break;
        }
        if (ix == 0) {
            short ns;
            std::memcpy(&ns, h + 114, 2);
            if (endianflag) swap2(&ns);
            if (ns != nt0)
                rc = fail(RTM_ERR_IO, "trace " + std::to_string(itrace_all) + " of " + path + " holds " +
                                          std::to_string(ns) + " samples, not nt0 = " + std::to_string(nt0));
        }
        for (int it = 0; it < nt0; it++) {
            float v = tr[it];
            if (endianflag) swap4(&v);
            seisobs[(size_t)it * ncols + ix] = v;
        }
    }
    std::fclose(f);
    return rc;
}

int read_params(const char *input_dir, rtm_params &p)
{
    std::memset(&p, 0, sizeof(p));
    std::string dir = input_dir ? input_dir : "./input";
    std::string cmdpath = dir + "/cmd.in";
    FILE *fp = std::fopen(cmdpath.c_str(), "r");
    if (!fp) return fail(RTM_ERR_IO, "cmd.in is not exist !");
    char buff[1024], cmd[256];
    if (!std::fgets(buff, sizeof(buff), fp) || std::fscanf(fp, "%255s", cmd) != 1) {
        std::fclose(fp);
        return fail(RTM_ERR_IO, "cmd.in does not name a parameter file");
    }
    std::fclose(fp);
    std::string ppath = dir + "/" + cmd;
    fp = std::fopen(ppath.c_str(), "r");
    if (!fp) return fail(RTM_ERR_IO, std::string(cmd) + " is not exist !");
    int ok = 1;
    auto skip2 = [&]() {
        ok &= std::fgets(buff, sizeof(buff), fp) != nullptr;
        ok &= std::fgets(buff, sizeof(buff), fp) != nullptr;
    };
    auto rf = [&](float *v) { ok &= std::fscanf(fp, "%f", v) == 1; };
    auto ri = [&](int *v) { ok &= std::fscanf(fp, "%d", v) == 1; };
    ok &= std::fgets(buff, sizeof(buff), fp) != nullptr;
    rf(&p.dt0); ri(&p.nt0); rf(&p.tsnap); skip2();
    rf(&p.xmax); rf(&p.zmax); rf(&p.dx0); rf(&p.dz0); skip2();
    rf(&p.fdom); rf(&p.amp); rf(&p.alp); skip2();
    rf(&p.spx0); rf(&p.spz0); rf(&p.dspx); skip2();
    rf(&p.offset); rf(&p.offsetmax); skip2();
    ri(&p.startshot); ri(&p.nshot); ri(&p.dshot); ri(&p.nshotall); skip2();
    ri(&p.npml); skip2();
    ri(&p.medium_flag); ri(&p.ismth); skip2();
    rf(&p.direct); rf(&p.direct0); skip2();
    ri(&p.idevice); skip2();
    ri(&p.flag_layout); skip2();
    ri(&p.mode); skip2();
    ri(&p.dataflag); skip2();
    ri(&p.sgyflag); skip2();
    ri(&p.endianflag); skip2();
    ri(&p.rhoflag); skip2();
    ok &= std::fscanf(fp, "%255s", p.vp_file) == 1;
    if (p.dataflag == 1) { skip2(); ok &= std::fscanf(fp, "%255s", p.shotgather_file) == 1; }
    if (p.rhoflag == 1) { skip2(); ok &= std::fscanf(fp, "%255s", p.rho_file) == 1; }
    std::fclose(fp);
    if (!ok) return fail(RTM_ERR_IO, std::string("parameter file ") + cmd + " is incomplete");
    return RTM_OK;
}

}  // namespace rtm
