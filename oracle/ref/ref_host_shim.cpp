// ref_host_shim.cpp — C-linkage wrappers around the reference's own host functions, so the
// tests can call the reference's C++ code (compiled from its sources under the reference
// checkout, see oracle/ref/Makefile) and pin the oracle and the product's host layer to it.
// TEST INFRASTRUCTURE ONLY: nothing in the product links this.
#include <cstdio>
#include <cstdlib>

#include "function.h"
#include "sgyhead.h"

void get_constant(float *vp, float fdom, float dx0, float dz0, int nx0, int nz0, int nt0,
                  float dt0, float *dx, float *dz, int *nx, int *nz, int *nt, float *dt, int *lx,
                  int *lz, float *vpmin, float *vpmax);
void get_parameter(char buff[40], int sgyflag, int *ntrace, short int *nsample, short int *dt,
                   int *endianflag);

void scanshotgather(char filename_shotgather[40], int **shotprofileId, int sgyflag, int *endianflag);

// RTM_GPU_velstr.cpp is compiled (with its main renamed) only for get_constant; it refers to
// the GPU entry points, which this host-only library never calls.
extern "C" void rtm_model() { std::abort(); }
extern "C" void rtm_real() { std::abort(); }

extern "C" {
void ref_Diff_coeffVelStrLiuyang(float *d, int n) { Diff_coeffVelStrLiuyang(d, n); }
void ref_Ricker(float *w, float fdom, int nt, float dt, int flag) { Ricker(w, fdom, nt, dt, flag); }
void ref_pmlvelsmooth1d(float *vp, int nx, int nz, int npml) { pmlvelsmooth1d(vp, nx, nz, npml); }
void ref_velsmooth1d(float *vp, int n1, int n2, int nsp) { velsmooth1d(vp, n1, n2, nsp); }
void ref_interpvel1(float *vp0, float *vp, int nx0, int nz0, int nx, int nz, int lx, int lz)
{
    interpvel1(vp0, vp, nx0, nz0, nx, nz, lx, lz);
}
void ref_extendvel1(float *vp, float *vp0, int nx, int nz, int npml) { extendvel1(vp, vp0, nx, nz, npml); }
void ref_extractvel1(float *t, float *v, int nx, int nz, int nx1, int nx2) { extractvel1(t, v, nx, nz, nx1, nx2); }
void ref_extractrho1(float *t, float *r, int nx, int nz, int nx1, int nx2) { extractrho1(t, r, nx, nz, nx1, nx2); }
void ref_laplacefd1d(int nx, int nz, int dx, int dz, float *img) { laplacefd1d(nx, nz, dx, dz, img); }
void ref_scaleimage1d(float *illum, float *grad, int n) { scaleimage1d(illum, grad, n); }
float ref_Maxval1(float *v, int n) { return Maxval1(v, n); }
void ref_get_constant(float *vp, float fdom, float dx0, float dz0, int nx0, int nz0, int nt0,
                      float dt0, float *dx, float *dz, int *nx, int *nz, int *nt, float *dt,
                      int *lx, int *lz, float *vpmin, float *vpmax)
{
    get_constant(vp, fdom, dx0, dz0, nx0, nz0, nt0, dt0, dx, dz, nx, nz, nt, dt, lx, lz, vpmin, vpmax);
}
// File I/O: paths are passed through unchanged (ReadVelMod prefixes "./input/").
void ref_Output1d(float *rec, int nt, int nx, float dt, char *path, int flag) { Output1d(rec, nt, nx, dt, path, flag); }
void ref_ReadVelMod(char *name, int nx, int nz, float *vp) { ReadVelMod(name, nx, nz, vp); }
void ref_Outseisfile1d(float *seis, int iTraceAll, int iTrace, int Offset, int sx, int gx, int Nt,
                       int Dt, float Dx, int Ntrace, int outflag, int sgyflag, int endianflag,
                       char *path)
{
    sgyheadkey k;
    k.iTraceAll = iTraceAll; k.iTrace = iTrace; k.Offset = Offset; k.sx = sx; k.gx = gx;
    k.Nt = (short)Nt; k.Dt = (short)Dt; k.Dx = Dx; k.Ntrace = Ntrace;
    Outseisfile1d(seis, k, outflag, sgyflag, endianflag, path);
}
// Returns the header keys read from the first trace: out_keys = {iTraceAll, iTrace, Offset,
// sx, gx, Nt, Dt, Ntrace}, out_dx = Dx.
void ref_Inseisfile1d(float *seis, int inflag, int sgyflag, char *path, int *out_keys, float *out_dx)
{
    sgyheadkey k;
    Inseisfile1d(seis, &k, inflag, sgyflag, path);
    out_keys[0] = k.iTraceAll; out_keys[1] = k.iTrace; out_keys[2] = k.Offset; out_keys[3] = k.sx;
    out_keys[4] = k.gx; out_keys[5] = k.Nt; out_keys[6] = k.Dt; out_keys[7] = k.Ntrace;
    *out_dx = k.Dx;
}
void ref_get_parameter(char *path, int sgyflag, int *ntrace, int *nsample, int *dt, int *endian)
{
    short ns = 0, d = 0;
    get_parameter(path, sgyflag, ntrace, &ns, &d, endian);
    *nsample = ns; *dt = d;
}
// scanshotgather (RTM_GPU_velstr.cpp:363-454) on ./seisReal/<name> under the working
// directory.  profile is [4][max_shots] (the rows of shotprofileId); the caller pre-fills it.
void ref_scanshotgather(char *name, int sgyflag, int *endianflag, int *profile, int max_shots)
{
    int *rows[4] = {profile, profile + max_shots, profile + 2 * max_shots, profile + 3 * max_shots};
    scanshotgather(name, rows, sgyflag, endianflag);
}
// Interpseis2d (Interp_function.cpp:245-264): seisobs [nt0][nx0] -> seiscal [nt][nx].  The
// output rows are zeroed first, so a branch that writes nothing leaves zeros.
void ref_Interpseis2d(float *seiscal, const float *seisobs, int nx, int nx0, int nt, int nt0, float dt, float dt0)
{
    float **out = Creat2dArray(nt, nx), **in = Creat2dArray(nt0, nx0);
    for (int i = 0; i < nt0; i++)
        for (int j = 0; j < nx0; j++) in[i][j] = seisobs[(size_t)i * nx0 + j];
    for (int i = 0; i < nt; i++)
        for (int j = 0; j < nx; j++) out[i][j] = 0.0f;
    Interpseis2d(out, in, nx, nx0, nt, nt0, dt, dt0);
    for (int i = 0; i < nt; i++)
        for (int j = 0; j < nx; j++) seiscal[(size_t)i * nx + j] = out[i][j];
    free2dArray(out, nt, nx);
    free2dArray(in, nt0, nx0);
}
// GeneralFKinterp (Interp_function.cpp:127-244): seisin [nt0][nx0] -> seisout [nt0][nx].
void ref_GeneralFKinterp(const float *seisin, float *seisout, int nx, int nx0, int nt0, int lx)
{
    float **out = Creat2dArray(nt0, nx), **in = Creat2dArray(nt0, nx0);
    for (int i = 0; i < nt0; i++)
        for (int j = 0; j < nx0; j++) in[i][j] = seisin[(size_t)i * nx0 + j];
    GeneralFKinterp(in, out, nx, nx0, nt0, lx);
    for (int i = 0; i < nt0; i++)
        for (int j = 0; j < nx; j++) seisout[(size_t)i * nx + j] = out[i][j];
    free2dArray(out, nt0, nx);
    free2dArray(in, nt0, nx0);
}
// Sincinterp (Interp_function.cpp:61-115): seisin [nt0][nx] -> seisout [nt][nx].
void ref_Sincinterp(const float *seisin, float *seisout, int nx, int nt, int nt0, float dt, float dt0)
{
    float **out = Creat2dArray(nt, nx), **in = Creat2dArray(nt0, nx);
    for (int i = 0; i < nt0; i++)
        for (int j = 0; j < nx; j++) in[i][j] = seisin[(size_t)i * nx + j];
    Sincinterp(in, out, nx, nt, nt0, dt, dt0);
    for (int i = 0; i < nt; i++)
        for (int j = 0; j < nx; j++) seisout[(size_t)i * nx + j] = out[i][j];
    free2dArray(out, nt, nx);
    free2dArray(in, nt0, nx);
}
}
