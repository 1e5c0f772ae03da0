/*
 * rtm_oracle.h — CPU restatement of the reference's 2D acoustic prestack RTM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The CUDA product is tested against this oracle; the product in
 * gubingluo_b200/ never uses it: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load it.  The product never links or calls it.
 *
 * Every function restates a piece of the reference (gubingluo/gubingluo) and cites the
 * file:line it follows.  The FP32 build ("_f32") mirrors the reference's float
 * arithmetic, including the sub-expressions the reference evaluates in double because of
 * double literals (PML c1/c2, mute travel time, illumination-normalised division).  The
 * FP64 build ("_f64") runs the identical discrete scheme in double precision.
 *
 * Parity pins: host-side pieces are compared against the reference's own C++ sources
 * compiled here (oracle/ref/Makefile -> oracle/_ref/libref_host.so); the device-side
 * scheme is compared against golden fixtures produced by the reference's CUDA code
 * rebuilt for sm_100a (oracle/ref/ref_harness.cu, tests/golden/).
 *
 * Grid conventions (reference rtm_model.cu:149-150): X = nxlen + 2*npml, Z = nz + 2*npml,
 * all arrays row-major [iz][ix].  p: Z*X, vx: Z*(X-1), vz: (Z-1)*X.
 * General npml >= 10 is supported; at npml == 32 the result equals the reference's
 * (whose PML kernels launch exactly two 32-wide blocks per side, kernel.cu:542-1185).
 */
#ifndef RTM_ORACLE_H
#define RTM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NORDER 20  /* common.h:56  N */
#define ORC_RADIUS 10  /* N/2 */

/* One shot's padded grid and acquisition. */
typedef struct {
    int X, Z, npml, nt;
    float dx, dz, dt;
    int nsx, nsz;        /* source node in padded coordinates */
    float amp, alp, fdom;
    int rz;              /* receiver row in padded coordinates (reference: npml) */
    int rx0, nrec;       /* first receiver column (padded) and receiver count */
    float vpmax;         /* PML velocity: sqrt(max v^2) of the forward model */
} orc_shot;

/* Geometry of one shot for a given acquisition layout (rtm_model.cu:122-154, 626-650,
 * 1122-1158, 1629-1665). */
typedef struct {
    int nx1, nx2, nxlength, noffset;
    int nsx, nsz, nxpad, nzpad;
    int rx0, nrec;
    /* SU/SEG-Y header keys of the shot's first trace */
    int iTraceAll, iTrace, Offset, sx, gx;
    unsigned short Nt, Dt;
    float Dx;
    int Ntrace;
} orc_geom;

/* ---- constants and 1-D/2-D setup arrays (bit-exact targets) ---- */
void orc_coef_table(float *c100);                      /* FD_function.cpp:73-165 */
void orc_ricker_device(float *w, float fdom, float dt, int nt);   /* kernel.cu:13-22 */
void orc_ricker_host(float *w, float fdom, int nt, float dt);     /* FD_function.cpp:7-24 */
void orc_pml_profiles(float *ddx, float *ddz, float *ddxvx, float *ddzvz,
                      float vpmax, float dx, float dz, int npml, int X, int Z); /* kernel.cu:174-269 */
void orc_norder(int *norder, int *norderx, int *norderz, int X, int Z);     /* kernel.cu:271-317 */
void orc_source(float *src, int X, int Z, int nsx, int nsz, float amp, float alp,
                float dx2, float dz2);                                      /* kernel.cu:23-35 */
void orc_mute(float *gather, const float *vp2, int X, int nsx, int nsz, int nt,
              int rz, int rx0, int nrec, int nw, int tlength, float dx2, float dz2,
              float rdt);                                                   /* kernel.cu:96-173 */
void orc_taper(float *taper, int nxlen, int nwin, float alpha);             /* kernel.cu:1591-1604 */
int  orc_taper_nwin(int nxlength);                                          /* rtm_model.cu:464-465 */
int  orc_geometry(orc_geom *g, int layout, int ishot, int nx, int nz, int nt, float dx,
                  float dz, float dt, int npml, float spx0, float spz0, float dspx,
                  float offset, float offsetmax);

/* ---- host model preparation (Velocity_function.cpp) ---- */
void orc_extractvel1(float *out, const float *v, int nx, int nz, int nx1, int nx2, int square);
void orc_extendvel1(float *pad, const float *in, int nxlen, int nz, int npml);
void orc_pmlvelsmooth1d(float *vp, int nx, int nz, int npml);
void orc_velsmooth1d(float *vp, int n1, int n2, int nsp);
void orc_interpvel1(const float *vp0, float *vp, int nx0, int nz0, int nx, int nz, int lx, int lz);
void orc_laplacefd1d(int nx, int nz, int dx, int dz, float *image);        /* image_function.cpp:44-79 */
void orc_scaleimage1d(const float *illum, float *grad, int n);             /* image_function.cpp:11-20 */
void orc_get_constant(const float *vp, float fdom, float dx0, float dz0, int nx0, int nz0,
                      int nt0, float dt0, float *dx, float *dz, int *nx, int *nz, int *nt,
                      float *dt, int *lx, int *lz, float *vpmin, float *vpmax);

/* ---- per-shot RTM (the hot path) ----
 * mode 0: model the gather in vp2f/rhof (written, unmuted, to `gather`), then migrate it.
 * mode 1: `gather` (nt*nrec) is the recorded data, migrated as given.
 * mute != 0 applies the direct-wave mute of kernel.cu:96-121 to the migrated copy, with the
 * velocities of vp2f (mute 1, rtm_model.cu: before smoothing) or of vp2b (mute 2, the
 * real-data driver rtm_real.cu:397-403, which mutes after smoothing).
 * vp2b/rhob: model of the backward pass (differs from the forward one only when the
 * reference smooths after the source pass, rtm_model.cu:402-408).
 * g1/illum: nz*nxlen interior images (untapered).  ps_out/p_out (optional, Z*X): the
 * reconstructed source and receiver pressure after the last backward step. */
int orc_shot_f32(const orc_shot *s, const float *vp2f, const float *rhof,
                 const float *vp2b, const float *rhob, const float *coef,
                 const float *wavelet, int mode, float *gather, int mute, int nw,
                 int tlength, float *g1, float *illum, float *ps_out, float *p_out);
int orc_shot_f64(const orc_shot *s, const float *vp2f, const float *rhof,
                 const float *vp2b, const float *rhob, const float *coef,
                 const float *wavelet, int mode, float *gather, int mute, int nw,
                 int tlength, double *g1, double *illum, double *ps_out, double *p_out);

/* orc_shot with the extra imaging conditions of the reference's backward loop
 * (rtm_model.cu:450-455, kernel.cu:1417-1522) accumulated into g2 (wavefield decomposition),
 * g3 (Poynting angle weighting, all angle bins summed), g3t (its true-amplitude variant) and
 * g4 (energy norm), nz*nxlen each, when extra != 0.  extra == 2 reproduces the reference's
 * indexing (vx read at the pressure cell's flat index on the (X-1)-wide vx arrays; receiver
 * vz in the source term of the Poynting vector); extra == 1 reads both at their own cells. */
int orc_shot_ex_f32(const orc_shot *s, const float *vp2f, const float *rhof,
                    const float *vp2b, const float *rhob, const float *coef,
                    const float *wavelet, int mode, float *gather, int mute, int nw,
                    int tlength, float *g1, float *illum, float *ps_out, float *p_out,
                    int extra, float *g2, float *g3, float *g3t, float *g4);
int orc_shot_ex_f64(const orc_shot *s, const float *vp2f, const float *rhof,
                    const float *vp2b, const float *rhob, const float *coef,
                    const float *wavelet, int mode, float *gather, int mute, int nw,
                    int tlength, double *g1, double *illum, double *ps_out, double *p_out,
                    int extra, double *g2, double *g3, double *g3t, double *g4);

/* Forward modelling only, nsteps steps from rest (source added, no strips).
 * Returns the final p (Z*X), vx (Z*(X-1)), vz ((Z-1)*X) and the gather (nsteps*nrec). */
int orc_forward_f32(const orc_shot *s, const float *vp2, const float *rho, const float *coef,
                    const float *wavelet, int nsteps, float *p, float *vx, float *vz,
                    float *gather);
int orc_forward_f64(const orc_shot *s, const float *vp2, const float *rho, const float *coef,
                    const float *wavelet, int nsteps, double *p, double *vx, double *vz,
                    double *gather);

/* Per-shot image finalisation (rtm_model.cu:462-488; kernel.cu:1556-1615):
 * taper g1 and illum, then image2s += g1/(illum+1e-6) (evaluated in double as in the
 * reference), image1 += g1, illum_total += illum, all at column offset nx1. */
void orc_finalize_f32(float *g1, float *illum, int nxlen, int nz, int nx, int nx1,
                      float *image1, float *image2s, float *illum_total);
void orc_finalize_f64(double *g1, double *illum, int nxlen, int nz, int nx, int nx1,
                      double *image1, double *image2s, double *illum_total);

/* The extra images of one shot (rtm_model.cu:466-487; kernel.cu:1556-1604): taper g2, g3, g4
 * and g3t like g1, then image3s/4s/5s += g2/g3/g4 / (illum + 1e-6) with the shot's tapered
 * illumination (call after orc_finalize, which tapers illum in place), image3m/4m/5m +=
 * g2/g3/g4 and imagetrue += g3t, at column offset nx1. */
void orc_finalize_extra_f32(float *g2, float *g3, float *g4, float *g3t, const float *illum, int nxlen, int nz,
                            int nx, int nx1, float *image3s, float *image4s, float *image5s, float *image3m,
                            float *image4m, float *image5m, float *imagetrue);
void orc_finalize_extra_f64(double *g2, double *g3, double *g4, double *g3t, const double *illum, int nxlen,
                            int nz, int nx, int nx1, double *image3s, double *image4s, double *image5s,
                            double *image3m, double *image4m, double *image5m, double *imagetrue);

/* Threads used by the OpenMP loops (1 when built without OpenMP). */
int orc_num_threads(void);

/* Seismic interpolation of the real-data path (orc_interp.c; Interp_function.cpp). */
void orc_kaiser(float *w, int n, double beta);
void orc_sinc_interp(const float *seisin, int ld_in, float *seisout, int nx, int nt, int nt0, float dt,
                     float dt0);
int orc_fk_interp(const float *seisin, float *seisout, int nx, int nx0, int nt0, int lx, int mirror);
int orc_interp_gather(const float *seisobs, int nx0, int nt0, float *seiscal, int nx, int nt, float dt,
                      float dt0, int mirror);

#ifdef __cplusplus
}
#endif
#endif
