/*
 * rtm_b200.h — C-ABI of librtm_b200.so, the B200 (sm_100a) implementation of the
 * gubingluo 2D acoustic prestack reverse-time-migration hot path.
 *
 * Plain C types only (ints, floats, pointers, sizes).  All arrays are host memory unless a
 * comment says otherwise; models and images are row-major [iz][ix] (x fastest), gathers
 * are [it][itrace] (trace fastest), exactly as in the reference.
 *
 * Reference interfaces replaced (gubingluo/gubingluo):
 *   rtm_model          <- extern "C" rtm_model   RTM_GPU_velstr.cpp:23-28, rtm_model.cu:12-17
 *   rtm_real           <- extern "C" rtm_real    rtm_real.cu:17-22 (the definition's argument list)
 *   rtm_migrate / rtm_batch / rtm_session_*  new: status-returning, file-free form of the same path
 *   rtm_scan_shotgather<- scanshotgather         RTM_GPU_velstr.cpp:363-454
 *   rtm_real_geometry  <- per-shot geometry      rtm_real.cu:134-157
 *   rtm_read_shot_traces <- trace reading        rtm_real.cu:379-394
 *   rtm_interp_gather  <- Interpseis2d           Interp_function.cpp:245-264
 *   rtm_read_params    <- parameter-file reader  RTM_GPU_velstr.cpp:60-120
 *   rtm_get_constant   <- get_constant           RTM_GPU_velstr.cpp:319-362
 *   rtm_shot_geometry  <- per-layout shot window rtm_model.cu:122-154, 626-650, 1122-1158, 1629-1665
 *   rtm_prepare_model  <- extractvel1/extractrho1/extendvel1/pmlvelsmooth1d/velsmooth1d
 *                         Velocity_function.cpp:2011-2073, :9-103, :199-313
 *   rtm_interp_model   <- interpvel1             Velocity_function.cpp:1946-1975
 *   rtm_laplace_image  <- laplacefd1d            image_function.cpp:44-79
 *   rtm_scale_image    <- scaleimage1d           image_function.cpp:11-20
 *   rtm_coef_table     <- Diff_coeffVelStrLiuyang FD_function.cpp:73-165 (+ table RTM_GPU_velstr.cpp:184-196)
 *   rtm_read_velocity  <- ReadVelMod             IO_function.cpp:9-35
 *   rtm_write_image_su <- Output1d               IO_function.cpp:366-422
 *   rtm_write_gather_su<- Outseisfile1d          IO_function.cpp:131-183 (+ sgyhead_function.cpp:351-383)
 *   rtm_read_gather_su <- Inseisfile1d/get_parameter IO_function.cpp:284-324, :226-283
 */
#ifndef RTM_B200_H
#define RTM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define RTM_OK 0
#define RTM_ERR_ARG -1      /* invalid argument or size */
#define RTM_ERR_CUDA -2     /* CUDA runtime error (device, launch, memory) */
#define RTM_ERR_IO -3       /* file missing, unreadable or malformed */
#define RTM_ERR_NOMEM -4    /* host or device allocation failed */
#define RTM_ERR_NUMERIC -5  /* a shot's image went NaN or infinite (the wavefield diverged) */

/* ---- storage precisions ---- */
#define RTM_PREC_FP32 0
#define RTM_PREC_FP16 1
#define RTM_PREC_BF16 2

/* One survey: model grid, time axis, source, acquisition layout and migration mode.
 * Field meanings follow the reference parameter file (RTM_GPU_velstr.cpp:76-120). */
typedef struct rtm_survey {
    int nx, nz, nt;          /* model size (after regridding) and time samples */
    float dx, dz, dt;
    int npml;                /* PML width in cells (any value >= 10) */
    float fdom, amp, alp;    /* Ricker peak frequency, source amplitude, Gaussian width */
    int layout;              /* 1 bilateral, 2 full array, 3 unilateral right, 4 unilateral left */
    float spx0, spz0, dspx;  /* first source position, source depth, source interval (m) */
    float offset, offsetmax; /* minimum offset (layouts 3/4) and aperture (layouts 1/3/4) */
    int mode;                /* 0: model each shot's gather first, 1: migrate given gathers */
    int medium_flag;         /* smooth the PML zone of the models (pmlvelsmooth1d) */
    int ismth;               /* >0: smooth v^2 and rho by a Gaussian of half-width ismth after the
                                source pass, as the reference does (rtm_model.cu:402-408) */
    float direct, direct0;   /* direct-wave mute: nw = direct/(fdom*dt), tlength = direct0/dt */
    int mute;                /* direct-wave mute: 0 none, 1 with the modelling model's velocities
                                (rtm_model.cu mutes before smoothing), 2 with the migration
                                model's (rtm_real.cu:397-403 mutes after smoothing) */
    int receiver_depth;      /* receiver row below z = 0 in cells (reference: 0) */
} rtm_survey;

typedef struct rtm_options {
    int device;              /* CUDA device ordinal */
    int strip_precision;     /* RTM_PREC_*: storage of the saved boundary strips */
    int gather_precision;    /* RTM_PREC_*: storage of the receiver gathers */
    int accum_fp64;          /* per-shot image/illumination accumulation: 0 fp32; 1 fp64; 2
                                compensated fp32 pairs (Kahan, 8 bytes like fp64); 3 fp64
                                totals of fp32 partial sums over 32 steps (the steps image into
                                fp32 partials, which a flush adds into the fp64 totals every 32
                                steps and after the last); with 1, 2 or 3 the stacked images and
                                the division are fp64 */
    int batch;               /* shots per launch; 0 = as many as fit in device memory */
    int use_graph;           /* 1: each pass's time loop (source pass; backward pass) runs as one
                                CUDA graph, captured the first time a launch shape (shots per
                                batch, tile counts) occurs and replayed for later batches of that
                                shape; 2: the same with grids rounded up to four significant bits
                                (blocks past the batch's tiles return), so batches of nearby
                                shapes share a graph.  Results are bit-identical to direct
                                launches.  Not used with tsnap snapshots, and per-kernel timing is
                                not sampled. */
    int verbose;             /* print per-batch progress like the reference */
    int extra_images;        /* the reference's other imaging conditions (kernel.cu:1417-1555):
                                0 off; 1 wavefield decomposition, Poynting-angle and energy-norm
                                images with vx and vz read at their own cells; 2 the same with the
                                reference's indexing (vx at the pressure cell's flat index on its
                                (X-1)-wide arrays, receiver vz in the source Poynting term), for
                                parity with its image3/4/5 outputs */
    float tsnap;             /* with verbose: print max |p| of every shot every tsnap seconds, as
                                the reference does (rtm_model.cu:271-273, 324-326, 415-417),
                                from an on-device reduction; 0 = none */
} rtm_options;

/* Geometry of one shot for the survey's layout (padded coordinates include the PML). */
typedef struct rtm_geometry {
    int nx1, nx2, nxlength, noffset;   /* model window [nx1, nx2] */
    int nsx, nsz, nxpad, nzpad;        /* source node, padded grid */
    int rz, rx0, nrec;                 /* receiver row, first receiver column, traces */
    int iTraceAll, iTrace, Offset, sx, gx, Nt, Dt, Ntrace;  /* SU header keys of trace 1 */
    float Dx;
} rtm_geometry;

typedef struct rtm_stats {
    double seconds_total;    /* wall time of rtm_session_run / rtm_migrate's migration */
    double gcell_updates;    /* cell-updates performed: nt*(2*X*Z + nxlen*nz) per shot */
    int shots;
    int batches;
    int kernel_launches;     /* launches of this library's kernels */
} rtm_stats;

/* ---- drop-in entry point (same symbol, signature and file side effects as the reference) ----
 * Writes ./seisReal/{ishot}seisreal.su in mode 0, reads it in mode 1, writes
 * the ./output/ temp images after shots with (ishot-1)%50 == 0 and ./output/{idevice}Imagetrue.su,
 * and overwrites the ten image arrays (nx*nz each).  image3*, image4*, image5* and Imagetrue
 * come from the reference's other imaging conditions (see rtm_options.extra_images): the
 * environment variable RTM_B200_EXTRA_IMAGES selects 1 (the default: vx and vz read at their
 * own cells), 2 (the reference's indexing) or 0 (left zero).  Errors are printed and
 * recorded in rtm_last_error(). */
void rtm_model(int idevice, int nshot, int startshot, int dshot, int mode, int medium_flag,
               int flag_layout, int sgyflag, int endianflag, int ismth, int nx, int nz, int nt,
               float dx, float dz, float dt, int npml, float direct, float direct0, float tsnap,
               float fdom, float spx0, float spz0, float dspx, float offset, float offsetmax,
               float amp, float alp, float *vp0, float *rho0, float *diffcoef, float *wavelet,
               float *image1, float *image2s, float *image3s, float *image4s, float *image5s,
               float *image2m, float *image3m, float *image4m, float *image5m, float *illum);

/* Drop-in for the reference's real-data driver (definition rtm_real.cu:17-22; the caller's
 * prototype RTM_GPU_velstr.cpp:30-35 declares `int nw, int tlength` where the definition has
 * `float direct, float direct0`: this symbol takes the definition's list).  For shots
 * startshot, startshot+dshot, ... <= nshot: geometry from shotprofileId[0..3][ishot-1] (sx,
 * trace count, first trace, offset; rtm_scan_shotgather), traces read from
 * ./seisReal/<filename_shotgather> (nt0 samples at dt0, receivers every dx0), resampled to
 * dx and dt (F-K in x, windowed sinc in t: rtm_interp_gather), muted in the migration model
 * and migrated on the device in batches.  vp0/rho0: the nz*nx model on the dx grid.  nx0,
 * nz0, dz0, lx, lz, tsnap, flag_layout and wavelet are accepted and not used, as in the
 * reference.  Writes the ./output/ temp images after shots with (ishot-1)%50 == 0 and
 * ./output/{idevice}Imagetrue.su, and overwrites the ten image arrays.  Environment: as for
 * rtm_model, plus RTM_B200_FK_MIRROR = 0 (default: the reference's negative-frequency
 * indexing in the F-K step) or 1 (the Hermitian partner).  Errors are printed and recorded
 * in rtm_last_error(). */
void rtm_real(int idevice, int nshot, int startshot, int dshot, int medium_flag, int flag_layout,
              int sgyflag, int endianflag, int ismth, int nx, int nz, int nt, float dx, float dz,
              float dt, int nx0, int nz0, int nt0, float dx0, float dz0, float dt0, int npml, int lx,
              int lz, float tsnap, float fdom, float spz0, float amp, float alp, float direct,
              float direct0, float *vp0, float *rho0, float *diffcoef, float *wavelet,
              char filename_shotgather[40], int **shotprofileId, float *image1, float *image2s,
              float *image3s, float *image4s, float *image5s, float *image2m, float *image3m,
              float *image4m, float *image5m, float *illum);

/* Last error message of this thread ("" when none). */
const char *rtm_last_error(void);

/* Library version string. */
const char *rtm_version(void);

/* ---- sessions: device-resident migration of a shot list ----
 * shots: shot numbers (1-based ishot of the reference).  vp/rho: nz*nx velocity (m/s) and
 * density (kg/m^3); vp_mig/rho_mig: model of the backward pass, NULL for the same model.
 * diffcoef: 10x10 coefficient table (rtm_coef_table), NULL for the built-in one. */
typedef struct rtm_session rtm_session;

int rtm_session_open(rtm_session **out, const rtm_survey *s, const rtm_options *o, const int *shots,
                     int nshots, const float *vp, const float *rho, const float *vp_mig,
                     const float *rho_mig, const float *diffcoef);
/* As rtm_session_open, with every shot's geometry given (geoms[k] for shot shots[k], e.g. from
 * rtm_real_geometry) instead of computed from the survey's layout; layout, spx0, dspx, offset
 * and offsetmax of the survey are then unused. */
int rtm_session_open_geometry(rtm_session **out, const rtm_survey *s, const rtm_options *o,
                              const int *shots, const rtm_geometry *geoms, int nshots,
                              const float *vp, const float *rho, const float *vp_mig,
                              const float *rho_mig, const float *diffcoef);
/* Mode 1: upload shot k's gather gathers[k] ([nt][nrec_k]), mute and pack it on the device. */
int rtm_session_set_gather(rtm_session *ss, int k, const float *gather);
/* Mode 1, recorded data: upload shot k's traces seisobs [nt0][nx0] (dt0, data spacing),
 * resample them on the device to [nt][nrec_k] (rtm_interp_gather; mirror as there), then
 * mute and pack as rtm_session_set_gather does. */
int rtm_session_set_gather_raw(rtm_session *ss, int k, const float *seisobs, int nx0, int nt0,
                               float dt0, int mirror);
/* Migrate every shot of the session; images accumulate on the device.  Inputs must be
 * resident (rtm_session_set_gather for mode 1). */
int rtm_session_run(rtm_session *ss, rtm_stats *stats);
/* Migrate shots [k0, k0+n) only; images accumulate.  A run (this or rtm_session_run) goes
 * in ceil(n / batch size) launches of equal size, to within one shot. */
int rtm_session_run_range(rtm_session *ss, int k0, int n, rtm_stats *stats);
/* Mode 0 only: model every shot's gather (forward pass with receiver sampling; no
 * migration), the reference's modelling pass (rtm_model.cu:266-290). */
int rtm_session_model(rtm_session *ss);
/* Device pointers of the stacked images (nz*nx, float or double per accum_fp64), for
 * reductions across GPUs; valid until rtm_session_close. */
int rtm_session_image_ptrs(rtm_session *ss, void **image1, void **image2s, void **image2m, void **illum);
/* Copy shot k's gather to the host, [nt][nrec_k]: mode 0, the modelled (unmuted) gather;
 * mode 1, the fp32 gather being migrated, after the direct-wave mute (cuda_mute1,
 * kernel.cu:96-121) when the survey's mute is on. */
int rtm_session_get_gather(rtm_session *ss, int k, float *gather);
/* Copy shot k's device PML damping profiles (cuda_pmlCoeffpx/pz/vx/vz, kernel.cu:174-269,
 * for the vpmax of the shot's model window): ddx [nxpad], ddz [nzpad], ddxvx [nxpad-1],
 * ddzvz [nzpad-1]; any pointer may be NULL.  For parity tests. */
int rtm_session_get_pml(rtm_session *ss, int k, float *ddx, float *ddz, float *ddxvx, float *ddzvz);
/* Copy the stacked images (nz*nx each; any pointer may be NULL). */
int rtm_session_get_images(rtm_session *ss, float *image1, float *image2s, float *image2m,
                           float *illum);
int rtm_session_get_images_f64(rtm_session *ss, double *image1, double *image2s, double *illum);
/* With options.extra_images != 0: the other imaging conditions' stacked images (nz*nx each,
 * any pointer may be NULL), replacing the reference's image3/4/5 and Imagetrue
 * (rtm_model.cu:466-487): wavefield decomposition (image3s, normalised by each shot's
 * illumination; image3m), Poynting-angle weighting (image4s, image4m), energy norm (image5s,
 * image5m) and the Poynting true-amplitude image (imagetrue). */
int rtm_session_get_images_extra(rtm_session *ss, float *image3s, float *image4s, float *image5s,
                                 float *image3m, float *image4m, float *image5m, float *imagetrue);
/* Zero the stacked images. */
int rtm_session_reset_images(rtm_session *ss);
/* Checkpoints (no counterpart in the reference, which only dumps partial images every 50
 * shots, rtm_model.cu:490-538, and resumes by hand from a new startshot without them).  Save
 * writes the stacked images as accumulated (fp32 or fp64; 4 images, 11 with extra_images)
 * with the count of shots already stacked, atomically (<path>.tmp renamed over <path>).
 * Load restores them into a session of the same configuration (hash of the survey, the
 * image options, the shots and their geometry, the models and the coefficients; refused
 * otherwise) and returns the count; running the remaining shots then gives the images of an
 * uninterrupted run bit for bit (shots are stacked in shot order whatever the batching). */
int rtm_session_save_checkpoint(rtm_session *ss, const char *path, int shots_done);
int rtm_session_load_checkpoint(rtm_session *ss, const char *path, int *shots_done);
/* Header of a checkpoint file (no device work); any output may be NULL. */
int rtm_checkpoint_info(const char *path, int *nx, int *nz, int *nshots, int *shots_done,
                        int *elem_bytes, unsigned long long *config_hash);
unsigned long long rtm_session_config_hash(rtm_session *ss);
/* Checking mode (no counterpart in the reference): with RTM_B200_GUARDS=1 in the environment
 * when a session opens, every device sub-allocation is followed by a guard band of a known
 * byte pattern, verified after setup, after every batch and after every resampling; a write
 * past the end of a buffer fails the call with RTM_ERR_CUDA naming the buffer.  Returns the
 * number of guard bands of the session (0 when the mode is off). */
int rtm_session_guard_count(rtm_session *ss);
/* Rows per stencil tile in use: forward and receiver velocity, reconstruction velocity,
 * forward and receiver pressure, reconstruction pressure (with the whole-step kernel, its tile
 * height in all four).  Chosen, with the kernel form of each family, per launch shape by timing
 * 8-, 16- and 32-row tiles in both forms before the first batch of that shape
 * (RTM_B200_TUNE=0, or RTM_B200_BZ_VEL / _VEL_RECON / _PRES / _PRES_RECON set, turns that off;
 * RTM_B200_BZ_PRES sets both pressure heights unless _PRES_RECON is given;
 * RTM_B200_KERNELS=scalar|vector fixes the form; choices persist across processes in
 * RTM_B200_TUNE_CACHE=<file>).  Any pointer may be NULL. */
int rtm_session_tile_heights(rtm_session *ss, int *bz_vel, int *bz_vel_recon, int *bz_pres, int *bz_pres_recon);
/* Run the tuner now for every launch shape of rtm_session_run_range(ss, k0, n) (no
 * migration), so that the timed run does not include its trial steps. */
int rtm_session_prepare(rtm_session *ss, int k0, int n);
/* Shots per launch (batch slots) of the session: options.batch, or as many as device memory
 * holds. */
int rtm_session_batch_size(rtm_session *ss);
/* Number of traces of shot k. */
int rtm_session_nrec(rtm_session *ss, int k);
/* cudaStream_t of the session (as void*), for event timing by the caller. */
void *rtm_session_stream(rtm_session *ss);
/* Per-launch device time of the named kernel family over the last run, measured with
 * events on the session stream for a sample of the steps: "vel_bwd", "pres_bwd",
 * "vel_fwd", "pres_fwd".  Returns the mean milliseconds per launch (-1 if not sampled). */
double rtm_session_kernel_ms(rtm_session *ss, const char *kernel, int *launches);
/* Final reconstructed source pressure and receiver pressure of the last shot run in slot k
 * of the last batch ([nzpad][nxpad]); for parity tests. */
int rtm_session_get_wavefields(rtm_session *ss, int slot, float *ps, float *pr);
void rtm_session_close(rtm_session *ss);

/* One call: open, upload (mode 1), run, fetch images, close. gathers_in (mode 1) and
 * gathers_out (mode 0) are arrays of nshots host pointers (NULL entries skipped). */
int rtm_migrate(const rtm_survey *s, const rtm_options *o, const int *shots, int nshots,
                const float *vp, const float *rho, const float *vp_mig, const float *rho_mig,
                const float *const *gathers_in, float *const *gathers_out, float *image1,
                float *image2s, float *image2m, float *illum, rtm_stats *stats);

/* The batched form as one descriptor (the same call as rtm_migrate): every shot of `shots`
 * migrated on one device in batches of options.batch (0: as many as fit), images stacked in
 * shot order and written to the four outputs (nz*nx each, overwritten; any may be NULL). */
typedef struct rtm_batch_desc {
    rtm_survey survey;
    rtm_options options;
    const int *shots;                 /* 1-based shot numbers */
    int nshots;
    const float *vp, *rho;            /* nz*nx modelling (mode 0) / migration model */
    const float *vp_mig, *rho_mig;    /* nz*nx backward-pass model, NULL for vp/rho */
    const float *const *gathers_in;   /* mode 1: nshots pointers to [nt][nrec_k] gathers */
    float *const *gathers_out;        /* mode 0: nshots pointers (NULL entries skipped), or NULL */
    float *image1, *image2s, *image2m, *illum;
} rtm_batch_desc;
int rtm_batch(const rtm_batch_desc *d, rtm_stats *stats);

/* Forward modelling only: nsteps source-pass steps of shot `ishot` from rest, in the model
 * vp/rho (nz*nx, as for sessions).  Outputs (any may be NULL): p [nzpad][nxpad],
 * vx [nzpad][nxpad-1], vz [nzpad-1][nxpad], gather [nsteps][nrec]. */
int rtm_forward(const rtm_survey *s, const rtm_options *o, int ishot, const float *vp, const float *rho,
                int nsteps, float *p, float *vx, float *vz, float *gather);

/* ---- host-side pieces of the path ---- */
int rtm_shot_geometry(const rtm_survey *s, int ishot, rtm_geometry *g);
void rtm_coef_table(float *c100);
/* Window [nx1, nx2] of the nz*nx models, square the velocity, pad by npml (edge
 * replication), optionally smooth the PML zone: out [nz+2npml][nxlen+2npml]. */
int rtm_prepare_model(const float *vp, const float *rho, int nx, int nz, int nx1, int nx2,
                      int npml, int medium_flag, float *vp2_pad, float *rho_pad);
int rtm_velsmooth(float *a, int n1, int n2, int nsp);
int rtm_pmlsmooth(float *a, int nxpad, int nzpad, int npml);
int rtm_interp_model(const float *vp0, float *vp, int nx0, int nz0, int nx, int nz, int lx, int lz);
void rtm_get_constant(const float *vp, float fdom, float dx0, float dz0, int nx0, int nz0, int nt0,
                      float dt0, float *dx, float *dz, int *nx, int *nz, int *nt, float *dt,
                      int *lx, int *lz, float *vpmin, float *vpmax);
void rtm_laplace_image(float *image, int nx, int nz, int dx, int dz);
/* GPU form of rtm_laplace_image that makes no device allocation.  No counterpart in the
 * reference, whose laplacefd1d (image_function.cpp:44-79) runs on the host only.  The image
 * passes through a fixed 48 MiB scratch area per device that is part of the library (input
 * copy + result, at most 6 Mi cells = 6291456 = nx*nz); larger images return RTM_ERR_ARG.
 * Runs on the calling thread's per-thread default stream of the current device and returns
 * when it has finished.  Calls on one device must not overlap (they share the scratch).  The
 * first call in each device context (again after cudaDeviceReset) looks up the scratch
 * address with that device current; make that first call before any stream capture begins.
 * Returns RTM_OK or an RTM_ERR_* code (message in rtm_last_error()). */
int rtm_laplace_image_noalloc(float *image, int nx, int nz, int dx, int dz);
void rtm_scale_image(const float *illum, float *image, int n);

/* ---- real-data path ---- */
/* scanshotgather (RTM_GPU_velstr.cpp:363-454) on a multi-shot SU (sgyflag 0) or SEG-Y (1)
 * file: byte order from the first header's ns/dt (*endianflag 1 = big-endian), then one row
 * per shot, a shot starting wherever sx changes: profile is [4][max_shots] with rows sx,
 * trace count, first trace number (from 1) and offset of the first trace (the rows of the
 * reference's shotprofileId).  Returns the number of shots (>= 0) or an RTM_ERR_* code. */
int rtm_scan_shotgather(const char *path, int sgyflag, int *endianflag, int *profile, int max_shots);
/* Geometry of one recorded shot (rtm_real.cu:134-157): receivers from `offset` to the right
 * of the source every dx0.  *ncols0 = traces on the data grid (the width nx0 that
 * rtm_interp_gather and rtm_session_set_gather_raw take).  Uses nx, nz, dx, dz, npml, spz0,
 * nt, dt and receiver_depth of s. */
int rtm_real_geometry(const rtm_survey *s, int sx, int offset, int ntrace, float dx0,
                      rtm_geometry *g, int *ncols0);
/* ntrace traces of nt0 samples from trace number itrace_all on (rtm_real.cu:379-394) into
 * seisobs [nt0][ncols]; columns from ntrace on are zero. */
int rtm_read_shot_traces(const char *path, int sgyflag, int endianflag, int nt0,
                         long long itrace_all, int ntrace, int ncols, float *seisobs);
/* Interpseis2d (Interp_function.cpp:245-264) on the GPU: seisobs [nt0][nx0] -> seiscal
 * [nt][nx].  nx > nx0: F-K interpolation by lx = (nx-1)/(nx0-1) (nx <= lx*nx0 required);
 * nt > nt0: 21-tap Kaiser-windowed sinc; neither: the first nt samples of the first nx
 * traces.  mirror 0 builds the negative frequencies of the F-K step with the reference's
 * indexing (one row off the Hermitian partner; for odd nt0 the first such row reads as zero
 * where the reference reads past its array), 1 from the Hermitian partner.  Host buffers;
 * synchronous on device `device`. */
int rtm_interp_gather(const float *seisobs, int nx0, int nt0, float *seiscal, int nx, int nt,
                      float dt, float dt0, int mirror, int device);

/* ---- files ---- */
typedef struct rtm_params {
    float dt0; int nt0; float tsnap;
    float xmax, zmax, dx0, dz0;
    float fdom, amp, alp;
    float spx0, spz0, dspx;
    float offset, offsetmax;
    int startshot, nshot, dshot, nshotall;
    int npml;
    int medium_flag, ismth;
    float direct, direct0;
    int idevice, flag_layout, mode, dataflag, sgyflag, endianflag, rhoflag;
    char vp_file[256], shotgather_file[256], rho_file[256];
} rtm_params;

/* Read "<dir>/cmd.in" (its 2nd line names the parameter file, read from <dir>). */
int rtm_read_params(const char *input_dir, rtm_params *p);
/* nx traces of 240-byte header + nz native floats -> vp [nz][nx]. */
int rtm_read_velocity(const char *path, int nx, int nz, float *vp);
int rtm_write_image_su(const char *path, const float *image, int nz, int nx, float d);
int rtm_write_gather_su(const char *path, const float *gather, const rtm_geometry *g, int nt,
                        int sgyflag, int endianflag);
/* Reads ntr traces of nt samples into gather [nt][ntr]; returns RTM_OK and the counts.
 * gather may be NULL to query the sizes only. */
int rtm_read_gather_su(const char *path, int sgyflag, float *gather, int *nt, int *ntr,
                       rtm_geometry *keys);

#ifdef __cplusplus
}
#endif
#endif
