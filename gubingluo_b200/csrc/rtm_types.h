// rtm_types.h — data layout shared by the host engine and the sm_100a kernels.
//
// One shot = one padded grid of X = nxlen + 2*npml columns by Z = nz + 2*npml rows
// (gubingluo rtm_model.cu:149-150).  Every 2-D array of a shot is stored row-major with a
// row pitch of `pitch` floats (a multiple of 32, so each row starts on a 128-byte boundary):
//   p  [Z][pitch]      pressure                       (reference d_p,  Z*X)
//   vx [Z][pitch]      x particle velocity, X-1 used  (reference d_vx, Z*(X-1))
//   vz [Z][pitch]      z particle velocity, Z-1 rows  (reference d_vz, (Z-1)*X)
//   sx, sz [Z][pitch]  split pressure parts, touched only in the PML band
//                      (reference pl1/pr1/pt1/pb1 and pl2/pr2/pt2/pb2)
// Model arrays (same pitch): inv_rho = 1/rho, kappa = rho*v^2.
// Boundary strips per time step (reference save_d_* layout, kernel.cu:1186-1293):
//   [vx lr: 2][nzi][10] [vz tb: 2][10][nxi] [p lr: 2][nzi][10] [p tb: 2][10][nxi]
// with nzi = Z - 2*npml, nxi = X - 2*npml.
#pragma once
#include <stdint.h>

#define RTM_RADIUS 10
#define RTM_BX 128       // stencil tile width: columns (= threads) per block
// rows per unrolled group of the velocity kernels (forward and receiver passes; the
// reconstruction) and of the pressure kernels (forward; receiver pass; reconstruction)
#ifndef RTM_GROUP_VEL
#define RTM_GROUP_VEL 2
#endif
#ifndef RTM_GROUP_VEL_RECON
#define RTM_GROUP_VEL_RECON 4
#endif
#ifndef RTM_GROUP_PRES
#define RTM_GROUP_PRES 2
#endif
#ifndef RTM_GROUP_PRES_RECV
#define RTM_GROUP_PRES_RECV 2
#endif
#ifndef RTM_GROUP_PRES_RECON
#define RTM_GROUP_PRES_RECON 4
#endif
#define RTM_MAX2(a, b) ((a) > (b) ? (a) : (b))
#define RTM_STAGE_W (RTM_BX + 24)                             // staged width: columns x0-12 .. x0+BX+11
// staged rows beyond a tile's BZ (the z window) of the velocity kernels' p and the pressure
// kernels' vz
#define RTM_STAGE_ZEXTRA_VEL \
    (2 * RTM_RADIUS + (RTM_GROUP_VEL > RTM_GROUP_VEL_RECON ? RTM_GROUP_VEL : RTM_GROUP_VEL_RECON) - 2)
#define RTM_STAGE_ZEXTRA_PRES \
    (2 * RTM_RADIUS + RTM_MAX2(RTM_GROUP_PRES, RTM_MAX2(RTM_GROUP_PRES_RECV, RTM_GROUP_PRES_RECON)) - 2)

// What one launch of the stencil kernels updates.
enum RtmWaveMode {
    RTM_WAVE_FWD = 0,        // forward propagation, full grid (modelling and source pass;
                             // the source pass saves its strips with k_strip_save)
    RTM_WAVE_RECEIVER = 2,   // receiver back-propagation (+ injection; imaging in the p update)
    RTM_WAVE_RECON = 3       // source-wavefield reconstruction (interior + restored strips)
};

enum RtmPrecision { RTM_FP32 = 0, RTM_FP16 = 1, RTM_BF16 = 2 };

// Per-shot PML coefficient block, stored contiguously on the device.  The split-field
// update is f = (c1*f - D)/c2 with c1 = 1 - dt*d/2, c2 = 2 - c1 (reference kernel.cu:596-598);
// the kernels multiply by ic2 = 1/c2.  Outside the bands c1 = ic2 = 1.
//   c1x[X], ic2x[X]     pressure x part       c1vx[X], ic2vx[X]   vx
//   c1z[Z], ic2z[Z]     pressure z part       c1vz[Z], ic2vz[Z]   vz
// plus the raw profiles ddx[X], ddz[Z], ddxvx[X], ddzvz[Z] (reference kernel.cu:174-269).
struct PmlOffsets {
    int c1x, ic2x, c1vx, ic2vx, c1z, ic2z, c1vz, ic2vz, ddx, ddz, ddxvx, ddzvz, total;
};

__host__ __device__ inline PmlOffsets pml_offsets(int X, int Z)
{
    PmlOffsets o;
    o.c1x = 0; o.ic2x = X; o.c1vx = 2 * X; o.ic2vx = 3 * X;
    o.c1z = 4 * X; o.ic2z = 4 * X + Z; o.c1vz = 4 * X + 2 * Z; o.ic2vz = 4 * X + 3 * Z;
    o.ddx = 4 * X + 4 * Z; o.ddz = 5 * X + 4 * Z; o.ddxvx = 5 * X + 5 * Z; o.ddzvz = 6 * X + 5 * Z;
    o.total = 6 * X + 6 * Z;
    return o;
}

struct WaveDev {
    float *p, *vx, *vz, *sx, *sz;
};

struct ShotDev {
    int X, Z, npml, pitch;
    int nxi, nzi;
    int nsx, nsz;
    int sbx0, sbz0, sbnx, sbnz;   // source stamp box (padded coordinates) and its size
    int rz, rx0, nrec;
    int ntx;                      // tiles along x (RTM_BX columns each)
    int strip_len;                // 40*(nxi+nzi)
    const float *inv_rho_f, *kappa_f;   // forward (source-pass) model
    const float *inv_rho_b, *kappa_b;   // backward (reconstruction + receiver) model
    const float *pml;                   // PmlOffsets block
    const float *src;                   // dt*source over the stamp box [sbnz][sbnx]
    WaveDev a;                          // source / reconstructed-source wavefield
    WaveDev b;                          // receiver wavefield
    // whole-step kernel (rtm_step.cu): the second buffers of p, vx, vz that a step writes
    // (sx, sz as in a and b), and which buffer a and b are (0 or 1: the tensor maps of their p)
    WaveDev an, bn;
    int par_a, par_b;
    void *strips;                       // [nt][strip_len] of the strip precision
    float *strip_scale;                 // [nt][4]  (fp16/bf16 strips)
    float *strip_stage;                 // fp32 staging ring for fp16/bf16 strips [ring][strip_len]
    void *gather;                       // [nt][nrec] of the gather precision
    float *gather_scale;                // [nt]
    void *g1, *illum;                   // [Z][pitch] float or double accumulators (interior cells used)
    double *g1t, *illt;                 // RTM_ACC_FP64_BLOCKED: [Z][pitch] fp64 totals (g1, illum: fp32 partials)
    const void *tmaps;                  // RTM_TMAP_COUNT TMA tensor maps (128 B each) of this shot's slot
    // the other imaging conditions (when enabled): accumulators g2 (decomposition), g3
    // (Poynting angle), g3t (true amplitude), g4 (energy norm), [Z][pitch] float or double;
    // the source and receiver pressures before the current backward step; v^2 of the
    // backward model
    void *gx[4];
    float *ps_pre, *p_pre;
    const float *vp2_b;
};

// Imaging accumulator of RTM_ACC_KAHAN: compensated fp32 pair (8 bytes, as a double), the
// accumulated value being s - c.
struct KahanAcc {
    float s, c;
    __host__ __device__ KahanAcc() : s(0.f), c(0.f) {}
    __host__ __device__ KahanAcc(int) : s(0.f), c(0.f) {}
};
// Per-shot accumulation of g1 and illum (rtm_options.accum_fp64): fp32, fp64, compensated fp32,
// or fp64 totals of fp32 partial sums over RTM_ACC_BLOCK steps (the partials are imaged as the
// fp32 form does and added into the totals, then cleared, every RTM_ACC_BLOCK steps and after
// the last one).
enum RtmAccum { RTM_ACC_FP32 = 0, RTM_ACC_FP64 = 1, RTM_ACC_KAHAN = 2, RTM_ACC_FP64_BLOCKED = 3 };
#define RTM_ACC_BLOCK 32

// TMA tensor maps of one slot: the staged fields of the two wavefields with the box each
// stencil kernel loads (velocity: p rows z0-9 .. z0+BZ+12, columns x0-12 .. x0+139;
// pressure: vx rows z0 .. z0+BZ-1 with the same columns, vz rows z0-10 .. z0+BZ+11,
// columns x0 .. x0+127).
// (A_P_RECON: the source pressure again, in the boxes of the velocity reconstruction's own tile
// height; A_VX_RECON / A_VZ_RECON: the source velocities in the boxes of the pressure
// reconstruction's own tile height)
// (whole-step kernel, per wavefield (A, B) and buffer (0, 1): STEP_*: p in the box of rows
// z0-19 .. z0+TZ+18, columns x0-24 .. x0+151; STEPVX_*: vx, rows z0 .. z0+TZ-1, columns
// x0-12 .. x0+139; STEPVZ_*: vz, rows z0-10 .. z0+TZ+9, columns x0 .. x0+127)
enum RtmTmap { RTM_TMAP_A_P = 0, RTM_TMAP_A_VX, RTM_TMAP_A_VZ, RTM_TMAP_B_P, RTM_TMAP_B_VX, RTM_TMAP_B_VZ,
               RTM_TMAP_A_P_RECON, RTM_TMAP_STEP_A0, RTM_TMAP_STEP_A1, RTM_TMAP_STEP_B0, RTM_TMAP_STEP_B1,
               RTM_TMAP_STEPVX_A0, RTM_TMAP_STEPVX_A1, RTM_TMAP_STEPVX_B0, RTM_TMAP_STEPVX_B1,
               RTM_TMAP_STEPVZ_A0, RTM_TMAP_STEPVZ_A1, RTM_TMAP_STEPVZ_B0, RTM_TMAP_STEPVZ_B1,
               RTM_TMAP_A_VX_RECON, RTM_TMAP_A_VZ_RECON, RTM_TMAP_COUNT };
#define RTM_TMAP_BYTES 128

// One block's work: the tile of `shot` whose top-left cell is (x0, z0).  x0 is a multiple of
// 4, so the staged box (from x0-12) starts on a 16-byte boundary.
struct TileRef {
    int shot;
    int x0, z0;
    int interior;   // 1: the tile lies in the interior and holds no source, receiver or strip
                    // cell, so the kernels take their branch-free body (set by the host)
};

// Kernel-wide constants of one launch.
struct StepArgs {
    const ShotDev *shots;
    const TileRef *tiles;
    const float *wavelet;   // [nt]
    const float *coef;      // [10][10] zero-padded Liu-Yang table
    float c10[10];          // full-order (half-order 10) coefficients, read from the constant bank
    float dt, dtx, dtz;
    int it;                 // time index
    int strip_prec, gather_prec, accum_fp64;
    int ring;               // staging-ring slot for fp16/bf16 strips
    int *err;               // device error flag: set non-zero by a kernel whose bounded wait gave up
    // fixed-grid launches (CUDA-graph replays whose grid covers the largest tile list of the
    // session): counts[list] is the batch's own tile count, blocks past it return at once;
    // counts == nullptr: the grid is the tile count
    const int *counts;
    int list;
    int prefetch;           // 1: the stencil kernels prefetch their tile's operand rows into L2
};

// One persistent pass (rtm_stencil.cu, k_pass): every step of the source pass or of the
// backward pass in one launch.  Blocks take work items from a device queue in the order
//   source pass, per step it:    velocity tiles, pressure tiles, strip save (one per shot)
//   backward pass, per step k:   reconstruction velocity tiles, reconstruction pressure
//                                tiles, receiver velocity tiles, receiver pressure tiles
// and wait, per shot, until the items an item depends on (all of the shot's items of the
// phases before it) are done: done[phase][shot] counts them.
struct PassArgs {
    StepArgs a;              // shots, wavelet, coefficients, precisions (tiles, it, ring per item)
    const TileRef *list[4];  // tile lists: source pass {vel, pres}; backward {vel recon, pres recon, vel, pres}
    int len[4];              // their lengths
    const int *per_shot;     // tiles per shot of each list: [4][B]
    int B;                   // stride of per_shot and done
    int nshots, nsteps, nt;  // shots of the batch; steps of the pass; time samples
    int save, record, strip_prec;
    unsigned *queue;         // next item (starts at 0)
    unsigned *done;          // [4][B] completed items per phase and shot (start at 0)
    long long wait_ns;       // bound on one wait for other blocks' items (then the error flag, 2)
    unsigned *trace;         // [trace_len] the item each block took last (for error reports)
    int trace_len;
};
