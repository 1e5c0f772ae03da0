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
#define RTM_TX 32        // tile width  (columns) of the stencil kernels
#define RTM_TZ 32        // tile height (rows)

enum RtmPrecision { RTM_FP32 = 0, RTM_FP16 = 1, RTM_BF16 = 2 };

// Per-shot PML/edge coefficient block, stored contiguously on the device:
//   c1x[X], c2x[X]      pressure x-part damping  (1,1 outside the x band)
//   c1vx[X], c2vx[X]    vx damping               (1,1 outside the x band)
//   c1z[Z], c2z[Z]      pressure z-part damping
//   c1vz[Z], c2vz[Z]    vz damping
// plus the raw profiles ddx[X], ddz[Z], ddxvx[X], ddzvz[Z] (reference kernel.cu:174-269).
struct PmlOffsets {
    int c1x, c2x, c1vx, c2vx, c1z, c2z, c1vz, c2vz, ddx, ddz, ddxvx, ddzvz, total;
};

__host__ __device__ inline PmlOffsets pml_offsets(int X, int Z)
{
    PmlOffsets o;
    o.c1x = 0; o.c2x = X; o.c1vx = 2 * X; o.c2vx = 3 * X;
    o.c1z = 4 * X; o.c2z = 4 * X + Z; o.c1vz = 4 * X + 2 * Z; o.c2vz = 4 * X + 3 * Z;
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
    int ntx;                      // tiles along x
    int strip_len;                // 40*(nxi+nzi)
    const float *inv_rho_f, *kappa_f;   // forward (source-pass) model
    const float *inv_rho_b, *kappa_b;   // backward (reconstruction + receiver) model
    const float *pml;                   // PmlOffsets block
    const float *src;                   // dt*source over the stamp box [sbnz][sbnx]
    WaveDev a;                          // source / reconstructed-source wavefield
    WaveDev b;                          // receiver wavefield
    void *strips;                       // [nt][strip_len] of the strip precision
    float *strip_scale;                 // [nt][4]  (fp16/bf16 strips)
    float *strip_stage;                 // fp32 staging ring for fp16/bf16 strips [ring][strip_len]
    void *gather;                       // [nt][nrec] of the gather precision
    float *gather_scale;                // [nt]
    void *g1, *illum;                   // [nzi][nxi] float or double accumulators
};

struct TileRef {
    int shot;
    int tile;
};

// Kernel-wide constants of one launch.
struct StepArgs {
    const ShotDev *shots;
    const TileRef *tiles;
    const float *wavelet;   // [nt]
    const float *coef;      // [10][10] zero-padded Liu-Yang table
    float dt, dtx, dtz;
    int it;                 // time index
    int strip_prec, gather_prec, accum_fp64;
    int ring;               // staging-ring slot for fp16/bf16 strips
};
