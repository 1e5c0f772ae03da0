// rtm_launch.h — host launchers of the kernels in rtm_kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include "rtm_types.h"

// mode: RtmWaveMode; bz: rows per tile (8, 16, 32 or 64); ntiles: length of the (shot, tile)
// list built for that bz.
void launch_vel(int mode, int bz, const StepArgs &a, int ntiles, cudaStream_t s);
void launch_pres(int mode, int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s);
// The same launches with four columns by U rows per thread (rtm_stencil_v.cu): same tile
// lists, staged boxes and results, 32 * bz / U threads per block.
void launch_vel4(int mode, int bz, const StepArgs &a, int ntiles, cudaStream_t s);
// A whole pass in one persistent launch (rtm_stencil.cu, k_pass): dir 0 the source pass, 1 the
// backward pass.  Only at the default tile heights (32, 16, 16); returns false otherwise.
bool launch_pass(int dir, const PassArgs &p, int bz_vel, int bz_vel_recon, int bz_pres, cudaStream_t s);
void launch_pres4(int mode, int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s);
// One whole time step (velocities and pressure) of one wavefield (rtm_step.cu): reads the
// shots' a / b fields, writes an / bn; tz rows per tile (16 or 32), 256 threads per block;
// `fast`: the tile list holds only interior tiles (the branch-free instance).
void launch_step(int mode, int tz, bool fast, const StepArgs &a, int ntiles, int record, cudaStream_t s);
size_t step_smem_bytes(int tz);
void launch_setup_pml(float *pml, int X, int Z, int npml, float dx, float dz, float dt, float vpmax, cudaStream_t s);
void launch_setup_source(float *src, int sbx0, int sbz0, int sbnx, int sbnz, int nsx, int nsz, float amp, float alp,
                         float dx2, float dz2, float dt, cudaStream_t s);
void launch_ricker(float *w, float fdom, float dt, int nt, cudaStream_t s);
void launch_mute(float *g, const float *vrow, int X, int nsx, int nsz, int nt, int rz, int rx0, int nrec, int nw,
                 int tlength, float dx2, float dz2, float rdt, cudaStream_t s);
void launch_strip_save(const ShotDev *shots, int nshots, int max_strip_len, int it, int ring, int prec,
                       cudaStream_t s);
void launch_strip_pack(const ShotDev *shots, int nshots, int it0, int ring0, int nsteps, int prec, cudaStream_t s);
void launch_gather_pack(const float *g, void *out, float *scale, int nt, int nrec, int prec, cudaStream_t s);
void launch_finalize(const void *fs, int nshots, int nx, int nz, int fp64, void *image1, void *image2s, void *image2m,
                     void *illum, int *nonfinite, cudaStream_t s);
// out[s] (zeroed by the caller) <- bits of max |p| over shot s's padded grid, side 0: source
// wavefield, 1: receiver wavefield; non-finite values count as +infinity.
void launch_absmax(const ShotDev *shots, int nshots, int side, unsigned *out, cudaStream_t s);
void launch_inject(const ShotDev *shots, int nshots, int maxrec, int it, float dt, int gather_prec, cudaStream_t s);
size_t finalize_shot_size();
void fill_finalize_shot(void *dst, const void *g1, const void *illum, const void *const *gx, int nx1, int nxi,
                        int nwin, int pitch, int npml, int acc);
void launch_image_extra(const ShotDev *shots, int nshots, int max_nxi, int max_nzi, int parity, int fp64,
                        float dx, float dz, float dt, cudaStream_t s);
// RTM_ACC_FP64_BLOCKED: every shot's fp32 partial sums g1, illum added into its fp64 totals
// and cleared, on the image interior (max_nxi x max_nzi: the batch's largest interior).
void launch_image_flush(const ShotDev *shots, int nshots, int max_nxi, int max_nzi, cudaStream_t s);
void launch_finalize_extra(const void *fs, int nshots, int nx, int nz, int fp64, void *const img[7], cudaStream_t s);
