// rtm_strip.cuh — saving one boundary-strip cell after a source-pass step (reference
// save_d_vxpml / save_d_vzpml / save_d_ppmllr / save_d_ppmltb, kernel.cu:1186-1293), shared
// by the strip-save kernel (rtm_kernels.cu) and the persistent source pass (rtm_stencil.cu).
// Strip layout per step: [vx lr 2][nzi][10] [vz tb 2][10][nxi] [p lr 2][nzi][10] [p tb 2][10][nxi].
#pragma once
#include "rtm_types.h"

// Value of strip cell idx (< S.strip_len) in the source wavefield's current fields.
__device__ __forceinline__ float strip_cell_value(const ShotDev &S, int idx)
{
    constexpr int R = RTM_RADIUS;
    const int X = S.X, Z = S.Z, npml = S.npml, nxi = S.nxi, nzi = S.nzi, pitch = S.pitch;
    const int lr = R * nzi, tb = R * nxi;
    int k = idx, z, x;
    const float *f;
    if (k < 2 * lr || (k >= 2 * lr + 2 * tb && k < 4 * lr + 2 * tb)) {   // left/right strips
        const bool pstrip = k >= 2 * lr;
        if (pstrip) k -= 2 * lr + 2 * tb;
        const int side = k >= lr ? 1 : 0, rem = k - side * lr;   // k < 2 * lr here
        const int q = rem / R;                                   // R: a constant divisor
        z = npml + q;
        const int c = rem - q * R;
        // vx right strip starts at X-npml-1 (vx has X-1 columns), p right strip at X-npml
        x = side == 0 ? npml - R + c : (pstrip ? X - npml : X - npml - 1) + c;
        f = pstrip ? S.a.p : S.a.vx;
    } else {                                                             // top/bottom strips
        const bool pstrip = k >= 4 * lr + 2 * tb;
        k -= pstrip ? 4 * lr + 2 * tb : 2 * lr;
        const int side = k >= tb ? 1 : 0, rem = k - side * tb;   // k < 2 * tb here
        // r = rem / nxi (< R): a float estimate (rem < 2^24, exact in fp32; the product's
        // rounding moves the estimate by at most one) corrected both ways, without the
        // integer division's instruction sequence
        int r = __float2int_rz(__int2float_rn(rem) * __frcp_rn(__int2float_rn(nxi)));
        r -= (r * nxi > rem) ? 1 : 0;
        r += ((r + 1) * nxi <= rem) ? 1 : 0;
        x = npml + (rem - r * nxi);
        // vz bottom strip starts at Z-npml-1 (vz has Z-1 rows), p bottom strip at Z-npml
        z = side == 0 ? npml - R + r : (pstrip ? Z - npml : Z - npml - 1) + r;
        f = pstrip ? S.a.p : S.a.vz;
    }
    return f[(size_t)z * pitch + x];
}

// Cell idx (< S.strip_len) of step it: fp32 strips straight to strips[it]; fp16/bf16 strips
// to the fp32 staging ring slot `ring` (packed later).
__device__ __forceinline__ void strip_save_cell(const ShotDev &S, int idx, int it, int ring, int prec)
{
    const float v = strip_cell_value(S, idx);
    if (prec == RTM_FP32) ((float *)S.strips)[(size_t)it * S.strip_len + idx] = v;
    else S.strip_stage[(size_t)ring * S.strip_len + idx] = v;
}
