// rtm_kernels.cu — per-shot setup, storage-precision, injection and stacking kernels of
// the RTM path (the time-step stencils are in rtm_stencil.cu).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "rtm_strip.cuh"
#include "rtm_types.h"

#define R RTM_RADIUS
#define RTM_PI 3.1415926535897932   // the reference's pi (common.h:11)

namespace {

__device__ __forceinline__ float load_gather(const StepArgs &a, const ShotDev &S, int j)
{
    size_t idx = (size_t)a.it * S.nrec + j;
    if (a.gather_prec == RTM_FP16) return __half2float(((const __half *)S.gather)[idx]) * S.gather_scale[a.it];
    if (a.gather_prec == RTM_BF16) return __bfloat162float(((const __nv_bfloat16 *)S.gather)[idx]) * S.gather_scale[a.it];
    return ((const float *)S.gather)[idx];
}

}  // namespace

// =====================================================================================
// Setup kernels (once per shot).

// PML profiles (reference kernel.cu:174-269) and the damping factors the stencil kernels
// use: c1 = 1 - dt*d/2, c2 = 2 - c1, evaluated in double as the reference does
// (kernel.cu:596-597), stored as c1 and 1/c2.  Outside the bands c1 = 1/c2 = 1.
__global__ void k_setup_pml(float *pml, int X, int Z, int npml, float dx, float dz, float dt, float vpmax)
{
    const PmlOffsets o = pml_offsets(X, Z);
    const int n = X > Z ? X : Z;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int axis = 0; axis < 2; axis++) {
            const int L = axis == 0 ? X : Z;
            const float h = axis == 0 ? dx : dz;
            if (i >= L) continue;
            float R_ = 1.0e-10;
            float d = npml * h;
            float d0 = 1.5 * vpmax * logf(1 / R_) / d;
            float temp;
            // pressure node profile (cuda_pmlCoeffpx/pz), n = L
            float dp = 0.0f;
            if (i < npml) { temp = (float)(npml - i); temp = temp / npml; temp = temp * temp; dp = d0 * temp; }
            if (i >= L - npml && i < L) { temp = (float)(i - L + npml + 1); temp = temp / npml; temp = temp * temp; dp = d0 * temp; }
            // velocity node profile (cuda_pmlCoeffvx/vz), n = L-1
            float dv = 0.0f;
            if (i < L - 1) {
                const int Lv = L - 1;
                if (i < npml) { temp = (float)(npml - i) - 0.5; temp = temp / npml; temp = temp * temp; dv = d0 * temp; }
                if (i >= Lv - npml && i < Lv) { temp = (float)(i - Lv + npml + 1) - 0.5; temp = temp / npml; temp = temp * temp; dv = d0 * temp; }
            }
            float c1p = 1.0 - 0.5 * dt * dp, c2p = 2.0 - c1p;
            float c1v = 1.0 - 0.5 * dt * dv, c2v = 2.0 - c1v;
            c2p = 1.0f / c2p;
            c2v = 1.0f / c2v;
            const bool bandp = (i < npml) || (i >= L - npml);
            const bool bandv = (i < npml) || (i >= L - npml - 1);
            if (axis == 0) {
                pml[o.ddx + i] = dp;
                pml[o.c1x + i] = bandp ? c1p : 1.0f;
                pml[o.ic2x + i] = bandp ? c2p : 1.0f;
                if (i < L - 1) pml[o.ddxvx + i] = dv;
                pml[o.c1vx + i] = (bandv && i < L - 1) ? c1v : 1.0f;
                pml[o.ic2vx + i] = (bandv && i < L - 1) ? c2v : 1.0f;
            } else {
                pml[o.ddz + i] = dp;
                pml[o.c1z + i] = bandp ? c1p : 1.0f;
                pml[o.ic2z + i] = bandp ? c2p : 1.0f;
                if (i < L - 1) pml[o.ddzvz + i] = dv;
                pml[o.c1vz + i] = (bandv && i < L - 1) ? c1v : 1.0f;
                pml[o.ic2vz + i] = (bandv && i < L - 1) ? c2v : 1.0f;
            }
        }
    }
}

// dt * Gaussian source over the stamp box (reference kernel.cu:23-35 then the dt factor of
// kernel.cu:45).
__global__ void k_setup_source(float *src, int sbx0, int sbz0, int sbnx, int sbnz, int nsx, int nsz,
                               float amp, float alp, float dx2, float dz2, float dt)
{
    const int n = sbnx * sbnz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int idz = sbz0 + i / sbnx, idx = sbx0 + i % sbnx;
        float dist = (idx - nsx) * (idx - nsx) * dx2 + (idz - nsz) * (idz - nsz) * dz2;
        float s = amp * expf(-alp * alp * dist);
        src[i] = dt * s;
    }
}

// Ricker wavelet, reference kernel.cu:13-22.
__global__ void k_ricker(float *w, float fdom, float dt, int nt)
{
    int it = threadIdx.x + blockDim.x * blockIdx.x;
    float temp = 3.1415926535897932 * fdom * fabs(it * dt - 1.0 / fdom);
    temp *= temp;
    if (it < nt) w[it] = (1.0 - 2.0 * temp) * expf(-temp);
}

// Direct-wave mute of one shot's fp32 gather, reference kernel.cu:96-173.  vrow holds v^2
// along the receiver row (indexed by padded column) followed by v^2 at the source node.
__global__ void k_mute(float *g, const float *vrow, int X, int nsx, int nsz, int nt, int rz, int rx0,
                       int nrec, int nw, int tlength, float dx2, float dz2, float rdt)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nrec) return;
    float vtemp = 0.482 * (1.0 / sqrtf(vrow[rx0 + idx]) + 1.0 / sqrtf(vrow[X]));
    float dist = (idx + rx0 - nsx) * (idx + rx0 - nsx) * dx2 + (rz - nsz) * (rz - nsz) * dz2;
    dist = sqrtf(dist);
    int temp = tlength < nt ? tlength : nt;
    int cut = ((int)(dist * vtemp * rdt) + nw) < nt ? ((int)(dist * vtemp * rdt) + nw) : nt;
    cut = cut > temp ? cut : temp;
    cut = cut < nt ? cut : nt;
    for (int it = blockIdx.y; it < nt && it <= cut; it += gridDim.y) g[(size_t)it * nrec + idx] = 0.0f;
}

// =====================================================================================
// Boundary strips of the source pass (reference save_d_vxpml / save_d_vzpml /
// save_d_ppmllr / save_d_ppmltb, kernel.cu:1186-1293): after step `it` of every shot of a
// batch, copy the ten cells inside each PML edge of vx, vz and p into the step's strip
// record, laid out [vx lr 2][nzi][10] [vz tb 2][10][nxi] [p lr 2][nzi][10] [p tb 2][10][nxi].
// fp32 strips go straight to strips[it]; fp16/bf16 strips go to the fp32 staging ring slot
// `ring` and are packed later.  Each thread copies CPT cells blockDim apart, its loads issued
// before its stores: 8 when the batch's strips fill the GPU several times over, so that a
// thread has several loads in flight (one cell per thread waited out the load latency in ~17
// rounds of resident threads at 64 shots); 1 for small batches, where more threads with one
// cell each finish sooner.  Grid (ceil(strip_len / (256 * CPT)), nshots).
template <int CPT>
__global__ void __launch_bounds__(256) k_strip_save(const ShotDev *shots, int it, int ring, int prec)
{
    const ShotDev &S = shots[blockIdx.y];
    const int i0 = blockIdx.x * blockDim.x * CPT + threadIdx.x;
    float v[CPT];
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        const int idx = i0 + c * blockDim.x;
        v[c] = idx < S.strip_len ? strip_cell_value(S, idx) : 0.0f;
    }
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        const int idx = i0 + c * blockDim.x;
        if (idx >= S.strip_len) break;
        if (prec == RTM_FP32) ((float *)S.strips)[(size_t)it * S.strip_len + idx] = v[c];
        else S.strip_stage[(size_t)ring * S.strip_len + idx] = v[c];
    }
}

// =====================================================================================
// Reduced-precision storage.

// Pack `nsteps` staged fp32 strip steps into fp16/bf16 with one exact power-of-two scale per
// (step, strip): grid (nsteps*4 strips, nshots).
__global__ void k_strip_pack(const ShotDev *shots, int it0, int ring0, int nsteps, int prec)
{
    __shared__ float s_max[32];
    const ShotDev &S = shots[blockIdx.y];
    const int step = blockIdx.x / 4, kind = blockIdx.x % 4;
    const long a = 2L * R * S.nzi, b = 2L * R * S.nxi;
    const long off[4] = {0, a, a + b, 2 * a + b};
    const long len[4] = {a, b, a, b};
    const float *src = S.strip_stage + (size_t)(ring0 + step) * S.strip_len + off[kind];
    float m = 0.0f;
    for (long i = threadIdx.x; i < len[kind]; i += blockDim.x) m = fmaxf(m, fabsf(src[i]));
    for (int s = 16; s > 0; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? s_max[threadIdx.x] : 0.0f;
        for (int s = 16; s > 0; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
        if (threadIdx.x == 0) s_max[0] = m;
    }
    __syncthreads();
    m = s_max[0];
    // power-of-two scale 2^e with |x| < 2^e (exact scaling, only the rounding of the narrow
    // type remains).  The values are divided by ldexpf, not multiplied by 1/scale: for a block
    // whose largest value is a subnormal float, 1/scale overflows to infinity
    int e = 0;
    if (m > 0.0f) frexpf(m, &e);
    const float scale = ldexpf(1.0f, e);
    const int it = it0 + step;
    if (threadIdx.x == 0) S.strip_scale[(size_t)it * 4 + kind] = scale;
    const size_t dst0 = (size_t)it * S.strip_len + off[kind];
    for (long i = threadIdx.x; i < len[kind]; i += blockDim.x) {
        float v = ldexpf(src[i], -e);
        if (prec == RTM_FP16) ((__half *)S.strips)[dst0 + i] = __float2half_rn(v);
        else ((__nv_bfloat16 *)S.strips)[dst0 + i] = __float2bfloat16_rn(v);
    }
}

// Pack an fp32 gather [nt][nrec] into fp16/bf16 with one power-of-two scale per time sample.
__global__ void k_gather_pack(const float *g, void *out, float *scale, int nt, int nrec, int prec)
{
    __shared__ float s_max[32];
    const int it = blockIdx.x;
    const float *row = g + (size_t)it * nrec;
    float m = 0.0f;
    for (int i = threadIdx.x; i < nrec; i += blockDim.x) m = fmaxf(m, fabsf(row[i]));
    for (int s = 16; s > 0; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? s_max[threadIdx.x] : 0.0f;
        for (int s = 16; s > 0; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
        if (threadIdx.x == 0) s_max[0] = m;
    }
    __syncthreads();
    m = s_max[0];
    int e = 0;   // as in k_strip_pack: 2^e > |x|, values divided by ldexpf
    if (m > 0.0f) frexpf(m, &e);
    if (threadIdx.x == 0) scale[it] = ldexpf(1.0f, e);
    for (int i = threadIdx.x; i < nrec; i += blockDim.x) {
        float v = ldexpf(row[i], -e);
        if (prec == RTM_FP16) ((__half *)out)[(size_t)it * nrec + i] = __float2half_rn(v);
        else ((__nv_bfloat16 *)out)[(size_t)it * nrec + i] = __float2bfloat16_rn(v);
    }
}

// =====================================================================================
// Per-batch image finalisation (reference rtm_model.cu:462-488, kernel.cu:1556-1615):
// each shot's g1 and illum are tapered laterally, then image2s += g1/(illum + 1e-6)
// (double division, as the reference's eps is a double literal), image1 += g1,
// image2m += g1, Illum += illum, at the shot's column offset nx1.  One thread per global
// image cell walks the batch's shots in order, so overlapping apertures stack in a fixed
// order.  Images are fp32 (reference) or fp64.
struct FinalizeShot {
    const void *g1, *illum;   // [Z][pitch]: interior cell (iz, lx) at (iz+npml)*pitch + lx+npml
    const void *gx[4];        // the other imaging conditions' g2, g3, g3t, g4 (null when off)
    int nx1, nxi, nwin, pitch, npml;
    int acc;                  // RtmAccum of g1 and illum (fp32, fp64 or compensated fp32 pairs)
};

// Value of a per-shot accumulator cell: fp32, fp64, or a compensated pair (s - c in double).
__device__ __forceinline__ double acc_value(const void *a, size_t ip, int acc)
{
    if (acc == RTM_ACC_FP64) return ((const double *)a)[ip];
    if (acc == RTM_ACC_KAHAN) {
        const float2 v = ((const float2 *)a)[ip];
        return (double)v.x - (double)v.y;
    }
    return ((const float *)a)[ip];
}

// Taper weight of interior column lx (cuda_taper_calculate, kernel.cu:1591-1604).
__device__ __forceinline__ float taper_at(int lx, int nwin, int nxl)
{
    const float alpha = 0.06f;
    float tp = 1.0f;
    if (lx < nwin) tp = expf(-alpha * alpha * (nwin - lx) * (nwin - lx));
    if (lx >= nxl - nwin && lx < nxl) tp = expf(-alpha * alpha * (lx - nxl + nwin + 1) * (lx - nxl + nwin + 1));
    if (lx >= nwin && lx < nxl - nwin) tp = 1.0f;
    return tp;
}

// nonfinite: lowest batch index of a shot whose g1 or illumination holds a NaN or infinity
// (a diverging run: unstable time step or invalid model values); left as set when none.
__global__ void k_finalize(const FinalizeShot *fs, int nshots, int nx, int nz, int fp64, void *image1,
                           void *image2s, void *image2m, void *illum_total, int *nonfinite)
{
    const long n = (long)nx * nz;
    int bad = nshots;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int iz = (int)(i / nx), ix = (int)(i - (long)iz * nx);
        for (int s = 0; s < nshots; s++) {
            const FinalizeShot f = fs[s];
            const int lx = ix - f.nx1;
            if (lx < 0 || lx >= f.nxi) continue;
            const float tp = taper_at(lx, f.nwin, f.nxi);
            const size_t ip = (size_t)(iz + f.npml) * f.pitch + lx + f.npml;
            if (fp64) {
                double g = acc_value(f.g1, ip, f.acc) * (double)tp;
                double il = acc_value(f.illum, ip, f.acc) * (double)tp;
                if (!isfinite(g) || !isfinite(il)) bad = min(bad, s);
                ((double *)image2s)[i] += g / (il + 1.0e-6);
                ((double *)image1)[i] += g;
                ((double *)image2m)[i] += g;
                ((double *)illum_total)[i] += il;
            } else {
                float g = ((const float *)f.g1)[ip] * tp;
                float il = ((const float *)f.illum)[ip] * tp;
                if (!isfinite(g) || !isfinite(il)) bad = min(bad, s);
                float *i2s = (float *)image2s;
                i2s[i] = i2s[i] + g / (il + 1.0e-6);
                ((float *)image1)[i] += g;
                ((float *)image2m)[i] += g;
                ((float *)illum_total)[i] += il;
            }
        }
    }
    if (bad < nshots) atomicMin(nonfinite, bad);
}

// Largest |p| of each shot's wavefield (a: source side, b: receiver side) over its padded
// grid, for the progress snapshots the reference prints every tsnap (rtm_model.cu:271-273,
// 324-326, 415-417); a NaN or infinity reads as +infinity.  out[s] holds the float's bits
// (non-negative floats order like their bit patterns) and must start at 0.
__global__ void k_absmax(const ShotDev *shots, int side, unsigned *out)
{
    const ShotDev &sh = shots[blockIdx.y];
    const float *p = side ? sh.b.p : sh.a.p;
    const long n = (long)sh.Z * sh.pitch;
    float m = 0.0f;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long iz = i / sh.pitch, ix = i - iz * sh.pitch;
        if (ix >= sh.X) continue;
        const float v = p[i];
        m = fmaxf(m, isfinite(v) ? fabsf(v) : INFINITY);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out + blockIdx.y, __float_as_uint(m));
}

void launch_absmax(const ShotDev *shots, int nshots, int side, unsigned *out, cudaStream_t s)
{
    dim3 grid(std::max(1, 148 * 4 / std::max(1, nshots)), nshots);
    k_absmax<<<grid, 256, 0, s>>>(shots, side, out);
}

// The other images of a batch (rtm_model.cu:466-487): taper g2, g3, g4 and g3t like g1, then
// image3s/4s/5s += g2/g3/g4 / (illum + 1e-6) with the shot's tapered illumination (the
// division in double, as cuda_applyics promotes it), image3m/4m/5m += g2/g3/g4, imagetrue +=
// g3t.  img = {image3s, image4s, image5s, image3m, image4m, image5m, imagetrue}.
struct ExtraImages {
    void *img[7];
};
template <typename T>
__global__ void k_finalize_extra(const FinalizeShot *fs, int nshots, int nx, int nz, ExtraImages out)
{
    const long n = (long)nx * nz;
    T *im[7];
    for (int k = 0; k < 7; k++) im[k] = (T *)out.img[k];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int iz = (int)(i / nx), ix = (int)(i - (long)iz * nx);
        for (int s = 0; s < nshots; s++) {
            const FinalizeShot f = fs[s];
            const int lx = ix - f.nx1;
            if (lx < 0 || lx >= f.nxi) continue;
            const T tp = (T)taper_at(lx, f.nwin, f.nxi);
            const size_t ip = (size_t)(iz + f.npml) * f.pitch + lx + f.npml;
            const T il = (T)acc_value(f.illum, ip, f.acc) * tp;
            const T g[4] = {((const T *)f.gx[0])[ip] * tp, ((const T *)f.gx[1])[ip] * tp,
                            ((const T *)f.gx[2])[ip] * tp, ((const T *)f.gx[3])[ip] * tp};
            const int gi[3] = {0, 1, 3};   // g2 -> image3, g3 -> image4, g4 -> image5
            for (int k = 0; k < 3; k++) {
                im[k][i] = (T)(im[k][i] + g[gi[k]] / (il + 1.0e-6));
                im[3 + k][i] += g[gi[k]];
            }
            im[6][i] += g[2];
        }
    }
}

// The reference's other imaging conditions for one backward step (kernel.cu:1417-1522;
// rtm_model.cu:450-455), run after the receiver update on the interior of every shot of a
// batch, one thread per cell, grid (ceil(nxi/32), ceil(nzi/8), nshots):
//   g2  += the up-down, down-up, left-right and right-left products of the decomposed
//          pressures (the reference keeps four arrays and adds them at the end);
//   g3  += ps p cos(theta), theta from the angle between the source and receiver Poynting
//          vectors (the reference bins it by whole degrees in 61 arrays and adds the bins at
//          the end; only the sum is used);
//   g3t += ps p 16 pi v / sin(theta);
//   g4  += -(ps - ps_pre)(p - p_pre)/(dt^2 v^2) + grad ps . grad p (centred differences).
// PAR = 1 reads vx as the reference does, at the pressure cell's flat index z*X + x on its
// (X-1)-wide vx arrays, and takes the receiver vz in the source Poynting term; PAR = 0 reads
// vx and vz at the cell itself.  Operand types follow the reference's expressions (float
// values, double literals).  Each cell's pressures then become the "before" values of the
// next (earlier) step.
template <int PAR, typename ACC>
__global__ void k_image_extra(const ShotDev *shots, float dx, float dz, float dt)
{
    const ShotDev &S = shots[blockIdx.z];
    const int ix = blockIdx.x * 32 + threadIdx.x, iz = blockIdx.y * 8 + threadIdx.y;
    if (ix >= S.nxi || iz >= S.nzi) return;
    const int X = S.X, pitch = S.pitch, npml = S.npml;
    const int z = iz + npml, x = ix + npml;
    const size_t id = (size_t)z * pitch + x;
    size_t ivx = id;
    if (PAR) {
        const long f = (long)z * X + x;
        ivx = (size_t)(f / (X - 1)) * pitch + (size_t)(f % (X - 1));
    }
    const float ps = S.a.p[id], p = S.b.p[id];
    const float vxs = S.a.vx[ivx], vx = S.b.vx[ivx], vzs = S.a.vz[id], vz = S.b.vz[id];
    const float v2 = S.vp2_b[id];
    ACC *g2 = (ACC *)S.gx[0], *g3 = (ACC *)S.gx[1], *g3t = (ACC *)S.gx[2], *g4 = (ACC *)S.gx[3];
    // decomposition (kernel.cu:1417-1451)
    {
        const float vectxs = -ps * vxs, vectzs = -ps * vzs, vectxr = -p * vx, vectzr = -p * vz;
        const float psu = vectzs < 0 ? ps : 0.0f, psd = vectzs > 0 ? ps : 0.0f;
        const float psl = vectxs < 0 ? ps : 0.0f, psr = vectxs > 0 ? ps : 0.0f;
        const float pu = vectzr < 0 ? p : 0.0f, pd = vectzr > 0 ? p : 0.0f;
        const float pl = vectxr < 0 ? p : 0.0f, pr = vectxr > 0 ? p : 0.0f;
        g2[id] += (ACC)(psu * pd + psd * pu + psl * pr + psr * pl);
    }
    // Poynting angle (kernel.cu:1452-1485)
    {
        const float ksx = ps * vxs, ksz = ps * (PAR ? vz : vzs), krx = p * vx, krz = p * vz;
        const float q = (ksx * ksx + ksz * ksz) * (krx * krx + krz * krz);
        const double den = sqrtf(q) > 0 ? (double)sqrtf(q) : 1.0e-6;
        float wt = (float)((double)(ksx * krx + ksz * krz) / den);
        if (wt >= -1.0 && wt <= 1.0) {
            wt = (float)(0.5 * (double)acosf(wt));
            wt = (float)(RTM_PI / 2.0 - (double)wt);
            if (wt > 0 && wt <= RTM_PI / 3.0) {
                const float c = ps * p * cosf(wt);
                const double t = (double)(ps * p) * 16.0 * RTM_PI * (double)sqrtf(v2) / (double)sinf(wt);
                g3[id] += (ACC)c;
                g3t[id] = (ACC)((double)g3t[id] + t);
            }
        }
    }
    // energy norm (kernel.cu:1486-1522)
    {
        const float *ap = S.a.p, *bp = S.b.p;
        const float psx = (float)(0.5 * (double)(ap[id + 1] - ap[id - 1]) / dx);
        const float psz = (float)(0.5 * (double)(ap[id + pitch] - ap[id - pitch]) / dz);
        const float px = (float)(0.5 * (double)(bp[id + 1] - bp[id - 1]) / dx);
        const float pz = (float)(0.5 * (double)(bp[id + pitch] - bp[id - pitch]) / dz);
        g4[id] += (ACC)(-(ps - S.ps_pre[id]) * (p - S.p_pre[id]) / (dt * dt * v2) + psx * px + psz * pz);
    }
    S.ps_pre[id] = ps;
    S.p_pre[id] = p;
}

// =====================================================================================
// Small per-batch helpers.

// Receiver injection of time sample `it` before the first backward step (rtm_model.cu:410).
__global__ void k_inject(const ShotDev *shots, int it, float dt, int gather_prec)
{
    const ShotDev &S = shots[blockIdx.y];
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= S.nrec) return;
    StepArgs a;
    a.it = it;
    a.gather_prec = gather_prec;
    float v = load_gather(a, S, j);
    S.b.p[(size_t)S.rz * S.pitch + S.rx0 + j] = dt * v;
}

// =====================================================================================
// Host launchers.
#include "rtm_launch.h"

void launch_setup_pml(float *pml, int X, int Z, int npml, float dx, float dz, float dt, float vpmax, cudaStream_t s)
{
    int n = X > Z ? X : Z;
    k_setup_pml<<<(n + 127) / 128, 128, 0, s>>>(pml, X, Z, npml, dx, dz, dt, vpmax);
}
void launch_setup_source(float *src, int sbx0, int sbz0, int sbnx, int sbnz, int nsx, int nsz, float amp, float alp,
                         float dx2, float dz2, float dt, cudaStream_t s)
{
    int n = sbnx * sbnz;
    k_setup_source<<<(n + 255) / 256, 256, 0, s>>>(src, sbx0, sbz0, sbnx, sbnz, nsx, nsz, amp, alp, dx2, dz2, dt);
}
void launch_ricker(float *w, float fdom, float dt, int nt, cudaStream_t s)
{
    k_ricker<<<(nt + 511) / 512, 512, 0, s>>>(w, fdom, dt, nt);
}
void launch_mute(float *g, const float *vrow, int X, int nsx, int nsz, int nt, int rz, int rx0, int nrec, int nw,
                 int tlength, float dx2, float dz2, float rdt, cudaStream_t s)
{
    dim3 grid((nrec + 127) / 128, 64);
    k_mute<<<grid, 128, 0, s>>>(g, vrow, X, nsx, nsz, nt, rz, rx0, nrec, nw, tlength, dx2, dz2, rdt);
}
void launch_strip_save(const ShotDev *shots, int nshots, int max_strip_len, int it, int ring, int prec,
                       cudaStream_t s)
{
    if ((long)nshots * max_strip_len >= 8L * 148 * 2048) {
        dim3 grid((max_strip_len + 256 * 8 - 1) / (256 * 8), nshots);
        k_strip_save<8><<<grid, 256, 0, s>>>(shots, it, ring, prec);
    } else {
        dim3 grid((max_strip_len + 255) / 256, nshots);
        k_strip_save<1><<<grid, 256, 0, s>>>(shots, it, ring, prec);
    }
}
void launch_strip_pack(const ShotDev *shots, int nshots, int it0, int ring0, int nsteps, int prec, cudaStream_t s)
{
    dim3 grid(nsteps * 4, nshots);
    k_strip_pack<<<grid, 512, 0, s>>>(shots, it0, ring0, nsteps, prec);
}
void launch_gather_pack(const float *g, void *out, float *scale, int nt, int nrec, int prec, cudaStream_t s)
{
    k_gather_pack<<<nt, 256, 0, s>>>(g, out, scale, nt, nrec, prec);
}
void launch_finalize(const void *fs, int nshots, int nx, int nz, int fp64, void *image1, void *image2s, void *image2m,
                     void *illum, int *nonfinite, cudaStream_t s)
{
    long n = (long)nx * nz;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_finalize<<<blocks, 256, 0, s>>>((const FinalizeShot *)fs, nshots, nx, nz, fp64, image1, image2s, image2m, illum,
                                      nonfinite);
}
// Flush of the blocked accumulation: total += partial, partial = 0, for the interior cells the
// imaging writes (x in [npml, X-npml), z in [npml, Z-npml)); one thread per cell, rows along
// x, so every access is coalesced (48 bytes per cell per flush).
__global__ void k_image_flush(const ShotDev *shots)
{
    const ShotDev &S = shots[blockIdx.z];
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, nzi = S.Z - 2 * S.npml;
    if (ix >= S.X - 2 * S.npml) return;
    float *g1 = (float *)S.g1, *il = (float *)S.illum;
    for (int iz = blockIdx.y; iz < nzi; iz += gridDim.y) {
        const size_t id = (size_t)(iz + S.npml) * S.pitch + (ix + S.npml);
        S.g1t[id] += (double)g1[id];
        S.illt[id] += (double)il[id];
        g1[id] = 0.f;
        il[id] = 0.f;
    }
}
void launch_image_flush(const ShotDev *shots, int nshots, int max_nxi, int max_nzi, cudaStream_t s)
{
    dim3 grid((max_nxi + 255) / 256, std::min(max_nzi, 65535), nshots);
    k_image_flush<<<grid, 256, 0, s>>>(shots);
}
void launch_image_extra(const ShotDev *shots, int nshots, int max_nxi, int max_nzi, int parity, int fp64,
                        float dx, float dz, float dt, cudaStream_t s)
{
    dim3 grid((max_nxi + 31) / 32, (max_nzi + 7) / 8, nshots), block(32, 8);
    if (parity) {
        if (fp64) k_image_extra<1, double><<<grid, block, 0, s>>>(shots, dx, dz, dt);
        else k_image_extra<1, float><<<grid, block, 0, s>>>(shots, dx, dz, dt);
    } else {
        if (fp64) k_image_extra<0, double><<<grid, block, 0, s>>>(shots, dx, dz, dt);
        else k_image_extra<0, float><<<grid, block, 0, s>>>(shots, dx, dz, dt);
    }
}
void launch_finalize_extra(const void *fs, int nshots, int nx, int nz, int fp64, void *const img[7], cudaStream_t s)
{
    long n = (long)nx * nz;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    ExtraImages out;
    for (int k = 0; k < 7; k++) out.img[k] = img[k];
    if (fp64) k_finalize_extra<double><<<blocks, 256, 0, s>>>((const FinalizeShot *)fs, nshots, nx, nz, out);
    else k_finalize_extra<float><<<blocks, 256, 0, s>>>((const FinalizeShot *)fs, nshots, nx, nz, out);
}
void launch_inject(const ShotDev *shots, int nshots, int maxrec, int it, float dt, int gather_prec, cudaStream_t s)
{
    dim3 grid((maxrec + 127) / 128, nshots);
    k_inject<<<grid, 128, 0, s>>>(shots, it, dt, gather_prec);
}
size_t finalize_shot_size() { return sizeof(FinalizeShot); }
void fill_finalize_shot(void *dst, const void *g1, const void *illum, const void *const *gx, int nx1, int nxi,
                        int nwin, int pitch, int npml, int acc)
{
    FinalizeShot f;
    f.acc = acc;
    f.g1 = g1;
    f.illum = illum;
    for (int k = 0; k < 4; k++) f.gx[k] = gx ? gx[k] : nullptr;
    f.nx1 = nx1;
    f.nxi = nxi;
    f.nwin = nwin;
    f.pitch = pitch;
    f.npml = npml;
    *(FinalizeShot *)dst = f;
}
