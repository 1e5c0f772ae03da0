// rtm_kernels.cu — sm_100a kernels of the RTM hot path.
//
// One time step of one wavefield is two launches over a flat (shot, tile) work list, so a
// batch of shots with different apertures shares every launch:
//   k_vel_*  : particle-velocity update (+ strip save / strip restore)
//   k_pres_* : pressure update with split-field PML (+ source, receiver sampling or
//              injection, strip save / restore, cross-correlation imaging)
// The reference runs the same step as 9-22 separate launches with z-major (uncoalesced)
// thread mapping (gubingluo kernel.cu:318-1416, rtm_model.cu:326-455).  Here lanes run
// along x (contiguous), tiles are staged in shared memory with their halos, and the PML
// is a per-cell predicate inside the same kernels: the reduced local FD order near the
// outer edge (reference cuda_norder*, kernel.cu:271-317) selects a row of the
// zero-padded coefficient table, so taps beyond the local order multiply exact zeros.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "rtm_types.h"

#define TX RTM_TX
#define TZ RTM_TZ
#define R RTM_RADIUS
#define NTHR 256          // 32 x 8 threads
#define ROWS_PER_THR (TZ / 8)

namespace {

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

// Stage rows [z0, z0+nr) x cols [x0, x0+nc) of field f (valid region xv x zv) into s[nr][nc];
// cells outside the valid region read as zero.
__device__ __forceinline__ void stage(float *s, const float *__restrict__ f, int pitch, int xv,
                                      int zv, int z0, int x0, int nr, int nc)
{
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int i = tid; i < nr * nc; i += NTHR) {
        int r = i / nc, c = i - r * nc;
        int z = z0 + r, x = x0 + c;
        float v = 0.0f;
        if (z >= 0 && z < zv && x >= 0 && x < xv) v = __ldg(&f[(size_t)z * pitch + x]);
        s[i] = v;
    }
}

__device__ __forceinline__ float load_strip(const void *base, size_t idx, int prec, float scale)
{
    if (prec == RTM_FP16) return __half2float(((const __half *)base)[idx]) * scale;
    if (prec == RTM_BF16) return __bfloat162float(((const __nv_bfloat16 *)base)[idx]) * scale;
    return ((const float *)base)[idx];
}

__device__ __forceinline__ void store_strip(const StepArgs &a, const ShotDev &S, size_t idx, float v)
{
    if (a.strip_prec == RTM_FP32)
        ((float *)S.strips)[(size_t)a.it * S.strip_len + idx] = v;
    else
        S.strip_stage[(size_t)a.ring * S.strip_len + idx] = v;
}

__device__ __forceinline__ float load_gather(const StepArgs &a, const ShotDev &S, int j)
{
    size_t idx = (size_t)a.it * S.nrec + j;
    if (a.gather_prec == RTM_FP16) return __half2float(((const __half *)S.gather)[idx]) * S.gather_scale[a.it];
    if (a.gather_prec == RTM_BF16) return __bfloat162float(((const __nv_bfloat16 *)S.gather)[idx]) * S.gather_scale[a.it];
    return ((const float *)S.gather)[idx];
}

// Strip element indices (reference save_d_*, kernel.cu:1186-1293).  Returns -1 when the
// cell is not part of that strip.
__device__ __forceinline__ long strip_idx_vx(const ShotDev &S, int z, int x)
{
    if (z < S.npml || z >= S.Z - S.npml) return -1;
    int iz = z - S.npml;
    if (x >= S.npml - R && x < S.npml) return (long)iz * R + (x - (S.npml - R));
    int xr = S.X - S.npml - 1;
    if (x >= xr && x < xr + R) return (long)R * S.nzi + (long)iz * R + (x - xr);
    return -1;
}
__device__ __forceinline__ long strip_idx_vz(const ShotDev &S, int z, int x)
{
    if (x < S.npml || x >= S.X - S.npml) return -1;
    long base = 2L * R * S.nzi;
    int ix = x - S.npml;
    if (z >= S.npml - R && z < S.npml) return base + (long)(z - (S.npml - R)) * S.nxi + ix;
    int zr = S.Z - S.npml - 1;
    if (z >= zr && z < zr + R) return base + (long)R * S.nxi + (long)(z - zr) * S.nxi + ix;
    return -1;
}
__device__ __forceinline__ long strip_idx_p(const ShotDev &S, int z, int x)
{
    long base = 2L * R * S.nzi + 2L * R * S.nxi;
    if (z >= S.npml && z < S.Z - S.npml) {
        int iz = z - S.npml;
        if (x >= S.npml - R && x < S.npml) return base + (long)iz * R + (x - (S.npml - R));
        int xr = S.X - S.npml;
        if (x >= xr && x < xr + R) return base + (long)R * S.nzi + (long)iz * R + (x - xr);
        return -1;
    }
    if (x >= S.npml && x < S.X - S.npml) {
        base += 2L * R * S.nzi;
        int ix = x - S.npml;
        if (z >= S.npml - R && z < S.npml) return base + (long)(z - (S.npml - R)) * S.nxi + ix;
        int zr = S.Z - S.npml;
        if (z >= zr && z < zr + R) return base + (long)R * S.nxi + (long)(z - zr) * S.nxi + ix;
    }
    return -1;
}
// Which of the four per-step strip scales an element index belongs to.
__device__ __forceinline__ int strip_kind(const ShotDev &S, long idx)
{
    long a = 2L * R * S.nzi, b = a + 2L * R * S.nxi, c = b + 2L * R * S.nzi;
    return idx < a ? 0 : (idx < b ? 1 : (idx < c ? 2 : 3));
}

// -------------------------------------------------------------------------------------
// velocity update of one wavefield at one cell; `sp` is the staged p window whose
// element (0,0) is grid cell (z0-9, x0-9), row stride SW.
constexpr int VW = TX + 2 * R - 1;   // 51: cols x0-9 .. x0+TX+9
constexpr int VH = TZ + 2 * R - 1;   // rows z0-9 .. z0+TZ+9

__device__ __forceinline__ float vx_diff(const float *sp, const float *cf, int lz, int lx)
{
    const float *row = &sp[(lz + R - 1) * VW + lx + R - 1];
    float d = 0.0f;
#pragma unroll
    for (int i = 1; i <= R; i++) d += cf[i - 1] * (row[i] - row[-i + 1]);
    return d;
}
__device__ __forceinline__ float vz_diff(const float *sp, const float *cf, int lz, int lx)
{
    const float *col = &sp[(lz + R - 1) * VW + lx + R - 1];
    float d = 0.0f;
#pragma unroll
    for (int i = 1; i <= R; i++) d += cf[i - 1] * (col[i * VW] - col[(-i + 1) * VW]);
    return d;
}

// pressure-kernel windows: vx rows [z0, z0+TZ) cols [x0-10, x0+TX+9); vz rows [z0-10, z0+TZ+9)
constexpr int PXW = TX + 2 * R - 1;  // 51
constexpr int PZH = TZ + 2 * R - 1;  // 51

__device__ __forceinline__ void p_diff(const float *svx, const float *svz, const float *cf, int lz,
                                       int lx, float &dxs, float &dzs)
{
    const float *row = &svx[lz * PXW + lx + R];
    const float *col = &svz[(lz + R) * TX + lx];
    float a = 0.0f, b = 0.0f;
#pragma unroll
    for (int i = 1; i <= R; i++) {
        a += cf[i - 1] * (row[i - 1] - row[-i]);
        b += cf[i - 1] * (col[(i - 1) * TX] - col[-i * TX]);
    }
    dxs = a;
    dzs = b;
}

__device__ __forceinline__ void load_coef(float *s_coef, const float *coef)
{
    const int tid = threadIdx.y * 32 + threadIdx.x;
    if (tid < 100) s_coef[tid] = coef[tid];
}

// Full-grid velocity update of wavefield w (forward modelling / receiver propagation).
__device__ __forceinline__ void vel_full(const ShotDev &S, const WaveDev &w, const float *sp,
                                         const float *s_coef, const float *__restrict__ inv_rho,
                                         float dtx, float dtz, int z0, int x0, bool save,
                                         const StepArgs &a)
{
    const PmlOffsets o = pml_offsets(S.X, S.Z);
    const int lx = threadIdx.x, x = x0 + lx;
#pragma unroll
    for (int k = 0; k < ROWS_PER_THR; k++) {
        const int lz = threadIdx.y + 8 * k, z = z0 + lz;
        if (z >= S.Z || x >= S.X) continue;
        const size_t id = (size_t)z * S.pitch + x;
        const float ir = __ldg(&inv_rho[id]);
        if (x < S.X - 1) {   // vx: reference kernel.cu:430-465 and :542-630
            int r = imin(imin(x + 1, S.X - 1 - x), R);
            float d = vx_diff(sp, &s_coef[(r - 1) * R], lz, lx);
            d = d * dtx * ir;
            float c2 = S.pml[o.c2vx + x];
            float v = w.vx[id];
            if (c2 == 1.0f) v = v - d;
            else v = (S.pml[o.c1vx + x] * v - d) / c2;
            w.vx[id] = v;
            if (save) {
                long si = strip_idx_vx(S, z, x);
                if (si >= 0) store_strip(a, S, si, v);
            }
        }
        if (z < S.Z - 1) {   // vz: reference kernel.cu:466-500 and :631-713
            int r = imin(imin(z + 1, S.Z - 1 - z), R);
            float d = vz_diff(sp, &s_coef[(r - 1) * R], lz, lx);
            d = d * dtz * ir;
            float c2 = S.pml[o.c2vz + z];
            float v = w.vz[id];
            if (c2 == 1.0f) v = v - d;
            else v = (S.pml[o.c1vz + z] * v - d) / c2;
            w.vz[id] = v;
            if (save) {
                long si = strip_idx_vz(S, z, x);
                if (si >= 0) store_strip(a, S, si, v);
            }
        }
    }
}

// Full-grid pressure update of wavefield w at one cell (no source / receiver handling).
// Returns false for the outer-edge cells, which the reference never updates.
__device__ __forceinline__ bool pres_full_cell(const ShotDev &S, const WaveDev &w, const float *svx,
                                               const float *svz, const float *s_coef,
                                               const float *__restrict__ kappa, float dtx,
                                               float dtz, int z, int x, int lz, int lx, float &pout)
{
    if (z < 1 || z > S.Z - 2 || x < 1 || x > S.X - 2) return false;
    const size_t id = (size_t)z * S.pitch + x;
    const bool xb = (x < S.npml) || (x >= S.X - S.npml);
    const bool zb = (z < S.npml) || (z >= S.Z - S.npml);
    int r = R;
    if (xb || zb) r = imin(imin(imin(z, x), imin(S.Z - 1 - z, S.X - 1 - x)), R);
    float dxs, dzs;
    p_diff(svx, svz, &s_coef[(r - 1) * R], lz, lx, dxs, dzs);
    const float kap = __ldg(&kappa[id]);
    dxs = dxs * dtx * kap;
    dzs = dzs * dtz * kap;
    float p;
    if (!xb && !zb) {   // interior, reference kernel.cu:501-541
        p = w.p[id] - (dxs + dzs);
    } else {            // split-field PML, reference kernel.cu:714-1185
        const PmlOffsets o = pml_offsets(S.X, S.Z);
        float s1 = w.sx[id], s2 = w.sz[id];
        float c2x = S.pml[o.c2x + x], c2z = S.pml[o.c2z + z];
        if (c2x == 1.0f) s1 = s1 - dxs;
        else s1 = (S.pml[o.c1x + x] * s1 - dxs) / c2x;
        if (c2z == 1.0f) s2 = s2 - dzs;
        else s2 = (S.pml[o.c1z + z] * s2 - dzs) / c2z;
        w.sx[id] = s1;
        w.sz[id] = s2;
        p = s1 + s2;
    }
    pout = p;
    return true;
}

__device__ __forceinline__ bool in_src(const ShotDev &S, int z, int x)
{
    return (unsigned)(z - S.sbz0) < (unsigned)S.sbnz && (unsigned)(x - S.sbx0) < (unsigned)S.sbnx;
}
__device__ __forceinline__ float src_at(const ShotDev &S, int z, int x)
{
    return S.src[(z - S.sbz0) * S.sbnx + (x - S.sbx0)];
}

}  // namespace

// =====================================================================================
// Forward pass (modelling / source wavefield).  Velocity update, optional strip save.
__global__ void __launch_bounds__(NTHR) k_vel_fwd(StepArgs a, int save)
{
    __shared__ float sp[VH * VW];
    __shared__ float s_coef[100];
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int x0 = (t.tile % S.ntx) * TX, z0 = (t.tile / S.ntx) * TZ;
    load_coef(s_coef, a.coef);
    stage(sp, S.a.p, S.pitch, S.X, S.Z, z0 - (R - 1), x0 - (R - 1), VH, VW);
    __syncthreads();
    vel_full(S, S.a, sp, s_coef, S.inv_rho_f, a.dtx, a.dtz, z0, x0, save != 0, a);
}

// Pressure update + source injection (+ receiver sampling, + strip save).
__global__ void __launch_bounds__(NTHR) k_pres_fwd(StepArgs a, int save, int record)
{
    __shared__ float svx[TZ * PXW];
    __shared__ float svz[PZH * TX];
    __shared__ float s_coef[100];
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int x0 = (t.tile % S.ntx) * TX, z0 = (t.tile / S.ntx) * TZ;
    load_coef(s_coef, a.coef);
    stage(svx, S.a.vx, S.pitch, S.X - 1, S.Z, z0, x0 - R, TZ, PXW);
    stage(svz, S.a.vz, S.pitch, S.X, S.Z - 1, z0 - R, x0, PZH, TX);
    __syncthreads();
    const float wit = a.wavelet[a.it];
    const int lx = threadIdx.x, x = x0 + lx;
#pragma unroll
    for (int k = 0; k < ROWS_PER_THR; k++) {
        const int lz = threadIdx.y + 8 * k, z = z0 + lz;
        if (z >= S.Z || x >= S.X) continue;
        const size_t id = (size_t)z * S.pitch + x;
        float p;
        bool upd = pres_full_cell(S, S.a, svx, svz, s_coef, S.kappa_f, a.dtx, a.dtz, z, x, lz, lx, p);
        if (!upd) p = S.a.p[id];
        if (in_src(S, z, x)) p += src_at(S, z, x) * wit;   // reference kernel.cu:36-47
        if (upd || in_src(S, z, x)) S.a.p[id] = p;
        if (record && z == S.rz && x >= S.rx0 && x < S.rx0 + S.nrec) {   // kernel.cu:48-71
            float *g = (float *)S.gather;
            g[(size_t)a.it * S.nrec + (x - S.rx0)] = p;
        }
        if (save) {
            long si = strip_idx_p(S, z, x);
            if (si >= 0) store_strip(a, S, si, p);
        }
    }
}

// =====================================================================================
// Backward pass: source reconstruction (wavefield a, interior only) and receiver
// propagation (wavefield b, full grid) in the same launches.
// Velocity: restore vx/vz strips of step it+1 into a; a += (dt/h)/rho * D(ps) (interior);
// b: full forward velocity update.  Reference rtm_model.cu:424-429, :440-443.
__global__ void __launch_bounds__(NTHR) k_vel_bwd(StepArgs a)
{
    __shared__ float sps[VH * VW];
    __shared__ float spr[VH * VW];
    __shared__ float s_coef[100];
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int x0 = (t.tile % S.ntx) * TX, z0 = (t.tile / S.ntx) * TZ;
    load_coef(s_coef, a.coef);
    stage(sps, S.a.p, S.pitch, S.X, S.Z, z0 - (R - 1), x0 - (R - 1), VH, VW);
    stage(spr, S.b.p, S.pitch, S.X, S.Z, z0 - (R - 1), x0 - (R - 1), VH, VW);
    __syncthreads();
    // receiver wavefield
    vel_full(S, S.b, spr, s_coef, S.inv_rho_b, a.dtx, a.dtz, z0, x0, false, a);
    // reconstruction
    const float *cf = &s_coef[(R - 1) * R];
    const int lx = threadIdx.x, x = x0 + lx;
    const int itn = a.it + 1;
    const size_t sbase = (size_t)itn * S.strip_len;
#pragma unroll
    for (int k = 0; k < ROWS_PER_THR; k++) {
        const int lz = threadIdx.y + 8 * k, z = z0 + lz;
        if (z >= S.Z || x >= S.X) continue;
        const size_t id = (size_t)z * S.pitch + x;
        const bool zin = (z >= S.npml && z < S.Z - S.npml);
        if (zin && x >= S.npml && x <= S.X - S.npml - 2) {   // kernel.cu:318-353
            float d = vx_diff(sps, cf, lz, lx);
            d = d * a.dtx * __ldg(&S.inv_rho_b[id]);
            S.a.vx[id] += d;
        } else {
            long si = strip_idx_vx(S, z, x);
            if (si >= 0) {   // read_d_vxpml, kernel.cu:1294-1320
                float sc = a.strip_prec ? S.strip_scale[(size_t)itn * 4 + 0] : 1.0f;
                S.a.vx[id] = load_strip(S.strips, sbase + si, a.strip_prec, sc);
            }
        }
        if (x >= S.npml && x < S.X - S.npml && z >= S.npml && z <= S.Z - S.npml - 2) {   // :354-388
            float d = vz_diff(sps, cf, lz, lx);
            d = d * a.dtz * __ldg(&S.inv_rho_b[id]);
            S.a.vz[id] += d;
        } else {
            long si = strip_idx_vz(S, z, x);
            if (si >= 0) {   // read_d_vzpml, kernel.cu:1321-1347
                float sc = a.strip_prec ? S.strip_scale[(size_t)itn * 4 + 1] : 1.0f;
                S.a.vz[id] = load_strip(S.strips, sbase + si, a.strip_prec, sc);
            }
        }
    }
}

// Pressure: restore p strips of step it into ps; ps += dt*rho*v^2 * D(v) (interior);
// ps -= dt*src*w[it]; receiver: full pressure update, overwrite the receiver row with
// dt*gather[it]; imaging g1 += ps*p, illum += ps*ps on the interior.
// Reference rtm_model.cu:431-452, kernel.cu:389-429, :72-95, :1401-1416.
__global__ void __launch_bounds__(NTHR) k_pres_bwd(StepArgs a)
{
    __shared__ float svxs[TZ * PXW];
    __shared__ float svzs[PZH * TX];
    __shared__ float svxr[TZ * PXW];
    __shared__ float svzr[PZH * TX];
    __shared__ float s_coef[100];
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int x0 = (t.tile % S.ntx) * TX, z0 = (t.tile / S.ntx) * TZ;
    load_coef(s_coef, a.coef);
    stage(svxs, S.a.vx, S.pitch, S.X - 1, S.Z, z0, x0 - R, TZ, PXW);
    stage(svzs, S.a.vz, S.pitch, S.X, S.Z - 1, z0 - R, x0, PZH, TX);
    stage(svxr, S.b.vx, S.pitch, S.X - 1, S.Z, z0, x0 - R, TZ, PXW);
    stage(svzr, S.b.vz, S.pitch, S.X, S.Z - 1, z0 - R, x0, PZH, TX);
    __syncthreads();
    const float wit = a.wavelet[a.it];
    const float *cf = &s_coef[(R - 1) * R];
    const size_t sbase = (size_t)a.it * S.strip_len;
    const int lx = threadIdx.x, x = x0 + lx;
#pragma unroll
    for (int k = 0; k < ROWS_PER_THR; k++) {
        const int lz = threadIdx.y + 8 * k, z = z0 + lz;
        if (z >= S.Z || x >= S.X) continue;
        const size_t id = (size_t)z * S.pitch + x;
        const bool interior = (z >= S.npml && z < S.Z - S.npml && x >= S.npml && x < S.X - S.npml);
        // --- reconstruction of the source wavefield
        float ps = S.a.p[id];
        bool wps = false;
        if (interior) {
            float dxs, dzs;
            p_diff(svxs, svzs, cf, lz, lx, dxs, dzs);
            const float kap = __ldg(&S.kappa_b[id]);
            dxs = dxs * a.dtx * kap;
            dzs = dzs * a.dtz * kap;
            ps += dxs + dzs;
            wps = true;
        } else {
            long si = strip_idx_p(S, z, x);
            if (si >= 0) {   // read_d_ppmllr / read_d_ppmltb, kernel.cu:1348-1400
                float sc = a.strip_prec ? S.strip_scale[(size_t)a.it * 4 + strip_kind(S, si)] : 1.0f;
                ps = load_strip(S.strips, sbase + si, a.strip_prec, sc);
                wps = true;
            }
        }
        if (in_src(S, z, x)) { ps -= src_at(S, z, x) * wit; wps = true; }
        if (wps) S.a.p[id] = ps;
        // --- receiver wavefield
        float p;
        bool upd = pres_full_cell(S, S.b, svxr, svzr, s_coef, S.kappa_b, a.dtx, a.dtz, z, x, lz, lx, p);
        if (z == S.rz && x >= S.rx0 && x < S.rx0 + S.nrec) {
            p = a.dt * load_gather(a, S, x - S.rx0);
            upd = true;
        }
        if (upd) S.b.p[id] = p;
        else p = S.b.p[id];
        // --- imaging
        if (interior) {
            size_t im = (size_t)(z - S.npml) * S.nxi + (x - S.npml);
            if (a.accum_fp64) {
                double *g1 = (double *)S.g1, *il = (double *)S.illum;
                g1[im] += (double)ps * (double)p;
                il[im] += (double)ps * (double)ps;
            } else {
                float *g1 = (float *)S.g1, *il = (float *)S.illum;
                g1[im] += ps * p;
                il[im] += ps * ps;
            }
        }
    }
}

// =====================================================================================
// Setup kernels (once per shot).

// PML profiles (reference kernel.cu:174-269) and the damping factors the stencil kernels
// use: c1 = 1 - dt*d/2, c2 = 2 - c1, evaluated in double as the reference does
// (kernel.cu:596-597).  Outside the bands c1 = c2 = 1.
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
            const bool bandp = (i < npml) || (i >= L - npml);
            const bool bandv = (i < npml) || (i >= L - npml - 1);
            if (axis == 0) {
                pml[o.ddx + i] = dp;
                pml[o.c1x + i] = bandp ? c1p : 1.0f;
                pml[o.c2x + i] = bandp ? c2p : 1.0f;
                if (i < L - 1) pml[o.ddxvx + i] = dv;
                pml[o.c1vx + i] = (bandv && i < L - 1) ? c1v : 1.0f;
                pml[o.c2vx + i] = (bandv && i < L - 1) ? c2v : 1.0f;
            } else {
                pml[o.ddz + i] = dp;
                pml[o.c1z + i] = bandp ? c1p : 1.0f;
                pml[o.c2z + i] = bandp ? c2p : 1.0f;
                if (i < L - 1) pml[o.ddzvz + i] = dv;
                pml[o.c1vz + i] = (bandv && i < L - 1) ? c1v : 1.0f;
                pml[o.c2vz + i] = (bandv && i < L - 1) ? c2v : 1.0f;
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
    // power-of-two scale so that |x|/scale <= 1 (exact scaling, only the rounding of the
    // narrow type remains)
    float scale = 1.0f;
    if (m > 0.0f) {
        int e;
        frexpf(m, &e);
        scale = ldexpf(1.0f, e);
    }
    const float inv = 1.0f / scale;
    const int it = it0 + step;
    if (threadIdx.x == 0) S.strip_scale[(size_t)it * 4 + kind] = scale;
    const size_t dst0 = (size_t)it * S.strip_len + off[kind];
    for (long i = threadIdx.x; i < len[kind]; i += blockDim.x) {
        float v = src[i] * inv;
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
    float sc = 1.0f;
    if (m > 0.0f) {
        int e;
        frexpf(m, &e);
        sc = ldexpf(1.0f, e);
    }
    if (threadIdx.x == 0) scale[it] = sc;
    const float inv = 1.0f / sc;
    for (int i = threadIdx.x; i < nrec; i += blockDim.x) {
        float v = row[i] * inv;
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
    const void *g1, *illum;
    int nx1, nxi, nwin;
};

__global__ void k_finalize(const FinalizeShot *fs, int nshots, int nx, int nz, int fp64, void *image1,
                           void *image2s, void *image2m, void *illum_total)
{
    const float alpha = 0.06f;
    const long n = (long)nx * nz;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int iz = (int)(i / nx), ix = (int)(i - (long)iz * nx);
        for (int s = 0; s < nshots; s++) {
            const FinalizeShot f = fs[s];
            const int lx = ix - f.nx1;
            if (lx < 0 || lx >= f.nxi) continue;
            const int nwin = f.nwin, nxl = f.nxi;
            float tp = 1.0f;
            if (lx < nwin) tp = expf(-alpha * alpha * (nwin - lx) * (nwin - lx));
            if (lx >= nxl - nwin && lx < nxl) tp = expf(-alpha * alpha * (lx - nxl + nwin + 1) * (lx - nxl + nwin + 1));
            if (lx >= nwin && lx < nxl - nwin) tp = 1.0f;
            const size_t ip = (size_t)iz * nxl + lx;
            if (fp64) {
                double g = ((const double *)f.g1)[ip] * (double)tp;
                double il = ((const double *)f.illum)[ip] * (double)tp;
                ((double *)image2s)[i] += g / (il + 1.0e-6);
                ((double *)image1)[i] += g;
                ((double *)image2m)[i] += g;
                ((double *)illum_total)[i] += il;
            } else {
                float g = ((const float *)f.g1)[ip] * tp;
                float il = ((const float *)f.illum)[ip] * tp;
                float *i2s = (float *)image2s;
                i2s[i] = i2s[i] + g / (il + 1.0e-6);
                ((float *)image1)[i] += g;
                ((float *)image2m)[i] += g;
                ((float *)illum_total)[i] += il;
            }
        }
    }
}

// Laplacian filter of a stacked image (reference laplacefd1d, image_function.cpp:44-79):
// integer dx, dz; second differences formed in double; border zeroed.
__global__ void k_laplace(const float *in, float *out, int nx, int nz, int dx, int dz)
{
    const long n = (long)nx * nz;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int iz = (int)(i / nx), ix = (int)(i - (long)iz * nx);
        if (ix == 0 || iz == 0 || ix == nx - 1 || iz == nz - 1) { out[i] = 0.0f; continue; }
        const float *r = &in[i];
        float t1 = (r[1] + r[-1] - 2.0 * r[0]) / (dx * dx);
        float t2 = (r[nx] + r[-nx] - 2.0 * r[0]) / (dz * dz);
        out[i] = t1 + t2;
    }
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

void launch_vel_fwd(const StepArgs &a, int ntiles, int save, cudaStream_t s)
{
    k_vel_fwd<<<ntiles, dim3(32, 8), 0, s>>>(a, save);
}
void launch_pres_fwd(const StepArgs &a, int ntiles, int save, int record, cudaStream_t s)
{
    k_pres_fwd<<<ntiles, dim3(32, 8), 0, s>>>(a, save, record);
}
void launch_vel_bwd(const StepArgs &a, int ntiles, cudaStream_t s)
{
    k_vel_bwd<<<ntiles, dim3(32, 8), 0, s>>>(a);
}
void launch_pres_bwd(const StepArgs &a, int ntiles, cudaStream_t s)
{
    k_pres_bwd<<<ntiles, dim3(32, 8), 0, s>>>(a);
}
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
                     void *illum, cudaStream_t s)
{
    long n = (long)nx * nz;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_finalize<<<blocks, 256, 0, s>>>((const FinalizeShot *)fs, nshots, nx, nz, fp64, image1, image2s, image2m, illum);
}
void launch_laplace(const float *in, float *out, int nx, int nz, int dx, int dz, cudaStream_t s)
{
    long n = (long)nx * nz;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_laplace<<<blocks, 256, 0, s>>>(in, out, nx, nz, dx, dz);
}
void launch_inject(const ShotDev *shots, int nshots, int maxrec, int it, float dt, int gather_prec, cudaStream_t s)
{
    dim3 grid((maxrec + 127) / 128, nshots);
    k_inject<<<grid, 128, 0, s>>>(shots, it, dt, gather_prec);
}
size_t finalize_shot_size() { return sizeof(FinalizeShot); }
void fill_finalize_shot(void *dst, const void *g1, const void *illum, int nx1, int nxi, int nwin)
{
    FinalizeShot f;
    f.g1 = g1;
    f.illum = illum;
    f.nx1 = nx1;
    f.nxi = nxi;
    f.nwin = nwin;
    *(FinalizeShot *)dst = f;
}
