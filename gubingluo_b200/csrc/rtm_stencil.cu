// rtm_stencil.cu — the time-step kernels of the RTM hot path (sm_100a).
//
// One launch updates one wavefield of every shot of a batch: a flat (shot, tile) work list
// maps each 128-thread block to a BX x BZ tile of one shot.  Each thread owns one grid
// column x and marches down the tile's BZ rows:
//   * the tile and its halo are staged once into shared memory with 16-byte cp.async copies
//     (zero-filled outside the grid), so every global access is a coalesced 128-byte row;
//   * x-derivatives read the staged row; z-derivatives read a 20-deep register queue that
//     the unrolled march rotates without moves (one shared load per row);
//   * the full-order coefficients come from the kernel-parameter constant bank; the reduced
//     local orders of the outer ten cells (reference cuda_norder*, kernel.cu:271-317) use
//     rows of the zero-padded coefficient table;
//   * PML damping, split pressure, source, receivers, strips and imaging are per-row or
//     per-column predicates of the same kernel.
// Reference equivalents (gubingluo kernel.cu): forward v :430-500 + :542-713, forward p
// :501-541 + :714-1185, reconstruction :318-429, strips :1186-1400, source :36-47,
// receivers :48-95, cross-correlation :1401-1416.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "rtm_launch.h"
#include "rtm_types.h"

namespace {

constexpr int BX = RTM_BX;         // threads (= columns) per block
constexpr int WW = BX + 24;        // staged width: columns x0-12 .. x0+BX+11 (16-byte aligned)
constexpr int R = RTM_RADIUS;
constexpr int QL = 20;             // register queue length (stencil taps along z)

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16(float *dst, const float *src, bool ok)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(ok ? 16 : 0));
}
__device__ __forceinline__ void cp_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// Rows [r0, r0+NR) and columns [c0, c0+NC) of field f into s[NR][NC]; c0 and NC are
// multiples of 4, rows outside [0, zrows) and columns outside [0, pitch) read as zero.
template <int NR, int NC>
__device__ __forceinline__ void stage(float *s, const float *__restrict__ f, int pitch, int zrows, int r0, int c0)
{
    constexpr int N4 = NC / 4;
    for (int i = threadIdx.x; i < NR * N4; i += BX) {
        const int r = i / N4, c = (i - r * N4) * 4;
        const int z = r0 + r, x = c0 + c;
        const bool ok = (unsigned)z < (unsigned)zrows && (unsigned)x < (unsigned)pitch;
        cp16(&s[r * NC + c], ok ? f + (size_t)z * pitch + x : f, ok);
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
    if (a.strip_prec == RTM_FP32) ((float *)S.strips)[(size_t)a.it * S.strip_len + idx] = v;
    else S.strip_stage[(size_t)a.ring * S.strip_len + idx] = v;
}

__device__ __forceinline__ float gather_at(const StepArgs &a, const ShotDev &S, int j)
{
    const size_t idx = (size_t)a.it * S.nrec + j;
    if (a.gather_prec == RTM_FP16) return __half2float(((const __half *)S.gather)[idx]) * S.gather_scale[a.it];
    if (a.gather_prec == RTM_BF16) return __bfloat162float(((const __nv_bfloat16 *)S.gather)[idx]) * S.gather_scale[a.it];
    return ((const float *)S.gather)[idx];
}

// Strip layout per step (reference save_d_*): [vx lr 2][nzi][10] [vz tb 2][10][nxi]
// [p lr 2][nzi][10] [p tb 2][10][nxi].
// Column part of the vx strip index for column x (-1: not a strip column).
__device__ __forceinline__ int strip_col_vx(int x, int X, int npml, int nzi)
{
    if (x >= npml - R && x < npml) return x - (npml - R);
    const int xr = X - npml - 1;
    if (x >= xr && x < xr + R) return R * nzi + (x - xr);
    return -1;
}
__device__ __forceinline__ int strip_col_plr(int x, int X, int npml, int nzi)
{
    if (x >= npml - R && x < npml) return x - (npml - R);
    const int xr = X - npml;
    if (x >= xr && x < xr + R) return R * nzi + (x - xr);
    return -1;
}
// Row part of the vz / p-top-bottom strip index for row z (-1: not a strip row); `first`
// is the first row of the bottom strip (Z-npml-1 for vz, Z-npml for p).
__device__ __forceinline__ int strip_row_tb(int z, int npml, int first, int nxi)
{
    if (z >= npml - R && z < npml) return (z - (npml - R)) * nxi;
    if (z >= first && z < first + R) return R * nxi + (z - first) * nxi;
    return -1;
}

}  // namespace

// =====================================================================================
// Velocity update.  MODE 0: forward, full grid; 1: forward + strip save; 2: receiver
// (backward model), full grid; 3: reconstruction of the source wavefield (interior only,
// vx/vz strips of step it+1 restored).
template <int BZ, int MODE>
__global__ void __launch_bounds__(BX) k_vel(const StepArgs a)
{
    constexpr int WH = BZ + 19;   // staged rows z0-9 .. z0+BZ+9
    extern __shared__ __align__(16) float sw[];
    __shared__ float s_tab[100];
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = (t.tile % S.ntx) * BX, z0 = (t.tile / S.ntx) * BZ;
    if (MODE == 3 && (z0 + BZ <= npml - R || z0 >= Z - npml + R || x0 + BX <= npml - R || x0 >= X - npml + R))
        return;   // tile outside the reconstruction region (interior + strips)
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ inv_rho = (MODE >= 2) ? S.inv_rho_b : S.inv_rho_f;
    stage<WH, WW>(sw, W.p, pitch, Z, z0 - 9, x0 - 12);
    if (threadIdx.x < 100) s_tab[threadIdx.x] = a.coef[threadIdx.x];
    cp_wait_all();
    __syncthreads();
    const int tx = threadIdx.x, x = x0 + tx;
    if (x >= X) return;   // no barrier below

    const PmlOffsets o = pml_offsets(X, Z);
    const int nzi = S.nzi, nxi = S.nxi;
    // per-column constants: vx order, coefficients and damping
    const bool has_vx = x < X - 1;
    const int rx = max(min(min(x + 1, X - 1 - x), R), 1);
    float cx[R];
#pragma unroll
    for (int i = 0; i < R; i++) cx[i] = (rx == R) ? a.c10[i] : s_tab[(rx - 1) * R + i];
    const bool bandvx = (x < npml) || (x >= X - npml - 1);
    const float c1vx = bandvx ? S.pml[o.c1vx + x] : 1.0f;
    const float ic2vx = bandvx ? S.pml[o.ic2vx + x] : 1.0f;
    const int svx_col = strip_col_vx(x, X, npml, nzi);
    const int svz_col = (x >= npml && x < X - npml) ? x - npml : -1;
    const bool rec_vx_col = (x >= npml && x <= X - npml - 2);
    const bool rec_vz_col = (x >= npml && x < X - npml);
    const size_t vstrip = 2 * (size_t)R * nzi;   // offset of the vz strips
    const size_t sbase_next = (size_t)(a.it + 1) * S.strip_len;

    float q[QL];   // q[(u + k) % QL] = p[z - 9 + k][x]
#pragma unroll
    for (int k = 0; k < QL - 1; k++) q[k] = sw[k * WW + tx + 12];

    const int zend = min(z0 + BZ, Z);
    for (int zb = z0; zb < zend; zb += QL) {
#pragma unroll
        for (int u = 0; u < QL; u++) {
            const int z = zb + u;
            if (z >= zend) break;
            q[(u + QL - 1) % QL] = sw[(z - z0 + 19) * WW + tx + 12];
            const float *row = &sw[(z - z0 + 9) * WW + tx + 12];
            const size_t id = (size_t)z * pitch + x;
            // ---------------- vx
            if (MODE == 3) {
                const bool zin = (z >= npml && z < Z - npml);
                if (zin && rec_vx_col) {   // kernel.cu:318-353 (vx += ...)
                    float d = 0.0f;
#pragma unroll
                    for (int i = 1; i <= R; i++) d += a.c10[i - 1] * (row[i] - row[1 - i]);
                    d = d * a.dtx * __ldg(&inv_rho[id]);
                    W.vx[id] += d;
                } else if (zin && svx_col >= 0) {   // read_d_vxpml, kernel.cu:1294-1320
                    const float sc = a.strip_prec ? S.strip_scale[(size_t)(a.it + 1) * 4 + 0] : 1.0f;
                    W.vx[id] = load_strip(S.strips, sbase_next + svx_col + (size_t)(z - npml) * R, a.strip_prec, sc);
                }
            } else if (has_vx) {
                float d = 0.0f;
#pragma unroll
                for (int i = 1; i <= R; i++) d += cx[i - 1] * (row[i] - row[1 - i]);
                d = d * a.dtx * __ldg(&inv_rho[id]);
                float v = W.vx[id];
                v = bandvx ? (c1vx * v - d) * ic2vx : v - d;
                W.vx[id] = v;
                if (MODE == 1 && svx_col >= 0 && z >= npml && z < Z - npml)
                    store_strip(a, S, svx_col + (size_t)(z - npml) * R, v);
            }
            // ---------------- vz
            if (z < Z - 1) {
                if (MODE == 3) {
                    if (rec_vz_col && z >= npml && z <= Z - npml - 2) {   // kernel.cu:354-388
                        float d = 0.0f;
#pragma unroll
                        for (int i = 1; i <= R; i++) d += a.c10[i - 1] * (q[(u + 9 + i) % QL] - q[(u + 10 - i) % QL]);
                        d = d * a.dtz * __ldg(&inv_rho[id]);
                        W.vz[id] += d;
                    } else if (svz_col >= 0) {
                        const int srow = strip_row_tb(z, npml, Z - npml - 1, nxi);
                        if (srow >= 0) {   // read_d_vzpml, kernel.cu:1321-1347
                            const float sc = a.strip_prec ? S.strip_scale[(size_t)(a.it + 1) * 4 + 1] : 1.0f;
                            W.vz[id] = load_strip(S.strips, sbase_next + vstrip + srow + svz_col, a.strip_prec, sc);
                        }
                    }
                } else {
                    const int rz = min(min(z + 1, Z - 1 - z), R);
                    float d = 0.0f;
                    if (rz == R) {
#pragma unroll
                        for (int i = 1; i <= R; i++) d += a.c10[i - 1] * (q[(u + 9 + i) % QL] - q[(u + 10 - i) % QL]);
                    } else {
                        const float *c = &s_tab[(rz - 1) * R];
#pragma unroll
                        for (int i = 1; i <= R; i++) d += c[i - 1] * (q[(u + 9 + i) % QL] - q[(u + 10 - i) % QL]);
                    }
                    d = d * a.dtz * __ldg(&inv_rho[id]);
                    float v = W.vz[id];
                    const bool bandvz = (z < npml) || (z >= Z - npml - 1);
                    if (bandvz) v = (S.pml[o.c1vz + z] * v - d) * S.pml[o.ic2vz + z];
                    else v = v - d;
                    W.vz[id] = v;
                    if (MODE == 1 && svz_col >= 0) {
                        const int srow = strip_row_tb(z, npml, Z - npml - 1, nxi);
                        if (srow >= 0) store_strip(a, S, vstrip + srow + svz_col, v);
                    }
                }
            }
        }
    }
}

// =====================================================================================
// Pressure update.  MODE 0: forward (+ source, + receiver sampling when `record`);
// 1: forward + strip save; 2: receiver (backward model): overwrite the receiver row with
// dt*gather[it], then image g1 += ps*p, illum += ps*ps; 3: reconstruction (interior, p
// strips of step it restored, source subtracted).
template <int BZ, int MODE>
__global__ void __launch_bounds__(BX) k_pres(const StepArgs a, int record)
{
    constexpr int XH = BZ;        // vx rows z0 .. z0+BZ-1, columns x0-12 .. x0+BX+11
    constexpr int ZH = BZ + 20;   // vz rows z0-10 .. z0+BZ+9, columns x0 .. x0+BX-1
    extern __shared__ __align__(16) float sm[];
    float *svx = sm;
    float *svz = sm + XH * WW;
    __shared__ float s_tab[100];
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = (t.tile % S.ntx) * BX, z0 = (t.tile / S.ntx) * BZ;
    if (MODE == 3 && (z0 + BZ <= npml - R || z0 >= Z - npml + R || x0 + BX <= npml - R || x0 >= X - npml + R))
        return;
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ kappa = (MODE >= 2) ? S.kappa_b : S.kappa_f;
    stage<XH, WW>(svx, W.vx, pitch, Z, z0, x0 - 12);
    stage<ZH, BX>(svz, W.vz, pitch, Z, z0 - 10, x0);
    if (threadIdx.x < 100) s_tab[threadIdx.x] = a.coef[threadIdx.x];
    cp_wait_all();
    __syncthreads();
    const int tx = threadIdx.x, x = x0 + tx;
    if (x >= X) return;

    const PmlOffsets o = pml_offsets(X, Z);
    const int nzi = S.nzi, nxi = S.nxi;
    const int rpx = max(min(min(x, X - 1 - x), R), 1);
    float cp[R];
#pragma unroll
    for (int i = 0; i < R; i++) cp[i] = (rpx == R) ? a.c10[i] : s_tab[(rpx - 1) * R + i];
    const bool xedge = (x < 1) || (x > X - 2);
    const bool xb = (x < npml) || (x >= X - npml);
    const float c1x = xb ? S.pml[o.c1x + x] : 1.0f;
    const float ic2x = xb ? S.pml[o.ic2x + x] : 1.0f;
    const bool in_src_col = (unsigned)(x - S.sbx0) < (unsigned)S.sbnx;
    const bool rec_col = (x >= S.rx0) && (x < S.rx0 + S.nrec);
    const int splr_col = strip_col_plr(x, X, npml, nzi);
    const int sptb_col = (x >= npml && x < X - npml) ? x - npml : -1;
    const size_t pstrip = 2 * (size_t)R * nzi + 2 * (size_t)R * nxi;   // offset of the p strips
    const size_t ptb = pstrip + 2 * (size_t)R * nzi;
    const bool xin = (x >= npml && x < X - npml);
    const float wit = a.wavelet[a.it];

    float q[QL];   // q[(u + k) % QL] = vz[z - 10 + k][x]
#pragma unroll
    for (int k = 0; k < QL - 1; k++) q[k] = svz[k * BX + tx];

    const int zend = min(z0 + BZ, Z);
    for (int zb = z0; zb < zend; zb += QL) {
#pragma unroll
        for (int u = 0; u < QL; u++) {
            const int z = zb + u;
            if (z >= zend) break;
            q[(u + QL - 1) % QL] = svz[(z - z0 + 19) * BX + tx];
            const float *row = &svx[(z - z0) * WW + tx + 12];
            const size_t id = (size_t)z * pitch + x;
            const bool zin = (z >= npml && z < Z - npml);
            if (MODE == 3) {
                // ---------------- reconstruction of the source pressure
                bool wr = false;
                float ps = 0.0f;
                if (zin && xin) {   // kernel.cu:389-429 (p += ...)
                    float dxs = 0.0f, dzs = 0.0f;
#pragma unroll
                    for (int i = 1; i <= R; i++) {
                        dxs += a.c10[i - 1] * (row[i - 1] - row[-i]);
                        dzs += a.c10[i - 1] * (q[(u + 9 + i) % QL] - q[(u + 10 - i) % QL]);
                    }
                    const float kap = __ldg(&kappa[id]);
                    dxs = dxs * a.dtx * kap;
                    dzs = dzs * a.dtz * kap;
                    ps = W.p[id] + (dxs + dzs);
                    wr = true;
                } else {   // read_d_ppmllr / read_d_ppmltb (step it), kernel.cu:1348-1400
                    long si = -1;
                    int kind = 2;
                    if (zin && splr_col >= 0) si = (long)(pstrip + splr_col + (size_t)(z - npml) * R);
                    else if (sptb_col >= 0) {
                        const int srow = strip_row_tb(z, npml, Z - npml, nxi);
                        if (srow >= 0) { si = (long)(ptb + srow + sptb_col); kind = 3; }
                    }
                    if (si >= 0) {
                        const float sc = a.strip_prec ? S.strip_scale[(size_t)a.it * 4 + kind] : 1.0f;
                        ps = load_strip(S.strips, (size_t)a.it * S.strip_len + si, a.strip_prec, sc);
                        wr = true;
                    }
                }
                if (in_src_col && (unsigned)(z - S.sbz0) < (unsigned)S.sbnz) {   // kernel.cu:36-47 (subtract)
                    if (!wr) ps = W.p[id];
                    ps -= S.src[(z - S.sbz0) * S.sbnx + (x - S.sbx0)] * wit;
                    wr = true;
                }
                if (wr) W.p[id] = ps;
                continue;
            }
            // ---------------- full-grid pressure update with split-field PML
            const bool zedge = (z < 1) || (z > Z - 2);
            float p;
            bool wr = false;
            if (!xedge && !zedge) {
                const int rpz = min(min(z, Z - 1 - z), R);
                float dxs = 0.0f, dzs = 0.0f;
                if (rpz == R) {
#pragma unroll
                    for (int i = 1; i <= R; i++) {
                        dxs += cp[i - 1] * (row[i - 1] - row[-i]);
                        dzs += cp[i - 1] * (q[(u + 9 + i) % QL] - q[(u + 10 - i) % QL]);
                    }
                } else {
                    const float *c = &s_tab[(min(rpx, rpz) - 1) * R];
#pragma unroll
                    for (int i = 1; i <= R; i++) {
                        dxs += c[i - 1] * (row[i - 1] - row[-i]);
                        dzs += c[i - 1] * (q[(u + 9 + i) % QL] - q[(u + 10 - i) % QL]);
                    }
                }
                const float kap = __ldg(&kappa[id]);
                dxs = dxs * a.dtx * kap;
                dzs = dzs * a.dtz * kap;
                const bool zb_ = !zin;
                if (!xb && !zb_) {
                    p = W.p[id] - (dxs + dzs);
                } else {
                    float s1 = W.sx[id], s2 = W.sz[id];
                    s1 = xb ? (c1x * s1 - dxs) * ic2x : s1 - dxs;
                    s2 = zb_ ? (S.pml[o.c1z + z] * s2 - dzs) * S.pml[o.ic2z + z] : s2 - dzs;
                    W.sx[id] = s1;
                    W.sz[id] = s2;
                    p = s1 + s2;
                }
                wr = true;
            }
            if (MODE != 2) {
                if (in_src_col && (unsigned)(z - S.sbz0) < (unsigned)S.sbnz) {   // kernel.cu:36-47 (add)
                    if (!wr) p = W.p[id];
                    p += S.src[(z - S.sbz0) * S.sbnx + (x - S.sbx0)] * wit;
                    wr = true;
                }
                if (wr) W.p[id] = p;
                if (record && z == S.rz && rec_col)   // kernel.cu:48-71
                    ((float *)S.gather)[(size_t)a.it * S.nrec + (x - S.rx0)] = p;
                if (MODE == 1) {
                    if (zin && splr_col >= 0) {
                        store_strip(a, S, pstrip + splr_col + (size_t)(z - npml) * R, wr ? p : W.p[id]);
                    } else if (sptb_col >= 0) {
                        const int srow = strip_row_tb(z, npml, Z - npml, nxi);
                        if (srow >= 0) store_strip(a, S, ptb + srow + sptb_col, wr ? p : W.p[id]);
                    }
                }
            } else {
                if (z == S.rz && rec_col) {   // kernel.cu:72-95 (overwrite)
                    p = a.dt * gather_at(a, S, x - S.rx0);
                    wr = true;
                }
                if (wr) W.p[id] = p;
                if (zin && xin) {   // kernel.cu:1401-1416
                    if (!wr) p = W.p[id];
                    const float ps = S.a.p[id];
                    const size_t im = (size_t)(z - npml) * nxi + (x - npml);
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
    }
}

// =====================================================================================
// Host launchers.
template <int BZ>
static size_t vel_smem() { return (size_t)(BZ + 19) * WW * sizeof(float); }
template <int BZ>
static size_t pres_smem() { return ((size_t)BZ * WW + (size_t)(BZ + 20) * BX) * sizeof(float); }

template <int BZ, int MODE>
static void vel_launch(const StepArgs &a, int ntiles, cudaStream_t s)
{
    static bool init = false;
    if (!init) {
        cudaFuncSetAttribute(k_vel<BZ, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vel_smem<BZ>());
        init = true;
    }
    k_vel<BZ, MODE><<<ntiles, BX, vel_smem<BZ>(), s>>>(a);
}
template <int BZ, int MODE>
static void pres_launch(const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    static bool init = false;
    if (!init) {
        cudaFuncSetAttribute(k_pres<BZ, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pres_smem<BZ>());
        init = true;
    }
    k_pres<BZ, MODE><<<ntiles, BX, pres_smem<BZ>(), s>>>(a, record);
}

template <int MODE>
static void vel_dispatch(int bz, const StepArgs &a, int ntiles, cudaStream_t s)
{
    if (bz == 16) vel_launch<16, MODE>(a, ntiles, s);
    else if (bz == 64) vel_launch<64, MODE>(a, ntiles, s);
    else vel_launch<32, MODE>(a, ntiles, s);
}
template <int MODE>
static void pres_dispatch(int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if (bz == 16) pres_launch<16, MODE>(a, ntiles, record, s);
    else if (bz == 64) pres_launch<64, MODE>(a, ntiles, record, s);
    else pres_launch<32, MODE>(a, ntiles, record, s);
}

void launch_vel(int mode, int bz, const StepArgs &a, int ntiles, cudaStream_t s)
{
    switch (mode) {
    case RTM_WAVE_FWD: vel_dispatch<0>(bz, a, ntiles, s); break;
    case RTM_WAVE_FWD_SAVE: vel_dispatch<1>(bz, a, ntiles, s); break;
    case RTM_WAVE_RECEIVER: vel_dispatch<2>(bz, a, ntiles, s); break;
    default: vel_dispatch<3>(bz, a, ntiles, s); break;
    }
}
void launch_pres(int mode, int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    switch (mode) {
    case RTM_WAVE_FWD: pres_dispatch<0>(bz, a, ntiles, record, s); break;
    case RTM_WAVE_FWD_SAVE: pres_dispatch<1>(bz, a, ntiles, record, s); break;
    case RTM_WAVE_RECEIVER: pres_dispatch<2>(bz, a, ntiles, 0, s); break;
    default: pres_dispatch<3>(bz, a, ntiles, 0, s); break;
    }
}
