// rtm_stencil.cu — the time-step kernels of the RTM hot path (sm_100a).
//
// One launch updates one wavefield of every shot of a batch: a flat (shot, tile) work list
// maps each 64-thread block to a BX x BZ tile (128 columns) of one shot.  Each thread owns
// two adjacent grid columns and marches down the tile's BZ rows:
//   * the tile and its halo are staged once into shared memory with 16-byte cp.async copies
//     (zero-filled outside the grid), so every global access is a coalesced row segment;
//   * x-derivatives of both columns read 11 8-byte shared words of the staged row;
//     z-derivatives read two 20-deep register queues that the unrolled march rotates without
//     moves (one 8-byte shared load per row);
//   * the per-cell operands of the next row are loaded before the current row is stored;
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

constexpr int BX = RTM_BX;         // columns per tile
constexpr int NT = BX / 2;         // threads per block (two adjacent columns each)
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
    for (int i = threadIdx.x; i < NR * N4; i += NT) {
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

// Damped or undamped update f' = (c1*f - d)*ic2; outside the PML c1 = ic2 = 1, which makes
// this exactly f - d.
__device__ __forceinline__ float damp(float f, float d, float c1, float ic2) { return (c1 * f - d) * ic2; }

__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float a, float b, bool va, bool vb)
{
    if (va && vb) *reinterpret_cast<float2 *>(p) = make_float2(a, b);
    else {
        if (va) p[0] = a;
        if (vb) p[1] = b;
    }
}

}  // namespace

// =====================================================================================
// Velocity update.  MODE 0: forward, full grid; 1: forward + strip save; 2: receiver
// (backward model), full grid; 3: reconstruction of the source wavefield (interior only,
// vx/vz strips of step it+1 restored).
template <int BZ, int MODE>
__global__ void __launch_bounds__(NT) k_vel(const StepArgs a)
{
    constexpr int WH = BZ + 19;   // staged rows z0-9 .. z0+BZ+9
    extern __shared__ __align__(16) float sw[];
    __shared__ float s_tab[100];
    __shared__ float s_c1vz[BZ], s_ic2vz[BZ];
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = (t.tile % S.ntx) * BX, z0 = (t.tile / S.ntx) * BZ;
    if (MODE == 3 && (z0 + BZ <= npml - R || z0 >= Z - npml + R || x0 + BX <= npml - R || x0 >= X - npml + R))
        return;   // tile outside the reconstruction region (interior + strips)
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ inv_rho = (MODE >= 2) ? S.inv_rho_b : S.inv_rho_f;
    const PmlOffsets o = pml_offsets(X, Z);
    stage<WH, WW>(sw, W.p, pitch, Z, z0 - 9, x0 - 12);
    for (int i = threadIdx.x; i < 100; i += NT) s_tab[i] = a.coef[i];
    for (int i = threadIdx.x; i < BZ; i += NT) {
        const int z = min(z0 + i, Z - 2);
        s_c1vz[i] = S.pml[o.c1vz + z];
        s_ic2vz[i] = S.pml[o.ic2vz + z];
    }
    cp_wait_all();
    __syncthreads();
    const int tx = threadIdx.x, xa = x0 + 2 * tx;   // columns xa, xa+1
    if (xa >= X) return;   // no barrier below

    const int nzi = S.nzi, nxi = S.nxi;
    float *__restrict__ vxp = W.vx;
    float *__restrict__ vzp = W.vz;
    // per-column constants
    bool hvx[2], hvz[2], rvx[2], rvz[2];
    float c1vx[2], ic2vx[2];
    int svx[2], svz[2];
    bool edge_order = false;
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int x = xa + c;
        hvz[c] = x < X;
        hvx[c] = x < X - 1;
        edge_order |= hvx[c] && (x < R - 1 || x > X - R - 1);
        const bool band = (x < npml) || (x >= X - npml - 1);
        c1vx[c] = (band && hvx[c]) ? S.pml[o.c1vx + x] : 1.0f;
        ic2vx[c] = (band && hvx[c]) ? S.pml[o.ic2vx + x] : 1.0f;
        svx[c] = hvx[c] ? strip_col_vx(x, X, npml, nzi) : -1;
        svz[c] = (x >= npml && x < X - npml) ? x - npml : -1;
        rvx[c] = (x >= npml && x <= X - npml - 2);
        rvz[c] = (x >= npml && x < X - npml);
    }
    // vx coefficient rows of the two columns (the reduced orders of the outer ten columns)
    const float *cx0 = &s_tab[(max(min(min(xa + 1, X - 1 - xa), R), 1) - 1) * R];
    const float *cx1 = &s_tab[(max(min(min(xa + 2, X - 2 - xa), R), 1) - 1) * R];
    const size_t vstrip = 2 * (size_t)R * nzi;
    const size_t sbase_next = (size_t)(a.it + 1) * S.strip_len;
    const float dtx = a.dtx, dtz = a.dtz;

    float qa[QL], qb[QL];   // q?[(u + k) % QL] = p[z - 9 + k][xa (+1)]
#pragma unroll
    for (int k = 0; k < QL - 1; k++) {
        const float2 f = ld2(&sw[k * WW + 2 * tx + 12]);
        qa[k] = f.x;
        qb[k] = f.y;
    }
    const int zend = min(z0 + BZ, Z);
    // operands of the next PF rows (1/rho, vx, vz of both columns): the loads of row z+PF are
    // issued while row z is computed, so each warp keeps PF rows of loads in flight
    constexpr int PF = 4;   // divides QL, so the slot of row z is the compile-time u % PF
    float2 n_ir[PF], n_vx[PF], n_vz[PF];
    auto load_row = [&](int z, int slot) {
        const unsigned id = (unsigned)z * pitch + xa;
        n_ir[slot] = __ldg(reinterpret_cast<const float2 *>(&inv_rho[id]));
        n_vx[slot] = ld2(&vxp[id]);
        n_vz[slot] = ld2(&vzp[id]);
    };
#pragma unroll
    for (int k = 0; k < PF; k++)
        if (z0 + k < zend) load_row(z0 + k, k);
    for (int zb = z0; zb < zend; zb += QL) {
#pragma unroll
        for (int u = 0; u < QL; u++) {
            const int z = zb + u;
            if (z >= zend) break;
            const int slot = u % PF;
            const float2 ir = n_ir[slot], ov = n_vx[slot], ow = n_vz[slot];
            if (z + PF < zend) load_row(z + PF, slot);
            {
                const float2 f = ld2(&sw[(z - z0 + 19) * WW + 2 * tx + 12]);
                qa[(u + QL - 1) % QL] = f.x;
                qb[(u + QL - 1) % QL] = f.y;
            }
            // v[k] = p[z][xa - 10 + k], k = 0..21
            float v[22];
            const float *rw = &sw[(z - z0 + 9) * WW + 2 * tx + 2];
#pragma unroll
            for (int j = 0; j < 11; j++) {
                const float2 f = ld2(&rw[2 * j]);
                v[2 * j] = f.x;
                v[2 * j + 1] = f.y;
            }
            float dx0 = 0.f, dx1 = 0.f, dz0 = 0.f, dz1 = 0.f;
            if (!edge_order) {
#pragma unroll
                for (int i = 1; i <= R; i++) {
                    dx0 += a.c10[i - 1] * (v[10 + i] - v[11 - i]);
                    dx1 += a.c10[i - 1] * (v[11 + i] - v[12 - i]);
                }
            } else {   // outer ten columns: local order (kernel.cu:542-630 with cuda_norderx)
#pragma unroll
                for (int i = 1; i <= R; i++) {
                    dx0 += cx0[i - 1] * (v[10 + i] - v[11 - i]);
                    dx1 += cx1[i - 1] * (v[11 + i] - v[12 - i]);
                }
            }
            const int rz = min(min(z + 1, Z - 1 - z), R);
            if (MODE == 3 || rz == R) {
#pragma unroll
                for (int i = 1; i <= R; i++) {
                    dz0 += a.c10[i - 1] * (qa[(u + 9 + i) % QL] - qa[(u + 10 - i) % QL]);
                    dz1 += a.c10[i - 1] * (qb[(u + 9 + i) % QL] - qb[(u + 10 - i) % QL]);
                }
            } else {   // top/bottom ten rows: local order (cuda_norderz)
                const float *cz = &s_tab[(rz - 1) * R];
#pragma unroll
                for (int i = 1; i <= R; i++) {
                    dz0 += cz[i - 1] * (qa[(u + 9 + i) % QL] - qa[(u + 10 - i) % QL]);
                    dz1 += cz[i - 1] * (qb[(u + 9 + i) % QL] - qb[(u + 10 - i) % QL]);
                }
            }
            const unsigned id = (unsigned)z * pitch + xa;
            if (MODE == 3) {
                // kernel.cu:318-388 (+=) on the interior; strips of step it+1 elsewhere
                const bool zin = (z >= npml && z < Z - npml);
                const bool zinv = (z >= npml && z <= Z - npml - 2);
                float nvx[2] = {ov.x, ov.y}, nvz[2] = {ow.x, ow.y};
                bool wvx[2] = {false, false}, wvz[2] = {false, false};
                const float ddx[2] = {dx0, dx1}, ddz[2] = {dz0, dz1}, irr[2] = {ir.x, ir.y};
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    if (zin && rvx[c]) {
                        nvx[c] += ddx[c] * dtx * irr[c];
                        wvx[c] = true;
                    } else if (zin && svx[c] >= 0) {   // read_d_vxpml, kernel.cu:1294-1320
                        const float sc = a.strip_prec ? S.strip_scale[(size_t)(a.it + 1) * 4 + 0] : 1.0f;
                        nvx[c] = load_strip(S.strips, sbase_next + svx[c] + (size_t)(z - npml) * R, a.strip_prec, sc);
                        wvx[c] = true;
                    }
                    if (zinv && rvz[c]) {
                        nvz[c] += ddz[c] * dtz * irr[c];
                        wvz[c] = true;
                    } else if (svz[c] >= 0 && z < Z - 1) {   // read_d_vzpml, kernel.cu:1321-1347
                        const int srow = strip_row_tb(z, npml, Z - npml - 1, nxi);
                        if (srow >= 0) {
                            const float sc = a.strip_prec ? S.strip_scale[(size_t)(a.it + 1) * 4 + 1] : 1.0f;
                            nvz[c] = load_strip(S.strips, sbase_next + vstrip + srow + svz[c], a.strip_prec, sc);
                            wvz[c] = true;
                        }
                    }
                }
                st2(&vxp[id], nvx[0], nvx[1], wvx[0], wvx[1]);
                st2(&vzp[id], nvz[0], nvz[1], wvz[0], wvz[1]);
                continue;
            }
            // kernel.cu:430-500 (interior) and :542-713 (PML): f' = (c1*f - d)*ic2
            const float nvx0 = damp(ov.x, dx0 * dtx * ir.x, c1vx[0], ic2vx[0]);
            const float nvx1 = damp(ov.y, dx1 * dtx * ir.y, c1vx[1], ic2vx[1]);
            st2(&vxp[id], nvx0, nvx1, hvx[0], hvx[1]);
            const bool zv = z < Z - 1;
            const float c1z = s_c1vz[z - z0], ic2z = s_ic2vz[z - z0];
            const float nvz0 = damp(ow.x, dz0 * dtz * ir.x, c1z, ic2z);
            const float nvz1 = damp(ow.y, dz1 * dtz * ir.y, c1z, ic2z);
            st2(&vzp[id], nvz0, nvz1, zv && hvz[0], zv && hvz[1]);
            if (MODE == 1) {   // save_d_vxpml / save_d_vzpml, kernel.cu:1186-1239
                if (z >= npml && z < Z - npml) {
                    if (svx[0] >= 0) store_strip(a, S, svx[0] + (size_t)(z - npml) * R, nvx0);
                    if (svx[1] >= 0) store_strip(a, S, svx[1] + (size_t)(z - npml) * R, nvx1);
                }
                const int srow = strip_row_tb(z, npml, Z - npml - 1, nxi);
                if (srow >= 0 && zv) {
                    if (svz[0] >= 0) store_strip(a, S, vstrip + srow + svz[0], nvz0);
                    if (svz[1] >= 0) store_strip(a, S, vstrip + srow + svz[1], nvz1);
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
template <int BZ, int MODE, typename ACC>
__global__ void __launch_bounds__(NT) k_pres(const StepArgs a, int record)
{
    constexpr int XH = BZ;        // vx rows z0 .. z0+BZ-1, columns x0-12 .. x0+BX+11
    constexpr int ZH = BZ + 20;   // vz rows z0-10 .. z0+BZ+9, columns x0 .. x0+BX-1
    extern __shared__ __align__(16) float sm[];
    float *svx = sm;
    float *svz = sm + XH * WW;
    __shared__ float s_tab[100];
    __shared__ float s_c1z[BZ], s_ic2z[BZ];
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = (t.tile % S.ntx) * BX, z0 = (t.tile / S.ntx) * BZ;
    if (MODE == 3 && (z0 + BZ <= npml - R || z0 >= Z - npml + R || x0 + BX <= npml - R || x0 >= X - npml + R))
        return;
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ kappa = (MODE >= 2) ? S.kappa_b : S.kappa_f;
    const PmlOffsets o = pml_offsets(X, Z);
    stage<XH, WW>(svx, W.vx, pitch, Z, z0, x0 - 12);
    stage<ZH, BX>(svz, W.vz, pitch, Z, z0 - 10, x0);
    for (int i = threadIdx.x; i < 100; i += NT) s_tab[i] = a.coef[i];
    for (int i = threadIdx.x; i < BZ; i += NT) {
        const int z = min(z0 + i, Z - 1);
        s_c1z[i] = S.pml[o.c1z + z];
        s_ic2z[i] = S.pml[o.ic2z + z];
    }
    cp_wait_all();
    __syncthreads();
    const int tx = threadIdx.x, xa = x0 + 2 * tx;
    if (xa >= X) return;

    const int nzi = S.nzi, nxi = S.nxi;
    float *__restrict__ pp = W.p;
    float *__restrict__ sxp = W.sx;
    float *__restrict__ szp = W.sz;
    const float *__restrict__ psp = S.a.p;
    ACC *__restrict__ g1p = (ACC *)S.g1;
    ACC *__restrict__ ilp = (ACC *)S.illum;
    // per-column constants
    bool upd[2], xb[2], xin[2], srcc[2], recc[2], valid[2];
    float c1x[2], ic2x[2];
    int splr[2], sptb[2];
    bool edge_order = false;
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int x = xa + c;
        valid[c] = x < X;
        upd[c] = x >= 1 && x <= X - 2;
        edge_order |= upd[c] && (x < R || x > X - 1 - R);
        xb[c] = (x < npml) || (x >= X - npml);
        xin[c] = valid[c] && !xb[c];
        c1x[c] = (xb[c] && valid[c]) ? S.pml[o.c1x + x] : 1.0f;
        ic2x[c] = (xb[c] && valid[c]) ? S.pml[o.ic2x + x] : 1.0f;
        srcc[c] = valid[c] && (unsigned)(x - S.sbx0) < (unsigned)S.sbnx;
        recc[c] = (x >= S.rx0) && (x < S.rx0 + S.nrec);
        splr[c] = valid[c] ? strip_col_plr(x, X, npml, nzi) : -1;
        sptb[c] = xin[c] ? x - npml : -1;
    }
    const int rpx0 = max(min(min(xa, X - 1 - xa), R), 1), rpx1 = max(min(min(xa + 1, X - 2 - xa), R), 1);
    const size_t pstrip = 2 * (size_t)R * nzi + 2 * (size_t)R * nxi;
    const size_t ptb = pstrip + 2 * (size_t)R * nzi;
    const float wit = a.wavelet[a.it];
    const float dtx = a.dtx, dtz = a.dtz;
    const bool any_band = xb[0] || xb[1];

    float qa[QL], qb[QL];   // q?[(u + k) % QL] = vz[z - 10 + k][xa (+1)]
#pragma unroll
    for (int k = 0; k < QL - 1; k++) {
        const float2 f = ld2(&svz[k * BX + 2 * tx]);
        qa[k] = f.x;
        qb[k] = f.y;
    }
    const int zend = min(z0 + BZ, Z);
    // operands of the next row
    float2 n_kap = make_float2(0.f, 0.f), n_p = n_kap, n_s1 = n_kap, n_s2 = n_kap, n_ps = n_kap;
    ACC n_g1[2] = {0, 0}, n_il[2] = {0, 0};
    auto load_row = [&](int z) {
        const unsigned id = (unsigned)z * pitch + xa;
        const bool zin = (z >= npml && z < Z - npml);
        n_kap = __ldg(reinterpret_cast<const float2 *>(&kappa[id]));
        n_p = ld2(&pp[id]);
        if (MODE != 3 && (any_band || !zin)) {
            n_s1 = ld2(&sxp[id]);
            n_s2 = ld2(&szp[id]);
        }
        if (MODE == 2 && zin && (xin[0] || xin[1])) {
            n_ps = __ldg(reinterpret_cast<const float2 *>(&psp[id]));
            const size_t im = (size_t)(z - npml) * nxi + (xa - npml);
            if (xin[0]) { n_g1[0] = g1p[im]; n_il[0] = ilp[im]; }
            if (xin[1]) { n_g1[1] = g1p[im + 1]; n_il[1] = ilp[im + 1]; }
        }
    };
    load_row(z0);
    for (int zb = z0; zb < zend; zb += QL) {
#pragma unroll
        for (int u = 0; u < QL; u++) {
            const int z = zb + u;
            if (z >= zend) break;
            const float2 kap = n_kap, op = n_p, os1 = n_s1, os2 = n_s2, ops = n_ps;
            const ACC og1[2] = {n_g1[0], n_g1[1]}, oil[2] = {n_il[0], n_il[1]};
            if (z + 1 < zend) load_row(z + 1);
            {
                const float2 f = ld2(&svz[(z - z0 + 19) * BX + 2 * tx]);
                qa[(u + QL - 1) % QL] = f.x;
                qb[(u + QL - 1) % QL] = f.y;
            }
            // w[k] = vx[z][xa - 10 + k], k = 0..21
            float w[22];
            const float *rw = &svx[(z - z0) * WW + 2 * tx + 2];
#pragma unroll
            for (int j = 0; j < 11; j++) {
                const float2 f = ld2(&rw[2 * j]);
                w[2 * j] = f.x;
                w[2 * j + 1] = f.y;
            }
            const int rpz = min(min(z, Z - 1 - z), R);
            float dx0 = 0.f, dx1 = 0.f, dz0 = 0.f, dz1 = 0.f;
            if (MODE == 3 || (!edge_order && rpz == R)) {
#pragma unroll
                for (int i = 1; i <= R; i++) {
                    dx0 += a.c10[i - 1] * (w[9 + i] - w[10 - i]);
                    dx1 += a.c10[i - 1] * (w[10 + i] - w[11 - i]);
                    dz0 += a.c10[i - 1] * (qa[(u + 9 + i) % QL] - qa[(u + 10 - i) % QL]);
                    dz1 += a.c10[i - 1] * (qb[(u + 9 + i) % QL] - qb[(u + 10 - i) % QL]);
                }
            } else {   // local order near the outer edge (kernel.cu:714-1185 with cuda_norder)
                const float *c0 = &s_tab[(max(min(rpx0, rpz), 1) - 1) * R];
                const float *c1 = &s_tab[(max(min(rpx1, rpz), 1) - 1) * R];
#pragma unroll
                for (int i = 1; i <= R; i++) {
                    dx0 += c0[i - 1] * (w[9 + i] - w[10 - i]);
                    dx1 += c1[i - 1] * (w[10 + i] - w[11 - i]);
                    dz0 += c0[i - 1] * (qa[(u + 9 + i) % QL] - qa[(u + 10 - i) % QL]);
                    dz1 += c1[i - 1] * (qb[(u + 9 + i) % QL] - qb[(u + 10 - i) % QL]);
                }
            }
            const unsigned id = (unsigned)z * pitch + xa;
            const bool zin = (z >= npml && z < Z - npml);
            const bool srcr = (unsigned)(z - S.sbz0) < (unsigned)S.sbnz;
            const float ddx[2] = {dx0 * dtx, dx1 * dtx}, ddz[2] = {dz0 * dtz, dz1 * dtz};
            const float kk[2] = {kap.x, kap.y}, p0[2] = {op.x, op.y};
            if (MODE == 3) {
                // ---------------- reconstruction: kernel.cu:389-429, strips of step it, source
                float ps[2] = {p0[0], p0[1]};
                bool wr[2] = {false, false};
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    if (zin && xin[c]) {
                        ps[c] = p0[c] + (ddx[c] * kk[c] + ddz[c] * kk[c]);
                        wr[c] = true;
                    } else {
                        long si = -1;
                        int kind = 2;
                        if (zin && splr[c] >= 0) si = (long)(pstrip + splr[c] + (size_t)(z - npml) * R);
                        else if (sptb[c] >= 0) {
                            const int srow = strip_row_tb(z, npml, Z - npml, nxi);
                            if (srow >= 0) { si = (long)(ptb + srow + sptb[c]); kind = 3; }
                        }
                        if (si >= 0) {   // read_d_ppmllr / read_d_ppmltb, kernel.cu:1348-1400
                            const float sc = a.strip_prec ? S.strip_scale[(size_t)a.it * 4 + kind] : 1.0f;
                            ps[c] = load_strip(S.strips, (size_t)a.it * S.strip_len + si, a.strip_prec, sc);
                            wr[c] = true;
                        }
                    }
                    if (srcr && srcc[c]) {   // kernel.cu:36-47 (subtract)
                        ps[c] -= S.src[(z - S.sbz0) * S.sbnx + (xa + c - S.sbx0)] * wit;
                        wr[c] = true;
                    }
                }
                st2(&pp[id], ps[0], ps[1], wr[0], wr[1]);
                continue;
            }
            // ---------------- full-grid pressure update with split-field PML
            const bool zupd = z >= 1 && z <= Z - 2;
            float pn[2] = {p0[0], p0[1]};
            bool wr[2] = {false, false};
            if (zupd) {
                if (zin && !any_band) {   // interior, kernel.cu:501-541
#pragma unroll
                    for (int c = 0; c < 2; c++) {
                        pn[c] = p0[c] - (ddx[c] * kk[c] + ddz[c] * kk[c]);
                        wr[c] = upd[c];
                    }
                } else {                  // split-field PML, kernel.cu:714-1185
                    const float c1z = s_c1z[z - z0], ic2z = s_ic2z[z - z0];
                    const float s1o[2] = {os1.x, os1.y}, s2o[2] = {os2.x, os2.y};
                    float s1n[2], s2n[2];
#pragma unroll
                    for (int c = 0; c < 2; c++) {
                        const float dxs = ddx[c] * kk[c], dzs = ddz[c] * kk[c];
                        if (zin && !xb[c]) {
                            pn[c] = p0[c] - (dxs + dzs);
                            s1n[c] = s1o[c];
                            s2n[c] = s2o[c];
                        } else {
                            s1n[c] = damp(s1o[c], dxs, c1x[c], ic2x[c]);
                            s2n[c] = damp(s2o[c], dzs, c1z, ic2z);
                            pn[c] = s1n[c] + s2n[c];
                        }
                        wr[c] = upd[c];
                    }
                    const bool sb0 = upd[0] && (xb[0] || !zin), sb1 = upd[1] && (xb[1] || !zin);
                    st2(&sxp[id], s1n[0], s1n[1], sb0, sb1);
                    st2(&szp[id], s2n[0], s2n[1], sb0, sb1);
                }
            }
            if (MODE != 2) {
                if (srcr) {   // kernel.cu:36-47 (add)
#pragma unroll
                    for (int c = 0; c < 2; c++)
                        if (srcc[c]) {
                            pn[c] += S.src[(z - S.sbz0) * S.sbnx + (xa + c - S.sbx0)] * wit;
                            wr[c] = true;
                        }
                }
                st2(&pp[id], pn[0], pn[1], wr[0], wr[1]);
                if (record && z == S.rz) {   // kernel.cu:48-71
#pragma unroll
                    for (int c = 0; c < 2; c++)
                        if (recc[c]) ((float *)S.gather)[(size_t)a.it * S.nrec + (xa + c - S.rx0)] = pn[c];
                }
                if (MODE == 1) {   // save_d_ppmllr / save_d_ppmltb, kernel.cu:1240-1293
#pragma unroll
                    for (int c = 0; c < 2; c++) {
                        if (zin && splr[c] >= 0) store_strip(a, S, pstrip + splr[c] + (size_t)(z - npml) * R, pn[c]);
                        else if (sptb[c] >= 0) {
                            const int srow = strip_row_tb(z, npml, Z - npml, nxi);
                            if (srow >= 0) store_strip(a, S, ptb + srow + sptb[c], pn[c]);
                        }
                    }
                }
            } else {
                if (z == S.rz) {   // kernel.cu:72-95 (overwrite)
#pragma unroll
                    for (int c = 0; c < 2; c++)
                        if (recc[c]) {
                            pn[c] = a.dt * gather_at(a, S, xa + c - S.rx0);
                            wr[c] = true;
                        }
                }
                st2(&pp[id], pn[0], pn[1], wr[0], wr[1]);
                if (zin) {   // kernel.cu:1401-1416
                    const size_t im = (size_t)(z - npml) * nxi + (xa - npml);
                    const float pss[2] = {ops.x, ops.y};
#pragma unroll
                    for (int c = 0; c < 2; c++)
                        if (xin[c]) {
                            g1p[im + c] = og1[c] + (ACC)pss[c] * (ACC)pn[c];
                            ilp[im + c] = oil[c] + (ACC)pss[c] * (ACC)pss[c];
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
    k_vel<BZ, MODE><<<ntiles, NT, vel_smem<BZ>(), s>>>(a);
}
template <int BZ, int MODE, typename ACC>
static void pres_launch_t(const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    static bool init = false;
    if (!init) {
        cudaFuncSetAttribute(k_pres<BZ, MODE, ACC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)pres_smem<BZ>());
        init = true;
    }
    k_pres<BZ, MODE, ACC><<<ntiles, NT, pres_smem<BZ>(), s>>>(a, record);
}
template <int BZ, int MODE>
static void pres_launch(const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if (MODE == 2 && a.accum_fp64) pres_launch_t<BZ, MODE, double>(a, ntiles, record, s);
    else pres_launch_t<BZ, MODE, float>(a, ntiles, record, s);
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
