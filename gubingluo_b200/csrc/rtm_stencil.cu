// rtm_stencil.cu — the time-step kernels of the RTM hot path (sm_100a).
//
// One launch updates one wavefield of every shot of a batch: a flat (shot, tile) work list
// maps each 128-thread block to a BX x BZ tile of one shot.  Each thread owns one grid
// column x and marches down the tile's BZ rows:
//   * the tile and its halo are staged once into shared memory by the tensor memory
//     accelerator (2-D cp.async.bulk.tensor boxes issued by one thread, completion on an
//     mbarrier; rows and columns outside the field arrive as zeros);
//   * x-derivatives read the staged row; z-derivatives read a (2R+U-1)-deep register window
//     that advances U rows per unrolled group (one shared load per row, a few register moves
//     per group), which keeps the loop body small enough for the instruction cache;
//   * the per-cell operands of the next group of U rows are loaded while the current group is
//     computed (the first group's while the tile is staged);
//   * the full-order coefficients come from the kernel-parameter constant bank.  Tiles that
//     reach the outer ten cells of the grid, where the local order is reduced (reference
//     cuda_norder*, kernel.cu:271-317), run the same groups with coefficients from rows of the
//     zero-padded table (the choice is per tile, so warps do not diverge); rows left over
//     after the last whole group take a compact one-row path;
//   * PML damping, split pressure, source, receivers, strip restore and imaging are per-row
//     or per-column predicates of the same kernel (strips are saved by k_strip_save after
//     each forward step).
// Reference equivalents (gubingluo kernel.cu): forward v :430-500 + :542-713, forward p
// :501-541 + :714-1185, reconstruction :318-429, strip restore :1294-1400, source :36-47,
// receivers :48-95, cross-correlation :1401-1416.
#include <atomic>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "rtm_launch.h"
#include "rtm_types.h"

namespace {

constexpr int BX = RTM_BX;          // threads (= columns) per block
constexpr int WW = RTM_STAGE_W;     // staged width: columns x0-12 .. x0+BX+11 (16-byte aligned)
constexpr int R = RTM_RADIUS;
// Rows per unrolled group (measured: 2 rows make the forward and receiver velocity kernels
// 2-5% faster than 4, and the reconstruction 24% slower; the forward and receiver pressure
// kernels are fastest at 2 rows with 7 resident blocks (72 registers), 4-9% faster than 4
// rows at 6 and 5 blocks, while the reconstruction pressure kernel is 4% slower that way
// than at 4 rows and 6 blocks).  The z window of U rows is 2R+U-1 deep; each kernel family
// stages the rows of its deepest window, so every mode reads one box height.
constexpr int UV = RTM_GROUP_VEL, UVR = RTM_GROUP_VEL_RECON;
constexpr int UP = RTM_GROUP_PRES, UPR = RTM_GROUP_PRES_RECV, UPC = RTM_GROUP_PRES_RECON;
constexpr int QNV_MAX = 2 * R + RTM_MAX2(UV, UVR) - 1;
constexpr int QNP_MAX = 2 * R + RTM_MAX2(UP, RTM_MAX2(UPR, UPC)) - 1;
static_assert(QNV_MAX - 1 == RTM_STAGE_ZEXTRA_VEL && QNP_MAX - 1 == RTM_STAGE_ZEXTRA_PRES,
              "staged rows beyond a tile must cover the z window");
#ifndef RTM_VEL_RECON_BLOCKS
#define RTM_VEL_RECON_BLOCKS 6   // resident blocks per SM of the reconstruction velocity kernel
#endif
// resident blocks per SM of the fp32 pressure kernels (forward; receiver pass; reconstruction)
#ifndef RTM_PRES_FWD_BLOCKS
#define RTM_PRES_FWD_BLOCKS 7
#endif
#ifndef RTM_PRES_RECV_BLOCKS
#define RTM_PRES_RECV_BLOCKS 7
#endif
#ifndef RTM_PRES_RECON_BLOCKS
#define RTM_PRES_RECON_BLOCKS 6
#endif
static_assert(WW == BX + 24, "staged width");
constexpr long kWaitLimit = 1L << 22;   // polls of a tile's TMA barrier before giving up


__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// ---- TMA tile staging ------------------------------------------------------------------
// One thread of the block initialises an mbarrier, announces the bytes of the tile's boxes and
// issues the 2-D TMA copies (cp.async.bulk.tensor, no multicast; boxes start at x0-12 or x0, a
// multiple of 4 floats, and rows or columns outside the field arrive as zeros); every thread
// then polls the barrier, at most kWaitLimit times.
__device__ __forceinline__ void mbar_init(unsigned long long *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_box(float *dst, const void *tmap, int x, int y, unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_done(unsigned long long *bar)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar))
        : "memory");
    return ok != 0;
}
// Wait for the tile; on giving up, flag the error, wait once more (bounded) for the copies
// still in flight and report false, so that the block returns without computing.
__device__ __forceinline__ bool tile_wait(unsigned long long *bar, int *err)
{
    for (long i = 0; i < kWaitLimit; i++)
        if (mbar_done(bar)) return true;
    atomicExch(err, 1);
    for (long i = 0; i < kWaitLimit; i++)
        if (mbar_done(bar)) break;
    return false;
}
__device__ __forceinline__ const void *tmap_of(const ShotDev &S, int which)
{
    return (const char *)S.tmaps + which * RTM_TMAP_BYTES;
}

__device__ __forceinline__ float load_strip(const void *base, size_t idx, int prec, float scale)
{
    if (prec == RTM_FP16) return __half2float(((const __half *)base)[idx]) * scale;
    if (prec == RTM_BF16) return __bfloat162float(((const __nv_bfloat16 *)base)[idx]) * scale;
    return ((const float *)base)[idx];
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

// Interior pressure update p - (dxs + dzs) and the cross-correlation terms, shared by the
// general and the interior-tile forms of the pressure kernel so that both give the same
// bits: the sum and the difference are rounded separately (no fused multiply-add), as the
// reference's host-order arithmetic and the oracle have them.
__device__ __forceinline__ float p_interior(float p0, float dxs, float dzs) { return __fsub_rn(p0, __fadd_rn(dxs, dzs)); }
template <typename ACC>
__device__ __forceinline__ void image_cell(ACC *__restrict__ g1p, ACC *__restrict__ ilp, unsigned id, ACC og1, ACC oil,
                                           float ps, float pn)
{
    g1p[id] = og1 + (ACC)ps * (ACC)pn;
    ilp[id] = oil + (ACC)ps * (ACC)ps;
}

// Damped or undamped update f' = (c1*f - d)*ic2; outside the PML c1 = ic2 = 1, which makes
// this exactly f - d.  Each operation is rounded on its own (no fused multiply-add), so the
// interior-tile bodies below, which write f - d, give the same bits.
__device__ __forceinline__ float damp(float f, float d, float c1, float ic2)
{
    return __fmul_rn(__fsub_rn(__fmul_rn(c1, f), d), ic2);
}
// Velocity increment (dt/h) * D * (1/rho), and the reconstruction updates, rounded the same
// way in every body.
__device__ __forceinline__ float vel_inc(float d, float dth, float ir) { return __fmul_rn(__fmul_rn(d, dth), ir); }
__device__ __forceinline__ float p_recon(float p0, float dxs, float dzs) { return __fadd_rn(p0, __fadd_rn(dxs, dzs)); }

// Advance the z window by N rows: q[k] <- q[k+N], then the N new entries from the staged
// column s (entry k of the advanced window is staged row dz + k, dz = rows advanced since
// the tile's first row).  `more` is false after the tile's last row: nothing is read then.
template <int N, int STRIDE, int QN>
__device__ __forceinline__ void advance(float (&q)[QN], const float *s, int dz, bool more)
{
#pragma unroll
    for (int k = 0; k + N < QN; k++) q[k] = q[k + N];
    if (more) {
#pragma unroll
        for (int j = 0; j < N; j++) q[QN - N + j] = s[(dz + QN - N + j) * STRIDE];
    }
}

// Shot integers used inside the row loops, read once per thread.
struct ShotK {
    int nxi, nzi, strip_len;
    int sbx0, sbnx, sbz0, sbnz;   // source box
    int rz, rx0, nrec;            // receiver line
};

__device__ __forceinline__ ShotK shot_ints(const ShotDev &S)
{
    ShotK k;
    k.nxi = S.nxi; k.nzi = S.nzi; k.strip_len = S.strip_len;
    k.sbx0 = S.sbx0; k.sbnx = S.sbnx; k.sbz0 = S.sbz0; k.sbnz = S.sbnz;
    k.rz = S.rz; k.rx0 = S.rx0; k.nrec = S.nrec;
    return k;
}

// Sum_{i=1..R} c(i-1) * (f(i) - g(i)) in tap order; c is a coefficient accessor.
template <typename C, typename F, typename G>
__device__ __forceinline__ float tap_sum(C c, F f, G g)
{
    float s0 = 0.f;
#pragma unroll
    for (int i = 1; i <= R; i++) s0 += c(i - 1) * (f(i) - g(i));
    return s0;
}

// Per-column constants of the velocity update.
struct VelCol {
    bool hvx;            // column x carries a vx cell (x < X-1)
    float c1vx, ic2vx;   // vx damping of this column
    int svx, svz;        // strip columns of the reconstruction (-1: none)
    bool rvx, rvz;       // reconstruction-interior columns
};

// Velocity update of one cell (x, z) from the raw derivative sums dx, dz.
template <int MODE>
__device__ __forceinline__ void vel_apply(const StepArgs &a, const ShotDev &S, const ShotK &k, const VelCol &cc,
                                          float *__restrict__ vxp, float *__restrict__ vzp, unsigned id, int z,
                                          int Z, int npml, float dx, float dz, float ir, float ov, float ow,
                                          float c1z, float ic2z)
{
    const float dtx = a.dtx, dtz = a.dtz;
    if (MODE == 3) {
        // kernel.cu:318-388 (+=) on the interior; strips of step it+1 elsewhere
        const bool zin = (z >= npml && z < Z - npml);
        const bool zinv = (z >= npml && z <= Z - npml - 2);
        if (zin && cc.rvx) vxp[id] = __fadd_rn(ov, vel_inc(dx, dtx, ir));
        else if (zin && cc.svx >= 0) {   // read_d_vxpml, kernel.cu:1294-1320
            const float sc = a.strip_prec ? S.strip_scale[(size_t)(a.it + 1) * 4 + 0] : 1.0f;
            vxp[id] = load_strip(S.strips, (size_t)(a.it + 1) * k.strip_len + cc.svx + (size_t)(z - npml) * R,
                                 a.strip_prec, sc);
        }
        if (zinv && cc.rvz) vzp[id] = __fadd_rn(ow, vel_inc(dz, dtz, ir));
        else if (cc.svz >= 0 && z < Z - 1) {   // read_d_vzpml, kernel.cu:1321-1347
            const int srow = strip_row_tb(z, npml, Z - npml - 1, k.nxi);
            if (srow >= 0) {
                const float sc = a.strip_prec ? S.strip_scale[(size_t)(a.it + 1) * 4 + 1] : 1.0f;
                vzp[id] = load_strip(S.strips,
                                     (size_t)(a.it + 1) * k.strip_len + 2 * (size_t)R * k.nzi + srow + cc.svz,
                                     a.strip_prec, sc);
            }
        }
        return;
    }
    // kernel.cu:430-500 (interior) and :542-713 (PML): f' = (c1*f - d)*ic2
    const float nvx = damp(ov, vel_inc(dx, dtx, ir), cc.c1vx, cc.ic2vx);
    if (cc.hvx) vxp[id] = nvx;
    const float nvz = damp(ow, vel_inc(dz, dtz, ir), c1z, ic2z);
    if (z < Z - 1) vzp[id] = nvz;
}

// Per-column constants of the pressure update.
struct PresCol {
    bool xb, xin;        // column in the x PML band / in the image interior
    bool srcc, recc;     // column in the source box / on the receiver line
    float c1x, ic2x;     // x damping of this column
    int splr, sptb;      // strip columns of the reconstruction (-1: none)
};

// Pressure update of one cell (x, z) from the raw derivative sums dx, dz; `upd` is false on
// the grid's edge rows and columns, which keep their pressure (kernel.cu:714-1185).
template <int MODE, typename ACC>
__device__ __forceinline__ void pres_apply(const StepArgs &a, const ShotDev &S, const ShotK &k, const PresCol &cc,
                                           float wit, float *__restrict__ pp, float *__restrict__ sxp,
                                           float *__restrict__ szp, ACC *__restrict__ g1p, ACC *__restrict__ ilp,
                                           unsigned id, int x, int z, int Z, int npml, bool upd, float dx,
                                           float dz, float kk, float p0, float s1o, float s2o, float ps, ACC og1,
                                           ACC oil, float c1z, float ic2z, int record)
{
    const float ddx = dx * a.dtx, ddz = dz * a.dtz;
    const bool zin = (z >= npml && z < Z - npml);
    const bool srcr = (unsigned)(z - k.sbz0) < (unsigned)k.sbnz;
    if (MODE == 3) {
        // reconstruction: kernel.cu:389-429, strips of step it, source subtracted
        float pn = p0;
        bool wr = false;
        if (zin && cc.xin) {
            pn = p_recon(p0, ddx * kk, ddz * kk);
            wr = true;
        } else {
            const size_t pstrip = 2 * (size_t)R * k.nzi + 2 * (size_t)R * k.nxi;
            long si = -1;
            int kind = 2;
            if (zin && cc.splr >= 0) si = (long)(pstrip + cc.splr + (size_t)(z - npml) * R);
            else if (cc.sptb >= 0) {
                const int srow = strip_row_tb(z, npml, Z - npml, k.nxi);
                if (srow >= 0) {
                    si = (long)(pstrip + 2 * (size_t)R * k.nzi + srow + cc.sptb);
                    kind = 3;
                }
            }
            if (si >= 0) {   // read_d_ppmllr / read_d_ppmltb, kernel.cu:1348-1400
                const float sc = a.strip_prec ? S.strip_scale[(size_t)a.it * 4 + kind] : 1.0f;
                pn = load_strip(S.strips, (size_t)a.it * k.strip_len + si, a.strip_prec, sc);
                wr = true;
            }
        }
        if (srcr && cc.srcc) {   // kernel.cu:36-47 (subtract)
            pn -= S.src[(z - k.sbz0) * k.sbnx + (x - k.sbx0)] * wit;
            wr = true;
        }
        if (wr) pp[id] = pn;
        return;
    }
    // full-grid pressure update with split-field PML
    float pn = p0;
    bool wr = false;
    if (upd) {
        const float dxs = ddx * kk, dzs = ddz * kk;
        if (zin && !cc.xb) pn = p_interior(p0, dxs, dzs);   // interior, kernel.cu:501-541
        else {                                      // split-field PML, kernel.cu:714-1185
            const float s1n = damp(s1o, dxs, cc.c1x, cc.ic2x);
            const float s2n = damp(s2o, dzs, c1z, ic2z);
            pn = s1n + s2n;
            sxp[id] = s1n;
            szp[id] = s2n;
        }
        wr = true;
    }
    if (MODE == 0) {
        if (srcr && cc.srcc) {   // kernel.cu:36-47 (add)
            pn += S.src[(z - k.sbz0) * k.sbnx + (x - k.sbx0)] * wit;
            wr = true;
        }
        if (wr) pp[id] = pn;
        if (record && z == k.rz && cc.recc)   // kernel.cu:48-71
            ((float *)S.gather)[(size_t)a.it * k.nrec + (x - k.rx0)] = pn;
    } else {
        if (z == k.rz && cc.recc) {   // kernel.cu:72-95 (overwrite)
            pn = a.dt * gather_at(a, S, x - k.rx0);
            wr = true;
        }
        if (wr) pp[id] = pn;
        if (zin && cc.xin) image_cell<ACC>(g1p, ilp, id, og1, oil, ps, pn);   // kernel.cu:1401-1416
    }
}

}  // namespace

// =====================================================================================
// Velocity update.  MODE 0: forward, full grid; 2: receiver (backward model), full grid;
// 3: reconstruction of the source wavefield (interior only, vx/vz strips of step it+1
// restored).
// Register budget (measured): 6 blocks per SM (80 registers, no spills) in every mode but the
// 8-row reconstruction tiles (5, which would spill at 6); with its interior-tile body the
// reconstruction runs 4% faster at 6 than at 5.
template <int BZ, int MODE>
__global__ void __launch_bounds__(BX, MODE == 3 ? (BZ == 8 ? 5 : RTM_VEL_RECON_BLOCKS) : 6) k_vel(const StepArgs a)
{
    constexpr int U = MODE == 3 ? UVR : UV, QN = 2 * R + U - 1;
    static_assert(BZ % U == 0, "interior tiles take whole row groups");
    constexpr int WH = BZ + QNV_MAX - 1;   // staged rows z0-9 .. z0+BZ+QNV_MAX-11 (the box height)
    extern __shared__ __align__(128) float sw[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ float s_tab[100];
    __shared__ float s_c1vz[BZ], s_ic2vz[BZ];
    const TileRef t = a.tiles[blockIdx.x];   // reconstruction: tiles of the interior + strips only
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = t.x0, z0 = t.z0;
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ inv_rho = (MODE >= 2) ? S.inv_rho_b : S.inv_rho_f;
    const PmlOffsets o = pml_offsets(X, Z);
    if (threadIdx.x == 0) {   // p rows z0-9 .. z0+BZ+12, columns x0-12 .. x0+139
        mbar_init(&s_bar);
        mbar_expect(&s_bar, WH * WW * sizeof(float));
        tma_box(sw, tmap_of(S, MODE == 2 ? RTM_TMAP_B_P : (MODE == 3 ? RTM_TMAP_A_P_RECON : RTM_TMAP_A_P)), x0 - 12,
                z0 - 9, &s_bar);
    }
    for (int i = threadIdx.x; i < 100; i += BX) s_tab[i] = a.coef[i];
    for (int i = threadIdx.x; i < BZ; i += BX) {
        const int z = min(z0 + i, Z - 2);
        s_c1vz[i] = S.pml[o.c1vz + z];
        s_ic2vz[i] = S.pml[o.ic2vz + z];
    }
    const int tx = threadIdx.x, x = x0 + tx;
    const ShotK k = shot_ints(S);
    float *__restrict__ vxp = W.vx;
    float *__restrict__ vzp = W.vz;
    VelCol cc;
    cc.hvx = x < X - 1;
    {
        const bool band = (x < npml) || (x >= X - npml - 1);
        cc.c1vx = (band && cc.hvx) ? S.pml[o.c1vx + x] : 1.0f;
        cc.ic2vx = (band && cc.hvx) ? S.pml[o.ic2vx + x] : 1.0f;
    }
    cc.svx = (MODE == 3 && cc.hvx) ? strip_col_vx(x, X, npml, k.nzi) : -1;
    cc.svz = (x >= npml && x < X - npml) ? x - npml : -1;
    cc.rvx = (x >= npml && x <= X - npml - 2);
    cc.rvz = (x >= npml && x < X - npml);
    // vx order of this column (cuda_norderx): full unless within ten cells of the edge
    const int ox = min(min(x + 1, X - 1 - x), R);
    const int zend = min(z0 + BZ, Z);
    // Tiles that reach the outer ten cells of the grid take the table-coefficient form of the
    // unrolled groups: vx order per column (cuda_norderx), vz order per row (cuda_norderz).
    // The reconstruction writes only cells at least npml >= R from the edge, where every
    // order is full.
    const bool edge_tile = MODE != 3 && (x0 < R || x0 + BX > X - R || z0 < R || zend > Z - R);
    const float *cxe = &s_tab[(max(ox, 1) - 1) * R];
    // operands of the first unrolled group, loaded while the tile is staged
    float cir[U], cov[U], cow[U];
    auto load_group = [&](int zg, float(&gir)[U], float(&gov)[U], float(&gow)[U]) {
        const unsigned g0 = (unsigned)zg * pitch + x;
#pragma unroll
        for (int u = 0; u < U; u++) {
            gir[u] = __ldg(&inv_rho[g0 + u * pitch]);
            gov[u] = vxp[g0 + u * pitch];
            gow[u] = vzp[g0 + u * pitch];
        }
    };
    if (x < X && z0 + U <= zend) load_group(z0, cir, cov, cow);
    __syncthreads();
    if (!tile_wait(&s_bar, a.err) || x >= X) return;   // no barrier below

    const float *col = &sw[tx + 12];   // staged column x: col[r*WW] = p[z0-9+r][x]
    float q[QN];                        // q[k] = p[z-9+k][x] at the current row z
#pragma unroll
    for (int j = 0; j < QN; j++) q[j] = col[j * WW];

    // interior tiles (TileRef.interior: every column in [npml, X-npml-1), every row in
    // [npml, Z-npml-1), where the velocity damping is 1 and no strip lies): the update
    // alone, in the arithmetic of the general body
    if (t.interior) {
#pragma unroll 1
        for (int z = z0; z < z0 + BZ; z += U) {
            float nir[U], nov[U], now[U];
            const bool more = z + 2 * U <= z0 + BZ;
            if (more) load_group(z + U, nir, nov, now);
            const unsigned id0 = (unsigned)z * pitch + x;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const float *rw = &col[(z + u - z0 + 9) * WW];
                const float dx = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return rw[i]; },
                                         [&](int i) { return rw[1 - i]; });
                const float dz = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return q[u + 9 + i]; },
                                         [&](int i) { return q[u + 10 - i]; });
                const unsigned id = id0 + u * pitch;
                if (MODE == 3) {
                    vxp[id] = __fadd_rn(cov[u], vel_inc(dx, a.dtx, cir[u]));
                    vzp[id] = __fadd_rn(cow[u], vel_inc(dz, a.dtz, cir[u]));
                } else {
                    vxp[id] = __fsub_rn(cov[u], vel_inc(dx, a.dtx, cir[u]));
                    vzp[id] = __fsub_rn(cow[u], vel_inc(dz, a.dtz, cir[u]));
                }
            }
            advance<U, WW>(q, col, z + U - z0, z + U < z0 + BZ);
            if (more) {
#pragma unroll
                for (int u = 0; u < U; u++) {
                    cir[u] = nir[u];
                    cov[u] = nov[u];
                    cow[u] = now[u];
                }
            }
        }
        return;
    }

    // one-row path for the rows after the last whole group: local orders from the table
    auto one_row = [&](int z) {
        const unsigned id = (unsigned)z * pitch + x;
        const float ir = __ldg(&inv_rho[id]), ov = vxp[id], ow = vzp[id];
        const float *rw = &col[(z - z0 + 9) * WW];
        const int oz = (MODE == 3) ? R : min(min(z + 1, Z - 1 - z), R);
        const float *cx = &s_tab[((MODE == 3) ? R - 1 : max(ox, 1) - 1) * R];
        const float *cz = &s_tab[(max(oz, 1) - 1) * R];
        float dx = 0.f, dz = 0.f;
#pragma unroll
        for (int i = 1; i <= R; i++) {
            dx += cx[i - 1] * (rw[i] - rw[1 - i]);
            dz += cz[i - 1] * (q[9 + i] - q[10 - i]);
        }
        vel_apply<MODE>(a, S, k, cc, vxp, vzp, id, z, Z, npml, dx, dz, ir, ov, ow, s_c1vz[z - z0],
                        s_ic2vz[z - z0]);
    };

    int z = z0;
    for (; z + U <= zend; z += U) {
        float nir[U], nov[U], now[U];
        const bool more = z + 2 * U <= zend;
        if (more) load_group(z + U, nir, nov, now);
        const unsigned id0 = (unsigned)z * pitch + x;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const float *rw = &col[(z + u - z0 + 9) * WW];
            float dx, dz;
            if (!edge_tile) {
                dx = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return rw[i]; },
                             [&](int i) { return rw[1 - i]; });
                dz = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return q[u + 9 + i]; },
                             [&](int i) { return q[u + 10 - i]; });
            } else {
                const int zz = z + u, oz = min(min(zz + 1, Z - 1 - zz), R);
                const float *cze = &s_tab[(max(oz, 1) - 1) * R];
                dx = tap_sum([&](int j) { return cxe[j]; }, [&](int i) { return rw[i]; },
                             [&](int i) { return rw[1 - i]; });
                dz = tap_sum([&](int j) { return cze[j]; }, [&](int i) { return q[u + 9 + i]; },
                             [&](int i) { return q[u + 10 - i]; });
            }
            vel_apply<MODE>(a, S, k, cc, vxp, vzp, id0 + u * pitch, z + u, Z, npml, dx, dz, cir[u], cov[u], cow[u],
                            s_c1vz[z + u - z0], s_ic2vz[z + u - z0]);
        }
        advance<U, WW>(q, col, z + U - z0, z + U < zend);
        if (more) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                cir[u] = nir[u];
                cov[u] = nov[u];
                cow[u] = now[u];
            }
        }
    }
    for (; z < zend; z++) {
        one_row(z);
        advance<1, WW>(q, col, z + 1 - z0, z + 1 < zend);
    }
}

// =====================================================================================
// Pressure update.  MODE 0: forward (+ source, + receiver sampling when `record`);
// 2: receiver (backward model): overwrite the receiver row with dt*gather[it], then image
// g1 += ps*p, illum += ps*ps; 3: reconstruction (interior, p strips of step it restored,
// source subtracted).
// Register budgets (measured, no spills): 7 blocks per SM (72 registers) for the forward and
// receiver passes in their 2-row groups, 6 (80 registers) for the reconstruction in 4-row
// groups, 4 for the receiver pass with fp64 accumulators (123 registers).  With 4-row groups
// the receiver pass needed 96 registers (5 blocks) and spilled when capped at 6.
//
// Interior tiles (TileRef.interior, set by the host for tiles whose every column lies in
// [npml, X-npml) and every row in [npml, Z-npml), with no source cell and no receiver) take
// a second body in the same kernel, chosen per block: the interior update alone, with no
// PML, source or receiver tests and no split-field loads, in the arithmetic of the general
// body's interior branch (for the reconstruction: tiles of the interior with no source cell).
template <int BZ, int MODE, typename ACC>
__global__ void __launch_bounds__(BX, MODE == 2   ? (sizeof(ACC) == 8 ? 4 : RTM_PRES_RECV_BLOCKS)
                                     : MODE == 3 ? RTM_PRES_RECON_BLOCKS
                                                 : RTM_PRES_FWD_BLOCKS)
    k_pres(const StepArgs a, int record)
{
    constexpr int U = MODE == 2 ? UPR : MODE == 3 ? UPC : UP, QN = 2 * R + U - 1;
    static_assert(BZ % U == 0, "interior tiles take whole row groups");
    constexpr int XH = BZ;            // vx rows z0 .. z0+BZ-1, columns x0-12 .. x0+BX+11
    constexpr int ZH = BZ + QNP_MAX - 1;   // vz rows z0-10 .. z0+BZ+QNP_MAX-12 (the box height), columns x0 ..
    extern __shared__ __align__(128) float sm[];
    float *svx = sm;
    float *svz = sm + XH * WW;   // XH * WW * 4 bytes is a multiple of 128
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ float s_tab[100];
    __shared__ float s_c1z[BZ], s_ic2z[BZ];
    const TileRef t = a.tiles[blockIdx.x];   // reconstruction: tiles of the interior + strips only
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = t.x0, z0 = t.z0;
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ kappa = (MODE >= 2) ? S.kappa_b : S.kappa_f;
    const PmlOffsets o = pml_offsets(X, Z);
    if (threadIdx.x == 0) {   // vx rows z0 .. z0+BZ-1 (columns x0-12 ..), vz rows z0-10 .. z0+BZ+11
        mbar_init(&s_bar);
        mbar_expect(&s_bar, (XH * WW + ZH * BX) * sizeof(float));
        tma_box(svx, tmap_of(S, MODE == 2 ? RTM_TMAP_B_VX : RTM_TMAP_A_VX), x0 - 12, z0, &s_bar);
        tma_box(svz, tmap_of(S, MODE == 2 ? RTM_TMAP_B_VZ : RTM_TMAP_A_VZ), x0, z0 - 10, &s_bar);
    }
    for (int i = threadIdx.x; i < 100; i += BX) s_tab[i] = a.coef[i];
    for (int i = threadIdx.x; i < BZ; i += BX) {
        const int z = min(z0 + i, Z - 1);
        s_c1z[i] = S.pml[o.c1z + z];
        s_ic2z[i] = S.pml[o.ic2z + z];
    }
    const int tx = threadIdx.x, x = x0 + tx;
    const ShotK k = shot_ints(S);
    float *__restrict__ pp = W.p;
    float *__restrict__ sxp = W.sx;
    float *__restrict__ szp = W.sz;
    const float *__restrict__ psp = S.a.p;
    ACC *__restrict__ g1p = (ACC *)S.g1;
    ACC *__restrict__ ilp = (ACC *)S.illum;
    PresCol cc;
    cc.xb = (x < npml) || (x >= X - npml);
    cc.xin = !cc.xb;
    cc.c1x = (cc.xb && x < X) ? S.pml[o.c1x + x] : 1.0f;
    cc.ic2x = (cc.xb && x < X) ? S.pml[o.ic2x + x] : 1.0f;
    cc.srcc = (unsigned)(x - k.sbx0) < (unsigned)k.sbnx;
    cc.recc = (x >= k.rx0) && (x < k.rx0 + k.nrec);
    cc.splr = (MODE == 3) ? strip_col_plr(x, X, npml, k.nzi) : -1;
    cc.sptb = cc.xin ? x - npml : -1;
    const float wit = a.wavelet[a.it];
    // local order of this column (cuda_norder): full unless within ten cells of the edge
    const int rpx = min(min(x, X - 1 - x), R);
    const int zend = min(z0 + BZ, Z);
    // tiles that reach the outer ten cells take the table-coefficient form of the groups
    const bool edge_tile = MODE != 3 && (x0 < R || x0 + BX > X - R || z0 < R || zend > Z - R);
    // operands of an unrolled group of rows
    float ckk[U], cp0[U], cs1[U], cs2[U], cps[U];
    ACC cg1[U], cil[U];
    auto load_group = [&](int zg, float(&gkk)[U], float(&gp0)[U], float(&gs1)[U], float(&gs2)[U],
                          float(&gps)[U], ACC(&gg1)[U], ACC(&gil)[U]) {
        const unsigned g0 = (unsigned)zg * pitch + x;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned id = g0 + u * pitch;
            const int zz = zg + u;
            const bool zin = (zz >= npml && zz < Z - npml);
            const bool band = cc.xb || !zin;
            gkk[u] = __ldg(&kappa[id]);
            // a band cell's new p is the sum of its split fields: its old p is needed only on
            // the grid's edge rows and columns, which keep it (edge tiles only)
            gp0[u] = (MODE != 3 && band && !edge_tile) ? 0.f : pp[id];
            gs1[u] = (MODE != 3 && band) ? sxp[id] : 0.f;
            gs2[u] = (MODE != 3 && band) ? szp[id] : 0.f;
            gps[u] = 0.f;
            gg1[u] = 0;
            gil[u] = 0;
            if (MODE == 2 && zin && cc.xin) {
                gps[u] = __ldg(&psp[id]);
                gg1[u] = g1p[id];
                gil[u] = ilp[id];
            }
        }
    };
    if (x < X && z0 + U <= zend) load_group(z0, ckk, cp0, cs1, cs2, cps, cg1, cil);
    __syncthreads();
    if (!tile_wait(&s_bar, a.err) || x >= X) return;

    const float *colx = &svx[tx + 12];   // colx[r*WW] = vx[z0+r][x]
    const float *colz = &svz[tx];        // colz[r*BX] = vz[z0-10+r][x]
    float q[QN];                          // q[k] = vz[z-10+k][x] at the current row z
#pragma unroll
    for (int j = 0; j < QN; j++) q[j] = colz[j * BX];

    if (t.interior) {
#pragma unroll 1
        for (int z = z0; z < z0 + BZ; z += U) {
            float nkk[U], np0[U], nps[U];
            ACC ng1[U], nil[U];
            const bool more = z + 2 * U <= z0 + BZ;
            if (more) {
                const unsigned g0 = (unsigned)(z + U) * pitch + x;
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const unsigned id = g0 + u * pitch;
                    nkk[u] = __ldg(&kappa[id]);
                    np0[u] = pp[id];
                    if (MODE == 2) {
                        nps[u] = __ldg(&psp[id]);
                        ng1[u] = g1p[id];
                        nil[u] = ilp[id];
                    }
                }
            }
            const unsigned id0 = (unsigned)z * pitch + x;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const float *rw = &colx[(z + u - z0) * WW];
                const float dx = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return rw[i - 1]; },
                                         [&](int i) { return rw[-i]; });
                const float dz = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return q[u + 9 + i]; },
                                         [&](int i) { return q[u + 10 - i]; });
                const float ddx = dx * a.dtx, ddz = dz * a.dtz;
                const float pn = MODE == 3 ? p_recon(cp0[u], ddx * ckk[u], ddz * ckk[u])
                                           : p_interior(cp0[u], ddx * ckk[u], ddz * ckk[u]);
                const unsigned id = id0 + u * pitch;
                pp[id] = pn;
                if (MODE == 2) image_cell<ACC>(g1p, ilp, id, cg1[u], cil[u], cps[u], pn);
            }
            advance<U, BX>(q, colz, z + U - z0, z + U < z0 + BZ);
            if (more) {
#pragma unroll
                for (int u = 0; u < U; u++) {
                    ckk[u] = nkk[u];
                    cp0[u] = np0[u];
                    if (MODE == 2) {
                        cps[u] = nps[u];
                        cg1[u] = ng1[u];
                        cil[u] = nil[u];
                    }
                }
            }
        }
        return;
    }

    // one-row path for the rows after the last whole group: local orders from the table
    auto one_row = [&](int z) {
        const unsigned id = (unsigned)z * pitch + x;
        const bool zin = (z >= npml && z < Z - npml);
        const bool band = cc.xb || !zin;
        const float kk = __ldg(&kappa[id]), p0 = pp[id];
        const float s1o = (MODE != 3 && band) ? sxp[id] : 0.f, s2o = (MODE != 3 && band) ? szp[id] : 0.f;
        float ps = 0.f;
        ACC og1 = 0, oil = 0;
        if (MODE == 2 && zin && cc.xin) {
            ps = __ldg(&psp[id]);
            og1 = g1p[id];
            oil = ilp[id];
        }
        const float *rw = &colx[(z - z0) * WW];
        const int rpz = min(min(z, Z - 1 - z), R);
        const int rp = (MODE == 3) ? R : min(rpx, rpz);
        const float *c = &s_tab[(max(rp, 1) - 1) * R];
        float dx = 0.f, dz = 0.f;
#pragma unroll
        for (int i = 1; i <= R; i++) {
            dx += c[i - 1] * (rw[i - 1] - rw[-i]);
            dz += c[i - 1] * (q[9 + i] - q[10 - i]);
        }
        pres_apply<MODE, ACC>(a, S, k, cc, wit, pp, sxp, szp, g1p, ilp, id, x, z, Z, npml, rp > 0, dx, dz, kk, p0,
                              s1o, s2o, ps, og1, oil, s_c1z[z - z0], s_ic2z[z - z0], record);
    };

    int z = z0;
    for (; z + U <= zend; z += U) {
        float nkk[U], np0[U], ns1[U], ns2[U], nps[U];
        ACC ng1[U], nil[U];
        const bool more = z + 2 * U <= zend;
        if (more) load_group(z + U, nkk, np0, ns1, ns2, nps, ng1, nil);
        const unsigned id0 = (unsigned)z * pitch + x;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const float *rw = &colx[(z + u - z0) * WW];
            float dx, dz;
            bool upd = true;
            if (!edge_tile) {
                dx = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return rw[i - 1]; },
                             [&](int i) { return rw[-i]; });
                dz = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return q[u + 9 + i]; },
                             [&](int i) { return q[u + 10 - i]; });
            } else {   // local order min(x, z distance to the edge, R); none on the edge itself
                const int zz = z + u, rp = min(rpx, min(min(zz, Z - 1 - zz), R));
                const float *cf = &s_tab[(max(rp, 1) - 1) * R];
                upd = rp > 0;
                dx = tap_sum([&](int j) { return cf[j]; }, [&](int i) { return rw[i - 1]; },
                             [&](int i) { return rw[-i]; });
                dz = tap_sum([&](int j) { return cf[j]; }, [&](int i) { return q[u + 9 + i]; },
                             [&](int i) { return q[u + 10 - i]; });
            }
            pres_apply<MODE, ACC>(a, S, k, cc, wit, pp, sxp, szp, g1p, ilp, id0 + u * pitch, x, z + u, Z, npml, upd,
                                  dx, dz, ckk[u], cp0[u], cs1[u], cs2[u], cps[u], cg1[u], cil[u], s_c1z[z + u - z0],
                                  s_ic2z[z + u - z0], record);
        }
        advance<U, BX>(q, colz, z + U - z0, z + U < zend);
        if (more) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                ckk[u] = nkk[u];
                cp0[u] = np0[u];
                cs1[u] = ns1[u];
                cs2[u] = ns2[u];
                cps[u] = nps[u];
                cg1[u] = ng1[u];
                cil[u] = nil[u];
            }
        }
    }
    for (; z < zend; z++) {
        one_row(z);
        advance<1, BX>(q, colz, z + 1 - z0, z + 1 < zend);
    }
}

// =====================================================================================
// Host launchers.
template <int BZ>
static size_t vel_smem() { return (size_t)(BZ + QNV_MAX - 1) * WW * sizeof(float); }
template <int BZ>
static size_t pres_smem() { return ((size_t)BZ * WW + (size_t)(BZ + QNP_MAX - 1) * BX) * sizeof(float); }

// The dynamic shared-memory limit of a kernel is an attribute of the kernel's instance on
// each device, so it is set once per device (bit d of `done`; a repeated set is harmless, so
// two host threads that meet here first both set it).
template <typename F>
static void set_smem_once(std::atomic<unsigned long long> &done, F *fn, size_t bytes)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;   // the launch reports the error
    const unsigned long long bit = (dev >= 0 && dev < 64) ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (bit) done.fetch_or(bit, std::memory_order_release);
}

template <int BZ, int MODE>
static void vel_launch(const StepArgs &a, int ntiles, cudaStream_t s)
{
    static std::atomic<unsigned long long> done{0};
    set_smem_once(done, k_vel<BZ, MODE>, vel_smem<BZ>());
    k_vel<BZ, MODE><<<ntiles, BX, vel_smem<BZ>(), s>>>(a);
}
template <int BZ, int MODE, typename ACC>
static void pres_launch_t(const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    static std::atomic<unsigned long long> done{0};
    set_smem_once(done, k_pres<BZ, MODE, ACC>, pres_smem<BZ>());
    k_pres<BZ, MODE, ACC><<<ntiles, BX, pres_smem<BZ>(), s>>>(a, record);
}
template <int BZ, int MODE>
static void pres_launch(const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if constexpr (MODE == 2) {
        if (a.accum_fp64) {
            pres_launch_t<BZ, MODE, double>(a, ntiles, record, s);
            return;
        }
    }
    pres_launch_t<BZ, MODE, float>(a, ntiles, record, s);
}

template <int MODE>
static void vel_dispatch(int bz, const StepArgs &a, int ntiles, cudaStream_t s)
{
    if (bz == 16) vel_launch<16, MODE>(a, ntiles, s);
    else if (bz == 8) vel_launch<8, MODE>(a, ntiles, s);
    else if (bz == 64) vel_launch<64, MODE>(a, ntiles, s);
    else vel_launch<32, MODE>(a, ntiles, s);
}
template <int MODE>
static void pres_dispatch(int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if (bz == 16) pres_launch<16, MODE>(a, ntiles, record, s);
    else if (bz == 8) pres_launch<8, MODE>(a, ntiles, record, s);
    else if (bz == 64) pres_launch<64, MODE>(a, ntiles, record, s);
    else pres_launch<32, MODE>(a, ntiles, record, s);
}

void launch_vel(int mode, int bz, const StepArgs &a, int ntiles, cudaStream_t s)
{
    switch (mode) {
    case RTM_WAVE_FWD: vel_dispatch<0>(bz, a, ntiles, s); break;
    case RTM_WAVE_RECEIVER: vel_dispatch<2>(bz, a, ntiles, s); break;
    default: vel_dispatch<3>(bz, a, ntiles, s); break;
    }
}
void launch_pres(int mode, int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    switch (mode) {
    case RTM_WAVE_FWD: pres_dispatch<0>(bz, a, ntiles, record, s); break;
    case RTM_WAVE_RECEIVER: pres_dispatch<2>(bz, a, ntiles, 0, s); break;
    default: pres_dispatch<3>(bz, a, ntiles, 0, s); break;
    }
}
