// rtm_stencil_common.cuh — device helpers shared by the stencil kernels (rtm_stencil.cu:
// one column per thread; rtm_stencil_v.cu: four columns by U rows per thread): tile staging
// by the tensor memory accelerator with bounded waits, strip indexing, and the update
// formulas, rounded operation by operation so that every kernel form gives the same bits.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

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
// Before an mbarrier's memory is initialised again (a block that stages one tile after
// another), the old object is invalidated; every wait on it has completed by then.
__device__ __forceinline__ void mbar_inval(unsigned long long *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
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
// True once the barrier's phase of the given parity (0: the first phase after init) is done.
__device__ __forceinline__ bool mbar_done(unsigned long long *bar, unsigned parity = 0)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the tile; on giving up, flag the error, wait once more (bounded) for the copies
// still in flight and report false, so that the block returns without computing.
__device__ __forceinline__ bool tile_wait(unsigned long long *bar, int *err, unsigned parity = 0)
{
    for (long i = 0; i < kWaitLimit; i++)
        if (mbar_done(bar, parity)) return true;
    // the first block to give up records where: its index, the barrier's shared address and
    // its 64-bit state word (err[1..5]; the host adds them to the error message)
    if (atomicCAS(err + 1, 0, 1) == 0) {
        unsigned long long w;
        asm volatile("ld.shared.b64 %0, [%1];\n" : "=l"(w) : "r"(smem_u32(bar)) : "memory");
        err[2] = (int)blockIdx.x;
        err[3] = (int)smem_u32(bar);
        err[4] = (int)(unsigned)w;
        err[5] = (int)(unsigned)(w >> 32);
    }
    atomicExch(err, 1);
    for (long i = 0; i < kWaitLimit; i++)
        if (mbar_done(bar, parity)) break;
    return false;
}
// Fixed-grid launches: true for the blocks past the batch's tile list (see StepArgs::counts).
__device__ __forceinline__ bool tile_beyond(const StepArgs &a) { return a.counts && (int)blockIdx.x >= a.counts[a.list]; }

// L2 prefetch of the operand rows of a tile: rows [z0, z1) of columns [x0, x0 + BX) of nf
// fields (element sizes es), one bulk prefetch per row and field, spread over the block's
// threads.  The kernels then find their per-cell operands in L2 instead of waiting on DRAM
// row group by row group.  Rows stop at the row pitch (x0 and the pitch are multiples of 4
// elements, so every address and size is a multiple of 16 bytes).
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}
// Rows [z0, z1) of one field, issued by the lanes of warp `w` of the block (wrapped to the
// block's warps).
__device__ __forceinline__ void prefetch_rows(const void *field, int es, int z0, int z1, int x0, int pitch, int w)
{
    if ((int)(threadIdx.x >> 5) != w % (int)(blockDim.x >> 5)) return;
    const unsigned bytes = (unsigned)(min(RTM_BX, pitch - x0) * es);
    for (int z = z0 + (int)(threadIdx.x & 31); z < z1; z += 32)
        prefetch_l2((const char *)field + ((size_t)z * pitch + x0) * es, bytes);
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
__device__ __forceinline__ ACC image_g1(ACC og1, float ps, float pn) { return og1 + (ACC)ps * (ACC)pn; }
template <typename ACC>
__device__ __forceinline__ ACC image_il(ACC oil, float ps) { return oil + (ACC)ps * (ACC)ps; }
// Compensated fp32 accumulator (Kahan): the running sum s and the compensation c, whose
// negative is the low-order part lost so far, so the sum is s - c.  Each term enters as
// fma(a, b, -c), the product exact before its one rounding.
__device__ __forceinline__ KahanAcc kahan_add(KahanAcc o, float a, float b)
{
    const float y = __fmaf_rn(a, b, -o.c);
    const float t = __fadd_rn(o.s, y);
    KahanAcc r;
    r.c = __fsub_rn(__fsub_rn(t, o.s), y);
    r.s = t;
    return r;
}
template <>
__device__ __forceinline__ KahanAcc image_g1<KahanAcc>(KahanAcc og1, float ps, float pn) { return kahan_add(og1, ps, pn); }
template <>
__device__ __forceinline__ KahanAcc image_il<KahanAcc>(KahanAcc oil, float ps) { return kahan_add(oil, ps, ps); }
template <typename ACC>
__device__ __forceinline__ void image_cell(ACC *__restrict__ g1p, ACC *__restrict__ ilp, unsigned id, ACC og1, ACC oil,
                                           float ps, float pn)
{
    g1p[id] = image_g1<ACC>(og1, ps, pn);
    ilp[id] = image_il<ACC>(oil, ps);
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

// x-derivatives of the U rows of one column group (U even) with rows u and u+1 as the two
// lanes of packed fp32 pairs (sm_100: one instruction for both lanes): each lane takes the
// difference, then a fused multiply-add, in tap order, as tap_sum's sum is compiled, so the
// results are tap_sum's bits with half the arithmetic instructions.  Row u's staged row
// starts at rw + u * WW; f(i) = row[i + FO], g(i) = row[GO - i].
template <int U, int FO, int GO, typename C>
__device__ __forceinline__ void dx_pairs(const float *rw, float (&dx)[U], C c)
{
    static_assert(U % 2 == 0, "rows are paired");
#pragma unroll
    for (int u = 0; u < U; u += 2) {
        const float *r0 = rw + u * WW, *r1 = r0 + WW;
        float2 s = make_float2(0.f, 0.f);
#pragma unroll
        for (int i = 1; i <= R; i++) {
            const float ci = c(i - 1);
            const float2 d = __fadd2_rn(make_float2(r0[i + FO], r1[i + FO]), make_float2(-r0[GO - i], -r1[GO - i]));
            s = __ffma2_rn(make_float2(ci, ci), d, s);
        }
        dx[u] = s.x;
        dx[u + 1] = s.y;
    }
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

// New vx / vz of one existing cell (x, z) from the raw derivative sums, for kernels that
// write every cell of a second buffer: the damped update (modes 0 and 2); in the
// reconstruction, the interior update, the restored strip of step it+1, or the old value
// where the reconstruction leaves the cell alone.  Same operations as vel_apply.
template <int MODE>
__device__ __forceinline__ float vx_value(const StepArgs &a, const ShotDev &S, const ShotK &k, const PmlOffsets &o,
                                          int x, int z, int X, int Z, int npml, float dx, float ir, float ov)
{
    if (MODE == 3) {
        const bool zin = (z >= npml && z < Z - npml);
        if (zin && x >= npml && x <= X - npml - 2) return __fadd_rn(ov, vel_inc(dx, a.dtx, ir));
        const int svx = strip_col_vx(x, X, npml, k.nzi);
        if (zin && svx >= 0) {   // read_d_vxpml, kernel.cu:1294-1320
            const float sc = a.strip_prec ? S.strip_scale[(size_t)(a.it + 1) * 4 + 0] : 1.0f;
            return load_strip(S.strips, (size_t)(a.it + 1) * k.strip_len + svx + (size_t)(z - npml) * R, a.strip_prec,
                              sc);
        }
        return ov;
    }
    const bool band = (x < npml) || (x >= X - npml - 1);
    const float c1 = band ? S.pml[o.c1vx + x] : 1.0f, ic2 = band ? S.pml[o.ic2vx + x] : 1.0f;
    return damp(ov, vel_inc(dx, a.dtx, ir), c1, ic2);
}
template <int MODE>
__device__ __forceinline__ float vz_value(const StepArgs &a, const ShotDev &S, const ShotK &k, const PmlOffsets &o,
                                          int x, int z, int X, int Z, int npml, float dz, float ir, float ow)
{
    if (MODE == 3) {
        const bool xin = (x >= npml && x < X - npml);
        if (z >= npml && z <= Z - npml - 2 && xin) return __fadd_rn(ow, vel_inc(dz, a.dtz, ir));
        if (xin) {
            const int srow = strip_row_tb(z, npml, Z - npml - 1, k.nxi);
            if (srow >= 0) {   // read_d_vzpml, kernel.cu:1321-1347
                const float sc = a.strip_prec ? S.strip_scale[(size_t)(a.it + 1) * 4 + 1] : 1.0f;
                return load_strip(S.strips, (size_t)(a.it + 1) * k.strip_len + 2 * (size_t)R * k.nzi + srow + (x - npml),
                                  a.strip_prec, sc);
            }
        }
        return ow;
    }
    return damp(ow, vel_inc(dz, a.dtz, ir), S.pml[o.c1vz + z], S.pml[o.ic2vz + z]);
}

// Per-column constants of the pressure update.
struct PresCol {
    bool xb, xin;        // column in the x PML band / in the image interior
    bool srcc, recc;     // column in the source box / on the receiver line
    float c1x, ic2x;     // x damping of this column
    int splr, sptb;      // strip columns of the reconstruction (-1: none)
};

// Pressure update of one cell (x, z) from the raw derivative sums dx, dz; `upd` is false on
// the grid's edge rows and columns, which keep their pressure (kernel.cu:714-1185).  Returns the
// cell's new pressure (its old one where nothing changes it) and sets *wr when the one-buffer
// kernels must store it; the split fields, the recorded gather and the imaging accumulators are
// written here.
template <int MODE, typename ACC>
__device__ __forceinline__ float pres_value(const StepArgs &a, const ShotDev &S, const ShotK &k, const PresCol &cc,
                                            float wit, float *__restrict__ sxp, float *__restrict__ szp,
                                            ACC *__restrict__ g1p, ACC *__restrict__ ilp, unsigned id, int x, int z,
                                            int Z, int npml, bool upd, float dx, float dz, float kk, float p0,
                                            float s1o, float s2o, float ps, ACC og1, ACC oil, float c1z, float ic2z,
                                            int record, bool *wr_out)
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
        *wr_out = wr;
        return pn;
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
        if (record && z == k.rz && cc.recc)   // kernel.cu:48-71
            ((float *)S.gather)[(size_t)a.it * k.nrec + (x - k.rx0)] = pn;
    } else {
        if (z == k.rz && cc.recc) {   // kernel.cu:72-95 (overwrite)
            pn = a.dt * gather_at(a, S, x - k.rx0);
            wr = true;
        }
        if (zin && cc.xin) image_cell<ACC>(g1p, ilp, id, og1, oil, ps, pn);   // kernel.cu:1401-1416
    }
    *wr_out = wr;
    return pn;
}

template <int MODE, typename ACC>
__device__ __forceinline__ void pres_apply(const StepArgs &a, const ShotDev &S, const ShotK &k, const PresCol &cc,
                                           float wit, float *__restrict__ pp, float *__restrict__ sxp,
                                           float *__restrict__ szp, ACC *__restrict__ g1p, ACC *__restrict__ ilp,
                                           unsigned id, int x, int z, int Z, int npml, bool upd, float dx,
                                           float dz, float kk, float p0, float s1o, float s2o, float ps, ACC og1,
                                           ACC oil, float c1z, float ic2z, int record)
{
    bool wr;
    const float pn = pres_value<MODE, ACC>(a, S, k, cc, wit, sxp, szp, g1p, ilp, id, x, z, Z, npml, upd, dx, dz, kk, p0,
                                           s1o, s2o, ps, og1, oil, c1z, ic2z, record, &wr);
    if (wr) pp[id] = pn;
}

}  // namespace
