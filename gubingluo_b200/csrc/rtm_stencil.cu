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
//     zero-padded table (the choice is per warp or per tile, so warps do not diverge); rows
//     left over after the last whole group take a compact one-row path;
//   * PML damping, split pressure, source, receivers, strip restore and imaging are per-row
//     or per-column predicates of the same kernel (strips are saved by k_strip_save after
//     each forward step).
// Reference equivalents (gubingluo kernel.cu): forward v :430-500 + :542-713, forward p
// :501-541 + :714-1185, reconstruction :318-429, strip restore :1294-1400, source :36-47,
// receivers :48-95, cross-correlation :1401-1416.
#include <algorithm>
#include <atomic>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "rtm_launch.h"
#include "rtm_types.h"

#include "rtm_stencil_common.cuh"
#include "rtm_strip.cuh"

// =====================================================================================
// Velocity update.  MODE 0: forward, full grid; 2: receiver (backward model), full grid;
// 3: reconstruction of the source wavefield (interior only, vx/vz strips of step it+1
// restored).
// Register budget (measured): 6 blocks per SM (80 registers, no spills) for the reconstruction
// and for the 32-row forward and receiver tiles (whose 33 KB of staged rows allow no more),
// 8 (64 registers, no spills) for the 8- and 16-row forward and receiver tiles, 5 for the
// 8-row reconstruction tiles (which would spill at 6); with its interior-tile body the
// reconstruction runs 4% faster at 6 than at 5.
// The work of one block on tile t (the kernels below, and the persistent pass kernel);
// `sw` is the block's dynamic shared memory; `use`: how many tiles the block has staged with
// this function before (the first use initialises the mbarrier, use n waits for its phase n).
template <int BZ, int MODE>
__device__ __forceinline__ void vel_tile(const StepArgs &a, const TileRef t, float *sw, unsigned use = 0)
{
    constexpr int U = MODE == 3 ? UVR : UV, QN = 2 * R + U - 1;
    static_assert(BZ % U == 0, "interior tiles take whole row groups");
    constexpr int WH = BZ + QNV_MAX - 1;   // staged rows z0-9 .. z0+BZ+QNV_MAX-11 (the box height)
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ float s_tab[100];
    __shared__ float s_c1vz[BZ], s_ic2vz[BZ];
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = t.x0, z0 = t.z0;
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ inv_rho = (MODE >= 2) ? S.inv_rho_b : S.inv_rho_f;
    const PmlOffsets o = pml_offsets(X, Z);
    if (threadIdx.x == 0) {   // p rows z0-9 .. z0+BZ+12, columns x0-12 .. x0+139
        if (use == 0) mbar_init(&s_bar);   // a persistent block keeps it between its tiles
        mbar_expect(&s_bar, WH * WW * sizeof(float));
        tma_box(sw, tmap_of(S, MODE == 2 ? RTM_TMAP_B_P : (MODE == 3 ? RTM_TMAP_A_P_RECON : RTM_TMAP_A_P)), x0 - 12,
                z0 - 9, &s_bar);
    }
    if (a.prefetch) {   // the tile's 1/rho, vx, vz rows into L2
        const int z1 = min(z0 + BZ, Z);
        prefetch_rows(inv_rho, 4, z0, z1, x0, pitch, 1);
        prefetch_rows(W.vx, 4, z0, z1, x0, pitch, 2);
        prefetch_rows(W.vz, 4, z0, z1, x0, pitch, 3);
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
    // Warps whose columns, or whose tile's rows, reach the outer ten cells of the grid take the
    // table-coefficient form of the unrolled groups: vx order per column (cuda_norderx), vz
    // order per row (cuda_norderz).  The others have the full order everywhere, whose table
    // row equals the constant coefficients, so either form gives the same bits; the choice is
    // per warp, so warps do not diverge.  The reconstruction writes only cells at least
    // npml >= R from the edge, where every order is full.
    const int xw0 = x0 + (tx & ~31);
    const bool edge_tile = MODE != 3 && (xw0 < R || xw0 + 32 > X - R || z0 < R || zend > Z - R);
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
    // the reconstruction leaves every column outside [npml-R, X-npml+R) alone
    const bool dead = x >= X || (MODE == 3 && (x < npml - R || x >= X - npml + R));
    if (!dead && z0 + U <= zend) load_group(z0, cir, cov, cow);
    __syncthreads();
    if (!tile_wait(&s_bar, a.err, use & 1u) || dead) return;   // no barrier below

    const float *col = &sw[tx + 12];   // staged column x: col[r*WW] = p[z0-9+r][x]
    float q[QN];                        // q[k] = p[z-9+k][x] at the current row z
#pragma unroll
    for (int j = 0; j < QN; j++) q[j] = col[j * WW];

    // interior tiles (TileRef.interior: every column in [npml, X-npml-1), every row in
    // [npml, Z-npml-1), where the velocity damping is 1 and no strip lies): the update
    // alone, in the arithmetic of the general body.  The 32-row forward and receiver tiles
    // unroll four row groups, so that the z window's shift becomes register renaming within
    // them (measured 1.5-2.5% faster; the pressure kernels and the smaller tiles were not
    // faster that way, or spilled)
    if (t.interior) {
#pragma unroll (MODE == 3 || BZ < 32 ? 1 : 4)
        for (int z = z0; z < z0 + BZ; z += U) {
            float nir[U], nov[U], now[U];
            const bool more = z + 2 * U <= z0 + BZ;
            if (more) load_group(z + U, nir, nov, now);
            const unsigned id0 = (unsigned)z * pitch + x;
            // x-derivatives in row pairs, the forward and receiver passes (0.5% faster; the
            // reconstruction's 4-row groups keep the scalar sums: paired, their registers spill)
            float dxs[U];
            if (MODE != 3) dx_pairs<U, 0, 1>(&col[(z - z0 + 9) * WW], dxs, [&](int j) { return a.c10[j]; });
#pragma unroll
            for (int u = 0; u < U; u++) {
                const float *rw = &col[(z + u - z0 + 9) * WW];
                const float dx = MODE != 3 ? dxs[u]
                                           : tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return rw[i]; },
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
        float dxs[U];
        if (MODE != 3 && !edge_tile) dx_pairs<U, 0, 1>(&col[(z - z0 + 9) * WW], dxs, [&](int j) { return a.c10[j]; });
#pragma unroll
        for (int u = 0; u < U; u++) {
            const float *rw = &col[(z + u - z0 + 9) * WW];
            float dx, dz;
            if (!edge_tile) {
                dx = MODE != 3 ? dxs[u]
                               : tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return rw[i]; },
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
// receiver passes in their 2-row groups (8 at 64 registers for the forward pass's 8-row
// tiles; the receiver pass spills there), 6 (80 registers) for the reconstruction in 4-row
// groups, 4 for the receiver pass with fp64 accumulators (123 registers).  With 4-row groups
// the receiver pass needed 96 registers (5 blocks) and spilled when capped at 6.
//
// Interior tiles (TileRef.interior, set by the host for tiles whose every column lies in
// [npml, X-npml) and every row in [npml, Z-npml), with no source cell and no receiver) take
// a second body in the same kernel, chosen per block: the interior update alone, with no
// PML, source or receiver tests and no split-field loads, in the arithmetic of the general
// body's interior branch (for the reconstruction: tiles of the interior with no source cell).
template <int BZ, int MODE, typename ACC>
__device__ __forceinline__ void pres_tile(const StepArgs &a, int record, const TileRef t, float *sm, unsigned use = 0)
{
    constexpr int U = MODE == 2 ? UPR : MODE == 3 ? UPC : UP, QN = 2 * R + U - 1;
    static_assert(BZ % U == 0, "interior tiles take whole row groups");
    constexpr int XH = BZ;            // vx rows z0 .. z0+BZ-1, columns x0-12 .. x0+BX+11
    constexpr int ZH = BZ + QNP_MAX - 1;   // vz rows z0-10 .. z0+BZ+QNP_MAX-12 (the box height), columns x0 ..
    float *svx = sm;
    float *svz = sm + XH * WW;   // XH * WW * 4 bytes is a multiple of 128
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ float s_tab[100];
    __shared__ float s_c1z[BZ], s_ic2z[BZ];
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = t.x0, z0 = t.z0;
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ kappa = (MODE >= 2) ? S.kappa_b : S.kappa_f;
    const PmlOffsets o = pml_offsets(X, Z);
    if (threadIdx.x == 0) {   // vx rows z0 .. z0+BZ-1 (columns x0-12 ..), vz rows z0-10 .. z0+BZ+11
        if (use == 0) mbar_init(&s_bar);   // a persistent block keeps it between its tiles
        mbar_expect(&s_bar, (XH * WW + ZH * BX) * sizeof(float));
        const int mvx = MODE == 2 ? RTM_TMAP_B_VX : MODE == 3 ? RTM_TMAP_A_VX_RECON : RTM_TMAP_A_VX;
        const int mvz = MODE == 2 ? RTM_TMAP_B_VZ : MODE == 3 ? RTM_TMAP_A_VZ_RECON : RTM_TMAP_A_VZ;
        tma_box(svx, tmap_of(S, mvx), x0 - 12, z0, &s_bar);
        tma_box(svz, tmap_of(S, mvz), x0, z0 - 10, &s_bar);
    }
    if (a.prefetch) {   // the tile's kappa and p rows (split fields, imaging operands) into L2
        const int z1 = min(z0 + BZ, Z);
        prefetch_rows(kappa, 4, z0, z1, x0, pitch, 1);
        prefetch_rows(W.p, 4, z0, z1, x0, pitch, 2);
        if (MODE != 3 && !t.interior) {
            prefetch_rows(W.sx, 4, z0, z1, x0, pitch, 3);
            prefetch_rows(W.sz, 4, z0, z1, x0, pitch, 4);
        }
        if (MODE == 2) {   // imaging operands of the interior rows
            const int i0 = max(z0, npml), i1 = min(z1, Z - npml);
            prefetch_rows(S.a.p, 4, i0, i1, x0, pitch, 5);
            prefetch_rows(S.g1, (int)sizeof(ACC), i0, i1, x0, pitch, 6);
            prefetch_rows(S.illum, (int)sizeof(ACC), i0, i1, x0, pitch, 7);
        }
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
    // warps whose columns, or whose tile's rows, reach the outer ten cells take the
    // table-coefficient form of the groups (per warp, as in the velocity kernel; per tile in
    // the receiver pass, whose larger body ran 2-4% slower with the choice per warp)
    const int xw0 = MODE == 2 ? x0 : x0 + (tx & ~31), xw1 = MODE == 2 ? x0 + BX : xw0 + 32;
    const bool edge_tile = MODE != 3 && (xw0 < R || xw1 > X - R || z0 < R || zend > Z - R);
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
    // the reconstruction leaves every column outside [npml-R, X-npml+R) alone
    const bool dead = x >= X || (MODE == 3 && (x < npml - R || x >= X - npml + R));
    if (!dead && z0 + U <= zend) load_group(z0, ckk, cp0, cs1, cs2, cps, cg1, cil);
    __syncthreads();
    if (!tile_wait(&s_bar, a.err, use & 1u) || dead) return;

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
            // the forward pass takes its x-derivatives in row pairs (2.3% faster); the receiver
            // and reconstruction passes were not faster that way (4% slower at 32-row tiles)
            float dxs[U];
            if (MODE == 0) dx_pairs<U, -1, 0>(&colx[(z - z0) * WW], dxs, [&](int j) { return a.c10[j]; });
            if constexpr (MODE == 0 && U == 2) {
                // the update of both rows in packed pairs as well: per lane the products and the
                // separately rounded sum and difference of p_interior, so the same bits
                float dz2[2];
#pragma unroll
                for (int u = 0; u < 2; u++)
                    dz2[u] = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return q[u + 9 + i]; },
                                     [&](int i) { return q[u + 10 - i]; });
                const float2 kk = make_float2(ckk[0], ckk[1]);
                const float2 dxs2 = __fmul2_rn(__fmul2_rn(make_float2(dxs[0], dxs[1]), make_float2(a.dtx, a.dtx)), kk);
                const float2 dzs2 = __fmul2_rn(__fmul2_rn(make_float2(dz2[0], dz2[1]), make_float2(a.dtz, a.dtz)), kk);
                const float2 sum = __fadd2_rn(dxs2, dzs2);
                const float2 pn = __fadd2_rn(make_float2(cp0[0], cp0[1]), make_float2(-sum.x, -sum.y));
                pp[id0] = pn.x;
                pp[id0 + pitch] = pn.y;
            } else {
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const float *rw = &colx[(z + u - z0) * WW];
                    const float dx = MODE == 0 ? dxs[u]
                                               : tap_sum([&](int j) { return a.c10[j]; },
                                                         [&](int i) { return rw[i - 1]; }, [&](int i) { return rw[-i]; });
                    const float dz = tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return q[u + 9 + i]; },
                                             [&](int i) { return q[u + 10 - i]; });
                    const float ddx = dx * a.dtx, ddz = dz * a.dtz;
                    const float pn = MODE == 3 ? p_recon(cp0[u], ddx * ckk[u], ddz * ckk[u])
                                               : p_interior(cp0[u], ddx * ckk[u], ddz * ckk[u]);
                    const unsigned id = id0 + u * pitch;
                    pp[id] = pn;
                    if (MODE == 2) image_cell<ACC>(g1p, ilp, id, cg1[u], cil[u], cps[u], pn);
                }
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
        float dxs[U];
        if (MODE == 0 && !edge_tile) dx_pairs<U, -1, 0>(&colx[(z - z0) * WW], dxs, [&](int j) { return a.c10[j]; });
#pragma unroll
        for (int u = 0; u < U; u++) {
            const float *rw = &colx[(z + u - z0) * WW];
            float dx, dz;
            bool upd = true;
            if (!edge_tile) {
                dx = MODE == 0 ? dxs[u]
                               : tap_sum([&](int j) { return a.c10[j]; }, [&](int i) { return rw[i - 1]; },
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

// The kernels: one block per tile of the launch's list (reconstruction: tiles of the
// interior and its strips only).
template <int BZ, int MODE>
__global__ void __launch_bounds__(BX, MODE == 3 ? (BZ == 8 ? 5 : RTM_VEL_RECON_BLOCKS) : BZ <= 16 ? 8 : 6)
    k_vel(const StepArgs a)
{
    extern __shared__ __align__(128) float sw[];
    if (tile_beyond(a)) return;   // fixed-grid launch: past this batch's tiles
    vel_tile<BZ, MODE>(a, a.tiles[blockIdx.x], sw);
}
template <int BZ, int MODE, typename ACC>
__global__ void __launch_bounds__(BX, MODE == 2   ? (sizeof(ACC) == 8 ? 4 : RTM_PRES_RECV_BLOCKS)
                                     : MODE == 3 ? RTM_PRES_RECON_BLOCKS
                                                 : BZ == 8 ? 8 : RTM_PRES_FWD_BLOCKS)
    k_pres(const StepArgs a, int record)
{
    extern __shared__ __align__(128) float sm[];
    if (tile_beyond(a)) return;
    pres_tile<BZ, MODE, ACC>(a, record, a.tiles[blockIdx.x], sm);
}

// =====================================================================================
// Persistent passes: every step of a pass in one launch (PassArgs).  Blocks claim items in
// queue order; an item waits only for items earlier in the queue, which blocks that are
// running have claimed, so the queue always drains.  Each wait is bounded (wait_ns of the
// global timer, and the error flag of any other block): on giving up, the block sets the
// error flag to 2 and every block leaves at its next item.  One block per SM slot, 128
// threads, the tile functions of the kernels above.

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ long long global_ns()
{
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Thread 0: wait until *c >= target (or give up: error flag 2).  Then order the items' writes
// before this block's tensor-memory loads (async proxy).
__device__ __forceinline__ bool wait_done(const unsigned *c, unsigned target, const PassArgs &P)
{
    if (ld_acquire(c) < target) {
        const long long t0 = global_ns();
        while (ld_acquire(c) < target) {
            if (global_ns() - t0 > P.wait_ns || *(volatile int *)P.a.err) {
                atomicCAS(P.a.err, 0, 2);
                return false;
            }
            __nanosleep(100);
        }
    }
    asm volatile("fence.proxy.async.global;\n" ::: "memory");
    return true;
}

// DIR 0: source pass (velocity, pressure, strip save per step; mode 0, strips fp32);
// DIR 1: backward pass (reconstruction velocity and pressure, receiver velocity and pressure
// with imaging).
template <int BZV, int BZVR, int BZP, typename ACC, int DIR>
__global__ void __launch_bounds__(BX, DIR == 0 ? 5 : 4) k_pass(const PassArgs P)
{
    extern __shared__ __align__(128) float sm[];
    __shared__ unsigned s_item;
    __shared__ int s_ok;
    const int n = P.nshots;
    const int ns = (DIR == 0 && P.save) ? n : 0;
    const int per = DIR == 0 ? P.len[0] + P.len[1] + ns : P.len[0] + P.len[1] + P.len[2] + P.len[3];
    const unsigned total = (unsigned)per * (unsigned)P.nsteps;
    const int *cnt = P.per_shot;
    unsigned uses[4] = {0, 0, 0, 0};   // tiles this block has staged with each phase's function
    for (;;) {
        __syncthreads();   // the previous item's shared memory is free
        if (threadIdx.x == 0) s_item = *(volatile int *)P.a.err ? total : atomicAdd(P.queue, 1u);
        __syncthreads();
        const unsigned item = s_item;
        if (item >= total) return;
        if (threadIdx.x == 0 && (int)blockIdx.x < P.trace_len) P.trace[blockIdx.x] = item;
        const int k = (int)(item / per);
        int r = (int)(item - (unsigned)k * per);
        StepArgs a = P.a;
        int ph, s;
        TileRef t{};
        if (DIR == 0) {
            a.it = k;
            a.ring = k % 32;
            if (r < P.len[0]) ph = 0, t = P.list[0][r], s = t.shot;
            else if (r < P.len[0] + P.len[1]) ph = 1, t = P.list[1][r - P.len[0]], s = t.shot;
            else ph = 2, s = r - P.len[0] - P.len[1];
        } else {
            a.it = P.nt - 2 - k;
            ph = 0;
            while (r >= P.len[ph]) r -= P.len[ph++];
            t = P.list[ph][r];
            s = t.shot;
        }
        if (threadIdx.x == 0) {
            bool ok = true;
            const unsigned *d = P.done;
            const int B = P.B;
            if (DIR == 0) {
                if (ph == 0) ok = ns ? wait_done(&d[2 * B + s], (unsigned)k, P)
                                     : wait_done(&d[1 * B + s], (unsigned)(k * cnt[1 * B + s]), P);
                else if (ph == 1) ok = wait_done(&d[0 * B + s], (unsigned)((k + 1) * cnt[0 * B + s]), P);
                else ok = wait_done(&d[1 * B + s], (unsigned)((k + 1) * cnt[1 * B + s]), P);
            } else {
                // 0 recon vel: after recon pres of step k-1; 1 recon pres: after recon vel of k and
                // the receiver pressure of k-1 (its imaging read the pressure being replaced);
                // 2 receiver vel: after receiver pres of k-1; 3 receiver pres: after receiver vel
                // of k and recon pres of k (its imaging reads that pressure)
                if (ph == 0) ok = wait_done(&d[1 * B + s], (unsigned)(k * cnt[1 * B + s]), P);
                else if (ph == 1) ok = wait_done(&d[0 * B + s], (unsigned)((k + 1) * cnt[0 * B + s]), P) &&
                                       wait_done(&d[3 * B + s], (unsigned)(k * cnt[3 * B + s]), P);
                else if (ph == 2) ok = wait_done(&d[3 * B + s], (unsigned)(k * cnt[3 * B + s]), P);
                else ok = wait_done(&d[2 * B + s], (unsigned)((k + 1) * cnt[2 * B + s]), P) &&
                          wait_done(&d[1 * B + s], (unsigned)((k + 1) * cnt[1 * B + s]), P);
            }
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) return;
        unsigned use = 0;
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (q == ph) use = uses[q]++;
        if (DIR == 0) {
            if (ph == 0) vel_tile<BZV, 0>(a, t, sm, use);
            else if (ph == 1) pres_tile<BZP, 0, float>(a, P.record, t, sm, use);
            else {
                const ShotDev &S = a.shots[s];
                for (int i = threadIdx.x; i < S.strip_len; i += BX) strip_save_cell(S, i, k, a.ring, P.strip_prec);
            }
        } else {
            if (ph == 0) vel_tile<BZVR, 3>(a, t, sm, use);
            else if (ph == 1) pres_tile<BZP, 3, float>(a, 0, t, sm, use);
            else if (ph == 2) vel_tile<BZV, 2>(a, t, sm, use);
            else pres_tile<BZP, 2, ACC>(a, 0, t, sm, use);
        }
        __syncthreads();   // every thread's writes of the item are done
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&P.done[ph * P.B + s], 1u);
        }
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
        if (a.accum_fp64 == RTM_ACC_FP64) {
            pres_launch_t<BZ, MODE, double>(a, ntiles, record, s);
            return;
        }
        if (a.accum_fp64 == RTM_ACC_KAHAN) {
            pres_launch_t<BZ, MODE, KahanAcc>(a, ntiles, record, s);
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

// Persistent passes at the default tile heights (32-row forward/receiver velocity tiles,
// 16-row reconstruction velocity and pressure tiles).  Returns false when the heights differ.
template <int DIR, typename ACC>
static void pass_launch_t(const PassArgs &p, int bzv, int bzp, cudaStream_t s)
{
    constexpr int BZV = 32, BZVR = 16, BZP = 16;
    static std::atomic<unsigned long long> done{0};
    const size_t bytes = std::max(std::max(vel_smem<BZV>(), vel_smem<BZVR>()), pres_smem<BZP>());
    set_smem_once(done, k_pass<BZV, BZVR, BZP, ACC, DIR>, bytes);
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pass<BZV, BZVR, BZP, ACC, DIR>, BX, bytes);
    (void)bzv;
    (void)bzp;
    k_pass<BZV, BZVR, BZP, ACC, DIR><<<sms * std::max(per_sm, 1), BX, bytes, s>>>(p);
}
bool launch_pass(int dir, const PassArgs &p, int bz_vel, int bz_vel_recon, int bz_pres, cudaStream_t s)
{
    if (bz_vel != 32 || bz_vel_recon != 16 || bz_pres != 16) return false;
    if (dir == 0) pass_launch_t<0, float>(p, bz_vel, bz_pres, s);
    else if (p.a.accum_fp64 == RTM_ACC_FP64) pass_launch_t<1, double>(p, bz_vel, bz_pres, s);
    else if (p.a.accum_fp64 == RTM_ACC_KAHAN) pass_launch_t<1, KahanAcc>(p, bz_vel, bz_pres, s);
    else pass_launch_t<1, float>(p, bz_vel, bz_pres, s);
    return true;
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
