// rtm_stencil_v.cu — the velocity and pressure kernels with four columns by U rows per thread
// (sm_100a).
//
// Same launches, tile lists, staged boxes and results (bit for bit) as the one-column kernels
// of rtm_stencil.cu.  Only the mapping of a tile's cells to threads differs: thread (g, r) of
// a block of 32 * BZ / U threads owns the four adjacent columns x0+4g .. x0+4g+3 and the U
// adjacent rows z0+U r .. z0+U r+U-1, so a warp is one group of U rows across the tile's 128
// columns.
//   * An x-derivative of the four columns reads seven 16-byte words of the staged row (the
//     28 values x-12 .. x+15) instead of 4 x 20 single words.
//   * The z-derivatives of the 4 x U cells read the U+19 staged rows they need as 16-byte
//     words, each row serving up to U outputs; the taps are accumulated in the order
//     i = 1 .. 10 of every other form.
//   * Per-cell operands (1/rho, kappa, the old fields, the imaging accumulators) are loaded
//     and, in interior tiles, stored as 16-byte words: field rows start on 128-byte
//     boundaries and x0 is a multiple of 4.
// The update formulas are the shared ones of rtm_stencil_common.cuh (vel_apply, pres_apply,
// damp, vel_inc, p_interior, p_recon, image_cell).  The reference kernels these replace are
// listed in rtm_stencil.cu.
#include <atomic>
#include <type_traits>

#include "rtm_launch.h"
#include "rtm_vec.cuh"


// =====================================================================================
// Velocity update (modes as k_vel in rtm_stencil.cu).  Block: 32 * BZ / U threads.
// Registers: at most 80; the reconstruction in two-row groups at most 72 (7 blocks of 128
// threads per SM at 8-row tiles, no spills), which measured 6% faster than at 79 registers and
// 6 blocks.
template <int BZ, int MODE, int U>
__global__ void __launch_bounds__(32 * BZ / U, min_blocks(32 * BZ / U, MODE == 3 && U == 2 ? 72 : 80)) k_vel4(const StepArgs a)
{
    static_assert(BZ % U == 0, "row groups tile the tile");
    constexpr int WH = BZ + QNV_MAX - 1;   // staged p rows z0-9 .. (the k_vel box)
    static_assert(WH >= BZ + 19, "the staged rows cover the z-derivatives");
    extern __shared__ __align__(128) float sw[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ float s_tab[100];
    __shared__ float s_c1vz[BZ], s_ic2vz[BZ];
    if (tile_beyond(a)) return;   // fixed-grid launch: past this batch's tiles
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = t.x0, z0 = t.z0;
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ inv_rho = (MODE >= 2) ? S.inv_rho_b : S.inv_rho_f;
    const PmlOffsets o = pml_offsets(X, Z);
    if (threadIdx.x == 0) {   // p rows z0-9 .., columns x0-12 .. x0+139
        mbar_init(&s_bar);
        mbar_expect(&s_bar, WH * WW * sizeof(float));
        tma_box(sw, tmap_of(S, MODE == 2 ? RTM_TMAP_B_P : (MODE == 3 ? RTM_TMAP_A_P_RECON : RTM_TMAP_A_P)), x0 - 12,
                z0 - 9, &s_bar);
    }
    for (int i = threadIdx.x; i < 100; i += blockDim.x) s_tab[i] = a.coef[i];
    for (int i = threadIdx.x; i < BZ; i += blockDim.x) {
        const int z = min(z0 + i, Z - 2);
        s_c1vz[i] = S.pml[o.c1vz + z];
        s_ic2vz[i] = S.pml[o.ic2vz + z];
    }
    const int g = threadIdx.x & 31, r = threadIdx.x >> 5;
    const int x = x0 + 4 * g, zr = z0 + U * r;
    float *__restrict__ vxp = W.vx;
    float *__restrict__ vzp = W.vz;
    // (the reconstruction leaves every column outside [npml-R, X-npml+R) alone)
    const bool live = x < X && zr < Z && (MODE != 3 || (x + 4 > npml - R && x < X - npml + R));
    // operands of the thread's cells, loaded while the tile is staged (x < X keeps the four
    // columns inside the row pitch, a multiple of 32 >= X)
    float4 ir[U], ov[U], ow[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const unsigned id = (unsigned)(zr + u) * pitch + x;
        if (live && zr + u < Z) {
            ir[u] = ldg4(&inv_rho[id]);
            ov[u] = ld4(&vxp[id]);
            ow[u] = ld4(&vzp[id]);
        } else {
            ir[u] = ov[u] = ow[u] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    __syncthreads();
    if (!tile_wait(&s_bar, a.err) || !live) return;   // no barrier below

    const float *rowbase = &sw[(U * r + 9) * WW + 4 * g];   // staged row of grid row zr, word of column x-12
    const float *colbase = &sw[(U * r) * WW + 4 * g + 12];  // group's first staged row, word of column x

    if (t.interior) {   // every cell interior, full orders, no strip: the update alone
        float dz[U][4];
        dz4<U, WW>(colbase, dz, [&](int, int, int j) { return a.c10[j]; });
#pragma unroll
        for (int u = 0; u < U; u++) {
            float dx[4];
            dx4<12, 13>(rowbase + u * WW, dx, [&](int, int j) { return a.c10[j]; });
            const unsigned id = (unsigned)(zr + u) * pitch + x;
            float nvx[4], nvz[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float irj = comp(ir[u], j);
                if (MODE == 3) {
                    nvx[j] = __fadd_rn(comp(ov[u], j), vel_inc(dx[j], a.dtx, irj));
                    nvz[j] = __fadd_rn(comp(ow[u], j), vel_inc(dz[u][j], a.dtz, irj));
                } else {
                    nvx[j] = __fsub_rn(comp(ov[u], j), vel_inc(dx[j], a.dtx, irj));
                    nvz[j] = __fsub_rn(comp(ow[u], j), vel_inc(dz[u][j], a.dtz, irj));
                }
            }
            st4(&vxp[id], f4(nvx));
            st4(&vzp[id], f4(nvz));
        }
        return;
    }

    const ShotK k = shot_ints(S);
    const int zend = min(z0 + BZ, Z);
    // tiles that reach the outer ten cells take table coefficients: vx order per column
    // (cuda_norderx), vz order per row (cuda_norderz); the reconstruction writes only cells
    // at least npml >= R from the edge, where every order is full
    const bool edge_tile = MODE != 3 && (x0 < R || x0 + BX > X - R || z0 < R || zend > Z - R);
    auto order = [&](int i, int n) { return max(min(min(i + 1, n - 1 - i), R), 1); };
    float dz[U][4];
    if (!edge_tile) dz4<U, WW>(colbase, dz, [&](int, int, int j) { return a.c10[j]; });
    else dz4<U, WW>(colbase, dz, [&](int u, int, int j) { return s_tab[(order(zr + u, Z) - 1) * R + j]; });
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int z = zr + u;
        if (z >= zend) break;
        float dx[4];
        if (!edge_tile) dx4<12, 13>(rowbase + u * WW, dx, [&](int, int j) { return a.c10[j]; });
        else dx4<12, 13>(rowbase + u * WW, dx, [&](int jj, int j) { return s_tab[(order(x + jj, X) - 1) * R + j]; });
        const unsigned id0 = (unsigned)z * pitch + x;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int xj = x + j;
            if (xj >= X) break;
            VelCol cc;
            cc.hvx = xj < X - 1;
            const bool band = (xj < npml) || (xj >= X - npml - 1);
            cc.c1vx = (band && cc.hvx) ? S.pml[o.c1vx + xj] : 1.0f;
            cc.ic2vx = (band && cc.hvx) ? S.pml[o.ic2vx + xj] : 1.0f;
            cc.svx = (MODE == 3 && cc.hvx) ? strip_col_vx(xj, X, npml, k.nzi) : -1;
            cc.svz = (xj >= npml && xj < X - npml) ? xj - npml : -1;
            cc.rvx = (xj >= npml && xj <= X - npml - 2);
            cc.rvz = (xj >= npml && xj < X - npml);
            vel_apply<MODE>(a, S, k, cc, vxp, vzp, id0 + j, z, Z, npml, dx[j], dz[u][j], comp(ir[u], j),
                            comp(ov[u], j), comp(ow[u], j), s_c1vz[z - z0], s_ic2vz[z - z0]);
        }
    }
}

// =====================================================================================
// Pressure update (modes as k_pres in rtm_stencil.cu).  Block: 32 * BZ / U threads.
// Registers: at most 80 (128 for the receiver pass with its imaging); the reconstruction in
// two-row groups at most 64 (8 blocks of 128 threads per SM at 8-row tiles, no spills), which
// measured 6-9% faster than at 77 registers and 6 blocks.
template <int BZ, int MODE, int U, typename ACC>
__global__ void __launch_bounds__(32 * BZ / U, min_blocks(32 * BZ / U, MODE == 2 ? 128 : MODE == 3 && U == 2 ? 64 : 80)) k_pres4(const StepArgs a, int record)
{
    static_assert(BZ % U == 0, "row groups tile the tile");
    constexpr int XH = BZ;                 // vx rows z0 .. z0+BZ-1, columns x0-12 .. x0+BX+11
    constexpr int ZH = BZ + QNP_MAX - 1;   // vz rows z0-10 .., columns x0 .. x0+BX-1
    static_assert(ZH >= BZ + 19, "the staged rows cover the z-derivatives");
    extern __shared__ __align__(128) float sm[];
    float *svx = sm;
    float *svz = sm + XH * WW;
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ float s_tab[100];
    __shared__ float s_c1z[BZ], s_ic2z[BZ];
    if (tile_beyond(a)) return;   // fixed-grid launch: past this batch's tiles
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = t.x0, z0 = t.z0;
    const WaveDev W = (MODE == 2) ? S.b : S.a;
    const float *__restrict__ kappa = (MODE >= 2) ? S.kappa_b : S.kappa_f;
    const PmlOffsets o = pml_offsets(X, Z);
    if (threadIdx.x == 0) {
        mbar_init(&s_bar);
        mbar_expect(&s_bar, (XH * WW + ZH * BX) * sizeof(float));
        const int mvx = MODE == 2 ? RTM_TMAP_B_VX : MODE == 3 ? RTM_TMAP_A_VX_RECON : RTM_TMAP_A_VX;
        const int mvz = MODE == 2 ? RTM_TMAP_B_VZ : MODE == 3 ? RTM_TMAP_A_VZ_RECON : RTM_TMAP_A_VZ;
        tma_box(svx, tmap_of(S, mvx), x0 - 12, z0, &s_bar);
        tma_box(svz, tmap_of(S, mvz), x0, z0 - 10, &s_bar);
    }
    for (int i = threadIdx.x; i < 100; i += blockDim.x) s_tab[i] = a.coef[i];
    for (int i = threadIdx.x; i < BZ; i += blockDim.x) {
        const int z = min(z0 + i, Z - 1);
        s_c1z[i] = S.pml[o.c1z + z];
        s_ic2z[i] = S.pml[o.ic2z + z];
    }
    const int g = threadIdx.x & 31, r = threadIdx.x >> 5;
    const int x = x0 + 4 * g, zr = z0 + U * r;
    float *__restrict__ pp = W.p;
    float *__restrict__ sxp = W.sx;
    float *__restrict__ szp = W.sz;
    const float *__restrict__ psp = S.a.p;
    ACC *__restrict__ g1p = (ACC *)S.g1;
    ACC *__restrict__ ilp = (ACC *)S.illum;
    // (the reconstruction leaves every column outside [npml-R, X-npml+R) alone)
    const bool live = x < X && zr < Z && (MODE != 3 || (x + 4 > npml - R && x < X - npml + R));
    const int zend = min(z0 + BZ, Z);
    const bool edge_tile = MODE != 3 && (x0 < R || x0 + BX > X - R || z0 < R || zend > Z - R);
    // columns of the x PML band / of the image interior among the thread's four
    bool xb[4], xin[4];
    bool anyxb = false, anyxin = false;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        xb[j] = (x + j < npml) || (x + j >= X - npml);
        xin[j] = !xb[j];
        anyxb |= xb[j];
        anyxin |= xin[j];
    }
    // operands of the thread's cells, loaded while the tile is staged
    float4 kk[U], p0[U], s1[U], s2[U], ps[U];
    ACC og1[U][4], oil[U][4];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int z = zr + u;
        const unsigned id = (unsigned)z * pitch + x;
        const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
        kk[u] = p0[u] = s1[u] = s2[u] = ps[u] = zero;
#pragma unroll
        for (int j = 0; j < 4; j++) og1[u][j] = oil[u][j] = 0;
        if (!live || z >= Z) continue;
        const bool zin = (z >= npml && z < Z - npml);
        kk[u] = ldg4(&kappa[id]);
        if (t.interior || MODE == 3) {
            p0[u] = ld4(&pp[id]);
        } else {
            const bool anyband = anyxb || !zin;
            // a band cell's new p is the sum of its split fields: the old p is needed only
            // for interior cells and, in edge tiles, on the grid's edge rows and columns
            if (edge_tile || anyxin && zin) p0[u] = ld4(&pp[id]);
            if (anyband) {
                s1[u] = ld4(&sxp[id]);
                s2[u] = ld4(&szp[id]);
            }
        }
        if (MODE == 2 && zin && anyxin) {
            ps[u] = ldg4(&psp[id]);
            ld_acc4<ACC>(&g1p[id], og1[u]);
            ld_acc4<ACC>(&ilp[id], oil[u]);
        }
    }
    __syncthreads();
    if (!tile_wait(&s_bar, a.err) || !live) return;

    const float *rowbase = &svx[(U * r) * WW + 4 * g];   // vx row of grid row zr, word of column x-12
    const float *colbase = &svz[(U * r) * BX + 4 * g];   // group's first staged vz row, word of column x

    if (t.interior) {
        float dz[U][4];
        dz4<U, BX>(colbase, dz, [&](int, int, int j) { return a.c10[j]; });
#pragma unroll
        for (int u = 0; u < U; u++) {
            float dx[4];
            dx4<11, 12>(rowbase + u * WW, dx, [&](int, int j) { return a.c10[j]; });
            const unsigned id = (unsigned)(zr + u) * pitch + x;
            float pn[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float ddx = dx[j] * a.dtx, ddz = dz[u][j] * a.dtz, kj = comp(kk[u], j);
                pn[j] = MODE == 3 ? p_recon(comp(p0[u], j), ddx * kj, ddz * kj)
                                  : p_interior(comp(p0[u], j), ddx * kj, ddz * kj);
            }
            st4(&pp[id], f4(pn));
            if (MODE == 2) {
                ACC ng1[4], nil[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    ng1[j] = image_g1<ACC>(og1[u][j], comp(ps[u], j), pn[j]);
                    nil[j] = image_il<ACC>(oil[u][j], comp(ps[u], j));
                }
                st_acc4<ACC>(&g1p[id], ng1);
                st_acc4<ACC>(&ilp[id], nil);
            }
        }
        return;
    }

    const ShotK k = shot_ints(S);
    const float wit = a.wavelet[a.it];
    // local order of a cell (cuda_norder): min(x and z distance to the edge, R); edge tiles
    // take the table coefficients of that order, and no update on the edge itself
    auto order = [&](int xj, int zz) { return min(min(min(xj, X - 1 - xj), min(zz, Z - 1 - zz)), R); };
    float dz[U][4];
    if (!edge_tile) dz4<U, BX>(colbase, dz, [&](int, int, int j) { return a.c10[j]; });
    else dz4<U, BX>(colbase, dz, [&](int u, int jj, int j) { return s_tab[(max(order(x + jj, zr + u), 1) - 1) * R + j]; });
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int z = zr + u;
        if (z >= zend) break;
        float dx[4];
        if (!edge_tile) dx4<11, 12>(rowbase + u * WW, dx, [&](int, int j) { return a.c10[j]; });
        else dx4<11, 12>(rowbase + u * WW, dx, [&](int jj, int j) { return s_tab[(max(order(x + jj, z), 1) - 1) * R + j]; });
        const unsigned id0 = (unsigned)z * pitch + x;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int xj = x + j;
            if (xj >= X) break;
            PresCol cc;
            cc.xb = xb[j];
            cc.xin = xin[j];
            cc.c1x = xb[j] ? S.pml[o.c1x + xj] : 1.0f;
            cc.ic2x = xb[j] ? S.pml[o.ic2x + xj] : 1.0f;
            cc.srcc = (unsigned)(xj - k.sbx0) < (unsigned)k.sbnx;
            cc.recc = (xj >= k.rx0) && (xj < k.rx0 + k.nrec);
            cc.splr = (MODE == 3) ? strip_col_plr(xj, X, npml, k.nzi) : -1;
            cc.sptb = xin[j] ? xj - npml : -1;
            const bool upd = !edge_tile || order(xj, z) > 0;
            pres_apply<MODE, ACC>(a, S, k, cc, wit, pp, sxp, szp, g1p, ilp, id0 + j, xj, z, Z, npml, upd, dx[j],
                                  dz[u][j], comp(kk[u], j), comp(p0[u], j), comp(s1[u], j), comp(s2[u], j),
                                  comp(ps[u], j), og1[u][j], oil[u][j], s_c1z[z - z0], s_ic2z[z - z0], record);
        }
    }
}

// =====================================================================================
// Host launchers.
namespace {

template <int BZ>
size_t vel_smem4() { return (size_t)(BZ + QNV_MAX - 1) * WW * sizeof(float); }
template <int BZ>
size_t pres_smem4() { return ((size_t)BZ * WW + (size_t)(BZ + QNP_MAX - 1) * BX) * sizeof(float); }

template <typename F>
void set_smem_once4(std::atomic<unsigned long long> &done, F *fn, size_t bytes)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;   // the launch reports the error
    const unsigned long long bit = (dev >= 0 && dev < 64) ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (bit) done.fetch_or(bit, std::memory_order_release);
}

template <int BZ, int MODE, int U>
void vel4_launch(const StepArgs &a, int ntiles, cudaStream_t s)
{
    static std::atomic<unsigned long long> done{0};
    set_smem_once4(done, k_vel4<BZ, MODE, U>, vel_smem4<BZ>());
    k_vel4<BZ, MODE, U><<<ntiles, 32 * BZ / U, vel_smem4<BZ>(), s>>>(a);
}
template <int BZ, int MODE, int U, typename ACC>
void pres4_launch(const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    static std::atomic<unsigned long long> done{0};
    set_smem_once4(done, k_pres4<BZ, MODE, U, ACC>, pres_smem4<BZ>());
    k_pres4<BZ, MODE, U, ACC><<<ntiles, 32 * BZ / U, pres_smem4<BZ>(), s>>>(a, record);
}

template <int MODE>
void vel4_dispatch(int bz, const StepArgs &a, int ntiles, cudaStream_t s)
{
    if (bz == 16) vel4_launch<16, MODE, 2>(a, ntiles, s);
    else if (bz == 8) vel4_launch<8, MODE, 2>(a, ntiles, s);
    else if (bz == 64) vel4_launch<64, MODE, 4>(a, ntiles, s);
    else vel4_launch<32, MODE, 2>(a, ntiles, s);
}
template <int MODE, typename ACC>
void pres4_dispatch_t(int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if (bz == 16) pres4_launch<16, MODE, 2, ACC>(a, ntiles, record, s);
    else if (bz == 8) pres4_launch<8, MODE, 2, ACC>(a, ntiles, record, s);
    else if (bz == 64) pres4_launch<64, MODE, 4, ACC>(a, ntiles, record, s);
    else pres4_launch<32, MODE, 2, ACC>(a, ntiles, record, s);
}
template <int MODE>
void pres4_dispatch(int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if constexpr (MODE == 2) {
        if (a.accum_fp64 == RTM_ACC_FP64) {
            pres4_dispatch_t<MODE, double>(bz, a, ntiles, record, s);
            return;
        }
        if (a.accum_fp64 == RTM_ACC_KAHAN) {
            pres4_dispatch_t<MODE, KahanAcc>(bz, a, ntiles, record, s);
            return;
        }
    }
    pres4_dispatch_t<MODE, float>(bz, a, ntiles, record, s);
}

}  // namespace

void launch_vel4(int mode, int bz, const StepArgs &a, int ntiles, cudaStream_t s)
{
    switch (mode) {
    case RTM_WAVE_FWD: vel4_dispatch<0>(bz, a, ntiles, s); break;
    case RTM_WAVE_RECEIVER: vel4_dispatch<2>(bz, a, ntiles, s); break;
    default: vel4_dispatch<3>(bz, a, ntiles, s); break;
    }
}
void launch_pres4(int mode, int bz, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    switch (mode) {
    case RTM_WAVE_FWD: pres4_dispatch<0>(bz, a, ntiles, record, s); break;
    case RTM_WAVE_RECEIVER: pres4_dispatch<2>(bz, a, ntiles, 0, s); break;
    default: pres4_dispatch<3>(bz, a, ntiles, 0, s); break;
    }
}
