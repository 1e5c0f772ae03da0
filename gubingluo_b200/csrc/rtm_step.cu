// rtm_step.cu — one whole time step (velocity and pressure) of one wavefield per launch
// (sm_100a).
//
// The split kernels (rtm_stencil.cu, rtm_stencil_v.cu) update the velocities of a step in
// one launch and the pressure in the next, so p, vx and vz cross HBM twice per step: 44 bytes
// per cell-update.  Here one launch does both, reading p, vx, vz, 1/rho and kappa once and
// writing p, vx and vz once (32 bytes).  The pressure update at a cell needs the new vx of the
// ten columns either side and the new vz of the ten rows above and below, so a block
// recomputes the new velocities of its tile's halo instead of waiting for its neighbours:
//
//   tile      128 columns x TZ rows of pressure cells (x0 a multiple of 4);
//   staged    by the tensor memory accelerator at the block's start, one barrier: the old p
//             of rows z0-19 .. z0+TZ+18, columns x0-24 .. x0+151; the old vx of rows
//             z0 .. z0+TZ-1, columns x0-12 .. x0+139; the old vz of rows z0-10 .. z0+TZ+9,
//             columns x0 .. x0+127 (off the grid: zeros);
//   phase A   new vx on the staged vx cells (x-derivatives of the staged p), in place in
//             shared memory; the tile's own cells also to HBM;
//   phase B   new vz on the staged vz cells (z-derivatives of the staged p), in place; the
//             tile's own rows also to HBM;
//   phase C   new p of the tile from the shared new velocities and the staged old p (with the
//             split PML fields, source, receivers, strips and imaging of the split pressure
//             kernels).
// So the per-shot fields cross HBM in bulk copies issued at once, and the only loads of a
// phase are the models 1/rho and kappa (shared by the shots of a survey window, mostly
// L2-resident) and, in the receiver pass, the imaging operands.
//
// Neighbouring tiles read the old fields while this one writes the new ones, so the fields
// p, vx, vz have two buffers each (ShotDev a/an, b/bn: before and after the step; the host
// swaps the roles after every step).  The split PML parts sx, sz belong to one cell each and
// stay in one buffer.  Every cell of a tile is written to the new buffers, including cells a
// step leaves unchanged, so both buffers hold the same values there.
//
// Work per phase is a list of tasks of four columns by two rows (the 16-byte words of
// rtm_vec.cuh), walked by the block's 256 threads.  Tiles whose cells and halo lie in the
// interior (no PML, source or receiver; full orders) are launched apart, as the branch-free
// instance FAST (fewer registers, more resident blocks); the others evaluate the per-cell
// updates of the split kernels (vx_value, vz_value, pres_value), so the results are the split
// kernels' bits.
#include <atomic>

#include "rtm_launch.h"
#include "rtm_vec.cuh"

namespace {

constexpr int kStepThreads = 256;
constexpr int PW = BX + 48;   // staged p columns x0-24 .. x0+151
constexpr int VXW = BX + 24;  // new vx columns x0-12 .. x0+139
constexpr int UQ = 2;         // rows per task

template <int TZ>
constexpr size_t step_smem_floats() { return (size_t)(TZ + 38) * PW + (size_t)TZ * VXW + (size_t)(TZ + 20) * BX; }

}  // namespace

template <int TZ, int MODE, typename ACC, bool FAST>
__global__ void __launch_bounds__(kStepThreads, (FAST && TZ == 16) ? 3 : 2) k_step(const StepArgs a, int record)
{
    constexpr int PH = TZ + 38, VZH = TZ + 20;
    constexpr int NQX = VXW / 4, NQ = BX / 4;   // quads of phase A; of phases B and C
    static_assert(TZ % UQ == 0 && VZH % UQ == 0, "two-row tasks");
    extern __shared__ __align__(128) float sm[];
    float *sp = sm;                   // [PH][PW]   old p
    float *svx = sp + PH * PW;        // [TZ][VXW]  old vx, then (updated in place) new vx
    float *svz = svx + TZ * VXW;      // [VZH][BX]  old vz, then new vz
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ float s_tab[100];
    if (tile_beyond(a)) return;   // fixed-grid launch: past this batch's tiles
    const TileRef t = a.tiles[blockIdx.x];
    const ShotDev &S = a.shots[t.shot];
    const int X = S.X, Z = S.Z, pitch = S.pitch, npml = S.npml;
    const int x0 = t.x0, z0 = t.z0;
    const WaveDev W = (MODE == 2) ? S.b : S.a;     // the wavefield before the step
    const WaveDev N = (MODE == 2) ? S.bn : S.an;   // after the step (p, vx, vz)
    const float *__restrict__ inv_rho = (MODE >= 2) ? S.inv_rho_b : S.inv_rho_f;
    const float *__restrict__ kappa = (MODE >= 2) ? S.kappa_b : S.kappa_f;
    const PmlOffsets o = pml_offsets(X, Z);
    if (threadIdx.x == 0) {   // old p (with both halos), old vx (x-halo), old vz (z-halo)
        mbar_init(&s_bar);
        mbar_expect(&s_bar, (PH * PW + TZ * VXW + VZH * BX) * sizeof(float));
        const int par = (MODE == 2) ? S.par_b : S.par_a;
        const int mp = (MODE == 2) ? RTM_TMAP_STEP_B0 : RTM_TMAP_STEP_A0;
        const int mx = (MODE == 2) ? RTM_TMAP_STEPVX_B0 : RTM_TMAP_STEPVX_A0;
        const int mz = (MODE == 2) ? RTM_TMAP_STEPVZ_B0 : RTM_TMAP_STEPVZ_A0;
        tma_box(sp, tmap_of(S, mp + par), x0 - 24, z0 - 19, &s_bar);
        tma_box(svx, tmap_of(S, mx + par), x0 - 12, z0, &s_bar);
        tma_box(svz, tmap_of(S, mz + par), x0, z0 - 10, &s_bar);
    }
    if (a.prefetch) {   // the models' rows of the tile and its halo into L2
        prefetch_rows(inv_rho, 4, max(z0 - 10, 0), min(z0 + TZ + 10, Z), x0, pitch, 1);
        prefetch_rows(kappa, 4, z0, min(z0 + TZ, Z), x0, pitch, 2);
    }
    for (int i = threadIdx.x; i < 100; i += kStepThreads) s_tab[i] = a.coef[i];
    __syncthreads();
    // every thread waits (bounded); the block goes on only if all saw the tile arrive
    if (!__syncthreads_and(tile_wait(&s_bar, a.err))) return;

    constexpr bool fast = FAST;   // the host launches interior tiles and the others apart
    const ShotK k = shot_ints(S);
    // general tiles whose cells of a phase all have full local orders use the full-order
    // coefficients like interior tiles (the table row of order R holds the same values)
    const bool edgeA = x0 - 12 < R - 1 || x0 + BX + 11 > X - 1 - R;         // vx orders (columns)
    const bool edgeB = z0 - 10 < R - 1 || z0 + TZ + 9 > Z - 1 - R;          // vz orders (rows)
    const bool edgeC = x0 < R || x0 + BX - 1 > X - 1 - R || z0 < R || z0 + TZ - 1 > Z - 1 - R;   // p orders
    auto c10 = [&](int j) { return a.c10[j]; };
    // local orders (cuda_norderx / cuda_norderz / cuda_norder), as table rows; at least 1
    auto ordv = [&](int i, int n) { return max(min(min(i + 1, n - 1 - i), R), 1); };

    // ---- phase A: new vx, columns x0-12 .. x0+139, rows z0 .. z0+TZ-1
#pragma unroll 1
    for (int task = threadIdx.x; task < NQX * (TZ / UQ); task += kStepThreads) {
        const int q = task % NQX, rg = task / NQX;
        const int x = x0 - 12 + 4 * q, zq = z0 + UQ * rg;
        const bool colin = x >= 0 && x < X;   // the quad lies in the row (x, X multiples of 4 apart from X)
        float4 ir[UQ], ov[UQ];
#pragma unroll
        for (int u = 0; u < UQ; u++) {
            const unsigned id = (unsigned)(zq + u) * pitch + x;
            ov[u] = lds4(&svx[(UQ * rg + u) * VXW + 4 * q]);   // staged old vx (zero off the grid)
            ir[u] = (colin && zq + u < Z) ? ldg4(&inv_rho[id]) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        const bool own = x >= x0 && x < x0 + BX;
#pragma unroll
        for (int u = 0; u < UQ; u++) {
            const int z = zq + u;
            const float *rw = &sp[(19 + UQ * rg + u) * PW + 4 * q];   // word of column x-12
            float dx[4], nv[4];
            if (fast) {
                dx4<12, 13>(rw, dx, [&](int, int j) { return c10(j); });
#pragma unroll
                for (int j = 0; j < 4; j++)
                    nv[j] = MODE == 3 ? __fadd_rn(comp(ov[u], j), vel_inc(dx[j], a.dtx, comp(ir[u], j)))
                                      : __fsub_rn(comp(ov[u], j), vel_inc(dx[j], a.dtx, comp(ir[u], j)));
            } else {
                if (edgeA) dx4<12, 13>(rw, dx, [&](int jj, int j) { return s_tab[(ordv(x + jj, X) - 1) * R + j]; });
                else dx4<12, 13>(rw, dx, [&](int, int j) { return c10(j); });
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int xj = x + j;
                    nv[j] = (xj >= 0 && xj < X - 1 && z < Z)
                                ? vx_value<MODE>(a, S, k, o, xj, z, X, Z, npml, dx[j], comp(ir[u], j), comp(ov[u], j))
                                : 0.f;
                }
            }
            st4(&svx[(UQ * rg + u) * VXW + 4 * q], f4(nv));
            if (own && z < Z) {
                const unsigned id = (unsigned)z * pitch + x;
                if (fast) st4(&N.vx[id], f4(nv));
                else
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (x + j < X - 1) N.vx[id + j] = nv[j];
            }
        }
    }

    // ---- phase B: new vz, columns x0 .. x0+127, rows z0-10 .. z0+TZ+9
#pragma unroll 1
    for (int task = threadIdx.x; task < NQ * (VZH / UQ); task += kStepThreads) {
        const int q = task % NQ, rg = task / NQ;
        const int x = x0 + 4 * q, zq = z0 - 10 + UQ * rg;
        float4 ir[UQ], ow[UQ];
#pragma unroll
        for (int u = 0; u < UQ; u++) {
            const int z = zq + u;
            const unsigned id = (unsigned)z * pitch + x;
            ow[u] = lds4(&svz[(UQ * rg + u) * BX + 4 * q]);   // staged old vz (zero off the grid)
            ir[u] = (x < X && z >= 0 && z < Z) ? ldg4(&inv_rho[id]) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        const float *col = &sp[(UQ * rg) * PW + 24 + 4 * q];   // staged row of grid row zq-9, word of column x
        float dz[UQ][4];
        if (fast || !edgeB) dz4<UQ, PW>(col, dz, [&](int, int, int j) { return c10(j); });
        else dz4<UQ, PW>(col, dz, [&](int u, int, int j) { return s_tab[(ordv(zq + u, Z) - 1) * R + j]; });
#pragma unroll
        for (int u = 0; u < UQ; u++) {
            const int z = zq + u;
            float nv[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (fast)
                    nv[j] = MODE == 3 ? __fadd_rn(comp(ow[u], j), vel_inc(dz[u][j], a.dtz, comp(ir[u], j)))
                                      : __fsub_rn(comp(ow[u], j), vel_inc(dz[u][j], a.dtz, comp(ir[u], j)));
                else
                    nv[j] = (x + j < X && z >= 0 && z < Z - 1)
                                ? vz_value<MODE>(a, S, k, o, x + j, z, X, Z, npml, dz[u][j], comp(ir[u], j),
                                                 comp(ow[u], j))
                                : 0.f;
            }
            st4(&svz[(UQ * rg + u) * BX + 4 * q], f4(nv));
            if (z >= z0 && z < z0 + TZ && z < Z - 1 && x < X) {
                const unsigned id = (unsigned)z * pitch + x;
                if (fast) st4(&N.vz[id], f4(nv));
                else
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (x + j < X) N.vz[id + j] = nv[j];
            }
        }
    }
    __syncthreads();

    // ---- phase C: new p of the tile
    float *__restrict__ sxp = W.sx;
    float *__restrict__ szp = W.sz;
    const float *__restrict__ psp = S.a.p;   // receiver pass: the reconstructed source pressure of this step
    ACC *__restrict__ g1p = (ACC *)S.g1;
    ACC *__restrict__ ilp = (ACC *)S.illum;
    const float wit = a.wavelet[a.it];
#pragma unroll 1
    for (int task = threadIdx.x; task < NQ * (TZ / UQ); task += kStepThreads) {
        const int q = task % NQ, rg = task / NQ;
        const int x = x0 + 4 * q, zq = z0 + UQ * rg;
        if (x >= X || zq >= Z) continue;
        bool xb[4], xin[4], anyxb = false, anyxin = false;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            xb[j] = (x + j < npml) || (x + j >= X - npml);
            xin[j] = !xb[j];
            anyxb |= xb[j];
            anyxin |= xin[j];
        }
        float4 kk[UQ], p0[UQ], s1[UQ], s2[UQ], ps[UQ];
        ACC og1[UQ][4], oil[UQ][4];
        // operands of row u of the task (the interior instance loads both rows before the
        // derivatives; the general one, short of registers, each row just before its use)
        auto load_row = [&](int u) {
            const int z = zq + u;
            const unsigned id = (unsigned)z * pitch + x;
            const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
            kk[u] = p0[u] = s1[u] = s2[u] = ps[u] = zero;
#pragma unroll
            for (int j = 0; j < 4; j++) og1[u][j] = oil[u][j] = 0;
            if (z >= Z) return;
            const bool zin = (z >= npml && z < Z - npml);
            kk[u] = ldg4(&kappa[id]);
            p0[u] = lds4(&sp[(19 + UQ * rg + u) * PW + 24 + 4 * q]);   // staged old p of the cell
            if (MODE != 3 && !fast && (anyxb || !zin)) {
                s1[u] = ld4(&sxp[id]);
                s2[u] = ld4(&szp[id]);
            }
            if (MODE == 2 && zin && anyxin) {
                ps[u] = ldg4(&psp[id]);
                ld_acc4<ACC>(&g1p[id], og1[u]);
                ld_acc4<ACC>(&ilp[id], oil[u]);
            }
        };
        if (fast)
#pragma unroll
            for (int u = 0; u < UQ; u++) load_row(u);
        const float *rowb = &svx[(UQ * rg) * VXW + 4 * q];   // new vx of row zq, word of column x-12
        const float *colb = &svz[(UQ * rg) * BX + 4 * q];    // new vz of row zq-10, word of column x
        float dz[UQ][4];
        if (fast || !edgeC) dz4<UQ, BX>(colb, dz, [&](int, int, int j) { return c10(j); });
        else
            dz4<UQ, BX>(colb, dz, [&](int u, int jj, int j) {
                const int xj = x + jj, zz = zq + u;
                const int rp = max(min(min(min(xj, X - 1 - xj), min(zz, Z - 1 - zz)), R), 1);
                return s_tab[(rp - 1) * R + j];
            });
#pragma unroll
        for (int u = 0; u < UQ; u++) {
            const int z = zq + u;
            if (z >= Z) break;
            if (!fast) load_row(u);
            const unsigned id = (unsigned)z * pitch + x;
            float dx[4], pn[4];
            if (fast) {
                dx4<11, 12>(rowb + u * VXW, dx, [&](int, int j) { return c10(j); });
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const float ddx = dx[j] * a.dtx, ddz = dz[u][j] * a.dtz, kj = comp(kk[u], j);
                    pn[j] = MODE == 3 ? p_recon(comp(p0[u], j), ddx * kj, ddz * kj)
                                      : p_interior(comp(p0[u], j), ddx * kj, ddz * kj);
                }
                st4(&N.p[id], f4(pn));
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
                continue;
            }
            if (edgeC)
                dx4<11, 12>(rowb + u * VXW, dx, [&](int jj, int j) {
                    const int xj = x + jj;
                    const int rp = max(min(min(min(xj, X - 1 - xj), min(z, Z - 1 - z)), R), 1);
                    return s_tab[(rp - 1) * R + j];
                });
            else dx4<11, 12>(rowb + u * VXW, dx, [&](int, int j) { return c10(j); });
            const float c1z = S.pml[o.c1z + z], ic2z = S.pml[o.ic2z + z];
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
                const bool upd = min(min(xj, X - 1 - xj), min(z, Z - 1 - z)) > 0;
                bool wr;
                N.p[id + j] = pres_value<MODE, ACC>(a, S, k, cc, wit, sxp, szp, g1p, ilp, id + j, xj, z, Z, npml, upd,
                                                    dx[j], dz[u][j], comp(kk[u], j), comp(p0[u], j), comp(s1[u], j),
                                                    comp(s2[u], j), comp(ps[u], j), og1[u][j], oil[u][j], c1z, ic2z,
                                                    record, &wr);
            }
        }
    }
}

// =====================================================================================
// Host launchers.
namespace {

template <int TZ, int MODE, typename ACC, bool FAST>
void step_launch(const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    static std::atomic<unsigned long long> done{0};
    const size_t bytes = step_smem_floats<TZ>() * sizeof(float);
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
        const unsigned long long bit = 1ull << dev;
        if (!(done.load(std::memory_order_acquire) & bit)) {
            cudaFuncSetAttribute(k_step<TZ, MODE, ACC, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            done.fetch_or(bit, std::memory_order_release);
        }
    }
    k_step<TZ, MODE, ACC, FAST><<<ntiles, kStepThreads, bytes, s>>>(a, record);
}
template <int MODE, typename ACC>
void step_dispatch_t(int tz, bool fast, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if (tz == 16) {
        if (fast) step_launch<16, MODE, ACC, true>(a, ntiles, record, s);
        else step_launch<16, MODE, ACC, false>(a, ntiles, record, s);
    } else {
        if (fast) step_launch<32, MODE, ACC, true>(a, ntiles, record, s);
        else step_launch<32, MODE, ACC, false>(a, ntiles, record, s);
    }
}
template <int MODE>
void step_dispatch(int tz, bool fast, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if constexpr (MODE == 2) {
        if (a.accum_fp64 == RTM_ACC_FP64) return step_dispatch_t<MODE, double>(tz, fast, a, ntiles, record, s);
        if (a.accum_fp64 == RTM_ACC_KAHAN) return step_dispatch_t<MODE, KahanAcc>(tz, fast, a, ntiles, record, s);
    }
    step_dispatch_t<MODE, float>(tz, fast, a, ntiles, record, s);
}

}  // namespace

size_t step_smem_bytes(int tz) { return (tz == 16 ? step_smem_floats<16>() : step_smem_floats<32>()) * sizeof(float); }

void launch_step(int mode, int tz, bool fast, const StepArgs &a, int ntiles, int record, cudaStream_t s)
{
    if (ntiles <= 0) return;
    switch (mode) {
    case RTM_WAVE_FWD: step_dispatch<0>(tz, fast, a, ntiles, record, s); break;
    case RTM_WAVE_RECEIVER: step_dispatch<2>(tz, fast, a, ntiles, 0, s); break;
    default: step_dispatch<3>(tz, fast, a, ntiles, 0, s); break;
    }
}
