// rtm_vec.cuh — 16-byte-word helpers of the kernels that give each thread four adjacent
// columns (rtm_stencil_v.cu, rtm_step.cu): shared and global float4 accesses, x- and
// z-derivative sums of four columns from staged rows, accumulator words.
#pragma once
#include <type_traits>

#include "rtm_stencil_common.cuh"

namespace {

__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
template <int J>
__device__ __forceinline__ float comp(const float4 &v)
{
    return J == 0 ? v.x : J == 1 ? v.y : J == 2 ? v.z : v.w;
}
__device__ __forceinline__ float comp(const float4 &v, int j)
{
    return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w;
}
__device__ __forceinline__ float4 f4(const float (&a)[4]) { return make_float4(a[0], a[1], a[2], a[3]); }

// Load four ACC values (16-byte aligned).
template <typename ACC>
__device__ __forceinline__ void ld_acc4(const ACC *p, ACC (&o)[4])
{
    if constexpr (std::is_same<ACC, KahanAcc>::value) {
        const float4 a = ld4((const float *)p), b = ld4((const float *)p + 4);
        o[0].s = a.x; o[0].c = a.y; o[1].s = a.z; o[1].c = a.w;
        o[2].s = b.x; o[2].c = b.y; o[3].s = b.z; o[3].c = b.w;
    } else if constexpr (sizeof(ACC) == 4) {
        const float4 v = ld4((const float *)p);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    } else {
        const double2 a = reinterpret_cast<const double2 *>(p)[0];
        const double2 b = reinterpret_cast<const double2 *>(p)[1];
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
}
template <typename ACC>
__device__ __forceinline__ void st_acc4(ACC *p, const ACC (&v)[4])
{
    if constexpr (std::is_same<ACC, KahanAcc>::value) {
        st4((float *)p, make_float4(v[0].s, v[0].c, v[1].s, v[1].c));
        st4((float *)p + 4, make_float4(v[2].s, v[2].c, v[3].s, v[3].c));
    } else if constexpr (sizeof(ACC) == 4) {
        st4((float *)p, make_float4(v[0], v[1], v[2], v[3]));
    } else {
        reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
    }
}

// x-derivative sums of four adjacent columns from one staged row.  `rw` points at the
// 16-byte word holding the column 12 to the left of the first output column, so a[k] is the
// value k-12 columns from it.  dx(j) = sum_i c(j, i-1) * (a[F + j + i] - a[G + j - i]) in tap
// order (velocity from p: F = 12, G = 13; pressure from vx: F = 11, G = 12).
// Paired lanes (sm_100 packed fp32: one instruction for two lanes, each lane rounded as a
// scalar operation): s += c * (f - g) per lane, the difference rounded, then a fused
// multiply-add, as the scalar sums are compiled.
#ifndef RTM_PACKED_FP32
#define RTM_PACKED_FP32 1
#endif
__device__ __forceinline__ float2 tap2(float2 s, float2 c, float2 f, float2 g)
{
    return __ffma2_rn(c, __fadd2_rn(f, make_float2(-g.x, -g.y)), s);
}

template <int F, int G, typename C>
__device__ __forceinline__ void dx4(const float *rw, float (&d)[4], C coef)
{
    float a[28];
#pragma unroll
    for (int q = 0; q < 7; q++) {
        const float4 v = lds4(rw + 4 * q);
        a[4 * q] = v.x; a[4 * q + 1] = v.y; a[4 * q + 2] = v.z; a[4 * q + 3] = v.w;
    }
#if RTM_PACKED_FP32
#pragma unroll
    for (int h = 0; h < 2; h++) {   // columns 2h, 2h+1
        float2 s = make_float2(0.f, 0.f);
#pragma unroll
        for (int i = 1; i <= R; i++)
            s = tap2(s, make_float2(coef(2 * h, i - 1), coef(2 * h + 1, i - 1)),
                     make_float2(a[F + 2 * h + i], a[F + 2 * h + 1 + i]), make_float2(a[G + 2 * h - i], a[G + 2 * h + 1 - i]));
        d[2 * h] = s.x;
        d[2 * h + 1] = s.y;
    }
#else
#pragma unroll
    for (int j = 0; j < 4; j++)
        d[j] = tap_sum([&](int i) { return coef(j, i); }, [&](int i) { return a[F + j + i]; },
                       [&](int i) { return a[G + j - i]; });
#endif
}

// z-derivative sums of 4 columns x U rows.  `col` points at the 16-byte word of the four
// columns in the staged row of index 0 of the group; output row u takes the rows u+i+9 and
// u-i+10 (velocity from p staged from z-9; pressure from vz staged from z-10).  Taps run in
// the outer loop, so each sum is accumulated in the order i = 1 .. 10 while only the rows of
// neighbouring taps are live.
template <int U, int STRIDE, typename C>
__device__ __forceinline__ void dz4(const float *col, float (&s)[U][4], C coef)
{
#if RTM_PACKED_FP32
    float2 s2[U][2];
#pragma unroll
    for (int u = 0; u < U; u++) s2[u][0] = s2[u][1] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 1; i <= R; i++) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            const float4 f = lds4(col + (u + i + 9) * STRIDE);
            const float4 g = lds4(col + (u - i + 10) * STRIDE);
            s2[u][0] = tap2(s2[u][0], make_float2(coef(u, 0, i - 1), coef(u, 1, i - 1)), make_float2(f.x, f.y),
                            make_float2(g.x, g.y));
            s2[u][1] = tap2(s2[u][1], make_float2(coef(u, 2, i - 1), coef(u, 3, i - 1)), make_float2(f.z, f.w),
                            make_float2(g.z, g.w));
        }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
        s[u][0] = s2[u][0].x; s[u][1] = s2[u][0].y; s[u][2] = s2[u][1].x; s[u][3] = s2[u][1].y;
    }
#else
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
        for (int j = 0; j < 4; j++) s[u][j] = 0.f;
#pragma unroll
    for (int i = 1; i <= R; i++) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            const float4 f = lds4(col + (u + i + 9) * STRIDE);
            const float4 g = lds4(col + (u - i + 10) * STRIDE);
#pragma unroll
            for (int j = 0; j < 4; j++) s[u][j] += coef(u, j, i - 1) * (comp(f, j) - comp(g, j));
        }
    }
#endif
}

// Resident blocks per SM that leave each of `threads` threads `regs` registers (the launch
// bounds of the kernels below: 80 registers, 128 for the receiver pressure update with its
// imaging operands; measured with -Xptxas -v, no spills at 16-row tiles in fp32 but 24 bytes
// in the receiver pressure update).
constexpr int min_blocks(int threads, int regs) { return 65536 / (threads * regs) > 0 ? 65536 / (threads * regs) : 1; }

}  // namespace
