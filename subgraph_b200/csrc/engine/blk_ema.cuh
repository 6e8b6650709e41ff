// Register-blocked eMA (device side of blk_sched.hpp).
//
// Lanes are the vertices of the tile (32, or 16 per half-warp); a warp (or
// half-warp) takes one block U at a time: it loads the held family's
// columns of its vertex into registers, then for every streamed column (one
// shared load) adds its products to the outputs of U that contain it.  All
// register indices are compile-time constants (fold expressions over the
// constexpr schedule), so the held values and the |U| accumulators stay in
// registers.  Multiply and add are separately rounded, in split order, as in
// the per-output loop (DataTableColMajor.cpp:492-493): the outputs are
// bit-identical to it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "blk_sched.hpp"
#include "stage.cuh"

namespace sg {
namespace blk {

template <int N, int P, int T, int C>
__device__ __forceinline__ void mac(float *acc, const float *h, float x)
{
    constexpr int o = Sched<N, P>::tab.po[T][C];
    constexpr int hi = Sched<N, P>::tab.ph[T][C];
    acc[o] = __fadd_rn(acc[o], __fmul_rn(h[hi], x));
}

template <int N, int P, int T, int... C>
__device__ __forceinline__ void stream_one(float *acc, const float *h, float x, std::integer_sequence<int, C...>)
{
    (mac<N, P, T, C>(acc, h, x), ...);
}

template <int N, int P, int T>
__device__ __forceinline__ void stream_at(float *acc, const float *h, const float *str_s, int col, int RS, int vi)
{
    if constexpr (T < Shape<N, P>::NS) {
        const float x = str_s[col * RS + vi];
        stream_one<N, P, T>(acc, h, x, std::make_integer_sequence<int, Shape<N, P>::PER>{});
    }
}

template <int N, int P, int G>
__device__ __forceinline__ void stream_group(float *acc, const float *h, const float *str_s, const int32_t *row, int RS,
                                             int vi)
{
    const int4 q = __ldg(reinterpret_cast<const int4 *>(row + Shape<N, P>::NH4) + G);
    stream_at<N, P, 4 * G + 0>(acc, h, str_s, q.x, RS, vi);
    stream_at<N, P, 4 * G + 1>(acc, h, str_s, q.y, RS, vi);
    stream_at<N, P, 4 * G + 2>(acc, h, str_s, q.z, RS, vi);
    stream_at<N, P, 4 * G + 3>(acc, h, str_s, q.w, RS, vi);
}

template <int N, int P, int... G>
__device__ __forceinline__ void stream_all(float *acc, const float *h, const float *str_s, const int32_t *row, int RS,
                                           int vi, std::integer_sequence<int, G...>)
{
    (stream_group<N, P, G>(acc, h, str_s, row, RS, vi), ...);
}

template <int N, int P, int I>
__device__ __forceinline__ void held_at(float *h, const float *held_s, int col, int RS, int vi)
{
    if constexpr (I < Shape<N, P>::NH) h[I] = held_s[col * RS + vi];
}

template <int N, int P, int G>
__device__ __forceinline__ void held_group(float *h, const float *held_s, const int32_t *row, int RS, int vi)
{
    const int4 q = __ldg(reinterpret_cast<const int4 *>(row) + G);
    held_at<N, P, 4 * G + 0>(h, held_s, q.x, RS, vi);
    held_at<N, P, 4 * G + 1>(h, held_s, q.y, RS, vi);
    held_at<N, P, 4 * G + 2>(h, held_s, q.z, RS, vi);
    held_at<N, P, 4 * G + 3>(h, held_s, q.w, RS, vi);
}

template <int N, int P, int... G>
__device__ __forceinline__ void held_all(float *h, const float *held_s, const int32_t *row, int RS, int vi,
                                         std::integer_sequence<int, G...>)
{
    (held_group<N, P, G>(h, held_s, row, RS, vi), ...);
}

template <int N, int P, int I>
__device__ __forceinline__ void out_at(const float *acc, float *out_s, int col, int TVP, int vi)
{
    if constexpr (I < Shape<N, P>::NO)
        if (col >= 0) out_s[col * TVP + vi] = acc[I];
}

template <int N, int P, int G>
__device__ __forceinline__ void out_group(const float *acc, float *out_s, const int32_t *row, int TVP, int vi)
{
    using S = Shape<N, P>;
    const int4 q = __ldg(reinterpret_cast<const int4 *>(row + S::NH4 + S::NS4) + G);
    out_at<N, P, 4 * G + 0>(acc, out_s, q.x, TVP, vi);
    out_at<N, P, 4 * G + 1>(acc, out_s, q.y, TVP, vi);
    out_at<N, P, 4 * G + 2>(acc, out_s, q.z, TVP, vi);
    out_at<N, P, 4 * G + 3>(acc, out_s, q.w, TVP, vi);
}

template <int N, int P, int... G>
__device__ __forceinline__ void out_all(const float *acc, float *out_s, const int32_t *row, int TVP, int vi,
                                        std::integer_sequence<int, G...>)
{
    (out_group<N, P, G>(acc, out_s, row, TVP, vi), ...);
}

// All blocks of the stage for the TV vertices of the tile (TV = 32 or 16);
// results go to out_s[column][vertex] (stride TVP).
template <int N, int P>
__device__ __forceinline__ void ema_blocks(const StageDesc &d, const float *agg_s, const float *main_s, float *out_s,
                                           int RS, int TVP, int TV, int warp, int nwarps, int lane)
{
    using S = Shape<N, P>;
    const float *held_s = S::kHoldMain ? main_s : agg_s;
    const float *str_s = S::kHoldMain ? agg_s : main_s;
    const int per_warp = 32 / TV;
    const int vi = lane % TV, sub = lane / TV;
    for (int b = warp * per_warp + sub; b < d.blk_nblocks; b += nwarps * per_warp) {
        const int32_t *row = d.blk + (size_t)b * S::ROW;
        float h[S::NH];
        held_all<N, P>(h, held_s, row, RS, vi, std::make_integer_sequence<int, S::NH4 / 4>{});
        float acc[S::NO];
#pragma unroll
        for (int o = 0; o < S::NO; ++o) acc[o] = 0.f;
        stream_all<N, P>(acc, h, str_s, row, RS, vi, std::make_integer_sequence<int, S::NS4 / 4>{});
        out_all<N, P>(acc, out_s, row, TVP, vi, std::make_integer_sequence<int, S::NO4 / 4>{});
    }
}

__device__ __forceinline__ void ema_blocked(const StageDesc &d, const float *agg_s, const float *main_s, float *out_s,
                                            int RS, int TVP, int TV, int warp, int nwarps, int lane)
{
    int k = 0;
#define SG_BLK_CASE(NN, PP) \
    if (++k == d.blk_shape) { ema_blocks<NN, PP>(d, agg_s, main_s, out_s, RS, TVP, TV, warp, nwarps, lane); return; }
    SG_BLK_SHAPES(SG_BLK_CASE)
#undef SG_BLK_CASE
}

}  // namespace blk
}  // namespace sg
