// Device bodies of the counting step, shared by the per-stage kernels and the
// persistent batched kernel.
//
// Arithmetic follows the reference's CPU code operation by operation (one
// lane sums one aggregated column over a vertex's neighbours in list order;
// every eMA product is accumulated in split order with separately rounded
// multiply and add), so vertices aggregated in one piece give the reference's
// FP32 values bit for bit (CSCGraph.hpp:242-307, DataTableColMajor.cpp:346-400).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "blk_ema.cuh"
#include "stage.cuh"

namespace sg {

__device__ __forceinline__ float ema_step(float acc, float agg, float mainv, bool scaled)
{
    if (scaled) {  // dst + (a * (double)b) * scale, rounded to float (DataTableColMajor.cpp:369)
        const double p = __dmul_rn(__dmul_rn((double)agg, (double)mainv), (double)1.0e-12f);
        return __double2float_rn(__dadd_rn((double)acc, p));
    }
    return __fadd_rn(acc, __fmul_rn(agg, mainv));   // dst + a*b without contraction (:492-493)
}
__device__ __forceinline__ double ema_step(double acc, double agg, double mainv, bool)
{
    return __dadd_rn(acc, __dmul_rn(agg, mainv));
}
// main is one-hot: the single non-zero split product is agg * 1
__device__ __forceinline__ float leaf_value(float agg, bool scaled)
{
    return scaled ? __double2float_rn(__dmul_rn((double)agg, (double)1.0e-12f)) : agg;
}
__device__ __forceinline__ double leaf_value(double agg, bool) { return agg; }

// 32-byte column chunks of table rows (rows are 32-byte aligned: pitches are
// multiples of 8 elements), loaded with one 256-bit load each.
struct __align__(32) F8 { float v[8]; };
struct __align__(32) D4 { double v[4]; };
template <typename T> struct Chunk;
template <> struct Chunk<float> {
    using type = F8;
    static constexpr int n = 8;
    __device__ static float get(const F8 &c, int i) { return c.v[i]; }
    __device__ static void add(F8 &a, const F8 &b)
    {
#pragma unroll
        for (int i = 0; i < 8; ++i) a.v[i] = __fadd_rn(a.v[i], b.v[i]);
    }
    __device__ static F8 zero()
    {
        F8 z;
#pragma unroll
        for (int i = 0; i < 8; ++i) z.v[i] = 0.f;
        return z;
    }
};
template <> struct Chunk<double> {
    using type = D4;
    static constexpr int n = 4;
    __device__ static double get(const D4 &c, int i) { return c.v[i]; }
    __device__ static void add(D4 &a, const D4 &b)
    {
#pragma unroll
        for (int i = 0; i < 4; ++i) a.v[i] = __dadd_rn(a.v[i], b.v[i]);
    }
    __device__ static D4 zero()
    {
        D4 z;
#pragma unroll
        for (int i = 0; i < 4; ++i) z.v[i] = 0.0;
        return z;
    }
};

// 16-byte chunks for the hub items, whose threads split the chunk's
// neighbours as well as its columns: narrower chunks give more of them.
template <typename T> struct Chunk16;
template <> struct Chunk16<float> {
    using type = float4;
    static constexpr int n = 4;
    __device__ static void add(float4 &a, const float4 &b)
    {
        a.x = __fadd_rn(a.x, b.x); a.y = __fadd_rn(a.y, b.y); a.z = __fadd_rn(a.z, b.z); a.w = __fadd_rn(a.w, b.w);
    }
    __device__ static float4 zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
};
template <> struct Chunk16<double> {
    using type = double2;
    static constexpr int n = 2;
    __device__ static void add(double2 &a, const double2 &b) { a.x = __dadd_rn(a.x, b.x); a.y = __dadd_rn(a.y, b.y); }
    __device__ static double2 zero() { return make_double2(0.0, 0.0); }
};

// Loads of count tables and partial rows.  The per-stage kernels read tables
// written by earlier launches (read-only for the launch: the non-coherent
// path); the persistent kernel reads tables produced inside the same launch,
// so it loads them through L2 (ld.global.cg), the point of coherence.
template <bool COH, typename P> __device__ __forceinline__ P ld_tab(const P *p) { return COH ? __ldcg(p) : __ldg(p); }
// 256-bit chunk loads: non-coherent (read-only for the launch), or through L2
template <bool COH> __device__ __forceinline__ F8 ld_tab(const F8 *p)
{
    F8 r;
    if (COH)
        asm volatile("ld.global.cg.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]), "=f"(r.v[6]),
                       "=f"(r.v[7])
                     : "l"(p)
                     : "memory");
    else
        asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
            : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]), "=f"(r.v[6]), "=f"(r.v[7])
            : "l"(p));
    return r;
}
template <bool COH> __device__ __forceinline__ D4 ld_tab(const D4 *p)
{
    D4 r;
    if (COH)
        asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];"
                     : "=d"(r.v[0]), "=d"(r.v[1]), "=d"(r.v[2]), "=d"(r.v[3])
                     : "l"(p)
                     : "memory");
    else
        asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(r.v[0]), "=d"(r.v[1]), "=d"(r.v[2]), "=d"(r.v[3]) : "l"(p));
    return r;
}

// The sum of n FP64 partials by one 256-thread block, in a fixed order with
// Kahan compensation, times `scale` (valid in thread 0).  A non-finite sum
// (an inf or NaN partial, which isPruned=0 runs reach) is returned as the
// plain sum: compensation would turn inf into NaN.
__device__ __forceinline__ double block_sum_partials(const double *p, int n, double scale, double *ss, double *cc,
                                                     double *pp)
{
    double s = 0.0, c = 0.0, plain = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = p[i];
        plain = __dadd_rn(plain, x);
        const double y = __dadd_rn(x, -c);
        const double t = __dadd_rn(s, y);
        c = __dadd_rn(__dadd_rn(t, -s), -y);
        s = t;
    }
    ss[threadIdx.x] = s;
    cc[threadIdx.x] = c;
    pp[threadIdx.x] = plain;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            ss[threadIdx.x] = __dadd_rn(ss[threadIdx.x], ss[threadIdx.x + w]);
            cc[threadIdx.x] = __dadd_rn(cc[threadIdx.x], cc[threadIdx.x + w]);
            pp[threadIdx.x] = __dadd_rn(pp[threadIdx.x], pp[threadIdx.x + w]);
        }
        __syncthreads();
    }
    const double r = isfinite(pp[0]) ? __dadd_rn(ss[0], -cc[0]) : pp[0];
    return __dmul_rn(r, scale);
}

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// Quotient by a tile-uniform divisor d for 0 <= i < n: multiply-high by
// m = floor((2^32-1)/d) + 1, exact while n*d < 2^32 (the error term i*(m*d -
// 2^32)/2^32 stays below 1/d); otherwise the plain division.
struct FastDiv {
    uint32_t m;
    int d;
    bool ok;
};
__device__ __forceinline__ FastDiv fast_div(int d, int n)
{
    FastDiv f;
    f.d = d;
    f.ok = d > 1 && (uint64_t)n * (uint64_t)d < (1ull << 32);
    f.m = f.ok ? 0xffffffffu / (uint32_t)d + 1u : 0u;
    return f;
}
__device__ __forceinline__ int fdiv(const FastDiv &f, int i)
{
    return f.ok ? (int)__umulhi((uint32_t)i, f.m) : i / f.d;
}

// Row stride (floats) of the aggregate and main rows in the packed layout: 32
// vertices plus 2 so that the 16 float2 of a half-warp cover all 32 banks.
constexpr int kPackedRow = 34;

// Shared-memory layout of a tile: [La_rows][RS] aggregate, [Lm_rows][RS] main
// rows (RS = TV+1, or kPackedRow for the packed eMA), [out_chunk][TV+1]
// output staging, then nb*TV doubles (root values) on a 16-byte boundary.
template <typename T>
__host__ __device__ inline size_t tile_smem_bytes(int La_rows, int Lm_rows, int out_chunk, int tv, bool packed, int nb = 1)
{
    const size_t rs = packed ? (size_t)kPackedRow : (size_t)(tv + 1);
    size_t b = (((size_t)(La_rows + Lm_rows) * rs + (size_t)out_chunk * (size_t)(tv + 1)) * sizeof(T) + 15) & ~(size_t)15;
    return b + (size_t)nb * tv * sizeof(double);
}

// packed FP32x2 arithmetic (sm_100a): two independent lanes, each rounded
// like __fmul_rn / __fadd_rn
__device__ __forceinline__ unsigned long long mul2_rn(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long add2_rn(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// ---------------------------------------------------------------------------
// One tile of one stage: TV consecutive (degree-ordered) vertices.
//   A. aggregation of the aux child's rows over each vertex's neighbours into
//      shared memory, transposed [column][vertex]: `gather_group` threads per
//      vertex, each owning gather_q 32-byte column chunks, neighbour ids and
//      rows fetched in batches of U before they are added (memory-level
//      parallelism without reordering the sums).  A one-hot aux child becomes
//      a per-color neighbour count.  Hub vertices add their partial rows.
//   B. the main child's rows of the tile, transposed the same way.
//   C. eMA.  Non-one-hot main: lanes = vertices, one output column per lane
//      group, split pairs as warp-uniform words, results staged and written
//      as contiguous rows.  One-hot main: each output is one aggregated
//      column (or zero), written directly as contiguous rows.  Root: a value
//      per vertex, reduced over the tile in a fixed order.
// The aggregate never leaves the chip.
// ---------------------------------------------------------------------------
template <typename T, int NT, int Q, bool PK = false, bool COH = false, bool BLK = false, int BN = 0, int BP = 0>
__device__ __forceinline__ void fused_tile(const StageDesc &d, int tile, unsigned char *smem_raw)
{
    using CT = Chunk<T>;
    using C = typename CT::type;
    constexpr int CH = CT::n;
    constexpr int NW = NT / 32;
    // neighbours per batch: 128 bytes of row chunks in flight per thread
    constexpr int U = 128 / (Q * (int)sizeof(C)) > 0 ? 128 / (Q * (int)sizeof(C)) : 1;
    const int TV = d.tile_v;
    const int TVP = TV + 1;
    const int RS = PK ? kPackedRow : TVP;          // row stride of the aggregate and main rows
    const int nbc = d.nb;                          // colorings of this launch
    const bool rooted = BLK && d.rooted;           // compacted rooted operands (one coloring)
    const int La_rows = d.aux_leaf ? nbc * d.k : (rooted ? d.r_La : d.aux_cols);
    const int Lm_rows = d.main_leaf ? 0 : (rooted ? d.r_Lm : d.main_cols);
    T *agg_s = reinterpret_cast<T *>(smem_raw);
    T *main_s = agg_s + (size_t)La_rows * RS;
    T *out_s = main_s + (size_t)Lm_rows * RS;
    const size_t root_off = (((size_t)(La_rows + Lm_rows) * RS + (size_t)d.out_chunk * TVP) * sizeof(T) + 15) & ~(size_t)15;
    double *root_s = reinterpret_cast<double *>(smem_raw + root_off);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int v0 = tile * TV;
    const int tv = min(TV, d.V - v0);
    const bool scaled = d.scaled != 0;

    // ---- A: aggregation ------------------------------------------------------
    if (d.aux_leaf) {
        // per-color neighbour counts (row b*k + c for coloring b): one thread per
        // (vertex, coloring), each owning its k counters (exact integers, no
        // atomics), neighbours in predicated batches of 8 with their loads in
        // flight together.  The colorings of a vertex are adjacent threads, so
        // that they share the neighbour ids and read the neighbour's colours
        // ([V][nb] bytes) together.
        const int nk = nbc * d.k;
        for (int vi = tid; vi < tv; vi += NT)
            for (int c = 0; c < nk; ++c) agg_s[c * RS + vi] = T(0);
        __syncthreads();
        for (int idx = tid; idx < nbc * tv; idx += NT) {
            const int vi = idx / nbc, b = idx - vi * nbc;
            const int v = v0 + vi;
            T *cnt = agg_s + (size_t)b * d.k * RS + vi;
            if (v < d.hub_count) {
                const T *p = reinterpret_cast<const T *>(d.hub_partial) + b * d.k;
                const int c0 = __ldg(d.hub_chunk_start + v), c1 = __ldg(d.hub_chunk_start + v + 1);
                for (int ch = c0; ch < c1; ++ch)
                    for (int c = 0; c < d.k; ++c)
                        cnt[c * RS] = add_rn(cnt[c * RS], ld_tab<COH>(p + (size_t)ch * d.hub_pitch + c));
                continue;
            }
            const int beg = __ldg(d.off + v), end = __ldg(d.off + v + 1);
            if (d.adjc && nbc == 1) {
                // colour-tagged neighbour ids: the colour comes with the id (top
                // 4 bits), one load a neighbour
                for (int e = beg; e < end; e += 8) {
                    int cl[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) cl[u] = e + u < end ? (int)((uint32_t)__ldg(d.adjc + e + u) >> 28) : -1;
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (cl[u] >= 0) cnt[cl[u] * RS] += T(1);
                }
                continue;
            }
            const uint8_t *col = d.color + b;
            for (int e = beg; e < end; e += 8) {
                int nb[8], cl[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) nb[u] = e + u < end ? __ldg(d.adj + e + u) : -1;
#pragma unroll
                for (int u = 0; u < 8; ++u) cl[u] = nb[u] >= 0 ? (int)__ldg(col + (size_t)nb[u] * d.cstride) : -1;
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (cl[u] >= 0) cnt[cl[u] * RS] += T(1);
            }
        }
    } else {
        const int G = d.gather_group;
        const int grp = tid / G, lane_g = tid - grp * G;
        const int ngrp = NT / G;
        const int nchunk = (d.aux_cols + CH - 1) / CH;
        const int rowc = d.aux_pitch / CH;
        const C *auxc = reinterpret_cast<const C *>(d.aux);
        // Work items: (vertex, chunk slots).  Grouped: the threads of group grp
        // take vertices grp, grp + ngrp, ...; thread lane_g owns chunks
        // lane_g + G*r.  Flat (d.cact): the tile's vertex v has
        // ceil(nact(c(v)) / Q) items over its active chunks; item l owns active
        // chunks l + n*r (n = the vertex's items), and the tile's items are
        // spread over all threads (s_pre: their prefix sums over the vertices).
        // A chunk slot at or past nchunk is idle.
        // (not in the persistent kernel, COH, which never sets cact)
        int *s_pre = nullptr;
        if constexpr (!COH) {
            __shared__ int s_pre_buf[33];
            s_pre = s_pre_buf;
        }
        const bool flat = !COH && d.cact != nullptr;
        if (flat) {
            if (warp == 0) {
                int n = 0;
                if (lane < tv) {
                    const int cv = __ldg(d.color + (size_t)(v0 + lane) * d.cstride);
                    n = ((int)__ldg(d.cact + (size_t)cv * d.cact_stride) + Q - 1) / Q;
                }
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, n, o);
                    if (lane >= o) n += y;
                }
                if (lane < tv) s_pre[lane + 1] = n;
                if (lane == 0) s_pre[0] = 0;
            }
            __syncthreads();
        }
        const int w_end = flat ? s_pre[tv] : tv;
        const int w_step = flat ? NT : ngrp;
        for (int wi = flat ? tid : (grp < ngrp ? grp : tv); wi < w_end; wi += w_step) {
            int vi, qv[Q];
            if (flat) {
                int lo = 0, hi = tv;   // s_pre[lo] <= wi < s_pre[hi]
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (s_pre[mid] <= wi) lo = mid;
                    else hi = mid;
                }
                vi = lo;
                const int l = wi - s_pre[vi], n = s_pre[vi + 1] - s_pre[vi];
                const uint16_t *ca = d.cact + (size_t)__ldg(d.color + (size_t)(v0 + vi) * d.cstride) * d.cact_stride;
                const int nact = __ldg(ca);
#pragma unroll
                for (int r = 0; r < Q; ++r) qv[r] = l + n * r < nact ? (int)__ldg(ca + 1 + l + n * r) : nchunk;
            } else {
                vi = wi;
#pragma unroll
                for (int r = 0; r < Q; ++r) qv[r] = lane_g + G * r;
            }
            {
                const int v = v0 + vi;
                C acc[Q];
                if (v < d.hub_count) {
                    const C *p = reinterpret_cast<const C *>(d.hub_partial);
                    const int prc = d.hub_pitch / CH;
                    const int c0 = __ldg(d.hub_chunk_start + v), c1 = __ldg(d.hub_chunk_start + v + 1);
#pragma unroll
                    for (int r = 0; r < Q; ++r) {
                        const int q = qv[r];
                        acc[r] = CT::zero();
                        if (q < nchunk)
                            for (int ch = c0; ch < c1; ++ch) CT::add(acc[r], ld_tab<COH>(p + (size_t)ch * prc + q));
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < Q; ++r) acc[r] = CT::zero();
                    const int beg = __ldg(d.off + v), end = __ldg(d.off + v + 1);
                    const int32_t *nbrs = d.adjc ? d.adjc : d.adj;
                    if (d.cmask) {
                        // colored neighbour ids: chunk q of a neighbour of color c_u is
                        // read only when bit c_u of this vertex color's mask is set
                        // (other chunks: exact zeros, or columns whose products meet
                        // an exact zero); a skipped slot adds +0
                        const uint16_t *cm = d.cmask + (size_t)__ldg(d.color + (size_t)v * d.cstride) * d.cmask_stride;
                        uint32_t msk[Q];
#pragma unroll
                        for (int r = 0; r < Q; ++r) {
                            const int q = qv[r];
                            msk[r] = q < nchunk ? (uint32_t)__ldg(cm + q) : 0u;
                        }
                        for (int e = beg; e < end; e += U) {
                            int nw[U];
#pragma unroll
                            for (int u = 0; u < U; ++u) nw[u] = e + u < end ? __ldg(nbrs + e + u) : 0;
                            C x[U][Q];
#pragma unroll
                            for (int u = 0; u < U; ++u)
#pragma unroll
                                for (int r = 0; r < Q; ++r) {
                                    const int q = qv[r];
                                    x[u][r] = (e + u < end && ((msk[r] >> ((uint32_t)nw[u] >> 28)) & 1u))
                                                  ? ld_tab<COH>(auxc + (size_t)(nw[u] & 0x0fffffff) * rowc + q)
                                                  : CT::zero();
                                }
#pragma unroll
                            for (int u = 0; u < U; ++u)
#pragma unroll
                                for (int r = 0; r < Q; ++r) CT::add(acc[r], x[u][r]);
                        }
                    } else if (qv[Q - 1] < nchunk) {
                        // every slot of this thread lies in the row: full batches of U
                        // neighbours without predicates, then the remaining ones singly
                        // (the same neighbour order, so the same sums)
                        const C *base = auxc + lane_g;
                        int e = beg;
                        for (; e + U <= end; e += U) {
                            int nb[U];
#pragma unroll
                            for (int u = 0; u < U; ++u) nb[u] = __ldg(nbrs + e + u) & 0x0fffffff;
                            C x[U][Q];
#pragma unroll
                            for (int u = 0; u < U; ++u) {
                                const C *row = base + (size_t)nb[u] * rowc;
#pragma unroll
                                for (int r = 0; r < Q; ++r) x[u][r] = ld_tab<COH>(row + G * r);
                            }
#pragma unroll
                            for (int u = 0; u < U; ++u)
#pragma unroll
                                for (int r = 0; r < Q; ++r) CT::add(acc[r], x[u][r]);
                        }
                        for (; e < end; ++e) {
                            const C *row = base + (size_t)(__ldg(nbrs + e) & 0x0fffffff) * rowc;
                            C x[Q];
#pragma unroll
                            for (int r = 0; r < Q; ++r) x[r] = ld_tab<COH>(row + G * r);
#pragma unroll
                            for (int r = 0; r < Q; ++r) CT::add(acc[r], x[r]);
                        }
                    } else {
                        // some slots past the row (the last threads of the group)
                        for (int e = beg; e < end; e += U) {
                            int nb[U];
#pragma unroll
                            for (int u = 0; u < U; ++u) nb[u] = e + u < end ? (__ldg(nbrs + e + u) & 0x0fffffff) : -1;
                            C x[U][Q];
#pragma unroll
                            for (int u = 0; u < U; ++u)
#pragma unroll
                                for (int r = 0; r < Q; ++r) {
                                    const int q = qv[r];
                                    x[u][r] = (q < nchunk && nb[u] >= 0) ? ld_tab<COH>(auxc + (size_t)nb[u] * rowc + q)
                                                                         : CT::zero();
                                }
#pragma unroll
                            for (int u = 0; u < U; ++u)
#pragma unroll
                                for (int r = 0; r < Q; ++r) CT::add(acc[r], x[u][r]);
                        }
                    }
                }
                if (rooted) {
                    // only the columns lacking this vertex's color, at their rooted rank
                    const uint32_t *ach = d.agg_chunk + (size_t)__ldg(d.color + (size_t)v * d.cstride) * nchunk;
#pragma unroll
                    for (int r = 0; r < Q; ++r) {
                        const int q = qv[r];
                        if (q < nchunk) {
                            const uint32_t w = __ldg(ach + q);
                            const uint32_t lack = w >> 16;
                            const int base = (int)(w & 0xffffu);
#pragma unroll
                            for (int i = 0; i < CH; ++i)
                                if (lack >> i & 1u)
                                    agg_s[(base + __popc(lack & ((1u << i) - 1u))) * RS + vi] = CT::get(acc[r], i);
                        }
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < Q; ++r) {
                        const int q = qv[r];
                        if (q < nchunk) {
#pragma unroll
                            for (int i = 0; i < CH; ++i) {
                                const int c = q * CH + i;
                                if (c < d.aux_cols) agg_s[c * RS + vi] = CT::get(acc[r], i);
                            }
                        }
                    }
                }
            }
        }
    }
    // ---- B: main rows --------------------------------------------------------------
    if (!d.main_leaf) {
        const T *mainp = reinterpret_cast<const T *>(d.main);
        if (rooted) {
            // the main columns holding this vertex's color, in rooted order
            for (int vi = warp; vi < tv; vi += NW) {
                const T *row = mainp + (size_t)(v0 + vi) * d.main_pitch;
                const int16_t *mf = d.main_full + (size_t)__ldg(d.color + (size_t)(v0 + vi) * d.cstride) * d.r_Lm;
                for (int c = lane; c < d.r_Lm; c += 32) main_s[c * RS + vi] = ld_tab<COH>(row + __ldg(mf + c));
            }
        } else {
            for (int vi = warp; vi < tv; vi += NW) {
                const T *row = mainp + (size_t)(v0 + vi) * d.main_pitch;
                for (int c = lane; c < d.main_cols; c += 32) main_s[c * RS + vi] = ld_tab<COH>(row + c);
            }
        }
    }
    __syncthreads();

    // ---- C: eMA ------------------------------------------------------------------------
    const int VPW = TV < 32 ? TV : 32;       // vertices per warp instruction
    const int OPI = 32 / VPW;                // outputs per warp instruction
    const int VB = TV / VPW;                 // vertex blocks of the tile
    const int lv = lane % VPW, osub = lane / VPW;
    if (d.is_root) {
        // root_s[b * TV + vi]: the root value of vertex vi in coloring b
        if (d.main_leaf) {
            for (int idx = tid; idx < nbc * tv; idx += NT) {
                const int b = idx / tv, vi = idx - b * tv;
                const int cv = __ldg(d.color + (size_t)(v0 + vi) * d.cstride + b);
                const int r = __ldg(d.rem + cv);
                root_s[b * TV + vi] = r >= 0 ? (double)agg_s[(b * d.a_cstride + r) * RS + vi] : 0.0;
            }
        } else {
            for (int u = warp; u < nbc * VB; u += NW) {
                if (osub != 0) continue;
                const int cb = u / VB, vi = (u - cb * VB) * VPW + lv;
                const T *mb = main_s + (size_t)cb * d.m_cstride * RS + vi;
                const T *ab = agg_s + (size_t)cb * d.a_cstride * RS + vi;
                double racc = 0.0;
                float facc = 0.f;
                for (int j = 0; j < d.S; ++j) {
                    const uint32_t pk = __ldg(d.split + (size_t)j * d.split_stride);
                    const T x = mb[(pk & 0xffffu) * RS];
                    const T y = ab[(pk >> 16) * RS];
                    if (sizeof(T) == 8) racc = __dadd_rn(racc, __dmul_rn((double)y, (double)x));
                    else if (d.root_float) facc = __fadd_rn(facc, __fmul_rn((float)y, (float)x));
                    else racc = __dadd_rn(racc, (double)__fmul_rn((float)y, (float)x));
                }
                if (vi < tv) root_s[cb * TV + vi] = (sizeof(T) == 4 && d.root_float) ? (double)facc : racc;
            }
        }
        __syncthreads();
        // one warp per coloring: the tile's vertices summed in a fixed order
        for (int cb = warp; cb < nbc; cb += NW) {
            double s = 0.0;
            for (int vi = lane; vi < tv; vi += 32) {
                s = __dadd_rn(s, root_s[cb * TV + vi]);
                if (d.root_vertex) d.root_vertex[v0 + vi] = root_s[cb * TV + vi];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_down_sync(0xffffffffu, s, o));
            if (lane == 0) d.root_partial[(size_t)cb * d.rp_stride + tile] = s;
        }
    } else if (d.main_leaf) {
        // one-hot main: out[o] = agg[set(o) \ {color}] when color is in set(o)
        // one flat, coalesced pass over the out_w written columns of the tile's
        // rows (column t = coloring b, output o)
        T *outp = reinterpret_cast<T *>(d.out);
        const int P = d.out_pitch, W = d.out_w;
        const FastDiv fd = fast_div(W, tv * W), fs = fast_div(d.s_cstride, W);
        for (int idx = tid; idx < tv * W; idx += NT) {
            const int vi = fdiv(fd, idx), t = idx - vi * W;
            const int b = fdiv(fs, t), o = t - b * d.s_cstride;
            T val = T(0);
            if (o < d.L_s) {
                const int cv = __ldg(d.color + (size_t)(v0 + vi) * d.cstride + b);
                const int r = __ldg(d.rem + o * d.k + cv);
                if (r >= 0) val = leaf_value(agg_s[(b * d.a_cstride + r) * RS + vi], scaled);
            }
            outp[(size_t)(v0 + vi) * P + t] = val;
        }
    } else if (BLK && d.packed == 2) {
        // register-blocked eMA over all output columns at once (blk_ema.cuh),
        // then the rows of the tile written out contiguously
        if constexpr (BLK && sizeof(T) == 4 && !PK) {
            T *outp = reinterpret_cast<T *>(d.out);
            const int P = d.out_pitch, W = d.out_w;
            if constexpr (BN > 0) blk::ema_blocks<BN, BP>(d, agg_s, main_s, out_s, RS, TVP, TV, warp, NW, lane);
            else blk::ema_blocked(d, agg_s, main_s, out_s, RS, TVP, TV, warp, NW, lane);
            __syncthreads();
            const FastDiv fd = fast_div(W, tv * W);
            if (rooted) {
                // rooted outputs back to the table's columns; sets lacking the
                // vertex's color are exact zeros
                for (int idx = tid; idx < tv * W; idx += NT) {
                    const int vj = fdiv(fd, idx), t = idx - vj * W;
                    T val = T(0);
                    if (t < d.L_s) {
                        const int r = __ldg(d.out_rank + (size_t)__ldg(d.color + (size_t)(v0 + vj) * d.cstride) * d.L_s + t);
                        if (r >= 0) val = out_s[r * TVP + vj];
                    }
                    outp[(size_t)(v0 + vj) * P + t] = val;
                }
            } else {
                for (int idx = tid; idx < tv * W; idx += NT) {
                    const int vj = fdiv(fd, idx), t = idx - vj * W;
                    outp[(size_t)(v0 + vj) * P + t] = t < d.L_s ? out_s[t * TVP + vj] : T(0);
                }
            }
            __syncthreads();
        }
    } else if (PK) {
        // packed eMA: lane = pair of vertices (2p, 2p+1) x a group of 4 output
        // columns; each operand is one 64-bit shared load at a byte offset taken
        // from the split tables, and the products / sums are FP32x2 operations
        // rounded like the scalar path.  A half-warp reads 16 consecutive
        // float2 of one row: all 32 banks once.
        T *outp = reinterpret_cast<T *>(d.out);
        const int P = d.out_pitch;
        const int SP4 = d.split_stride / 4;
        const int pr = lane & 15, osub = lane >> 4;
        const char *sb = reinterpret_cast<const char *>(smem_raw) + pr * 8;
        for (int o0 = 0; o0 < d.L_s; o0 += d.out_chunk) {
            const int oc = min(d.out_chunk, d.L_s - o0);
            const int ngroups = (oc + 7) / 8;
            for (int unit = warp; unit < ngroups; unit += NW) {
                const int ol = (unit * 2 + osub) * 4;
                if (ol >= oc) continue;
                const uint4 *ap = reinterpret_cast<const uint4 *>(d.aoff + o0 + ol);
                const uint4 *mp = reinterpret_cast<const uint4 *>(d.moff + o0 + ol);
                unsigned long long a0 = 0, a1 = 0, a2 = 0, a3 = 0;
                int j = 0;
                for (; j + 4 <= d.S; j += 4) {
                    uint4 A[4], M[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        A[u] = __ldg(ap + (size_t)(j + u) * SP4);
                        M[u] = __ldg(mp + (size_t)(j + u) * SP4);
                    }
                    unsigned long long pv[4][4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        pv[u][0] = mul2_rn(*reinterpret_cast<const unsigned long long *>(sb + A[u].x),
                                           *reinterpret_cast<const unsigned long long *>(sb + M[u].x));
                        pv[u][1] = mul2_rn(*reinterpret_cast<const unsigned long long *>(sb + A[u].y),
                                           *reinterpret_cast<const unsigned long long *>(sb + M[u].y));
                        pv[u][2] = mul2_rn(*reinterpret_cast<const unsigned long long *>(sb + A[u].z),
                                           *reinterpret_cast<const unsigned long long *>(sb + M[u].z));
                        pv[u][3] = mul2_rn(*reinterpret_cast<const unsigned long long *>(sb + A[u].w),
                                           *reinterpret_cast<const unsigned long long *>(sb + M[u].w));
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        a0 = add2_rn(a0, pv[u][0]);
                        a1 = add2_rn(a1, pv[u][1]);
                        a2 = add2_rn(a2, pv[u][2]);
                        a3 = add2_rn(a3, pv[u][3]);
                    }
                }
                for (; j < d.S; ++j) {
                    const uint4 A = __ldg(ap + (size_t)j * SP4), M = __ldg(mp + (size_t)j * SP4);
                    a0 = add2_rn(a0, mul2_rn(*reinterpret_cast<const unsigned long long *>(sb + A.x),
                                             *reinterpret_cast<const unsigned long long *>(sb + M.x)));
                    a1 = add2_rn(a1, mul2_rn(*reinterpret_cast<const unsigned long long *>(sb + A.y),
                                             *reinterpret_cast<const unsigned long long *>(sb + M.y)));
                    a2 = add2_rn(a2, mul2_rn(*reinterpret_cast<const unsigned long long *>(sb + A.z),
                                             *reinterpret_cast<const unsigned long long *>(sb + M.z)));
                    a3 = add2_rn(a3, mul2_rn(*reinterpret_cast<const unsigned long long *>(sb + A.w),
                                             *reinterpret_cast<const unsigned long long *>(sb + M.w)));
                }
                const unsigned long long av[4] = {a0, a1, a2, a3};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (ol + u < oc) {
                        out_s[(ol + u) * TVP + 2 * pr] = __uint_as_float((unsigned)(av[u] & 0xffffffffull));
                        out_s[(ol + u) * TVP + 2 * pr + 1] = __uint_as_float((unsigned)(av[u] >> 32));
                    }
                }
            }
            __syncthreads();
            const int ow = (o0 + oc == d.L_s) ? d.out_w - o0 : oc;
            const FastDiv fd = fast_div(ow, tv * ow);
            for (int idx = tid; idx < tv * ow; idx += NT) {
                const int vj = fdiv(fd, idx), t = idx - vj * ow;
                outp[(size_t)(v0 + vj) * P + o0 + t] = t < oc ? out_s[t * TVP + vj] : T(0);
            }
            __syncthreads();
        }
    } else {
        // each lane accumulates 4 consecutive output columns of its vertex at once
        // (4 independent chains); the split table is stored [j][column] so one
        // 16-byte warp-uniform load gives the 4 (main, aux) pairs of split j.
        // Columns are "wide": w = b * s_cstride + o over the launch's colorings
        // (one coloring: w = o < L_s, the row padding filled at the end).
        T *outp = reinterpret_cast<T *>(d.out);
        const int P = d.out_pitch;
        const int SP = d.split_stride;
        const int WW = nbc == 1 ? d.L_s : nbc * d.s_cstride;
        const FastDiv fs = fast_div(d.s_cstride, WW);
        for (int o0 = 0; o0 < WW; o0 += d.out_chunk) {
            const int oc = min(d.out_chunk, WW - o0);
            const int ngroups = (oc + 4 * OPI - 1) / (4 * OPI);
            for (int unit = warp; unit < VB * ngroups; unit += NW) {
                const int vb = unit % VB, og = unit / VB;
                const int ol = (og * OPI + osub) * 4;
                if (ol >= oc) continue;
                const int vi = vb * VPW + lv;
                const int w = o0 + ol;
                const int b = nbc == 1 ? 0 : fdiv(fs, w), o = w - b * d.s_cstride;
                if (o >= d.L_s) {   // a group of row padding (several colorings)
                    for (int u = 0; u < 4; ++u)
                        if (ol + u < oc) out_s[(ol + u) * TVP + vi] = T(0);
                    continue;
                }
                const T *mb = main_s + (size_t)b * d.m_cstride * RS + vi;
                const T *ab = agg_s + (size_t)b * d.a_cstride * RS + vi;
                const uint4 *sp = reinterpret_cast<const uint4 *>(d.split + o);
                const size_t sstep = (size_t)(SP / 4);
                T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
                int j = 0;
                // blocks of 4 splits: the 4 split words, then the 32 operands,
                // then the 16 multiply-adds (4 chains, each in split order)
                for (; j + 4 <= d.S; j += 4) {
                    uint4 pk[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) pk[u] = __ldg(sp + (size_t)(j + u) * sstep);
                    T ag[4][4], mn[4][4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        ag[u][0] = ab[(pk[u].x >> 16) * RS]; mn[u][0] = mb[(pk[u].x & 0xffffu) * RS];
                        ag[u][1] = ab[(pk[u].y >> 16) * RS]; mn[u][1] = mb[(pk[u].y & 0xffffu) * RS];
                        ag[u][2] = ab[(pk[u].z >> 16) * RS]; mn[u][2] = mb[(pk[u].z & 0xffffu) * RS];
                        ag[u][3] = ab[(pk[u].w >> 16) * RS]; mn[u][3] = mb[(pk[u].w & 0xffffu) * RS];
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        a0 = ema_step(a0, ag[u][0], mn[u][0], scaled);
                        a1 = ema_step(a1, ag[u][1], mn[u][1], scaled);
                        a2 = ema_step(a2, ag[u][2], mn[u][2], scaled);
                        a3 = ema_step(a3, ag[u][3], mn[u][3], scaled);
                    }
                }
                for (; j < d.S; ++j) {
                    const uint4 pk = __ldg(sp + (size_t)j * sstep);
                    a0 = ema_step(a0, ab[(pk.x >> 16) * RS], mb[(pk.x & 0xffffu) * RS], scaled);
                    a1 = ema_step(a1, ab[(pk.y >> 16) * RS], mb[(pk.y & 0xffffu) * RS], scaled);
                    a2 = ema_step(a2, ab[(pk.z >> 16) * RS], mb[(pk.z & 0xffffu) * RS], scaled);
                    a3 = ema_step(a3, ab[(pk.w >> 16) * RS], mb[(pk.w & 0xffffu) * RS], scaled);
                }
                // columns past L_s inside the group are row padding: zero
                const T av[4] = {a0, a1, a2, a3};
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (ol + u < oc) out_s[(ol + u) * TVP + vi] = o + u < d.L_s ? av[u] : T(0);
            }
            __syncthreads();
            // one coloring: the last chunk zero-fills the row padding up to out_w
            const int ow = (nbc == 1 && o0 + oc == d.L_s) ? d.out_w - o0 : oc;
            const FastDiv fd = fast_div(ow, tv * ow);
            for (int idx = tid; idx < tv * ow; idx += NT) {
                const int vj = fdiv(fd, idx), t = idx - vj * ow;
                outp[(size_t)(v0 + vj) * P + o0 + t] = t < oc ? out_s[t * TVP + vj] : T(0);
            }
            __syncthreads();
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Exact-order hub aggregation.  item = (hub vertex, group of 32 columns), one
// warp per item, neighbours in batches of BR (32 or 64).  The sum of a column over a hub's neighbour list in list
// order -- the reference's order (CSCGraph.hpp:242-307), so the row equals
// the per-tile aggregation bit for bit -- is one dependent chain of tens of
// thousands of adds, fed by loads whose latency must be hidden:
//   copies: the 32-column slices of a batch of BR neighbours go straight into
//           a shared-memory tile (row u = neighbour u's slice) with cp.async,
//           16 bytes a lane, a copy instruction moving whole slices (full
//           sectors), NSLOT batches ahead (a ring of tiles per warp);
//   adds:   lane l reads column l of the BR rows (conflict-free shared loads)
//           one batch ahead and adds them in order.
// Neighbour ids travel through the same pipeline: lane l copies ids l, l + 32,
// ... of a batch (cp.async, 4 bytes) into a ring of NSLOT + 1 id slots, in the commit
// group of the rows of the batch NSLOT earlier, so no step waits on a global
// load: every wait is cp.async.wait_group for a group issued NSLOT - 2
// batches earlier.  A lane waits for its own copies and __syncwarp makes the
// whole tile (and id slot) visible; the rings belong to the warp, so nothing
// wider is synchronised.  The result is the hub's single partial row (row v:
// every hub is one chunk).  Batches of 64 halve the per-batch work around the
// adds (one wait, commit and slot update for 64 neighbours) at twice the
// registers and tile bytes.
// ---------------------------------------------------------------------------
// row stride (elements) of a staging tile: a multiple of 16 bytes whose word
// offset between rows is 4 mod 32, so that the column reads are free of bank
// conflicts (a copy phase of eight lanes writes 128 contiguous bytes)
template <typename T> __host__ __device__ constexpr int hub_stage_stride() { return sizeof(T) == 4 ? 36 : 34; }
template <typename T, int BR = 32> __host__ __device__ constexpr int hub_tile_elems() { return BR * hub_stage_stride<T>(); }
// id slots of a warp's ring (one batch of BR ids each)
template <int NSLOT> __host__ __device__ constexpr int hub_id_slots() { return NSLOT + 1; }
// shared-memory bytes of one warp: the tile ring and the id ring
template <typename T, int NSLOT, int BR = 32> __host__ __device__ constexpr size_t hub_warp_bytes()
{
    return (size_t)NSLOT * hub_tile_elems<T, BR>() * sizeof(T) + (size_t)hub_id_slots<NSLOT>() * BR * sizeof(int32_t);
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}
// the same with the shared-memory address given as a 32-bit shared-window offset
__device__ __forceinline__ void cp_async16_s(uint32_t sa, const void *gmem)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4_s(uint32_t sa, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}
// copies of `n` source bytes (n <= the copy size) whose remaining bytes are
// zero-filled: n = 0 writes zeros and reads nothing
__device__ __forceinline__ void cp_async16_zs(uint32_t sa, const void *gmem, uint32_t n)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async4_zs(uint32_t sa, const void *gmem, uint32_t n)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename T, int NSLOT, int BR>
__device__ __forceinline__ void hub_item_exact(const HubArgs &h, int item, unsigned char *wsmem)
{
    static_assert(NSLOT >= 3, "one batch in flight besides the two in registers");
    static_assert(BR == 32 || BR == 64, "batches of 32 or 64 neighbours");
    constexpr int SS = hub_stage_stride<T>();
    constexpr int TILE = hub_tile_elems<T, BR>();
    constexpr int PC = 16 / sizeof(T);   // columns per 16-byte piece
    constexpr int NP = 32 / PC;          // pieces per 32-column slice = lanes per neighbour of one copy
    constexpr int NPI = 32 / NP;         // neighbours per warp copy (whole 128-/256-byte slices)
    constexpr int RPL = BR / NPI;        // rows per lane group = copies per batch
    constexpr int IDR = hub_id_slots<NSLOT>();
    constexpr uint32_t TILE_B = TILE * sizeof(T), IDS_B = BR * sizeof(int32_t);
    const T *ring = reinterpret_cast<const T *>(wsmem);
    const int32_t *ids = reinterpret_cast<const int32_t *>(wsmem + (size_t)NSLOT * TILE_B);
    const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(wsmem);
    const uint32_t ids_s = ring_s + NSLOT * TILE_B;
    const int lane = threadIdx.x & 31;
    // lane group ln copies piece lr of rows ln * RPL .. ln * RPL + RPL - 1, one
    // row a copy: each copy instruction moves NPI whole slices (full sectors)
    const int ln = lane / NP, lr = lane % NP;
    const int ngrp = (h.L_a + 31) / 32;
    const int v = item / ngrp, grp = item - v * ngrp;
    const int c0 = grp * 32;                                   // first column of the slice
    const bool lr_in = c0 + (lr + 1) * PC <= h.aux_pitch;      // this lane's piece lies inside the row
    const int beg = __ldg(h.off + v), deg = __ldg(h.off + v + 1) - beg;
    const int nbt = (deg + BR - 1) / BR;
    // this lane's piece of row 0 (a lane whose piece lies past the row copies
    // the slice's first piece instead: columns past the row are never
    // written out), and its first tile row in slot 0
    const uint64_t src0 = reinterpret_cast<uint64_t>(reinterpret_cast<const T *>(h.aux) + c0 + (lr_in ? lr * PC : 0));
    const uint32_t row_bytes = (uint32_t)h.aux_pitch * (uint32_t)sizeof(T);
    const uint32_t dst0 = ring_s + (uint32_t)((ln * RPL * SS + lr * PC) * sizeof(T));
    // with group masks the ids carry their colour (top 4 bits) and a
    // neighbour's slice is copied only when this group needs its colour
    const bool masked = h.gmask != nullptr;
    const int32_t *adj_v = (masked ? h.adjc : h.adj) + beg;
    const uint32_t gm =
        masked ? (uint32_t)__ldg(h.gmask + (size_t)__ldg(h.color + (size_t)v * h.cstride) * h.gmask_stride + grp) : ~0u;
    // ids lane, lane + 32, ... of batch j into the id slot at byte offset
    // `slot_b` (zero past the list: a valid row that is never added)
    auto fetch_ids = [&](int j, uint32_t slot_b) {
#pragma unroll
        for (int i = 0; i < BR / 32; ++i) {
            const int e = j * BR + i * 32 + lane;
            const bool in = e < deg;
            cp_async4_zs(ids_s + slot_b + (i * 32 + lane) * 4, adj_v + (in ? e : 0), in ? 4u : 0u);
        }
    };
    // A batch's copy plan for this lane: the source of each of its RPL pieces
    // and, bit k of `need`, whether piece k is read (else zero-filled).
    uint64_t src[RPL];
    uint32_t need = 0;
    auto plan = [&](uint32_t is_b) {
        const int4 *bid = reinterpret_cast<const int4 *>(ids + is_b / 4 + ln * RPL);
        need = 0;
#pragma unroll
        for (int q = 0; q < RPL / 4; ++q) {
            const int4 t = bid[q];
            const uint32_t w[4] = {(uint32_t)t.x, (uint32_t)t.y, (uint32_t)t.z, (uint32_t)t.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                src[4 * q + i] = src0 + (uint64_t)(w[i] & 0x0fffffffu) * row_bytes;
                need |= (gm >> (w[i] >> 28) & 1u) << (4 * q + i);
            }
        }
    };
    auto piece = [&](int k) -> uint32_t { return (need >> k & 1u) * 16u; };
    // batch b's copies into the ring slot at byte offset ts_b: every row of a
    // full batch, the rows inside the list of the last one, none past it
    auto copy = [&](int b, uint32_t ts_b) {
        const int left = deg - b * BR;
        const uint32_t d = dst0 + ts_b;
        if (left >= BR) {
#pragma unroll
            for (int k = 0; k < RPL; ++k)
                cp_async16_zs(d + (uint32_t)(k * SS * sizeof(T)), reinterpret_cast<const void *>(src[k]), piece(k));
        } else if (left > 0) {
#pragma unroll
            for (int k = 0; k < RPL; ++k)
                if (ln * RPL + k < left)
                    cp_async16_zs(d + (uint32_t)(k * SS * sizeof(T)), reinterpret_cast<const void *>(src[k]), piece(k));
        }
    };
    auto load = [&](T(&x)[BR], uint32_t ts_b) {
        const T *tile = ring + ts_b / sizeof(T) + lane;
#pragma unroll
        for (int u = 0; u < BR; ++u) x[u] = tile[u * SS];
    };
    // ids of batches 0 .. NSLOT - 1 first; batch j >= NSLOT has its ids
    // fetched with batch j - NSLOT's rows, into the slot of batch j - NSLOT - 1
    // (whose ids the previous plan read: hence the __syncwarp)
    for (int j = 0; j < NSLOT; ++j) fetch_ids(j, j * IDS_B);
    cp_async_commit();
    cp_async_wait<0>();
    __syncwarp();
    for (int b = 0; b < NSLOT - 1; ++b) {
        plan(b * IDS_B);
        copy(b, b * TILE_B);
        __syncwarp();
        fetch_ids(b + NSLOT, (b == 0 ? IDR - 1 : b - 1) * IDS_B);
        cp_async_commit();
    }
    plan((NSLOT - 1) * IDS_B);
    // Step b: add batch b (read by the step before); copy batch b + NSLOT - 1
    // (planned by the step before) and fetch the ids of batch b + 2 NSLOT - 1;
    // wait for batch b + 1 and read it into registers; plan batch b + NSLOT.
    // Steps b < nbt - NSLOT copy and add full batches and have no branch, so
    // that the copies, the shared loads and the plan fill the latency of the
    // add chains; the last NSLOT steps copy what is left of the list and add
    // the last batch under a predicate.  Slots (byte offsets) advance by one.
    uint32_t ts_b = (NSLOT - 1) * TILE_B, is_b = (NSLOT - 1) * IDS_B, ls_b = TILE_B;
    T acc = T(0);
    auto step = [&](int b, T(&cur)[BR], T(&nxt)[BR], bool tail, bool last) {
        // the adds of batch b first (its rows are in registers since the step
        // before): the copies, waits, shared loads and plan of the batches
        // ahead below are independent of them and fill the latency of the
        // dependent add chain
        if (!last) {
#pragma unroll
            for (int u = 0; u < BR; ++u) acc = add_rn(acc, cur[u]);
        } else {
            const int n = deg - b * BR;
#pragma unroll
            for (int u = 0; u < BR; ++u)
                if (u < n) acc = add_rn(acc, cur[u]);
        }
        if (!tail) {
#pragma unroll
            for (int k = 0; k < RPL; ++k)
                cp_async16_zs(dst0 + ts_b + (uint32_t)(k * SS * sizeof(T)), reinterpret_cast<const void *>(src[k]), piece(k));
        } else {
            copy(b + NSLOT - 1, ts_b);
        }
        fetch_ids(b + 2 * NSLOT - 1, is_b == 0 ? (IDR - 1) * IDS_B : is_b - IDS_B);
        cp_async_commit();            // always, so that the group count stays in step
        ts_b = ts_b == (NSLOT - 1) * TILE_B ? 0 : ts_b + TILE_B;
        is_b = is_b == (IDR - 1) * IDS_B ? 0 : is_b + IDS_B;
        cp_async_wait<NSLOT - 2>();   // this lane's copies of batch b + 1 (and older) have landed
        __syncwarp();                 // and so have the other lanes'; the slots read two steps ago may be refilled
        load(nxt, ls_b);              // batch b + 1 (unused past the list)
        ls_b = ls_b == (NSLOT - 1) * TILE_B ? 0 : ls_b + TILE_B;
        plan(is_b);                   // batch b + NSLOT: its ids landed with batch b's rows
    };
    T x[BR], y[BR];
    cp_async_wait<NSLOT - 2>();   // batch 0
    __syncwarp();
    load(x, 0);
    const int main_end = nbt - NSLOT;
    int b = 0;
    for (; b + 1 < main_end; b += 2) {
        step(b, x, y, false, false);
        step(b + 1, y, x, false, false);
    }
    for (; b + 1 < nbt; b += 2) {
        step(b, x, y, true, false);
        step(b + 1, y, x, true, b + 2 == nbt);
    }
    if (b < nbt) step(b, x, y, true, true);
    cp_async_wait<0>();
    if (c0 + lane < h.L_a) reinterpret_cast<T *>(h.partial)[(size_t)v * h.row_pitch + c0 + lane] = acc;
}

// ---------------------------------------------------------------------------
// One hub item: the neighbour chunk `item` of a hub vertex, summed into a
// partial row.  Threads are (neighbour lane r, column chunk q); lane r sums
// the chunk's neighbours r, r+R, ... in order, and the R lane sums are added
// in lane order: a fixed summation order.  A one-hot aux child counts colors.
// Needs NT * 32 bytes of shared memory (the lane partials), 32-byte aligned.
// ---------------------------------------------------------------------------
template <typename T, int NT, bool COH = false>
__device__ __forceinline__ void hub_item(const HubArgs &h, int item, unsigned char *smem_raw)
{
    using CT = Chunk16<T>;
    using C = typename CT::type;
    constexpr int CH = CT::n;
    int lo = 0, hi = h.hub_count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(h.chunk_start + mid) <= item) lo = mid; else hi = mid - 1;
    }
    const int v = lo;
    const int c = item - __ldg(h.chunk_start + v);
    const int beg = __ldg(h.off + v) + c * h.chunk;
    const int end = min(__ldg(h.off + v + 1), beg + h.chunk);
    T *prow = reinterpret_cast<T *>(h.partial) + (size_t)item * h.row_pitch;
    if (h.k_leaf) {
        // colour counts of the chunk's neighbours, k per coloring (nb * k <= 256)
        const int nk = h.nb * h.k_leaf;
        uint32_t *cnt = reinterpret_cast<uint32_t *>(smem_raw);
        for (int i = threadIdx.x; i < nk; i += NT) cnt[i] = 0;
        __syncthreads();
        if (h.nb == 1 && h.adjc) {   // colour-tagged ids: one load a neighbour
            for (int e = beg + (int)threadIdx.x; e < end; e += NT) atomicAdd(&cnt[(uint32_t)__ldg(h.adjc + e) >> 28], 1u);
        } else if (h.nb == 1 && h.cstride == 1) {
            for (int e = beg + (int)threadIdx.x; e < end; e += NT) atomicAdd(&cnt[__ldg(h.color + __ldg(h.adj + e))], 1u);
        } else {
            for (int e = beg + (int)threadIdx.x; e < end; e += NT) {
                const uint8_t *cp = h.color + (size_t)__ldg(h.adj + e) * h.cstride;
                for (int b = 0; b < h.nb; ++b) atomicAdd(&cnt[b * h.k_leaf + __ldg(cp + b)], 1u);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nk; i += NT) prow[i] = (T)cnt[i];
        __syncthreads();
        return;
    }
    C *lanes = reinterpret_cast<C *>(smem_raw);
    const int nchunk = (h.L_a + CH - 1) / CH;
    const int rowc = h.aux_pitch / CH;
    const C *auxc = reinterpret_cast<const C *>(h.aux);
    for (int base = 0; base < nchunk; base += NT) {
        const int cols = min(NT, nchunk - base);
        const int R = NT / cols;
        const int r = threadIdx.x / cols, q = base + (int)threadIdx.x - r * cols;
        C acc = CT::zero();
        if (r < R) {
            int e = beg + r;
            for (; e + 3 * R < end; e += 4 * R) {
                const C x0 = ld_tab<COH>(auxc + (size_t)__ldg(h.adj + e) * rowc + q);
                const C x1 = ld_tab<COH>(auxc + (size_t)__ldg(h.adj + e + R) * rowc + q);
                const C x2 = ld_tab<COH>(auxc + (size_t)__ldg(h.adj + e + 2 * R) * rowc + q);
                const C x3 = ld_tab<COH>(auxc + (size_t)__ldg(h.adj + e + 3 * R) * rowc + q);
                CT::add(acc, x0);
                CT::add(acc, x1);
                CT::add(acc, x2);
                CT::add(acc, x3);
            }
            for (; e < end; e += R) CT::add(acc, ld_tab<COH>(auxc + (size_t)__ldg(h.adj + e) * rowc + q));
            lanes[threadIdx.x] = acc;
        }
        __syncthreads();
        if ((int)threadIdx.x < cols) {
            C s = lanes[threadIdx.x];
            for (int rr = 1; rr < R; ++rr) CT::add(s, lanes[rr * cols + threadIdx.x]);
            reinterpret_cast<C *>(prow)[base + threadIdx.x] = s;
        }
        __syncthreads();
    }
}

}  // namespace sg
