// Device kernels of the color-coding counting path, written for sm_100a.
//
// The count tables are vertex-major (row v = the v-th vertex's color-set
// columns), so the neighbour aggregation reads whole contiguous rows with
// 128-bit loads.  Every aggregated column is summed by one lane in the order
// of the vertex's neighbour list, and every eMA product is accumulated in the
// order of the split table with separately rounded multiply and add: for
// vertices below the hub threshold the FP32 results equal the reference's
// CPU arithmetic (CSCGraph.hpp:242-307, DataTableColMajor.cpp:346-400) bit
// for bit.
#include "kernels.cuh"

#include <algorithm>
#include <cstdio>

namespace sg {

// ---------------------------------------------------------------------------
// K1: coloring.  The glibc TYPE_3 stream after srand(seed) is the lag-31
// recurrence s_m = s_{m-3} + s_{m-31} (mod 2^32) started from a 31-word
// window; rand() number v is s_{341+v} >> 1 (CountMat.cpp:979-991 draws
// rand() % k for v = 0..V-1 on one thread).  With P(x) = x^31 - x^28 - 1,
// s_{m0+t} = sum_i [x^t mod P]_i * s_{m0+i}, so every block rebuilds its own
// start window from the jump polynomial x^{m0} and every thread then needs one
// 31-term dot product.  All arithmetic is exact modulo 2^32.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kColorBlock) k_color(ColorArgs a)
{
    __shared__ uint32_t W[31];
    const int b = blockIdx.x;
    const int col = blockIdx.y;
    const uint32_t *w0 = a.window + 31 * col;
    if (threadIdx.x < 31) {
        uint32_t q[31];
#pragma unroll
        for (int j = 0; j < 31; ++j) q[j] = a.jump[b * 31 + j];
        for (int s = 0; s < (int)threadIdx.x; ++s) {   // q <- x*q mod P
            uint32_t t = q[30];
#pragma unroll
            for (int j = 30; j > 0; --j) q[j] = q[j - 1];
            q[0] = t;
            q[28] += t;
        }
        uint32_t acc = 0;
#pragma unroll
        for (int j = 0; j < 31; ++j) acc += q[j] * w0[j];
        W[threadIdx.x] = acc;
    }
    __syncthreads();
    const int64_t v = (int64_t)b * kColorBlock + threadIdx.x;
    if (v < a.V) {
        uint32_t s = 0;
#pragma unroll
        for (int i = 0; i < 31; ++i) s += __ldg(a.coef + i * kColorBlock + threadIdx.x) * W[i];
        const int r = (int)(s >> 1);
        a.color[col * a.color_stride + a.perm[v]] = (uint8_t)(r % a.k);
    }
}

void launch_color(const ColorArgs &a, int ncolorings, cudaStream_t st)
{
    if (a.V == 0 || ncolorings == 0) return;
    dim3 grid(a.nblocks, ncolorings);
    k_color<<<grid, kColorBlock, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// Relabelling: internal vertex v = original iperm[v]; its neighbour list keeps
// the original order (which fixes the summation order) with ids mapped
// through perm.  One warp per vertex.
// ---------------------------------------------------------------------------
__global__ void k_remap(int32_t V, const int32_t *__restrict__ old_off, const int32_t *__restrict__ old_adj,
                        const int32_t *__restrict__ new_off, const int32_t *__restrict__ iperm,
                        const int32_t *__restrict__ perm, int32_t *__restrict__ new_adj)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = w; v < V; v += nw) {
        const int32_t o = iperm[v];
        const int32_t b = old_off[o], e = old_off[o + 1], d = new_off[v];
        for (int32_t i = b + lane; i < e; i += 32) new_adj[d + (i - b)] = perm[old_adj[i]];
    }
}

void launch_remap(int32_t V, const int32_t *old_off, const int32_t *old_adj, const int32_t *new_off,
                  const int32_t *iperm, const int32_t *perm, int32_t *new_adj, cudaStream_t st)
{
    if (V == 0) return;
    int blocks = std::min<int64_t>(((int64_t)V * 32 + 255) / 256, 148 * 16);
    k_remap<<<blocks, 256, 0, st>>>(V, old_off, old_adj, new_off, iperm, perm, new_adj);
}

// ---------------------------------------------------------------------------
// Arithmetic of the eMA step, per table type and mode.
// ---------------------------------------------------------------------------
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

template <typename T> struct Chunk;
template <> struct Chunk<float> {
    using type = float4;
    static constexpr int n = 4;
    __device__ static float get(const float4 &v, int i) { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }
    __device__ static void add(float4 &a, const float4 &b)
    {
        a.x = __fadd_rn(a.x, b.x); a.y = __fadd_rn(a.y, b.y); a.z = __fadd_rn(a.z, b.z); a.w = __fadd_rn(a.w, b.w);
    }
    __device__ static float4 zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
};
template <> struct Chunk<double> {
    using type = double2;
    static constexpr int n = 2;
    __device__ static double get(const double2 &v, int i) { return i == 0 ? v.x : v.y; }
    __device__ static void add(double2 &a, const double2 &b) { a.x = __dadd_rn(a.x, b.x); a.y = __dadd_rn(a.y, b.y); }
    __device__ static double2 zero() { return make_double2(0.0, 0.0); }
};

// ---------------------------------------------------------------------------
// K2: one sub-template step, fused.  A CTA owns a tile of TV consecutive
// (degree-ordered) vertices:
//   A. aggregation of the aux child's rows over each vertex's neighbours
//      into shared memory, transposed [column][vertex]; a one-hot aux child
//      (size 1) turns into a per-color neighbour count;
//   B. the main child's rows of the tile, transposed the same way;
//   C. eMA: lanes = vertices, one output column per lane group, split pairs
//      read as warp-uniform words; results staged in shared memory and
//      written as contiguous rows (or reduced per vertex at the root).
// The aggregate never leaves the chip.
// ---------------------------------------------------------------------------
template <typename T, int TV, int Q>
__global__ void __launch_bounds__(kFusedThreads) k_fused(StageDesc d)
{
    using CT = Chunk<T>;
    using C = typename CT::type;
    constexpr int CH = CT::n;
    constexpr int NW = kFusedThreads / 32;
    constexpr int TVP = TV + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int La_rows = d.aux_leaf ? d.k : d.L_a;
    const int Lm_rows = d.main_leaf ? 0 : d.L_m;
    T *agg_s = reinterpret_cast<T *>(smem_raw);
    T *main_s = agg_s + (size_t)La_rows * TVP;
    T *out_s = main_s + (size_t)Lm_rows * TVP;
    // per-vertex root values after the tables, on a 16-byte boundary
    const size_t root_off = ((size_t)(La_rows + Lm_rows + d.out_chunk) * TVP * sizeof(T) + 15) & ~(size_t)15;
    double *root_s = reinterpret_cast<double *>(smem_raw + root_off);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = d.gather_group;
    const int lane_g = tid & (G - 1);
    const int grp = tid / G, ngrp = kFusedThreads / G;
    const int nchunk = (d.L_a + CH - 1) / CH;
    const int rowc = d.aux_pitch / CH;
    const C *auxc = reinterpret_cast<const C *>(d.aux);
    const T *mainp = reinterpret_cast<const T *>(d.main);
    T *outp = reinterpret_cast<T *>(d.out);
    const T *hub = reinterpret_cast<const T *>(d.hub_agg);

    for (int tile = blockIdx.x; tile < d.ntiles; tile += gridDim.x) {
        const int v0 = tile * TV;
        const int tv = min(TV, d.V - v0);

        // ---- A: aggregation ------------------------------------------------
        if (d.aux_leaf) {
            // neighbour color histogram, exact integer counts
            for (int vi = warp; vi < tv; vi += NW) {
                const int v = v0 + vi;
                if (v < d.hub_count) {
                    if (lane < d.k) agg_s[lane * TVP + vi] = hub[(size_t)v * d.hub_pitch + lane];
                    continue;
                }
                const int beg = __ldg(d.off + v), end = __ldg(d.off + v + 1);
                uint32_t cnt = 0;
                for (int e = beg; e < end; e += 32) {
                    const int c = (e + lane < end) ? (int)__ldg(d.color + __ldg(d.adj + e + lane)) : 255;
                    for (int cc = 0; cc < d.k; ++cc) {
                        const unsigned bal = __ballot_sync(0xffffffffu, c == cc);
                        if (lane == cc) cnt += __popc(bal);
                    }
                }
                if (lane < d.k) agg_s[lane * TVP + vi] = (T)cnt;
            }
        } else {
            for (int vi = grp; vi < tv; vi += ngrp) {
                const int v = v0 + vi;
                if (v < d.hub_count) {
                    for (int c = lane_g; c < d.L_a; c += G) agg_s[c * TVP + vi] = hub[(size_t)v * d.hub_pitch + c];
                    continue;
                }
                const int beg = __ldg(d.off + v), end = __ldg(d.off + v + 1);
                for (int base = 0; base < nchunk; base += G * Q) {
                    C acc[Q];
#pragma unroll
                    for (int r = 0; r < Q; ++r) acc[r] = CT::zero();
                    int e = beg;
                    for (; e + 4 <= end; e += 4) {
                        const int n0 = __ldg(d.adj + e), n1 = __ldg(d.adj + e + 1);
                        const int n2 = __ldg(d.adj + e + 2), n3 = __ldg(d.adj + e + 3);
                        const C *r0 = auxc + (size_t)n0 * rowc, *r1 = auxc + (size_t)n1 * rowc;
                        const C *r2 = auxc + (size_t)n2 * rowc, *r3 = auxc + (size_t)n3 * rowc;
#pragma unroll
                        for (int r = 0; r < Q; ++r) {
                            const int q = base + lane_g + G * r;
                            if (q < nchunk) {
                                const C x0 = __ldg(r0 + q), x1 = __ldg(r1 + q), x2 = __ldg(r2 + q), x3 = __ldg(r3 + q);
                                CT::add(acc[r], x0);
                                CT::add(acc[r], x1);
                                CT::add(acc[r], x2);
                                CT::add(acc[r], x3);
                            }
                        }
                    }
                    for (; e < end; ++e) {
                        const C *r0 = auxc + (size_t)__ldg(d.adj + e) * rowc;
#pragma unroll
                        for (int r = 0; r < Q; ++r) {
                            const int q = base + lane_g + G * r;
                            if (q < nchunk) CT::add(acc[r], __ldg(r0 + q));
                        }
                    }
#pragma unroll
                    for (int r = 0; r < Q; ++r) {
                        const int q = base + lane_g + G * r;
#pragma unroll
                        for (int i = 0; i < CH; ++i) {
                            const int c = q * CH + i;
                            if (q < nchunk && c < d.L_a) agg_s[c * TVP + vi] = CT::get(acc[r], i);
                        }
                    }
                }
            }
        }
        // ---- B: main rows ----------------------------------------------------
        if (!d.main_leaf) {
            for (int vi = warp; vi < tv; vi += NW) {
                const T *row = mainp + (size_t)(v0 + vi) * d.main_pitch;
                for (int c = lane; c < d.L_m; c += 32) main_s[c * TVP + vi] = __ldg(row + c);
            }
        }
        __syncthreads();

        // ---- C: eMA ------------------------------------------------------------
        const bool scaled = d.scaled != 0;
        if (d.is_root) {
            if (d.main_leaf) {
                for (int vi = tid; vi < tv; vi += kFusedThreads) {
                    const int cv = __ldg(d.color + v0 + vi);
                    const int r = __ldg(d.rem + cv);
                    const T a = r >= 0 ? agg_s[r * TVP + vi] : T(0);
                    root_s[vi] = (double)a;
                }
            } else if (warp == 0) {
                constexpr int OPI = 32 / TV;
                const int vi = lane % TV;
                if (lane / TV == 0 || OPI == 1) {
                    double racc = 0.0;
                    float facc = 0.f;
                    for (int j = 0; j < d.S; ++j) {
                        const uint32_t pk = __ldg(d.split + j);
                        const T x = main_s[(pk & 0xffffu) * TVP + vi];
                        const T y = agg_s[(pk >> 16) * TVP + vi];
                        if (sizeof(T) == 8) racc = __dadd_rn(racc, __dmul_rn((double)y, (double)x));
                        else if (d.root_float) facc = __fadd_rn(facc, __fmul_rn((float)y, (float)x));
                        else racc = __dadd_rn(racc, (double)__fmul_rn((float)y, (float)x));
                    }
                    if (vi < tv) root_s[vi] = (sizeof(T) == 4 && d.root_float) ? (double)facc : racc;
                }
            }
            __syncthreads();
            if (warp == 0) {
                // fixed-order tree over the tile's vertices
                double s = 0.0;
                for (int vi = lane; vi < tv; vi += 32) {
                    s = __dadd_rn(s, root_s[vi]);
                    if (d.root_vertex) d.root_vertex[v0 + vi] = root_s[vi];
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_down_sync(0xffffffffu, s, o));
                if (lane == 0) d.root_partial[tile] = s;
            }
        } else if (d.main_leaf) {
            // one-hot main: out[o] = agg[set(o) \ {color}] if color in set(o)
            const int P = d.out_pitch;
            for (int idx = tid; idx < tv * P; idx += kFusedThreads) {
                const int vi = idx / P, o = idx - vi * P;
                T val = T(0);
                if (o < d.L_s) {
                    const int cv = __ldg(d.color + v0 + vi);
                    const int r = __ldg(d.rem + o * d.k + cv);
                    if (r >= 0) val = leaf_value(agg_s[r * TVP + vi], scaled);
                }
                outp[(size_t)(v0 + vi) * P + o] = val;
            }
        } else {
            constexpr int OPI = 32 / TV;
            const int vi = lane % TV, osub = lane / TV;
            const int P = d.out_pitch;
            for (int o0 = 0; o0 < d.L_s; o0 += d.out_chunk) {
                const int oc = min(d.out_chunk, d.L_s - o0);
                for (int ol = warp * OPI + osub; ol < oc; ol += NW * OPI) {
                    const uint32_t *sp = d.split + (size_t)(o0 + ol) * d.S;
                    T acc = T(0);
                    for (int j = 0; j < d.S; ++j) {
                        const uint32_t pk = __ldg(sp + j);
                        acc = ema_step(acc, agg_s[(pk >> 16) * TVP + vi], main_s[(pk & 0xffffu) * TVP + vi], scaled);
                    }
                    out_s[ol * TVP + vi] = acc;
                }
                __syncthreads();
                const int ow = (o0 + oc == d.L_s) ? P - o0 : oc;   // last chunk also zero-fills the pitch padding
                for (int idx = tid; idx < tv * ow; idx += kFusedThreads) {
                    const int vj = idx / ow, t = idx - vj * ow;
                    outp[(size_t)(v0 + vj) * P + o0 + t] = t < oc ? out_s[t * TVP + vj] : T(0);
                }
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
bool plan_fused(StageDesc &d, bool fp64, int sm_count, FusedConfig &cfg)
{
    const size_t es = fp64 ? 8 : 4;
    const int CH = fp64 ? 2 : 4;
    const int La_rows = d.aux_leaf ? d.k : d.L_a;
    const int Lm_rows = d.main_leaf ? 0 : d.L_m;
    const int nchunk = (d.L_a + CH - 1) / CH;
    // lanes per vertex in the gather: enough that a lane holds <= 8 chunks
    int G = 1;
    while (G < 32 && G * 4 < nchunk) G *= 2;
    int q = (nchunk + G - 1) / G;
    q = q <= 1 ? 1 : q <= 2 ? 2 : q <= 4 ? 4 : 8;
    d.gather_group = d.aux_leaf ? 32 : G;
    cfg.q = d.aux_leaf ? 1 : q;
    const size_t limit_fast = 113 * 1024, limit_max = 227 * 1024;
    for (int pass = 0; pass < 2; ++pass) {
        const size_t limit = pass == 0 ? limit_fast : limit_max;
        for (int tv : {32, 16, 8}) {
            const int oc = (d.is_root || d.main_leaf) ? 0 : std::min(d.L_s, 64);
            size_t bytes = ((size_t)(La_rows + Lm_rows + oc) * (tv + 1) * es + 15) / 16 * 16;
            bytes += (size_t)tv * sizeof(double);
            if (bytes <= limit) {
                cfg.tile_v = tv;
                cfg.smem = bytes;
                d.tile_v = tv;
                d.out_chunk = oc;
                d.ntiles = (d.V + tv - 1) / tv;
                cfg.grid = sm_count;   // scaled by the occupancy at launch
                return true;
            }
        }
    }
    return false;
}

template <typename T, int TV>
static void launch_fused_q(const StageDesc &d, const FusedConfig &cfg, cudaStream_t st)
{
    auto go = [&](auto kern) {
        if (cfg.smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFusedThreads, cfg.smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        const int grid = std::max(1, std::min(d.ntiles, cfg.grid * per_sm));
        kern<<<grid, kFusedThreads, cfg.smem, st>>>(d);
    };
    switch (cfg.q) {
    case 1: go(k_fused<T, TV, 1>); break;
    case 2: go(k_fused<T, TV, 2>); break;
    case 4: go(k_fused<T, TV, 4>); break;
    default: go(k_fused<T, TV, 8>); break;
    }
}

void launch_fused(const StageDesc &d, bool fp64, const FusedConfig &cfg, cudaStream_t st)
{
    if (d.V == 0) return;
    if (fp64) {
        if (cfg.tile_v == 32) launch_fused_q<double, 32>(d, cfg, st);
        else if (cfg.tile_v == 16) launch_fused_q<double, 16>(d, cfg, st);
        else launch_fused_q<double, 8>(d, cfg, st);
    } else {
        if (cfg.tile_v == 32) launch_fused_q<float, 32>(d, cfg, st);
        else if (cfg.tile_v == 16) launch_fused_q<float, 16>(d, cfg, st);
        else launch_fused_q<float, 8>(d, cfg, st);
    }
}

// ---------------------------------------------------------------------------
// Hub aggregation: item = (hub vertex, neighbour chunk).  One CTA per item,
// threads over the row's 16-byte chunks, neighbours of the chunk in order.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_hub_partial(HubArgs h)
{
    using CT = Chunk<T>;
    using C = typename CT::type;
    constexpr int CH = CT::n;
    for (int item = blockIdx.x; item < h.total_chunks; item += gridDim.x) {
        // hub of this chunk: last hub whose first chunk <= item
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
            // per-color counts of the chunk: exact integers, any order
            __shared__ uint32_t cnt[32];
            if (threadIdx.x < 32) cnt[threadIdx.x] = 0;
            __syncthreads();
            for (int e = beg + (int)threadIdx.x; e < end; e += blockDim.x)
                atomicAdd(&cnt[__ldg(h.color + __ldg(h.adj + e))], 1u);
            __syncthreads();
            if ((int)threadIdx.x < h.k_leaf) prow[threadIdx.x] = (T)cnt[threadIdx.x];
            __syncthreads();
        } else {
            const int nchunk = (h.L_a + CH - 1) / CH;
            const int rowc = h.aux_pitch / CH;
            const C *auxc = reinterpret_cast<const C *>(h.aux);
            for (int q = threadIdx.x; q < nchunk; q += blockDim.x) {
                C acc = CT::zero();
                int e = beg;
                for (; e + 4 <= end; e += 4) {
                    const C x0 = __ldg(auxc + (size_t)__ldg(h.adj + e) * rowc + q);
                    const C x1 = __ldg(auxc + (size_t)__ldg(h.adj + e + 1) * rowc + q);
                    const C x2 = __ldg(auxc + (size_t)__ldg(h.adj + e + 2) * rowc + q);
                    const C x3 = __ldg(auxc + (size_t)__ldg(h.adj + e + 3) * rowc + q);
                    CT::add(acc, x0);
                    CT::add(acc, x1);
                    CT::add(acc, x2);
                    CT::add(acc, x3);
                }
                for (; e < end; ++e) CT::add(acc, __ldg(auxc + (size_t)__ldg(h.adj + e) * rowc + q));
                reinterpret_cast<C *>(prow)[q] = acc;
            }
        }
    }
}

template <typename T>
__global__ void k_hub_combine(HubArgs h, int ncols)
{
    for (int v = blockIdx.x; v < h.hub_count; v += gridDim.x) {
        const int c0 = __ldg(h.chunk_start + v), c1 = __ldg(h.chunk_start + v + 1);
        const T *p = reinterpret_cast<const T *>(h.partial);
        T *out = reinterpret_cast<T *>(h.hub_agg) + (size_t)v * h.row_pitch;
        for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
            T acc = p[(size_t)c0 * h.row_pitch + c];
            for (int ch = c0 + 1; ch < c1; ++ch) {
                const T x = p[(size_t)ch * h.row_pitch + c];
                if (sizeof(T) == 8) acc = (T)__dadd_rn((double)acc, (double)x);
                else acc = (T)__fadd_rn((float)acc, (float)x);
            }
            out[c] = acc;
        }
    }
}

void launch_hub(const HubArgs &h, bool fp64, int sm_count, cudaStream_t st)
{
    if (h.hub_count == 0) return;
    const int grid = std::max(1, std::min(h.total_chunks, sm_count * 8));
    const int ncols = h.k_leaf ? h.k_leaf : h.L_a;
    if (fp64) {
        k_hub_partial<double><<<grid, 256, 0, st>>>(h);
        k_hub_combine<double><<<std::min(h.hub_count, sm_count * 4), 256, 0, st>>>(h, ncols);
    } else {
        k_hub_partial<float><<<grid, 256, 0, st>>>(h);
        k_hub_combine<float><<<std::min(h.hub_count, sm_count * 4), 256, 0, st>>>(h, ncols);
    }
}

// ---------------------------------------------------------------------------
// K3: the per-coloring sum of the root partials, FP64 with Kahan
// compensation, in a fixed order (one CTA, strided per thread, then a
// fixed-shape tree), times the scale (1e12 for the pruned modes).
// ---------------------------------------------------------------------------
__global__ void k_root_reduce(const double *__restrict__ partial, int32_t n, double scale, double *out)
{
    __shared__ double ss[256], cc[256];
    double s = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double y = __dadd_rn(partial[i], -c);
        const double t = __dadd_rn(s, y);
        c = __dadd_rn(__dadd_rn(t, -s), -y);
        s = t;
    }
    ss[threadIdx.x] = s;
    cc[threadIdx.x] = c;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            ss[threadIdx.x] = __dadd_rn(ss[threadIdx.x], ss[threadIdx.x + w]);
            cc[threadIdx.x] = __dadd_rn(cc[threadIdx.x], cc[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = __dmul_rn(__dadd_rn(ss[0], -cc[0]), scale);
}

void launch_root_reduce(const double *partial, int32_t n, double scale, double *out, cudaStream_t st)
{
    k_root_reduce<<<1, 256, 0, st>>>(partial, n, scale, out);
}

}  // namespace sg
