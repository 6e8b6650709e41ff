// The batched form: one persistent launch runs every (coloring, sub-template)
// stage of a batch of colorings from a work queue.
//
// Items are numbered stage by stage in an order where every stage comes after
// the stages it reads (sub-templates in processing order, colorings
// interleaved), so a claimed item only ever waits for lower-numbered items,
// which were claimed by CTAs that are already running: the queue cannot
// deadlock.  A stage's completion is an item counter; a CTA's thread 0 waits
// on the counters of the stage's inputs with acquire loads, bounded by a
// cycle budget after which it raises the batch's error flag (every later wait
// then returns at once and the host reports SG_ERR_TIMEOUT).  Tables produced
// inside the launch are read through L2 (fused_tile<..., COH = true>).
#include "kernels.cuh"
#include "tile.cuh"

namespace sg {

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <typename T>
__device__ __forceinline__ void batch_fused(const StageDesc &d, int tile, unsigned char *smem)
{
    constexpr int NT = kBatchThreads;
    if (sizeof(T) == 4 && d.packed == 1) {
        switch (d.gather_q) {
        case 1: fused_tile<T, NT, 1, true, true>(d, tile, smem); break;
        case 2: fused_tile<T, NT, 2, true, true>(d, tile, smem); break;
        default: fused_tile<T, NT, 4, true, true>(d, tile, smem); break;
        }
    } else {
        switch (d.gather_q) {
        case 1: fused_tile<T, NT, 1, false, true>(d, tile, smem); break;
        case 2: fused_tile<T, NT, 2, false, true>(d, tile, smem); break;
        default: fused_tile<T, NT, 4, false, true>(d, tile, smem); break;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kBatchThreads, 2)
    k_persistent(const BatchStage *__restrict__ stages, int nstages, int total_items, int *done, BatchCtl *ctl,
                 long long wait_cycles, unsigned long long *stage_end)
{
    extern __shared__ __align__(32) unsigned char smem_raw[];
    __shared__ BatchStage st;
    __shared__ int s_item, s_stage, s_skip, s_cur;
    if (threadIdx.x == 0) s_cur = -1;   // the stage whose descriptor is in `st`
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(&ctl->next_item, 1);
            if (s_item == 0 && stage_end) ctl->t0 = global_ns();
        }
        __syncthreads();
        const int item = s_item;
        if (item >= total_items) break;
        if (threadIdx.x == 0) {
            int lo = 0, hi = nstages - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (stages[mid].first_item <= item) lo = mid; else hi = mid - 1;
            }
            s_stage = lo;
            const BatchStage &bs = stages[lo];
            for (int q = 0; q < bs.ndeps; ++q) {
                const int dep = bs.deps[q];
                const int need = stages[dep].nitems;
                const long long t0 = clock64();
                while (ld_acquire(done + dep) < need) {
                    if (ld_acquire(&ctl->error)) break;
                    if (clock64() - t0 > wait_cycles) {
                        if (atomicCAS(&ctl->error, 0, 1) == 0) ctl->error_stage = lo;
                        break;
                    }
                    __nanosleep(256);
                }
            }
            s_skip = ld_acquire(&ctl->error);
        }
        __syncthreads();
        if (s_stage != s_cur) {   // the stage descriptor into shared memory, when it changes
            const int *src = reinterpret_cast<const int *>(stages + s_stage);
            int *dst = reinterpret_cast<int *>(&st);
            for (int i = threadIdx.x; i < (int)(sizeof(BatchStage) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) s_cur = s_stage;   // read again only after the barriers below
        if (!s_skip) {
            const int local = item - st.first_item;
            if (st.kind == kStageHub) {
                const int c1 = min((local + 1) * kHubItemChunks, st.h.total_chunks);
                for (int ch = local * kHubItemChunks; ch < c1; ++ch) hub_item<T, kBatchThreads, true>(st.h, ch, smem_raw);
            } else {
                const int t0 = local * st.tiles_per_item;
                const int t1 = min(t0 + st.tiles_per_item, st.d.ntiles);
                for (int t = t0; t < t1; ++t) batch_fused<T>(st.d, t, smem_raw);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const int prev = atomicAdd(done + s_stage, 1);
            // the CTA that completes a stage stamps its end (job latencies)
            if (stage_end && prev + 1 == st.nitems) stage_end[s_stage] = global_ns();
        }
    }
}

// per-slot root sums of a batch (one CTA per coloring slot), FP64 Kahan in a
// fixed order like k_root_reduce
__global__ void k_root_reduce_slots(const double *__restrict__ partial, int64_t slot_stride, int32_t n,
                                    const int32_t *__restrict__ n_slot, double scale, double *out)
{
    __shared__ double ss[256], cc[256], pp[256];
    const double *p = partial + (size_t)blockIdx.x * slot_stride;
    if (n_slot) n = n_slot[blockIdx.x];   // jobs of different templates: their own tile counts
    const double r = block_sum_partials(p, n, scale, ss, cc, pp);
    if (threadIdx.x == 0) out[blockIdx.x] = r;
}

cudaError_t launch_persistent(const BatchStage *stages, int nstages, int total_items, int *done, BatchCtl *ctl,
                              long long wait_cycles, size_t smem, bool fp64, int sm_count, cudaStream_t st,
                              unsigned long long *stage_end)
{
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        // every resident CTA claims items (a claimed item only waits for items
        // claimed earlier by running CTAs, so residency needs no guarantee)
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchThreads, smem) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        kern<<<sm_count * per_sm, kBatchThreads, smem, st>>>(stages, nstages, total_items, done, ctl, wait_cycles,
                                                               stage_end);
    };
    if (fp64) go(k_persistent<double>);
    else go(k_persistent<float>);
    return cudaGetLastError();
}

void launch_root_reduce_slots(const double *partial, int64_t slot_stride, int32_t n, double scale, double *out,
                              int nslots, cudaStream_t st, const int32_t *n_slot)
{
    if (nslots > 0) k_root_reduce_slots<<<nslots, 256, 0, st>>>(partial, slot_stride, n, n_slot, scale, out);
}

}  // namespace sg
