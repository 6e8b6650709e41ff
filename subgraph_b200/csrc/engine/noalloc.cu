// sg_colors_noalloc: the coloring kernel for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc: frameworks that reserve all device
// memory in their own pool at start-up and hand out only views of it, and
// pipelines where an allocation's implicit device synchronisation is not
// acceptable.  This entry point allocates nothing: the caller passes the output
// buffer, and the kernel's scratch (the jump-ahead polynomials of the glibc
// stream) lives in the file-scope array below, which every GPU that loads the
// library holds until the process exits.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../../include/sg_api.h"

namespace sg {
void glibc_window(uint32_t seed, uint32_t w[31]);
void set_last_error(const std::string &msg);   // the message sg_last_error() returns
}

namespace {

constexpr int kBlock = 1024;                                 // vertices per block
constexpr int64_t kMaxVertices = int64_t(1) << 26;           // 67,108,864
constexpr int64_t kMaxBlocks = kMaxVertices / kBlock;        // 65,536
// scratch words: [31][kBlock] coefficients of x^t, then [kMaxBlocks][31] jump
// polynomials x^(341 + b*kBlock) mod P  (8.3 MB in all)
constexpr int64_t kCoefWords = 31 * kBlock;
constexpr int64_t kScratchWords = kCoefWords + kMaxBlocks * 31;

static __device__ __align__(256) uint32_t g_color_scratch[kScratchWords];

struct DeviceSetup {
    uint32_t *scratch = nullptr;   // device address of g_color_scratch on this device
};
std::mutex g_mu;
std::vector<DeviceSetup> g_setup;

using Poly = std::vector<uint32_t>;

Poly mulmod(const Poly &a, const Poly &b)
{
    uint32_t c[61] = {0};
    for (int i = 0; i < 31; ++i)
        if (a[i])
            for (int j = 0; j < 31; ++j) c[i + j] += a[i] * b[j];
    for (int d = 60; d >= 31; --d) {   // x^31 = x^28 + 1
        c[d - 3] += c[d];
        c[d - 31] += c[d];
    }
    return Poly(c, c + 31);
}

Poly xpow(uint64_t n)
{
    Poly r(31, 0), b(31, 0);
    r[0] = 1;
    b[1] = 1;
    for (; n; n >>= 1) {
        if (n & 1) r = mulmod(r, b);
        b = mulmod(b, b);
    }
    return r;
}

struct Window {
    uint32_t w[31];
};

// colors[v] = rand() % k for v = 0..V-1 after srand(seed), in vertex order
// (the reference's CountMat::colorInit on one thread, CountMat.cpp:979-991)
__global__ void __launch_bounds__(kBlock) k_color_noalloc(int32_t V, int32_t k, Window w0, int32_t *colors)
{
    __shared__ uint32_t W[31];
    const uint32_t *coef = g_color_scratch;
    const uint32_t *jump = g_color_scratch + kCoefWords + (size_t)blockIdx.x * 31;
    if (threadIdx.x < 31) {
        uint32_t q[31];
#pragma unroll
        for (int j = 0; j < 31; ++j) q[j] = jump[j];
        for (int s = 0; s < (int)threadIdx.x; ++s) {
            const uint32_t t = q[30];
#pragma unroll
            for (int j = 30; j > 0; --j) q[j] = q[j - 1];
            q[0] = t;
            q[28] += t;
        }
        uint32_t acc = 0;
#pragma unroll
        for (int j = 0; j < 31; ++j) acc += q[j] * w0.w[j];
        W[threadIdx.x] = acc;
    }
    __syncthreads();
    const int64_t v = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    if (v < V) {
        uint32_t s = 0;
#pragma unroll
        for (int i = 0; i < 31; ++i) s += coef[i * kBlock + threadIdx.x] * W[i];
        colors[v] = (int32_t)(s >> 1) % k;
    }
}

sg_status fail(sg_status code, const std::string &msg)
{
    sg::set_last_error("sg_colors_noalloc: " + msg);
    return code;
}

// Fills the whole scratch array for the current device: the coefficients of
// x^t (t < kBlock) and the jump polynomials of every block a call of up to
// kMaxVertices vertices can launch.  None of it depends on the seed or on V, so
// it is written once per device and only read afterwards.  The copy is a plain
// synchronous cudaMemcpy from host memory (no device allocation).
sg_status setup_device(DeviceSetup &ds)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_color_scratch);
    if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    std::vector<uint32_t> tab((size_t)kScratchWords);
    Poly q(31, 0);
    q[0] = 1;
    for (int t = 0; t < kBlock; ++t) {
        for (int i = 0; i < 31; ++i) tab[(size_t)i * kBlock + t] = q[i];
        const uint32_t top = q[30];
        for (int j = 30; j > 0; --j) q[j] = q[j - 1];
        q[0] = top;
        q[28] += top;
    }
    Poly J = xpow(341), step = xpow(kBlock);
    for (int64_t b = 0; b < kMaxBlocks; ++b) {
        std::memcpy(&tab[(size_t)(kCoefWords + b * 31)], J.data(), 31 * 4);
        J = mulmod(J, step);
    }
    e = cudaMemcpy(p, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("scratch set-up: ") + cudaGetErrorString(e));
    ds.scratch = (uint32_t *)p;
    return SG_OK;
}

}  // namespace

extern "C" sg_status sg_colors_noalloc(int32_t V, int32_t k, uint32_t seed, int32_t *d_colors, void *stream)
{
    try {
        if (V < 0 || V > kMaxVertices) {
            return fail(SG_ERR_INVALID,
                        "V must be in [0, 2^26] (the scratch array holds jump tables for 2^26 vertices)");
        }
        if (k < 1 || (V > 0 && !d_colors)) {
            return fail(SG_ERR_INVALID, "k must be >= 1 and the output buffer non-null");
        }
        if (V == 0) return SG_OK;
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            return fail(SG_ERR_CUDA, "no current CUDA device");
        }
        {
            std::lock_guard<std::mutex> lk(g_mu);
            if ((int)g_setup.size() <= dev) g_setup.resize(dev + 1);
            if (!g_setup[dev].scratch) {
                const sg_status st = setup_device(g_setup[dev]);
                if (st != SG_OK) return st;
            }
        }
        cudaStream_t st = (cudaStream_t)stream;
        const int64_t nblocks = (V + kBlock - 1) / kBlock;
        Window w0;
        sg::glibc_window(seed, w0.w);
        k_color_noalloc<<<(unsigned)nblocks, kBlock, 0, st>>>(V, k, w0, d_colors);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            return fail(SG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
        }
        return SG_OK;
    } catch (const std::bad_alloc &) {
        return fail(SG_ERR_OOM, "host allocation failed");
    } catch (const std::exception &ex) {
        return fail(SG_ERR_CUDA, ex.what());
    }
}
