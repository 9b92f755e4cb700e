// Allocation-free 2-norm (include/eqg_noalloc.h).
//
// Same arithmetic as the runtime's two-norm: squares summed per block, the
// block sums added by the last block to finish.  The block sums and the
// completion counter live in g_noalloc_scratch, a file-scope device array,
// instead of runtime-allocated scratch, so the call allocates nothing.
#include "eqg.h"
#include "eqg_noalloc.h"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace eqg {
void set_last_error(const std::string& msg);
}

namespace {

constexpr int kNoallocThreads = 256;
constexpr int64_t kNoallocMaxBlocks = EQG_NOALLOC_MAX_ELEMENTS / kNoallocThreads;

// kNoallocMaxBlocks block sums, then one word for the completion counter:
// 512 KiB per device, held from module load until process exit.
static __device__ __align__(256) double g_noalloc_scratch[kNoallocMaxBlocks + 32];

__global__ void two_norm_noalloc_kernel(const double* __restrict__ x, int64_t n, double* __restrict__ result,
                                        double* scratch)
{
    __shared__ double sh[kNoallocThreads];
    __shared__ bool last;
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kNoallocMaxBlocks);
    const int64_t i = (int64_t)blockIdx.x * kNoallocThreads + threadIdx.x;
    const double v = i < n ? x[i] : 0.0;
    sh[threadIdx.x] = v * v;
    __syncthreads();
    for (int s = kNoallocThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scratch[blockIdx.x] = sh[0];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kNoallocThreads) acc += ((volatile double*)scratch)[b];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kNoallocThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *result = sqrt(sh[0]);
        *counter = 0u;
    }
}

// Device address of the scratch array, looked up once per device with that
// device current.
std::mutex g_addr_mutex;
double* g_addr[256] = {nullptr};

int scratch_address(double** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        eqg::set_last_error(std::string("eqg_two_norm_noalloc: cudaGetDevice failed: ") + cudaGetErrorString(e));
        return EQG_ERR_DEVICE;
    }
    if (dev < 0 || dev >= 256) {
        eqg::set_last_error("eqg_two_norm_noalloc: device index out of range");
        return EQG_ERR_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            eqg::set_last_error(std::string("eqg_two_norm_noalloc: cudaGetSymbolAddress failed: ") +
                                cudaGetErrorString(e));
            return EQG_ERR_DEVICE;
        }
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return EQG_OK;
}

}  // namespace

extern "C" int eqg_two_norm_noalloc(const double* x, int64_t n, double* result, void* stream)
{
    if (n < 0 || n > EQG_NOALLOC_MAX_ELEMENTS) {
        eqg::set_last_error("eqg_two_norm_noalloc: n = " + std::to_string(n) + " is outside [0, " +
                            std::to_string(EQG_NOALLOC_MAX_ELEMENTS) + "] (the scratch holds " +
                            std::to_string(kNoallocMaxBlocks) + " partial sums of 256 elements)");
        return EQG_ERR_ARG;
    }
    if (!result || (!x && n > 0)) {
        eqg::set_last_error("eqg_two_norm_noalloc: null input or output pointer");
        return EQG_ERR_ARG;
    }
    double* scratch = nullptr;
    const int st = scratch_address(&scratch);
    if (st != EQG_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the completion counter must start at zero; the partial sums need no clearing
    cudaError_t e = cudaMemsetAsync(scratch + kNoallocMaxBlocks, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess) {
        const int64_t blocks = n > 0 ? (n + kNoallocThreads - 1) / kNoallocThreads : 1;
        two_norm_noalloc_kernel<<<(unsigned)blocks, kNoallocThreads, 0, s>>>(x, n, result, scratch);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        eqg::set_last_error(std::string("eqg_two_norm_noalloc: ") + cudaGetErrorString(e));
        return EQG_ERR_DEVICE;
    }
    return EQG_OK;
}
