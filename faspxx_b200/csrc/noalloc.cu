// noalloc.cu -- fasp_gpu_vec_dot_noalloc: the dot product of fasp_gpu_vec_dot for callers
// that must not allocate device memory.
//
// fasp_gpu_vec_dot creates a per-thread context on first use (a stream, reduction scratch,
// pinned host memory). Some callers cannot do that: an application whose memory pool has
// reserved the device memory up front and forbids further driver allocations, and
// latency-critical loops in which cudaMalloc/cudaFree would synchronize the device. This
// variant keeps its scratch in a file-scope device array instead, created with the module
// and held by every GPU that loads the library until the process exits:
//   - one partial sum per block (kNoAllocMaxBlocks doubles), a block ticket and the result,
//     about 32 KB in all;
//   - each block sums a fixed chunk of kNoAllocChunk elements, so n is limited to
//     kNoAllocMaxBlocks * kNoAllocChunk = 8,388,608; larger n returns ERROR_VEC_SIZE (-14)
//     without touching the GPU.
// It runs on the device chosen by fasp_gpu_init (the calling thread's current device is
// switched to it for the call and restored afterwards), on that device's legacy default
// stream, and blocks until the result has been copied to the host.
// Every call shares the one array and leaves its contents behind: the ticket is cleared at
// the start of each call, the partials and the result are overwritten. Calls whose work
// overlaps on the GPU (several host threads, or device work still running from an earlier
// call on another stream) race on the array; callers must serialise them.
// The first call on each device looks up the array's device address (cudaGetSymbolAddress)
// with that device current and keeps it for later calls; make that first call before any
// stream capture begins. The kept address does not survive cudaDeviceReset (the module is
// reloaded and the array may move): do not use this entry point after a device reset.
#include <mutex>

#include "../../include/fasp_b200.h"
#include "internal.h"

namespace fb {

constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocPerThread = 8;
constexpr int kNoAllocChunk = kNoAllocBlock * kNoAllocPerThread;  // elements per block
constexpr int kNoAllocMaxBlocks = 4096;
constexpr unsigned long long kNoAllocMaxN =
    (unsigned long long)kNoAllocMaxBlocks * kNoAllocChunk;        // 8,388,608

struct NoAllocScratch {
    double   partials[kNoAllocMaxBlocks];
    unsigned ticket;
    unsigned pad;
    double   result;
};

static __device__ __align__(256) NoAllocScratch g_dot_scratch;

// Block b sums elements [b*chunk, (b+1)*chunk) in a fixed order; the last block to finish
// adds the partials in block order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(kNoAllocBlock)
k_dot_noalloc(uint32_t n, const double* __restrict__ a, const double* __restrict__ b,
              NoAllocScratch* s)
{
    __shared__ bool amLast;
    const size_t base = (size_t)blockIdx.x * kNoAllocChunk + threadIdx.x;
    double acc[1] = {0.0};
    const int ops[1] = {kSum};
#pragma unroll
    for (int k = 0; k < kNoAllocPerThread; ++k) {
        const size_t i = base + (size_t)k * kNoAllocBlock;
        if (i < n) acc[0] = fma(a[i], b[i], acc[0]);
    }
    block_reduce<1>(acc, ops);
    if (threadIdx.x == 0) {
        s->partials[blockIdx.x] = acc[0];
        __threadfence();
        amLast = atomicAdd(&s->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!amLast) return;
    __threadfence();
    double tot[1] = {0.0};
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
        tot[0] += __ldcg(&s->partials[i]);
    block_reduce<1>(tot, ops);
    if (threadIdx.x == 0) {
        s->result = tot[0];
        s->ticket = 0;
    }
}

// Device address of g_dot_scratch per device, looked up once with that device current.
static NoAllocScratch* scratch_for_current_device(int* err)
{
    constexpr int kMaxDevices = 64;
    static NoAllocScratch* addr[kMaxDevices] = {};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        *err = kErrNoDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_dot_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            *err = kErrCuda;
            return nullptr;
        }
        addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *err = kOk;
    return addr[dev];
}

} // namespace fb

extern "C" int fasp_gpu_vec_dot_noalloc(uint32_t n, const double* a, const double* b,
                                        double* result)
{
    using namespace fb;
    if (!result || (n && (!a || !b))) return kErrInputPar;
    if ((unsigned long long)n > kNoAllocMaxN) {
        std::fprintf(stderr,
                     "fasp_gpu_vec_dot_noalloc: n = %u exceeds the static scratch limit of "
                     "%llu elements\n",
                     n, kNoAllocMaxN);
        return kErrVecSize;
    }
    if (n == 0) {
        *result = 0.0;
        return kOk;
    }
    // run on the library's device; the caller's current device is restored on return
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) {
        cudaGetLastError();
        return kErrNoDevice;
    }
    const int dev = library_device();
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        return kErrNoDevice;
    }
    int err = kOk;
    NoAllocScratch* s = scratch_for_current_device(&err);
    if (s) {
        const int grid = (int)((n + kNoAllocChunk - 1) / kNoAllocChunk);
        // legacy default stream: ordered after the caller's earlier default-stream work
        if (cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned), 0) != cudaSuccess) err = kErrCuda;
        if (!err) {
            k_dot_noalloc<<<grid, kNoAllocBlock, 0, 0>>>(n, a, b, s);
            if (cudaGetLastError() != cudaSuccess) err = kErrCuda;
        }
        if (!err && cudaMemcpy(result, &s->result, sizeof(double), cudaMemcpyDeviceToHost) !=
                        cudaSuccess)
            err = kErrCuda;
        if (err) cudaGetLastError();
    }
    if (prev != dev) cudaSetDevice(prev);
    return err;
}
