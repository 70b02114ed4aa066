// segsort.cuh -- device building blocks for constructing CSR matrices: an exclusive scan
// of row counts and a segmented sort of 64-bit keys within row segments (register bitonic
// networks for short rows, a shared-memory bitonic network per segment of up to 4,096
// keys, merge passes above that). Used by the ReadMat conversions (ingest.cu) and the
// sparse matrix product (spgemm.cu). Everything here has internal linkage.
#pragma once

#include <algorithm>
#include <vector>

#include "internal.h"

namespace fb {
namespace {


constexpr int      kScanThreads = 256;
constexpr uint32_t kTile = kScanThreads * 8; // elements per scan tile
constexpr int      kSegMax = 4096;           // keys one block sorts in shared memory
constexpr int      kSegThreads = 512;
constexpr uint64_t kPad = ~0ull;

// Device memory released when the conversion returns (cudaFree waits for the device).
struct Tmp {
    std::vector<void*> ptrs;
    ~Tmp()
    {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    int get(T** p, size_t count)
    {
        *p = nullptr;
        if (cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            return kErrAlloc;
        }
        ptrs.push_back(*p);
        return kOk;
    }
};

inline int grid_for(size_t work, int block)
{
    return (int)std::max<size_t>(1, std::min<size_t>((work + block - 1) / block, 148 * 16));
}

// ---- exclusive scan of uint32 counts: out[0] = 0, out[i+1] = out[i] + in[i] ----------------

// Exclusive scan of one value per thread across the block; *total gets the block's sum.
__device__ uint32_t block_exclusive(uint32_t v, uint32_t* total)
{
    __shared__ uint32_t ws[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < nw ? ws[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        ws[lane] = s;
    }
    __syncthreads();
    const uint32_t excl = x - v + (wid ? ws[wid - 1] : 0u);
    *total = ws[nw - 1];
    __syncthreads();
    return excl;
}

__global__ void __launch_bounds__(kScanThreads) k_tile_sums(uint32_t n, const uint32_t* __restrict__ in,
                                                             uint32_t* __restrict__ sums)
{
    const size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * 8;
    uint32_t s = 0;
    for (int j = 0; j < 8; ++j)
        if (base + j < n) s += in[base + j];
    uint32_t total;
    block_exclusive(s, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One block: exclusive scan of the tile sums in place; out[n] = the grand total.
__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t nt, uint32_t* __restrict__ sums,
                                                     uint32_t* __restrict__ outTotal)
{
    uint32_t carry = 0;
    for (size_t c0 = 0; c0 < nt; c0 += (size_t)blockDim.x * 8) {
        const size_t base = c0 + (size_t)threadIdx.x * 8;
        uint32_t v[8], s = 0;
        for (int j = 0; j < 8; ++j) {
            v[j] = base + j < nt ? sums[base + j] : 0u;
            s += v[j];
        }
        uint32_t total;
        uint32_t e = block_exclusive(s, &total) + carry;
        for (int j = 0; j < 8; ++j) {
            if (base + j < nt) sums[base + j] = e;
            e += v[j];
        }
        carry += total;
    }
    if (threadIdx.x == 0) *outTotal = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(uint32_t n, const uint32_t* __restrict__ in,
                                                              const uint32_t* __restrict__ sums,
                                                              uint32_t* __restrict__ out)
{
    const size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * 8;
    uint32_t v[8], s = 0;
    for (int j = 0; j < 8; ++j) {
        v[j] = base + j < n ? in[base + j] : 0u;
        s += v[j];
    }
    uint32_t total;
    uint32_t e = block_exclusive(s, &total) + sums[blockIdx.x];
    for (int j = 0; j < 8; ++j) {
        if (base + j < n) out[base + j] = e;
        e += v[j];
    }
}

// out has n + 1 entries; tileSums has ceil(n / kTile) entries. n > 0.
int scan_counts(cudaStream_t s, uint32_t n, const uint32_t* in, uint32_t* out, uint32_t* tileSums)
{
    const uint32_t nt = (uint32_t)((n + (size_t)kTile - 1) / kTile);
    k_tile_sums<<<nt, kScanThreads, 0, s>>>(n, in, tileSums);
    k_scan_sums<<<1, 1024, 0, s>>>(nt, tileSums, out + n);
    k_scan_apply<<<nt, kScanThreads, 0, s>>>(n, in, tileSums, out);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

// ---- row sorts ------------------------------------------------------------------------------

// Rows with lo < length <= G, one group of G lanes per row, bitonic network in registers.
// Every lane of the warp takes part in every shuffle; rows outside the class sort padding.
template <int G>
__global__ void __launch_bounds__(256) k_sort_short(uint32_t nrow, uint32_t lo,
                                                    const uint32_t* __restrict__ rowPtr,
                                                    uint64_t* __restrict__ keys)
{
    const int lane = threadIdx.x % G;
    const size_t groups = (size_t)gridDim.x * blockDim.x / G;
    for (size_t r0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G; r0 < (nrow + groups - 1) / groups * groups;
         r0 += groups) {
        uint32_t b = 0, len = 0;
        if (r0 < nrow) {
            b = rowPtr[r0];
            len = rowPtr[r0 + 1] - b;
        }
        const bool mine = r0 < nrow && len > lo && len <= (uint32_t)G;
        uint64_t v = mine && (uint32_t)lane < len ? keys[b + lane] : kPad;
#pragma unroll
        for (int k = 2; k <= G; k <<= 1)
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                const uint64_t o = __shfl_xor_sync(0xffffffffu, v, j, G);
                const bool keepMin = ((lane & j) == 0) == ((lane & k) == 0);
                v = keepMin ? (o < v ? o : v) : (o > v ? o : v);
            }
        if (mine && (uint32_t)lane < len) keys[b + lane] = v;
    }
}

// One block per segment (start, length <= kSegMax): bitonic network in shared memory.
__global__ void __launch_bounds__(kSegThreads) k_sort_segment(const uint2* __restrict__ segs,
                                                               uint64_t* __restrict__ keys)
{
    __shared__ uint64_t sh[kSegMax];
    const uint2 sg = segs[blockIdx.x];
    uint32_t P = 64;
    while (P < sg.y) P <<= 1;
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) sh[i] = i < sg.y ? keys[sg.x + i] : kPad;
    __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const uint64_t a = sh[i], c = sh[l];
                    if ((a > c) == ((i & k) == 0)) {
                        sh[i] = c;
                        sh[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (uint32_t i = threadIdx.x; i < sg.y; i += blockDim.x) keys[sg.x + i] = sh[i];
}

// Number of keys in a[0, n) below k (a sorted ascending).
__device__ __forceinline__ uint32_t count_below(const uint64_t* a, uint32_t n, uint64_t k)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (a[mid] < k)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// One merge pass over long rows (start, length): sorted runs of w keys are merged in pairs.
// A key's place in the merged pair is its place in its own run plus the number of keys below
// it in the other run (keys are unique, so no two keys compete for a place).
__global__ void k_merge_pass(uint32_t nh, const uint2* __restrict__ rows, uint32_t w,
                             const uint64_t* __restrict__ in, uint64_t* __restrict__ out)
{
    for (uint32_t h = blockIdx.y; h < nh; h += gridDim.y) {
        const uint2 rg = rows[h];
        const uint64_t* src = in + rg.x;
        uint64_t* dst = out + rg.x;
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < rg.y;
             i += (size_t)gridDim.x * blockDim.x) {
            const size_t run = i / w;
            const size_t left = (run & ~(size_t)1) * w;
            const size_t right = left + w;
            const uint64_t k = src[i];
            size_t pos;
            if (right >= rg.y) {
                pos = i; // an unpaired last run stays where it is
            } else if ((run & 1) == 0) {
                const uint32_t rn = (uint32_t)std::min<size_t>(w, rg.y - right);
                pos = i + count_below(src + right, rn, k);
            } else {
                pos = left + (i - right) + count_below(src + left, w, k);
            }
            dst[pos] = k;
        }
    }
}

__global__ void k_copy_rows(uint32_t nh, const uint2* __restrict__ rows,
                            const uint64_t* __restrict__ in, uint64_t* __restrict__ out)
{
    for (uint32_t h = blockIdx.y; h < nh; h += gridDim.y) {
        const uint2 rg = rows[h];
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < rg.y;
             i += (size_t)gridDim.x * blockDim.x)
            out[rg.x + i] = in[rg.x + i];
    }
}

int read_flag(cudaStream_t s, const int* dflag, int* hflag)
{
    FB_CUDA(cudaMemcpyAsync(hflag, dflag, sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    return kOk;
}

template <typename T>
int stage(Tmp& t, cudaStream_t s, const T* src, size_t count, bool onDevice, const T** out)
{
    if (onDevice) {
        *out = src;
        return kOk;
    }
    T* d = nullptr;
    int e = t.get(&d, count);
    if (e) return e;
    FB_CUDA(cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
    *out = d;
    return kOk;
}


// Sorts the keys of every row segment [rowPtr[r], rowPtr[r + 1]) ascending (rowPtr on the
// device, 0-based; keys unique within a row, so the order is fully determined).
int sort_row_keys(Ctx& c, Tmp& t, uint32_t nrow, const uint32_t* rowPtr, uint64_t* keys,
                  uint32_t nkeys)
{
    cudaStream_t s = c.stream;
    int e;
    std::vector<uint32_t> hrp((size_t)nrow + 1);
    FB_CUDA(cudaMemcpyAsync(hrp.data(), rowPtr, hrp.size() * 4, cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    // row classes by length
    std::vector<uint2> segs, huge;
    uint32_t maxHuge = 0;
    bool small8 = false, small32 = false;
    for (uint32_t r = 0; r < nrow; ++r) {
        const uint32_t b = hrp[r], len = hrp[r + 1] - b;
        if (len <= 1) continue;
        if (len <= 8) {
            small8 = true;
        } else if (len <= 32) {
            small32 = true;
        } else if (len <= (uint32_t)kSegMax) {
            segs.push_back(make_uint2(b, len));
        } else {
            for (uint32_t o = 0; o < len; o += kSegMax)
                segs.push_back(make_uint2(b + o, std::min<uint32_t>(kSegMax, len - o)));
            huge.push_back(make_uint2(b, len));
            maxHuge = std::max(maxHuge, len);
        }
    }
    if (small8) k_sort_short<8><<<grid_for((size_t)nrow * 8, 256), 256, 0, s>>>(nrow, 1, rowPtr, keys);
    if (small32) k_sort_short<32><<<grid_for((size_t)nrow * 32, 256), 256, 0, s>>>(nrow, 8, rowPtr, keys);
    FB_CUDA(cudaGetLastError());
    uint2* dseg = nullptr;
    if (!segs.empty()) {
        if ((e = t.get(&dseg, segs.size()))) return e;
        FB_CUDA(cudaMemcpyAsync(dseg, segs.data(), segs.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
        for (size_t o = 0; o < segs.size(); o += 0x7fffffffu) {
            const size_t cnt = std::min<size_t>(segs.size() - o, 0x7fffffffu);
            k_sort_segment<<<(unsigned)cnt, kSegThreads, 0, s>>>(dseg + o, keys);
        }
        FB_CUDA(cudaGetLastError());
    }
    if (!huge.empty()) {
        uint2* dh = nullptr;
        uint64_t* alt = nullptr;
        if ((e = t.get(&dh, huge.size())) || (e = t.get(&alt, nkeys))) return e;
        FB_CUDA(cudaMemcpyAsync(dh, huge.data(), huge.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
        const uint32_t nh = (uint32_t)huge.size();
        const dim3 g((unsigned)std::min<size_t>((maxHuge + 255) / 256, 1024), std::min<uint32_t>(nh, 65535));
        uint64_t *src = keys, *dst = alt;
        for (uint64_t w = kSegMax; w < maxHuge; w *= 2) {
            k_merge_pass<<<g, 256, 0, s>>>(nh, dh, (uint32_t)w, src, dst);
            std::swap(src, dst);
        }
        if (src != keys) k_copy_rows<<<g, 256, 0, s>>>(nh, dh, src, keys);
        FB_CUDA(cudaGetLastError());
    }

    return kOk;
}

} // namespace
} // namespace fb
