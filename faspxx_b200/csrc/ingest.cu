// ingest.cu -- a CSRx matrix built on the device from the arrays that FASP++'s file readers
// produce, with the conversions of ReadMat (src/ReadData.cxx:361-446) done as GPU scans and
// sorts instead of host loops:
//
//   MatrixMarket triplets, 0-based (ReadMTX, ReadData.cxx:98-218), then MTXtoMAT
//   (src/MATUtil.cxx:416-436): MTXtoCSR's counting sort by row (:252-300), SortCSRRow
//   (:439-476), CSRtoMAT (:303-413);
//
//   raw CSR arrays (ReadCSR, ReadData.cxx:221-358): the 1-based shift (:350-353), then
//   SortCSRRow and CSRtoMAT as ReadMat's .csr branch does (ReadData.cxx:376-400).
//
// The order both reference paths produce, and this file reproduces: rows ascending; in a
// row, columns ascending, and entries with equal columns (duplicates are kept, not summed)
// in input order, since the counting sort and the insertion sort are both stable. A row
// without a diagonal entry gets an explicit 0.0 at its sorted place.
//
// Every entry is carried as one 64-bit key (column << 32 | input position): keys are unique,
// so any correct sort of a row's keys is the stable order, and the value is gathered through
// the position at the end. Rows are sorted by length class: groups of 8 or 32 lanes with a
// register bitonic network (short rows), one block with a shared-memory bitonic network per
// segment of up to 4096 keys, and merge passes (rank by binary search) above that.
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

// ---- input checks (CheckCSR, MATUtil.cxx:110-174, before any indexed access) ---------------

__global__ void k_check_coo(uint32_t nnz, uint32_t nrow, uint32_t mcol,
                            const uint32_t* __restrict__ rowInd, const uint32_t* __restrict__ colInd,
                            int* __restrict__ bad)
{
    for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz;
         j += (size_t)gridDim.x * blockDim.x)
        if (rowInd[j] >= nrow || colInd[j] >= mcol) *bad = 1;
}

// Row pointers start at 0, or at 1 for 1-based files (ReadCSR shifts those,
// ReadData.cxx:350-353); monotone; rowPtr[nrow] - rowPtr[0] == nnz; shifted columns < mcol.
__global__ void k_check_csr(uint32_t nrow, uint32_t mcol, uint32_t nnz,
                            const uint32_t* __restrict__ rowPtr, const uint32_t* __restrict__ colInd,
                            int* __restrict__ bad)
{
    const uint32_t base = rowPtr[0];
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0 && (base > 1u || rowPtr[nrow] - base != nnz || rowPtr[nrow] < base)) *bad = 1;
    if (base > 1u) return;
    for (size_t i = tid; i < nrow; i += (size_t)gridDim.x * blockDim.x)
        if (rowPtr[i] > rowPtr[i + 1]) *bad = 1;
    for (size_t k = tid; k < nnz; k += (size_t)gridDim.x * blockDim.x)
        if (colInd[k] - base >= mcol) *bad = 1; // a 0 in a 1-based file wraps and fails too
}

// ---- keys in row segments -----------------------------------------------------------------

__global__ void k_count_rows(uint32_t nnz, const uint32_t* __restrict__ rowInd,
                             uint32_t* __restrict__ cnt)
{
    for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz;
         j += (size_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[rowInd[j]], 1u);
}

// MTXtoCSR step 3 (MATUtil.cxx:278-286) with an atomic slot per row: the order inside a row
// is arbitrary here and fixed by the row sort, which orders by (column, position).
__global__ void k_scatter_coo(uint32_t nnz, const uint32_t* __restrict__ rowInd,
                              const uint32_t* __restrict__ colInd, const uint32_t* __restrict__ rowPtr,
                              uint32_t* __restrict__ fill, uint64_t* __restrict__ keys)
{
    for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz;
         j += (size_t)gridDim.x * blockDim.x) {
        const uint32_t r = rowInd[j];
        const uint32_t p = rowPtr[r] + atomicAdd(&fill[r], 1u);
        keys[p] = (uint64_t)colInd[j] << 32 | (uint64_t)j;
    }
}

__global__ void k_keys_csr(uint32_t nrow, uint32_t nnz, const uint32_t* __restrict__ rowPtr,
                           const uint32_t* __restrict__ colInd, uint32_t* __restrict__ rowPtr0,
                           uint64_t* __restrict__ keys)
{
    const uint32_t base = rowPtr[0];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i <= nrow;
         i += (size_t)gridDim.x * blockDim.x)
        rowPtr0[i] = rowPtr[i] - base;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (size_t)gridDim.x * blockDim.x)
        keys[k] = (uint64_t)(colInd[k] - base) << 32 | (uint64_t)k;
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

// ---- CSRtoMAT: explicit zero diagonals (MATUtil.cxx:303-413) ----------------------------------

// Keys of row i with column below i, in a sorted row.
__device__ __forceinline__ uint32_t below_diag(const uint64_t* keys, uint32_t b, uint32_t e, uint32_t i)
{
    return count_below(keys + b, e - b, (uint64_t)i << 32);
}

__global__ void k_diag_missing(uint32_t nrow, uint32_t mcol, const uint32_t* __restrict__ rowPtr,
                               const uint64_t* __restrict__ keys, uint32_t* __restrict__ miss,
                               int* __restrict__ bad)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrow;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t b = rowPtr[i], e = rowPtr[i + 1];
        const uint32_t p = b + below_diag(keys, b, e, (uint32_t)i);
        const bool has = p < e && (uint32_t)(keys[p] >> 32) == (uint32_t)i;
        miss[i] = has ? 0u : 1u;
        if (!has && i >= mcol) *bad = 1; // CheckCSR rejects the inserted column
    }
}

__global__ void k_gather(uint32_t nrow, uint32_t nnz, const uint32_t* __restrict__ rowPtr,
                         const uint32_t* __restrict__ add, const uint32_t* __restrict__ miss,
                         const uint64_t* __restrict__ keys, const double* __restrict__ values,
                         uint32_t* __restrict__ rowPtr2, uint32_t* __restrict__ colInd2,
                         double* __restrict__ val2)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (size_t i = tid; i <= nrow; i += stride) rowPtr2[i] = rowPtr[i] + add[i];
    for (size_t p = tid; p < nnz; p += stride) {
        uint32_t lo = 0, hi = nrow; // the row r with rowPtr[r] <= p < rowPtr[r + 1]
        while (hi - lo > 1) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (rowPtr[mid] <= p)
                lo = mid;
            else
                hi = mid;
        }
        const uint64_t k = keys[p];
        const uint32_t col = (uint32_t)(k >> 32);
        const size_t q = p + add[lo] + (miss[lo] && col > lo ? 1u : 0u);
        colInd2[q] = col;
        val2[q] = values[(uint32_t)k];
    }
    for (size_t i = tid; i < nrow; i += stride)
        if (miss[i]) {
            const uint32_t b = rowPtr[i], e = rowPtr[i + 1];
            const size_t q = (size_t)b + add[i] + below_diag(keys, b, e, (uint32_t)i);
            colInd2[q] = (uint32_t)i;
            val2[q] = 0.0;
        }
}

int read_flag(cudaStream_t s, const int* dflag, int* hflag)
{
    FB_CUDA(cudaMemcpyAsync(hflag, dflag, sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    return kOk;
}

// Sorts the rows of keys (row segments given by the 0-based rowPtr, on the device), inserts
// the missing diagonals and uploads the result into M.
int finish(Ctx& c, Tmp& t, uint32_t nrow, uint32_t mcol, uint32_t nnz, uint32_t* rowPtr,
           uint64_t* keys, const double* values, int* bad, Mat& M)
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
        if ((e = t.get(&dh, huge.size())) || (e = t.get(&alt, nnz))) return e;
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

    // explicit zero diagonals
    uint32_t *miss = nullptr, *add = nullptr, *tiles = nullptr;
    if ((e = t.get(&miss, nrow)) || (e = t.get(&add, (size_t)nrow + 1)) ||
        (e = t.get(&tiles, (nrow + (size_t)kTile - 1) / kTile)))
        return e;
    k_diag_missing<<<grid_for(nrow, 256), 256, 0, s>>>(nrow, mcol, rowPtr, keys, miss, bad);
    FB_CUDA(cudaGetLastError());
    if ((e = scan_counts(s, nrow, miss, add, tiles))) return e;
    int hbad = 0;
    uint32_t added = 0;
    FB_CUDA(cudaMemcpyAsync(&added, add + nrow, 4, cudaMemcpyDeviceToHost, s));
    if ((e = read_flag(s, bad, &hbad))) return e;
    if (hbad) return kErrMatData;
    const uint64_t nnz2 = (uint64_t)nnz + added;
    if (nnz2 > 0xffffffffull) return kErrMatSize;
    uint32_t *rp2 = nullptr, *ci2 = nullptr;
    double* va2 = nullptr;
    if ((e = t.get(&rp2, (size_t)nrow + 1)) || (e = t.get(&ci2, nnz2)) || (e = t.get(&va2, nnz2)))
        return e;
    k_gather<<<grid_for(std::max<size_t>(nnz, nrow), 256), 256, 0, s>>>(nrow, nnz, rowPtr, add, miss,
                                                                       keys, values, rp2, ci2, va2);
    FB_CUDA(cudaGetLastError());
    FB_CUDA(cudaStreamSynchronize(s));
    return m_upload(M, nrow, mcol, (uint32_t)nnz2, rp2, ci2, va2, false, s);
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

} // namespace

int m_from_coo(Ctx& c, uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowInd,
               const uint32_t* colInd, const double* values, bool onDevice, Mat& M)
{
    if (!rowInd || !colInd || !values) return kErrInputPar;
    if (nrow == 0 || mcol == 0 || nnz == 0) return kErrMatSize;
    cudaStream_t s = c.stream;
    Tmp t;
    int e;
    const uint32_t *ri = nullptr, *ci = nullptr;
    const double* va = nullptr;
    if ((e = stage(t, s, rowInd, nnz, onDevice, &ri)) || (e = stage(t, s, colInd, nnz, onDevice, &ci)) ||
        (e = stage(t, s, values, nnz, onDevice, &va)))
        return e;
    int* bad = nullptr;
    uint32_t *cnt = nullptr, *rp = nullptr, *tiles = nullptr;
    uint64_t* keys = nullptr;
    if ((e = t.get(&bad, 1)) || (e = t.get(&cnt, nrow)) || (e = t.get(&rp, (size_t)nrow + 1)) ||
        (e = t.get(&tiles, (nrow + (size_t)kTile - 1) / kTile)) || (e = t.get(&keys, nnz)))
        return e;
    FB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    k_check_coo<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, nrow, mcol, ri, ci, bad);
    FB_CUDA(cudaGetLastError());
    int hbad = 0;
    if ((e = read_flag(s, bad, &hbad))) return e;
    if (hbad) return kErrMatData;
    FB_CUDA(cudaMemsetAsync(cnt, 0, (size_t)nrow * 4, s));
    k_count_rows<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, ri, cnt);
    FB_CUDA(cudaGetLastError());
    if ((e = scan_counts(s, nrow, cnt, rp, tiles))) return e;
    FB_CUDA(cudaMemsetAsync(cnt, 0, (size_t)nrow * 4, s));
    k_scatter_coo<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, ri, ci, rp, cnt, keys);
    FB_CUDA(cudaGetLastError());
    return finish(c, t, nrow, mcol, nnz, rp, keys, va, bad, M);
}

int m_from_csr_raw(Ctx& c, uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                   const uint32_t* colInd, const double* values, bool onDevice, Mat& M)
{
    if (!rowPtr || !colInd || !values) return kErrInputPar;
    if (nrow == 0 || mcol == 0 || nnz == 0) return kErrMatSize;
    cudaStream_t s = c.stream;
    Tmp t;
    int e;
    const uint32_t *rpIn = nullptr, *ci = nullptr;
    const double* va = nullptr;
    if ((e = stage(t, s, rowPtr, (size_t)nrow + 1, onDevice, &rpIn)) ||
        (e = stage(t, s, colInd, nnz, onDevice, &ci)) || (e = stage(t, s, values, nnz, onDevice, &va)))
        return e;
    int* bad = nullptr;
    uint32_t* rp = nullptr;
    uint64_t* keys = nullptr;
    if ((e = t.get(&bad, 1)) || (e = t.get(&rp, (size_t)nrow + 1)) || (e = t.get(&keys, nnz))) return e;
    FB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    k_check_csr<<<grid_for(std::max(nnz, nrow), 256), 256, 0, s>>>(nrow, mcol, nnz, rpIn, ci, bad);
    FB_CUDA(cudaGetLastError());
    int hbad = 0;
    if ((e = read_flag(s, bad, &hbad))) return e;
    if (hbad) return kErrMatData;
    k_keys_csr<<<grid_for(std::max(nnz, nrow + 1u), 256), 256, 0, s>>>(nrow, nnz, rpIn, ci, rp, keys);
    FB_CUDA(cudaGetLastError());
    return finish(c, t, nrow, mcol, nnz, rp, keys, va, bad, M);
}

} // namespace fb
