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

#include "segsort.cuh"

namespace fb {
namespace {

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

// Sorts the rows of keys (row segments given by the 0-based rowPtr, on the device), inserts
// the missing diagonals and uploads the result into M.
int finish(Ctx& c, Tmp& t, uint32_t nrow, uint32_t mcol, uint32_t nnz, uint32_t* rowPtr,
           uint64_t* keys, const double* values, int* bad, Mat& M)
{
    cudaStream_t s = c.stream;
    int e;
    if ((e = sort_row_keys(c, t, nrow, rowPtr, keys, nnz))) return e;

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
