// spmv.cu -- CSRx matrices in HBM: upload and validation, SpMV (MAT::Apply), residual
// (MAT::Residual), CSR->CSC transpose (MAT::TransInPlace), the lanes-per-row autotuner and
// the sampled outer product of the adjoint gradient.
//
// SpMV mapping: a group of L lanes (L = 1, 2, ..., 32) owns one row; the lanes stride over
// the row's entries so that a warp reads 32/L consecutive rows' values and column indices
// as one contiguous, coalesced stream; x is gathered through L1/L2 (the stencil rows touch
// nearby columns, so x stays cache resident). L = 1 is the scalar thread-per-row kernel and
// L = 32 the warp-per-row vector kernel; L is chosen from the mean row length or timed.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <unordered_map>
#include <vector>

#include "internal.h"

namespace fb {

constexpr int kSlotResidualXinf = kSlots - 1;

// y = A x (RES: r = b - A x, with the x ~ 0 shortcut of MAT::Residual) on stencil masks of
// the fixed 5- or 7-point shape (SH), W consecutive rows per thread (stencil_group).
template <typename T, int SH, bool RES>
__global__ void __launch_bounds__(kBlock) k_stencil_vec(CSRView<T> A, const T* __restrict__ x,
                                                        const T* __restrict__ b,
                                                        T* __restrict__ y,
                                                        const double* __restrict__ xinf)
{
    using VT = Vec16<T>;
    using V = typename VT::V;
    constexpr int W = VT::W;
    const bool shortcut = RES && *xinf < kCloseZero;
    const uint32_t nw = A.nrow / W, stride = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31u;
    const V* xv = reinterpret_cast<const V*>(x);
    const V* bv = reinterpret_cast<const V*>(b);
    V* yv = reinterpret_cast<V*>(y);
    // the loop bound is the same on every lane of a warp (all lanes shuffle)
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g - lane < nw; g += stride) {
        const bool act = g < nw;
        T s[W];
#pragma unroll
        for (int j = 0; j < W; ++j) s[j] = T(0);
        if (!shortcut) {
            V c;
            stencil_group<T, SH>(A, g, nw, act, [&](uint32_t h) { return xv[h]; }, c, s);
        }
        if (act) {
            if (RES) {
                const V bb = bv[g];
#pragma unroll
                for (int j = 0; j < W; ++j) s[j] = VT::at(bb, j) - s[j];
            }
            yv[g] = VT::make(s);
        }
    }
}


template <typename T, int L, bool PAT>
__global__ void __launch_bounds__(kBlock) k_spmv(CSRView<T> A, const T* __restrict__ x,
                                                 T* __restrict__ y)
{
    if (L == 1) { // thread per row, or warp tiles of plain CSR: short rows (stencils)
        for_rows<T, PAT>(A, [&](uint32_t j) { return x[j]; }, [&](size_t r, T s) { y[r] = s; });
        return;
    }
    const int lane = threadIdx.x & (L - 1);
    const size_t warpRows = 32 / L;
    const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
    const size_t sub = (threadIdx.x & 31) / L;
    for (size_t base = gw * warpRows; base < A.nrow; base += nwarps * warpRows) {
        const size_t r = base + sub;
        T s = T(0);
        if (r < A.nrow) {
            const uint32_t b = A.rowPtr[r], e = A.rowPtr[r + 1];
            for (uint32_t k = b + lane; k < e; k += L) {
                const T xv = x[ld_stream(A.colInd + k)];
                s = PAT ? s + xv : fma(ld_stream(A.val + k), xv, s);
            }
        }
        s = group_sum<L>(s);
        if (lane == 0 && r < A.nrow) y[r] = s;
    }
}

// r = b - A x, or r = b when the device flag says NormInf(x) < CLOSE_ZERO (MAT.cxx:459-462).
template <typename T, int L>
__global__ void __launch_bounds__(kBlock) k_residual(CSRView<T> A, const T* __restrict__ b,
                                                     const T* __restrict__ x,
                                                     T* __restrict__ r,
                                                     const double* __restrict__ xinf)
{
    const bool shortcut = *xinf < kCloseZero;
    if (L == 1) {
        if (shortcut) {
            for (size_t row = (size_t)blockIdx.x * blockDim.x + threadIdx.x; row < A.nrow;
                 row += (size_t)gridDim.x * blockDim.x)
                r[row] = b[row] - T(0);
        } else {
            for_rows<T, false>(A, [&](uint32_t j) { return x[j]; },
                               [&](size_t row, T s) { r[row] = b[row] - s; });
        }
        return;
    }
    const int lane = threadIdx.x & (L - 1);
    const size_t warpRows = 32 / L;
    const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
    const size_t sub = (threadIdx.x & 31) / L;
    for (size_t base = gw * warpRows; base < A.nrow; base += nwarps * warpRows) {
        const size_t row = base + sub;
        T s = T(0);
        if (row < A.nrow && !shortcut) {
            const uint32_t bb = A.rowPtr[row], e = A.rowPtr[row + 1];
            for (uint32_t k = bb + lane; k < e; k += L) s = fma(A.val[k], x[A.colInd[k]], s);
        }
        s = group_sum<L>(s);
        if (lane == 0 && row < A.nrow) r[row] = b[row] - s;
    }
}

static int spmv_grid(const Ctx& c, uint32_t nrow, int L)
{
    long long threads = (long long)nrow * L;
    long long g = (threads + kBlock - 1) / kBlock;
    long long cap = (long long)c.nsm * 8; // resident at 2048 threads per SM
    return (int)std::max<long long>(1, std::min(g, cap));
}

// Lanes per row from the mean row length: one thread per row up to 16 entries (measured
// fastest for 5- and 7-point stencils on B200), then about 8 entries per lane.
int lanes_for(double mean)
{
    if (mean <= 16) return 1;
    int L = 2;
    while (L < 32 && L * 8 < mean) L *= 2;
    return L;
}

template <typename T>
static int launch_spmv(Ctx& c, CSRView<T> A, int L, const T* x, T* y)
{
    if (A.nrow == 0) return kOk;
    const int need = spmv_grid(c, A.nrow, L);
    const bool pat = A.val == nullptr && !A.gnz;
    if (L == 1 && !pat) {
        const int sh = stencil_vec_shape(A, x, y, x);
        if (sh) {
            auto gv = [&](auto kern) {
                const int g = std::min(need, resident_grid(c, (const void*)kern, kBlock));
                kern<<<g, kBlock, 0, c.stream>>>(A, x, (const T*)nullptr, y, (const double*)nullptr);
            };
            ++c.launches;
            if (sh == 5)
                gv(k_stencil_vec<T, 5, false>);
            else
                gv(k_stencil_vec<T, 7, false>);
            FB_CUDA(cudaGetLastError());
            return kOk;
        }
    }
    const size_t tiles = L == 1 ? with_tiles(A, kBlock) : 0;
    auto go = [&](auto kern) {
        CSRView<T> V = A;
        size_t smem = tiles;
        if (smem && !tiles_fit((const void*)kern, smem)) V.tiles = 0, smem = 0;
        const int g = std::min(need, resident_grid(c, (const void*)kern, kBlock, smem));
        kern<<<g, kBlock, smem, c.stream>>>(V, x, y);
    };
#define SPMV_CASE(LL)                                                                     \
    case LL:                                                                              \
        if (pat)                                                                          \
            go(k_spmv<T, LL, true>);                                                      \
        else                                                                              \
            go(k_spmv<T, LL, false>);                                                     \
        break;
    ++c.launches;
    switch (L) {
        SPMV_CASE(1)
        SPMV_CASE(2)
        SPMV_CASE(4)
        SPMV_CASE(8)
        SPMV_CASE(16)
        SPMV_CASE(32)
        default: return kErrInputPar;
    }
#undef SPMV_CASE
    FB_CUDA(cudaGetLastError());
    return kOk;
}

int m_spmv(Ctx& c, const Mat& A, const double* x, double* y)
{
    return launch_spmv<double>(c, A.v64(), A.lanes, x, y);
}

int m_spmv32(Ctx& c, const Mat& A, const float* x, float* y)
{
    return launch_spmv<float>(c, A.v32(), A.lanes, x, y);
}

template <typename T>
static int residual_t(Ctx& c, const Mat& A, CSRView<T> V, const T* b, const T* x, T* r,
                      const double* xinf)
{
    if (A.nrow == 0) return kOk;
    if (!V.val && !V.gnz) return kErrMatData; // MAT::Residual reads values (MAT.cxx:466)
    if (!xinf) {
        double* slot = c.dslot + kSlotResidualXinf;
        int e = v_norminf(c, A.mcol, x, slot);
        if (e) return e;
        xinf = slot;
    }
    const int need = spmv_grid(c, A.nrow, A.lanes);
    if (A.lanes == 1) {
        const int sh = stencil_vec_shape(V, x, b, r);
        if (sh) {
            auto gv = [&](auto kern) {
                const int g = std::min(need, resident_grid(c, (const void*)kern, kBlock));
                kern<<<g, kBlock, 0, c.stream>>>(V, x, b, r, xinf);
            };
            ++c.launches;
            if (sh == 5)
                gv(k_stencil_vec<T, 5, true>);
            else
                gv(k_stencil_vec<T, 7, true>);
            FB_CUDA(cudaGetLastError());
            return kOk;
        }
    }
    const size_t tiles = A.lanes == 1 ? with_tiles(V, kBlock) : 0;
    auto go = [&](auto kern) {
        CSRView<T> W = V;
        size_t smem = tiles;
        if (smem && !tiles_fit((const void*)kern, smem)) W.tiles = 0, smem = 0;
        const int g = std::min(need, resident_grid(c, (const void*)kern, kBlock, smem));
        kern<<<g, kBlock, smem, c.stream>>>(W, b, x, r, xinf);
    };
    ++c.launches;
    switch (A.lanes) {
        case 1: go(k_residual<T, 1>); break;
        case 2: go(k_residual<T, 2>); break;
        case 4: go(k_residual<T, 4>); break;
        case 8: go(k_residual<T, 8>); break;
        case 16: go(k_residual<T, 16>); break;
        default: go(k_residual<T, 32>); break;
    }
    FB_CUDA(cudaGetLastError());
    return kOk;
}

int m_residual(Ctx& c, const Mat& A, const double* b, const double* x, double* r,
               const double* xinf)
{
    return residual_t<double>(c, A, A.v64(), b, x, r, xinf);
}

int m_residual(Ctx& c, const Mat& A, const float* b, const float* x, float* r,
               const double* xinf)
{
    if (!A.val && !A.grid) return kErrMatData;
    return residual_t<float>(c, A, A.v32(), b, x, r, xinf);
}

// ---- setup-time kernels ----------------------------------------------------------------

// MAT::FormDiagPtr (MAT.cxx:917-928): first position whose column equals the row; rows
// without a diagonal keep 0. GetDiag (MAT.cxx:256-267) reads values there (1 if pattern).
__global__ void k_diag(uint32_t nrow, const uint32_t* __restrict__ rowPtr,
                       const uint32_t* __restrict__ colInd, const double* __restrict__ val,
                       uint32_t* __restrict__ diagPtr, double* __restrict__ diag)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrow;
         i += (size_t)gridDim.x * blockDim.x) {
        uint32_t d = 0;
        for (uint32_t k = rowPtr[i]; k < rowPtr[i + 1]; ++k)
            if (colInd[k] == i) {
                d = k;
                break;
            }
        diagPtr[i] = d;
        if (diag) diag[i] = val ? val[d] : 1.0;
    }
}

__global__ void k_to_f32(size_t n, const double* __restrict__ a, float* __restrict__ b)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

static int dmalloc(void** p, size_t bytes)
{
    // 32 spare bytes keep vectorised/bulk tail accesses inside the allocation (the warp
    // tiles' 16-byte loads read up to 3 entries past the last one)
    cudaError_t e = cudaMalloc(p, bytes + 32);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return kErrAlloc;
    }
    return kOk;
}

void m_free(Mat& M)
{
    cudaFree(M.rowPtr);
    cudaFree(M.colInd);
    cudaFree(M.diagPtr);
    cudaFree(M.val);
    cudaFree(M.val32);
    cudaFree(M.diag);
    cudaFree(M.rcCls);
    cudaFree(M.rcOff);
    cudaFree(M.rcDelta);
    cudaFree(M.rcVal);
    cudaFree(M.rcVal32);
    cudaFree(M.skMask);
    cudaFree(M.cd16);
    M = Mat();
}

// ---- 16-bit column offsets ------------------------------------------------------------------
// cd16[k] = colInd[k] - row(k) when every entry is within 32,767 columns of its row (banded
// FDM/FEM matrices up to bandwidths of 32,767, the 128^3 Laplacian's is 16,384): the
// thread-per-row kernels then read 2 bytes per entry instead of 4 and form the column by one
// add, with the entries and their order unchanged -- the same results bit for bit.
__global__ void k_col16(uint32_t nrow, const uint32_t* __restrict__ rowPtr,
                        const uint32_t* __restrict__ colInd, int16_t* __restrict__ out,
                        unsigned* __restrict__ outOfRange)
{
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrow;
         r += (size_t)gridDim.x * blockDim.x) {
        bool bad = false;
        for (uint32_t k = rowPtr[r]; k < rowPtr[r + 1]; ++k) {
            const long long d = (long long)colInd[k] - (long long)r;
            if (d < -32767 || d > 32767)
                bad = true;
            else
                out[k] = (int16_t)d;
        }
        if (bad) atomicOr(outOfRange, 1u);
    }
}

int m_build_col16(Mat& M, cudaStream_t s)
{
    if (M.grid || M.nnz == 0 || !M.colInd || M.cd16) return kOk;
    int16_t* out = nullptr;
    unsigned* flag = nullptr;
    int e;
    if ((e = dmalloc((void**)&out, ((size_t)M.nnz + 8) * 2)) ||
        (e = dmalloc((void**)&flag, 4))) {
        cudaFree(out);
        return e;
    }
    FB_CUDA(cudaMemsetAsync(flag, 0, 4, s));
    k_col16<<<std::max(1, std::min(ceil_div(M.nrow, kBlock), 148 * 8)), kBlock, 0, s>>>(
        M.nrow, M.rowPtr, M.colInd, out, flag);
    FB_CUDA(cudaGetLastError());
    unsigned h = 0;
    FB_CUDA(cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    cudaFree(flag);
    if (h) {
        cudaFree(out); // some entry is too far from its row: keep 32-bit columns only
        return kOk;
    }
    M.cd16 = out;
    return kOk;
}

// The most entries any 256-row tile covers once widened to multiples of 4: the block tiles
// of csr_tile_rows take a matrix only when every tile fits a stage.
__global__ void k_tile_span(uint32_t nrow, const uint32_t* __restrict__ rowPtr,
                            unsigned* __restrict__ span)
{
    const size_t ntiles = ((size_t)nrow + kTileRows - 1) / kTileRows;
    unsigned m = 0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntiles;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t r0 = t * kTileRows;
        const size_t r1 = r0 + kTileRows < nrow ? r0 + kTileRows : nrow;
        const unsigned long long a = rowPtr[r0] & ~3u;
        const unsigned long long ar = ((unsigned long long)rowPtr[r1] + 3) & ~3ull;
        const unsigned long long w = ar - a;
        m = max(m, (unsigned)(w < 0xffffffffull ? w : 0xffffffffull));
    }
    atomicMax(span, m);
}

int m_tile_span(Mat& M, cudaStream_t s)
{
    M.tileSpan = 0;
    if (M.grid || M.nrow == 0 || !M.rowPtr) return kOk;
    unsigned* d = nullptr;
    int e;
    if ((e = dmalloc((void**)&d, 4))) return e;
    FB_CUDA(cudaMemsetAsync(d, 0, 4, s));
    const int tiles = ceil_div(M.nrow, (int)kTileRows);
    k_tile_span<<<std::max(1, std::min(ceil_div(tiles, kBlock), 148 * 8)), kBlock, 0, s>>>(
        M.nrow, M.rowPtr, d);
    FB_CUDA(cudaGetLastError());
    unsigned h = 0;
    FB_CUDA(cudaMemcpyAsync(&h, d, 4, cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    cudaFree(d);
    M.tileSpan = h;
    return kOk;
}

unsigned tile_timeouts_spmv() { return tile_timeouts(); }

// ---- row classes ------------------------------------------------------------------------
// A row's class is its length, its column offsets col - row and its values (bit patterns),
// in CSR order. Constant-coefficient stencil matrices have a handful of classes (interior,
// faces, edges, corners), so the SpMV streams a 2-byte class id per row instead of 8 to 12
// bytes per entry. The table is built only when it stays small against the matrix.

constexpr uint32_t kRcMaxClasses = 4096;
constexpr uint32_t kRcMaxRowLen = 64;

struct RowClasses {
    std::vector<uint16_t> cls;
    std::vector<uint32_t> off{0};
    std::vector<int32_t>  delta;
    std::vector<double>   val;
};

static bool build_row_classes(uint32_t nrow, const uint32_t* rp, const uint32_t* ci,
                              const double* v, RowClasses& R)
{
    if (nrow == 0 || nrow > 0x7fffffffu) return false;
    const size_t nnz = rp[nrow];
    const size_t maxEntries = std::max<size_t>(64, nnz / 8);
    R.cls.resize(nrow);
    std::unordered_map<uint64_t, std::vector<uint32_t>> buckets;
    for (uint32_t row = 0; row < nrow; ++row) {
        const uint32_t b = rp[row], e = rp[row + 1], len = e - b;
        if (len > kRcMaxRowLen) return false;
        uint64_t h = 1469598103934665603ull ^ len;
        for (uint32_t k = b; k < e; ++k) {
            const uint64_t d = (uint64_t)(uint32_t)(int32_t)((int64_t)ci[k] - (int64_t)row);
            uint64_t bits;
            std::memcpy(&bits, &v[k], 8);
            h = (h ^ d) * 1099511628211ull;
            h = (h ^ bits) * 1099511628211ull;
        }
        auto& cand = buckets[h];
        uint32_t id = 0xffffffffu;
        for (uint32_t c : cand) {
            const uint32_t cb = R.off[c], ce = R.off[c + 1];
            if (ce - cb != len) continue;
            bool same = true;
            for (uint32_t k = 0; k < len && same; ++k)
                same = R.delta[cb + k] == (int32_t)((int64_t)ci[b + k] - (int64_t)row) &&
                       std::memcmp(&R.val[cb + k], &v[b + k], 8) == 0;
            if (same) {
                id = c;
                break;
            }
        }
        if (id == 0xffffffffu) {
            id = (uint32_t)R.off.size() - 1;
            if (id >= kRcMaxClasses || R.delta.size() + len > maxEntries) return false;
            for (uint32_t k = b; k < e; ++k) {
                const int64_t d = (int64_t)ci[k] - (int64_t)row;
                if (d < INT32_MIN || d > INT32_MAX) return false;
                R.delta.push_back((int32_t)d);
                R.val.push_back(v[k]);
            }
            R.off.push_back((uint32_t)R.delta.size());
            cand.push_back(id);
        }
        R.cls[row] = (uint16_t)id;
    }
    return true;
}

// Stencil masks: when the classes' column offsets, taken together, are at most kMaxStencil
// distinct values each carrying one value (bitwise) wherever it occurs, and every class
// lists its offsets in ascending order (the CSR order), each row is a bit mask over that
// sorted offset list. Summing the present entries in list order is the CSR order.
static bool build_stencil_masks(const RowClasses& R, Mat& T, std::vector<uint16_t>& rowMask)
{
    std::map<int32_t, double> U;
    const uint32_t C = (uint32_t)R.off.size() - 1;
    for (uint32_t c = 0; c < C; ++c)
        for (uint32_t k = R.off[c]; k < R.off[c + 1]; ++k) {
            if (k > R.off[c] && R.delta[k] <= R.delta[k - 1]) return false;
            auto it = U.find(R.delta[k]);
            if (it == U.end())
                U.emplace(R.delta[k], R.val[k]);
            else if (std::memcmp(&it->second, &R.val[k], 8) != 0)
                return false;
        }
    if (U.empty() || U.size() > (size_t)kMaxStencil) return false;
    std::map<int32_t, int> pos;
    T.skLen = 0;
    for (auto& kv : U) {
        pos[kv.first] = (int)T.skLen;
        T.skDelta[T.skLen] = kv.first;
        T.skVal[T.skLen] = kv.second;
        ++T.skLen;
    }
    std::vector<uint16_t> cm(C, 0);
    for (uint32_t c = 0; c < C; ++c)
        for (uint32_t k = R.off[c]; k < R.off[c + 1]; ++k) cm[c] |= (uint16_t)(1u << pos[R.delta[k]]);
    rowMask.resize(R.cls.size());
    for (size_t r = 0; r < R.cls.size(); ++r) rowMask[r] = cm[R.cls[r]];
    return true;
}

static int upload_row_classes(Mat& T, const RowClasses& R, cudaStream_t s)
{
    const uint32_t C = (uint32_t)R.off.size() - 1, E = (uint32_t)R.delta.size();
    int e;
    if ((e = dmalloc((void**)&T.rcCls, (size_t)T.nrow * 2 + 16)) ||
        (e = dmalloc((void**)&T.rcOff, ((size_t)C + 1) * 4)) ||
        (e = dmalloc((void**)&T.rcDelta, (size_t)E * 4 + 16)) ||
        (e = dmalloc((void**)&T.rcVal, (size_t)E * 8 + 16)))
        return e;
    FB_CUDA(cudaMemcpyAsync(T.rcCls, R.cls.data(), (size_t)T.nrow * 2, cudaMemcpyHostToDevice, s));
    FB_CUDA(cudaMemcpyAsync(T.rcOff, R.off.data(), ((size_t)C + 1) * 4, cudaMemcpyHostToDevice, s));
    FB_CUDA(cudaMemcpyAsync(T.rcDelta, R.delta.data(), (size_t)E * 4, cudaMemcpyHostToDevice, s));
    FB_CUDA(cudaMemcpyAsync(T.rcVal, R.val.data(), (size_t)E * 8, cudaMemcpyHostToDevice, s));
    std::vector<uint16_t> rowMask;
    if (build_stencil_masks(R, T, rowMask)) {
        if ((e = dmalloc((void**)&T.skMask, (size_t)T.nrow * 2 + 16))) return e;
        FB_CUDA(cudaMemcpyAsync(T.skMask, rowMask.data(), (size_t)T.nrow * 2,
                                cudaMemcpyHostToDevice, s));
    } else {
        T.skLen = 0;
    }
    FB_CUDA(cudaStreamSynchronize(s)); // the host vectors die with the caller
    T.rcClasses = C;
    T.rcEntries = E;
    T.rcOn = true;
    return kOk;
}

// CheckCSR (src/MATUtil.cxx:110-174) on host arrays: sizes, monotone row pointers, column
// indices in range. A failed check returns ERROR_MAT_DATA and uploads nothing, so no kernel
// ever indexes outside the matrix.
static int check_csr(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                     const uint32_t* colInd)
{
    if (nrow == 0 || mcol == 0 || nnz == 0) return kErrMatSize;
    if (rowPtr[0] != 0 || rowPtr[nrow] != nnz) return kErrMatData;
    for (uint32_t j = 0; j < nrow; ++j)
        if (rowPtr[j] > rowPtr[j + 1]) return kErrMatData;
    for (uint32_t k = 0; k < nnz; ++k)
        if (colInd[k] >= mcol) return kErrMatData;
    return kOk;
}

int m_upload(Mat& M, uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
             const uint32_t* colInd, const double* values, bool hostPtrs, cudaStream_t s)
{
    std::vector<uint32_t> hrp, hci;
    const uint32_t* crp = rowPtr;
    const uint32_t* cci = colInd;
    if (!hostPtrs) {
        // device arrays: validate a host copy before any kernel touches them
        hrp.resize((size_t)nrow + 1);
        hci.resize(nnz);
        FB_CUDA(cudaMemcpy(hrp.data(), rowPtr, hrp.size() * 4, cudaMemcpyDeviceToHost));
        FB_CUDA(cudaMemcpy(hci.data(), colInd, hci.size() * 4, cudaMemcpyDeviceToHost));
        crp = hrp.data();
        cci = hci.data();
    }
    int e = check_csr(nrow, mcol, nnz, crp, cci);
    if (e) return e;
    uint32_t maxLen = 0;
    for (uint32_t j = 0; j < nrow; ++j) maxLen = std::max(maxLen, crp[j + 1] - crp[j]);

    Mat T;
    T.nrow = nrow;
    T.mcol = mcol;
    T.nnz = nnz;
    T.maxRowLen = maxLen;
    T.meanRowLen = (double)nnz / nrow;
    cudaGetDevice(&T.dev);
    const cudaMemcpyKind kind = hostPtrs ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if ((e = dmalloc((void**)&T.rowPtr, ((size_t)nrow + 1) * 4)) ||
        (e = dmalloc((void**)&T.colInd, (size_t)nnz * 4)) ||
        (e = dmalloc((void**)&T.diagPtr, (size_t)nrow * 4)) ||
        (e = dmalloc((void**)&T.diag, (size_t)nrow * 8)) ||
        (values && (e = dmalloc((void**)&T.val, (size_t)nnz * 8)))) {
        m_free(T);
        return e;
    }
    FB_CUDA(cudaMemcpyAsync(T.rowPtr, rowPtr, ((size_t)nrow + 1) * 4, kind, s));
    FB_CUDA(cudaMemcpyAsync(T.colInd, colInd, (size_t)nnz * 4, kind, s));
    if (values) FB_CUDA(cudaMemcpyAsync(T.val, values, (size_t)nnz * 8, kind, s));
    k_diag<<<std::max(1, std::min(ceil_div(nrow, kBlock), 148 * 8)), kBlock, 0, s>>>(
        nrow, T.rowPtr, T.colInd, T.val, T.diagPtr, T.diag);
    FB_CUDA(cudaGetLastError());
    T.lanes = lanes_for(T.meanRowLen);
    std::vector<double> hv;
    const double* cv = values;
    if (values && !hostPtrs) {
        hv.resize(nnz);
        FB_CUDA(cudaMemcpy(hv.data(), values, (size_t)nnz * 8, cudaMemcpyDeviceToHost));
        cv = hv.data();
    }
    if (values && nrow == mcol && nrow > 0) { // one diagonal value (bitwise) in every row?
        bool same = true, first = true;
        double d0 = 0.0;
        for (uint32_t r = 0; r < nrow && same; ++r) {
            bool found = false;
            for (uint32_t k = crp[r]; k < crp[r + 1]; ++k)
                if (cci[k] == r) {
                    found = true;
                    if (first) {
                        d0 = cv[k];
                        first = false;
                    } else if (std::memcmp(&cv[k], &d0, 8) != 0) {
                        same = false;
                    }
                    break;
                }
            same = same && found;
        }
        T.diagConst = same && d0 != 0.0;
        T.diagValue = d0;
    }
    if (values && T.lanes == 1) {
        RowClasses R;
        if (build_row_classes(nrow, crp, cci, cv, R) && (e = upload_row_classes(T, R, s))) {
            m_free(T);
            return e;
        }
    }
    if ((e = m_build_col16(T, s)) || (e = m_tile_span(T, s))) {
        m_free(T);
        return e;
    }
    FB_CUDA(cudaStreamSynchronize(s));
    M = T;
    return kOk;
}

int Mat::ensure32(cudaStream_t s)
{
    if (!val) return kOk;
    int e;
    if (!val32) {
        if ((e = dmalloc((void**)&val32, (size_t)nnz * 4))) return e;
        k_to_f32<<<std::max(1, std::min(ceil_div(nnz, kBlock), 148 * 8)), kBlock, 0, s>>>(
            nnz, val, val32);
        FB_CUDA(cudaGetLastError());
    }
    if (rcVal && !rcVal32) {
        if ((e = dmalloc((void**)&rcVal32, (size_t)rcEntries * 4 + 16))) return e;
        k_to_f32<<<std::max(1, std::min(ceil_div(rcEntries, kBlock), 148 * 8)), kBlock, 0, s>>>(
            rcEntries, rcVal, rcVal32);
        FB_CUDA(cudaGetLastError());
    }
    return kOk;
}

// ---- transpose: CSR -> CSC in exactly MAT::TransInPlace's order (MAT.cxx:479-538) -------
// Column counts by atomics, an exclusive scan, a scatter that records each entry's original
// position, then each output row (input column) sorted by original position: since CSR
// positions increase with the row index, that is the ascending-row order the reference's
// row-by-row scatter produces.

__global__ void k_col_count(uint32_t nnz, const uint32_t* __restrict__ colInd,
                            uint32_t* __restrict__ cnt)
{
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (size_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[colInd[k]], 1u);
}

// single-block exclusive scan of cnt[0..m) into out[0..m]
__global__ void k_scan(uint32_t m, const uint32_t* __restrict__ cnt, uint32_t* __restrict__ out)
{
    __shared__ uint32_t warpTot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t base = 0; base < m; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t v = i < m ? cnt[i] : 0, incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warpTot[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            uint32_t w = lane < (int)(blockDim.x >> 5) ? warpTot[lane] : 0, wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            warpTot[lane] = wi - w; // exclusive warp offsets
        }
        __syncthreads();
        if (i < m) out[i] = carry + warpTot[wid] + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += warpTot[wid] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[m] = carry;
}

__global__ void k_row_of(uint32_t nrow, const uint32_t* __restrict__ rowPtr,
                         uint32_t* __restrict__ rowOf)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrow;
         i += (size_t)gridDim.x * blockDim.x)
        for (uint32_t k = rowPtr[i]; k < rowPtr[i + 1]; ++k) rowOf[k] = (uint32_t)i;
}

__global__ void k_scatter_pos(uint32_t nnz, const uint32_t* __restrict__ colInd,
                              const uint32_t* __restrict__ tRowPtr, uint32_t* __restrict__ fill,
                              uint32_t* __restrict__ pos)
{
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (size_t)gridDim.x * blockDim.x) {
        const uint32_t c = colInd[k];
        const uint32_t slot = tRowPtr[c] + atomicAdd(&fill[c], 1u);
        pos[slot] = (uint32_t)k;
    }
}

// sort each segment of pos by value (insertion sort per thread), then gather rows/values
__global__ void k_sort_gather(uint32_t m, const uint32_t* __restrict__ tRowPtr,
                              uint32_t* __restrict__ pos, const uint32_t* __restrict__ rowOf,
                              const double* __restrict__ val, uint32_t* __restrict__ tColInd,
                              double* __restrict__ tVal)
{
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < m;
         c += (size_t)gridDim.x * blockDim.x) {
        const uint32_t b = tRowPtr[c], e = tRowPtr[c + 1];
        for (uint32_t i = b + 1; i < e; ++i) {
            const uint32_t key = pos[i];
            uint32_t j = i;
            while (j > b && pos[j - 1] > key) {
                pos[j] = pos[j - 1];
                --j;
            }
            pos[j] = key;
        }
        for (uint32_t i = b; i < e; ++i) {
            const uint32_t p = pos[i];
            tColInd[i] = rowOf[p];
            if (val) tVal[i] = val[p];
        }
    }
}

// The transpose of a grid operator is the grid operator with every offset negated (the
// same coefficients), in ascending order of the negated flattened offsets.
static int grid_transpose(Ctx& c, const Mat& A, Mat& T)
{
    std::vector<int32_t> dx(A.skLen), dy(A.skLen), dz(A.skLen);
    for (uint32_t k = 0; k < A.skLen; ++k) {
        dx[k] = -A.gd[0][k];
        dy[k] = -A.gd[1][k];
        dz[k] = -A.gd[2][k];
    }
    return m_create_stencil(T, A.gdim[0], A.gdim[1], A.gdim[2], A.skLen, dx.data(), dy.data(),
                            dz.data(), A.skVal, c.stream);
}

int m_transpose(Ctx& c, const Mat& A, Mat& T)
{
    if (A.grid) return grid_transpose(c, A, T);
    const uint32_t m = A.mcol, n = A.nrow, nnz = A.nnz;
    Mat R;
    R.nrow = m;
    R.mcol = n;
    R.nnz = nnz;
    R.dev = A.dev;
    uint32_t *cnt = nullptr, *fill = nullptr, *pos = nullptr, *rowOf = nullptr;
    int e;
    if ((e = dmalloc((void**)&R.rowPtr, ((size_t)m + 1) * 4)) ||
        (e = dmalloc((void**)&R.colInd, (size_t)nnz * 4)) ||
        (e = dmalloc((void**)&R.diagPtr, (size_t)m * 4)) ||
        (e = dmalloc((void**)&R.diag, (size_t)m * 8)) ||
        (A.val && (e = dmalloc((void**)&R.val, (size_t)nnz * 8))) ||
        (e = dmalloc((void**)&cnt, (size_t)m * 4)) || (e = dmalloc((void**)&fill, (size_t)m * 4)) ||
        (e = dmalloc((void**)&pos, (size_t)nnz * 4)) ||
        (e = dmalloc((void**)&rowOf, (size_t)nnz * 4))) {
        m_free(R);
        cudaFree(cnt);
        cudaFree(fill);
        cudaFree(pos);
        cudaFree(rowOf);
        return e;
    }
    cudaStream_t s = c.stream;
    const int gn = std::max(1, std::min(ceil_div(nnz, kBlock), c.nsm * 8));
    const int gm = std::max(1, std::min(ceil_div(m, kBlock), c.nsm * 8));
    const int gr = std::max(1, std::min(ceil_div(n, kBlock), c.nsm * 8));
    FB_CUDA(cudaMemsetAsync(cnt, 0, (size_t)m * 4, s));
    FB_CUDA(cudaMemsetAsync(fill, 0, (size_t)m * 4, s));
    k_col_count<<<gn, kBlock, 0, s>>>(nnz, A.colInd, cnt);
    k_scan<<<1, 1024, 0, s>>>(m, cnt, R.rowPtr);
    k_row_of<<<gr, kBlock, 0, s>>>(n, A.rowPtr, rowOf);
    k_scatter_pos<<<gn, kBlock, 0, s>>>(nnz, A.colInd, R.rowPtr, fill, pos);
    k_sort_gather<<<gm, kBlock, 0, s>>>(m, R.rowPtr, pos, rowOf, A.val, R.colInd, R.val);
    k_diag<<<gm, kBlock, 0, s>>>(m, R.rowPtr, R.colInd, R.val, R.diagPtr, R.diag);
    FB_CUDA(cudaGetLastError());
    FB_CUDA(cudaStreamSynchronize(s));
    cudaFree(cnt);
    cudaFree(fill);
    cudaFree(pos);
    cudaFree(rowOf);
    R.meanRowLen = (double)nnz / m;
    std::vector<uint32_t> hrp((size_t)m + 1);
    FB_CUDA(cudaMemcpy(hrp.data(), R.rowPtr, hrp.size() * 4, cudaMemcpyDeviceToHost));
    for (uint32_t j = 0; j < m; ++j) R.maxRowLen = std::max(R.maxRowLen, hrp[j + 1] - hrp[j]);
    R.lanes = A.lanes;
    if ((e = m_build_col16(R, s)) || (e = m_tile_span(R, s))) {
        m_free(R);
        return e;
    }
    T = R;
    return kOk;
}

// ---- autotuner: time each lanes-per-row choice on this matrix ---------------------------
int m_autotune(Ctx& c, Mat& A)
{
    if (A.grid) return kOk; // grid operators run thread per row (lanes = 1) only
    double *x = nullptr, *y = nullptr;
    int e;
    if ((e = dmalloc((void**)&x, (size_t)A.mcol * 8)) || (e = dmalloc((void**)&y, (size_t)A.nrow * 8))) {
        cudaFree(x);
        return e;
    }
    FB_CUDA(cudaMemsetAsync(x, 0, (size_t)A.mcol * 8, c.stream));
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best = 1e30f;
    int bestL = A.lanes;
    const int orig = A.lanes;
    for (int L = 1; L <= 32; L *= 2) {
        if (L > 2 * (int)A.maxRowLen && L > 1) break;
        A.lanes = L;
        for (int w = 0; w < 2; ++w) m_spmv(c, A, x, y);
        cudaEventRecord(t0, c.stream);
        for (int r = 0; r < 5; ++r) m_spmv(c, A, x, y);
        cudaEventRecord(t1, c.stream);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        if (ms < best) {
            best = ms;
            bestL = L;
        }
    }
    A.lanes = cudaGetLastError() == cudaSuccess ? bestL : orig;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(x);
    cudaFree(y);
    return kOk;
}

// ---- sampled outer product: dA_k = scale * lam[row(k)] * x[col(k)] ----------------------
__global__ void k_sampled_outer(CSRView<double> A, const double* __restrict__ lam,
                                const double* __restrict__ x, double scale,
                                double* __restrict__ dA)
{
    // one warp per 32 rows' worth of entries: lanes stride the contiguous entry range
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.nrow;
         i += (size_t)gridDim.x * blockDim.x) {
        const double li = scale * lam[i];
        for (uint32_t k = A.rowPtr[i]; k < A.rowPtr[i + 1]; ++k) dA[k] = li * x[A.colInd[k]];
    }
}

int m_sampled_outer(Ctx& c, const Mat& A, const double* lam, const double* x, double scale,
                    double* dA)
{
    if (A.grid) return kErrInputPar; // no stored entries to differentiate
    const int g = std::max(1, std::min(ceil_div(A.nrow, kBlock), c.nsm * 8));
    k_sampled_outer<<<g, kBlock, 0, c.stream>>>(A.v64(), lam, x, scale, dA);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

// ---- MAT::MultTransposeAdd: v = A^T v1 + v2 (MAT.cxx:541-606) ---------------------------
// T is A's exact transpose (m_transpose, the order of MAT::TransInPlace). As the reference,
// each v[i] starts from v2[i] and adds the products of row i of T left to right, each
// product rounded before the add (no fused multiply-add), so the results are the
// reference's bit for bit wherever its loop bounds are right (structurally symmetric A).
// Pattern-only matrices count every stored entry as 1, as MAT::Apply does; a grid operator
// walks its stencil points in ascending offset, which is its CSR order.
template <bool GRID, bool PAT>
__global__ void k_mult_transpose_add(CSRView<double> T, const double* __restrict__ v1,
                                     const double* __restrict__ v2, double* __restrict__ v)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < T.nrow;
         i += (size_t)gridDim.x * blockDim.x) {
        double acc = v2[i];
        if (GRID) {
            const uint32_t m = grid_mask(T, (uint32_t)i);
            for (uint32_t k = 0; k < T.ulen; ++k)
                if ((m >> k) & 1u)
                    acc = __dadd_rn(acc, __dmul_rn(v1[(long long)i + T.udelta[k]], T.uval[k]));
        } else {
            const uint32_t b = T.rowPtr[i], e = T.rowPtr[i + 1];
            for (uint32_t k = b; k < e; ++k)
                acc = __dadd_rn(acc, PAT ? v1[T.colInd[k]]
                                         : __dmul_rn(v1[T.colInd[k]], T.val[k]));
        }
        v[i] = acc;
    }
}

int m_mult_transpose_add(Ctx& c, const Mat& T, const double* v1, const double* v2, double* v)
{
    if (T.nrow == 0) return kOk;
    const int g = std::max(1, std::min(ceil_div(T.nrow, kBlock), c.nsm * 8));
    CSRView<double> V = T.view<double>(T.val, nullptr);
    if (T.grid)
        k_mult_transpose_add<true, false><<<g, kBlock, 0, c.stream>>>(V, v1, v2, v);
    else if (!T.val)
        k_mult_transpose_add<false, true><<<g, kBlock, 0, c.stream>>>(V, v1, v2, v);
    else
        k_mult_transpose_add<false, false><<<g, kBlock, 0, c.stream>>>(V, v1, v2, v);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

// ---- structured-grid (matrix-free) operators --------------------------------------------
// The GPU counterpart of the reference's matrix-free LOP example (example/TestMatFree.cxx:
// 26-176): y = A x on an nx x ny x nz grid with a constant-coefficient stencil, Dirichlet
// truncation at the faces, without any stored matrix. Rows are grid points in x-fastest
// order; a row's entries are the stencil points inside the grid in ascending column order,
// so every kernel computes exactly what it computes on the assembled CSR matrix.

__global__ void k_fill_const(uint32_t n, double v, double* __restrict__ y)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        y[i] = v;
}

int m_create_stencil(Mat& M, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t npts,
                     const int32_t* dx, const int32_t* dy, const int32_t* dz, const double* coef,
                     cudaStream_t s)
{
    if (!dx || !dy || !dz || !coef) return kErrInputPar;
    if (nx == 0 || ny == 0 || nz == 0) return kErrMatSize;
    const uint64_t n64 = (uint64_t)nx * ny * nz;
    if (n64 > 0xffffffffull || (uint64_t)nx * ny > 0xffffffffull) return kErrMatSize;
    if (npts == 0 || npts > (uint32_t)kMaxStencil) return kErrInputPar;
    struct Pt {
        int64_t flat;
        int32_t d[3];
        double  v;
    };
    std::vector<Pt> pts(npts);
    for (uint32_t k = 0; k < npts; ++k) {
        const int32_t d[3] = {dx[k], dy[k], dz[k]};
        for (int a = 0; a < 3; ++a)
            if (d[a] < -3 || d[a] > 3) return kErrInputPar; // reach of at most 3 points
        pts[k] = Pt{(int64_t)d[0] + (int64_t)nx * ((int64_t)d[1] + (int64_t)ny * d[2]),
                    {d[0], d[1], d[2]}, coef[k]};
    }
    // points that reach past the grid in some dimension are never inside it: dropped (in a
    // grid one point thick, such points could share a flattened offset with real ones)
    const uint32_t ext[3] = {nx, ny, nz};
    pts.erase(std::remove_if(pts.begin(), pts.end(),
                             [&](const Pt& p) {
                                 for (int a = 0; a < 3; ++a)
                                     if ((uint32_t)std::abs(p.d[a]) >= ext[a]) return true;
                                 return false;
                             }),
              pts.end());
    npts = (uint32_t)pts.size();
    // a present neighbour (ix + dx, iy + dy, iz + dz) is column row + flat, so ascending
    // flattened offset is the CSR column order of every row
    std::sort(pts.begin(), pts.end(), [](const Pt& a, const Pt& b) { return a.flat < b.flat; });
    for (uint32_t k = 1; k < npts; ++k)
        if (pts[k].flat == pts[k - 1].flat) return kErrInputPar;
    Mat T;
    T.grid = true;
    T.nrow = T.mcol = (uint32_t)n64;
    T.gdim[0] = nx;
    T.gdim[1] = ny;
    T.gdim[2] = nz;
    T.skLen = npts;
    uint64_t nnz = 0;
    double diagv = 0.0;
    bool hasDiag = false;
    for (uint32_t k = 0; k < npts; ++k) {
        T.skDelta[k] = (int32_t)pts[k].flat;
        T.skVal[k] = pts[k].v;
        uint64_t cnt = 1;
        for (int a = 0; a < 3; ++a) {
            T.gd[a][k] = (int8_t)pts[k].d[a];
            const uint32_t r = (uint32_t)std::abs(pts[k].d[a]);
            cnt *= r < ext[a] ? ext[a] - r : 0;
        }
        nnz += cnt;
        if (pts[k].flat == 0) {
            hasDiag = true;
            diagv = pts[k].v;
        }
    }
    if (nnz > 0xffffffffull) return kErrMatSize;
    T.nnz = (uint32_t)nnz;
    T.lanes = 1;
    T.maxRowLen = npts;
    T.meanRowLen = (double)nnz / (double)n64;
    T.diagConst = hasDiag && diagv != 0.0;
    T.diagValue = diagv;
    cudaGetDevice(&T.dev);
    int e;
    if ((e = dmalloc((void**)&T.diag, (size_t)T.nrow * 8))) return e;
    k_fill_const<<<std::max(1, std::min(ceil_div(T.nrow, kBlock), 148 * 8)), kBlock, 0, s>>>(
        T.nrow, diagv, T.diag);
    FB_CUDA(cudaGetLastError());
    FB_CUDA(cudaStreamSynchronize(s));
    M = T;
    return kOk;
}

void m_grid_csr(const Mat& M, std::vector<uint32_t>& rowPtr, std::vector<uint32_t>& colInd,
                std::vector<double>& values)
{
    const uint32_t nx = M.gdim[0], ny = M.gdim[1], nz = M.gdim[2];
    rowPtr.assign((size_t)M.nrow + 1, 0);
    colInd.clear();
    values.clear();
    colInd.reserve(M.nnz);
    values.reserve(M.nnz);
    uint32_t row = 0;
    for (uint32_t iz = 0; iz < nz; ++iz)
        for (uint32_t iy = 0; iy < ny; ++iy)
            for (uint32_t ix = 0; ix < nx; ++ix, ++row) {
                for (uint32_t k = 0; k < M.skLen; ++k) {
                    const int64_t jx = (int64_t)ix + M.gd[0][k], jy = (int64_t)iy + M.gd[1][k],
                                  jz = (int64_t)iz + M.gd[2][k];
                    if (jx < 0 || jy < 0 || jz < 0 || jx >= nx || jy >= ny || jz >= nz) continue;
                    colInd.push_back((uint32_t)((int64_t)row + M.skDelta[k]));
                    values.push_back(M.skVal[k]);
                }
                rowPtr[(size_t)row + 1] = (uint32_t)colInd.size();
            }
}

} // namespace fb
