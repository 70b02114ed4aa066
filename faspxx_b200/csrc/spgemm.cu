// spgemm.cu -- sparse matrix algebra on the device: the product C = L R, MAT::Mult
// (src/MAT.cxx:715-800) with its exact result:
//   * the columns of row i of C appear in the order in which the loop over L's row i
//     (entries k in CSR order) and, for each, R's row colInd[k] (entries l in CSR order)
//     first meets them -- MAT::Mult does not sort its rows;
//   * C(i, c) = 0 + sum of L(i,k) R(k,l) over the (k, l) pairs with column c, added in that
//     same loop order, each product rounded before it is added.
// On the GPU: every (k, l) pair of a row is a candidate with the 64-bit key
// column << 32 | position (position = its index in the loop order), the keys of each row are
// sorted (equal columns become adjacent, in loop order), each run of one column is summed in
// order and remembered by its first position, and a second sort by first position restores
// MAT::Mult's column order. Products are computed and stored before they are added, so no
// multiply-add is fused. Further down: the sum C = a A + b B, MAT::Add.
#include "segsort.cuh"

namespace fb {
namespace {

// candidates per row, and their total in 64 bits (a product can have more than 2^32)
__global__ void k_mult_count(uint32_t n, const uint32_t* __restrict__ lrp,
                             const uint32_t* __restrict__ lci, const uint32_t* __restrict__ rrp,
                             uint32_t* __restrict__ cnt, unsigned long long* __restrict__ total)
{
    unsigned long long mine = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        unsigned long long c = 0;
        for (uint32_t k = lrp[i]; k < lrp[i + 1]; ++k) {
            const uint32_t j = lci[k];
            c += rrp[j + 1] - rrp[j];
        }
        cnt[i] = c > 0xffffffffull ? 0xffffffffu : (uint32_t)c;
        mine += c;
    }
    if (mine) atomicAdd(total, mine);
}

// keys (column << 32 | position in the row's loop order) and the rounded products
__global__ void k_mult_expand(uint32_t n, const uint32_t* __restrict__ lrp,
                              const uint32_t* __restrict__ lci, const double* __restrict__ lva,
                              const uint32_t* __restrict__ rrp, const uint32_t* __restrict__ rci,
                              const double* __restrict__ rva, const uint32_t* __restrict__ coff,
                              uint64_t* __restrict__ keys, double* __restrict__ prod)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        uint32_t p = 0;
        const size_t base = coff[i];
        for (uint32_t k = lrp[i]; k < lrp[i + 1]; ++k) {
            const uint32_t j = lci[k];
            const double a = lva[k];
            for (uint32_t l = rrp[j]; l < rrp[j + 1]; ++l, ++p) {
                keys[base + p] = (uint64_t)rci[l] << 32 | p;
                prod[base + p] = a * rva[l];
            }
        }
    }
}

// distinct columns per row (the keys of each row sorted)
__global__ void k_mult_distinct(uint32_t n, const uint32_t* __restrict__ coff,
                                const uint64_t* __restrict__ keys, uint32_t* __restrict__ nout)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        uint32_t d = 0;
        for (uint32_t q = coff[i]; q < coff[i + 1]; ++q)
            if (q == coff[i] || (keys[q] >> 32) != (keys[q - 1] >> 32)) ++d;
        nout[i] = d;
    }
}

// one entry per distinct column: its sum in loop order, its column, and the key
// first position << 32 | group index that orders the row as MAT::Mult does
__global__ void k_mult_groups(uint32_t n, const uint32_t* __restrict__ coff,
                              const uint64_t* __restrict__ keys, const double* __restrict__ prod,
                              const uint32_t* __restrict__ crp, uint64_t* __restrict__ okeys,
                              uint32_t* __restrict__ gcol, double* __restrict__ gsum)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t b = coff[i], e = coff[i + 1];
        uint32_t g = 0;
        for (uint32_t q = b; q < e;) {
            const uint32_t col = (uint32_t)(keys[q] >> 32);
            const uint32_t first = (uint32_t)keys[q];
            double s = 0.0;
            for (; q < e && (uint32_t)(keys[q] >> 32) == col; ++q)
                s = __dadd_rn(s, prod[(size_t)b + (uint32_t)keys[q]]);
            const size_t o = (size_t)crp[i] + g;
            okeys[o] = (uint64_t)first << 32 | g;
            gcol[o] = col;
            gsum[o] = s;
            ++g;
        }
    }
}

__global__ void k_mult_out(uint32_t n, const uint32_t* __restrict__ crp,
                           const uint64_t* __restrict__ okeys, const uint32_t* __restrict__ gcol,
                           const double* __restrict__ gsum, uint32_t* __restrict__ cci,
                           double* __restrict__ cva)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        for (uint32_t q = crp[i]; q < crp[i + 1]; ++q) {
            const size_t src = (size_t)crp[i] + (uint32_t)okeys[q];
            cci[q] = gcol[src];
            cva[q] = gsum[src];
        }
}

} // namespace

int m_mult(Ctx& c, const Mat& L, const Mat& R, Mat& C)
{
    if (L.grid || R.grid || !L.val || !R.val) return kErrInputPar; // stored values needed
    if (L.mcol != R.nrow) return kErrNonmatch;
    if (L.nrow == 0 || R.mcol == 0) return kErrMatSize;
    cudaStream_t s = c.stream;
    const uint32_t n = L.nrow;
    Tmp t;
    int e;
    uint32_t *cnt = nullptr, *coff = nullptr, *tiles = nullptr;
    unsigned long long* total = nullptr;
    if ((e = t.get(&cnt, n)) || (e = t.get(&coff, (size_t)n + 1)) ||
        (e = t.get(&tiles, (n + (size_t)kTile - 1) / kTile)) || (e = t.get(&total, 1)))
        return e;
    FB_CUDA(cudaMemsetAsync(total, 0, sizeof(unsigned long long), s));
    const int g = grid_for(n, 256);
    k_mult_count<<<g, 256, 0, s>>>(n, L.rowPtr, L.colInd, R.rowPtr, cnt, total);
    FB_CUDA(cudaGetLastError());
    unsigned long long htotal = 0;
    FB_CUDA(cudaMemcpyAsync(&htotal, total, sizeof(htotal), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    if (htotal == 0) return kErrMatSize; // MAT::Mult would build a matrix with no entries
    if (htotal > 0xffffffffull) return kErrMatSize;
    const uint32_t ncand = (uint32_t)htotal;
    if ((e = scan_counts(s, n, cnt, coff, tiles))) return e;
    uint64_t* keys = nullptr;
    double* prod = nullptr;
    if ((e = t.get(&keys, ncand)) || (e = t.get(&prod, ncand))) return e;
    k_mult_expand<<<g, 256, 0, s>>>(n, L.rowPtr, L.colInd, L.val, R.rowPtr, R.colInd, R.val,
                                    coff, keys, prod);
    FB_CUDA(cudaGetLastError());
    if ((e = sort_row_keys(c, t, n, coff, keys, ncand))) return e;
    uint32_t *nout = cnt, *crp = nullptr;
    if ((e = t.get(&crp, (size_t)n + 1))) return e;
    k_mult_distinct<<<g, 256, 0, s>>>(n, coff, keys, nout);
    FB_CUDA(cudaGetLastError());
    if ((e = scan_counts(s, n, nout, crp, tiles))) return e;
    uint32_t nnzC = 0;
    FB_CUDA(cudaMemcpyAsync(&nnzC, crp + n, 4, cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    uint64_t* okeys = nullptr;
    uint32_t *gcol = nullptr, *cci = nullptr;
    double *gsum = nullptr, *cva = nullptr;
    if ((e = t.get(&okeys, nnzC)) || (e = t.get(&gcol, nnzC)) || (e = t.get(&gsum, nnzC)) ||
        (e = t.get(&cci, nnzC)) || (e = t.get(&cva, nnzC)))
        return e;
    k_mult_groups<<<g, 256, 0, s>>>(n, coff, keys, prod, crp, okeys, gcol, gsum);
    FB_CUDA(cudaGetLastError());
    if ((e = sort_row_keys(c, t, n, crp, okeys, nnzC))) return e;
    k_mult_out<<<g, 256, 0, s>>>(n, crp, okeys, gcol, gsum, cci, cva);
    FB_CUDA(cudaGetLastError());
    FB_CUDA(cudaStreamSynchronize(s));
    return m_upload(C, n, R.mcol, nnzC, crp, cci, cva, false, s);
}

namespace {

// ---- MAT::Add (src/MAT.cxx:652-713): C = a A + b B -------------------------------------------
// Row i of C: A's entries in order as a A(i,k); then each entry of B's row in order is added
// to the first entry of A's row with its column -- or to the first of B's entries already
// appended to this row, the one extra slot MAT::Add's search window reaches -- else appended
// as b B(i,k); finally each row sorted by column, stably (SortCSRRow). Products and sums are
// rounded separately as the reference rounds them.

__global__ void k_add_rows(uint32_t n, double a, double b, const uint32_t* __restrict__ arp,
                           const uint32_t* __restrict__ aci, const double* __restrict__ ava,
                           const uint32_t* __restrict__ brp, const uint32_t* __restrict__ bci,
                           const double* __restrict__ bva, uint32_t* __restrict__ tci,
                           double* __restrict__ tva, uint32_t* __restrict__ nout)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t base = (size_t)arp[i] + brp[i];
        const uint32_t c1 = arp[i + 1] - arp[i];
        uint32_t cnt = 0;
        for (uint32_t k = arp[i]; k < arp[i + 1]; ++k, ++cnt) {
            tci[base + cnt] = aci[k];
            tva[base + cnt] = __dmul_rn(a, ava[k]);
        }
        for (uint32_t k = brp[i]; k < brp[i + 1]; ++k) {
            const uint32_t col = bci[k];
            const double v = __dmul_rn(b, bva[k]);
            const uint32_t window = cnt > c1 ? c1 + 1 : c1;
            uint32_t l = 0;
            for (; l < window; ++l)
                if (tci[base + l] == col) break;
            if (l < window) {
                tva[base + l] = __dadd_rn(tva[base + l], v);
            } else {
                tci[base + cnt] = col;
                tva[base + cnt] = v;
                ++cnt;
            }
        }
        nout[i] = cnt;
    }
}

__global__ void k_add_keys(uint32_t n, const uint32_t* __restrict__ arp,
                           const uint32_t* __restrict__ brp, const uint32_t* __restrict__ crp,
                           const uint32_t* __restrict__ tci, uint64_t* __restrict__ keys)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t base = (size_t)arp[i] + brp[i];
        for (uint32_t q = crp[i]; q < crp[i + 1]; ++q) {
            const uint32_t p = q - crp[i];
            keys[q] = (uint64_t)tci[base + p] << 32 | p;
        }
    }
}

__global__ void k_add_out(uint32_t n, const uint32_t* __restrict__ arp,
                          const uint32_t* __restrict__ brp, const uint32_t* __restrict__ crp,
                          const uint64_t* __restrict__ keys, const double* __restrict__ tva,
                          uint32_t* __restrict__ cci, double* __restrict__ cva)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t base = (size_t)arp[i] + brp[i];
        for (uint32_t q = crp[i]; q < crp[i + 1]; ++q) {
            cci[q] = (uint32_t)(keys[q] >> 32);
            cva[q] = tva[base + (uint32_t)keys[q]];
        }
    }
}

} // namespace

int m_add(Ctx& c, double a, const Mat& A, double b, const Mat& B, Mat& C)
{
    if (A.grid || B.grid || !A.val || !B.val) return kErrInputPar;
    if (A.nrow != B.nrow || A.mcol != B.mcol) return kErrNonmatch;
    const uint64_t cap = (uint64_t)A.nnz + B.nnz;
    if (cap > 0xffffffffull) return kErrMatSize;
    cudaStream_t s = c.stream;
    const uint32_t n = A.nrow;
    Tmp t;
    int e;
    uint32_t *tci = nullptr, *nout = nullptr, *crp = nullptr, *tiles = nullptr, *cci = nullptr;
    double *tva = nullptr, *cva = nullptr;
    uint64_t* keys = nullptr;
    if ((e = t.get(&tci, cap)) || (e = t.get(&tva, cap)) || (e = t.get(&nout, n)) ||
        (e = t.get(&crp, (size_t)n + 1)) || (e = t.get(&tiles, (n + (size_t)kTile - 1) / kTile)))
        return e;
    const int g = grid_for(n, 256);
    k_add_rows<<<g, 256, 0, s>>>(n, a, b, A.rowPtr, A.colInd, A.val, B.rowPtr, B.colInd, B.val,
                                 tci, tva, nout);
    FB_CUDA(cudaGetLastError());
    if ((e = scan_counts(s, n, nout, crp, tiles))) return e;
    uint32_t nnzC = 0;
    FB_CUDA(cudaMemcpyAsync(&nnzC, crp + n, 4, cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    if ((e = t.get(&keys, nnzC)) || (e = t.get(&cci, nnzC)) || (e = t.get(&cva, nnzC))) return e;
    k_add_keys<<<g, 256, 0, s>>>(n, A.rowPtr, B.rowPtr, crp, tci, keys);
    FB_CUDA(cudaGetLastError());
    if ((e = sort_row_keys(c, t, n, crp, keys, nnzC))) return e;
    k_add_out<<<g, 256, 0, s>>>(n, A.rowPtr, B.rowPtr, crp, keys, tva, cci, cva);
    FB_CUDA(cudaGetLastError());
    FB_CUDA(cudaStreamSynchronize(s));
    return m_upload(C, n, A.mcol, nnzC, crp, cci, cva, false, s);
}

} // namespace fb
