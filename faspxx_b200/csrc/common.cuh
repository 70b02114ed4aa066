// common.cuh -- shared device helpers of the B200 iterative-solve library.
//
// Reductions are deterministic: every kernel that reduces runs on a fixed grid, each block
// reduces its grid-stride share in a fixed shuffle order and writes one partial per value;
// the last block to finish (ticket counter) sums the partials in a fixed order and runs the
// kernel's scalar "finalize" step on one thread. Reruns are therefore bit-identical.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

namespace fb {

constexpr int kBlock = 256;          // threads per block for vector kernels
constexpr int kMaxRedValues = 16;    // values one fused reduction may carry
constexpr int kMaxGrid = 148 * 16;   // upper bound of any reducing grid (partials sizing)

struct Scratch {
    double*   partials;  // [kMaxRedValues][kMaxGrid]
    unsigned* ticket;    // one counter, always returned to 0 by the last block
};

enum RedOp { kSum = 0, kMax = 1 };

__device__ __forceinline__ double red_ident(int op) { return op == kMax ? 0.0 : 0.0; }

__device__ __forceinline__ double red_apply(double a, double b, int op)
{
    // max of magnitudes: operands are |.| >= 0 or NaN; fmax drops a NaN like VEC::NormInf
    return op == kMax ? fmax(a, b) : a + b;
}

__device__ __forceinline__ double warp_reduce(double v, int op)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = red_apply(v, __shfl_down_sync(0xffffffffu, v, o), op);
    return v;
}

// Reduces acc[0..NV) over the block; on return thread 0 holds the block totals.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&acc)[NV], const int (&ops)[NV])
{
    __shared__ double sh[32][NV];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = warp_reduce(acc[k], ops[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[wid][k] = acc[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = lane < nw ? sh[lane][k] : red_ident(ops[k]);
            acc[k] = warp_reduce(t, ops[k]);
        }
    }
    __syncthreads();
}

// One thread's share of the partials of every block: value k of block b sits at
// partials[k * kMaxGrid + b]; the thread sums blocks threadIdx.x, +blockDim.x, ... in that
// order. The loads of U consecutive block indices (all NV values) are issued before their
// adds, so the last block waits for about gridDim / (blockDim U) L2 round trips instead of
// one per block index and value.
template <int NV>
__device__ __forceinline__ void sum_partials(const double* partials, const int (&ops)[NV],
                                             double (&tot)[NV])
{
    constexpr int U = NV >= 8 ? 1 : 8 / NV;
#pragma unroll
    for (int k = 0; k < NV; ++k) tot[k] = red_ident(ops[k]);
    const int nb = (int)gridDim.x, bd = (int)blockDim.x;
    for (int b0 = threadIdx.x; b0 < nb; b0 += U * bd) {
        double v[U][NV];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int b = b0 + u * bd;
#pragma unroll
            for (int k = 0; k < NV; ++k)
                v[u][k] = b < nb ? __ldcg(&partials[k * kMaxGrid + b]) : red_ident(ops[k]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k = 0; k < NV; ++k) tot[k] = red_apply(tot[k], v[u][k], ops[k]);
    }
}

// Called by thread 0 of every block after its partials are written: true in exactly one
// block, the last to arrive, which returns the counter to 0. The ticket is one acq_rel
// atomic: its release half publishes this block's partials, and in the last block its
// acquire half (with the __syncthreads that follows in the caller) orders the partial
// loads after every block's release -- no separate fences (the last block's full fence
// cost ~0.35 us per reduction on B200). Counting in per-group counters first, to spread
// the atomics over several addresses, measured slower: the completing block pays two
// dependent atomics instead of one.
__device__ __forceinline__ bool last_block_ticket(unsigned* ticket)
{
    unsigned prev;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(prev) : "l"(ticket)
                 : "memory");
    if (prev != gridDim.x - 1) return false;
    *ticket = 0;
    return true;
}

// Grid-wide deterministic reduction. Every thread of every block must call it (after its
// grid-stride work). The last block runs fin(totals) on thread 0. Returns nothing useful to
// other threads.
template <int NV, typename Fin>
__device__ __forceinline__ void grid_reduce(double (&acc)[NV], const int (&ops)[NV],
                                            Scratch s, Fin fin)
{
    __shared__ bool amLast;
    block_reduce<NV>(acc, ops);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) s.partials[k * kMaxGrid + blockIdx.x] = acc[k];
        amLast = last_block_ticket(s.ticket);
    }
    __syncthreads();
    if (!amLast) return;
    double tot[NV];
    sum_partials<NV>(s.partials, ops, tot);
    block_reduce<NV>(tot, ops);
    if (threadIdx.x == 0) fin(tot);
}

// grid_reduce for kernels whose finalize runs a solver's scalar state machine on a control
// block in global memory. That code is a chain of dependent reads and writes of the block's
// fields; run on global memory, every link costs an L2 round trip while the rest of the GPU
// waits for the kernel to end. Here the last block loads the whole control block into
// shared memory with one parallel read (issued before the partials are summed, so the two
// overlap), thread 0 runs fin(ctl_in_shared_memory, totals), and the block writes it back.
// Only the last block touches the control block after the ticket: every other block has
// read what it needs before its own reduction.
template <int NV, typename Ctl, typename Fin>
__device__ __forceinline__ void grid_reduce_ctl(double (&acc)[NV], const int (&ops)[NV],
                                                Scratch s, Ctl* gctl, Fin fin)
{
    static_assert(sizeof(Ctl) % 4 == 0, "control block copied in 4-byte words");
    constexpr int kWords = (int)(sizeof(Ctl) / 4);
    __shared__ bool amLast;
    __shared__ __align__(16) uint32_t sc[kWords];
    block_reduce<NV>(acc, ops);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) s.partials[k * kMaxGrid + blockIdx.x] = acc[k];
        amLast = last_block_ticket(s.ticket);
    }
    __syncthreads();
    if (!amLast) return;
    uint32_t* g = reinterpret_cast<uint32_t*>(gctl);
    for (int w = threadIdx.x; w < kWords; w += blockDim.x) sc[w] = __ldcg(g + w);
    double tot[NV];
    sum_partials<NV>(s.partials, ops, tot);
    block_reduce<NV>(tot, ops); // ends with a barrier: sc is complete
    if (threadIdx.x == 0) fin(reinterpret_cast<Ctl*>(sc), tot);
    __syncthreads();
    for (int w = threadIdx.x; w < kWords; w += blockDim.x) __stcg(g + w, sc[w]);
}

// Reduction over L consecutive lanes (L a power of two <= 32), result in the group's lane 0.
template <int L, typename T>
__device__ __forceinline__ T group_sum(T v)
{
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, L);
    return v;
}

// CSRx matrix view: 32-bit unsigned indices as in FASP++'s MAT (src/MAT.hxx:43-47).
constexpr int kMaxStencil = 16;

template <typename T>
struct CSRView {
    uint32_t        nrow, mcol, nnz;
    const uint32_t* rowPtr;
    const uint32_t* colInd;
    // 16-bit column offsets (optional, thread-per-row kernels): colInd[k] - row as int16_t,
    // present when every entry of the matrix is within 32,767 columns of its row; the
    // thread-per-row kernels then stream 2 bytes per entry instead of 4.
    const int16_t*  cd16;
    const T*        val;   // nullptr: pattern only (every stored entry is 1)
    // Row classes (optional, thread-per-row kernels): rows with identical column offsets
    // (col - row) and values share one table entry; cls[row] picks it. Entries of class k
    // are [coff[k], coff[k+1]) in cdelta / cval, in the row's CSR order.
    const uint16_t* cls;
    const uint32_t* coff;
    const int32_t*  cdelta;
    const T*        cval;
    // Stencil masks (optional, thread-per-row kernels): every row is a subset of one sorted
    // list of column offsets udelta[0..ulen) whose values uval are the same in every row
    // that has them (constant coefficients, truncated at the boundary); mask[row] says which
    // are present. The lists travel in the kernel's parameter space, so a row costs one
    // 2-byte load plus its gathers.
    const uint16_t* mask;
    uint32_t        ulen;
    int32_t         udelta[kMaxStencil];
    T               uval[kMaxStencil];
    // Structured-grid form (a matrix-free operator, no stored matrix; gnz == 0: not one).
    // Row i is the grid point (ix, iy, iz), i = ix + nx (iy + ny iz); its entries are the
    // stencil list above truncated at the faces, and its mask is computed from the
    // coordinates: in dimension d, with t = min(coordinate, 3) and u = min(extent - 1 -
    // coordinate, 3), the offsets present are glo[4d + t] & ghi[4d + u] (every offset
    // reaches at most 3 points in each dimension). Division by nx and nx ny uses
    // multiply-high with precomputed constants (FastDiv).
    uint32_t        gnx, gny, gnz, gnxy;
    uint32_t        gmx, gmxy;      // FastDiv multipliers for nx and nx ny
    uint8_t         gsx[2], gsxy[2]; // and their shifts
    uint16_t        glo[12], ghi[12];
    // Block tiles of plain CSR (csr_tile_rows): tileSpan is the most entries any 256-row
    // tile covers once widened to multiples of 4 (from the upload; 0 unknown), and tiles is
    // set by a launch that gives its blocks the tile stages (with_tiles).
    uint32_t        tileSpan;
    uint32_t        tiles;
};

// Division of a 32-bit unsigned n by a divisor fixed at launch (Granlund and Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994, Figure 4.1): with
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, t = mulhi(m, n),
// n / d = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0) for every n < 2^32.
struct FastDiv {
    uint32_t m;
    uint8_t  s1, s2;
    static FastDiv make(uint32_t d)
    {
        uint32_t l = 0;
        while (l < 32 && (1ull << l) < d) ++l;
        FastDiv f;
        f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
        f.s1 = (uint8_t)(l < 1 ? l : 1);
        f.s2 = (uint8_t)(l > 1 ? l - 1 : 0);
        return f;
    }
};

__device__ __forceinline__ uint32_t fast_div(uint32_t n, uint32_t m, uint32_t s1, uint32_t s2)
{
    const uint32_t t = __umulhi(m, n);
    return (t + ((n - t) >> s1)) >> s2;
}

// The stencil mask of grid row `row` (structured-grid form); V is any view with the g*
// fields of CSRView.
template <typename V>
__device__ __forceinline__ uint32_t grid_mask(const V& A, uint32_t row)
{
    const uint32_t iz = fast_div(row, A.gmxy, A.gsxy[0], A.gsxy[1]);
    const uint32_t rem = row - iz * A.gnxy;
    const uint32_t iy = fast_div(rem, A.gmx, A.gsx[0], A.gsx[1]);
    const uint32_t ix = rem - iy * A.gnx;
    auto dim = [&](int d, uint32_t c, uint32_t N) {
        const uint32_t t = c < 3u ? c : 3u, u = N - 1u - c < 3u ? N - 1u - c : 3u;
        return (uint32_t)A.glo[4 * d + t] & (uint32_t)A.ghi[4 * d + u];
    };
    return dim(0, ix, A.gnx) & dim(1, iy, A.gny) & dim(2, iz, A.gnz);
}

// The matrix is streamed once per SpMV: evict-first loads keep it from displacing the
// vectors, which are reused every iteration and fit in the 126 MB L2 at the benchmark sizes.
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p) { return __ldcs(p); }
__device__ __forceinline__ int16_t ld_stream(const int16_t* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }

// sum_k val[k] * xv(col[k]) over one row [b, e) on one thread, left to right (the order of
// MAT::Apply, src/MAT.cxx:378-419). Entries go in predicated chunks of 4 with the chunk's
// column/value loads issued before any gather, so a 7-entry stencil row has all its
// matrix loads in flight at once.
template <typename T, bool PAT, typename XV>
__device__ __forceinline__ T row_dot(const CSRView<T>& A, size_t row, uint32_t b, uint32_t e,
                                     XV xv)
{
    T s = T(0);
#pragma unroll 2
    for (uint32_t k = b; k < e; k += 4) {
        uint32_t c[4];
        T v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool in = k + u < e;
            if (A.cd16)
                c[u] = in ? (uint32_t)((long long)row + ld_stream(A.cd16 + k + u)) : 0u;
            else
                c[u] = in ? ld_stream(A.colInd + k + u) : 0u;
            v[u] = PAT ? T(in ? 1 : 0) : (in ? ld_stream(A.val + k + u) : T(0));
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < e) s = fma(v[u], xv(c[u]), s);
    }
    return s;
}

// Two CSR rows r0, r1 on one thread, interleaved: both rows' pointers, then both rows'
// chunks of four column/value loads, then their gathers, then the FMAs, each row left to
// right as row_dot sums it (the same bits). A thread that walks its rows one at a time waits
// for three dependent round trips per row (row pointer, entries, gathers); two at a time it
// waits half as often.
template <typename T, typename XV>
__device__ __forceinline__ void row_dot2(const CSRView<T>& A, size_t r0, size_t r1, XV xv,
                                         T& s0, T& s1)
{
    const uint32_t b0 = ld_stream(A.rowPtr + r0), e0 = ld_stream(A.rowPtr + r0 + 1);
    const uint32_t b1 = ld_stream(A.rowPtr + r1), e1 = ld_stream(A.rowPtr + r1 + 1);
    s0 = T(0);
    s1 = T(0);
    for (uint32_t k = 0; b0 + k < e0 || b1 + k < e1; k += 4) {
        uint32_t c0[4], c1[4];
        T v0[4], v1[4], x0[4], x1[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool in0 = b0 + k + u < e0, in1 = b1 + k + u < e1;
            c0[u] = in0 ? ld_stream(A.colInd + b0 + k + u) : 0u;
            c1[u] = in1 ? ld_stream(A.colInd + b1 + k + u) : 0u;
            v0[u] = in0 ? ld_stream(A.val + b0 + k + u) : T(0);
            v1[u] = in1 ? ld_stream(A.val + b1 + k + u) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            x0[u] = b0 + k + u < e0 ? xv(c0[u]) : T(0);
            x1[u] = b1 + k + u < e1 ? xv(c1[u]) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (b0 + k + u < e0) s0 = fma(v0[u], x0[u], s0);
            if (b1 + k + u < e1) s1 = fma(v1[u], x1[u], s1);
        }
    }
}

// ---- block tiles of plain CSR, streamed by bulk async copies ------------------------------
// Thread per row streams each row's column indices and values on its own: the lanes of a
// warp read 4-byte words some 28 bytes apart (a 7-entry row), and a thread has one row's
// loads in flight at a time, too few bytes to cover the latency of HBM. A block tile takes
// 256 consecutive rows, one per thread, whose entries are one contiguous range: one thread
// copies the tile's row pointers, column indices and values into shared memory with bulk
// asynchronous copies (cp.async.bulk, completion counted in bytes on an mbarrier), two
// tiles ahead, so the copy engine keeps the stream in flight while the threads gather x for
// the current tile. Each thread sums its row from the stage in CSR order with one FMA per
// entry (the bits of row_dot). The copies start at an entry index that is a multiple of 4
// (16-byte aligned) and run to the next multiple of 4 past the tile's last entry: up to 3
// entries beyond nnz, inside the spare bytes every matrix array is allocated with.
constexpr uint32_t kTileRows = 256; // rows per tile = threads per block
constexpr int kTileStages = 2;
constexpr uint32_t kTileRp = kTileRows + 4;

template <typename T>
struct TileShape {
    // bytes per stage: 2 stages and the kernels' own static shared memory (at most 3 KB)
    // stay under the 48 KB a launch gets without opting in; FP32 takes less so that more
    // blocks fit on an SM. Both hold a 256-row tile of a 7-point stencil (1,798 entries).
    static constexpr uint32_t bytes = sizeof(T) == 8 ? 22800u : 16000u;
    static constexpr uint32_t cap = ((bytes - kTileRp * 4u) / (4u + sizeof(T))) & ~3u;
};

template <typename T>
struct alignas(16) TileStage {
    uint32_t rp[kTileRp];
    uint32_t c[TileShape<T>::cap];
    T v[TileShape<T>::cap];
};

template <typename T>
struct alignas(16) TileSmem {
    TileStage<T> st[kTileStages];
    unsigned long long full[kTileStages]; // mbarriers: one phase per copied tile
    uint32_t a[kTileStages];              // the stage's first entry index
    uint32_t ok[kTileStages];             // entries staged (else only the row pointers)
    uint32_t bad;                         // a tile wait ran out: the block leaves
};

// Waits that ran out (a bulk copy that never completed): counted here, per translation
// unit, and read by tile_timeouts() on the host. The block then stops: it waits (bounded
// again) for the copies it still has in flight and returns, leaving the rest of its rows
// unwritten.
static __device__ unsigned fb_tile_timeouts;

extern __shared__ __align__(16) unsigned char fb_tile_smem[];

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// An L2 policy that marks the lines it touches first to evict: the matrix is streamed once
// per product, and at normal priority it would push the solver's vectors (reused every
// iteration, resident in the 126 MB L2 at the benchmark sizes) out of L2, as the
// evict-first loads (ld_stream) of the row-at-a-time kernels do not.
__device__ __forceinline__ unsigned long long l2_evict_first()
{
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              unsigned long long* bar, unsigned long long pol)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
                 ".L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
                 : "memory");
}

// At most 2^20 polls (each try_wait itself suspends for a bounded time), then false.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, uint32_t parity)
{
    for (uint32_t it = 0; it < (1u << 20); ++it) {
        uint32_t done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
                     "selp.u32 %0, 1, 0, p; }"
                     : "=r"(done)
                     : "r"(smem_addr(bar)), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// Rows of a plain CSR view in block tiles; own(row, sum) on the row's thread. Block b takes
// tiles b, b + G, b + 2G, ... (G = gridDim.x), so thread t of the grid owns rows t, t + S,
// t + 2S, ... (S = the grid's threads) in that order, as the row-at-a-time loops do. Every
// thread of the block calls it (it synchronises the block). A tile whose entries do not fit
// a stage (only possible when the caller ignored the span check of with_tiles) is summed
// from global memory.
template <typename T, bool PAT, typename XV, typename OWN>
__device__ __forceinline__ void csr_tile_rows(const CSRView<T>& A, TileSmem<T>& sm, XV xv,
                                              OWN own)
{
    constexpr uint32_t CAP = TileShape<T>::cap;
    const size_t n = A.nrow;
    const size_t ntiles = (n + kTileRows - 1) / kTileRows;
    const uint32_t tid = threadIdx.x;
    const size_t mine =
        blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const unsigned long long pol = tid == 0 ? l2_evict_first() : 0ull;
    auto issue = [&](size_t k) { // thread 0: tile k of this block into stage k % stages
        const int s = (int)(k % kTileStages);
        const size_t r0 = (blockIdx.x + k * gridDim.x) * kTileRows;
        const size_t rows = n - r0 < kTileRows ? n - r0 : kTileRows;
        const uint32_t beg = A.rowPtr[r0], end = A.rowPtr[r0 + rows];
        const uint32_t a = beg & ~3u, ar = (uint32_t)(((size_t)end + 3) & ~size_t(3));
        const bool ok = ar - a <= CAP;
        const uint32_t rpn = (uint32_t)((rows + 1 + 3) & ~size_t(3));
        const uint32_t eb = PAT ? 4u : 4u + (uint32_t)sizeof(T);
        sm.a[s] = a;
        sm.ok[s] = ok ? 1u : 0u;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         smem_addr(&sm.full[s])),
                     "r"(rpn * 4u + (ok ? (ar - a) * eb : 0u))
                     : "memory");
        bulk_copy_g2s(sm.st[s].rp, A.rowPtr + r0, rpn * 4u, &sm.full[s], pol);
        if (ok && ar > a) {
            bulk_copy_g2s(sm.st[s].c, A.colInd + a, (ar - a) * 4u, &sm.full[s], pol);
            if (!PAT)
                bulk_copy_g2s(sm.st[s].v, A.val + a, (ar - a) * (uint32_t)sizeof(T),
                              &sm.full[s], pol);
        }
    };
    if (tid == 0) {
        sm.bad = 0;
        for (int s = 0; s < kTileStages; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&sm.full[s]))
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (size_t k = 0; k < (size_t)kTileStages && k < mine; ++k) issue(k);
    }
    __syncthreads();
    for (size_t k = 0; k < mine; ++k) {
        const int s = (int)(k % kTileStages);
        const bool landed = mbar_wait_bounded(&sm.full[s], (uint32_t)((k / kTileStages) & 1));
        if (!landed) {
            atomicAdd(&fb_tile_timeouts, 1u);
            sm.bad = 1;
        }
        const size_t row = (blockIdx.x + k * gridDim.x) * kTileRows + tid;
        if (landed && row < n) {
            const TileStage<T>& st = sm.st[s];
            const uint32_t b = st.rp[tid], e = st.rp[tid + 1];
            T sum = T(0);
            if (sm.ok[s]) {
                const uint32_t a = sm.a[s];
#pragma unroll 2
                for (uint32_t k4 = b; k4 < e; k4 += 4) {
                    uint32_t cc[4];
                    T v[4], xs[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const bool in = k4 + u < e;
                        cc[u] = in ? st.c[k4 + u - a] : 0u;
                        v[u] = PAT ? T(in ? 1 : 0) : (in ? st.v[k4 + u - a] : T(0));
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) xs[u] = k4 + u < e ? xv(cc[u]) : T(0);
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (k4 + u < e) sum = fma(v[u], xs[u], sum);
                }
            } else {
                sum = row_dot<T, PAT>(A, row, b, e, xv);
            }
            own(row, sum);
        }
        __syncthreads(); // stage s is free again
        if (sm.bad) { // every thread sees it after the barrier: leave together
            if (tid == 0) // the copies this block still has in flight (tiles k .. k + 1)
                for (size_t j = k; j < k + kTileStages && j < mine; ++j)
                    mbar_wait_bounded(&sm.full[j % kTileStages],
                                      (uint32_t)((j / kTileStages) & 1));
            return;
        }
        if (tid == 0 && k + kTileStages < mine) issue(k + kTileStages);
    }
}

// Row `row` of A times the gathered vector, through the row-class table when A has one
// (2 bytes streamed per row instead of the row's column indices and values), else through
// the CSR arrays. Both accumulate the entries in CSR order with one FMA each, so the two
// storage forms give bit-identical results.
template <typename T, bool PAT, typename XV>
__device__ __forceinline__ T row_apply(const CSRView<T>& A, size_t row, XV xv)
{
    if (!PAT && (A.mask || A.gnz)) {
        const uint32_t m = A.gnz ? grid_mask(A, (uint32_t)row) : (uint32_t)__ldcs(A.mask + row);
        T s = T(0);
        // chunks of 8 offsets: a 7-point row issues all its gathers before the first FMA
        // (loading every offset at a clamped index instead, so that the gathers need not
        // wait for the mask, measured slower on B200: 12.9 vs 10.4 ms per mixed 128^3 solve)
#pragma unroll
        for (int c0 = 0; c0 < kMaxStencil; c0 += 8) {
            if (c0 >= (int)A.ulen) break;
            T xs[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int k = c0 + u;
                const bool in = k < (int)A.ulen && ((m >> k) & 1u);
                xs[u] = in ? xv((uint32_t)((long long)row + A.udelta[k])) : T(0);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int k = c0 + u;
                if (k < (int)A.ulen && ((m >> k) & 1u)) s = fma(A.uval[k], xs[u], s);
            }
        }
        return s;
    }
    if (!PAT && A.cls) {
        const uint32_t k = __ldcs(A.cls + row);
        const uint32_t b = __ldg(A.coff + k), e = __ldg(A.coff + k + 1);
        T s = T(0);
#pragma unroll 2
        for (uint32_t i = b; i < e; i += 4) {
            T v[4], xs[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool in = i + u < e;
                const long long d = in ? (long long)__ldg(A.cdelta + i + u) : 0;
                v[u] = in ? __ldg(A.cval + i + u) : T(0);
                xs[u] = in ? xv((uint32_t)((long long)row + d)) : T(0);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (i + u < e) s = fma(v[u], xs[u], s);
        }
        return s;
    }
    const uint32_t b = ld_stream(A.rowPtr + row), e = ld_stream(A.rowPtr + row + 1);
    return row_dot<T, PAT>(A, row, b, e, xv);
}

// Every row of A once, own(row, sum) on the thread that owns it: thread t of the grid owns
// rows t, t + S, t + 2S, ... (S = the grid's threads) in that order. Views launched with
// block tiles (A.tiles, see with_tiles) stream them; call it with every thread of the block.
template <typename T, bool PAT, typename XV, typename OWN>
__device__ __forceinline__ void for_rows(const CSRView<T>& A, XV xv, OWN own)
{
    if (A.tiles) {
        csr_tile_rows<T, PAT>(A, *reinterpret_cast<TileSmem<T>*>(fb_tile_smem), xv, own);
        return;
    }
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t row = (size_t)blockIdx.x * blockDim.x + threadIdx.x; row < A.nrow;
         row += stride)
        own(row, row_apply<T, PAT>(A, row, xv));
}

// Block tiles for a plain CSR view (no row classes, stencil masks, grid form or 16-bit
// offsets) whose every 256-row tile fits a stage (tileSpan, from the upload), with 16-byte
// aligned arrays, launched with blocks of kTileRows threads: marks the view and returns the
// dynamic shared memory its kernel must be launched with (0, view unmarked, otherwise).
// Launchers then call tiles_fit with the kernel, which unmarks the view again when the
// kernel's static shared memory and the stages together exceed 48 KB.
template <typename T>
inline size_t with_tiles(CSRView<T>& V, int block)
{
    auto al = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
    const bool ok = V.nrow > 0 && !V.cls && !V.mask && !V.gnz && !V.cd16 &&
                    V.tileSpan > 0 && V.tileSpan <= TileShape<T>::cap &&
                    block == (int)kTileRows && al(V.rowPtr) && al(V.colInd) &&
                    (!V.val || al(V.val));
    V.tiles = ok ? 1u : 0u;
    return ok ? sizeof(TileSmem<T>) : 0;
}

// This translation unit's count of tile waits that ran out.
static inline unsigned tile_timeouts()
{
    unsigned v = 0;
    if (cudaMemcpyFromSymbol(&v, fb_tile_timeouts, sizeof(v)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return v;
}

// Programmatic dependent launch: a kernel launched with the programmatic-serialization
// attribute may start while its predecessor drains; pdl_wait() blocks until the predecessor
// has completed and its writes are visible (a no-op for an ordinary launch), pdl_release()
// lets the successor be scheduled. Every kernel that uses them calls pdl_wait() before its
// first global-memory access.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The fixed stencil shape of a stencil-mask view (the vector-row SpMV kernels' SH): 5 or 7 when its sorted offsets are
// [-S1, -1, 0, 1, S1] or [-S2, -S1, -1, 0, 1, S1, S2] with S1, S2 multiples of 4, else 0.
template <typename V>
inline int stencil_shape(const V& A)
{
    if (A.ulen != 5 && A.ulen != 7) return 0;
    const int mid = (int)A.ulen / 2;
    if (A.udelta[mid] != 0 || A.udelta[mid - 1] != -1 || A.udelta[mid + 1] != 1) return 0;
    for (int k = 0; k < (int)A.ulen; ++k)
        if ((k < mid - 1 || k > mid + 1) && A.udelta[k] % 4 != 0) return 0;
    return (int)A.ulen;
}

// 16-byte groups of rows: four FP32 or two FP64 values.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using V = float4;
    using type = float4;
    static constexpr int W = 4;
    __device__ static float at(const float4& v, int j)
    {
        return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
    }
    __device__ static float4 zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    // (prev last, v.x, v.y, v.z) and (v.y, v.z, v.w, next first): the -1 and +1 neighbours
    __device__ static float4 down(float prevLast, const float4& v)
    {
        return make_float4(prevLast, v.x, v.y, v.z);
    }
    __device__ static float4 up(const float4& v, float nextFirst)
    {
        return make_float4(v.y, v.z, v.w, nextFirst);
    }
    __device__ static float first(const float4& v) { return v.x; }
    __device__ static float last(const float4& v) { return v.w; }
    __device__ static float4 make(const float* s) { return make_float4(s[0], s[1], s[2], s[3]); }
};
template <>
struct Vec16<double> {
    using V = double2;
    using type = double2;
    static constexpr int W = 2;
    __device__ static double at(const double2& v, int j) { return j == 0 ? v.x : v.y; }
    __device__ static double2 zero() { return make_double2(0.0, 0.0); }
    __device__ static double2 down(double prevLast, const double2& v)
    {
        return make_double2(prevLast, v.x);
    }
    __device__ static double2 up(const double2& v, double nextFirst)
    {
        return make_double2(v.y, nextFirst);
    }
    __device__ static double first(const double2& v) { return v.x; }
    __device__ static double last(const double2& v) { return v.y; }
    __device__ static double2 make(const double* s) { return make_double2(s[0], s[1]); }
};

// The vector-row stencil kernel applies: stencil masks (or a grid operator) of the 5- or
// 7-point shape, a square matrix, n % W == 0, 16-byte aligned vectors and aligned masks.
template <typename T>
inline int stencil_vec_shape(const CSRView<T>& A, const void* p0, const void* p1,
                             const void* p2)
{
    constexpr int W = 16 / (int)sizeof(T);
    auto al = [](const void* p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) == 0; };
    if (!(A.mask || A.gnz) || A.nrow != A.mcol || A.nrow % W != 0 || A.nrow >= (1u << 30))
        return 0;
    if (!al(p0, 16) || !al(p1, 16) || !al(p2, 16) || (A.mask && !al(A.mask, 2 * W))) return 0;
    return stencil_shape(A);
}

// The W row sums of rows W g .. W g + W - 1 (a 16-byte group) of a stencil-mask view (or
// grid operator) of the fixed 5- or 7-point shape SH, gathering the vector whose group h
// gv(h) returns (h < nw = n / W); c = gv(g). Lanes of a warp hold consecutive groups and
// every lane calls it (the loop bound is warp-uniform; act = g < nw): offsets -1/+1 come
// from the neighbouring lanes' groups by shuffles (lanes 0 and 31 fetch the group beyond
// the warp), +-S from aligned groups, fetched for every group inside [0, nw) whatever the
// masks say (a needed element lies in [0, n) and n % W == 0, so its group does too).
// Each row sums its entries in offset order with one FMA each, as row_apply does.
template <typename T, int SH, typename GV>
__device__ __forceinline__ void stencil_group(const CSRView<T>& A, uint32_t g, uint32_t nw,
                                              bool act, GV gv, typename Vec16<T>::V& c,
                                              T (&s)[Vec16<T>::W])
{
    using VT = Vec16<T>;
    using V = typename VT::V;
    constexpr int W = VT::W, MID = SH / 2;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t m[W];
#pragma unroll
    for (int j = 0; j < W; ++j) m[j] = 0u;
    c = VT::zero();
    if (act) {
        c = gv(g);
        if (A.gnz) {
#pragma unroll
            for (int j = 0; j < W; ++j) m[j] = grid_mask(A, W * g + (uint32_t)j);
        } else if constexpr (W == 4) {
            const uint2 mm = __ldg(reinterpret_cast<const uint2*>(A.mask) + g);
            m[0] = mm.x & 0xffffu;
            m[1] = mm.x >> 16;
            m[2] = mm.y & 0xffffu;
            m[3] = mm.y >> 16;
        } else {
            const uint32_t mm = __ldg(reinterpret_cast<const uint32_t*>(A.mask) + g);
            m[0] = mm & 0xffffu;
            m[1] = mm >> 16;
        }
    }
    T pl = __shfl_up_sync(0xffffffffu, VT::last(c), 1);
    T nf = __shfl_down_sync(0xffffffffu, VT::first(c), 1);
    if (lane == 0 && act && g > 0) pl = VT::last(gv(g - 1));
    if (lane == 31 && act && g + 1 < nw) nf = VT::first(gv(g + 1));
    V xs[SH];
#pragma unroll
    for (int k = 0; k < SH; ++k) {
        if (k == MID) {
            xs[k] = c;
        } else if (k == MID - 1) {
            xs[k] = VT::down(pl, c);
        } else if (k == MID + 1) {
            xs[k] = VT::up(c, nf);
        } else {
            const uint32_t ga = g + (uint32_t)(A.udelta[k] / W); // wrapped
            xs[k] = act && ga < nw ? gv(ga) : VT::zero();
        }
    }
#pragma unroll
    for (int j = 0; j < W; ++j)
#pragma unroll
        for (int k = 0; k < SH; ++k)
            if ((m[j] >> k) & 1u) s[j] = fma(A.uval[k], VT::at(xs[k], j), s[j]);
}

__host__ __device__ inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

} // namespace fb

#define FB_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            std::fprintf(stderr, "fasp_b200: CUDA error %s at %s:%d\n",                      \
                         cudaGetErrorString(e_), __FILE__, __LINE__);                        \
            return ::fb::kErrCuda;                                                           \
        }                                                                                    \
    } while (0)
