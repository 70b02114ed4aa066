// dcgs2.cu -- the Arnoldi step of GMRES (GMRES.cxx:160-210, the orthogonalisation of
// :169-175) as classical Gram-Schmidt with delayed re-orthogonalisation (DCGS2: Bielich,
// Langou, Thomas, Swirydowicz, Yamazaki, Boman, "Low-synch Gram-Schmidt with delayed
// reorthogonalization for Krylov solvers", Parallel Computing 112, 2022).
//
// Step j starts from the orthonormal q_0 .. q_{j-1} (Q) and u, the candidate for q_j
// projected once against Q, in basis slot j. It runs the product w = A M u and two passes
// over the basis:
//   dots    a = Q^T u, b = Q^T w, c = u^T w, d = u^T u in one grid reduction; the last block
//           then re-orthogonalises u in exact arithmetic (t = sqrt(d - a^T a), q_j = (u -
//           Q a) / t), completes Hessenberg column j - 1 (+= a, subdiagonal t), applies the
//           reference's Givens step to it, and forms the tentative column j of A M q_j =
//           (w - Q_{j+1} H a) / t: h = (b - H a) / t, h_j = ((c - a^T b) / t - t a_{j-1}) / t
//   update  q_j = (u - Q a) / t into slot j and u_{j+1} = (w - Q b - q_j g) / t into slot
//           j + 1, g = (c - a^T b) / t, the candidate projected once against q_0 .. q_j
// Each pass streams the basis once, where CGS2 streams it three times (multi-dot, fused
// projection + multi-dot, projection + norm) and then scales the new vector: 2j + 6
// vectors of traffic per step instead of 3j + 10, and two launches instead of five.
// Iteration i of the reference (Hessenberg column i - 1) completes in the dots pass of
// step i; a restart cycle of s iterations ends with a dots pass without a product.
//
// Both passes stream 12 KB chunks of each vector through a ring of shared-memory stages
// with bulk asynchronous copies (cp.async.bulk, completion counted in bytes on an
// mbarrier), issued by one thread six stages ahead of the consuming threads; block b takes
// the contiguous element range b of the grid, chunk by chunk, and per chunk the vectors in
// a fixed order (u, w, then Q). Sums are fixed-order: a thread adds its 6 (FP64) or 12
// (FP32) elements of an item, the warp a shuffle tree, each warp its items in chunk order,
// the block its warps in order and the last block the blocks in order -- reruns give the
// same bits.
#include <algorithm>
#include <mutex>
#include <set>
#include <utility>

#include "common.cuh"
#include "gmres.cuh"

namespace fb {

// 12 KB stages, six per block, two blocks per SM: of rings of 4-12 stages of 4-20 KB, with
// two or three blocks per SM, this one ran the 96^3 GMRES(30) profile fastest (5.05 ms for
// 60 steps; 6 x 16 KB 5.47, 8 x 12 KB 5.08, 12 x 8 KB 5.6, three blocks per SM 6.3-8.0)
constexpr uint32_t kDcStageBytes = 12288;
constexpr int      kDcStages = 6;
constexpr int      kDcThreads = 256;
constexpr int      kDcWarps = kDcThreads / 32;
constexpr int      kDcMaxNV = 2 * kDcMaxK + 2; // values of one dots pass
constexpr int      kDcMaxGrid = 384;            // blocks of a pass (a multiple of 32)

template <typename T>
struct DcShape {
    static constexpr int      W = Vec16<T>::W;                    // elements per 16 bytes
    static constexpr uint32_t C = kDcStageBytes / sizeof(T);      // elements per chunk
    static constexpr int      G = (int)(C / W) / kDcThreads;      // 16-byte groups a thread
};

struct alignas(16) DcRing {
    unsigned char      st[kDcStages][kDcStageBytes];
    unsigned long long full[kDcStages];
    int                bad;
};

// The basis, the product and the step.
template <typename T>
struct DcArgs {
    T*       V;    // basis slots 0 .. j + 1, leading dimension ld
    size_t   ld;
    const T* w;    // A M u (null in the closing dots pass of a cycle)
    uint32_t n;
    int      j;
};

// The contiguous element range of this block: a multiple of the 16-byte group.
template <typename T>
__device__ __forceinline__ void dc_range(uint32_t n, size_t& e0, size_t& e1)
{
    constexpr int W = DcShape<T>::W;
    const size_t per = (((size_t)n + gridDim.x - 1) / gridDim.x + W - 1) / W * W;
    e0 = std::min((size_t)n, (size_t)blockIdx.x * per);
    e1 = std::min((size_t)n, e0 + per);
}

// A bulk copy at the default L2 priority: the basis is read again in the next pass and the
// next step, and stays in L2 while it fits.
__device__ __forceinline__ void bulk_copy_g2s_plain(void* dst, const void* src, uint32_t bytes,
                                                    unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Streams the items of the block's range through the ring: chunk after chunk, vectors
// v = 0 .. nItem-1 of src(v) per chunk. consume(v, base, stage, len) runs on every thread
// once the item's bytes have landed (base: the chunk's first element), the block
// synchronises after each item and thread 0 then refills that stage. ready() runs on every
// thread once the first copies are in flight, before the first item (a kernel that may start
// before its predecessor has finished waits for it there). Items are walked with
// counters (no division: a 64-bit division by nItem per item had made the passes
// instruction-bound). The copies start on 16-byte boundaries (the range starts are) and
// round their length up to 16 bytes: at most 8 bytes past the last element, inside every
// vector's allocation. False when a wait ran out: the block has then drained its copies in
// flight (bounded) and stopped.
template <typename T, typename Src, typename Consume, typename Ready>
__device__ __forceinline__ bool dc_stream(DcRing& ring, size_t e0, size_t e1, int nItem, Src src,
                                          Consume consume, Ready ready,
                                          uint32_t pre = (uint32_t)kDcStages)
{
    constexpr uint32_t C = DcShape<T>::C;
    const uint32_t tid = threadIdx.x;
    const uint32_t total = (uint32_t)((e1 - e0 + C - 1) / C) * (uint32_t)nItem;
    // the issuing thread's position: the next item to copy
    int iv = 0, is = 0;
    size_t ib = e0;
    auto issue = [&]() {
        const uint32_t len = (uint32_t)std::min((size_t)C, e1 - ib);
        const uint32_t bytes = (len * (uint32_t)sizeof(T) + 15u) & ~15u;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         smem_addr(&ring.full[is])),
                     "r"(bytes)
                     : "memory");
        bulk_copy_g2s_plain(ring.st[is], src(iv) + ib, bytes, &ring.full[is]);
        if (++is == kDcStages) is = 0;
        if (++iv == nItem) {
            iv = 0;
            ib += C;
        }
    };
    if (tid == 0) {
        ring.bad = 0;
        for (int q = 0; q < kDcStages; ++q)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&ring.full[q]))
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (uint32_t k = 0; k < pre && k < (uint32_t)kDcStages && k < total; ++k) issue();
    }
    // every thread: false leaves before the first item (the block drains its first copies)
    if (!ready()) {
        if (tid == 0)
            for (uint32_t q = 0; q < pre && q < (uint32_t)kDcStages && q < total; ++q)
                mbar_wait_bounded(&ring.full[q], 0u);
        return false;
    }
    // the rest of the first stages: items that may only be read once ready() has passed
    if (tid == 0)
        for (uint32_t k = pre; k < (uint32_t)kDcStages && k < total; ++k) issue();
    __syncthreads();
    int v = 0, st = 0;
    uint32_t ph = 0;
    size_t base = e0;
    for (uint32_t k = 0; k < total; ++k) {
        // the consumers hold warp-collective sums: a warp consumes only if all its lanes saw
        // the bytes land
        const bool mine = mbar_wait_bounded(&ring.full[st], ph);
        const bool landed = __all_sync(0xffffffffu, mine);
        if (!landed) {
            if (!mine) atomicAdd(&fb_tile_timeouts, 1u);
            ring.bad = 1;
        }
        if (landed)
            consume(v, base, (const T*)ring.st[st], (uint32_t)std::min((size_t)C, e1 - base));
        __syncthreads(); // stage st is free again
        if (ring.bad) {
            if (tid == 0) // the copies still in flight: items k .. k + stages - 1
                for (uint32_t i = 0, q = st, p = ph; i < (uint32_t)kDcStages && k + i < total;
                     ++i) {
                    mbar_wait_bounded(&ring.full[q], p);
                    if (++q == (uint32_t)kDcStages) q = 0, p ^= 1u;
                }
            return false;
        }
        if (tid == 0 && k + kDcStages < total) issue();
        if (++st == kDcStages) st = 0, ph ^= 1u;
        if (++v == nItem) {
            v = 0;
            base += C;
        }
    }
    return true;
}

// A thread's elements of a chunk: groups tid, tid + 256, ... (a warp reads 512 contiguous
// bytes per group); entries at or past len read as zero.
template <typename T>
__device__ __forceinline__ void dc_load(const T* st, uint32_t len,
                                        T (&r)[DcShape<T>::G][DcShape<T>::W])
{
    using S = DcShape<T>;
    using VT = typename Vec16<T>::type;
#pragma unroll
    for (int g = 0; g < S::G; ++g) {
        const uint32_t i0 = (uint32_t)(g * kDcThreads + threadIdx.x) * S::W;
        if (i0 + S::W <= len) {
            *(VT*)r[g] = *(const VT*)(st + i0);
        } else {
#pragma unroll
            for (int e = 0; e < S::W; ++e) r[g][e] = i0 + e < len ? st[i0 + e] : T(0);
        }
    }
}

template <typename T>
__device__ __forceinline__ T dc_dot(const T (&x)[DcShape<T>::G][DcShape<T>::W],
                                    const T (&y)[DcShape<T>::G][DcShape<T>::W])
{
    T s = T(0);
#pragma unroll
    for (int g = 0; g < DcShape<T>::G; ++g)
#pragma unroll
        for (int e = 0; e < DcShape<T>::W; ++e) s = fma(x[g][e], y[g][e], s);
    return s;
}

// Warp sums of 16 values at once (a butterfly reduce-scatter): each level halves the values
// a lane holds and exchanges the other half with its partner, 8 + 4 + 2 + 1 + 1 shuffles of
// a double instead of 16 x 5. Returns value (lane >> 1) & 15 summed over the warp (lanes 2r
// and 2r + 1 both hold value r). Every sum is a fixed tree over the lanes, the same on every
// run (a + b and b + a are the same bits).
__device__ __forceinline__ double warp_sum16(const double (&x)[16])
{
    const uint32_t lane = threadIdx.x & 31;
    double y[8], z[4], t[2];
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const double send = b4 ? x[i] : x[i + 8];
        y[i] = (b4 ? x[i + 8] : x[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double send = b3 ? y[i] : y[i + 4];
        z[i] = (b3 ? y[i + 4] : y[i]) + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const double send = b2 ? z[i] : z[i + 2];
        t[i] = (b2 ? z[i + 2] : z[i]) + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    const double send = b1 ? t[0] : t[1];
    const double u = (b1 ? t[1] : t[0]) + __shfl_xor_sync(0xffffffffu, send, 2);
    return u + __shfl_xor_sync(0xffffffffu, u, 1);
}

// ---- the dots pass and the step's scalar work ----------------------------------------

// The product w = A M u of the step, formed by the dots pass itself on stencil masks of the
// fixed 5- or 7-point shape SH: each thread forms its 16-byte groups of w from the
// gathered u (stencil_group: the row sums of k_gm_apply_vec, bit for bit; MODE 1 folds
// diagInv into the gather, MODE 2 scales the result), stores them for the update pass and
// keeps them for the dots. It saves the product's launch and the re-read of w.
template <typename T>
struct DcApply {
    CSRView<T> A;
    const T*   dinv;
    T*         wout;
};

// Value slots: a_l at l, then (with w) b_l at j + l, c at 2j, and d last.
template <typename T, bool HASW, int SH = 0, int MODE = 0>
__global__ void __launch_bounds__(kDcThreads, 2)
k_dc_dots(DcArgs<T> P, Scratch s, GmLayout L, GmCtl* g, DcApply<T> Ap)
{
    constexpr bool FUSE = HASW && SH != 0;
    constexpr int WI = HASW && !FUSE ? 1 : 0; // w streamed as item 1
    extern __shared__ __align__(16) unsigned char dc_raw[];
    DcRing& ring = *reinterpret_cast<DcRing*>(dc_raw);
    __shared__ double wacc[kDcWarps][kDcMaxNV];
    __shared__ double tot[kDcMaxNV];
    __shared__ double col[kDcMaxK + 2], hcol[kDcMaxK], var[2];
    __shared__ GmCtl gs;
    __shared__ bool amLast;
    // launched programmatically after the product or the previous update pass: every input
    // may still be in flight until the grid dependency resolves; the update pass that
    // follows may be scheduled as soon as blocks of this one start
    pdl_wait();
    pdl_release();
    if (g->stop) return;
    using S = DcShape<T>;
    const int j = P.j;
    const int nv = HASW ? 2 * j + 2 : j + 1;
    const int nItem = 1 + WI + j;
    const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int v = tid; v < kDcWarps * nv; v += kDcThreads) wacc[v / nv][v % nv] = 0.0;
    size_t e0, e1;
    dc_range<T>(P.n, e0, e1);
    __syncthreads();
    T u[S::G][S::W], w[S::G][S::W];
    // a thread's products with Q_l for the window of 8 basis vectors l0 .. l0 + 7 (slot
    // l & 7), summed over the warp when the window is full or the chunk's basis ends
    double wa[8], wb[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) wa[q] = wb[q] = 0.0;
    auto src = [&](int v) -> const T* {
        if (v == 0) return P.V + (size_t)j * P.ld;
        if (WI && v == 1) return P.w;
        return P.V + (size_t)(v - 1 - WI) * P.ld;
    };
    auto add = [&](int slot, double x) { // the warp's sum of an item, lane 0 keeps it
        x = warp_reduce(x, kSum);
        if (lane == 0) wacc[wid][slot] += x;
    };
    // the fused product: the thread's groups of w = A M u (every lane of a warp takes part)
    auto product = [&](size_t base, uint32_t len) {
        if constexpr (FUSE) {
            using VT = Vec16<T>;
            using V = typename VT::V;
            const V* uv = reinterpret_cast<const V*>(P.V + (size_t)j * P.ld);
            const V* dv = reinterpret_cast<const V*>(Ap.dinv);
            const uint32_t nw = P.n / S::W;
            auto gather = [&](uint32_t h) {
                const V a = uv[h];
                if (MODE != 1) return a;
                const V d = dv[h];
                T t[S::W];
#pragma unroll
                for (int e = 0; e < S::W; ++e) t[e] = VT::at(a, e) * VT::at(d, e);
                return VT::make(t);
            };
#pragma unroll
            for (int r = 0; r < S::G; ++r) {
                const uint32_t i0 = (uint32_t)(r * kDcThreads + tid) * S::W;
                const uint32_t gi = (uint32_t)(base / S::W) + (uint32_t)(r * kDcThreads + tid);
                // every group of the vector takes part, so that a lane's neighbours in the
                // shuffles are the real groups g - 1 and g + 1 also past the end of this
                // block's range; only the block's own groups are stored and summed
                const bool act = gi < nw, own = i0 + S::W <= len;
                T sum[S::W];
#pragma unroll
                for (int e = 0; e < S::W; ++e) sum[e] = T(0);
                V cgrp;
                stencil_group<T, SH>(Ap.A, gi, nw, act, gather, cgrp, sum);
                if (own && MODE == 2) {
                    const V d = dv[gi];
#pragma unroll
                    for (int e = 0; e < S::W; ++e) sum[e] = sum[e] * VT::at(d, e);
                }
                if (own) reinterpret_cast<V*>(Ap.wout)[gi] = VT::make(sum);
#pragma unroll
                for (int e = 0; e < S::W; ++e) w[r][e] = own ? sum[e] : T(0);
            }
        }
    };
    const bool ok = dc_stream<T>(ring, e0, e1, nItem, src,
                                 [&](int v, size_t base, const T* st, uint32_t len) {
        if (v == 0) {
            dc_load<T>(st, len, u);
            add(nv - 1, (double)dc_dot<T>(u, u));
            if (FUSE) {
                product(base, len);
                add(2 * j, (double)dc_dot<T>(u, w));
            }
        } else if (WI && v == 1) {
            dc_load<T>(st, len, w);
            add(2 * j, (double)dc_dot<T>(u, w));
        } else {
            const int l = v - 1 - WI;
            T q[S::G][S::W];
            dc_load<T>(st, len, q);
            const double pa = (double)dc_dot<T>(q, u);
            const double pb = HASW ? (double)dc_dot<T>(q, w) : 0.0;
            const int r = l & 7;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (i == r) {
                    wa[i] = pa;
                    wb[i] = pb;
                }
            if (r == 7 || l == j - 1) { // the window's warp sums: slot l0 + i (a), j + l0 + i (b)
                double x[16];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    x[i] = wa[i];
                    x[i + 8] = wb[i];
                    wa[i] = wb[i] = 0.0;
                }
                const double sum = warp_sum16(x);
                const int r2 = (int)(lane >> 1) & 15, i = r2 & 7, l0 = l - r;
                if (!(lane & 1) && l0 + i < j && (HASW || r2 < 8))
                    wacc[wid][(r2 < 8 ? 0 : j) + l0 + i] += sum;
            }
        }
    }, [] { return true; });
    // a block that stopped early still takes its ticket, with NaN partials: the step then
    // sees t = NaN and breaks the cycle off (the reference's breakdown exit)
    __syncthreads();
    for (int v = tid; v < nv; v += kDcThreads) {
        double a = 0.0;
        for (int q = 0; q < kDcWarps; ++q) a += wacc[q][v];
        s.partials[(size_t)v * gridDim.x + blockIdx.x] = ok ? a : (double)NAN;
    }
    __syncthreads();
    if (tid == 0) amLast = last_block_ticket(s.ticket);
    __syncthreads();
    if (!amLast) return;
    // totals: warp q adds value v = q, q + 8, ... over the blocks (lane l takes blocks l,
    // l + 32, ... in order, then a shuffle tree); a lane's loads for a value are issued
    // together, two values at a time
    const uint32_t G = gridDim.x;
    for (int v0 = wid; v0 < nv; v0 += 2 * kDcWarps) {
        double x[2][kDcMaxGrid / 32];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int q = 0; q < kDcMaxGrid / 32; ++q) {
                const int v = v0 + h * kDcWarps;
                const uint32_t b = lane + 32u * q;
                x[h][q] = v < nv && b < G ? __ldcg(&s.partials[(size_t)v * G + b]) : 0.0;
            }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            double a = 0.0;
#pragma unroll
            for (int q = 0; q < kDcMaxGrid / 32; ++q) a += x[h][q];
            a = warp_reduce(a, kSum);
            if (lane == 0 && v0 + h * kDcWarps < nv) tot[v0 + h * kDcWarps] = a;
        }
    }
    // the finalize reads the Hessenberg columns 0 .. j-2 and the rotations from shared memory
    // (the ring's stages are free now): loaded by all threads at once rather than one
    // dependent global load at a time
    double* Hs = reinterpret_cast<double*>(ring.st); // [j][j], row i from column i - 1
    double* snS = Hs + (size_t)kDcMaxK * kDcMaxK;
    double* csS = snS + kDcMaxK;
    const size_t m = L.m;
    for (int e = tid; e < j * j; e += kDcThreads) {
        const int i = e / j, l = e - i * j;
        if (l + 1 >= i && l < j - 1) Hs[e] = L.hraw[(size_t)i * m + l];
    }
    for (int i = tid; i < j; i += kDcThreads) {
        snS[i] = L.hsin[i];
        csS[i] = L.hcos[i];
    }
    if (tid == 32) gs = *g;
    if (tid == 64 && j >= 1) {
        var[0] = L.var[j - 1];
        var[1] = L.var[j];
    }
    __syncthreads();
#define HR(i, l) L.hraw[(size_t)(i) * m + (l)]
    const double* A = tot;     // a_l
    const double* B = tot + j; // b_l (with w)
    double t = 1.0, tinv = 1.0;
    if (j >= 1) {
        // re-orthogonalisation of u: column j - 1 gains a, its subdiagonal is ||u - Q a||
        double ssq = 0.0;
        for (int l = 0; l < j; ++l) ssq = fma(A[l], A[l], ssq);
        const double t2 = tot[nv - 1] - ssq;
        t = t2 > 0.0 ? sqrt(t2) : (t2 <= 0.0 ? 0.0 : t2); // a NaN stays NaN
        tinv = 1.0 / t;
        for (int i = tid; i <= j; i += kDcThreads) {
            const double v = i < j ? HR(i, j - 1) + A[i] : t;
            col[i] = v;
            HR(i, j - 1) = v;
        }
        __syncthreads();
    }
    // the tentative column j: h_i = (b_i - sum_l H(i, l) a_l) / t, rows i < j, in l order
    double hj = 0.0, gco = 0.0;
    if (HASW) {
        if (j == 0) {
            gco = hj = tot[2 * j];
        } else {
            for (int i = tid; i < j; i += kDcThreads) {
                double acc = B[i];
                for (int l = i > 0 ? i - 1 : 0; l < j; ++l)
                    acc = fma(-(l == j - 1 ? col[i] : Hs[i * j + l]), A[l], acc);
                hcol[i] = acc * tinv;
            }
            double ab = 0.0;
            for (int l = 0; l < j; ++l) ab = fma(A[l], B[l], ab);
            gco = (tot[2 * j] - ab) * tinv;
            hj = (gco - t * A[j - 1]) * tinv;
        }
    }
    __syncthreads();
    if (tid == 0 && j >= 1) { // iteration j: the Givens step on the completed column j - 1
        auto C = [&](int i) -> double& { return col[i]; };
        auto Sn = [&](int i) { return snS[i]; };
        auto Cs = [&](int i) { return csS[i]; };
        auto Var = [&](int i) -> double& { return var[i == j - 1 ? 0 : 1]; };
        gm_givens_serial(L, j, j - 1, t, C, Sn, Cs, Var, &gs);
        L.var[j - 1] = var[0];
        L.var[j] = var[1];
        *g = gs;
    }
    __syncthreads();
    if (j >= 1)
        for (int i = tid; i <= j; i += kDcThreads) L.hh[(size_t)i * m + (j - 1)] = col[i];
    if constexpr (HASW) {
        if (gs.stop) return;
        for (int i = tid; i <= j; i += kDcThreads) HR(i, j) = i < j ? hcol[i] : hj;
        for (int l = tid; l < j; l += kDcThreads) {
            L.ca[l] = A[l];
            L.cb[l] = B[l];
        }
        if (tid == 0) {
            L.cs[0] = gco;
            L.cs[1] = tinv;
        }
    }
#undef HR
}

// ---- the update pass -----------------------------------------------------------------

// WLAST: w, written by a dots pass that formed the product, is each chunk's last item, and
// only the items before the first w are copied ahead of the grid dependency.
template <typename T, bool WLAST = false>
__global__ void __launch_bounds__(kDcThreads, 2) k_dc_update(DcArgs<T> P, GmLayout L,
                                                             const GmCtl* g)
{
    extern __shared__ __align__(16) unsigned char dc_raw[];
    DcRing& ring = *reinterpret_cast<DcRing*>(dc_raw);
    __shared__ T ca[kDcMaxK], cb[kDcMaxK];
    pdl_release(); // the next step's first kernel waits for this one's completion itself
    using S = DcShape<T>;
    using VT = typename Vec16<T>::type;
    const int j = P.j;
    const int nItem = 2 + j;
    const uint32_t tid = threadIdx.x;
    T gco = T(0), tinv = T(1);
    size_t e0, e1;
    dc_range<T>(P.n, e0, e1);
    // launched programmatically after the dots pass: the copies of u, w and the basis start
    // at once (the dots pass writes none of them: only the Hessenberg state and the
    // coefficients), and the coefficients are read once it has finished
    auto ready = [&]() {
        pdl_wait();
        if (g->stop) return false;
        for (int l = tid; l < j; l += kDcThreads) {
            ca[l] = (T)L.ca[l];
            cb[l] = (T)L.cb[l];
        }
        gco = (T)L.cs[0];
        tinv = (T)L.cs[1];
        return true;
    };
    T u[S::G][S::W], w[S::G][S::W], sa[S::G][S::W], sb[S::G][S::W];
    T* qj = P.V + (size_t)j * P.ld;
    T* un = P.V + (size_t)(j + 1) * P.ld;
    const int wv = WLAST ? nItem - 1 : 1; // w's place in a chunk
    auto src = [&](int v) -> const T* {
        if (v == 0) return P.V + (size_t)j * P.ld;
        if (v == wv) return P.w;
        return P.V + (size_t)(v - (WLAST ? 1 : 2)) * P.ld;
    };
    dc_stream<T>(ring, e0, e1, nItem, src, [&](int v, size_t base, const T* st, uint32_t len) {
        if (v == 0) {
            dc_load<T>(st, len, u);
#pragma unroll
            for (int q = 0; q < S::G; ++q)
#pragma unroll
                for (int e = 0; e < S::W; ++e) sa[q][e] = sb[q][e] = T(0);
        } else if (v == wv) {
            dc_load<T>(st, len, w);
        } else {
            const int l = v - (WLAST ? 1 : 2);
            T q[S::G][S::W];
            dc_load<T>(st, len, q);
            const T al = ca[l], bl = cb[l];
#pragma unroll
            for (int r = 0; r < S::G; ++r)
#pragma unroll
                for (int e = 0; e < S::W; ++e) {
                    sa[r][e] = fma(al, q[r][e], sa[r][e]);
                    sb[r][e] = fma(bl, q[r][e], sb[r][e]);
                }
        }
        if (v == nItem - 1) { // the chunk's last item: q_j and u_{j+1}
#pragma unroll
            for (int r = 0; r < S::G; ++r) {
                const uint32_t i0 = (uint32_t)(r * kDcThreads + tid) * S::W;
                T qo[S::W], uo[S::W];
#pragma unroll
                for (int e = 0; e < S::W; ++e) {
                    qo[e] = j > 0 ? (u[r][e] - sa[r][e]) * tinv : u[r][e];
                    const T x = fma(-qo[e], gco, w[r][e] - sb[r][e]);
                    uo[e] = j > 0 ? x * tinv : x;
                }
                if (i0 + S::W <= len) {
                    if (j > 0) *(VT*)(qj + base + i0) = Vec16<T>::make(qo);
                    *(VT*)(un + base + i0) = Vec16<T>::make(uo);
                } else {
#pragma unroll
                    for (int e = 0; e < S::W; ++e)
                        if (i0 + e < len) {
                            if (j > 0) qj[base + i0 + e] = qo[e];
                            un[base + i0 + e] = uo[e];
                        }
                }
            }
        }
    }, ready, WLAST ? (uint32_t)wv : (uint32_t)kDcStages);
}

// ---- launchers -------------------------------------------------------------------------

// The shared-memory opt-in above 48 KB, once per kernel and device.
static void dc_optin(const void* kern)
{
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (done.insert({kern, dev}).second)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(DcRing));
}

// Launches kern with programmatic stream serialization (the kernel waits for its predecessor
// with pdl_wait before reading anything).
template <typename... P, typename... A>
static int dc_launch(void (*kern)(P...), int grid, size_t smem, cudaStream_t st, A&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kDcThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    FB_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...));
    return kOk;
}

// Resident blocks (two per SM), at least 1024 elements a block, and no more blocks than the
// reduction scratch holds partials of nv values for.
static int dc_grid(const Ctx& c, const void* fn, uint32_t n, int nv)
{
    int g = resident_grid(c, fn, kDcThreads, sizeof(DcRing));
    g = std::min(g, (int)std::max<uint32_t>(1u, (n + 1023) / 1024));
    g = std::min(g, (kMaxRedValues * kMaxGrid) / std::max(nv, 1));
    g = std::min(g, kDcMaxGrid);
    return std::max(g, 1);
}

template <typename T>
int dc_dots(Ctx& c, uint32_t n, int j, T* V, size_t ld, const T* w, const GmLayout& L,
            GmCtl* g)
{
    if (j > kDcMaxK) return kErrInputPar;
    DcArgs<T> P{V, ld, w, n, j};
    DcApply<T> none{};
    ++c.launches;
    int e;
    if (w) {
        auto kern = k_dc_dots<T, true>;
        dc_optin((const void*)kern);
        e = dc_launch(kern, dc_grid(c, (const void*)kern, n, 2 * j + 2), sizeof(DcRing),
                      c.stream, P, c.red, L, g, none);
    } else {
        auto kern = k_dc_dots<T, false>;
        dc_optin((const void*)kern);
        e = dc_launch(kern, dc_grid(c, (const void*)kern, n, j + 1), sizeof(DcRing), c.stream,
                      P, c.red, L, g, none);
    }
    if (e) return e;
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int dc_dots_apply(Ctx& c, const CSRView<T>& A, int mode, const T* dinv, uint32_t n, int j,
                  T* V, size_t ld, T* w, const GmLayout& L, GmCtl* g)
{
    if (j > kDcMaxK) return kErrInputPar;
    const int sh = stencil_vec_shape(A, V + (size_t)j * ld, w,
                                     mode == 0 ? (const void*)w : (const void*)dinv);
    if (!sh) return kErrInputPar;
    DcArgs<T> P{V, ld, w, n, j};
    DcApply<T> Ap{A, dinv, w};
    ++c.launches;
    auto go = [&](auto kern) {
        dc_optin((const void*)kern);
        return dc_launch(kern, dc_grid(c, (const void*)kern, n, 2 * j + 2), sizeof(DcRing),
                         c.stream, P, c.red, L, g, Ap);
    };
    int e;
    if (sh == 5)
        e = mode == 0 ? go(k_dc_dots<T, true, 5, 0>)
                      : mode == 1 ? go(k_dc_dots<T, true, 5, 1>) : go(k_dc_dots<T, true, 5, 2>);
    else
        e = mode == 0 ? go(k_dc_dots<T, true, 7, 0>)
                      : mode == 1 ? go(k_dc_dots<T, true, 7, 1>) : go(k_dc_dots<T, true, 7, 2>);
    if (e) return e;
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int dc_update(Ctx& c, uint32_t n, int j, T* V, size_t ld, const T* w, const GmLayout& L,
              const GmCtl* g, bool wlast)
{
    if (j > kDcMaxK) return kErrInputPar;
    DcArgs<T> P{V, ld, w, n, j};
    ++c.launches;
    auto kern = wlast ? k_dc_update<T, true> : k_dc_update<T, false>;
    dc_optin((const void*)kern);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)dc_grid(c, (const void*)kern, n, 1));
    cfg.blockDim = dim3(kDcThreads);
    cfg.dynamicSmemBytes = sizeof(DcRing);
    cfg.stream = c.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    FB_CUDA(cudaLaunchKernelEx(&cfg, kern, P, L, g));
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template int dc_dots<double>(Ctx&, uint32_t, int, double*, size_t, const double*,
                             const GmLayout&, GmCtl*);
template int dc_dots<float>(Ctx&, uint32_t, int, float*, size_t, const float*, const GmLayout&,
                            GmCtl*);
template int dc_update<double>(Ctx&, uint32_t, int, double*, size_t, const double*,
                               const GmLayout&, const GmCtl*, bool);
template int dc_update<float>(Ctx&, uint32_t, int, float*, size_t, const float*,
                              const GmLayout&, const GmCtl*, bool);
template int dc_dots_apply<double>(Ctx&, const CSRView<double>&, int, const double*, uint32_t,
                                   int, double*, size_t, double*, const GmLayout&, GmCtl*);
template int dc_dots_apply<float>(Ctx&, const CSRView<float>&, int, const float*, uint32_t,
                                  int, float*, size_t, float*, const GmLayout&, GmCtl*);

unsigned tile_timeouts_dcgs2() { return tile_timeouts(); }

} // namespace fb
