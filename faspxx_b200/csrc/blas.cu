// blas.cu -- vector kernels: the VEC operations of FASP++ (src/VEC.cxx) on device memory.
//
// All are bandwidth-bound, grid-stride loops on coalesced 8-byte accesses. Reductions use the
// deterministic two-pass grid reduction of common.cuh and deliver their result to a device
// scalar, so a following kernel can consume it without a host round trip. Sums use FMA and
// a different association than the reference's 4 interleaved partial sums (VEC.cxx:424-485);
// results agree to rounding, not bit for bit.
#include <cstdint>
#include <map>
#include <tuple>
#include <mutex>
#include <type_traits>

#include "internal.h"

namespace fb {

#define GRID_STRIDE(i, n) \
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)(n); \
         i += (size_t)gridDim.x * blockDim.x)

int resident_grid(const Ctx& c, const void* fn, int block, size_t smem)
{
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, size_t>, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(fn, block, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, smem) != cudaSuccess ||
        nb < 1) {
        cudaGetLastError();
        nb = 1;
    }
    long long g = (long long)nb * c.nsm;
    if (g > kMaxGrid) g = kMaxGrid;
    cache[key] = (int)g;
    return (int)g;
}

bool tiles_fit(const void* fn, size_t smem)
{
    static std::mutex mu;
    static std::map<const void*, size_t> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(fn);
    if (it == cache.end()) {
        cudaFuncAttributes at{};
        if (cudaFuncGetAttributes(&at, fn) != cudaSuccess) {
            cudaGetLastError();
            at.sharedSizeBytes = 48 * 1024; // unknown: no tiles
        }
        it = cache.emplace(fn, at.sharedSizeBytes).first;
    }
    return it->second + smem <= 48 * 1024;
}

int Ctx::grid(long long work, int perBlock, int perSM) const
{
    long long g = (work + perBlock - 1) / perBlock;
    long long cap = (long long)nsm * perSM;
    if (cap > kMaxGrid) cap = kMaxGrid;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// ---- reductions ------------------------------------------------------------------------
// T = double (the reference's arithmetic) or float (mixed-precision inner solves: each
// thread accumulates in T, the block and grid stages in FP64).

template <typename T>
__global__ void k_dot(uint32_t n, const T* __restrict__ a, const T* __restrict__ b, Scratch s,
                      double* dres)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    T t = T(0);
    GRID_STRIDE(i, n) t = fma(a[i], b[i], t);
    double acc[1] = {(double)t};
    const int ops[1] = {kSum};
    grid_reduce<1>(acc, ops, s, [=] __device__(const double* v) { *dres = v[0]; });
}

template <typename T>
__global__ void k_norm2(uint32_t n, const T* __restrict__ a, Scratch s, double* dres)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    T t = T(0);
    GRID_STRIDE(i, n) t = fma(a[i], a[i], t);
    double acc[1] = {(double)t};
    const int ops[1] = {kSum};
    grid_reduce<1>(acc, ops, s, [=] __device__(const double* v) { *dres = sqrt(v[0]); });
}

template <typename T>
__global__ void k_norminf(uint32_t n, const T* __restrict__ a, Scratch s, double* dres)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    T t = T(0);
    GRID_STRIDE(i, n) t = fmax(t, fabs(a[i]));
    double acc[1] = {(double)t};
    const int ops[1] = {kMax};
    grid_reduce<1>(acc, ops, s, [=] __device__(const double* v) { *dres = v[0]; });
}

template <typename T>
int v_dot(Ctx& c, uint32_t n, const T* a, const T* b, double* dres)
{
    ++c.launches;
    FB_CUDA(launch_pdl(k_dot<T>, dim3((unsigned)c.grid(n, kBlock)), dim3(kBlock), 0, c.stream, n,
                       a, b, c.red, dres));
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int v_norm2(Ctx& c, uint32_t n, const T* a, double* dres)
{
    ++c.launches;
    FB_CUDA(launch_pdl(k_norm2<T>, dim3((unsigned)c.grid(n, kBlock)), dim3(kBlock), 0, c.stream,
                       n, a, c.red, dres));
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int v_norminf(Ctx& c, uint32_t n, const T* a, double* dres)
{
    ++c.launches;
    FB_CUDA(launch_pdl(k_norminf<T>, dim3((unsigned)c.grid(n, kBlock)), dim3(kBlock), 0,
                       c.stream, n, a, c.red, dres));
    FB_CUDA(cudaGetLastError());
    return kOk;
}

// ---- updates ---------------------------------------------------------------------------

template <typename T>
__global__ void k_axpy(uint32_t n, Scal a, const T* __restrict__ x, T* __restrict__ y)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    const T av = (T)eval(a);
    GRID_STRIDE(i, n) y[i] = fma(av, x[i], y[i]);
}

template <typename T>
__global__ void k_xpay(uint32_t n, Scal a, const T* __restrict__ x, T* __restrict__ y)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    const T av = (T)eval(a);
    GRID_STRIDE(i, n) y[i] = fma(av, y[i], x[i]);
}

template <typename T>
__global__ void k_axpby(uint32_t n, Scal a, Scal b, const T* __restrict__ y, T* __restrict__ x)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    const T av = (T)eval(a), bv = (T)eval(b);
    GRID_STRIDE(i, n) x[i] = fma(av, x[i], bv * y[i]);
}

template <typename T>
__global__ void k_waxpby(uint32_t n, Scal a, const T* __restrict__ v1, Scal b,
                         const T* __restrict__ v2, T* __restrict__ w)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    const T av = (T)eval(a), bv = (T)eval(b);
    GRID_STRIDE(i, n) w[i] = fma(av, v1[i], bv * v2[i]);
}

template <typename T>
__global__ void k_scale(uint32_t n, Scal a, T* __restrict__ x)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    const T av = (T)eval(a);
    GRID_STRIDE(i, n) x[i] *= av;
}

template <typename T>
__global__ void k_set(uint32_t n, T v, T* __restrict__ x)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    GRID_STRIDE(i, n) x[i] = v;
}

template <typename T>
__global__ void k_pmult(uint32_t n, const T* __restrict__ d, T* __restrict__ x)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    GRID_STRIDE(i, n) x[i] *= d[i];
}

template <typename T>
__global__ void k_add(uint32_t n, const T* __restrict__ d, T* __restrict__ x)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    GRID_STRIDE(i, n) x[i] += d[i];
}

// Jacobi::Setup (src/Iter.cxx:45-47): diagInv = weight * (1 / diag), two roundings as there.
__global__ void k_recip_scale(uint32_t n, double w, const double* __restrict__ d,
                              double* __restrict__ out)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    GRID_STRIDE(i, n) out[i] = (1.0 / d[i]) * w;
}

#define LAUNCH_EW(kernel, n, ...)                                                          \
    do {                                                                                   \
        if ((n) == 0) return kOk;                                                          \
        FB_CUDA(launch_pdl(kernel, dim3((unsigned)c.grid((n), kBlock)), dim3(kBlock), 0,   \
                           c.stream, (n), __VA_ARGS__));                                   \
        ++c.launches;                                                                      \
        FB_CUDA(cudaGetLastError());                                                       \
        return kOk;                                                                        \
    } while (0)

template <typename T>
int v_axpy(Ctx& c, uint32_t n, Scal a, const T* x, T* y) { LAUNCH_EW(k_axpy<T>, n, a, x, y); }
template <typename T>
int v_xpay(Ctx& c, uint32_t n, Scal a, const T* x, T* y) { LAUNCH_EW(k_xpay<T>, n, a, x, y); }
template <typename T>
int v_axpby(Ctx& c, uint32_t n, Scal a, Scal b, const T* y, T* x)
{
    LAUNCH_EW(k_axpby<T>, n, a, b, y, x);
}
template <typename T>
int v_waxpby(Ctx& c, uint32_t n, Scal a, const T* v1, Scal b, const T* v2, T* w)
{
    LAUNCH_EW(k_waxpby<T>, n, a, v1, b, v2, w);
}
template <typename T>
int v_scale(Ctx& c, uint32_t n, Scal a, T* x) { LAUNCH_EW(k_scale<T>, n, a, x); }
template <typename T>
int v_set(Ctx& c, uint32_t n, double v, T* x) { LAUNCH_EW(k_set<T>, n, (T)v, x); }
template <typename T>
int v_pmult(Ctx& c, uint32_t n, const T* d, T* x) { LAUNCH_EW(k_pmult<T>, n, d, x); }
template <typename T>
int v_add(Ctx& c, uint32_t n, const T* d, T* x) { LAUNCH_EW(k_add<T>, n, d, x); }
int v_recip_scale(Ctx& c, uint32_t n, double w, const double* d, double* out)
{
    LAUNCH_EW(k_recip_scale, n, w, d, out);
}

// L2 flush by reading: every 16-byte group of buf is loaded through L2 (ld.global.cg); the
// store is taken only if the XOR of all loaded words equals a value the caller never
// writes, which keeps the loads without writing anything in practice.
__global__ void __launch_bounds__(256) k_l2_flush_read(const uint4* __restrict__ buf, size_t n16,
                                                       unsigned* __restrict__ sink)
{
    unsigned acc = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint4 v = __ldcg(buf + i);
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if (acc == 0x9e3779b9u) *sink = acc;
}

int l2_flush_read(Ctx& c, const void* buf, size_t bytes)
{
    const size_t n16 = bytes / 16;
    if (n16 == 0) return kOk;
    const int grid = c.nsm * 8;
    k_l2_flush_read<<<grid, 256, 0, c.stream>>>(static_cast<const uint4*>(buf), n16,
                                               const_cast<unsigned*>(static_cast<const unsigned*>(buf)));
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int v_copy(Ctx& c, uint32_t n, const T* src, T* dst)
{
    if (n == 0 || src == dst) return kOk;
    FB_CUDA(cudaMemcpyAsync(dst, src, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice,
                            c.stream));
    return kOk;
}

// ---- classical Gram-Schmidt building blocks ------------------------------------------
// V holds basis vectors at V + j*ld. KC vectors are handled per launch; the coefficients
// h stay FP64 for either vector type. When V, w and the stride allow it (16-byte aligned
// vectors, ld a multiple of the vector width), each thread reads 16-byte vectors of
// consecutive elements (VEC = 1), which keeps more bytes in flight per thread; the few
// elements past the last full vector are read one by one.

constexpr int KC = 8;

// Grid of the Gram-Schmidt kernels (one grid for all three, so the fused kernel maps
// elements to threads exactly as the separate ones): 3 blocks per SM, all resident at once
// (each kernel is compiled for 3 blocks of kBlock threads) -- one wave, each thread keeping
// several 16-byte loads per vector in flight, and few partials for the grid reduction.
static int mgrid(const Ctx& c, uint32_t n) { return c.grid(n, kBlock, 3); }

template <typename T>
static bool vec_ok(const T* V, size_t ld, const T* w)
{
    return ((reinterpret_cast<uintptr_t>(V) | reinterpret_cast<uintptr_t>(w)) & 15) == 0 &&
           ld % Vec16<T>::W == 0;
}

// The Gram-Schmidt kernels take the number of basis vectors of a launch, K, at compile time:
// every 16-byte load of an element group (w and the K basis vectors) is issued before the
// group's FMAs, and with K <= 3 each thread takes two groups per step, so a thread keeps
// K + 1 or 2 (K + 1) loads in flight instead of waiting on each vector in turn (the
// one-wave grid gives each thread only a few steps). The groups, and the elements in each
// group, are accumulated in the same order as one group at a time, so the results do not
// depend on the grouping. Two groups per step only for K <= 3: more would exceed the 85
// registers a thread has at 3 blocks of kBlock threads per SM.
template <int K>
__host__ __device__ constexpr int gs_unroll() { return K <= 3 ? 2 : 1; }

// dres[j] = (V_j, w), j < K
template <typename T, int VEC, int K>
__global__ void __launch_bounds__(kBlock, 3)
k_multidot(uint32_t n, const T* __restrict__ V, size_t ld, const T* __restrict__ w, Scratch s,
           double* dres, const int* stop)
{
    if (stop && *stop) return;
    using VT = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::W;
    constexpr int U = gs_unroll<K>();
    T t[K];
    double acc[K];
    int ops[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        t[j] = T(0);
        ops[j] = kSum;
    }
    size_t i0 = 0;
    if (VEC) {
        const size_t nv = n / W, stride = (size_t)gridDim.x * blockDim.x;
        size_t iv = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        for (; iv + (U - 1) * stride < nv; iv += U * stride) {
            T wv[U][W], vv[U][K][W];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                *(VT*)wv[u] = ((const VT*)w)[iv + u * stride];
#pragma unroll
                for (int j = 0; j < K; ++j)
                    *(VT*)vv[u][j] = ((const VT*)(V + j * ld))[iv + u * stride];
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int e = 0; e < W; ++e) t[j] = fma(vv[u][j][e], wv[u][e], t[j]);
        }
        for (; iv < nv; iv += stride) {
            T wv[W], vv[K][W];
            *(VT*)wv = ((const VT*)w)[iv];
#pragma unroll
            for (int j = 0; j < K; ++j) *(VT*)vv[j] = ((const VT*)(V + j * ld))[iv];
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int e = 0; e < W; ++e) t[j] = fma(vv[j][e], wv[e], t[j]);
        }
        i0 = nv * W;
    }
    for (size_t i = i0 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const T wi = w[i];
#pragma unroll
        for (int j = 0; j < K; ++j) t[j] = fma(V[j * ld + i], wi, t[j]);
    }
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = (double)t[j];
    grid_reduce<K>(acc, ops, s, [=] __device__(const double* v) {
        for (int j = 0; j < K; ++j) dres[j] = v[j];
    });
}

// w -= sign * sum_j h[j] V_j (j < K); with dnorm != null also ||w_new|| -> *dnorm.
template <typename T, int VEC, int K>
__global__ void __launch_bounds__(kBlock, 3)
k_multiaxpy(uint32_t n, const T* __restrict__ V, size_t ld, const double* __restrict__ h,
            double sign, T* __restrict__ w, Scratch s, double* dnorm, const int* stop)
{
    if (stop && *stop) return;
    using VT = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::W;
    constexpr int U = gs_unroll<K>();
    T hj[K];
#pragma unroll
    for (int j = 0; j < K; ++j) hj[j] = (T)(sign * h[j]);
    T t = T(0);
    size_t i0 = 0;
    if (VEC) {
        const size_t nv = n / W, stride = (size_t)gridDim.x * blockDim.x;
        size_t iv = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        for (; iv + (U - 1) * stride < nv; iv += U * stride) {
            T wv[U][W], vv[U][K][W];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                *(VT*)wv[u] = ((const VT*)w)[iv + u * stride];
#pragma unroll
                for (int j = 0; j < K; ++j)
                    *(VT*)vv[u][j] = ((const VT*)(V + j * ld))[iv + u * stride];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int e = 0; e < W; ++e) wv[u][e] = fma(-hj[j], vv[u][j][e], wv[u][e]);
                ((VT*)w)[iv + u * stride] = *(VT*)wv[u];
#pragma unroll
                for (int e = 0; e < W; ++e) t = fma(wv[u][e], wv[u][e], t);
            }
        }
        for (; iv < nv; iv += stride) {
            T wv[W], vv[K][W];
            *(VT*)wv = ((const VT*)w)[iv];
#pragma unroll
            for (int j = 0; j < K; ++j) *(VT*)vv[j] = ((const VT*)(V + j * ld))[iv];
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int e = 0; e < W; ++e) wv[e] = fma(-hj[j], vv[j][e], wv[e]);
            ((VT*)w)[iv] = *(VT*)wv;
#pragma unroll
            for (int e = 0; e < W; ++e) t = fma(wv[e], wv[e], t);
        }
        i0 = nv * W;
    }
    for (size_t i = i0 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        T wi = w[i];
#pragma unroll
        for (int j = 0; j < K; ++j) wi = fma(-hj[j], V[j * ld + i], wi);
        w[i] = wi;
        t = fma(wi, wi, t);
    }
    double acc[1] = {(double)t};
    const int ops[1] = {kSum};
    if (dnorm) grid_reduce<1>(acc, ops, s, [=] __device__(const double* v) { *dnorm = sqrt(v[0]); });
}

// CGS2's second projection and its re-orthogonalisation dots in one pass over the basis,
// for K <= 8 vectors (what fits in registers with every load hoisted): w -= sum_j h[j] V_j,
// then dres[j] = (V_j, w_new), each basis vector loaded once. Each element's FMA sequence,
// each thread's elements (the same grid and mapping as k_multidot) and the reduction order
// equal those of k_multiaxpy followed by k_multidot, so the results are bit-identical to
// the two passes; V is read once instead of twice.
template <typename T>
__host__ __device__ constexpr int kf() { return 8; }

template <typename T, int VEC, int K>
__global__ void __launch_bounds__(kBlock, 3)
k_multiaxpy_dot(uint32_t n, const T* __restrict__ V, size_t ld, const double* __restrict__ h,
                T* __restrict__ w, Scratch s, double* dres, const int* stop)
{
    if (stop && *stop) return;
    using VT = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::W;
    constexpr int U = gs_unroll<K>();
    __shared__ T hs[K];
    if (threadIdx.x < K) hs[threadIdx.x] = (T)(1.0 * h[threadIdx.x]);
    __syncthreads();
    T t[K];
#pragma unroll
    for (int j = 0; j < K; ++j) t[j] = T(0);
    size_t i0 = 0;
    if (VEC) {
        const size_t nv = n / W, stride = (size_t)gridDim.x * blockDim.x;
        size_t iv = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        for (; iv + (U - 1) * stride < nv; iv += U * stride) {
            T wv[U][W], vv[U][K][W];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                *(VT*)wv[u] = ((const VT*)w)[iv + u * stride];
#pragma unroll
                for (int j = 0; j < K; ++j)
                    *(VT*)vv[u][j] = ((const VT*)(V + j * ld))[iv + u * stride];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int e = 0; e < W; ++e) wv[u][e] = fma(-hs[j], vv[u][j][e], wv[u][e]);
                ((VT*)w)[iv + u * stride] = *(VT*)wv[u];
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int e = 0; e < W; ++e) t[j] = fma(vv[u][j][e], wv[u][e], t[j]);
            }
        }
        for (; iv < nv; iv += stride) {
            T wv[W], vv[K][W];
            *(VT*)wv = ((const VT*)w)[iv];
#pragma unroll
            for (int j = 0; j < K; ++j) *(VT*)vv[j] = ((const VT*)(V + j * ld))[iv];
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int e = 0; e < W; ++e) wv[e] = fma(-hs[j], vv[j][e], wv[e]);
            ((VT*)w)[iv] = *(VT*)wv;
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int e = 0; e < W; ++e) t[j] = fma(vv[j][e], wv[e], t[j]);
        }
        i0 = nv * W;
    }
    for (size_t i = i0 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        T wi = w[i];
#pragma unroll
        for (int j = 0; j < K; ++j) wi = fma(-hs[j], V[j * ld + i], wi);
        w[i] = wi;
#pragma unroll
        for (int j = 0; j < K; ++j) t[j] = fma(V[j * ld + i], wi, t[j]);
    }
    double acc[K];
    int ops[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        acc[j] = (double)t[j];
        ops[j] = kSum;
    }
    grid_reduce<K>(acc, ops, s, [=] __device__(const double* v) {
        for (int j = 0; j < K; ++j) dres[j] = v[j];
    });
}

// Compile-time K from a runtime count k in [1, KMAX]: calls f(std::integral_constant<int, K>).
template <int KMAX, typename F>
static void with_k(int k, F&& f)
{
    switch (k) {
        case 1: f(std::integral_constant<int, 1>()); break;
        case 2: f(std::integral_constant<int, 2>()); break;
        case 3: f(std::integral_constant<int, 3>()); break;
        case 4: f(std::integral_constant<int, 4>()); break;
        case 5: f(std::integral_constant<int, 5>()); break;
        case 6: f(std::integral_constant<int, 6>()); break;
        case 7: f(std::integral_constant<int, 7>()); break;
        case 8: f(std::integral_constant<int, 8>()); break;
        default:
            if constexpr (KMAX > 8) {
                switch (k) {
                    case 9: f(std::integral_constant<int, 9>()); break;
                    case 10: f(std::integral_constant<int, 10>()); break;
                    case 11: f(std::integral_constant<int, 11>()); break;
                    case 12: f(std::integral_constant<int, 12>()); break;
                    case 13: f(std::integral_constant<int, 13>()); break;
                    case 14: f(std::integral_constant<int, 14>()); break;
                    case 15: f(std::integral_constant<int, 15>()); break;
                    default: f(std::integral_constant<int, 16>()); break;
                }
            }
            break;
    }
}

// ---- one launch per Gram-Schmidt pass ---------------------------------------------------
// k_gs handles up to kGsMaxK basis vectors in one launch (a GMRES(30) Arnoldi step has up
// to 31), so a CGS2 step is three launches whatever its size instead of three per 8
// vectors: each launch has a fixed cost (ramp, one-wave tail, the reduction's last block)
// of about 5 us on B200, against 10-20 us of streaming. MODE 0: dres[j] = (V_j, w);
// MODE 1: w -= sum_j h[j] V_j, then dres[j] = (V_j, w_new); MODE 2: w -= sign sum_j h[j] V_j
// and, with dnorm, ||w_new||. Each thread walks its 16-byte element groups (grid stride,
// the same groups in every mode) and, per group, the basis vectors in batches of
// gs_batch loads issued before their FMAs; its dot accumulators live in shared memory
// (k x blockDim values), so k does not cost registers. MODE 1 reads each vector's group
// again for the dots right after the projection used it: from L1 or L2, not from DRAM, so
// the fused pass streams V once. A thread adds its groups in order, the block adds its
// threads in a fixed tree and the last block adds the blocks in order: MODE 1's dots equal
// MODE 2 (sign 1) followed by MODE 0 bit for bit, and reruns give the same bits.
constexpr int kGsMaxK = 32;
// basis vectors per batch when two element groups share it (2 in the fused mode, which
// keeps both groups of w live across its two passes)
template <int MODE>
__host__ __device__ constexpr int gs_pair() { return MODE == 1 ? 2 : 4; }
// loads in flight per batch: 8 basis groups, 4 in the fused mode (which also keeps w's
// group live across its two passes; 8 there exceeds the 85-register budget)
template <int MODE>
__host__ __device__ constexpr int gs_batch() { return MODE == 1 ? 4 : 8; }

template <typename T>
static size_t gs_smem(int k) { return (size_t)k * kBlock * sizeof(T) + kGsMaxK * sizeof(T); }

template <typename T, int MODE>
__global__ void __launch_bounds__(kBlock, 3)
k_gs(uint32_t n, int k, const T* __restrict__ V, size_t ld, const double* __restrict__ h,
     double sign, T* __restrict__ w, Scratch s, double* dres, double* dnorm, const int* stop)
{
    extern __shared__ __align__(16) unsigned char gs_raw[];
    T* sacc = reinterpret_cast<T*>(gs_raw);           // [k][blockDim]
    T* sh = sacc + (size_t)k * blockDim.x;            // [kGsMaxK] coefficients (sign folded)
    __shared__ bool amLast;
    pdl_wait(); // launched programmatically (gs_launch)
    pdl_release();
    if (stop && *stop) return;
    using VT = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::W;
    constexpr int B = gs_batch<MODE>();
    const uint32_t tid = threadIdx.x, bd = blockDim.x;
    if (MODE >= 1)
        for (int j = tid; j < k; j += bd) sh[j] = (T)(sign * h[j]);
    if (MODE <= 1)
        for (int j = 0; j < k; ++j) sacc[j * bd + tid] = T(0);
    __syncthreads();
    T nrm = T(0);
    auto project = [&](T* wv, auto load) {
        for (int j0 = 0; j0 < k; j0 += B) {
            T vv[B][W];
#pragma unroll
            for (int u = 0; u < B; ++u)
                if (j0 + u < k) load(j0 + u, vv[u]);
#pragma unroll
            for (int u = 0; u < B; ++u)
                if (j0 + u < k)
#pragma unroll
                    for (int e = 0; e < W; ++e) wv[e] = fma(-sh[j0 + u], vv[u][e], wv[e]);
        }
    };
    auto dots = [&](const T* wv, auto load) {
        for (int j0 = 0; j0 < k; j0 += B) {
            T vv[B][W];
#pragma unroll
            for (int u = 0; u < B; ++u)
                if (j0 + u < k) load(j0 + u, vv[u]);
#pragma unroll
            for (int u = 0; u < B; ++u)
                if (j0 + u < k) {
                    T a = sacc[(j0 + u) * bd + tid];
#pragma unroll
                    for (int e = 0; e < W; ++e) a = fma(vv[u][e], wv[e], a);
                    sacc[(j0 + u) * bd + tid] = a;
                }
        }
    };
    // 16-byte groups, two at a time: a thread's groups iv and iv + stride share each batch
    // of gs_pair basis vectors, so twice as many loads are in flight per wait and a thread
    // waits half as often; each dot still adds group iv's elements before group iv +
    // stride's
    constexpr int kGsPair = gs_pair<MODE>();
    const size_t nv = n / W, stride = (size_t)gridDim.x * bd;
    for (size_t iv = (size_t)blockIdx.x * bd + tid; iv < nv; iv += 2 * stride) {
        const int ng = iv + stride < nv ? 2 : 1;
        const size_t ivs[2] = {iv, iv + stride};
        T wv[2][W];
#pragma unroll
        for (int u = 0; u < 2; ++u)
            if (u < ng) *(VT*)wv[u] = ((const VT*)w)[ivs[u]];
        auto batch = [&](int j0, T (&vv)[2][kGsPair][W]) {
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int q = 0; q < kGsPair; ++q)
                    if (u < ng && j0 + q < k)
                        *(VT*)vv[u][q] = ((const VT*)(V + (j0 + q) * ld))[ivs[u]];
        };
        if (MODE >= 1) {
            for (int j0 = 0; j0 < k; j0 += kGsPair) {
                T vv[2][kGsPair][W];
                batch(j0, vv);
#pragma unroll
                for (int u = 0; u < 2; ++u)
#pragma unroll
                    for (int q = 0; q < kGsPair; ++q)
                        if (u < ng && j0 + q < k)
#pragma unroll
                            for (int e = 0; e < W; ++e)
                                wv[u][e] = fma(-sh[j0 + q], vv[u][q][e], wv[u][e]);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u)
                if (u < ng) {
                    ((VT*)w)[ivs[u]] = *(VT*)wv[u];
#pragma unroll
                    for (int e = 0; e < W; ++e) nrm = fma(wv[u][e], wv[u][e], nrm);
                }
        }
        if (MODE <= 1) {
            for (int j0 = 0; j0 < k; j0 += kGsPair) {
                T vv[2][kGsPair][W];
                batch(j0, vv);
#pragma unroll
                for (int q = 0; q < kGsPair; ++q)
                    if (j0 + q < k) {
                        T a = sacc[(j0 + q) * bd + tid];
#pragma unroll
                        for (int u = 0; u < 2; ++u)
                            if (u < ng)
#pragma unroll
                                for (int e = 0; e < W; ++e) a = fma(vv[u][q][e], wv[u][e], a);
                        sacc[(j0 + q) * bd + tid] = a;
                    }
            }
        }
    }
    for (size_t i = nv * W + (size_t)blockIdx.x * bd + tid; i < n; i += (size_t)gridDim.x * bd) {
        auto ld1 = [&](int j, T* out) {
            out[0] = V[j * ld + i];
#pragma unroll
            for (int e = 1; e < W; ++e) out[e] = T(0);
        };
        T wv[W];
        wv[0] = w[i];
#pragma unroll
        for (int e = 1; e < W; ++e) wv[e] = T(0);
        if (MODE >= 1) {
            project(wv, ld1);
            w[i] = wv[0];
            nrm = fma(wv[0], wv[0], nrm);
        }
        if (MODE <= 1) dots(wv, ld1);
    }
    if (MODE == 2) {
        double acc[1] = {(double)nrm};
        const int ops[1] = {kSum};
        if (dnorm) grid_reduce<1>(acc, ops, s, [=] __device__(const double* v) { *dnorm = sqrt(v[0]); });
        return;
    }
    // block partials: warp g adds column j = g, g + warps, ... over the block's threads
    // (lane l sums threads l, l + 32, ... in order, then a shuffle tree)
    __syncthreads();
    const int lane = tid & 31, wid = tid >> 5, nwarp = bd >> 5;
    for (int j = wid; j < k; j += nwarp) {
        double a = 0.0;
        for (uint32_t t = lane; t < bd; t += 32) a += (double)sacc[j * bd + t];
        a = warp_reduce(a, kSum);
        if (lane == 0) s.partials[(size_t)j * gridDim.x + blockIdx.x] = a;
    }
    __syncthreads();
    if (tid == 0) amLast = last_block_ticket(s.ticket);
    __syncthreads();
    if (!amLast) return;
    // the last block: dres[j] = the blocks' partials added in block order (lane l takes
    // blocks l, l + 32, ..., then a shuffle tree)
    for (int j = wid; j < k; j += nwarp) {
        double a = 0.0;
        for (uint32_t b = lane; b < gridDim.x; b += 32)
            a += __ldcg(&s.partials[(size_t)j * gridDim.x + b]);
        a = warp_reduce(a, kSum);
        if (lane == 0) dres[j] = a;
    }
}

// Launches k_gs over the basis in chunks of kGsMaxK vectors. MODE 1 with more than one
// chunk runs as MODE 2 over every chunk, then MODE 0 over every chunk (the projection must
// be complete before any dot).
template <typename T, int MODE>
static int gs_launch(Ctx& c, uint32_t n, int k, const T* V, size_t ld, const double* h,
                     double sign, T* w, double* dres, double* dnorm, const int* stop)
{
    // the shared-memory opt-in above 48 KB, once per device
    static bool attr[64] = {};
    if (c.dev < 0 || c.dev >= 64) return kErrNoDevice;
    if (!attr[c.dev]) {
        FB_CUDA(cudaFuncSetAttribute(k_gs<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)gs_smem<T>(kGsMaxK)));
        attr[c.dev] = true;
    }
    const int g = mgrid(c, n);
    for (int j0 = 0; j0 < k; j0 += kGsMaxK) {
        const int kk = k - j0 < kGsMaxK ? k - j0 : kGsMaxK;
        const bool last = j0 + kGsMaxK >= k;
        ++c.launches;
        FB_CUDA(launch_pdl(k_gs<T, MODE>, dim3((unsigned)g), dim3(kBlock), gs_smem<T>(kk),
                           c.stream, n, kk, V + j0 * ld, ld, h ? h + j0 : nullptr, sign, w,
                           c.red, dres ? dres + j0 : nullptr, last ? dnorm : nullptr, stop));
        FB_CUDA(cudaGetLastError());
    }
    return kOk;
}

template <typename T>
int v_multidot(Ctx& c, uint32_t n, int k, const T* V, size_t ld, const T* w, double* dres,
               const int* stop)
{
    if (vec_ok(V, ld, w))
        return gs_launch<T, 0>(c, n, k, V, ld, nullptr, 1.0, const_cast<T*>(w), dres, nullptr,
                               stop);
    const bool vec = vec_ok(V, ld, w);
    for (int j0 = 0; j0 < k; j0 += KC) {
        const int kk = k - j0 < KC ? k - j0 : KC;
        ++c.launches;
        with_k<KC>(kk, [&](auto KK) {
            constexpr int K = decltype(KK)::value;
            if (vec)
                k_multidot<T, 1, K><<<mgrid(c, n), kBlock, 0, c.stream>>>(
                    n, V + j0 * ld, ld, w, c.red, dres + j0, stop);
            else
                k_multidot<T, 0, K><<<mgrid(c, n), kBlock, 0, c.stream>>>(
                    n, V + j0 * ld, ld, w, c.red, dres + j0, stop);
        });
        FB_CUDA(cudaGetLastError());
    }
    return kOk;
}

template <typename T>
int v_multiaxpy(Ctx& c, uint32_t n, int k, const T* V, size_t ld, const double* h,
                double sign, T* w, double* dnorm, const int* stop)
{
    if (vec_ok(V, ld, (const T*)w))
        return gs_launch<T, 2>(c, n, k, V, ld, h, sign, w, nullptr, dnorm, stop);
    const bool vec = vec_ok(V, ld, (const T*)w);
    for (int j0 = 0; j0 < k; j0 += KC) {
        const int kk = k - j0 < KC ? k - j0 : KC;
        const bool last = j0 + KC >= k;
        ++c.launches;
        with_k<KC>(kk, [&](auto KK) {
            constexpr int K = decltype(KK)::value;
            if (vec)
                k_multiaxpy<T, 1, K><<<mgrid(c, n), kBlock, 0, c.stream>>>(
                    n, V + j0 * ld, ld, h + j0, sign, w, c.red, last ? dnorm : nullptr, stop);
            else
                k_multiaxpy<T, 0, K><<<mgrid(c, n), kBlock, 0, c.stream>>>(
                    n, V + j0 * ld, ld, h + j0, sign, w, c.red, last ? dnorm : nullptr, stop);
        });
        FB_CUDA(cudaGetLastError());
    }
    return kOk;
}

template <typename T>
int v_multiaxpy_dot(Ctx& c, uint32_t n, int k, const T* V, size_t ld, const double* h, T* w,
                    double* dres, const int* stop)
{
    if (vec_ok(V, ld, (const T*)w)) {
        if (k <= kGsMaxK)
            return gs_launch<T, 1>(c, n, k, V, ld, h, 1.0, w, dres, nullptr, stop);
        int e = gs_launch<T, 2>(c, n, k, V, ld, h, 1.0, w, nullptr, nullptr, stop);
        return e ? e : gs_launch<T, 0>(c, n, k, V, ld, nullptr, 1.0, w, dres, nullptr, stop);
    }
    if (k > kf<T>()) {
        int e = v_multiaxpy(c, n, k, V, ld, h, 1.0, w, (double*)nullptr, stop);
        return e ? e : v_multidot(c, n, k, V, ld, (const T*)w, dres, stop);
    }
    ++c.launches;
    const bool vec = vec_ok(V, ld, (const T*)w);
    with_k<kf<T>()>(k, [&](auto KK) {
        constexpr int K = decltype(KK)::value;
        if (vec)
            k_multiaxpy_dot<T, 1, K><<<mgrid(c, n), kBlock, 0, c.stream>>>(n, V, ld, h, w, c.red,
                                                                           dres, stop);
        else
            k_multiaxpy_dot<T, 0, K><<<mgrid(c, n), kBlock, 0, c.stream>>>(n, V, ld, h, w, c.red,
                                                                           dres, stop);
    });
    FB_CUDA(cudaGetLastError());
    return kOk;
}

#define FB_VEC_INSTANTIATE(T)                                                              \
    template int v_dot<T>(Ctx&, uint32_t, const T*, const T*, double*);                   \
    template int v_norm2<T>(Ctx&, uint32_t, const T*, double*);                           \
    template int v_norminf<T>(Ctx&, uint32_t, const T*, double*);                         \
    template int v_axpy<T>(Ctx&, uint32_t, Scal, const T*, T*);                           \
    template int v_xpay<T>(Ctx&, uint32_t, Scal, const T*, T*);                           \
    template int v_axpby<T>(Ctx&, uint32_t, Scal, Scal, const T*, T*);                    \
    template int v_waxpby<T>(Ctx&, uint32_t, Scal, const T*, Scal, const T*, T*);         \
    template int v_scale<T>(Ctx&, uint32_t, Scal, T*);                                    \
    template int v_set<T>(Ctx&, uint32_t, double, T*);                                    \
    template int v_copy<T>(Ctx&, uint32_t, const T*, T*);                                 \
    template int v_pmult<T>(Ctx&, uint32_t, const T*, T*);                                \
    template int v_add<T>(Ctx&, uint32_t, const T*, T*);                                  \
    template int v_multidot<T>(Ctx&, uint32_t, int, const T*, size_t, const T*, double*,  \
                               const int*);                                               \
    template int v_multiaxpy<T>(Ctx&, uint32_t, int, const T*, size_t, const double*,     \
                                double, T*, double*, const int*);                         \
    template int v_multiaxpy_dot<T>(Ctx&, uint32_t, int, const T*, size_t, const double*, \
                                    T*, double*, const int*);
FB_VEC_INSTANTIATE(double)
FB_VEC_INSTANTIATE(float)
#undef FB_VEC_INSTANTIATE

} // namespace fb
