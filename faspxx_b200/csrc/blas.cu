// blas.cu -- vector kernels: the VEC operations of FASP++ (src/VEC.cxx) on device memory.
//
// All are bandwidth-bound, grid-stride loops on coalesced 8-byte accesses. Reductions use the
// deterministic two-pass grid reduction of common.cuh and deliver their result to a device
// scalar, so a following kernel can consume it without a host round trip. Sums use FMA and
// a different association than the reference's 4 interleaved partial sums (VEC.cxx:424-485);
// results agree to rounding, not bit for bit.
#include <map>
#include <mutex>

#include "internal.h"

namespace fb {

#define GRID_STRIDE(i, n) \
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)(n); \
         i += (size_t)gridDim.x * blockDim.x)

int resident_grid(const Ctx& c, const void* fn, int block)
{
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(fn, block);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, 0) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 1;
    }
    long long g = (long long)nb * c.nsm;
    if (g > kMaxGrid) g = kMaxGrid;
    cache[key] = (int)g;
    return (int)g;
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

__global__ void k_dot(uint32_t n, const double* __restrict__ a, const double* __restrict__ b,
                      Scratch s, double* dres)
{
    double acc[1] = {0.0};
    const int ops[1] = {kSum};
    GRID_STRIDE(i, n) acc[0] = fma(a[i], b[i], acc[0]);
    grid_reduce<1>(acc, ops, s, [=] __device__(const double* t) { *dres = t[0]; });
}

__global__ void k_norm2(uint32_t n, const double* __restrict__ a, Scratch s, double* dres)
{
    double acc[1] = {0.0};
    const int ops[1] = {kSum};
    GRID_STRIDE(i, n) acc[0] = fma(a[i], a[i], acc[0]);
    grid_reduce<1>(acc, ops, s, [=] __device__(const double* t) { *dres = sqrt(t[0]); });
}

__global__ void k_norminf(uint32_t n, const double* __restrict__ a, Scratch s, double* dres)
{
    double acc[1] = {0.0};
    const int ops[1] = {kMax};
    GRID_STRIDE(i, n) acc[0] = fmax(acc[0], fabs(a[i]));
    grid_reduce<1>(acc, ops, s, [=] __device__(const double* t) { *dres = t[0]; });
}

int v_dot(Ctx& c, uint32_t n, const double* a, const double* b, double* dres)
{
    ++c.launches;
    k_dot<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(n, a, b, c.red, dres);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

int v_norm2(Ctx& c, uint32_t n, const double* a, double* dres)
{
    ++c.launches;
    k_norm2<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(n, a, c.red, dres);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

int v_norminf(Ctx& c, uint32_t n, const double* a, double* dres)
{
    ++c.launches;
    k_norminf<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(n, a, c.red, dres);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

// ---- updates ---------------------------------------------------------------------------

__global__ void k_axpy(uint32_t n, Scal a, const double* __restrict__ x, double* __restrict__ y)
{
    const double av = eval(a);
    GRID_STRIDE(i, n) y[i] = fma(av, x[i], y[i]);
}

__global__ void k_xpay(uint32_t n, Scal a, const double* __restrict__ x, double* __restrict__ y)
{
    const double av = eval(a);
    GRID_STRIDE(i, n) y[i] = fma(av, y[i], x[i]);
}

__global__ void k_axpby(uint32_t n, Scal a, Scal b, const double* __restrict__ y,
                        double* __restrict__ x)
{
    const double av = eval(a), bv = eval(b);
    GRID_STRIDE(i, n) x[i] = fma(av, x[i], bv * y[i]);
}

__global__ void k_waxpby(uint32_t n, Scal a, const double* __restrict__ v1, Scal b,
                         const double* __restrict__ v2, double* __restrict__ w)
{
    const double av = eval(a), bv = eval(b);
    GRID_STRIDE(i, n) w[i] = fma(av, v1[i], bv * v2[i]);
}

__global__ void k_scale(uint32_t n, Scal a, double* __restrict__ x)
{
    const double av = eval(a);
    GRID_STRIDE(i, n) x[i] *= av;
}

__global__ void k_set(uint32_t n, double v, double* __restrict__ x)
{
    GRID_STRIDE(i, n) x[i] = v;
}

__global__ void k_pmult(uint32_t n, const double* __restrict__ d, double* __restrict__ x)
{
    GRID_STRIDE(i, n) x[i] *= d[i];
}

__global__ void k_add(uint32_t n, const double* __restrict__ d, double* __restrict__ x)
{
    GRID_STRIDE(i, n) x[i] += d[i];
}

// Jacobi::Setup (src/Iter.cxx:45-47): diagInv = weight * (1 / diag), two roundings as there.
__global__ void k_recip_scale(uint32_t n, double w, const double* __restrict__ d,
                              double* __restrict__ out)
{
    GRID_STRIDE(i, n) out[i] = (1.0 / d[i]) * w;
}

#define LAUNCH_EW(kernel, n, ...)                                                          \
    do {                                                                                   \
        if ((n) == 0) return kOk;                                                          \
        kernel<<<c.grid((n), kBlock), kBlock, 0, c.stream>>>((n), __VA_ARGS__);            \
        ++c.launches;                                                                      \
        FB_CUDA(cudaGetLastError());                                                       \
        return kOk;                                                                        \
    } while (0)

int v_axpy(Ctx& c, uint32_t n, Scal a, const double* x, double* y) { LAUNCH_EW(k_axpy, n, a, x, y); }
int v_xpay(Ctx& c, uint32_t n, Scal a, const double* x, double* y) { LAUNCH_EW(k_xpay, n, a, x, y); }
int v_axpby(Ctx& c, uint32_t n, Scal a, Scal b, const double* y, double* x)
{
    LAUNCH_EW(k_axpby, n, a, b, y, x);
}
int v_waxpby(Ctx& c, uint32_t n, Scal a, const double* v1, Scal b, const double* v2, double* w)
{
    LAUNCH_EW(k_waxpby, n, a, v1, b, v2, w);
}
int v_scale(Ctx& c, uint32_t n, Scal a, double* x) { LAUNCH_EW(k_scale, n, a, x); }
int v_set(Ctx& c, uint32_t n, double v, double* x) { LAUNCH_EW(k_set, n, v, x); }
int v_pmult(Ctx& c, uint32_t n, const double* d, double* x) { LAUNCH_EW(k_pmult, n, d, x); }
int v_add(Ctx& c, uint32_t n, const double* d, double* x) { LAUNCH_EW(k_add, n, d, x); }
int v_recip_scale(Ctx& c, uint32_t n, double w, const double* d, double* out)
{
    LAUNCH_EW(k_recip_scale, n, w, d, out);
}

int v_copy(Ctx& c, uint32_t n, const double* src, double* dst)
{
    if (n == 0 || src == dst) return kOk;
    FB_CUDA(cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice,
                            c.stream));
    return kOk;
}

// ---- classical Gram-Schmidt building blocks ------------------------------------------
// V holds basis vectors at V + j*ld. KC vectors are handled per launch.

constexpr int KC = 8;

// dres[j] = (V_j, w), j in [j0, j0+k)
__global__ void k_multidot(uint32_t n, int k, const double* __restrict__ V, size_t ld,
                           const double* __restrict__ w, Scratch s, double* dres)
{
    double acc[KC];
    int ops[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) {
        acc[j] = 0.0;
        ops[j] = kSum;
    }
    GRID_STRIDE(i, n)
    {
        const double wi = w[i];
#pragma unroll
        for (int j = 0; j < KC; ++j)
            if (j < k) acc[j] = fma(V[j * ld + i], wi, acc[j]);
    }
    grid_reduce<KC>(acc, ops, s, [=] __device__(const double* t) {
        for (int j = 0; j < k; ++j) dres[j] = t[j];
    });
}

// w -= sign * sum_j h[j] V_j; with dnorm != null also ||w_new|| -> *dnorm.
__global__ void k_multiaxpy(uint32_t n, int k, const double* __restrict__ V, size_t ld,
                            const double* __restrict__ h, double sign, double* __restrict__ w,
                            Scratch s, double* dnorm)
{
    double hj[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) hj[j] = j < k ? sign * h[j] : 0.0;
    double acc[1] = {0.0};
    const int ops[1] = {kSum};
    GRID_STRIDE(i, n)
    {
        double wi = w[i];
#pragma unroll
        for (int j = 0; j < KC; ++j)
            if (j < k) wi = fma(-hj[j], V[j * ld + i], wi);
        w[i] = wi;
        acc[0] = fma(wi, wi, acc[0]);
    }
    if (dnorm) grid_reduce<1>(acc, ops, s, [=] __device__(const double* t) { *dnorm = sqrt(t[0]); });
}

int v_multidot(Ctx& c, uint32_t n, int k, const double* V, size_t ld, const double* w,
               double* dres)
{
    for (int j0 = 0; j0 < k; j0 += KC) {
        const int kk = k - j0 < KC ? k - j0 : KC;
        ++c.launches;
    k_multidot<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(n, kk, V + j0 * ld, ld, w, c.red,
                                                                 dres + j0);
        FB_CUDA(cudaGetLastError());
    }
    return kOk;
}

int v_multiaxpy(Ctx& c, uint32_t n, int k, const double* V, size_t ld, const double* h,
                double sign, double* w, double* dnorm)
{
    for (int j0 = 0; j0 < k; j0 += KC) {
        const int kk = k - j0 < KC ? k - j0 : KC;
        const bool last = j0 + KC >= k;
        ++c.launches;
    k_multiaxpy<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(
            n, kk, V + j0 * ld, ld, h + j0, sign, w, c.red, last ? dnorm : nullptr);
        FB_CUDA(cudaGetLastError());
    }
    return kOk;
}

} // namespace fb
