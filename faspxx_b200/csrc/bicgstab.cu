// bicgstab.cu -- kernels and engine of the device-driven BiCGStab (see bicgstab.cuh).
//
// The scalar part of BiCGStab::Solve runs on one thread at the end of each fused kernel's
// deterministic grid reduction, on the control block in device memory. The branches that need
// vector work the four kernels do not do -- the safe-guard copy (BiCGStab.cxx:133), the
// stagnation check with its true residual and restart (:141-162) and the false-convergence
// check (:164-175) -- set status = kEsc; the host finishes them and relaunches bi_resume.
// Operand order of every update follows the reference's VEC calls (WAXPBY is
// fma(a, v1, b * v2), XPAY with a = 1 is fma(1, y, x)), and a Jacobi sweep from zero is
// diagInv .* v, which is what Jacobi::Solve computes from a zero guess.
#include <cstring>
#include <utility>

#include "bicgstab.cuh"

namespace fb {

#define GRID_STRIDE(i, n) \
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)(n); \
         i += (size_t)gridDim.x * blockDim.x)

__device__ __forceinline__ void bi_rec(BiCtl* c, unsigned k, double v)
{
    const unsigned g = k + c->histOffset;
    if (c->hist && g < c->histCap) c->hist[g] = v * c->histScale;
}

__device__ __forceinline__ void bi_done(BiCtl* c, int code)
{
    c->code = code;
    c->status = kDone;
}

__device__ __forceinline__ void bi_esc(BiCtl* c, int reason, int phase, const double* red)
{
    for (int k = 0; k < 5; ++k) c->red[k] = red[k];
    c->reason = reason;
    c->phase = phase;
    c->status = kEsc;
}

// Loop top (BiCGStab.cxx:79-87), ++numIter, rjr0star and alpha (:88-102).
// t = {(ptmp, r0*), (rj, r0*), (rj, rj)}.
__device__ void bi_after_p(BiCtl* c, const double* t)
{
    if (c->numIter >= c->maxIter) {
        bi_done(c, c->code);
        return;
    }
    if (c->numIter == c->minIter) {
        const double resAbs = sqrt(t[2]);
        c->resAbs = resAbs;
        c->denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;
        c->resRel = resAbs / c->denAbs;
        bi_rec(c, c->numIter, resAbs);
        if (c->resRel < c->relTol || resAbs < c->absTol) {
            bi_done(c, c->code);
            return;
        }
    }
    c->numIter += 1;
    c->rjr0star = t[1];
    c->tmp12 = t[0];
    if (fabs(t[0]) > 1e-40) {
        c->alpha = c->rjr0star / t[0];
    } else {
        bi_rec(c, c->numIter, c->resAbs);
        bi_done(c, kErrDivZero);
    }
}

// The checks after the update (BiCGStab.cxx:117-175) from `phase` on, then beta (:177-183).
// red = {(r,r), (r,r0*), max|x|, (p,p), (x,x)}.
__device__ void bi_checks(BiCtl* c, const double* red, int phase)
{
    bool stop = false;
    if (c->numIter >= c->minIter) {
        if (phase <= 0) {
            c->resAbs = sqrt(red[0]);
            c->resRel = c->resAbs / c->denAbs;
            c->ratio = c->resAbs / c->resAbsOld;
            if (c->numIter >= c->savIter && c->resAbs < c->resAbsOld) {
                bi_esc(c, kBiSave, 1, red);
                return;
            }
            if (c->reliable) { // the host folds x and recomputes r in FP64, then phase 3
                if (c->resAbs > c->rmax) c->rmax = c->resAbs;
                if (c->resAbs < c->delta * c->rmax) {
                    bi_esc(c, kBiRefresh, 3, red);
                    return;
                }
            }
        }
        if (phase <= 1 && c->ratio > kKsmChkRatio && c->numIter > c->minIter) {
            if (red[2] < c->solStagTol) {
                c->code = kErrSolStag;
                stop = true;
            } else {
                const double xRelDiff = fabs(c->alpha) * sqrt(red[3]) / sqrt(red[4]);
                if (c->stagStep <= kMaxStagNum && xRelDiff < c->solStagTol) {
                    bi_esc(c, kBiStag, 2, red);
                    return;
                }
            }
        }
        if (phase <= 2 && !stop && c->resRel < c->relTol) {
            bi_esc(c, kBiCheck, 3, red);
            return;
        }
        bi_rec(c, c->numIter, c->resAbs);
        if (stop) {
            bi_done(c, c->code);
            return;
        }
    }
    if (c->numIter < c->maxIter) {
        c->resAbsOld = c->resAbs;
        c->rjr0startmp = c->rjr0star;
        c->rjr0star = red[1];
        c->beta = c->rjr0star / c->rjr0startmp * c->alpha / c->omega;
    } else {
        bi_done(c, c->code);
    }
}

// pj = rj + beta (pj_old - omega ptmp_old) (BiCGStab.cxx:184-185, the previous iteration's
// direction update, formed for every gathered entry in the reference's operand order:
// tmp = fma(1, pj, -omega ptmp), pj = fma(1, rj, beta tmp)) and ptmp = D (A pj) with the
// loop-top sums; pj and ptmp of the owned rows go to the
// other buffer of each pair, and the finalize flips c->par to it. SH = 5 or 7: stencil
// masks of that fixed shape, 16-byte row groups per thread (stencil_group; each row's
// product is the same bits, the partial sums group the rows by W). JAC = 2 (reliable
// updates on a matrix whose diagonal varies): ptmp = A (D pj), the right-preconditioned
// product, so that the recursive residual stays b - A x (the reference's order keeps it so
// only when D commutes with A).
template <typename T, int L, int JAC, int SH = 0>
__global__ void __launch_bounds__(kBlock) bi_p(CSRView<T> A, T* __restrict__ p0,
                                               T* __restrict__ p1, T* __restrict__ t0,
                                               T* __restrict__ t1, const T* __restrict__ rj,
                                               const T* __restrict__ r0s,
                                               const T* __restrict__ dinv, BiCtl* c, Scratch s)
{
    pdl_wait();
    pdl_release();
    if (c->status != kRun) return;
    static_assert(SH == 0 || JAC != 2, "right preconditioning runs the row kernels");
    const int par = c->par;
    const T* __restrict__ pOld = par ? p1 : p0;
    const T* __restrict__ tOld = par ? t1 : t0;
    T* __restrict__ pNew = par ? p0 : p1;
    T* __restrict__ tNew = par ? t0 : t1;
    const T beta = (T)c->beta, nomega = (T)(-c->omega);
    auto pat = [&](size_t j) { // the updated pj at j
        const T tmp = fma(T(1), pOld[j], nomega * tOld[j]);
        return fma(T(1), rj[j], beta * tmp);
    };
    T a0 = 0, a1 = 0, a2 = 0;
    auto own = [&](size_t row, T ap) {
        const T pt = JAC == 1 ? ap * dinv[row] : ap;
        tNew[row] = pt;
        const T r = rj[row], r0 = r0s[row];
        a0 = fma(pt, r0, a0);
        a1 = fma(r, r0, a1);
        a2 = fma(r, r, a2);
    };
    auto xv = [&](uint32_t j) { return JAC == 2 ? pat(j) * dinv[j] : pat(j); };
    if constexpr (SH != 0) {
        using VT = Vec16<T>;
        using V = typename VT::V;
        constexpr int W = VT::W;
        const uint32_t nw = A.nrow / W, stride = gridDim.x * blockDim.x;
        const V* rv = reinterpret_cast<const V*>(rj);
        const V* pv = reinterpret_cast<const V*>(pOld);
        const V* tv = reinterpret_cast<const V*>(tOld);
        auto pg = [&](uint32_t h) { // pj at group h
            const V r = rv[h], p = pv[h], t = tv[h];
            T e[W];
#pragma unroll
            for (int j = 0; j < W; ++j) {
                const T tmp = fma(T(1), VT::at(p, j), nomega * VT::at(t, j));
                e[j] = fma(T(1), VT::at(r, j), beta * tmp);
            }
            return VT::make(e);
        };
        for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g - (threadIdx.x & 31u) < nw;
             g += stride) {
            const bool act = g < nw;
            T sm[W];
#pragma unroll
            for (int j = 0; j < W; ++j) sm[j] = T(0);
            V cg;
            stencil_group<T, SH>(A, g, nw, act, pg, cg, sm);
            if (act) {
                reinterpret_cast<V*>(pNew)[g] = cg; // the group's own pj
#pragma unroll
                for (int j = 0; j < W; ++j) own((size_t)W * g + j, sm[j]);
            }
        }
    } else if (L == 1) {
        for (size_t row = (size_t)blockIdx.x * blockDim.x + threadIdx.x; row < A.nrow;
             row += (size_t)gridDim.x * blockDim.x) {
            pNew[row] = pat(row);
            own(row, row_apply<T, false>(A, row, xv));
        }
    } else {
        const int lane = threadIdx.x & (L - 1);
        const size_t warpRows = 32 / L;
        const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
        const size_t sub = (threadIdx.x & 31) / L;
        for (size_t base = gw * warpRows; base < A.nrow; base += nwarps * warpRows) {
            const size_t row = base + sub;
            T sum = T(0);
            if (row < A.nrow)
                for (uint32_t k = A.rowPtr[row] + lane; k < A.rowPtr[row + 1]; k += L)
                    sum = fma(A.val[k], xv(A.colInd[k]), sum);
            sum = group_sum<L>(sum);
            if (lane == 0 && row < A.nrow) {
                pNew[row] = pat(row);
                own(row, sum);
            }
        }
    }
    double a[3] = {(double)a0, (double)a1, (double)a2};
    const int ops[3] = {kSum, kSum, kSum};
    grid_reduce_ctl<3>(a, ops, s, c, [=] __device__(BiCtl* cs, const double* t) {
        if (cs->bench) return;
        cs->par ^= 1;
        bi_after_p(cs, t);
    });
}

// sj = rj - alpha ptmp (on the fly for the gathers, stored for the owned rows),
// stmp = D (A sj), omega = (stmp, sj) / (stmp, stmp)  (BiCGStab.cxx:103-113). SH as bi_p,
// with sj's groups formed from rj and ptmp by the same FMA.
template <typename T, int L, int JAC, int SH = 0>
__global__ void __launch_bounds__(kBlock) bi_s(CSRView<T> A, const T* __restrict__ rj,
                                               const T* __restrict__ t0,
                                               const T* __restrict__ t1,
                                               const T* __restrict__ dinv, T* __restrict__ sj,
                                               T* __restrict__ stmp, BiCtl* c, Scratch s)
{
    pdl_wait();
    pdl_release();
    if (c->status != kRun) return;
    const T* __restrict__ ptmp = c->par ? t1 : t0;
    static_assert(SH == 0 || JAC != 2, "right preconditioning runs the row kernels");
    const T nalpha = (T)(-c->alpha);
    auto sv = [&](uint32_t j) { return fma(T(1), rj[j], nalpha * ptmp[j]); };
    auto gv = [&](uint32_t j) { return JAC == 2 ? sv(j) * dinv[j] : sv(j); };
    T a0 = 0, a1 = 0;
    auto own = [&](size_t row, T as) {
        const T sjv = sv((uint32_t)row);
        sj[row] = sjv;
        const T st = JAC == 1 ? as * dinv[row] : as;
        stmp[row] = st;
        a0 = fma(st, sjv, a0);
        a1 = fma(st, st, a1);
    };
    if constexpr (SH != 0) {
        using VT = Vec16<T>;
        using V = typename VT::V;
        constexpr int W = VT::W;
        const uint32_t nw = A.nrow / W, stride = gridDim.x * blockDim.x;
        const V* rv = reinterpret_cast<const V*>(rj);
        const V* tv = reinterpret_cast<const V*>(ptmp);
        auto sg = [&](uint32_t h) { // sj at group h
            const V r = rv[h], t = tv[h];
            T e[W];
#pragma unroll
            for (int j = 0; j < W; ++j) e[j] = fma(T(1), VT::at(r, j), nalpha * VT::at(t, j));
            return VT::make(e);
        };
        for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g - (threadIdx.x & 31u) < nw;
             g += stride) {
            const bool act = g < nw;
            T sm[W];
#pragma unroll
            for (int j = 0; j < W; ++j) sm[j] = T(0);
            V c;
            stencil_group<T, SH>(A, g, nw, act, sg, c, sm);
            if (act)
#pragma unroll
                for (int j = 0; j < W; ++j) own((size_t)W * g + j, sm[j]);
        }
    } else if (L == 1) {
        for (size_t row = (size_t)blockIdx.x * blockDim.x + threadIdx.x; row < A.nrow;
             row += (size_t)gridDim.x * blockDim.x)
            own(row, row_apply<T, false>(A, row, gv));
    } else {
        const int lane = threadIdx.x & (L - 1);
        const size_t warpRows = 32 / L;
        const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
        const size_t sub = (threadIdx.x & 31) / L;
        for (size_t base = gw * warpRows; base < A.nrow; base += nwarps * warpRows) {
            const size_t row = base + sub;
            T sum = T(0);
            if (row < A.nrow)
                for (uint32_t k = A.rowPtr[row] + lane; k < A.rowPtr[row + 1]; k += L)
                    sum = fma(A.val[k], gv(A.colInd[k]), sum);
            sum = group_sum<L>(sum);
            if (lane == 0 && row < A.nrow) own(row, sum);
        }
    }
    double a[2] = {(double)a0, (double)a1};
    const int ops[2] = {kSum, kSum};
    grid_reduce_ctl<2>(a, ops, s, c, [=] __device__(BiCtl* cs, const double* t) {
        if (!cs->bench) cs->omega = t[0] / t[1];
    });
}

// x += alpha D pj + omega D sj, rj = sj - omega stmp, then the checks (BiCGStab.cxx:114-183).
// VEC: every vector is read and written in 16-byte groups (2 FP64 / 4 FP32 elements), so a
// thread keeps six 16-byte loads in flight per step instead of six scalar ones; the few
// elements past the last full group go one at a time.
template <typename T>
struct BiXSums {
    T rr = 0, rr0 = 0, xm = 0, pp = 0, xx = 0;
};

template <typename T, int JAC>
__device__ __forceinline__ void bi_x_elem(T alpha, T omega, T nomega, T p, T sv, T d, T& xi,
                                          T st, T r0, T& r, BiXSums<T>& a)
{
    const T mp = JAC ? p * d : p;
    const T ms = JAC ? sv * d : sv;
    const T tmp = fma(alpha, mp, omega * ms);
    xi = fma(T(1), xi, tmp);
    r = fma(T(1), sv, nomega * st);
    a.rr = fma(r, r, a.rr);
    a.rr0 = fma(r, r0, a.rr0);
    a.xm = fmax(a.xm, fabs(xi));
    a.pp = fma(p, p, a.pp);
    a.xx = fma(xi, xi, a.xx);
}

template <typename T, int JAC, int VEC>
__global__ void __launch_bounds__(kBlock) bi_x(uint32_t n, T* __restrict__ x, T* __restrict__ rj,
                                               const T* __restrict__ p0,
                                               const T* __restrict__ p1,
                                               const T* __restrict__ sj,
                                               const T* __restrict__ stmp,
                                               const T* __restrict__ r0s,
                                               const T* __restrict__ dinv, BiCtl* c, Scratch s)
{
    pdl_wait();
    pdl_release();
    if (c->status != kRun) return;
    const T* __restrict__ pj = c->par ? p1 : p0;
    const T alpha = (T)c->alpha, omega = (T)c->omega, nomega = (T)(-c->omega);
    BiXSums<T> a;
    uint32_t i0 = 0;
    if (VEC) {
        using VT = typename Vec16<T>::type;
        constexpr int W = Vec16<T>::W;
        const uint32_t nv = n / W;
        GRID_STRIDE(iv, nv)
        {
            T p[W], sv[W], d[W], xi[W], st[W], r0[W], r[W];
            *(VT*)p = ((const VT*)pj)[iv];
            *(VT*)sv = ((const VT*)sj)[iv];
            if (JAC) *(VT*)d = ((const VT*)dinv)[iv];
            *(VT*)xi = ((const VT*)x)[iv];
            *(VT*)st = ((const VT*)stmp)[iv];
            *(VT*)r0 = ((const VT*)r0s)[iv];
#pragma unroll
            for (int e = 0; e < W; ++e)
                bi_x_elem<T, JAC>(alpha, omega, nomega, p[e], sv[e], JAC ? d[e] : T(1), xi[e],
                                  st[e], r0[e], r[e], a);
            ((VT*)x)[iv] = *(VT*)xi;
            ((VT*)rj)[iv] = *(VT*)r;
        }
        i0 = nv * W;
    }
    for (uint32_t i = i0 + blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        T xi = x[i], r;
        bi_x_elem<T, JAC>(alpha, omega, nomega, pj[i], sj[i], JAC ? dinv[i] : T(1), xi, stmp[i],
                          r0s[i], r, a);
        x[i] = xi;
        rj[i] = r;
    }
    double red[5] = {(double)a.rr, (double)a.rr0, (double)a.xm, (double)a.pp, (double)a.xx};
    const int ops[5] = {kSum, kSum, kMax, kSum, kSum};
    grid_reduce_ctl<5>(red, ops, s, c, [=] __device__(BiCtl* cs, const double* t) {
        if (!cs->bench) bi_checks(cs, t, 0);
    });
}

// After the host finished an escalated branch (rj may have been recomputed and pj zeroed):
// the two sums of rj, then the checks continue at c->phase.
template <typename T>
__global__ void __launch_bounds__(kBlock) bi_resume(uint32_t n, const T* __restrict__ rj,
                                                    const T* __restrict__ r0s, BiCtl* c,
                                                    Scratch s)
{
    T rr = 0, rr0 = 0;
    GRID_STRIDE(i, n)
    {
        rr = fma(rj[i], rj[i], rr);
        rr0 = fma(rj[i], r0s[i], rr0);
    }
    double a[2] = {(double)rr, (double)rr0};
    const int ops[2] = {kSum, kSum};
    grid_reduce_ctl<2>(a, ops, s, c, [=] __device__(BiCtl* cs, const double* t) {
        const double red[5] = {t[0], t[1], cs->red[2], cs->red[3], cs->red[4]};
        cs->status = kRun;
        cs->reason = kBiNone;
        bi_checks(cs, red, cs->phase);
    });
}

// ---- engine ------------------------------------------------------------------------------

template <typename T>
static CSRView<T> bi_view(const Mat& A);
template <>
CSRView<double> bi_view<double>(const Mat& A) { return A.v64(); }
template <>
CSRView<float> bi_view<float>(const Mat& A) { return A.v32(); }

// A launch that may overlap the previous kernel's tail (programmatic dependent launch): the
// kernels wait for it to complete (pdl_wait) before their first memory access.
template <typename... P, typename... A>
static void bi_launch(void (*kern)(P...), int grid, cudaStream_t s, bool pdl, A&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kBlock);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

template <typename T>
int BiEngine<T>::launch_iter()
{
    const CSRView<T> V = bi_view<T>(*A);
    const int L = A->lanes;
    const long long rows = (long long)n * L;
    const int needS = c->grid(rows, kBlock);
    const int needV = c->grid(n, kBlock);
    auto fit = [&](const void* k, int need) { return std::min(need, resident_grid(*c, k, kBlock)); };
    T *p0 = pj2[0], *p1 = pj2[1], *t0 = ptmp2[0], *t1 = ptmp2[1];
#define BI_SPMV(KP, KS, LL, JJ)                                                            \
    do {                                                                                   \
        bi_launch(KP<T, LL, JJ>, fit((const void*)KP<T, LL, JJ>, needS), c->stream, pdl, V,  \
                  p0, p1, t0, t1, (const T*)rj, (const T*)r0s, dinv, ctl, c->red);          \
        bi_launch(KS<T, LL, JJ>, fit((const void*)KS<T, LL, JJ>, needS), c->stream, pdl, V,  \
                  (const T*)rj, (const T*)t0, (const T*)t1, dinv, sj, stmp, ctl, c->red);   \
    } while (0)
    // 16-byte row groups on 5- and 7-point stencil masks (bi_p / bi_s with SH)
    auto al16 = [](const void* q) { return ((uintptr_t)q & 15) == 0; };
    const int sh = L == 1 && al16(p1) && al16(t1) && al16(r0s) && al16(sj) && al16(stmp)
                       ? stencil_vec_shape(V, p0, rj, t0)
                       : 0;
#define BI_SPMV_SH(JJ, SS)                                                                 \
    do {                                                                                   \
        bi_launch(bi_p<T, 1, JJ, SS>, fit((const void*)bi_p<T, 1, JJ, SS>, needV),         \
                  c->stream, pdl, V, p0, p1, t0, t1, (const T*)rj, (const T*)r0s, dinv, ctl, \
                  c->red);                                                                 \
        bi_launch(bi_s<T, 1, JJ, SS>, fit((const void*)bi_s<T, 1, JJ, SS>, needV),         \
                  c->stream, pdl, V, (const T*)rj, (const T*)t0, (const T*)t1, dinv, sj,    \
                  stmp, ctl, c->red);                                                      \
    } while (0)
#define BI_LANES(JJ)                                                                       \
    switch (sh ? -sh : L) {                                                                \
        case -5: BI_SPMV_SH(JJ, 5); break;                                                 \
        case -7: BI_SPMV_SH(JJ, 7); break;                                                 \
        case 1: BI_SPMV(bi_p, bi_s, 1, JJ); break;                                         \
        case 2: BI_SPMV(bi_p, bi_s, 2, JJ); break;                                         \
        case 4: BI_SPMV(bi_p, bi_s, 4, JJ); break;                                         \
        case 8: BI_SPMV(bi_p, bi_s, 8, JJ); break;                                         \
        case 16: BI_SPMV(bi_p, bi_s, 16, JJ); break;                                       \
        default: BI_SPMV(bi_p, bi_s, 32, JJ); break;                                       \
    }
    // 16-byte groups when every vector bi_x touches starts on a 16-byte boundary
    const bool vx = (((uintptr_t)x | (uintptr_t)rj | (uintptr_t)p0 | (uintptr_t)p1 |
                      (uintptr_t)sj | (uintptr_t)stmp | (uintptr_t)r0s |
                      (uintptr_t)(jacobi ? dinv : p0)) & 15) == 0;
    auto launch_x = [&](auto kern) {
        bi_launch(kern, fit((const void*)kern, needV), c->stream, pdl, n, x, rj, (const T*)p0,
                  (const T*)p1, (const T*)sj, (const T*)stmp, (const T*)r0s, dinv, ctl, c->red);
    };
    if (jacobi && rightPcd) { // A (D v): the row kernels (no stencil groups)
        switch (L) {
            case 1: BI_SPMV(bi_p, bi_s, 1, 2); break;
            case 2: BI_SPMV(bi_p, bi_s, 2, 2); break;
            case 4: BI_SPMV(bi_p, bi_s, 4, 2); break;
            case 8: BI_SPMV(bi_p, bi_s, 8, 2); break;
            case 16: BI_SPMV(bi_p, bi_s, 16, 2); break;
            default: BI_SPMV(bi_p, bi_s, 32, 2); break;
        }
        if (vx)
            launch_x(bi_x<T, 1, 1>);
        else
            launch_x(bi_x<T, 1, 0>);
    } else if (jacobi) {
        BI_LANES(1)
        if (vx)
            launch_x(bi_x<T, 1, 1>);
        else
            launch_x(bi_x<T, 1, 0>);
    } else {
        BI_LANES(0)
        if (vx)
            launch_x(bi_x<T, 0, 1>);
        else
            launch_x(bi_x<T, 0, 0>);
    }
#undef BI_LANES
#undef BI_SPMV_SH
#undef BI_SPMV
    if (!capturing) c->launches += 3;
    FB_CUDA(cudaGetLastError());
    return kOk;
}

// The checks resume at c->phase and end with beta; the direction update of the same
// iteration (BiCGStab.cxx:184-185, after every branch of the checks, a restart's pj = 0
// included) is the next bi_p's, which forms it from whatever the host left in pj(par).
template <typename T>
int BiEngine<T>::launch_resume()
{
    ++c->launches;
    bi_resume<T><<<c->grid(n, kBlock), kBlock, 0, c->stream>>>(n, rj, r0s, ctl, c->red);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int BiEngine<T>::push_ctl()
{
    FB_CUDA(cudaMemcpyAsync(ctl, hctl, sizeof(BiCtl), cudaMemcpyHostToDevice, c->stream));
    return kOk;
}

template <typename T>
int BiEngine<T>::pull_ctl()
{
    FB_CUDA(cudaMemcpyAsync(hctl, ctl, sizeof(BiCtl), cudaMemcpyDeviceToHost, c->stream));
    FB_CUDA(cudaStreamSynchronize(c->stream));
    return kOk;
}

template <typename T>
int BiEngine<T>::init(Ctx* ctx, const Mat* M, int jac, const T* dinvv, bool graph)
{
    c = ctx;
    A = M;
    n = M->nrow;
    jacobi = jac;
    dinv = dinvv;
    useGraph = graph;
    const size_t bytes = ((size_t)n + 4) * sizeof(T);
    T** vecs[] = {&x, &rj, &r0s, &pj2[0], &pj2[1], &ptmp2[0], &ptmp2[1], &sj, &stmp};
    for (T** v : vecs)
        if (cudaMalloc(v, bytes) != cudaSuccess) {
            cudaGetLastError();
            destroy();
            return kErrAlloc;
        }
    if (cudaMalloc(&ctl, sizeof(BiCtl)) || cudaMallocHost(&hctl, sizeof(BiCtl)) ||
        cudaMallocHost(&hstatus, sizeof(int))) {
        cudaGetLastError();
        destroy();
        return kErrAlloc;
    }
    std::memset(hctl, 0, sizeof(BiCtl));
    hctl->histScale = 1.0;
    if (useGraph) {
        cudaGraph_t g;
        FB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        capturing = true;
        for (int i = 0; i < itersPerGraph; ++i) launch_iter();
        capturing = false;
        cudaMemcpyAsync(hstatus, &ctl->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
        FB_CUDA(cudaStreamEndCapture(c->stream, &g));
        FB_CUDA(cudaGraphInstantiate(&gexec, g, 0));
        cudaGraphDestroy(g);
    }
    return kOk;
}

template <typename T>
void BiEngine<T>::destroy()
{
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    T** vecs[] = {&x, &rj, &r0s, &pj2[0], &pj2[1], &ptmp2[0], &ptmp2[1], &sj, &stmp};
    for (T** v : vecs) {
        cudaFree(*v);
        *v = nullptr;
    }
    cudaFree(ctl);
    ctl = nullptr;
    if (hctl) cudaFreeHost(hctl);
    if (hstatus) cudaFreeHost(hstatus);
    hctl = nullptr;
    hstatus = nullptr;
}

// Two graph launches in flight; after each completes its status word says whether to go on.
template <typename T>
int BiEngine<T>::run(unsigned* launches)
{
    if (!useGraph) {
        for (;;) {
            for (int i = 0; i < itersPerGraph; ++i) {
                int e = launch_iter();
                if (e) return e;
            }
            FB_CUDA(cudaMemcpyAsync(hstatus, &ctl->status, sizeof(int), cudaMemcpyDeviceToHost,
                                    c->stream));
            FB_CUDA(cudaStreamSynchronize(c->stream));
            if (launches) *launches += 3 * itersPerGraph;
            if (*hstatus != kRun) return kOk;
        }
    }
    cudaEvent_t ev[2];
    FB_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    FB_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    *hstatus = kRun;
    int cur = 0;
    FB_CUDA(cudaGraphLaunch(gexec, c->stream));
    FB_CUDA(cudaEventRecord(ev[cur], c->stream));
    int err = kOk;
    for (;;) {
        if (cudaGraphLaunch(gexec, c->stream) != cudaSuccess ||
            cudaEventRecord(ev[cur ^ 1], c->stream) != cudaSuccess) {
            err = kErrCuda;
            break;
        }
        if (launches) *launches += 3 * itersPerGraph;
        if (cudaEventSynchronize(ev[cur]) != cudaSuccess) {
            err = kErrCuda;
            break;
        }
        if (*hstatus != kRun) break;
        cur ^= 1;
    }
    if (launches) *launches += 3 * itersPerGraph;
    cudaStreamSynchronize(c->stream);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return err;
}

template struct BiEngine<double>;
template struct BiEngine<float>;

} // namespace fb
