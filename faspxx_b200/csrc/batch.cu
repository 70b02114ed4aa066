// batch.cu -- many independent Jacobi-PCG solves in one persistent launch.
//
// The systems are the diagonal blocks of one CSRx matrix (global row and column indices,
// block k = rows sysRow[k]..sysRow[k+1]); each has nrhs right-hand sides stored right-hand-
// side-major, b[r * N + row]. A fixed grid of blocks pulls work items from an atomic queue
// ordered by decreasing size (longest first balances the tail); one work item is one
// system with all its right-hand sides, so every matrix entry is loaded once for all of
// them. A CUDA block runs CG for its system with block-level reductions only: no grid-wide
// synchronisation, no host round trip, convergence decided on the device. Each iteration
// is two passes over the system's rows:
//   1. q = A p with p = z + beta p_old formed on the fly (double-buffered p), and (q, p);
//   2. x += alpha p, r -= alpha q, z = diagInv .* r, and (r, r), (z, r).
// The CG recurrences are those of CG::Solve (src/CG.cxx:69-234) with x0 = 0 and the
// stopping test ||r|| < relTol ||r0||; right-hand sides converge (and freeze) separately.
// Precision FP64, or FP32 (values, vectors and per-thread sums) inside FP64 refinement:
// r = b - A x in FP64, the FP32 CG solves A e = r / ||r|| to innerTol, x += ||r|| e.
#include <algorithm>
#include <numeric>
#include <vector>

#include "../../include/fasp_b200.h"
#include "internal.h"

namespace fb {

constexpr int kMaxRhs = 4;

template <typename T>
struct BatchArgs {
    uint32_t        count, nrhs, N;
    const uint32_t* sysRow;
    const uint32_t* order;
    const uint32_t* rowPtr;
    const uint32_t* colInd;
    const T*        val;
    const T*        dinv;
    const T*        b;        // rhs-major [nrhs][N]
    T*              x;
    T*              r;
    T*              z;
    T*              p0;
    T*              p1;
    T*              q;
    uint32_t*       iters;    // [count][nrhs], accumulated across calls (refinement)
    double*         resRel;   // [count][nrhs] final relative residual estimate
    double          relTol;
    uint32_t        maxIter;
    unsigned*       queue;
};

template <int NV>
__device__ __forceinline__ void bsum(double (&v)[NV])
{
    int ops[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) ops[k] = kSum;
    block_reduce<NV>(v, ops);
}

// Two 512-thread blocks per SM (at most 64 registers; FP64 with four right-hand sides took
// 97 and ran one block): twice the warps to hide the latency of each pass, measured 124.8
// against 152.5 ms (FP64) on the 4,096-system batch on B200 despite a few spilled registers.
template <typename T, int NR>
__global__ void __launch_bounds__(512, 2) batch_pcg(BatchArgs<T> a)
{
    __shared__ unsigned item;
    __shared__ double sh[3 * kMaxRhs];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item = atomicAdd(a.queue, 1u);
        __syncthreads();
        if (item >= a.count) return;
        const uint32_t sys = a.order[item];
        const uint32_t r0 = a.sysRow[sys], r1 = a.sysRow[sys + 1];
        // start: x = 0, r = b, z = diagInv .* r, (r, r), (z, r)
        double acc[2 * NR];
#pragma unroll
        for (int k = 0; k < 2 * NR; ++k) acc[k] = 0.0;
        for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
            const T d = a.dinv[i];
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                const size_t o = (size_t)k * a.N + i;
                const T bi = a.b[o];
                a.x[o] = T(0);
                a.r[o] = bi;
                a.z[o] = d * bi;
                acc[k] += (double)bi * bi;
                acc[NR + k] += (double)(d * bi) * bi;
            }
        }
        bsum<2 * NR>(acc);
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < 2 * NR; ++k) sh[k] = acc[k];
        __syncthreads();
        double tol[NR], rz[NR], beta[NR];
        bool active[NR];
        int nact = 0;
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            tol[k] = a.relTol * sqrt(sh[k]);
            rz[k] = sh[NR + k];
            beta[k] = 0.0;
            active[k] = sqrt(sh[k]) > tol[k] && sh[k] > 0.0;
            nact += active[k];
        }
        uint32_t it = 0;
        int par = 0;
        double last[NR];
        uint32_t itk[NR]; // each right-hand side's own count: the iteration that stopped it
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            last[k] = 1.0;
            itk[k] = 0;
        }
        while (nact > 0 && it < a.maxIter) {
            ++it;
            const T* pOld = par ? a.p1 : a.p0;
            T* pNew = par ? a.p0 : a.p1;
            // pass 1: q = A p, p formed on the fly; (q, p)
            double pq[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) pq[k] = 0.0;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const uint32_t kb = a.rowPtr[i], ke = a.rowPtr[i + 1];
                T s[NR];
#pragma unroll
                for (int k = 0; k < NR; ++k) s[k] = T(0);
                for (uint32_t e = kb; e < ke; ++e) {
                    const uint32_t j = __ldg(a.colInd + e);
                    const T v = __ldg(a.val + e);
#pragma unroll
                    for (int k = 0; k < NR; ++k) {
                        if (!active[k]) continue;
                        const size_t o = (size_t)k * a.N + j;
                        const T pj = it == 1 ? a.z[o] : fma((T)beta[k], pOld[o], a.z[o]);
                        s[k] = fma(v, pj, s[k]);
                    }
                }
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    if (!active[k]) continue;
                    const size_t o = (size_t)k * a.N + i;
                    const T pi = it == 1 ? a.z[o] : fma((T)beta[k], pOld[o], a.z[o]);
                    pNew[o] = pi;
                    a.q[o] = s[k];
                    pq[k] += (double)s[k] * pi;
                }
            }
            bsum<NR>(pq);
            if (threadIdx.x == 0)
#pragma unroll
                for (int k = 0; k < NR; ++k) sh[k] = pq[k];
            __syncthreads();
            T alpha[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) alpha[k] = active[k] && sh[k] != 0.0 ? (T)(rz[k] / sh[k]) : T(0);
            // pass 2: x += alpha p, r -= alpha q, z = diagInv .* r; (r, r), (z, r)
            double red[2 * NR];
#pragma unroll
            for (int k = 0; k < 2 * NR; ++k) red[k] = 0.0;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const T d = a.dinv[i];
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    if (!active[k]) continue;
                    const size_t o = (size_t)k * a.N + i;
                    const T xi = fma(alpha[k], pNew[o], a.x[o]);
                    const T ri = fma(-alpha[k], a.q[o], a.r[o]);
                    const T zi = d * ri;
                    a.x[o] = xi;
                    a.r[o] = ri;
                    a.z[o] = zi;
                    red[k] += (double)ri * ri;
                    red[NR + k] += (double)zi * ri;
                }
            }
            bsum<2 * NR>(red);
            if (threadIdx.x == 0)
#pragma unroll
                for (int k = 0; k < 2 * NR; ++k) sh[k] = red[k];
            __syncthreads();
            nact = 0;
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                if (!active[k]) continue;
                const double res = sqrt(sh[k]);
                last[k] = res;
                if (res < tol[k] || !(sh[NR + k] == sh[NR + k])) {
                    active[k] = false;
                    itk[k] = it;
                } else {
                    beta[k] = sh[NR + k] / rz[k];
                    rz[k] = sh[NR + k];
                    ++nact;
                }
            }
            par ^= 1;
        }
#pragma unroll
        for (int k = 0; k < NR; ++k)
            if (threadIdx.x == k) {
                a.iters[(size_t)sys * a.nrhs + k] += active[k] ? it : itk[k];
                a.resRel[(size_t)sys * a.nrhs + k] =
                    tol[k] > 0 ? last[k] * a.relTol / tol[k] : 0.0;
            }
    }
}

// Mixed precision with reliable updates, block-local: the CG iterations run in FP32 on the
// system scaled by s = ||b|| (x0 = 0), and whenever a right-hand side's recursive residual
// meets the stop test or has fallen by delta since its last refresh, the block refreshes
// every active right-hand side in FP64 (the block owns the whole system, so this needs only
// __syncthreads): x64 += s x32, x32 = 0, r = b - A x64 in FP64 with the FP64 values, r32 =
// r / s, z32 = diagInv .* r32. The stop test is applied to the FP64 residual; otherwise CG
// goes on with the same p and beta = (z, r)_refreshed / (z, r)_old.
struct BatchRel {
    const double* val64;
    const double* b64;
    double*       x64;
    double        delta;
};

template <int NR>
__global__ void __launch_bounds__(512) batch_pcg_rel(BatchArgs<float> a, BatchRel f)
{
    // per right-hand side scalars, uniform across the block: thread 0 updates them after
    // each block reduction, the others read them after the barrier
    struct Rhs {
        double   rz, rzold, beta, rmax, res, true0, prev, sc, pq;
        float    alpha;
        int      active, fresh, stall, trig;
        unsigned its; // the iteration that stopped this right-hand side
    };
    __shared__ Rhs st[kMaxRhs];
    __shared__ unsigned item;
    __shared__ double sh[3 * kMaxRhs];
    __shared__ int nact, refresh;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item = atomicAdd(a.queue, 1u);
        __syncthreads();
        if (item >= a.count) return;
        const uint32_t sys = a.order[item];
        const uint32_t r0 = a.sysRow[sys], r1 = a.sysRow[sys + 1];
        const size_t N = a.N;
        // ||b|| per right-hand side (FP64), the scale s
        {
            double bb[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) bb[k] = 0.0;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x)
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    const double bi = f.b64[k * N + i];
                    bb[k] = fma(bi, bi, bb[k]);
                }
            bsum<NR>(bb);
            if (threadIdx.x == 0)
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    const double nb = sqrt(bb[k]);
                    st[k].true0 = nb;
                    st[k].prev = nb;
                    st[k].sc = nb > 0.0 ? nb : 1.0;
                    st[k].active = nb > 0.0;
                    st[k].fresh = 1; // the next p is z (first iteration, or after a restart)
                    st[k].stall = 0;
                    st[k].beta = 0.0;
                    st[k].its = 0;
                }
            __syncthreads();
        }
        // start: x = 0, r32 = b / s, z32 = diagInv .* r32, (r,r), (z,r)
        {
            double acc[2 * NR];
#pragma unroll
            for (int k = 0; k < 2 * NR; ++k) acc[k] = 0.0;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const float d = a.dinv[i];
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    const size_t o = k * N + i;
                    f.x64[o] = 0.0;
                    const float ri = (float)(f.b64[o] / st[k].sc);
                    const float zi = d * ri;
                    a.x[o] = 0.0f;
                    a.r[o] = ri;
                    a.z[o] = zi;
                    acc[k] += (double)ri * ri;
                    acc[NR + k] += (double)zi * ri;
                }
            }
            bsum<2 * NR>(acc);
            if (threadIdx.x == 0) {
                int na = 0;
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    st[k].rz = acc[NR + k];
                    st[k].res = sqrt(acc[k]);
                    st[k].rmax = st[k].res;
                    na += st[k].active;
                }
                nact = na;
            }
            __syncthreads();
        }
        uint32_t it = 0;
        int par = 0;
        while (nact > 0 && it < a.maxIter) {
            ++it;
            const float* pOld = par ? a.p1 : a.p0;
            float* pNew = par ? a.p0 : a.p1;
            int act[NR], fr[NR];
            float bt[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                act[k] = st[k].active;
                fr[k] = st[k].fresh;
                bt[k] = (float)st[k].beta;
            }
            // pass 1: q = A p with p = z + beta p_old on the fly, (q, p)
            double pq[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) pq[k] = 0.0;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const uint32_t kb = a.rowPtr[i], ke = a.rowPtr[i + 1];
                float s[NR];
#pragma unroll
                for (int k = 0; k < NR; ++k) s[k] = 0.f;
                for (uint32_t e = kb; e < ke; ++e) {
                    const uint32_t j = __ldg(a.colInd + e);
                    const float v = __ldg(a.val + e);
#pragma unroll
                    for (int k = 0; k < NR; ++k) {
                        if (!act[k]) continue;
                        const size_t o = k * N + j;
                        const float pj = fr[k] ? a.z[o] : fmaf(bt[k], pOld[o], a.z[o]);
                        s[k] = fmaf(v, pj, s[k]);
                    }
                }
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    if (!act[k]) continue;
                    const size_t o = k * N + i;
                    const float pi = fr[k] ? a.z[o] : fmaf(bt[k], pOld[o], a.z[o]);
                    pNew[o] = pi;
                    a.q[o] = s[k];
                    pq[k] += (double)s[k] * pi;
                }
            }
            bsum<NR>(pq);
            if (threadIdx.x == 0)
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    st[k].alpha = st[k].active && pq[k] != 0.0 ? (float)(st[k].rz / pq[k]) : 0.f;
                    st[k].fresh = 0;
                }
            __syncthreads();
            // pass 2: x += alpha p, r -= alpha q, z = diagInv .* r; (r,r), (z,r)
            float al[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) al[k] = st[k].alpha;
            double red[2 * NR];
#pragma unroll
            for (int k = 0; k < 2 * NR; ++k) red[k] = 0.0;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const float d = a.dinv[i];
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    if (!act[k]) continue;
                    const size_t o = k * N + i;
                    const float xi = fmaf(al[k], pNew[o], a.x[o]);
                    const float ri = fmaf(-al[k], a.q[o], a.r[o]);
                    const float zi = d * ri;
                    a.x[o] = xi;
                    a.r[o] = ri;
                    a.z[o] = zi;
                    red[k] += (double)ri * ri;
                    red[NR + k] += (double)zi * ri;
                }
            }
            bsum<2 * NR>(red);
            if (threadIdx.x == 0) {
                int rf = 0;
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    st[k].trig = 0;
                    if (!st[k].active) continue;
                    const double res = sqrt(red[k]);
                    st[k].res = res;
                    if (res > st[k].rmax) st[k].rmax = res;
                    st[k].rzold = st[k].rz;
                    if (res < a.relTol || res < f.delta * st[k].rmax || !(red[k] == red[k])) {
                        rf = 1;
                        st[k].trig = 1;
                    } else {
                        st[k].beta = red[NR + k] / st[k].rz;
                        st[k].rz = red[NR + k];
                    }
                }
                refresh = rf;
            }
            __syncthreads();
            if (refresh) { // block-uniform
                // 1. x64 += s x32, x32 = 0
                for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x)
#pragma unroll
                    for (int k = 0; k < NR; ++k) {
                        if (!act[k]) continue;
                        const size_t o = k * N + i;
                        f.x64[o] = fma(st[k].sc, (double)a.x[o], f.x64[o]);
                        a.x[o] = 0.0f;
                    }
                __syncthreads();
                // 2. r = b - A x64 in FP64; r32 = r / s; z32 = diagInv .* r32
                double rr[3 * NR];
#pragma unroll
                for (int k = 0; k < 3 * NR; ++k) rr[k] = 0.0;
                for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                    const float d = a.dinv[i];
#pragma unroll
                    for (int k = 0; k < NR; ++k) {
                        if (!act[k]) continue;
                        double sum = 0.0;
                        for (uint32_t e = a.rowPtr[i]; e < a.rowPtr[i + 1]; ++e)
                            sum = fma(f.val64[e], f.x64[k * N + a.colInd[e]], sum);
                        const size_t o = k * N + i;
                        const double ri = f.b64[o] - sum;
                        const float r32 = (float)(ri / st[k].sc);
                        const float z32 = d * r32;
                        a.r[o] = r32;
                        a.z[o] = z32;
                        rr[k] = fma(ri, ri, rr[k]);
                        rr[NR + k] += (double)r32 * r32;
                        rr[2 * NR + k] += (double)z32 * r32;
                    }
                }
                bsum<3 * NR>(rr);
                if (threadIdx.x == 0)
#pragma unroll
                    for (int k = 0; k < NR; ++k) {
                        if (!st[k].active) continue;
                        const double tr = sqrt(rr[k]);
                        // three refreshes of its own in a row gaining less than sqrt(delta):
                        // the tolerance is below what the FP32 iterations attain here (a
                        // refresh another right-hand side asked for is not counted)
                        if (st[k].trig) {
                            st[k].stall = tr > sqrt(f.delta) * st[k].prev ? st[k].stall + 1 : 0;
                            st[k].prev = tr;
                        }
                        if (tr < a.relTol * st[k].true0 || !(tr == tr) || st[k].stall >= 3) {
                            st[k].active = 0;
                            st[k].its = it;
                            st[k].res = tr / st[k].sc;
                        } else {
                            const double rs = sqrt(rr[NR + k]);
                            // a refreshed residual far above the recursive one: p = z
                            if (rs > 4.0 * st[k].res) st[k].fresh = 1;
                            // beta from the refreshed residual and the (z, r) of the previous
                            // iteration
                            st[k].beta = rr[2 * NR + k] / st[k].rzold;
                            st[k].rz = rr[2 * NR + k];
                            st[k].rmax = rs;
                            st[k].res = rs;
                        }
                    }
                __syncthreads();
            }
            if (threadIdx.x == 0) {
                int na = 0;
#pragma unroll
                for (int k = 0; k < NR; ++k) na += st[k].active;
                nact = na;
            }
            __syncthreads();
            par ^= 1;
        }
        // right-hand sides still active at maxIter: fold the FP32 correction
        for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x)
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                if (!st[k].active) continue;
                const size_t o = k * N + i;
                f.x64[o] = fma(st[k].sc, (double)a.x[o], f.x64[o]);
            }
        if (threadIdx.x < NR) {
            const int k = threadIdx.x;
            a.iters[(size_t)sys * a.nrhs + k] += st[k].active ? it : st[k].its;
            a.resRel[(size_t)sys * a.nrhs + k] =
                st[k].true0 > 0 ? st[k].res * st[k].sc / st[k].true0 : 0.0;
        }
    }
}

// FP64 residual of every system and right-hand side, r64 = b - A x (the outer step of the
// mixed solve), with ||r|| per (system, rhs) and the FP32 right-hand side r / ||r||.
__global__ void __launch_bounds__(256) batch_residual(uint32_t count, uint32_t nrhs, uint32_t N,
                                                      const uint32_t* sysRow,
                                                      const uint32_t* rowPtr,
                                                      const uint32_t* colInd, const double* val,
                                                      const double* b, const double* x,
                                                      double* r64, double* rnorm)
{
    // one block per (system, rhs)
    const uint32_t id = blockIdx.x;
    if (id >= count * nrhs) return;
    const uint32_t sys = id / nrhs, k = id % nrhs;
    const uint32_t r0 = sysRow[sys], r1 = sysRow[sys + 1];
    double acc[1] = {0.0};
    for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        double s = 0.0;
        for (uint32_t e = rowPtr[i]; e < rowPtr[i + 1]; ++e)
            s = fma(val[e], x[(size_t)k * N + colInd[e]], s);
        const double ri = b[(size_t)k * N + i] - s;
        r64[(size_t)k * N + i] = ri;
        acc[0] = fma(ri, ri, acc[0]);
    }
    bsum<1>(acc);
    if (threadIdx.x == 0) rnorm[id] = sqrt(acc[0]);
}

__global__ void batch_scale_to32(uint32_t count, uint32_t nrhs, uint32_t N,
                                 const uint32_t* sysRow, const double* r64,
                                 const double* rnorm, float* b32)
{
    const uint32_t id = blockIdx.x;
    if (id >= count * nrhs) return;
    const uint32_t sys = id / nrhs, k = id % nrhs;
    const double s = rnorm[id] > 0 ? 1.0 / rnorm[id] : 0.0;
    for (uint32_t i = sysRow[sys] + threadIdx.x; i < sysRow[sys + 1]; i += blockDim.x)
        b32[(size_t)k * N + i] = (float)(r64[(size_t)k * N + i] * s);
}

__global__ void batch_update64(uint32_t count, uint32_t nrhs, uint32_t N,
                               const uint32_t* sysRow, const double* rnorm, const float* e32,
                               double* x)
{
    const uint32_t id = blockIdx.x;
    if (id >= count * nrhs) return;
    const uint32_t sys = id / nrhs, k = id % nrhs;
    const double s = rnorm[id];
    for (uint32_t i = sysRow[sys] + threadIdx.x; i < sysRow[sys + 1]; i += blockDim.x)
        x[(size_t)k * N + i] = fma(s, (double)e32[(size_t)k * N + i], x[(size_t)k * N + i]);
}

__global__ void batch_dinv(uint32_t N, const double* diag, double* d64, float* d32)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x) {
        const double v = 1.0 / diag[i];
        d64[i] = v;
        d32[i] = (float)v;
    }
}

} // namespace fb

using namespace fb;

struct fasp_gpu_batch_s {
    Ctx       c;
    Mat       M;
    uint32_t  count = 0, nrhs = 0;
    uint32_t* sysRow = nullptr;
    uint32_t* order = nullptr;
    double*   dinv = nullptr;
    float*    dinv32 = nullptr;
    double *  r64 = nullptr, *z64 = nullptr, *p0 = nullptr, *p1 = nullptr, *q64 = nullptr;
    float *   b32 = nullptr, *x32 = nullptr, *r32 = nullptr, *z32 = nullptr, *p032 = nullptr,
          *p132 = nullptr, *q32 = nullptr;
    double*   rnorm = nullptr;
    double*   resRel = nullptr;
    uint32_t* iters = nullptr;
    unsigned* queue = nullptr;
    int       block = 256;  // autotuned
    int       blocksPerSM = 4;
    double    lastMs = 0.0;
};

namespace {

template <typename T>
int launch_batch(fasp_gpu_batch_s& B, BatchArgs<T> a)
{
    const int grid = B.c.nsm * B.blocksPerSM;
    cudaMemsetAsync(B.queue, 0, sizeof(unsigned), B.c.stream);
    switch (B.nrhs) {
        case 1: batch_pcg<T, 1><<<grid, B.block, 0, B.c.stream>>>(a); break;
        case 2: batch_pcg<T, 2><<<grid, B.block, 0, B.c.stream>>>(a); break;
        case 3: batch_pcg<T, 3><<<grid, B.block, 0, B.c.stream>>>(a); break;
        default: batch_pcg<T, 4><<<grid, B.block, 0, B.c.stream>>>(a); break;
    }
    B.c.launches += 1;
    return cudaGetLastError() == cudaSuccess ? kOk : kErrCuda;
}

} // namespace

extern "C" {

int fasp_gpu_batch_create(uint32_t count, const uint32_t* sysRow, uint32_t nnz,
                          const uint32_t* rowPtr, const uint32_t* colInd, const double* values,
                          uint32_t nrhs, fasp_gpu_batch* out)
{
    if (!out || !sysRow || !rowPtr || !colInd || !values || count == 0 || nrhs == 0 ||
        nrhs > (uint32_t)kMaxRhs)
        return kErrInputPar;
    *out = nullptr;
    std::vector<uint32_t> hs(count + 1);
    if (cudaMemcpy(hs.data(), sysRow, (count + 1) * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return kErrCuda;
    for (uint32_t k = 0; k < count; ++k)
        if (hs[k + 1] <= hs[k]) return kErrMatData; // empty or unordered system
    if (hs[0] != 0) return kErrMatData;
    const uint32_t N = hs[count];
    fasp_gpu_batch h = new (std::nothrow) fasp_gpu_batch_s();
    if (!h) return kErrAlloc;
    int e = h->c.init(library_device());
    // the matrix upload validates the structure (CheckCSR) before any kernel reads it
    if (!e) e = m_upload(h->M, N, N, nnz, rowPtr, colInd, values, false, h->c.stream);
    if (!e) {
        // each row's columns must stay inside its own system (block diagonal)
        std::vector<uint32_t> rp(N + 1), ci(nnz);
        cudaMemcpy(rp.data(), h->M.rowPtr, (N + 1) * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(ci.data(), h->M.colInd, (size_t)nnz * 4, cudaMemcpyDeviceToHost);
        for (uint32_t k = 0; k < count && !e; ++k)
            for (uint32_t i = hs[k]; i < hs[k + 1] && !e; ++i)
                for (uint32_t q = rp[i]; q < rp[i + 1]; ++q)
                    if (ci[q] < hs[k] || ci[q] >= hs[k + 1]) {
                        e = kErrMatData;
                        break;
                    }
    }
    h->count = count;
    h->nrhs = nrhs;
    const size_t vN = (size_t)nrhs * N;
    auto dm = [&](void** p, size_t bytes) {
        if (!e && cudaMalloc(p, bytes + 16) != cudaSuccess) {
            cudaGetLastError();
            e = kErrAlloc;
        }
    };
    dm((void**)&h->sysRow, (count + 1) * 4);
    dm((void**)&h->order, count * 4);
    dm((void**)&h->dinv, N * 8);
    dm((void**)&h->dinv32, N * 4);
    dm((void**)&h->r64, vN * 8);
    dm((void**)&h->z64, vN * 8);
    dm((void**)&h->p0, vN * 8);
    dm((void**)&h->p1, vN * 8);
    dm((void**)&h->q64, vN * 8);
    dm((void**)&h->b32, vN * 4);
    dm((void**)&h->x32, vN * 4);
    dm((void**)&h->r32, vN * 4);
    dm((void**)&h->z32, vN * 4);
    dm((void**)&h->p032, vN * 4);
    dm((void**)&h->p132, vN * 4);
    dm((void**)&h->q32, vN * 4);
    dm((void**)&h->rnorm, (size_t)count * nrhs * 8);
    dm((void**)&h->resRel, (size_t)count * nrhs * 8);
    dm((void**)&h->iters, (size_t)count * nrhs * 4);
    dm((void**)&h->queue, 16);
    if (!e) e = h->M.ensure32(h->c.stream);
    if (!e) {
        // longest systems first
        std::vector<uint32_t> ord(count);
        std::iota(ord.begin(), ord.end(), 0u);
        std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
            return hs[a + 1] - hs[a] > hs[b + 1] - hs[b];
        });
        cudaMemcpy(h->sysRow, hs.data(), (count + 1) * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(h->order, ord.data(), count * 4, cudaMemcpyHostToDevice);
        batch_dinv<<<std::max(1, std::min(ceil_div(N, 256), 148 * 8)), 256, 0, h->c.stream>>>(
            N, h->M.diag, h->dinv, h->dinv32);
        if (cudaStreamSynchronize(h->c.stream) != cudaSuccess) e = kErrCuda;
    }
    if (e) {
        fasp_gpu_batch_destroy(h);
        return e;
    }
    *out = h;
    return kOk;
}

int fasp_gpu_batch_destroy(fasp_gpu_batch h)
{
    if (!h) return kOk;
    cudaStreamSynchronize(h->c.stream);
    m_free(h->M);
    for (void* p : {(void*)h->sysRow, (void*)h->order, (void*)h->dinv, (void*)h->dinv32,
                    (void*)h->r64, (void*)h->z64, (void*)h->p0, (void*)h->p1, (void*)h->q64,
                    (void*)h->b32, (void*)h->x32, (void*)h->r32, (void*)h->z32,
                    (void*)h->p032, (void*)h->p132, (void*)h->q32, (void*)h->rnorm,
                    (void*)h->resRel, (void*)h->iters, (void*)h->queue})
        cudaFree(p);
    h->c.destroy();
    delete h;
    return kOk;
}

int fasp_gpu_batch_set_shape(fasp_gpu_batch h, int block, int blocksPerSM)
{
    if (!h || (block != 128 && block != 256 && block != 512) || blocksPerSM < 1 ||
        blocksPerSM > 16 || block * blocksPerSM > 2048)
        return kErrInputPar;
    h->block = block;
    h->blocksPerSM = blocksPerSM;
    return kOk;
}

int fasp_gpu_batch_solve(fasp_gpu_batch h, const double* b, double* x, double relTol,
                         uint32_t maxIter, int precision, double innerRelTol,
                         uint32_t* iters, double* resRel)
{
    if (!h || !b || !x || relTol <= 0) return kErrInputPar;
    TraceRange trace("fasp batch solve");
    fasp_gpu_batch_s& B = *h;
    const uint32_t N = B.M.nrow, cnt = B.count, nr = B.nrhs;
    const size_t vN = (size_t)nr * N;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, B.c.stream);
    cudaMemsetAsync(B.iters, 0, (size_t)cnt * nr * 4, B.c.stream);
    int e = kOk;
    if (precision == FASP_GPU_FP64) {
        BatchArgs<double> a{cnt, nr, N, B.sysRow, B.order, B.M.rowPtr, B.M.colInd, B.M.val,
                            B.dinv, b, x, B.r64, B.z64, B.p0, B.p1, B.q64, B.iters, B.resRel,
                            relTol, maxIter, B.queue};
        e = launch_batch<double>(B, a);
    } else if (precision == FASP_GPU_MIXED_RELIABLE) {
        BatchArgs<float> a{cnt, nr, N, B.sysRow, B.order, B.M.rowPtr, B.M.colInd, B.M.val32,
                           B.dinv32, nullptr, B.x32, B.r32, B.z32, B.p032, B.p132, B.q32,
                           B.iters, B.resRel, relTol, maxIter, B.queue};
        const BatchRel f{B.M.val, b, x, innerRelTol > 0 && innerRelTol < 1 ? innerRelTol : 1e-2};
        const int grid = B.c.nsm * B.blocksPerSM;
        cudaMemsetAsync(B.queue, 0, sizeof(unsigned), B.c.stream);
        switch (nr) {
            case 1: batch_pcg_rel<1><<<grid, B.block, 0, B.c.stream>>>(a, f); break;
            case 2: batch_pcg_rel<2><<<grid, B.block, 0, B.c.stream>>>(a, f); break;
            case 3: batch_pcg_rel<3><<<grid, B.block, 0, B.c.stream>>>(a, f); break;
            default: batch_pcg_rel<4><<<grid, B.block, 0, B.c.stream>>>(a, f); break;
        }
        B.c.launches += 1;
        if (cudaGetLastError() != cudaSuccess) e = kErrCuda;
    } else {
        // FP64 refinement around FP32 inner solves, x0 = 0
        cudaMemsetAsync(x, 0, vN * 8, B.c.stream);
        const double inner = innerRelTol > 0 ? innerRelTol : 1e-4;
        int steps = 0;
        const int maxSteps = 2 + (int)(std::log(relTol) / std::log(inner)) + 4;
        std::vector<double> hn((size_t)cnt * nr), h0;
        for (; steps < maxSteps; ++steps) {
            batch_residual<<<cnt * nr, 256, 0, B.c.stream>>>(cnt, nr, N, B.sysRow, B.M.rowPtr,
                                                           B.M.colInd, B.M.val, b, x, B.r64,
                                                           B.rnorm);
            cudaMemcpyAsync(hn.data(), B.rnorm, hn.size() * 8, cudaMemcpyDeviceToHost,
                            B.c.stream);
            cudaStreamSynchronize(B.c.stream);
            if (steps == 0) h0 = hn;
            bool done = true;
            for (size_t k = 0; k < hn.size(); ++k)
                if (hn[k] > relTol * h0[k]) done = false;
            if (done) break;
            batch_scale_to32<<<cnt * nr, 256, 0, B.c.stream>>>(cnt, nr, N, B.sysRow, B.r64,
                                                             B.rnorm, B.b32);
            BatchArgs<float> a{cnt, nr, N, B.sysRow, B.order, B.M.rowPtr, B.M.colInd,
                               B.M.val32, B.dinv32, B.b32, B.x32, B.r32, B.z32, B.p032,
                               B.p132, B.q32, B.iters, B.resRel, inner, maxIter, B.queue};
            if ((e = launch_batch<float>(B, a))) break;
            batch_update64<<<cnt * nr, 256, 0, B.c.stream>>>(cnt, nr, N, B.sysRow, B.rnorm,
                                                           B.x32, x);
            B.c.launches += 3;
        }
        if (!e) {
            // final FP64 relative residual per (system, rhs)
            for (size_t k = 0; k < hn.size(); ++k) hn[k] = h0[k] > 0 ? hn[k] / h0[k] : 0.0;
            cudaMemcpyAsync(B.resRel, hn.data(), hn.size() * 8, cudaMemcpyHostToDevice,
                            B.c.stream);
        }
    }
    cudaEventRecord(t1, B.c.stream);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    B.lastMs = ms;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (!e && cudaGetLastError() != cudaSuccess) e = kErrCuda;
    if (!e && iters &&
        cudaMemcpyAsync(iters, B.iters, (size_t)cnt * nr * 4, cudaMemcpyDeviceToHost, B.c.stream))
        e = kErrCuda;
    if (!e && resRel &&
        cudaMemcpyAsync(resRel, B.resRel, (size_t)cnt * nr * 8, cudaMemcpyDeviceToHost,
                        B.c.stream))
        e = kErrCuda;
    if (!e && cudaStreamSynchronize(B.c.stream) != cudaSuccess) e = kErrCuda;
    return e;
}

int fasp_gpu_batch_solve_async(fasp_gpu_batch h, const double* b, double* x, double relTol,
                               uint32_t maxIter, int precision, double innerRelTol,
                               uint32_t* iters, double* resRel, fasp_gpu_stream stream)
{
    if (!h) return kErrInputPar;
    return on_stream(h->c, reinterpret_cast<cudaStream_t>(stream), [&]() {
        return fasp_gpu_batch_solve(h, b, x, relTol, maxIter, precision, innerRelTol, iters,
                                    resRel);
    });
}

int fasp_gpu_batch_last_time(fasp_gpu_batch h, double* ms)
{
    if (!h || !ms) return kErrInputPar;
    *ms = h->lastMs;
    return kOk;
}

} // extern "C"
