// solvers.cu -- the SOL subclasses of FASP++ on the GPU.
//
// Each solver keeps the reference's control flow statement by statement (file:line cited
// per function) while every vector operation is a kernel on the solver's stream. Scalars
// stay on the device (kernels read them through Scal) until a branch needs one on the host.
// CG with an Identity or single-sweep Jacobi preconditioner runs device-driven (cg.cu); the
// other configurations run the host-orchestrated restatement below.
#include <cmath>
#include <cstring>
#include <limits>
#include <type_traits>

#include <new>

#include "gmres.cuh"
#include "solver.h"

namespace fb {

static const double kNaN = std::numeric_limits<double>::quiet_NaN();

// scalar slots of the solver context
enum {
    SL_T0 = 0, SL_T1, SL_T2, SL_T3, SL_T4, SL_T5, SL_T6, SL_T7,
    SL_XINF = 16,  // NormInf of a residual's x (MAT::Residual shortcut)
    SL_ONE = 17,   // constant 1: disables the shortcut (MAT::Apply + XPAY paths)
    SL_XINF2 = 18, // the fused Jacobi sweeps' second NormInf slot (ping-pong with SL_XINF)
    SL_JRES = 19,  // ||r|| of the sweep that tests convergence
};

double SolverImpl::fetch(const double* dptr)
{
    double v = kNaN;
    if (cudaMemcpyAsync(c.hslot, dptr, sizeof(double), cudaMemcpyDeviceToHost, c.stream) ==
            cudaSuccess &&
        cudaStreamSynchronize(c.stream) == cudaSuccess)
        v = c.hslot[0];
    return v;
}

// A->Apply(x, r); r.XPAY(-1.0, b)  -> r = b - A x without the NormInf shortcut
template <typename T>
static int apply_residual(Ctx& c, const Mat& A, const T* b, const T* x, T* r)
{
    return m_residual(c, A, b, x, r, c.dslot + SL_ONE);
}

// ---- Jacobi (src/Iter.cxx) ---------------------------------------------------------------

template <typename T>
__global__ void k_jacobi_update(uint32_t n, const T* __restrict__ dinv,
                                const T* __restrict__ work, T* __restrict__ x,
                                Scratch s, double* dxinf)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    // work .*= diagInv; x += work (Iter.cxx:91-92); also NormInf(x_new) for the next
    // residual's shortcut test
    T m = T(0);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const T xi = x[i] + work[i] * dinv[i];
        x[i] = xi;
        m = fmax(m, fabs(xi));
    }
    double acc[1] = {(double)m};
    const int ops[1] = {kMax};
    grid_reduce<1>(acc, ops, s, [=] __device__(const double* t) { *dxinf = t[0]; });
}

template <typename T>
static CSRView<T> pcd_view(const Mat& A);
template <>
CSRView<double> pcd_view<double>(const Mat& A) { return A.v64(); }
template <>
CSRView<float> pcd_view<float>(const Mat& A) { return A.v32(); }

// One Jacobi sweep in one pass (Jacobi::Solve, Iter.cxx:83-92, with MAT::Residual,
// MAT.cxx:455-476): r = b - A x_in, or r = b when NormInf(x_in) < CLOSE_ZERO; x_out = x_in
// + diagInv .* r; NormInf(x_out) for the next sweep's shortcut and, with NORM, ||r|| -- the
// residual of x_in, which Jacobi::Solve tests before it updates x. Each row is summed as
// MAT::Residual's thread-per-row kernel sums it and updated with the same expression as
// k_jacobi_update, so the sweeps give the two-kernel path's x bit for bit. x_in and x_out
// are different vectors (every row reads x_in's neighbours).
template <typename T, bool NORM>
__global__ void __launch_bounds__(kBlock) k_jacobi_sweep(CSRView<T> A, const T* __restrict__ b,
                                                         const T* __restrict__ xin,
                                                         const T* __restrict__ dinv,
                                                         T* __restrict__ xout,
                                                         const double* __restrict__ xinfIn,
                                                         Scratch s, double* xinfOut,
                                                         double* rnorm)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    const bool shortcut = *xinfIn < kCloseZero;
    T m = T(0), rr = T(0);
    auto xv = [&](uint32_t j) { return xin[j]; };
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.nrow;
         i += (size_t)gridDim.x * blockDim.x) {
        const T sum = shortcut ? T(0) : row_apply<T, false>(A, i, xv);
        const T r = b[i] - sum;
        const T xi = xin[i] + r * dinv[i];
        xout[i] = xi;
        m = fmax(m, fabs(xi));
        if (NORM) rr = fma(r, r, rr);
    }
    if (NORM) {
        double acc[2] = {(double)m, (double)rr};
        const int ops[2] = {kMax, kSum};
        grid_reduce<2>(acc, ops, s, [=] __device__(const double* t) {
            *xinfOut = t[0];
            *rnorm = sqrt(t[1]);
        });
    } else {
        double acc[1] = {(double)m};
        const int ops[1] = {kMax};
        grid_reduce<1>(acc, ops, s, [=] __device__(const double* t) { *xinfOut = t[0]; });
    }
}

// A whole Jacobi::Solve (Iter.cxx:56-112) on a small matrix in one single-block launch:
// NormInf(x), then per sweep the residual (with MAT::Residual's shortcut) into work, its
// norm and Jacobi::Solve's convergence test when numIter >= minIter, and x += diagInv .*
// work, each phase separated by a block barrier. A coarse MG level thus costs one launch
// instead of 2 per sweep. The sums of each row and the updates are those of the
// multi-block kernels, so x is the same bit for bit; the residual norms that decide when
// to stop are block reductions in a fixed order (the tests' outcome can differ from the
// multi-block reductions' only at the rounding level).
constexpr uint32_t kJacobiBlockRows = 16384;
constexpr int kJacobiBlockThreads = 1024;

// The block's sum or max of v, returned to EVERY thread (warp_reduce leaves its result in
// lane 0 only; it is broadcast), so that the branches taken on it -- the residual
// shortcut, the convergence test -- are the same in the whole block and every thread
// reaches the same barriers.
__device__ __forceinline__ double block_allreduce(double v, int op, double* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_reduce(v, op);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    const double t = warp_reduce(lane < nw ? sh[lane] : red_ident(op), op);
    return __shfl_sync(0xffffffffu, t, 0); // each warp forms the same value in the same order
}

template <typename T>
__global__ void __launch_bounds__(kJacobiBlockThreads) k_jacobi_block(
    CSRView<T> A, const T* __restrict__ b, T* __restrict__ x, const T* __restrict__ dinv,
    T* __restrict__ work, fasp_gpu_params prm)
{
    pdl_wait(); // may be launched programmatically (launch_pdl)
    pdl_release();
    __shared__ double sh[32];
    const uint32_t n = A.nrow;
    auto xv = [&](uint32_t j) { return x[j]; };
    double m = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, (double)fabs(x[i]));
    double xinf = block_allreduce(m, kMax, sh);
    double denAbs = 1.0;
    for (uint32_t it = 0; it < prm.maxIter; ++it) {
        const bool shortcut = xinf < kCloseZero;
        T rr = T(0);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const T sum = shortcut ? T(0) : row_apply<T, false>(A, i, xv);
            const T r = b[i] - sum;
            work[i] = r;
            rr = fma(r, r, rr);
        }
        if (it >= prm.minIter) {
            const double resAbs = sqrt(block_allreduce((double)rr, kSum, sh));
            if (it == prm.minIter) denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;
            if (resAbs / denAbs < prm.relTol || resAbs < prm.absTol) break;
        }
        __syncthreads(); // every row's residual read the old x
        m = 0.0;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const T xi = x[i] + work[i] * dinv[i];
            x[i] = xi;
            m = fmax(m, (double)fabs(xi));
        }
        xinf = block_allreduce(m, kMax, sh); // its barriers order the writes of x
    }
}

int Pcd::setup(Ctx& c, const Mat* M, int t, double w, const fasp_gpu_params& p)
{
    type = t;
    weight = w;
    prm = p;
    A = M;
    if (type != 1) return kOk;
    const size_t n = M->nrow;
    if (cudaMalloc(&dinv, (n + 2) * 8) || cudaMalloc(&dinv32, (n + 4) * 4) ||
        cudaMalloc(&work, (n + 2) * 8)) {
        cudaGetLastError();
        return kErrAlloc;
    }
    // Jacobi::Setup: GetDiag, Reciprocal, Scale(weight) (Iter.cxx:45-47)
    int e = v_recip_scale(c, M->nrow, weight, M->diag, dinv);
    if (e) return e;
    return to32(c, M->nrow, dinv, dinv32);
}

// type 2 (MG preconditioner): one MG::Solve on the preconditioner's own solver object
static int pcd_mg_apply(SolverImpl* s, const double* b, double* x);
static void pcd_mg_free(SolverImpl* s);

void Pcd::destroy()
{
    if (mg) {
        pcd_mg_free(mg);
        mg = nullptr;
    }
    cudaFree(dinv);
    cudaFree(dinv32);
    cudaFree(work);
    cudaFree(work32);
    dinv = nullptr;
    dinv32 = nullptr;
    work = nullptr;
    work32 = nullptr;
}

// Identity::Solve (Iter.cxx:16-20) or Jacobi::Solve (Iter.cxx:56-112).
template <typename T>
int Pcd::solve(Ctx& c, const T* b, T* x, std::vector<double>* hist, double* norm2,
               double* normInf)
{
    const uint32_t n = A->nrow;
    if (type == 0) return v_copy(c, n, b, x);
    if (type == 2) {
        if constexpr (std::is_same<T, float>::value)
            return kErrPcdType; // FP32 inner solves have no MG preconditioner
        else
            return pcd_mg_apply(mg, b, x);
    }
    T* work;
    const T* dinv;
    if constexpr (std::is_same<T, float>::value) {
        if (!work32 && cudaMalloc(&work32, ((size_t)n + 4) * 4) != cudaSuccess) {
            cudaGetLastError();
            return kErrAlloc;
        }
        work = work32;
        dinv = dinv32;
    } else {
        work = this->work;
        dinv = this->dinv;
    }
    auto fetch = [&](const double* d) {
        double v = kNaN;
        cudaMemcpyAsync(c.hslot + 1, d, 8, cudaMemcpyDeviceToHost, c.stream);
        cudaStreamSynchronize(c.stream);
        v = c.hslot[1];
        return v;
    };
    auto rec = [&](uint32_t k, double v) {
        if (!hist) return;
        if (k >= hist->size()) hist->resize((size_t)k + 1, kNaN);
        (*hist)[k] = v;
    };
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0;
    const CSRView<T> V = pcd_view<T>(*A);
    const bool fusable = A->lanes == 1 && (V.val || V.gnz) && (const void*)b != (const void*)x;
    if (fusable && !hist && !norm2 && !normInf && n <= kJacobiBlockRows) {
        // nothing reads the norms back: the whole solve in one single-block launch
        ++c.launches;
        FB_CUDA(launch_pdl(k_jacobi_block<T>, dim3(1), dim3(kJacobiBlockThreads), 0, c.stream, V, b,
                           x, dinv, work, prm));
        FB_CUDA(cudaGetLastError());
        numIter = prm.maxIter; // the convergence test ran on the device
        return kOk;
    }
    if (fusable) {
        // one launch per sweep; x and work take turns as the sweep's input and output
        double* xinf[2] = {c.dslot + SL_XINF, c.dslot + SL_XINF2};
        int e = v_norminf(c, n, x, xinf[0]);
        if (e) return e;
        T* cur = x;
        T* nxt = work;
        int p = 0;
        auto sweep = [&](auto kern) {
            const int g = std::min(c.grid(n, kBlock), resident_grid(c, (const void*)kern, kBlock));
            launch_pdl(kern, dim3((unsigned)g), dim3(kBlock), 0, c.stream, V, b, (const T*)cur,
                       dinv, nxt, (const double*)xinf[p], c.red, xinf[p ^ 1], c.dslot + SL_JRES);
        };
        numIter = 0;
        while (numIter < prm.maxIter) {
            const bool test = numIter >= prm.minIter;
            ++c.launches;
            if (test)
                sweep(k_jacobi_sweep<T, true>);
            else
                sweep(k_jacobi_sweep<T, false>);
            FB_CUDA(cudaGetLastError());
            if (test) {
                resAbs = fetch(c.dslot + SL_JRES);
                if (numIter == prm.minIter) denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;
                resRel = resAbs / denAbs;
                rec(numIter, resAbs);
                if (resRel < prm.relTol || resAbs < prm.absTol) break; // x_in stays
            }
            std::swap(cur, nxt);
            p ^= 1;
            ++numIter;
        }
        if (cur != x && (e = v_copy(c, n, (const T*)cur, x))) return e;
        if (!(numIter == prm.minIter && numIter == prm.maxIter)) {
            if ((e = m_residual(c, *A, b, x, work, xinf[p]))) return e;
            v_norm2(c, n, work, c.dslot + SL_T7);
            v_norminf(c, n, work, c.dslot + SL_T6);
            resAbs = fetch(c.dslot + SL_T7);
            const double ni = fetch(c.dslot + SL_T6);
            if (norm2) *norm2 = resAbs;
            if (normInf) *normInf = ni;
            rec(numIter, resAbs);
        }
        return kOk;
    }
    double* xinf = c.dslot + SL_XINF;
    int e = v_norminf(c, n, x, xinf);
    if (e) return e;
    numIter = 0;
    while (numIter < prm.maxIter) {
        if ((e = m_residual(c, *A, b, x, work, xinf))) return e;
        if (numIter >= prm.minIter) {
            v_norm2(c, n, work, c.dslot + SL_T7);
            resAbs = fetch(c.dslot + SL_T7);
            if (numIter == prm.minIter) denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;
            resRel = resAbs / denAbs;
            rec(numIter, resAbs);
            if (resRel < prm.relTol || resAbs < prm.absTol) break;
        }
        ++c.launches;
        FB_CUDA(launch_pdl(k_jacobi_update<T>, dim3((unsigned)c.grid(n, kBlock)), dim3(kBlock), 0,
                           c.stream, n, dinv, (const T*)work, x, c.red, xinf));
        FB_CUDA(cudaGetLastError());
        ++numIter;
    }
    if (!(numIter == prm.minIter && numIter == prm.maxIter)) {
        if ((e = m_residual(c, *A, b, x, work, xinf))) return e;
        v_norm2(c, n, work, c.dslot + SL_T7);
        v_norminf(c, n, work, c.dslot + SL_T6);
        resAbs = fetch(c.dslot + SL_T7);
        const double ni = fetch(c.dslot + SL_T6);
        if (norm2) *norm2 = resAbs;
        if (normInf) *normInf = ni;
        rec(numIter, resAbs);
    }
    return kOk;
}

template int Pcd::solve<double>(Ctx&, const double*, double*, std::vector<double>*, double*,
                                double*);
template int Pcd::solve<float>(Ctx&, const float*, float*, std::vector<double>*, double*,
                               double*);

// ---- setup -------------------------------------------------------------------------------

template <typename T>
static int alloc_vecs(std::vector<T*>& w, int k, uint32_t n)
{
    const size_t bytes = ((size_t)n + 4) * sizeof(T);
    for (int i = 0; i < k; ++i) {
        T* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return kErrAlloc;
        }
        cudaMemset(p, 0, bytes);
        w.push_back(p);
    }
    return kOk;
}

int SolverImpl::setup(fasp_gpu_mat Mh)
{
    if (!Mh) return kErrInputPar;
    destroy(); // a second Setup releases everything the first one allocated
    Ah = Mh;
    A = &Mh->M;
    n = A->nrow;
    if (A->nrow != A->mcol) return kErrMatSize;
    int e;
    const double one = 1.0;
    FB_CUDA(cudaMemcpyAsync(c.dslot + SL_ONE, &one, 8, cudaMemcpyHostToDevice, c.stream));
    FB_CUDA(cudaStreamSynchronize(c.stream));
    const int alg = cfg.alg;
    if (alg == FASP_GPU_JACOBI) {
        // the solver is itself a Jacobi object with its own weight and SOLParams
        if ((e = pcd.setup(c, A, 1, cfg.weight, cfg.prm))) return e;
        FB_CUDA(cudaStreamSynchronize(c.stream));
        return kOk;
    }
    if (cfg.pcd < 0 || cfg.pcd > 2) return kErrPcdType;
    if (cfg.pcd == 2) {
        // MG as the preconditioner (SOL::SetupPCD with an MG object, SOL.cxx:249): an MG
        // solver on the same matrix and stream, with this solver's MG settings and the
        // preconditioner's SOLParams (pcdPrm), transfers included when set
        if (cfg.precision != FASP_GPU_FP64) return kErrPcdType;
        SolverImpl* m = new (std::nothrow) SolverImpl();
        if (!m) return kErrAlloc;
        m->cfg = cfg;
        m->cfg.alg = FASP_GPU_MG;
        m->cfg.prm = cfg.pcdPrm;
        m->cfg.pcd = 0;
        m->c = c; // shares the stream and reduction scratch (never destroyed by m)
        m->mgIn = mgIn;
        pcd.type = 2;
        pcd.A = A;
        pcd.prm = cfg.pcdPrm;
        pcd.mg = m;
        if ((e = m->setup(Mh))) return e;
    } else if ((e = pcd.setup(c, A, cfg.pcd, cfg.pcdWeight, cfg.pcdPrm))) {
        return e;
    }
    switch (alg) {
        case FASP_GPU_CG: {
            if ((e = alloc_vecs(w, 5, n))) return e; // rk pk zk ax safe
            dhistCap = cfg.prm.maxIter + 2;
            if (cudaMalloc(&dhist, (size_t)dhistCap * 8) != cudaSuccess) return kErrAlloc;
            const bool fusable = cfg.pcd == 0 || (pcd.pure() && pcd.prm.maxIter == 1);
            if (fusable && cfg.precision == FASP_GPU_FP64) {
                cg64 = new CGEngine<double>();
                cg64->wantPersistent = cfg.persistent != 0;
                cg64->wantCluster = cfg.persistent == 2;
                cg64->barLimit = barLimit;
                cg64->pdl = cfg.overlapLaunch != 0;
                // Jacobi::Setup's diagInv = (1 / diag) * weight, one value for all rows
                cg64->constDiag = cfg.pcd == 1 && A->diagConst;
                cg64->zc = (1.0 / A->diagValue) * pcd.weight;
                if ((e = cg64->init(&c, A, cfg.pcd, pcd.dinv, cfg.useGraph != 0))) return e;
            }
            if (cfg.precision == FASP_GPU_MIXED || cfg.precision == FASP_GPU_MIXED_RELIABLE) {
                if (!fusable) return kErrPcdType; // mixed mode fuses its preconditioner
                if ((e = Ah->M.ensure32(c.stream))) return e;
                cg32 = new CGEngine<float>();
                cg32->wantPersistent = cfg.persistent != 0;
                cg32->wantCluster = cfg.persistent == 2;
                cg32->barLimit = barLimit;
                cg32->pdl = cfg.overlapLaunch != 0;
                cg32->recurrence = cfg.fp32Recurrence != 0;
                cg32->constDiag = cfg.pcd == 1 && A->diagConst;
                cg32->zc = (1.0 / A->diagValue) * pcd.weight;
                if ((e = cg32->init(&c, A, cfg.pcd, pcd.dinv32, cfg.useGraph != 0))) return e;
            }
            break;
        }
        case FASP_GPU_BICGSTAB: {
            if (cfg.precision == FASP_GPU_MIXED) {
                // FP64: the outer residual; FP32: the inner solve's 12 vectors + b, e
                if ((e = alloc_vecs(w, 1, n)) || (e = alloc_vecs(w32, 14, n))) return e;
                if ((e = Ah->M.ensure32(c.stream))) return e;
            } else if (cfg.precision == FASP_GPU_MIXED_RELIABLE) {
                // FP64 x and residual; the FP32 engine holds the iteration's vectors
                if ((e = alloc_vecs(w, 2, n))) return e;
                if ((e = Ah->M.ensure32(c.stream))) return e;
            } else if ((e = alloc_vecs(w, 12, n))) {
                return e;
            }
            // Identity or one Jacobi sweep from zero: the device-driven engine
            const bool fusable = (A->val || A->grid) && (cfg.pcd == 0 || (pcd.pure() && pcd.prm.maxIter == 1));
            if (fusable) {
                dhistCap = cfg.prm.maxIter + 2;
                if (cudaMalloc(&dhist, (size_t)dhistCap * 8) != cudaSuccess) return kErrAlloc;
                if (cfg.precision == FASP_GPU_MIXED ||
                    cfg.precision == FASP_GPU_MIXED_RELIABLE) {
                    bi32 = new BiEngine<float>();
                    bi32->pdl = cfg.overlapLaunch != 0;
                    bi32->rightPcd = cfg.precision == FASP_GPU_MIXED_RELIABLE && cfg.pcd == 1 &&
                                     !A->diagConst;
                    if ((e = bi32->init(&c, A, cfg.pcd, pcd.dinv32, cfg.useGraph != 0))) return e;
                } else {
                    bi64 = new BiEngine<double>();
                    bi64->pdl = cfg.overlapLaunch != 0;
                    if ((e = bi64->init(&c, A, cfg.pcd, pcd.dinv, cfg.useGraph != 0))) return e;
                }
            } else if (cfg.precision == FASP_GPU_MIXED_RELIABLE) {
                return kErrPcdType; // reliable updates run in the fused FP32 engine
            }
            break;
        }
        case FASP_GPU_GMRES:
        case FASP_GPU_FGMRES: {
            // GMRES::Setup (GMRES.cxx:38-88) / FGMRES::Setup (FGMRES.cxx:23-80)
            const uint32_t maxR = cfg.maxRestart ? cfg.maxRestart : 30;
            const uint32_t minR = cfg.maxRestart ? cfg.minRestart : 10;
            restart = cfg.prm.restart;
            maxRestart = maxR > cfg.prm.maxIter ? cfg.prm.maxIter : maxR;
            minRestart = minR > maxRestart ? maxRestart : minR;
            if (restart > maxRestart)
                restart = maxRestart;
            else if (restart < minRestart)
                restart = minRestart;
            if (maxRestart == 0 || restart == 0) return kErrInputPar;
            ldV = ((size_t)n + 31) & ~(size_t)31; // every basis vector 256-byte aligned
            if (cfg.precision == FASP_GPU_MIXED) {
                // FP64 outer residual; FP32 wk tmp safe + b, e and the FP32 bases
                if ((e = alloc_vecs(w, 1, n)) || (e = alloc_vecs(w32, 5, n))) return e;
                if ((e = Ah->M.ensure32(c.stream))) return e;
                const size_t vb = (size_t)(maxRestart + 1) * ldV * 4;
                if (cudaMalloc(&V32, vb + 16) != cudaSuccess) return kErrAlloc;
                cudaMemset(V32, 0, vb);
                if (alg == FASP_GPU_FGMRES) {
                    if (cudaMalloc(&Z32, vb + 16) != cudaSuccess) return kErrAlloc;
                    cudaMemset(Z32, 0, vb);
                }
            } else {
                if ((e = alloc_vecs(w, 3, n))) return e; // wk tmp safe
                const size_t vb = (size_t)(maxRestart + 1) * ldV * 8;
                if (cudaMalloc(&V, vb + 16) != cudaSuccess) return kErrAlloc;
                cudaMemset(V, 0, vb);
                if (alg == FASP_GPU_FGMRES) {
                    if (cudaMalloc(&Z, vb + 16) != cudaSuccess) return kErrAlloc;
                    cudaMemset(Z, 0, vb);
                }
            }
            const size_t gmSize = gm_layout_size(maxRestart);
            if (cudaMalloc(&gm, gmSize * 8) != cudaSuccess) return kErrAlloc;
            cudaMemset(gm, 0, gmSize * 8);
            if (cudaMalloc(&gmc, sizeof(GmCtl)) != cudaSuccess ||
                cudaMallocHost(&hgmc, sizeof(GmCtl)) != cudaSuccess)
                return kErrAlloc;
            dhistCap = cfg.prm.maxIter + 2;
            if (cudaMalloc(&dhist, (size_t)dhistCap * 8) != cudaSuccess) return kErrAlloc;
            break;
        }
        case FASP_GPU_MG: {
            if (!mgIn.empty()) {
                if ((e = alloc_vecs(w, 1, n))) return e; // r
                if ((e = mg_setup_transfers())) return e;
                break;
            }
            // MG::SetupALL + SetupLevel with identity transfers (MG.cxx:26-79)
            if ((e = alloc_vecs(w, 1, n))) return e; // r
            const uint32_t L = cfg.mgLevels;
            mgSmooth.resize(L);
            mgCoarse.resize(L);
            for (uint32_t l = 0; l < L; ++l) {
                if ((e = mgSmooth[l].setup(c, A, 1, cfg.mgSmoothWeight, cfg.mgSmoothPrm))) return e;
                if ((e = mgCoarse[l].setup(c, A, 1, cfg.mgCoarseWeight, cfg.mgCoarsePrm))) return e;
            }
            std::vector<double*> lv;
            if ((e = alloc_vecs(lv, 2 * L, n))) return e;
            for (uint32_t l = 0; l < L; ++l) {
                mgB.push_back(lv[2 * l]);
                mgX.push_back(lv[2 * l + 1]);
            }
            break;
        }
        default:
            return kErrSolverType;
    }
    FB_CUDA(cudaStreamSynchronize(c.stream));
    return kOk;
}

void SolverImpl::clean()
{
    // SOL::Clean: restart value restored, Krylov bases zeroed (GMRES.cxx:91-111,
    // FGMRES.cxx:83-105)
    if (cfg.alg == FASP_GPU_GMRES || cfg.alg == FASP_GPU_FGMRES) {
        restart = cfg.prm.restart;
        if (restart > maxRestart)
            restart = maxRestart;
        else if (restart < minRestart)
            restart = minRestart;
        const size_t vb = (size_t)(maxRestart + 1) * ldV * 8;
        if (V) cudaMemsetAsync(V, 0, vb, c.stream);
        if (Z) cudaMemsetAsync(Z, 0, vb, c.stream);
        if (V32) cudaMemsetAsync(V32, 0, vb / 2, c.stream);
        if (Z32) cudaMemsetAsync(Z32, 0, vb / 2, c.stream);
        cudaStreamSynchronize(c.stream);
    }
}

void SolverImpl::destroy()
{
    for (double* p : w) cudaFree(p);
    w.clear();
    for (float* p : w32) cudaFree(p);
    w32.clear();
    cudaFree(V32);
    cudaFree(Z32);
    V32 = Z32 = nullptr;
    cudaFree(V);
    cudaFree(Z);
    cudaFree(gm);
    cudaFree(gmc);
    if (hgmc) cudaFreeHost(hgmc);
    gmc = nullptr;
    hgmc = nullptr;
    cudaFree(safe);
    cudaFree(dhist);
    cudaFree(hostB);
    cudaFree(hostX);
    V = Z = gm = safe = dhist = hostB = hostX = nullptr;
    pcd.destroy();
    for (auto& p : mgSmooth) p.destroy();
    for (auto& p : mgCoarse) p.destroy();
    for (double* p : mgB) cudaFree(p);
    for (double* p : mgX) cudaFree(p);
    for (double* p : mgRes) cudaFree(p);
    mgRes.clear();
    for (Mat* m : mgOwn) {
        m_free(*m);
        delete m;
    }
    mgOwn.clear();
    mgA.clear();
    mgP.clear();
    mgR.clear();
    mgSmooth.clear();
    mgCoarse.clear();
    mgB.clear();
    mgX.clear();
    if (cg64) {
        cg64->destroy();
        delete cg64;
        cg64 = nullptr;
    }
    if (cg32) {
        cg32->destroy();
        delete cg32;
        cg32 = nullptr;
    }
    if (bi64) {
        bi64->destroy();
        delete bi64;
        bi64 = nullptr;
    }
    if (bi32) {
        bi32->destroy();
        delete bi32;
        bi32 = nullptr;
    }
    if (adj) {
        adj->destroy();
        adj->c.destroy();
        delete adj;
        adj = nullptr;
    }
}

// ---- CG (src/CG.cxx:53-249) ---------------------------------------------------------------

int SolverImpl::cg_generic(const double* b, double* x, fasp_gpu_info* info)
{
    const fasp_gpu_params& P = cfg.prm;
    double *rk = w[0], *pk = w[1], *zk = w[2], *ax = w[3], *sv = w[4];
    double* d = c.dslot;
    int err = kOk, e;
    const unsigned maxStag = kMaxStagNum;
    const double solStagTol = 1e-4 * P.relTol, solZeroTol = kCloseZero;
    unsigned stagStep = 0, moreStep = 0;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, ratio = 0.0, resAbsOld = 1.0;
    double alpha = 0.0, beta, tmpa, tmpb;
    uint32_t numIter = 0;

    if ((e = apply_residual(c, *A, b, x, rk))) return e;
    v_set(c, n, 0.0, zk);
    if ((e = pcd.solve(c, rk, zk))) return e;
    v_copy(c, n, zk, pk);
    v_dot(c, n, zk, rk, d + SL_T0);
    tmpa = fetch(d + SL_T0);

    while (numIter < P.maxIter) {
        if (numIter == P.minIter) {
            v_norm2(c, n, rk, d + SL_T1);
            resAbs = fetch(d + SL_T1);
            resAbsOld = resAbs;
            denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;
            resRel = resAbs / denAbs;
            rec(numIter, resAbs);
            if (resRel < P.relTol || resAbs < P.absTol) break;
        }
        ++numIter;
        m_spmv(c, *A, pk, ax);
        v_dot(c, n, ax, pk, d + SL_T0);
        tmpb = fetch(d + SL_T0);
        if (std::fabs(tmpb) > kCloseZero * kCloseZero)
            alpha = tmpa / tmpb;
        else {
            v_axpy(c, n, Scal::h(alpha), pk, x);
            v_axpy(c, n, Scal::h(-alpha), ax, rk);
            v_norm2(c, n, rk, d + SL_T1);
            resAbs = fetch(d + SL_T1);
            resRel = resAbs / denAbs;
            if (resRel > P.relTol && resAbs > P.absTol) err = kErrDivZero;
            rec(numIter, resAbs);
            break;
        }
        v_axpy(c, n, Scal::h(alpha), pk, x);
        v_axpy(c, n, Scal::h(-alpha), ax, rk);
        if (numIter >= P.minIter) {
            bool stop = false;
            v_norm2(c, n, rk, d + SL_T1);
            resAbs = fetch(d + SL_T1);
            resRel = resAbs / denAbs;
            ratio = resAbs / resAbsOld;
            if (numIter >= P.savIter && resAbs < resAbsOld) v_copy(c, n, x, sv);
            if (ratio > kKsmChkRatio) {
                v_norminf(c, n, x, d + SL_T2);
                const double xNormInf = fetch(d + SL_T2);
                if (xNormInf < solZeroTol) {
                    err = kErrSolStag;
                    stop = true;
                } else {
                    v_norm2(c, n, pk, d + SL_T3);
                    v_norm2(c, n, x, d + SL_T4);
                    const double xRelDiff =
                        std::fabs(alpha) * fetch(d + SL_T3) / fetch(d + SL_T4);
                    if ((stagStep <= maxStag) && (xRelDiff < solStagTol)) {
                        apply_residual(c, *A, b, x, rk);
                        v_norm2(c, n, rk, d + SL_T1);
                        resAbs = fetch(d + SL_T1);
                        resRel = resAbs / denAbs;
                        if (resRel < P.relTol || resAbs < P.absTol)
                            stop = true;
                        else if (stagStep >= maxStag) {
                            err = kErrStag;
                            stop = true;
                        } else {
                            v_set(c, n, 0.0, pk);
                            ++stagStep;
                        }
                    }
                }
            }
            if (!stop && resRel < P.relTol) {
                apply_residual(c, *A, b, x, rk);
                v_norm2(c, n, rk, d + SL_T1);
                resAbs = fetch(d + SL_T1);
                resRel = resAbs / denAbs;
                if (resRel < P.relTol || resAbs < P.absTol)
                    stop = true;
                else if (moreStep >= P.restart) {
                    err = kErrTolSmall;
                    stop = true;
                } else {
                    v_set(c, n, 0.0, pk); // CG.cxx:213 resizes pk to 0; zero is the intent
                    ++moreStep;
                }
            }
            rec(numIter, resAbs);
            if (stop) break;
        }
        if (numIter < P.maxIter) {
            resAbsOld = resAbs;
            v_set(c, n, 0.0, zk);
            if ((e = pcd.solve(c, rk, zk))) return e;
            v_dot(c, n, zk, rk, d + SL_T0);
            tmpb = fetch(d + SL_T0);
            beta = tmpb / tmpa;
            tmpa = tmpb;
            v_xpay(c, n, Scal::h(beta), zk, pk);
        }
    }
    info->numIter = numIter;
    info->code = err;
    if (!(numIter == P.minIter && numIter == P.maxIter)) {
        info->norm2 = resAbs;
        v_norminf(c, n, rk, d + SL_T2);
        info->normInf = fetch(d + SL_T2);
    }
    if (numIter > P.savIter) v_copy(c, n, sv, x);
    FB_CUDA(cudaStreamSynchronize(c.stream));
    return kOk;
}

__global__ void k_fill(uint32_t n, double v, double* x)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        x[i] = v;
}

int SolverImpl::cg_device(const double* b, double* x, fasp_gpu_info* info)
{
    const fasp_gpu_params& P = cfg.prm;
    CGEngine<double>& E = *cg64;
    CGCtl& h = *E.hctl;
    std::vector<std::pair<uint32_t, double>> patches; // history entries set by the host
    int e;
    std::memset(&h, 0, sizeof(CGCtl));
    h.maxIter = P.maxIter;
    h.minIter = P.minIter;
    h.savIter = P.savIter;
    h.restart = P.restart;
    h.relTol = P.relTol;
    h.absTol = P.absTol;
    h.solStagTol = 1e-4 * P.relTol;
    h.hist = dhist;
    h.histCap = dhistCap;
    h.histScale = 1.0;
    ++c.launches;
    k_fill<<<c.grid(dhistCap, kBlock), kBlock, 0, c.stream>>>(dhistCap, kNaN, dhist);
    v_copy(c, n, x, E.x);
    if ((e = apply_residual(c, *A, b, E.x, E.r))) return e;
    if ((e = E.push_ctl()) || (e = E.launch_init()) || (e = E.pull_ctl())) return e;
    unsigned launches = 0;
    info->escalations = 0;
    for (int guard = 0; h.status != kDone; ++guard) {
        if (h.status == kRun) {
            if ((e = E.run(&launches)) || (e = E.pull_ctl())) return e;
            c.launches += launches;
            launches = 0;
            continue;
        }
        // kEsc: the host finishes the branch the device could not (CG.cxx references)
        info->escalations++;
        const int reason = h.reason;
        double* p = E.cur_p();
        auto true_res = [&]() {
            apply_residual(c, *A, b, E.x, E.r);
            v_norm2(c, n, E.r, c.dslot + SL_T1);
            h.resAbs = fetch(c.dslot + SL_T1);
            h.resRel = h.resAbs / h.denAbs;
        };
        bool finished = false;
        if (reason == kBreakdown) { // CG.cxx:107-118
            v_axpy(c, n, Scal::h(h.alpha), p, E.x);
            v_axpy(c, n, Scal::h(-h.alpha), E.q, E.r);
            v_norm2(c, n, E.r, c.dslot + SL_T1);
            h.resAbs = fetch(c.dslot + SL_T1);
            h.resRel = h.resAbs / h.denAbs;
            if (h.resRel > P.relTol && h.resAbs > P.absTol) h.code = kErrDivZero;
            patches.push_back({h.numIter, h.resAbs});
            finished = true;
        } else if (reason == kSave) { // CG.cxx:138
            if (!safe && cudaMalloc(&safe, ((size_t)n + 2) * 8) != cudaSuccess) return kErrAlloc;
            v_copy(c, n, E.x, safe);
        } else if (reason == kStag) { // CG.cxx:153-181
            true_res();
            if (h.resRel < P.relTol || h.resAbs < P.absTol) {
                patches.push_back({h.numIter, h.resAbs});
                finished = true;
            } else if (h.stagStep >= kMaxStagNum) {
                h.code = kErrStag;
                patches.push_back({h.numIter, h.resAbs});
                finished = true;
            } else {
                h.pzero = 1;
                ++h.stagStep;
            }
        } else if (reason == kCheck3) { // CG.cxx:186-215
            true_res();
            if (h.resRel < P.relTol || h.resAbs < P.absTol) {
                patches.push_back({h.numIter, h.resAbs});
                finished = true;
            } else if (h.moreStep >= P.restart) {
                h.code = kErrTolSmall;
                patches.push_back({h.numIter, h.resAbs});
                finished = true;
            } else {
                h.pzero = 1;
                ++h.moreStep;
            }
        }
        if (finished) {
            h.status = kDone;
            if ((e = E.push_ctl())) return e;
            break;
        }
        h.status = kRun;
        if ((e = E.push_ctl()) || (e = E.launch_resume()) || (e = E.pull_ctl())) return e;
        if (guard > (int)P.maxIter + 64) return kErrCuda; // cannot happen: each pass advances
    }
    info->numIter = h.numIter;
    info->code = h.code;
    info->norm2 = kNaN;
    info->normInf = kNaN;
    if (!(h.numIter == P.minIter && h.numIter == P.maxIter)) {
        info->norm2 = h.resAbs;
        v_norminf(c, n, E.r, c.dslot + SL_T2);
        info->normInf = fetch(c.dslot + SL_T2);
    }
    v_copy(c, n, E.x, x);
    if (h.numIter > P.savIter && safe) v_copy(c, n, safe, x);
    const uint32_t len = std::min<uint32_t>(h.numIter + 1, dhistCap);
    hist.assign(len, kNaN);
    FB_CUDA(cudaMemcpyAsync(hist.data(), dhist, (size_t)len * 8, cudaMemcpyDeviceToHost, c.stream));
    FB_CUDA(cudaStreamSynchronize(c.stream));
    for (auto& pt : patches) rec(pt.first, pt.second);
    (void)launches;
    return kOk;
}

// Mixed precision: FP64 residual and update around FP32 inner CG solves (no reference
// counterpart). Each outer step solves A e = r / ||r|| in FP32 to innerRelTol, then
// x += ||r|| e in FP64; it stops when ||b - A x|| / ||b - A x0|| < relTol (or < absTol).
int SolverImpl::cg_mixed(const double* b, double* x, fasp_gpu_info* info)
{
    const fasp_gpu_params& P = cfg.prm;
    CGEngine<float>& E = *cg32;
    CGCtl& h = *E.hctl;
    double *x64 = w[0], *r64 = w[1];
    int e;
    v_copy(c, n, x, x64);
    const double innerTol = cfg.innerRelTol > 0 ? cfg.innerRelTol : 1e-4;
    const uint32_t innerMax = cfg.innerMaxIter ? cfg.innerMaxIter : P.maxIter;
    const uint32_t maxOuter = cfg.maxOuter ? cfg.maxOuter : 50;
    ++c.launches;
    k_fill<<<c.grid(dhistCap, kBlock), kBlock, 0, c.stream>>>(dhistCap, kNaN, dhist);
    uint32_t total = 0, outer = 0;
    double den = 1.0, rn = 0.0;
    int code = kOk;
    std::vector<std::pair<uint32_t, double>> outerHist;
    for (;;) {
        if ((e = apply_residual(c, *A, b, x64, r64))) return e;
        v_norm2(c, n, r64, c.dslot + SL_T1);
        rn = fetch(c.dslot + SL_T1);
        if (outer == 0) den = (kCloseZero > rn) ? kCloseZero : rn;
        outerHist.push_back({total, rn});
        if (rn / den < P.relTol || rn < P.absTol) break;
        if (outer >= maxOuter || total >= P.maxIter || !std::isfinite(rn)) {
            code = kErrMaxIt;
            break;
        }
        if ((e = convert_scaled(c, n, r64, 1.0 / rn, E.r)) || (e = set32(c, n, E.x))) return e;
        std::memset(&h, 0, sizeof(CGCtl));
        h.maxIter = std::min<uint32_t>(innerMax, P.maxIter - total);
        h.minIter = 0;
        h.savIter = 0xffffffffu;
        h.inner = 1;
        h.innerTol = innerTol;
        h.relTol = innerTol;
        h.hist = dhist;
        h.histCap = dhistCap;
        h.histOffset = total;
        h.histScale = rn;
        if ((e = E.push_ctl()) || (e = E.launch_init()) || (e = E.pull_ctl())) return e;
        unsigned gl = 0;
        if (h.status == kRun && ((e = E.run(&gl)) || (e = E.pull_ctl()))) return e;
        c.launches += gl;
        const uint32_t it = h.numIter;
        total += it;
        if ((e = E.apply_pending_x()) || (e = update_from32(c, n, rn, E.x, x64))) return e;
        ++outer;
        if (it == 0) {
            code = h.code ? h.code : kErrMaxIt;
            if ((e = apply_residual(c, *A, b, x64, r64))) return e;
            v_norm2(c, n, r64, c.dslot + SL_T1);
            rn = fetch(c.dslot + SL_T1);
            break;
        }
    }
    info->numIter = total;
    info->outerIter = outer;
    info->code = code;
    info->norm2 = rn;
    v_norminf(c, n, r64, c.dslot + SL_T2);
    info->normInf = fetch(c.dslot + SL_T2);
    v_copy(c, n, x64, x);
    const uint32_t len = std::min<uint32_t>(total + 1, dhistCap);
    hist.assign(len, kNaN);
    FB_CUDA(cudaMemcpyAsync(hist.data(), dhist, (size_t)len * 8, cudaMemcpyDeviceToHost, c.stream));
    FB_CUDA(cudaStreamSynchronize(c.stream));
    for (auto& pt : outerHist) rec(pt.first, pt.second);
    return kOk;
}

// Mixed precision with reliable updates (no reference counterpart): one FP32 PCG run whose
// vectors are scaled by s = ||b - A x0||. Whenever the FP32 recursive residual meets the
// stop test or has fallen by delta (innerRelTol) since the last refresh, the host folds the
// FP32 correction into x in FP64 (x += s e, e = 0), recomputes r = b - A x in FP64, stops
// if ||r|| / ||r0|| < relTol (or ||r|| < absTol), and otherwise continues the same Krylov
// process from the refreshed residual: p is kept and beta = (z, r) / (z, r)_old uses the
// refreshed r (the reliable-update scheme of Sleijpen and van der Vorst, 1996). Unlike
// restarted refinement the conjugate directions survive each refresh, so the iteration
// count stays that of FP64 CG while the SpMV and vector traffic is FP32.
int SolverImpl::cg_reliable(const double* b, double* x, fasp_gpu_info* info)
{
    const fasp_gpu_params& P = cfg.prm;
    CGEngine<float>& E = *cg32;
    CGCtl& h = *E.hctl;
    double *x64 = w[0], *r64 = w[1];
    int e;
    v_copy(c, n, x, x64);
    const double delta = cfg.innerRelTol > 0 && cfg.innerRelTol < 1 ? cfg.innerRelTol : 1e-2;
    ++c.launches;
    k_fill<<<c.grid(dhistCap, kBlock), kBlock, 0, c.stream>>>(dhistCap, kNaN, dhist);
    std::vector<std::pair<uint32_t, double>> patches;
    auto true_res = [&](double* rn) {
        int err = apply_residual(c, *A, b, x64, r64);
        if (err) return err;
        if ((err = v_norm2(c, n, r64, c.dslot + SL_T1))) return err;
        *rn = fetch(c.dslot + SL_T1);
        return (int)kOk;
    };
    double rn = 0.0;
    if ((e = true_res(&rn))) return e;
    const double den = (kCloseZero > rn) ? kCloseZero : rn;
    double hostPrev = den;
    patches.push_back({0u, rn});
    int code = kOk;
    uint32_t iters = 0, refreshes = 0, hostRefreshes = 0, hostStall = 0;
    bool converged = rn / den < P.relTol || rn < P.absTol;
    if (!converged && std::isfinite(rn) && P.maxIter > 0) {
        const double s = rn;
        if ((e = convert_scaled(c, n, r64, 1.0 / s, E.r)) || (e = set32(c, n, E.x))) return e;
        std::memset(&h, 0, sizeof(CGCtl));
        h.maxIter = P.maxIter;
        h.minIter = 0;
        h.savIter = 0xffffffffu;
        h.inner = 1;
        h.reliable = 1;
        h.innerTol = P.relTol * den / s;
        h.relTol = P.relTol;
        h.absTol = P.absTol;
        h.absTolIn = P.absTol / s;
        h.delta = delta;
        h.hist = dhist;
        h.histCap = dhistCap;
        h.histScale = s;
        // graph and plain engines refresh inside their kernels; the persistent one escalates
        h.devRefresh = E.persistent ? 0 : 1;
        h.den64 = den;
        h.resPrev = den;
        h.rb = b;
        h.rx = x64;
        h.rr = r64;
        h.rval = A->val;
        h.rcval = A->rcVal;
        for (int u = 0; u < kMaxStencil; ++u) {
            h.skval[u] = A->skVal[u];
            h.skdelta[u] = A->skDelta[u];
        }
        if ((e = E.push_ctl()) || (e = E.launch_init()) || (e = E.pull_ctl())) return e;
        h.rmax = h.resAbs;
        if ((e = E.push_ctl())) return e;
        for (uint32_t guard = 0;; ++guard) {
            if (h.status == kRun || h.status == kRefresh) {
                unsigned gl = 0;
                if ((e = E.run(&gl)) || (e = E.pull_ctl())) return e;
                c.launches += gl;
                continue;
            }
            if (h.status == kDone && h.converged) { // the last device refresh passed the test
                rn = h.res64;
                converged = true;
                break;
            }
            if (h.status == kDone && h.code == kErrTolSmall) { // refreshes stopped gaining
                rn = h.res64;
                code = kErrTolSmall;
                break;
            }
            // a host refresh: the stop test or delta reached (persistent engine), or the end
            // of the FP32 run (maxIter, breakdown)
            TraceRange refresh("fasp reliable refresh");
            if ((e = E.apply_pending_x()) || (e = update_from32(c, n, s, E.x, x64)) ||
                (e = set32(c, n, E.x)))
                return e;
            if ((e = true_res(&rn))) return e;
            ++hostRefreshes;
            patches.push_back({h.numIter, rn});
            converged = rn / den < P.relTol || rn < P.absTol;
            hostStall = rn > std::sqrt(delta) * hostPrev ? hostStall + 1 : 0;
            hostPrev = rn;
            if (!converged && hostStall >= 3) code = kErrTolSmall;
            if (h.status == kDone || converged || !std::isfinite(rn) || guard > P.maxIter ||
                code != kOk) {
                if (h.status == kDone && h.code != kOk) code = h.code;
                break;
            }
            if ((e = convert_scaled(c, n, r64, 1.0 / s, E.r))) return e;
            if (rn / s > 4.0 * h.resAbs) h.pzero = 1; // see cg_after_refresh
            h.rmax = rn / s;
            h.phase = 1;
            if ((e = E.push_ctl()) || (e = E.launch_resume()) || (e = E.pull_ctl())) return e;
        }
        iters = h.numIter;
        refreshes = hostRefreshes + h.refreshes;
    }
    if (!converged && code == kOk) code = kErrMaxIt;
    info->numIter = iters;
    info->outerIter = refreshes;
    info->escalations = hostRefreshes;
    info->code = code;
    info->norm2 = rn;
    v_norminf(c, n, r64, c.dslot + SL_T2);
    info->normInf = fetch(c.dslot + SL_T2);
    v_copy(c, n, x64, x);
    const uint32_t len = std::min<uint32_t>(iters + 1, dhistCap);
    hist.assign(len, kNaN);
    FB_CUDA(cudaMemcpyAsync(hist.data(), dhist, (size_t)len * 8, cudaMemcpyDeviceToHost, c.stream));
    FB_CUDA(cudaStreamSynchronize(c.stream));
    for (auto& pt : patches) rec(pt.first, pt.second);
    return kOk;
}

// BiCGStab with reliable updates (no reference counterpart; the scheme of cg_reliable): the
// FP32 engine iterates on the residual scaled by s = ||b - A x0|| and accumulates its
// correction e. Whenever its recursive residual has fallen by delta (innerRelTol, default
// 1e-3: the fewest refreshes without extra iterations on B200 at 96^3) since the
// last refresh, or meets the stop test, or the run ends, the host folds x += s e in FP64,
// recomputes r = b - A x in FP64 and stops if ||r|| / ||r0|| < relTol (or ||r|| < absTol);
// otherwise the same Krylov process continues from the refreshed residual: p and r0* are
// kept, (r, r0*) and beta come from the refreshed r (bi_resume at phase 3). The save and
// stagnation tests of the reference look at the whole solution, which the FP32 correction
// is not, so they are off; a refresh that gains less than sqrt(delta) three times in a row
// ends the solve with ERROR_SOLVER_TOLSMALL.
int SolverImpl::bicgstab_reliable(const double* b, double* x, fasp_gpu_info* info)
{
    const fasp_gpu_params& P = cfg.prm;
    if (!bi32) return kErrPcdType;
    BiEngine<float>& E = *bi32;
    BiCtl& h = *E.hctl;
    double *x64 = w[0], *r64 = w[1];
    int e;
    v_copy(c, n, x, x64);
    const double delta = cfg.innerRelTol > 0 && cfg.innerRelTol < 1 ? cfg.innerRelTol : 1e-3;
    ++c.launches;
    k_fill<<<c.grid(dhistCap, kBlock), kBlock, 0, c.stream>>>(dhistCap, kNaN, dhist);
    std::vector<std::pair<uint32_t, double>> patches;
    auto true_res = [&](double* rn) {
        int err = apply_residual(c, *A, b, x64, r64);
        if (err) return err;
        if ((err = v_norm2(c, n, r64, c.dslot + SL_T1))) return err;
        *rn = fetch(c.dslot + SL_T1);
        return (int)kOk;
    };
    double rn = 0.0;
    if ((e = true_res(&rn))) return e;
    const double den = (kCloseZero > rn) ? kCloseZero : rn;
    patches.push_back({0u, rn});
    int code = kOk;
    uint32_t iters = 0, refreshes = 0, stall = 0;
    double prev = den;
    bool converged = rn / den < P.relTol || rn < P.absTol;
    if (!converged && std::isfinite(rn) && P.maxIter > 0) {
        const double s = rn;
        // e = 0, r = (b - A x) / s, r0* = p = r (BiCGStab.cxx:70-78 on the scaled system;
        // the first bi_p forms p = r from zeroed direction buffers and beta = omega = 0)
        if ((e = convert_scaled(c, n, r64, 1.0 / s, E.rj)) || (e = set32(c, n, E.x))) return e;
        v_copy(c, n, (const float*)E.rj, E.r0s);
        if ((e = set32(c, n, E.pj(0))) || (e = set32(c, n, E.ptmp2[0]))) return e;
        std::memset(&h, 0, sizeof(BiCtl));
        h.status = kRun;
        h.code = kOk;
        h.minIter = 0;
        h.maxIter = P.maxIter;
        h.savIter = 0xffffffffu;
        h.restart = P.restart;
        h.relTol = P.relTol * den / s;
        h.absTol = P.absTol / s;
        h.solStagTol = 0.0;           // no solution-stagnation stop on the correction
        h.stagStep = kMaxStagNum + 1; // nor a stagnation restart
        h.resAbs = h.resRel = h.denAbs = h.resAbsOld = 1.0;
        h.hist = dhist;
        h.histCap = dhistCap;
        h.histOffset = 0;
        h.histScale = s;
        h.reliable = 1;
        h.delta = delta;
        h.rmax = 1.0; // ||r / s|| at the start
        if ((e = E.push_ctl())) return e;
        unsigned launches = 0;
        for (uint32_t guard = 0;; ++guard) {
            if (h.status == kRun) {
                if ((e = E.run(&launches)) || (e = E.pull_ctl())) return e;
                c.launches += launches;
                launches = 0;
                continue;
            }
            // a refresh, the FP32 stop test, or the end of the run (maxIter, breakdown)
            TraceRange refresh("fasp reliable refresh");
            if ((e = update_from32(c, n, s, E.x, x64)) || (e = set32(c, n, E.x))) return e;
            if ((e = true_res(&rn))) return e;
            ++refreshes;
            patches.push_back({h.numIter, rn});
            converged = rn / den < P.relTol || rn < P.absTol;
            stall = rn > std::sqrt(delta) * prev ? stall + 1 : 0;
            prev = rn;
            if (!converged && stall >= 3) code = kErrTolSmall;
            if (h.status == kDone || converged || !std::isfinite(rn) || guard > P.maxIter ||
                code != kOk) {
                if (!converged && h.status == kDone && h.code != kOk) code = h.code;
                break;
            }
            if ((e = convert_scaled(c, n, r64, 1.0 / s, E.rj))) return e;
            h.resAbs = rn / s;
            h.resRel = h.resAbs / h.denAbs;
            h.rmax = h.resAbs;
            h.phase = 3;
            h.status = kRun;
            if ((e = E.push_ctl()) || (e = E.launch_resume()) || (e = E.pull_ctl())) return e;
        }
        iters = h.numIter;
    }
    if (!converged && code == kOk) code = kErrMaxIt;
    info->numIter = iters;
    info->outerIter = refreshes;
    info->escalations = refreshes;
    info->code = code;
    info->norm2 = rn;
    v_norminf(c, n, r64, c.dslot + SL_T2);
    info->normInf = fetch(c.dslot + SL_T2);
    v_copy(c, n, x64, x);
    const uint32_t len = std::min<uint32_t>(iters + 1, dhistCap);
    hist.assign(len, kNaN);
    FB_CUDA(cudaMemcpyAsync(hist.data(), dhist, (size_t)len * 8, cudaMemcpyDeviceToHost, c.stream));
    FB_CUDA(cudaStreamSynchronize(c.stream));
    for (auto& pt : patches) rec(pt.first, pt.second);
    return kOk;
}

// ---- BiCGStab (src/BiCGStab.cxx:68-270) ---------------------------------------------------

template <typename T>
int SolverImpl::bicgstab(const T* b, T* x, fasp_gpu_info* info, const fasp_gpu_params& P,
                         Space<T> S)
{
    if constexpr (std::is_same<T, double>::value) {
        if (bi64) return bicgstab_engine(*bi64, b, x, info, P, S);
    } else {
        if (bi32) return bicgstab_engine(*bi32, b, x, info, P, S);
    }
    std::vector<T*>& w = *S.w;
    T *r0star = w[0], *tmp = w[1], *apj = w[2], *asj = w[3], *pj = w[4], *rj = w[5],
      *sj = w[6], *ptmp = w[7], *stmp = w[8], *ms = w[9], *mp = w[10], *sv = w[11];
    double* d = c.dslot;
    int err = kOk, e;
    const unsigned maxStag = kMaxStagNum;
    const double solStagTol = 1e-4 * P.relTol;
    unsigned stagStep = 0, moreStep = 0;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, ratio = 0.0, resAbsOld = 1.0;
    double alpha = 0.0, beta, rjr0star = 0.0, rjr0startmp, omega = 0.0, tmp12;
    uint32_t numIter = 0;

    m_spmv(c, *A, x, tmp);
    v_waxpby(c, n, Scal::h(1.0), b, Scal::h(-1.0), tmp, rj);
    v_copy(c, n, rj, r0star);
    v_copy(c, n, rj, pj);

    while (numIter < P.maxIter) {
        if (numIter == P.minIter) {
            v_norm2(c, n, rj, d + SL_T1);
            resAbs = fetch(d + SL_T1);
            denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;
            resRel = resAbs / denAbs;
            rec(numIter, resAbs);
            if (resRel < P.relTol || resAbs < P.absTol) break;
        }
        ++numIter;
        v_dot(c, n, rj, r0star, d + SL_T0);
        m_spmv(c, *A, pj, apj);
        v_set(c, n, 0.0, ptmp);
        if ((e = pcd.solve(c, apj, ptmp))) return e;
        v_dot(c, n, ptmp, r0star, d + SL_T2);
        rjr0star = fetch(d + SL_T0);
        tmp12 = fetch(d + SL_T2);
        if (std::fabs(tmp12) > 1e-40)
            alpha = rjr0star / tmp12;
        else {
            err = kErrDivZero;
            rec(numIter, resAbs);
            break;
        }
        v_waxpby(c, n, Scal::h(1.0), rj, Scal::h(-alpha), ptmp, sj);
        m_spmv(c, *A, sj, asj);
        v_set(c, n, 0.0, stmp);
        if ((e = pcd.solve(c, asj, stmp))) return e;
        v_dot(c, n, stmp, sj, d + SL_T3);
        v_dot(c, n, stmp, stmp, d + SL_T4);
        omega = fetch(d + SL_T3) / fetch(d + SL_T4);
        v_set(c, n, 0.0, mp);
        if ((e = pcd.solve(c, pj, mp))) return e;
        v_set(c, n, 0.0, ms);
        if ((e = pcd.solve(c, sj, ms))) return e;
        v_waxpby(c, n, Scal::h(alpha), mp, Scal::h(omega), ms, tmp);
        v_xpay(c, n, Scal::h(1.0), tmp, x);
        v_waxpby(c, n, Scal::h(1.0), sj, Scal::h(-omega), stmp, rj);

        if (numIter >= P.minIter) {
            bool stop = false;
            v_norm2(c, n, rj, d + SL_T1);
            resAbs = fetch(d + SL_T1);
            resRel = resAbs / denAbs;
            ratio = resAbs / resAbsOld;
            if (numIter >= P.savIter && resAbs < resAbsOld) v_copy(c, n, x, sv);
            if (ratio > kKsmChkRatio && numIter > P.minIter) {
                v_norminf(c, n, x, d + SL_T2);
                const double xNorminf = fetch(d + SL_T2);
                if (xNorminf < solStagTol) {
                    err = kErrSolStag;
                    stop = true;
                } else {
                    v_norm2(c, n, pj, d + SL_T3);
                    v_norm2(c, n, x, d + SL_T4);
                    const double xRelDiff =
                        std::fabs(alpha) * fetch(d + SL_T3) / fetch(d + SL_T4);
                    if ((stagStep <= maxStag) && (xRelDiff < solStagTol)) {
                        apply_residual(c, *A, b, x, rj);
                        v_norm2(c, n, rj, d + SL_T1);
                        resAbs = fetch(d + SL_T1);
                        resRel = resAbs / denAbs;
                        if (resRel < P.relTol || resAbs < P.absTol)
                            stop = true;
                        else if (stagStep >= maxStag) {
                            err = kErrStag;
                            stop = true;
                        } else {
                            v_set(c, n, 0.0, pj);
                            ++stagStep;
                        }
                    }
                }
            }
            if (!stop && resRel < P.relTol) {
                apply_residual(c, *A, b, x, rj);
                v_norm2(c, n, rj, d + SL_T1);
                resAbs = fetch(d + SL_T1);
                resRel = resAbs / denAbs;
                if (resRel < P.relTol || resAbs < P.absTol)
                    stop = true;
                else if (moreStep >= P.restart) {
                    err = kErrTolSmall;
                    stop = true;
                } else {
                    v_set(c, n, 0.0, pj);
                    ++moreStep;
                }
            }
            rec(numIter, resAbs);
            if (stop) break;
        }
        if (numIter < P.maxIter) {
            resAbsOld = resAbs;
            rjr0startmp = rjr0star;
            v_dot(c, n, rj, r0star, d + SL_T0);
            rjr0star = fetch(d + SL_T0);
            beta = rjr0star / rjr0startmp * alpha / omega;
            v_waxpby(c, n, Scal::h(1.0), pj, Scal::h(-omega), ptmp, tmp);
            v_waxpby(c, n, Scal::h(1.0), rj, Scal::h(beta), tmp, pj);
        }
    }
    info->numIter = numIter;
    info->code = err;
    if (!(numIter == P.minIter && numIter == P.maxIter)) {
        info->norm2 = resAbs;
        v_norminf(c, n, rj, d + SL_T2);
        info->normInf = fetch(d + SL_T2);
    }
    if (numIter > P.savIter) v_copy(c, n, sv, x);
    FB_CUDA(cudaStreamSynchronize(c.stream));
    return kOk;
}

// Device-driven BiCGStab: the same control flow as bicgstab() above, run by the kernels of
// bicgstab.cu; the host finishes the branches they escalate (BiCGStab.cxx references).
template <typename T>
int SolverImpl::bicgstab_engine(BiEngine<T>& E, const T* b, T* x, fasp_gpu_info* info,
                                const fasp_gpu_params& P, Space<T> S)
{
    BiCtl& h = *E.hctl;
    T* sv = (*S.w)[11];
    std::vector<std::pair<uint32_t, double>> patches; // raw values, recorded through rec()
    int e;
    // BiCGStab.cxx:70-78: rj = b - A x, r0star = rj, pj = rj (the first bi_p forms pj =
    // rj + beta (pj(0) - omega ptmp(0)) with beta = omega = 0 from zeroed buffers)
    v_copy(c, n, (const T*)x, E.x);
    if ((e = m_spmv(c, *A, (const T*)E.x, E.sj))) return e;
    v_waxpby(c, n, Scal::h(1.0), b, Scal::h(-1.0), (const T*)E.sj, E.rj);
    v_copy(c, n, (const T*)E.rj, E.r0s);
    v_set(c, n, 0.0, E.pj(0));
    v_set(c, n, 0.0, E.ptmp2[0]);
    std::memset(&h, 0, sizeof(BiCtl));
    h.status = P.maxIter > 0 ? kRun : kDone;
    h.code = kOk;
    h.minIter = P.minIter;
    h.maxIter = P.maxIter;
    h.savIter = P.savIter;
    h.restart = P.restart;
    h.relTol = P.relTol;
    h.absTol = P.absTol;
    h.solStagTol = 1e-4 * P.relTol;
    h.resAbs = h.resRel = h.denAbs = h.resAbsOld = 1.0;
    h.hist = dhist;
    h.histCap = dhistCap;
    h.histOffset = histOff;
    h.histScale = histScale;
    ++c.launches;
    k_fill<<<c.grid(dhistCap, kBlock), kBlock, 0, c.stream>>>(dhistCap, kNaN, dhist);
    if ((e = E.push_ctl())) return e;
    unsigned launches = 0;
    info->escalations = 0;
    auto true_res = [&]() { // rj = b - A x, resAbs, resRel (BiCGStab.cxx:146-149, 166-169)
        apply_residual(c, *A, b, (const T*)E.x, E.rj);
        v_norm2(c, n, (const T*)E.rj, c.dslot + SL_T1);
        h.resAbs = fetch(c.dslot + SL_T1);
        h.resRel = h.resAbs / h.denAbs;
    };
    for (uint32_t guard = 0; h.status != kDone; ++guard) {
        if (h.status == kRun) {
            if ((e = E.run(&launches)) || (e = E.pull_ctl())) return e;
            c.launches += launches;
            launches = 0;
            continue;
        }
        info->escalations++;
        bool stop = false;
        if (h.reason == kBiSave) { // :133
            v_copy(c, n, (const T*)E.x, sv);
        } else if (h.reason == kBiStag) { // :144-162
            true_res();
            if (h.resRel < P.relTol || h.resAbs < P.absTol) {
                stop = true;
            } else if (h.stagStep >= kMaxStagNum) {
                h.code = kErrStag;
                stop = true;
            } else {
                v_set(c, n, 0.0, E.pj(h.par));
                ++h.stagStep;
            }
        } else if (h.reason == kBiCheck) { // :164-175
            true_res();
            if (h.resRel < P.relTol || h.resAbs < P.absTol) {
                stop = true;
            } else if (h.moreStep >= P.restart) {
                h.code = kErrTolSmall;
                stop = true;
            } else {
                v_set(c, n, 0.0, E.pj(h.par));
                ++h.moreStep;
            }
        }
        if (stop) { // rec(numIter, resAbs) and leave the loop (:176-177)
            patches.push_back({h.numIter, h.resAbs});
            h.status = kDone;
            if ((e = E.push_ctl())) return e;
            break;
        }
        h.status = kRun;
        if ((e = E.push_ctl()) || (e = E.launch_resume()) || (e = E.pull_ctl())) return e;
        if (guard > P.maxIter + 64) return kErrCuda; // cannot happen: each pass advances
    }
    info->numIter = h.numIter;
    info->code = h.code;
    if (!(h.numIter == P.minIter && h.numIter == P.maxIter)) {
        info->norm2 = h.resAbs;
        v_norminf(c, n, (const T*)E.rj, c.dslot + SL_T2);
        info->normInf = fetch(c.dslot + SL_T2);
    }
    v_copy(c, n, (const T*)E.x, x);
    if (h.numIter > P.savIter) v_copy(c, n, (const T*)sv, x);
    // the device recorded scaled entries at histOff + k; the host's through rec()
    const uint32_t len = std::min<uint32_t>(histOff + h.numIter + 1, dhistCap);
    std::vector<double> dh(len, kNaN);
    FB_CUDA(cudaMemcpyAsync(dh.data(), dhist, (size_t)len * 8, cudaMemcpyDeviceToHost, c.stream));
    FB_CUDA(cudaStreamSynchronize(c.stream));
    if (hist.size() < len) hist.resize(len, kNaN);
    for (uint32_t k = histOff; k < len; ++k)
        if (std::isfinite(dh[k])) hist[k] = dh[k];
    for (auto& pt : patches) rec(pt.first, pt.second);
    return kOk;
}

// ---- GMRES / FGMRES: the Hessenberg least-squares stays in FP64 on the device -----------

// GMRES.cxx:168-203 after the dots: hh[j][c1] (CGS2: h1+h2), t = ||w||, then the Givens
// step of gm_givens_serial on a shared-memory copy of the column.
__global__ void __launch_bounds__(128) k_gmres_givens(GmLayout L, int count, int c1, int cgs,
                                                      const double* tnorm, GmCtl* g)
{
    pdl_wait(); // launched programmatically
    pdl_release();
    if (g && g->stop) return;
    const size_t m = L.m;
#define HH(i, j) L.hh[(size_t)(i) * m + (j)]
    // the column c1, the previous rotations, var[c1] and the control block, loaded by all
    // threads at once; one thread then runs the reference's serial sequence on shared
    // memory, with the same operations and order
    __shared__ double col[kGmShared + 1], sn[kGmShared], cs[kGmShared], var[2];
    __shared__ GmCtl gs;
    const bool sh = count <= kGmShared;
    if (sh) {
        for (int j = threadIdx.x; j < count; j += blockDim.x) {
            col[j] = cgs ? L.h1[j] + L.h2[j] : HH(j, c1);
            sn[j] = L.hsin[j];
            cs[j] = L.hcos[j];
        }
    }
    if (threadIdx.x == 32) var[0] = L.var[c1];
    if (threadIdx.x == 64 && g) gs = *g;
    __syncthreads();
    if (threadIdx.x == 0) {
        if (!sh && cgs)
            for (int j = 0; j < count; ++j) HH(j, c1) = L.h1[j] + L.h2[j];
        auto C = [&](int j) -> double& { return sh ? col[j] : HH(j, c1); };
        auto S = [&](int j) { return sh ? sn[j] : L.hsin[j]; };
        auto K = [&](int j) { return sh ? cs[j] : L.hcos[j]; };
        auto Var = [&](int j) -> double& { return var[j == c1 ? 0 : 1]; };
        var[1] = L.var[count];
        gm_givens_serial(L, count, c1, *tnorm, C, S, K, Var, g ? &gs : nullptr);
        L.var[c1] = var[0];
        L.var[count] = var[1];
        if (g) *g = gs;
    }
    if (sh) {
        __syncthreads();
        for (int j = threadIdx.x; j <= count; j += blockDim.x) HH(j, c1) = col[j];
    }
#undef HH
}

// GMRES.cxx:213-219 (signed loop): back substitution into var[0..count)
// Restart lengths up to 64 stage the triangle and var in shared memory (loaded by all
// threads at once) before thread 0 runs the same serial sequence: one thread's dependent
// global loads had cost about 40 us per cycle.
constexpr int kGmBack = 64;

__global__ void __launch_bounds__(128) k_gmres_backsolve(GmLayout L, int count, int c1)
{
    const size_t m = L.m;
#define HH(i, j) L.hh[(size_t)(i) * m + (j)]
    __shared__ double hs[kGmBack * kGmBack], vs[kGmBack];
    if (count < 1) return; // every cycle makes at least one step
    if (count <= kGmBack) {
        for (int e = threadIdx.x; e < count * count; e += blockDim.x) {
            const int i = e / count, j = e - i * count;
            if (j >= i) hs[e] = HH(i, j);
        }
        for (int i = threadIdx.x; i < count; i += blockDim.x) vs[i] = L.var[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            vs[c1] = vs[c1] / hs[c1 * count + c1];
            for (int k = count - 2; k >= 0; --k) {
                double t = 0.0;
                for (int j = k + 1; j < count; ++j) t -= hs[k * count + j] * vs[j];
                t += vs[k];
                vs[k] = t / hs[k * count + k];
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < count; i += blockDim.x) L.var[i] = vs[i];
        return;
    }
    if (threadIdx.x != 0) return;
    L.var[c1] = L.var[c1] / HH(c1, c1);
    for (int k = count - 2; k >= 0; --k) {
        double t = 0.0;
        for (int j = k + 1; j < count; ++j) t -= HH(k, j) * L.var[j];
        t += L.var[k];
        L.var[k] = t / HH(k, k);
    }
#undef HH
}

__global__ void k_set_scalar(double* dst, double v) { *dst = v; }

template <typename T>
static int orthogonalize(SolverImpl& S, const GmLayout& L, int count, int c1, const T* V, T* wv)
{
    Ctx& c = S.c;
    const uint32_t n = S.n;
    const size_t ld = S.ldV;
    double* tn = c.dslot + SL_T5;
    if (S.cfg.orth == FASP_GPU_ORTH_MGS) { // GMRES.cxx:169-172
        for (int j = 0; j < count; ++j) {
            double* hj = L.hh + (size_t)j * L.m + c1;
            v_dot(c, n, (const T*)wv, V + j * ld, hj);
            v_axpby(c, n, Scal::h(1.0), Scal::d(hj, -1.0), V + j * ld, wv);
        }
        v_norm2(c, n, (const T*)wv, tn);
    } else { // CGS2: two fused multi-dot / multi-AXPY passes
        v_multidot(c, n, count, V, ld, (const T*)wv, L.h1);
        v_multiaxpy_dot(c, n, count, V, ld, L.h1, wv, L.h2);
        v_multiaxpy(c, n, count, V, ld, L.h2, 1.0, wv, tn);
    }
    ++c.launches;
    FB_CUDA(launch_pdl(k_gmres_givens, dim3(1), dim3(128), 0, c.stream, L, count, c1,
                       (int)(S.cfg.orth != FASP_GPU_ORTH_MGS), (const double*)tn,
                       (GmCtl*)nullptr));
    FB_CUDA(cudaGetLastError());
    v_scale(c, n, Scal::dinv(tn), wv);
    return kOk;
}

// ---- restart cycles without host round trips (Identity or one Jacobi sweep, CGS2) -------

bool SolverImpl::gm_device_cycles(bool flexible) const
{
    // Identity or one Jacobi sweep (from zero for GMRES, from the warm start Z_j for
    // FGMRES); MGS keeps the reference's per-vector op sequence with a host-read scalar
    (void)flexible;
    return gmc && dhist && (A->val || A->grid) && cfg.orth != FASP_GPU_ORTH_MGS &&
           (pcd.type == 0 || (pcd.pure() && pcd.prm.maxIter == 1));
}

// The preconditioned product of an Arnoldi step: mode 0 y = A v (Identity), 1 y = A (D v)
// (right Jacobi from zero: the sweep is diagInv .* v), 2 y = D (A v) (left Jacobi).
template <typename T, int L, int MODE>
__global__ void __launch_bounds__(kBlock) k_gm_apply(CSRView<T> A, const T* __restrict__ v,
                                                     const T* __restrict__ dinv,
                                                     T* __restrict__ y, const int* stop)
{
    if (*stop) return;
    auto xv = [&](uint32_t j) { return MODE == 1 ? v[j] * dinv[j] : v[j]; };
    auto out = [&](size_t row, T sum) { y[row] = MODE == 2 ? sum * dinv[row] : sum; };
    if (L == 1) { // thread per row, or block tiles of plain CSR (A.tiles)
        for_rows<T, false>(A, xv, out);
        return;
    }
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
        if (lane == 0 && row < A.nrow) out(row, sum);
    }
}

// The same product on stencil masks of the fixed 5- or 7-point shape SH: W consecutive rows
// per thread in 16-byte groups (stencil_group, as MAT::Apply's vector-row kernel), the
// preconditioner folded into the gather (mode 1: v .* diagInv per element) or the result
// (mode 2). Each row sum is the one k_gm_apply forms, bit for bit.
template <typename T, int SH, int MODE>
__global__ void __launch_bounds__(kBlock) k_gm_apply_vec(CSRView<T> A, const T* __restrict__ v,
                                                         const T* __restrict__ dinv,
                                                         T* __restrict__ y, const int* stop)
{
    pdl_wait(); // launched programmatically in the DCGS2 cycles: v may still be in flight
    pdl_release();
    if (*stop) return;
    using VT = Vec16<T>;
    using V = typename VT::V;
    constexpr int W = VT::W;
    const uint32_t nw = A.nrow / W, stride = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31u;
    const V* vv = reinterpret_cast<const V*>(v);
    const V* dv = reinterpret_cast<const V*>(dinv);
    V* yv = reinterpret_cast<V*>(y);
    auto gather = [&](uint32_t h) {
        const V a = vv[h];
        if (MODE != 1) return a;
        const V d = dv[h];
        T t[W];
#pragma unroll
        for (int e = 0; e < W; ++e) t[e] = VT::at(a, e) * VT::at(d, e);
        return VT::make(t);
    };
    // the loop bound is the same on every lane of a warp (all lanes shuffle)
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g - lane < nw; g += stride) {
        const bool act = g < nw;
        T s[W];
#pragma unroll
        for (int e = 0; e < W; ++e) s[e] = T(0);
        V c;
        stencil_group<T, SH>(A, g, nw, act, gather, c, s);
        if (act) {
            if (MODE == 2) {
                const V d = dv[g];
#pragma unroll
                for (int e = 0; e < W; ++e) s[e] = s[e] * VT::at(d, e);
            }
            yv[g] = VT::make(s);
        }
    }
}

// w *= 1 / t (Scale by a device scalar, as v_scale(Scal::dinv(t)))
template <typename T>
__global__ void k_gm_scale(uint32_t n, const double* __restrict__ tn, T* __restrict__ w,
                           const int* stop)
{
    pdl_wait(); // launched programmatically
    pdl_release();
    if (*stop) return;
    const T inv = (T)(1.0 / *tn);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        w[i] *= inv;
}

// FGMRES with one Jacobi sweep from the warm start Z_j (Jacobi::Solve with minIter =
// maxIter = 1, Iter.cxx:56-112, as FGMRES.cxx:158-159 calls it): NormInf(Z_j) for the
// residual's shortcut, then t = Z_j + diagInv .* (V_j - A Z_j) into a work vector; the
// step's product A t stores t back into Z_j (k_fg_apply), so every gather reads the old Z_j.
template <typename T>
__global__ void k_fg_norminf(uint32_t n, const T* __restrict__ z, Scratch s, double* dres,
                             const int* stop)
{
    pdl_wait(); // launched programmatically
    pdl_release();
    if (*stop) return;
    T m = T(0);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(z[i]));
    double acc[1] = {(double)m};
    const int ops[1] = {kMax};
    grid_reduce<1>(acc, ops, s, [=] __device__(const double* t) { *dres = t[0]; });
}

template <typename T, int L>
__global__ void __launch_bounds__(kBlock) k_fg_sweep(CSRView<T> A, const T* __restrict__ v,
                                                     const T* __restrict__ zj,
                                                     const T* __restrict__ dinv,
                                                     const double* __restrict__ zinf,
                                                     T* __restrict__ t, const int* stop)
{
    pdl_wait(); // launched programmatically
    pdl_release();
    if (*stop) return;
    const bool shortcut = *zinf < kCloseZero; // MAT::Residual (MAT.cxx:459-462)
    auto xv = [&](uint32_t j) { return zj[j]; };
    auto out = [&](size_t row, T sum) {
        const T work = v[row] - sum;
        t[row] = zj[row] + work * dinv[row];
    };
    if (L == 1) {
        for (size_t row = (size_t)blockIdx.x * blockDim.x + threadIdx.x; row < A.nrow;
             row += (size_t)gridDim.x * blockDim.x)
            out(row, shortcut ? T(0) : row_apply<T, false>(A, row, xv));
        return;
    }
    const int lane = threadIdx.x & (L - 1);
    const size_t warpRows = 32 / L;
    const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
    const size_t sub = (threadIdx.x & 31) / L;
    for (size_t base = gw * warpRows; base < A.nrow; base += nwarps * warpRows) {
        const size_t row = base + sub;
        T sum = T(0);
        if (row < A.nrow && !shortcut)
            for (uint32_t k = A.rowPtr[row] + lane; k < A.rowPtr[row + 1]; k += L)
                sum = fma(A.val[k], xv(A.colInd[k]), sum);
        sum = group_sum<L>(sum);
        if (lane == 0 && row < A.nrow) out(row, sum);
    }
}

// y = A t and z = t (the preconditioned basis vector Z_j of FGMRES, FGMRES.cxx:159-160)
template <typename T, int L>
__global__ void __launch_bounds__(kBlock) k_fg_apply(CSRView<T> A, const T* __restrict__ t,
                                                     T* __restrict__ z, T* __restrict__ y,
                                                     const int* stop)
{
    pdl_wait(); // launched programmatically
    pdl_release();
    if (*stop) return;
    auto xv = [&](uint32_t j) { return t[j]; };
    if (L == 1) { // thread per row, or block tiles of plain CSR (A.tiles)
        for_rows<T, false>(A, xv, [&](size_t row, T sum) {
            y[row] = sum;
            z[row] = t[row];
        });
        return;
    }
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
            y[row] = sum;
            z[row] = t[row];
        }
    }
}

template <typename T, typename F>
static void lanes_launch(Ctx& c, const Mat& A, F&& go)
{
    switch (A.lanes) {
        case 1: go(std::integral_constant<int, 1>()); break;
        case 2: go(std::integral_constant<int, 2>()); break;
        case 4: go(std::integral_constant<int, 4>()); break;
        case 8: go(std::integral_constant<int, 8>()); break;
        case 16: go(std::integral_constant<int, 16>()); break;
        default: go(std::integral_constant<int, 32>()); break;
    }
}

template <typename T, int MODE>
static void gm_apply_launch(Ctx& c, const Mat& A, CSRView<T> V, const T* v, const T* dinv,
                            T* y, const int* stop)
{
    if (A.lanes == 1) { // fixed 5- or 7-point stencil masks: 16-byte row groups
        const int sh = stencil_vec_shape(V, v, y, MODE == 0 ? (const void*)v : (const void*)dinv);
        if (sh) {
            auto gv = [&](auto kern) {
                const int g = std::min(c.grid((long long)V.nrow / Vec16<T>::W, kBlock),
                                       resident_grid(c, (const void*)kern, kBlock));
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)g);
                cfg.blockDim = dim3(kBlock);
                cfg.stream = c.stream;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                at[0].val.programmaticStreamSerializationAllowed = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                cudaLaunchKernelEx(&cfg, kern, V, v, dinv, y, stop);
            };
            if (sh == 5)
                gv(k_gm_apply_vec<T, 5, MODE>);
            else
                gv(k_gm_apply_vec<T, 7, MODE>);
            return;
        }
    }
    const int need = c.grid((long long)A.nrow * A.lanes, kBlock);
    const size_t tiles = A.lanes == 1 ? with_tiles(V, kBlock) : 0;
    auto go = [&](auto kern) {
        CSRView<T> W = V;
        size_t smem = tiles;
        if (smem && !tiles_fit((const void*)kern, smem)) W.tiles = 0, smem = 0;
        kern<<<std::min(need, resident_grid(c, (const void*)kern, kBlock, smem)), kBlock, smem,
               c.stream>>>(W, v, dinv, y, stop);
    };
    switch (A.lanes) {
        case 1: go(k_gm_apply<T, 1, MODE>); break;
        case 2: go(k_gm_apply<T, 2, MODE>); break;
        case 4: go(k_gm_apply<T, 4, MODE>); break;
        case 8: go(k_gm_apply<T, 8, MODE>); break;
        case 16: go(k_gm_apply<T, 16, MODE>); break;
        default: go(k_gm_apply<T, 32, MODE>); break;
    }
}

template <typename T>
static CSRView<T> gm_view(const Mat& A);
template <>
CSRView<double> gm_view<double>(const Mat& A) { return A.v64(); }
template <>
CSRView<float> gm_view<float>(const Mat& A) { return A.v32(); }

// Enqueues up to `steps` Arnoldi steps of one restart cycle (GMRES.cxx:160-210 /
// :371-402) with no host synchronisation, then reads the cycle's outcome: count, numIter,
// the last estimate, and merges the device's history records. left: GMRES::LSolve.
template <typename T>
static int gm_cycle_device(SolverImpl& S, const GmLayout& L, T* V, uint32_t steps, bool left,
                           uint32_t& count, uint32_t& numIter, double& resAbs, double denAbs,
                           const fasp_gpu_params& P, int& stopped, T* wbuf, T* Z = nullptr,
                           T* tmp = nullptr)
{
    Ctx& c = S.c;
    const uint32_t n = S.n;
    const size_t ld = S.ldV;
    GmCtl& h = *S.hgmc;
    const uint32_t iter0 = numIter;
    std::memset(&h, 0, sizeof(GmCtl));
    h.numIter = numIter;
    h.minIter = P.minIter;
    h.resAbs = resAbs;
    h.denAbs = denAbs;
    h.relTol = P.relTol;
    h.absTol = P.absTol;
    h.hist = S.dhist;
    h.histCap = S.dhistCap;
    h.histOffset = S.histOff;
    h.histScale = S.histScale;
    FB_CUDA(cudaMemcpyAsync(S.gmc, &h, sizeof(GmCtl), cudaMemcpyHostToDevice, c.stream));
    const int* stop = &S.gmc->stop;
    const CSRView<T> AV = gm_view<T>(*S.A);
    const T* dinv;
    if constexpr (std::is_same<T, float>::value)
        dinv = S.pcd.dinv32;
    else
        dinv = S.pcd.dinv;
    const int mode = S.pcd.type == 0 ? 0 : (left ? 2 : 1);
    double* tn = c.dslot + SL_T5;
    const int needS = c.grid((long long)n * S.A->lanes, kBlock);
    // DCGS2 (dcgs2.cu): step j applies A M to the candidate u_j in slot j, then one dots
    // pass completes iteration j (Hessenberg column j - 1) and one update pass writes q_j and
    // the next candidate; a dots pass without a product closes the cycle
    const bool dc = S.cfg.orth == FASP_GPU_ORTH_DCGS2 && !Z && wbuf && S.maxRestart <= kDcMaxK;
    // FP32 cycles on stencil masks of the fixed 5- or 7-point shape: the dots pass forms the
    // product (96^3 mixed GMRES(30) 11.3 against 11.8 ms); in FP64 the gathers' wait inside
    // the streaming pass cost more than the saved launch (17.9 against 17.5 ms)
    const bool fuse = sizeof(T) == 4 && dc && S.A->lanes == 1 &&
                      stencil_vec_shape(AV, V, wbuf,
                                        mode == 0 ? (const void*)wbuf : (const void*)dinv) != 0;
    for (uint32_t k = 1; dc && k <= steps; ++k) {
        const uint32_t j = k - 1;
        const T* u = V + j * ld;
        int e;
        if (fuse) {
            if ((e = dc_dots_apply<T>(c, AV, mode, dinv, n, (int)j, V, ld, wbuf, L, S.gmc)))
                return e;
        } else {
            if (mode == 0)
                gm_apply_launch<T, 0>(c, *S.A, AV, u, dinv, wbuf, stop);
            else if (mode == 1)
                gm_apply_launch<T, 1>(c, *S.A, AV, u, dinv, wbuf, stop);
            else
                gm_apply_launch<T, 2>(c, *S.A, AV, u, dinv, wbuf, stop);
            ++c.launches;
            if ((e = dc_dots<T>(c, n, (int)j, V, ld, wbuf, L, S.gmc))) return e;
        }
        if ((e = dc_update<T>(c, n, (int)j, V, ld, wbuf, L, S.gmc, fuse))) return e;
    }
    if (dc) {
        int e;
        if ((e = dc_dots<T>(c, n, (int)steps, V, ld, (const T*)nullptr, L, S.gmc))) return e;
    }
    for (uint32_t k = 1; !dc && k <= steps; ++k) {
        const T* vin = V + (k - 1) * ld;
        T* vnew = V + k * ld;
        if (Z) { // FGMRES: Z_{k-1} = P(V_{k-1}) from its warm start, then A Z_{k-1}
            T* zj = Z + (k - 1) * ld;
            const T* t = vin;
            if (S.pcd.type != 0) {
                FB_CUDA(launch_pdl(k_fg_norminf<T>, dim3((unsigned)c.grid(n, kBlock)),
                                   dim3(kBlock), 0, c.stream, n, (const T*)zj, c.red,
                                   c.dslot + SL_T6, stop));
                lanes_launch<T>(c, *S.A, [&](auto LL) {
                    auto kern = k_fg_sweep<T, decltype(LL)::value>;
                    launch_pdl(kern,
                               dim3((unsigned)std::min(
                                   needS, resident_grid(c, (const void*)kern, kBlock))),
                               dim3(kBlock), 0, c.stream, AV, vin, (const T*)zj, dinv,
                               (const double*)(c.dslot + SL_T6), tmp, stop);
                });
                t = tmp;
                c.launches += 2;
            }
            lanes_launch<T>(c, *S.A, [&](auto LL) {
                auto kern = k_fg_apply<T, decltype(LL)::value>;
                CSRView<T> W = AV;
                size_t smem = S.A->lanes == 1 ? with_tiles(W, kBlock) : 0;
                if (smem && !tiles_fit((const void*)kern, smem)) W.tiles = 0, smem = 0;
                launch_pdl(kern,
                           dim3((unsigned)std::min(
                               needS, resident_grid(c, (const void*)kern, kBlock, smem))),
                           dim3(kBlock), smem, c.stream, W, t, zj, vnew, stop);
            });
        } else if (mode == 0)
            gm_apply_launch<T, 0>(c, *S.A, AV, vin, dinv, vnew, stop);
        else if (mode == 1)
            gm_apply_launch<T, 1>(c, *S.A, AV, vin, dinv, vnew, stop);
        else
            gm_apply_launch<T, 2>(c, *S.A, AV, vin, dinv, vnew, stop);
        v_multidot(c, n, (int)k, (const T*)V, ld, (const T*)vnew, L.h1, stop);
        v_multiaxpy_dot(c, n, (int)k, (const T*)V, ld, L.h1, vnew, L.h2, stop);
        v_multiaxpy(c, n, (int)k, (const T*)V, ld, L.h2, 1.0, vnew, tn, stop);
        FB_CUDA(launch_pdl(k_gmres_givens, dim3(1), dim3(128), 0, c.stream, L, (int)k,
                           (int)k - 1, 1, (const double*)tn, S.gmc));
        FB_CUDA(launch_pdl(k_gm_scale<T>, dim3((unsigned)c.grid(n, kBlock)), dim3(kBlock), 0,
                           c.stream, n, (const double*)tn, vnew, stop));
        c.launches += 3;
    }
    FB_CUDA(cudaGetLastError());
    FB_CUDA(cudaMemcpyAsync(&h, S.gmc, sizeof(GmCtl), cudaMemcpyDeviceToHost, c.stream));
    const uint32_t off = S.histOff + iter0 + 1;
    const uint32_t cnt = std::min<uint32_t>(steps, S.dhistCap > off ? S.dhistCap - off : 0);
    std::vector<double> dh(cnt);
    if (cnt)
        FB_CUDA(cudaMemcpyAsync(dh.data(), S.dhist + off, (size_t)cnt * 8,
                                cudaMemcpyDeviceToHost, c.stream));
    FB_CUDA(cudaStreamSynchronize(c.stream));
    count = h.count;
    numIter = h.numIter;
    resAbs = h.resAbs;
    stopped = h.stop;
    for (uint32_t k = 0; k < cnt && iter0 + 1 + k <= numIter; ++k)
        if (std::isfinite(dh[k])) {
            const uint32_t g = off + k;
            if (g >= S.hist.size()) S.hist.resize((size_t)g + 1, kNaN);
            S.hist[g] = dh[k];
        }
    return kOk;
}

static void adapt_restart(SolverImpl& S, double cr, bool inclusive)
{
    const double maxCr = 0.99026806874157040, minCr = 0.17364817766693041;
    const unsigned dec = 3;
    const bool mid = inclusive ? (cr <= maxCr && cr >= minCr) : (cr < maxCr && cr > minCr);
    if (cr > maxCr)
        S.restart = S.maxRestart;
    else if (mid) {
        if (S.restart - dec > S.minRestart) // unsigned, as USI
            S.restart -= dec;
        else
            S.restart = S.maxRestart;
    }
    if (S.restart > S.maxRestart) S.restart = S.maxRestart; // guard against the wrap
}

// GMRES::RSolve (GMRES.cxx:114-280) and FGMRES::Solve (FGMRES.cxx:108-271)
template <typename T>
int SolverImpl::gmres_right(const T* b, T* x, fasp_gpu_info* info, const fasp_gpu_params& P,
                            Space<T> S, bool flexible)
{
    std::vector<T*>& w = *S.w;
    T *wk = w[0], *tmp = w[1], *sv = w[2];
    T *V = S.V, *Z = S.Z;
    const size_t ld = ldV;
    const GmLayout L = gm_layout(gm, maxRestart);
    double* d = c.dslot;
    int err = kOk, e;
    double ri, rj, cr = 1.0;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, resAbsOld = 1.0;
    uint32_t count = 1, count_1 = 2, numIter = 0;

    const bool devCycle = gm_device_cycles(flexible);
    if (devCycle) {
        ++c.launches;
        k_fill<<<c.grid(dhistCap, kBlock), kBlock, 0, c.stream>>>(dhistCap, kNaN, dhist);
    }
    v_copy(c, n, x, sv);
    apply_residual(c, *A, b, x, V);
    v_norm2(c, n, V, d + SL_T1);
    resAbs = ri = fetch(d + SL_T1);
    denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;

    while (numIter < P.maxIter) {
        if (numIter == P.minIter) {
            resRel = resAbs / denAbs;
            resAbsOld = resAbs;
            rec(numIter, resAbs);
            if (resRel < P.relTol || resAbs < P.absTol) break;
        }
        if (resAbs < kSmallDbl) break;
        ++c.launches;
        k_set_scalar<<<1, 1, 0, c.stream>>>(L.var, resAbs);
        v_scale(c, n, Scal::h(1 / resAbs), V);

        count = 0;
        if (devCycle) { // the whole cycle on the device, one synchronisation
            const uint32_t steps = std::min<uint32_t>(restart, P.maxIter - numIter);
            int stopped = 0;
            if ((e = gm_cycle_device<T>(*this, L, V, steps, false, count, numIter, resAbs, denAbs,
                                        P, stopped, wk, flexible ? Z : nullptr, tmp)))
                return e;
            count_1 = count - 1;
            if (!(stopped == 1 && count == 1)) { // a breakdown step updates nothing
                resRel = resAbs / denAbs;
                resAbsOld = resAbs;
            }
        }
        while (!devCycle && count < restart && numIter < P.maxIter) {
            ++numIter;
            count_1 = count++;
            T* vnew = V + count * ld;
            if (flexible) {
                v_set(c, n, 0.0, tmp);
                if ((e = pcd.solve(c, V + count_1 * ld, Z + count_1 * ld))) return e;
                m_spmv(c, *A, Z + count_1 * ld, vnew);
            } else {
                v_set(c, n, 0.0, tmp);
                if ((e = pcd.solve(c, V + count_1 * ld, tmp))) return e;
                m_spmv(c, *A, tmp, vnew);
            }
            if ((e = orthogonalize<T>(*this, L, count, count_1, V, vnew))) return e;
            FB_CUDA(cudaMemcpyAsync(c.hslot + 2, L.out, 16, cudaMemcpyDeviceToHost, c.stream));
            FB_CUDA(cudaStreamSynchronize(c.stream));
            if (c.hslot[3] == 0.0) break;
            resAbs = c.hslot[2];
            resRel = resAbs / denAbs;
            resAbsOld = resAbs;
            rec(numIter, resAbs);
            if ((resAbs < P.absTol || resRel < P.relTol) && numIter > P.minIter) break;
        }

        ++c.launches;

        k_gmres_backsolve<<<1, 128, 0, c.stream>>>(L, (int)count, (int)count_1);
        v_set(c, n, 0.0, wk);
        v_multiaxpy(c, n, (int)count, flexible ? Z : V, ld, L.var, -1.0, wk, nullptr);
        if (flexible) {
            v_axpy(c, n, Scal::h(1.0), wk, x);
        } else {
            v_set(c, n, 0.0, tmp);
            if ((e = pcd.solve(c, wk, tmp))) return e;
            v_axpy(c, n, Scal::h(1.0), tmp, x);
        }
        if (numIter >= P.savIter && resAbs < resAbsOld) v_copy(c, n, x, sv);
        if (numIter > P.maxIter) {
            err = kErrMaxIt;
            break;
        }
        apply_residual(c, *A, b, x, V);
        v_norm2(c, n, V, d + SL_T1);
        resAbs = rj = fetch(d + SL_T1);
        resRel = resAbs / denAbs;
        rec(numIter, resAbs);
        if ((resRel < P.relTol || resAbs < P.absTol) && numIter >= P.minIter) break;
        cr = rj / ri;
        ri = rj;
        adapt_restart(*this, cr, flexible);
    }
    info->numIter = numIter;
    info->code = err;
    if (!(numIter == P.minIter && numIter == P.maxIter)) {
        v_norm2(c, n, V, d + SL_T1);
        v_norminf(c, n, V, d + SL_T2);
        info->norm2 = fetch(d + SL_T1);
        info->normInf = fetch(d + SL_T2);
    }
    if (numIter > P.savIter) v_copy(c, n, sv, x);
    FB_CUDA(cudaStreamSynchronize(c.stream));
    return kOk;
}

// GMRES::LSolve (GMRES.cxx:283-453)
template <typename T>
int SolverImpl::gmres_left(const T* b, T* x, fasp_gpu_info* info, const fasp_gpu_params& P,
                           Space<T> S)
{
    std::vector<T*>& w = *S.w;
    T *wk = w[0], *tmp = w[1], *sv = w[2];
    T *V = S.V;
    const size_t ld = ldV;
    const GmLayout L = gm_layout(gm, maxRestart);
    double* d = c.dslot;
    int err = kOk, e;
    double ri, rj, cr = 1.0;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, resAbsOld = 1.0;
    uint32_t count = 1, count_1 = 2, numIter = 0;

    const bool devCycle = gm_device_cycles(false);
    if (devCycle) {
        ++c.launches;
        k_fill<<<c.grid(dhistCap, kBlock), kBlock, 0, c.stream>>>(dhistCap, kNaN, dhist);
    }
    v_copy(c, n, x, sv);
    apply_residual(c, *A, b, x, tmp);
    v_norm2(c, n, tmp, d + SL_T1);
    ri = fetch(d + SL_T1);
    v_set(c, n, 0.0, V);
    if ((e = pcd.solve(c, tmp, V))) return e;
    v_norm2(c, n, V, d + SL_T1);
    resAbs = fetch(d + SL_T1);
    denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;

    while (numIter < P.maxIter) {
        if (numIter == P.minIter) {
            resRel = resAbs / denAbs;
            resAbsOld = resAbs;
            rec(numIter, resAbs);
            if (resRel < P.relTol || resAbs < P.absTol) break;
        }
        if (resAbs < kSmallDbl) break;
        ++c.launches;
        k_set_scalar<<<1, 1, 0, c.stream>>>(L.var, resAbs);
        v_scale(c, n, Scal::h(1 / resAbs), V);

        count = 0;
        if (devCycle) { // the whole cycle on the device, one synchronisation
            const uint32_t steps = std::min<uint32_t>(restart, P.maxIter - numIter);
            int stopped = 0;
            if ((e = gm_cycle_device<T>(*this, L, V, steps, true, count, numIter, resAbs, denAbs,
                                        P, stopped, wk)))
                return e;
            count_1 = count - 1;
            if (!(stopped == 1 && count == 1)) {
                resAbsOld = resAbs;
                resRel = resAbs / denAbs;
            }
        }
        while (!devCycle && count < restart && numIter < P.maxIter) {
            ++numIter;
            count_1 = count++;
            T* vnew = V + count * ld;
            m_spmv(c, *A, V + count_1 * ld, tmp);
            v_set(c, n, 0.0, vnew);
            if ((e = pcd.solve(c, tmp, vnew))) return e;
            if ((e = orthogonalize<T>(*this, L, count, count_1, V, vnew))) return e;
            FB_CUDA(cudaMemcpyAsync(c.hslot + 2, L.out, 16, cudaMemcpyDeviceToHost, c.stream));
            FB_CUDA(cudaStreamSynchronize(c.stream));
            if (c.hslot[3] == 0.0) break;
            resAbs = c.hslot[2];
            resAbsOld = resAbs;
            resRel = resAbs / denAbs;
            rec(numIter, resAbs);
            if ((resAbs < P.absTol || resRel < P.relTol) && numIter > P.minIter) break;
        }

        ++c.launches;

        k_gmres_backsolve<<<1, 128, 0, c.stream>>>(L, (int)count, (int)count_1);
        v_set(c, n, 0.0, wk);
        v_multiaxpy(c, n, (int)count, V, ld, L.var, -1.0, wk, nullptr);
        v_axpy(c, n, Scal::h(1.0), wk, x);
        if (numIter >= P.savIter && resAbs < resAbsOld) v_copy(c, n, x, sv);
        if (numIter > P.maxIter) {
            err = kErrMaxIt;
            break;
        }
        apply_residual(c, *A, b, x, tmp);
        v_norm2(c, n, tmp, d + SL_T1);
        rj = fetch(d + SL_T1);
        v_set(c, n, 0.0, V);
        if ((e = pcd.solve(c, tmp, V))) return e;
        v_norm2(c, n, V, d + SL_T1);
        resAbs = fetch(d + SL_T1);
        resRel = resAbs / denAbs;
        rec(numIter, resAbs);
        if ((resRel < P.relTol || resAbs < P.absTol) && numIter >= P.minIter) break;
        cr = rj / ri;
        ri = rj;
        adapt_restart(*this, cr, false);
    }
    info->numIter = numIter;
    info->code = err;
    if (!(numIter == P.minIter && numIter == P.maxIter)) {
        v_norm2(c, n, tmp, d + SL_T1);
        v_norminf(c, n, tmp, d + SL_T2);
        info->norm2 = fetch(d + SL_T1);
        info->normInf = fetch(d + SL_T2);
    }
    if (numIter > P.savIter) v_copy(c, n, sv, x);
    FB_CUDA(cudaStreamSynchronize(c.stream));
    return kOk;
}

// ---- Jacobi as a solver (Iter.cxx:56-112) --------------------------------------------------

int SolverImpl::jacobi(const double* b, double* x, fasp_gpu_info* info)
{
    double n2 = kNaN, ni = kNaN;
    int e = pcd.solve(c, b, x, &hist, &n2, &ni);
    if (e) return e;
    info->code = kOk;
    info->numIter = pcd.numIter;
    info->norm2 = n2;
    info->normInf = ni;
    return kOk;
}

// ---- MG (src/MG.cxx:105-210), identity transfers, residual with the top-level A ----------

void SolverImpl::mg_cycle(const double* b, double* x)
{
    const uint32_t NL = (uint32_t)mgSmooth.size();
    double* r = w[0];
    if (NL > 0) {
        ++mgLevel;
        if ((uint32_t)mgLevel - NL == 0) return;
        const uint32_t L = (uint32_t)mgLevel;
        mgSmooth[L].solve(c, b, x);
        m_residual(c, *A, b, x, r, nullptr);
        v_copy(c, n, r, mgB[L]);     // restriction: IdentityMatrix::Apply (MAT.cxx:1095)
        v_set(c, n, 0.0, mgX[L]);
        if (L + 1 - NL == 0)
            mgCoarse[L].solve(c, mgB[L], mgX[L]);
        else
            for (uint32_t i = 0; i < cfg.mgCycles; ++i) mg_cycle(mgB[L], mgX[L]);
        v_copy(c, n, mgX[L], r);     // prolongation
        v_axpy(c, n, Scal::h(1.0), r, x);
        mgSmooth[L].solve(c, b, x);
        --mgLevel;
    } else {
        v_copy(c, n, b, x);
    }
}

static int pcd_mg_apply(SolverImpl* s, const double* b, double* x)
{
    fasp_gpu_info info{};
    const fasp_gpu_config& k = s->cfg;
    const bool fixed = k.prm.minIter == k.prm.maxIter && k.mgSmoothPrm.minIter == k.mgSmoothPrm.maxIter &&
                       k.mgCoarsePrm.minIter == k.mgCoarsePrm.maxIter;
    if (!fixed) return s->mg(b, x, &info);
    for (const auto& g : s->mgGraphs)
        if (g.b == b && g.x == x) {
            FB_CUDA(cudaGraphLaunch(g.exec, s->c.stream));
            return kOk;
        }
    cudaStream_t st = s->c.stream;
    FB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    s->capturing = true;
    const int e = s->mg(b, x, &info);
    s->capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    cudaGraphExec_t exec = nullptr;
    if (!e && ce == cudaSuccess && graph &&
        cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        cudaGraphDestroy(graph);
        s->mgGraphs.push_back({b, x, exec});
        FB_CUDA(cudaGraphLaunch(exec, st));
        return kOk;
    }
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return e ? e : kErrCuda;
}

static void pcd_mg_free(SolverImpl* s)
{
    for (auto& g : s->mgGraphs) cudaGraphExecDestroy(g.exec);
    s->mgGraphs.clear();
    s->destroy();
    delete s;
}

// ---- MG with transfer operators (no reference counterpart) -------------------------------
// The reference's MG cycle (MG.cxx:105-152) with what its identity-transfer setup leaves
// out: level l's residual uses its own operator A_l (the reference always uses the top-level
// A, MG.cxx:119), the residual is restricted by R_l and the correction prolongated by P_l
// (the reference stores one operator for both, MG.cxx:42-43). The smoother of level l runs
// on A_l and the coarse solver on A_{l+1}. Missing restrictions are P_l's exact transpose;
// missing coarse operators the Galerkin products R_l (A_l P_l), formed with MAT::Mult.

int SolverImpl::mg_setup_transfers()
{
    const uint32_t L = cfg.mgLevels;
    if (L == 0 || mgIn.size() != L) return kErrInputPar;
    int e;
    mgA.assign(1, A);
    mgP.clear();
    mgR.clear();
    auto own = [&]() {
        Mat* m = new Mat();
        mgOwn.push_back(m);
        return m;
    };
    for (uint32_t l = 0; l < L; ++l) {
        if (!mgIn[l].P) return kErrInputPar;
        const Mat* Al = mgA[l];
        const Mat* P = &mgIn[l].P->M;
        if (P->nrow != Al->nrow) return kErrNonmatch;
        const uint32_t nc = P->mcol;
        const Mat* R = nullptr;
        if (mgIn[l].R) {
            R = &mgIn[l].R->M;
        } else {
            Mat* T = own();
            if ((e = m_transpose(c, *P, *T))) return e;
            R = T;
        }
        if (R->nrow != nc || R->mcol != Al->nrow) return kErrNonmatch;
        const Mat* Ac = nullptr;
        if (mgIn[l].Ac) {
            Ac = &mgIn[l].Ac->M;
        } else {
            Mat AP;
            if ((e = m_mult(c, *Al, *P, AP))) return e;
            Mat* G = own();
            e = m_mult(c, *R, AP, *G);
            m_free(AP);
            if (e) return e;
            Ac = G;
        }
        if (Ac->nrow != nc || Ac->mcol != nc) return kErrNonmatch;
        mgA.push_back(Ac);
        mgP.push_back(P);
        mgR.push_back(R);
    }
    mgSmooth.resize(L);
    mgCoarse.resize(L);
    for (uint32_t l = 0; l < L; ++l) {
        if ((e = mgSmooth[l].setup(c, mgA[l], 1, cfg.mgSmoothWeight, cfg.mgSmoothPrm)))
            return e;
        if ((e = mgCoarse[l].setup(c, mgA[l + 1], 1, cfg.mgCoarseWeight, cfg.mgCoarsePrm)))
            return e;
        std::vector<double*> v;
        if ((e = alloc_vecs(v, 2, mgA[l + 1]->nrow))) return e;
        mgB.push_back(v[0]);
        mgX.push_back(v[1]);
        std::vector<double*> r;
        if (l > 0) {
            if ((e = alloc_vecs(r, 1, mgA[l]->nrow))) return e;
            mgRes.push_back(r[0]);
        } else {
            mgRes.push_back(nullptr); // level 0 uses the solver's residual vector
        }
    }
    return kOk;
}

void SolverImpl::mg_cycle_transfer(const double* b, double* x)
{
    const uint32_t NL = (uint32_t)mgP.size();
    ++mgLevel;
    if ((uint32_t)mgLevel == NL) return;
    const uint32_t l = (uint32_t)mgLevel;
    const Mat& Al = *mgA[l];
    double* r = l == 0 ? w[0] : mgRes[l];
    mgSmooth[l].solve(c, b, x);                        // pre-smoothing on A_l
    m_residual(c, Al, b, x, r, nullptr);               // r = b - A_l x
    m_spmv(c, *mgR[l], r, mgB[l]);                     // b_{l+1} = R_l r
    v_set(c, mgA[l + 1]->nrow, 0.0, mgX[l]);
    if (l + 1 == NL)
        mgCoarse[l].solve(c, mgB[l], mgX[l]);          // coarsest: on A_{l+1}
    else
        for (uint32_t i = 0; i < cfg.mgCycles; ++i) mg_cycle_transfer(mgB[l], mgX[l]);
    m_spmv(c, *mgP[l], mgX[l], r);                     // P_l e_{l+1}
    v_axpy(c, Al.nrow, Scal::h(1.0), r, x);
    mgSmooth[l].solve(c, b, x);                        // post-smoothing
    --mgLevel;
}

int SolverImpl::mg(const double* b, double* x, fasp_gpu_info* info)
{
    const fasp_gpu_params& P = cfg.prm;
    double* r = w[0];
    double* d = c.dslot;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0;
    uint32_t numIter = 0;
    mgLevel = -1;
    while (numIter < P.maxIter) {
        m_residual(c, *A, b, x, r, nullptr);
        if (numIter >= P.minIter) {
            v_norm2(c, n, r, d + SL_T1);
            resAbs = fetch(d + SL_T1);
            if (numIter == P.minIter) denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;
            resRel = resAbs / denAbs;
            rec(numIter, resAbs);
            if (resRel < P.relTol || resAbs < P.absTol) break;
        }
        if (mgP.empty())
            mg_cycle(b, x);
        else
            mg_cycle_transfer(b, x);
        ++numIter;
    }
    info->numIter = numIter;
    info->code = kOk;
    if (!(numIter == P.minIter && numIter == P.maxIter)) {
        m_residual(c, *A, b, x, r, nullptr);
        v_norm2(c, n, r, d + SL_T1);
        v_norminf(c, n, r, d + SL_T2);
        info->norm2 = resAbs = fetch(d + SL_T1);
        info->normInf = fetch(d + SL_T2);
        rec(numIter, resAbs);
    }
    if (!capturing) FB_CUDA(cudaStreamSynchronize(c.stream));
    return kOk;
}

// ---- mixed-precision BiCGStab / GMRES / FGMRES ------------------------------------------
// FP64 iterative refinement (no reference counterpart): r = b - A x in FP64, the inner solver
// runs its unchanged control flow in FP32 on A e = r / ||r|| (FP32 matrix values, vectors
// and per-thread accumulation; FP64 block and grid reductions, and the GMRES Hessenberg and
// Givens least-squares in FP64) to innerRelTol, then x += ||r|| e in FP64. Stops when
// ||b - A x|| / ||b - A x0|| < relTol (or < absTol), after maxOuter steps, or when the
// inner solve makes no iteration. History: inner residuals scaled back by ||r|| at their
// global iteration index, each outer FP64 true residual at the index where it was taken.
int SolverImpl::refine(const double* b, double* x, fasp_gpu_info* info)
{
    const fasp_gpu_params& P = cfg.prm;
    double* r64 = w[0];
    float* b32 = w32[w32.size() - 2];
    float* e32 = w32[w32.size() - 1];
    std::vector<float*> inner(w32.begin(), w32.end() - 2);
    Space<float> S{&inner, V32, Z32};
    const double innerTol = cfg.innerRelTol > 0 ? cfg.innerRelTol : 1e-4;
    const uint32_t innerMax = cfg.innerMaxIter ? cfg.innerMaxIter : P.maxIter;
    const uint32_t maxOuter = cfg.maxOuter ? cfg.maxOuter : 50;
    uint32_t total = 0, outer = 0;
    double den = 1.0, rn = 0.0;
    int code = kOk, e;
    std::vector<std::pair<uint32_t, double>> outerHist;
    for (;;) {
        if ((e = apply_residual(c, *A, b, (const double*)x, r64))) return e;
        v_norm2(c, n, (const double*)r64, c.dslot + SL_T1);
        rn = fetch(c.dslot + SL_T1);
        if (outer == 0) den = (kCloseZero > rn) ? kCloseZero : rn;
        outerHist.push_back({total, rn});
        if (rn / den < P.relTol || rn < P.absTol) break;
        if (outer >= maxOuter || total >= P.maxIter || !std::isfinite(rn)) {
            code = kErrMaxIt;
            break;
        }
        if ((e = convert_scaled(c, n, r64, 1.0 / rn, b32)) || (e = set32(c, n, e32))) return e;
        fasp_gpu_params Q = P;
        Q.relTol = innerTol;
        Q.absTol = 0.0;
        Q.minIter = 0;
        Q.maxIter = std::min<uint32_t>(innerMax, P.maxIter - total);
        Q.savIter = 0xffffffffu;
        fasp_gpu_info ii;
        std::memset(&ii, 0, sizeof(ii));
        histOff = total;
        histScale = rn;
        if (cfg.alg == FASP_GPU_BICGSTAB)
            e = bicgstab<float>(b32, e32, &ii, Q, S);
        else if (cfg.alg == FASP_GPU_FGMRES)
            e = gmres_right<float>(b32, e32, &ii, Q, S, true);
        else if (cfg.leftPrecond)
            e = gmres_left<float>(b32, e32, &ii, Q, S);
        else
            e = gmres_right<float>(b32, e32, &ii, Q, S, false);
        histOff = 0;
        histScale = 1.0;
        if (e) return e;
        total += ii.numIter;
        if ((e = update_from32(c, n, rn, e32, x))) return e;
        ++outer;
        if (ii.numIter == 0) {
            code = ii.code ? ii.code : kErrMaxIt;
            if ((e = apply_residual(c, *A, b, (const double*)x, r64))) return e;
            v_norm2(c, n, (const double*)r64, c.dslot + SL_T1);
            rn = fetch(c.dslot + SL_T1);
            outerHist.push_back({total, rn});
            break;
        }
    }
    info->numIter = total;
    info->outerIter = outer;
    info->code = code;
    info->norm2 = rn;
    v_norminf(c, n, (const double*)r64, c.dslot + SL_T2);
    info->normInf = fetch(c.dslot + SL_T2);
    for (auto& pt : outerHist) rec(pt.first, pt.second);
    FB_CUDA(cudaStreamSynchronize(c.stream));
    return kOk;
}

// ---- dispatch ------------------------------------------------------------------------------

int SolverImpl::solve(const double* b, double* x, fasp_gpu_info* info)
{
    if (!A) return kErrInputPar;
    static const char* const kAlg[] = {"?", "CG", "BiCGStab", "?", "GMRES", "FGMRES"};
    static const char* const kPrec[] = {"FP64", "MIXED", "MIXED_RELIABLE"};
    const char* an = cfg.alg >= 0 && cfg.alg <= 5 ? kAlg[cfg.alg]
                     : cfg.alg == FASP_GPU_JACOBI ? "Jacobi"
                     : cfg.alg == FASP_GPU_MG     ? "MG"
                                                  : "?";
    const char* pn = cfg.precision >= 0 && cfg.precision <= 2 ? kPrec[cfg.precision] : "?";
    TraceRange trace(std::string("fasp solve ") + an + " " + pn);
    fasp_gpu_info tmp;
    if (!info) info = &tmp;
    std::memset(info, 0, sizeof(*info));
    info->norm2 = 1e60; // SOL() initial norms (SOL.hxx:46-51)
    info->normInf = 1e60;
    hist.clear();
    const unsigned long long l0 = c.launches;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, c.stream);
    int e;
    switch (cfg.alg) {
        case FASP_GPU_CG:
            if (cfg.precision == FASP_GPU_MIXED)
                e = cg_mixed(b, x, info);
            else if (cfg.precision == FASP_GPU_MIXED_RELIABLE)
                e = cg_reliable(b, x, info);
            else if (cg64)
                e = cg_device(b, x, info);
            else
                e = cg_generic(b, x, info);
            break;
        case FASP_GPU_BICGSTAB:
            if (cfg.precision == FASP_GPU_MIXED)
                e = refine(b, x, info);
            else if (cfg.precision == FASP_GPU_MIXED_RELIABLE)
                e = bicgstab_reliable(b, x, info);
            else
                e = bicgstab<double>(b, x, info, cfg.prm, sp64());
            break;
        case FASP_GPU_GMRES:
            if (cfg.precision == FASP_GPU_MIXED)
                e = refine(b, x, info);
            else if (cfg.leftPrecond)
                e = gmres_left<double>(b, x, info, cfg.prm, sp64());
            else
                e = gmres_right<double>(b, x, info, cfg.prm, sp64(), false);
            break;
        case FASP_GPU_FGMRES:
            e = cfg.precision == FASP_GPU_MIXED
                    ? refine(b, x, info)
                    : gmres_right<double>(b, x, info, cfg.prm, sp64(), true);
            break;
        case FASP_GPU_JACOBI: e = jacobi(b, x, info); break;
        case FASP_GPU_MG: e = mg(b, x, info); break;
        default: e = kErrSolverType;
    }
    cudaEventRecord(t1, c.stream);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    lastMs = ms;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (e == kOk && cudaGetLastError() != cudaSuccess) e = kErrCuda;
    if (hist.size() < (size_t)info->numIter + 1) hist.resize((size_t)info->numIter + 1, kNaN);
    info->launches = (uint32_t)(c.launches - l0);
    return e;
}

unsigned tile_timeouts_solvers() { return tile_timeouts() + tile_timeouts_dcgs2(); }

} // namespace fb
