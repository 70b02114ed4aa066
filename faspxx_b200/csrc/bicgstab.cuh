// bicgstab.cuh -- device-driven BiCGStab (BiCGStab::Solve, src/BiCGStab.cxx:68-270) for FP64
// and for the FP32 inner solves of mixed-precision refinement, with an Identity or one-sweep
// Jacobi preconditioner fused into the kernels.
#pragma once

#include "cg.cuh"

namespace fb {

enum BiReason { kBiNone = 0, kBiSave = 1, kBiStag = 2, kBiCheck = 3, kBiRefresh = 4 };

// The locals of BiCGStab::Solve (BiCGStab.cxx:70-82) and the parameters it reads, in device
// memory so that the finalize thread of each fused kernel runs the reference's control flow.
struct BiCtl {
    int      status, reason, code, phase;
    int      bench;     // 1: kernel timing, the finalize steps do nothing
    unsigned numIter, minIter, maxIter, savIter, restart, stagStep, moreStep;
    double   relTol, absTol, solStagTol;
    double   resAbs, resRel, denAbs, ratio, resAbsOld;
    double   alpha, omega, beta, rjr0star, rjr0startmp, tmp12;
    double   red[5];    // (r,r), (r,r0*), max|x|, (p,p), (x,x) of the last update kernel
    double*  hist;
    unsigned histCap;
    unsigned histOffset;
    double   histScale;
    // reliable updates (FP32 iterations of MIXED_RELIABLE): escalate kBiRefresh once the
    // recursive residual has fallen below delta x its largest value since the last refresh
    int      reliable;
    double   delta, rmax;
    // which of the two direction buffers (pj, ptmp) holds the current iteration's values:
    // bi_p reads the other pair and flips it in its finalize
    int      par;
};

// One iteration is three kernels (Jacobi from zero is a diagonal scaling, D = weight/diag):
//   bi_p      pj = rj + beta (pj_old - omega ptmp_old), the previous iteration's direction
//             update (:184-185), formed for every gathered entry and stored for the owned
//             rows into the other buffer of a pair; ptmp = D A pj, with (ptmp, r0*),
//             (rj, r0*) and (rj, rj) (the loop top, BiCGStab.cxx:79-102). beta = 0 at the
//             start makes pj = rj (:78).
//   bi_s      sj = rj - alpha ptmp formed on the fly, stmp = D A sj, with (stmp, sj) and
//             (stmp, stmp)                                                  (:103-113)
//   bi_x      x += alpha D pj + omega D sj, rj = sj - omega stmp, with (r,r), (r,r0*), max|x|,
//             (p,p), (x,x) and the checks of :117-175 ending with beta       (:114-183)
template <typename T>
struct BiEngine {
    Ctx*       c = nullptr;
    const Mat* A = nullptr;
    int        jacobi = 0;
    const T*   dinv = nullptr;
    T *x = nullptr, *rj = nullptr, *r0s = nullptr, *sj = nullptr, *stmp = nullptr;
    T *pj2[2] = {nullptr, nullptr}, *ptmp2[2] = {nullptr, nullptr}; // chosen by ctl->par
    T* pj(int par) const { return pj2[par & 1]; } // the direction of iteration par
    BiCtl*     ctl = nullptr;     // device
    BiCtl*     hctl = nullptr;    // pinned host copy
    int*       hstatus = nullptr; // pinned, written at the end of every graph launch
    cudaGraphExec_t gexec = nullptr;
    int        itersPerGraph = 8;
    bool       useGraph = true;
    bool       pdl = true; // programmatic dependent launch between the iteration's kernels
    // Jacobi applied on the right, ptmp = A (D pj) and stmp = A (D sj), so that the
    // recursive residual is b - A x whatever the diagonal (reliable updates replace it by
    // the true residual); false: the reference's D (A pj), the same when D is a constant
    bool       rightPcd = false;
    bool       capturing = false;
    uint32_t   n = 0;

    int  init(Ctx* ctx, const Mat* M, int jac, const T* dinvv, bool graph);
    void destroy();
    int  run(unsigned* launches);
    int  launch_iter();
    int  launch_resume();
    int  push_ctl();
    int  pull_ctl();
};

extern template struct BiEngine<double>;
extern template struct BiEngine<float>;

} // namespace fb
