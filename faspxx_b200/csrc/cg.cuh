// cg.cuh -- device-driven preconditioned CG (CG::Solve, src/CG.cxx:53-249) for FP64 and
// for the FP32 inner solves of mixed-precision refinement.
#pragma once

#include "internal.h"

namespace fb {

// kRefresh: a reliable update is in progress inside the iteration kernels (the next cg_spmv
// folds x into FP64, the next cg_update recomputes the FP64 residual); the host keeps going.
enum CGStatus { kRun = 0, kDone = 1, kEsc = 2, kRefresh = 3 };
enum CGReason { kNoReason = 0, kBreakdown = 1, kSave = 2, kStag = 3, kCheck3 = 4, kReliable = 5 };

// The locals of CG::Solve (CG.cxx:55-64) plus the parameters it reads, kept in device
// memory so that the finalize thread of each fused kernel can run the reference's control
// flow between iterations without a host round trip.
// Grid barrier state of the persistent kernel (device memory, zero at creation). limit:
// polls a block makes at one barrier before it gives up (0: 2^24, on the order of a second).
struct GridBar {
    unsigned count, gen, error, limit;
};

struct CGCtl {
    int      status, reason, code, phase;
    int      pmode;     // 0: p = z (first iteration or restart), 1: p = z + beta p
    int      par;       // which of the two p buffers holds the current direction
    int      pzero;     // the host zeroed p (a restart): next p = z
    int      xpend;     // lean FP32 engine: x += alpha p of the last iteration not yet applied
    // one reduction per iteration (FP32 engines with the recurrence and z = zc r or z = r):
    // cg_spmv also sums (r,r), (r,q), (q,q) and runs the checks of the update on
    // (r - alpha q, r - alpha q) = (r,r) - 2 alpha (r,q) + alpha^2 (q,q); cg_update only
    // updates r, and skips the slot after a refresh (skipUpd == numIter + 1)
    int      onered;
    unsigned skipUpd;
    double   zc;        // the constant diagInv when the Jacobi diagonal is one value (z = zc r)
    int      inner;     // 1: inner solve of mixed refinement (plain relative stop)
    int      reliable;  // 1 (with inner): FP32 iterations with FP64 reliable updates
    int      bench;     // 1: kernel timing, the finalize steps do nothing
    unsigned numIter, stagStep, moreStep;
    unsigned maxIter, minIter, savIter, restart;
    double   relTol, absTol, solStagTol, innerTol;
    double   tmpa, tmpb, alpha, beta, resAbs, resRel, denAbs, ratio, resAbsOld, xRelDiff;
    double   delta;     // reliable: refresh when resAbs < delta * rmax
    double   rmax;      // reliable: largest recursive residual since the last refresh
    double   absTolIn;  // reliable: absolute tolerance in the scaled units of the FP32 vectors
    // reliable updates run by the iteration kernels (graph and plain engines): the FP64
    // side, the stop test on the FP64 residual (relTol, absTol, den64) and its outcome
    int      devRefresh;
    int      converged;
    unsigned refreshes;
    unsigned stall;     // consecutive refreshes whose FP64 residual fell by less than sqrt(delta)
    double   den64, res64, resPrev;
    const double* rb;   // b
    double*  rx;        // x (FP64)
    double*  rr;        // r = b - A x (FP64), written by each refresh
    const double* rval; // FP64 values of the matrix (same structure as the FP32 view)
    const double* rcval;// FP64 values of its row-class table (when the FP32 view uses one)
    double   skval[kMaxStencil]; // FP64 stencil values (when the FP32 view uses masks)
    int32_t  skdelta[kMaxStencil];
    double   red[5];    // rr, zr, xx, max|x|, pp saved at an escalation
    double*  hist;
    unsigned histCap;
    unsigned histOffset; // global index of this solve's iteration 0 (mixed refinement)
    double   histScale;  // inner solves record scale * residual
};

// Plane columns of the CG SpMV on 3D seven-point stencil masks (cg_spmv with V4 and SH = 7;
// groups of rpg = 4 FP32 or 2 FP64 rows): the matrix is nz planes of p4 groups (the offset
// +-S2 = rpg p4 rows is one plane), and a thread walks `chunk` consecutive planes of one
// column of groups, so that the z (or p) groups at -S2, 0 and +S2 of a plane are the
// previous, current and next plane's group of the same column, held in registers.
// p4 == 0: not in use.
struct MarchPlan {
    uint32_t p4 = 0, nz = 0, chunk = 0;
};

// Device-driven PCG on one square matrix. T = double (the reference's arithmetic) or
// float (inner solves). The preconditioner is fused: identity (z aliases r) or one Jacobi
// sweep from zero, z = weight/diag .* r (Jacobi::Solve with minIter = maxIter = 1).
template <typename T>
struct CGEngine {
    Ctx*       c = nullptr;
    const Mat* A = nullptr;
    int        jacobi = 0;
    const T*   dinv = nullptr;
    // a constant diagInv (every diagonal entry equal): z = zc r is formed where it is used
    // and never stored, with the same values as the stored z (graph and plain engines)
    bool       constDiag = false;
    double     zc = 0.0;
    int        jmode() const { return !jacobi ? 0 : (constDiag && !wantPersistent ? 2 : 1); }
    T *x = nullptr, *r = nullptr, *z = nullptr, *q = nullptr, *P0 = nullptr, *P1 = nullptr;
    CGCtl*     ctl = nullptr;    // device
    CGCtl*     hctl = nullptr;   // pinned host copy
    int*       hstatus = nullptr;// pinned, written at the end of every graph launch
    cudaGraphExec_t gexec = nullptr;
    int        itersPerGraph = 16;
    bool       useGraph = true;
    bool       capturing = false;
    bool       pdl = true;      // programmatic dependent launch of the iteration kernels
    bool       recurrence = false; // q = A z + beta q_old (FP32 engines; p single-buffered)
    // with the recurrence (not persistent): x += alpha p is applied by the next cg_spmv for
    // its own rows and cg_update keeps to r, z and two sums (the FP32 loop reads no others)
    bool       lean() const { return recurrence && !persistent; }
    // one grid reduction per iteration (see CGCtl::onered)
    bool       onered() const
    {
        return lean() && sizeof(T) == 4 && (jmode() == 2 || jmode() == 0);
    }
    // applies a pending x += alpha p (host side, after the device loop stopped)
    int        apply_pending_x();
    uint32_t   n = 0;
    // persistent engine: one cooperative launch runs the iterations
    bool       wantPersistent = true; // set before init
    bool       persistent = false;
    // ... as one thread-block cluster (wantCluster, set before init with wantPersistent):
    // cgrid blocks of 1024 threads meeting at the hardware cluster barrier
    bool       wantCluster = false;
    bool       cluster = false;
    int        cgrid = 0;
    // ... with the vectors in the cluster's distributed shared memory, 2^dshift rows a block,
    // when they fit (dsBytes of dynamic shared memory a block)
    bool       dsmem = false;
    int        dshift = 0;
    size_t     dsBytes = 0;
    int        pgrid = 0;
    GridBar*   bar = nullptr;
    unsigned   barLimit = 0;      // GridBar::limit written before each persistent launch
    int        run_persistent(unsigned iterCap);

    int  init(Ctx* ctx, const Mat* M, int jac, const T* dinvv, bool graph);
    void destroy();
    // Runs iterations until the control block leaves kRun; returns kOk or an error.
    int  run(unsigned* launches);
    // Kernels: start from the residual in r and the guess in x.
    int  launch_init();
    int  launch_iter();
    void launch_spmv_kernel();
    void launch_update_kernel();
    int  launch_resume();
    int  time_kernels(unsigned reps, int flushL2, double* ms);
    int  push_ctl();   // hctl -> ctl
    int  pull_ctl();   // ctl -> hctl (synchronous)
    T*   cur_p() const { return hctl->par ? P1 : P0; }
};

extern template struct CGEngine<double>;
extern template struct CGEngine<float>;

int convert_scaled(Ctx& c, uint32_t n, const double* src, double inv_scale, float* dst);
int update_from32(Ctx& c, uint32_t n, double scale, const float* e, double* x);
int set32(Ctx& c, uint32_t n, float* x);
int to32(Ctx& c, uint32_t n, const double* src, float* dst);

} // namespace fb
