// solver.h -- the solver object behind fasp_gpu_solver (SOL and its subclasses).
#pragma once

#include <limits>
#include <vector>

#include "../../include/fasp_b200.h"
#include "bicgstab.cuh"
#include "cg.cuh"
#include "internal.h"

struct fasp_gpu_mat_s {
    fb::Mat         M;
    fb::Ctx         c;            // stream for matrix-level calls
    fasp_gpu_mat_s* T = nullptr;  // cached exact transpose (adjoint solves), owned
};

namespace fb {

// The in-cycle state of a GMRES restart cycle run without host round trips: k_gmres_givens
// updates it after every Arnoldi step and sets stop (1: breakdown, 2: converged); the other
// step kernels return at once when it is set.
struct GmCtl {
    int      stop;
    unsigned count;     // steps of this cycle done, a breakdown step included
    unsigned numIter, minIter;
    double   resAbs, denAbs, relTol, absTol;
    double*  hist;
    unsigned histCap, histOffset;
    double   histScale;
};

// The preconditioner of a solver: Identity (Iter.cxx:16-20) or Jacobi (Iter.cxx:29-112).
struct SolverImpl;

struct Pcd {
    int             type = 0;    // 0 identity, 1 Jacobi, 2 MG (one MG solve, prm its SOLParams)
    fasp_gpu_params prm{};
    double          weight = 1.0;
    const Mat*      A = nullptr;
    double*         dinv = nullptr;   // weight / diag
    float*          dinv32 = nullptr;
    double*         work = nullptr;
    float*          work32 = nullptr; // FP32 sweeps of mixed-precision inner solves (lazy)
    uint32_t        numIter = 0;
    SolverImpl*     mg = nullptr;     // type 2: the MG solver it runs (owned)
    bool pure() const { return type == 1 && prm.minIter == prm.maxIter; }
    int  setup(Ctx& c, const Mat* M, int t, double w, const fasp_gpu_params& p);
    void destroy();
    // Solve(b, x): x is read as the initial guess (callers zero it where the reference does).
    // T = float runs the same sweeps on the FP32 matrix values and diagInv.
    template <typename T>
    int  solve(Ctx& c, const T* b, T* x, std::vector<double>* hist = nullptr,
               double* norm2 = nullptr, double* normInf = nullptr);
};

// The vectors one precision of a host-orchestrated solver works on.
template <typename T>
struct Space {
    std::vector<T*>* w = nullptr;  // work vectors
    T*               V = nullptr;  // GMRES/FGMRES basis, (maxRestart+1) x n
    T*               Z = nullptr;  // FGMRES preconditioned basis
};

struct SolverImpl {
    fasp_gpu_config cfg{};
    unsigned        barLimit = 0;   // persistent CG: polls per grid barrier (0: 2^24)
    Ctx             c;
    Mat*            A = nullptr;    // bound by Setup (borrowed)
    fasp_gpu_mat    Ah = nullptr;
    Pcd             pcd;
    uint32_t        n = 0;
    // work vectors (FP64)
    std::vector<double*> w;
    double*         V = nullptr;    // GMRES/FGMRES basis, (maxRestart+1) x n
    double*         Z = nullptr;    // FGMRES preconditioned basis
    // FP32 copies for the inner solves of mixed-precision BiCGStab / GMRES / FGMRES
    std::vector<float*> w32;
    float*          V32 = nullptr;
    float*          Z32 = nullptr;
    // history entries are stored at histOff + k, scaled by histScale (inner solves)
    uint32_t        histOff = 0;
    double          histScale = 1.0;
    double*         gm = nullptr;   // device Hessenberg block: hh, hcos, hsin, var, dots
    GmCtl*          gmc = nullptr;  // device in-cycle state, and its pinned host copy
    GmCtl*          hgmc = nullptr;
    uint32_t        maxRestart = 0, minRestart = 0, restart = 0;
    size_t          ldV = 0;        // stride of the GMRES/FGMRES bases (n padded to 32)
    // MG (identity transfers): per level smoother and coarse solver, coarse b and x
    std::vector<Pcd> mgSmooth, mgCoarse;
    std::vector<double*> mgB, mgX;
    int             mgLevel = -1;
    // MG with transfer operators: what the caller set per coarse level (borrowed handles,
    // kept across Setup calls), and what Setup resolved: the level operators A_0 .. A_L,
    // P_l, R_l, the restrictions and Galerkin operators it formed itself (owned), and a
    // residual vector per level below the finest
    struct MgIn {
        fasp_gpu_mat P = nullptr, R = nullptr, Ac = nullptr;
    };
    std::vector<MgIn>        mgIn;
    std::vector<const Mat*>  mgA, mgP, mgR;
    std::vector<Mat*>        mgOwn;
    std::vector<double*>     mgRes;
    int  mg_setup_transfers();
    void mg_cycle_transfer(const double* b, double* x);
    // MG as a preconditioner: when no step of its solve reads a norm on the host (minIter =
    // maxIter for the MG object, its smoothers and its coarse solver), the whole solve is a
    // fixed kernel sequence; it is captured once per (b, x) pair and replayed as a graph
    struct MgGraph {
        const double*   b;
        double*         x;
        cudaGraphExec_t exec;
    };
    std::vector<MgGraph> mgGraphs;
    bool capturing = false;
    // device-driven CG
    CGEngine<double>* cg64 = nullptr;
    CGEngine<float>*  cg32 = nullptr;
    // device-driven BiCGStab (Identity or one Jacobi sweep as preconditioner)
    BiEngine<double>* bi64 = nullptr;
    BiEngine<float>*  bi32 = nullptr;
    double*         safe = nullptr;
    double*         dhist = nullptr;
    double*         hostB = nullptr;  // staging of the host entry point
    double*         hostX = nullptr;
    uint32_t        dhistCap = 0;
    // results
    std::vector<double> hist;
    double          lastMs = 0.0;
    // adjoint
    SolverImpl*     adj = nullptr;

    int  setup(fasp_gpu_mat M);
    int  solve(const double* b, double* x, fasp_gpu_info* info);
    void clean();
    void destroy();

    // solver bodies (host-orchestrated, device vectors)
    int cg_generic(const double* b, double* x, fasp_gpu_info* info);
    int cg_device(const double* b, double* x, fasp_gpu_info* info);
    int cg_mixed(const double* b, double* x, fasp_gpu_info* info);
    int cg_reliable(const double* b, double* x, fasp_gpu_info* info);
    int bicgstab_reliable(const double* b, double* x, fasp_gpu_info* info);
    template <typename T>
    int bicgstab(const T* b, T* x, fasp_gpu_info* info, const fasp_gpu_params& P, Space<T> S);
    template <typename T>
    int bicgstab_engine(BiEngine<T>& E, const T* b, T* x, fasp_gpu_info* info,
                        const fasp_gpu_params& P, Space<T> S);
    template <typename T>
    int gmres_right(const T* b, T* x, fasp_gpu_info* info, const fasp_gpu_params& P,
                    Space<T> S, bool flexible);
    template <typename T>
    int gmres_left(const T* b, T* x, fasp_gpu_info* info, const fasp_gpu_params& P, Space<T> S);
    bool gm_device_cycles(bool flexible) const;
    // FP64 iterative refinement around FP32 inner BiCGStab / GMRES / FGMRES solves
    int refine(const double* b, double* x, fasp_gpu_info* info);
    Space<double> sp64() { return Space<double>{&w, V, Z}; }
    Space<float>  sp32() { return Space<float>{&w32, V32, Z32}; }
    int jacobi(const double* b, double* x, fasp_gpu_info* info);
    int mg(const double* b, double* x, fasp_gpu_info* info);
    void mg_cycle(const double* b, double* x);

    // helpers
    double fetch(const double* dptr);
    void   rec(uint32_t k, double v)
    {
        k += histOff;
        if (k >= hist.size()) hist.resize((size_t)k + 1, std::numeric_limits<double>::quiet_NaN());
        hist[k] = v * histScale;
    }
};

} // namespace fb

struct fasp_gpu_solver_s {
    fb::SolverImpl s;
};
