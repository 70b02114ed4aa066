/*
 * faspxx_b200.hxx -- C++ façade of the B200 iterative-solve library with the FASP++ API.
 *
 * Header-only, over the C ABI in fasp_b200.h (link with -lfasp_b200). The classes keep the
 * names, members and return codes of FASP++ so that a driver such as example/TestPCG.cxx
 * switches to the GPU by changing its includes and adding `using namespace fasp_b200;`:
 *
 *   VEC    host vector (src/VEC.hxx): the values a Solve copies in and out
 *   DVEC   device vector resident in HBM (no reference counterpart; avoids the copies)
 *   LOP    linear operator base (src/LOP.hxx:22-66)
 *   MAT    CSRx matrix (src/MAT.hxx:39-213), uploaded once at construction
 *   SOL    solver base (src/SOL.hxx:24-126) with SOLParams setters and getters
 *   CG, BiCGStab, GMRES, FGMRES, Jacobi, Identity, MG<MAT>   (src/*.hxx)
 *   Krylov(A, b, x, pcd, params)                             (src/Krylov.cxx:16-53)
 *
 * Differences a caller sees: operators must be MAT (a host-side user LOP cannot be applied
 * on the GPU, so Setup returns ERROR_SOLVER_TYPE for it); Solve blocks until the device is
 * done; FaspRetCode values are the reference's.
 */
#ifndef FASPXX_B200_HXX
#define FASPXX_B200_HXX

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <string>
#include <vector>

#include "fasp_b200.h"

namespace fasp_b200 {

typedef int          INT;
typedef unsigned int USI;
typedef double       DBL;

/* FaspRetCode (src/RetCode.hxx:24-55) */
enum FaspRetCode {
    SUCCESS = 0, ERROR_OPEN_FILE = -10, ERROR_INPUT_FILE = -11, ERROR_INPUT_PAR = -12,
    ERROR_VEC_SIZE = -14, ERROR_MAT_SIZE = -15, ERROR_NONMATCH_SIZE = -16,
    ERROR_MAT_DATA = -17, ERROR_DIVIDE_ZERO = -18, ERROR_MAT_ZERODIAG = -19,
    ERROR_ALLOC_MEM = -20, ERROR_SOLVER_TYPE = -30, ERROR_SOLVER_PCD_TYPE = -31,
    ERROR_SOLVER_STAG = -32, ERROR_SOLVER_SOLSTAG = -33, ERROR_SOLVER_TOLSMALL = -34,
    ERROR_SOLVER_MAXIT = -39
};

/* Output and SOLType (src/Param.hxx:27-54) */
enum Output { PRINT_NONE = 0, PRINT_MIN = 2, PRINT_SOME = 4, PRINT_MORE = 6, PRINT_MAX = 8 };
enum SOLType {
    SOLVER_CG = 1, SOLVER_BICGSTAB = 2, SOLVER_MINRES = 3, SOLVER_GMRES = 4,
    SOLVER_FGMRES = 5, SOLVER_VFGMRES = 6, SOLVER_JACOBI = 11, SOLVER_MG = 21
};

/* SOLParams (src/Param.hxx:57-80) */
struct SOLParams {
    SOLType     type = SOLVER_CG;
    std::string algName = "cg";
    USI         maxIter = 1, minIter = 0, savIter = 100000, restart = 30;
    double      relTol = 1e-6, absTol = 1e-8;
    Output      verbose = PRINT_NONE;
};

/* Host vector with the VEC constructors the solvers' callers use (src/VEC.hxx:40-62). */
class VEC {
public:
    std::vector<DBL> values;
    VEC() = default;
    explicit VEC(const USI& size, const DBL& value = 0.0) : values(size, value) {}
    explicit VEC(const std::vector<DBL>& src) : values(src) {}
    VEC(const USI& size, const DBL* src) : values(src, src + size) {}
    void SetValues(const USI& size, const DBL& value = 0.0) { values.assign(size, value); }
    void SetValues(const std::vector<DBL>& src) { values = src; }
    void SetValues(const USI& size, const DBL* a) { values.assign(a, a + size); }
    USI  GetSize() const { return (USI)values.size(); }
    DBL&       operator[](const USI& i) { return values[i]; }
    const DBL& operator[](const USI& i) const { return values[i]; }
};

/* Device vector: one allocation in HBM (no reference counterpart). */
class DVEC {
    double* p_ = nullptr;
    USI     n_ = 0;
public:
    DVEC() = default;
    explicit DVEC(USI n) : n_(n) { fasp_gpu_malloc((void**)&p_, (size_t)n * 8 + 16); }
    explicit DVEC(const VEC& v) : DVEC(v.GetSize()) { Upload(v); }
    DVEC(const DVEC&) = delete;
    DVEC& operator=(const DVEC&) = delete;
    ~DVEC() { if (p_) fasp_gpu_free(p_); }
    int  Upload(const VEC& v) { return fasp_gpu_memcpy_h2d(p_, v.values.data(), (size_t)n_ * 8); }
    int  Download(VEC& v) const { v.values.resize(n_); return fasp_gpu_memcpy_d2h(v.values.data(), p_, (size_t)n_ * 8); }
    double*       data() { return p_; }
    const double* data() const { return p_; }
    USI  GetSize() const { return n_; }
    DBL  Dot(const DVEC& v) const { double r = 0; fasp_gpu_vec_dot(n_, p_, v.p_, &r); return r; }
    DBL  Norm2() const { double r = 0; fasp_gpu_vec_norm2(n_, p_, &r); return r; }
    DBL  NormInf() const { double r = 0; fasp_gpu_vec_norminf(n_, p_, &r); return r; }
    void AXPY(const DBL& a, const DVEC& x) { fasp_gpu_vec_axpy(n_, a, x.p_, p_); }
    void XPAY(const DBL& a, const DVEC& x) { fasp_gpu_vec_xpay(n_, a, x.p_, p_); }
    void AXPBY(const DBL& a, const DBL& b, const DVEC& y) { fasp_gpu_vec_axpby(n_, a, b, y.p_, p_); }
    void WAXPBY(const DBL& a, const DVEC& v1, const DBL& b, const DVEC& v2) { fasp_gpu_vec_waxpby(n_, a, v1.p_, b, v2.p_, p_); }
    void Scale(const DBL& a) { fasp_gpu_vec_scale(n_, a, p_); }
};

/* Linear operator (src/LOP.hxx:22-66). */
class LOP {
protected:
    USI nrow = 0, mcol = 0;
public:
    virtual ~LOP() = default;
    USI GetRowSize() const { return nrow; }
    USI GetColSize() const { return mcol; }
    virtual fasp_gpu_mat Device() const { return nullptr; } /* null: not GPU-resident */
};

/* CSRx matrix in HBM (src/MAT.hxx:39-213). */
class MAT : public LOP {
    fasp_gpu_mat h_ = nullptr;
    USI          nnz_ = 0;
    int          err_ = 0;
    void create(USI n, USI m, USI nnz, const DBL* v, const USI* ci, const USI* rp)
    {
        nrow = n; mcol = m; nnz_ = nnz;
        err_ = fasp_gpu_mat_create(n, m, nnz, rp, ci, v, &h_);
    }
public:
    MAT() = default;
    /* MAT(nrow, mcol, nnz, values, colInd, rowPtr) (MAT.cxx:41-57) */
    MAT(const USI& n, const USI& m, const USI& nnz, const std::vector<DBL>& values,
        const std::vector<USI>& colInd, const std::vector<USI>& rowPtr)
    {
        create(n, m, nnz, values.data(), colInd.data(), rowPtr.data());
    }
    /* sparsity structure only (MAT.cxx:60-75) */
    MAT(const USI& n, const USI& m, const USI& nnz, const std::vector<USI>& colInd,
        const std::vector<USI>& rowPtr)
    {
        create(n, m, nnz, nullptr, colInd.data(), rowPtr.data());
    }
    MAT(const MAT&) = delete;
    MAT& operator=(const MAT&) = delete;
    MAT(MAT&& o) noexcept { *this = std::move(o); }
    MAT& operator=(MAT&& o) noexcept
    {
        std::swap(h_, o.h_); std::swap(nnz_, o.nnz_); std::swap(err_, o.err_);
        std::swap(nrow, o.nrow); std::swap(mcol, o.mcol);
        return *this;
    }
    ~MAT() override { if (h_) fasp_gpu_mat_destroy(h_); }
    int  Status() const { return err_; }     /* ERROR_MAT_DATA when CheckCSR fails */
    USI  GetNNZ() const { return nnz_; }
    fasp_gpu_mat Device() const override { return h_; }
    void Apply(const DVEC& v, DVEC& w) const { fasp_gpu_mat_apply(h_, v.data(), w.data()); }
    void Residual(const DVEC& b, const DVEC& x, DVEC& r) const
    {
        fasp_gpu_mat_residual(h_, b.data(), x.data(), r.data());
    }
    /* B200 option: matrix form of the SpMV kernels, 0 CSR, 1 row classes, 2 row classes
     * with stencil masks (bit-identical results; set before a solver's Setup) */
    void SetRowClass(int mode) { fasp_gpu_mat_set_rowclass(h_, mode); }
    /* MAT::TransInPlace (MAT.cxx:479-538) */
    void TransInPlace()
    {
        fasp_gpu_mat t = nullptr;
        if (fasp_gpu_mat_transpose(h_, &t) == 0) {
            fasp_gpu_mat_destroy(h_);
            h_ = t;
            std::swap(nrow, mcol);
        }
    }
};

/* Solver base (src/SOL.hxx:24-126). */
class SOL {
protected:
    fasp_gpu_config cfg_{};
    const LOP*      A = nullptr;
    fasp_gpu_solver h_ = nullptr;
    fasp_gpu_info   info_{};
    bool            dirty_ = true;
    explicit SOL(int alg) { fasp_gpu_default_config(&cfg_, alg); info_.norm2 = info_.normInf = 1e60; }
    int build()
    {
        if (!A || !A->Device()) return ERROR_SOLVER_TYPE;
        if (h_ && !dirty_) return SUCCESS;
        if (h_) fasp_gpu_solver_destroy(h_);
        h_ = nullptr;
        int e = fasp_gpu_solver_create(&cfg_, &h_);
        if (!e) e = fasp_gpu_solver_setup(h_, A->Device());
        dirty_ = e != 0;
        return e;
    }
public:
    virtual ~SOL() { if (h_) fasp_gpu_solver_destroy(h_); }
    SOL(const SOL&) = delete;
    SOL& operator=(const SOL&) = delete;
    void SetOutput(Output) {}
    void SetMaxIter(USI v) { cfg_.prm.maxIter = v; dirty_ = true; }
    void SetMinIter(USI v) { cfg_.prm.minIter = v; dirty_ = true; }
    void SetSavIter(USI v) { cfg_.prm.savIter = v; dirty_ = true; }
    void SetRestart(USI v) { cfg_.prm.restart = v; dirty_ = true; }
    void SetRelTol(double v) { cfg_.prm.relTol = v; dirty_ = true; }
    void SetAbsTol(double v) { cfg_.prm.absTol = v; dirty_ = true; }
    /* B200 options */
    void SetPrecision(int p) { cfg_.precision = p; dirty_ = true; }
    void SetInnerRelTol(double t) { cfg_.innerRelTol = t; dirty_ = true; }
    void SetOrth(int o) { cfg_.orth = o; dirty_ = true; }
    void SetUseGraph(bool on) { cfg_.useGraph = on ? 1 : 0; dirty_ = true; }
    void SetPersistent(bool on) { cfg_.persistent = on ? 1 : 0; dirty_ = true; }
    void SetOverlapLaunch(bool on) { cfg_.overlapLaunch = on ? 1 : 0; dirty_ = true; }
    void SetFP32Recurrence(bool on) { cfg_.fp32Recurrence = on ? 1 : 0; dirty_ = true; }
    const fasp_gpu_config& Config() const { return cfg_; }
    /* SOL::SetupPCD (SOL.cxx:249): Identity or Jacobi */
    virtual void SetupPCD(SOL& pc) { pc.AsPreconditionerOf(cfg_); dirty_ = true; }
    virtual void AsPreconditionerOf(fasp_gpu_config& c) const { c.pcd = 0; }
    virtual FaspRetCode Setup(const LOP& op)
    {
        A = &op;
        dirty_ = true;
        return (FaspRetCode)build();
    }
    /* Solve(b, x) with host vectors: copies in, solves on the GPU, copies x back */
    virtual FaspRetCode Solve(const VEC& b, VEC& x)
    {
        int e = build();
        if (e) return (FaspRetCode)e;
        e = fasp_gpu_solver_solve_host(h_, b.values.data(), x.values.data(), &info_);
        return (FaspRetCode)(e ? e : info_.code);
    }
    /* Solve(b, x) with device vectors */
    FaspRetCode Solve(const DVEC& b, DVEC& x)
    {
        int e = build();
        if (e) return (FaspRetCode)e;
        e = fasp_gpu_solver_solve(h_, b.data(), x.data(), &info_);
        return (FaspRetCode)(e ? e : info_.code);
    }
    virtual void Clean() { if (h_) fasp_gpu_solver_clean(h_); }
    double GetNorm2() const { return info_.norm2; }
    double GetInfNorm() const { return info_.normInf; }
    USI    GetIterations() const { return info_.numIter; }
    const fasp_gpu_info& Info() const { return info_; }
};

class CG : public SOL { public: CG() : SOL(FASP_GPU_CG) {} };
class BiCGStab : public SOL { public: BiCGStab() : SOL(FASP_GPU_BICGSTAB) {} };

class GMRES : public SOL {
public:
    GMRES() : SOL(FASP_GPU_GMRES) {}
    void SetRightPrecond() { cfg_.leftPrecond = 0; dirty_ = true; }
    void SetLeftPrecond() { cfg_.leftPrecond = 1; dirty_ = true; }
    void SetMaxMinRestart(const USI maxR, const USI minR)
    {
        cfg_.maxRestart = maxR; cfg_.minRestart = minR; dirty_ = true;
    }
};

class FGMRES : public SOL {
public:
    FGMRES() : SOL(FASP_GPU_FGMRES) {}
    void SetMaxMinRestart(const USI maxR, const USI minR)
    {
        cfg_.maxRestart = maxR; cfg_.minRestart = minR; dirty_ = true;
    }
};

class Identity : public SOL {
public:
    Identity() : SOL(FASP_GPU_IDENTITY) {}
    FaspRetCode Setup(const LOP&) override { return SUCCESS; }
};

/* Jacobi / weighted Jacobi (src/Iter.hxx:42-71): a solver, or the preconditioner of one. */
class Jacobi : public SOL {
public:
    Jacobi() : SOL(FASP_GPU_JACOBI) {}
    explicit Jacobi(DBL weight) : SOL(FASP_GPU_JACOBI) { cfg_.weight = weight; }
    void SetWeight(const DBL w) { cfg_.weight = w; dirty_ = true; }
    FaspRetCode Setup(const MAT& M) { return SOL::Setup(M); }
    void AsPreconditionerOf(fasp_gpu_config& c) const override
    {
        c.pcd = 1;
        c.pcdWeight = cfg_.weight;
        c.pcdPrm = cfg_.prm;
    }
};

/* Abstract MG with identity transfers and Jacobi level solvers (src/MG.hxx:44-106). */
template <class TTT>
class MG : public SOL {
public:
    MG() : SOL(FASP_GPU_MG) {}
    FaspRetCode SetupALL(const TTT& M, const USI numLevels)
    {
        cfg_.mgLevels = numLevels;
        return SOL::Setup(M);
    }
    void SetNumCycles(USI n) { cfg_.mgCycles = n; dirty_ = true; }
    /* SetupLevel(A, level, &IdentityMatrix, &smoother, &coarseSolver): the Jacobi objects'
     * weights and SOLParams become the level solvers (the same for every level here). */
    FaspRetCode SetupLevel(const TTT&, const USI, const void*, const Jacobi& smoother,
                           const Jacobi& coarse)
    {
        cfg_.mgSmoothWeight = smoother.Config().weight;
        cfg_.mgSmoothPrm = smoother.Config().prm;
        cfg_.mgCoarseWeight = coarse.Config().weight;
        cfg_.mgCoarsePrm = coarse.Config().prm;
        dirty_ = true;
        return SUCCESS;
    }
};

/* Krylov() dispatcher (src/Krylov.cxx:16-53), including SetSolTypeFromName
 * (src/SOL.cxx:127-161); unknown names fall back to CG as there. */
inline FaspRetCode Krylov(LOP& A, VEC& b, VEC& x, SOL& pcd, SOLParams& params)
{
    std::string name = params.algName;
    for (char& ch : name) ch = (char)std::tolower((unsigned char)ch);
    SOL* sol = nullptr;
    if (name == "bicgstab") sol = new BiCGStab();
    else if (name == "gmres") sol = new GMRES();
    else if (name == "fgmres") sol = new FGMRES();
    else sol = new CG();
    sol->SetMaxIter(params.maxIter);
    sol->SetMinIter(params.minIter);
    sol->SetSavIter(params.savIter);
    sol->SetRestart(params.restart);
    sol->SetRelTol(params.relTol);
    sol->SetAbsTol(params.absTol);
    sol->SetupPCD(pcd);
    FaspRetCode code = sol->Setup(A);
    if (code == SUCCESS) code = sol->Solve(b, x);
    delete sol; /* the reference leaks it (Krylov.cxx:24-52) */
    return code;
}

} // namespace fasp_b200

#endif
