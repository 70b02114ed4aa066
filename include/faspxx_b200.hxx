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
 *   CG, BiCGStab, GMRES, FGMRES, Jacobi, Identity, MG<MAT>   (src/CG.hxx and the others)
 *   Krylov(A, b, x, pcd, params)                             (src/Krylov.cxx:16-53)
 *   ReadMat(file, MAT&)                                      (src/ReadData.cxx:361-446)
 *   StencilLOP  matrix-free grid operator, the GPU form of a user LOP such as the one of
 *               example/TestMatFree.cxx:26-176 (no reference class of this name)
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
#include <fstream>
#include <string>
#include <utility>
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
    void adopt(int e, fasp_gpu_mat h)
    {
        err_ = e;
        if (e) return;
        if (h_) fasp_gpu_mat_destroy(h_);
        h_ = h;
        fasp_gpu_mat_info(h_, &nrow, &mcol, &nnz_);
    }
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
    /* MAT::MultTransposeAdd (MAT.cxx:541-606): v = A^T v1 + v2, on a transpose formed once */
    void MultTransposeAdd(const DVEC& v1, const DVEC& v2, DVEC& v) const
    {
        fasp_gpu_mat_mult_transpose_add(h_, v1.data(), v2.data(), v.data());
    }
    /* B200 option: matrix form of the SpMV kernels, 0 CSR, 1 row classes, 2 row classes
     * with stencil masks (bit-identical results; set before a solver's Setup) */
    void SetRowClass(int mode) { fasp_gpu_mat_set_rowclass(h_, mode); }
    /* MAT::Mult (MAT.cxx:715-800): *this = matl * matr, formed on the GPU */
    void Mult(const MAT& matl, const MAT& matr)
    {
        fasp_gpu_mat h = nullptr;
        const int e = fasp_gpu_mat_mult(matl.h_, matr.h_, &h);
        adopt(e, h);
    }
    /* MAT::Add (MAT.cxx:652-713): *this = a * mat1 + b * mat2, formed on the GPU */
    void Add(const DBL a, const MAT& mat1, const DBL b, const MAT& mat2)
    {
        fasp_gpu_mat h = nullptr;
        const int e = fasp_gpu_mat_add(a, mat1.h_, b, mat2.h_, &h);
        adopt(e, h);
    }
    /* MTXtoMAT / ReadCSR's conversions on the GPU from the readers' arrays (see ReadMat) */
    int FromCOO(USI n, USI m, const std::vector<USI>& rowInd, const std::vector<USI>& colInd,
                const std::vector<DBL>& values)
    {
        fasp_gpu_mat h = nullptr;
        const int e = fasp_gpu_mat_create_coo(n, m, (USI)values.size(), rowInd.data(),
                                              colInd.data(), values.data(), 0, &h);
        adopt(e, h);
        return e;
    }
    int FromCSRRaw(USI n, const std::vector<USI>& rowPtr, const std::vector<USI>& colInd,
                   const std::vector<DBL>& values)
    {
        fasp_gpu_mat h = nullptr;
        const int e = fasp_gpu_mat_create_csr_raw(n, n, (USI)values.size(), rowPtr.data(),
                                                  colInd.data(), values.data(), 0, &h);
        adopt(e, h);
        return e;
    }
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

/* Matrix-free operator on an nx x ny x nz grid (nz = 1: 2D, ny = nz = 1: 1D): a
 * constant-coefficient stencil of up to 16 points (dx, dy, dz in -3..3) truncated at the
 * faces, row ix + nx (iy + ny iz), nothing stored -- what a user LOP like the one of
 * example/TestMatFree.cxx computes, in a form the GPU applies (fasp_gpu_mat_create_stencil). */
class StencilLOP : public LOP {
    fasp_gpu_mat h_ = nullptr;
    int          err_ = 0;
public:
    StencilLOP(USI nx, USI ny, USI nz, const std::vector<int32_t>& dx,
               const std::vector<int32_t>& dy, const std::vector<int32_t>& dz,
               const std::vector<DBL>& coef)
    {
        nrow = mcol = nx * ny * nz;
        err_ = fasp_gpu_mat_create_stencil(nx, ny, nz, (USI)coef.size(), dx.data(), dy.data(),
                                           dz.data(), coef.data(), &h_);
    }
    StencilLOP(const StencilLOP&) = delete;
    StencilLOP& operator=(const StencilLOP&) = delete;
    ~StencilLOP() override { if (h_) fasp_gpu_mat_destroy(h_); }
    int Status() const { return err_; }
    fasp_gpu_mat Device() const override { return h_; }
    void Apply(const DVEC& v, DVEC& w) const { fasp_gpu_mat_apply(h_, v.data(), w.data()); }
};

/* ReadMat (src/ReadData.cxx:361-446): a .csr or .mtx file by its extension. The text is
 * read here on the host as ReadCSR / ReadMTX read it; the conversions (the 1-based shift,
 * the row sorts, the zero diagonals) run on the GPU. */
inline FaspRetCode ReadMat(const char* fileName, MAT& dst)
{
    const std::string f(fileName);
    if (f.size() <= 4) return ERROR_INPUT_FILE;
    std::string ext = f.substr(f.size() - 3);
    for (char& ch : ext) ch = (char)std::tolower((unsigned char)ch);
    std::ifstream in(fileName);
    if (!in.is_open()) return ERROR_OPEN_FILE;
    if (ext == "csr") {
        USI n = 0;
        if (!(in >> n) || n == 0) return ERROR_INPUT_PAR;
        std::vector<USI> rp(n + 1);
        for (auto& v : rp)
            if (!(in >> v)) return ERROR_INPUT_FILE;
        const USI nnz = rp[n] - rp[0];
        std::vector<USI> ci(nnz);
        std::vector<DBL> va(nnz);
        for (auto& v : ci)
            if (!(in >> v)) return ERROR_INPUT_FILE;
        for (auto& v : va)
            if (!(in >> v)) return ERROR_INPUT_FILE;
        return (FaspRetCode)dst.FromCSRRaw(n, rp, ci, va);
    }
    if (ext == "mtx") {
        std::string line;
        while (in.peek() == '%' && std::getline(in, line)) {}
        USI n = 0, m = 0, nnz = 0;
        if (!(in >> n >> m >> nnz)) return ERROR_INPUT_FILE;
        std::vector<USI> ri(nnz), ci(nnz);
        std::vector<DBL> va(nnz);
        for (USI k = 0; k < nnz; ++k) {
            if (!(in >> ri[k] >> ci[k] >> va[k])) return ERROR_INPUT_FILE;
            --ri[k];
            --ci[k];
        }
        return (FaspRetCode)dst.FromCOO(n, m, ri, ci, va);
    }
    return ERROR_INPUT_FILE;
}

/* Solver base (src/SOL.hxx:24-126). */
class SOL {
protected:
    fasp_gpu_config cfg_{};
    const LOP*      A = nullptr;
    fasp_gpu_solver h_ = nullptr;
    fasp_gpu_info   info_{};
    bool            dirty_ = true;
    const SOL*      pcdObj_ = nullptr; /* the preconditioner object given to SetupPCD */
    explicit SOL(int alg) { fasp_gpu_default_config(&cfg_, alg); info_.norm2 = info_.normInf = 1e60; }
    /* MG transfer levels of this solver, or of the MG object that preconditions it */
    virtual int SetTransfers(fasp_gpu_solver) const { return SUCCESS; }
    int build()
    {
        if (!A || !A->Device()) return ERROR_SOLVER_TYPE;
        if (h_ && !dirty_) return SUCCESS;
        if (h_) fasp_gpu_solver_destroy(h_);
        h_ = nullptr;
        int e = fasp_gpu_solver_create(&cfg_, &h_);
        if (!e) e = SetTransfers(h_);
        if (!e && pcdObj_) e = pcdObj_->SetTransfers(h_);
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
    /* SOL::SetupPCD (SOL.cxx:249): Identity, Jacobi or MG */
    virtual void SetupPCD(SOL& pc)
    {
        pc.AsPreconditionerOf(cfg_);
        pcdObj_ = &pc;
        dirty_ = true;
    }
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
    using SOL::Setup;
    FaspRetCode Setup(const MAT& M) { return SOL::Setup(M); }
    void AsPreconditionerOf(fasp_gpu_config& c) const override
    {
        c.pcd = 1;
        c.pcdWeight = cfg_.weight;
        c.pcdPrm = cfg_.prm;
    }
};

/* Abstract MG with identity transfers and Jacobi level solvers (src/MG.hxx:44-106), or,
 * with SetTransfer for every coarse level, MG with restriction/prolongation operators and
 * per-level operators (B200; fasp_gpu_solver_set_mg_transfer). As the preconditioner of a
 * Krylov solver (SetupPCD) it runs one MG solve with its own SOLParams. */
template <class TTT>
class MG : public SOL {
    struct Level {
        const MAT* P;
        const MAT* R;
        const MAT* Ac;
    };
    std::vector<Level> levels_;
    int SetTransfers(fasp_gpu_solver h) const override
    {
        for (size_t l = 0; l < levels_.size(); ++l) {
            const Level& v = levels_[l];
            if (!v.P) continue;
            const int e = fasp_gpu_solver_set_mg_transfer(h, (uint32_t)l, v.P->Device(),
                                                          v.R ? v.R->Device() : nullptr,
                                                          v.Ac ? v.Ac->Device() : nullptr);
            if (e) return e;
        }
        return SUCCESS;
    }
public:
    MG() : SOL(FASP_GPU_MG) {}
    /* level `level` (0 = finest): prolongation P from level+1, restriction R (nullptr: the
     * transpose of P), coarse operator Ac (nullptr: the Galerkin product R A P) */
    void SetTransfer(USI level, const MAT& P, const MAT* R = nullptr, const MAT* Ac = nullptr)
    {
        if (levels_.size() <= level) levels_.resize(level + 1, Level{nullptr, nullptr, nullptr});
        levels_[level] = Level{&P, R, Ac};
        dirty_ = true;
    }
    void AsPreconditionerOf(fasp_gpu_config& c) const override
    {
        c.pcd = 2;
        c.pcdPrm = cfg_.prm;
        c.mgLevels = cfg_.mgLevels;
        c.mgCycles = cfg_.mgCycles;
        c.mgSmoothWeight = cfg_.mgSmoothWeight;
        c.mgSmoothPrm = cfg_.mgSmoothPrm;
        c.mgCoarseWeight = cfg_.mgCoarseWeight;
        c.mgCoarsePrm = cfg_.mgCoarsePrm;
    }
    /* the numLevels of SetupALL without binding a matrix (for a preconditioner) */
    void SetNumLevels(USI numLevels) { cfg_.mgLevels = numLevels; dirty_ = true; }
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
