/*
 * ref_shim.cxx -- exposes the FASP++ reference solvers through the oracle C API
 * (fasp_oracle.h). TEST INFRASTRUCTURE ONLY: it is compiled together with the reference
 * sources by build_ref.sh into _ref/liboracle_ref.so, so that tests can run the real
 * reference next to the C restatement and the GPU library on the same inputs.
 *
 * The residual history comes from the reference's own iteration table: the main solver
 * runs with verbose = PRINT_MAX (SOL::PrintInfo prints every iteration when
 * verbose > PRINT_SOME, src/SOL.cxx:46-64), std::cout is captured during Solve, and
 * each "iter | resRel | resAbs |" row fills hist[iter]. Those values carry the
 * 6 significant digits the reference prints.
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "BiCGStab.hxx"
#include "CG.hxx"
#include "FGMRES.hxx"
#include "GMRES.hxx"
#include "Iter.hxx"
#include "MAT.hxx"
#include "MATUtil.hxx"
#include "MG.hxx"
#include "ReadData.hxx"
#include "VEC.hxx"

#include "fasp_oracle.h"

namespace {

struct RefHandle {
    orc_config_t           cfg;
    MAT                    mat;
    SOL*                   sol = nullptr;
    SOL*                   pcd = nullptr;
    std::vector<Jacobi*>   levelSolvers;
    std::vector<IdentityMatrix*> transfers;
    std::string            log;
};

void apply_params(SOL& s, const orc_params_t& p, Output verbose)
{
    s.SetOutput(verbose);
    s.SetMaxIter(p.maxIter);
    s.SetMinIter(p.minIter);
    s.SetSavIter(p.savIter);
    s.SetRestart(p.restart);
    s.SetRelTol(p.relTol);
    s.SetAbsTol(p.absTol);
}

Jacobi* make_jacobi(const orc_params_t& p, double w, const MAT& A)
{
    Jacobi* j = new Jacobi();
    apply_params(*j, p, PRINT_NONE);
    j->SetWeight(w);
    j->Setup(A);
    return j;
}

} // namespace

extern "C" {

void orc_default_params(orc_params_t* p)
{
    SOLParams d;
    p->maxIter = d.maxIter;
    p->minIter = d.minIter;
    p->savIter = d.savIter;
    p->restart = d.restart;
    p->relTol  = d.relTol;
    p->absTol  = d.absTol;
}

void orc_default_config(orc_config_t* c, int alg)
{
    std::memset(c, 0, sizeof(*c));
    c->alg = alg;
    orc_default_params(&c->prm);
    c->weight = 1.0;
    c->pcdWeight = 1.0;
    orc_default_params(&c->pcdPrm);
    c->mgLevels = 3;
    c->mgCycles = 1;
    c->mgSmoothWeight = 1.0;
    c->mgCoarseWeight = 1.0;
    orc_default_params(&c->mgSmoothPrm);
    orc_default_params(&c->mgCoarsePrm);
}

void* orc_create(const orc_config_t* cfg, uint32_t nrow, uint32_t mcol, uint32_t nnz,
                 const uint32_t* rowPtr, const uint32_t* colInd, const double* values)
{
    if (!cfg || nrow == 0 || mcol == 0 || nnz == 0) return nullptr;
    RefHandle* h = new RefHandle();
    h->cfg = *cfg;
    std::vector<USI> rp(rowPtr, rowPtr + nrow + 1), ci(colInd, colInd + nnz);
    if (values) {
        std::vector<DBL> va(values, values + nnz);
        h->mat = MAT(nrow, mcol, nnz, va, ci, rp);
    } else {
        h->mat = MAT(nrow, mcol, nnz, ci, rp);
    }
    const Output loud = PRINT_MAX;

    if (cfg->pcd == 1)
        h->pcd = make_jacobi(cfg->pcdPrm, cfg->pcdWeight, h->mat);
    else
        h->pcd = new Identity();

    std::ostringstream sink; // Setup prints parameters at this verbosity
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    switch (cfg->alg) {
        case ORC_CG: {
            CG* s = new CG();
            apply_params(*s, cfg->prm, loud);
            s->SetupPCD(*h->pcd);
            s->Setup(h->mat);
            h->sol = s;
            break;
        }
        case ORC_BICGSTAB: {
            BiCGStab* s = new BiCGStab();
            apply_params(*s, cfg->prm, loud);
            s->SetupPCD(*h->pcd);
            s->Setup(h->mat);
            h->sol = s;
            break;
        }
        case ORC_GMRES:
        case ORC_GMRES_LEFT: {
            GMRES* s = new GMRES();
            apply_params(*s, cfg->prm, loud);
            if (cfg->maxRestart) s->SetMaxMinRestart(cfg->maxRestart, cfg->minRestart);
            if (cfg->alg == ORC_GMRES_LEFT) s->SetLeftPrecond();
            s->SetupPCD(*h->pcd);
            s->Setup(h->mat);
            h->sol = s;
            break;
        }
        case ORC_FGMRES: {
            FGMRES* s = new FGMRES();
            apply_params(*s, cfg->prm, loud);
            if (cfg->maxRestart) s->SetMaxMinRestart(cfg->maxRestart, cfg->minRestart);
            s->SetupPCD(*h->pcd);
            s->Setup(h->mat);
            h->sol = s;
            break;
        }
        case ORC_JACOBI: {
            Jacobi* s = new Jacobi();
            apply_params(*s, cfg->prm, loud);
            s->SetWeight(cfg->weight);
            s->Setup(h->mat);
            h->sol = s;
            break;
        }
        case ORC_MG: {
            MG<MAT>* s = new MG<MAT>();
            apply_params(*s, cfg->prm, loud);
            const USI L = cfg->mgLevels;
            s->SetupALL(h->mat, L);
            for (USI i = 0; i < L; ++i) {
                IdentityMatrix* t = new IdentityMatrix(h->mat.GetRowSize());
                Jacobi* sm = make_jacobi(cfg->mgSmoothPrm, cfg->mgSmoothWeight, h->mat);
                Jacobi* co = make_jacobi(cfg->mgCoarsePrm, cfg->mgCoarseWeight, h->mat);
                h->transfers.push_back(t);
                h->levelSolvers.push_back(sm);
                h->levelSolvers.push_back(co);
                s->SetupLevel(h->mat, i, t, sm, co);
            }
            s->SetNumCycles(cfg->mgCycles);
            h->sol = s;
            break;
        }
        default:
            break;
    }
    std::cout.rdbuf(old);
    if (!h->sol) {
        delete h->pcd;
        delete h;
        return nullptr;
    }
    return h;
}

int orc_solve(void* hv, const double* b, double* x, uint32_t* numIter, double* norm2,
              double* normInf, double* hist, uint32_t histCap)
{
    RefHandle* h = static_cast<RefHandle*>(hv);
    const USI nrow = h->mat.GetRowSize(), mcol = h->mat.GetColSize();
    VEC vb(nrow, b), vx(mcol, x);
    std::ostringstream cap;
    std::streambuf* old = std::cout.rdbuf(cap.rdbuf());
    const FaspRetCode code = h->sol->Solve(vb, vx);
    std::cout.rdbuf(old);
    h->log = cap.str();
    for (USI i = 0; i < mcol; ++i) x[i] = vx[i];
    if (numIter) *numIter = h->sol->GetIterations();
    if (norm2) *norm2 = h->sol->GetNorm2();
    if (normInf) *normInf = h->sol->GetInfNorm();
    for (uint32_t k = 0; k < histCap; ++k) hist[k] = NAN;
    std::istringstream in(h->log);
    std::string line;
    while (std::getline(in, line)) {
        unsigned it;
        double rr, ra;
        if (std::sscanf(line.c_str(), "%u | %lf | %lf |", &it, &rr, &ra) == 3 && it < histCap)
            hist[it] = ra;
    }
    return static_cast<int>(code);
}

void orc_clean(void* hv)
{
    RefHandle* h = static_cast<RefHandle*>(hv);
    if (h->cfg.alg == ORC_GMRES || h->cfg.alg == ORC_GMRES_LEFT ||
        h->cfg.alg == ORC_FGMRES || h->cfg.alg == ORC_CG || h->cfg.alg == ORC_BICGSTAB)
        h->sol->Clean();
}

void orc_destroy(void* hv)
{
    RefHandle* h = static_cast<RefHandle*>(hv);
    if (!h) return;
    /* SOL has no virtual destructor (src/SOL.hxx:54): delete through the real type. */
    switch (h->cfg.alg) {
        case ORC_CG: delete static_cast<CG*>(h->sol); break;
        case ORC_BICGSTAB: delete static_cast<BiCGStab*>(h->sol); break;
        case ORC_GMRES:
        case ORC_GMRES_LEFT: delete static_cast<GMRES*>(h->sol); break;
        case ORC_FGMRES: delete static_cast<FGMRES*>(h->sol); break;
        case ORC_JACOBI: delete static_cast<Jacobi*>(h->sol); break;
        case ORC_MG: delete static_cast<MG<MAT>*>(h->sol); break;
        default: break;
    }
    if (h->cfg.pcd == 1)
        delete static_cast<Jacobi*>(h->pcd);
    else
        delete static_cast<Identity*>(h->pcd);
    for (auto* j : h->levelSolvers) delete j;
    for (auto* t : h->transfers) delete t;
    delete h;
}

void orc_spmv(uint32_t nrow, const uint32_t* rowPtr, const uint32_t* colInd,
              const double* values, const double* x, double* y)
{
    const uint32_t nnz = rowPtr[nrow];
    uint32_t mcol = 0;
    for (uint32_t k = 0; k < nnz; ++k) mcol = colInd[k] + 1 > mcol ? colInd[k] + 1 : mcol;
    if (mcol < nrow) mcol = nrow;
    std::vector<USI> rp(rowPtr, rowPtr + nrow + 1), ci(colInd, colInd + nnz);
    MAT A;
    if (values) {
        std::vector<DBL> va(values, values + nnz);
        A = MAT(nrow, mcol, nnz, va, ci, rp);
    } else {
        A = MAT(nrow, mcol, nnz, ci, rp);
    }
    VEC vx(mcol, x), vy(nrow, 0.0);
    A.Apply(vx, vy);
    for (uint32_t i = 0; i < nrow; ++i) y[i] = vy[i];
}

void orc_residual(uint32_t nrow, uint32_t mcol, const uint32_t* rowPtr,
                  const uint32_t* colInd, const double* values, const double* b,
                  const double* x, double* r)
{
    const uint32_t nnz = rowPtr[nrow];
    std::vector<USI> rp(rowPtr, rowPtr + nrow + 1), ci(colInd, colInd + nnz);
    std::vector<DBL> va(values, values + nnz);
    MAT A(nrow, mcol, nnz, va, ci, rp);
    VEC vb(nrow, b), vx(mcol, x), vr(nrow, 0.0);
    A.Residual(vb, vx, vr);
    for (uint32_t i = 0; i < nrow; ++i) r[i] = vr[i];
}

double orc_dot(uint32_t n, const double* a, const double* b)
{
    VEC va(n, a), vb(n, b);
    return va.Dot(vb);
}

double orc_norm2(uint32_t n, const double* a)
{
    VEC va(n, a);
    return va.Norm2();
}

double orc_norminf(uint32_t n, const double* a)
{
    VEC va(n, a);
    return va.NormInf();
}

void orc_transpose(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                   const uint32_t* colInd, const double* values, uint32_t* tRowPtr,
                   uint32_t* tColInd, double* tValues, uint32_t* tDiagPtr)
{
    std::vector<USI> rp(rowPtr, rowPtr + nrow + 1), ci(colInd, colInd + nnz);
    MAT A;
    if (values) {
        std::vector<DBL> va(values, values + nnz);
        A = MAT(nrow, mcol, nnz, va, ci, rp);
    } else {
        A = MAT(nrow, mcol, nnz, ci, rp);
    }
    A.TransInPlace();
    int* trp = A.GetRowPtr();
    int* tci = A.GetColInd();
    for (uint32_t i = 0; i <= mcol; ++i) tRowPtr[i] = (uint32_t)trp[i];
    for (uint32_t k = 0; k < nnz; ++k) tColInd[k] = (uint32_t)tci[k];
    delete[] trp;
    delete[] tci;
    if (values && tValues) {
        double* tv = A.GetValues();
        for (uint32_t k = 0; k < nnz; ++k) tValues[k] = tv[k];
        delete[] tv;
    }
    if (tDiagPtr) {
        /* MAT keeps diagPtr private; FormDiagPtr's search is restated here. */
        for (uint32_t j = 0; j < mcol; ++j) {
            tDiagPtr[j] = 0;
            for (uint32_t k = tRowPtr[j]; k < tRowPtr[j + 1]; ++k)
                if (tColInd[k] == j) {
                    tDiagPtr[j] = k;
                    break;
                }
        }
    }
}

int orc_mult_transpose_add(uint32_t nrow, uint32_t mcol, const uint32_t* rowPtr,
                           const uint32_t* colInd, const double* values, const double* v1,
                           const double* v2, double* v)
{
    /* the reference's last loop reads A's rowPtr[i + 1] for every row i of A^T (MAT.cxx:603):
     * past its end unless A is square; a pattern-only A reads its empty values array */
    if (nrow != mcol || !values) return ORC_REF_UNDEFINED;
    const uint32_t nnz = rowPtr[nrow];
    std::vector<USI> rp(rowPtr, rowPtr + nrow + 1), ci(colInd, colInd + nnz);
    std::vector<DBL> va(values, values + nnz);
    MAT A(nrow, mcol, nnz, va, ci, rp);
    VEC a(nrow, v1), b(mcol, v2), out(mcol, 0.0);
    A.MultTransposeAdd(a, b, out);
    for (uint32_t i = 0; i < mcol; ++i) v[i] = out[i];
    return 0;
}

void orc_diagptr(uint32_t nrow, const uint32_t* rowPtr, const uint32_t* colInd,
                 uint32_t* diagPtr)
{
    for (uint32_t j = 0; j < nrow; ++j) {
        diagPtr[j] = 0;
        for (uint32_t k = rowPtr[j]; k < rowPtr[j + 1]; ++k)
            if (colInd[k] == j) {
                diagPtr[j] = k;
                break;
            }
    }
}

/* The MAT's arrays; *nnzOut = 0 for an empty MAT. */
static void copy_mat(const MAT& A, uint32_t* nnzOut, uint32_t* rowPtr, uint32_t* colInd,
                     double* values)
{
    *nnzOut = A.GetNNZ();
    if (*nnzOut == 0) return;
    int* rp = A.GetRowPtr();
    int* ci = A.GetColInd();
    double* va = A.GetValues();
    for (uint32_t i = 0; i <= A.GetRowSize(); ++i) rowPtr[i] = (uint32_t)rp[i];
    for (uint32_t k = 0; k < *nnzOut; ++k) {
        colInd[k] = (uint32_t)ci[k];
        values[k] = va[k];
    }
    delete[] rp;
    delete[] ci;
    delete[] va;
}

/* Inputs on which SortCSRRow or CSRtoMAT index out of bounds (fasp_oracle.h): rp is the
 * 0-based row pointer of the rows as they reach SortCSRRow. */
static bool row0_undefined(const std::vector<USI>& rp, const std::vector<USI>& ci)
{
    if (rp.size() < 2) return false;
    if (rp[1] == rp[0]) return true; /* empty first row: CSRtoMAT reads colInd[end - 1] */
    for (USI k = rp[0] + 1; k < rp[1]; ++k)
        if (ci[k] < ci[rp[0]]) return true; /* SortCSRRow moves it to position 0 */
    return false;
}

int orc_mtx_to_mat(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowInd,
                   const uint32_t* colInd, const double* values, uint32_t* nnzOut,
                   uint32_t* rowPtr, uint32_t* colIndOut, double* valuesOut)
{
    *nnzOut = 0;
    std::vector<USI> ri(rowInd, rowInd + nnz), ci(colInd, colInd + nnz);
    std::vector<DBL> va(values, values + nnz);
    /* the first row as MTXtoCSR's stable scatter hands it to SortCSRRow */
    std::vector<USI> rp0{0, 0}, ci0;
    for (uint32_t j = 0; j < nnz; ++j) {
        if (ri[j] >= nrow) return ORC_REF_UNDEFINED;
        if (ri[j] == 0) ci0.push_back(ci[j]);
    }
    rp0[1] = (USI)ci0.size();
    if (row0_undefined(rp0, ci0)) return ORC_REF_UNDEFINED;
    MAT A;
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    const FaspRetCode code = MTXtoMAT(nrow, mcol, nnz, ri, ci, va, A);
    std::cout.rdbuf(old);
    copy_mat(A, nnzOut, rowPtr, colIndOut, valuesOut);
    return static_cast<int>(code);
}

int orc_csr_to_mat(uint32_t nrow, uint32_t nnz, const uint32_t* rowPtr, const uint32_t* colInd,
                   const double* values, uint32_t* nnzOut, uint32_t* rowPtrOut,
                   uint32_t* colIndOut, double* valuesOut)
{
    *nnzOut = 0;
    std::vector<USI> rp(rowPtr, rowPtr + nrow + 1), ci(colInd, colInd + nnz);
    std::vector<DBL> va(values, values + nnz);
    USI row = nrow, col = nrow, nz = nnz;
    if (rp[0] == 1) { /* ReadCSR's shift, ReadData.cxx:350-353 */
        for (auto& v : rp) --v;
        for (auto& v : ci) --v;
    }
    /* SortCSRRow sorts before it checks: only well-formed row pointers reach it */
    if (rp[0] != 0 || rp[nrow] != nnz) return ORC_REF_UNDEFINED;
    for (uint32_t i = 0; i < nrow; ++i)
        if (rp[i] > rp[i + 1]) return ORC_REF_UNDEFINED;
    if (row0_undefined(rp, ci)) return ORC_REF_UNDEFINED;
    MAT A;
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    FaspRetCode code = SortCSRRow(row, col, nz, rp, ci, va); /* ReadData.cxx:376-400 */
    if (code >= 0) code = CSRtoMAT(row, col, nz, va, ci, rp, A);
    std::cout.rdbuf(old);
    copy_mat(A, nnzOut, rowPtrOut, colIndOut, valuesOut);
    return static_cast<int>(code);
}

int orc_mat_mult(uint32_t nl, uint32_t ml, const uint32_t* rpl, const uint32_t* cil,
                 const double* val, uint32_t mr, const uint32_t* rpr, const uint32_t* cir,
                 const double* var, uint32_t cap, uint32_t* nnzC, uint32_t* rpC,
                 uint32_t* ciC, double* vaC)
{
    std::vector<USI> lrp(rpl, rpl + nl + 1), lci(cil, cil + rpl[nl]);
    std::vector<DBL> lva(val, val + rpl[nl]);
    std::vector<USI> rrp(rpr, rpr + ml + 1), rci(cir, cir + rpr[ml]);
    std::vector<DBL> rva(var, var + rpr[ml]);
    MAT L(nl, ml, rpl[nl], lva, lci, lrp), R(ml, mr, rpr[ml], rva, rci, rrp), C;
    C.Mult(L, R);
    *nnzC = C.GetNNZ();
    if (*nnzC > cap) return -1;
    int* rp = C.GetRowPtr();
    int* ci = C.GetColInd();
    double* va = C.GetValues();
    for (uint32_t i = 0; i <= nl; ++i) rpC[i] = (uint32_t)rp[i];
    for (uint32_t k = 0; k < *nnzC; ++k) {
        ciC[k] = (uint32_t)ci[k];
        vaC[k] = va[k];
    }
    delete[] rp;
    delete[] ci;
    delete[] va;
    return 0;
}

int orc_mat_add(uint32_t n, uint32_t m, double a, const uint32_t* arp, const uint32_t* aci,
                const double* ava, double b, const uint32_t* brp, const uint32_t* bci,
                const double* bva, uint32_t* nnzC, uint32_t* rpC, uint32_t* ciC, double* vaC)
{
    /* row 0 as MAT::Add builds it before sorting: A's columns, then B's unmatched ones */
    std::vector<USI> row0(aci, aci + arp[1]);
    for (uint32_t k = brp[0]; k < brp[1]; ++k) {
        bool hit = false;
        for (USI c : row0) hit = hit || c == bci[k];
        if (!hit) row0.push_back(bci[k]);
    }
    std::vector<USI> rp0{0, (USI)row0.size()};
    if (!row0.empty() && row0_undefined(rp0, row0)) return ORC_REF_UNDEFINED;
    std::vector<USI> arpv(arp, arp + n + 1), aciv(aci, aci + arp[n]);
    std::vector<DBL> avav(ava, ava + arp[n]);
    std::vector<USI> brpv(brp, brp + n + 1), bciv(bci, bci + brp[n]);
    std::vector<DBL> bvav(bva, bva + brp[n]);
    MAT A(n, m, arp[n], avav, aciv, arpv), B(n, m, brp[n], bvav, bciv, brpv), C;
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    C.Add(a, A, b, B);
    std::cout.rdbuf(old);
    copy_mat(C, nnzC, rpC, ciC, vaC);
    return 0;
}

/* ReadMat (src/ReadData.cxx:361-446) of a .csr/.mtx file: call once with NULL arrays to
 * get nrow and nnz, then with arrays of those sizes. Returns the FaspRetCode. */
int orc_ref_readmat(const char* path, uint32_t* nrow, uint32_t* nnz, uint32_t* rowPtr,
                    uint32_t* colInd, double* values)
{
    MAT A;
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    const FaspRetCode code = ReadMat(path, A);
    std::cout.rdbuf(old);
    if (code < 0) return static_cast<int>(code);
    *nrow = A.GetRowSize();
    *nnz = A.GetNNZ();
    if (rowPtr && colInd && values) {
        int* rp = A.GetRowPtr();
        int* ci = A.GetColInd();
        double* va = A.GetValues();
        for (uint32_t i = 0; i <= *nrow; ++i) rowPtr[i] = (uint32_t)rp[i];
        for (uint32_t k = 0; k < *nnz; ++k) {
            colInd[k] = (uint32_t)ci[k];
            values[k] = va[k];
        }
        delete[] rp;
        delete[] ci;
        delete[] va;
    }
    return static_cast<int>(code);
}

} // extern "C"

