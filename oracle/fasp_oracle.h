/*
 * fasp_oracle.h -- CPU ORACLE for the iterative-solve path. TEST INFRASTRUCTURE ONLY.
 *
 * This header is shared by two interchangeable CPU back ends that tests load side by side:
 *   - liboracle_port.so  : fasp_oracle.c, a plain-C restatement of the FASP++ algorithms
 *                          (each function cites the reference file:line it follows);
 *   - _ref/liboracle_ref.so : ref_shim.cxx linked against the FASP++ sources compiled from
 *                          their own tree (build_ref.sh), used to pin the restatement.
 * Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline leg and the
 * reference arm) may load either library, and only as the checker or the timed CPU
 * baseline -- never as part of the product path.
 *
 * Index arrays are 32-bit unsigned, like the reference's USI. values == NULL means a
 * pattern-only matrix (MAT.cxx:420-451 treats every stored entry as 1).
 */
#ifndef FASP_ORACLE_H
#define FASP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Solver kinds; numbers follow SOLType (src/Param.hxx:36-54). GMRES_LEFT is the
 * left-preconditioned GMRES::LSolve (src/GMRES.cxx:283-453). */
enum {
    ORC_IDENTITY   = 0,
    ORC_CG         = 1,
    ORC_BICGSTAB   = 2,
    ORC_GMRES      = 4,
    ORC_FGMRES     = 5,
    ORC_JACOBI     = 11,
    ORC_MG         = 21,
    ORC_GMRES_LEFT = 104
};

/* Mirrors SOLParams (src/Param.hxx:57-80) minus the name/verbosity fields. */
typedef struct {
    uint32_t maxIter, minIter, savIter, restart;
    double   relTol, absTol;
} orc_params_t;

typedef struct {
    int          alg;        /* ORC_* above */
    orc_params_t prm;        /* the solver's own SOLParams */
    double       weight;     /* Jacobi weight when alg == ORC_JACOBI (Iter.hxx:45) */
    uint32_t     maxRestart, minRestart; /* GMRES/FGMRES::SetMaxMinRestart; 0,0 = 30,10 */
    int          pcd;        /* preconditioner: 0 identity, 1 Jacobi */
    double       pcdWeight;
    orc_params_t pcdPrm;     /* the Jacobi preconditioner's SOLParams */
    uint32_t     mgLevels;   /* MG: number of coarse levels (TestMG.cxx:80) */
    uint32_t     mgCycles;   /* MG: SetNumCycles (MG.cxx:19-23) */
    double       mgSmoothWeight, mgCoarseWeight;
    orc_params_t mgSmoothPrm, mgCoarsePrm;
} orc_config_t;

/* SOLParams() defaults (src/Param.hxx:68-79). */
void orc_default_params(orc_params_t* p);
void orc_default_config(orc_config_t* c, int alg);

/* A solver object bound to one CSRx matrix: the Setup(...) of the reference. The
 * arrays are copied. Returns NULL on a bad config. */
void* orc_create(const orc_config_t* cfg, uint32_t nrow, uint32_t mcol, uint32_t nnz,
                 const uint32_t* rowPtr, const uint32_t* colInd, const double* values);

/* Solve(b, x): x is the initial guess in and the solution out. hist[k] receives the
 * residual norm the solver holds at the end of iteration k (k = 0..numIter, entries the
 * solver never computes are NaN). Returns the FaspRetCode. */
int orc_solve(void* h, const double* b, double* x, uint32_t* numIter, double* norm2,
              double* normInf, double* hist, uint32_t histCap);

/* Clean(): reset work vectors (FGMRES Z basis included). */
void orc_clean(void* h);
void orc_destroy(void* h);

/* Elementary operators on a CSRx matrix given by arrays. */
void   orc_spmv(uint32_t nrow, const uint32_t* rowPtr, const uint32_t* colInd,
                const double* values, const double* x, double* y);
void   orc_residual(uint32_t nrow, uint32_t mcol, const uint32_t* rowPtr,
                    const uint32_t* colInd, const double* values, const double* b,
                    const double* x, double* r);
double orc_dot(uint32_t n, const double* a, const double* b);
double orc_norm2(uint32_t n, const double* a);
double orc_norminf(uint32_t n, const double* a);
/* MAT::TransInPlace: (nrow x mcol) -> (mcol x nrow); outputs sized mcol+1, nnz, nnz, mcol. */
void   orc_transpose(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                     const uint32_t* colInd, const double* values, uint32_t* tRowPtr,
                     uint32_t* tColInd, double* tValues, uint32_t* tDiagPtr);
/* MAT::MultTransposeAdd (MAT.cxx:541-606): v = A^T v1 + v2 for A (nrow x mcol); v1 has
 * nrow entries, v2 and v mcol. v starts as v2 and each v[i] adds the products of column i in
 * the transpose's order (ascending row). The reference bounds each row of the transpose by
 * A's own rowPtr[i + 1] (MAT.cxx:603); the restatement uses the transpose's row end, which
 * is the same whenever A's row pointers equal its transpose's (structurally symmetric A).
 * values == NULL: every stored entry counts as 1, as in MAT::Apply. Returns 0. The
 * reference shim returns ORC_REF_UNDEFINED for nrow != mcol (its loop then reads past
 * A's row pointers). */
int    orc_mult_transpose_add(uint32_t nrow, uint32_t mcol, const uint32_t* rowPtr,
                              const uint32_t* colInd, const double* values, const double* v1,
                              const double* v2, double* v);
/* MAT::FormDiagPtr */
void   orc_diagptr(uint32_t nrow, const uint32_t* rowPtr, const uint32_t* colInd,
                   uint32_t* diagPtr);

/* ReadMat's conversions (src/ReadData.cxx:361-446). Outputs hold nrow + 1, nnz + nrow and
 * nnz + nrow entries; *nnzOut = the nnz of the resulting MAT, 0 when it is left empty.
 * orc_mtx_to_mat: MTXtoMAT (src/MATUtil.cxx:416-436) of ReadMTX's 0-based triplets;
 *   returns MTXtoMAT's code, which is SUCCESS even when CSRtoMAT's check fails.
 * orc_csr_to_mat: ReadCSR's 1-based shift (ReadData.cxx:350-353), SortCSRRow and
 *   CSRtoMAT (ReadData.cxx:376-400) of a square matrix's raw CSR arrays; returns the code.
 * The reference library returns ORC_REF_UNDEFINED, without calling the reference, for
 * inputs on which the reference reads or writes out of bounds: a row index >= nrow; an
 * entry of row 0 that sorts before the row's first entry (SortCSRRow's unsigned index
 * wraps, MATUtil.cxx:459); an empty first row without a diagonal (CSRtoMAT reads
 * colInd[-1], :369). */
#define ORC_REF_UNDEFINED (-1000)
int    orc_mtx_to_mat(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowInd,
                      const uint32_t* colInd, const double* values, uint32_t* nnzOut,
                      uint32_t* rowPtr, uint32_t* colIndOut, double* valuesOut);
int    orc_csr_to_mat(uint32_t nrow, uint32_t nnz, const uint32_t* rowPtr,
                      const uint32_t* colInd, const double* values, uint32_t* nnzOut,
                      uint32_t* rowPtrOut, uint32_t* colIndOut, double* valuesOut);

/* The right-hand side of the reference's matrix-free example (example/TestMatFree.cxx:41-85,
 * Poisson2D.hxx TEST_PROBLEM 1) on the (dim-1)^2 interior grid. Port library only. */
void   orc_matfree_rhs(int dim, double* b);

/* MAT::Mult (src/MAT.cxx:715-800): C = L R (L: nl x ml, R: ml x mr). cap = capacity of
 * ciC/vaC in entries; rpC holds nl + 1. Returns 0, or -1 when cap is too small (*nnzC is
 * then the size needed). */
int    orc_mat_mult(uint32_t nl, uint32_t ml, const uint32_t* rpl, const uint32_t* cil,
                    const double* val, uint32_t mr, const uint32_t* rpr, const uint32_t* cir,
                    const double* var, uint32_t cap, uint32_t* nnzC, uint32_t* rpC,
                    uint32_t* ciC, double* vaC);

/* Port library only: MG with transfer operators (the B200 library's
 * fasp_gpu_solver_set_mg_transfer) on a handle made by orc_create with alg ORC_MG: level l
 * gets prolongation P (n_l x n_{l+1}), restriction R (n_{l+1} x n_l) and the operator
 * A_{l+1} (an x an). MG::MGCycle (src/MG.cxx:105-152) then runs with level l's residual
 * on A_l, R and P as the transfers, the smoother of level l on A_l and the coarse solver
 * on A_{l+1}. Every coarse level must be set before orc_solve. */
int    orc_mg_set_level(void* h, uint32_t level,
                        uint32_t pn, uint32_t pm, uint32_t pnnz, const uint32_t* prp,
                        const uint32_t* pci, const double* pva,
                        uint32_t rn, uint32_t rm, uint32_t rnnz, const uint32_t* rrp,
                        const uint32_t* rci, const double* rva,
                        uint32_t an, uint32_t annz, const uint32_t* arp, const uint32_t* aci,
                        const double* ava);

/* MAT::Add (src/MAT.cxx:652-713): C = a A + b B (n x m each); outputs hold nnz(A) + nnz(B)
 * entries and n + 1 row pointers. The reference library returns ORC_REF_UNDEFINED, without
 * calling the reference, when the sort of a row 0 would move an entry to the front
 * (SortCSRRow's unsigned index wraps). */
int    orc_mat_add(uint32_t n, uint32_t m, double a, const uint32_t* arp, const uint32_t* aci,
                   const double* ava, double b, const uint32_t* brp, const uint32_t* bci,
                   const double* bva, uint32_t* nnzC, uint32_t* rpC, uint32_t* ciC,
                   double* vaC);

/* Reference library only (_ref/liboracle_ref.so): ReadMat of a .csr/.mtx file. */
int    orc_ref_readmat(const char* path, uint32_t* nrow, uint32_t* nnz, uint32_t* rowPtr,
                       uint32_t* colInd, double* values);

#ifdef __cplusplus
}
#endif
#endif
