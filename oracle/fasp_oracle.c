/*
 * fasp_oracle.c -- CPU ORACLE (test infrastructure only; see fasp_oracle.h).
 *
 * A plain-C restatement of the FASP++ iterative-solve path. Every routine follows one
 * reference routine statement by statement so that, compiled with -ffp-contract=off,
 * it reproduces the reference's floating-point results bit for bit (the summation
 * orders of VEC::Dot / Norm2 and the row loop of MAT::Apply are kept). References are
 * to FaspDevTeam/faspxx paths.
 *
 * Where the reference has undefined behaviour, the restatement does what the code
 * plainly intends, and the same change is applied to the reference build that pins it
 * (oracle/build_ref.sh):
 *   - CG.cxx:213 `pk.SetValues(0.0)` resizes pk to length 0 (then reads it): here pk=0.
 *   - GMRES.cxx:214,224,386,396 and FGMRES.cxx:209,219 count an unsigned index down
 *     with `k >= 0`: here the loops are signed.
 *   - GMRES/FGMRES size `var` by the problem size (GMRES.cxx:53): here by
 *     max(n, maxRestart + 1).
 *   - CG breakdown on the first iteration reads an uninitialised alpha: here alpha = 0.
 * One guard goes beyond the reference: an adaptive restart that wraps below zero in
 * unsigned arithmetic (GMRES.cxx:261-262 with restart < 3) is capped at maxRestart.
 */
#include "fasp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* FaspRetCode values (src/RetCode.hxx:24-55) and constants (include/Faspxx.hxx:31-46). */
#define SUCCESS 0
#define ERROR_INPUT_PAR -12
#define ERROR_DIVIDE_ZERO -18
#define ERROR_SOLVER_STAG -32
#define ERROR_SOLVER_SOLSTAG -33
#define ERROR_SOLVER_TOLSMALL -34
#define ERROR_SOLVER_MAXIT -39
#define CLOSE_ZERO 1e-20
#define SMALL_DBL (-1e+60)
#define KSM_CHK_RATIO 0.95
#define MAX_STAG_NUM 20u
#define MAX_ITER_NUM 100000u
/* Variable-restart constants (src/GMRES.hxx:46-48, src/FGMRES.hxx:47-49). */
#define MAX_CR 0.99026806874157040
#define MIN_CR 0.17364817766693041
#define RESTART_DECREASE 3u

/* ------------------------------------------------------------------------------------
 * VEC restatement (src/VEC.cxx). Loops keep the reference's 4-way partial sums.
 * ---------------------------------------------------------------------------------- */

/* VEC::Dot, VEC.cxx:468-485 */
double orc_dot(uint32_t n, const double* a, const double* b)
{
    const uint32_t len = n - n % 4;
    double d1 = 0.0, d2 = 0.0, d3 = 0.0, d4 = 0.0;
    uint32_t i;
    for (i = 0; i < len; i += 4) {
        d1 += a[i] * b[i];
        d2 += a[i + 1] * b[i + 1];
        d3 += a[i + 2] * b[i + 2];
        d4 += a[i + 3] * b[i + 3];
    }
    for (i = len; i < n; ++i) d1 += a[i] * b[i];
    return d1 + d2 + d3 + d4;
}

/* VEC::Norm2, VEC.cxx:424-438 (std::pow(v, 2) is v*v exactly) */
double orc_norm2(uint32_t n, const double* a)
{
    const uint32_t len = n - n % 4;
    double t1 = 0.0, t2 = 0.0, t3 = 0.0, t4 = 0.0;
    uint32_t i;
    for (i = 0; i < len; i += 4) {
        t1 += a[i] * a[i];
        t2 += a[i + 1] * a[i + 1];
        t3 += a[i + 2] * a[i + 2];
        t4 += a[i + 3] * a[i + 3];
    }
    for (i = len; i < n; ++i) t1 += a[i] * a[i];
    return sqrt(t1 + t2 + t3 + t4);
}

/* VEC::NormInf, VEC.cxx:441-465 (a NaN never wins a `>` comparison) */
double orc_norminf(uint32_t n, const double* a)
{
    const uint32_t len = n - n % 4;
    double m1 = 0.0, m2 = 0.0, m3 = 0.0, m4 = 0.0, t;
    uint32_t i;
    for (i = 0; i < len; i += 4) {
        t = fabs(a[i]);
        if (t > m1) m1 = t;
        t = fabs(a[i + 1]);
        if (t > m2) m2 = t;
        t = fabs(a[i + 2]);
        if (t > m3) m3 = t;
        t = fabs(a[i + 3]);
        if (t > m4) m4 = t;
    }
    for (i = len; i < n; ++i) {
        t = fabs(a[i]);
        if (t > m1) m1 = t;
    }
    m1 = m1 >= m2 ? m1 : m2;
    m3 = m3 >= m4 ? m3 : m4;
    return m1 > m3 ? m1 : m3;
}

/* VEC::AXPY, VEC.cxx:245-256: y += a*x */
static void v_axpy(uint32_t n, double a, const double* x, double* y)
{
    for (uint32_t i = 0; i < n; ++i) y[i] += a * x[i];
}

/* VEC::XPAY, VEC.cxx:259-271: y = a*y + x */
static void v_xpay(uint32_t n, double a, const double* x, double* y)
{
    for (uint32_t i = 0; i < n; ++i) y[i] = a * y[i] + x[i];
}

/* VEC::AXPBY, VEC.cxx:274-326: x = a*x + b*y (the a==1 / b==1 cases give the same
 * values, since multiplication by 1.0 is exact) */
static void v_axpby(uint32_t n, double a, double b, const double* y, double* x)
{
    for (uint32_t i = 0; i < n; ++i) x[i] = a * x[i] + b * y[i];
}

/* VEC::WAXPBY, VEC.cxx:329-379: w = a*v1 + b*v2 */
static void v_waxpby(uint32_t n, double a, const double* v1, double b, const double* v2,
                     double* w)
{
    for (uint32_t i = 0; i < n; ++i) w[i] = a * v1[i] + b * v2[i];
}

/* VEC::Scale, VEC.cxx:154-165 */
static void v_scale(uint32_t n, double a, double* x)
{
    for (uint32_t i = 0; i < n; ++i) x[i] *= a;
}

static void v_set(uint32_t n, double v, double* x)
{
    for (uint32_t i = 0; i < n; ++i) x[i] = v;
}

static void v_copy(uint32_t n, const double* src, double* dst)
{
    if (n) memcpy(dst, src, (size_t)n * sizeof(double));
}

/* ------------------------------------------------------------------------------------
 * MAT restatement (src/MAT.cxx)
 * ---------------------------------------------------------------------------------- */

typedef struct {
    uint32_t  nrow, mcol, nnz;
    uint32_t* rowPtr;
    uint32_t* colInd;
    uint32_t* diagPtr;
    double*   values; /* NULL: pattern only */
} omat_t;

/* MAT::Apply, MAT.cxx:373-452. The 4/5/6-entry unrolled cases sum in the same
 * left-to-right order as the general loop, so one loop restates all of them. */
void orc_spmv(uint32_t nrow, const uint32_t* rowPtr, const uint32_t* colInd,
              const double* values, const double* v, double* w)
{
    for (uint32_t i = 0; i < nrow; ++i) {
        const uint32_t begin = rowPtr[i], end = rowPtr[i + 1];
        double s;
        if (values) {
            s = values[begin] * v[colInd[begin]];
            for (uint32_t k = begin + 1; k < end; ++k) s += values[k] * v[colInd[k]];
        } else {
            s = v[colInd[begin]];
            for (uint32_t k = begin + 1; k < end; ++k) s += v[colInd[k]];
        }
        w[i] = s;
    }
}

/* MAT::Residual, MAT.cxx:455-476, including the x ~ 0 shortcut r = b (:459-462). */
void orc_residual(uint32_t nrow, uint32_t mcol, const uint32_t* rowPtr,
                  const uint32_t* colInd, const double* values, const double* b,
                  const double* x, double* r)
{
    if (orc_norminf(mcol, x) < CLOSE_ZERO) {
        v_copy(nrow, b, r);
        return;
    }
    for (uint32_t i = 0; i < nrow; ++i) {
        const uint32_t begin = rowPtr[i];
        double s = b[i] - values[begin] * x[colInd[begin]];
        for (uint32_t k = begin + 1; k < rowPtr[i + 1]; ++k) s -= values[k] * x[colInd[k]];
        r[i] = s;
    }
}

/* MAT::FormDiagPtr, MAT.cxx:917-928 (a row without a diagonal keeps 0) */
void orc_diagptr(uint32_t nrow, const uint32_t* rowPtr, const uint32_t* colInd,
                 uint32_t* diagPtr)
{
    for (uint32_t j = 0; j < nrow; ++j) {
        diagPtr[j] = 0;
        for (uint32_t k = rowPtr[j]; k < rowPtr[j + 1]; ++k) {
            if (colInd[k] == j) {
                diagPtr[j] = k;
                break;
            }
        }
    }
}

/* MAT::TransInPlace, MAT.cxx:479-538: counting sort by column into rowPtr[c+2],
 * prefix sum from index 2, then a row-ordered scatter through rowPtr[c+1]. */
void orc_transpose(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                   const uint32_t* colInd, const double* values, uint32_t* tRowPtr,
                   uint32_t* tColInd, double* tValues, uint32_t* tDiagPtr)
{
    const uint32_t m = mcol;
    for (uint32_t i = 0; i <= m; ++i) tRowPtr[i] = 0;
    for (uint32_t j = 0; j < nnz; ++j) {
        const uint32_t i = colInd[j];
        if (i < m - 1) ++tRowPtr[i + 2];
    }
    for (uint32_t i = 2; i <= m; ++i) tRowPtr[i] += tRowPtr[i - 1];
    for (uint32_t i = 0; i < nrow; ++i) {
        for (uint32_t p = rowPtr[i]; p < rowPtr[i + 1]; ++p) {
            const uint32_t j = colInd[p] + 1;
            const uint32_t k = tRowPtr[j];
            tColInd[k] = i;
            if (values && tValues) tValues[k] = values[p];
            tRowPtr[j] = k + 1;
        }
    }
    if (tDiagPtr) orc_diagptr(m, tRowPtr, tColInd, tDiagPtr);
}

/* MAT::MultTransposeAdd, MAT.cxx:541-606: the transpose formed as TransInPlace forms it
 * (:556-590), then v = v2 (:592) and v[i] += v1[col] * value over row i of the transpose in
 * order (:595-605), each product rounded before the add. */
int orc_mult_transpose_add(uint32_t nrow, uint32_t mcol, const uint32_t* rowPtr,
                           const uint32_t* colInd, const double* values, const double* v1,
                           const double* v2, double* v)
{
    const uint32_t nnz = rowPtr[nrow];
    uint32_t* trp = (uint32_t*)calloc((size_t)mcol + 2, sizeof(uint32_t));
    uint32_t* tci = (uint32_t*)malloc(((size_t)nnz + 1) * sizeof(uint32_t));
    double*   tva = values ? (double*)malloc(((size_t)nnz + 1) * sizeof(double)) : NULL;
    if (!trp || !tci || (values && !tva)) {
        free(trp);
        free(tci);
        free(tva);
        return -20;
    }
    orc_transpose(nrow, mcol, nnz, rowPtr, colInd, values, trp, tci, tva, NULL);
    for (uint32_t i = 0; i < mcol; ++i) {
        double acc = v2[i];
        for (uint32_t j = trp[i]; j < trp[i + 1]; ++j) {
            const double prod = v1[tci[j]] * (tva ? tva[j] : 1.0);
            acc += prod;
        }
        v[i] = acc;
    }
    free(trp);
    free(tci);
    free(tva);
    return 0;
}

/* ------------------------------------------------------------------------------------
 * ReadMat's conversions (src/ReadData.cxx:361-446, src/MATUtil.cxx:110-476)
 * ---------------------------------------------------------------------------------- */

#define ERROR_MAT_DATA -17

/* CheckCSR, MATUtil.cxx:110-174 (the array-size checks hold by construction here). */
static int check_csr(uint32_t row, uint32_t col, uint32_t nnz, const uint32_t* colInd,
                     const uint32_t* rowPtr)
{
    if (row == 0 || col == 0 || nnz == 0) return SUCCESS;
    if (nnz != rowPtr[row] - rowPtr[0]) return ERROR_MAT_DATA;
    for (uint32_t j = 0; j < row; ++j)
        if (rowPtr[j] > rowPtr[j + 1]) return ERROR_MAT_DATA;
    for (uint32_t j = 0; j < row; ++j)
        for (uint32_t k = rowPtr[j]; k < rowPtr[j + 1]; ++k)
            if (colInd[k] >= col) return ERROR_MAT_DATA;
    return SUCCESS;
}

/* SortCSRRow, MATUtil.cxx:439-476: a stable insertion sort of each row by column (the
 * reference's unsigned inner index is signed here; it wraps when an entry of row 0 moves
 * to the front). */
static void sort_rows(uint32_t row, const uint32_t* rowPtr, uint32_t* colInd, double* values)
{
    for (uint32_t j = 0; j < row; ++j) {
        const int64_t begin = rowPtr[j], end = rowPtr[j + 1];
        for (int64_t k = begin + 1; k < end; ++k) {
            const uint32_t index = colInd[k];
            const double data = values[k];
            int64_t l = k - 1;
            for (; l >= begin && index < colInd[l]; --l) {
                colInd[l + 1] = colInd[l];
                values[l + 1] = values[l];
            }
            colInd[l + 1] = index;
            values[l + 1] = data;
        }
    }
}

/* CSRtoMAT, MATUtil.cxx:303-413: rows without a diagonal entry get 0.0 after their
 * entries of smaller column; then CheckCSR. Output arrays hold nnz + row entries.
 * Returns the code; *nnzOut = 0 when the check fails (the MAT is not set). */
static int csr_to_mat(uint32_t row, uint32_t col, uint32_t nnz, const double* values,
                      const uint32_t* colInd, const uint32_t* rowPtr, uint32_t* nnzOut,
                      uint32_t* rpOut, uint32_t* ciOut, double* vaOut)
{
    uint32_t count = 0, added = 0;
    rpOut[0] = 0;
    for (uint32_t i = 0; i < row; ++i) {
        const uint32_t begin = rowPtr[i], end = rowPtr[i + 1];
        int found = 0;
        for (uint32_t k = begin; k < end; ++k)
            if (colInd[k] == i) {
                found = 1;
                break;
            }
        uint32_t k = begin;
        if (!found) {
            for (; k < end && colInd[k] < i; ++k) {
                vaOut[count] = values[k];
                ciOut[count++] = colInd[k];
            }
            vaOut[count] = 0.0;
            ciOut[count++] = i;
            ++added;
        }
        for (; k < end; ++k) {
            vaOut[count] = values[k];
            ciOut[count++] = colInd[k];
        }
        rpOut[i + 1] = rowPtr[i + 1] + added;
    }
    *nnzOut = 0;
    const int code = check_csr(row, col, nnz + added, ciOut, rpOut);
    if (code == SUCCESS) *nnzOut = nnz + added;
    return code;
}

int orc_mtx_to_mat(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowInd,
                   const uint32_t* colInd, const double* values, uint32_t* nnzOut,
                   uint32_t* rowPtr, uint32_t* colIndOut, double* valuesOut)
{
    *nnzOut = 0;
    for (uint32_t j = 0; j < nnz; ++j)
        if (rowInd[j] >= nrow) return ERROR_MAT_DATA; /* the reference writes out of bounds */
    /* MTXtoCSR, MATUtil.cxx:252-300: count, prefix, scatter in input order, shift back */
    uint32_t* rp = (uint32_t*)calloc((size_t)nrow + 1, 4);
    uint32_t* ci = (uint32_t*)malloc((size_t)nnz * 4 + 4);
    double* va = (double*)malloc((size_t)nnz * 8 + 8);
    for (uint32_t j = 0; j < nnz; ++j) ++rp[rowInd[j] + 1];
    for (uint32_t i = 1; i < nrow; ++i) rp[i] += rp[i - 1];
    for (uint32_t j = 0; j < nnz; ++j) {
        const uint32_t p = rp[rowInd[j]]++;
        ci[p] = colInd[j];
        va[p] = values[j];
    }
    for (uint32_t i = nrow; i > 0; --i) rp[i] = rp[i - 1];
    rp[0] = 0;
    sort_rows(nrow, rp, ci, va);
    /* MTXtoMAT (MATUtil.cxx:416-436) ignores the codes of its three steps */
    csr_to_mat(nrow, mcol, nnz, va, ci, rp, nnzOut, rowPtr, colIndOut, valuesOut);
    free(rp);
    free(ci);
    free(va);
    return SUCCESS;
}

int orc_csr_to_mat(uint32_t nrow, uint32_t nnz, const uint32_t* rowPtr, const uint32_t* colInd,
                   const double* values, uint32_t* nnzOut, uint32_t* rowPtrOut,
                   uint32_t* colIndOut, double* valuesOut)
{
    *nnzOut = 0;
    uint32_t* rp = (uint32_t*)malloc(((size_t)nrow + 1) * 4);
    uint32_t* ci = (uint32_t*)malloc((size_t)nnz * 4 + 4);
    double* va = (double*)malloc((size_t)nnz * 8 + 8);
    memcpy(rp, rowPtr, ((size_t)nrow + 1) * 4);
    memcpy(ci, colInd, (size_t)nnz * 4);
    memcpy(va, values, (size_t)nnz * 8);
    if (rp[0] == 1) { /* ReadCSR, ReadData.cxx:350-353 */
        for (uint32_t i = 0; i <= nrow; ++i) rp[i]--;
        for (uint32_t k = 0; k < nnz; ++k) ci[k]--;
    }
    /* ReadMat's .csr branch (ReadData.cxx:376-400): SortCSRRow, then CSRtoMAT; the sort's
     * check runs first here so that a bad rowPtr is never followed */
    int code = (rp[0] == 0) ? check_csr(nrow, nrow, nnz, ci, rp) : ERROR_MAT_DATA;
    if (code == SUCCESS) {
        sort_rows(nrow, rp, ci, va);
        code = csr_to_mat(nrow, nrow, nnz, va, ci, rp, nnzOut, rowPtrOut, colIndOut, valuesOut);
    }
    free(rp);
    free(ci);
    free(va);
    return code;
}

/* ------------------------------------------------------------------------------------
 * Solver objects (src/SOL.hxx, CG.cxx, BiCGStab.cxx, GMRES.cxx, FGMRES.cxx, Iter.cxx,
 * MG.cxx)
 * ---------------------------------------------------------------------------------- */

typedef struct osol osol_t;
struct osol {
    int          alg;
    orc_params_t prm;
    const omat_t* A;
    osol_t*      pcd;
    double       norm2, normInf;
    uint32_t     numIter;
    uint32_t     len;
    double*      hist;
    uint32_t     histCap;
    /* Jacobi */
    double  weight;
    double* diagInv;
    double* work;
    /* CG / BiCGStab work vectors */
    double *rk, *pk, *zk, *ax, *safe;
    double *r0star, *tmp, *apj, *asj, *sj, *ptmp, *stmp, *ms, *mp;
    /* GMRES / FGMRES */
    uint32_t maxRestart, minRestart, restart;
    double **V, **Z;
    double *hh, *hsin, *hcos, *var, *wk;
    /* MG */
    uint32_t numLevels;
    uint32_t* numCycles;
    osol_t**  smoothers;
    osol_t**  coarse;
    double**  lb;
    double**  lx;
    double*   mgr;
    int       level;
    /* MG with transfer operators (orc_mg_set_level): lA[l] = A_{l+1}, lP[l], lR[l], and the
     * residual vector lr[l] of level l >= 1 */
    omat_t**  lA;
    omat_t**  lP;
    omat_t**  lR;
    double**  lr;
};

typedef struct {
    omat_t  mat;
    osol_t* sol;
    osol_t* pcd;
} ohandle_t;

static double* dalloc(uint32_t n)
{
    return (double*)calloc(n ? n : 1, sizeof(double));
}

static void rec(osol_t* s, uint32_t k, double v)
{
    if (s->hist && k < s->histCap) s->hist[k] = v;
}

static int sol_solve(osol_t* s, const double* b, double* x);

/* Identity::Solve, Iter.cxx:16-20 */
static int identity_solve(osol_t* s, const double* b, double* x)
{
    v_copy(s->len, b, x);
    return SUCCESS;
}

/* Jacobi::Setup, Iter.cxx:29-53: diagInv = weight * (1 / diag) */
static void jacobi_setup(osol_t* s, const omat_t* A)
{
    s->A       = A;
    s->len     = A->mcol;
    s->work    = dalloc(A->mcol > A->nrow ? A->mcol : A->nrow);
    s->diagInv = dalloc(A->nrow);
    for (uint32_t j = 0; j < A->nrow; ++j)
        s->diagInv[j] = A->values ? A->values[A->diagPtr[j]] : 1.0; /* MAT::GetDiag */
    for (uint32_t j = 0; j < A->nrow; ++j) s->diagInv[j] = 1.0 / s->diagInv[j];
    v_scale(A->nrow, s->weight, s->diagInv);
}

/* Jacobi::Solve, Iter.cxx:56-112 */
static int jacobi_solve(osol_t* s, const double* b, double* x)
{
    const omat_t* A = s->A;
    const orc_params_t* P = &s->prm;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, resAbsOld = 1.0;
    (void)resRel;
    s->numIter = 0;
    while (s->numIter < P->maxIter) {
        orc_residual(A->nrow, A->mcol, A->rowPtr, A->colInd, A->values, b, x, s->work);
        if (s->numIter >= P->minIter) {
            resAbs = orc_norm2(A->nrow, s->work);
            if (s->numIter == P->minIter) denAbs = (CLOSE_ZERO > resAbs) ? CLOSE_ZERO : resAbs;
            resRel = resAbs / denAbs;
            rec(s, s->numIter, resAbs);
            if (resRel < P->relTol || resAbs < P->absTol) break;
            resAbsOld = resAbs;
        }
        for (uint32_t i = 0; i < A->nrow; ++i) s->work[i] *= s->diagInv[i]; /* PointwiseMult */
        for (uint32_t i = 0; i < A->nrow; ++i) x[i] += s->work[i];          /* operator+= */
        ++s->numIter;
    }
    (void)resAbsOld;
    if (!(s->numIter == P->minIter && s->numIter == P->maxIter)) {
        orc_residual(A->nrow, A->mcol, A->rowPtr, A->colInd, A->values, b, x, s->work);
        s->norm2 = resAbs = orc_norm2(A->nrow, s->work);
        s->normInf = orc_norminf(A->nrow, s->work);
        rec(s, s->numIter, resAbs);
    }
    return SUCCESS;
}

/* CG::Solve, CG.cxx:53-249 */
static int cg_solve(osol_t* s, const double* b, double* x)
{
    const omat_t* A = s->A;
    const orc_params_t* P = &s->prm;
    const uint32_t n = s->len;
    int err = SUCCESS;
    const uint32_t maxStag = MAX_STAG_NUM;
    const double solStagTol = 1e-4 * P->relTol;
    const double solZeroTol = CLOSE_ZERO;
    uint32_t stagStep = 0, moreStep = 0;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, ratio = 0.0, resAbsOld = 1.0;
    double alpha = 0.0, beta, tmpa, tmpb;

    s->numIter = 0;
    orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->rk);
    v_xpay(n, -1.0, b, s->rk);
    v_set(n, 0.0, s->zk);
    sol_solve(s->pcd, s->rk, s->zk);
    v_copy(n, s->zk, s->pk);
    tmpa = orc_dot(n, s->zk, s->rk);

    while (s->numIter < P->maxIter) {
        if (s->numIter == P->minIter) {
            resAbs    = orc_norm2(n, s->rk);
            resAbsOld = resAbs;
            denAbs    = (CLOSE_ZERO > resAbs) ? CLOSE_ZERO : resAbs;
            resRel    = resAbs / denAbs;
            rec(s, s->numIter, resAbs);
            if (resRel < P->relTol || resAbs < P->absTol) break;
        }
        ++s->numIter;
        orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, s->pk, s->ax);
        tmpb = orc_dot(n, s->ax, s->pk);
        if (fabs(tmpb) > CLOSE_ZERO * CLOSE_ZERO)
            alpha = tmpa / tmpb;
        else {
            v_axpy(n, alpha, s->pk, x);
            v_axpy(n, -alpha, s->ax, s->rk);
            resAbs = orc_norm2(n, s->rk);
            resRel = resAbs / denAbs;
            if (resRel > P->relTol && resAbs > P->absTol) err = ERROR_DIVIDE_ZERO;
            rec(s, s->numIter, resAbs);
            break;
        }
        v_axpy(n, alpha, s->pk, x);
        v_axpy(n, -alpha, s->ax, s->rk);

        if (s->numIter >= P->minIter) {
            int stop = 0;
            resAbs = orc_norm2(n, s->rk);
            resRel = resAbs / denAbs;
            ratio  = resAbs / resAbsOld;
            if (s->numIter >= P->savIter && resAbs < resAbsOld) v_copy(n, x, s->safe);
            if (ratio > KSM_CHK_RATIO) {
                const double xNormInf = orc_norminf(n, x);
                if (xNormInf < solZeroTol) {
                    err = ERROR_SOLVER_SOLSTAG;
                    stop = 1;
                } else {
                    const double xRelDiff =
                        fabs(alpha) * orc_norm2(n, s->pk) / orc_norm2(n, x);
                    if ((stagStep <= maxStag) && (xRelDiff < solStagTol)) {
                        orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->rk);
                        v_xpay(n, -1.0, b, s->rk);
                        resAbs = orc_norm2(n, s->rk);
                        resRel = resAbs / denAbs;
                        if (resRel < P->relTol || resAbs < P->absTol)
                            stop = 1;
                        else if (stagStep >= maxStag) {
                            err  = ERROR_SOLVER_STAG;
                            stop = 1;
                        } else {
                            v_set(n, 0.0, s->pk);
                            ++stagStep;
                        }
                    }
                }
            }
            if (!stop && resRel < P->relTol) {
                orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->rk);
                v_xpay(n, -1.0, b, s->rk);
                resAbs = orc_norm2(n, s->rk);
                resRel = resAbs / denAbs;
                if (resRel < P->relTol || resAbs < P->absTol)
                    stop = 1;
                else if (moreStep >= P->restart) {
                    err  = ERROR_SOLVER_TOLSMALL;
                    stop = 1;
                } else {
                    v_set(n, 0.0, s->pk); /* CG.cxx:213, see the file header */
                    ++moreStep;
                }
            }
            rec(s, s->numIter, resAbs);
            if (stop) break;
        }

        if (s->numIter < P->maxIter) {
            resAbsOld = resAbs;
            v_set(n, 0.0, s->zk);
            sol_solve(s->pcd, s->rk, s->zk);
            tmpb = orc_dot(n, s->zk, s->rk);
            beta = tmpb / tmpa;
            tmpa = tmpb;
            v_xpay(n, beta, s->zk, s->pk);
        }
    }
    if (!(s->numIter == P->minIter && s->numIter == P->maxIter)) {
        s->norm2   = resAbs;
        s->normInf = orc_norminf(n, s->rk);
    }
    if (s->numIter > P->savIter) v_copy(n, s->safe, x);
    return err;
}

/* BiCGStab::Solve, BiCGStab.cxx:68-270 */
static int bicgstab_solve(osol_t* s, const double* b, double* x)
{
    const omat_t* A = s->A;
    const orc_params_t* P = &s->prm;
    const uint32_t n = s->len;
    int err = SUCCESS;
    const uint32_t maxStag = MAX_STAG_NUM;
    const double solStagTol = 1e-4 * P->relTol;
    uint32_t stagStep = 0, moreStep = 0;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, ratio = 0.0, resAbsOld = 1.0;
    double alpha = 0.0, beta, rjr0star = 0.0, rjr0startmp, omega = 0.0, tmp12;

    s->numIter = 0;
    orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->tmp);
    v_waxpby(n, 1.0, b, -1.0, s->tmp, s->rk);
    v_copy(n, s->rk, s->r0star);
    v_copy(n, s->rk, s->pk);

    while (s->numIter < P->maxIter) {
        if (s->numIter == P->minIter) {
            resAbs = orc_norm2(n, s->rk);
            denAbs = (CLOSE_ZERO > resAbs) ? CLOSE_ZERO : resAbs;
            resRel = resAbs / denAbs;
            rec(s, s->numIter, resAbs);
            if (resRel < P->relTol || resAbs < P->absTol) break;
        }
        ++s->numIter;
        rjr0star = orc_dot(n, s->rk, s->r0star);
        orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, s->pk, s->apj);
        v_set(n, 0.0, s->ptmp);
        sol_solve(s->pcd, s->apj, s->ptmp);
        tmp12 = orc_dot(n, s->ptmp, s->r0star);
        if (fabs(tmp12) > 1e-40)
            alpha = rjr0star / tmp12;
        else {
            err = ERROR_DIVIDE_ZERO;
            rec(s, s->numIter, resAbs);
            break;
        }
        v_waxpby(n, 1.0, s->rk, -alpha, s->ptmp, s->sj);
        orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, s->sj, s->asj);
        v_set(n, 0.0, s->stmp);
        sol_solve(s->pcd, s->asj, s->stmp);
        omega = orc_dot(n, s->stmp, s->sj) / orc_dot(n, s->stmp, s->stmp);
        v_set(n, 0.0, s->mp);
        sol_solve(s->pcd, s->pk, s->mp);
        v_set(n, 0.0, s->ms);
        sol_solve(s->pcd, s->sj, s->ms);
        v_waxpby(n, alpha, s->mp, omega, s->ms, s->tmp);
        v_xpay(n, 1.0, s->tmp, x);
        v_waxpby(n, 1.0, s->sj, -omega, s->stmp, s->rk);

        if (s->numIter >= P->minIter) {
            int stop = 0;
            resAbs = orc_norm2(n, s->rk);
            resRel = resAbs / denAbs;
            ratio  = resAbs / resAbsOld;
            if (s->numIter >= P->savIter && resAbs < resAbsOld) v_copy(n, x, s->safe);
            if (ratio > KSM_CHK_RATIO && s->numIter > P->minIter) {
                const double xNorminf = orc_norminf(n, x);
                if (xNorminf < solStagTol) {
                    err  = ERROR_SOLVER_SOLSTAG;
                    stop = 1;
                } else {
                    const double xRelDiff =
                        fabs(alpha) * orc_norm2(n, s->pk) / orc_norm2(n, x);
                    if ((stagStep <= maxStag) && (xRelDiff < solStagTol)) {
                        orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->rk);
                        v_xpay(n, -1.0, b, s->rk);
                        resAbs = orc_norm2(n, s->rk);
                        resRel = resAbs / denAbs;
                        if (resRel < P->relTol || resAbs < P->absTol)
                            stop = 1;
                        else if (stagStep >= maxStag) {
                            err  = ERROR_SOLVER_STAG;
                            stop = 1;
                        } else {
                            v_set(n, 0.0, s->pk);
                            ++stagStep;
                        }
                    }
                }
            }
            if (!stop && resRel < P->relTol) {
                orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->rk);
                v_xpay(n, -1.0, b, s->rk);
                resAbs = orc_norm2(n, s->rk);
                resRel = resAbs / denAbs;
                if (resRel < P->relTol || resAbs < P->absTol)
                    stop = 1;
                else if (moreStep >= P->restart) {
                    err  = ERROR_SOLVER_TOLSMALL;
                    stop = 1;
                } else {
                    v_set(n, 0.0, s->pk);
                    ++moreStep;
                }
            }
            rec(s, s->numIter, resAbs);
            if (stop) break;
        }

        if (s->numIter < P->maxIter) {
            resAbsOld   = resAbs;
            rjr0startmp = rjr0star;
            rjr0star    = orc_dot(n, s->rk, s->r0star);
            beta        = rjr0star / rjr0startmp * alpha / omega;
            v_waxpby(n, 1.0, s->pk, -omega, s->ptmp, s->tmp);
            v_waxpby(n, 1.0, s->rk, beta, s->tmp, s->pk);
        }
    }
    if (!(s->numIter == P->minIter && s->numIter == P->maxIter)) {
        s->norm2   = resAbs;
        s->normInf = orc_norminf(n, s->rk);
    }
    if (s->numIter > P->savIter) v_copy(n, s->safe, x);
    return err;
}

#define HH(s, i, j) ((s)->hh[(size_t)(i) * (s)->maxRestart + (j)])

/* Givens/Hessenberg step shared by GMRES::RSolve (GMRES.cxx:173-203), GMRES::LSolve
 * (:345-375) and FGMRES::Solve (:168-198). Returns 0 when t is not > SMALL_DBL (the
 * reference leaves the restart cycle), 1 otherwise. w is the new basis vector. */
static int arnoldi_givens(osol_t* s, uint32_t count, uint32_t count_1, double* w)
{
    const uint32_t n = s->len;
    double t, gamma;
    for (uint32_t j = 0; j < count; ++j) {
        HH(s, j, count_1) = orc_dot(n, w, s->V[j]);
        v_axpby(n, 1.0, -HH(s, j, count_1), s->V[j], w);
    }
    t = orc_norm2(n, w);
    HH(s, count, count_1) = t;
    if (fabs(t) > SMALL_DBL)
        v_scale(n, 1.0 / t, w);
    else
        return 0;
    for (uint32_t j = 1; j < count; ++j) {
        t                   = HH(s, j - 1, count_1);
        HH(s, j - 1, count_1) = s->hsin[j - 1] * HH(s, j, count_1) + s->hcos[j - 1] * t;
        HH(s, j, count_1)   = -s->hsin[j - 1] * t + s->hcos[j - 1] * HH(s, j, count_1);
    }
    t = HH(s, count, count_1) * HH(s, count, count_1);
    t += HH(s, count_1, count_1) * HH(s, count_1, count_1);
    t = sqrt(t);
    gamma            = t > SMALL_DBL ? t : SMALL_DBL;
    s->hcos[count_1] = HH(s, count_1, count_1) / gamma;
    s->hsin[count_1] = HH(s, count, count_1) / gamma;
    HH(s, count_1, count_1) =
        s->hsin[count_1] * HH(s, count, count_1) + s->hcos[count_1] * HH(s, count_1, count_1);
    s->var[count]   = -s->hsin[count_1] * s->var[count_1];
    s->var[count_1] = s->hcos[count_1] * s->var[count_1];
    return 1;
}

/* Back substitution (GMRES.cxx:213-219, signed loop) then
 * wk = var[count_1]*B[count_1] + sum_{j=count-2..0} var[j]*B[j] (:221-224). */
static void gmres_combine(osol_t* s, uint32_t count, uint32_t count_1, double** B)
{
    const uint32_t n = s->len;
    double t;
    s->var[count_1] = s->var[count_1] / HH(s, count_1, count_1);
    for (int k = (int)count - 2; k >= 0; --k) {
        t = 0.0;
        for (uint32_t j = (uint32_t)k + 1; j < count; ++j) t -= HH(s, k, j) * s->var[j];
        t += s->var[k];
        s->var[k] = t / HH(s, k, k);
    }
    v_copy(n, B[count_1], s->wk);
    v_scale(n, s->var[count_1], s->wk);
    for (int j = (int)count - 2; j >= 0; --j) v_axpby(n, 1.0, s->var[j], B[j], s->wk);
}

/* Variable restart, GMRES.cxx:255-265 (strict) and FGMRES.cxx:246-256 (inclusive). */
static void adapt_restart(osol_t* s, double cr, int inclusive)
{
    const int mid = inclusive ? (cr <= MAX_CR && cr >= MIN_CR) : (cr < MAX_CR && cr > MIN_CR);
    if (cr > MAX_CR)
        s->restart = s->maxRestart;
    else if (mid) {
        if (s->restart - RESTART_DECREASE > s->minRestart) /* unsigned, as USI */
            s->restart -= RESTART_DECREASE;
        else
            s->restart = s->maxRestart;
    }
    if (s->restart > s->maxRestart) s->restart = s->maxRestart; /* see file header */
}

/* GMRES::RSolve (GMRES.cxx:114-280) and FGMRES::Solve (FGMRES.cxx:108-271): flexible
 * keeps the preconditioned vectors in Z and does not zero Z[j] before pcd->Solve. */
static int gmres_right_solve(osol_t* s, const double* b, double* x, int flexible)
{
    const omat_t* A = s->A;
    const orc_params_t* P = &s->prm;
    const uint32_t n = s->len;
    int err = SUCCESS;
    double t, ri, rj, cr = 1.0;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, resAbsOld = 1.0;
    uint32_t count = 1, count_1 = 2;

    s->numIter = 0;
    v_copy(n, x, s->safe);
    orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->V[0]);
    v_xpay(n, -1.0, b, s->V[0]);
    resAbs = ri = orc_norm2(n, s->V[0]);
    denAbs = flexible ? ((resAbs > CLOSE_ZERO) ? resAbs : CLOSE_ZERO)
                      : ((CLOSE_ZERO > resAbs) ? CLOSE_ZERO : resAbs);

    while (s->numIter < P->maxIter) {
        if (s->numIter == P->minIter) {
            resRel    = resAbs / denAbs;
            resAbsOld = resAbs;
            rec(s, s->numIter, resAbs);
            if (resRel < P->relTol || resAbs < P->absTol) break;
        }
        if (resAbs < SMALL_DBL) break;
        s->var[0] = resAbs;
        v_scale(n, 1 / resAbs, s->V[0]);

        count = 0;
        while (count < s->restart && s->numIter < P->maxIter) {
            ++s->numIter;
            count_1 = count++;
            if (flexible) {
                v_set(n, 0.0, s->tmp);
                sol_solve(s->pcd, s->V[count_1], s->Z[count_1]);
                orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, s->Z[count_1], s->V[count]);
            } else {
                v_set(n, 0.0, s->tmp);
                sol_solve(s->pcd, s->V[count_1], s->tmp);
                orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, s->tmp, s->V[count]);
            }
            if (!arnoldi_givens(s, count, count_1, s->V[count])) break;
            resAbs    = fabs(s->var[count]);
            resRel    = resAbs / denAbs;
            resAbsOld = resAbs;
            rec(s, s->numIter, resAbs);
            if ((resAbs < P->absTol || resRel < P->relTol) && s->numIter > P->minIter) break;
        }

        if (flexible) {
            gmres_combine(s, count, count_1, s->Z);
            v_axpy(n, 1.0, s->wk, x);
        } else {
            gmres_combine(s, count, count_1, s->V);
            v_set(n, 0.0, s->tmp);
            sol_solve(s->pcd, s->wk, s->tmp);
            v_axpy(n, 1.0, s->tmp, x);
        }
        if (s->numIter >= P->savIter && resAbs < resAbsOld) v_copy(n, x, s->safe);
        if (s->numIter > P->maxIter) {
            err = ERROR_SOLVER_MAXIT;
            break;
        }
        orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->V[0]);
        v_xpay(n, -1.0, b, s->V[0]);
        resAbs = rj = orc_norm2(n, s->V[0]);
        resRel = resAbs / denAbs;
        rec(s, s->numIter, resAbs);
        if ((resRel < P->relTol || resAbs < P->absTol) && s->numIter >= P->minIter) break;
        cr = rj / ri;
        ri = rj;
        adapt_restart(s, cr, flexible);
    }
    (void)t;
    if (!(s->numIter == P->minIter && s->numIter == P->maxIter)) {
        s->norm2   = orc_norm2(n, s->V[0]);
        s->normInf = orc_norminf(n, s->V[0]);
    }
    if (s->numIter > P->savIter) v_copy(n, s->safe, x);
    return err;
}

/* GMRES::LSolve, GMRES.cxx:283-453 */
static int gmres_left_solve(osol_t* s, const double* b, double* x)
{
    const omat_t* A = s->A;
    const orc_params_t* P = &s->prm;
    const uint32_t n = s->len;
    int err = SUCCESS;
    double ri, rj, cr = 1.0;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, resAbsOld = 1.0;
    uint32_t count = 1, count_1 = 2;

    s->numIter = 0;
    v_copy(n, x, s->safe);
    orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->tmp);
    v_xpay(n, -1.0, b, s->tmp);
    ri = orc_norm2(n, s->tmp);
    v_set(n, 0.0, s->V[0]);
    sol_solve(s->pcd, s->tmp, s->V[0]);
    resAbs = orc_norm2(n, s->V[0]);
    denAbs = (CLOSE_ZERO > resAbs) ? CLOSE_ZERO : resAbs;

    while (s->numIter < P->maxIter) {
        if (s->numIter == P->minIter) {
            resRel    = resAbs / denAbs;
            resAbsOld = resAbs;
            rec(s, s->numIter, resAbs);
            if (resRel < P->relTol || resAbs < P->absTol) break;
        }
        if (resAbs < SMALL_DBL) break;
        s->var[0] = resAbs;
        v_scale(n, 1 / resAbs, s->V[0]);

        count = 0;
        while (count < s->restart && s->numIter < P->maxIter) {
            ++s->numIter;
            count_1 = count++;
            orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, s->V[count_1], s->tmp);
            v_set(n, 0.0, s->V[count]);
            sol_solve(s->pcd, s->tmp, s->V[count]);
            if (!arnoldi_givens(s, count, count_1, s->V[count])) break;
            resAbs    = fabs(s->var[count]);
            resAbsOld = resAbs;
            resRel    = resAbs / denAbs;
            rec(s, s->numIter, resAbs);
            if ((resAbs < P->absTol || resRel < P->relTol) && s->numIter > P->minIter) break;
        }

        gmres_combine(s, count, count_1, s->V);
        v_axpy(n, 1.0, s->wk, x);
        if (s->numIter >= P->savIter && resAbs < resAbsOld) v_copy(n, x, s->safe);
        if (s->numIter > P->maxIter) {
            err = ERROR_SOLVER_MAXIT;
            break;
        }
        orc_spmv(A->nrow, A->rowPtr, A->colInd, A->values, x, s->tmp);
        v_xpay(n, -1.0, b, s->tmp);
        rj = orc_norm2(n, s->tmp);
        v_set(n, 0.0, s->V[0]);
        sol_solve(s->pcd, s->tmp, s->V[0]);
        resAbs = orc_norm2(n, s->V[0]);
        resRel = resAbs / denAbs;
        rec(s, s->numIter, resAbs);
        if ((resRel < P->relTol || resAbs < P->absTol) && s->numIter >= P->minIter) break;
        cr = rj / ri;
        ri = rj;
        adapt_restart(s, cr, 0);
    }
    if (!(s->numIter == P->minIter && s->numIter == P->maxIter)) {
        s->norm2   = orc_norm2(n, s->tmp);
        s->normInf = orc_norminf(n, s->tmp);
    }
    if (s->numIter > P->savIter) v_copy(n, s->safe, x);
    return err;
}

/* MG::MGCycle, MG.cxx:105-152, with IdentityMatrix transfers (MAT.cxx:1095) as the
 * reference's MG driver sets them up (example/TestMG.cxx:85-94). The residual always
 * uses the top-level operator (MG.cxx:119). */
static void mg_cycle(osol_t* s, const double* b, double* x)
{
    const omat_t* A = s->A;
    const uint32_t n = s->len;
    if (s->lP) {
        /* with transfer operators: the same cycle, level l's residual with A_l, restriction
         * R_l, prolongation P_l (the B200 library's fasp_gpu_solver_set_mg_transfer) */
        ++s->level;
        if ((uint32_t)s->level == s->numLevels) return;
        const uint32_t l = (uint32_t)s->level;
        const omat_t* Al = l == 0 ? A : s->lA[l - 1];
        double* r = l == 0 ? s->mgr : s->lr[l];
        const omat_t *R = s->lR[l], *P = s->lP[l];
        sol_solve(s->smoothers[l], b, x);
        orc_residual(Al->nrow, Al->mcol, Al->rowPtr, Al->colInd, Al->values, b, x, r);
        orc_spmv(R->nrow, R->rowPtr, R->colInd, R->values, r, s->lb[l]);
        v_set(s->lA[l]->nrow, 0.0, s->lx[l]);
        if (l + 1 == s->numLevels)
            sol_solve(s->coarse[l], s->lb[l], s->lx[l]);
        else
            for (uint32_t i = 0; i < s->numCycles[l]; ++i) mg_cycle(s, s->lb[l], s->lx[l]);
        orc_spmv(P->nrow, P->rowPtr, P->colInd, P->values, s->lx[l], r);
        v_axpy(Al->nrow, 1.0, r, x);
        sol_solve(s->smoothers[l], b, x);
        --s->level;
        return;
    }
    if (s->numLevels > 0) {
        ++s->level;
        if ((uint32_t)s->level - s->numLevels == 0) return;
        const uint32_t L = (uint32_t)s->level;
        sol_solve(s->smoothers[L], b, x);
        orc_residual(A->nrow, A->mcol, A->rowPtr, A->colInd, A->values, b, x, s->mgr);
        v_copy(n, s->mgr, s->lb[L]);
        v_set(n, 0.0, s->lx[L]);
        if (L + 1 - s->numLevels == 0)
            sol_solve(s->coarse[L], s->lb[L], s->lx[L]);
        else
            for (uint32_t i = 0; i < s->numCycles[L]; ++i) mg_cycle(s, s->lb[L], s->lx[L]);
        v_copy(n, s->lx[L], s->mgr);
        v_axpy(n, 1.0, s->mgr, x);
        sol_solve(s->smoothers[L], b, x);
        --s->level;
    } else {
        v_copy(n, b, x);
    }
}

/* MG::Solve, MG.cxx:155-210 */
static int mg_solve(osol_t* s, const double* b, double* x)
{
    const omat_t* A = s->A;
    const orc_params_t* P = &s->prm;
    const uint32_t n = s->len;
    double resAbs = 1.0, resRel = 1.0, denAbs = 1.0, resAbsOld = 1.0;
    (void)resRel;
    s->numIter = 0;
    while (s->numIter < P->maxIter) {
        orc_residual(A->nrow, A->mcol, A->rowPtr, A->colInd, A->values, b, x, s->mgr);
        if (s->numIter >= P->minIter) {
            resAbs = orc_norm2(n, s->mgr);
            if (s->numIter == P->minIter) denAbs = (CLOSE_ZERO > resAbs) ? CLOSE_ZERO : resAbs;
            resRel = resAbs / denAbs;
            rec(s, s->numIter, resAbs);
            if (resRel < P->relTol || resAbs < P->absTol) break;
            resAbsOld = resAbs;
        }
        mg_cycle(s, b, x);
        ++s->numIter;
    }
    (void)resAbsOld;
    if (!(s->numIter == P->minIter && s->numIter == P->maxIter)) {
        orc_residual(A->nrow, A->mcol, A->rowPtr, A->colInd, A->values, b, x, s->mgr);
        s->norm2 = resAbs = orc_norm2(n, s->mgr);
        s->normInf = orc_norminf(n, s->mgr);
        rec(s, s->numIter, resAbs);
    }
    return SUCCESS;
}

static int sol_solve(osol_t* s, const double* b, double* x)
{
    switch (s->alg) {
        case ORC_IDENTITY: return identity_solve(s, b, x);
        case ORC_JACOBI: return jacobi_solve(s, b, x);
        case ORC_CG: return cg_solve(s, b, x);
        case ORC_BICGSTAB: return bicgstab_solve(s, b, x);
        case ORC_GMRES: return gmres_right_solve(s, b, x, 0);
        case ORC_FGMRES: return gmres_right_solve(s, b, x, 1);
        case ORC_GMRES_LEFT: return gmres_left_solve(s, b, x);
        case ORC_MG: return mg_solve(s, b, x);
        default: return ERROR_INPUT_PAR;
    }
}

/* ------------------------------------------------------------------------------------
 * Object management: the Setup(...) of each solver.
 * ---------------------------------------------------------------------------------- */

void orc_default_params(orc_params_t* p)
{
    p->maxIter = 1;
    p->minIter = 0;
    p->savIter = MAX_ITER_NUM;
    p->restart = 30;
    p->relTol  = 1e-6;
    p->absTol  = 1e-8;
}

void orc_default_config(orc_config_t* c, int alg)
{
    memset(c, 0, sizeof(*c));
    c->alg = alg;
    orc_default_params(&c->prm);
    c->weight = 1.0;
    c->pcd = 0;
    c->pcdWeight = 1.0;
    orc_default_params(&c->pcdPrm);
    c->mgLevels = 3;
    c->mgCycles = 1;
    c->mgSmoothWeight = 1.0;
    c->mgCoarseWeight = 1.0;
    orc_default_params(&c->mgSmoothPrm);
    orc_default_params(&c->mgCoarsePrm);
}

static osol_t* new_sol(int alg, const orc_params_t* prm, const omat_t* A)
{
    osol_t* s = (osol_t*)calloc(1, sizeof(osol_t));
    s->alg = alg;
    s->prm = *prm;
    s->A = A;
    s->len = A->mcol;
    s->norm2 = 1e60;
    s->normInf = 1e60;
    s->level = -1;
    return s;
}

static osol_t* new_jacobi(const orc_params_t* prm, double weight, const omat_t* A)
{
    osol_t* s = new_sol(ORC_JACOBI, prm, A);
    s->weight = weight;
    jacobi_setup(s, A);
    return s;
}

static void omat_free(omat_t* m)
{
    if (!m) return;
    free(m->rowPtr); free(m->colInd); free(m->diagPtr); free(m->values);
    free(m);
}

static void free_sol(osol_t* s)
{
    if (!s) return;
    if (s->lP)
        for (uint32_t l = 0; l < s->numLevels; ++l) {
            omat_free(s->lA[l]);
            omat_free(s->lP[l]);
            omat_free(s->lR[l]);
            free(s->lr[l]);
        }
    free(s->lA); free(s->lP); free(s->lR); free(s->lr);
    free(s->diagInv); free(s->work);
    free(s->rk); free(s->pk); free(s->zk); free(s->ax); free(s->safe);
    free(s->r0star); free(s->tmp); free(s->apj); free(s->asj); free(s->sj);
    free(s->ptmp); free(s->stmp); free(s->ms); free(s->mp);
    if (s->V) for (uint32_t j = 0; j <= s->maxRestart; ++j) free(s->V[j]);
    if (s->Z) for (uint32_t j = 0; j <= s->maxRestart; ++j) free(s->Z[j]);
    free(s->V); free(s->Z);
    free(s->hh); free(s->hsin); free(s->hcos); free(s->var); free(s->wk);
    if (s->smoothers)
        for (uint32_t l = 0; l < s->numLevels; ++l) {
            free_sol(s->smoothers[l]);
            free_sol(s->coarse[l]);
            free(s->lb[l]);
            free(s->lx[l]);
        }
    free(s->smoothers); free(s->coarse); free(s->lb); free(s->lx);
    free(s->numCycles); free(s->mgr);
    free(s);
}

/* GMRES::Setup (GMRES.cxx:38-88) / FGMRES::Setup (FGMRES.cxx:23-80) */
static void gmres_setup(osol_t* s, uint32_t maxR, uint32_t minR, int flexible)
{
    const uint32_t n = s->len;
    s->restart = s->prm.restart;
    s->maxRestart = maxR > s->prm.maxIter ? s->prm.maxIter : maxR;
    s->minRestart = minR > s->maxRestart ? s->maxRestart : minR;
    const uint32_t m = s->maxRestart;
    s->wk = dalloc(n);
    s->tmp = dalloc(n);
    s->safe = dalloc(n);
    s->var = dalloc(n > m + 1 ? n : m + 1);
    s->hcos = dalloc(m + 1);
    s->hsin = dalloc(m ? m : 1);
    s->hh = dalloc((m + 1) * (m ? m : 1));
    s->V = (double**)calloc(m + 1, sizeof(double*));
    for (uint32_t j = 0; j <= m; ++j) s->V[j] = dalloc(n);
    if (flexible) {
        s->Z = (double**)calloc(m + 1, sizeof(double*));
        for (uint32_t j = 0; j <= m; ++j) s->Z[j] = dalloc(n);
    }
    if (s->restart > s->maxRestart)
        s->restart = s->maxRestart;
    else if (s->restart < s->minRestart)
        s->restart = s->minRestart;
}

/* MG::SetupALL (MG.cxx:54-79) + SetupLevel (:26-51) as in TestMG.cxx:80-97: identity
 * transfers, Jacobi smoothers and coarse solvers; prm = the MG object's SOLParams. */
static osol_t* new_mg(const orc_config_t* cfg, const orc_params_t* prm, const omat_t* M)
{
    const uint32_t n = M->mcol;
    osol_t* s = new_sol(ORC_MG, prm, M);
    const uint32_t L = cfg->mgLevels;
    s->numLevels = L;
    s->mgr = dalloc(n);
    if (L) {
        s->numCycles = (uint32_t*)calloc(L, sizeof(uint32_t));
        s->smoothers = (osol_t**)calloc(L, sizeof(osol_t*));
        s->coarse = (osol_t**)calloc(L, sizeof(osol_t*));
        s->lb = (double**)calloc(L, sizeof(double*));
        s->lx = (double**)calloc(L, sizeof(double*));
        for (uint32_t l = 0; l < L; ++l) {
            s->numCycles[l] = cfg->mgCycles;
            s->smoothers[l] = new_jacobi(&cfg->mgSmoothPrm, cfg->mgSmoothWeight, M);
            s->coarse[l] = new_jacobi(&cfg->mgCoarsePrm, cfg->mgCoarseWeight, M);
            s->lb[l] = dalloc(n);
            s->lx[l] = dalloc(n);
        }
    }
    return s;
}

void* orc_create(const orc_config_t* cfg, uint32_t nrow, uint32_t mcol, uint32_t nnz,
                 const uint32_t* rowPtr, const uint32_t* colInd, const double* values)
{
    if (!cfg || nrow == 0 || mcol == 0 || nnz == 0) return NULL;
    ohandle_t* h = (ohandle_t*)calloc(1, sizeof(ohandle_t));
    omat_t* M = &h->mat;
    M->nrow = nrow;
    M->mcol = mcol;
    M->nnz = nnz;
    M->rowPtr = (uint32_t*)malloc((nrow + 1) * sizeof(uint32_t));
    M->colInd = (uint32_t*)malloc(nnz * sizeof(uint32_t));
    M->diagPtr = (uint32_t*)malloc(nrow * sizeof(uint32_t));
    memcpy(M->rowPtr, rowPtr, (nrow + 1) * sizeof(uint32_t));
    memcpy(M->colInd, colInd, nnz * sizeof(uint32_t));
    if (values) {
        M->values = (double*)malloc(nnz * sizeof(double));
        memcpy(M->values, values, nnz * sizeof(double));
    }
    orc_diagptr(nrow, M->rowPtr, M->colInd, M->diagPtr);

    const uint32_t n = mcol;
    if (cfg->pcd == 1)
        h->pcd = new_jacobi(&cfg->pcdPrm, cfg->pcdWeight, M);
    else if (cfg->pcd == 2) /* an MG object as the preconditioner (SOL::SetupPCD) */
        h->pcd = new_mg(cfg, &cfg->pcdPrm, M);
    else
        h->pcd = new_sol(ORC_IDENTITY, &cfg->pcdPrm, M);

    osol_t* s = NULL;
    switch (cfg->alg) {
        case ORC_CG:
            s = new_sol(ORC_CG, &cfg->prm, M);
            s->zk = dalloc(n); s->pk = dalloc(n); s->rk = dalloc(n);
            s->ax = dalloc(n); s->safe = dalloc(n);
            break;
        case ORC_BICGSTAB:
            s = new_sol(ORC_BICGSTAB, &cfg->prm, M);
            s->r0star = dalloc(n); s->tmp = dalloc(n); s->apj = dalloc(n);
            s->asj = dalloc(n); s->pk = dalloc(n); s->rk = dalloc(n); s->sj = dalloc(n);
            s->ptmp = dalloc(n); s->stmp = dalloc(n); s->ms = dalloc(n);
            s->mp = dalloc(n); s->safe = dalloc(n);
            break;
        case ORC_GMRES:
        case ORC_GMRES_LEFT:
        case ORC_FGMRES: {
            s = new_sol(cfg->alg, &cfg->prm, M);
            const uint32_t maxR = cfg->maxRestart ? cfg->maxRestart : 30;
            const uint32_t minR = cfg->maxRestart ? cfg->minRestart : 10;
            gmres_setup(s, maxR, minR, cfg->alg == ORC_FGMRES);
            if (s->maxRestart == 0 || s->restart == 0) {
                free_sol(s);
                s = NULL;
            }
            break;
        }
        case ORC_JACOBI:
            s = new_jacobi(&cfg->prm, cfg->weight, M);
            break;
        case ORC_MG:
            s = new_mg(cfg, &cfg->prm, M);
            break;
        default:
            break;
    }
    if (!s) {
        free_sol(h->pcd);
        free(M->rowPtr); free(M->colInd); free(M->diagPtr); free(M->values);
        free(h);
        return NULL;
    }
    s->pcd = h->pcd;
    h->sol = s;
    return h;
}

int orc_solve(void* hv, const double* b, double* x, uint32_t* numIter, double* norm2,
              double* normInf, double* hist, uint32_t histCap)
{
    ohandle_t* h = (ohandle_t*)hv;
    osol_t* s = h->sol;
    for (uint32_t k = 0; k < histCap; ++k) hist[k] = NAN;
    s->hist = hist;
    s->histCap = histCap;
    const int code = sol_solve(s, b, x);
    s->hist = NULL;
    if (numIter) *numIter = s->numIter;
    if (norm2) *norm2 = s->norm2;
    if (normInf) *normInf = s->normInf;
    return code;
}

/* Clean() of the solvers (CG.cxx:43-50, GMRES.cxx:91-111, FGMRES.cxx:83-105) */
void orc_clean(void* hv)
{
    ohandle_t* h = (ohandle_t*)hv;
    osol_t* s = h->sol;
    const uint32_t n = s->len;
    if (s->alg == ORC_GMRES || s->alg == ORC_GMRES_LEFT || s->alg == ORC_FGMRES) {
        s->restart = s->prm.restart;
        if (s->restart > s->maxRestart)
            s->restart = s->maxRestart;
        else if (s->restart < s->minRestart)
            s->restart = s->minRestart;
        for (uint32_t j = 0; j <= s->maxRestart; ++j) {
            v_set(n, 0.0, s->V[j]);
            if (s->Z) v_set(n, 0.0, s->Z[j]);
        }
    }
}

void orc_destroy(void* hv)
{
    ohandle_t* h = (ohandle_t*)hv;
    if (!h) return;
    free_sol(h->sol);
    free_sol(h->pcd);
    free(h->mat.rowPtr); free(h->mat.colInd); free(h->mat.diagPtr); free(h->mat.values);
    free(h);
}

/* ------------------------------------------------------------------------------------
 * The reference's matrix-free example problem (example/TestMatFree.cxx:41-85 with
 * example/Poisson2D.hxx, TEST_PROBLEM 1): the right-hand side AssembleRHS builds on the
 * (dim-1) x (dim-1) interior grid, h = 1/dim, point (k, j) at index (k-1)(dim-1) + j-1.
 * u = sin(pi x) sin(pi y) vanishes on the boundary, so every point gets h^2 Load(k h, j h)
 * (the boundary terms the example adds are 0.0 there); Load is evaluated in the example's
 * operation order with the C library's sin.
 * ---------------------------------------------------------------------------------- */
void orc_matfree_rhs(int dim, double* b)
{
    const double pi = 3.14159265358979323846264338327950288;
    const double h = 1.0 / dim;
    const double h2 = h * h;
    const int dim1 = dim - 1;
    for (int k = 1; k <= dim1; ++k)
        for (int j = 1; j <= dim1; ++j) {
            const double x = k * h, y = j * h;
            const double load = 2 * pi * pi * sin(pi * x) * sin(pi * y);
            b[(size_t)(k - 1) * dim1 + (j - 1)] = h2 * load;
        }
}

/* ------------------------------------------------------------------------------------
 * MAT::Mult, src/MAT.cxx:715-800: C = L R. The columns of row i of C are listed in the
 * order in which the loop over L's row i (k ascending) and R's row colInd[k] (l ascending)
 * first meets them; C(i,c) = 0 + each matching L(i,k) R(k,l) in that loop order. (The
 * reference finds a column by a linear search of the row's list; a column-to-slot table
 * gives the same list and the same additions in the same order.)
 * ---------------------------------------------------------------------------------- */
int orc_mat_mult(uint32_t nl, uint32_t ml, const uint32_t* rpl, const uint32_t* cil,
                 const double* val, uint32_t mr, const uint32_t* rpr, const uint32_t* cir,
                 const double* var, uint32_t cap, uint32_t* nnzC, uint32_t* rpC,
                 uint32_t* ciC, double* vaC)
{
    (void)ml;
    uint32_t* slot = (uint32_t*)malloc((size_t)(mr ? mr : 1) * sizeof(uint32_t));
    for (uint32_t c = 0; c < mr; ++c) slot[c] = 0xffffffffu;
    uint32_t count = 0;
    int fits = 1;
    rpC[0] = 0;
    for (uint32_t i = 0; i < nl; ++i) {
        const uint32_t start = count;
        for (uint32_t k = rpl[i]; k < rpl[i + 1]; ++k)
            for (uint32_t l = rpr[cil[k]]; l < rpr[cil[k] + 1]; ++l) {
                const uint32_t c = cir[l];
                if (slot[c] == 0xffffffffu) {
                    slot[c] = count;
                    if (count < cap) {
                        ciC[count] = c;
                        vaC[count] = 0.0;
                    } else {
                        fits = 0;
                    }
                    ++count;
                }
                if (fits) vaC[slot[c]] += val[k] * var[l];
            }
        for (uint32_t q = start; q < count && q < cap; ++q) slot[ciC[q]] = 0xffffffffu;
        if (!fits) /* keep counting: reset the table from R's rows again */
            for (uint32_t k = rpl[i]; k < rpl[i + 1]; ++k)
                for (uint32_t l = rpr[cil[k]]; l < rpr[cil[k] + 1]; ++l) slot[cir[l]] = 0xffffffffu;
        rpC[i + 1] = count;
    }
    free(slot);
    *nnzC = count;
    return fits ? 0 : -1;
}

static omat_t* omat_copy(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rp,
                         const uint32_t* ci, const double* va)
{
    omat_t* m = (omat_t*)calloc(1, sizeof(omat_t));
    m->nrow = nrow;
    m->mcol = mcol;
    m->nnz = nnz;
    m->rowPtr = (uint32_t*)malloc(((size_t)nrow + 1) * sizeof(uint32_t));
    m->colInd = (uint32_t*)malloc(((size_t)nnz + 1) * sizeof(uint32_t));
    m->diagPtr = (uint32_t*)malloc(((size_t)nrow + 1) * sizeof(uint32_t));
    m->values = (double*)malloc(((size_t)nnz + 1) * sizeof(double));
    memcpy(m->rowPtr, rp, ((size_t)nrow + 1) * sizeof(uint32_t));
    memcpy(m->colInd, ci, (size_t)nnz * sizeof(uint32_t));
    memcpy(m->values, va, (size_t)nnz * sizeof(double));
    orc_diagptr(nrow, m->rowPtr, m->colInd, m->diagPtr);
    return m;
}

int orc_mg_set_level(void* hv, uint32_t level,
                     uint32_t pn, uint32_t pm, uint32_t pnnz, const uint32_t* prp,
                     const uint32_t* pci, const double* pva,
                     uint32_t rn, uint32_t rm, uint32_t rnnz, const uint32_t* rrp,
                     const uint32_t* rci, const double* rva,
                     uint32_t an, uint32_t annz, const uint32_t* arp, const uint32_t* aci,
                     const double* ava)
{
    ohandle_t* h = (ohandle_t*)hv;
    osol_t* s = h ? h->sol : NULL;
    if (s && s->alg != ORC_MG) s = h->pcd; /* the MG preconditioner of a Krylov solver */
    if (!s || s->alg != ORC_MG || level >= s->numLevels) return ERROR_INPUT_PAR;
    const uint32_t L = s->numLevels;
    if (!s->lP) {
        s->lA = (omat_t**)calloc(L, sizeof(omat_t*));
        s->lP = (omat_t**)calloc(L, sizeof(omat_t*));
        s->lR = (omat_t**)calloc(L, sizeof(omat_t*));
        s->lr = (double**)calloc(L, sizeof(double*));
    }
    omat_free(s->lA[level]);
    omat_free(s->lP[level]);
    omat_free(s->lR[level]);
    s->lP[level] = omat_copy(pn, pm, pnnz, prp, pci, pva);
    s->lR[level] = omat_copy(rn, rm, rnnz, rrp, rci, rva);
    s->lA[level] = omat_copy(an, an, annz, arp, aci, ava);
    /* the coarse solver of this level and the smoother of the next one run on A_{level+1} */
    osol_t* old = s->coarse[level];
    s->coarse[level] = new_jacobi(&old->prm, old->weight, s->lA[level]);
    free_sol(old);
    if (level + 1 < L) {
        old = s->smoothers[level + 1];
        s->smoothers[level + 1] = new_jacobi(&old->prm, old->weight, s->lA[level]);
        free_sol(old);
        free(s->lr[level + 1]);
        s->lr[level + 1] = dalloc(an);
    }
    free(s->lb[level]);
    free(s->lx[level]);
    s->lb[level] = dalloc(an);
    s->lx[level] = dalloc(an);
    return SUCCESS;
}

/* MAT::Add, src/MAT.cxx:652-713: C = a A + b B. Row i: A's entries as a*A(i,k); each entry
 * of B's row (in order) is added to the first entry of the row so far with its column among
 * A's entries and the first appended B entry (the reference searches countrow + 1 slots), or
 * appended as b*B(i,k); then SortCSRRow. Outputs hold nnz(A) + nnz(B) entries. */
int orc_mat_add(uint32_t n, uint32_t m, double a, const uint32_t* arp, const uint32_t* aci,
                const double* ava, double b, const uint32_t* brp, const uint32_t* bci,
                const double* bva, uint32_t* nnzC, uint32_t* rpC, uint32_t* ciC, double* vaC)
{
    (void)m;
    uint32_t count = 0;
    rpC[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t start = count, c1 = arp[i + 1] - arp[i];
        for (uint32_t k = arp[i]; k < arp[i + 1]; ++k) {
            ciC[count] = aci[k];
            vaC[count] = a * ava[k];
            ++count;
        }
        for (uint32_t k = brp[i]; k < brp[i + 1]; ++k) {
            const uint32_t window = (count - start > c1) ? c1 + 1 : c1;
            uint32_t l = 0;
            for (; l < window; ++l)
                if (ciC[start + l] == bci[k]) break;
            if (l < window) {
                vaC[start + l] = vaC[start + l] + b * bva[k];
            } else {
                ciC[count] = bci[k];
                vaC[count] = b * bva[k];
                ++count;
            }
        }
        rpC[i + 1] = count;
    }
    sort_rows(n, rpC, ciC, vaC);
    *nnzC = count;
    return SUCCESS;
}

