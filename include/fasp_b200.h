/*
 * fasp_b200.h -- C ABI of the B200 (sm_100a) iterative-solve library.
 *
 * Drop-in device backend for the iterative-solve path of FASP++ (FaspDevTeam/faspxx):
 * the CSRx matrix (src/MAT.hxx), the VEC kernels the solvers use (src/VEC.hxx) and the
 * SOL-derived solvers CG, BiCGStab, GMRES, FGMRES, Jacobi and the abstract MG
 * (src/SOL.hxx, CG.hxx, BiCGStab.hxx, GMRES.hxx, FGMRES.hxx, Iter.hxx, MG.hxx), with the
 * SOLParams of src/Param.hxx:57-80. Plain pointers and sizes only; every function returns
 * an int that is a FaspRetCode value (src/RetCode.hxx:24-55) or one of the
 * FASP_GPU_ERROR_* codes below. Index arrays are 32-bit unsigned like the reference's USI.
 *
 * Threading: one handle per host thread. All device work of a handle runs on the handle's
 * own CUDA stream; calls that return results block until they are ready.
 *
 * Streams: every call that enqueues device work per operation or per solve has an _async
 * form that takes the caller's CUDA stream (fasp_gpu_stream, the runtime's cudaStream_t).
 * It orders its device work after all work the caller enqueued on that stream before the
 * call, and orders all work the caller enqueues on the stream after the call after it, with
 * two events and no device-wide synchronisation; the handle's own stream still runs the work
 * (its reduction scratch and control blocks belong to it). Operator and VEC forms return
 * once the work is enqueued (reductions then write their result to DEVICE memory); solver
 * forms return once the solve has finished on the device (the solvers decide convergence
 * from device scalars) and fill info as the blocking forms do.
 */
#ifndef FASP_B200_H
#define FASP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FASP_GPU_ABI_VERSION 1

/* Device-layer failures (outside the FaspRetCode range). */
#define FASP_GPU_ERROR_CUDA (-101)
#define FASP_GPU_ERROR_NO_DEVICE (-102)

/* Solver kinds: SOLType numbers (src/Param.hxx:36-54). */
enum fasp_gpu_alg {
    FASP_GPU_IDENTITY = 0,
    FASP_GPU_CG = 1,
    FASP_GPU_BICGSTAB = 2,
    FASP_GPU_GMRES = 4,
    FASP_GPU_FGMRES = 5,
    FASP_GPU_JACOBI = 11,
    FASP_GPU_MG = 21
};

/* Arithmetic of a solve. */
enum fasp_gpu_precision {
    FASP_GPU_FP64 = 0,  /* every vector and reduction in FP64, the reference's arithmetic */
    FASP_GPU_MIXED = 1, /* FP32 inner Krylov iterations inside FP64 iterative refinement */
    FASP_GPU_MIXED_RELIABLE = 2 /* CG and BiCGStab (with Identity or one Jacobi sweep): one
                                   FP32 Krylov run with FP64 reliable updates of x and r; the
                                   search direction survives each update. Other solvers:
                                   ERROR_SOLVER_TYPE at creation. */
};

/* Gram-Schmidt variant of the GMRES/FGMRES Arnoldi step. */
enum fasp_gpu_orth {
    FASP_GPU_ORTH_CGS2 = 0, /* classical GS + one reorthogonalisation, fused multi-dot/AXPY */
    FASP_GPU_ORTH_MGS = 1,  /* modified GS, the reference's op sequence (GMRES.cxx:169-172) */
    FASP_GPU_ORTH_DCGS2 = 2 /* the default of fasp_gpu_default_config: CGS2 with the
                               re-orthogonalisation delayed into the next step, two passes over
                               the basis per step; used by GMRES restart cycles on the device
                               (Identity or one Jacobi sweep, restart length up to 48), the
                               other configurations and FGMRES run CGS2 */
};

/* SOLParams (src/Param.hxx:57-80) without the name and verbosity fields. */
typedef struct {
    uint32_t maxIter, minIter, savIter, restart;
    double   relTol, absTol;
} fasp_gpu_params;

/* Everything a reference driver sets on a solver and its preconditioner. The first
 * block mirrors the oracle's configuration so parity tests pass both the same values. */
typedef struct {
    int             alg;        /* fasp_gpu_alg */
    fasp_gpu_params prm;        /* SOL::Set{Max,Min,Sav}Iter, SetRestart, SetRelTol, ... */
    double          weight;     /* Jacobi::SetWeight when alg == FASP_GPU_JACOBI */
    uint32_t        maxRestart, minRestart; /* GMRES/FGMRES::SetMaxMinRestart; 0,0 = 30,10 */
    int             pcd;        /* preconditioner: 0 Identity, 1 Jacobi, 2 MG (an MG solve with
                                   SOLParams pcdPrm and the mg* settings below, plus any
                                   fasp_gpu_solver_set_mg_transfer levels; FP64 only) */
    double          pcdWeight;  /* its Jacobi weight */
    fasp_gpu_params pcdPrm;     /* its SOLParams (maxIter = minIter = sweeps in the examples) */
    uint32_t        mgLevels, mgCycles; /* MG::SetupALL levels, MG::SetNumCycles */
    double          mgSmoothWeight, mgCoarseWeight;
    fasp_gpu_params mgSmoothPrm, mgCoarsePrm;
    /* B200 options (no reference counterpart) */
    int             leftPrecond; /* GMRES::SetLeftPrecond (GMRES.cxx:28) */
    int             precision;   /* fasp_gpu_precision */
    int             orth;        /* fasp_gpu_orth (default DCGS2) */
    double          innerRelTol; /* MIXED: relative tolerance of each FP32 inner solve;
                                    MIXED_RELIABLE: an FP64 update each time the FP32
                                    residual has fallen by this factor (0 or >= 1: 1e-2
                                    for CG, 1e-3 for BiCGStab) */
    uint32_t        innerMaxIter;/* MIXED: iteration cap of each inner solve */
    uint32_t        maxOuter;    /* MIXED: refinement steps cap */
    int             useGraph;    /* 1: device-driven iterations captured in CUDA graphs */
    int             persistent;  /* 1: device-driven CG runs all iterations in one
                                    cooperative launch (when the device allows it);
                                    2: ... as one thread-block cluster of 16 blocks (8
                                    where 16 is refused) meeting at the hardware
                                    cluster barrier, the vectors in the cluster's
                                    distributed shared memory when they fit (n up to
                                    65,536 FP64 / 131,072 FP32): faster than the
                                    graphs only for the smallest systems;
                                    default 0: CUDA graphs of the two fused kernels */
    int             overlapLaunch; /* 1 (default): the CG and BiCGStab iteration kernels
                                    use programmatic dependent launch, each one's launch
                                    overlapping its predecessor's reduction tail */
    int             fp32Recurrence; /* MIXED, MIXED_RELIABLE CG: 1 (default) = the FP32
                                    iterations form q = A p as A z + beta q_old (the SpMV
                                    gathers one vector); 0 = as the reference, A (z + beta p) */
} fasp_gpu_config;

/* Outcome of one Solve. */
typedef struct {
    int      code;        /* FaspRetCode */
    uint32_t numIter;     /* SOL::GetIterations (MIXED: inner iterations summed) */
    double   norm2;       /* SOL::GetNorm2 */
    double   normInf;     /* SOL::GetInfNorm */
    uint32_t outerIter;   /* MIXED: refinement steps; otherwise 0 */
    uint32_t escalations; /* device-driven CG: rare branches handed back to the host */
    uint32_t launches;    /* kernels this Solve launched (graph nodes included) */
} fasp_gpu_info;

typedef struct fasp_gpu_mat_s*    fasp_gpu_mat;
typedef struct fasp_gpu_solver_s* fasp_gpu_solver;
/* A CUDA stream: the same type as the CUDA runtime's cudaStream_t (struct CUstream_st*), so
 * a cudaStream_t passes unchanged; NULL is the legacy default stream. */
typedef struct CUstream_st*       fasp_gpu_stream;

/* ---- library ------------------------------------------------------------------------ */
int         fasp_gpu_init(int device);              /* select the device; checks sm_100 */
int         fasp_gpu_abi_version(void);
const char* fasp_gpu_strerror(int code);            /* GetRetCode (src/RetCode.cxx:19-83) */
void        fasp_gpu_default_config(fasp_gpu_config* cfg, int alg); /* SOLParams() defaults */

/* ---- device memory helpers (so hosts need no CUDA runtime of their own) -------------- */
int fasp_gpu_malloc(void** dptr, size_t bytes);
int fasp_gpu_free(void* dptr);
int fasp_gpu_memcpy_h2d(void* dst, const void* src, size_t bytes);
int fasp_gpu_memcpy_d2h(void* dst, const void* src, size_t bytes);
int fasp_gpu_memset(void* dptr, int value, size_t bytes); /* every byte set to value */
int fasp_gpu_synchronize(void);
int fasp_gpu_host_alloc(void** hptr, size_t bytes); /* page-locked host memory */
int fasp_gpu_host_free(void* hptr);

/* ---- MAT: CSRx matrix in HBM (src/MAT.hxx, MAT.cxx) --------------------------------- */
/* MAT(nrow, mcol, nnz, values, colInd, rowPtr) (MAT.cxx:41-57) from HOST arrays; the
 * diagonal pointers are formed as FormDiagPtr does (MAT.cxx:917-928). values == NULL
 * builds a sparsity structure (MAT.cxx:60-75). Structure is checked like CheckCSR
 * (MATUtil.cxx:110-174): ERROR_MAT_DATA and no upload if it fails. */
int fasp_gpu_mat_create(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                        const uint32_t* colInd, const double* values, fasp_gpu_mat* out);
/* Same from DEVICE arrays (copied). */
int fasp_gpu_mat_create_device(uint32_t nrow, uint32_t mcol, uint32_t nnz,
                               const uint32_t* rowPtr, const uint32_t* colInd,
                               const double* values, fasp_gpu_mat* out);
/* ReadMat (src/ReadData.cxx:361-446) after its readers, on the device: the arrays that
 * ReadMTX (ReadData.cxx:98-218) returns -- 0-based row and column indices of nnz entries in
 * any order -- converted as MTXtoMAT does (src/MATUtil.cxx:416-436): rows counted and
 * scattered (MTXtoCSR, :252-300), each row sorted by column with equal columns kept in
 * input order (SortCSRRow, :439-476; duplicates are kept, not summed), and an explicit 0.0
 * diagonal inserted in rows without one (CSRtoMAT, :303-413). onDevice != 0: the three
 * arrays are device memory; otherwise host memory. ERROR_MAT_DATA for an index out of
 * range or a row >= mcol without a diagonal (the reference's MTXtoMAT leaves the MAT empty
 * and returns SUCCESS there); ERROR_MAT_SIZE for a zero size. */
int fasp_gpu_mat_create_coo(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowInd,
                            const uint32_t* colInd, const double* values, int onDevice,
                            fasp_gpu_mat* out);
/* The .csr branch of ReadMat on the device: the arrays ReadCSR (ReadData.cxx:221-358)
 * reads -- rowPtr[nrow + 1], colInd[nnz], values[nnz], 0-based or 1-based (rowPtr[0] == 1;
 * shifted as ReadData.cxx:350-353 does) with rows in any column order -- then SortCSRRow
 * and CSRtoMAT as above. ReadCSR's files are square: pass mcol = nrow for them.
 * ERROR_MAT_DATA when rowPtr[0] is neither 0 nor 1, rowPtr is not monotone,
 * rowPtr[nrow] - rowPtr[0] != nnz, or a column is out of range. */
int fasp_gpu_mat_create_csr_raw(uint32_t nrow, uint32_t mcol, uint32_t nnz,
                                const uint32_t* rowPtr, const uint32_t* colInd,
                                const double* values, int onDevice, fasp_gpu_mat* out);
/* A matrix-free operator (the LOP of example/TestMatFree.cxx:26-39, applied as in its
 * MatFree::Apply, :97-176, generalised): y = A x on an nx x ny x nz grid (ny = nz = 1 for
 * 1D, nz = 1 for 2D), point (ix, iy, iz) being row ix + nx (iy + ny iz), with the
 * constant-coefficient stencil sum_k coef[k] x(ix + dx[k], iy + dy[k], iz + dz[k]) over the
 * stencil points inside the grid (Dirichlet truncation at the faces). Nothing is stored:
 * kernels compute each row's points from its coordinates. Every operation gives the same
 * results as on the assembled CSR matrix (entries in ascending column order); a grid
 * operator is accepted wherever a matrix is, except the sampled outer product (no stored
 * entries, ERROR_INPUT_PAR) and SpMV lanes other than 1. npts <= 16, |dx|,|dy|,|dz| <= 3,
 * no two points at the same offset (ERROR_INPUT_PAR); points that reach past the grid in
 * some dimension (|dx| >= nx, ...) have no entries and are dropped; the diagonal (Jacobi) is the
 * coefficient of (0,0,0), 0 when absent. Download returns the CSR arrays it applies. */
int fasp_gpu_mat_create_stencil(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t npts,
                                const int32_t* dx, const int32_t* dy, const int32_t* dz,
                                const double* coef, fasp_gpu_mat* out);
/* MAT::Mult (MAT.cxx:715-800): *out = L R on the device, with MAT::Mult's exact result --
 * the columns of each row in the order in which the loop over L's row and R's rows first
 * meets them (rows are not sorted), each entry 0 + the products of that column added in the
 * same loop order. ERROR_MAT_NONMATCH (-16) unless L's columns = R's rows; ERROR_INPUT_PAR
 * for a pattern-only matrix or a grid operator (no stored values); ERROR_MAT_SIZE when the
 * product has no entries or more than 2^32 - 1 intermediate products. */
int fasp_gpu_mat_mult(fasp_gpu_mat L, fasp_gpu_mat R, fasp_gpu_mat* out);
/* MAT::Add (MAT.cxx:652-713): *out = a A + b B on the device, with MAT::Add's exact result
 * -- each row: A's entries as a A(i,k), then every entry of B's row added (b B(i,k)) to the
 * first of A's entries with its column, or to the first of B's entries already appended to
 * the row (the reference's search window), else appended; then the row sorted by column,
 * stably (SortCSRRow). ERROR_MAT_NONMATCH for different sizes; ERROR_INPUT_PAR for a
 * pattern-only matrix or a grid operator. */
int fasp_gpu_mat_add(double a, fasp_gpu_mat A, double b, fasp_gpu_mat B, fasp_gpu_mat* out);
int fasp_gpu_mat_destroy(fasp_gpu_mat A);
/* GetRowSize / GetColSize / GetNNZ (LOP.hxx:50-53, MAT.hxx:113) */
int fasp_gpu_mat_info(fasp_gpu_mat A, uint32_t* nrow, uint32_t* mcol, uint32_t* nnz);
/* GetRowPtr / GetColInd / GetValues / diagPtr to HOST arrays (MAT.cxx:627-649); any may be
 * NULL. */
int fasp_gpu_mat_download(fasp_gpu_mat A, uint32_t* rowPtr, uint32_t* colInd, double* values,
                          uint32_t* diagPtr);
/* MAT::Apply, w = A v (MAT.cxx:373-452), device vectors. */
int fasp_gpu_mat_apply(fasp_gpu_mat A, const double* v, double* w);
/* MAT::Residual, r = b - A x with its x ~ 0 shortcut (MAT.cxx:455-476). */
int fasp_gpu_mat_residual(fasp_gpu_mat A, const double* b, const double* x, double* r);
/* MAT::TransInPlace (MAT.cxx:479-538) into a new handle; structure and order bit-exact. */
int fasp_gpu_mat_transpose(fasp_gpu_mat A, fasp_gpu_mat* out);
/* MAT::MultTransposeAdd, v = A^T v1 + v2 (MAT.cxx:541-606), device vectors: v1 has nrow
 * entries, v2 and v mcol. The transpose is formed once (MAT::TransInPlace's order, as
 * fasp_gpu_mat_transpose) and cached on A -- the reference rebuilds it on every call. Each
 * v[i] starts from v2[i] and adds the products of column i of A in ascending row order,
 * each product rounded before the add: the reference's results bit for bit. The reference
 * bounds each column by A's own rowPtr[i + 1] (MAT.cxx:603), which is right only when A's row
 * pointers equal its transpose's (structurally symmetric A, every workload here); this
 * function uses the transpose's own bounds for every A, rectangular included. Pattern-only
 * matrices count each stored entry as 1 (as MAT::Apply; the reference reads its empty
 * values array), grid operators their stencil. */
int fasp_gpu_mat_mult_transpose_add(fasp_gpu_mat A, const double* v1, const double* v2,
                                    double* v);
/* MAT::GetDiag (MAT.cxx:256-267) into a device vector. */
int fasp_gpu_mat_diag(fasp_gpu_mat A, double* diag);
/* Rows-per-warp autotuner: times every lanes-per-row choice on A; returns the pick. */
int fasp_gpu_mat_autotune(fasp_gpu_mat A, int* lanes);
int fasp_gpu_mat_set_lanes(fasp_gpu_mat A, int lanes);
/* Compressed forms of constant-coefficient matrices for the thread-per-row SpMV (lanes = 1),
 * both with the CSR entry order and one FMA per entry, so results are bit-identical to CSR:
 *  - row classes: rows with identical column offsets (col - row) and values share one table
 *    entry; a row streams a 2-byte class id instead of its indices and values. Built at
 *    upload when the rows fall into at most 4096 classes whose table is at most nnz/8
 *    entries;
 *  - stencil masks: when every class is a subset of one sorted list of at most 16 offsets
 *    with one value each, a row is a 16-bit mask over that list, which the kernels receive
 *    as launch parameters (no table reads at all).
 * mode 0 = CSR, 1 = row classes, 2 = row classes with stencil masks (the default when
 * built). Set it before a solver's Setup, which captures the matrix form. info reports the
 * mode in use, the class count, table entries and the stencil length (0 = no masks). */
int fasp_gpu_mat_set_rowclass(fasp_gpu_mat A, int mode);
int fasp_gpu_mat_rowclass_info(fasp_gpu_mat A, int* mode, uint32_t* classes, uint32_t* entries,
                               uint32_t* stencil);
/* 16-bit column offsets of the CSR form (opt-in): built at upload (and for transposes) when
 * every stored entry lies within 32,767 columns of its row -- banded FDM/FEM matrices, the
 * 128^3 Laplacian's bandwidth is 16,384 -- as colInd[k] - row; with on = 1 the
 * thread-per-row kernels (lanes = 1) stream 2 bytes per entry for the columns instead of 4
 * and form each column by one add. The entries and their order are unchanged, so results
 * are bit-identical. Off by default: on B200 the 2-byte loads measured slower than the
 * 4-byte colInd (128^3 CSR CG, FP32 iterations 17.4 against 14.9 ms). Set it before a
 * solver's Setup; info reports whether the offsets exist and whether they are in use. */
int fasp_gpu_mat_set_col16(fasp_gpu_mat A, int on);
int fasp_gpu_mat_col16_info(fasp_gpu_mat A, int* built, int* inUse);
/* Block tiles of the CSR form (thread-per-row kernels, lanes = 1): 256 consecutive rows per
 * block, their row pointers, column indices and values copied into shared memory by bulk
 * asynchronous copies two tiles ahead of the threads that sum the rows (each row in CSR
 * order with one FMA per entry: results bit-identical to the row-at-a-time kernels). span =
 * the most entries a tile covers, widened to multiples of 4; fits64 / fits32 = every tile
 * fits a stage with the FP64 values / the FP32 value copy (1812 / 1868 entries: a 7-point
 * 3D or 5-point 2D stencil fits, a 9-point 2D one does not); inUse = the plain CSR form is
 * the one in use (no row classes, stencil masks or 16-bit offsets) with lanes = 1, so the
 * tiles run wherever the tile fits. */
int fasp_gpu_mat_tile_info(fasp_gpu_mat A, uint32_t* span, int* fits64, int* fits32,
                           int* inUse);
/* Tile waits that ran out since the library was loaded: a bulk copy that never completed,
 * after which the kernel went on with what the stage held. 0 on a healthy device. */
int fasp_gpu_tile_timeouts(uint32_t* count);
/* Average duration (ms) of one MAT::Apply over reps launches on FP64 (fp32 = 0) or the FP32
 * value copy (fp32 = 1), timed with CUDA events on the matrix's stream (inputs: x = 0). */
int fasp_gpu_mat_time_apply(fasp_gpu_mat A, uint32_t reps, int fp32, int flushL2,
                            double* ms);
/* Sampled outer product on A's pattern: dA[k] = scale * lam[row(k)] * x[col(k)]. The
 * matrix gradient dL/dA of x = A^-1 b is the case scale = -1 (no reference counterpart). */
int fasp_gpu_mat_sampled_outer(fasp_gpu_mat A, const double* lam, const double* x,
                               double scale, double* dA);
/* Stream-ordered forms of MAT::Apply, MAT::Residual, MAT::MultTransposeAdd and the sampled
 * outer product (see Streams above): they return once the work is enqueued. The first
 * MultTransposeAdd on a matrix forms its transpose synchronously. */
int fasp_gpu_mat_apply_async(fasp_gpu_mat A, const double* v, double* w, fasp_gpu_stream stream);
int fasp_gpu_mat_residual_async(fasp_gpu_mat A, const double* b, const double* x, double* r,
                                fasp_gpu_stream stream);
int fasp_gpu_mat_mult_transpose_add_async(fasp_gpu_mat A, const double* v1, const double* v2,
                                          double* v, fasp_gpu_stream stream);
int fasp_gpu_mat_sampled_outer_async(fasp_gpu_mat A, const double* lam, const double* x,
                                     double scale, double* dA, fasp_gpu_stream stream);

/* ---- VEC kernels on device vectors (src/VEC.cxx) ------------------------------------ */
int fasp_gpu_vec_dot(uint32_t n, const double* a, const double* b, double* result);    /* :468 */
int fasp_gpu_vec_norm2(uint32_t n, const double* a, double* result);                   /* :424 */
int fasp_gpu_vec_norminf(uint32_t n, const double* a, double* result);                 /* :441 */
int fasp_gpu_vec_axpy(uint32_t n, double a, const double* x, double* y);               /* :245 */
int fasp_gpu_vec_xpay(uint32_t n, double a, const double* x, double* y);               /* :259 */
int fasp_gpu_vec_axpby(uint32_t n, double a, double b, const double* y, double* x);    /* :274 */
int fasp_gpu_vec_waxpby(uint32_t n, double a, const double* v1, double b, const double* v2,
                        double* w);                                                    /* :329 */
int fasp_gpu_vec_scale(uint32_t n, double a, double* x);                               /* :154 */
/* Stream-ordered forms of the VEC operations above (see Streams): reductions write their
 * FP64 result to the DEVICE address dres; all return once the work is enqueued. They run on
 * the calling thread's VEC context, so calls from one thread are ordered among themselves. */
int fasp_gpu_vec_dot_async(uint32_t n, const double* a, const double* b, double* dres,
                           fasp_gpu_stream stream);
int fasp_gpu_vec_norm2_async(uint32_t n, const double* a, double* dres, fasp_gpu_stream stream);
int fasp_gpu_vec_norminf_async(uint32_t n, const double* a, double* dres,
                               fasp_gpu_stream stream);
int fasp_gpu_vec_axpy_async(uint32_t n, double a, const double* x, double* y,
                            fasp_gpu_stream stream);
int fasp_gpu_vec_xpay_async(uint32_t n, double a, const double* x, double* y,
                            fasp_gpu_stream stream);
int fasp_gpu_vec_axpby_async(uint32_t n, double a, double b, const double* y, double* x,
                             fasp_gpu_stream stream);
int fasp_gpu_vec_waxpby_async(uint32_t n, double a, const double* v1, double b,
                              const double* v2, double* w, fasp_gpu_stream stream);
int fasp_gpu_vec_scale_async(uint32_t n, double a, double* x, fasp_gpu_stream stream);
/* No counterpart in the reference. The dot product of fasp_gpu_vec_dot for callers that
 * cannot allocate device memory (for example an application whose memory pool has reserved
 * the device memory up front and forbids further driver allocations, or a latency-critical
 * loop where cudaMalloc/cudaFree would synchronize the device). It calls no allocator: its
 * reduction scratch (about 32 KB) is a static device array that every GPU loading this
 * library holds until exit. n is limited to 8,388,608 elements; larger n returns
 * ERROR_VEC_SIZE. It runs on the device chosen by fasp_gpu_init (from any host thread; the
 * thread's current device is restored on return), on that device's legacy default stream,
 * and blocks until *result (host) is written. All calls share the one scratch array: calls
 * that overlap on the GPU race and must be serialised by the caller. The first call on each
 * device looks up the array's address with that device current and keeps it; make it
 * before any stream capture begins, and do not call this entry point after
 * cudaDeviceReset (the kept address is then stale). */
int fasp_gpu_vec_dot_noalloc(uint32_t n, const double* a, const double* b, double* result);

/* ---- SOL: solvers (src/SOL.hxx and subclasses) -------------------------------------- */
int fasp_gpu_solver_create(const fasp_gpu_config* cfg, fasp_gpu_solver* out);
/* Setup(const LOP& A): binds A (the caller keeps it alive, as SOL keeps a raw pointer,
 * SOL.hxx:28), builds the preconditioner (Jacobi::Setup, Iter.cxx:29-53) and work space. */
int fasp_gpu_solver_setup(fasp_gpu_solver s, fasp_gpu_mat A);
/* MG with transfer operators (no reference counterpart: the reference's MG::SetupLevel
 * stores one operator as both restriction and prolongation, MG.cxx:42-43, and every level's
 * residual uses the top-level matrix, MG.cxx:119, so only identity transfers work there).
 * Call before fasp_gpu_solver_setup for every coarse level l = 0 .. mgLevels - 1 (level 0
 * is the Setup matrix; with pcd = 2 the levels belong to the MG preconditioner): P = prolongation from level l+1 to level l (n_l x n_{l+1}); R =
 * restriction (n_{l+1} x n_l), NULL for the exact transpose of P; Ac = the level-(l+1)
 * operator, NULL for the Galerkin product R (A_l P) formed with MAT::Mult on the GPU. The
 * cycle is the reference's (pre-smoothing, residual, restriction, coarse solve or the next
 * level's cycles, prolongation, correction, post-smoothing) with level l's smoother on A_l,
 * the coarse solver on A_mgLevels and each residual on its own level's operator. Handles
 * are borrowed: keep them alive while the solver uses them. Setup returns ERROR_INPUT_PAR
 * when a level is missing and ERROR_MAT_NONMATCH for inconsistent sizes. */
int fasp_gpu_solver_set_mg_transfer(fasp_gpu_solver s, uint32_t level, fasp_gpu_mat P,
                                    fasp_gpu_mat R, fasp_gpu_mat Ac);
/* Solve(b, x) on DEVICE vectors: x is the initial guess in, the solution out. */
int fasp_gpu_solver_solve(fasp_gpu_solver s, const double* b, double* x, fasp_gpu_info* info);
/* Solve(b, x) ordered on the caller's stream (see Streams): the solve starts after the
 * caller's earlier work on `stream` (for example the kernel that forms b) and the caller's
 * later work on `stream` starts after it, with no device-wide synchronisation. Returns once
 * the solve has finished, with info filled. */
int fasp_gpu_solver_solve_async(fasp_gpu_solver s, const double* b, double* x,
                                fasp_gpu_info* info, fasp_gpu_stream stream);
/* Solve(b, x) on HOST vectors: copies in, solves, copies out (end-to-end path). */
int fasp_gpu_solver_solve_host(fasp_gpu_solver s, const double* b, double* x,
                               fasp_gpu_info* info);
/* Residual norms the last Solve held at the end of each iteration (NaN where the solver
 * computes none); *len receives numIter + 1. */
int fasp_gpu_solver_history(fasp_gpu_solver s, double* hist, uint32_t cap, uint32_t* len);
int fasp_gpu_solver_clean(fasp_gpu_solver s);     /* SOL::Clean */
int fasp_gpu_solver_destroy(fasp_gpu_solver s);
/* Device time of the last Solve (or adjoint solve) in milliseconds (CUDA events around its
 * device work). */
int fasp_gpu_solver_last_time(fasp_gpu_solver s, double* ms);
/* Persistent CG engine (persistent = 1): the number of polls a thread block makes at one
 * software grid barrier before it gives up (0, the default: 2^24 polls with a 32 ns sleep,
 * on the order of a second). A barrier that gives up raises an error flag that makes every
 * block leave the kernel; the solve then returns FASP_GPU_ERROR_CUDA and the context stays
 * usable (no counterpart in the reference; a failure-detection bound and its test hook). */
int fasp_gpu_solver_set_barrier_limit(fasp_gpu_solver s, uint32_t polls);
/* Device-driven CG only: average duration (ms) of each of its two fused kernels over reps
 * launches, timed alone with CUDA events on the solver's stream (control logic bypassed;
 * the solver's internal vectors are overwritten). ms must hold 3 values: ms[0] SpMV
 * kernel, ms[1] update kernel, ms[2] one iteration of the persistent kernel (0 when the
 * solver does not use it). Times the FP32 engine when the solver is MIXED. */
int fasp_gpu_solver_kernel_times(fasp_gpu_solver s, uint32_t reps, int flushL2, double* ms);

/* ---- adjoint (no reference counterpart) --------------------------------------------- */
/* Solve A^T lam = g with the same Krylov kernels on the exact CSC transpose of the bound
 * matrix (built once, cached). */
int fasp_gpu_solver_solve_adjoint(fasp_gpu_solver s, const double* g, double* lam,
                                  fasp_gpu_info* info);
/* The same, ordered on the caller's stream (see Streams). */
int fasp_gpu_solver_solve_adjoint_async(fasp_gpu_solver s, const double* g, double* lam,
                                        fasp_gpu_info* info, fasp_gpu_stream stream);

/* ---- batched CG (no reference counterpart) ------------------------------------------ */
/* count independent SPD systems solved by Jacobi-PCG in one persistent launch. The systems
 * are the diagonal blocks of one CSRx matrix on the DEVICE (global row/column indices;
 * system k owns rows sysRow[k]..sysRow[k+1]-1 and its columns must stay inside that range;
 * sysRow also on the device). nrhs (1..4) right-hand sides per system, stored
 * right-hand-side-major: b[r * N + row], N = sysRow[count]. */
typedef struct fasp_gpu_batch_s* fasp_gpu_batch;
int fasp_gpu_batch_create(uint32_t count, const uint32_t* sysRow, uint32_t nnz,
                          const uint32_t* rowPtr, const uint32_t* colInd,
                          const double* values, uint32_t nrhs, fasp_gpu_batch* out);
/* Thread-block shape of the persistent launch: block (128, 256 or 512 threads) and blocks
 * per SM; the autotuner in the Python/C++ layers times the choices. */
int fasp_gpu_batch_set_shape(fasp_gpu_batch bt, int block, int blocksPerSM);
/* Solves all systems from x0 = 0 to ||r|| < relTol ||b|| per right-hand side (device b, x).
 * precision FASP_GPU_MIXED runs FP32 inner CG to innerRelTol inside FP64 refinement;
 * FASP_GPU_MIXED_RELIABLE runs FP32 CG iterations with block-local FP64 reliable updates
 * (innerRelTol = the refresh factor, default 1e-2), the FP64 iteration count.
 * iters (host, count*nrhs, may be NULL): iterations per right-hand side; resRel (host,
 * may be NULL): final relative residual per right-hand side. */
int fasp_gpu_batch_solve(fasp_gpu_batch bt, const double* b, double* x, double relTol,
                         uint32_t maxIter, int precision, double innerRelTol,
                         uint32_t* iters, double* resRel);
/* The same, ordered on the caller's stream (see Streams); returns once the batch is solved. */
int fasp_gpu_batch_solve_async(fasp_gpu_batch bt, const double* b, double* x, double relTol,
                               uint32_t maxIter, int precision, double innerRelTol,
                               uint32_t* iters, double* resRel, fasp_gpu_stream stream);
int fasp_gpu_batch_last_time(fasp_gpu_batch bt, double* ms);
int fasp_gpu_batch_destroy(fasp_gpu_batch bt);

#ifdef __cplusplus
}
#endif
#endif /* FASP_B200_H */
