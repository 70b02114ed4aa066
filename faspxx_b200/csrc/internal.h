// internal.h -- host-side structures and kernel launchers shared by the library's sources.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace fb {

// Launches kern with programmatic stream serialization: the kernel calls pdl_wait() before
// its first read of anything a predecessor wrote, so its launch overlaps the predecessor's
// tail without changing what it reads.
template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*kern)(P...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, A&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// An NVTX range over a scope: the solver's phases (matrix upload, setup, solve, the
// reliable-update refreshes, batched solves) appear as named ranges under a tracing tool
// (Nsight Systems, ncu --nvtx); with no tool attached the calls return at once.
struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    explicit TraceRange(const std::string& name) { nvtxRangePushA(name.c_str()); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

// Return codes: the FaspRetCode values of FASP++ (src/RetCode.hxx:24-55), plus two for the
// device layer.
enum Err {
    kOk = 0,
    kErrInputPar = -12,
    kErrVecSize = -14,
    kErrMatSize = -15,
    kErrNonmatch = -16,
    kErrMatData = -17,
    kErrDivZero = -18,
    kErrZeroDiag = -19,
    kErrAlloc = -20,
    kErrSolverType = -30,
    kErrPcdType = -31,
    kErrStag = -32,
    kErrSolStag = -33,
    kErrTolSmall = -34,
    kErrMaxIt = -39,
    kErrCuda = -101,
    kErrNoDevice = -102,
};

// Constants of include/Faspxx.hxx:31-46.
constexpr double kCloseZero = 1e-20;
constexpr double kSmallDbl = -1e+60;
constexpr double kKsmChkRatio = 0.95;
constexpr unsigned kMaxStagNum = 20;

// A scalar operand: a host value, or (m * *p) / (m / *p when inv) read on the device, so
// that one kernel can consume another's reduction without a host round trip.
struct Scal {
    double        v;
    const double* p;
    double        m;
    int           inv;
    static Scal h(double x) { return Scal{x, nullptr, 1.0, 0}; }
    static Scal d(const double* q, double mul = 1.0) { return Scal{0.0, q, mul, 0}; }
    static Scal dinv(const double* q, double mul = 1.0) { return Scal{0.0, q, mul, 1}; }
};

__device__ __forceinline__ double eval(const Scal& s)
{
    if (!s.p) return s.v;
    return s.inv ? s.m / *s.p : s.m * *s.p;
}

constexpr int kSlots = 256;

// Execution context: one stream, its reduction scratch and scalar slots.
struct Ctx {
    int          dev = 0;
    int          nsm = 148;
    cudaStream_t stream = nullptr;
    bool         ownStream = false;
    Scratch      red{nullptr, nullptr};
    double*      dslot = nullptr;  // device scalars [kSlots]
    double*      hslot = nullptr;  // pinned host mirror [kSlots]
    unsigned long long launches = 0; // kernels launched on this context
    cudaEvent_t  joinEv[2] = {nullptr, nullptr}; // stream-ordering events (created on use)
    int init(int device);
    void destroy();
    // Stream ordering with a caller's stream (the _async entry points): join_from makes this
    // context's stream wait for all work enqueued on `user` so far; join_to makes `user` wait
    // for all work enqueued on this context's stream so far. No-ops when user == stream.
    int  join_from(cudaStream_t user);
    int  join_to(cudaStream_t user);
    // fixed-size grids (reductions depend on them): at most perSM blocks per SM
    int  grid(long long work, int perBlock, int perSM = 8) const;
    int  sync();
    int  fetch(int slot, double* out);               // read one device scalar (synchronous)
};

// The device chosen by fasp_gpu_init (capi.cu).
int library_device();

// Runs `work` (which enqueues on c.stream) ordered after everything the caller enqueued on
// `user` before the call, and orders the caller's later work on `user` after it.
template <typename F>
int on_stream(Ctx& c, cudaStream_t user, F&& work)
{
    int e = c.join_from(user);
    if (!e) e = work();
    const int j = c.join_to(user);
    return e ? e : j;
}

// Blocks of `fn` at `block` threads that are resident at once on the whole device (one
// wave): SM count x the occupancy limit (registers, shared memory), capped at kMaxGrid.
// Grid-stride kernels launched with min(work, this) never run a partial second wave.
int resident_grid(const Ctx& c, const void* fn, int block, size_t smem = 0);
// Whether fn's static shared memory plus smem bytes of block tiles stay within the 48 KB a
// launch gets without opting in (else the launcher runs the kernel without tiles).
bool tiles_fit(const void* fn, size_t smem);

// Reads `bytes` of `buf` (a multiple of 16) through L2 on stream s and writes nothing (blas.cu):
// after a read of more than the L2's 126 MB, L2 holds only clean lines of buf, so a kernel
// timed next reads its inputs from HBM without paying to write back dirty lines first.
int l2_flush_read(Ctx& c, const void* buf, size_t bytes);

// Average device time (ms) of one call of `launch` over reps calls, CUDA events on c.stream.
// flushL2 = 0: the calls run back to back between two events (inputs that fit L2 stay
// there). flushL2 = 1: every call follows a 256 MB read that evicts L2 (126 MB) and leaves
// it clean, so its inputs come from HBM and no write-back of dirty lines lands in it; the
// reps (flush, call) pairs run back to back between two events, the reps flushes alone are
// timed the same way, and the difference is the calls' time. Timing each call alone between
// its own two events instead would add the launch latency of an idle stream (measured
// about 14 us on B200, against a 42 us SpMV) to every call.
template <typename F>
int time_launches(Ctx& c, unsigned reps, int flushL2, F&& launch, double* ms)
{
    void* flush = nullptr;
    const size_t fbytes = (size_t)256 << 20;
    if (flushL2 && cudaMalloc(&flush, fbytes) != cudaSuccess) {
        cudaGetLastError();
        return kErrAlloc;
    }
    if (flushL2) cudaMemsetAsync(flush, 0, fbytes, c.stream);
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    int e = kOk;
    auto window = [&](bool withCall, bool withFlush, double* out) {
        cudaEventRecord(t0, c.stream);
        for (unsigned k = 0; k < reps && !e; ++k) {
            if (withFlush) l2_flush_read(c, flush, fbytes);
            if (withCall) e = launch();
        }
        cudaEventRecord(t1, c.stream);
        cudaEventSynchronize(t1);
        float t = 0.f;
        cudaEventElapsedTime(&t, t0, t1);
        *out = t;
    };
    double tot = 0.0;
    if (!flushL2) {
        window(true, false, &tot);
    } else {
        double pair = 0.0, alone = 0.0;
        if (!e) { // untimed warm-up pair
            l2_flush_read(c, flush, fbytes);
            e = launch();
        }
        window(true, true, &pair);
        window(false, true, &alone);
        tot = pair > alone ? pair - alone : 0.0;
    }
    *ms = tot / reps;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(flush);
    if (cudaGetLastError() != cudaSuccess && !e) e = kErrCuda;
    return e;
}

// CSRx matrix resident in device memory.
struct Mat {
    uint32_t  nrow = 0, mcol = 0, nnz = 0;
    uint32_t* rowPtr = nullptr;
    uint32_t* colInd = nullptr;
    uint32_t* diagPtr = nullptr;
    double*   val = nullptr;     // nullptr: pattern only
    float*    val32 = nullptr;   // FP32 copy for the mixed-precision inner solves (lazy)
    double*   diag = nullptr;    // GetDiag (1 for pattern-only)
    int       lanes = 8;         // lanes per row of the SpMV (autotuned or from row lengths)
    bool      diagConst = false; // every row stores a diagonal entry, all with one value
    int16_t*  cd16 = nullptr;    // colInd - row when every entry is within 32,767 columns
    bool      cd16On = false;    // the thread-per-row kernels use cd16 (opt-in: measured
                                 // slower than the 32-bit colInd on B200)
    uint32_t  tileSpan = 0;      // most entries of a 256-row tile (m_tile_span), 0 unknown
    double    diagValue = 0.0;
    uint32_t  maxRowLen = 0;
    double    meanRowLen = 0;
    int       dev = 0;
    // row-class form (built at upload when the rows fall into few classes; see CSRView)
    uint16_t* rcCls = nullptr;
    uint32_t* rcOff = nullptr;
    int32_t*  rcDelta = nullptr;
    double*   rcVal = nullptr;
    float*    rcVal32 = nullptr;
    uint32_t  rcClasses = 0, rcEntries = 0;
    bool      rcOn = false;      // used by the thread-per-row kernels when built and enabled
    // stencil-mask form (built with the classes when they are subsets of one stencil)
    uint16_t* skMask = nullptr;
    bool      skOn = true;       // masks used when built (and row classes are on)
    uint32_t  skLen = 0;
    int32_t   skDelta[kMaxStencil] = {};
    double    skVal[kMaxStencil] = {};
    // structured-grid (matrix-free) operator: no CSR arrays; the stencil is skLen / skDelta /
    // skVal (flattened offsets, ascending) with per-dimension offsets gd[3][k]
    bool      grid = false;
    uint32_t  gdim[3] = {0, 0, 0};
    int8_t    gd[3][kMaxStencil] = {};
    template <typename T>
    CSRView<T> view(const T* v, const T* cv) const
    {
        CSRView<T> V{};
        V.nrow = nrow;
        V.mcol = mcol;
        V.nnz = nnz;
        V.rowPtr = rowPtr;
        V.colInd = colInd;
        V.cd16 = (cd16On && !(rcOn && rcCls && v && cv)) ? cd16 : nullptr;
        V.val = v;
        V.tileSpan = tileSpan;
        if (grid) {
            V.ulen = skLen;
            for (uint32_t u = 0; u < skLen; ++u) {
                V.udelta[u] = skDelta[u];
                V.uval[u] = (T)skVal[u];
            }
            V.gnx = gdim[0];
            V.gny = gdim[1];
            V.gnz = gdim[2];
            V.gnxy = gdim[0] * gdim[1];
            const FastDiv fx = FastDiv::make(gdim[0]), fxy = FastDiv::make(V.gnxy);
            V.gmx = fx.m;
            V.gsx[0] = fx.s1;
            V.gsx[1] = fx.s2;
            V.gmxy = fxy.m;
            V.gsxy[0] = fxy.s1;
            V.gsxy[1] = fxy.s2;
            for (int d = 0; d < 3; ++d)
                for (int t = 0; t < 4; ++t) {
                    uint32_t lo = 0, hi = 0;
                    for (uint32_t u = 0; u < skLen; ++u) {
                        if (gd[d][u] >= -t) lo |= 1u << u;
                        if (gd[d][u] <= t) hi |= 1u << u;
                    }
                    V.glo[4 * d + t] = (uint16_t)lo;
                    V.ghi[4 * d + t] = (uint16_t)hi;
                }
            return V;
        }
        if (rcOn && rcCls && v && cv) {
            V.cls = rcCls;
            V.coff = rcOff;
            V.cdelta = rcDelta;
            V.cval = cv;
            if (skMask && skOn) {
                V.mask = skMask;
                V.ulen = skLen;
                for (uint32_t u = 0; u < skLen; ++u) {
                    V.udelta[u] = skDelta[u];
                    V.uval[u] = (T)skVal[u];
                }
            }
        }
        return V;
    }
    CSRView<double> v64() const { return view<double>(val, rcVal); }
    CSRView<float>  v32() const { return view<float>(val32, rcVal32); }
    int ensure32(cudaStream_t s);
};

// ---- vector kernels (blas.cu) ---------------------------------------------------------
// T = double or float (explicitly instantiated for both). Reductions write their FP64 result
// to a device scalar (dres); vector updates take Scal.
template <typename T> int v_dot(Ctx& c, uint32_t n, const T* a, const T* b, double* dres);
template <typename T> int v_norm2(Ctx& c, uint32_t n, const T* a, double* dres);
template <typename T> int v_norminf(Ctx& c, uint32_t n, const T* a, double* dres);
template <typename T> int v_axpy(Ctx& c, uint32_t n, Scal a, const T* x, T* y);   // y += a x
template <typename T> int v_xpay(Ctx& c, uint32_t n, Scal a, const T* x, T* y);   // y = a y + x
template <typename T>
int v_axpby(Ctx& c, uint32_t n, Scal a, Scal b, const T* y, T* x);                 // x = a x + b y
template <typename T>
int v_waxpby(Ctx& c, uint32_t n, Scal a, const T* v1, Scal b, const T* v2, T* w); // w = a v1 + b v2
template <typename T> int v_scale(Ctx& c, uint32_t n, Scal a, T* x);
template <typename T> int v_set(Ctx& c, uint32_t n, double v, T* x);
template <typename T> int v_copy(Ctx& c, uint32_t n, const T* src, T* dst);
template <typename T> int v_pmult(Ctx& c, uint32_t n, const T* d, T* x);          // x *= d
template <typename T> int v_add(Ctx& c, uint32_t n, const T* d, T* x);            // x += d
int v_recip_scale(Ctx& c, uint32_t n, double w, const double* d, double* out); // out = w*(1/d)
// Classical Gram-Schmidt blocks over a basis stored at V + j*ld:
// dres[j] = (V_j, w) for j < k, in one pass over w;
// A non-null stop (device flag) turns the launches into no-ops once it is set.
template <typename T>
int v_multidot(Ctx& c, uint32_t n, int k, const T* V, size_t ld, const T* w, double* dres,
               const int* stop = nullptr);
// w -= sign * sum_j h[j] V_j (h on the device); dnorm (nullable) receives ||w_new||.
template <typename T>
int v_multiaxpy(Ctx& c, uint32_t n, int k, const T* V, size_t ld, const double* h,
                double sign, T* w, double* dnorm, const int* stop = nullptr);
// w -= sum_j h[j] V_j then dres[j] = (V_j, w), in one pass for k <= 8 (bit-identical to
// v_multiaxpy followed by v_multidot, which it falls back to above)
template <typename T>
int v_multiaxpy_dot(Ctx& c, uint32_t n, int k, const T* V, size_t ld, const double* h, T* w,
                    double* dres, const int* stop = nullptr);

// ---- sparse kernels (spmv.cu) ---------------------------------------------------------
int m_upload(Mat& M, uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
             const uint32_t* colInd, const double* values, bool hostPtrs, cudaStream_t s);
// A structured-grid operator (no stored matrix): nx x ny x nz points, npts stencil points
// (dx, dy, dz) with coefficients, truncated at the faces (spmv.cu).
int m_create_stencil(Mat& M, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t npts,
                     const int32_t* dx, const int32_t* dy, const int32_t* dz, const double* coef,
                     cudaStream_t s);
// C = L R exactly as MAT::Mult (src/MAT.cxx:715-800) forms it (spgemm.cu).
int m_mult(Ctx& c, const Mat& L, const Mat& R, Mat& C);
// C = a A + b B exactly as MAT::Add (src/MAT.cxx:652-713) forms it (spgemm.cu).
int m_add(Ctx& c, double a, const Mat& A, double b, const Mat& B, Mat& C);
// The CSR arrays of a grid operator, generated on the host (downloads and tests).
void m_grid_csr(const Mat& M, std::vector<uint32_t>& rowPtr, std::vector<uint32_t>& colInd,
                std::vector<double>& values);
void m_free(Mat& M);
// ReadMat's conversions on the device (ingest.cu): MTXtoMAT of 0-based triplets, and
// ReadCSR's shift + SortCSRRow + CSRtoMAT of raw CSR arrays (0- or 1-based).
int m_from_coo(Ctx& c, uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowInd,
               const uint32_t* colInd, const double* values, bool onDevice, Mat& M);
int m_from_csr_raw(Ctx& c, uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                   const uint32_t* colInd, const double* values, bool onDevice, Mat& M);
int m_spmv(Ctx& c, const Mat& A, const double* x, double* y);           // y = A x
int m_spmv32(Ctx& c, const Mat& A, const float* x, float* y);
inline int m_spmv(Ctx& c, const Mat& A, const float* x, float* y) { return m_spmv32(c, A, x, y); }
// r = b - A x with the x ~ 0 shortcut of MAT::Residual; the NormInf(x) comes from xinf
// (device scalar computed by the caller) unless xinf is null (then computed here). The
// float overload runs on the matrix's FP32 values (Mat::ensure32 first).
int m_residual(Ctx& c, const Mat& A, const double* b, const double* x, double* r,
               const double* xinf);
int m_residual(Ctx& c, const Mat& A, const float* b, const float* x, float* r,
               const double* xinf);
int m_transpose(Ctx& c, const Mat& A, Mat& T);                            // CSR -> CSC, exact
// Builds M.cd16 (16-bit column offsets) when every |col - row| <= 32767; otherwise leaves it
// null. Synchronises the stream.
int m_build_col16(Mat& M, cudaStream_t s);
// Mat::tileSpan from the row pointers (the block tiles' fit test, csr_tile_rows).
int m_tile_span(Mat& M, cudaStream_t s);
// Tile waits that ran out in the kernels of spmv.cu and solvers.cu (bulk copies that never
// landed).
unsigned tile_timeouts_spmv();
unsigned tile_timeouts_solvers();
// v = A^T v1 + v2 on T = m_transpose(A), in MAT::MultTransposeAdd's order (MAT.cxx:541-606)
int m_mult_transpose_add(Ctx& c, const Mat& T, const double* v1, const double* v2, double* v);
int lanes_for(double meanRowLen);                                         // SpMV mapping
int m_autotune(Ctx& c, Mat& A);
// dA[k] = scale * lam[row(k)] * x[col(k)] on the sparsity pattern (sampled outer product)
int m_sampled_outer(Ctx& c, const Mat& A, const double* lam, const double* x, double scale,
                    double* dA);

} // namespace fb
