// capi.cu -- the extern "C" entry points declared in include/fasp_b200.h.
#include <cstring>
#include <new>

#include "solver.h"

using namespace fb;

namespace fb {

int Ctx::init(int device)
{
    dev = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return kErrNoDevice;
    }
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    nsm = v > 0 ? v : 148;
    if (nsm * 16 > kMaxGrid) nsm = kMaxGrid / 16;
    FB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    ownStream = true;
    FB_CUDA(cudaMalloc(&red.partials, sizeof(double) * kMaxRedValues * kMaxGrid));
    FB_CUDA(cudaMalloc(&red.ticket, sizeof(unsigned) * 4));
    FB_CUDA(cudaMemset(red.ticket, 0, sizeof(unsigned) * 4));
    FB_CUDA(cudaMalloc(&dslot, sizeof(double) * kSlots));
    FB_CUDA(cudaMemset(dslot, 0, sizeof(double) * kSlots));
    FB_CUDA(cudaMallocHost(&hslot, sizeof(double) * kSlots));
    return kOk;
}

void Ctx::destroy()
{
    if (stream) cudaStreamSynchronize(stream);
    for (cudaEvent_t& ev : joinEv)
        if (ev) {
            cudaEventDestroy(ev);
            ev = nullptr;
        }
    cudaFree(red.partials);
    cudaFree(red.ticket);
    cudaFree(dslot);
    if (hslot) cudaFreeHost(hslot);
    if (ownStream && stream) cudaStreamDestroy(stream);
    red = Scratch{nullptr, nullptr};
    dslot = nullptr;
    hslot = nullptr;
    stream = nullptr;
}

int Ctx::join_from(cudaStream_t user)
{
    if (user == stream) return kOk;
    if (!joinEv[0]) FB_CUDA(cudaEventCreateWithFlags(&joinEv[0], cudaEventDisableTiming));
    FB_CUDA(cudaEventRecord(joinEv[0], user));
    FB_CUDA(cudaStreamWaitEvent(stream, joinEv[0], 0));
    return kOk;
}

int Ctx::join_to(cudaStream_t user)
{
    if (user == stream) return kOk;
    if (!joinEv[1]) FB_CUDA(cudaEventCreateWithFlags(&joinEv[1], cudaEventDisableTiming));
    FB_CUDA(cudaEventRecord(joinEv[1], stream));
    FB_CUDA(cudaStreamWaitEvent(user, joinEv[1], 0));
    return kOk;
}

int Ctx::sync()
{
    FB_CUDA(cudaStreamSynchronize(stream));
    return kOk;
}

int Ctx::fetch(int slot, double* out)
{
    FB_CUDA(cudaMemcpyAsync(hslot + slot, dslot + slot, 8, cudaMemcpyDeviceToHost, stream));
    FB_CUDA(cudaStreamSynchronize(stream));
    *out = hslot[slot];
    return kOk;
}

} // namespace fb

static int g_device = 0;

namespace fb {
int library_device() { return g_device; }
} // namespace fb

// Per-thread context for the stand-alone VEC entry points.
static Ctx* vec_ctx(int* err)
{
    static thread_local Ctx* c = nullptr;
    static thread_local int cdev = -1;
    if (c && cdev == g_device) return c;
    if (c) {
        c->destroy();
        delete c;
    }
    c = new Ctx();
    *err = c->init(g_device);
    cdev = g_device;
    return c;
}

static cudaStream_t user_stream(fasp_gpu_stream s) { return reinterpret_cast<cudaStream_t>(s); }

// Stream-ordered VEC operations on the calling thread's context.
template <typename F>
static int vec_async(fasp_gpu_stream st, F&& work)
{
    int err = 0;
    Ctx* c = vec_ctx(&err);
    if (err) return err;
    return on_stream(*c, user_stream(st), [&]() { return work(*c); });
}

// A handle whose matrix is built by `build` on the handle's own stream.
template <typename F>
static int mat_build(fasp_gpu_mat* out, F build)
{
    if (!out) return kErrInputPar;
    *out = nullptr;
    fasp_gpu_mat h = new (std::nothrow) fasp_gpu_mat_s();
    if (!h) return kErrAlloc;
    int e = h->c.init(g_device);
    if (!e) e = build(h);
    if (e) {
        h->c.destroy();
        delete h;
        return e;
    }
    *out = h;
    return kOk;
}

extern "C" {

int fasp_gpu_abi_version(void) { return FASP_GPU_ABI_VERSION; }

int fasp_gpu_init(int device)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return FASP_GPU_ERROR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return FASP_GPU_ERROR_NO_DEVICE;
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) return FASP_GPU_ERROR_NO_DEVICE; // built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return FASP_GPU_ERROR_CUDA;
    g_device = device;
    return kOk;
}

const char* fasp_gpu_strerror(int code)
{
    switch (code) {
        case 0: return "Successful return";
        case -10: return "Cannot open file";
        case -11: return "Wrong input file";
        case -12: return "Wrong input parameters";
        case -14: return "Wrong vector size";
        case -15: return "Wrong matrix size";
        case -16: return "Sizes do not match";
        case -17: return "Wrong matrix data";
        case -18: return "Divided by zero";
        case -19: return "Matrix has zero diagonal entries";
        case -20: return "Cannot allocate memory";
        case -30: return "Unknown solver type";
        case -31: return "Unknown preconditioner type";
        case -32: return "Iterative solver stagnates";
        case -33: return "Iterative solver's solution is too small";
        case -34: return "Iterative solver's tolerance is too small";
        case -39: return "Maximal iteration number reached";
        case FASP_GPU_ERROR_CUDA: return "CUDA runtime error";
        case FASP_GPU_ERROR_NO_DEVICE: return "No sm_100 CUDA device available";
        default: return "Unknown error";
    }
}

void fasp_gpu_default_config(fasp_gpu_config* cfg, int alg)
{
    std::memset(cfg, 0, sizeof(*cfg));
    const fasp_gpu_params d{1u, 0u, 100000u, 30u, 1e-6, 1e-8}; // SOLParams() (Param.hxx:68-79)
    cfg->alg = alg;
    cfg->prm = d;
    cfg->weight = 1.0;
    cfg->pcd = 0;
    cfg->pcdWeight = 1.0;
    cfg->pcdPrm = d;
    cfg->mgLevels = 3;
    cfg->mgCycles = 1;
    cfg->mgSmoothWeight = 1.0;
    cfg->mgCoarseWeight = 1.0;
    cfg->mgSmoothPrm = d;
    cfg->mgCoarsePrm = d;
    cfg->precision = FASP_GPU_FP64;
    cfg->orth = FASP_GPU_ORTH_DCGS2;
    cfg->innerRelTol = 1e-4;
    cfg->innerMaxIter = 0;
    cfg->maxOuter = 50;
    cfg->useGraph = 1;
    cfg->persistent = 0;
    cfg->overlapLaunch = 1;
    cfg->fp32Recurrence = 1;
}

// ---- memory ---------------------------------------------------------------------------

int fasp_gpu_malloc(void** p, size_t bytes)
{
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return kErrAlloc;
    }
    return kOk;
}

int fasp_gpu_free(void* p)
{
    FB_CUDA(cudaFree(p));
    return kOk;
}

int fasp_gpu_memcpy_h2d(void* dst, const void* src, size_t bytes)
{
    FB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return kOk;
}

int fasp_gpu_memcpy_d2h(void* dst, const void* src, size_t bytes)
{
    FB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return kOk;
}

int fasp_gpu_memset(void* dst, int value, size_t bytes)
{
    FB_CUDA(cudaMemset(dst, value, bytes));
    return kOk;
}

int fasp_gpu_synchronize(void)
{
    FB_CUDA(cudaDeviceSynchronize());
    return kOk;
}

int fasp_gpu_host_alloc(void** p, size_t bytes)
{
    if (cudaMallocHost(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return kErrAlloc;
    }
    return kOk;
}

int fasp_gpu_host_free(void* p)
{
    FB_CUDA(cudaFreeHost(p));
    return kOk;
}

// ---- MAT ------------------------------------------------------------------------------

static int mat_create(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                      const uint32_t* colInd, const double* values, bool host,
                      fasp_gpu_mat* out)
{
    TraceRange trace("fasp matrix upload");
    if (!out || !rowPtr || !colInd) return kErrInputPar;
    *out = nullptr;
    fasp_gpu_mat h = new (std::nothrow) fasp_gpu_mat_s();
    if (!h) return kErrAlloc;
    int e = h->c.init(g_device);
    if (!e) e = m_upload(h->M, nrow, mcol, nnz, rowPtr, colInd, values, host, h->c.stream);
    if (e) {
        h->c.destroy();
        delete h;
        return e;
    }
    *out = h;
    return kOk;
}

int fasp_gpu_mat_create(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowPtr,
                        const uint32_t* colInd, const double* values, fasp_gpu_mat* out)
{
    return mat_create(nrow, mcol, nnz, rowPtr, colInd, values, true, out);
}

int fasp_gpu_mat_create_device(uint32_t nrow, uint32_t mcol, uint32_t nnz,
                               const uint32_t* rowPtr, const uint32_t* colInd,
                               const double* values, fasp_gpu_mat* out)
{
    return mat_create(nrow, mcol, nnz, rowPtr, colInd, values, false, out);
}

int fasp_gpu_mat_create_coo(uint32_t nrow, uint32_t mcol, uint32_t nnz, const uint32_t* rowInd,
                            const uint32_t* colInd, const double* values, int onDevice,
                            fasp_gpu_mat* out)
{
    return mat_build(out, [&](fasp_gpu_mat h) {
        return m_from_coo(h->c, nrow, mcol, nnz, rowInd, colInd, values, onDevice != 0, h->M);
    });
}

int fasp_gpu_mat_create_csr_raw(uint32_t nrow, uint32_t mcol, uint32_t nnz,
                                const uint32_t* rowPtr, const uint32_t* colInd,
                                const double* values, int onDevice, fasp_gpu_mat* out)
{
    return mat_build(out, [&](fasp_gpu_mat h) {
        return m_from_csr_raw(h->c, nrow, mcol, nnz, rowPtr, colInd, values, onDevice != 0,
                              h->M);
    });
}

int fasp_gpu_mat_create_stencil(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t npts,
                                const int32_t* dx, const int32_t* dy, const int32_t* dz,
                                const double* coef, fasp_gpu_mat* out)
{
    return mat_build(out, [&](fasp_gpu_mat h) {
        return m_create_stencil(h->M, nx, ny, nz, npts, dx, dy, dz, coef, h->c.stream);
    });
}

int fasp_gpu_mat_mult(fasp_gpu_mat L, fasp_gpu_mat R, fasp_gpu_mat* out)
{
    if (!L || !R) return kErrInputPar;
    return mat_build(out, [&](fasp_gpu_mat h) { return m_mult(h->c, L->M, R->M, h->M); });
}

int fasp_gpu_mat_add(double a, fasp_gpu_mat A, double b, fasp_gpu_mat B, fasp_gpu_mat* out)
{
    if (!A || !B) return kErrInputPar;
    return mat_build(out, [&](fasp_gpu_mat h) { return m_add(h->c, a, A->M, b, B->M, h->M); });
}

int fasp_gpu_mat_destroy(fasp_gpu_mat A)
{
    if (!A) return kOk;
    cudaStreamSynchronize(A->c.stream);
    if (A->T) fasp_gpu_mat_destroy(A->T);
    m_free(A->M);
    A->c.destroy();
    delete A;
    return kOk;
}

int fasp_gpu_mat_info(fasp_gpu_mat A, uint32_t* nrow, uint32_t* mcol, uint32_t* nnz)
{
    if (!A) return kErrInputPar;
    if (nrow) *nrow = A->M.nrow;
    if (mcol) *mcol = A->M.mcol;
    if (nnz) *nnz = A->M.nnz;
    return kOk;
}

int fasp_gpu_mat_download(fasp_gpu_mat A, uint32_t* rowPtr, uint32_t* colInd, double* values,
                          uint32_t* diagPtr)
{
    if (!A) return kErrInputPar;
    const Mat& M = A->M;
    if (M.grid) { // no stored matrix: the CSR arrays it applies, generated on the host
        std::vector<uint32_t> rp, ci;
        std::vector<double> va;
        m_grid_csr(M, rp, ci, va);
        if (rowPtr) std::memcpy(rowPtr, rp.data(), rp.size() * 4);
        if (colInd) std::memcpy(colInd, ci.data(), ci.size() * 4);
        if (values) std::memcpy(values, va.data(), va.size() * 8);
        if (diagPtr)
            for (uint32_t i = 0; i < M.nrow; ++i) {
                diagPtr[i] = 0;
                for (uint32_t k = rp[i]; k < rp[i + 1]; ++k)
                    if (ci[k] == i) {
                        diagPtr[i] = k;
                        break;
                    }
            }
        return kOk;
    }
    if (rowPtr) FB_CUDA(cudaMemcpy(rowPtr, M.rowPtr, ((size_t)M.nrow + 1) * 4, cudaMemcpyDeviceToHost));
    if (colInd) FB_CUDA(cudaMemcpy(colInd, M.colInd, (size_t)M.nnz * 4, cudaMemcpyDeviceToHost));
    if (values && M.val) FB_CUDA(cudaMemcpy(values, M.val, (size_t)M.nnz * 8, cudaMemcpyDeviceToHost));
    if (diagPtr) FB_CUDA(cudaMemcpy(diagPtr, M.diagPtr, (size_t)M.nrow * 4, cudaMemcpyDeviceToHost));
    return kOk;
}

int fasp_gpu_mat_apply(fasp_gpu_mat A, const double* v, double* w)
{
    if (!A || !v || !w) return kErrInputPar;
    int e = m_spmv(A->c, A->M, v, w);
    if (e) return e;
    return A->c.sync();
}

int fasp_gpu_mat_residual(fasp_gpu_mat A, const double* b, const double* x, double* r)
{
    if (!A || !b || !x || !r) return kErrInputPar;
    int e = m_residual(A->c, A->M, b, x, r, nullptr);
    if (e) return e;
    return A->c.sync();
}

// A's exact transpose, built once and cached on the handle (adjoint solves and
// MultTransposeAdd share it).
static int cached_transpose(fasp_gpu_mat A)
{
    if (A->T) return kOk;
    return fasp_gpu_mat_transpose(A, &A->T);
}

int fasp_gpu_mat_mult_transpose_add(fasp_gpu_mat A, const double* v1, const double* v2,
                                    double* v)
{
    if (!A || !v1 || !v2 || !v) return kErrInputPar;
    int e = cached_transpose(A);
    if (!e) e = m_mult_transpose_add(A->c, A->T->M, v1, v2, v);
    if (e) return e;
    return A->c.sync();
}

int fasp_gpu_mat_apply_async(fasp_gpu_mat A, const double* v, double* w, fasp_gpu_stream st)
{
    if (!A || !v || !w) return kErrInputPar;
    return on_stream(A->c, user_stream(st), [&]() { return m_spmv(A->c, A->M, v, w); });
}

int fasp_gpu_mat_residual_async(fasp_gpu_mat A, const double* b, const double* x, double* r,
                                fasp_gpu_stream st)
{
    if (!A || !b || !x || !r) return kErrInputPar;
    return on_stream(A->c, user_stream(st),
                     [&]() { return m_residual(A->c, A->M, b, x, r, nullptr); });
}

int fasp_gpu_mat_mult_transpose_add_async(fasp_gpu_mat A, const double* v1, const double* v2,
                                          double* v, fasp_gpu_stream st)
{
    if (!A || !v1 || !v2 || !v) return kErrInputPar;
    int e = cached_transpose(A);
    if (e) return e;
    return on_stream(A->c, user_stream(st),
                     [&]() { return m_mult_transpose_add(A->c, A->T->M, v1, v2, v); });
}

int fasp_gpu_mat_transpose(fasp_gpu_mat A, fasp_gpu_mat* out)
{
    if (!A || !out) return kErrInputPar;
    *out = nullptr;
    fasp_gpu_mat h = new (std::nothrow) fasp_gpu_mat_s();
    if (!h) return kErrAlloc;
    int e = h->c.init(g_device);
    if (!e) e = m_transpose(A->c, A->M, h->M);
    if (e) {
        h->c.destroy();
        delete h;
        return e;
    }
    *out = h;
    return kOk;
}

int fasp_gpu_mat_diag(fasp_gpu_mat A, double* diag)
{
    if (!A || !diag) return kErrInputPar;
    FB_CUDA(cudaMemcpy(diag, A->M.diag, (size_t)A->M.nrow * 8, cudaMemcpyDeviceToDevice));
    return kOk;
}

int fasp_gpu_mat_autotune(fasp_gpu_mat A, int* lanes)
{
    if (!A) return kErrInputPar;
    int e = m_autotune(A->c, A->M);
    if (lanes) *lanes = A->M.lanes;
    return e;
}

int fasp_gpu_mat_set_lanes(fasp_gpu_mat A, int lanes)
{
    if (!A || lanes < 1 || lanes > 32 || (lanes & (lanes - 1))) return kErrInputPar;
    if (A->M.grid && lanes != 1) return kErrInputPar; // grid operators: thread per row
    A->M.lanes = lanes;
    return kOk;
}

int fasp_gpu_mat_set_rowclass(fasp_gpu_mat A, int mode)
{
    if (!A || mode < 0 || mode > 2) return kErrInputPar;
    if (A->M.grid) return kOk; // a grid operator has no stored form to choose
    A->M.rcOn = mode >= 1 && A->M.rcCls != nullptr;
    A->M.skOn = mode == 2;
    return kOk;
}

int fasp_gpu_mat_set_col16(fasp_gpu_mat A, int on)
{
    if (!A) return kErrInputPar;
    A->M.cd16On = on != 0;
    return kOk;
}

int fasp_gpu_mat_col16_info(fasp_gpu_mat A, int* built, int* inUse)
{
    if (!A) return kErrInputPar;
    if (built) *built = A->M.cd16 != nullptr;
    if (inUse) *inUse = A->M.cd16 != nullptr && A->M.cd16On && !A->M.rcOn;
    return kOk;
}

int fasp_gpu_mat_tile_info(fasp_gpu_mat A, uint32_t* span, int* fits64, int* fits32,
                           int* inUse)
{
    if (!A) return kErrInputPar;
    const Mat& M = A->M;
    const bool f64 = M.tileSpan > 0 && M.tileSpan <= TileShape<double>::cap;
    const bool f32 = M.tileSpan > 0 && M.tileSpan <= TileShape<float>::cap;
    if (span) *span = M.tileSpan;
    if (fits64) *fits64 = f64;
    if (fits32) *fits32 = f32;
    if (inUse) *inUse = !M.grid && !M.rcOn && !(M.cd16 && M.cd16On) && M.lanes == 1;
    return kOk;
}

int fasp_gpu_tile_timeouts(uint32_t* count)
{
    if (!count) return kErrInputPar;
    *count = tile_timeouts_spmv() + tile_timeouts_solvers();
    return kOk;
}

int fasp_gpu_mat_rowclass_info(fasp_gpu_mat A, int* mode, uint32_t* classes, uint32_t* entries,
                               uint32_t* stencil)
{
    if (!A) return kErrInputPar;
    const Mat& M = A->M;
    if (mode) *mode = M.grid ? 3 : (!M.rcOn ? 0 : (M.skOn && M.skMask ? 2 : 1));
    if (classes) *classes = M.rcClasses;
    if (entries) *entries = M.rcEntries;
    if (stencil) *stencil = (M.skMask || M.grid) ? M.skLen : 0;
    return kOk;
}

int fasp_gpu_mat_time_apply(fasp_gpu_mat A, uint32_t reps, int fp32, int flushL2, double* ms)
{
    if (!A || !ms || reps == 0) return kErrInputPar;
    Ctx& c = A->c;
    Mat& M = A->M;
    int e;
    if (fp32 && (e = M.ensure32(c.stream))) return e;
    const size_t es = fp32 ? 4 : 8;
    void *x = nullptr, *y = nullptr;
    if (cudaMalloc(&x, (size_t)M.mcol * es + 16) || cudaMalloc(&y, (size_t)M.nrow * es + 16)) {
        cudaGetLastError();
        cudaFree(x);
        return kErrAlloc;
    }
    FB_CUDA(cudaMemsetAsync(x, 0, (size_t)M.mcol * es, c.stream));
    auto one = [&]() {
        return fp32 ? m_spmv32(c, M, (const float*)x, (float*)y)
                    : m_spmv(c, M, (const double*)x, (double*)y);
    };
    for (int w = 0; w < 3; ++w)
        if ((e = one())) break;
    if (!e) e = time_launches(c, reps, flushL2, one, ms);
    cudaFree(x);
    cudaFree(y);
    FB_CUDA(cudaGetLastError());
    return e;
}

int fasp_gpu_mat_sampled_outer(fasp_gpu_mat A, const double* lam, const double* x,
                               double scale, double* dA)
{
    if (!A || !lam || !x || !dA) return kErrInputPar;
    int e = m_sampled_outer(A->c, A->M, lam, x, scale, dA);
    if (e) return e;
    return A->c.sync();
}

int fasp_gpu_mat_sampled_outer_async(fasp_gpu_mat A, const double* lam, const double* x,
                                     double scale, double* dA, fasp_gpu_stream st)
{
    if (!A || !lam || !x || !dA) return kErrInputPar;
    return on_stream(A->c, user_stream(st),
                     [&]() { return m_sampled_outer(A->c, A->M, lam, x, scale, dA); });
}

// ---- VEC ------------------------------------------------------------------------------

static int vec_reduce(int which, uint32_t n, const double* a, const double* b, double* result)
{
    int err = 0;
    Ctx* c = vec_ctx(&err);
    if (err) return err;
    if (!result) return kErrInputPar;
    if (which == 0)
        err = v_dot(*c, n, a, b, c->dslot);
    else if (which == 1)
        err = v_norm2(*c, n, a, c->dslot);
    else
        err = v_norminf(*c, n, a, c->dslot);
    if (err) return err;
    return c->fetch(0, result);
}

int fasp_gpu_vec_dot(uint32_t n, const double* a, const double* b, double* r) { return vec_reduce(0, n, a, b, r); }
int fasp_gpu_vec_norm2(uint32_t n, const double* a, double* r) { return vec_reduce(1, n, a, nullptr, r); }
int fasp_gpu_vec_norminf(uint32_t n, const double* a, double* r) { return vec_reduce(2, n, a, nullptr, r); }

#define VEC_CALL(expr)            \
    int err = 0;                  \
    Ctx* c = vec_ctx(&err);       \
    if (err) return err;          \
    err = (expr);                 \
    if (err) return err;          \
    return c->sync();

int fasp_gpu_vec_axpy(uint32_t n, double a, const double* x, double* y) { VEC_CALL(v_axpy(*c, n, Scal::h(a), x, y)) }
int fasp_gpu_vec_xpay(uint32_t n, double a, const double* x, double* y) { VEC_CALL(v_xpay(*c, n, Scal::h(a), x, y)) }
int fasp_gpu_vec_axpby(uint32_t n, double a, double b, const double* y, double* x)
{
    VEC_CALL(v_axpby(*c, n, Scal::h(a), Scal::h(b), y, x))
}
int fasp_gpu_vec_waxpby(uint32_t n, double a, const double* v1, double b, const double* v2, double* w)
{
    VEC_CALL(v_waxpby(*c, n, Scal::h(a), v1, Scal::h(b), v2, w))
}
int fasp_gpu_vec_scale(uint32_t n, double a, double* x) { VEC_CALL(v_scale(*c, n, Scal::h(a), x)) }

int fasp_gpu_vec_dot_async(uint32_t n, const double* a, const double* b, double* dres,
                           fasp_gpu_stream st)
{
    if (!dres) return kErrInputPar;
    return vec_async(st, [&](Ctx& c) { return v_dot(c, n, a, b, dres); });
}
int fasp_gpu_vec_norm2_async(uint32_t n, const double* a, double* dres, fasp_gpu_stream st)
{
    if (!dres) return kErrInputPar;
    return vec_async(st, [&](Ctx& c) { return v_norm2(c, n, a, dres); });
}
int fasp_gpu_vec_norminf_async(uint32_t n, const double* a, double* dres, fasp_gpu_stream st)
{
    if (!dres) return kErrInputPar;
    return vec_async(st, [&](Ctx& c) { return v_norminf(c, n, a, dres); });
}
int fasp_gpu_vec_axpy_async(uint32_t n, double a, const double* x, double* y, fasp_gpu_stream st)
{
    return vec_async(st, [&](Ctx& c) { return v_axpy(c, n, Scal::h(a), x, y); });
}
int fasp_gpu_vec_xpay_async(uint32_t n, double a, const double* x, double* y, fasp_gpu_stream st)
{
    return vec_async(st, [&](Ctx& c) { return v_xpay(c, n, Scal::h(a), x, y); });
}
int fasp_gpu_vec_axpby_async(uint32_t n, double a, double b, const double* y, double* x,
                             fasp_gpu_stream st)
{
    return vec_async(st, [&](Ctx& c) { return v_axpby(c, n, Scal::h(a), Scal::h(b), y, x); });
}
int fasp_gpu_vec_waxpby_async(uint32_t n, double a, const double* v1, double b, const double* v2,
                              double* w, fasp_gpu_stream st)
{
    return vec_async(st,
                     [&](Ctx& c) { return v_waxpby(c, n, Scal::h(a), v1, Scal::h(b), v2, w); });
}
int fasp_gpu_vec_scale_async(uint32_t n, double a, double* x, fasp_gpu_stream st)
{
    return vec_async(st, [&](Ctx& c) { return v_scale(c, n, Scal::h(a), x); });
}

// ---- SOL ------------------------------------------------------------------------------

int fasp_gpu_solver_create(const fasp_gpu_config* cfg, fasp_gpu_solver* out)
{
    if (!cfg || !out) return kErrInputPar;
    *out = nullptr;
    switch (cfg->alg) {
        case FASP_GPU_CG: case FASP_GPU_BICGSTAB: case FASP_GPU_GMRES: case FASP_GPU_FGMRES:
        case FASP_GPU_JACOBI: case FASP_GPU_MG: break;
        default: return kErrSolverType;
    }
    if (cfg->precision == FASP_GPU_MIXED && cfg->alg != FASP_GPU_CG &&
        cfg->alg != FASP_GPU_BICGSTAB && cfg->alg != FASP_GPU_GMRES &&
        cfg->alg != FASP_GPU_FGMRES)
        return kErrSolverType;
    if (cfg->precision == FASP_GPU_MIXED_RELIABLE && cfg->alg != FASP_GPU_CG &&
        cfg->alg != FASP_GPU_BICGSTAB)
        return kErrSolverType;
    if (cfg->precision < FASP_GPU_FP64 || cfg->precision > FASP_GPU_MIXED_RELIABLE)
        return kErrInputPar;
    fasp_gpu_solver h = new (std::nothrow) fasp_gpu_solver_s();
    if (!h) return kErrAlloc;
    h->s.cfg = *cfg;
    int e = h->s.c.init(g_device);
    if (e) {
        h->s.c.destroy();
        delete h;
        return e;
    }
    *out = h;
    return kOk;
}

int fasp_gpu_solver_setup(fasp_gpu_solver s, fasp_gpu_mat A)
{
    if (!s || !A) return kErrInputPar;
    TraceRange trace("fasp solver setup");
    s->s.destroy();
    return s->s.setup(A);
}

int fasp_gpu_solver_set_mg_transfer(fasp_gpu_solver s, uint32_t level, fasp_gpu_mat P,
                                    fasp_gpu_mat R, fasp_gpu_mat Ac)
{
    if (!s || !P || level > 64) return kErrInputPar;
    auto& in = s->s.mgIn;
    if (in.size() <= level) in.resize(level + 1);
    in[level].P = P;
    in[level].R = R;
    in[level].Ac = Ac;
    return kOk;
}

int fasp_gpu_solver_solve(fasp_gpu_solver s, const double* b, double* x, fasp_gpu_info* info)
{
    if (!s || !b || !x) return kErrInputPar;
    return s->s.solve(b, x, info);
}

int fasp_gpu_solver_solve_async(fasp_gpu_solver s, const double* b, double* x,
                                fasp_gpu_info* info, fasp_gpu_stream st)
{
    if (!s || !b || !x) return kErrInputPar;
    return on_stream(s->s.c, user_stream(st), [&]() { return s->s.solve(b, x, info); });
}

int fasp_gpu_solver_solve_host(fasp_gpu_solver s, const double* b, double* x, fasp_gpu_info* info)
{
    if (!s || !b || !x || !s->s.A) return kErrInputPar;
    SolverImpl& S = s->s;
    const size_t bytes = (size_t)S.n * 8;
    if (!S.hostB) {
        // device staging for the host entry point, kept for the solver's lifetime
        if (cudaMalloc(&S.hostB, bytes + 16) || cudaMalloc(&S.hostX, bytes + 16)) {
            cudaGetLastError();
            return kErrAlloc;
        }
    }
    int e = kOk;
    if (cudaMemcpyAsync(S.hostB, b, bytes, cudaMemcpyHostToDevice, S.c.stream) ||
        cudaMemcpyAsync(S.hostX, x, bytes, cudaMemcpyHostToDevice, S.c.stream))
        e = kErrCuda;
    if (!e) e = S.solve(S.hostB, S.hostX, info);
    if (!e && (cudaMemcpyAsync(x, S.hostX, bytes, cudaMemcpyDeviceToHost, S.c.stream) ||
               cudaStreamSynchronize(S.c.stream)))
        e = kErrCuda;
    return e;
}

int fasp_gpu_solver_history(fasp_gpu_solver s, double* hist, uint32_t cap, uint32_t* len)
{
    if (!s) return kErrInputPar;
    const auto& H = s->s.hist;
    if (len) *len = (uint32_t)H.size();
    if (hist)
        for (uint32_t k = 0; k < cap && k < H.size(); ++k) hist[k] = H[k];
    return kOk;
}

int fasp_gpu_solver_clean(fasp_gpu_solver s)
{
    if (!s) return kErrInputPar;
    s->s.clean();
    return kOk;
}

int fasp_gpu_solver_destroy(fasp_gpu_solver s)
{
    if (!s) return kOk;
    s->s.destroy();
    s->s.c.destroy();
    delete s;
    return kOk;
}

int fasp_gpu_solver_last_time(fasp_gpu_solver s, double* ms)
{
    if (!s || !ms) return kErrInputPar;
    *ms = s->s.lastMs;
    return kOk;
}

int fasp_gpu_solver_set_barrier_limit(fasp_gpu_solver s, uint32_t polls)
{
    if (!s) return kErrInputPar;
    SolverImpl& S = s->s;
    S.barLimit = polls;
    if (S.cg64) S.cg64->barLimit = polls;
    if (S.cg32) S.cg32->barLimit = polls;
    return kOk;
}

int fasp_gpu_solver_kernel_times(fasp_gpu_solver s, uint32_t reps, int flushL2, double* ms)
{
    if (!s || !ms || reps == 0) return kErrInputPar;
    SolverImpl& S = s->s;
    if (S.cg32) return S.cg32->time_kernels(reps, flushL2, ms);
    if (S.cg64) return S.cg64->time_kernels(reps, flushL2, ms);
    return kErrSolverType;
}

// The adjoint solver: a solver of s's configuration bound to the cached exact transpose.
static int adjoint_solver(fasp_gpu_solver s)
{
    SolverImpl& S = s->s;
    fasp_gpu_mat Ah = S.Ah;
    // MAT::TransInPlace into a handle cached on (and destroyed with) the matrix
    int e = cached_transpose(Ah);
    if (e) return e;
    if (!S.adj) {
        // a solver of the same configuration bound to A^T
        S.adj = new (std::nothrow) SolverImpl();
        if (!S.adj) return kErrAlloc;
        S.adj->cfg = S.cfg;
        e = S.adj->c.init(g_device);
        if (!e) e = S.adj->setup(Ah->T);
        if (e) {
            S.adj->destroy();
            S.adj->c.destroy();
            delete S.adj;
            S.adj = nullptr;
            return e;
        }
    }
    return kOk;
}

int fasp_gpu_solver_solve_adjoint(fasp_gpu_solver s, const double* g, double* lam,
                                  fasp_gpu_info* info)
{
    if (!s || !g || !lam || !s->s.Ah) return kErrInputPar;
    SolverImpl& S = s->s;
    int e = adjoint_solver(s);
    if (e) return e;
    e = S.adj->solve(g, lam, info);
    S.lastMs = S.adj->lastMs; // last_time reports the most recent solve, adjoint included
    return e;
}

int fasp_gpu_solver_solve_adjoint_async(fasp_gpu_solver s, const double* g, double* lam,
                                        fasp_gpu_info* info, fasp_gpu_stream st)
{
    if (!s || !g || !lam || !s->s.Ah) return kErrInputPar;
    SolverImpl& S = s->s;
    int e = adjoint_solver(s);
    if (e) return e;
    e = on_stream(S.adj->c, user_stream(st), [&]() { return S.adj->solve(g, lam, info); });
    S.lastMs = S.adj->lastMs;
    return e;
}

} // extern "C"
