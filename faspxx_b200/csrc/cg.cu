// cg.cu -- kernels and engine of the device-driven PCG (see cg.cuh).
//
// One iteration is two fused kernels:
//   cg_spmv   ax = A p with p = z + beta p_old formed on the fly for every gathered
//             entry (the XPAY of CG.cxx:233 folded into the SpMV), p written once for the
//             owned rows, and the partials of (ax, p) (CG.cxx:101-104);
//   cg_update x += alpha p, r -= alpha ax, z = diagInv .* r, with the partials of
//             (r,r), (z,r), (x,x), max|x| and (p,p) (CG.cxx:122-133,141-152,224-228).
// The last block of each kernel reduces the partials in a fixed order and runs the
// scalar part of CG::Solve on one thread. Branches that need more vector work than these
// two kernels do (breakdown, safe-guard copy, stagnation restart, false-convergence check)
// set status = kEsc and are finished by the host, which then relaunches cg_resume.
#include <cstring>
#include <type_traits>
#include <utility>

#include <cooperative_groups.h>

#include "cg.cuh"

namespace fb {

#define GRID_STRIDE(i, n) \
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)(n); \
         i += (size_t)gridDim.x * blockDim.x)

__device__ __forceinline__ void cg_rec(CGCtl* c, unsigned k, double v)
{
    const unsigned g = k + c->histOffset;
    if (c->hist && g < c->histCap) c->hist[g] = v * c->histScale;
}

__device__ __forceinline__ void cg_done(CGCtl* c, int code)
{
    c->code = code;
    c->status = kDone;
}

__device__ __forceinline__ void cg_esc(CGCtl* c, int reason, int phase, const double* red)
{
    for (int k = 0; k < 5; ++k) c->red[k] = red[k];
    c->reason = reason;
    c->phase = phase;
    c->status = kEsc;
}

// while (numIter < maxIter) + the minIter check at the top of the loop (CG.cxx:82-91).
__device__ void cg_looptop(CGCtl* c, double rr)
{
    if (c->numIter >= c->maxIter) {
        cg_done(c, c->code);
        return;
    }
    if (c->numIter == c->minIter) {
        const double resAbs = sqrt(rr);
        c->resAbs = resAbs;
        c->resAbsOld = resAbs;
        c->denAbs = (kCloseZero > resAbs) ? kCloseZero : resAbs;
        c->resRel = resAbs / c->denAbs;
        cg_rec(c, c->numIter, resAbs);
        if (c->inner ? (c->resRel < c->innerTol) : (c->resRel < c->relTol || resAbs < c->absTol))
            cg_done(c, c->code);
    }
}

// Prepare for the next iteration (CG.cxx:219-234), then the next loop top.
__device__ void cg_prepare_next(CGCtl* c, double zr, double rr)
{
    if (c->numIter < c->maxIter) {
        c->resAbsOld = c->resAbs;
        const double beta = zr / c->tmpa;
        c->tmpa = zr;
        c->beta = beta;
        c->pmode = c->pzero ? 0 : 1;
        c->pzero = 0;
    }
    cg_looptop(c, rr);
}

// CG.cxx:99-119: ++numIter, then alpha = tmpa / (ax, p) unless |(ax, p)| <= 1e-40.
__device__ void cg_after_spmv(CGCtl* c, double tmpb)
{
    c->numIter += 1;
    c->tmpb = tmpb;
    if (fabs(tmpb) > kCloseZero * kCloseZero) {
        c->alpha = c->tmpa / tmpb;
        c->xpend = 1;
    } else if (c->inner)
        cg_done(c, kErrDivZero);
    else {
        const double red[5] = {0, 0, 0, 0, 0};
        cg_esc(c, kBreakdown, 0, red);
    }
}

// CG.cxx:130-216 from `phase` on; red = {rr, zr, xx, max|x|, pp} of the updated vectors.
__device__ void cg_checks(CGCtl* c, const double* red, int phase)
{
    if (c->inner) {
        const double resAbs = sqrt(red[0]);
        c->resAbs = resAbs;
        c->resRel = resAbs / c->denAbs;
        cg_rec(c, c->numIter, resAbs);
        if (c->reliable) {
            // Reliable updates: hand x and r to the host for an FP64 refresh when the
            // recursive residual meets the stop test or has fallen by delta since the last
            // refresh. phase 1 = resumed right after a refresh (the host checked the stop).
            if (resAbs > c->rmax) c->rmax = resAbs;
            if (phase < 1 && (c->resRel < c->innerTol || resAbs < c->absTolIn ||
                              resAbs < c->delta * c->rmax)) {
                if (c->devRefresh) {
                    c->status = kRefresh;
                    c->reason = kReliable;
                } else {
                    cg_esc(c, kReliable, 1, red);
                }
                return;
            }
            cg_prepare_next(c, red[1], red[0]);
            return;
        }
        if (c->resRel < c->innerTol) {
            cg_done(c, kOk);
            return;
        }
        cg_prepare_next(c, red[1], red[0]);
        return;
    }
    const unsigned it = c->numIter;
    if (it >= c->minIter) {
        if (phase <= 0) {
            c->resAbs = sqrt(red[0]);
            c->resRel = c->resAbs / c->denAbs;
            c->ratio = c->resAbs / c->resAbsOld;
            if (it >= c->savIter && c->resAbs < c->resAbsOld) {
                cg_esc(c, kSave, 1, red);
                return;
            }
        }
        if (phase <= 1 && c->ratio > kKsmChkRatio) {
            if (red[3] < kCloseZero) { // Check I: x vanishes
                cg_rec(c, it, c->resAbs);
                cg_done(c, kErrSolStag);
                return;
            }
            const double xRelDiff = fabs(c->alpha) * sqrt(red[4]) / sqrt(red[2]);
            if ((c->stagStep <= kMaxStagNum) && (xRelDiff < c->solStagTol)) { // Check II
                c->xRelDiff = xRelDiff;
                cg_esc(c, kStag, 2, red);
                return;
            }
        }
        if (phase <= 2 && c->resRel < c->relTol) { // Check III: confirm with b - A x
            cg_esc(c, kCheck3, 3, red);
            return;
        }
        cg_rec(c, it, c->resAbs);
    }
    cg_prepare_next(c, red[1], red[0]);
}

// After the FP64 residual of a reliable update: t = {(r,r) FP64, (r,r) and (z,r) of the
// rescaled FP32 copy}. Stops when the FP64 test passes; otherwise the FP32 iteration goes
// on from the refreshed residual with the same p (beta = (z,r) / (z,r)_old).
__device__ void cg_after_refresh(CGCtl* c, const double* t)
{
    const double rn = sqrt(t[0]);
    c->res64 = rn;
    c->refreshes += 1;
    c->reason = kNoReason;
    c->xpend = 0; // the fold applied it
    const bool conv = rn / c->den64 < c->relTol || rn < c->absTol;
    // three refreshes in a row without real progress: the tolerance is below what FP32
    // iterations with FP64 refreshes attain here (ERROR_SOLVER_TOLSMALL)
    c->stall = rn > sqrt(c->delta) * c->resPrev ? c->stall + 1 : 0;
    c->resPrev = rn;
    if (conv || !isfinite(rn) || c->stall >= 3) {
        c->converged = conv ? 1 : 0;
        cg_rec(c, c->numIter, rn / c->histScale);
        cg_done(c, conv ? kOk : kErrTolSmall);
        return;
    }
    c->status = kRun;
    // A refreshed residual far above the recursive one (a start at the rounding floor, or
    // FP32 drift) carries none of the Krylov space p was built for: beta would be huge and
    // p would swamp it, so the direction restarts from z (p = z).
    if (rn / c->histScale > 4.0 * c->resAbs) c->pzero = 1;
    c->rmax = sqrt(t[1]);
    // one-reduction engines refresh in the cg_spmv slot: the cg_update slot that follows has
    // nothing to update
    if (c->onered) c->skipUpd = c->numIter + 1;
    const double red[5] = {t[1], t[2], 0.0, 0.0, 0.0};
    cg_checks(c, red, 1);
    cg_rec(c, c->numIter, rn / c->histScale);
}

// Reliable update, part 1 (in the cg_spmv slot): x64 += s x32, x32 = 0.
// A lean engine first applies the pending x += alpha p of the last iteration.
__device__ __forceinline__ void cg_refresh_fold(uint32_t n, float* x32, const float* p,
                                                const CGCtl* c)
{
    double* x64 = c->rx;
    const double s = c->histScale;
    const float alpha = (float)c->alpha;
    const bool pend = p && c->xpend;
    GRID_STRIDE(i, n)
    {
        const float xi = pend ? fmaf(alpha, p[i], x32[i]) : x32[i];
        x64[i] = fma(s, (double)xi, x64[i]);
        x32[i] = 0.0f;
    }
}

// The structure of the FP32 view that the FP64 refresh residual walks (small enough to pass
// by value; the stencil offsets and all FP64 values come from the control block).
struct RefreshView {
    uint32_t        nrow, ulen;
    const uint32_t* rowPtr;
    const uint32_t* colInd;
    const uint16_t* cls;
    const uint32_t* coff;
    const int32_t*  cdelta;
    const uint16_t* mask;
    // structured-grid form (see CSRView)
    uint32_t        gnx, gny, gnz, gnxy, gmx, gmxy;
    uint8_t         gsx[2], gsxy[2];
    uint16_t        glo[12], ghi[12];
};

__device__ __forceinline__ RefreshView refresh_view(const CSRView<float>& A)
{
    RefreshView R;
    R.nrow = A.nrow;
    R.ulen = A.ulen;
    R.rowPtr = A.rowPtr;
    R.colInd = A.colInd;
    R.cls = A.cls;
    R.coff = A.coff;
    R.cdelta = A.cdelta;
    R.mask = A.mask;
    R.gnx = A.gnx;
    R.gny = A.gny;
    R.gnz = A.gnz;
    R.gnxy = A.gnxy;
    R.gmx = A.gmx;
    R.gmxy = A.gmxy;
    for (int k = 0; k < 2; ++k) {
        R.gsx[k] = A.gsx[k];
        R.gsxy[k] = A.gsxy[k];
    }
    for (int k = 0; k < 12; ++k) {
        R.glo[k] = A.glo[k];
        R.ghi[k] = A.ghi[k];
    }
    return R;
}

// Row `row` of the FP64 matrix: the same storage form and entry order as row_apply.
template <typename XV>
__device__ __forceinline__ double row_fp64(const RefreshView& A, const CGCtl* c, size_t row,
                                           XV xv)
{
    double s = 0.0;
    if (A.mask || A.gnz) {
        const uint32_t m = A.gnz ? grid_mask(A, (uint32_t)row) : (uint32_t)__ldcs(A.mask + row);
        for (uint32_t k = 0; k < A.ulen; ++k)
            if ((m >> k) & 1u)
                s = fma(c->skval[k], xv((uint32_t)((long long)row + c->skdelta[k])), s);
        return s;
    }
    if (A.cls) {
        const uint32_t k = __ldcs(A.cls + row);
        for (uint32_t i = A.coff[k]; i < A.coff[k + 1]; ++i)
            s = fma(c->rcval[i], xv((uint32_t)((long long)row + A.cdelta[i])), s);
        return s;
    }
    for (uint32_t k = A.rowPtr[row]; k < A.rowPtr[row + 1]; ++k)
        s = fma(c->rval[k], xv(A.colInd[k]), s);
    return s;
}

// Reliable update, part 2 (in the cg_update slot): r64 = b - A x64 on the FP64 values,
// r32 = r64 / s, z32 = diagInv .* r32, with the three sums of cg_after_refresh. Not inlined:
// it runs a few times per solve and must not cost the update kernel registers.
template <int JAC>
__device__ __noinline__ void cg_refresh_residual(RefreshView A, float* r32, float* z32,
                                                 const float* dinv32, CGCtl* c, Scratch s)
{
    const double* b = c->rb;
    const double* x64 = c->rx;
    double* r64 = c->rr;
    const double inv = 1.0 / c->histScale;
    double rr64 = 0.0;
    float rr = 0.f, zr = 0.f;
    GRID_STRIDE(row, A.nrow)
    {
        const double ax = row_fp64(A, c, row, [&](uint32_t j) { return x64[j]; });
        const double ri = b[row] - ax;
        r64[row] = ri;
        const float r32i = (float)(ri * inv);
        r32[row] = r32i;
        float zi = r32i;
        if (JAC == 1) {
            zi = dinv32[row] * r32i;
            z32[row] = zi;
        } else if (JAC == 2) {
            zi = (float)c->zc * r32i;
        }
        rr64 = fma(ri, ri, rr64);
        rr = fmaf(r32i, r32i, rr);
        zr = fmaf(zi, r32i, zr);
    }
    double a[3] = {rr64, (double)rr, (double)zr};
    const int ops[3] = {kSum, kSum, kSum};
    grid_reduce_ctl<3>(a, ops, s, c, [=] __device__(CGCtl* cs, const double* t) {
        cg_after_refresh(cs, t);
    });
}

// ---- kernels ---------------------------------------------------------------------------

template <typename T>
struct V16;
template <>
struct V16<float> {
    typedef float4 t;
    enum { W = 4 };
};
template <>
struct V16<double> {
    typedef double2 t;
    enum { W = 2 };
};

// Component j of a float4 (j a constant after unrolling).
__device__ __forceinline__ float f4c(const float4& v, int j)
{
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

// Elements s .. s+3 of the eight-element run (a, b); s is the same on every thread.
__device__ __forceinline__ float4 f4shift(const float4& a, const float4& b, int s)
{
    switch (s) {
        case 0: return a;
        case 1: return make_float4(a.y, a.z, a.w, b.x);
        case 2: return make_float4(a.z, a.w, b.x, b.y);
        default: return make_float4(a.w, b.x, b.y, b.z);
    }
}

// REC = 0: q = A p with p = z + beta p_old formed on the fly for every gathered entry (the
// reference's order: XPAY, then Apply); p is double-buffered.
// REC = 2: REC = 1 with one reduction per iteration (CGCtl::onered; z is r or zc r).
// REC = 1 (FP32 iterations of the mixed-precision solves): the recurrence
// q = A p = A z + beta q_old, so the SpMV gathers z alone and p, q update in place for the
// owned row (half the gathers). Its rounding differs from A p by a term that beta < 1 damps;
// the FP64 refreshes of reliable updates correct the residual it feeds.
// Blocks per SM: FP32 6 (40 registers), one-reduction FP32 5 (its extra sums spill under
// 40 registers and the spills cost more than the sixth block), FP64 5, lanes 4, vector rows
// 3 (80 registers; 4 blocks at 64 registers spilled and measured slower).
// V4 (stencil masks of at most 8 offsets): consecutive rows per thread with 16-byte loads,
// four for the FP32 recurrences, two for FP64 (REC = 0, fixed shapes only); the host checks
// n % 4 (FP64: n % 2) == 0, a square matrix and 16-byte aligned vectors (8- or 4-byte
// aligned masks). SH = 5 or 7: the offsets are
// known to be [-S1, -1, 0, 1, S1] or [-S2, -S1, -1, 0, 1, S1, S2] with S1, S2 multiples of
// 4 (the 2D and 3D Laplacian stencils on lexicographic grids), so that every gather is one
// aligned 16-byte word or a fixed shift of the row's own and a neighbouring word.
template <typename T, int L, int REC, int JZ, bool V4 = false, int SH = 0>
__global__ void __launch_bounds__(kBlock, (V4 ? 3 : (L > 1 ? 4 : (sizeof(T) == 4 ? (REC == 2 ? 5 : 6) : 5))))
    cg_spmv(CSRView<T> A, const T* __restrict__ z, T* P0, T* P1, T* __restrict__ q, T* x,
            CGCtl* c, Scratch s, MarchPlan mp)
{
    static_assert(REC != 2 || JZ != 1, "one-reduction iterations need z = r or z = zc r");
    constexpr bool ONE = REC == 2;
    pdl_wait();
    pdl_release();
    // every control field of the launch, loaded together ahead of the status test (one
    // round trip to L2 instead of two dependent ones)
    const int status = c->status;
    const int mode = c->pmode, par = c->par;
    const bool xpend = REC && c->xpend;
    const T alphaPrev = (T)c->alpha;
    const T zc = (T)c->zc;
    const T beta = (T)c->beta;
    if (status != kRun) {
        if constexpr (std::is_same<T, float>::value) {
            if (status == kRefresh) {
                if constexpr (ONE) // the cg_update slot folded x: the FP64 residual comes here
                    cg_refresh_residual<JZ>(refresh_view(A),
                                            const_cast<T*>(z), nullptr, nullptr, c, s);
                else
                    cg_refresh_fold(A.nrow, x, REC ? P0 : nullptr, c);
            }
        }
        return;
    }
    // JZ = 2: z = zc r is formed here from r (passed as z), never stored
    auto zat = [&](size_t j) { return JZ == 2 ? zc * z[j] : z[j]; };
    const T* __restrict__ pOld = par ? P1 : P0;
    T* __restrict__ pNew = par ? P0 : P1;
    T acc = T(0), rr = T(0), rq = T(0), qq = T(0);
    // the owned row's p and q from its product `sum`
    auto own = [&](size_t row, T sum) {
        const T zraw = z[row];
        const T zi = JZ == 2 ? zc * zraw : zraw;
        if (REC) {
            const T po = P0[row];
            if (xpend) x[row] = fma(alphaPrev, po, x[row]); // the last iteration's x update
            const T pi = mode ? fma(beta, po, zi) : zi;
            const T qi = mode ? fma(beta, q[row], sum) : sum;
            P0[row] = pi;
            q[row] = qi;
            acc = fma(qi, pi, acc);
            if (ONE) { // zraw is r
                rr = fma(zraw, zraw, rr);
                rq = fma(zraw, qi, rq);
                qq = fma(qi, qi, qq);
            }
        } else {
            const T pi = mode ? fma(beta, pOld[row], zi) : zi;
            pNew[row] = pi;
            q[row] = sum;
            acc = fma(sum, pi, acc);
        }
    };
    // REC with JZ = 2: the gathers read r itself and the row's sum is scaled once,
    // A z = zc (A r), instead of forming zc r_j for every gathered entry
    auto gv = [&](uint32_t j) {
        if (REC) return JZ == 2 ? z[j] : zat(j);
        return mode ? fma(beta, pOld[j], zat(j)) : zat(j);
    };
    auto ownr = [&](size_t row, T sum) { own(row, (REC && JZ == 2) ? zc * sum : sum); };
    // rows 4g .. 4g+3 from the masks m, the values xs[k] at each offset and the row's own
    // z, p, q, x: the row-per-thread arithmetic operation for operation (the same bits);
    // only the order in which a thread adds its rows into the partial sums differs
    auto group4 = [&](const uint32_t (&m)[4], const float4 (&xs)[8], const float4& zr4,
                      const float4& po4, const float4& qo4, const float4& xo4, float* pn,
                      float* qn, float* xn) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float sum = 0.f;
#pragma unroll
            for (int k = 0; k < (SH ? SH : 8); ++k)
                if ((m[j] >> k) & 1u) sum = fmaf((float)A.uval[k], f4c(xs[k], j), sum);
            if (JZ == 2) sum = (float)zc * sum;
            const float zraw = f4c(zr4, j);
            const float zi = JZ == 2 ? (float)zc * zraw : zraw;
            const float po = f4c(po4, j);
            xn[j] = fmaf((float)alphaPrev, po, f4c(xo4, j));
            pn[j] = mode ? fmaf((float)beta, po, zi) : zi;
            qn[j] = mode ? fmaf((float)beta, f4c(qo4, j), sum) : sum;
            acc = fmaf(qn[j], pn[j], (float)acc);
            if (ONE) {
                rr = fmaf(zraw, zraw, (float)rr);
                rq = fmaf(zraw, qn[j], (float)rq);
                qq = fmaf(qn[j], qn[j], (float)qq);
            }
        }
    };
    if constexpr (V4 && L == 1 && REC && sizeof(T) == 4) {
        // Rows 4g .. 4g+3 on one thread, lanes of a warp on consecutive groups g. Offset
        // d takes the rows' values
        //   d % 4 == 0:  from the aligned group g + d/4 (one 16-byte load);
        //   |d| < 4:     from this lane's own group and its neighbours' (warp shuffles; lanes
        //                0 and 31 load the group beyond the warp);
        //   otherwise:   from the aligned groups g + floor(d/4) and the one after it.
        // A needed element lies in [0, n) and n % 4 == 0, so its whole group does too; the
        // loads are issued for every group inside [0, n / 4) whatever the masks say, so
        // that they do not wait for the mask load (the masks only pick the FMAs). Group
        // indices are 32-bit and wrap (n / 4 < 2^30, |d| < 2^31), so one unsigned compare
        // bounds them. Each row's sum, p, q and x follow the row-per-thread path operation
        // for operation (the same bits); only the order in which a thread adds its rows
        // into the partial sums differs. With a fixed shape (SH) the offsets' kinds are known
        // at compile time (no per-offset branches or selects), and SH = 7 with a MarchPlan
        // walks columns of planes (below).
        const uint32_t n4 = A.nrow >> 2, stride = gridDim.x * blockDim.x;
        const uint32_t lane = threadIdx.x & 31u;
        const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4* z4 = reinterpret_cast<const float4*>(z);
        float4* p4 = reinterpret_cast<float4*>(P0);
        float4* q4 = reinterpret_cast<float4*>(q);
        float4* x4 = reinterpret_cast<float4*>(x);
        int npos = SH ? 1 : 0, nneg = SH ? 1 : 0; // reach of the offsets 0 < |d| < 4
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (!SH && k < (int)A.ulen) {
                const int d = A.udelta[k];
                if (d > npos && d < 4) npos = d;
                if (-d > nneg && d > -4) nneg = -d;
            }
        if (SH == 7 && mp.p4) {
            // Plane columns (MarchPlan, cols = p4 groups a plane): item w = (column w % cols,
            // chunk w / cols) walks groups g = column + k cols over the planes k of its chunk.
            // cols % 32 == 0, so a warp's lanes share the chunk and hold consecutive columns
            // (every lane takes part in the shuffles); the -S2 / +S2 groups rotate through
            // registers, one new z load a step.
            const uint32_t cols = mp.p4, nz = mp.nz, C = mp.chunk;
            const uint32_t items = cols * ((nz + C - 1) / C);
            const int o1 = A.udelta[1] >> 2, o5 = A.udelta[5] >> 2; // -S1 / 4, S1 / 4
            for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w - lane < items;
                 w += stride) {
                if (w >= items) break; // whole warps (items % 32 == 0)
                const uint32_t k0 = (w / cols) * C, k1 = min(k0 + C, nz);
                uint32_t g = w % cols + k0 * cols;
                float4 below = k0 > 0 ? z4[g - cols] : zero, cur = z4[g];
                for (uint32_t k = k0; k < k1; ++k, g += cols) {
                    const float4 above = k + 1 < nz ? z4[g + cols] : zero;
                    const float4 po4 = p4[g], qo4 = q4[g];
                    const float4 xo4 = xpend ? x4[g] : zero;
                    uint32_t m[4];
                    if (A.gnz) {
#pragma unroll
                        for (int j = 0; j < 4; ++j) m[j] = grid_mask(A, 4u * g + (uint32_t)j);
                    } else {
                        const uint2 mm = __ldg(reinterpret_cast<const uint2*>(A.mask) + g);
                        m[0] = mm.x & 0xffffu;
                        m[1] = mm.x >> 16;
                        m[2] = mm.y & 0xffffu;
                        m[3] = mm.y >> 16;
                    }
                    const uint32_t ga = g + (uint32_t)o1, gb = g + (uint32_t)o5;
                    const float4 s1lo = ga < n4 ? z4[ga] : zero, s1hi = gb < n4 ? z4[gb] : zero;
                    float4 pv = zero, nx = zero;
                    pv.w = __shfl_up_sync(0xffffffffu, cur.w, 1);
                    nx.x = __shfl_down_sync(0xffffffffu, cur.x, 1);
                    if (lane == 0 && g > 0) pv = z4[g - 1];
                    if (lane == 31 && g + 1 < n4) nx = z4[g + 1];
                    float4 xs[8];
                    xs[0] = below;
                    xs[1] = s1lo;
                    xs[2] = make_float4(pv.w, cur.x, cur.y, cur.z);
                    xs[3] = cur;
                    xs[4] = make_float4(cur.y, cur.z, cur.w, nx.x);
                    xs[5] = s1hi;
                    xs[6] = above;
                    xs[7] = zero;
                    float pn[4], qn[4], xn[4];
                    group4(m, xs, cur, po4, qo4, xo4, pn, qn, xn);
                    p4[g] = make_float4(pn[0], pn[1], pn[2], pn[3]);
                    q4[g] = make_float4(qn[0], qn[1], qn[2], qn[3]);
                    if (xpend) x4[g] = make_float4(xn[0], xn[1], xn[2], xn[3]);
                    below = cur;
                    cur = above;
                }
            }
        } else
        // the loop bound is the same on every lane of a warp (all lanes shuffle)
        for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g - lane < n4; g += stride) {
            const bool act = g < n4;
            float4 zr4 = zero, po4 = zero, qo4 = zero, xo4 = zero;
            uint32_t m[4] = {0u, 0u, 0u, 0u};
            if (act) {
                zr4 = z4[g];
                po4 = p4[g];
                qo4 = q4[g];
                if (xpend) xo4 = x4[g];
                if (A.gnz) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) m[j] = grid_mask(A, 4u * g + (uint32_t)j);
                } else {
                    const uint2 mm = __ldg(reinterpret_cast<const uint2*>(A.mask) + g);
                    m[0] = mm.x & 0xffffu;
                    m[1] = mm.x >> 16;
                    m[2] = mm.y & 0xffffu;
                    m[3] = mm.y >> 16;
                }
            }
            float4 pv = zero, nx = zero; // groups g - 1 and g + 1
            if (nneg) {
                pv.w = __shfl_up_sync(0xffffffffu, zr4.w, 1);
                if (nneg > 1) pv.z = __shfl_up_sync(0xffffffffu, zr4.z, 1);
                if (nneg > 2) pv.y = __shfl_up_sync(0xffffffffu, zr4.y, 1);
                if (lane == 0 && act && g > 0) pv = z4[g - 1];
            }
            if (npos) {
                nx.x = __shfl_down_sync(0xffffffffu, zr4.x, 1);
                if (npos > 1) nx.y = __shfl_down_sync(0xffffffffu, zr4.y, 1);
                if (npos > 2) nx.z = __shfl_down_sync(0xffffffffu, zr4.z, 1);
                if (lane == 31 && g + 1 < n4) nx = z4[g + 1];
            }
            float4 xs[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                xs[k] = zero;
                if (SH) { // fixed shape: offsets -1, 0, 1 sit at SH/2 - 1 .. SH/2
                    if (k >= SH) continue;
                    if (k == SH / 2) {
                        xs[k] = zr4;
                    } else if (k == SH / 2 - 1) {
                        xs[k] = make_float4(pv.w, zr4.x, zr4.y, zr4.z);
                    } else if (k == SH / 2 + 1) {
                        xs[k] = make_float4(zr4.y, zr4.z, zr4.w, nx.x);
                    } else {
                        const uint32_t ga = g + (uint32_t)(A.udelta[k] >> 2);
                        if (act && ga < n4) xs[k] = z4[ga];
                    }
                } else if (k < (int)A.ulen) {
                    const int d = A.udelta[k];
                    const uint32_t ga = g + (uint32_t)(d >> 2); // floor(d / 4), wrapped
                    if ((d & 3) == 0) {
                        if (act && ga < n4) xs[k] = z4[ga];
                    } else if (d > -4 && d < 4) {
                        xs[k] = d > 0 ? f4shift(zr4, nx, d) : f4shift(pv, zr4, 4 + d);
                    } else {
                        float4 a = zero, b = zero;
                        if (act && ga < n4) a = z4[ga];
                        if (act && ga + 1u < n4) b = z4[ga + 1u];
                        xs[k] = f4shift(a, b, d & 3);
                    }
                }
            }
            float pn[4], qn[4], xn[4];
            // inactive lanes hold zeros: their terms add +0 to the partial sums
            group4(m, xs, zr4, po4, qo4, xo4, pn, qn, xn);
            if (act) {
                p4[g] = make_float4(pn[0], pn[1], pn[2], pn[3]);
                q4[g] = make_float4(qn[0], qn[1], qn[2], qn[3]);
                if (xpend) x4[g] = make_float4(xn[0], xn[1], xn[2], xn[3]);
            }
        }
    } else if constexpr (V4 && L == 1 && !REC && sizeof(T) == 8 && SH != 0) {
        // FP64 in the reference's order (p = z + beta p_old formed for every gathered entry,
        // CG.cxx:233 folded into the SpMV): rows 2g, 2g+1 on one thread, lanes on
        // consecutive groups; the gathered p of group h comes from z and p_old at h with the
        // row-per-thread formula, -1/+1 from the neighbouring lanes' groups (shuffles; lanes
        // 0 and 31 form the group beyond the warp), +-S1 (and +-S2 outside a plane walk) from
        // aligned groups. Each row's sum and its p, q follow the row-per-thread path
        // operation for operation (the same bits); the partial sums group rows by two.
        const uint32_t n2 = A.nrow >> 1, stride = gridDim.x * blockDim.x;
        const uint32_t lane = threadIdx.x & 31u;
        const double2 zero = make_double2(0.0, 0.0);
        const double2* z2 = reinterpret_cast<const double2*>(z);
        const double2* po2 = reinterpret_cast<const double2*>(pOld);
        double2* pn2 = reinterpret_cast<double2*>(pNew);
        double2* q2 = reinterpret_cast<double2*>(q);
        constexpr int MID = SH / 2;
        auto pat = [&](uint32_t h) { // the gathered p of rows 2h, 2h+1
            const double2 zz = z2[h];
            const double a = JZ == 2 ? (double)zc * zz.x : zz.x;
            const double b = JZ == 2 ? (double)zc * zz.y : zz.y;
            if (!mode) return make_double2(a, b);
            const double2 o = po2[h];
            return make_double2(fma((double)beta, o.x, a), fma((double)beta, o.y, b));
        };
        auto masks = [&](uint32_t g, uint32_t& m0, uint32_t& m1) {
            if (A.gnz) {
                m0 = grid_mask(A, 2u * g);
                m1 = grid_mask(A, 2u * g + 1u);
            } else {
                const uint32_t mm = __ldg(reinterpret_cast<const uint32_t*>(A.mask) + g);
                m0 = mm & 0xffffu;
                m1 = mm >> 16;
            }
        };
        // the two rows' sums from the values at each offset, then p, q and (q, p)
        auto rows2 = [&](uint32_t g, uint32_t m0, uint32_t m1, const double2 (&xs)[SH],
                         const double2& pc) {
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int k = 0; k < SH; ++k) {
                if ((m0 >> k) & 1u) s0 = fma((double)A.uval[k], xs[k].x, s0);
                if ((m1 >> k) & 1u) s1 = fma((double)A.uval[k], xs[k].y, s1);
            }
            pn2[g] = pc;
            q2[g] = make_double2(s0, s1);
            acc = fma(s0, pc.x, (double)acc);
            acc = fma(s1, pc.y, (double)acc);
        };
        // -1 / +1 neighbours of a warp's consecutive groups
        auto sides = [&](uint32_t g, bool act, const double2& pc, double2& pv, double2& nx) {
            pv = zero;
            nx = zero;
            pv.y = __shfl_up_sync(0xffffffffu, pc.y, 1);
            nx.x = __shfl_down_sync(0xffffffffu, pc.x, 1);
            if (lane == 0 && act && g > 0) pv = pat(g - 1);
            if (lane == 31 && act && g + 1 < n2) nx = pat(g + 1);
        };
        bool walked = false;
        if constexpr (SH == 7) {
          if (mp.p4) {
            walked = true;
            // plane columns (MarchPlan with two-row groups: cols = S2 / 2 per plane)
            const uint32_t cols = mp.p4, nz = mp.nz, C = mp.chunk;
            const uint32_t items = cols * ((nz + C - 1) / C);
            const int o1 = A.udelta[1] >> 1, o5 = A.udelta[5] >> 1;
            for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w - lane < items;
                 w += stride) {
                if (w >= items) break; // whole warps (items % 32 == 0)
                const uint32_t k0 = (w / cols) * C, k1 = min(k0 + C, nz);
                uint32_t g = w % cols + k0 * cols;
                double2 below = k0 > 0 ? pat(g - cols) : zero, cur = pat(g);
                for (uint32_t k = k0; k < k1; ++k, g += cols) {
                    const double2 above = k + 1 < nz ? pat(g + cols) : zero;
                    uint32_t m0, m1;
                    masks(g, m0, m1);
                    const uint32_t ga = g + (uint32_t)o1, gb = g + (uint32_t)o5;
                    double2 xs[SH];
                    xs[0] = below;
                    xs[1] = ga < n2 ? pat(ga) : zero;
                    double2 pv, nx;
                    sides(g, true, cur, pv, nx);
                    xs[2] = make_double2(pv.y, cur.x);
                    xs[3] = cur;
                    xs[4] = make_double2(cur.y, nx.x);
                    xs[5] = gb < n2 ? pat(gb) : zero;
                    xs[6] = above;
                    rows2(g, m0, m1, xs, cur);
                    below = cur;
                    cur = above;
                }
            }
          }
        }
        if (!walked) {
            // the loop bound is the same on every lane of a warp (all lanes shuffle)
            for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g - lane < n2;
                 g += stride) {
                const bool act = g < n2;
                double2 pc = zero;
                uint32_t m0 = 0u, m1 = 0u;
                if (act) {
                    pc = pat(g);
                    masks(g, m0, m1);
                }
                double2 pv, nx;
                sides(g, act, pc, pv, nx);
                double2 xs[SH];
#pragma unroll
                for (int k = 0; k < SH; ++k) {
                    if (k == MID) {
                        xs[k] = pc;
                    } else if (k == MID - 1) {
                        xs[k] = make_double2(pv.y, pc.x);
                    } else if (k == MID + 1) {
                        xs[k] = make_double2(pc.y, nx.x);
                    } else {
                        const uint32_t ga = g + (uint32_t)(A.udelta[k] >> 1);
                        xs[k] = act && ga < n2 ? pat(ga) : zero;
                    }
                }
                if (act) rows2(g, m0, m1, xs, pc);
            }
        }
    } else if (L == 1 && REC && (A.mask || A.gnz) && A.ulen <= 8) {
        // stencil masks of at most 8 offsets (the 5- and 7-point stencils): 32-bit row
        // indices, each gather one signed offset from the row's own address, and no
        // offset-count tests (the mask has no bits at or above ulen)
        const uint32_t n32 = A.nrow, stride = gridDim.x * blockDim.x;
        for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < n32; row += stride) {
            // masks kept in L2 (the FP32 working set fits), or computed (grid operators)
            const uint32_t m = A.gnz ? grid_mask(A, row) : (uint32_t)__ldg(A.mask + row);
            const T* zr = z + row;
            T xs[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) xs[k] = ((m >> k) & 1u) ? zr[A.udelta[k]] : T(0);
            T sum = T(0);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if ((m >> k) & 1u) sum = fma(A.uval[k], xs[k], sum);
            ownr(row, sum);
        }
    } else if (L == 1 && REC && sizeof(T) == 4 && !A.mask && !A.gnz && !A.cls && !A.cd16) {
        // plain CSR in the FP32 recurrence kernels: rows row and row + stride on one thread
        // (row_dot2; each row's sum in the row-per-thread order, rows owned in the same
        // order, so the same bits); 128^3 CSR mixed solve 14.27 against 14.84 ms on B200.
        // The other kernels spill at their register budgets with it.
        const size_t stride = (size_t)gridDim.x * blockDim.x;
        size_t row = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        for (; row + stride < A.nrow; row += 2 * stride) {
            T s0, s1;
            row_dot2(A, row, row + stride, gv, s0, s1);
            ownr(row, s0);
            ownr(row + stride, s1);
        }
        if (row < A.nrow) ownr(row, row_apply<T, false>(A, row, gv));
    } else if (L == 1) { // thread per row
        const size_t stride = (size_t)gridDim.x * blockDim.x;
        for (size_t row = (size_t)blockIdx.x * blockDim.x + threadIdx.x; row < A.nrow;
             row += stride)
            ownr(row, row_apply<T, false>(A, row, gv));
    }
    const int lane = threadIdx.x & (L - 1);
    const size_t warpRows = 32 / L;
    const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
    const size_t sub = (threadIdx.x & 31) / L;
    for (size_t base = gw * warpRows; L > 1 && base < A.nrow; base += nwarps * warpRows) {
        const size_t row = base + sub;
        T sum = T(0);
        if (row < A.nrow) {
            const uint32_t b = A.rowPtr[row], e = A.rowPtr[row + 1];
            for (uint32_t k = b + lane; k < e; k += L) sum = fma(A.val[k], gv(A.colInd[k]), sum);
        }
        sum = group_sum<L>(sum);
        if (lane == 0 && row < A.nrow) ownr(row, sum);
    }
    if constexpr (ONE) {
        double a[4] = {(double)acc, (double)rr, (double)rq, (double)qq};
        const int ops[4] = {kSum, kSum, kSum, kSum};
        grid_reduce_ctl<4>(a, ops, s, c, [=] __device__(CGCtl* cs, const double* t) {
            if (cs->bench) return;
            // alpha from (r,z) of this r (not the value carried from the last iteration),
            // then the update's checks on the residual that cg_update will form
            const double f = JZ == 2 ? cs->zc : 1.0;
            cs->tmpa = f * t[1];
            cg_after_spmv(cs, t[0]);
            if (cs->status != kRun) return;
            const double al = cs->alpha;
            double rn = t[1] - 2.0 * al * t[2] + al * al * t[3];
            if (rn < 0.0) rn = 0.0;
            const double red[5] = {rn, f * rn, 0.0, 0.0, 0.0};
            cg_checks(cs, red, 0);
        });
    } else {
        double a[1] = {(double)acc};
        const int ops[1] = {kSum};
        grid_reduce_ctl<1>(a, ops, s, c, [=] __device__(CGCtl* cs, const double* t) {
            if (!REC) cs->par = par ^ 1;
            if (!cs->bench) cg_after_spmv(cs, t[0]);
        });
    }
}

template <typename T, int JAC>
__global__ void __launch_bounds__(kBlock, 4) cg_update(uint32_t n, T* __restrict__ x,
                                                    T* __restrict__ r, T* __restrict__ z,
                                                    const T* P0, const T* P1,
                                                    const T* __restrict__ q,
                                                    const T* __restrict__ dinv, CGCtl* c,
                                                    Scratch s, CSRView<T> A)
{
    pdl_wait();
    pdl_release();
    if (c->status != kRun) {
        if constexpr (std::is_same<T, float>::value)
            if (c->status == kRefresh)
                cg_refresh_residual<JAC>(refresh_view(A),
                                         r, z, dinv, c, s);
        return;
    }
    const T alpha = (T)c->alpha;
    const T zc = (T)c->zc;
    const T* __restrict__ p = c->par ? P1 : P0;
    T rr = 0, zr = 0, xx = 0, xm = 0, pp = 0;
    auto one = [&](T pi, T& xi, T& ri, T qi, T di, T& zi) {
        xi = fma(alpha, pi, xi);
        ri = fma(-alpha, qi, ri);
        zi = JAC == 1 ? di * ri : (JAC == 2 ? zc * ri : ri);
        rr = fma(ri, ri, rr);
        zr = fma(zi, ri, zr);
        xx = fma(xi, xi, xx);
        xm = fmax(xm, fabs(xi));
        pp = fma(pi, pi, pp);
    };
    // 16-byte accesses: all vectors are the engine's own 256-byte aligned allocations
    using V = typename V16<T>::t;
    constexpr int W = V16<T>::W;
    const size_t nv = n / W;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    // FP32: two grid-stride steps per pass, all ten 16-byte loads issued before any use,
    // doubling the bytes in flight per thread (the kernel is latency-bound at one step; the
    // FP64 variant would spill under the 64-register cap).
    constexpr bool kTwo = std::is_same<T, float>::value;
    size_t i = tid;
    for (; kTwo && i + stride < nv; i += 2 * stride) {
        T pa[2][W], xa[2][W], ra[2][W], qa[2][W], da[2][W];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const size_t k = i + h * stride;
            *(V*)pa[h] = ((const V*)p)[k];
            *(V*)xa[h] = ((const V*)x)[k];
            *(V*)ra[h] = ((const V*)r)[k];
            *(V*)qa[h] = ((const V*)q)[k];
            if (JAC == 1) *(V*)da[h] = ((const V*)dinv)[k];
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const size_t k = i + h * stride;
            // z overwrites q's registers: q is dead once r is updated
#pragma unroll
            for (int u = 0; u < W; ++u)
                one(pa[h][u], xa[h][u], ra[h][u], qa[h][u], JAC == 1 ? da[h][u] : T(0),
                    qa[h][u]);
            ((V*)x)[k] = *(V*)xa[h];
            ((V*)r)[k] = *(V*)ra[h];
            if (JAC == 1) ((V*)z)[k] = *(V*)qa[h];
        }
    }
    for (; i < nv; i += stride) {
        T pa[W], xa[W], ra[W], qa[W], da[W];
        *(V*)pa = ((const V*)p)[i];
        *(V*)xa = ((const V*)x)[i];
        *(V*)ra = ((const V*)r)[i];
        *(V*)qa = ((const V*)q)[i];
        if (JAC == 1) *(V*)da = ((const V*)dinv)[i];
#pragma unroll
        for (int u = 0; u < W; ++u)
            one(pa[u], xa[u], ra[u], qa[u], JAC == 1 ? da[u] : T(0), qa[u]);
        ((V*)x)[i] = *(V*)xa;
        ((V*)r)[i] = *(V*)ra;
        if (JAC == 1) ((V*)z)[i] = *(V*)qa;
    }
    for (size_t i = nv * W + tid; i < n; i += stride) {
        T xi = x[i], ri = r[i], zi;
        one(p[i], xi, ri, q[i], JAC == 1 ? dinv[i] : T(0), zi);
        x[i] = xi;
        r[i] = ri;
        if (JAC == 1) z[i] = zi;
    }
    double a[5] = {(double)rr, (double)zr, (double)xx, (double)xm, (double)pp};
    const int ops[5] = {kSum, kSum, kSum, kMax, kSum};
    grid_reduce_ctl<5>(a, ops, s, c, [=] __device__(CGCtl* cs, const double* t) {
        if (!cs->bench) cg_checks(cs, t, 0);
    });
}

// The lean FP32 update (engines with the recurrence): r -= alpha q, z = D r and the two sums
// (r,r), (z,r) that the FP32 loop reads; x is updated by the next cg_spmv.
template <typename T, int JAC>
__global__ void __launch_bounds__(kBlock, 4) cg_update_lean(uint32_t n, T* __restrict__ r,
                                                         T* __restrict__ z,
                                                         const T* __restrict__ q,
                                                         const T* __restrict__ dinv, CGCtl* c,
                                                         Scratch s, CSRView<T> A)
{
    pdl_wait();
    pdl_release();
    if (c->status != kRun) {
        if constexpr (std::is_same<T, float>::value)
            if (c->status == kRefresh)
                cg_refresh_residual<JAC>(refresh_view(A),
                                         r, z, dinv, c, s);
        return;
    }
    const T alpha = (T)c->alpha;
    const T zc = (T)c->zc;
    T rr = 0, zr = 0;
    using V = typename V16<T>::t;
    constexpr int W = V16<T>::W;
    const size_t nv = n / W;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    // two grid-stride steps per pass with all loads issued first (more bytes in flight per
    // thread on the small grid), then the single-step remainder; same order of sums
    size_t i = tid;
    auto step = [&](T (&ra)[W], T (&qa)[W], const T (&da)[W], size_t k) {
#pragma unroll
        for (int u = 0; u < W; ++u) {
            ra[u] = fma(-alpha, qa[u], ra[u]);
            qa[u] = JAC == 1 ? da[u] * ra[u] : (JAC == 2 ? zc * ra[u] : ra[u]); // z in q's regs
            rr = fma(ra[u], ra[u], rr);
            zr = fma(qa[u], ra[u], zr);
        }
        ((V*)r)[k] = *(V*)ra;
        if (JAC == 1) ((V*)z)[k] = *(V*)qa;
    };
    for (; i + stride < nv; i += 2 * stride) {
        T ra[2][W], qa[2][W], da[2][W];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            *(V*)ra[h] = ((const V*)r)[i + h * stride];
            *(V*)qa[h] = ((const V*)q)[i + h * stride];
            if (JAC == 1) *(V*)da[h] = ((const V*)dinv)[i + h * stride];
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) step(ra[h], qa[h], da[h], i + h * stride);
    }
    for (; i < nv; i += stride) {
        T ra[W], qa[W], da[W];
        *(V*)ra = ((const V*)r)[i];
        *(V*)qa = ((const V*)q)[i];
        if (JAC == 1) *(V*)da = ((const V*)dinv)[i];
        step(ra, qa, da, i);
    }
    for (size_t i = nv * W + tid; i < n; i += stride) {
        const T ri = fma(-alpha, q[i], r[i]);
        const T zi = JAC == 1 ? dinv[i] * ri : (JAC == 2 ? zc * ri : ri);
        r[i] = ri;
        if (JAC == 1) z[i] = zi;
        rr = fma(ri, ri, rr);
        zr = fma(zi, ri, zr);
    }
    double a[2] = {(double)rr, (double)zr};
    const int ops[2] = {kSum, kSum};
    grid_reduce_ctl<2>(a, ops, s, c, [=] __device__(CGCtl* cs, const double* t) {
        const double red[5] = {t[0], t[1], 0.0, 0.0, 0.0};
        if (!cs->bench) cg_checks(cs, red, 0);
    });
}

// The update of one-reduction engines: r -= alpha q, no sums (cg_spmv ran the checks). In a
// refresh it folds x (the FP64 residual follows in the next cg_spmv slot).
template <typename T>
__global__ void __launch_bounds__(kBlock, 4) cg_update_r(uint32_t n, T* __restrict__ r,
                                                      const T* __restrict__ q, T* x,
                                                      const T* P0, CGCtl* c)
{
    pdl_wait();
    pdl_release();
    using V = typename V16<T>::t;
    constexpr int W = V16<T>::W;
    const size_t nv = n / W;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    // the thread's first two groups are loaded with the control fields (they do not
    // depend on them), so the launch waits for one L2 round trip before its FMAs, not two
    T ra[2][W], qa[2][W];
    bool has[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        has[h] = tid + h * stride < nv;
        if (has[h]) {
            *(V*)ra[h] = ((const V*)r)[tid + h * stride];
            *(V*)qa[h] = ((const V*)q)[tid + h * stride];
        }
    }
    const int st = c->status;
    const unsigned skipUpd = c->skipUpd, numIter = c->numIter;
    const T alpha = (T)c->alpha;
    if (st != kRun) {
        if constexpr (std::is_same<T, float>::value)
            if (st == kRefresh) cg_refresh_fold(n, x, P0, c);
        return;
    }
    if (skipUpd == numIter + 1) return;
#pragma unroll
    for (int h = 0; h < 2; ++h)
        if (has[h]) {
#pragma unroll
            for (int u = 0; u < W; ++u) ra[h][u] = fma(-alpha, qa[h][u], ra[h][u]);
            ((V*)r)[tid + h * stride] = *(V*)ra[h];
        }
    size_t i = tid + 2 * stride;
    for (; i + stride < nv; i += 2 * stride) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            *(V*)ra[h] = ((const V*)r)[i + h * stride];
            *(V*)qa[h] = ((const V*)q)[i + h * stride];
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
#pragma unroll
            for (int u = 0; u < W; ++u) ra[h][u] = fma(-alpha, qa[h][u], ra[h][u]);
            ((V*)r)[i + h * stride] = *(V*)ra[h];
        }
    }
    for (; i < nv; i += stride) {
        T ra[W], qa[W];
        *(V*)ra = ((const V*)r)[i];
        *(V*)qa = ((const V*)q)[i];
#pragma unroll
        for (int u = 0; u < W; ++u) ra[u] = fma(-alpha, qa[u], ra[u]);
        ((V*)r)[i] = *(V*)ra;
    }
    for (size_t k = nv * W + tid; k < n; k += stride) r[k] = fma(-alpha, q[k], r[k]);
}

// Start of CG::Solve after rk = b - A x (CG.cxx:69-79): z = B(r), tmpa = (z, r), p = z.
template <typename T, int JAC>
__global__ void __launch_bounds__(kBlock) cg_start(uint32_t n, const T* __restrict__ r,
                                                   T* __restrict__ z, const T* __restrict__ dinv,
                                                   CGCtl* c, Scratch s)
{
    T rr = 0, zr = 0;
    const T zc = (T)c->zc;
    GRID_STRIDE(i, n)
    {
        const T ri = r[i];
        T zi = ri;
        if (JAC == 1) {
            zi = dinv[i] * ri;
            z[i] = zi;
        } else if (JAC == 2) {
            zi = zc * ri;
        }
        rr = fma(ri, ri, rr);
        zr = fma(zi, ri, zr);
    }
    double a[2] = {(double)rr, (double)zr};
    const int ops[2] = {kSum, kSum};
    grid_reduce_ctl<2>(a, ops, s, c, [=] __device__(CGCtl* cs, const double* t) {
        cs->status = kRun;
        cs->numIter = 0;
        cs->code = kOk;
        cs->tmpa = t[1];
        cs->pmode = 0;
        cs->pzero = 0;
        cs->resAbs = 1.0;
        cs->resRel = 1.0;
        cs->denAbs = 1.0;
        cs->ratio = 0.0;
        cs->resAbsOld = 1.0;
        cs->alpha = 0.0;
        cs->xpend = 0;
        cg_looptop(cs, t[0]);
    });
}

// After the host finished an escalated branch (r may have been recomputed): z = B(r), then
// the control flow continues at c->phase with fresh (r,r), (z,r).
template <typename T, int JAC>
__global__ void __launch_bounds__(kBlock) cg_resume(uint32_t n, const T* __restrict__ r,
                                                    T* __restrict__ z,
                                                    const T* __restrict__ dinv, CGCtl* c,
                                                    Scratch s)
{
    T rr = 0, zr = 0;
    const T zc = (T)c->zc;
    GRID_STRIDE(i, n)
    {
        const T ri = r[i];
        T zi = ri;
        if (JAC == 1) {
            zi = dinv[i] * ri;
            z[i] = zi;
        } else if (JAC == 2) {
            zi = zc * ri;
        }
        rr = fma(ri, ri, rr);
        zr = fma(zi, ri, zr);
    }
    double a[2] = {(double)rr, (double)zr};
    const int ops[2] = {kSum, kSum};
    grid_reduce_ctl<2>(a, ops, s, c, [=] __device__(CGCtl* cs, const double* t) {
        const double red[5] = {t[0], t[1], cs->red[2], cs->red[3], cs->red[4]};
        cs->status = kRun;
        cs->reason = kNoReason;
        cg_checks(cs, red, cs->phase);
    });
}

// ---- persistent kernel: every iteration in one cooperative launch -----------------------
// The two phases of an iteration (the cg_spmv and cg_update work above) are separated by
// a grid barrier. Instead of one last block finishing each reduction, every block reads
// all block partials after the barrier and sums them in the same fixed order, so all
// blocks hold bit-identical scalars and run the same control flow on a shared-memory copy
// of the control block; block 0 writes it back when the launch ends. Vectors that other
// blocks wrote inside this launch are read with ld.global.cg (L2), since L1 is not coherent.

constexpr int kPBlock = 256;
constexpr int kSlotPhase1 = kMaxRedValues - 1; // partial slot of the SpMV phase

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Software grid barrier for a co-resident (cooperatively launched) grid. The spin is
// bounded: after bar->limit polls (0: 2^24) it raises bar->error and every block leaves the
// kernel -- a block that was released before the error leaves at its next barrier, where it
// sees the flag -- so no block waits for good.
__device__ bool grid_sync(GridBar* bar, unsigned* gen)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned g = *gen;
        int good = 1;
        __threadfence();
        const unsigned arrived = atomicAdd(&bar->count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicExch(&bar->gen, g + 1);
        } else {
            unsigned spins = 0;
            const unsigned limit = bar->limit ? bar->limit : (1u << 24);
            while (ld_acquire_u32(&bar->gen) == g) {
                if (ld_acquire_u32(&bar->error)) {
                    good = 0;
                    break;
                }
                if (++spins > limit) {
                    atomicExch(&bar->error, 1u);
                    good = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        *gen = g + 1;
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// The one-cluster variant of the persistent kernel (small systems): its blocks are one
// thread-block cluster, co-scheduled by construction, and meet at the hardware cluster
// barrier (release/acquire at cluster scope orders the partials and vectors in global memory
// that the other blocks read next) instead of the atomic grid barrier. Every block takes the
// same branches on bit-identical scalars, as at a __syncthreads.
__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

constexpr int kCBlock = 1024; // threads per block of the one-cluster kernel

// Sum of the partials of slot k over all blocks, fixed order; every block gets the same.
template <int NV>
__device__ __forceinline__ void all_reduce_partials(const Scratch s, const int (&slot)[NV],
                                                    const int (&ops)[NV], double (&tot)[NV])
{
    // the slots are consecutive (0..4, or the single phase-1 slot)
    sum_partials<NV>(s.partials + slot[0] * kMaxGrid, ops, tot);
    block_reduce<NV>(tot, ops);
}

template <int NV>
__device__ __forceinline__ void write_partials(Scratch s, const int (&slot)[NV],
                                               const int (&ops)[NV], double (&acc)[NV])
{
    block_reduce<NV>(acc, ops);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) s.partials[slot[k] * kMaxGrid + blockIdx.x] = acc[k];
}

template <typename T, int JAC, bool CL = false>
__global__ void __launch_bounds__(CL ? kCBlock : kPBlock, CL ? 1 : 4)
cg_persistent(CSRView<T> A, T* x, T* r, T* z, T* P0, T* P1, T* q, const T* __restrict__ dinv,
              CGCtl* gctl, Scratch s, GridBar* bar, unsigned iterCap)
{
    __shared__ CGCtl c;
    __shared__ unsigned gen;
    __shared__ double bc[5];
    if (threadIdx.x == 0) {
        c = *gctl;
        if (!CL) gen = ld_acquire_u32(&bar->gen);
    }
    __syncthreads();
    auto sync = [&]() -> bool {
        if constexpr (CL) {
            cluster_sync_all();
            return true;
        } else {
            return grid_sync(bar, &gen);
        }
    };
    const uint32_t n = A.nrow;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const T* zz = JAC ? z : r;
    unsigned done = 0;
    while (c.status == kRun && done < iterCap) {
        // phase 1: ax = A p with p = z + beta p_old formed on the fly, and (ax, p)
        {
            const int mode = c.pmode, par = c.par;
            const T beta = (T)c.beta;
            const T* pOld = par ? P1 : P0;
            T* pNew = par ? P0 : P1;
            T acc = T(0);
            for (size_t row = tid; row < n; row += stride) {
                const T sum = row_apply<T, false>(A, row, [&](uint32_t j) {
                    return mode ? fma(beta, __ldcg(pOld + j), __ldcg(zz + j)) : __ldcg(zz + j);
                });
                const T pi = mode ? fma(beta, __ldcg(pOld + row), __ldcg(zz + row))
                                  : __ldcg(zz + row);
                pNew[row] = pi;
                q[row] = sum;
                acc = fma(sum, pi, acc);
            }
            double a[1] = {(double)acc};
            const int sl[1] = {kSlotPhase1}, ops[1] = {kSum};
            write_partials<1>(s, sl, ops, a);
            if (!sync()) return;
            double t[1];
            all_reduce_partials<1>(s, sl, ops, t);
            if (threadIdx.x == 0) {
                c.par = par ^ 1;
                if (!c.bench) cg_after_spmv(&c, t[0]);
            }
            __syncthreads();
            if (c.status != kRun) break;
        }
        // phase 2: x += alpha p, r -= alpha ax, z = diagInv .* r, and the five reductions
        {
            const T alpha = (T)c.alpha;
            const T* p = c.par ? P1 : P0;
            T rr = 0, zr = 0, xx = 0, xm = 0, pp = 0;
            for (size_t i = tid; i < n; i += stride) {
                const T pi = __ldcg(p + i);
                const T xi = fma(alpha, pi, __ldcg(x + i));
                const T ri = fma(-alpha, __ldcg(q + i), __ldcg(r + i));
                x[i] = xi;
                r[i] = ri;
                T zi = ri;
                if (JAC) {
                    zi = __ldg(dinv + i) * ri;
                    z[i] = zi;
                }
                rr = fma(ri, ri, rr);
                zr = fma(zi, ri, zr);
                xx = fma(xi, xi, xx);
                xm = fmax(xm, fabs(xi));
                pp = fma(pi, pi, pp);
            }
            double a[5] = {(double)rr, (double)zr, (double)xx, (double)xm, (double)pp};
            const int sl[5] = {0, 1, 2, 3, 4}, ops[5] = {kSum, kSum, kSum, kMax, kSum};
            write_partials<5>(s, sl, ops, a);
            if (!sync()) return;
            double t[5];
            all_reduce_partials<5>(s, sl, ops, t);
            if (threadIdx.x == 0) {
                for (int k = 0; k < 5; ++k) bc[k] = t[k];
                if (!c.bench) cg_checks(&c, bc, 0);
            }
            __syncthreads();
        }
        ++done;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *gctl = c;
}

// ---- small systems: one cluster, the vectors in distributed shared memory ---------------
// cg_persistent's iteration for a system whose vectors fit in the shared memory of one
// cluster: block b holds rows [b S, (b + 1) S) of x, r, z, both direction buffers and q in
// its own shared memory (S a power of two) and gathers the columns that other blocks own
// through distributed shared memory; the block partials are exchanged the same way and every
// block adds them in rank order, so all blocks take the same branches on the same scalars.
// Nothing of an iteration goes through L2 but the matrix and diagInv. The slices are loaded
// from the engine's vectors at entry and stored back at exit, where the host-side branches
// (escalations, reliable refreshes) read them; a block leaves only after the last cluster
// barrier, so no block reads the shared memory of one that has gone.
constexpr int kDsVecs = 6; // x, r, z, P0, P1, q
// rows a thread holds at most: a block's slice is at most 4,096 FP64 or 8,192 FP32 rows
// (six vectors in 227 KB), 1,024 threads a block
template <typename T>
constexpr int kDsRows = sizeof(T) == 8 ? 4 : 8;

template <typename T, int JAC>
__global__ void __launch_bounds__(kCBlock, 1)
cg_dsmem(CSRView<T> A, T* x, T* r, T* z, T* P0, T* P1, T* q, const T* __restrict__ dinv,
         CGCtl* gctl, unsigned iterCap, int shift)
{
    namespace cgx = cooperative_groups;
    cgx::cluster_group cl = cgx::this_cluster();
    extern __shared__ __align__(16) unsigned char ds_raw[];
    const uint32_t S = 1u << shift;
    T* sx = reinterpret_cast<T*>(ds_raw);
    T* sr = sx + S;
    T* sz = sr + S;
    T* sp0 = sz + S;
    T* sp1 = sp0 + S;
    T* sq = sp1 + S;
    __shared__ CGCtl c;
    __shared__ double part[2][5]; // this block's totals: the product phase, the update phase
    __shared__ double gath[16][5]; // every block's totals, fetched one block per thread
    __shared__ double bc[5];
    const uint32_t n = A.nrow, rank = cl.block_rank(), nb = cl.num_blocks();
    const uint32_t r0 = rank << shift;
    const uint32_t rows = r0 < n ? min(S, n - r0) : 0u;
    const uint32_t tid = threadIdx.x, bd = blockDim.x;
    for (uint32_t i = tid; i < rows; i += bd) {
        sx[i] = x[r0 + i];
        sr[i] = r[r0 + i];
        if (JAC) sz[i] = z[r0 + i];
        sp0[i] = P0[r0 + i];
        sp1[i] = P1[r0 + i];
        sq[i] = q[r0 + i];
    }
    if (tid == 0) c = *gctl;
    cl.sync();
    T* szz = JAC ? sz : sr;
    auto at = [&](T* base, uint32_t j) -> T {
        const uint32_t o = j >> shift, l = j & (S - 1u);
        return o == rank ? base[l] : cl.map_shared_rank(base, o)[l];
    };
    // a thread's rows i = tid + u blockDim (u < R), unrolled so that their loads overlap;
    // its diagInv entries stay in registers for the whole launch
    constexpr int R = kDsRows<T>;
    T dv[R];
#pragma unroll
    for (int u = 0; u < R; ++u) {
        const uint32_t i = tid + u * bd;
        dv[u] = JAC && i < rows ? __ldg(dinv + r0 + i) : T(0);
    }
    unsigned done = 0;
    while (c.status == kRun && done < iterCap) {
        // phase 1: ax = A p with p = z + beta p_old formed on the fly, and (ax, p)
        {
            const int mode = c.pmode, par = c.par;
            const T beta = (T)c.beta;
            T* pOld = par ? sp1 : sp0;
            T* pNew = par ? sp0 : sp1;
            T sum[R], pv[R];
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const uint32_t i = tid + u * bd;
                sum[u] = pv[u] = T(0);
                if (i < rows) {
                    sum[u] = row_apply<T, false>(A, r0 + i, [&](uint32_t j) {
                        return mode ? fma(beta, at(pOld, j), at(szz, j)) : at(szz, j);
                    });
                    pv[u] = mode ? fma(beta, pOld[i], szz[i]) : szz[i];
                }
            }
            T acc = T(0);
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const uint32_t i = tid + u * bd;
                if (i < rows) {
                    pNew[i] = pv[u];
                    sq[i] = sum[u];
                    acc = fma(sum[u], pv[u], acc);
                }
            }
            double a[1] = {(double)acc};
            const int ops[1] = {kSum};
            block_reduce<1>(a, ops);
            if (tid == 0) part[0][0] = a[0];
            cl.sync();
            if (tid < nb) gath[tid][0] = *cl.map_shared_rank(&part[0][0], tid);
            __syncthreads();
            if (tid == 0) {
                double t = 0.0;
                for (uint32_t b = 0; b < nb; ++b) t += gath[b][0];
                c.par = par ^ 1;
                if (!c.bench) cg_after_spmv(&c, t);
            }
            __syncthreads();
            if (c.status != kRun) break;
        }
        // phase 2: x += alpha p, r -= alpha ax, z = diagInv .* r, and the five reductions
        {
            const T alpha = (T)c.alpha;
            const T* p = c.par ? sp1 : sp0;
            T rr = 0, zr = 0, xx = 0, xm = 0, pp = 0;
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const uint32_t i = tid + u * bd;
                if (i >= rows) continue;
                const T pi = p[i];
                const T xi = fma(alpha, pi, sx[i]);
                const T ri = fma(-alpha, sq[i], sr[i]);
                sx[i] = xi;
                sr[i] = ri;
                T zi = ri;
                if (JAC) {
                    zi = dv[u] * ri;
                    sz[i] = zi;
                }
                rr = fma(ri, ri, rr);
                zr = fma(zi, ri, zr);
                xx = fma(xi, xi, xx);
                xm = fmax(xm, fabs(xi));
                pp = fma(pi, pi, pp);
            }
            double a[5] = {(double)rr, (double)zr, (double)xx, (double)xm, (double)pp};
            const int ops[5] = {kSum, kSum, kSum, kMax, kSum};
            block_reduce<5>(a, ops);
            if (tid == 0)
                for (int k = 0; k < 5; ++k) part[1][k] = a[k];
            cl.sync();
            if (tid < nb) {
                const double* pb = cl.map_shared_rank(&part[1][0], tid);
                for (int k = 0; k < 5; ++k) gath[tid][k] = pb[k];
            }
            __syncthreads();
            if (tid == 0) {
                double t[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                for (uint32_t b = 0; b < nb; ++b)
                    for (int k = 0; k < 5; ++k) t[k] = red_apply(t[k], gath[b][k], ops[k]);
                for (int k = 0; k < 5; ++k) bc[k] = t[k];
                if (!c.bench) cg_checks(&c, bc, 0);
            }
            __syncthreads();
        }
        ++done;
    }
    cl.sync(); // every remote read of this block's slices is done
    for (uint32_t i = tid; i < rows; i += bd) {
        x[r0 + i] = sx[i];
        r[r0 + i] = sr[i];
        if (JAC) z[r0 + i] = sz[i];
        P0[r0 + i] = sp0[i];
        P1[r0 + i] = sp1[i];
        q[r0 + i] = sq[i];
    }
    if (rank == 0 && tid == 0) *gctl = c;
}

// ---- engine ------------------------------------------------------------------------------

static int spmv_grid_cg(const Ctx& c, uint32_t nrow, int L)
{
    long long g = ((long long)nrow * L + kBlock - 1) / kBlock;
    long long cap = (long long)c.nsm * 8;
    if (cap > kMaxGrid) cap = kMaxGrid;
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

template <typename T>
static CSRView<T> view_of(const Mat& A);
template <>
CSRView<double> view_of<double>(const Mat& A) { return A.v64(); }
template <>
CSRView<float> view_of<float>(const Mat& A) { return A.v32(); }

// Launch with programmatic stream serialization when pdl is set (captured into the graph as
// a programmatic edge), so the kernel's launch overlaps its predecessor's reduction tail.
template <typename... P, typename... A>
static void launch_overlapped_smem(void (*kern)(P...), int grid, size_t smem, cudaStream_t s,
                                   bool pdl, A&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kBlock);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}
template <typename... P, typename... A>
static void launch_overlapped(void (*kern)(P...), int grid, cudaStream_t s, bool pdl,
                              A&&... args)
{
    launch_overlapped_smem(kern, grid, 0, s, pdl, std::forward<A>(args)...);
}


// The plane columns of a 3D seven-point stencil (SH = 7) with offsets +-S2, S2 a multiple
// of 32 groups of rpg rows (a warp's groups stay in one plane) dividing n: chunk planes per
// thread, so that grid x kBlock threads cover every (column, chunk) item in one pass.
template <typename V>
static MarchPlan march_plan(const V& A, int sh, int grid, int rpg)
{
    MarchPlan mp;
    if (sh != 7 || A.udelta[0] != -A.udelta[6]) return mp;
    const long long s2 = A.udelta[6];
    if (s2 % (32 * rpg) != 0 || (long long)A.nrow % s2 != 0 || (long long)A.nrow / s2 < 2)
        return mp;
    const long long p4 = s2 / rpg, nz = (long long)A.nrow / s2;
    const long long threads = (long long)grid * kBlock;
    long long chunk = (nz * p4 + threads - 1) / threads;
    if (chunk < 1) chunk = 1;
    mp.p4 = (uint32_t)p4;
    mp.nz = (uint32_t)nz;
    mp.chunk = (uint32_t)chunk;
    return mp;
}

// The two fused kernels, each on one resident wave (grid from the occupancy limit).
template <typename T>
void CGEngine<T>::launch_spmv_kernel()
{
    const CSRView<T> V = view_of<T>(*A);
    const int need = spmv_grid_cg(*c, A->nrow, A->lanes);
    const int jm = jmode();
    const T* zz = jm == 1 ? z : r;
    const int sh = stencil_shape(V);
    // The fused iteration kernels walk CSR rows one at a time, without block tiles: with its
    // p, q, x updates per row a tile's block barrier stalls every warp on the slowest one,
    // and on B200 the 128^3 CSR solves measured slower with tiles (mixed 16.3 against 14.9
    // ms, FP64 28.9 against 25.0 ms) although the product alone is faster.
    auto go = [&](auto kern) {
        const int g = std::min(need, resident_grid(*c, (const void*)kern, kBlock));
        launch_overlapped(kern, g, c->stream, pdl, V, zz, P0, P1, q, x, ctl, c->red,
                          march_plan(V, sh, g, sizeof(T) == 4 ? 4 : 2));
    };
    auto al = [](const void* p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) == 0; };
    // vector rows (stencil masks, see cg_spmv): four per thread for the FP32 recurrences,
    // two for FP64 on the 5- and 7-point shapes
    const bool base = A->lanes == 1 && (V.mask || V.gnz) && V.ulen <= 8 && V.nrow == V.mcol &&
                      V.nrow < (1u << 30) && al(zz, 16) && al(P0, 16) && al(q, 16);
    const bool v4 = sizeof(T) == 4
                        ? base && recurrence && V.nrow % 4 == 0 && al(x, 16) &&
                              (V.gnz || al(V.mask, 8))
                        : base && !recurrence && sh != 0 && V.nrow % 2 == 0 && al(P1, 16) &&
                              (V.gnz || al(V.mask, 4));
#define CG_SPMV_LANES(RR, JJ)                                                              \
    switch (v4 ? 0 : A->lanes) {                                                           \
        case 0:                                                                            \
            if (sh == 5)                                                                   \
                go(cg_spmv<T, 1, RR, JJ, (sizeof(T) == 4 ? RR > 0 : RR == 0), 5>);         \
            else if (sh == 7)                                                              \
                go(cg_spmv<T, 1, RR, JJ, (sizeof(T) == 4 ? RR > 0 : RR == 0), 7>);         \
            else                                                                           \
                go(cg_spmv<T, 1, RR, JJ, (RR > 0 && sizeof(T) == 4)>);                     \
            break;                                                                         \
        case 1: go(cg_spmv<T, 1, RR, JJ>); break;                                          \
        case 2: go(cg_spmv<T, 2, RR, JJ>); break;                                          \
        case 4: go(cg_spmv<T, 4, RR, JJ>); break;                                          \
        case 8: go(cg_spmv<T, 8, RR, JJ>); break;                                          \
        case 16: go(cg_spmv<T, 16, RR, JJ>); break;                                        \
        default: go(cg_spmv<T, 32, RR, JJ>); break;                                        \
    }
    if (onered() && jm == 2) {
        CG_SPMV_LANES(2, 2)
    } else if (onered()) {
        CG_SPMV_LANES(2, 0)
    } else if (recurrence && jm == 2) {
        CG_SPMV_LANES(1, 2)
    } else if (recurrence) {
        CG_SPMV_LANES(1, 0)
    } else if (jm == 2) {
        CG_SPMV_LANES(0, 2)
    } else {
        CG_SPMV_LANES(0, 0)
    }
#undef CG_SPMV_LANES
}

template <typename T>
void CGEngine<T>::launch_update_kernel()
{
    const int need = c->grid(n / V16<T>::W + 1, kBlock, 16);
    const CSRView<T> V = view_of<T>(*A);
    auto go = [&](auto kern, T* zz) {
        const int g = std::min(need, resident_grid(*c, (const void*)kern, kBlock));
        launch_overlapped(kern, g, c->stream, pdl, n, x, r, zz, P0, P1, q, dinv, ctl, c->red, V);
    };
    const int jm = jmode();
    if (onered()) {
        const int g = std::min(need, resident_grid(*c, (const void*)cg_update_r<T>, kBlock));
        launch_overlapped(cg_update_r<T>, g, c->stream, pdl, n, r, (const T*)q, x,
                          (const T*)P0, ctl);
        return;
    }
    if (lean()) {
        auto gl = [&](auto kern, T* zz) {
            const int g = std::min(need, resident_grid(*c, (const void*)kern, kBlock));
            launch_overlapped(kern, g, c->stream, pdl, n, r, zz, q, dinv, ctl, c->red, V);
        };
        if (jm == 2)
            gl(cg_update_lean<T, 2>, r);
        else if (jm == 1)
            gl(cg_update_lean<T, 1>, z);
        else
            gl(cg_update_lean<T, 0>, r);
        return;
    }
    if (jm == 2)
        go(cg_update<T, 2>, r);
    else if (jm == 1)
        go(cg_update<T, 1>, z);
    else
        go(cg_update<T, 0>, r);
}

template <typename T>
int CGEngine<T>::apply_pending_x()
{
    if (!lean() || !hctl->xpend) return kOk;
    hctl->xpend = 0;
    int e = v_axpy(*c, n, Scal::h(hctl->alpha), (const T*)P0, x);
    if (e) return e;
    return push_ctl();
}

template <typename T>
int CGEngine<T>::launch_iter()
{
    if (!capturing) c->launches += 2;
    launch_spmv_kernel();
    launch_update_kernel();
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int CGEngine<T>::launch_init()
{
    const int g2 = c->grid(n, kBlock);
    ++c->launches;
    const int jm = persistent ? jacobi : jmode();
    if (jm == 2)
        cg_start<T, 2><<<g2, kBlock, 0, c->stream>>>(n, r, r, dinv, ctl, c->red);
    else if (jm == 1)
        cg_start<T, 1><<<g2, kBlock, 0, c->stream>>>(n, r, z, dinv, ctl, c->red);
    else
        cg_start<T, 0><<<g2, kBlock, 0, c->stream>>>(n, r, r, dinv, ctl, c->red);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int CGEngine<T>::launch_resume()
{
    const int g2 = c->grid(n, kBlock);
    ++c->launches;
    const int jm = persistent ? jacobi : jmode();
    if (jm == 2)
        cg_resume<T, 2><<<g2, kBlock, 0, c->stream>>>(n, r, r, dinv, ctl, c->red);
    else if (jm == 1)
        cg_resume<T, 1><<<g2, kBlock, 0, c->stream>>>(n, r, z, dinv, ctl, c->red);
    else
        cg_resume<T, 0><<<g2, kBlock, 0, c->stream>>>(n, r, r, dinv, ctl, c->red);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int CGEngine<T>::push_ctl()
{
    hctl->zc = zc;
    hctl->onered = onered() ? 1 : 0;
    FB_CUDA(cudaMemcpyAsync(ctl, hctl, sizeof(CGCtl), cudaMemcpyHostToDevice, c->stream));
    return kOk;
}

template <typename T>
int CGEngine<T>::pull_ctl()
{
    FB_CUDA(cudaMemcpyAsync(hctl, ctl, sizeof(CGCtl), cudaMemcpyDeviceToHost, c->stream));
    FB_CUDA(cudaStreamSynchronize(c->stream));
    return kOk;
}

template <typename T>
int CGEngine<T>::init(Ctx* ctx, const Mat* M, int jac, const T* dinvv, bool graph)
{
    c = ctx;
    A = M;
    n = M->nrow;
    jacobi = jac;
    dinv = dinvv;
    useGraph = graph;
    const size_t bytes = ((size_t)n + 4) * sizeof(T);
    if (cudaMalloc(&x, bytes) || cudaMalloc(&r, bytes) || cudaMalloc(&q, bytes) ||
        cudaMalloc(&P0, bytes) || cudaMalloc(&P1, bytes) ||
        (jacobi && cudaMalloc(&z, bytes)) || cudaMalloc(&ctl, sizeof(CGCtl)) ||
        cudaMallocHost(&hctl, sizeof(CGCtl)) || cudaMallocHost(&hstatus, sizeof(int))) {
        cudaGetLastError();
        destroy();
        return kErrAlloc;
    }
    if (!jacobi) z = r;
    std::memset(hctl, 0, sizeof(CGCtl));
    hctl->histScale = 1.0;
    FB_CUDA(cudaMemsetAsync(P0, 0, bytes, c->stream));
    FB_CUDA(cudaMemsetAsync(P1, 0, bytes, c->stream));
    if (useGraph) {
        // itersPerGraph iterations + a status read-back, captured once; kernels read every
        // scalar from the control block, so the graph never needs updating.
        cudaGraph_t g;
        FB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        capturing = true;
        for (int i = 0; i < itersPerGraph; ++i) launch_iter();
        capturing = false;
        cudaMemcpyAsync(hstatus, &ctl->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
        FB_CUDA(cudaStreamEndCapture(c->stream, &g));
        FB_CUDA(cudaGraphInstantiate(&gexec, g, 0));
        cudaGraphDestroy(g);
    }
    if (wantPersistent && wantCluster) {
        // the vectors in distributed shared memory: 16 (else 8) blocks of 2^k rows each
        const void* fd = jacobi ? (const void*)cg_dsmem<T, 1> : (const void*)cg_dsmem<T, 0>;
        cudaFuncSetAttribute(fd, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaGetLastError();
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev);
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, fd) != cudaSuccess) {
            cudaGetLastError();
            optin = 0;
        }
        for (int cs : {16, 8}) {
            int k = 0;
            while (((size_t)cs << k) < (size_t)n) ++k;
            const size_t bytes = (size_t)kDsVecs * ((size_t)1 << k) * sizeof(T);
            if (bytes + fa.sharedSizeBytes > (size_t)optin) continue;
            if (((size_t)1 << k) > (size_t)kDsRows<T> * kCBlock) continue;
            if (cudaFuncSetAttribute(fd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bytes) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)cs);
            cfg.blockDim = dim3(kCBlock);
            cfg.dynamicSmemBytes = bytes;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = (unsigned)cs;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int nc = 0;
            if (cudaOccupancyMaxActiveClusters(&nc, fd, &cfg) == cudaSuccess && nc >= 1) {
                cgrid = cs;
                dshift = k;
                dsBytes = bytes;
                dsmem = cluster = persistent = true;
                return kOk;
            }
            cudaGetLastError();
        }
    }
    if (wantPersistent && wantCluster) {
        // one cluster of 16 blocks (8 if the device refuses the non-portable size)
        const void* fn = jacobi ? (const void*)cg_persistent<T, 1, true>
                                : (const void*)cg_persistent<T, 0, true>;
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaGetLastError();
        for (int cs : {16, 8}) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)cs);
            cfg.blockDim = dim3(kCBlock);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = (unsigned)cs;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int nc = 0;
            if (cudaOccupancyMaxActiveClusters(&nc, fn, &cfg) == cudaSuccess && nc >= 1) {
                cgrid = cs;
                break;
            }
            cudaGetLastError();
        }
        if (cgrid > 0) {
            // the control flow needs no barrier state, but the kernel takes the pointer
            if (cudaMalloc(&bar, sizeof(GridBar)) != cudaSuccess) {
                cudaGetLastError();
                return kErrAlloc;
            }
            FB_CUDA(cudaMemsetAsync(bar, 0, sizeof(GridBar), c->stream));
            cluster = persistent = true;
            return kOk;
        }
    }
    if (wantPersistent) {
        // one cooperative launch needs every block resident: size the grid from occupancy
        int coop = 0, nb = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->dev);
        if (jacobi)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, cg_persistent<T, 1>, kPBlock, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, cg_persistent<T, 0>, kPBlock, 0);
        cudaGetLastError();
        if (nb > 4) nb = 4;
        pgrid = nb * c->nsm;
        if (pgrid > kMaxGrid) pgrid = kMaxGrid;
        if (coop && nb > 0) {
            if (cudaMalloc(&bar, sizeof(GridBar)) != cudaSuccess) {
                cudaGetLastError();
                return kErrAlloc;
            }
            FB_CUDA(cudaMemsetAsync(bar, 0, sizeof(GridBar), c->stream));
            persistent = true;
        }
    }
    return kOk;
}

// One cooperative launch that iterates until the control block leaves kRun or iterCap
// iterations have run. A barrier time-out (bar->error) is reported as a CUDA error.
template <typename T>
int CGEngine<T>::run_persistent(unsigned iterCap)
{
    CSRView<T> V = view_of<T>(*A);
    T* zz = jacobi ? z : r;
    Scratch s = c->red;
    if (dsmem) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)cgrid);
        cfg.blockDim = dim3(kCBlock);
        cfg.dynamicSmemBytes = dsBytes;
        cfg.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)cgrid;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (jacobi)
            FB_CUDA(cudaLaunchKernelEx(&cfg, cg_dsmem<T, 1>, V, x, r, zz, P0, P1, q, dinv, ctl,
                                       iterCap, dshift));
        else
            FB_CUDA(cudaLaunchKernelEx(&cfg, cg_dsmem<T, 0>, V, x, r, zz, P0, P1, q, dinv, ctl,
                                       iterCap, dshift));
        FB_CUDA(cudaStreamSynchronize(c->stream));
        return kOk;
    }
    if (cluster) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)cgrid);
        cfg.blockDim = dim3(kCBlock);
        cfg.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)cgrid;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (jacobi)
            FB_CUDA(cudaLaunchKernelEx(&cfg, cg_persistent<T, 1, true>, V, x, r, zz, P0, P1, q,
                                       dinv, ctl, s, bar, iterCap));
        else
            FB_CUDA(cudaLaunchKernelEx(&cfg, cg_persistent<T, 0, true>, V, x, r, zz, P0, P1, q,
                                       dinv, ctl, s, bar, iterCap));
        FB_CUDA(cudaStreamSynchronize(c->stream));
        return kOk;
    }
    void* args[] = {&V, &x, &r, &zz, &P0, &P1, &q, (void*)&dinv, &ctl, &s, &bar, &iterCap};
    const void* fn = jacobi ? (const void*)cg_persistent<T, 1> : (const void*)cg_persistent<T, 0>;
    FB_CUDA(cudaMemcpyAsync(&bar->limit, &barLimit, sizeof(unsigned), cudaMemcpyHostToDevice,
                            c->stream));
    FB_CUDA(cudaLaunchCooperativeKernel(fn, pgrid, kPBlock, args, 0, c->stream));
    GridBar hb;
    FB_CUDA(cudaMemcpyAsync(&hb, bar, sizeof(GridBar), cudaMemcpyDeviceToHost, c->stream));
    FB_CUDA(cudaStreamSynchronize(c->stream));
    if (hb.error) {
        // every block has left (the flag releases the others); reset for the next launch
        cudaMemsetAsync(bar, 0, sizeof(GridBar), c->stream);
        cudaStreamSynchronize(c->stream);
        return kErrCuda;
    }
    return kOk;
}

template <typename T>
void CGEngine<T>::destroy()
{
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    cudaFree(x);
    cudaFree(r);
    cudaFree(q);
    cudaFree(P0);
    cudaFree(P1);
    if (jacobi) cudaFree(z);
    cudaFree(ctl);
    cudaFree(bar);
    bar = nullptr;
    persistent = cluster = dsmem = false;
    cgrid = 0;
    if (hctl) cudaFreeHost(hctl);
    if (hstatus) cudaFreeHost(hstatus);
    x = r = z = q = P0 = P1 = nullptr;
    ctl = nullptr;
    hctl = nullptr;
    hstatus = nullptr;
}

// Keeps two graph launches in flight; after each completes, its status word says whether
// to go on. Overshoot after the end is a few no-op kernels (each checks status first).
template <typename T>
int CGEngine<T>::run(unsigned* launches)
{
    if (persistent) {
        const int e = run_persistent(0xffffffffu);
        if (launches) *launches += 1;
        return e;
    }
    if (!useGraph) {
        // plain launches, status polled every itersPerGraph iterations
        for (;;) {
            for (int i = 0; i < itersPerGraph; ++i) {
                int e = launch_iter();
                if (e) return e;
            }
            FB_CUDA(cudaMemcpyAsync(hstatus, &ctl->status, sizeof(int), cudaMemcpyDeviceToHost,
                                    c->stream));
            FB_CUDA(cudaStreamSynchronize(c->stream));
            if (launches) *launches += 2 * itersPerGraph;
            if (*hstatus != kRun && *hstatus != kRefresh) return kOk;
        }
    }
    cudaEvent_t ev[2];
    FB_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    FB_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    *hstatus = kRun;
    int cur = 0;
    FB_CUDA(cudaGraphLaunch(gexec, c->stream));
    FB_CUDA(cudaEventRecord(ev[cur], c->stream));
    int err = kOk;
    for (;;) {
        if (cudaGraphLaunch(gexec, c->stream) != cudaSuccess ||
            cudaEventRecord(ev[cur ^ 1], c->stream) != cudaSuccess) {
            err = kErrCuda;
            break;
        }
        if (launches) *launches += 2 * itersPerGraph;
        if (cudaEventSynchronize(ev[cur]) != cudaSuccess) {
            err = kErrCuda;
            break;
        }
        // hstatus was written by the graph that ev[cur] follows (stream order)
        if (*hstatus != kRun && *hstatus != kRefresh) break;
        cur ^= 1;
    }
    if (launches) *launches += 2 * itersPerGraph;
    cudaStreamSynchronize(c->stream);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return err;
}

// Times each fused kernel alone: reps launches of cg_spmv, then reps of cg_update, each
// bracketed by events on the engine's stream, with the control block in bench mode.
template <typename T>
int CGEngine<T>::time_kernels(unsigned reps, int flushL2, double* ms)
{
    std::memset(hctl, 0, sizeof(CGCtl));
    hctl->status = kRun;
    hctl->bench = 1;
    hctl->pmode = 1;
    hctl->beta = 0.5;
    hctl->alpha = 1e-3;
    hctl->histScale = 1.0;
    int e = push_ctl();
    if (e) return e;
    auto spmv = [&]() {
        launch_spmv_kernel();
        return (int)kOk;
    };
    auto update = [&]() {
        launch_update_kernel();
        return (int)kOk;
    };
    for (int w = 0; w < 3; ++w) {
        spmv();
        update();
    }
    if ((e = time_launches(*c, reps, flushL2, spmv, &ms[0])) ||
        (e = time_launches(*c, reps, flushL2, update, &ms[1])))
        return e;
    ms[2] = 0.0;
    if (persistent) {
        // the persistent kernel, reps iterations in one launch (bench mode: no control flow)
        if ((e = push_ctl())) return e;
        run_persistent(2);
        if ((e = push_ctl())) return e;
        auto all = [&]() { return run_persistent(reps); };
        if ((e = time_launches(*c, 1, flushL2, all, &ms[2]))) return e;
        ms[2] /= reps;
    }
    hctl->bench = 0;
    hctl->status = kDone;
    e = push_ctl();
    if (e) return e;
    FB_CUDA(cudaStreamSynchronize(c->stream));
    FB_CUDA(cudaGetLastError());
    return kOk;
}

template struct CGEngine<double>;
template struct CGEngine<float>;

// ---- mixed-precision helpers -----------------------------------------------------------

__global__ void k_convert_scaled(uint32_t n, const double* __restrict__ src, double inv,
                                 float* __restrict__ dst)
{
    GRID_STRIDE(i, n) dst[i] = (float)(src[i] * inv);
}

__global__ void k_update_from32(uint32_t n, double scale, const float* __restrict__ e,
                                double* __restrict__ x)
{
    GRID_STRIDE(i, n) x[i] = fma(scale, (double)e[i], x[i]);
}

__global__ void k_set32(uint32_t n, float* __restrict__ x)
{
    GRID_STRIDE(i, n) x[i] = 0.0f;
}

__global__ void k_to32(uint32_t n, const double* __restrict__ s, float* __restrict__ d)
{
    GRID_STRIDE(i, n) d[i] = (float)s[i];
}

int convert_scaled(Ctx& c, uint32_t n, const double* src, double inv, float* dst)
{
    ++c.launches;
    k_convert_scaled<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(n, src, inv, dst);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

int update_from32(Ctx& c, uint32_t n, double scale, const float* e, double* x)
{
    ++c.launches;
    k_update_from32<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(n, scale, e, x);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

int set32(Ctx& c, uint32_t n, float* x)
{
    ++c.launches;
    k_set32<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(n, x);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

int to32(Ctx& c, uint32_t n, const double* s, float* d)
{
    ++c.launches;
    k_to32<<<c.grid(n, kBlock), kBlock, 0, c.stream>>>(n, s, d);
    FB_CUDA(cudaGetLastError());
    return kOk;
}

} // namespace fb
