// gmres.cuh -- the device-side Hessenberg least-squares state of GMRES/FGMRES (GMRES.cxx:
// 114-280, FGMRES.cxx:108-271) shared by the Gram-Schmidt variants: the rotated Hessenberg
// hh, the Givens sines and cosines, the right-hand side var, and the Givens step that
// completes one Hessenberg column.
#pragma once

#include "internal.h"
#include "solver.h"

namespace fb {

struct GmLayout {
    double *hh, *hcos, *hsin, *var, *h1, *h2, *out;
    // delayed reorthogonalisation: the Hessenberg before rotation (column j - 1 final once
    // step j has re-orthogonalised its vector, column j tentative), and the coefficients the
    // update pass of step j reads: ca[0..j) and cb[0..j), then cs = {g, 1/t}
    double *hraw, *ca, *cb, *cs;
    size_t  m;
};

// Doubles of the layout for restart length m.
inline size_t gm_layout_size(size_t m)
{
    return (m + 1) * m + (m + 1) + m + (m + 1) + 2 * (m + 1) + 4 + (m + 1) * m + 2 * (m + 1) + 4;
}

inline GmLayout gm_layout(double* gm, size_t m)
{
    GmLayout L;
    L.m = m;
    L.hh = gm;
    L.hcos = L.hh + (m + 1) * m;
    L.hsin = L.hcos + (m + 1);
    L.var = L.hsin + m;
    L.h1 = L.var + (m + 1);
    L.h2 = L.h1 + (m + 1);
    L.out = L.h2 + (m + 1);
    L.hraw = L.out + 4;
    L.ca = L.hraw + (m + 1) * m;
    L.cb = L.ca + (m + 1);
    L.cs = L.cb + (m + 1);
    return L;
}

// Basis vectors a DCGS2 step handles: restart lengths up to this use it.
constexpr int kDcMaxK = 48;

// Hessenberg columns up to this length are staged in shared memory by the Givens kernel.
constexpr int kGmShared = 512;

// GMRES.cxx:168-209 after the Arnoldi step, on one thread: C(count) = t, then the previous
// rotations applied to column c1 in order, the new rotation, the updated right-hand side and
// the residual estimate |var[count]| (out[0]); out[1] = 0 when t is not > SMALL_DBL (the
// reference leaves the restart cycle before rotating). With a control block g: numIter is
// incremented (the top of the step, GMRES.cxx:162), the estimate recorded in the history,
// and the in-cycle stop test of GMRES.cxx:205-209 applied. C(j) is the column entry j, S(j)
// / K(j) the sine / cosine of rotation j and Var(j) entry j of the right-hand side, each a
// reference into shared memory in the callers, as is g: one thread's chain of dependent
// global loads and stores (about 10 L2 round trips) had cost several microseconds a step.
template <typename CF, typename SF, typename KF, typename VF>
__device__ __forceinline__ void gm_givens_serial(const GmLayout& L, int count, int c1, double t,
                                                 CF C, SF S, KF K, VF Var, GmCtl* g)
{
    C(count) = t;
    if (g) {
        g->numIter += 1;
        g->count = count;
    }
    if (!(fabs(t) > kSmallDbl)) {
        L.out[1] = 0.0;
        if (g) g->stop = 1;
        return;
    }
    L.out[1] = 1.0;
    for (int j = 1; j < count; ++j) {
        t = C(j - 1);
        C(j - 1) = S(j - 1) * C(j) + K(j - 1) * t;
        C(j) = -S(j - 1) * t + K(j - 1) * C(j);
    }
    t = C(count) * C(count);
    t += C(c1) * C(c1);
    t = sqrt(t);
    const double gamma = t > kSmallDbl ? t : kSmallDbl;
    const double cs = C(c1) / gamma, sn = C(count) / gamma;
    L.hcos[c1] = cs;
    L.hsin[c1] = sn;
    C(c1) = sn * C(count) + cs * C(c1);
    Var(count) = -sn * Var(c1);
    Var(c1) = cs * Var(c1);
    const double resAbs = fabs(Var(count));
    L.out[0] = resAbs;
    if (g) {
        g->resAbs = resAbs;
        const unsigned k = g->numIter + g->histOffset;
        if (g->hist && k < g->histCap) g->hist[k] = resAbs * g->histScale;
        if ((resAbs < g->absTol || resAbs / g->denAbs < g->relTol) && g->numIter > g->minIter)
            g->stop = 2;
    }
}

template <typename T>
int dc_dots(Ctx& c, uint32_t n, int j, T* V, size_t ld, const T* w, const GmLayout& L, GmCtl* g);
template <typename T>
int dc_update(Ctx& c, uint32_t n, int j, T* V, size_t ld, const T* w, const GmLayout& L,
              const GmCtl* g, bool wlast);
// The dots pass of step j forming the product w = A M u itself (mode 0: A u, 1: A (D u),
// 2: D (A u)) on stencil masks of the fixed 5- or 7-point shape; kErrInputPar when the
// matrix or the vectors do not have that form (the caller then launches the product).
template <typename T>
int dc_dots_apply(Ctx& c, const CSRView<T>& A, int mode, const T* dinv, uint32_t n, int j,
                  T* V, size_t ld, T* w, const GmLayout& L, GmCtl* g);
unsigned tile_timeouts_dcgs2();

} // namespace fb
