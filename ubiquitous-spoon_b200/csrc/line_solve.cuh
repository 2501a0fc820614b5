// Line solves of the wall-normal band systems, one GPU thread per line
// (a column of a field, or one part of a spectral column): the band rows of
// an implicit z solve, the wall closures that fold the ghost rows out of it
// and recover them afterwards, and the tridiagonal / heptadiagonal
// recurrences.  Shared by the reference step functions (steps.cu) and the
// fully implicit scheme of the engine (kernels_channel.cu).
//
// Scratch for nl lines is stored [k][line] (one array per quantity), so
// that consecutive threads touch consecutive addresses.
#pragma once

#include "closures.h"
#include <cuda_runtime.h>

namespace lines {

namespace closure = cf::closure;


// The fourth-order coefficients a1, a2, b1, b2 (fourth.c:3-6) in use.
struct Coef {
    double a1, a2, b1, b2;
};

struct Lines {
    double *a, *b, *c, *d, *e, *f, *g, *r, *x;   // band rows, right-hand side, solution
    double *p, *q, *s;                           // factorisation work (heptdag p, q, r / tridag gam)
    long long nl;                                // number of lines
    int* err;                                    // set to 1 on a zero pivot (may be null)
};

// Element k of quantity v on line l.
#define LN(v, k) (L.v[(long long) (k) * L.nl + l])
#define LN_FAIL() do { if (L.err) *L.err = 1; return; } while (0)

// tridag.c:4-26 on rows off .. off+n-1 of line l (gam in p).
__device__ inline void line_tridag(const Lines& L, long long l, int off, int n)
{
    double bet = LN(b, off);
    if (bet == 0.0) LN_FAIL();
    LN(x, off) = LN(r, off) / bet;
    for (int j = 1; j < n; j++) {
        const int k = off + j;
        LN(p, k) = LN(c, k - 1) / bet;
        bet = LN(b, k) - LN(a, k) * LN(p, k);
        if (bet == 0.0) LN_FAIL();
        LN(x, k) = (LN(r, k) - LN(a, k) * LN(x, k - 1)) / bet;
    }
    for (int j = n - 2; j >= 0; j--) {
        const int k = off + j;
        LN(x, k) -= LN(p, k + 1) * LN(x, k + 1);
    }
}

// heptdag.c:5-61 on rows off .. off+n-1 of line l: h = r, result in x (which
// holds s until the back substitution overwrites it); p, q, s hold p, q, r.
__device__ inline void line_heptdag(const Lines& L, long long l, int off, int n)
{
    auto A = [&](int i) { return LN(a, off + i); };
    auto B = [&](int i) { return LN(b, off + i); };
    auto C = [&](int i) { return LN(c, off + i); };
    auto D = [&](int i) { return LN(d, off + i); };
    auto E = [&](int i) { return LN(e, off + i); };
    auto F = [&](int i) { return LN(f, off + i); };
    auto Gq = [&](int i) { return LN(g, off + i); };
    auto H = [&](int i) { return LN(r, off + i); };
    auto P = [&](int i) -> double& { return LN(p, off + i); };
    auto Q = [&](int i) -> double& { return LN(q, off + i); };
    auto R = [&](int i) -> double& { return LN(s, off + i); };
    auto S = [&](int i) -> double& { return LN(x, off + i); };
    double den = D(0);
    if (den == 0.0) LN_FAIL();
    P(0) = E(0) / den;
    Q(0) = F(0) / den;
    R(0) = Gq(0) / den;
    S(0) = H(0) / den;
    den = D(1) - C(1) * P(0);
    if (den == 0.0) LN_FAIL();
    P(1) = (E(1) - C(1) * Q(0)) / den;
    Q(1) = (F(1) - C(1) * R(0)) / den;
    R(1) = (Gq(1)) / den;
    S(1) = (H(1) - C(1) * S(0)) / den;
    double bet = C(2) - B(2) * P(0);
    den = D(2) - B(2) * Q(0) - bet * P(1);
    if (den == 0.0) LN_FAIL();
    P(2) = (E(2) - B(2) * R(0) - bet * Q(1)) / den;
    Q(2) = (F(2) - bet * R(1)) / den;
    R(2) = (Gq(2)) / den;
    S(2) = (H(2) - B(2) * S(0) - bet * S(1)) / den;
    for (int i = 3; i < n; i++) {
        const double alp = B(i) - A(i) * P(i - 3);
        bet = C(i) - A(i) * Q(i - 3) - alp * P(i - 2);
        den = D(i) - A(i) * R(i - 3) - alp * Q(i - 2) - bet * P(i - 1);
        if (den == 0.0) LN_FAIL();
        P(i) = (E(i) - alp * R(i - 2) - bet * Q(i - 1)) / den;
        Q(i) = (F(i) - bet * R(i - 1)) / den;
        R(i) = (Gq(i)) / den;
        S(i) = (H(i) - A(i) * S(i - 3) - alp * S(i - 2) - bet * S(i - 1)) / den;
    }
    // x aliases s: each x(i) overwrites s(i) after s(i+1..i+3) became x
    S(n - 2) = S(n - 2) - P(n - 2) * S(n - 1);
    S(n - 3) = S(n - 3) - P(n - 3) * S(n - 2) - Q(n - 3) * S(n - 1);
    for (int i = n - 4; i >= 0; i--) S(i) = S(i) - P(i) * S(i + 1) - Q(i) * S(i + 2) - R(i) * S(i + 3);
}

// ================================================ wall closures of the line solves
//
// The closures themselves (stencil, reduce, fill; cell-centred fields and
// the pressure, face fields) are in closures.h, shared with the engine's
// host factorisations; here they run over one line of the [k][line] band
// storage.  k is the first ghost row below (bot) or above (top) the interior.

struct Rows {
    const Lines& L;
    long long l;
    CF_HD double& a(int k) const { return L.a[(long long) k * L.nl + l]; }
    CF_HD double& b(int k) const { return L.b[(long long) k * L.nl + l]; }
    CF_HD double& c(int k) const { return L.c[(long long) k * L.nl + l]; }
    CF_HD double& d(int k) const { return L.d[(long long) k * L.nl + l]; }
    CF_HD double& e(int k) const { return L.e[(long long) k * L.nl + l]; }
    CF_HD double& f(int k) const { return L.f[(long long) k * L.nl + l]; }
    CF_HD double& g(int k) const { return L.g[(long long) k * L.nl + l]; }
    CF_HD double& r(int k) const { return L.r[(long long) k * L.nl + l]; }
    CF_HD double& x(int k) const { return L.x[(long long) k * L.nl + l]; }
    // set row k to (a..g | rhs)
    __device__ inline void set(int k, double va, double vb, double vc, double vd, double ve, double vf, double vg,
                        double vr) const
    {
        closure::set_row(*this, k, va, vb, vc, vd, ve, vf, vg, vr);
    }
};

__device__ inline void cell_stencil_bot2(const Rows& R, const double* dz, int k, double bc, bool neumann)
{
    closure::cell_stencil_bot2(R, dz, k, bc, neumann);
}
__device__ inline void cell_stencil_top2(const Rows& R, const double* dz, int k, double bc, bool neumann)
{
    closure::cell_stencil_top2(R, dz, k, bc, neumann);
}
__device__ inline void cell_reduce_bot2(const Rows& R, int k) { closure::cell_reduce_bot2(R, k); }
__device__ inline void cell_reduce_top2(const Rows& R, int k) { closure::cell_reduce_top2(R, k); }
__device__ inline void cell_fill_bot2(const Rows& R, int k) { closure::cell_fill_bot2(R, k); }
__device__ inline void cell_fill_top2(const Rows& R, int k) { closure::cell_fill_top2(R, k); }
__device__ inline void cell_stencil_bot4(const Rows& R, const double* dz, int k, double bc, bool neumann, const Coef& cf)
{
    closure::cell_stencil_bot4(R, dz, k, bc, neumann, cf.a1, cf.a2);
}
__device__ inline void cell_stencil_top4(const Rows& R, const double* dz, int k, double bc, bool neumann, const Coef& cf)
{
    closure::cell_stencil_top4(R, dz, k, bc, neumann, cf.a1, cf.a2);
}
__device__ inline void cell_reduce_bot4(const Rows& R, int k) { closure::cell_reduce_bot4(R, k); }
__device__ inline void cell_reduce_top4(const Rows& R, int k) { closure::cell_reduce_top4(R, k); }
__device__ inline void cell_fill_bot4(const Rows& R, int k) { closure::cell_fill_bot4(R, k); }
__device__ inline void cell_fill_top4(const Rows& R, int k) { closure::cell_fill_top4(R, k); }

__device__ inline void face_stencil2(const Rows& R, int k, double bc) { closure::face_stencil2(R, k, bc); }
__device__ inline void face_reduce_bot2(const Rows& R, int k) { closure::face_reduce_bot2(R, k); }
__device__ inline void face_reduce_top2(const Rows& R, int k) { closure::face_reduce_top2(R, k); }
__device__ inline void face_fill2(const Rows& R, int k) { closure::face_fill2(R, k); }
__device__ inline void face_stencil_bot4(const Rows& R, const double* dz, int k, double bc, const Coef& cf)
{
    closure::face_stencil_bot4(R, dz, k, bc, cf.a1, cf.a2);
}
__device__ inline void face_stencil_top4(const Rows& R, const double* dz, int k, double bc, const Coef& cf)
{
    closure::face_stencil_top4(R, dz, k, bc, cf.a1, cf.a2);
}
__device__ inline void face_reduce_bot4(const Rows& R, int k) { closure::face_reduce_bot4(R, k); }
__device__ inline void face_reduce_top4(const Rows& R, int k) { closure::face_reduce_top4(R, k); }
__device__ inline void face_fill_bot4(const Rows& R, int k) { closure::face_fill_bot4(R, k); }
__device__ inline void face_fill_top4(const Rows& R, int k) { closure::face_fill_top4(R, k); }

// ============================================================ band rows and solve
//
// The band of an implicit z solve, row k (interior).  Cell fields and the
// pressure use the metric denominators dz[k] times the half-cell spacings,
// face fields dzp1h times the cell widths (diffuseu.c:173-283,
// diffusew.c:175-287, pressure.c:293-443).  t is nudt or dt; the spectral
// forms subtract the wavenumber terms lamx, lamy; all but the pressure add
// the volume dvol on the diagonal.

struct BandArgs {
    int order;
    bool face;           // w: face metrics
    bool spectral;       // subtract lamx, lamy terms
    bool plus_dvol;      // + dvol on the diagonal
    double t, dx, dy;
    bool xy_volume;      // dvol includes dx*dy
};

__device__ inline void band_row(const Rows& R, const double* dz, int k, const BandArgs& A, const Coef& cf, double lamx,
                         double lamy, double& dvol_out)
{
    const double t = A.t;
    double dvol, Dm3 = 0, Dp3 = 0, Dm1, Dp1;
    if (!A.face) {
        const double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
        const double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
        dvol = A.xy_volume ? A.dx * A.dy * dz[k] : dz[k];
        Dm1 = dzm1h * dz[k];
        Dp1 = dzp1h * dz[k];
        if (A.order == 4) {
            Dm3 = 0.5 * (dz[k - 2] + dz[k - 1]) * dz[k];
            Dp3 = 0.5 * (dz[k + 2] + dz[k + 1]) * dz[k];
        }
    } else {
        const double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
        dvol = A.xy_volume ? A.dx * A.dy * dzp1h : dzp1h;
        Dm1 = dz[k] * dzp1h;
        Dp1 = dz[k + 1] * dzp1h;
        if (A.order == 4) {
            Dm3 = dz[k - 1] * dzp1h;
            Dp3 = dz[k + 2] * dzp1h;
        }
    }
    double diag;
    if (A.order == 2) {
        R.a(k) = +dvol * t / Dm1;
        R.c(k) = +dvol * t / Dp1;
        diag = -dvol * t / Dm1 - dvol * t / Dp1;
    } else {
        const double A1 = cf.a1, A2 = cf.a2;
        R.a(k) = +A2 * A2 * dvol * t / Dm3;
        R.g(k) = +A2 * A2 * dvol * t / Dp3;
        R.b(k) = +A1 * A2 * dvol * t / Dm1 + A1 * A2 * dvol * t / Dm3;
        R.f(k) = +A1 * A2 * dvol * t / Dp1 + A1 * A2 * dvol * t / Dp3;
        R.c(k) = -A1 * A2 * dvol * t / Dp1 - A1 * A2 * dvol * t / Dm3 + A1 * A1 * dvol * t / Dm1;
        R.e(k) = -A1 * A2 * dvol * t / Dm1 - A1 * A2 * dvol * t / Dp3 + A1 * A1 * dvol * t / Dp1;
        diag = -A2 * A2 * dvol * t / Dm3 - A2 * A2 * dvol * t / Dp3 - A1 * A1 * dvol * t / Dm1 - A1 * A1 * dvol * t / Dp1;
    }
    if (A.spectral) diag = diag - lamx * dvol * t / (A.dx * A.dx) - lamy * dvol * t / (A.dy * A.dy);
    if (A.plus_dvol) diag = diag + dvol;
    if (A.order == 2) R.b(k) = diag;
    else R.d(k) = diag;
    dvol_out = dvol;
}

// Closure kinds: cell fields / pressure with Neumann or Dirichlet walls, face fields.
struct WallSpec {
    bool face;
    bool neumann_bot, neumann_top;   // cell kind only
    double bc_bot, bc_top;
};

// One column: band rows (interior), walls, reduction, solve of n rows, ghost
// fill.  r must already hold the interior right-hand side.
__device__ inline void solve_line(const Rows& R, const Lines& L, long long l, const double* dz, int g, int n2, int order,
                           const WallSpec& W, const Coef& cf)
{
    const int kb = g - 1;
    const int kt = W.face ? n2 - g - 1 : n2 - g;
    const int n = W.face ? n2 - 2 * g - 1 : n2 - 2 * g;
    if (order == 2) {
        if (W.face) {
            face_stencil2(R, kb, W.bc_bot);
            face_stencil2(R, kt, W.bc_top);
            face_reduce_bot2(R, kb);
            face_reduce_top2(R, kt);
        } else {
            cell_stencil_bot2(R, dz, kb, W.bc_bot, W.neumann_bot);
            cell_stencil_top2(R, dz, kt, W.bc_top, W.neumann_top);
            cell_reduce_bot2(R, kb);
            cell_reduce_top2(R, kt);
        }
        line_tridag(L, l, g, n);
        if (W.face) {
            face_fill2(R, kb);
            face_fill2(R, kt);
        } else {
            cell_fill_bot2(R, kb);
            cell_fill_top2(R, kt);
        }
    } else {
        if (W.face) {
            face_stencil_bot4(R, dz, kb, W.bc_bot, cf);
            face_stencil_top4(R, dz, kt, W.bc_top, cf);
            face_reduce_bot4(R, kb);
            face_reduce_top4(R, kt);
        } else {
            cell_stencil_bot4(R, dz, kb, W.bc_bot, W.neumann_bot, cf);
            cell_stencil_top4(R, dz, kt, W.bc_top, W.neumann_top, cf);
            cell_reduce_bot4(R, kb);
            cell_reduce_top4(R, kt);
        }
        line_heptdag(L, l, g, n);
        if (W.face) {
            face_fill_bot4(R, kb);
            face_fill_top4(R, kt);
        } else {
            cell_fill_bot4(R, kb);
            cell_fill_top4(R, kt);
        }
    }
}

}  // namespace lines
