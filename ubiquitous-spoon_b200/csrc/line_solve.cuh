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

#include <cuda_runtime.h>

namespace lines {

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
// A closure adds the wall rows of a column's band system (stencil), folds
// them out of the first interior rows (reduce) and recovers the ghost values
// from the solution (fill).  Cell-centred fields and the pressure share one
// set (diffuseu.c:572-940, pressure.c:505-769: Neumann or Dirichlet at the
// wall); face fields have their own (diffusew.c:555-905: the wall value is a
// Dirichlet condition on the face itself).  k is the first ghost row below
// (bot) or above (top) the interior.

struct Rows {
    const Lines& L;
    long long l;
    __device__ double& a(int k) const { return L.a[(long long) k * L.nl + l]; }
    __device__ double& b(int k) const { return L.b[(long long) k * L.nl + l]; }
    __device__ double& c(int k) const { return L.c[(long long) k * L.nl + l]; }
    __device__ double& d(int k) const { return L.d[(long long) k * L.nl + l]; }
    __device__ double& e(int k) const { return L.e[(long long) k * L.nl + l]; }
    __device__ double& f(int k) const { return L.f[(long long) k * L.nl + l]; }
    __device__ double& g(int k) const { return L.g[(long long) k * L.nl + l]; }
    __device__ double& r(int k) const { return L.r[(long long) k * L.nl + l]; }
    __device__ double& x(int k) const { return L.x[(long long) k * L.nl + l]; }
    // set row k to (a..g | rhs)
    __device__ inline void set(int k, double va, double vb, double vc, double vd, double ve, double vf, double vg,
                        double vr) const
    {
        a(k) = va; b(k) = vb; c(k) = vc; d(k) = vd; e(k) = ve; f(k) = vf; g(k) = vg; r(k) = vr;
    }
};

// ---- cell fields and pressure, second order (three-band rows a, b, c)
__device__ inline void cell_stencil_bot2(const Rows& R, const double* dz, int k, double bc, bool neumann)
{
    const double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
    R.a(k) = 0.0;
    if (neumann) { R.b(k) = -1.0 / dzp1h; R.c(k) = +1.0 / dzp1h; }
    else { R.b(k) = 0.5; R.c(k) = 0.5; }
    R.r(k) = bc;
}
__device__ inline void cell_stencil_top2(const Rows& R, const double* dz, int k, double bc, bool neumann)
{
    const double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
    if (neumann) { R.a(k) = -1.0 / dzm1h; R.b(k) = +1.0 / dzm1h; }
    else { R.a(k) = 0.5; R.b(k) = 0.5; }
    R.c(k) = 0.0;
    R.r(k) = bc;
}
__device__ inline void cell_reduce_bot2(const Rows& R, int k)
{
    const double fac = R.a(k + 1) / R.b(k);
    R.a(k + 1) -= R.b(k) * fac;
    R.b(k + 1) -= R.c(k) * fac;
    R.r(k + 1) -= R.r(k) * fac;
}
__device__ inline void cell_reduce_top2(const Rows& R, int k)
{
    const double fac = R.c(k - 1) / R.b(k);
    R.c(k - 1) -= R.b(k) * fac;
    R.b(k - 1) -= R.a(k) * fac;
    R.r(k - 1) -= R.r(k) * fac;
}
__device__ inline void cell_fill_bot2(const Rows& R, int k) { R.x(k) = (R.c(k) * R.x(k + 1) - R.r(k)) / -R.b(k); }
__device__ inline void cell_fill_top2(const Rows& R, int k) { R.x(k) = (R.a(k) * R.x(k - 1) - R.r(k)) / -R.b(k); }

// ---- cell fields and pressure, fourth order (seven-band rows a..g)
__device__ inline void cell_stencil_bot4(const Rows& R, const double* dz, int k, double bc, bool neumann, const Coef& cf)
{
    const double A1 = cf.a1, A2 = cf.a2;
    const double dzp3h = 0.5 * (dz[k + 2] + dz[k + 1]);
    const double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
    const double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
    // row k: the fourth-order second difference across the wall vanishes
    R.set(k, 0.0, -A2 / dzm1h, -A1 / dzm1h - 2.0 * -A2 / dzp1h, +A1 / dzm1h - 2.0 * -A1 / dzp1h - A2 / dzp3h,
          +A2 / dzm1h - 2.0 * +A1 / dzp1h - A1 / dzp3h, -2.0 * +A2 / dzp1h + A1 / dzp3h, +A2 / dzp3h, 0.0);
    // row k-1: the boundary condition
    if (neumann) R.set(k - 1, 0.0, 0.0, 0.0, -A2 / dzp1h, -A1 / dzp1h, +A1 / dzp1h, +A2 / dzp1h, bc);
    else R.set(k - 1, 0.0, 0.0, 0.0, 0.5 * A2, 0.5 * (A1 + 2.0 * A2), 0.5 * (A1 + 2.0 * A2), 0.5 * A2, bc);
    // row k-2: even extension of the outermost ghost
    R.set(k - 2, 0.0, 0.0, 0.0, 0.0, 0.0, -1.0, +1.0, 0.0);
}
__device__ inline void cell_stencil_top4(const Rows& R, const double* dz, int k, double bc, bool neumann, const Coef& cf)
{
    const double A1 = cf.a1, A2 = cf.a2;
    const double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
    const double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
    const double dzm3h = 0.5 * (dz[k - 2] + dz[k - 1]);
    R.set(k, -A2 / dzm3h, -A1 / dzm3h - 2.0 * -A2 / dzm1h, +A1 / dzm3h - 2.0 * -A1 / dzm1h - A2 / dzp1h,
          +A2 / dzm3h - 2.0 * +A1 / dzm1h - A1 / dzp1h, -2.0 * +A2 / dzm1h + A1 / dzp1h, +A2 / dzp1h, 0.0, 0.0);
    if (neumann) R.set(k + 1, -A2 / dzm1h, -A1 / dzm1h, +A1 / dzm1h, +A2 / dzm1h, 0.0, 0.0, 0.0, bc);
    else R.set(k + 1, 0.5 * A2, 0.5 * (A1 + 2.0 * A2), 0.5 * (A1 + 2.0 * A2), 0.5 * A2, 0.0, 0.0, 0.0, bc);
    R.set(k + 2, -1.0, +1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
}
// Fold the three wall rows (pivots b(k), d(k-1), f(k-2)) out of rows k+1..k+3.
__device__ inline void cell_reduce_bot4(const Rows& R, int k)
{
    double fac = R.a(k + 1) / R.b(k);
    R.a(k + 1) -= R.b(k) * fac; R.b(k + 1) -= R.c(k) * fac; R.c(k + 1) -= R.d(k) * fac;
    R.d(k + 1) -= R.e(k) * fac; R.e(k + 1) -= R.f(k) * fac; R.f(k + 1) -= R.g(k) * fac;
    fac = R.b(k + 1) / R.d(k - 1);
    R.b(k + 1) -= R.d(k - 1) * fac; R.c(k + 1) -= R.e(k - 1) * fac; R.d(k + 1) -= R.f(k - 1) * fac;
    R.e(k + 1) -= R.g(k - 1) * fac; R.r(k + 1) -= R.r(k - 1) * fac;
    fac = R.c(k + 1) / R.f(k - 2);
    R.c(k + 1) -= R.f(k - 2) * fac; R.d(k + 1) -= R.g(k - 2) * fac;
    fac = R.a(k + 2) / R.d(k - 1);
    R.a(k + 2) -= R.d(k - 1) * fac; R.b(k + 2) -= R.e(k - 1) * fac; R.c(k + 2) -= R.f(k - 1) * fac;
    R.d(k + 2) -= R.g(k - 1) * fac; R.r(k + 2) -= R.r(k - 1) * fac;
    fac = R.b(k + 2) / R.f(k - 2);
    R.b(k + 2) -= R.f(k - 2) * fac; R.c(k + 2) -= R.g(k - 2) * fac;
    fac = R.a(k + 3) / R.f(k - 2);
    R.a(k + 3) -= R.f(k - 2) * fac; R.b(k + 3) -= R.g(k - 2) * fac;
}
// Fold the wall rows (pivots f(k), d(k+1), b(k+2)) out of rows k-1..k-3.
__device__ inline void cell_reduce_top4(const Rows& R, int k)
{
    double fac = R.g(k - 1) / R.f(k);
    R.g(k - 1) -= R.f(k) * fac; R.f(k - 1) -= R.e(k) * fac; R.e(k - 1) -= R.d(k) * fac;
    R.d(k - 1) -= R.c(k) * fac; R.c(k - 1) -= R.b(k) * fac; R.b(k - 1) -= R.a(k) * fac;
    fac = R.f(k - 1) / R.d(k + 1);
    R.f(k - 1) -= R.d(k + 1) * fac; R.e(k - 1) -= R.c(k + 1) * fac; R.d(k - 1) -= R.b(k + 1) * fac;
    R.c(k - 1) -= R.a(k + 1) * fac; R.r(k - 1) -= R.r(k + 1) * fac;
    fac = R.e(k - 1) / R.b(k + 2);
    R.e(k - 1) -= R.b(k + 2) * fac; R.d(k - 1) -= R.a(k + 2) * fac;
    fac = R.g(k - 2) / R.d(k + 1);
    R.g(k - 2) -= R.d(k + 1) * fac; R.f(k - 2) -= R.c(k + 1) * fac; R.e(k - 2) -= R.b(k + 1) * fac;
    R.d(k - 2) -= R.a(k + 1) * fac; R.r(k - 2) -= R.r(k + 1) * fac;
    fac = R.f(k - 2) / R.b(k + 2);
    R.f(k - 2) -= R.b(k + 2) * fac; R.e(k - 2) -= R.a(k + 2) * fac;
    fac = R.g(k - 3) / R.b(k + 2);
    R.g(k - 3) -= R.b(k + 2) * fac; R.f(k - 3) -= R.a(k + 2) * fac;
}
__device__ inline void cell_fill_bot4(const Rows& R, int k)
{
    R.x(k) = (R.g(k - 2) * R.x(k + 1)) / -R.f(k - 2);
    R.x(k - 1) = (R.e(k - 1) * R.x(k) + R.f(k - 1) * R.x(k + 1) + R.g(k - 1) * R.x(k + 2) - R.r(k - 1)) / -R.d(k - 1);
    R.x(k - 2) = (R.c(k) * R.x(k - 1) + R.d(k) * R.x(k) + R.e(k) * R.x(k + 1) + R.f(k) * R.x(k + 2)
                  + R.g(k) * R.x(k + 3)) / -R.b(k);
}
__device__ inline void cell_fill_top4(const Rows& R, int k)
{
    R.x(k) = (R.a(k + 2) * R.x(k - 1)) / -R.b(k + 2);
    R.x(k + 1) = (R.a(k + 1) * R.x(k - 2) + R.b(k + 1) * R.x(k - 1) + R.c(k + 1) * R.x(k) - R.r(k + 1)) / -R.d(k + 1);
    R.x(k + 2) = (R.a(k) * R.x(k - 3) + R.b(k) * R.x(k - 2) + R.c(k) * R.x(k - 1) + R.d(k) * R.x(k)
                  + R.e(k) * R.x(k + 1)) / -R.f(k);
}

// ---- face fields (w), second order: the wall face value is the unknown
__device__ inline void face_stencil2(const Rows& R, int k, double bc) { R.a(k) = 0.0; R.b(k) = 1.0; R.c(k) = 0.0; R.r(k) = bc; }
__device__ inline void face_reduce_bot2(const Rows& R, int k)
{
    const double fac = R.a(k + 1) / R.b(k);
    R.a(k + 1) -= R.b(k) * fac;
    R.r(k + 1) -= R.r(k) * fac;
}
__device__ inline void face_reduce_top2(const Rows& R, int k)
{
    const double fac = R.c(k - 1) / R.b(k);
    R.c(k - 1) -= R.b(k) * fac;
    R.r(k - 1) -= R.r(k) * fac;
}
__device__ inline void face_fill2(const Rows& R, int k) { R.x(k) = (-R.r(k)) / -R.b(k); }

// ---- face fields (w), fourth order
__device__ inline void face_stencil_bot4(const Rows& R, const double* dz, int k, double bc, const Coef& cf)
{
    const double A1 = cf.a1, A2 = cf.a2, dzp0 = dz[k], dzp1 = dz[k + 1];
    R.set(k, 0.0, -A2 / dzp0, -A1 / dzp0 + A2 / dzp1, +A1 / dzp0 + A1 / dzp1, +A2 / dzp0 - A1 / dzp1, -A2 / dzp1, 0.0,
          0.0);
    R.set(k - 1, 0.0, 0.0, 0.0, -1.0, +2.0, -1.0, 0.0, 0.0);
    R.set(k - 2, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, bc);
}
__device__ inline void face_stencil_top4(const Rows& R, const double* dz, int k, double bc, const Coef& cf)
{
    const double A1 = cf.a1, A2 = cf.a2, dzp0 = dz[k], dzp1 = dz[k + 1];
    R.set(k, 0.0, -A2 / dzp0, -A1 / dzp0 + A2 / dzp1, +A1 / dzp0 + A1 / dzp1, +A2 / dzp0 - A1 / dzp1, -A2 / dzp1, 0.0,
          0.0);
    R.set(k + 1, 0.0, -1.0, +2.0, -1.0, 0.0, 0.0, 0.0, 0.0);
    R.set(k + 2, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, bc);
}
__device__ inline void face_reduce_bot4(const Rows& R, int k)
{
    double fac = R.a(k + 1) / R.b(k);
    R.a(k + 1) -= R.b(k) * fac; R.b(k + 1) -= R.c(k) * fac; R.c(k + 1) -= R.d(k) * fac;
    R.d(k + 1) -= R.e(k) * fac; R.e(k + 1) -= R.f(k) * fac;
    fac = R.b(k + 1) / R.d(k - 1);
    R.b(k + 1) -= R.d(k - 1) * fac; R.c(k + 1) -= R.e(k - 1) * fac; R.d(k + 1) -= R.f(k - 1) * fac;
    fac = R.c(k + 1) / R.f(k - 2);
    R.c(k + 1) -= R.f(k - 2) * fac; R.r(k + 1) -= R.r(k - 2) * fac;
    fac = R.a(k + 2) / R.d(k - 1);
    R.a(k + 2) -= R.d(k - 1) * fac; R.b(k + 2) -= R.e(k - 1) * fac; R.c(k + 2) -= R.f(k - 1) * fac;
    fac = R.b(k + 2) / R.f(k - 2);
    R.b(k + 2) -= R.f(k - 2) * fac; R.r(k + 2) -= R.r(k - 2) * fac;
    fac = R.a(k + 3) / R.f(k - 2);
    R.a(k + 3) -= R.f(k - 2) * fac; R.r(k + 3) -= R.r(k - 2) * fac;
}
__device__ inline void face_reduce_top4(const Rows& R, int k)
{
    double fac = R.g(k - 1) / R.f(k);
    R.g(k - 1) -= R.f(k) * fac; R.f(k - 1) -= R.e(k) * fac; R.e(k - 1) -= R.d(k) * fac;
    R.d(k - 1) -= R.c(k) * fac; R.c(k - 1) -= R.b(k) * fac;
    fac = R.f(k - 1) / R.d(k + 1);
    R.f(k - 1) -= R.d(k + 1) * fac; R.e(k - 1) -= R.c(k + 1) * fac; R.d(k - 1) -= R.b(k + 1) * fac;
    fac = R.e(k - 1) / R.b(k + 2);
    R.e(k - 1) -= R.b(k + 2) * fac; R.r(k - 1) -= R.r(k + 2) * fac;
    fac = R.g(k - 2) / R.d(k + 1);
    R.g(k - 2) -= R.d(k + 1) * fac; R.f(k - 2) -= R.c(k + 1) * fac; R.e(k - 2) -= R.b(k + 1) * fac;
    fac = R.f(k - 2) / R.b(k + 2);
    R.f(k - 2) -= R.b(k + 2) * fac; R.r(k - 2) -= R.r(k + 2) * fac;
    fac = R.g(k - 3) / R.b(k + 2);
    R.g(k - 3) -= R.b(k + 2) * fac; R.r(k - 3) -= R.r(k + 2) * fac;
}
__device__ inline void face_fill_bot4(const Rows& R, int k)
{
    R.x(k) = (-R.r(k - 2)) / -R.f(k - 2);
    R.x(k - 1) = (R.e(k - 1) * R.x(k) + R.f(k - 1) * R.x(k + 1)) / -R.d(k - 1);
    R.x(k - 2) = (R.c(k) * R.x(k - 1) + R.d(k) * R.x(k) + R.e(k) * R.x(k + 1) + R.f(k) * R.x(k + 2)) / -R.b(k);
}
__device__ inline void face_fill_top4(const Rows& R, int k)
{
    R.x(k) = (-R.r(k + 2)) / -R.b(k + 2);
    R.x(k + 1) = (R.b(k + 1) * R.x(k - 1) + R.c(k + 1) * R.x(k)) / -R.d(k + 1);
    R.x(k + 2) = (R.b(k) * R.x(k - 2) + R.c(k) * R.x(k - 1) + R.d(k) * R.x(k) + R.e(k) * R.x(k + 1)) / -R.f(k);
}

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
