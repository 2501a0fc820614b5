// Wall closures of the wall-normal band systems, in one place for the two
// users: the host factorisations of the engine (host_band.cpp) and the
// device step functions (line_solve.cuh, steps.cu).  Both must reproduce the
// reference's closures operation for operation -- the step functions equal
// the reference bit for bit -- so the operation order is the reference's.
//
// A closure adds the wall rows of a column's band system (stencil), folds
// them out of the first interior rows (reduce) and recovers the ghost values
// from the solution (fill).  Cell-centred fields and the pressure share one
// set (diffuseu.c:572-940, pressure.c:446-770: Neumann or Dirichlet at the
// wall); face fields have their own (diffusew.c:555-905: the wall value is a
// Dirichlet condition on the face itself).  k is the first ghost row below
// (bot) or above (top) the interior.
//
// R is the band storage: R.a(k) .. R.g(k), R.r(k) (right-hand side) and
// R.x(k) (solution) return double&.  Second-order systems use a, b, c only.
// The reductions can record the amounts they subtract from the diagonal
// (dsub, optional): the pressure solve keeps the column-independent
// off-diagonal work and adds its per-column diagonal afterwards.
//
// Compiled without floating-point contraction by both users (a contracted
// multiply-add would round once where the reference rounds twice).
#pragma once

#ifdef __CUDACC__
#define CF_HD __host__ __device__
#else
#define CF_HD
#endif

namespace cf {
namespace closure {

template <class R>
CF_HD inline void set_row(const R& B, int k, double va, double vb, double vc, double vd, double ve, double vf,
                          double vg, double vr)
{
    B.a(k) = va; B.b(k) = vb; B.c(k) = vc; B.d(k) = vd; B.e(k) = ve; B.f(k) = vf; B.g(k) = vg; B.r(k) = vr;
}

// ---- cell fields and pressure, second order (three-band rows a, b, c)
// ghost_stencil_bot2 / top2 (diffuseu.c:617-640, pressure.c:446-468)
template <class R>
CF_HD inline void cell_stencil_bot2(const R& B, const double* dz, int k, double bc, bool neumann)
{
    const double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
    B.a(k) = 0.0;
    if (neumann) { B.b(k) = -1.0 / dzp1h; B.c(k) = +1.0 / dzp1h; }
    else { B.b(k) = 0.5; B.c(k) = 0.5; }
    B.r(k) = bc;
}
template <class R>
CF_HD inline void cell_stencil_top2(const R& B, const double* dz, int k, double bc, bool neumann)
{
    const double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
    if (neumann) { B.a(k) = -1.0 / dzm1h; B.b(k) = +1.0 / dzm1h; }
    else { B.a(k) = 0.5; B.b(k) = 0.5; }
    B.c(k) = 0.0;
    B.r(k) = bc;
}
// ghost_reduce_bot2 / top2 (diffuseu.c:643-664)
template <class R>
CF_HD inline void cell_reduce_bot2(const R& B, int k)
{
    const double fac = B.a(k + 1) / B.b(k);
    B.a(k + 1) -= B.b(k) * fac;
    B.b(k + 1) -= B.c(k) * fac;
    B.r(k + 1) -= B.r(k) * fac;
}
template <class R>
CF_HD inline void cell_reduce_top2(const R& B, int k)
{
    const double fac = B.c(k - 1) / B.b(k);
    B.c(k - 1) -= B.b(k) * fac;
    B.b(k - 1) -= B.a(k) * fac;
    B.r(k - 1) -= B.r(k) * fac;
}
// ghost_fill_bot2 / top2 (diffuseu.c:667-682)
template <class R>
CF_HD inline void cell_fill_bot2(const R& B, int k) { B.x(k) = (B.c(k) * B.x(k + 1) - B.r(k)) / -B.b(k); }
template <class R>
CF_HD inline void cell_fill_top2(const R& B, int k) { B.x(k) = (B.a(k) * B.x(k - 1) - B.r(k)) / -B.b(k); }

// ---- cell fields and pressure, fourth order (seven-band rows a..g)
// ghost_stencil_bot4 / top4 (diffuseu.c:703-802, pressure.c:617-700)
template <class R>
CF_HD inline void cell_stencil_bot4(const R& B, const double* dz, int k, double bc, bool neumann, double A1,
                                    double A2)
{
    const double dzp3h = 0.5 * (dz[k + 2] + dz[k + 1]);
    const double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
    const double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
    // row k: the fourth-order second difference across the wall vanishes
    set_row(B, k, 0.0, -A2 / dzm1h, -A1 / dzm1h - 2.0 * -A2 / dzp1h, +A1 / dzm1h - 2.0 * -A1 / dzp1h - A2 / dzp3h,
            +A2 / dzm1h - 2.0 * +A1 / dzp1h - A1 / dzp3h, -2.0 * +A2 / dzp1h + A1 / dzp3h, +A2 / dzp3h, 0.0);
    // row k-1: the boundary condition
    if (neumann) set_row(B, k - 1, 0.0, 0.0, 0.0, -A2 / dzp1h, -A1 / dzp1h, +A1 / dzp1h, +A2 / dzp1h, bc);
    else set_row(B, k - 1, 0.0, 0.0, 0.0, 0.5 * A2, 0.5 * (A1 + 2.0 * A2), 0.5 * (A1 + 2.0 * A2), 0.5 * A2, bc);
    // row k-2: even extension of the outermost ghost
    set_row(B, k - 2, 0.0, 0.0, 0.0, 0.0, 0.0, -1.0, +1.0, 0.0);
}
template <class R>
CF_HD inline void cell_stencil_top4(const R& B, const double* dz, int k, double bc, bool neumann, double A1,
                                    double A2)
{
    const double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
    const double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
    const double dzm3h = 0.5 * (dz[k - 2] + dz[k - 1]);
    set_row(B, k, -A2 / dzm3h, -A1 / dzm3h - 2.0 * -A2 / dzm1h, +A1 / dzm3h - 2.0 * -A1 / dzm1h - A2 / dzp1h,
            +A2 / dzm3h - 2.0 * +A1 / dzm1h - A1 / dzp1h, -2.0 * +A2 / dzm1h + A1 / dzp1h, +A2 / dzp1h, 0.0, 0.0);
    if (neumann) set_row(B, k + 1, -A2 / dzm1h, -A1 / dzm1h, +A1 / dzm1h, +A2 / dzm1h, 0.0, 0.0, 0.0, bc);
    else set_row(B, k + 1, 0.5 * A2, 0.5 * (A1 + 2.0 * A2), 0.5 * (A1 + 2.0 * A2), 0.5 * A2, 0.0, 0.0, 0.0, bc);
    set_row(B, k + 2, -1.0, +1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
}
// ghost_reduce_bot4 (diffuseu.c:807-850): fold the three wall rows (pivots
// b(k), d(k-1), f(k-2)) out of rows k+1..k+3.  dsub[0][0..2]: the diagonal
// subtractions of row k+1, dsub[1][0]: of row k+2.
template <class R>
CF_HD inline void cell_reduce_bot4(const R& B, int k, double (*dsub)[3] = nullptr)
{
    double fac, t;
    fac = B.a(k + 1) / B.b(k);
    B.a(k + 1) -= B.b(k) * fac; B.b(k + 1) -= B.c(k) * fac; B.c(k + 1) -= B.d(k) * fac;
    t = B.e(k) * fac; B.d(k + 1) -= t; if (dsub) dsub[0][0] = t;
    B.e(k + 1) -= B.f(k) * fac; B.f(k + 1) -= B.g(k) * fac;
    fac = B.b(k + 1) / B.d(k - 1);
    B.b(k + 1) -= B.d(k - 1) * fac; B.c(k + 1) -= B.e(k - 1) * fac;
    t = B.f(k - 1) * fac; B.d(k + 1) -= t; if (dsub) dsub[0][1] = t;
    B.e(k + 1) -= B.g(k - 1) * fac; B.r(k + 1) -= B.r(k - 1) * fac;
    fac = B.c(k + 1) / B.f(k - 2);
    B.c(k + 1) -= B.f(k - 2) * fac;
    t = B.g(k - 2) * fac; B.d(k + 1) -= t; if (dsub) dsub[0][2] = t;
    fac = B.a(k + 2) / B.d(k - 1);
    B.a(k + 2) -= B.d(k - 1) * fac; B.b(k + 2) -= B.e(k - 1) * fac; B.c(k + 2) -= B.f(k - 1) * fac;
    t = B.g(k - 1) * fac; B.d(k + 2) -= t; if (dsub) dsub[1][0] = t;
    B.r(k + 2) -= B.r(k - 1) * fac;
    fac = B.b(k + 2) / B.f(k - 2);
    B.b(k + 2) -= B.f(k - 2) * fac; B.c(k + 2) -= B.g(k - 2) * fac;
    fac = B.a(k + 3) / B.f(k - 2);
    B.a(k + 3) -= B.f(k - 2) * fac; B.b(k + 3) -= B.g(k - 2) * fac;
}
// ghost_reduce_top4 (diffuseu.c:853-896): pivots f(k), d(k+1), b(k+2) out of
// rows k-1..k-3; dsub rows k-1 (three), k-2 (one).
template <class R>
CF_HD inline void cell_reduce_top4(const R& B, int k, double (*dsub)[3] = nullptr)
{
    double fac, t;
    fac = B.g(k - 1) / B.f(k);
    B.g(k - 1) -= B.f(k) * fac; B.f(k - 1) -= B.e(k) * fac; B.e(k - 1) -= B.d(k) * fac;
    t = B.c(k) * fac; B.d(k - 1) -= t; if (dsub) dsub[0][0] = t;
    B.c(k - 1) -= B.b(k) * fac; B.b(k - 1) -= B.a(k) * fac;
    fac = B.f(k - 1) / B.d(k + 1);
    B.f(k - 1) -= B.d(k + 1) * fac; B.e(k - 1) -= B.c(k + 1) * fac;
    t = B.b(k + 1) * fac; B.d(k - 1) -= t; if (dsub) dsub[0][1] = t;
    B.c(k - 1) -= B.a(k + 1) * fac; B.r(k - 1) -= B.r(k + 1) * fac;
    fac = B.e(k - 1) / B.b(k + 2);
    B.e(k - 1) -= B.b(k + 2) * fac;
    t = B.a(k + 2) * fac; B.d(k - 1) -= t; if (dsub) dsub[0][2] = t;
    fac = B.g(k - 2) / B.d(k + 1);
    B.g(k - 2) -= B.d(k + 1) * fac; B.f(k - 2) -= B.c(k + 1) * fac; B.e(k - 2) -= B.b(k + 1) * fac;
    t = B.a(k + 1) * fac; B.d(k - 2) -= t; if (dsub) dsub[1][0] = t;
    B.r(k - 2) -= B.r(k + 1) * fac;
    fac = B.f(k - 2) / B.b(k + 2);
    B.f(k - 2) -= B.b(k + 2) * fac; B.e(k - 2) -= B.a(k + 2) * fac;
    fac = B.g(k - 3) / B.b(k + 2);
    B.g(k - 3) -= B.b(k + 2) * fac; B.f(k - 3) -= B.a(k + 2) * fac;
}
// ghost_fill_bot4 / top4 (diffuseu.c:899-940)
template <class R>
CF_HD inline void cell_fill_bot4(const R& B, int k)
{
    B.x(k) = (B.g(k - 2) * B.x(k + 1)) / -B.f(k - 2);
    B.x(k - 1) = (B.e(k - 1) * B.x(k) + B.f(k - 1) * B.x(k + 1) + B.g(k - 1) * B.x(k + 2) - B.r(k - 1)) / -B.d(k - 1);
    B.x(k - 2) = (B.c(k) * B.x(k - 1) + B.d(k) * B.x(k) + B.e(k) * B.x(k + 1) + B.f(k) * B.x(k + 2)
                  + B.g(k) * B.x(k + 3)) / -B.b(k);
}
template <class R>
CF_HD inline void cell_fill_top4(const R& B, int k)
{
    B.x(k) = (B.a(k + 2) * B.x(k - 1)) / -B.b(k + 2);
    B.x(k + 1) = (B.a(k + 1) * B.x(k - 2) + B.b(k + 1) * B.x(k - 1) + B.c(k + 1) * B.x(k) - B.r(k + 1)) / -B.d(k + 1);
    B.x(k + 2) = (B.a(k) * B.x(k - 3) + B.b(k) * B.x(k - 2) + B.c(k) * B.x(k - 1) + B.d(k) * B.x(k)
                  + B.e(k) * B.x(k + 1)) / -B.f(k);
}

// ---- face fields (w), second order: the wall face value is the unknown
// (diffusew.c:617-668)
template <class R>
CF_HD inline void face_stencil2(const R& B, int k, double bc)
{
    B.a(k) = 0.0; B.b(k) = 1.0; B.c(k) = 0.0; B.r(k) = bc;
}
template <class R>
CF_HD inline void face_reduce_bot2(const R& B, int k)
{
    const double fac = B.a(k + 1) / B.b(k);
    B.a(k + 1) -= B.b(k) * fac;
    B.r(k + 1) -= B.r(k) * fac;
}
template <class R>
CF_HD inline void face_reduce_top2(const R& B, int k)
{
    const double fac = B.c(k - 1) / B.b(k);
    B.c(k - 1) -= B.b(k) * fac;
    B.r(k - 1) -= B.r(k) * fac;
}
template <class R>
CF_HD inline void face_fill2(const R& B, int k) { B.x(k) = (-B.r(k)) / -B.b(k); }

// ---- face fields (w), fourth order (diffusew.c:691-884)
template <class R>
CF_HD inline void face_stencil_bot4(const R& B, const double* dz, int k, double bc, double A1, double A2)
{
    const double dzp0 = dz[k], dzp1 = dz[k + 1];
    set_row(B, k, 0.0, -A2 / dzp0, -A1 / dzp0 + A2 / dzp1, +A1 / dzp0 + A1 / dzp1, +A2 / dzp0 - A1 / dzp1,
            -A2 / dzp1, 0.0, 0.0);
    set_row(B, k - 1, 0.0, 0.0, 0.0, -1.0, +2.0, -1.0, 0.0, 0.0);
    set_row(B, k - 2, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, bc);
}
template <class R>
CF_HD inline void face_stencil_top4(const R& B, const double* dz, int k, double bc, double A1, double A2)
{
    const double dzp0 = dz[k], dzp1 = dz[k + 1];
    set_row(B, k, 0.0, -A2 / dzp0, -A1 / dzp0 + A2 / dzp1, +A1 / dzp0 + A1 / dzp1, +A2 / dzp0 - A1 / dzp1,
            -A2 / dzp1, 0.0, 0.0);
    set_row(B, k + 1, 0.0, -1.0, +2.0, -1.0, 0.0, 0.0, 0.0, 0.0);
    set_row(B, k + 2, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, bc);
}
// dsub[0][0..1]: the two diagonal subtractions of row k+1
template <class R>
CF_HD inline void face_reduce_bot4(const R& B, int k, double (*dsub)[3] = nullptr)
{
    double fac, t;
    fac = B.a(k + 1) / B.b(k);
    B.a(k + 1) -= B.b(k) * fac; B.b(k + 1) -= B.c(k) * fac; B.c(k + 1) -= B.d(k) * fac;
    t = B.e(k) * fac; B.d(k + 1) -= t; if (dsub) dsub[0][0] = t;
    B.e(k + 1) -= B.f(k) * fac;
    fac = B.b(k + 1) / B.d(k - 1);
    B.b(k + 1) -= B.d(k - 1) * fac; B.c(k + 1) -= B.e(k - 1) * fac;
    t = B.f(k - 1) * fac; B.d(k + 1) -= t; if (dsub) dsub[0][1] = t;
    fac = B.c(k + 1) / B.f(k - 2);
    B.c(k + 1) -= B.f(k - 2) * fac; B.r(k + 1) -= B.r(k - 2) * fac;
    fac = B.a(k + 2) / B.d(k - 1);
    B.a(k + 2) -= B.d(k - 1) * fac; B.b(k + 2) -= B.e(k - 1) * fac; B.c(k + 2) -= B.f(k - 1) * fac;
    fac = B.b(k + 2) / B.f(k - 2);
    B.b(k + 2) -= B.f(k - 2) * fac; B.r(k + 2) -= B.r(k - 2) * fac;
    fac = B.a(k + 3) / B.f(k - 2);
    B.a(k + 3) -= B.f(k - 2) * fac; B.r(k + 3) -= B.r(k - 2) * fac;
}
// dsub[0][0..1]: the two diagonal subtractions of row k-1
template <class R>
CF_HD inline void face_reduce_top4(const R& B, int k, double (*dsub)[3] = nullptr)
{
    double fac, t;
    fac = B.g(k - 1) / B.f(k);
    B.g(k - 1) -= B.f(k) * fac; B.f(k - 1) -= B.e(k) * fac; B.e(k - 1) -= B.d(k) * fac;
    t = B.c(k) * fac; B.d(k - 1) -= t; if (dsub) dsub[0][0] = t;
    B.c(k - 1) -= B.b(k) * fac;
    fac = B.f(k - 1) / B.d(k + 1);
    B.f(k - 1) -= B.d(k + 1) * fac; B.e(k - 1) -= B.c(k + 1) * fac;
    t = B.b(k + 1) * fac; B.d(k - 1) -= t; if (dsub) dsub[0][1] = t;
    fac = B.e(k - 1) / B.b(k + 2);
    B.e(k - 1) -= B.b(k + 2) * fac; B.r(k - 1) -= B.r(k + 2) * fac;
    fac = B.g(k - 2) / B.d(k + 1);
    B.g(k - 2) -= B.d(k + 1) * fac; B.f(k - 2) -= B.c(k + 1) * fac; B.e(k - 2) -= B.b(k + 1) * fac;
    fac = B.f(k - 2) / B.b(k + 2);
    B.f(k - 2) -= B.b(k + 2) * fac; B.r(k - 2) -= B.r(k + 2) * fac;
    fac = B.g(k - 3) / B.b(k + 2);
    B.g(k - 3) -= B.b(k + 2) * fac; B.r(k - 3) -= B.r(k + 2) * fac;
}
template <class R>
CF_HD inline void face_fill_bot4(const R& B, int k)
{
    B.x(k) = (-B.r(k - 2)) / -B.f(k - 2);
    B.x(k - 1) = (B.e(k - 1) * B.x(k) + B.f(k - 1) * B.x(k + 1)) / -B.d(k - 1);
    B.x(k - 2) = (B.c(k) * B.x(k - 1) + B.d(k) * B.x(k) + B.e(k) * B.x(k + 1) + B.f(k) * B.x(k + 2)) / -B.b(k);
}
template <class R>
CF_HD inline void face_fill_top4(const R& B, int k)
{
    B.x(k) = (-B.r(k + 2)) / -B.b(k + 2);
    B.x(k + 1) = (B.b(k + 1) * B.x(k - 1) + B.c(k + 1) * B.x(k)) / -B.d(k + 1);
    B.x(k + 2) = (B.b(k) * B.x(k - 2) + B.c(k) * B.x(k - 1) + B.d(k) * B.x(k) + B.e(k) * B.x(k + 1)) / -B.f(k);
}

}  // namespace closure
}  // namespace cf
