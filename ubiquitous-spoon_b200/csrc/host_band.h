// Host-side construction of the column-independent parts of the wall-normal
// line solves (1-D, O(n2) work, done once per RK3 substep coefficient set).
//
// The implicit-diffusion matrices of solve_helmholtz1d_{u,w}{2,4}
// (reference diffuseu.c:173-283, diffusew.c:175-287) depend only on k, dz and
// the diffusion coefficient, never on the column, so their factorisation is
// computed here once and the device only streams right-hand sides.  The
// pressure matrices (pressure.c:293-443) differ per wavenumber only through
// the main diagonal; everything else is built here.  All arithmetic follows
// the reference's expression order so device results can match it bit for bit.
#pragma once

#include <vector>

namespace cf {

constexpr double A1 = 1.125 / 1.0;   // fourth.c:3
constexpr double A2 = -0.125 / 3.0;  // fourth.c:4
constexpr double B1 = 1.125 / 2.0;   // fourth.c:5
constexpr double B2 = -0.125 / 2.0;  // fourth.c:6

extern const double RK3_ALP[3], RK3_BET[3], RK3_GAM[3], RK3_ZET[3];  // rk3.c:3-6

enum BcKind { BC_DIRICHLET = 0, BC_NEUMANN = 1 };

// A banded column of length n2 (rows a..g act on x[k-3..k+3]; the tridiagonal
// variants use a, b, c on x[k-1..k+1]).
struct Band {
    int n2 = 0;
    std::vector<double> a, b, c, d, e, f, g, r, x;
    explicit Band(int n2_) : n2(n2_), a(n2_, 0.0), b(n2_, 0.0), c(n2_, 0.0), d(n2_, 0.0),
                             e(n2_, 0.0), f(n2_, 0.0), g(n2_, 0.0), r(n2_, 0.0), x(n2_, 0.0) {}
};

// Factorisation of a column-independent reduced band system over rows
// [k0, k0 + n) of a column, in the recurrence form used on the device:
//   s_i = (((r_i - F3_i s_{i-3}) - F2_i s_{i-2}) - F1_i s_{i-1}) / DEN_i
//   x_i = ((s_i - P_i x_{i+1}) - Q_i x_{i+2}) - R_i x_{i+3}
// (tridiagonal: F2 = F3 = Q = R = 0).  Same operations as tridag.c:4-26 and
// heptdag.c:5-61 applied to the right-hand side.
struct LineFactor {
    int k0 = 0, n = 0, width = 3;
    std::vector<double> F1, F2, F3, DEN, P, Q, R;
};

// Ghost-cell fill coefficients of one wall (the stencil rows of
// ghost_stencil_{bot,top}{2,4}); rows[0..2] = rows k, k-1, k-2 (bottom) or
// k, k+1, k+2 (top), 7 coefficients a..g each.
struct WallRows {
    double row[3][7];
};

// Everything the device needs for one implicit solve (field type, order,
// diffusion coefficient): the factorisation, the wall closures used to
// recover ghost values, the boundary-lifting term hbc and the Green's
// function of a unit-rate forcing (for the mass-flux control).
struct ImplicitSet {
    LineFactor fac;
    WallRows bot, top;       // closure rows for the solve's own ghost fill (bc = 0)
    std::vector<double> hbc; // H(-nubdt) applied to the zero field with wall BC, interior rows
    std::vector<double> green;  // solve(gamdt) over all n2 rows (u and c only)
    double green_stats[4] = {0, 0, 0, 0};  // z-average, bottom/top wall gradient, centreline
};

// Grid metrics of one instance (chanfast.c:140-192).
struct Metrics {
    int order, nx, ny, nz, gz, n2;
    double lx, ly, lz, dx, dy;
    std::vector<double> dz;
};

Metrics make_metrics(int order, int nx, int ny, int nz, int gz, double lx, double ly, double lz);

// Stencil rows used by apply_bc_u / apply_bc_w (bc value enters separately).
WallRows bc_rows_u(const Metrics& m, bool bottom);
WallRows bc_rows_w(const Metrics& m, bool bottom);

// Fill the ghost rows of one column `x` (length n2) from its interior, as
// apply_bc_u{2,4} / apply_bc_w{2,4} do, with wall values bc_bot / bc_top.
void apply_bc_u_col(const Metrics& m, std::vector<double>& x, double bc_bot, double bc_top);
void apply_bc_w_col(const Metrics& m, std::vector<double>& x, double bc_bot, double bc_top);

// 1-D Helmholtz operator h = x + nudt d2x/dz2 on interior rows
// (helmholtz1d_operator_{u,w}{2,4}); other rows of h untouched.
void helmholtz_u_col(const Metrics& m, const std::vector<double>& x, std::vector<double>& h, double nudt);
void helmholtz_w_col(const Metrics& m, const std::vector<double>& x, std::vector<double>& h, double nudt);

// Implicit-solve set for u-type (cell-centred) or w-type (face) fields.
// nuadt/nubdt: explicit and implicit diffusion coefficients of the substep,
// gamdt: RK3 gamma*dt, bc_bot/bc_top: wall values, kappa: diffusivity used
// in the wall-gradient statistics.
ImplicitSet make_implicit_u(const Metrics& m, double nubdt, double gamdt, double bc_bot,
                            double bc_top, double kappa, bool want_green);
ImplicitSet make_implicit_w(const Metrics& m, double nubdt, double bc_bot, double bc_top);

// Per-row coefficients of the fused forward sweep used on the device:
//   s_i = sum_m cu_m x_{k+m} + cf f_k + cg g_k + c0 - f1 s_{i-1} - f2 s_{i-2} - f3 s_{i-3}
// which is, up to rounding, ((H(nuadt) x + gamdt f + zetdt g - hbc) dvol - F.s) / DEN
// (chanfast.c:469-482 with the forward half of tridag/heptdag).  Row i holds
// [cu_{-H..H}, cf, cg, c0, f1, f2, f3] with H = 1 (order 2) or 3 (order 4).
std::vector<double> fused_rows(const Metrics& m, const ImplicitSet& s, bool is_w, double nuadt,
                               double gamdt, double zetdt);
inline int fused_width(int order) { return (order == 2 ? 3 : 7) + 6; }

// Per-row coefficients of the channel scheme's Helmholtz right-hand side
// (channel.c:455-467 and its v, c, w counterparts), z part:
//   h_k = sum_m cu_m x_{k+m} + cf f_k + cg g_k + c0
// = x + nuadt d2x/dz2 + gamdt f + zetdt g - hbc; the device adds
// nuadt (d2/dx2 + d2/dy2) x.  Same row layout as fused_rows, f1..f3 = 0.
std::vector<double> channel_rows(const Metrics& m, const ImplicitSet& s, bool is_w, double nuadt,
                                 double gamdt, double zetdt);

// Solve one column with an ImplicitSet factorisation (host reference of the
// device kernel; used for the Green's function and for tests).
void solve_column(const ImplicitSet& s, const Metrics& m, bool is_w, std::vector<double>& rhs_h,
                  std::vector<double>& out);

// Pressure Poisson column data (pressure_poisson{2,4}).  Interior band rows
// a..g with the column-independent part of the main diagonal in dpart; the
// two closure variants (0: Neumann/Neumann, 1: Dirichlet bottom for the mean
// mode) give the reduced rows near the walls and the diagonal corrections,
// applied on the device in the listed order.
struct PoissonSet {
    int width;
    std::vector<double> a, b, c, e, f, g;   // per interior row (reduced for variant 0)
    std::vector<double> dpart, dvol;        // diagonal partial sum, cell volume dx*dy*dz
    // Rows near the walls whose off-diagonals differ between the variants:
    // variant v, boundary row index q (0..5 = k0, k0+1, k0+2, top-3, top-2, top-1):
    double red[2][6][7];    // a..g after reduction (d unused)
    double dsub[2][6][3];   // diagonal subtractions, in order
    WallRows bot[2], top;   // closure rows for the ghost fill
    std::vector<double> lamx, lamy;  // modified wavenumbers (pressure.c:312-315 / 376-389)
};
PoissonSet make_poisson(const Metrics& m, double dt);

// Per-wavenumber band of solve_helmholtz_{u,w}{2,4} (diffuseu.c:398-614,
// diffusew.c:466-614) with Dirichlet walls and zero wall values, in the same
// form: rows GZ .. GZ+n-1 (n = nz for cell-centred fields, nz - 1 for w),
// diagonal dpart - lamx cx - lamy cy with cx = dvol nudt / dx^2 applied on
// the device, both closure variants equal (no special mean mode).
PoissonSet make_helmholtz_spectral(const Metrics& m, double nudt, bool is_w);

// Bulk statistics of an xy-averaged profile (chanfast.c:485-509):
// out = {z-average, kappa*d/dz at bottom, at top, centreline}.
void profile_stats(const Metrics& m, const double* avg, double kappa, double out[4]);
double z_average(const Metrics& m, const double* avg);

// z coordinates of cell centres / faces (get.c:458-487).
std::vector<double> z_at_p(const Metrics& m);
std::vector<double> z_at_w(const Metrics& m);

}  // namespace cf
