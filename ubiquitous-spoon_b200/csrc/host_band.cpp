// Host-side 1-D band construction; see host_band.h.  Every formula below
// restates the reference closure or band row named beside it, keeping its
// evaluation order (x86-64 builds without FMA contraction).
#include "host_band.h"
#include "closures.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace cf {

const double RK3_ALP[3] = {29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0};
const double RK3_BET[3] = {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0};
const double RK3_GAM[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
const double RK3_ZET[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

Metrics make_metrics(int order, int nx, int ny, int nz, int gz, double lx, double ly, double lz)
{
    Metrics m;
    m.order = order;
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    m.gz = gz;
    m.n2 = nz + 2 * gz;
    m.lx = lx;
    m.ly = ly;
    m.lz = lz;
    m.dx = lx / (double) nx;  // chanfast.c:141-142
    m.dy = ly / (double) ny;
    m.dz.assign(m.n2, 0.0);
    for (int iz = 0; iz < nz; iz++)  // chanfast.c:184-189
        m.dz[iz + gz] = lz * 0.5 * (std::cos(M_PI * (double) iz / (double) nz)
                                    - std::cos(M_PI * (double) (iz + 1) / (double) nz));
    for (int k = 0; k < gz; k++) m.dz[k] = m.dz[2 * gz - k - 1];  // ghost_even_z (ghost.c:31-54)
    for (int k = m.n2 - gz; k < m.n2; k++) m.dz[k] = m.dz[2 * (m.n2 - gz) - k - 1];
    return m;
}

// ---------------------------------------------------------------- closures
// Cell-centred fields and pressure (diffuseu.c:617-940, pressure.c:446-770),
// face fields (diffusew.c:617-884): closures.h, shared with the device step
// functions, over a view of the Band.

struct BandRef {
    Band& B;
    double& a(int k) const { return B.a[k]; }
    double& b(int k) const { return B.b[k]; }
    double& c(int k) const { return B.c[k]; }
    double& d(int k) const { return B.d[k]; }
    double& e(int k) const { return B.e[k]; }
    double& f(int k) const { return B.f[k]; }
    double& g(int k) const { return B.g[k]; }
    double& r(int k) const { return B.r[k]; }
    double& x(int k) const { return B.x[k]; }
};

static void u_stencil_bot2(Band& B, const std::vector<double>& dz, int k, double bc, BcKind t)
{
    closure::cell_stencil_bot2(BandRef{B}, dz.data(), k, bc, t == BC_NEUMANN);
}
static void u_stencil_top2(Band& B, const std::vector<double>& dz, int k, double bc, BcKind t)
{
    closure::cell_stencil_top2(BandRef{B}, dz.data(), k, bc, t == BC_NEUMANN);
}
static void u_reduce_bot2(Band& B, int k) { closure::cell_reduce_bot2(BandRef{B}, k); }
static void u_reduce_top2(Band& B, int k) { closure::cell_reduce_top2(BandRef{B}, k); }
static void u_fill_bot2(Band& B, int k) { closure::cell_fill_bot2(BandRef{B}, k); }
static void u_fill_top2(Band& B, int k) { closure::cell_fill_top2(BandRef{B}, k); }
static void u_stencil_bot4(Band& B, const std::vector<double>& dz, int k, double bc, BcKind t)
{
    closure::cell_stencil_bot4(BandRef{B}, dz.data(), k, bc, t == BC_NEUMANN, A1, A2);
}
static void u_stencil_top4(Band& B, const std::vector<double>& dz, int k, double bc, BcKind t)
{
    closure::cell_stencil_top4(BandRef{B}, dz.data(), k, bc, t == BC_NEUMANN, A1, A2);
}
// `dsub` (optional) receives the diagonal subtractions (closures.h)
static void u_reduce_bot4(Band& B, int k, double dsub[3][3]) { closure::cell_reduce_bot4(BandRef{B}, k, dsub); }
static void u_reduce_top4(Band& B, int k, double dsub[3][3]) { closure::cell_reduce_top4(BandRef{B}, k, dsub); }
static void u_fill_bot4(Band& B, int k) { closure::cell_fill_bot4(BandRef{B}, k); }
static void u_fill_top4(Band& B, int k) { closure::cell_fill_top4(BandRef{B}, k); }

static void w_stencil2(Band& B, int k, double bc) { closure::face_stencil2(BandRef{B}, k, bc); }
static void w_reduce_bot2(Band& B, int k) { closure::face_reduce_bot2(BandRef{B}, k); }
static void w_reduce_top2(Band& B, int k) { closure::face_reduce_top2(BandRef{B}, k); }
static void w_fill2(Band& B, int k) { closure::face_fill2(BandRef{B}, k); }
static void w_stencil_bot4(Band& B, const std::vector<double>& dz, int k, double bc)
{
    closure::face_stencil_bot4(BandRef{B}, dz.data(), k, bc, A1, A2);
}
static void w_stencil_top4(Band& B, const std::vector<double>& dz, int k, double bc)
{
    closure::face_stencil_top4(BandRef{B}, dz.data(), k, bc, A1, A2);
}
static void w_reduce_bot4(Band& B, int k, double dsub[3][3] = nullptr) { closure::face_reduce_bot4(BandRef{B}, k, dsub); }
static void w_reduce_top4(Band& B, int k, double dsub[3][3] = nullptr) { closure::face_reduce_top4(BandRef{B}, k, dsub); }
static void w_fill_bot4(Band& B, int k) { closure::face_fill_bot4(BandRef{B}, k); }
static void w_fill_top4(Band& B, int k) { closure::face_fill_top4(BandRef{B}, k); }

static WallRows rows_of(const Band& B, int k0, int step)
{
    WallRows w;
    for (int q = 0; q < 3; q++) {
        int k = k0 + q * step;
        const double* src[7] = {&B.a[k], &B.b[k], &B.c[k], &B.d[k], &B.e[k], &B.f[k], &B.g[k]};
        for (int t = 0; t < 7; t++) w.row[q][t] = *src[t];
    }
    return w;
}

WallRows bc_rows_u(const Metrics& m, bool bottom)
{
    Band B(m.n2);
    int kb = m.gz - 1, kt = m.n2 - m.gz;
    if (m.order == 2) {
        if (bottom) { u_stencil_bot2(B, m.dz, kb, 0.0, BC_DIRICHLET); return rows_of(B, kb, -1); }
        u_stencil_top2(B, m.dz, kt, 0.0, BC_DIRICHLET);
        return rows_of(B, kt, +1);
    }
    if (bottom) { u_stencil_bot4(B, m.dz, kb, 0.0, BC_DIRICHLET); return rows_of(B, kb, -1); }
    u_stencil_top4(B, m.dz, kt, 0.0, BC_DIRICHLET);
    return rows_of(B, kt, +1);
}

WallRows bc_rows_w(const Metrics& m, bool bottom)
{
    Band B(m.n2);
    int kb = m.gz - 1, kt = m.n2 - m.gz - 1;
    if (m.order == 2) {
        w_stencil2(B, bottom ? kb : kt, 0.0);
        return rows_of(B, bottom ? kb : kt, bottom ? -1 : +1);
    }
    if (bottom) { w_stencil_bot4(B, m.dz, kb, 0.0); return rows_of(B, kb, -1); }
    w_stencil_top4(B, m.dz, kt, 0.0);
    return rows_of(B, kt, +1);
}

void apply_bc_u_col(const Metrics& m, std::vector<double>& x, double bc_bot, double bc_top)
{
    // apply_bc_u2 / apply_bc_u4 (diffuseu.c:37-104)
    Band B(m.n2);
    B.x = x;
    int kb = m.gz - 1, kt = m.n2 - m.gz;
    if (m.order == 2) {
        u_stencil_bot2(B, m.dz, kb, bc_bot, BC_DIRICHLET);
        u_stencil_top2(B, m.dz, kt, bc_top, BC_DIRICHLET);
        u_fill_bot2(B, kb);
        u_fill_top2(B, kt);
    } else {
        u_stencil_bot4(B, m.dz, kb, bc_bot, BC_DIRICHLET);
        u_stencil_top4(B, m.dz, kt, bc_top, BC_DIRICHLET);
        u_fill_bot4(B, kb);
        u_fill_top4(B, kt);
    }
    x = B.x;
}

void apply_bc_w_col(const Metrics& m, std::vector<double>& x, double bc_bot, double bc_top)
{
    // apply_bc_w2 / apply_bc_w4 (diffusew.c:37-104)
    Band B(m.n2);
    B.x = x;
    int kb = m.gz - 1, kt = m.n2 - m.gz - 1;
    if (m.order == 2) {
        w_stencil2(B, kb, bc_bot);
        w_stencil2(B, kt, bc_top);
        w_fill2(B, kb);
        w_fill2(B, kt);
    } else {
        w_stencil_bot4(B, m.dz, kb, bc_bot);
        w_stencil_top4(B, m.dz, kt, bc_top);
        w_fill_bot4(B, kb);
        w_fill_top4(B, kt);
    }
    x = B.x;
}

// One row of helmholtz1d_operator_u{2,4} (diffuseu.c:121-131 / 149-169).
static double helmholtz_u_at(const Metrics& m, const double* u, int k, double nudt)
{
    const auto& dz = m.dz;
    if (m.order == 2) {
        double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
        double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
        return u[k] + nudt * (((u[k + 1] - u[k]) / dzp1h - (u[k] - u[k - 1]) / dzm1h) / dz[k]);
    }
    double wp3h = A1 * (u[k + 2] - u[k + 1]) + A2 * (u[k + 3] - u[k]);
    double wp1h = A1 * (u[k + 1] - u[k]) + A2 * (u[k + 2] - u[k - 1]);
    double wm1h = A1 * (u[k] - u[k - 1]) + A2 * (u[k + 1] - u[k - 2]);
    double wm3h = A1 * (u[k - 1] - u[k - 2]) + A2 * (u[k] - u[k - 3]);
    double dzp3h = 0.5 * (dz[k + 2] + dz[k + 1]);
    double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
    double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
    double dzm3h = 0.5 * (dz[k - 2] + dz[k - 1]);
    return u[k] + nudt * ((A1 * (wp1h / dzp1h - wm1h / dzm1h) + A2 * (wp3h / dzp3h - wm3h / dzm3h)) / dz[k]);
}

// One row of helmholtz1d_operator_w{2,4} (diffusew.c:121-132 / 150-171).
static double helmholtz_w_at(const Metrics& m, const double* w, int k, double nudt)
{
    const auto& dz = m.dz;
    double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
    if (m.order == 2) {
        double dzp1 = dz[k + 1], dzm0 = dz[k];
        return w[k] + nudt * (((w[k + 1] - w[k]) / dzp1 - (w[k] - w[k - 1]) / dzm0) / dzp1h);
    }
    double wp3h = A1 * (w[k + 2] - w[k + 1]) + A2 * (w[k + 3] - w[k]);
    double wp1h = A1 * (w[k + 1] - w[k]) + A2 * (w[k + 2] - w[k - 1]);
    double wm1h = A1 * (w[k] - w[k - 1]) + A2 * (w[k + 1] - w[k - 2]);
    double wm3h = A1 * (w[k - 1] - w[k - 2]) + A2 * (w[k] - w[k - 3]);
    double dzp2 = dz[k + 2], dzp1 = dz[k + 1], dzm0 = dz[k], dzm1 = dz[k - 1];
    return w[k] + nudt * ((A1 * (wp1h / dzp1 - wm1h / dzm0) + A2 * (wp3h / dzp2 - wm3h / dzm1)) / dzp1h);
}

void helmholtz_u_col(const Metrics& m, const std::vector<double>& u, std::vector<double>& h, double nudt)
{
    for (int k = m.gz; k < m.n2 - m.gz; k++) h[k] = helmholtz_u_at(m, u.data(), k, nudt);
}

void helmholtz_w_col(const Metrics& m, const std::vector<double>& w, std::vector<double>& h, double nudt)
{
    for (int k = m.gz; k < m.n2 - m.gz - 1; k++) h[k] = helmholtz_w_at(m, w.data(), k, nudt);
}

// ------------------------------------------------------- factorisation

static LineFactor factor_band(const Band& B, int k0, int n, int width)
{
    LineFactor L;
    L.k0 = k0;
    L.n = n;
    L.width = width;
    L.F1.assign(n, 0.0); L.F2.assign(n, 0.0); L.F3.assign(n, 0.0); L.DEN.assign(n, 0.0);
    L.P.assign(n, 0.0); L.Q.assign(n, 0.0); L.R.assign(n, 0.0);
    auto A = [&](int i) { return B.a[k0 + i]; };
    auto Bb = [&](int i) { return B.b[k0 + i]; };
    auto C = [&](int i) { return B.c[k0 + i]; };
    if (width == 3) {  // tridag.c:4-26
        double bet = Bb(0);
        if (bet == 0.0) throw std::runtime_error("zero pivot");
        L.DEN[0] = bet;
        std::vector<double> gam(n, 0.0);
        for (int j = 1; j < n; j++) {
            gam[j] = C(j - 1) / bet;
            bet = Bb(j) - A(j) * gam[j];
            if (bet == 0.0) throw std::runtime_error("zero pivot");
            L.F1[j] = A(j);
            L.DEN[j] = bet;
        }
        for (int j = 0; j < n - 1; j++) L.P[j] = gam[j + 1];
        return L;
    }
    // heptdag.c:5-61
    auto D = [&](int i) { return B.d[k0 + i]; };
    auto E = [&](int i) { return B.e[k0 + i]; };
    auto F = [&](int i) { return B.f[k0 + i]; };
    auto G = [&](int i) { return B.g[k0 + i]; };
    std::vector<double> p(n), q(n), r(n);
    double den, alp, bet;
    den = D(0);
    if (den == 0.0) throw std::runtime_error("zero pivot");
    p[0] = E(0) / den; q[0] = F(0) / den; r[0] = G(0) / den;
    L.DEN[0] = den;
    den = D(1) - C(1) * p[0];
    if (den == 0.0) throw std::runtime_error("zero pivot");
    p[1] = (E(1) - C(1) * q[0]) / den; q[1] = (F(1) - C(1) * r[0]) / den; r[1] = (G(1)) / den;
    L.F1[1] = C(1); L.DEN[1] = den;
    bet = C(2) - Bb(2) * p[0];
    den = D(2) - Bb(2) * q[0] - bet * p[1];
    if (den == 0.0) throw std::runtime_error("zero pivot");
    p[2] = (E(2) - Bb(2) * r[0] - bet * q[1]) / den; q[2] = (F(2) - bet * r[1]) / den; r[2] = (G(2)) / den;
    L.F2[2] = Bb(2); L.F1[2] = bet; L.DEN[2] = den;
    for (int i = 3; i < n; i++) {
        alp = Bb(i) - A(i) * p[i - 3];
        bet = C(i) - A(i) * q[i - 3] - alp * p[i - 2];
        den = D(i) - A(i) * r[i - 3] - alp * q[i - 2] - bet * p[i - 1];
        if (den == 0.0) throw std::runtime_error("zero pivot");
        p[i] = (E(i) - alp * r[i - 2] - bet * q[i - 1]) / den;
        q[i] = (F(i) - bet * r[i - 1]) / den;
        r[i] = (G(i)) / den;
        L.F3[i] = A(i); L.F2[i] = alp; L.F1[i] = bet; L.DEN[i] = den;
    }
    // Back substitution uses p, q, r of rows < n-1 (x[n-1] = s[n-1]).
    for (int i = 0; i < n - 1; i++) L.P[i] = p[i];
    for (int i = 0; i < n - 2; i++) L.Q[i] = q[i];
    for (int i = 0; i < n - 3; i++) L.R[i] = r[i];
    return L;
}

static void apply_factor(const LineFactor& L, const double* rhs, double* x)
{
    std::vector<double> s(L.n + 3, 0.0);
    double* sp = s.data() + 3;
    for (int i = 0; i < L.n; i++)
        sp[i] = (((rhs[i] - L.F3[i] * sp[i - 3]) - L.F2[i] * sp[i - 2]) - L.F1[i] * sp[i - 1]) / L.DEN[i];
    std::vector<double> y(L.n + 3, 0.0);
    for (int i = L.n - 1; i >= 0; i--)
        y[i] = ((sp[i] - L.P[i] * y[i + 1]) - L.Q[i] * y[i + 2]) - L.R[i] * y[i + 3];
    for (int i = 0; i < L.n; i++) x[i] = y[i];
}

// Interior band rows of solve_helmholtz1d_u{2,4} (diffuseu.c:190-201, 239-268);
// with area = dx*dy, the z part of solve_helmholtz_u{2,4} (diffuseu.c:430-445,
// 564-590), whose cell volume is dx*dy*dz.
static void band_rows_u(const Metrics& m, Band& B, double nudt, double area = 1.0)
{
    const auto& dz = m.dz;
    for (int k = m.gz; k < m.n2 - m.gz; k++) {
        double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
        double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
        double dvol = area * dz[k];
        if (m.order == 2) {
            B.a[k] = +dvol * nudt / (dzm1h * dz[k]);
            B.c[k] = +dvol * nudt / (dzp1h * dz[k]);
            B.b[k] = -dvol * nudt / (dzm1h * dz[k]) - dvol * nudt / (dzp1h * dz[k]) + dvol;
        } else {
            double dzp3h = 0.5 * (dz[k + 2] + dz[k + 1]);
            double dzm3h = 0.5 * (dz[k - 2] + dz[k - 1]);
            B.a[k] = +A2 * A2 * dvol * nudt / (dzm3h * dz[k]);
            B.g[k] = +A2 * A2 * dvol * nudt / (dzp3h * dz[k]);
            B.b[k] = +A1 * A2 * dvol * nudt / (dzm1h * dz[k]) + A1 * A2 * dvol * nudt / (dzm3h * dz[k]);
            B.f[k] = +A1 * A2 * dvol * nudt / (dzp1h * dz[k]) + A1 * A2 * dvol * nudt / (dzp3h * dz[k]);
            B.c[k] = -A1 * A2 * dvol * nudt / (dzp1h * dz[k]) - A1 * A2 * dvol * nudt / (dzm3h * dz[k])
                     + A1 * A1 * dvol * nudt / (dzm1h * dz[k]);
            B.e[k] = -A1 * A2 * dvol * nudt / (dzm1h * dz[k]) - A1 * A2 * dvol * nudt / (dzp3h * dz[k])
                     + A1 * A1 * dvol * nudt / (dzp1h * dz[k]);
            B.d[k] = -A2 * A2 * dvol * nudt / (dzm3h * dz[k]) - A2 * A2 * dvol * nudt / (dzp3h * dz[k])
                     - A1 * A1 * dvol * nudt / (dzm1h * dz[k]) - A1 * A1 * dvol * nudt / (dzp1h * dz[k])
                     + dvol;
        }
    }
}

// Interior band rows of solve_helmholtz1d_w{2,4} (diffusew.c:192-205, 242-272);
// with area = dx*dy, the z part of solve_helmholtz_w{2,4} (diffusew.c:494-509,
// 571-597).
static void band_rows_w(const Metrics& m, Band& B, double nudt, double area = 1.0)
{
    const auto& dz = m.dz;
    for (int k = m.gz; k < m.n2 - m.gz - 1; k++) {
        double dzp1 = dz[k + 1], dzm0 = dz[k];
        double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
        double dvol = area * dzp1h;
        if (m.order == 2) {
            B.a[k] = +dvol * nudt / (dzm0 * dzp1h);
            B.c[k] = +dvol * nudt / (dzp1 * dzp1h);
            B.b[k] = -dvol * nudt / (dzm0 * dzp1h) - dvol * nudt / (dzp1 * dzp1h) + dvol;
        } else {
            double dzp2 = dz[k + 2], dzm1 = dz[k - 1];
            B.a[k] = +A2 * A2 * dvol * nudt / (dzm1 * dzp1h);
            B.g[k] = +A2 * A2 * dvol * nudt / (dzp2 * dzp1h);
            B.b[k] = +A1 * A2 * dvol * nudt / (dzm0 * dzp1h) + A1 * A2 * dvol * nudt / (dzm1 * dzp1h);
            B.f[k] = +A1 * A2 * dvol * nudt / (dzp1 * dzp1h) + A1 * A2 * dvol * nudt / (dzp2 * dzp1h);
            B.c[k] = -A1 * A2 * dvol * nudt / (dzp1 * dzp1h) - A1 * A2 * dvol * nudt / (dzm1 * dzp1h)
                     + A1 * A1 * dvol * nudt / (dzm0 * dzp1h);
            B.e[k] = -A1 * A2 * dvol * nudt / (dzm0 * dzp1h) - A1 * A2 * dvol * nudt / (dzp2 * dzp1h)
                     + A1 * A1 * dvol * nudt / (dzp1 * dzp1h);
            B.d[k] = -A2 * A2 * dvol * nudt / (dzm1 * dzp1h) - A2 * A2 * dvol * nudt / (dzp2 * dzp1h)
                     - A1 * A1 * dvol * nudt / (dzm0 * dzp1h) - A1 * A1 * dvol * nudt / (dzp1 * dzp1h)
                     + dvol;
        }
    }
}

double z_average(const Metrics& m, const double* avg)
{
    // get_z_avg (get.c:490-502)
    double a = 0.0, l = 0.0;
    for (int k = m.gz; k < m.nz + m.gz; k++) {
        a += avg[k] * m.dz[k];
        l += m.dz[k];
    }
    return a / l;
}

void profile_stats(const Metrics& m, const double* avg, double kappa, double out[4])
{
    // chanfast.c:487-496 (order 2) / 1411-1420 (order 4)
    int g = m.gz, n2 = m.n2, nz = m.nz;
    const auto& dz = m.dz;
    out[0] = z_average(m, avg);
    if (m.order == 4) {
        out[1] = kappa * (A1 * (avg[g] - avg[g - 1]) + A2 * (avg[g + 1] - avg[g - 2])) / (0.5 * (dz[g] + dz[g - 1]));
        out[2] = kappa * (A1 * (avg[n2 - g] - avg[n2 - g - 1]) + A2 * (avg[n2 - g + 1] - avg[n2 - g - 2]))
                 / (0.5 * (dz[n2 - g] + dz[n2 - g - 1]));
    } else {
        out[1] = kappa * (avg[g] - avg[g - 1]) / (0.5 * (dz[g] + dz[g - 1]));
        out[2] = kappa * (avg[n2 - g] - avg[n2 - g - 1]) / (0.5 * (dz[n2 - g] + dz[n2 - g - 1]));
    }
    out[3] = nz % 2 == 0 ? 0.5 * (avg[g + nz / 2 - 1] + avg[g + nz / 2]) : avg[g + nz / 2];
}

ImplicitSet make_implicit_u(const Metrics& m, double nubdt, double gamdt, double bc_bot,
                            double bc_top, double kappa, bool want_green)
{
    ImplicitSet S;
    int kb = m.gz - 1, kt = m.n2 - m.gz;
    Band B(m.n2);
    band_rows_u(m, B, -nubdt);
    if (m.order == 2) {
        u_stencil_bot2(B, m.dz, kb, 0.0, BC_DIRICHLET);
        u_stencil_top2(B, m.dz, kt, 0.0, BC_DIRICHLET);
        S.bot = rows_of(B, kb, -1);
        S.top = rows_of(B, kt, +1);
        u_reduce_bot2(B, kb);
        u_reduce_top2(B, kt);
        S.fac = factor_band(B, m.gz, m.nz, 3);
    } else {
        u_stencil_bot4(B, m.dz, kb, 0.0, BC_DIRICHLET);
        u_stencil_top4(B, m.dz, kt, 0.0, BC_DIRICHLET);
        S.bot = rows_of(B, kb, -1);
        S.top = rows_of(B, kt, +1);
        u_reduce_bot4(B, kb, nullptr);
        u_reduce_top4(B, kt, nullptr);
        S.fac = factor_band(B, m.gz, m.nz, 7);
    }
    // Boundary lifting (chanfast.c:473-477): bc := 0, apply_bc(bc), hbc = H(-nubdt) bc.
    std::vector<double> bc(m.n2, 0.0), hbc(m.n2, 0.0);
    apply_bc_u_col(m, bc, bc_bot, bc_top);
    helmholtz_u_col(m, bc, hbc, -nubdt);
    S.hbc = hbc;
    if (want_green) {
        std::vector<double> h(m.n2, gamdt), out(m.n2, 0.0);
        solve_column(S, m, false, h, out);
        S.green = out;
        profile_stats(m, out.data(), kappa, S.green_stats);
    }
    return S;
}

ImplicitSet make_implicit_w(const Metrics& m, double nubdt, double bc_bot, double bc_top)
{
    ImplicitSet S;
    int kb = m.gz - 1, kt = m.n2 - m.gz - 1;
    Band B(m.n2);
    band_rows_w(m, B, -nubdt);
    if (m.order == 2) {
        w_stencil2(B, kb, 0.0);
        w_stencil2(B, kt, 0.0);
        S.bot = rows_of(B, kb, -1);
        S.top = rows_of(B, kt, +1);
        w_reduce_bot2(B, kb);
        w_reduce_top2(B, kt);
        S.fac = factor_band(B, m.gz, m.nz - 1, 3);
    } else {
        w_stencil_bot4(B, m.dz, kb, 0.0);
        w_stencil_top4(B, m.dz, kt, 0.0);
        S.bot = rows_of(B, kb, -1);
        S.top = rows_of(B, kt, +1);
        w_reduce_bot4(B, kb);
        w_reduce_top4(B, kt);
        S.fac = factor_band(B, m.gz, m.nz - 1, 7);
    }
    std::vector<double> bc(m.n2, 0.0), hbc(m.n2, 0.0);
    apply_bc_w_col(m, bc, bc_bot, bc_top);
    helmholtz_w_col(m, bc, hbc, -nubdt);
    S.hbc = hbc;
    return S;
}

void solve_column(const ImplicitSet& s, const Metrics& m, bool is_w, std::vector<double>& h,
                  std::vector<double>& out)
{
    // r = h * dvol (diffuseu.c:200, diffusew.c:204); the ghost rows carry
    // bc = 0 so the elimination leaves r unchanged.
    int k0 = s.fac.k0, n = s.fac.n;
    std::vector<double> r(n);
    for (int i = 0; i < n; i++) {
        int k = k0 + i;
        double dvol = is_w ? 0.5 * (m.dz[k + 1] + m.dz[k]) : m.dz[k];
        r[i] = h[k] * dvol;
    }
    Band B(m.n2);
    apply_factor(s.fac, r.data(), &B.x[k0]);
    // ghost fill with the solve's closure rows (bc = 0)
    auto put = [&](const WallRows& w, int k, int step) {
        for (int q = 0; q < 3; q++) {
            int kk = k + q * step;
            B.a[kk] = w.row[q][0]; B.b[kk] = w.row[q][1]; B.c[kk] = w.row[q][2]; B.d[kk] = w.row[q][3];
            B.e[kk] = w.row[q][4]; B.f[kk] = w.row[q][5]; B.g[kk] = w.row[q][6]; B.r[kk] = 0.0;
        }
    };
    int kb = m.gz - 1, kt = is_w ? m.n2 - m.gz - 1 : m.n2 - m.gz;
    if (m.order == 2) {
        put(s.bot, kb, -1);
        put(s.top, kt, +1);
        if (is_w) { w_fill2(B, kb); w_fill2(B, kt); }
        else { u_fill_bot2(B, kb); u_fill_top2(B, kt); }
    } else {
        put(s.bot, kb, -1);
        put(s.top, kt, +1);
        if (is_w) { w_fill_bot4(B, kb); w_fill_top4(B, kt); }
        else { u_fill_bot4(B, kb); u_fill_top4(B, kt); }
    }
    out = B.x;
}

// Stencil coefficients of the 1-D Helmholtz operator on rows k0 .. k0+n-1:
// the operator is linear, so its coefficients are its response to unit columns.
static std::vector<double> operator_coefs(const Metrics& m, int k0, int n, bool is_w, double nudt)
{
    const int H = m.order == 2 ? 1 : 3;
    std::vector<double> L((size_t) n * (2 * H + 1), 0.0);
    std::vector<double> e(m.n2, 0.0);
    for (int i = 0; i < n; i++) {
        int k = k0 + i;
        for (int off = -H; off <= H; off++) {
            e[k + off] = 1.0;
            L[(size_t) i * (2 * H + 1) + off + H] = is_w ? helmholtz_w_at(m, e.data(), k, nudt)
                                                         : helmholtz_u_at(m, e.data(), k, nudt);
            e[k + off] = 0.0;
        }
    }
    return L;
}

std::vector<double> fused_rows(const Metrics& m, const ImplicitSet& s, bool is_w, double nuadt,
                               double gamdt, double zetdt)
{
    const int H = m.order == 2 ? 1 : 3;
    const int W = fused_width(m.order);
    const int k0 = s.fac.k0, n = s.fac.n;
    const std::vector<double> L = operator_coefs(m, k0, n, is_w, nuadt);
    std::vector<double> rows((size_t) n * W, 0.0);
    for (int i = 0; i < n; i++) {
        int k = k0 + i;
        double dvol = is_w ? 0.5 * (m.dz[k + 1] + m.dz[k]) : m.dz[k];
        double iden = 1.0 / s.fac.DEN[i];
        double* r = &rows[(size_t) i * W];
        for (int t = 0; t < 2 * H + 1; t++) r[t] = dvol * L[(size_t) i * (2 * H + 1) + t] * iden;
        r[2 * H + 1] = dvol * gamdt * iden;
        r[2 * H + 2] = dvol * zetdt * iden;
        r[2 * H + 3] = -dvol * s.hbc[k] * iden;
        r[2 * H + 4] = s.fac.F1[i] * iden;
        r[2 * H + 5] = s.fac.F2[i] * iden;
        r[2 * H + 6] = s.fac.F3[i] * iden;
    }
    return rows;
}

std::vector<double> channel_rows(const Metrics& m, const ImplicitSet& s, bool is_w, double nuadt,
                                 double gamdt, double zetdt)
{
    const int H = m.order == 2 ? 1 : 3;
    const int W = fused_width(m.order);
    const int k0 = s.fac.k0, n = s.fac.n;
    const std::vector<double> L = operator_coefs(m, k0, n, is_w, nuadt);
    std::vector<double> rows((size_t) n * W, 0.0);
    for (int i = 0; i < n; i++) {
        double* r = &rows[(size_t) i * W];
        for (int t = 0; t < 2 * H + 1; t++) r[t] = L[(size_t) i * (2 * H + 1) + t];
        r[2 * H + 1] = gamdt;
        r[2 * H + 2] = zetdt;
        r[2 * H + 3] = -s.hbc[k0 + i];
    }
    return rows;
}

// Modified wavenumbers of the x-y second difference, the same for the
// pressure Poisson and the spectral Helmholtz solves (pressure.c:312-315,
// 376-389; diffuseu.c:426-429, 547-560).
static void modified_wavenumbers(const Metrics& m, PoissonSet& P)
{
    auto lam = [&](int n, int i) {
        double c1 = std::cos(2.0 * M_PI * 1.0 * (double) i / (double) n);
        if (m.order == 2) return 2.0 - 2.0 * c1;
        double c2 = std::cos(2.0 * M_PI * 2.0 * (double) i / (double) n);
        double c3 = std::cos(2.0 * M_PI * 3.0 * (double) i / (double) n);
        return (2.0 * A2 * A2 + 2.0 * A1 * A1) + (4.0 * A1 * A2 - 2.0 * A1 * A1) * c1
               + (-4.0 * A1 * A2) * c2 + (-2.0 * A2 * A2) * c3;
    };
    P.lamx.resize(m.nx / 2 + 1);
    for (int i = 0; i <= m.nx / 2; i++) P.lamx[i] = lam(m.nx, i);
    P.lamy.resize(m.ny);
    for (int j = 0; j < m.ny; j++) P.lamy[j] = lam(m.ny, j);
}

PoissonSet make_helmholtz_spectral(const Metrics& m, double nudt, bool is_w)
{
    PoissonSet P;
    P.width = m.order == 2 ? 3 : 7;
    const auto& dz = m.dz;
    const int n2 = m.n2, g = m.gz;
    const int n = is_w ? m.nz - 1 : m.nz;
    const int kb = g - 1, kt = g + n;   // wall ghost row / face below and above the rows
    const double area = m.dx * m.dy;
    Band B(n2);
    if (is_w) band_rows_w(m, B, nudt, area);
    else band_rows_u(m, B, nudt, area);
    P.dpart.assign(n2, 0.0);
    P.dvol.assign(n2, 0.0);
    for (int k = g; k < g + n; k++) {
        // column-independent part of the diagonal; the wavenumber terms are
        // cx = dvol nudt / dx^2, cy = dvol nudt / dy^2 (added on the device)
        P.dvol[k] = area * (is_w ? 0.5 * (dz[k + 1] + dz[k]) : dz[k]);
        double& dg = m.order == 2 ? B.b[k] : B.d[k];
        P.dpart[k] = dg;
        dg = 0.0;
    }
    double ds_b[3][3] = {{0}}, ds_t[3][3] = {{0}};
    if (m.order == 2) {
        if (is_w) { w_stencil2(B, kb, 0.0); w_stencil2(B, kt, 0.0); }
        else { u_stencil_bot2(B, dz, kb, 0.0, BC_DIRICHLET); u_stencil_top2(B, dz, kt, 0.0, BC_DIRICHLET); }
        P.bot[0] = rows_of(B, kb, -1);
        P.top = rows_of(B, kt, +1);
        // ghost_reduce_{bot,top}2: the diagonal of the first / last row loses c[kb]*fac / a[kt]*fac
        double fac = B.a[kb + 1] / B.b[kb];
        B.a[kb + 1] -= B.b[kb] * fac;
        ds_b[0][0] = B.c[kb] * fac;
        double fact = B.c[kt - 1] / B.b[kt];
        B.c[kt - 1] -= B.b[kt] * fact;
        ds_t[0][0] = B.a[kt] * fact;
    } else if (is_w) {
        w_stencil_bot4(B, dz, kb, 0.0);
        w_stencil_top4(B, dz, kt, 0.0);
        P.bot[0] = rows_of(B, kb, -1);
        P.top = rows_of(B, kt, +1);
        w_reduce_bot4(B, kb, ds_b);
        w_reduce_top4(B, kt, ds_t);
    } else {
        u_stencil_bot4(B, dz, kb, 0.0, BC_DIRICHLET);
        u_stencil_top4(B, dz, kt, 0.0, BC_DIRICHLET);
        P.bot[0] = rows_of(B, kb, -1);
        P.top = rows_of(B, kt, +1);
        u_reduce_bot4(B, kb, ds_b);
        u_reduce_top4(B, kt, ds_t);
    }
    P.bot[1] = P.bot[0];
    const int rows[6] = {g, g + 1, g + 2, g + n - 3, g + n - 2, g + n - 1};
    for (int q = 0; q < 6; q++) {
        int k = rows[q];
        const double vals[7] = {B.a[k], B.b[k], B.c[k], B.d[k], B.e[k], B.f[k], B.g[k]};
        for (int t = 0; t < 7; t++) P.red[0][q][t] = vals[t];
        for (int t = 0; t < 3; t++) P.dsub[0][q][t] = 0.0;
    }
    for (int t = 0; t < 3; t++) P.dsub[0][0][t] = ds_b[0][t];
    P.dsub[0][1][0] = ds_b[1][0];
    for (int t = 0; t < 3; t++) P.dsub[0][5][t] = ds_t[0][t];
    P.dsub[0][4][0] = ds_t[1][0];
    std::memcpy(P.red[1], P.red[0], sizeof(P.red[0]));
    std::memcpy(P.dsub[1], P.dsub[0], sizeof(P.dsub[0]));
    P.a.assign(n2, 0.0); P.b.assign(n2, 0.0); P.c.assign(n2, 0.0);
    P.e.assign(n2, 0.0); P.f.assign(n2, 0.0); P.g.assign(n2, 0.0);
    for (int k = g; k < g + n; k++) {
        P.a[k] = B.a[k]; P.b[k] = B.b[k]; P.c[k] = B.c[k];
        P.e[k] = B.e[k]; P.f[k] = B.f[k]; P.g[k] = B.g[k];
    }
    modified_wavenumbers(m, P);
    return P;
}

PoissonSet make_poisson(const Metrics& m, double dt)
{
    PoissonSet P;
    P.width = m.order == 2 ? 3 : 7;
    const auto& dz = m.dz;
    double dx = m.dx, dy = m.dy;
    int n2 = m.n2, g = m.gz, nz = m.nz;
    P.dpart.assign(n2, 0.0);
    P.dvol.assign(n2, 0.0);
    Band B(n2);
    for (int k = g; k < n2 - g; k++) {  // pressure.c:317-330 / 391-418
        double dzp1h = 0.5 * (dz[k + 1] + dz[k]);
        double dzm1h = 0.5 * (dz[k - 1] + dz[k]);
        double dvol = dx * dy * dz[k];
        P.dvol[k] = dvol;
        if (m.order == 2) {
            B.a[k] = +dvol * dt / (dzm1h * dz[k]);
            B.c[k] = +dvol * dt / (dzp1h * dz[k]);
            P.dpart[k] = -dvol * dt / (dzm1h * dz[k]) - dvol * dt / (dzp1h * dz[k]);
        } else {
            double dzp3h = 0.5 * (dz[k + 2] + dz[k + 1]);
            double dzm3h = 0.5 * (dz[k - 2] + dz[k - 1]);
            B.a[k] = +A2 * A2 * dvol * dt / (dzm3h * dz[k]);
            B.g[k] = +A2 * A2 * dvol * dt / (dzp3h * dz[k]);
            B.b[k] = +A1 * A2 * dvol * dt / (dzm1h * dz[k]) + A1 * A2 * dvol * dt / (dzm3h * dz[k]);
            B.f[k] = +A1 * A2 * dvol * dt / (dzp1h * dz[k]) + A1 * A2 * dvol * dt / (dzp3h * dz[k]);
            B.c[k] = -A1 * A2 * dvol * dt / (dzp1h * dz[k]) - A1 * A2 * dvol * dt / (dzm3h * dz[k])
                     + A1 * A1 * dvol * dt / (dzm1h * dz[k]);
            B.e[k] = -A1 * A2 * dvol * dt / (dzm1h * dz[k]) - A1 * A2 * dvol * dt / (dzp3h * dz[k])
                     + A1 * A1 * dvol * dt / (dzp1h * dz[k]);
            P.dpart[k] = -A2 * A2 * dvol * dt / (dzm3h * dz[k]) - A2 * A2 * dvol * dt / (dzp3h * dz[k])
                         - A1 * A1 * dvol * dt / (dzm1h * dz[k]) - A1 * A1 * dvol * dt / (dzp1h * dz[k]);
        }
    }
    int kb = g - 1, kt = n2 - g;
    for (int v = 0; v < 2; v++) {
        Band V = B;  // diagonal handled separately: keep d = 0 here
        for (int k = g; k < n2 - g; k++) { if (m.order == 2) V.b[k] = 0.0; else V.d[k] = 0.0; }
        BcKind bk = v == 1 ? BC_DIRICHLET : BC_NEUMANN;  // pressure.c:331-338
        double ds_b[3][3] = {{0}}, ds_t[3][3] = {{0}};
        if (m.order == 2) {
            u_stencil_bot2(V, dz, kb, 0.0, bk);
            u_stencil_top2(V, dz, kt, 0.0, BC_NEUMANN);
            P.bot[v] = rows_of(V, kb, -1);
            if (v == 0) P.top = rows_of(V, kt, +1);
            // reduce_bot2: the diagonal of row kb+1 loses c[kb]*fac
            double fac = V.a[kb + 1] / V.b[kb];
            V.a[kb + 1] -= V.b[kb] * fac;
            ds_b[0][0] = V.c[kb] * fac;
            double fact = V.c[kt - 1] / V.b[kt];
            V.c[kt - 1] -= V.b[kt] * fact;
            ds_t[0][0] = V.a[kt] * fact;
        } else {
            u_stencil_bot4(V, dz, kb, 0.0, bk);
            u_stencil_top4(V, dz, kt, 0.0, BC_NEUMANN);
            P.bot[v] = rows_of(V, kb, -1);
            if (v == 0) P.top = rows_of(V, kt, +1);
            u_reduce_bot4(V, kb, ds_b);
            u_reduce_top4(V, kt, ds_t);
        }
        int rows[6] = {g, g + 1, g + 2, n2 - g - 3, n2 - g - 2, n2 - g - 1};
        for (int q = 0; q < 6; q++) {
            int k = rows[q];
            const double vals[7] = {V.a[k], V.b[k], V.c[k], V.d[k], V.e[k], V.f[k], V.g[k]};
            for (int t = 0; t < 7; t++) P.red[v][q][t] = vals[t];
            for (int t = 0; t < 3; t++) P.dsub[v][q][t] = 0.0;
        }
        // bottom: rows g (q=0) three subtractions, g+1 (q=1) one; top: n2-g-1 (q=5) three, n2-g-2 (q=4) one
        for (int t = 0; t < 3; t++) P.dsub[v][0][t] = ds_b[0][t];
        P.dsub[v][1][0] = ds_b[1][0];
        for (int t = 0; t < 3; t++) P.dsub[v][5][t] = ds_t[0][t];
        P.dsub[v][4][0] = ds_t[1][0];
        if (v == 0) {
            P.a.assign(n2, 0.0); P.b.assign(n2, 0.0); P.c.assign(n2, 0.0);
            P.e.assign(n2, 0.0); P.f.assign(n2, 0.0); P.g.assign(n2, 0.0);
            for (int k = g; k < n2 - g; k++) {
                P.a[k] = V.a[k]; P.b[k] = V.b[k]; P.c[k] = V.c[k];
                P.e[k] = V.e[k]; P.f[k] = V.f[k]; P.g[k] = V.g[k];
            }
        }
    }
    (void) nz;
    modified_wavenumbers(m, P);
    return P;
}

std::vector<double> z_at_p(const Metrics& m)
{
    std::vector<double> z(m.n2);
    z[0] = 0.5 * m.dz[0];
    for (int k = 1; k < m.n2; k++) z[k] = z[k - 1] + 0.5 * (m.dz[k - 1] + m.dz[k]);
    double z0 = 0.5 * (z[m.gz - 1] + z[m.gz]);
    for (int k = 0; k < m.n2; k++) z[k] -= z0;
    return z;
}

std::vector<double> z_at_w(const Metrics& m)
{
    std::vector<double> z(m.n2);
    z[0] = m.dz[0];
    for (int k = 1; k < m.n2; k++) z[k] = z[k - 1] + m.dz[k];
    double z0 = z[m.gz - 1];
    for (int k = 0; k < m.n2; k++) z[k] -= z0;
    return z;
}

}  // namespace cf
