// Step functions of the reference (advect.h, diffuseu.h, diffusew.h,
// pressure.h, scalar.h, rk3.h, fourth.h, tridag.h, heptdag.h) with their
// names, signatures and field layout, computed on the GPU.
//
// Every function takes host arrays in the reference's padded d3tensor layout
// (index (i*n1 + j)*n2 + k, k wall-normal and fastest, d3tensor.c:9-42),
// copies the arrays it reads to the current CUDA device, runs one or two
// kernels over exactly the index ranges the reference loops cover, and copies
// the arrays it writes back.  They exist so that code written against the
// reference's step functions links against this library unchanged, and so
// that each function can be checked against the reference on its own; the
// time-stepping engine (cf_* in chanfast_cuda.h) does not use them.
//
// Arithmetic follows the reference's expressions operation for operation and
// this file is compiled without FMA contraction, with IEEE division, so the
// results equal the reference's bit for bit.  The modified wavenumbers of the
// spectral solves (cos of the mode angle) are evaluated on the host with the
// reference's expression, and boundary-condition callbacks are sampled on the
// host once per column.
//
// Module state mirrors the reference: *_initialize{2,4} selects the order of
// a module (diffuseu, diffusew, pressure) and the functions of the other
// order refuse to run.  Where the reference calls check() and aborts (order
// mismatch, unknown boundary-condition type, zero pivot, too few rows), these
// functions leave their outputs untouched (or, for a zero pivot found on the
// device, partially written), record a status and message
// (cf_steps_status / cf_steps_message) and return.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "chanfast_steps.h"
#include "line_solve.cuh"

using namespace lines;

// ------------------------------------------------------------ constants
// rk3.c:3-6, fourth.c:3-6 (data symbols with the reference's names)
extern "C" {
const double rk3_alp[] = {29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0};
const double rk3_bet[] = {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0};
const double rk3_gam[] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
const double rk3_zet[] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
double a1 = 1.125 / 1.0;
double a2 = -0.125 / 3.0;
double b1 = 1.125 / 2.0;
double b2 = -0.125 / 2.0;
}

namespace {

// ------------------------------------------------------------ status
std::mutex g_mu;
int g_status = CF_STEPS_OK;
std::string g_message;

void fail(int status, const std::string& msg)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_status = status;
    g_message = msg;
    std::fprintf(stderr, "chanfast_steps: %s\n", msg.c_str());
}

void ok()
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_status = CF_STEPS_OK;
    g_message.clear();
}

bool cuda_ok(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return true;
    fail(CF_STEPS_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// Orders selected by the *_initialize functions (0: not initialised).
int g_order_u = 0, g_order_w = 0, g_order_p = 0;
int g_nz_u = 0, g_nz_w = 0, g_nz_p = 0;

bool need_order(int have, int want, const char* fn)
{
    if (have == want) return true;
    fail(CF_STEPS_EORDER, std::string(fn) + ": module initialised for order " + std::to_string(have)
                              + ", function needs order " + std::to_string(want));
    return false;
}

// Device copy of a host array: uploaded on construction when `in`,
// downloaded on finish() when `out`.
struct Dev {
    double* d = nullptr;
    double* h = nullptr;
    size_t n = 0;
    bool out = false;
    bool good = true;
    Dev(double* host, size_t count, bool in, bool out_)
        : h(host), n(count), out(out_)
    {
        good = cuda_ok(cudaMalloc(&d, n * sizeof(double)), "cudaMalloc");
        if (good && in) good = cuda_ok(cudaMemcpy(d, h, n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
        if (good && !in) good = cuda_ok(cudaMemset(d, 0, n * sizeof(double)), "cudaMemset");
    }
    Dev(const Dev&) = delete;
    bool finish()
    {
        if (!good) return false;
        if (out) return cuda_ok(cudaMemcpy(h, d, n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
        return true;
    }
    ~Dev()
    {
        if (d) cudaFree(d);
    }
};

bool all_good(std::initializer_list<const Dev*> v)
{
    for (const Dev* p : v)
        if (!p->good) return false;
    return true;
}

bool sync_launch(const char* fn)
{
    if (!cuda_ok(cudaGetLastError(), fn)) return false;
    return cuda_ok(cudaDeviceSynchronize(), fn);
}

// Grid geometry of one call.
struct Box {
    int n0, n1, n2, gz;
    __host__ __device__ long long at(int i, int j, int k) const { return ((long long) i * n1 + j) * n2 + k; }
    size_t size() const { return (size_t) n0 * n1 * n2; }
};

Box box_of(int local_nx, int local_ny, int nz, int gx, int gy, int gz)
{
    return Box{local_nx + 2 * gx, local_ny + 2 * gy, nz + 2 * gz, gz};
}

// One thread per (i, j, k) of [i0, i1) x [j0, j1) x [k0, k1), k fastest.
template <class F>
__global__ void k_range(int i0, int i1, int j0, int j1, int k0, int k1, F f)
{
    const long long nk = k1 - k0, nj = j1 - j0, ni = i1 - i0;
    const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ni * nj * nk) return;
    const int k = k0 + (int) (t % nk);
    const long long r = t / nk;
    const int j = j0 + (int) (r % nj);
    const int i = i0 + (int) (r / nj);
    f(i, j, k);
}

template <class F>
void launch_range(int i0, int i1, int j0, int j1, int k0, int k1, F f)
{
    if (i1 <= i0 || j1 <= j0 || k1 <= k0) return;
    const long long n = (long long) (i1 - i0) * (j1 - j0) * (k1 - k0);
    k_range<<<(unsigned) ((n + 255) / 256), 256>>>(i0, i1, j0, j1, k0, k1, f);
}

// One thread per item t in [0, n).
template <class F>
__global__ void k_items(long long n, F f)
{
    const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) f(t);
}

template <class F>
void launch_items(long long n, F f)
{
    if (n <= 0) return;
    k_items<<<(unsigned) ((n + 127) / 128), 128>>>(n, f);
}

// The fourth-order coefficients as the reference's globals hold them now.
Coef coef_now() { return Coef{::a1, ::a2, ::b1, ::b2}; }

}  // namespace

// ============================================================== band solves
//
// Column scratch: one array of n2 values per quantity and per line, stored
// [k][line] so that the threads of a warp (consecutive lines) touch
// consecutive addresses.

namespace {

// Scratch for `nl` lines of n2 rows (all quantities zeroed).
struct LineStore {
    double* base = nullptr;
    int* err = nullptr;
    Lines L{};
    bool good = false;
    LineStore(long long nl, int n2)
    {
        const size_t per = (size_t) nl * n2;
        good = cuda_ok(cudaMalloc(&base, 12 * per * sizeof(double)), "cudaMalloc") &&
               cuda_ok(cudaMalloc(&err, sizeof(int)), "cudaMalloc");
        if (!good) return;
        good = cuda_ok(cudaMemset(base, 0, 12 * per * sizeof(double)), "cudaMemset") &&
               cuda_ok(cudaMemset(err, 0, sizeof(int)), "cudaMemset");
        double* q[12];
        for (int t = 0; t < 12; t++) q[t] = base + t * per;
        L = Lines{q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], q[9], q[10], q[11], nl, err};
    }
    ~LineStore()
    {
        if (base) cudaFree(base);
        if (err) cudaFree(err);
    }
    // false (and a recorded status) when a line met a zero pivot
    bool pivots_ok(const char* fn) const
    {
        int e = 0;
        if (!cuda_ok(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost), fn)) return false;
        if (e) {
            fail(CF_STEPS_EPIVOT, std::string(fn) + ": zero pivot in a band solve");
            return false;
        }
        return true;
    }
};

}  // namespace

extern "C" {

int cf_steps_status(void)
{
    std::lock_guard<std::mutex> lock(g_mu);
    return g_status;
}

const char* cf_steps_message(void)
{
    std::lock_guard<std::mutex> lock(g_mu);
    return g_message.c_str();
}

// tridag.c:4-26, one line on the device.
void tridag(double a[], double b[], double c[], double r[], double u[], int n)
{
    if (n < 1) { fail(CF_STEPS_EINVAL, "tridag: n < 1"); return; }
    LineStore S(1, n);
    if (!S.good) return;
    Lines L = S.L;
    const size_t bytes = (size_t) n * sizeof(double);
    if (!cuda_ok(cudaMemcpy(L.a, a, bytes, cudaMemcpyHostToDevice), "tridag") ||
        !cuda_ok(cudaMemcpy(L.b, b, bytes, cudaMemcpyHostToDevice), "tridag") ||
        !cuda_ok(cudaMemcpy(L.c, c, bytes, cudaMemcpyHostToDevice), "tridag") ||
        !cuda_ok(cudaMemcpy(L.r, r, bytes, cudaMemcpyHostToDevice), "tridag"))
        return;
    launch_items(1, [=] __device__(long long l) { line_tridag(L, l, 0, n); });
    if (!sync_launch("tridag") || !S.pivots_ok("tridag")) return;
    if (cuda_ok(cudaMemcpy(u, L.x, bytes, cudaMemcpyDeviceToHost), "tridag")) ok();
}

// heptdag.c:5-61, one line on the device (h: right-hand side, x: solution).
void heptdag(double a[], double b[], double c[], double d[], double e[], double f[], double g[], double h[],
             double x[], int n)
{
    if (n < 3) { fail(CF_STEPS_EINVAL, "heptdag: n < 3"); return; }
    LineStore S(1, n);
    if (!S.good) return;
    Lines L = S.L;
    const size_t bytes = (size_t) n * sizeof(double);
    double* src[8] = {a, b, c, d, e, f, g, h};
    double* dst[8] = {L.a, L.b, L.c, L.d, L.e, L.f, L.g, L.r};
    for (int t = 0; t < 8; t++)
        if (!cuda_ok(cudaMemcpy(dst[t], src[t], bytes, cudaMemcpyHostToDevice), "heptdag")) return;
    launch_items(1, [=] __device__(long long l) { line_heptdag(L, l, 0, n); });
    if (!sync_launch("heptdag") || !S.pivots_ok("heptdag")) return;
    if (cuda_ok(cudaMemcpy(x, L.x, bytes, cudaMemcpyDeviceToHost), "heptdag")) ok();
}

}  // extern "C"

// ================================================================ advect.h

namespace {

// massflux{x,y,z}2 (advect.c:6-85): face mass fluxes averaged to the faces
// of the advected component, over i < n0-1, j < n1-1, k < n2-1.
void massflux2(int axis, double u[], double v[], double w[], double mu[], double mv[], double mw[],
               int lnx, int lny, int nz, int gx, int gy, int gz, double dx, double dy, double dz[])
{
    const Box B = box_of(lnx, lny, nz, gx, gy, gz);
    Dev U(u, B.size(), true, false), V(v, B.size(), true, false), W(w, B.size(), true, false);
    Dev MU(mu, B.size(), true, true), MV(mv, B.size(), true, true), MW(mw, B.size(), true, true);
    Dev DZ(dz, B.n2, true, false);
    if (!all_good({&U, &V, &W, &MU, &MV, &MW, &DZ})) return;
    const double *pu = U.d, *pv = V.d, *pw = W.d, *pdz = DZ.d;
    double *pmu = MU.d, *pmv = MV.d, *pmw = MW.d;
    launch_range(0, B.n0 - 1, 0, B.n1 - 1, 0, B.n2 - 1, [=] __device__(int i, int j, int k) {
        const long long ijk = B.at(i, j, k);
        const long long nb = axis == 0 ? B.at(i + 1, j, k) : (axis == 1 ? B.at(i, j + 1, k) : B.at(i, j, k + 1));
        const double dzm0 = pdz[k];
        const double dzn = axis == 2 ? pdz[k + 1] : dzm0;   // metric of the neighbour
        pmu[ijk] = 0.5 * (dy * dzm0 * pu[ijk] + dy * dzn * pu[nb]);
        pmv[ijk] = 0.5 * (dx * dzm0 * pv[ijk] + dx * dzn * pv[nb]);
        pmw[ijk] = 0.5 * (dx * dy * pw[ijk] + dx * dy * pw[nb]);
    });
    if (sync_launch("massflux2") && MU.finish() && MV.finish() && MW.finish()) ok();
}

// massflux{x,y,z}4 (advect.c:88-283): first the wall rewrite of every column
// (u, v mirrored into the first ghost row, w extrapolated into two, :100-131),
// then fourth-order interpolated fluxes over 1 <= i < n0-2, 1 <= j < n1-2,
// 1 <= k < n2-2.
void massflux4(int axis, double u[], double v[], double w[], double mu[], double mv[], double mw[],
               int lnx, int lny, int nz, int gx, int gy, int gz, double dx, double dy, double dz[])
{
    const Box B = box_of(lnx, lny, nz, gx, gy, gz);
    Dev U(u, B.size(), true, true), V(v, B.size(), true, true), W(w, B.size(), true, true);
    Dev MU(mu, B.size(), true, true), MV(mv, B.size(), true, true), MW(mw, B.size(), true, true);
    Dev DZ(dz, B.n2, true, false);
    if (!all_good({&U, &V, &W, &MU, &MV, &MW, &DZ})) return;
    double *pu = U.d, *pv = V.d, *pw = W.d, *pmu = MU.d, *pmv = MV.d, *pmw = MW.d;
    const double* pdz = DZ.d;
    const Coef cf = coef_now();
    launch_range(0, B.n0, 0, B.n1, 0, 1, [=] __device__(int i, int j, int) {
        int k = B.gz - 1;
        pu[B.at(i, j, k)] = pu[B.at(i, j, k + 1)];
        pv[B.at(i, j, k)] = pv[B.at(i, j, k + 1)];
        pw[B.at(i, j, k - 1)] = 2.0 * pw[B.at(i, j, k)] - pw[B.at(i, j, k + 1)];
        pw[B.at(i, j, k - 2)] = 2.0 * pw[B.at(i, j, k)] - pw[B.at(i, j, k + 2)];
        k = B.n2 - B.gz;
        pu[B.at(i, j, k)] = pu[B.at(i, j, k - 1)];
        pv[B.at(i, j, k)] = pv[B.at(i, j, k - 1)];
        k = B.n2 - B.gz - 1;
        pw[B.at(i, j, k + 1)] = 2.0 * pw[B.at(i, j, k)] - pw[B.at(i, j, k - 1)];
        pw[B.at(i, j, k + 2)] = 2.0 * pw[B.at(i, j, k)] - pw[B.at(i, j, k - 2)];
    });
    launch_range(1, B.n0 - 2, 1, B.n1 - 2, 1, B.n2 - 2, [=] __device__(int i, int j, int k) {
        auto nb = [&](int s) {   // neighbour s = -1, 1, 2 along the axis
            return axis == 0 ? B.at(i + s, j, k) : (axis == 1 ? B.at(i, j + s, k) : B.at(i, j, k + s));
        };
        const long long ijk = B.at(i, j, k), m1 = nb(-1), p1 = nb(1), p2 = nb(2);
        const double dzm0 = pdz[k];
        const double dzm1 = axis == 2 ? pdz[k - 1] : dzm0, dzp1 = axis == 2 ? pdz[k + 1] : dzm0,
                     dzp2 = axis == 2 ? pdz[k + 2] : dzm0;
        pmu[ijk] = cf.b1 * (dy * dzm0 * pu[ijk] + dy * dzp1 * pu[p1]) + cf.b2 * (dy * dzm1 * pu[m1] + dy * dzp2 * pu[p2]);
        pmv[ijk] = cf.b1 * (dx * dzm0 * pv[ijk] + dx * dzp1 * pv[p1]) + cf.b2 * (dx * dzm1 * pv[m1] + dx * dzp2 * pv[p2]);
        pmw[ijk] = cf.b1 * (dx * dy * pw[ijk] + dx * dy * pw[p1]) + cf.b2 * (dx * dy * pw[m1] + dx * dy * pw[p2]);
    });
    if (sync_launch("massflux4") && U.finish() && V.finish() && W.finish() && MU.finish() && MV.finish() &&
        MW.finish())
        ok();
}

// advect{u,v,w}{2,4} (advect.c:286-734): conservative flux divergence of q
// carried by the face mass fluxes (mx, my, mz); f is zeroed first.  Cell
// fields (u, v) use the wall value qbc for the wall-adjacent z fluxes; w
// lives on faces and is divided by the face volume.
template <int ORDER, bool IS_W>
void advect(double q[], double mx[], double my[], double mz[], double f[], int lnx, int lny, int nz, int gx,
            int gy, int gz, double dx, double dy, double dz[])
{
    const Box B = box_of(lnx, lny, nz, gx, gy, gz);
    Dev Q(q, B.size(), true, false), MX(mx, B.size(), true, false), MY(my, B.size(), true, false),
        MZ(mz, B.size(), true, false), Fo(f, B.size(), false, true), DZ(dz, B.n2, true, false);
    if (!all_good({&Q, &MX, &MY, &MZ, &Fo, &DZ})) return;
    const double *pq = Q.d, *px = MX.d, *py = MY.d, *pz = MZ.d, *pdz = DZ.d;
    double* pf = Fo.d;
    const Coef cf = coef_now();
    const int h = ORDER == 2 ? 1 : 3;
    const int ktop = IS_W ? B.n2 - B.gz - 1 : B.n2 - B.gz;
    launch_range(h, B.n0 - h, h, B.n1 - h, B.gz, ktop, [=] __device__(int i, int j, int k) {
        auto Qa = [&](int di, int dj, int dk) { return pq[B.at(i + di, j + dj, k + dk)]; };
        auto X = [&](int di) { return px[B.at(i + di, j, k)]; };
        auto Y = [&](int dj) { return py[B.at(i, j + dj, k)]; };
        auto Z = [&](int dk) { return pz[B.at(i, j, k + dk)]; };
        const double q0 = Qa(0, 0, 0);
        const int n2 = B.n2, g = B.gz;
        const double vol = IS_W ? dx * dy * (0.5 * (pdz[k + 1] + pdz[k])) : dx * dy * pdz[k];
        double xph = X(0) * 0.5 * (q0 + Qa(1, 0, 0));
        double yph = Y(0) * 0.5 * (q0 + Qa(0, 1, 0));
        double zph = Z(0) * 0.5 * (q0 + Qa(0, 0, 1));
        double xmh = X(-1) * 0.5 * (q0 + Qa(-1, 0, 0));
        double ymh = Y(-1) * 0.5 * (q0 + Qa(0, -1, 0));
        double zmh = Z(-1) * 0.5 * (q0 + Qa(0, 0, -1));
        if (ORDER == 2) {
            if (!IS_W) {
                // wall values 0.5 (q[g-1] + q[g]), 0.5 (q[n2-g-1] + q[n2-g])
                const double qbot = 0.5 * (Qa(0, 0, g - 1 - k) + Qa(0, 0, g - k));
                const double qtop = 0.5 * (Qa(0, 0, n2 - g - 1 - k) + Qa(0, 0, n2 - g - k));
                if (k == n2 - g - 1) zph = Z(0) * qtop;
                if (k == g) zmh = Z(-1) * qbot;
            }
            pf[B.at(i, j, k)] = -((xph - xmh) + (yph - ymh) + (zph - zmh)) / vol;
        } else {
            double xp3 = X(1) * 0.5 * (q0 + Qa(3, 0, 0));
            double yp3 = Y(1) * 0.5 * (q0 + Qa(0, 3, 0));
            double zp3 = Z(1) * 0.5 * (q0 + Qa(0, 0, 3));
            double xm3 = X(-2) * 0.5 * (q0 + Qa(-3, 0, 0));
            double ym3 = Y(-2) * 0.5 * (q0 + Qa(0, -3, 0));
            double zm3 = Z(-2) * 0.5 * (q0 + Qa(0, 0, -3));
            if (!IS_W) {
                // fourth-order wall values (advect.c:488-503)
                const int kb = g - 1, kt = n2 - g;
                const double qbot = 0.5 * cf.a2 * (Qa(0, 0, kb - 1 - k) + Qa(0, 0, kb + 2 - k))
                                  + 0.5 * (cf.a1 + 2.0 * cf.a2) * (Qa(0, 0, kb - k) + Qa(0, 0, kb + 1 - k));
                const double qtop = 0.5 * cf.a2 * (Qa(0, 0, kt - 2 - k) + Qa(0, 0, kt + 1 - k))
                                  + 0.5 * (cf.a1 + 2.0 * cf.a2) * (Qa(0, 0, kt - 1 - k) + Qa(0, 0, kt - k));
                if (k == n2 - g - 1) {
                    zph = Z(0) * qtop;
                    zp3 = -Z(-1) * 0.5 * (Qa(0, 0, -2) + Qa(0, 0, 1)) + 2.0 * Z(0) * qtop;
                }
                if (k == n2 - g - 2) zp3 = Z(1) * qtop;
                if (k == g) {
                    zmh = Z(-1) * qbot;
                    zm3 = -Z(0) * 0.5 * (Qa(0, 0, 2) + Qa(0, 0, -1)) + 2.0 * Z(-1) * qbot;
                }
                if (k == g + 1) zm3 = Z(-2) * qbot;
            }
            pf[B.at(i, j, k)] = -((cf.a1 * (xph - xmh) + cf.a2 * (xp3 - xm3)) + (cf.a1 * (yph - ymh) + cf.a2 * (yp3 - ym3))
                                  + (cf.a1 * (zph - zmh) + cf.a2 * (zp3 - zm3))) / vol;
        }
    });
    if (sync_launch("advect") && Fo.finish()) ok();
}

}  // namespace

extern "C" {

void massfluxx2(double u[], double v[], double w[], double muphx[], double mvphx[], double mwphx[], int local_nx,
                int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    massflux2(0, u, v, w, muphx, mvphx, mwphx, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void massfluxy2(double u[], double v[], double w[], double muphy[], double mvphy[], double mwphy[], int local_nx,
                int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    massflux2(1, u, v, w, muphy, mvphy, mwphy, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void massfluxz2(double u[], double v[], double w[], double muphz[], double mvphz[], double mwphz[], int local_nx,
                int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    massflux2(2, u, v, w, muphz, mvphz, mwphz, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void massfluxx4(double u[], double v[], double w[], double muphx[], double mvphx[], double mwphx[], int local_nx,
                int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    massflux4(0, u, v, w, muphx, mvphx, mwphx, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void massfluxy4(double u[], double v[], double w[], double muphy[], double mvphy[], double mwphy[], int local_nx,
                int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    massflux4(1, u, v, w, muphy, mvphy, mwphy, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void massfluxz4(double u[], double v[], double w[], double muphz[], double mvphz[], double mwphz[], int local_nx,
                int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    massflux4(2, u, v, w, muphz, mvphz, mwphz, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void advectu2(double u[], double muphx[], double mvphx[], double mwphx[], double fu[], int local_nx, int local_ny,
              int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    advect<2, false>(u, muphx, mvphx, mwphx, fu, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void advectv2(double v[], double muphy[], double mvphy[], double mwphy[], double fv[], int local_nx, int local_ny,
              int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    advect<2, false>(v, muphy, mvphy, mwphy, fv, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void advectw2(double w[], double muphz[], double mvphz[], double mwphz[], double fw[], int local_nx, int local_ny,
              int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    advect<2, true>(w, muphz, mvphz, mwphz, fw, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void advectu4(double u[], double muphx[], double mvphx[], double mwphx[], double fu[], int local_nx, int local_ny,
              int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    advect<4, false>(u, muphx, mvphx, mwphx, fu, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void advectv4(double v[], double muphy[], double mvphy[], double mwphy[], double fv[], int local_nx, int local_ny,
              int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    advect<4, false>(v, muphy, mvphy, mwphy, fv, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void advectw4(double w[], double muphz[], double mvphz[], double mwphz[], double fw[], int local_nx, int local_ny,
              int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    advect<4, true>(w, muphz, mvphz, mwphz, fw, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}

// ================================================================ scalar.h

// add_buoyancy2 (scalar.c:6-35): c averaged to the u, v faces over
// i < n0-1, j < n1-1 (interior k) and to the w faces (k < n2-g-1).
void add_buoyancy2(double c[], double fu[], double fv[], double fw[], double betg_x, double betg_y, double betg_z,
                   int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z)
{
    const Box B = box_of(local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z);
    Dev C(c, B.size(), true, false), FU(fu, B.size(), true, true), FV(fv, B.size(), true, true),
        FW(fw, B.size(), true, true);
    if (!all_good({&C, &FU, &FV, &FW})) return;
    const double* pc = C.d;
    double *pu = FU.d, *pv = FV.d, *pw = FW.d;
    launch_range(0, B.n0 - 1, 0, B.n1 - 1, B.gz, B.n2 - B.gz, [=] __device__(int i, int j, int k) {
        const long long ijk = B.at(i, j, k);
        pu[ijk] += 0.5 * (pc[ijk] + pc[B.at(i + 1, j, k)]) * betg_x;
        pv[ijk] += 0.5 * (pc[ijk] + pc[B.at(i, j + 1, k)]) * betg_y;
        if (k < B.n2 - B.gz - 1) pw[ijk] += 0.5 * (pc[ijk] + pc[B.at(i, j, k + 1)]) * betg_z;
    });
    if (sync_launch("add_buoyancy2") && FU.finish() && FV.finish() && FW.finish()) ok();
}

// add_buoyancy4 (scalar.c:38-76): fourth-order face interpolation of c over
// 1 <= i < n0-2, 1 <= j < n1-2.
void add_buoyancy4(double c[], double fu[], double fv[], double fw[], double betg_x, double betg_y, double betg_z,
                   int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z)
{
    const Box B = box_of(local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z);
    Dev C(c, B.size(), true, false), FU(fu, B.size(), true, true), FV(fv, B.size(), true, true),
        FW(fw, B.size(), true, true);
    if (!all_good({&C, &FU, &FV, &FW})) return;
    const double* pc = C.d;
    double *pu = FU.d, *pv = FV.d, *pw = FW.d;
    const Coef cf = coef_now();
    launch_range(1, B.n0 - 2, 1, B.n1 - 2, B.gz, B.n2 - B.gz, [=] __device__(int i, int j, int k) {
        auto Cv = [&](int di, int dj, int dk) { return pc[B.at(i + di, j + dj, k + dk)]; };
        const long long ijk = B.at(i, j, k);
        const double cphx = cf.b1 * (Cv(0, 0, 0) + Cv(1, 0, 0)) + cf.b2 * (Cv(-1, 0, 0) + Cv(2, 0, 0));
        const double cphy = cf.b1 * (Cv(0, 0, 0) + Cv(0, 1, 0)) + cf.b2 * (Cv(0, -1, 0) + Cv(0, 2, 0));
        pu[ijk] += cphx * betg_x;
        pv[ijk] += cphy * betg_y;
        if (k < B.n2 - B.gz - 1) {
            const double cphz = cf.b1 * (Cv(0, 0, 0) + Cv(0, 0, 1)) + cf.b2 * (Cv(0, 0, -1) + Cv(0, 0, 2));
            pw[ijk] += cphz * betg_z;
        }
    });
    if (sync_launch("add_buoyancy4") && FU.finish() && FV.finish() && FW.finish()) ok();
}

// advect_scalar (scalar.c:79-110): divergence of the scalar face fluxes over
// 1 <= i < n0, 1 <= j < n1, interior k; fc is zeroed first.
void advect_scalar(double mucphx[], double mvcphy[], double mwcphz[], double fc[], int local_nx, int local_ny,
                   int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    const Box B = box_of(local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z);
    Dev X(mucphx, B.size(), true, false), Y(mvcphy, B.size(), true, false), Z(mwcphz, B.size(), true, false),
        FC(fc, B.size(), false, true), DZ(dz, B.n2, true, false);
    if (!all_good({&X, &Y, &Z, &FC, &DZ})) return;
    const double *px = X.d, *py = Y.d, *pz = Z.d, *pdz = DZ.d;
    double* pf = FC.d;
    launch_range(1, B.n0, 1, B.n1, B.gz, B.n2 - B.gz, [=] __device__(int i, int j, int k) {
        const long long ijk = B.at(i, j, k);
        pf[ijk] = -((px[ijk] - px[B.at(i - 1, j, k)]) + (py[ijk] - py[B.at(i, j - 1, k)])
                    + (pz[ijk] - pz[B.at(i, j, k - 1)])) / (dx * dy * pdz[k]);
    });
    if (sync_launch("advect_scalar") && FC.finish()) ok();
}

// flux_quick (scalar.c:113-162): QUICK face values of c, upwinded on the sign
// of the face mass flux, times that flux, over 1 <= i < n0-2, 1 <= j < n1-2,
// 1 <= k < n2-2.
void flux_quick(double u[], double v[], double w[], double c[], double mucphx[], double mvcphy[], double mwcphz[],
                int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy,
                double dz[])
{
    const Box B = box_of(local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z);
    Dev U(u, B.size(), true, false), V(v, B.size(), true, false), W(w, B.size(), true, false),
        C(c, B.size(), true, false), X(mucphx, B.size(), true, true), Y(mvcphy, B.size(), true, true),
        Z(mwcphz, B.size(), true, true), DZ(dz, B.n2, true, false);
    if (!all_good({&U, &V, &W, &C, &X, &Y, &Z, &DZ})) return;
    const double *pu = U.d, *pv = V.d, *pw = W.d, *pc = C.d, *pdz = DZ.d;
    double *px = X.d, *py = Y.d, *pz = Z.d;
    launch_range(1, B.n0 - 2, 1, B.n1 - 2, 1, B.n2 - 2, [=] __device__(int i, int j, int k) {
        const double q = -0.125;
        auto Cv = [&](int di, int dj, int dk) { return pc[B.at(i + di, j + dj, k + dk)]; };
        const long long ijk = B.at(i, j, k);
        const double mu = dy * pdz[k] * pu[ijk];
        const double mv = dx * pdz[k] * pv[ijk];
        const double mw = dx * dy * pw[ijk];
        const double c0 = Cv(0, 0, 0);
        double cphx = 0.5 * (c0 + Cv(1, 0, 0));
        double cphy = 0.5 * (c0 + Cv(0, 1, 0));
        double cphz = 0.5 * (c0 + Cv(0, 0, 1));
        cphx += mu > 0.0 ? q * (Cv(1, 0, 0) - 2.0 * c0 + Cv(-1, 0, 0)) : q * (Cv(2, 0, 0) - 2.0 * Cv(1, 0, 0) + c0);
        cphy += mv > 0.0 ? q * (Cv(0, 1, 0) - 2.0 * c0 + Cv(0, -1, 0)) : q * (Cv(0, 2, 0) - 2.0 * Cv(0, 1, 0) + c0);
        cphz += mw > 0.0 ? q * (Cv(0, 0, 1) - 2.0 * c0 + Cv(0, 0, -1)) : q * (Cv(0, 0, 2) - 2.0 * Cv(0, 0, 1) + c0);
        px[ijk] = mu * cphx;
        py[ijk] = mv * cphy;
        pz[ijk] = mw * cphz;
    });
    if (sync_launch("flux_quick") && X.finish() && Y.finish() && Z.finish()) ok();
}

}  // extern "C"

// ============================================================ line solves

namespace {

// solve_helmholtz1d_{u,w}{2,4}: every (i, j) column of h, result in u.
void solve_1d(const char* fn, bool face, int order, double u[], double h[], int lnx, int lny, int nz, int gx, int gy,
              int gz, double dz[], double nudt, double avg_bot, double avg_top, bool nb, bool nt)
{
    const Box B = box_of(lnx, lny, nz, gx, gy, gz);
    const long long nl = (long long) B.n0 * B.n1;
    Dev U(u, B.size(), true, true), H(h, B.size(), true, false), DZ(dz, B.n2, true, false);
    if (!all_good({&U, &H, &DZ})) return;
    LineStore S(nl, B.n2);
    if (!S.good) return;
    const Lines L = S.L;
    const double *ph = H.d, *pdz = DZ.d;
    double* pu = U.d;
    const Coef cf = coef_now();
    const BandArgs BA{order, face, false, true, nudt, 0.0, 0.0, false};
    const WallSpec W{face, nb, nt, avg_bot, avg_top};
    launch_items(nl, [=] __device__(long long l) {
        const Rows R{L, l};
        const int g = B.gz, n2 = B.n2;
        const int kend = face ? n2 - g - 1 : n2 - g;
        for (int k = g; k < kend; k++) {
            double dvol;
            band_row(R, pdz, k, BA, cf, 0.0, 0.0, dvol);
            R.r(k) = ph[l * n2 + k] * dvol;
        }
        solve_line(R, L, l, pdz, g, n2, order, W, cf);
        for (int k = 0; k < n2; k++) pu[l * n2 + k] = R.x(k);
    });
    if (sync_launch(fn) && S.pivots_ok(fn) && U.finish()) ok();
}

// Modified wavenumbers of modes ix = start .. start+n-1 of an n_total grid
// (pressure.c:312-315 second order, :376-389 fourth order), evaluated on the
// host with the reference's expression.
std::vector<double> modified_wavenumbers(int order, int n_total, int start, int n, const Coef& cf)
{
    std::vector<double> lam(n);
    const double A1 = cf.a1, A2 = cf.a2;
    for (int q = 0; q < n; q++) {
        const int ix = q + start;
        const double c1 = cos(2.0 * M_PI * 1.0 * (double) ix / (double) n_total);
        if (order == 2) {
            lam[q] = 2.0 - 2.0 * c1;
        } else {
            const double c2 = cos(2.0 * M_PI * 2.0 * (double) ix / (double) n_total);
            const double c3 = cos(2.0 * M_PI * 3.0 * (double) ix / (double) n_total);
            lam[q] = (2.0 * A2 * A2 + 2.0 * A1 * A1) + (4.0 * A1 * A2 - 2.0 * A1 * A1) * c1 + (-4.0 * A1 * A2) * c2
                   + (-2.0 * A2 * A2) * c3;
        }
    }
    return lam;
}

enum SpectralKind { SPEC_HELMHOLTZ, SPEC_POISSON };

// solve_helmholtz_{u,w}{2,4} and pressure_poisson{2,4}: the Re and Im parts
// of every (kx, ky) column of the z-pencil spectrum cout[lnx][lny][n2][2].
void solve_spectral(const char* fn, SpectralKind kind, bool face, int order, double* cout, int nx, int lnx,
                    int x_start, int ny, int lny, int y_start, int nz, int gz, double dx, double dy, double dz[],
                    double t, double avg_bot, double avg_top, bool nb, bool nt)
{
    const int n2 = nz + 2 * gz;
    const long long ncol = (long long) lnx * lny;
    const long long nl = 2 * ncol;
    const Coef cf = coef_now();
    std::vector<double> lx = modified_wavenumbers(order, nx, x_start, lnx, cf);
    std::vector<double> ly = modified_wavenumbers(order, ny, y_start, lny, cf);
    Dev CO(cout, (size_t) ncol * n2 * 2, true, true), DZ(dz, n2, true, false), LX(lx.data(), lnx, true, false),
        LY(ly.data(), lny, true, false);
    if (!all_good({&CO, &DZ, &LX, &LY})) return;
    LineStore S(nl, n2);
    if (!S.good) return;
    const Lines L = S.L;
    const double *pdz = DZ.d, *plx = LX.d, *ply = LY.d;
    double* pc = CO.d;
    const BandArgs BA{order, face, true, kind == SPEC_HELMHOLTZ, t, dx, dy, true};
    launch_items(nl, [=] __device__(long long l) {
        const Rows R{L, l};
        const long long col = l >> 1;
        const int rc = (int) (l & 1);
        const int lix = (int) (col / lny), liy = (int) (col - (long long) lix * lny);
        const bool mean = lix + x_start == 0 && liy + y_start == 0;
        const int g = gz;
        const int kend = face ? n2 - g - 1 : n2 - g;
        for (int k = g; k < kend; k++) {
            double dvol;
            band_row(R, pdz, k, BA, cf, plx[lix], ply[liy], dvol);
            R.r(k) = pc[(col * n2 + k) * 2 + rc] * dvol;
        }
        WallSpec W;
        if (kind == SPEC_POISSON) {
            // mean mode: Dirichlet (value 0) at the bottom, else Neumann (pressure.c:324-331)
            W = WallSpec{false, !mean, true, 0.0, 0.0};
        } else {
            const bool m = mean && rc == 0;   // the wall values enter the mean real part only
            W = WallSpec{face, nb, nt, m ? avg_bot : 0.0, m ? avg_top : 0.0};
        }
        solve_line(R, L, l, pdz, g, n2, order, W, cf);
        for (int k = 0; k < n2; k++) pc[(col * n2 + k) * 2 + rc] = R.x(k);
    });
    if (sync_launch(fn) && S.pivots_ok(fn) && CO.finish()) ok();
}

// apply_bc_{u,w}{2,4}: ghost values of every (i, j) column from its interior
// and the wall values bc_bot(x[i], y[j]), bc_top(x[i], y[j]).
void apply_bc(const char* fn, bool face, int order, double u[], int lnx, int lny, int nz, int gx, int gy, int gz,
              double xs[], double ys[], double dz[], double (*bc_bot)(double, double),
              double (*bc_top)(double, double), bool nb, bool nt)
{
    const Box B = box_of(lnx, lny, nz, gx, gy, gz);
    const long long nl = (long long) B.n0 * B.n1;
    std::vector<double> vb(nl), vt(nl);
    for (int i = 0; i < B.n0; i++)
        for (int j = 0; j < B.n1; j++) {
            vb[(long long) i * B.n1 + j] = bc_bot(xs[i], ys[j]);
            vt[(long long) i * B.n1 + j] = bc_top(xs[i], ys[j]);
        }
    Dev U(u, B.size(), true, true), DZ(dz, B.n2, true, false), VB(vb.data(), nl, true, false),
        VT(vt.data(), nl, true, false);
    if (!all_good({&U, &DZ, &VB, &VT})) return;
    LineStore S(nl, B.n2);
    if (!S.good) return;
    const Lines L = S.L;
    const double *pdz = DZ.d, *pb = VB.d, *pt = VT.d;
    double* pu = U.d;
    const Coef cf = coef_now();
    launch_items(nl, [=] __device__(long long l) {
        const Rows R{L, l};
        const int g = B.gz, n2 = B.n2;
        for (int k = 0; k < n2; k++) R.x(k) = pu[l * n2 + k];
        const int kb = g - 1, kt = face ? n2 - g - 1 : n2 - g;
        if (order == 2) {
            if (face) {
                face_stencil2(R, kb, pb[l]);
                face_stencil2(R, kt, pt[l]);
                face_fill2(R, kb);
                face_fill2(R, kt);
            } else {
                cell_stencil_bot2(R, pdz, kb, pb[l], nb);
                cell_stencil_top2(R, pdz, kt, pt[l], nt);
                cell_fill_bot2(R, kb);
                cell_fill_top2(R, kt);
            }
        } else {
            if (face) {
                face_stencil_bot4(R, pdz, kb, pb[l], cf);
                face_stencil_top4(R, pdz, kt, pt[l], cf);
                face_fill_bot4(R, kb);
                face_fill_top4(R, kt);
            } else {
                cell_stencil_bot4(R, pdz, kb, pb[l], nb, cf);
                cell_stencil_top4(R, pdz, kt, pt[l], nt, cf);
                cell_fill_bot4(R, kb);
                cell_fill_top4(R, kt);
            }
        }
        for (int k = 0; k < n2; k++) pu[l * n2 + k] = R.x(k);
    });
    if (sync_launch(fn) && U.finish()) ok();
}

// Boundary-condition type codes of the reference headers.
constexpr int DIRICHU_ = 0, NEUMANU_ = 1, DIRICHW_ = 20;

bool cell_bctype(int t, bool& neumann, const char* fn)
{
    if (t == DIRICHU_ || t == NEUMANU_) {
        neumann = t == NEUMANU_;
        return true;
    }
    fail(CF_STEPS_EINVAL, std::string(fn) + ": boundary-condition type must be DIRICHU or NEUMANU");
    return false;
}

bool face_bctype(int t, const char* fn)
{
    if (t == DIRICHW_) return true;
    fail(CF_STEPS_EINVAL, std::string(fn) + ": boundary-condition type must be DIRICHW");
    return false;
}

}  // namespace

// ============================================================ stencil operators

namespace {

// Staggered differences of a field along one axis around point 0 (value at
// offset s given by P(s)): fourth-order face differences at +3/2, +1/2,
// -1/2, -3/2.
struct Diff4 {
    double p3, p1, m1, m3;
};
template <class P>
__device__ Diff4 diff4(P q, double A1, double A2)
{
    return Diff4{A1 * (q(2) - q(1)) + A2 * (q(3) - q(0)), A1 * (q(1) - q(0)) + A2 * (q(2) - q(-1)),
                 A1 * (q(0) - q(-1)) + A2 * (q(1) - q(-2)), A1 * (q(-1) - q(-2)) + A2 * (q(0) - q(-3))};
}
// second difference from staggered differences with face spacings hp*, hm*
// and cell spacing hc
__device__ double second4(const Diff4& D, double hp1, double hm1, double hp3, double hm3, double hc, double A1, double A2)
{
    return (A1 * (D.p1 / hp1 - D.m1 / hm1) + A2 * (D.p3 / hp3 - D.m3 / hm3)) / hc;
}
template <class P>
__device__ double second2(P q, double hp, double hm, double hc)
{
    return ((q(1) - q(0)) / hp - (q(0) - q(-1)) / hm) / hc;
}

// Which operator, for operator_kernel.
enum OpKind { OP_HELM1D, OP_LAPXY, OP_HELM3D, OP_PLAP };

// helmholtz1d_operator, add_laplacexy_operator, helmholtz_operator
// (diffuseu.c:107-459, diffusew.c:107-463) and pressure_laplacian
// (pressure.c:208-290): out = in + s (z part) / out += s (xy part) /
// out = in + s (x + y + z) / out = s (x + y + z), with s = nudt, nu or dt.
template <int ORDER, bool FACE, OpKind OP>
void stencil_op(const char* fn, double u[], double h[], int lnx, int lny, int nz, int gx, int gy, int gz, double dx,
                double dy, double dz[], double s)
{
    const Box B = box_of(lnx, lny, nz, gx, gy, gz);
    Dev U(u, B.size(), true, false), H(h, B.size(), true, true), DZ(dz, B.n2, true, false);
    if (!all_good({&U, &H, &DZ})) return;
    const double* pu = U.d;
    const double* pdz = DZ.d;
    double* ph = H.d;
    const Coef cf = coef_now();
    const int hx = OP == OP_HELM1D ? 0 : (ORDER == 2 ? 1 : 3);
    const int kend = FACE ? B.n2 - B.gz - 1 : B.n2 - B.gz;
    launch_range(hx, B.n0 - hx, hx, B.n1 - hx, B.gz, kend, [=] __device__(int i, int j, int k) {
        const double A1 = cf.a1, A2 = cf.a2;
        const long long ijk = B.at(i, j, k);
        auto X = [&](int d) { return pu[B.at(i + d, j, k)]; };
        auto Y = [&](int d) { return pu[B.at(i, j + d, k)]; };
        auto Z = [&](int d) { return pu[B.at(i, j, k + d)]; };
        // z metrics: cell fields at centres, face fields on faces
        double zx;
        if (ORDER == 2) {
            if (!FACE) zx = second2(Z, 0.5 * (pdz[k + 1] + pdz[k]), 0.5 * (pdz[k - 1] + pdz[k]), pdz[k]);
            else zx = second2(Z, pdz[k + 1], pdz[k], 0.5 * (pdz[k + 1] + pdz[k]));
        } else {
            const Diff4 D = diff4(Z, A1, A2);
            if (!FACE)
                zx = second4(D, 0.5 * (pdz[k + 1] + pdz[k]), 0.5 * (pdz[k - 1] + pdz[k]), 0.5 * (pdz[k + 2] + pdz[k + 1]),
                             0.5 * (pdz[k - 2] + pdz[k - 1]), pdz[k], A1, A2);
            else zx = second4(D, pdz[k + 1], pdz[k], pdz[k + 2], pdz[k - 1], 0.5 * (pdz[k + 1] + pdz[k]), A1, A2);
        }
        if (OP == OP_HELM1D) {
            ph[ijk] = pu[ijk] + s * zx;
            return;
        }
        double xx, yy;
        if (ORDER == 2) {
            xx = second2(X, dx, dx, dx);
            yy = second2(Y, dy, dy, dy);
        } else {
            xx = second4(diff4(X, A1, A2), dx, dx, dx, dx, dx, A1, A2);
            yy = second4(diff4(Y, A1, A2), dy, dy, dy, dy, dy, A1, A2);
        }
        if (OP == OP_LAPXY) ph[ijk] += s * (xx + yy);
        else if (OP == OP_HELM3D) ph[ijk] = pu[ijk] + s * (xx + yy + zx);
        else ph[ijk] = s * (xx + yy + zx);
    });
    if (sync_launch(fn) && H.finish()) ok();
}

// divergence{2,4} (pressure.c:40-117); the fourth-order form first
// extrapolates w into the ghost faces below and above (in place).
template <int ORDER>
void divergence(double u[], double v[], double w[], double d[], int lnx, int lny, int nz, int gx, int gy, int gz,
                double dx, double dy, double dz[])
{
    const Box B = box_of(lnx, lny, nz, gx, gy, gz);
    Dev U(u, B.size(), true, false), V(v, B.size(), true, false), W(w, B.size(), true, ORDER == 4),
        Dd(d, B.size(), true, true), DZ(dz, B.n2, true, false);
    if (!all_good({&U, &V, &W, &Dd, &DZ})) return;
    const double *pu = U.d, *pv = V.d, *pdz = DZ.d;
    double *pw = W.d, *pd = Dd.d;
    const Coef cf = coef_now();
    if (ORDER == 4)
        launch_range(0, B.n0, 0, B.n1, 0, 1, [=] __device__(int i, int j, int) {
            int k = B.gz - 1;
            pw[B.at(i, j, k - 1)] = 2.0 * pw[B.at(i, j, k)] - pw[B.at(i, j, k + 1)];
            k = B.n2 - B.gz - 1;
            pw[B.at(i, j, k + 1)] = 2.0 * pw[B.at(i, j, k)] - pw[B.at(i, j, k - 1)];
        });
    const int lo = ORDER == 2 ? 1 : 2, hi = ORDER == 2 ? 0 : 1;
    launch_range(lo, B.n0 - hi, lo, B.n1 - hi, B.gz, B.n2 - B.gz, [=] __device__(int i, int j, int k) {
        const long long ijk = B.at(i, j, k);
        auto Ux = [&](int s) { return pu[B.at(i + s, j, k)]; };
        auto Vy = [&](int s) { return pv[B.at(i, j + s, k)]; };
        auto Wz = [&](int s) { return pw[B.at(i, j, k + s)]; };
        if (ORDER == 2)
            pd[ijk] = (Ux(0) - Ux(-1)) / dx + (Vy(0) - Vy(-1)) / dy + (Wz(0) - Wz(-1)) / pdz[k];
        else
            pd[ijk] = (cf.a1 * (Ux(0) - Ux(-1)) + cf.a2 * (Ux(1) - Ux(-2))) / dx
                    + (cf.a1 * (Vy(0) - Vy(-1)) + cf.a2 * (Vy(1) - Vy(-2))) / dy
                    + (cf.a1 * (Wz(0) - Wz(-1)) + cf.a2 * (Wz(1) - Wz(-2))) / pdz[k];
    });
    if (sync_launch("divergence") && W.finish() && Dd.finish()) ok();
}

// project{2,4} (pressure.c:120-205): u, v over the interior rows, w over the
// faces from the bottom wall face up.
template <int ORDER>
void project(double u[], double v[], double w[], double p[], int lnx, int lny, int nz, int gx, int gy, int gz,
             double dx, double dy, double dz[], double dt)
{
    const Box B = box_of(lnx, lny, nz, gx, gy, gz);
    Dev U(u, B.size(), true, true), V(v, B.size(), true, true), W(w, B.size(), true, true),
        P(p, B.size(), true, false), DZ(dz, B.n2, true, false);
    if (!all_good({&U, &V, &W, &P, &DZ})) return;
    const double *pp = P.d, *pdz = DZ.d;
    double *pu = U.d, *pv = V.d, *pw = W.d;
    const Coef cf = coef_now();
    const int lo = ORDER == 2 ? 0 : 1, hi = ORDER == 2 ? 1 : 2;
    launch_range(lo, B.n0 - hi, lo, B.n1 - hi, B.gz - 1, B.n2 - B.gz, [=] __device__(int i, int j, int k) {
        const long long ijk = B.at(i, j, k);
        auto Px = [&](int s) { return pp[B.at(i + s, j, k)]; };
        auto Py = [&](int s) { return pp[B.at(i, j + s, k)]; };
        auto Pz = [&](int s) { return pp[B.at(i, j, k + s)]; };
        if (k >= B.gz) {
            if (ORDER == 2) {
                pu[ijk] -= (Px(1) - Px(0)) * dt / dx;
                pv[ijk] -= (Py(1) - Py(0)) * dt / dy;
            } else {
                const double up1h = cf.a1 * (Px(1) - Px(0)) + cf.a2 * (Px(2) - Px(-1));
                const double vp1h = cf.a1 * (Py(1) - Py(0)) + cf.a2 * (Py(2) - Py(-1));
                pu[ijk] -= up1h * dt / dx;
                pv[ijk] -= vp1h * dt / dy;
            }
        }
        const double dzp1h = 0.5 * (pdz[k + 1] + pdz[k]);
        if (ORDER == 2) pw[ijk] -= (Pz(1) - Pz(0)) * dt / dzp1h;
        else pw[ijk] -= (cf.a1 * (Pz(1) - Pz(0)) + cf.a2 * (Pz(2) - Pz(-1))) * dt / dzp1h;
    });
    if (sync_launch("project") && U.finish() && V.finish() && W.finish()) ok();
}

bool init_module(int& order_slot, int& nz_slot, int order, int nz, int gz, const char* fn)
{
    const int min_nz = order == 2 ? 2 : 6, min_g = order == 2 ? 1 : 3;
    if (nz < min_nz || gz < min_g) {
        fail(CF_STEPS_EINVAL, std::string(fn) + ": needs nz >= " + std::to_string(min_nz) + " and nghost_z >= "
                                  + std::to_string(min_g));
        return false;
    }
    order_slot = order;
    nz_slot = nz;
    ok();
    return true;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- diffuseu.h

void diffuseu_initialize2(int nz, int nghost_z) { init_module(g_order_u, g_nz_u, 2, nz, nghost_z, "diffuseu_initialize2"); }
void diffuseu_initialize4(int nz, int nghost_z) { init_module(g_order_u, g_nz_u, 4, nz, nghost_z, "diffuseu_initialize4"); }
void diffuseu_finalize2(void) { if (need_order(g_order_u, 2, "diffuseu_finalize2")) ok(); }
void diffuseu_finalize4(void) { if (need_order(g_order_u, 4, "diffuseu_finalize4")) ok(); }

#define CF_APPLY_BC(NAME, FACE, ORD, MOD)                                                                          \
    void NAME(double u[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double xs[], \
              double ys[], double dz[], double (*bc_bot)(double, double), double (*bc_top)(double, double),         \
              int bctype_bot, int bctype_top)                                                                       \
    {                                                                                                               \
        if (!need_order(MOD, ORD, #NAME)) return;                                                                   \
        bool nb = false, nt = false;                                                                                \
        if (FACE) {                                                                                                 \
            if (!face_bctype(bctype_bot, #NAME) || !face_bctype(bctype_top, #NAME)) return;                         \
        } else if (!cell_bctype(bctype_bot, nb, #NAME) || !cell_bctype(bctype_top, nt, #NAME)) {                    \
            return;                                                                                                 \
        }                                                                                                           \
        apply_bc(#NAME, FACE, ORD, u, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, xs, ys, dz, bc_bot,     \
                 bc_top, nb, nt);                                                                                   \
    }

// apply_bc_u{2,4} (diffuseu.c:37-104), apply_bc_w{2,4} (diffusew.c:37-104)
CF_APPLY_BC(apply_bc_u2, false, 2, g_order_u)
CF_APPLY_BC(apply_bc_u4, false, 4, g_order_u)
CF_APPLY_BC(apply_bc_w2, true, 2, g_order_w)
CF_APPLY_BC(apply_bc_w4, true, 4, g_order_w)
#undef CF_APPLY_BC

#define CF_SOLVE1D(NAME, FACE, ORD, MOD)                                                                           \
    void NAME(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, \
              double dz[], double nudt, double avg_bot, double avg_top, int bctype_bot, int bctype_top)             \
    {                                                                                                               \
        if (!need_order(MOD, ORD, #NAME)) return;                                                                   \
        bool nb = false, nt = false;                                                                                \
        if (FACE) {                                                                                                 \
            if (!face_bctype(bctype_bot, #NAME) || !face_bctype(bctype_top, #NAME)) return;                         \
        } else if (!cell_bctype(bctype_bot, nb, #NAME) || !cell_bctype(bctype_top, nt, #NAME)) {                    \
            return;                                                                                                 \
        }                                                                                                           \
        solve_1d(#NAME, FACE, ORD, u, h, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dz, nudt, avg_bot,   \
                 avg_top, nb, nt);                                                                                  \
    }

// solve_helmholtz1d_u{2,4} (diffuseu.c:173-283), _w{2,4} (diffusew.c:175-287)
CF_SOLVE1D(solve_helmholtz1d_u2, false, 2, g_order_u)
CF_SOLVE1D(solve_helmholtz1d_u4, false, 4, g_order_u)
CF_SOLVE1D(solve_helmholtz1d_w2, true, 2, g_order_w)
CF_SOLVE1D(solve_helmholtz1d_w4, true, 4, g_order_w)
#undef CF_SOLVE1D

#define CF_SOLVE3D(NAME, FACE, ORD, MOD)                                                                           \
    void NAME(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny, int local_y_start, \
              int nz, int nghost_z, double dx, double dy, double dz[], double nudt, double avg_bot, double avg_top, \
              int bctype_bot, int bctype_top)                                                                       \
    {                                                                                                               \
        if (!need_order(MOD, ORD, #NAME)) return;                                                                   \
        bool nb = false, nt = false;                                                                                \
        if (FACE) {                                                                                                 \
            if (!face_bctype(bctype_bot, #NAME) || !face_bctype(bctype_top, #NAME)) return;                         \
        } else if (!cell_bctype(bctype_bot, nb, #NAME) || !cell_bctype(bctype_top, nt, #NAME)) {                    \
            return;                                                                                                 \
        }                                                                                                           \
        solve_spectral(#NAME, SPEC_HELMHOLTZ, FACE, ORD, &cout[0][0], nx, local_nx, local_x_start, ny, local_ny,    \
                       local_y_start, nz, nghost_z, dx, dy, dz, nudt, avg_bot, avg_top, nb, nt);                    \
    }

// solve_helmholtz_u{2,4} (diffuseu.c:460-569), _w{2,4} (diffusew.c:466-552)
CF_SOLVE3D(solve_helmholtz_u2, false, 2, g_order_u)
CF_SOLVE3D(solve_helmholtz_u4, false, 4, g_order_u)
CF_SOLVE3D(solve_helmholtz_w2, true, 2, g_order_w)
CF_SOLVE3D(solve_helmholtz_w4, true, 4, g_order_w)
#undef CF_SOLVE3D

#define CF_OP_Z(NAME, FACE, ORD, MOD)                                                                              \
    void NAME(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, \
              double dz[], double nudt)                                                                             \
    {                                                                                                               \
        if (!need_order(MOD, ORD, #NAME)) return;                                                                   \
        stencil_op<ORD, FACE, OP_HELM1D>(#NAME, u, h, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, 0.0,    \
                                         0.0, dz, nudt);                                                            \
    }
// helmholtz1d_operator_u{2,4} (diffuseu.c:107-170), _w{2,4} (diffusew.c:107-172)
CF_OP_Z(helmholtz1d_operator_u2, false, 2, g_order_u)
CF_OP_Z(helmholtz1d_operator_u4, false, 4, g_order_u)
CF_OP_Z(helmholtz1d_operator_w2, true, 2, g_order_w)
CF_OP_Z(helmholtz1d_operator_w4, true, 4, g_order_w)
#undef CF_OP_Z

#define CF_OP_XY(NAME, FACE, ORD, MOD)                                                                             \
    void NAME(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, \
              double dx, double dy, double nu)                                                                      \
    {                                                                                                               \
        if (!need_order(MOD, ORD, #NAME)) return;                                                                   \
        const int n2 = nz + 2 * nghost_z;                                                                           \
        std::vector<double> dz1(n2, 1.0); /* no z part: any positive metric */                                      \
        stencil_op<ORD, FACE, OP_LAPXY>(#NAME, u, h, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy,  \
                                        dz1.data(), nu);                                                            \
    }
// add_laplacexy_operator_u{2,4} (diffuseu.c:286-359), _w{2,4} (diffusew.c:290-363)
CF_OP_XY(add_laplacexy_operator_u2, false, 2, g_order_u)
CF_OP_XY(add_laplacexy_operator_u4, false, 4, g_order_u)
CF_OP_XY(add_laplacexy_operator_w2, true, 2, g_order_w)
CF_OP_XY(add_laplacexy_operator_w4, true, 4, g_order_w)
#undef CF_OP_XY

#define CF_OP_3D(NAME, FACE, ORD, MOD)                                                                             \
    void NAME(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, \
              double dx, double dy, double dz[], double nudt)                                                       \
    {                                                                                                               \
        if (!need_order(MOD, ORD, #NAME)) return;                                                                   \
        stencil_op<ORD, FACE, OP_HELM3D>(#NAME, u, h, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, \
                                         dz, nudt);                                                                 \
    }
// helmholtz_operator_u{2,4} (diffuseu.c:362-457), _w{2,4} (diffusew.c:366-463)
CF_OP_3D(helmholtz_operator_u2, false, 2, g_order_u)
CF_OP_3D(helmholtz_operator_u4, false, 4, g_order_u)
CF_OP_3D(helmholtz_operator_w2, true, 2, g_order_w)
CF_OP_3D(helmholtz_operator_w4, true, 4, g_order_w)
#undef CF_OP_3D

// ---------------------------------------------------------------- diffusew.h

void diffusew_initialize2(int nz, int nghost_z) { init_module(g_order_w, g_nz_w, 2, nz, nghost_z, "diffusew_initialize2"); }
void diffusew_initialize4(int nz, int nghost_z) { init_module(g_order_w, g_nz_w, 4, nz, nghost_z, "diffusew_initialize4"); }
void diffusew_finalize2(void) { if (need_order(g_order_w, 2, "diffusew_finalize2")) ok(); }
void diffusew_finalize4(void) { if (need_order(g_order_w, 4, "diffusew_finalize4")) ok(); }

// ---------------------------------------------------------------- pressure.h

void pressure_initialize2(int nz, int nghost_z) { init_module(g_order_p, g_nz_p, 2, nz, nghost_z, "pressure_initialize2"); }
void pressure_initialize4(int nz, int nghost_z) { init_module(g_order_p, g_nz_p, 4, nz, nghost_z, "pressure_initialize4"); }
void pressure_finalize2(void) { if (need_order(g_order_p, 2, "pressure_finalize2")) ok(); }
void pressure_finalize4(void) { if (need_order(g_order_p, 4, "pressure_finalize4")) ok(); }

void divergence2(double u[], double v[], double w[], double d[], int local_nx, int local_ny, int nz, int nghost_x,
                 int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    if (need_order(g_order_p, 2, "divergence2"))
        divergence<2>(u, v, w, d, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void divergence4(double u[], double v[], double w[], double d[], int local_nx, int local_ny, int nz, int nghost_x,
                 int nghost_y, int nghost_z, double dx, double dy, double dz[])
{
    if (need_order(g_order_p, 4, "divergence4"))
        divergence<4>(u, v, w, d, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz);
}
void project2(double u[], double v[], double w[], double p[], int local_nx, int local_ny, int nz, int nghost_x,
              int nghost_y, int nghost_z, double dx, double dy, double dz[], double dt)
{
    if (need_order(g_order_p, 2, "project2"))
        project<2>(u, v, w, p, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz, dt);
}
void project4(double u[], double v[], double w[], double p[], int local_nx, int local_ny, int nz, int nghost_x,
              int nghost_y, int nghost_z, double dx, double dy, double dz[], double dt)
{
    if (need_order(g_order_p, 4, "project4"))
        project<4>(u, v, w, p, local_nx, local_ny, nz, nghost_x, nghost_y, nghost_z, dx, dy, dz, dt);
}
void pressure_laplacian2(double p[], double l[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y,
                         int nghost_z, double dx, double dy, double dz[], double dt)
{
    if (need_order(g_order_p, 2, "pressure_laplacian2"))
        stencil_op<2, false, OP_PLAP>("pressure_laplacian2", p, l, local_nx, local_ny, nz, nghost_x, nghost_y,
                                      nghost_z, dx, dy, dz, dt);
}
void pressure_laplacian4(double p[], double l[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y,
                         int nghost_z, double dx, double dy, double dz[], double dt)
{
    if (need_order(g_order_p, 4, "pressure_laplacian4"))
        stencil_op<4, false, OP_PLAP>("pressure_laplacian4", p, l, local_nx, local_ny, nz, nghost_x, nghost_y,
                                      nghost_z, dx, dy, dz, dt);
}
void pressure_poisson2(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny,
                       int local_y_start, int nz, int nghost_z, double dx, double dy, double dz[], double dt)
{
    if (need_order(g_order_p, 2, "pressure_poisson2"))
        solve_spectral("pressure_poisson2", SPEC_POISSON, false, 2, &cout[0][0], nx, local_nx, local_x_start, ny,
                       local_ny, local_y_start, nz, nghost_z, dx, dy, dz, dt, 0.0, 0.0, true, true);
}
void pressure_poisson4(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny,
                       int local_y_start, int nz, int nghost_z, double dx, double dy, double dz[], double dt)
{
    if (need_order(g_order_p, 4, "pressure_poisson4"))
        solve_spectral("pressure_poisson4", SPEC_POISSON, false, 4, &cout[0][0], nx, local_nx, local_x_start, ny,
                       local_ny, local_y_start, nz, nghost_z, dx, dy, dz, dt, 0.0, 0.0, true, true);
}

}  // extern "C"
