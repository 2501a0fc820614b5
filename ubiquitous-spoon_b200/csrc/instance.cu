// Instance management and the C ABI of libchanfast_cuda.so.
//
// One cf_instance = one channel-flow state resident in device memory plus
// the per-substep coefficient sets.  cf_step issues, per RK3 substep, the
// kernel sequence that replaces the body of chanfast.c:395-656 (order 2) /
// 1319-1580 (order 4):
//   ghosts -> rhs -> solve u -> mass control u -> solve v -> solve c ->
//   scalar-mean control c -> solve w -> divergence+x FFT -> y FFT ->
//   Poisson -> inverse y FFT -> inverse x FFT -> projection
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cctype>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "chanfast_cuda.h"
#include "engine.cuh"
#include "batch.cuh"
#include "host_band.h"

using namespace cf;

namespace {

thread_local std::string g_last_error;

#define CF_CUDA(call)                                                                 \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);        \
            return e_ == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA;            \
        }                                                                             \
    } while (0)

// ------------------------------------------------------------ utility kernels

constexpr unsigned long long GOLDEN = 0x9E3779B97F4A7C15ull;

__device__ __forceinline__ double uniform_pm1(unsigned long long key, unsigned long long idx)
{
    // SplitMix64 output function of (key | idx); xi in [-1, 1)
    unsigned long long z = (key | idx) + GOLDEN;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    double m = (double) (z >> 11);
    return m * 0x1p-53 * 2.0 - 1.0;
}

__global__ void k_init_raw(Geo G, double* u, double* v, double* w, double* c, const double* zp,
                           unsigned long long seed, double amp, double c_amp)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    const int k = blockIdx.z;
    if (j >= G.ny) return;
    const long long d = ((long long) k * G.nx + i) * G.ny + j;
    const int iz = k - GZ;
    if (iz < 0 || iz >= G.nz) {
        u[d] = 0.0; v[d] = 0.0; w[d] = 0.0; c[d] = 0.0;
        return;
    }
    const unsigned long long gidx = ((unsigned long long) i * G.ny + j) * G.nz + iz;
    const double ucl = 1.5;
    const double z = zp[k];
    double xu = uniform_pm1((seed * 4 + 0) << 40, gidx);
    double xv = uniform_pm1((seed * 4 + 1) << 40, gidx);
    double xw = uniform_pm1((seed * 4 + 2) << 40, gidx);
    double xc = uniform_pm1((seed * 4 + 3) << 40, gidx);
    u[d] = 1.5 * (1.0 - (z - 1.0) * (z - 1.0)) + amp * ucl * xu;
    v[d] = amp * ucl * xv;
    w[d] = iz == G.nz - 1 ? 0.0 : amp * ucl * xw;   // face n2-gz-1 is the top wall
    c[d] = -0.5 + z / 2.0 + c_amp * xc;
}

// Host layout [A][B][K] (A = nx + 2 ox, B = ny + 2 oy, K rows starting at
// device row oz)  <->  device layout [n2][nx][ny].
__global__ void k_host2dev(Geo G, const double* __restrict__ src, double* __restrict__ dst,
                           int B, int K, int ox, int oy, int oz)
{
    __shared__ double tile[32][33];
    const int k0 = blockIdx.x * 32, j0 = blockIdx.y * 32, i = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int jj = ty; jj < 32; jj += 8) {
        int j = j0 + jj, kk = k0 + tx;
        if (j < G.ny && kk < K) tile[jj][tx] = src[((long long) (i + ox) * B + (j + oy)) * K + kk];
    }
    __syncthreads();
    for (int kq = ty; kq < 32; kq += 8) {
        int kk = k0 + kq, j = j0 + tx;
        if (j < G.ny && kk < K) dst[((long long) (kk + oz) * G.nx + i) * G.ny + j] = tile[tx][kq];
    }
}

__global__ void k_dev2host(Geo G, const double* __restrict__ src, double* __restrict__ dst,
                           int A, int B, int K, int ox, int oy, int oz)
{
    __shared__ double tile[32][33];
    const int k0 = blockIdx.x * 32, b0 = blockIdx.y * 32, a = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    int i = a - ox;
    i = ((i % G.nx) + G.nx) % G.nx;
    for (int kq = ty; kq < 32; kq += 8) {
        int kk = k0 + kq, b = b0 + tx;
        if (b < B && kk < K) {
            int j = ((b - oy) % G.ny + G.ny) % G.ny;
            tile[kq][tx] = src[((long long) (kk + oz) * G.nx + i) * G.ny + j];
        }
    }
    __syncthreads();
    for (int bb = ty; bb < 32; bb += 8) {
        int b = b0 + bb, kk = k0 + tx;
        if (b < B && kk < K) dst[((long long) a * B + b) * K + kk] = tile[tx][bb];
    }
    (void) A;
}

template <int ORDER>
__global__ void k_max_div(Geo G, const double* u, const double* v, const double* w, double* blockmax)
{
    __shared__ double red[256];
    const int nx = G.nx, ny = G.ny, n2 = G.n2;
    double m = 0.0;
    const long long total = (long long) G.nz * G.plane;
    for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long) gridDim.x * blockDim.x) {
        int k = GZ + (int) (t / G.plane);
        long long rem = t - (long long) (k - GZ) * G.plane;
        int i = (int) (rem / ny), j = (int) (rem - (long long) i * ny);
        auto I = [&](int kk, int ii, int jj) {
            ii = ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii);
            jj = jj < 0 ? jj + ny : (jj >= ny ? jj - ny : jj);
            return ((long long) kk * nx + ii) * ny + jj;
        };
        double d;
        if (ORDER == 2) {
            d = (u[I(k, i, j)] - u[I(k, i - 1, j)]) / G.dx + (v[I(k, i, j)] - v[I(k, i, j - 1)]) / G.dy
              + (w[I(k, i, j)] - w[I(k - 1, i, j)]) / G.dz[k];
        } else {
            const int kb = GZ - 1, kt = n2 - GZ - 1;
            double wkm2 = (k - 2 == kb - 1) ? 2.0 * w[I(kb, i, j)] - w[I(kb + 1, i, j)] : w[I(k - 2, i, j)];
            double wkp1 = (k + 1 == kt + 1) ? 2.0 * w[I(kt, i, j)] - w[I(kt - 1, i, j)] : w[I(k + 1, i, j)];
            d = (A1 * (u[I(k, i, j)] - u[I(k, i - 1, j)]) + A2 * (u[I(k, i + 1, j)] - u[I(k, i - 2, j)])) / G.dx
              + (A1 * (v[I(k, i, j)] - v[I(k, i, j - 1)]) + A2 * (v[I(k, i, j + 1)] - v[I(k, i, j - 2)])) / G.dy
              + (A1 * (w[I(k, i, j)] - w[I(k - 1, i, j)]) + A2 * (wkp1 - wkm2)) / G.dz[k];
        }
        m = fmax(m, fabs(d));
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) blockmax[blockIdx.x] = red[0];
}

// get_cfl (get.c:390-416) over interior cells
__global__ void k_cfl(Geo G, const double* u, const double* v, const double* w, double dt, double* blockmax)
{
    __shared__ double red[256];
    double m = 0.0;
    const long long total = (long long) G.nz * G.plane;
    for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long) gridDim.x * blockDim.x) {
        int k = GZ + (int) (t / G.plane);
        long long d = (long long) GZ * G.plane + t;
        double dzph = 0.5 * (G.dz[k] + G.dz[k + 1]);
        double c;
        if (m < (c = fabs(u[d]) * dt / G.dx)) m = c;
        if (m < (c = fabs(v[d]) * dt / G.dy)) m = c;
        if (m < (c = fabs(w[d]) * dt / dzph)) m = c;
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) blockmax[blockIdx.x] = red[0];
}

// ---- cf_max_divergence_noalloc -------------------------------------------
// Scratch of the allocation-free divergence check: one partial maximum per
// interior k-plane plus one result slot, in file-scope device memory.  Every
// GPU that loads this library holds these 64 KiB until the process exits.
constexpr int CF_NOALLOC_MAX_ROWS = 8191;
static __device__ __align__(256) double g_divmax_rows[CF_NOALLOC_MAX_ROWS + 1];

// Same per-point operator as k_max_div (divergence{2,4}, pressure.c:40-117);
// block b reduces interior plane k = GZ + b into rowmax[b].
template <int ORDER>
__global__ void k_max_div_rows(Geo G, const double* u, const double* v, const double* w, double* rowmax)
{
    __shared__ double red[256];
    const int nx = G.nx, ny = G.ny, n2 = G.n2;
    const int k = GZ + blockIdx.x;
    double m = 0.0;
    for (long long t = threadIdx.x; t < G.plane; t += blockDim.x) {
        int i = (int) (t / ny), j = (int) (t - (long long) i * ny);
        auto I = [&](int kk, int ii, int jj) {
            ii = ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii);
            jj = jj < 0 ? jj + ny : (jj >= ny ? jj - ny : jj);
            return ((long long) kk * nx + ii) * ny + jj;
        };
        double d;
        if (ORDER == 2) {
            d = (u[I(k, i, j)] - u[I(k, i - 1, j)]) / G.dx + (v[I(k, i, j)] - v[I(k, i, j - 1)]) / G.dy
              + (w[I(k, i, j)] - w[I(k - 1, i, j)]) / G.dz[k];
        } else {
            const int kb = GZ - 1, kt = n2 - GZ - 1;
            double wkm2 = (k - 2 == kb - 1) ? 2.0 * w[I(kb, i, j)] - w[I(kb + 1, i, j)] : w[I(k - 2, i, j)];
            double wkp1 = (k + 1 == kt + 1) ? 2.0 * w[I(kt, i, j)] - w[I(kt - 1, i, j)] : w[I(k + 1, i, j)];
            d = (A1 * (u[I(k, i, j)] - u[I(k, i - 1, j)]) + A2 * (u[I(k, i + 1, j)] - u[I(k, i - 2, j)])) / G.dx
              + (A1 * (v[I(k, i, j)] - v[I(k, i, j - 1)]) + A2 * (v[I(k, i, j + 1)] - v[I(k, i, j - 2)])) / G.dy
              + (A1 * (w[I(k, i, j)] - w[I(k - 1, i, j)]) + A2 * (wkp1 - wkm2)) / G.dz[k];
        }
        m = fmax(m, fabs(d));
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) rowmax[blockIdx.x] = red[0];
}

__global__ void k_max_rows_final(const double* rowmax, int n, double* result)
{
    __shared__ double red[256];
    double m = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) m = fmax(m, rowmax[t]);
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *result = red[0];
}

// ----------------------------------------------------------- statistics
//
// Plane statistics of get.c on the device, one block per row k, fixed
// summation order (the reference sums serially, so they agree to rounding):
// mode 0 the mean of a (get_xy_avg, :281-302), mode 1 the mean of
// (a - abar)(b - bbar) (get_xy_corr, :132-172), mode 2 the mean of
// pow(a - abar, en) (get_xy_moment, :94-129).
__global__ void k_row_stat(Geo G, const double* __restrict__ a, const double* __restrict__ b,
                           const double* __restrict__ abar, const double* __restrict__ bbar, int mode, double en,
                           double* __restrict__ out)
{
    __shared__ double red[256];
    const int k = blockIdx.x;
    const long long P = G.plane;
    const double* ak = a + k * P;
    const double* bk = b ? b + k * P : nullptr;
    const double am = abar ? abar[k] : 0.0, bm = bbar ? bbar[k] : 0.0;
    double s = 0.0;
    for (long long c = threadIdx.x; c < P; c += blockDim.x) {
        const double x = ak[c];
        if (mode == 0) s += x;
        else if (mode == 1) s += (x - am) * (bk[c] - bm);
        else s += pow(x - am, en);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = red[0] * (1.0 / ((double) G.nx * (double) G.ny));
}

// Cross spectrum of one column: Re, Im of uhat conj(vhat) (get.c:26-31).
__device__ __forceinline__ double2 cross(const double2 u, const double2 v)
{
    return make_double2(u.x * v.x + u.y * v.y, u.y * v.x - u.x * v.y);
}

// get_xy_spec (get.c:5-91), x spectrum: specx[ix][k] = sum over iy of the
// cross spectrum, the (0, 0) mode left out.  One block per (ix, k).
__global__ void k_specx(Geo G, const double2* __restrict__ uh, const double2* __restrict__ vh,
                        double* __restrict__ specx)
{
    __shared__ double2 red[256];
    const int ix = blockIdx.x, k = blockIdx.y, ny = G.ny;
    const long long base = ((long long) k * G.nkx + ix) * ny;
    double2 s = make_double2(0.0, 0.0);
    for (int iy = threadIdx.x; iy < ny; iy += blockDim.x) {
        if (ix == 0 && iy == 0) continue;
        const double2 c = cross(uh[base + iy], vh[base + iy]);
        s.x += c.x;
        s.y += c.y;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) {
            red[threadIdx.x].x += red[threadIdx.x + o].x;
            red[threadIdx.x].y += red[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        specx[((long long) ix * G.n2 + k) * 2] = red[0].x;
        specx[((long long) ix * G.n2 + k) * 2 + 1] = red[0].y;
    }
}

// y spectrum: specy[iy][k], iy in [0, ny/2], sums over ix the column iy and,
// for the modes whose conjugate column is not stored (0 < ix, except
// ix = nx/2 with nx even), the column ny - iy with its imaginary part
// negated; ix = 0 contributes for iy > 0 only.  One block per (iy, k).
__global__ void k_specy(Geo G, const double2* __restrict__ uh, const double2* __restrict__ vh,
                        double* __restrict__ specy)
{
    __shared__ double2 red[256];
    const int iyt = blockIdx.x, k = blockIdx.y, nx = G.nx, ny = G.ny, nkx = G.nkx;
    const int iyc = (ny - iyt) % ny;
    double2 s = make_double2(0.0, 0.0);
    for (int ix = threadIdx.x; ix < nkx; ix += blockDim.x) {
        const long long base = ((long long) k * nkx + ix) * ny;
        if (ix == 0) {
            if (iyt > 0) {
                const double2 c = cross(uh[base + iyt], vh[base + iyt]);
                s.x += c.x;
                s.y += c.y;
            }
        } else if (nx % 2 == 0 && ix == nx / 2) {
            const double2 c = cross(uh[base + iyt], vh[base + iyt]);
            s.x += c.x;
            s.y += c.y;
        } else {
            const double2 c = cross(uh[base + iyt], vh[base + iyt]);
            const double2 d = cross(uh[base + iyc], vh[base + iyc]);
            s.x += c.x + d.x;
            s.y += c.y - d.y;
        }
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) {
            red[threadIdx.x].x += red[threadIdx.x + o].x;
            red[threadIdx.x].y += red[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        specy[((long long) iyt * G.n2 + k) * 2] = red[0].x;
        specy[((long long) iyt * G.n2 + k) * 2 + 1] = red[0].y;
    }
}

// ------------------------------------------------------------ host helpers

// Packs host vectors into one device allocation.
struct Arena {
    std::vector<double> h;
    size_t add(const std::vector<double>& v)
    {
        size_t off = h.size();
        h.insert(h.end(), v.begin(), v.end());
        while (h.size() % 4) h.push_back(0.0);  // 32-byte alignment of every table
        return off;
    }
};

WallRowsD to_dev(const WallRows& w)
{
    WallRowsD d;
    std::memcpy(d.row, w.row, sizeof(d.row));
    return d;
}

std::vector<int> fft_radices(int n)
{
    std::vector<int> r;
    while (n % 8 == 0 && n > 8) { r.push_back(8); n /= 8; }
    if (n == 8) { r.push_back(8); n = 1; }
    while (n % 4 == 0) { r.push_back(4); n /= 4; }
    while (n % 2 == 0) { r.push_back(2); n /= 2; }
    while (n % 3 == 0) { r.push_back(3); n /= 3; }
    while (n % 5 == 0) { r.push_back(5); n /= 5; }
    if (n != 1) r.clear();
    return r;
}

}  // namespace

struct SetOffsets {
    size_t F1, F2, F3, DEN, P, Q, R, hbc, green, rows;
    int k0, n;
    WallRowsD bot, top;
    double gstats[4];
};

struct PoissonOffsets {
    size_t a, b, c, e, f, g, dpart, dvol, cx, cy;
    PoissonSet host;
};

struct cf_instance {
    cf_config cfg;
    Metrics m;
    Geo geo;
    // y transforms fused with the Poisson solve (k_poisson_fft, ny = 256 or
    // 512): by default where its one block per kx gives the GPU enough
    // blocks (nx/2 + 1 at least half the SM count); CF_FUSE_PRESSURE=1 at
    // creation fuses wherever supported, CF_FUSE_PRESSURE=0 never
    bool fuse_pressure = true;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double *u = nullptr, *v = nullptr, *w = nullptr, *c = nullptr, *p = nullptr;
    double* fbuf[4] = {nullptr, nullptr, nullptr, nullptr};
    double* gbuf[4] = {nullptr, nullptr, nullptr, nullptr};
    double2* spec = nullptr;
    double* scratch = nullptr;
    double* partial = nullptr;     // per-warp row sums of the u solve
    double* partial_c = nullptr;   // and of the c solve
    double* avg = nullptr;
    double* avg_c = nullptr;        // channel scheme: xy-average of c (avg holds u's)
    double* dscal = nullptr;        // [0] mdpdx, [1] dcdt, [2] non-finite flag, [3] copy-wait fault flag
    // channel scheme with the fused Helmholtz solves: device records [3][4]
    // (substep set, field u v w c) of k_poisson_fft_batch without FILL
    void* hrec = nullptr;
    bool stall_copies = false;      // test hook (cf_debug_stall_copies)
    long long* dcount = nullptr;    // device substep counter (log row)
    double* dlog = nullptr;
    int log_cap = 0;
    double* staging = nullptr;
    size_t staging_elems = 0;
    double* coef = nullptr;         // arena of all tables
    double* lamx = nullptr;         // inside coef
    double* lamy = nullptr;
    double* zp = nullptr;
    double2 *twx = nullptr, *twy = nullptr;
    FftPlan px, py;
    double c8 = 0.0;
    // per substep s (0..2): sets for u, v, c, w and the Poisson solve
    SetOffsets set[3][4];
    PoissonOffsets hspec[3][3];     // channel scheme: spectral Helmholtz sets of u and v, c, w
    PoissonOffsets pois[3];
    PoissonOffsets pois_init;
    WallRowsD bc_ub, bc_ut, bc_wb, bc_wt;
    long substep = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    long long log_rows_host = 0;
};

namespace {

int check_config(const cf_config* c)
{
    if (!c) return CF_EINVAL;
    if (c->order != 2 && c->order != 4) return CF_EINVAL;
    if (c->ngz != GZ) return CF_EINVAL;
    if (c->nx < 4 || c->ny < 4 || c->nz < (c->order == 4 ? 6 : 4)) return CF_EINVAL;
    if (c->ngx < 0 || c->ngy < 0) return CF_EINVAL;
    if (c->nx > FFT_MAX_N || c->ny > FFT_MAX_N) return CF_EINVAL;
    if (fft_radices(c->nx).empty() || fft_radices(c->ny).empty()) return CF_EINVAL;
    if (!(c->dt > 0.0) || !(c->nu >= 0.0) || !(c->prandtl > 0.0)) return CF_EINVAL;
    if (!(c->lx > 0.0) || !(c->ly > 0.0) || !(c->lz > 0.0)) return CF_EINVAL;
    if (c->scheme != CF_SCHEME_CHANFAST && c->scheme != CF_SCHEME_CHANNEL) return CF_EINVAL;
    // the fully implicit scheme batches its x transforms with the
    // power-of-two kernels; its fourth-order w solve has nz - 1 rows, of
    // which the three next to each wall carry the closure (nz >= 8)
    if (c->scheme == CF_SCHEME_CHANNEL && (!fftx_batched_supported(c->nx) || (c->order == 4 && c->nz < 8)))
        return CF_EINVAL;
    return CF_OK;
}

// Build every per-substep coefficient table for time step dt and upload.
int build_helm_records(cf_instance* I);
bool helm_fused(const cf_instance* I);

int build_tables(cf_instance* I, double dt)
{
    const cf_config& C = I->cfg;
    const Metrics& m = I->m;
    Arena A;
    const bool channel = C.scheme == CF_SCHEME_CHANNEL;
    auto addfac = [&](SetOffsets& so, const ImplicitSet& s, bool is_w, double nuadt, double gamdt,
                      double zetdt) {
        so.rows = A.add(channel ? channel_rows(m, s, is_w, nuadt, gamdt, zetdt)
                                : fused_rows(m, s, is_w, nuadt, gamdt, zetdt));
        so.k0 = s.fac.k0;
        so.n = s.fac.n;
        so.F1 = A.add(s.fac.F1); so.F2 = A.add(s.fac.F2); so.F3 = A.add(s.fac.F3);
        so.DEN = A.add(s.fac.DEN); so.P = A.add(s.fac.P); so.Q = A.add(s.fac.Q); so.R = A.add(s.fac.R);
        so.hbc = A.add(s.hbc);
        so.green = A.add(s.green.empty() ? std::vector<double>(m.n2, 0.0) : s.green);
        so.bot = to_dev(s.bot);
        so.top = to_dev(s.top);
        std::memcpy(so.gstats, s.green_stats, sizeof(so.gstats));
    };
    double uf = C.setuframe, vf = C.setvframe;
    try {
        for (int s = 0; s < 3; s++) {
            double nubdt = C.nu * RK3_BET[s] * dt;
            double gamdt = RK3_GAM[s] * dt;
            // chanfast.c:61-68: u, v walls at -frame, scalar -0.5 / +0.5, w 0
            ImplicitSet su = make_implicit_u(m, nubdt, gamdt, 0.0 - uf, 0.0 - uf, C.nu, true);
            ImplicitSet sv = make_implicit_u(m, nubdt, gamdt, 0.0 - vf, 0.0 - vf, C.nu, false);
            ImplicitSet sc = make_implicit_u(m, nubdt / C.prandtl, gamdt, -0.5, +0.5, C.nu / C.prandtl, true);
            ImplicitSet sw = make_implicit_w(m, nubdt, 0.0, 0.0);
            double nuadt = C.nu * RK3_ALP[s] * dt, zetdt = RK3_ZET[s] * dt;
            addfac(I->set[s][0], su, false, nuadt, gamdt, zetdt);
            addfac(I->set[s][1], sv, false, nuadt, gamdt, zetdt);
            addfac(I->set[s][2], sc, false, nuadt / C.prandtl, gamdt, zetdt);
            addfac(I->set[s][3], sw, true, nuadt, gamdt, zetdt);
        }
    } catch (const std::exception&) {
        g_last_error = "zero pivot in a line-solve factorisation";
        return CF_EPIVOT;
    }
    auto addpois = [&](PoissonOffsets& po, double pdt) {
        po.host = make_poisson(m, pdt);
        po.a = A.add(po.host.a); po.b = A.add(po.host.b); po.c = A.add(po.host.c);
        po.e = A.add(po.host.e); po.f = A.add(po.host.f); po.g = A.add(po.host.g);
        po.dpart = A.add(po.host.dpart); po.dvol = A.add(po.host.dvol);
        // diagonal factors of the wavenumber terms (pressure.c:326-327, 414-415)
        std::vector<double> cx(po.host.dvol.size()), cy(po.host.dvol.size());
        for (size_t k = 0; k < cx.size(); k++) {
            cx[k] = po.host.dvol[k] * pdt / (m.dx * m.dx);
            cy[k] = po.host.dvol[k] * pdt / (m.dy * m.dy);
        }
        po.cx = A.add(cx); po.cy = A.add(cy);
    };
    for (int s = 0; s < 3; s++) addpois(I->pois[s], (RK3_ALP[s] + RK3_BET[s]) * dt);
    addpois(I->pois_init, 1.0);
    if (channel) {
        // spectral Helmholtz sets with nudt = -nubdt (channel.c:471-478, 547-552, 576-581, 652-657)
        auto addspec = [&](PoissonOffsets& po, double nudt, bool is_w) {
            po.host = make_helmholtz_spectral(m, nudt, is_w);
            po.a = A.add(po.host.a); po.b = A.add(po.host.b); po.c = A.add(po.host.c);
            po.e = A.add(po.host.e); po.f = A.add(po.host.f); po.g = A.add(po.host.g);
            po.dpart = A.add(po.host.dpart); po.dvol = A.add(po.host.dvol);
            std::vector<double> cx(po.host.dvol.size()), cy(po.host.dvol.size());
            for (size_t k = 0; k < cx.size(); k++) {
                cx[k] = po.host.dvol[k] * nudt / (m.dx * m.dx);
                cy[k] = po.host.dvol[k] * nudt / (m.dy * m.dy);
            }
            po.cx = A.add(cx); po.cy = A.add(cy);
        };
        for (int s = 0; s < 3; s++) {
            double nubdt = C.nu * RK3_BET[s] * dt;
            addspec(I->hspec[s][0], -nubdt, false);
            addspec(I->hspec[s][1], -nubdt / C.prandtl, false);
            addspec(I->hspec[s][2], -nubdt, true);
        }
    }
    size_t o_lamx = A.add(I->pois_init.host.lamx);
    size_t o_lamy = A.add(I->pois_init.host.lamy);
    // metrics
    int n2 = m.n2;
    std::vector<double> dzp1h(n2, 0.0), dzm1h(n2, 0.0), dzp3h(n2, 0.0), dzm3h(n2, 0.0), dydz(n2), dxdz(n2);
    for (int k = 0; k < n2; k++) {
        if (k + 1 < n2) dzp1h[k] = 0.5 * (m.dz[k + 1] + m.dz[k]);
        if (k >= 1) dzm1h[k] = 0.5 * (m.dz[k - 1] + m.dz[k]);
        if (k + 2 < n2) dzp3h[k] = 0.5 * (m.dz[k + 2] + m.dz[k + 1]);
        if (k >= 2) dzm3h[k] = 0.5 * (m.dz[k - 2] + m.dz[k - 1]);
        dydz[k] = m.dy * m.dz[k];
        dxdz[k] = m.dx * m.dz[k];
    }
    std::vector<double> ivol(n2, 0.0), ivolw(n2, 0.0), idzp1h(n2, 0.0), idz(n2, 0.0);
    for (int k = 0; k < n2; k++) {
        ivol[k] = 1.0 / (m.dx * m.dy * m.dz[k]);
        idz[k] = 1.0 / m.dz[k];
        if (k + 1 < n2) {
            ivolw[k] = 1.0 / (m.dx * m.dy * dzp1h[k]);
            idzp1h[k] = 1.0 / dzp1h[k];
        }
    }
    size_t o_dz = A.add(m.dz), o_p1 = A.add(dzp1h), o_m1 = A.add(dzm1h), o_p3 = A.add(dzp3h),
           o_m3 = A.add(dzm3h), o_dydz = A.add(dydz), o_dxdz = A.add(dxdz), o_iv = A.add(ivol),
           o_ivw = A.add(ivolw), o_idz = A.add(idzp1h), o_idzc = A.add(idz);
    size_t o_zp = A.add(z_at_p(m));

    if (I->coef) { cudaFree(I->coef); I->coef = nullptr; }
    CF_CUDA(cudaMalloc(&I->coef, A.h.size() * sizeof(double)));
    CF_CUDA(cudaMemcpy(I->coef, A.h.data(), A.h.size() * sizeof(double), cudaMemcpyHostToDevice));
    double* b = I->coef;
    Geo& G = I->geo;
    G.dz = b + o_dz; G.dzp1h = b + o_p1; G.dzm1h = b + o_m1; G.dzp3h = b + o_p3; G.dzm3h = b + o_m3;
    G.dydz = b + o_dydz; G.dxdz = b + o_dxdz; G.ivol = b + o_iv; G.ivolw = b + o_ivw;
    G.idzp1h = b + o_idz;
    G.idz = b + o_idzc;
    I->lamx = b + o_lamx;
    I->lamy = b + o_lamy;
    I->zp = b + o_zp;
    I->cfg.dt = dt;
    // a new graph is needed whenever the tables move
    if (I->gexec) { cudaGraphExecDestroy(I->gexec); I->gexec = nullptr; }
    if (I->graph) { cudaGraphDestroy(I->graph); I->graph = nullptr; }
    if (helm_fused(I)) {
        const int hr = build_helm_records(I);
        if (hr) return hr;
    }
    return CF_OK;
}

FactorD factor_of(cf_instance* I, const SetOffsets& so)
{
    double* b = I->coef;
    FactorD f;
    f.k0 = so.k0;
    f.n = so.n;
    f.F1 = b + so.F1; f.F2 = b + so.F2; f.F3 = b + so.F3; f.DEN = b + so.DEN;
    f.P = b + so.P; f.Q = b + so.Q; f.R = b + so.R;
    return f;
}

PoissonArgs poisson_args(cf_instance* I, const PoissonOffsets& po, double pdt)
{
    double* b = I->coef;
    PoissonArgs A;
    A.spec = I->spec;
    A.scratch = I->scratch;
    A.a = b + po.a; A.b = b + po.b; A.c = b + po.c; A.e = b + po.e; A.f = b + po.f; A.g = b + po.g;
    A.dpart = b + po.dpart; A.dvol = b + po.dvol;
    A.cx = b + po.cx; A.cy = b + po.cy;
    A.lamx = I->lamx;
    A.lamy = I->lamy;
    std::memcpy(A.red, po.host.red, sizeof(A.red));
    std::memcpy(A.dsub, po.host.dsub, sizeof(A.dsub));
    A.bot[0] = to_dev(po.host.bot[0]);
    A.bot[1] = to_dev(po.host.bot[1]);
    A.top = to_dev(po.host.top);
    A.dt = pdt;
    A.dxdx = I->m.dx * I->m.dx;
    A.dydy = I->m.dy * I->m.dy;
    A.nrows = I->cfg.nz;
    A.avg = nullptr;
    A.abot = A.atop = WallRowsD{};
    A.abc_bot = A.abc_top = 0.0;
    return A;
}

// Optional per-kernel timing: events recorded after each launch group.
struct Timeline {
    cudaEvent_t ev[CF_NKERNEL_GROUPS + 1];
    int n = 0;
    void mark(cudaStream_t st) { cudaEventRecord(ev[n++], st); }
};

// Where the launches of a z-implicit substep go.  The base class launches
// each stage at once on the instance stream (and marks the timeline between
// launch groups); the batch (cf_batch below) overrides every stage to record
// it instead, and later runs each stage of many instances as one launch.
struct Sink {
    cudaStream_t st = nullptr;
    Timeline* tl = nullptr;
    virtual ~Sink() = default;
    virtual void mark() { if (tl) tl->mark(st); }
    virtual void ghosts(const Geo& G, const GhostArgs& A) { launch_ghosts(G, A, st); }
    virtual void rhs(const Geo& G, const RhsArgs& A) { launch_rhs(G, A, false, st); }
    virtual void back4(const Geo& G, const SolveBatch& B) { launch_back4(G, B, st); }
    virtual void mass(const Geo& G, const double* partial, double* avg, const MassArgs& M)
    {
        launch_mass(G, partial, avg, M, st);
    }
    virtual void div_fftx(const Geo& G, const DivArgs& A) { launch_div_fftx(G, A, st); }
    virtual void ffty(const Geo& G, const FftyArgs& A, int nrows) { launch_ffty(G, A, nrows, st); }
    virtual void poisson(const Geo& G, const PoissonArgs& A) { launch_poisson(G, A, st); }
    // the y transforms fused with the Poisson solve (power-of-two ny)
    virtual bool fused_pressure(const Geo& G) const { return poisson_fft_supported(G); }
    virtual void poisson_fft(const Geo& G, const PoissonFftArgs& A) { launch_poisson_fft(G, A, st); }
    virtual void c2r(const Geo& G, const C2rArgs& A, int nrows) { launch_fftx_c2r(G, A, nrows, st); }
    virtual void project(const Geo& G, const ProjArgs& A) { launch_project(G, A, st); }
};

// Divergence -> FFT -> Poisson -> inverse FFT -> projection with step `pdt`.
// With `corr`, the lazily applied mass-flux corrections of substep set `s`
// are folded in (divergence and projection read u + G_u * mdpdx, c + G_c * dcdt).
void pressure_sequence(cf_instance* I, const PoissonOffsets& po, double pdt, int s, bool corr, Sink& K)
{
    const Geo& G = I->geo;
    double* b = I->coef;
    // the divergence field of the power-of-two path lives in p, which the
    // inverse transform below rewrites completely
    DivArgs D{I->u, I->v, I->w, corr ? b + I->set[s][0].green : nullptr, corr ? I->dscal : nullptr,
              I->spec, I->px, I->c8, I->p};
    K.div_fftx(G, D);
    K.mark();
    if (I->fuse_pressure && K.fused_pressure(G)) {
        // one launch; its time is the Poisson group's, the y-transform groups stay empty
        K.mark();
        PoissonFftArgs F{poisson_args(I, po, pdt), I->py.tw, I->c8, I->dscal + 3, I->stall_copies ? 1 : 0};
        K.poisson_fft(G, F);
        K.mark();
        K.mark();
    } else {
        FftyArgs Y{I->spec, I->py, -1, GZ, I->c8};
        K.ffty(G, Y, G.nz);
        K.mark();
        K.poisson(G, poisson_args(I, po, pdt));
        K.mark();
        FftyArgs Yb{I->spec, I->py, +1, 0, I->c8};
        K.ffty(G, Yb, G.n2);
        K.mark();
    }
    C2rArgs X{I->spec, {I->p, nullptr, nullptr, nullptr}, I->px, I->c8, 0, 0};
    K.c2r(G, X, G.n2);
    K.mark();
    ProjArgs P;
    P.u = I->u; P.v = I->v; P.w = I->w; P.c = I->c; P.p = I->p;
    P.gu = corr ? b + I->set[s][0].green : nullptr;
    P.gc = corr ? b + I->set[s][2].green : nullptr;
    P.mu = corr ? I->dscal : nullptr;
    P.mc = corr ? I->dscal + 1 : nullptr;
    P.dt = pdt;
    P.dtdx = pdt / I->m.dx;
    P.dtdy = pdt / I->m.dy;
    K.project(G, P);
    K.mark();
}

void pressure_sequence(cf_instance* I, const PoissonOffsets& po, double pdt, int s, bool corr,
                       Timeline* tl = nullptr)
{
    Sink K;
    K.st = I->stream;
    K.tl = tl;
    pressure_sequence(I, po, pdt, s, corr, K);
}

// Mass-flux (u, q = 0) or scalar-mean (c, q = 2) control of substep set s
// from the xy-average profile in `avg` (chanfast.c:485-529, 572-616).
MassArgs mass_args(cf_instance* I, int s, int q, const double* avg)
{
    const cf_config& C = I->cfg;
    const SetOffsets& so = I->set[s][q];
    MassArgs M;
    M.avg = avg;
    M.dz = I->geo.dz;
    M.order = C.order;
    M.nz = C.nz;
    M.n2 = I->geo.n2;
    M.kappa = q == 0 ? C.nu : C.nu / C.prandtl;
    std::memcpy(M.green, so.gstats, sizeof(M.green));
    M.mode = q == 0 ? C.uvolavgmode : C.cvolavgmode;
    M.target = q == 0 ? C.want_uvolavg - C.setuframe : C.want_cvolavg;
    M.fixed = q == 0 ? -C.dpdx : 0.0;
    M.m_out = I->dscal + (q == 0 ? 0 : 1);
    M.counter = I->dcount;
    M.log_base = I->dlog;
    M.log_cap = I->log_cap;
    M.col = q == 0 ? 0 : 5;
    M.advance = q == 2 ? 1 : 0;
    M.nonfinite = I->dscal + 2;
    return M;
}

// The implicit half of a channel-scheme substep (channel.c:455-657 and
// :1405-1607): k_rhs has left h in the g buffers (slots u, v, w, c, one
// contiguous block); transform the four fields, solve per wavenumber, and
// transform back into u, v, w, c; then apply_bc and the two controls.
void enqueue_implicit3d(cf_instance* I, int s, Timeline* tl)
{
    const cf_config& C = I->cfg;
    const Geo& G = I->geo;
    cudaStream_t st = I->stream;
    const long long fstride = G.plane * G.n2;      // between the g buffers
    const long long sstride = G.splane * G.n2;     // between the four spectra
    R2cArgs X{I->gbuf[0], I->spec, I->px, I->c8, GZ, fstride, sstride};
    launch_fftx_r2c(G, X, G.nz, 4, st);
    if (helm_fused(I)) {
        // y transforms and the four solves in one launch (records of set s)
        BatchLaunch L;
        L.recs = static_cast<const char*>(I->hrec) + 4 * s * sizeof(BatchRec<PoissonFftArgs>);
        L.n = 4;
        L.blocks = 4u * (unsigned) G.nkx;
        L.smem = 0;
        L.block = dim3(1);
        launch_helmholtz_fft_batch(L, G.order, G.ny, st);
    } else {
        FftyArgs Y{I->spec, I->py, -1, GZ, I->c8, sstride};
        launch_ffty(G, Y, G.nz, st, 4);
        // slot order u, v, w, c; sets u/v 0, c 1, w 2
        const int set_of_slot[4] = {0, 0, 2, 1};
        for (int f = 0; f < 4; f++) {
            PoissonArgs H = poisson_args(I, I->hspec[s][set_of_slot[f]], 0.0);
            H.spec = I->spec + f * sstride;
            H.nrows = f == 2 ? C.nz - 1 : C.nz;
            if (f == 0 || f == 3) {   // u, c: the xy-average profile for the controls
                H.avg = f == 0 ? I->avg : I->avg_c;
                H.abot = I->bc_ub;
                H.atop = I->bc_ut;
                H.abc_bot = f == 0 ? 0.0 - C.setuframe : -0.5;
                H.abc_top = f == 0 ? 0.0 - C.setuframe : +0.5;
            }
            launch_helmholtz_spectral(G, H, st);
        }
        FftyArgs Yb{I->spec, I->py, +1, GZ, I->c8, sstride};
        launch_ffty(G, Yb, G.nz, st, 4);
    }
    C2rArgs Xb{I->spec, {I->u, I->v, I->w, I->c}, I->px, I->c8, GZ, sstride};
    launch_fftx_c2r(G, Xb, G.nz, st, 4);
    GhostArgs GA;
    GA.F = Fields{I->u, I->v, I->w, I->c};
    GA.ub = I->bc_ub; GA.ut = I->bc_ut; GA.wb = I->bc_wb; GA.wt = I->bc_wt;
    GA.bc_u = 0.0 - C.setuframe;
    GA.bc_v = 0.0 - C.setvframe;
    GA.bc_c_bot = -0.5;
    GA.bc_c_top = +0.5;
    GA.bc_w = 0.0;
    launch_ghosts(G, GA, st, false);
    if (tl) tl->mark(st);
    launch_mass_control(mass_args(I, s, 0, I->avg), st);
    if (tl) tl->mark(st);
    launch_mass_control(mass_args(I, s, 2, I->avg_c), st);
    if (tl) tl->mark(st);
}

// One RK3 substep of instance I through sink K.  The fully implicit scheme
// is not batched: its launches go to K's stream directly.
void enqueue_substep(cf_instance* I, Sink& K)
{
    const cf_config& C = I->cfg;
    const Geo& G = I->geo;
    const int s = (int) (I->substep % 3);
    const double dt = C.dt;
    const bool channel = C.scheme == CF_SCHEME_CHANNEL;
    for (int q = 0; q < 4; q++) std::swap(I->fbuf[q], I->gbuf[q]);   // chanfast.c:397-402

    GhostArgs GA;
    GA.F = Fields{I->u, I->v, I->w, I->c};
    GA.ub = I->bc_ub; GA.ut = I->bc_ut; GA.wb = I->bc_wb; GA.wt = I->bc_wt;
    GA.bc_u = 0.0 - C.setuframe;
    GA.bc_v = 0.0 - C.setvframe;
    GA.bc_c_bot = -0.5;
    GA.bc_c_top = +0.5;
    GA.bc_w = 0.0;
    K.mark();
    K.ghosts(G, GA);
    K.mark();

    // RHS + forward sweeps; set index of each f slot (u, v, w, c) among the
    // implicit-solve sets (u, v, c, w)
    // chanfast: x-y diffusion explicit in f with nu; channel: implicit, in
    // h with nu alpha dt (channel.c:450-458)
    const double nuadt = C.nu * RK3_ALP[s] * dt;
    RhsArgs R{I->u, I->v, I->w, I->c, I->fbuf[0], I->fbuf[1], I->fbuf[2], I->fbuf[3],
              channel ? nuadt : C.nu, channel ? nuadt / C.prandtl : C.nu / C.prandtl,
              C.betg_x, C.betg_y, C.betg_z};
    const int set_of_slot[4] = {0, 1, 3, 2};
    for (int f = 0; f < 4; f++) {
        R.sw[f].g = I->gbuf[f];
        // u and c: f += mdpdx / dcdt of the previous substep's control step
        R.sw[f].gshift = f == 0 ? I->dscal : (f == 3 ? I->dscal + 1 : nullptr);
        R.sw[f].rows = I->coef + I->set[s][set_of_slot[f]].rows;
    }
    R.wbot = I->bc_wb;
    R.wtop = I->bc_wt;
    R.wbc_bot = 0.0;
    R.wbc_top = 0.0;
    if (channel) {
        launch_rhs(G, R, true, K.st);
        K.mark();
        enqueue_implicit3d(I, s, K.tl);
        pressure_sequence(I, I->pois[s], (RK3_ALP[s] + RK3_BET[s]) * dt, s, true, K);
        I->substep++;
        return;
    }
    K.rhs(G, R);
    K.mark();

    double* fields[4] = {I->u, I->v, I->c, I->w};
    const int fidx[4] = {0, 1, 3, 2};   // u, v, c, w -> f/g slots (u, v, w, c)
    double bcb[4] = {0.0 - C.setuframe, 0.0 - C.setvframe, -0.5, 0.0};
    double bct[4] = {0.0 - C.setuframe, 0.0 - C.setvframe, +0.5, 0.0};
    double* partial[4] = {I->partial, nullptr, I->partial_c, nullptr};
    SolveBatch SB;
    for (int q = 0; q < 4; q++) {
        const SetOffsets& so = I->set[s][q];
        const bool is_w = q == 3;
        SolveArgs& S = SB.a[q];
        S.x = fields[q];
        S.s = I->gbuf[fidx[q]];   // the forward sweep in k_rhs left s there
        S.fac = factor_of(I, so);
        S.bc_bot = bcb[q];
        S.bc_top = bct[q];
        S.bcb = is_w ? I->bc_wb : I->bc_ub;
        S.bct = is_w ? I->bc_wt : I->bc_ut;
        S.partial = partial[q];
    }
    K.back4(G, SB);
    K.mark();
    for (int q = 0; q < 4; q += 2) {   // mass-flux control (u), scalar-mean control (c)
        // each control has its own average buffer, so batched stages of
        // different instances and fields never share one
        double* avg = q == 0 ? I->avg : I->avg_c;
        K.mass(G, partial[q], avg, mass_args(I, s, q, avg));
        K.mark();
    }
    pressure_sequence(I, I->pois[s], (RK3_ALP[s] + RK3_BET[s]) * dt, s, true, K);
    I->substep++;
}

void enqueue_substep(cf_instance* I, Timeline* tl = nullptr)
{
    Sink K;
    K.st = I->stream;
    K.tl = tl;
    enqueue_substep(I, K);
}

// ------------------------------------------------------------------ batches
//
// A batch runs the same stage of many z-implicit instances as one launch:
// BatchSink records each instance's stage arguments (with its geometry and
// its own grid) instead of launching; compile() groups the records of a
// stage by kernel variant (order; transform size for the power-of-two
// transforms), lays them out in one device block with each record's first
// flat block, and turns every group into one batched launch (batch.cuh).

// ST_PSOLVE: y transforms and Poisson solve, per member either the three
// separate launches or the fused one (the member's own choice, so that a
// member's result does not depend on its neighbours in a batch)
enum StageKind { ST_GHOSTS, ST_RHS, ST_BACK4, ST_MASS, ST_DIV, ST_PSOLVE, ST_C2R, ST_PROJECT };

struct BatchStage {
    int kind = -1;
    std::vector<BatchRec<GhostArgs>> ghosts;
    std::vector<BatchRec<RhsArgs>> rhs;
    std::vector<BatchRec<SolveBatch>> back4;
    std::vector<BatchRec<RowAvgArgs>> rowavg;
    std::vector<BatchRec<MassArgs>> control;
    std::vector<BatchRec<DivArgs>> div;        // power-of-two nx: the divergence ...
    std::vector<BatchRec<R2cArgs>> r2c;        // ... then its x transform
    std::vector<BatchRec<DivArgs>> div_fftx;   // other nx: both in one kernel
    std::vector<BatchRec<FftyArgs>> ffty;       // forward y transforms ...
    std::vector<BatchRec<PoissonArgs>> poisson; // ... Poisson solves ...
    std::vector<BatchRec<FftyArgs>> ffty_bwd;   // ... inverse y transforms
    std::vector<BatchRec<PoissonFftArgs>> pfft; // fused members
    std::vector<BatchRec<C2rArgs>> c2r;
    std::vector<BatchRec<ProjArgs>> project;
};

template <class Args>
BatchRec<Args> batch_rec(const Geo& G, const Args& A, dim3 g)
{
    BatchRec<Args> r;
    r.G = G;
    r.A = A;
    r.gx = g.x;
    r.gy = g.y;
    r.gz = g.z;
    r.begin = 0;
    return r;
}

// The fully implicit scheme's four spectral Helmholtz solves run fused with
// their y transforms (k_poisson_fft_batch, FILL off) where the pressure
// solve of the instance is fused.
bool helm_fused(const cf_instance* I)
{
    return I->cfg.scheme == CF_SCHEME_CHANNEL && I->fuse_pressure && poisson_fft_supported(I->geo);
}

// Scratch of one field's Helmholtz solve (k_poisson_fft's multiplier rows).
size_t helm_scratch_stride(const cf_instance* I)
{
    const Geo& G = I->geo;
    return (size_t) (I->cfg.order == 4 ? 3 : 1) * G.n2 * G.nkx * (G.ny / 2 + 2);
}

// Records of the fused solves of u, v, w, c for each substep set: the
// arguments enqueue_implicit3d gives the separate solves, each field with its
// own spectrum and scratch, its blocks after the previous field's.
int build_helm_records(cf_instance* I)
{
    const cf_config& C = I->cfg;
    const Geo& G = I->geo;
    const long long sstride = G.splane * G.n2;
    const int set_of_slot[4] = {0, 0, 2, 1};
    std::vector<BatchRec<PoissonFftArgs>> recs;
    for (int s = 0; s < 3; s++) {
        for (int f = 0; f < 4; f++) {
            PoissonArgs H = poisson_args(I, I->hspec[s][set_of_slot[f]], 0.0);
            H.spec = I->spec + f * sstride;
            H.scratch = I->scratch + f * helm_scratch_stride(I);
            H.nrows = f == 2 ? C.nz - 1 : C.nz;
            if (f == 0 || f == 3) {   // u, c: the xy-average profile for the controls
                H.avg = f == 0 ? I->avg : I->avg_c;
                H.abot = I->bc_ub;
                H.atop = I->bc_ut;
                H.abc_bot = f == 0 ? 0.0 - C.setuframe : -0.5;
                H.abc_top = f == 0 ? 0.0 - C.setuframe : +0.5;
            }
            PoissonFftArgs F{H, I->py.tw, I->c8, I->dscal + 3, 0};
            BatchRec<PoissonFftArgs> r = batch_rec(G, F, dim3(G.nkx));
            r.begin = (unsigned) (f * G.nkx);
            recs.push_back(r);
        }
    }
    const size_t bytes = recs.size() * sizeof(BatchRec<PoissonFftArgs>);
    if (!I->hrec) CF_CUDA(cudaMalloc(&I->hrec, bytes));
    CF_CUDA(cudaMemcpy(I->hrec, recs.data(), bytes, cudaMemcpyHostToDevice));
    return CF_OK;
}

struct BatchSink : Sink {
    std::vector<BatchStage> stages;
    size_t cursor = 0;
    bool mismatch = false;
    bool fuse = false;   // members may take the fused y-transform + Poisson launch
    size_t psolve = 0;   // the open ST_PSOLVE stage of a member's separate launches
    BatchStage& next(int kind)
    {
        if (cursor == stages.size()) {
            stages.emplace_back();
            stages.back().kind = kind;
        }
        BatchStage& S = stages[cursor++];
        if (S.kind != kind) mismatch = true;
        return S;
    }
    void mark() override {}
    void ghosts(const Geo& G, const GhostArgs& A) override
    {
        next(ST_GHOSTS).ghosts.push_back(batch_rec(G, A, grid_ghosts(G)));
    }
    void rhs(const Geo& G, const RhsArgs& A) override { next(ST_RHS).rhs.push_back(batch_rec(G, A, grid_rhs(G))); }
    void back4(const Geo& G, const SolveBatch& B) override
    {
        next(ST_BACK4).back4.push_back(batch_rec(G, B, grid_back4(G)));
    }
    void mass(const Geo& G, const double* partial, double* avg, const MassArgs& M) override
    {
        BatchStage& S = next(ST_MASS);
        S.rowavg.push_back(batch_rec(G, row_average_args(G, partial, avg), dim3(G.n2)));
        S.control.push_back(batch_rec(G, M, dim3(1)));
    }
    void div_fftx(const Geo& G, const DivArgs& A) override
    {
        BatchStage& S = next(ST_DIV);
        if (batch_pow2(G.nx)) {
            S.div.push_back(batch_rec(G, A, grid_div(G)));
            R2cArgs R{A.dv, A.spec, A.px, A.c8, GZ, 0, 0};
            S.r2c.push_back(batch_rec(G, R, grid_r2c(G, G.nz, 1)));
        } else {
            S.div_fftx.push_back(batch_rec(G, A, grid_div_fftx(G)));
        }
    }
    // forward y transform (opens the member's ST_PSOLVE stage), Poisson,
    // inverse y transform
    void ffty(const Geo& G, const FftyArgs& A, int nrows) override
    {
        if (A.sign < 0) {
            next(ST_PSOLVE);
            psolve = cursor - 1;
            stages[psolve].ffty.push_back(batch_rec(G, A, grid_ffty(G, nrows, 1)));
        } else {
            stages[psolve].ffty_bwd.push_back(batch_rec(G, A, grid_ffty(G, nrows, 1)));
        }
    }
    void poisson(const Geo& G, const PoissonArgs& A) override
    {
        stages[psolve].poisson.push_back(batch_rec(G, A, grid_poisson(G)));
    }
    bool fused_pressure(const Geo& G) const override { return fuse && poisson_fft_supported(G); }
    void poisson_fft(const Geo& G, const PoissonFftArgs& A) override
    {
        next(ST_PSOLVE).pfft.push_back(batch_rec(G, A, dim3(G.nkx)));
    }
    void c2r(const Geo& G, const C2rArgs& A, int nrows) override
    {
        next(ST_C2R).c2r.push_back(batch_rec(G, A, grid_c2r(G, nrows, 1)));
    }
    void project(const Geo& G, const ProjArgs& A) override
    {
        next(ST_PROJECT).project.push_back(batch_rec(G, A, grid_project(G)));
    }
};

enum BatchKernel { BK_GHOSTS, BK_RHS, BK_BACK4, BK_ROWAVG, BK_CONTROL, BK_DIV, BK_R2C, BK_DIV_FFTX, BK_FFTY,
                   BK_POISSON, BK_PFFT, BK_C2R, BK_PROJECT };

struct BatchOp {
    int kernel;
    int key;              // order, or the transform size (0: generic transforms)
    BatchLaunch L;        // L.recs holds a byte offset into the program's record block until upload
};

struct BatchProgram {
    std::vector<char> blob;    // host copy of every record
    void* dblob = nullptr;     // device copy (the launches read it)
    std::vector<BatchOp> ops;
    int substeps = 0;
};

// Append one group per key of `recs` to P: records laid out contiguously
// with their first flat blocks, one batched launch each.
template <class Args, class KeyFn, class SmemFn>
void add_groups(BatchProgram& P, int kernel, const std::vector<BatchRec<Args>>& recs, KeyFn key, SmemFn smem,
                dim3 block = dim3(1, 1, 1))
{
    std::map<int, std::vector<BatchRec<Args>>> groups;
    for (const auto& r : recs) groups[key(r)].push_back(r);
    for (auto& kv : groups) {
        auto& g = kv.second;
        // the members with the tallest columns first: blocks start roughly in
        // index order, so the longest-running ones are not left for the end
        std::stable_sort(g.begin(), g.end(), [](const auto& a, const auto& b) { return a.G.n2 > b.G.n2; });
        unsigned begin = 0;
        size_t sm = 0;
        for (auto& r : g) {
            r.begin = begin;
            begin += r.gx * r.gy * r.gz;
            sm = std::max(sm, (size_t) smem(r));
        }
        size_t off = (P.blob.size() + 255) / 256 * 256;
        P.blob.resize(off + g.size() * sizeof(BatchRec<Args>));
        std::memcpy(P.blob.data() + off, g.data(), g.size() * sizeof(BatchRec<Args>));
        BatchOp op;
        op.kernel = kernel;
        op.key = kv.first;
        op.L.recs = reinterpret_cast<const void*>(off);
        op.L.n = (int) g.size();
        op.L.blocks = begin;
        op.L.smem = sm;
        op.L.block = block;
        P.ops.push_back(op);
    }
}

// Block shape of a batched launch of a tuned kernel: every record of a batch
// is recorded with the batch's one launch shape (record()).
dim3 back4_block(const std::vector<BatchRec<SolveBatch>>& r)
{
    return dim3(r.empty() ? 128 : r[0].G.shape.solve_threads);
}
dim3 poisson_block(const std::vector<BatchRec<PoissonArgs>>& r)
{
    return dim3(r.empty() ? 128 : r[0].G.shape.pois_threads);
}
dim3 project_block(const std::vector<BatchRec<ProjArgs>>& r)
{
    return r.empty() ? dim3(32, 4) : dim3(r[0].G.shape.proj_bx, r[0].G.shape.proj_by);
}

void compile(const BatchSink& K, BatchProgram& P)
{
    auto order = [](const auto& r) { return r.G.order; };
    auto none = [](const auto&) { return 0; };
    // transform kernels are per size where the size has its own kernels
    auto keynx = [](const auto& r) { return fft_kernel_key(r.G.nx); };
    auto keyny = [](const auto& r) { return fft_kernel_key(r.G.ny); };
    auto smem_nx = [](const auto& r) { return batch_pow2(r.G.nx) ? (size_t) 0 : fft_generic_smem(r.G.nx, false); };
    auto smem_ny = [](const auto& r) { return batch_pow2(r.G.ny) ? (size_t) 0 : fft_generic_smem(r.G.ny, true); };
    for (const BatchStage& S : K.stages) {
        switch (S.kind) {
        case ST_GHOSTS: add_groups(P, BK_GHOSTS, S.ghosts, order, none); break;
        case ST_RHS: add_groups(P, BK_RHS, S.rhs, order, none); break;
        case ST_BACK4: add_groups(P, BK_BACK4, S.back4, order, none, back4_block(S.back4)); break;
        case ST_MASS:
            add_groups(P, BK_ROWAVG, S.rowavg, none, none);
            add_groups(P, BK_CONTROL, S.control, none, none);
            break;
        case ST_DIV:
            add_groups(P, BK_DIV, S.div, order, none);
            add_groups(P, BK_R2C, S.r2c, keynx, none);
            add_groups(P, BK_DIV_FFTX, S.div_fftx, [](const auto& r) { return 1024 * fft_kernel_key(r.G.nx) + r.G.order; },
                       smem_nx);
            break;
        case ST_PSOLVE:
            add_groups(P, BK_FFTY, S.ffty, keyny, smem_ny);
            add_groups(P, BK_POISSON, S.poisson, order, none, poisson_block(S.poisson));
            add_groups(P, BK_FFTY, S.ffty_bwd, keyny, smem_ny);
            add_groups(P, BK_PFFT, S.pfft, [](const auto& r) { return 8 * r.G.ny + r.G.order; }, none);
            break;
        case ST_C2R: add_groups(P, BK_C2R, S.c2r, keynx, smem_nx); break;
        default: add_groups(P, BK_PROJECT, S.project, order, none, project_block(S.project)); break;
        }
    }
}

int upload(BatchProgram& P, cudaStream_t st)
{
    CF_CUDA(cudaMallocAsync(&P.dblob, std::max<size_t>(P.blob.size(), 256), st));
    CF_CUDA(cudaMemcpyAsync(P.dblob, P.blob.data(), P.blob.size(), cudaMemcpyHostToDevice, st));
    for (BatchOp& op : P.ops)
        op.L.recs = static_cast<const char*>(P.dblob) + reinterpret_cast<size_t>(op.L.recs);
    return CF_OK;
}

void run_program(const BatchProgram& P, cudaStream_t st)
{
    for (const BatchOp& op : P.ops) {
        const BatchLaunch& L = op.L;
        switch (op.kernel) {
        case BK_GHOSTS: launch_ghosts_batch(L, op.key, st); break;
        case BK_RHS: launch_rhs_batch(L, op.key, st); break;
        case BK_BACK4: launch_back4_batch(L, op.key, st); break;
        case BK_ROWAVG: launch_row_average_batch(L, st); break;
        case BK_CONTROL: launch_mass_control_batch(L, st); break;
        case BK_DIV: launch_div_batch(L, op.key, st); break;
        case BK_R2C: launch_r2c_batch(L, op.key, st); break;
        case BK_DIV_FFTX: launch_div_fftx_batch(L, op.key % 1024, op.key / 1024, st); break;
        case BK_FFTY: launch_ffty_batch(L, op.key, st); break;
        case BK_POISSON: launch_poisson_batch(L, op.key, st); break;
        case BK_PFFT: launch_poisson_fft_batch(L, op.key, st); break;
        case BK_C2R: launch_c2r_batch(L, op.key, st); break;
        default: launch_project_batch(L, op.key, st); break;
        }
    }
}

// Record `nsub` substeps of every member into K (this advances each member's
// host-side substep counter and f/g roles, as stepping would), every member
// with the launch shape `shape` (a batched launch has one block shape; the
// members' own shapes are put back afterwards).
int record_sink(const std::vector<cf_instance*>& v, int nsub, const LaunchShape& shape, BatchSink& K)
{
    std::vector<LaunchShape> own;
    for (cf_instance* I : v) {
        own.push_back(I->geo.shape);
        I->geo.shape = shape;
    }
    int rc = CF_OK;
    for (int q = 0; q < nsub && rc == CF_OK; q++) {
        const size_t base = K.stages.size();
        size_t per = 0;
        for (size_t m = 0; m < v.size(); m++) {
            K.cursor = base;
            enqueue_substep(v[m], K);
            const size_t n = K.cursor - base;
            if (m == 0) per = n;
            if (n != per || K.mismatch) {
                g_last_error = "batch members emit different stage sequences";
                rc = CF_EINVAL;
                break;
            }
        }
    }
    for (size_t m = 0; m < v.size(); m++) v[m]->geo.shape = own[m];
    return rc;
}

int record(const std::vector<cf_instance*>& v, int nsub, BatchProgram& P, const LaunchShape& shape)
{
    BatchSink K;
    K.fuse = true;
    const int rc = record_sink(v, nsub, shape, K);
    if (rc) return rc;
    compile(K, P);
    P.substeps = nsub;
    return CF_OK;
}

// Order the batch stream after each member's stream (before) or each member
// stream after the batch stream (after).
int join_streams(const std::vector<cf_instance*>& v, cudaStream_t st, cudaEvent_t ev, bool before)
{
    if (before) {
        for (cf_instance* I : v) {
            if (I->stream == st) continue;
            CF_CUDA(cudaEventRecord(ev, I->stream));
            CF_CUDA(cudaStreamWaitEvent(st, ev, 0));
        }
    } else {
        CF_CUDA(cudaEventRecord(ev, st));
        for (cf_instance* I : v)
            if (I->stream != st) CF_CUDA(cudaStreamWaitEvent(I->stream, ev, 0));
    }
    return CF_OK;
}

int check_members(cf_instance* const* v, int n)
{
    if (!v || n <= 0) return CF_EINVAL;
    for (int m = 0; m < n; m++) {
        if (!v[m]) return CF_EINVAL;
        if (v[m]->cfg.scheme != CF_SCHEME_CHANFAST || v[m]->device != v[0]->device) return CF_EINVAL;
        for (int q = 0; q < m; q++)
            if (v[q] == v[m]) return CF_EINVAL;
    }
    return CF_OK;
}

}  // namespace

// Members are stepped by two programs, the substeps 0-2 and 3-5 of a
// two-step cycle (six substeps restore every member's f/g roles); the whole
// cycle replays as one CUDA graph.
struct cf_batch {
    std::vector<cf_instance*> v;
    std::vector<long> expect;       // each member's substep count the programs expect
    std::vector<double*> coef;      // each member's table block the records point into
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    BatchProgram half[2];
    int cursor = 0;                 // the half that runs next
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t ev = nullptr;
    LaunchShape shape;              // launch shape of the tuned kernels (tune_batch)
};

// ====================================================================== tuner
//
// Launch-shape autotuner.  Three kernels run with any of a few block shapes
// and give the same results (LaunchShape, engine.cuh): k_back4 (columns per
// block), k_poisson / k_helmholtz_spectral (column pairs per block) and
// k_project (2-D block).  The tuner captures one substep's arguments of those
// stages, times every candidate shape of each kernel with CUDA events on the
// instance's stream (one warm-up launch, then TUNE_REPS launches), and keeps
// the fastest.  Choices are cached per configuration for the process, and in
// the text file named by CF_TUNE_CACHE when that is set (one line per key:
// key solve pois proj_bx proj_by), so every size is timed once.
//
// * A single instance is tuned when it is created, before it holds any state:
//   the timed launches write its fields (zeroed again afterwards), its
//   spectrum and its scratch.
// * A batch is tuned when it is created (cf_batch_create), on its own batched
//   launches with every output those launches write redirected to scratch
//   device memory, so the members' state is untouched.  It is skipped (the
//   default shapes are used) when that scratch would not fit in free memory.
//   cf_batch_step uses the cached shape of its member set, else the defaults.
//
// CF_TUNE=0 in the environment, or cf_set_tuning(0), turns tuning off.

namespace {

const int TUNE_SOLVE[] = {64, 128};
const int TUNE_POIS[] = {64, 128};
const int TUNE_PROJ[][2] = {{32, 2}, {32, 4}, {32, 8}, {64, 2}};
constexpr int TUNE_REPS = 3;

std::mutex g_tune_mu;
std::map<std::string, LaunchShape> g_tune_cache;
bool g_tune_file_read = false;
int g_tune_mode = -1;   // -1: not decided yet (CF_TUNE), 0 off, 1 on

bool tune_enabled()
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune_mode < 0) {
        const char* e = std::getenv("CF_TUNE");
        g_tune_mode = (e && e[0] == '0') ? 0 : 1;
    }
    return g_tune_mode == 1;
}

bool shape_valid(const LaunchShape& S)
{
    bool a = false, b = false, c = false;
    for (int t : TUNE_SOLVE) a |= S.solve_threads == t;
    for (int t : TUNE_POIS) b |= S.pois_threads == t;
    for (const auto& t : TUNE_PROJ) c |= S.proj_bx == t[0] && S.proj_by == t[1];
    return a && b && c;
}

// Cache file: "key solve pois proj_bx proj_by" per line; unreadable or
// malformed lines are ignored.
void tune_read_file_locked()
{
    if (g_tune_file_read) return;
    g_tune_file_read = true;
    const char* path = std::getenv("CF_TUNE_CACHE");
    if (!path || !*path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char key[512];
    LaunchShape S;
    while (std::fscanf(f, "%511s %d %d %d %d", key, &S.solve_threads, &S.pois_threads, &S.proj_bx, &S.proj_by) == 5)
        if (shape_valid(S)) g_tune_cache[key] = S;
    std::fclose(f);
}

bool tune_lookup(const std::string& key, LaunchShape& out)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_read_file_locked();
    auto it = g_tune_cache.find(key);
    if (it == g_tune_cache.end()) return false;
    out = it->second;
    return true;
}

void tune_store(const std::string& key, const LaunchShape& S)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = S;
    const char* path = std::getenv("CF_TUNE_CACHE");
    if (!path || !*path) return;
    if (FILE* f = std::fopen(path, "a")) {
        std::fprintf(f, "%s %d %d %d %d\n", key.c_str(), S.solve_threads, S.pois_threads, S.proj_bx, S.proj_by);
        std::fclose(f);
    }
}

// Device model, compute capability and SM count: launch shapes tuned on one
// model are not reused on another (a cache file may be shared).  One
// whitespace-free token, as the cache file's first field.
std::string device_tag(int device)
{
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return "unknown";
    std::string name = p.name;
    for (char& ch : name)
        if (!std::isalnum((unsigned char) ch)) ch = '_';
    return name + "-cc" + std::to_string(p.major) + std::to_string(p.minor) + "-sm"
         + std::to_string(p.multiProcessorCount);
}

std::string config_key(const cf_instance* I)
{
    const cf_config& C = I->cfg;
    return "o" + std::to_string(C.order) + "s" + std::to_string(C.scheme) + "-" + std::to_string(C.nx) + "x"
         + std::to_string(C.ny) + "x" + std::to_string(C.nz);
}

// Key of a member set: its configurations with their counts, sorted.  A
// set of many distinct configurations is keyed by the 64-bit FNV-1a hash of
// that list instead, so that every key fits one cache-file field.
std::string batch_key(const std::vector<cf_instance*>& v)
{
    std::map<std::string, int> n;
    for (const cf_instance* I : v) n[config_key(I)]++;
    std::string list;
    for (const auto& kv : n) list += ":" + kv.first + "*" + std::to_string(kv.second);
    const std::string head = device_tag(v[0]->device) + ":batch";
    if (list.size() <= 400) return head + list;
    unsigned long long h = 1469598103934665603ull;
    for (unsigned char ch : list) {
        h ^= ch;
        h *= 1099511628211ull;
    }
    char hex[24];
    std::snprintf(hex, sizeof hex, "%016llx", h);
    return head + ":h" + hex;
}

// Mean device time of `launch` over TUNE_REPS launches after one warm-up.
template <class F>
int time_launch(cudaStream_t st, F launch, float& ms)
{
    cudaEvent_t a, b;
    CF_CUDA(cudaEventCreate(&a));
    CF_CUDA(cudaEventCreate(&b));
    launch();
    cudaEventRecord(a, st);
    for (int r = 0; r < TUNE_REPS; r++) launch();
    cudaEventRecord(b, st);
    cudaError_t e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaGetLastError();
    float t = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) {
        g_last_error = std::string("tuning: ") + cudaGetErrorString(e);
        return CF_ECUDA;
    }
    ms = t / TUNE_REPS;
    return CF_OK;
}

// Arguments of the tuned stages of one substep.
struct CaptureSink : Sink {
    Geo G{};
    bool has_back4 = false, has_pois = false, has_proj = false;
    SolveBatch back4_args{};
    PoissonArgs pois_args{};
    ProjArgs proj_args{};
    void mark() override {}
    void ghosts(const Geo&, const GhostArgs&) override {}
    void rhs(const Geo&, const RhsArgs&) override {}
    void back4(const Geo& g, const SolveBatch& B) override { G = g; back4_args = B; has_back4 = true; }
    void mass(const Geo&, const double*, double*, const MassArgs&) override {}
    void div_fftx(const Geo&, const DivArgs&) override {}
    void ffty(const Geo&, const FftyArgs&, int) override {}
    void poisson(const Geo& g, const PoissonArgs& A) override { G = g; pois_args = A; has_pois = true; }
    bool fused_pressure(const Geo&) const override { return false; }   // capture the separate solve
    void c2r(const Geo&, const C2rArgs&, int) override {}
    void project(const Geo& g, const ProjArgs& A) override { G = g; proj_args = A; has_proj = true; }
};

// Fastest candidate of each tuned kernel; `run(kind, shape)` launches that
// kernel once with the shape (kind 0 back4, 1 Poisson, 2 projection).
template <class Run>
int tune_shapes(cudaStream_t st, bool with_back4, Run run, LaunchShape& best)
{
    best = LaunchShape{};
    float bt = 1e30f, t = 0.0f;
    if (with_back4) {
        for (int c : TUNE_SOLVE) {
            LaunchShape S = best;
            S.solve_threads = c;
            int rc = time_launch(st, [&] { run(0, S); }, t);
            if (rc) return rc;
            if (t < bt) { bt = t; best.solve_threads = c; }
        }
    }
    bt = 1e30f;
    for (int c : TUNE_POIS) {
        LaunchShape S = best;
        S.pois_threads = c;
        int rc = time_launch(st, [&] { run(1, S); }, t);
        if (rc) return rc;
        if (t < bt) { bt = t; best.pois_threads = c; }
    }
    bt = 1e30f;
    for (const auto& c : TUNE_PROJ) {
        LaunchShape S = best;
        S.proj_bx = c[0];
        S.proj_by = c[1];
        int rc = time_launch(st, [&] { run(2, S); }, t);
        if (rc) return rc;
        if (t < bt) { bt = t; best.proj_bx = c[0]; best.proj_by = c[1]; }
    }
    return CF_OK;
}

}  // namespace

// Tune a newly created instance (no state yet); cached per configuration.
int tune_instance(cf_instance* I)
{
    if (!tune_enabled()) return CF_OK;
    const std::string key = device_tag(I->device) + ":" + config_key(I);
    LaunchShape S;
    if (tune_lookup(key, S)) {
        I->geo.shape = S;
        return CF_OK;
    }
    CaptureSink K;
    double* fb[4];
    double* gb[4];
    for (int q = 0; q < 4; q++) { fb[q] = I->fbuf[q]; gb[q] = I->gbuf[q]; }
    const long sub = I->substep;
    if (I->cfg.scheme == CF_SCHEME_CHANNEL) pressure_sequence(I, I->pois[0], I->cfg.dt, 0, true, K);
    else enqueue_substep(I, K);
    for (int q = 0; q < 4; q++) { I->fbuf[q] = fb[q]; I->gbuf[q] = gb[q]; }
    I->substep = sub;
    if (!K.has_pois || !K.has_proj) return CF_OK;
    auto run = [&](int kind, const LaunchShape& sh) {
        Geo G = K.G;
        G.shape = sh;
        if (kind == 0) launch_back4(G, K.back4_args, I->stream);
        else if (kind == 1) launch_poisson(G, K.pois_args, I->stream);
        else launch_project(G, K.proj_args, I->stream);
    };
    int rc = tune_shapes(I->stream, K.has_back4, run, S);
    if (rc) return rc;
    // the timed launches wrote the fields: zero them as creation leaves them
    const size_t fbytes = (size_t) I->geo.plane * I->geo.n2 * sizeof(double);
    for (double* f : {I->u, I->v, I->w, I->c}) CF_CUDA(cudaMemsetAsync(f, 0, fbytes, I->stream));
    CF_CUDA(cudaStreamSynchronize(I->stream));
    I->geo.shape = S;
    tune_store(key, S);
    return CF_OK;
}

// Launch shape of a member set for cf_batch_step: cached, else the defaults.
LaunchShape batch_cached_shape(const std::vector<cf_instance*>& v)
{
    LaunchShape S;
    if (tune_enabled()) tune_lookup(batch_key(v), S);
    return S;
}

// Tune the batched launches of a member set (cf_batch_create); outputs
// redirected to scratch.  The members' host state is restored.
int tune_batch(const std::vector<cf_instance*>& v, cudaStream_t st, LaunchShape& out)
{
    out = LaunchShape{};
    if (!tune_enabled()) return CF_OK;
    const std::string key = batch_key(v);
    if (tune_lookup(key, out)) return CF_OK;
    // one substep of every member, recorded and put back
    std::vector<std::array<double*, 8>> fg(v.size());
    std::vector<long> sub(v.size());
    for (size_t m = 0; m < v.size(); m++) {
        for (int q = 0; q < 4; q++) { fg[m][q] = v[m]->fbuf[q]; fg[m][4 + q] = v[m]->gbuf[q]; }
        sub[m] = v[m]->substep;
    }
    BatchSink K;
    int rc = record_sink(v, 1, LaunchShape{}, K);
    for (size_t m = 0; m < v.size(); m++) {
        for (int q = 0; q < 4; q++) { v[m]->fbuf[q] = fg[m][q]; v[m]->gbuf[q] = fg[m][4 + q]; }
        v[m]->substep = sub[m];
    }
    if (rc) return rc;
    std::vector<BatchRec<SolveBatch>> back4;
    std::vector<BatchRec<PoissonArgs>> pois;
    std::vector<BatchRec<ProjArgs>> proj;
    for (const BatchStage& S : K.stages) {
        if (S.kind == ST_BACK4) back4 = S.back4;
        if (S.kind == ST_PSOLVE) pois = S.poisson;
        if (S.kind == ST_PROJECT) proj = S.project;
    }
    if (back4.size() != v.size() || pois.size() != v.size() || proj.size() != v.size()) return CF_OK;
    // scratch: four fields and two row-sum blocks per member
    size_t need = 0;
    std::vector<size_t> off(v.size());
    for (size_t m = 0; m < v.size(); m++) {
        const Geo& G = v[m]->geo;
        const size_t nw = (size_t) ((G.plane + SOLVE_THREADS_MAX - 1) / SOLVE_THREADS_MAX) * (SOLVE_THREADS_MAX / 32);
        off[m] = need;
        need += 4 * (size_t) G.plane * G.n2 + 2 * nw * G.n2;
    }
    size_t free_b = 0, total_b = 0;
    CF_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (need * sizeof(double) > free_b / 2) return CF_OK;   // no room: defaults
    double* scr = nullptr;
    CF_CUDA(cudaMalloc(&scr, need * sizeof(double)));
    for (size_t m = 0; m < v.size(); m++) {
        const Geo& G = v[m]->geo;
        const size_t fsz = (size_t) G.plane * G.n2;
        double* base = scr + off[m];
        const size_t nw = (size_t) ((G.plane + SOLVE_THREADS_MAX - 1) / SOLVE_THREADS_MAX) * (SOLVE_THREADS_MAX / 32);
        for (int q = 0; q < 4; q++) back4[m].A.a[q].x = base + q * fsz;
        back4[m].A.a[0].partial = back4[m].A.a[0].partial ? base + 4 * fsz : nullptr;
        back4[m].A.a[2].partial = back4[m].A.a[2].partial ? base + 4 * fsz + nw * G.n2 : nullptr;
        proj[m].A.u = base;
        proj[m].A.v = base + fsz;
        proj[m].A.w = base + 2 * fsz;
        proj[m].A.c = base + 3 * fsz;
    }
    // one program per candidate (records regridded with the candidate
    // shape), built and uploaded at its first (warm-up) launch
    std::map<std::array<int, 5>, BatchProgram> progs;
    auto run = [&](int kind, const LaunchShape& sh) {
        const std::array<int, 5> code{kind, sh.solve_threads, sh.pois_threads, sh.proj_bx, sh.proj_by};
        auto it = progs.find(code);
        if (it != progs.end()) {
            run_program(it->second, st);
            return;
        }
        BatchProgram P;
        auto order = [](const auto& r) { return r.G.order; };
        auto none = [](const auto&) { return 0; };
        if (kind == 0) {
            auto recs = back4;
            for (auto& r : recs) { r.G.shape = sh; dim3 g = grid_back4(r.G); r.gx = g.x; r.gy = g.y; r.gz = g.z; }
            add_groups(P, BK_BACK4, recs, order, none, back4_block(recs));
        } else if (kind == 1) {
            auto recs = pois;
            for (auto& r : recs) { r.G.shape = sh; dim3 g = grid_poisson(r.G); r.gx = g.x; r.gy = g.y; r.gz = g.z; }
            add_groups(P, BK_POISSON, recs, order, none, poisson_block(recs));
        } else {
            auto recs = proj;
            for (auto& r : recs) { r.G.shape = sh; dim3 g = grid_project(r.G); r.gx = g.x; r.gy = g.y; r.gz = g.z; }
            add_groups(P, BK_PROJECT, recs, order, none, project_block(recs));
        }
        if (upload(P, st) != CF_OK) return;
        run_program(P, st);
        progs.emplace(code, P);
    };
    rc = tune_shapes(st, true, run, out);
    cudaStreamSynchronize(st);
    for (auto& kv : progs)
        if (kv.second.dblob) cudaFree(kv.second.dblob);
    cudaFree(scr);
    if (rc) {
        out = LaunchShape{};
        return rc;
    }
    tune_store(key, out);
    return CF_OK;
}

// ======================================================================= C ABI

extern "C" {

const char* cf_strerror(int status)
{
    switch (status) {
    case CF_OK: return "ok";
    case CF_EINVAL: return "invalid argument or unsupported configuration";
    case CF_ENOMEM: return "out of memory";
    case CF_ECUDA: return g_last_error.empty() ? "CUDA runtime error" : g_last_error.c_str();
    case CF_EPIVOT: return "zero pivot in a band factorisation";
    case CF_ENONFINITE: return "non-finite value";
    case CF_EIO: return "file I/O error";
    case CF_ETIMEOUT: return "a device wait for an asynchronous copy gave up";
    default: return "unknown status";
    }
}

int cf_destroy(cf_instance* I)
{
    if (!I) return CF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(I->device);
    if (I->stream) cudaStreamSynchronize(I->stream);
    if (I->gexec) cudaGraphExecDestroy(I->gexec);
    if (I->graph) cudaGraphDestroy(I->graph);
    // fbuf[0] and gbuf[0] are the bases of the two four-field blocks
    void* bufs[] = {I->u, I->v, I->w, I->c, I->p, I->fbuf[0], I->gbuf[0], I->spec, I->scratch, I->partial,
                    I->partial_c, I->avg, I->avg_c, I->dscal, I->dcount, I->dlog, I->staging, I->coef, I->twx,
                    I->twy};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (I->hrec) cudaFree(I->hrec);
    if (I->own_stream && I->stream) cudaStreamDestroy(I->stream);
    cudaSetDevice(prev);
    delete I;
    return CF_OK;
}

static int create_impl(const cf_config* cfg, void* stream, cf_instance* I)
{
    I->cfg = *cfg;
    const cf_config& C = *cfg;
    CF_CUDA(cudaGetDevice(&I->device));
    I->m = make_metrics(C.order, C.nx, C.ny, C.nz, GZ, C.lx, C.ly, C.lz);
    Geo& G = I->geo;
    G.order = C.order;
    G.nx = C.nx;
    G.ny = C.ny;
    G.nz = C.nz;
    G.n2 = C.nz + 2 * GZ;
    G.nkx = C.nx / 2 + 1;
    G.plane = (long long) C.nx * C.ny;
    G.splane = (long long) G.nkx * C.ny;
    G.dx = I->m.dx;
    G.dy = I->m.dy;
    G.dxdy = I->m.dx * I->m.dy;
    G.idx = 1.0 / I->m.dx;
    G.idy = 1.0 / I->m.dy;
    if (stream) {
        I->stream = (cudaStream_t) stream;
    } else {
        CF_CUDA(cudaStreamCreateWithFlags(&I->stream, cudaStreamNonBlocking));
        I->own_stream = true;
    }
    const size_t fb = (size_t) G.plane * G.n2 * sizeof(double);
    double** fl[] = {&I->u, &I->v, &I->w, &I->c, &I->p};
    for (double** pp : fl) {
        CF_CUDA(cudaMalloc(pp, fb));
        CF_CUDA(cudaMemsetAsync(*pp, 0, fb, I->stream));
    }
    // the previous- and current-stage right-hand sides of u, v, w, c: two
    // blocks of four consecutive fields (the channel scheme transforms a
    // block in one batched launch)
    for (double** blk : {I->fbuf, I->gbuf}) {
        CF_CUDA(cudaMalloc(&blk[0], 4 * fb));
        CF_CUDA(cudaMemsetAsync(blk[0], 0, 4 * fb, I->stream));
        for (int q = 1; q < 4; q++) blk[q] = blk[0] + q * G.plane * G.n2;
    }
    const size_t nspec = (C.scheme == CF_SCHEME_CHANNEL ? 4 : 1) * (size_t) G.splane * G.n2;
    CF_CUDA(cudaMalloc(&I->spec, nspec * sizeof(double2)));
    CF_CUDA(cudaMemsetAsync(I->spec, 0, nspec * sizeof(double2), I->stream));
    const int nscr = C.order == 4 ? 3 : 1;
    size_t nscratch = (size_t) nscr * G.splane * G.n2;
    if (helm_fused(I)) nscratch = std::max(nscratch, 4 * helm_scratch_stride(I));   // one per field
    CF_CUDA(cudaMalloc(&I->scratch, nscratch * sizeof(double)));
    // per-warp partial sums of k_back4, for its largest block size
    const long long nwarps = ((G.plane + SOLVE_THREADS_MAX - 1) / SOLVE_THREADS_MAX) * (SOLVE_THREADS_MAX / 32);
    CF_CUDA(cudaMalloc(&I->partial, (size_t) nwarps * G.n2 * sizeof(double)));
    CF_CUDA(cudaMalloc(&I->partial_c, (size_t) nwarps * G.n2 * sizeof(double)));
    CF_CUDA(cudaMalloc(&I->avg, (size_t) G.n2 * sizeof(double)));
    CF_CUDA(cudaMalloc(&I->avg_c, (size_t) G.n2 * sizeof(double)));
    CF_CUDA(cudaMalloc(&I->dscal, 8 * sizeof(double)));
    CF_CUDA(cudaMemsetAsync(I->dscal, 0, 8 * sizeof(double), I->stream));
    CF_CUDA(cudaMalloc(&I->dcount, sizeof(long long)));
    CF_CUDA(cudaMemsetAsync(I->dcount, 0, sizeof(long long), I->stream));
    I->log_cap = 3 * 4096;
    CF_CUDA(cudaMalloc(&I->dlog, (size_t) I->log_cap * LOG_COLS * sizeof(double)));
    CF_CUDA(cudaMemsetAsync(I->dlog, 0, (size_t) I->log_cap * LOG_COLS * sizeof(double), I->stream));
    // FFT plans
    auto plan = [&](int n, FftPlan& P, double2*& tw) -> int {
        std::vector<int> r = fft_radices(n);
        P.n = n;
        P.nstages = (int) r.size();
        for (int q = 0; q < P.nstages; q++) P.radix[q] = r[q];
        std::vector<double2> t(n);
        for (int q = 0; q < n; q++) {
            double a = 2.0 * M_PI * (double) q / (double) n;
            t[q] = make_double2(std::cos(a), -std::sin(a));
        }
        CF_CUDA(cudaMalloc(&tw, n * sizeof(double2)));
        CF_CUDA(cudaMemcpy(tw, t.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
        P.tw = tw;
        return CF_OK;
    };
    int rc = plan(C.nx, I->px, I->twx);
    if (rc) return rc;
    rc = plan(C.ny, I->py, I->twy);
    if (rc) return rc;
    I->c8 = std::cos(M_PI / 4.0);
    CF_CUDA(fft_set_smem_limits(std::max(C.nx, C.ny)));
    CF_CUDA(rhs_set_smem_limits());
    I->bc_ub = to_dev(bc_rows_u(I->m, true));
    I->bc_ut = to_dev(bc_rows_u(I->m, false));
    I->bc_wb = to_dev(bc_rows_w(I->m, true));
    I->bc_wt = to_dev(bc_rows_w(I->m, false));
    rc = build_tables(I, C.dt);
    if (rc) return rc;
    CF_CUDA(cudaStreamSynchronize(I->stream));
    return tune_instance(I);
}

int cf_create(const cf_config* cfg, void* stream, cf_instance** out)
{
    if (!out) return CF_EINVAL;
    *out = nullptr;
    int rc = check_config(cfg);
    if (rc) return rc;
    cf_instance* I = new (std::nothrow) cf_instance();
    if (!I) return CF_ENOMEM;
    const char* fp = std::getenv("CF_FUSE_PRESSURE");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 0;
    if (fp && fp[0] == '0') I->fuse_pressure = false;
    else if (fp && fp[0] == '1') I->fuse_pressure = true;
    else I->fuse_pressure = sms > 0 && 2 * (cfg->nx / 2 + 1) >= sms;
    rc = create_impl(cfg, stream, I);
    if (rc) {
        cf_destroy(I);
        return rc;
    }
    *out = I;
    return CF_OK;
}

static double* field_ptr(cf_instance* I, int f)
{
    switch (f) {
    case CF_U: return I->u;
    case CF_V: return I->v;
    case CF_W: return I->w;
    case CF_C: return I->c;
    case CF_P: return I->p;
    default: return nullptr;
    }
}

static int layout_dims(cf_instance* I, int layout, int& A, int& B, int& K, int& ox, int& oy, int& oz)
{
    const cf_config& C = I->cfg;
    if (layout == CF_LAYOUT_PADDED) {
        A = C.nx + 2 * C.ngx; B = C.ny + 2 * C.ngy; K = C.nz + 2 * GZ;
        ox = C.ngx; oy = C.ngy; oz = 0;
    } else if (layout == CF_LAYOUT_INTERIOR) {
        A = C.nx; B = C.ny; K = C.nz;
        ox = 0; oy = 0; oz = GZ;
    } else {
        return CF_EINVAL;
    }
    return CF_OK;
}

static int ensure_staging(cf_instance* I, size_t n)
{
    if (I->staging_elems >= n) return CF_OK;
    if (I->staging) cudaFree(I->staging);
    I->staging = nullptr;
    I->staging_elems = 0;
    CF_CUDA(cudaMalloc(&I->staging, n * sizeof(double)));
    I->staging_elems = n;
    return CF_OK;
}

int cf_set_field(cf_instance* I, int field, const double* host, int layout)
{
    if (!I || !host || field < CF_U || field > CF_C) return CF_EINVAL;
    int A, B, K, ox, oy, oz;
    if (layout_dims(I, layout, A, B, K, ox, oy, oz)) return CF_EINVAL;
    size_t n = (size_t) A * B * K;
    int rc = ensure_staging(I, n);
    if (rc) return rc;
    CF_CUDA(cudaMemcpyAsync(I->staging, host, n * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    dim3 blk(32, 8), grd((K + 31) / 32, (I->geo.ny + 31) / 32, I->geo.nx);
    k_host2dev<<<grd, blk, 0, I->stream>>>(I->geo, I->staging, field_ptr(I, field), B, K, ox, oy, oz);
    CF_CUDA(cudaGetLastError());
    CF_CUDA(cudaMemsetAsync(I->dscal + 2, 0, 2 * sizeof(double), I->stream));
    CF_CUDA(cudaStreamSynchronize(I->stream));
    return CF_OK;
}

int cf_get_field(cf_instance* I, int field, double* host, int layout)
{
    if (!I || !host || field < CF_U || field > CF_P) return CF_EINVAL;
    int A, B, K, ox, oy, oz;
    if (layout_dims(I, layout, A, B, K, ox, oy, oz)) return CF_EINVAL;
    size_t n = (size_t) A * B * K;
    int rc = ensure_staging(I, n);
    if (rc) return rc;
    dim3 blk(32, 8), grd((K + 31) / 32, (B + 31) / 32, A);
    k_dev2host<<<grd, blk, 0, I->stream>>>(I->geo, field_ptr(I, field), I->staging, A, B, K, ox, oy, oz);
    CF_CUDA(cudaGetLastError());
    CF_CUDA(cudaMemcpyAsync(host, I->staging, n * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    CF_CUDA(cudaStreamSynchronize(I->stream));
    return CF_OK;
}

int cf_init_fields(cf_instance* I, unsigned long long seed, double amp, double c_amp)
{
    if (!I) return CF_EINVAL;
    const Geo& G = I->geo;
    dim3 blk(128), grd((G.ny + 127) / 128, G.nx, G.n2);
    k_init_raw<<<grd, blk, 0, I->stream>>>(G, I->u, I->v, I->w, I->c, I->zp, seed, amp, c_amp);
    CF_CUDA(cudaGetLastError());
    CF_CUDA(cudaMemsetAsync(I->dscal + 2, 0, 2 * sizeof(double), I->stream));
    pressure_sequence(I, I->pois_init, 1.0, 0, false);
    CF_CUDA(cudaGetLastError());
    CF_CUDA(cudaStreamSynchronize(I->stream));
    return CF_OK;
}

int cf_step(cf_instance* I, int nsub)
{
    if (!I || nsub < 0) return CF_EINVAL;
    for (int q = 0; q < nsub; q++) {
        enqueue_substep(I);
        CF_CUDA(cudaGetLastError());
    }
    return CF_OK;
}

int cf_step_graph(cf_instance* I, int nsteps)
{
    if (!I || nsteps < 0) return CF_EINVAL;
    // align to the start of an RK3 step
    while (I->substep % 3 != 0 && nsteps > 0) {
        int rc = cf_step(I, 1);
        if (rc) return rc;
    }
    // The graph holds two RK3 steps: an even number of f/g swaps leaves the
    // buffer roles where capture found them.
    while (nsteps >= 2) {
        if (!I->gexec) {
            long saved = I->substep;
            CF_CUDA(cudaStreamBeginCapture(I->stream, cudaStreamCaptureModeThreadLocal));
            for (int q = 0; q < 6; q++) enqueue_substep(I);
            cudaError_t e = cudaStreamEndCapture(I->stream, &I->graph);
            I->substep = saved;
            CF_CUDA(e);
            CF_CUDA(cudaGraphInstantiate(&I->gexec, I->graph, 0));
        }
        CF_CUDA(cudaGraphLaunch(I->gexec, I->stream));
        I->substep += 6;
        nsteps -= 2;
    }
    if (nsteps > 0) return cf_step(I, 3 * nsteps);
    return CF_OK;
}

// CF_ENONFINITE once a mass-control kernel has found a NaN / Inf bulk mean
// of u or c, CF_ETIMEOUT once a kernel gave up waiting for one of its own
// asynchronous copies (the caller has synchronised the instance's stream).
// Both flags are cleared when fields are set again.
static int finite_status(cf_instance* I)
{
    double flag[2] = {0.0, 0.0};
    CF_CUDA(cudaMemcpy(flag, I->dscal + 2, sizeof(flag), cudaMemcpyDeviceToHost));
    if (flag[1] != 0.0) return CF_ETIMEOUT;
    return flag[0] != 0.0 ? CF_ENONFINITE : CF_OK;
}

int cf_sync(cf_instance* I)
{
    if (!I) return CF_EINVAL;
    CF_CUDA(cudaStreamSynchronize(I->stream));
    return finite_status(I);
}

long cf_substeps_done(const cf_instance* I) { return I ? I->substep : CF_EINVAL; }

long cf_get_log(cf_instance* I, double* out, long max_rows)
{
    if (!I || max_rows < 0) return CF_EINVAL;
    CF_CUDA(cudaStreamSynchronize(I->stream));
    if (int rc = finite_status(I)) return rc;
    long long count = 0;
    CF_CUDA(cudaMemcpy(&count, I->dcount, sizeof(count), cudaMemcpyDeviceToHost));
    long long avail = count < I->log_cap ? count : I->log_cap;
    long long nret = avail < max_rows ? avail : max_rows;
    if (!out || nret == 0) return (long) nret;
    std::vector<double> all((size_t) I->log_cap * LOG_COLS);
    CF_CUDA(cudaMemcpy(all.data(), I->dlog, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (long long r = 0; r < nret; r++) {
        long long row = count - nret + r;
        std::memcpy(out + r * LOG_COLS, all.data() + (row % I->log_cap) * LOG_COLS, LOG_COLS * sizeof(double));
    }
    return (long) nret;
}

int cf_max_divergence(cf_instance* I, double* out)
{
    if (!I || !out) return CF_EINVAL;
    const int nb = 592;
    double* d = nullptr;
    CF_CUDA(cudaMalloc(&d, nb * sizeof(double)));
    if (I->cfg.order == 2) k_max_div<2><<<nb, 256, 0, I->stream>>>(I->geo, I->u, I->v, I->w, d);
    else k_max_div<4><<<nb, 256, 0, I->stream>>>(I->geo, I->u, I->v, I->w, d);
    std::vector<double> h(nb);
    cudaError_t e = cudaMemcpyAsync(h.data(), d, nb * sizeof(double), cudaMemcpyDeviceToHost, I->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(I->stream);
    cudaFree(d);
    CF_CUDA(e);
    double m = 0.0;
    for (double x : h) m = std::fmax(m, x);
    *out = m;
    return CF_OK;
}

// Device address of g_divmax_rows on each device, looked up once per device
// (with that device current) by the first cf_max_divergence_noalloc call there.
static std::mutex g_noalloc_mu;
static double* g_noalloc_rows[256] = {};

int cf_max_divergence_noalloc(cf_instance* I, double* out)
{
    if (!I || !out) return CF_EINVAL;
    if (I->cfg.nz > CF_NOALLOC_MAX_ROWS) {
        g_last_error = "cf_max_divergence_noalloc: nz exceeds its fixed scratch of "
                       + std::to_string(CF_NOALLOC_MAX_ROWS) + " rows";
        return CF_EINVAL;
    }
    if (I->device < 0 || I->device >= 256) return CF_EINVAL;
    int prev = 0;
    CF_CUDA(cudaGetDevice(&prev));
    if (prev != I->device) CF_CUDA(cudaSetDevice(I->device));
    double* rows = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_rows[I->device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_divmax_rows);
            if (e != cudaSuccess) {
                g_last_error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                if (prev != I->device) cudaSetDevice(prev);
                return CF_ECUDA;
            }
            g_noalloc_rows[I->device] = (double*) p;
        }
        rows = g_noalloc_rows[I->device];
    }
    const int nz = I->cfg.nz;
    if (I->cfg.order == 2) k_max_div_rows<2><<<nz, 256, 0, I->stream>>>(I->geo, I->u, I->v, I->w, rows);
    else k_max_div_rows<4><<<nz, 256, 0, I->stream>>>(I->geo, I->u, I->v, I->w, rows);
    k_max_rows_final<<<1, 256, 0, I->stream>>>(rows, nz, rows + CF_NOALLOC_MAX_ROWS);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, rows + CF_NOALLOC_MAX_ROWS, sizeof(double), cudaMemcpyDeviceToHost, I->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(I->stream);
    if (prev != I->device) cudaSetDevice(prev);
    CF_CUDA(e);
    return CF_OK;
}

int cf_cfl(cf_instance* I, double dt, double* cfl)
{
    if (!I || !cfl) return CF_EINVAL;
    const int nb = 592;
    double* d = nullptr;
    CF_CUDA(cudaMalloc(&d, nb * sizeof(double)));
    k_cfl<<<nb, 256, 0, I->stream>>>(I->geo, I->u, I->v, I->w, dt, d);
    std::vector<double> h(nb);
    cudaError_t e = cudaMemcpyAsync(h.data(), d, nb * sizeof(double), cudaMemcpyDeviceToHost, I->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(I->stream);
    cudaFree(d);
    CF_CUDA(e);
    double m = 0.0;
    for (double x : h) m = std::fmax(m, x);
    *cfl = m;
    return CF_OK;
}

int cf_set_dt(cf_instance* I, double dt)
{
    if (!I || !(dt > 0.0)) return CF_EINVAL;
    CF_CUDA(cudaStreamSynchronize(I->stream));
    return build_tables(I, dt);
}

int cf_device_field(cf_instance* I, int field, double** dev_ptr, long long* n_elems)
{
    if (!I || !dev_ptr) return CF_EINVAL;
    double* p = field_ptr(I, field);
    if (!p) return CF_EINVAL;
    *dev_ptr = p;
    if (n_elems) *n_elems = I->geo.plane * I->geo.n2;
    return CF_OK;
}

int cf_profile(cf_instance* I, int nsub, double* ms)
{
    if (!I || !ms || nsub <= 0) return CF_EINVAL;
    Timeline tl;
    for (int g = 0; g <= CF_NKERNEL_GROUPS; g++) CF_CUDA(cudaEventCreate(&tl.ev[g]));
    for (int g = 0; g < CF_NKERNEL_GROUPS; g++) ms[g] = 0.0;
    int rc = CF_OK;
    for (int q = 0; q < nsub && rc == CF_OK; q++) {
        tl.n = 0;
        enqueue_substep(I, &tl);
        cudaError_t e = cudaStreamSynchronize(I->stream);
        if (e != cudaSuccess || tl.n != CF_NKERNEL_GROUPS + 1) {
            g_last_error = cudaGetErrorString(e);
            rc = CF_ECUDA;
            break;
        }
        for (int g = 0; g < CF_NKERNEL_GROUPS; g++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, tl.ev[g], tl.ev[g + 1]);
            ms[g] += t;
        }
    }
    for (int g = 0; g <= CF_NKERNEL_GROUPS; g++) cudaEventDestroy(tl.ev[g]);
    return rc;
}

int cf_batch_step(cf_instance** members, int n, int nsub, void* stream)
{
    int rc = check_members(members, n);
    if (rc) return rc;
    if (nsub < 0) return CF_EINVAL;
    if (nsub == 0) return CF_OK;
    std::vector<cf_instance*> v(members, members + n);
    cudaStream_t st = stream ? (cudaStream_t) stream : v[0]->stream;
    BatchProgram P;
    rc = record(v, nsub, P, batch_cached_shape(v));
    if (rc) return rc;
    cudaEvent_t ev;
    CF_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    rc = join_streams(v, st, ev, true);
    if (rc == CF_OK) rc = upload(P, st);
    if (rc == CF_OK) {
        run_program(P, st);
        cudaError_t e = cudaGetLastError();
        cudaFreeAsync(P.dblob, st);
        if (e != cudaSuccess) {
            g_last_error = cudaGetErrorString(e);
            rc = CF_ECUDA;
        }
    }
    if (rc == CF_OK) rc = join_streams(v, st, ev, false);
    cudaEventDestroy(ev);
    return rc;
}

int cf_set_tuning(int on)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_mode = on ? 1 : 0;
    return CF_OK;
}

static void shape_out(const LaunchShape& S, int* out)
{
    out[0] = S.solve_threads;
    out[1] = S.pois_threads;
    out[2] = S.proj_bx;
    out[3] = S.proj_by;
}

int cf_get_launch_shape(const cf_instance* I, int shape[4])
{
    if (!I || !shape) return CF_EINVAL;
    shape_out(I->geo.shape, shape);
    return CF_OK;
}

int cf_set_launch_shape(cf_instance* I, const int shape[4])
{
    if (!I || !shape) return CF_EINVAL;
    LaunchShape S;
    S.solve_threads = shape[0];
    S.pois_threads = shape[1];
    S.proj_bx = shape[2];
    S.proj_by = shape[3];
    if (!shape_valid(S)) return CF_EINVAL;
    I->geo.shape = S;
    // the captured graph holds the old launches
    if (I->gexec) { cudaGraphExecDestroy(I->gexec); I->gexec = nullptr; }
    if (I->graph) { cudaGraphDestroy(I->graph); I->graph = nullptr; }
    return CF_OK;
}

int cf_batch_get_launch_shape(const cf_batch* B, int shape[4])
{
    if (!B || !shape) return CF_EINVAL;
    shape_out(B->shape, shape);
    return CF_OK;
}

int cf_batch_destroy(cf_batch* B)
{
    if (!B) return CF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(B->device);
    if (B->stream) cudaStreamSynchronize(B->stream);
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    if (B->graph) cudaGraphDestroy(B->graph);
    for (BatchProgram& P : B->half)
        if (P.dblob) cudaFree(P.dblob);
    if (B->ev) cudaEventDestroy(B->ev);
    if (B->own_stream && B->stream) cudaStreamDestroy(B->stream);
    cudaSetDevice(prev);
    delete B;
    return CF_OK;
}

static int batch_create_impl(cf_batch* B, cf_instance** members, int n, void* stream, bool tune)
{
    B->v.assign(members, members + n);
    B->device = members[0]->device;
    if (stream) {
        B->stream = (cudaStream_t) stream;
    } else {
        CF_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
        B->own_stream = true;
    }
    CF_CUDA(cudaEventCreateWithFlags(&B->ev, cudaEventDisableTiming));
    int trc = join_streams(B->v, B->stream, B->ev, true);   // members' pending work first
    if (trc == CF_OK) {
        if (tune) trc = tune_batch(B->v, B->stream, B->shape);
        else B->shape = batch_cached_shape(B->v);
    }
    if (trc) return trc;
    std::vector<long> start;
    for (cf_instance* I : B->v) start.push_back(I->substep);
    for (int h = 0; h < 2; h++) {
        int rc = record(B->v, 3, B->half[h], B->shape);
        if (rc) {
            for (size_t m = 0; m < B->v.size(); m++) B->v[m]->substep = start[m];
            return rc;
        }
    }
    // recording stepped the host state through the whole cycle: the f/g
    // roles are back, the counters are put back
    for (size_t m = 0; m < B->v.size(); m++) {
        B->v[m]->substep = start[m];
        B->coef.push_back(B->v[m]->coef);
    }
    B->expect = start;
    for (BatchProgram& P : B->half) {
        int rc = upload(P, B->stream);
        if (rc) return rc;
    }
    CF_CUDA(cudaStreamSynchronize(B->stream));
    return CF_OK;
}

int cf_batch_create(cf_instance** members, int n, void* stream, cf_batch** out)
{
    return cf_batch_create_opts(members, n, stream, 0, out);
}

int cf_batch_create_opts(cf_instance** members, int n, void* stream, int flags, cf_batch** out)
{
    if (!out || (flags & ~CF_BATCH_NO_TUNE)) return CF_EINVAL;
    *out = nullptr;
    int rc = check_members(members, n);
    if (rc) return rc;
    cf_batch* B = new (std::nothrow) cf_batch();
    if (!B) return CF_ENOMEM;
    int prev = 0;
    CF_CUDA(cudaGetDevice(&prev));
    CF_CUDA(cudaSetDevice(members[0]->device));
    rc = batch_create_impl(B, members, n, stream, !(flags & CF_BATCH_NO_TUNE));
    cudaSetDevice(prev);
    if (rc) {
        cf_batch_destroy(B);
        return rc;
    }
    *out = B;
    return CF_OK;
}

// Run half h of the cycle eagerly and move the members' host state with it.
static int batch_half(cf_batch* B, int h)
{
    run_program(B->half[h], B->stream);
    CF_CUDA(cudaGetLastError());
    for (size_t m = 0; m < B->v.size(); m++) {
        cf_instance* I = B->v[m];
        for (int q = 0; q < 3; q++)
            for (int f = 0; f < 4; f++) std::swap(I->fbuf[f], I->gbuf[f]);
        I->substep += 3;
        B->expect[m] += 3;
    }
    B->cursor ^= 1;
    return CF_OK;
}

int cf_batch_run(cf_batch* B, int nsteps)
{
    if (!B || nsteps < 0) return CF_EINVAL;
    for (size_t m = 0; m < B->v.size(); m++) {
        // stepped outside the batch, or its tables rebuilt (cf_set_dt): the
        // recorded programs no longer describe it
        if (B->v[m]->substep != B->expect[m] || B->v[m]->coef != B->coef[m]) {
            g_last_error = "batch member changed outside the batch; create the batch again";
            return CF_EINVAL;
        }
    }
    int prev = 0;
    CF_CUDA(cudaGetDevice(&prev));
    CF_CUDA(cudaSetDevice(B->device));
    int rc = join_streams(B->v, B->stream, B->ev, true);
    if (rc == CF_OK && nsteps > 0 && B->cursor == 1) {
        rc = batch_half(B, 1);
        nsteps--;
    }
    while (rc == CF_OK && nsteps >= 2) {
        if (!B->gexec) {
            cudaError_t e = cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                run_program(B->half[0], B->stream);
                run_program(B->half[1], B->stream);
                e = cudaStreamEndCapture(B->stream, &B->graph);
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&B->gexec, B->graph, 0);
            if (e != cudaSuccess) {
                g_last_error = std::string("batch graph: ") + cudaGetErrorString(e);
                rc = CF_ECUDA;
                break;
            }
        }
        cudaError_t e = cudaGraphLaunch(B->gexec, B->stream);
        if (e != cudaSuccess) {
            g_last_error = cudaGetErrorString(e);
            rc = CF_ECUDA;
            break;
        }
        for (size_t m = 0; m < B->v.size(); m++) {
            B->v[m]->substep += 6;
            B->expect[m] += 6;
        }
        nsteps -= 2;
    }
    if (rc == CF_OK && nsteps == 1) rc = batch_half(B, 0);
    if (rc == CF_OK) rc = join_streams(B->v, B->stream, B->ev, false);
    cudaSetDevice(prev);
    return rc;
}

int cf_batch_sync(cf_batch* B)
{
    if (!B) return CF_EINVAL;
    CF_CUDA(cudaStreamSynchronize(B->stream));
    return CF_OK;
}

int cf_batch_launches_per_substep(const cf_batch* B)
{
    if (!B) return CF_EINVAL;
    return (int) ((B->half[0].ops.size() + B->half[1].ops.size()) / 6);
}

// Row statistics into host `out` (n2 values); mode as k_row_stat.
static int row_stat(cf_instance* I, int fa, int fb, int mode, double en, double* out)
{
    if (!I || !out) return CF_EINVAL;
    const double* a = field_ptr(I, fa);
    const double* b = mode == 1 ? field_ptr(I, fb) : nullptr;
    if (!a || (mode == 1 && !b)) return CF_EINVAL;
    const Geo& G = I->geo;
    cudaStream_t st = I->stream;
    double* d = nullptr;
    CF_CUDA(cudaMallocAsync(&d, 3 * (size_t) G.n2 * sizeof(double), st));
    double *abar = d + G.n2, *bbar = d + 2 * G.n2;
    if (mode != 0) k_row_stat<<<G.n2, 256, 0, st>>>(G, a, nullptr, nullptr, nullptr, 0, 0.0, abar);
    if (mode == 1) k_row_stat<<<G.n2, 256, 0, st>>>(G, b, nullptr, nullptr, nullptr, 0, 0.0, bbar);
    k_row_stat<<<G.n2, 256, 0, st>>>(G, a, b, mode ? abar : nullptr, mode == 1 ? bbar : nullptr, mode, en, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, (size_t) G.n2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    CF_CUDA(e);
    return CF_OK;
}

int cf_xy_avg(cf_instance* I, int field, double* avg) { return row_stat(I, field, -1, 0, 0.0, avg); }

int cf_xy_corr(cf_instance* I, int fa, int fb, double* corr) { return row_stat(I, fa, fb, 1, 0.0, corr); }

int cf_xy_moment(cf_instance* I, int field, double en, double* moment)
{
    return row_stat(I, field, -1, 2, en, moment);
}

int cf_xy_spec(cf_instance* I, int fa, int fb, double* specx, double* specy)
{
    if (!I || !specx || !specy) return CF_EINVAL;
    const double* a = field_ptr(I, fa);
    const double* b = field_ptr(I, fb);
    if (!a || !b) return CF_EINVAL;
    const Geo& G = I->geo;
    cudaStream_t st = I->stream;
    const size_t nsx = (size_t) (G.nx / 2 + 1) * G.n2 * 2, nsy = (size_t) (G.ny / 2 + 1) * G.n2 * 2;
    const size_t nspec = (size_t) G.splane * G.n2;
    double2* vh = nullptr;
    double* out = nullptr;
    CF_CUDA(cudaMallocAsync(&out, (nsx + nsy) * sizeof(double), st));
    if (fb != fa) CF_CUDA(cudaMallocAsync(&vh, nspec * sizeof(double2), st));
    // FFT3D_FWD of both fields over all n2 rows (chanfast.c:758-765)
    launch_fft2d_field(G, a, I->spec, I->px, I->py, I->c8, st);
    if (vh) launch_fft2d_field(G, b, vh, I->px, I->py, I->c8, st);
    const double2* v2 = vh ? vh : I->spec;
    k_specx<<<dim3(G.nkx, G.n2), 256, 0, st>>>(G, I->spec, v2, out);
    k_specy<<<dim3(G.ny / 2 + 1, G.n2), 256, 0, st>>>(G, I->spec, v2, out + nsx);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(specx, out, nsx * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(specy, out + nsx, nsy * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(out, st);
    if (vh) cudaFreeAsync(vh, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    CF_CUDA(e);
    return CF_OK;
}

int cf_z_coords(const cf_instance* I, double* zp, double* zw)
{
    if (!I) return CF_EINVAL;
    const std::vector<double> p = z_at_p(I->m), w = z_at_w(I->m);
    if (zp) std::memcpy(zp, p.data(), p.size() * sizeof(double));
    if (zw) std::memcpy(zw, w.data(), w.size() * sizeof(double));
    return CF_OK;
}

unsigned long long cf_instance_bytes(const cf_config* c)
{
    if (check_config(c) != CF_OK) return 0;
    // the allocations of create_impl and build_tables
    const unsigned long long n2 = c->nz + 2 * GZ, plane = (unsigned long long) c->nx * c->ny;
    const unsigned long long splane = (unsigned long long) (c->nx / 2 + 1) * c->ny;
    const unsigned long long fb = plane * n2 * 8;
    unsigned long long b = 5 * fb + 8 * fb;                                     // u v w c p, f and g blocks
    b += (c->scheme == CF_SCHEME_CHANNEL ? 4 : 1) * splane * n2 * 16;          // spectra
    unsigned long long scr = (c->order == 4 ? 3 : 1) * splane * n2 * 8;        // band-solve scratch
    if (c->scheme == CF_SCHEME_CHANNEL && (c->ny == 256 || c->ny == 512)) {
        // the fused spectral solves may take one scratch per field, and their records
        const unsigned long long per = (c->order == 4 ? 3ull : 1ull) * n2 * (c->nx / 2 + 1) * (c->ny / 2 + 2) * 8;
        scr = std::max(scr, 4 * per) + 65536;
    }
    b += scr;
    const unsigned long long nwarps = (plane + SOLVE_THREADS_MAX - 1) / SOLVE_THREADS_MAX * (SOLVE_THREADS_MAX / 32);
    b += 2 * nwarps * n2 * 8 + 2 * n2 * 8 + 64 + 8;                            // row sums, averages, scalars
    b += 3ull * 4096 * LOG_COLS * 8;                                           // log ring
    b += (unsigned long long) (c->nx + c->ny) * 16;                            // twiddles
    b += n2 * 8 * 512 + (unsigned long long) (c->nx + c->ny) * 8;              // coefficient tables (bound)
    b += (unsigned long long) (c->nx + 2 * c->ngx) * (c->ny + 2 * c->ngy) * n2 * 8;   // staging
    return b;
}

int cf_debug_stall_copies(cf_instance* I, int on)
{
    if (!I) return CF_EINVAL;
    I->stall_copies = on != 0;
    // a captured graph holds the launches as they were
    if (I->gexec) { cudaGraphExecDestroy(I->gexec); I->gexec = nullptr; }
    if (I->graph) { cudaGraphDestroy(I->graph); I->graph = nullptr; }
    return CF_OK;
}

int cf_pressure_fused(const cf_instance* I)
{
    if (!I) return CF_EINVAL;
    return I->fuse_pressure && poisson_fft_supported(I->geo) ? 1 : 0;
}

int cf_launches_per_substep(const cf_instance* I)
{
    // pressure: div+fftx (two launches for power-of-two nx), ffty, poisson,
    // ffty, fftx_c2r, project.  chanfast: ghosts, rhs + forward sweeps, the
    // four back substitutions, 2 x (row average + mass control).  channel
    // (power-of-two nx only): ghosts, rhs + Helmholtz right-hand sides, fftx,
    // ffty, four spectral solves, ffty, fftx_c2r, apply_bc, 2 x mass control.
    // With power-of-two ny the y transforms and the Poisson solve are one
    // launch (two fewer).
    if (!I) return CF_EINVAL;
    const int pressure = (fftx_batched_supported(I->cfg.nx) ? 7 : 6) - (I->fuse_pressure && poisson_fft_supported(I->geo) ? 2 : 0);
    // the channel scheme's y transforms and four spectral solves: 6 launches, or 1 fused
    return (I->cfg.scheme == CF_SCHEME_CHANNEL ? (helm_fused(I) ? 8 : 13) : 7) + pressure;
}

}  // extern "C"
