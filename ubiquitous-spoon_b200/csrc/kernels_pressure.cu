// Pressure projection: divergence, 2-D real FFT over (x, y), per-wavenumber
// banded Poisson solve in z, inverse FFT, projection.
//
//   k_div_fftx   divergence{2,4} (pressure.c:40-117) fused with the real DFT
//                along x and its 1/nx scaling (fft.c:38-51, 161-177)
//   k_ffty       complex DFT along y, forward with 1/ny (fft.c:97-118,186-202)
//                or backward unscaled
//   k_poisson    pressure_poisson{2,4} (pressure.c:293-443): one thread per
//                (kx, ky) column, Re and Im sharing one factorisation
//   k_fftx_c2r   inverse real DFT along x (fft.c:53-63, 180-183): the
//                half spectrum is completed by Hermitian symmetry, the
//                imaginary parts of the DC and Nyquist bins are ignored
//   k_project    project{2,4} (pressure.c:120-194) fused with the lazily
//                applied mass-flux / scalar-mean corrections of the substep
//                (chanfast.c:516-519, 603-606)
//
// FFTs run in shared memory: a Stockham autosort mixed-radix (2/3/4/5/8)
// transform over L lines of one thread block, twiddles from a host table.
#include <algorithm>
#include <type_traits>

#include "engine.cuh"
#include "host_band.h"
#include "wall.cuh"
#include "batch.cuh"

namespace cf {

__device__ __forceinline__ int wrapp(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by s*i (s = +-1)
__device__ __forceinline__ double2 cmul_si(double2 a, int s)
{
    return s > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

struct FftCtx {
    double2* buf;
    int N, L;
    bool line_major;      // element (pos, line) at buf[line*N + pos], else buf[pos*L + line]
    int sign;             // -1 forward, +1 backward
    const double2* tw;    // exp(-2 pi i m / N)
    double c8;            // cos(pi/4) from the host table
};

__device__ __forceinline__ int fidx(const FftCtx& F, int pos, int line)
{
    return F.line_major ? line * F.N + pos : pos * F.L + line;
}

__device__ __forceinline__ double2 twid(const FftCtx& F, int m)
{
    double2 t = __ldg(&F.tw[m]);
    if (F.sign > 0) t.y = -t.y;
    return t;
}

template <int R>
__device__ __forceinline__ void dft_small(double2* v, const FftCtx& F)
{
    const int s = F.sign;
    if (R == 2) {
        double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        double2 t2 = cadd(v[1], v[3]), t3 = cmul_si(csub(v[1], v[3]), s);
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    } else if (R == 8) {
        double2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft_small<4>(e, F);
        dft_small<4>(o, F);
        const double c = F.c8;
        // W8^1 = c (1 + s i), W8^2 = s i, W8^3 = c (-1 + s i)
        double2 o1 = make_double2(c * (o[1].x - s * o[1].y), c * (o[1].y + s * o[1].x));
        double2 o2 = cmul_si(o[2], s);
        double2 o3 = make_double2(c * (-o[3].x - s * o[3].y), c * (-o[3].y + s * o[3].x));
        v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);   v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);   v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);   v[7] = csub(e[3], o3);
    } else {
        // generic (3, 5): roots of unity from the host table
        double2 out[R];
        const int step = F.N / R;
#pragma unroll
        for (int q = 0; q < R; q++) {
            double2 acc = v[0];
#pragma unroll
            for (int r = 1; r < R; r++) acc = cadd(acc, cmul(v[r], twid(F, ((r * q) % R) * step)));
            out[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < R; q++) v[q] = out[q];
    }
}

// One Stockham stage of radix R (Ns = product of the previous radices).
template <int R, int MAXB>
__device__ void fft_stage(const FftCtx& F, int Ns)
{
    const int NR = F.N / R;
    const int nb = NR * F.L;
    const int nthr = blockDim.x, tid = threadIdx.x;
    double2 v[MAXB][R];
    int jj[MAXB], ll[MAXB];
#pragma unroll
    for (int t = 0; t < MAXB; t++) {
        int b = tid + t * nthr;
        jj[t] = -1;
        if (b < nb) {
            int line, j;
            if (F.line_major) { line = b / NR; j = b - line * NR; }
            else { j = b / F.L; line = b - j * F.L; }
            jj[t] = j;
            ll[t] = line;
            int k = j % Ns;
            int tstep = F.N / (Ns * R);
#pragma unroll
            for (int r = 0; r < R; r++) {
                double2 a = F.buf[fidx(F, j + r * NR, line)];
                if (r > 0 && k > 0) a = cmul(a, twid(F, (r * k * tstep) % F.N));
                v[t][r] = a;
            }
            dft_small<R>(v[t], F);
        }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < MAXB; t++) {
        if (jj[t] < 0) continue;
        int j = jj[t], k = j % Ns;
        int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) F.buf[fidx(F, idxD + r * Ns, ll[t])] = v[t][r];
    }
    __syncthreads();
}

// Full transform; `plan` radices multiply to N.  MAXC bounds N*L/blockDim.
template <int MAXC>
__device__ void fft_run(const FftCtx& F, const FftPlan& plan)
{
    int Ns = 1;
    for (int s = 0; s < plan.nstages; s++) {
        int R = plan.radix[s];
        switch (R) {
        case 2: fft_stage<2, MAXC / 2>(F, Ns); break;
        case 3: fft_stage<3, MAXC / 3 + 1>(F, Ns); break;
        case 4: fft_stage<4, MAXC / 4>(F, Ns); break;
        case 5: fft_stage<5, MAXC / 5 + 1>(F, Ns); break;
        default: fft_stage<8, MAXC / 8>(F, Ns); break;
        }
        Ns *= R;
    }
}

constexpr int FFT_L = 8;        // lines per block (x transforms: 8 consecutive j)
constexpr int FFT_THREADS = 256;
constexpr int FFT_MAXC = 16;    // N * L / threads for N <= 512

// ---------------------------------------------- transforms of a fixed size
//
// The same Stockham stages with the size known at compile time: the radix
// sequence (that of fft_radices: 8s, then 4s, 2s, 3s, 5s), every index and
// twiddle exponent fold to constants, and the y transforms' line-major
// buffer is padded by one slot per 8 (plus one per line) so that the
// first stages' strided writes spread over the banks.  Used for the sizes
// of STATIC_FFT_SIZES; other non-power-of-two sizes take the runtime plan.

__host__ __device__ constexpr int radix_count(int n)
{
    int c = 0;
    while (n % 8 == 0 && n > 8) { c++; n /= 8; }
    if (n == 8) { c++; n = 1; }
    while (n % 4 == 0) { c++; n /= 4; }
    while (n % 2 == 0) { c++; n /= 2; }
    while (n % 3 == 0) { c++; n /= 3; }
    while (n % 5 == 0) { c++; n /= 5; }
    return c;
}

__host__ __device__ constexpr int radix_at(int n, int s)
{
    int c = 0;
    while (n % 8 == 0 && n > 8) { if (c++ == s) return 8; n /= 8; }
    if (n == 8) { if (c++ == s) return 8; n = 1; }
    while (n % 4 == 0) { if (c++ == s) return 4; n /= 4; }
    while (n % 2 == 0) { if (c++ == s) return 2; n /= 2; }
    while (n % 3 == 0) { if (c++ == s) return 3; n /= 3; }
    while (n % 5 == 0) { if (c++ == s) return 5; n /= 5; }
    return 1;
}

template <int N>
__host__ __device__ constexpr int lm_stride() { return N + N / 8 + 1; }

// Slot of element `pos` of line `line`: line-major padded (y transforms)
// or position-major with FFT_L interleaved lines (x transforms).
template <int N, bool LM>
__device__ __forceinline__ int sslot(int pos, int line)
{
    return LM ? line * lm_stride<N>() + pos + (pos >> 3) : pos * FFT_L + line;
}

template <int N, bool LM, int R, int NS>
__device__ __forceinline__ void fft_stage_s(double2* buf, const FftCtx& F)
{
    constexpr int NR = N / R, NB = NR * FFT_L;
    constexpr int MAXB = (NB + FFT_THREADS - 1) / FFT_THREADS;
    constexpr int TSTEP = N / (NS * R);
    const int tid = threadIdx.x;
    double2 v[MAXB][R];
#pragma unroll
    for (int t = 0; t < MAXB; t++) {
        const int b = tid + t * FFT_THREADS;
        if (b < NB) {
            const int line = LM ? b / NR : b % FFT_L;
            const int j = LM ? b - line * NR : b / FFT_L;
            const int k = j % NS;
            // twiddles w^r of w = exp(-+2 pi i k TSTEP / N): w, w^2 and w^4
            // from the table, w^3, w^5, w^6, w^7 as products (fewer table
            // reads; the transforms are bound by the load pipe)
            double2 cw[8];
            if (k > 0) {
                const int m = k * TSTEP;
                cw[1] = twid(F, m);
                if constexpr (R > 2) cw[2] = twid(F, 2 * m);
                if constexpr (R > 3) cw[3] = cmul(cw[1], cw[2]);
                if constexpr (R > 4) cw[4] = twid(F, 4 * m);
                if constexpr (R > 5) {
                    cw[5] = cmul(cw[1], cw[4]);
                    cw[6] = cmul(cw[2], cw[4]);
                    cw[7] = cmul(cw[3], cw[4]);
                }
            }
#pragma unroll
            for (int r = 0; r < R; r++) {
                double2 a = buf[sslot<N, LM>(j + r * NR, line)];
                if (r > 0 && k > 0) a = cmul(a, cw[r]);
                v[t][r] = a;
            }
            dft_small<R>(v[t], F);
        }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < MAXB; t++) {
        const int b = tid + t * FFT_THREADS;
        if (b < NB) {
            const int line = LM ? b / NR : b % FFT_L;
            const int j = LM ? b - line * NR : b / FFT_L;
            const int k = j % NS;
            const int idxD = (j / NS) * NS * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) buf[sslot<N, LM>(idxD + r * NS, line)] = v[t][r];
        }
    }
    __syncthreads();
}

template <int N, bool LM, int S = 0, int NS = 1>
__device__ __forceinline__ void fft_static(double2* buf, const FftCtx& F)
{
    if constexpr (S < radix_count(N)) {
        constexpr int R = radix_at(N, S);
        fft_stage_s<N, LM, R, NS>(buf, F);
        fft_static<N, LM, S + 1, NS * R>(buf, F);
    }
}

// Sizes with a fixed-size transform kernel (besides the power-of-two ones).
#define STATIC_FFT_SIZES(X) X(48) X(96) X(192) X(384) X(160) X(320)

static bool static_fft_size(int n)
{
#define CASE_(n_) case n_:
    switch (n) {
    STATIC_FFT_SIZES(CASE_) return true;
    default: return false;
    }
#undef CASE_
}

// Dynamic shared memory of the generic transforms of size n.
size_t fft_generic_smem(int n, bool line_major)
{
    if (static_fft_size(n) && line_major) return (size_t) FFT_L * (n + n / 8 + 1) * sizeof(double2);
    return (size_t) n * FFT_L * sizeof(double2);
}

// --------------------------------------------------------- divergence + x FFT


// N: the transform size when it is fixed at compile time, 0 for the runtime plan
template <int ORDER, int N>
__device__ __forceinline__ void k_div_fftx_body(const Geo& G, const DivArgs& A, uint3 bid)
{
    extern __shared__ double2 sbuf[];
    const int k = GZ + A.kshift + bid.y;
    const int j0 = bid.x * FFT_L;
    const int nx = N ? N : G.nx, ny = G.ny, n2 = G.n2;
    const double dx = G.dx, dy = G.dy, dzk = G.dz[k];
    const double uc = A.mu ? A.gu[k] * (*A.mu) : 0.0;   // chanfast.c:516-519
    const bool corr = A.mu != nullptr;
    auto I = [&](int kk, int i, int j) { return ((long long) kk * nx + i) * ny + j; };
    const int kb = GZ - 1, kt = n2 - GZ - 1;
    for (int idx = threadIdx.x; idx < nx * FFT_L; idx += blockDim.x) {
        int i = idx / FFT_L, jj = idx - i * FFT_L, j = j0 + jj;
        double d = 0.0;
        if (j < ny && A.src) {
            d = __ldg(A.src + I(k, i, j));
        } else if (j < ny) {
            auto U = [&](int di) { double t = __ldg(A.u + I(k, wrapp(i + di, nx), j)); return corr ? t + uc : t; };
            auto V = [&](int dj) { return __ldg(A.v + I(k, i, wrapp(j + dj, ny))); };
            auto Wr = [&](int kk) { return __ldg(A.w + I(kk, i, j)); };
            if (ORDER == 2) {
                d = (U(0) - U(-1)) / dx + (V(0) - V(-1)) / dy + (Wr(k) - Wr(k - 1)) / dzk;
            } else {
                double wkm2 = (k - 2 == kb - 1) ? 2.0 * Wr(kb) - Wr(kb + 1) : Wr(k - 2);  // pressure.c:80-87
                double wkp1 = (k + 1 == kt + 1) ? 2.0 * Wr(kt) - Wr(kt - 1) : Wr(k + 1);  // pressure.c:88-95
                d = (A1 * (U(0) - U(-1)) + A2 * (U(1) - U(-2))) / dx
                  + (A1 * (V(0) - V(-1)) + A2 * (V(1) - V(-2))) / dy
                  + (A1 * (Wr(k) - Wr(k - 1)) + A2 * (wkp1 - wkm2)) / dzk;
            }
        }
        sbuf[i * FFT_L + jj] = make_double2(d, 0.0);
    }
    __syncthreads();
    FftCtx F{sbuf, nx, FFT_L, false, -1, A.px.tw, A.c8};
    if constexpr (N > 0) fft_static<N, false>(sbuf, F);
    else fft_run<FFT_MAXC>(F, A.px);
    const int nkx = G.nkx;
    const double scale = 1.0 / (double) nx;
    for (int idx = threadIdx.x; idx < nkx * FFT_L; idx += blockDim.x) {
        int kx = idx / FFT_L, jj = idx - kx * FFT_L, j = j0 + jj;
        if (j >= ny) continue;
        double2 t = sbuf[kx * FFT_L + jj];
        t.x *= scale;
        t.y *= scale;
        A.spec[((long long) k * nkx + kx) * ny + j] = t;
    }
}

template <int ORDER, int N>
__global__ void __launch_bounds__(FFT_THREADS) k_div_fftx(Geo G, DivArgs A)
{
    k_div_fftx_body<ORDER, N>(G, A, blockIdx);
}

template <int ORDER, int N>
__global__ void __launch_bounds__(FFT_THREADS) k_div_fftx_batch(const BatchRec<DivArgs>* r, int n)
{
    uint3 b;
    const BatchRec<DivArgs>& R = batch_locate(r, n, b);
    k_div_fftx_body<ORDER, N>(R.G, R.A, b);
}

// ------------------------------------------------------------------ y FFT


template <int N>
__device__ __forceinline__ void k_ffty_body(const Geo& G, const FftyArgs& A, uint3 bid)
{
    extern __shared__ double2 sbuf[];
    const int k = A.kfirst + bid.y;
    const int kx0 = bid.x * FFT_L;
    const int ny = N ? N : G.ny, nkx = G.nkx;
    const int nl = min(FFT_L, nkx - kx0);
    double2* base = A.spec + bid.z * A.fstride + ((long long) k * nkx + kx0) * ny;
    auto slot = [&](int idx) {   // idx = line * ny + pos
        if constexpr (N > 0) {
            const int line = idx / N, pos = idx - line * N;
            return sslot<N, true>(pos, line);
        } else {
            return idx;
        }
    };
    for (int idx = threadIdx.x; idx < FFT_L * ny; idx += blockDim.x) {
        int line = idx / ny;
        sbuf[slot(idx)] = line < nl ? base[idx] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    FftCtx F{sbuf, ny, FFT_L, true, A.sign, A.py.tw, A.c8};
    if constexpr (N > 0) fft_static<N, true>(sbuf, F);
    else fft_run<FFT_MAXC>(F, A.py);
    const double scale = 1.0 / (double) ny;
    for (int idx = threadIdx.x; idx < nl * ny; idx += blockDim.x) {
        double2 t = sbuf[slot(idx)];
        if (A.sign < 0) { t.x *= scale; t.y *= scale; }
        base[idx] = t;
    }
}

template <int N>
__global__ void __launch_bounds__(FFT_THREADS) k_ffty(Geo G, FftyArgs A)
{
    k_ffty_body<N>(G, A, blockIdx);
}

template <int N>
__global__ void __launch_bounds__(FFT_THREADS) k_ffty_batch(const BatchRec<FftyArgs>* r, int n)
{
    uint3 b;
    const BatchRec<FftyArgs>& R = batch_locate(r, n, b);
    k_ffty_body<N>(R.G, R.A, b);
}

// ---------------------------------------------------------- inverse x FFT


template <int N>
__device__ __forceinline__ void k_fftx_c2r_body(const Geo& G, const C2rArgs& A, uint3 bid)
{
    extern __shared__ double2 sbuf[];
    const int k = A.kfirst + bid.y;
    const int j0 = bid.x * FFT_L;
    const int nx = N ? N : G.nx, ny = G.ny, nkx = G.nkx;
    const double2* spec = A.spec + bid.z * A.fstride;
    for (int idx = threadIdx.x; idx < nx * FFT_L; idx += blockDim.x) {
        int pos = idx / FFT_L, jj = idx - pos * FFT_L, j = j0 + jj;
        double2 t = make_double2(0.0, 0.0);
        if (j < ny) {
            if (pos < nkx) {
                t = spec[((long long) k * nkx + pos) * ny + j];
                if (pos == 0 || 2 * pos == nx) t.y = 0.0;
            } else {
                t = spec[((long long) k * nkx + (nx - pos)) * ny + j];
                t.y = -t.y;
            }
        }
        sbuf[pos * FFT_L + jj] = t;
    }
    __syncthreads();
    FftCtx F{sbuf, nx, FFT_L, false, +1, A.px.tw, A.c8};
    if constexpr (N > 0) fft_static<N, false>(sbuf, F);
    else fft_run<FFT_MAXC>(F, A.px);
    double* const pz = bid.z == 0 ? A.p[0] : bid.z == 1 ? A.p[1] : bid.z == 2 ? A.p[2] : A.p[3];
    for (int idx = threadIdx.x; idx < nx * FFT_L; idx += blockDim.x) {
        int i = idx / FFT_L, jj = idx - i * FFT_L, j = j0 + jj;
        if (j < ny) pz[((long long) k * nx + i) * ny + j] = sbuf[i * FFT_L + jj].x;
    }
}

template <int N>
__global__ void __launch_bounds__(FFT_THREADS) k_fftx_c2r(Geo G, C2rArgs A)
{
    k_fftx_c2r_body<N>(G, A, blockIdx);
}

template <int N>
__global__ void __launch_bounds__(FFT_THREADS) k_fftx_c2r_batch(const BatchRec<C2rArgs>* r, int n)
{
    uint3 b;
    const BatchRec<C2rArgs>& R = batch_locate(r, n, b);
    k_fftx_c2r_body<N>(R.G, R.A, b);
}

// ------------------------------------------------------------ Poisson in z

// Async global -> shared copies ordered with the thread's other memory
// accesses ("memory" clobber): a ring slot is refilled right after it is read.
__device__ __forceinline__ void cp_async16_ordered(double2* dst, const double2* src)
{
    unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_ordered() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_ordered() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }


template <int ORDER>
__device__ __forceinline__ void fill_bot(const WallRowsD& R, double x0, double x1, double x2,
                                         double& g1, double& g2, double& g3)
{
    // ghost_fill_bot{2,4} with r = 0 (pressure.c:516-522, 728-747)
    if (ORDER == 2) {
        g1 = (R.row[0][2] * x0 - 0.0) / -R.row[0][1];
        g2 = g3 = 0.0;
    } else {
        g1 = (R.row[2][6] * x0) / -R.row[2][5];
        g2 = (R.row[1][4] * g1 + R.row[1][5] * x0 + R.row[1][6] * x1 - 0.0) / -R.row[1][3];
        g3 = (R.row[0][2] * g2 + R.row[0][3] * g1 + R.row[0][4] * x0 + R.row[0][5] * x1
              + R.row[0][6] * x2) / -R.row[0][1];
    }
}

template <int ORDER>
__device__ __forceinline__ void fill_top(const WallRowsD& R, double x0, double x1, double x2,
                                         double& g1, double& g2, double& g3)
{
    // ghost_fill_top{2,4} with r = 0 (pressure.c:525-531, 750-769)
    if (ORDER == 2) {
        g1 = (R.row[0][0] * x0 - 0.0) / -R.row[0][1];
        g2 = g3 = 0.0;
    } else {
        g1 = (R.row[2][0] * x0) / -R.row[2][1];
        g2 = (R.row[1][0] * x1 + R.row[1][1] * x0 + R.row[1][2] * g1 - 0.0) / -R.row[1][3];
        g3 = (R.row[0][0] * x2 + R.row[0][1] * x1 + R.row[0][2] * x0 + R.row[0][3] * g1
              + R.row[0][4] * g2) / -R.row[0][5];
    }
}

// xy-average profile of a Helmholtz solution from its (kx, ky) = (0, 0)
// column: rows GZ .. GZ+n-1 already hold the solved values; the wall ghost
// rows follow from the field's apply_bc closure, which is affine with
// column-independent coefficients and so commutes with the average.  This is
// get_xy_avg (get.c:281-302) of the field after apply_bc (channel.c:480-486),
// rows the closure does not write being zero as they are there.
template <int ORDER>
__device__ void average_walls(const PoissonArgs& A, int n2)
{
    double* avg = A.avg;
    const int kb = GZ - 1, kt = GZ + A.nrows;
    double g1, g2, g3;
    bc_u_bot<ORDER>(A.abot, A.abc_bot, avg[kb + 1], avg[kb + 2], avg[kb + 3], g1, g2, g3);
    for (int k = 0; k < GZ; k++) avg[k] = 0.0;
    avg[kb] = g1;
    if (ORDER == 4) { avg[kb - 1] = g2; avg[kb - 2] = g3; }
    bc_u_top<ORDER>(A.atop, A.abc_top, avg[kt - 1], avg[kt - 2], avg[kt - 3], g1, g2, g3);
    for (int k = kt; k < n2; k++) avg[k] = 0.0;
    avg[kt] = g1;
    if (ORDER == 4) { avg[kt + 1] = g2; avg[kt + 2] = g3; }
}

// Band rows of one (kx, +-ky) column pair: the interior stencil rows with the
// pair's diagonal, and the closure-reduced rows 0..2 and n-3..n-1 (var 1 is
// the (0, 0) mode's closure, pressure.c:331-338).
struct PairRows {
    const PoissonArgs& A;
    double lamx, lamy;
    int var, n;
    __device__ __forceinline__ int bq(int i) const { return i < 3 ? i : (i >= n - 3 ? 6 - (n - i) : -1); }
    // Coefficients of interior row i from its staged table values
    // st = (a, b, c, e, f, g, dpart, cx, cy) of row k = GZ + i.
    __device__ __forceinline__ void coef_from(int i, const double* st, double* cf) const
    {
        const int q = bq(i);
        double d = (st[6] - lamx * st[7]) - lamy * st[8];   // cx = dv dt / dx^2, cy = dv dt / dy^2
        if (q >= 0) {
            d = ((d - A.dsub[var][q][0]) - A.dsub[var][q][1]) - A.dsub[var][q][2];
            for (int t = 0; t < 7; t++) cf[t] = A.red[var][q][t];
        } else {
            cf[0] = st[0]; cf[1] = st[1]; cf[2] = st[2];
            cf[4] = st[3]; cf[5] = st[4]; cf[6] = st[5];
        }
        cf[3] = d;
    }
    // Table value f of row k: a, b, c, e, f, g, dpart, cx, cy, dvol.
    __device__ __forceinline__ double table(int f, int k) const
    {
        switch (f) {
        case 0: return A.a[k];
        case 1: return A.b[k];
        case 2: return A.c[k];
        case 3: return A.e[k];
        case 4: return A.f[k];
        case 5: return A.g[k];
        case 6: return A.dpart[k];
        case 7: return A.cx[k];
        case 8: return A.cy[k];
        default: return A.dvol[k];
        }
    }
    // Coefficients of interior row i (k = GZ + i).
    __device__ __forceinline__ void coef(int i, double* cf) const
    {
        const int k = GZ + i;
        double st[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, A.dpart[k], A.cx[k], A.cy[k]};
        if (bq(i) < 0) {   // closure rows take their band from red
            st[0] = A.a[k]; st[1] = A.b[k]; st[2] = A.c[k];
            st[3] = A.e[k]; st[4] = A.f[k]; st[5] = A.g[k];
        }
        coef_from(i, st, cf);
    }
};

// heptdag.c:5-61 for two complex right-hand sides sharing one factorisation,
// one row per step().  One elimination formula serves every row: with zero
// history (p, q, r, s of rows -3..-1) it reduces exactly to the special forms
// of rows 0..2.
struct HeptSweep {
    double p3 = 0, q3 = 0, r3 = 0, p2 = 0, q2 = 0, r2 = 0, p1 = 0, q1 = 0, r1 = 0;   // rows i-3, i-2, i-1
    double2 s3A = {0, 0}, s2A = {0, 0}, s1A = {0, 0}, s3B = {0, 0}, s2B = {0, 0}, s1B = {0, 0};
    // cf: the row's band (a b c d e f g); hA, hB: right-hand sides already
    // scaled by the cell volume.  Out: the row's multipliers p, q, r and the
    // forward-substituted values.
    __device__ __forceinline__ void step(const double* cf, double2 hA, double2 hB, double& p, double& q, double& r,
                                         double2& svA, double2& svB)
    {
        const double a = cf[0], b = cf[1], c = cf[2], d = cf[3], e = cf[4], f = cf[5], g = cf[6];
        const double alp = b - a * p3;
        const double bet = c - a * q3 - alp * p2;
        const double den = d - a * r3 - alp * q2 - bet * p1;
        const double iden = 1.0 / den;
        p = (e - alp * r2 - bet * q1) * iden;
        q = (f - bet * r1) * iden;
        r = g * iden;
        svA = make_double2((hA.x - a * s3A.x - alp * s2A.x - bet * s1A.x) * iden,
                           (hA.y - a * s3A.y - alp * s2A.y - bet * s1A.y) * iden);
        svB = make_double2((hB.x - a * s3B.x - alp * s2B.x - bet * s1B.x) * iden,
                           (hB.y - a * s3B.y - alp * s2B.y - bet * s1B.y) * iden);
        p3 = p2; q3 = q2; r3 = r2; p2 = p1; q2 = q1; r2 = r1; p1 = p; q1 = q; r1 = r;
        s3A = s2A; s2A = s1A; s1A = svA;
        s3B = s2B; s2B = s1B; s1B = svB;
    }
};

// Back substitution of one heptdag row (heptdag.c:50-55); the previous row's
// x1 enters last: one dependent operation per row.
__device__ __forceinline__ double2 hept_back(double2 sv, double p, double q, double r, double2 x1, double2 x2,
                                             double2 x3)
{
    return make_double2(((sv.x - r * x3.x) - q * x2.x) - p * x1.x, ((sv.y - r * x3.y) - q * x2.y) - p * x1.y);
}

// Banded solve of a pair of (kx, ky) columns over spectrum rows
// GZ .. GZ+n-1: pressure_poisson{2,4} (pressure.c:293-443) with FILL (the
// wall ghost rows of the solution are filled from the closure, as p needs
// them), or solve_helmholtz_{u,w}{2,4} (diffuseu.c:398-614,
// diffusew.c:466-614) without (the field's apply_bc follows the inverse
// transform).  The band matrix depends on ky only through cos(2 pi ky / ny),
// so columns ky and ny - ky share one factorisation: one thread per pair
// eliminates both (Re and Im of each), storing the multipliers once.  ky = 0
// and, for even ny, ky = ny/2 pair with themselves (solved twice, stored
// identically).
template <int ORDER, bool FILL>
__device__ __forceinline__ void band_column(const Geo& G, const PoissonArgs& A, uint3 bid)
{
    const long long ncol = G.splane;
    const int ny = G.ny, n2 = G.n2, n = A.nrows;
    const int nky = ny / 2 + 1;                       // pairs per kx
    const long long npair = (long long) G.nkx * nky;
    const long long pair = (long long) bid.x * blockDim.x + threadIdx.x;
    if (pair >= npair) return;
    const int kx = (int) (pair / nky), ky = (int) (pair - (long long) kx * nky);
    const int kyb = (ny - ky) % ny;
    const long long colA = (long long) kx * ny + ky, colB = (long long) kx * ny + kyb;
    const int var = (kx == 0 && ky == 0) ? 1 : 0;   // pressure.c:331-338
    const double lamx = A.lamx[kx], lamy = A.lamy[ky];
    const bool stats = !FILL && A.avg != nullptr && pair == 0;
    double2* sp = A.spec;
    auto SA = [&](int k) -> double2& { return sp[(long long) k * ncol + colA]; };
    auto SB = [&](int k) -> double2& { return sp[(long long) k * ncol + colB]; };
    auto scal = [](double2 v, double f) { return make_double2(v.x * f, v.y * f); };
    const PairRows rows{A, lamx, lamy, var, n};
    auto coef = [&](int i, double* cf) { rows.coef(i, cf); };
    auto at = [&](double* base, int k) -> double& { return base[(long long) k * npair + pair]; };

    if (ORDER == 2) {
        // tridag.c:4-26; the diagonal is cf[3], the off-diagonals cf[0], cf[2]
        double* gam = A.scratch;
        double cfv[7];
        coef(0, cfv);
        double ibet = 1.0 / cfv[3];
        const double dv0 = A.dvol[GZ];
        const double2 r0A = SA(GZ), r0B = SB(GZ);
        double2 uA = make_double2(r0A.x * dv0 * ibet, r0A.y * dv0 * ibet);
        double2 uB = make_double2(r0B.x * dv0 * ibet, r0B.y * dv0 * ibet);
        SA(GZ) = uA;
        SB(GZ) = uB;
        double cprev = cfv[2];
        for (int i = 1; i < n; i++) {
            const int k = GZ + i;
            coef(i, cfv);
            double gm = cprev * ibet;
            ibet = 1.0 / (cfv[3] - cfv[0] * gm);
            at(gam, k) = gm;
            const double dv = A.dvol[k];
            const double2 rA = SA(k), rB = SB(k);
            uA = make_double2((rA.x * dv - cfv[0] * uA.x) * ibet, (rA.y * dv - cfv[0] * uA.y) * ibet);
            uB = make_double2((rB.x * dv - cfv[0] * uB.x) * ibet, (rB.y * dv - cfv[0] * uB.y) * ibet);
            SA(k) = uA;
            SB(k) = uB;
            cprev = cfv[2];
        }
        double2 nA = uA, nB = uB;
        const double2 topA = uA, topB = uB;
        double2 b0A = uA, b0B = uB;
        if (stats) A.avg[GZ + n - 1] = uA.x;
        for (int i = n - 2; i >= 0; i--) {
            const int k = GZ + i;
            const double gm = at(gam, k + 1);
            double2 tA = SA(k), tB = SB(k);
            tA.x -= gm * nA.x;
            tA.y -= gm * nA.y;
            tB.x -= gm * nB.x;
            tB.y -= gm * nB.y;
            SA(k) = tA;
            SB(k) = tB;
            nA = tA;
            nB = tB;
            if (stats) A.avg[k] = tA.x;
            if (i == 0) { b0A = tA; b0B = tB; }
        }
        if (FILL) {
            auto fill = [&](auto S, double2 b0, double2 top) {
                double g1, g2, g3, h1;
                fill_bot<2>(A.bot[var], b0.x, 0.0, 0.0, g1, g2, g3);
                fill_bot<2>(A.bot[var], b0.y, 0.0, 0.0, h1, g2, g3);
                S(GZ - 1) = make_double2(g1, h1);
                fill_top<2>(A.top, top.x, 0.0, 0.0, g1, g2, g3);
                fill_top<2>(A.top, top.y, 0.0, 0.0, h1, g2, g3);
                S(n2 - GZ) = make_double2(g1, h1);
                for (int k = 0; k < GZ - 1; k++) S(k) = make_double2(0.0, 0.0);
                for (int k = n2 - GZ + 1; k < n2; k++) S(k) = make_double2(0.0, 0.0);
            };
            fill(SA, b0A, topA);
            fill(SB, b0B, topB);
        } else {
            if (GZ + n < n2 - GZ) {   // w: the top wall face
                SA(GZ + n) = make_double2(0.0, 0.0);
                SB(GZ + n) = make_double2(0.0, 0.0);
            }
            if (stats) average_walls<2>(A, n2);
        }
        return;
    }

    // heptdag.c:5-61 with per-pair pivots (HeptSweep); p, q, r spill to
    // scratch.  In the forward sweep each thread keeps the spectrum values of the next
    // POIS_PF rows of both columns in flight as cp.async copies into its own
    // slots of a shared-memory ring; none of those rows has been rewritten yet.
    double* Pp = A.scratch;
    double* Qp = A.scratch + (long long) n2 * npair;
    double* Rp = A.scratch + 2 * (long long) n2 * npair;
    extern __shared__ double2 pring[];
    const int t = threadIdx.x;
    const int nt = blockDim.x;
    auto fslot = [&](int i, int c) { return pring + ((i % POIS_PF) * 2 + c) * nt + t; };
    auto ffetch = [&](int i) {
        if (i < n) {
            cp_async16_ordered(fslot(i, 0), &SA(GZ + i));
            cp_async16_ordered(fslot(i, 1), &SB(GZ + i));
        }
        cp_async_commit_ordered();
    };
    for (int i = 0; i < POIS_PF; i++) ffetch(i);
    HeptSweep H;
    double cf[7];
    for (int i = 0; i < n; i++) {
        const int k = GZ + i;
        cp_async_wait_ordered<POIS_PF - 1>();
        double2 hA = *fslot(i, 0), hB = *fslot(i, 1);
        ffetch(i + POIS_PF);
        coef(i, cf);
        const double dv = A.dvol[k];
        hA = scal(hA, dv);
        hB = scal(hB, dv);
        double p, q, r;
        double2 svA, svB;
        H.step(cf, hA, hB, p, q, r, svA, svB);
        at(Pp, k) = p; at(Qp, k) = q; at(Rp, k) = r;
        SA(k) = svA;
        SB(k) = svB;
    }
    cp_async_wait_ordered<0>();

    // back substitution (heptdag.c:50-55), same general form (x2 = x3 = 0 at
    // the top).  s, p, q, r of row i - POIS_PB are loaded into registers while
    // row i is computed (plain loads: these rows were stored by this thread).
    double2 lsA[POIS_PB], lsB[POIS_PB];
    double lp[POIS_PB], lq[POIS_PB], lr[POIS_PB];
    auto bload = [&](int i, int u) {
        if (i >= 0) {
            const int k = GZ + i;
            lsA[u] = SA(k); lsB[u] = SB(k); lp[u] = at(Pp, k); lq[u] = at(Qp, k); lr[u] = at(Rp, k);
        }
    };
#pragma unroll
    for (int u = 0; u < POIS_PB; u++) bload(n - 2 - u, u);
    double2 x1A = SA(GZ + n - 1), x2A = make_double2(0, 0), x3A = x2A;
    double2 x1B = SB(GZ + n - 1), x2B = x2A, x3B = x2A;
    if (stats) A.avg[GZ + n - 1] = x1A.x;
    for (int i0 = n - 2; i0 >= 0; i0 -= POIS_PB) {
#pragma unroll
        for (int u = 0; u < POIS_PB; u++) {
            const int i = i0 - u;
            if (i >= 0) {
                const double2 svA = lsA[u], svB = lsB[u];
                const double p = lp[u], q = lq[u], r = lr[u];
                bload(i - POIS_PB, u);
                const double2 xA = hept_back(svA, p, q, r, x1A, x2A, x3A);
                const double2 xB = hept_back(svB, p, q, r, x1B, x2B, x3B);
                SA(GZ + i) = xA;
                SB(GZ + i) = xB;
                if (stats) A.avg[GZ + i] = xA.x;
                x3A = x2A; x2A = x1A; x1A = xA;
                x3B = x2B; x2B = x1B; x1B = xB;
            }
        }
    }
    if (!FILL) {
        if (GZ + n < n2 - GZ) {   // w: the top wall face
            SA(GZ + n) = make_double2(0.0, 0.0);
            SB(GZ + n) = make_double2(0.0, 0.0);
        }
        if (stats) average_walls<4>(A, n2);
        return;
    }
    // wall rows of the solution: bottom rows 0..2 are the last three results,
    // top rows n-1..n-3 are read back
    auto fill = [&](auto S, double2 x1, double2 x2, double2 x3) {
        double2 bt[3] = {x1, x2, x3};
        if (n < 3)
            for (int i = 0; i < 3; i++) bt[i] = i < n ? S(GZ + i) : make_double2(0.0, 0.0);
        double2 tp[3];
        for (int i = 0; i < 3; i++) tp[i] = n - 1 - i >= 0 ? S(GZ + n - 1 - i) : make_double2(0.0, 0.0);
        double g1, g2, g3, h1, h2, h3;
        fill_bot<4>(A.bot[var], bt[0].x, bt[1].x, bt[2].x, g1, g2, g3);
        fill_bot<4>(A.bot[var], bt[0].y, bt[1].y, bt[2].y, h1, h2, h3);
        S(GZ - 1) = make_double2(g1, h1);
        S(GZ - 2) = make_double2(g2, h2);
        S(GZ - 3) = make_double2(g3, h3);
        fill_top<4>(A.top, tp[0].x, tp[1].x, tp[2].x, g1, g2, g3);
        fill_top<4>(A.top, tp[0].y, tp[1].y, tp[2].y, h1, h2, h3);
        S(n2 - GZ) = make_double2(g1, h1);
        S(n2 - GZ + 1) = make_double2(g2, h2);
        S(n2 - GZ + 2) = make_double2(g3, h3);
    };
    fill(SA, x1A, x2A, x3A);
    fill(SB, x1B, x2B, x3B);
}

template <int ORDER>
__global__ void __launch_bounds__(POIS_THREADS_MAX, 4) k_poisson(Geo G, PoissonArgs A)
{
    band_column<ORDER, true>(G, A, blockIdx);
}

template <int ORDER>
__global__ void __launch_bounds__(POIS_THREADS_MAX, 4) k_poisson_batch(const BatchRec<PoissonArgs>* r, int n)
{
    uint3 b;
    const BatchRec<PoissonArgs>& R = batch_locate(r, n, b);
    band_column<ORDER, true>(R.G, R.A, b);
}

template <int ORDER>
__global__ void __launch_bounds__(POIS_THREADS_MAX, 4) k_helmholtz_spectral(Geo G, PoissonArgs A)
{
    band_column<ORDER, false>(G, A, blockIdx);
}

// ------------------------------------------------------------ projection


template <int ORDER>
__device__ __forceinline__ void k_project_body(const Geo& G, const ProjArgs& A, uint3 bid)
{
    const int j = bid.x * blockDim.x + threadIdx.x;
    const int i = bid.y * blockDim.y + threadIdx.y;
    const int k = bid.z;
    if (j >= G.ny || i >= G.nx) return;
    const int nx = G.nx, ny = G.ny, n2 = G.n2;
    auto I = [&](int kk, int ii, int jj) {
        return ((long long) kk * nx + wrapp(ii, nx)) * ny + wrapp(jj, ny);
    };
    const long long ijk = I(k, i, j);
    const double* __restrict__ p = A.p;
    const double dt = A.dt;
    const bool inner = k >= GZ && k < n2 - GZ;
    double u = A.u[ijk];
    if (A.mu) u = u + A.gu[k] * (*A.mu);      // chanfast.c:516-519
    if (inner) {
        double up1h;
        if (ORDER == 2) up1h = __ldg(p + I(k, i + 1, j)) - __ldg(p + ijk);
        else up1h = A1 * (__ldg(p + I(k, i + 1, j)) - __ldg(p + ijk)) + A2 * (__ldg(p + I(k, i + 2, j)) - __ldg(p + I(k, i - 1, j)));
        u = u - up1h * A.dtdx;
        double vp1h;
        if (ORDER == 2) vp1h = __ldg(p + I(k, i, j + 1)) - __ldg(p + ijk);
        else vp1h = A1 * (__ldg(p + I(k, i, j + 1)) - __ldg(p + ijk)) + A2 * (__ldg(p + I(k, i, j + 2)) - __ldg(p + I(k, i, j - 1)));
        A.v[ijk] = A.v[ijk] - vp1h * A.dtdy;
    }
    A.u[ijk] = u;
    if (k >= GZ - 1 && k < n2 - GZ) {
        double wp1h;
        if (ORDER == 2) wp1h = __ldg(p + I(k + 1, i, j)) - __ldg(p + ijk);
        else wp1h = A1 * (__ldg(p + I(k + 1, i, j)) - __ldg(p + ijk)) + A2 * (__ldg(p + I(k + 2, i, j)) - __ldg(p + I(k - 1, i, j)));
        A.w[ijk] = A.w[ijk] - wp1h * (dt * G.idzp1h[k]);
    }
    if (A.mc) A.c[ijk] = A.c[ijk] + A.gc[k] * (*A.mc);   // chanfast.c:603-606
}

template <int ORDER>
__global__ void __launch_bounds__(PROJ_THREADS_MAX) k_project(Geo G, ProjArgs A)
{
    k_project_body<ORDER>(G, A, blockIdx);
}

template <int ORDER>
__global__ void __launch_bounds__(PROJ_THREADS_MAX) k_project_batch(const BatchRec<ProjArgs>* r, int n)
{
    uint3 b;
    const BatchRec<ProjArgs>& R = batch_locate(r, n, b);
    k_project_body<ORDER>(R.G, R.A, b);
}

// ------------------------------------------------- power-of-two fast path
// N = 64, 128, 256, 512.  Each thread holds 8 elements of one line, at
// positions t + q*T (T = N/8, q = 0..7), in registers.  One leading radix-2
// or radix-4 stage when log2(N) is not a multiple of 3, then radix-8 stages.
// The leading stage reads the natural slots and the last radix-8 stage
// (Ns = T) leaves output position t + r*T in slot r, so global loads and
// stores are in natural order and coalesced.  Between stages the values go
// through shared memory padded by one complex per 8 (no bank conflicts).

__device__ __forceinline__ int pad8(int p) { return p + (p >> 3); }

template <int R>
__device__ __forceinline__ void bfly(double2* w, int s, double c8)
{
    if (R == 2) {
        double2 a = w[0], b = w[1];
        w[0] = cadd(a, b);
        w[1] = csub(a, b);
    } else if (R == 4) {
        double2 t0 = cadd(w[0], w[2]), t1 = csub(w[0], w[2]);
        double2 t2 = cadd(w[1], w[3]), t3 = cmul_si(csub(w[1], w[3]), s);
        w[0] = cadd(t0, t2);
        w[2] = csub(t0, t2);
        w[1] = cadd(t1, t3);
        w[3] = csub(t1, t3);
    } else {
        double2 e[4] = {w[0], w[2], w[4], w[6]}, o[4] = {w[1], w[3], w[5], w[7]};
        bfly<4>(e, s, c8);
        bfly<4>(o, s, c8);
        double2 o1 = make_double2(c8 * (o[1].x - s * o[1].y), c8 * (o[1].y + s * o[1].x));
        double2 o2 = cmul_si(o[2], s);
        double2 o3 = make_double2(c8 * (-o[3].x - s * o[3].y), c8 * (-o[3].y + s * o[3].x));
        w[0] = cadd(e[0], o[0]); w[4] = csub(e[0], o[0]);
        w[1] = cadd(e[1], o1);   w[5] = csub(e[1], o1);
        w[2] = cadd(e[2], o2);   w[6] = csub(e[2], o2);
        w[3] = cadd(e[3], o3);   w[7] = csub(e[3], o3);
    }
}

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

// Block-wide barrier of the transforms; FftBar256 is the named barrier of
// the first 256 threads (the transform threads of a larger block).
struct CtaBar {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct FftBar256 {
    __device__ __forceinline__ void operator()() const { asm volatile("bar.sync 1, 256;\n" ::: "memory"); }
};

__host__ __device__ constexpr int p2_lead_radix(int n)
{
    return ilog2c(n) % 3 == 0 ? 8 : (ilog2c(n) % 3 == 1 ? 2 : 4);
}

// Twiddles of the radix-8 stages of a power-of-two transform in the order a
// stage reads them: stage Ns (Ns = R0, 8 R0, .. < N) holds w^(r k N/(8 Ns))
// at [Ns - R0 + (r-1) Ns + k], r = 1..7, k < Ns (7 (N - R0) / 7 entries in
// all; at most N).  A warp then reads consecutive entries, free of bank
// conflicts.  tw: exp(-2 pi i m / N).
template <int N>
__device__ __forceinline__ void fill_stage_twiddles(double2* dst, const double2* __restrict__ tw, int tid, int nthreads)
{
    constexpr int R0 = p2_lead_radix(N);
    for (int e = tid; e < N - R0; e += nthreads) {
        int Ns = R0;
        while (e >= Ns - R0 + 7 * Ns) Ns *= 8;   // the stage holding entry e
        const int o = e - (Ns - R0), r = 1 + o / Ns, k = o - (r - 1) * Ns;
        dst[e] = __ldg(&tw[r * k * (N / (8 * Ns))]);
    }
}

// In-place transform of one line; every thread that `bar` synchronises must
// call it.  sl: this line's padded shared buffer.  TWM 0: tw is
// exp(-2 pi i m / (tws N)) in global memory, read with stride tws; TWM 1: tw
// is the stage table of fill_stage_twiddles<N> in shared memory.
template <int N, class Bar = CtaBar, int TWM = 0>
__device__ void fft_p2_line(double2 (&v)[8], int t, double2* sl, const double2* __restrict__ tw, int sign,
                            double c8, int tws = 1, Bar bar = Bar())
{
    constexpr int T = N / 8;
    constexpr int R0 = p2_lead_radix(N);
    {   // leading stage, Ns = 1: no twiddles; output position j*R0 + r
        constexpr int NB = 8 / R0;
#pragma unroll
        for (int m = 0; m < NB; m++) {
            double2 w[R0];
#pragma unroll
            for (int r = 0; r < R0; r++) w[r] = v[m + r * NB];
            bfly<R0>(w, sign, c8);
            const int j = t + m * T;
#pragma unroll
            for (int r = 0; r < R0; r++) sl[pad8(j * R0 + r)] = w[r];
        }
    }
    bar();
#pragma unroll
    for (int Ns = R0; Ns < N; Ns *= 8) {
        double2 w[8];
#pragma unroll
        for (int r = 0; r < 8; r++) w[r] = sl[pad8(t + r * T)];
        bar();
        const int k = t % Ns;
        const int step = N / (Ns * 8);
        if (k && TWM == 1) {
#pragma unroll
            for (int r = 1; r < 8; r++) {
                double2 c = tw[Ns - R0 + (r - 1) * Ns + k];
                if (sign > 0) c.y = -c.y;
                w[r] = cmul(w[r], c);
            }
        } else if (k) {
            // Twiddles w^r, r = 1..7, of w = exp(-+2 pi i k step / N): three
            // from the table (w, w^2, w^4), the rest as their products.
            // Seven table reads per stage made the transforms bound by the
            // load pipe, not by HBM; a product adds at most a few ulps.
            double2 c1 = __ldg(&tw[tws * k * step]), c2 = __ldg(&tw[tws * 2 * k * step]);
            double2 c4 = __ldg(&tw[tws * 4 * k * step]);
            if (sign > 0) { c1.y = -c1.y; c2.y = -c2.y; c4.y = -c4.y; }
            const double2 c3 = cmul(c1, c2);
            const double2 cw[8] = {c1, c1, c2, c3, c4, cmul(c1, c4), cmul(c2, c4), cmul(c3, c4)};
#pragma unroll
            for (int r = 1; r < 8; r++) w[r] = cmul(w[r], cw[r]);
        }
        bfly<8>(w, sign, c8);
        if (Ns * 8 == N) {
#pragma unroll
            for (int r = 0; r < 8; r++) v[r] = w[r];
        } else {
            const int base = (t / Ns) * Ns * 8 + k;
#pragma unroll
            for (int r = 0; r < 8; r++) sl[pad8(base + r * Ns)] = w[r];
            bar();
        }
    }
}

// 256 threads per block: 2048 / N lines of N / 8 threads (x transforms: the
// lines are consecutive j, so each load or store of a warp covers runs of
// consecutive j; y transforms: the lines are consecutive kx)
__host__ __device__ constexpr int p2_lines(int n) { return 2048 / n; }
__host__ __device__ constexpr int p2_pad(int n) { return n + n / 8; }
// Line stride of the x transforms, whose consecutive lanes are different
// lines: a quarter-warp (8 lanes of 16 bytes) spans 8 lines at one position
// (N <= 256; an odd stride in 16-byte units puts them in 8 distinct bank
// groups) or 4 lines at two consecutive positions (N = 512; stride = 2 mod 8).
__host__ __device__ constexpr int p2_stride_x(int n) { return p2_pad(n) + (p2_lines(n) >= 8 ? 1 : 2); }

// Divergence of the power-of-two path as its own streaming kernel
// (divergence{2,4}, pressure.c:40-117).  A block owns an 8 (i) x 32 (j)
// tile and climbs DV_KC planes.  Per plane, u with its x halo (rows i-2 ..
// i+8) and v with its y halo (columns j-2 .. j+33, an even width) are staged
// in shared memory by cp.async, double-buffered one plane ahead, so each
// value crosses L2 once; for even ny the copies are 16-byte pairs that
// bypass L1.  w is carried up the column in a register window (the next
// row loaded one plane ahead), and at the walls that window supplies the
// extrapolated w of pressure.c:80-95.  The x transform then reads the
// result as a real field.
constexpr int DV_I = 8, DV_J = 32, DV_KC = 16;

__device__ __forceinline__ void dv_cp8(double* dst, const double* src)
{
    unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void dv_cp16(double* dst, const double* src)   // L2 only
{
    unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

template <int ORDER>
__device__ __forceinline__ void k_div_body(const Geo& G, const DivArgs& A, uint3 bid)
{
    __shared__ __align__(16) double su[2][DV_I + 3][DV_J];   // u, rows i0-2 .. i0+8
    __shared__ __align__(16) double sv[2][DV_I][DV_J + 4];   // v, columns j0-2 .. j0+33
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * DV_J + tx;
    const int j0 = bid.x * DV_J, i0 = bid.y * DV_I;
    const int nx = G.nx, ny = G.ny, n2 = G.n2;
    const long long plane = G.plane;
    const int k0 = GZ + bid.z * DV_KC;
    const int k1 = min(k0 + DV_KC, n2 - GZ);
    const int i = i0 + ty, j = j0 + tx;
    const bool valid = i < nx && j < ny;
    // this thread's halo elements (even ny: one pair of u, one pair of v;
    // odd ny: at most two of u, two of v): their offsets within a plane,
    // the same for every plane, computed once.  For even ny a pair starts
    // at an even y index (j0 is even, the v halo starts 2 before), so it
    // never straddles the periodic wrap and its addresses are 16-byte aligned.
    constexpr int NU = (DV_I + 3) * DV_J, NV = DV_I * (DV_J + 4), NT = DV_I * DV_J;
    const bool pairs = (ny & 1) == 0;
    int uoff[2], voff[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int e = tid + q * NT;
        if (pairs) {   // pair e of u (e < NU/2) and of v (e < NV/2)
            const int r = e / (DV_J / 2), c = 2 * (e - r * (DV_J / 2));
            int ii = (i0 - 2 + r) % nx; if (ii < 0) ii += nx;
            uoff[q] = 2 * e < NU ? ii * ny + min(j0 + c, ny - 2) : 0;
            const int rv = e / ((DV_J + 4) / 2), cv = 2 * (e - rv * ((DV_J + 4) / 2));
            int jj = (j0 - 2 + cv) % ny; if (jj < 0) jj += ny;
            voff[q] = 2 * e < NV ? min(i0 + rv, nx - 1) * ny + jj : 0;
        } else {
            const int r = e / DV_J, c = e - r * DV_J;
            int ii = (i0 - 2 + r) % nx; if (ii < 0) ii += nx;
            uoff[q] = e < NU ? ii * ny + min(j0 + c, ny - 1) : 0;
            const int rv = e / (DV_J + 4), cv = e - rv * (DV_J + 4);
            int jj = (j0 - 2 + cv) % ny; if (jj < 0) jj += ny;
            voff[q] = e < NV ? min(i0 + rv, nx - 1) * ny + jj : 0;
        }
    }
    auto load = [&](int kk, int buf) {
        const double* uk = A.u + kk * plane;
        const double* vk = A.v + kk * plane;
        if (pairs) {
            if (2 * tid < NU) dv_cp16(&su[buf][0][0] + 2 * tid, uk + uoff[0]);
            if (2 * tid < NV) dv_cp16(&sv[buf][0][0] + 2 * tid, vk + voff[0]);
        } else {
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int e = tid + q * NT;
                if (e < NU) dv_cp8(&su[buf][0][0] + e, uk + uoff[q]);
                if (e < NV) dv_cp8(&sv[buf][0][0] + e, vk + voff[q]);
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    const bool corr = A.mu != nullptr;
    const double mu = corr ? *A.mu : 0.0;
    const int kb = GZ - 1, kt = n2 - GZ - 1;
    const long long c = valid ? (long long) i * ny + j : 0;
    const double* __restrict__ wp = A.w + c;
    load(k0, 0);
    // w at rows k-2 .. k (order 4) / k-1, k (order 2) for the first row
    double w0 = ORDER == 4 ? __ldg(wp + (k0 - 2) * plane) : 0.0;
    double w1 = __ldg(wp + (k0 - 1) * plane);
    double w2 = __ldg(wp + k0 * plane);
    double w3n = __ldg(wp + (k0 + 1) * plane);   // row k+1, loaded one plane ahead
    for (int k = k0; k < k1; k++) {
        const int buf = (k - k0) & 1;
        if (k + 1 < k1) load(k + 1, buf ^ 1);
        else asm volatile("cp.async.commit_group;\n" ::: "memory");
        const double w3 = w3n;   // row k+1 (a ghost row at the top: unused there)
        if (k + 1 < k1) w3n = __ldg(wp + (k + 2) * plane);   // rows up to k1 <= n2 - GZ, as before
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncthreads();
        const double uc = corr ? A.gu[k] * mu : 0.0;   // chanfast.c:516-519
        auto U = [&](int d) { return corr ? su[buf][ty + 2 + d][tx] + uc : su[buf][ty + 2 + d][tx]; };
        auto V = [&](int d) { return sv[buf][ty][tx + 2 + d]; };
        const double idzk = G.idz[k];
        double d;
        if (ORDER == 2) {
            d = (U(0) - U(-1)) * G.idx + (V(0) - V(-1)) * G.idy + (w2 - w1) * idzk;
        } else {
            const double wkm2 = (k - 2 == kb - 1) ? 2.0 * w1 - w2 : w0;   // pressure.c:80-87
            const double wkp1 = (k + 1 == kt + 1) ? 2.0 * w2 - w1 : w3;   // pressure.c:88-95
            d = (A1 * (U(0) - U(-1)) + A2 * (U(1) - U(-2))) * G.idx
              + (A1 * (V(0) - V(-1)) + A2 * (V(1) - V(-2))) * G.idy
              + (A1 * (w2 - w1) + A2 * (wkp1 - wkm2)) * idzk;
        }
        if (valid) A.dv[k * plane + c] = d;
        w0 = w1; w1 = w2; w2 = w3;
        __syncthreads();   // this buffer is refilled two planes on
    }
}

template <int ORDER>
__global__ void __launch_bounds__(DV_I * DV_J) k_div(Geo G, DivArgs A)
{
    k_div_body<ORDER>(G, A, blockIdx);
}

template <int ORDER>
__global__ void __launch_bounds__(DV_I * DV_J) k_div_batch(const BatchRec<DivArgs>* r, int n)
{
    uint3 b;
    const BatchRec<DivArgs>& R = batch_locate(r, n, b);
    k_div_body<ORDER>(R.G, R.A, b);
}

// Real-to-complex x transform (fftx_d2c, pressure.c:122-160, scaled by 1/N)
// as a complex transform of half length: z[m] = x[2m] + i x[2m+1], Z = FFT(z),
// X[k] = E[k] + exp(-2 pi i k/N) O[k] with E, O the transforms of the even and
// odd samples, E = (Z[k] + conj Z[M-k]) / 2, O = (Z[k] - conj Z[M-k]) / 2i.
// A line is M = N/2 points, 8 per thread; 256 / (M/8) lines of consecutive j
// per block.
template <int N>
__device__ __forceinline__ void k_fftx_r2c_p2_body(const Geo& G, const R2cArgs& A, uint3 bid)
{
    extern __shared__ double2 sbuf[];
    constexpr int M = N / 2, T = M / 8, L = p2_lines(M);
    const int l = threadIdx.x % L, t = threadIdx.x / L;
    const int k = A.kfirst + bid.y;
    const int j = bid.x * L + l;
    const bool valid = j < G.ny;
    const int ny = G.ny;
    const double* row = A.src + bid.z * A.src_fstride + (long long) k * G.nx * ny + (valid ? j : 0);
    double2 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int m = t + q * T;
        v[q] = make_double2(__ldg(row + (long long) (2 * m) * ny), __ldg(row + (long long) (2 * m + 1) * ny));
    }
    double2* sl = sbuf + l * p2_stride_x(M);
    fft_p2_line<M>(v, t, sl, A.px.tw, -1, A.c8, 2);
    // Z in natural order through this line's buffer (the transform's last
    // reads of it are behind its final barrier)
#pragma unroll
    for (int r = 0; r < 8; r++) sl[pad8(t + r * T)] = v[r];
    __syncthreads();
    if (!valid) return;
    const double scale = 1.0 / (double) N;
    double2* out = A.spec + bid.z * A.spec_fstride + (long long) k * G.nkx * ny + j;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int kx = t + q * T;
        const double2 a = sl[pad8(kx)];
        const double2 zb = sl[pad8((M - kx) & (M - 1))];
        const double er = 0.5 * (a.x + zb.x), ei = 0.5 * (a.y - zb.y);   // E
        const double orr = 0.5 * (a.y + zb.y), oi = -0.5 * (a.x - zb.x); // O
        const double2 w = __ldg(&A.px.tw[kx]);                            // exp(-2 pi i kx/N)
        out[(long long) kx * ny] = make_double2((er + (w.x * orr - w.y * oi)) * scale,
                                                (ei + (w.x * oi + w.y * orr)) * scale);
    }
    if (t == 0) {   // Nyquist: X[N/2] = E[0] - O[0], real
        const double2 z0 = sl[pad8(0)];
        out[(long long) M * ny] = make_double2((z0.x - z0.y) * scale, 0.0);
    }
}

// Four resident blocks per SM (64 registers instead of 80, no spills):
// 32 warps instead of 24 keep more lines' loads in flight; at 512 x 512 x
// 384 the x transform with the divergence takes 0.943 instead of 0.960 ms.
// The batched variant keeps 80 registers: capped, it spills at 64 and 128.
template <int N>
__global__ void __launch_bounds__(256, 4) k_fftx_r2c_p2(Geo G, R2cArgs A)
{
    k_fftx_r2c_p2_body<N>(G, A, blockIdx);
}

template <int N>
__global__ void __launch_bounds__(256) k_fftx_r2c_p2_batch(const BatchRec<R2cArgs>* r, int n)
{
    uint3 b;
    const BatchRec<R2cArgs>& R = batch_locate(r, n, b);
    k_fftx_r2c_p2_body<N>(R.G, R.A, b);
}

template <int N>
__device__ __forceinline__ void k_ffty_p2_body(const Geo& G, const FftyArgs& A, uint3 bid)
{
    extern __shared__ double2 sbuf[];
    constexpr int T = N / 8, L = p2_lines(N);
    const int t = threadIdx.x % T, l = threadIdx.x / T;
    const int k = A.kfirst + bid.y;
    const int kx = bid.x * L + l;
    const int nkx = G.nkx;
    const bool valid = kx < nkx;
    double2* base = A.spec + bid.z * A.fstride + ((long long) k * nkx + (valid ? kx : 0)) * N;
    double2 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = valid ? base[t + q * T] : make_double2(0.0, 0.0);
    fft_p2_line<N>(v, t, sbuf + l * p2_pad(N), A.py.tw, A.sign, A.c8);
    if (!valid) return;
    const double scale = 1.0 / (double) N;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        double2 x = v[q];
        if (A.sign < 0) { x.x *= scale; x.y *= scale; }
        base[t + q * T] = x;
    }
}

template <int N>
__global__ void __launch_bounds__(256, 4) k_ffty_p2(Geo G, FftyArgs A)
{
    k_ffty_p2_body<N>(G, A, blockIdx);
}

template <int N>
__global__ void __launch_bounds__(256, 4) k_ffty_p2_batch(const BatchRec<FftyArgs>* r, int n)
{
    uint3 b;
    const BatchRec<FftyArgs>& R = batch_locate(r, n, b);
    k_ffty_p2_body<N>(R.G, R.A, b);
}

// ------------------------------------ y transforms fused with the Poisson solve

// Bulk copies global -> shared completing on an mbarrier (no multicast), and
// the barrier's bounded wait.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned) __cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* b)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(b)) : "memory");
}
// generic-proxy accesses of shared memory before a bulk copy into it
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Wait for phase `parity` of barrier b to complete; false after about one
// second without completion (global timer), or after 2^26 polls should the
// timer not advance.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* b, unsigned parity)
{
    const unsigned a = smem_u32(b);
    const unsigned long long t0 = global_ns();
    for (unsigned it = 0; it < (1u << 26); it++) {
        unsigned ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok) : "r"(a), "r"(parity) : "memory");
        if (ok) return true;
        if (global_ns() - t0 > 1000000000ull) return false;
    }
    return false;
}

// k_poisson_fft: one block per kx does the forward y transform of that kx's
// interior rows (ffty_i2o, fft.c:186-202, with its 1/ny), the Poisson band
// solve of its (ky, ny - ky) column pairs with the wall ghost rows filled
// (pressure_poisson{2,4}, pressure.c:293-443), and the inverse y transform of
// all n2 rows (ffty_o2i), for ny = 512.  The spectrum makes one round trip
// through HBM instead of three; the transforms and the elimination are those
// of k_ffty_p2 and band_column.
//
// Two roles, each in its own warps.  Transform warps (the first 256
// threads: L = 4 lines of 64 threads) and solver warps (one thread per
// column pair, 257 of 288 threads) hand row groups of L rows to each other
// through two shared buffers (named barriers FULL / EMPTY per buffer), so
// that one role works on a group while the other works on the next.
//   Forward: rows arrive by bulk copies two groups ahead; the transform
//   warps transform a group, scale it by 1/ny and stage the group's band
//   rows; the solvers advance their pairs' elimination through it, storing
//   the forward-substituted values in place and the multipliers in scratch
//   (rows of ny/2 + 2 values, 16-byte aligned).
//   Back: groups top down; the solvers back-substitute a group (its inputs
//   as bulk copies two groups ahead at order 4, two rows ahead through
//   registers at order 2) and the six wall ghost rows, the transform warps
//   transform and store each.
constexpr int PF_FT = 256;                  // transform threads
template <int N>
__host__ __device__ constexpr int pfft_solvers() { return (N / 2 + 1 + 31) / 32 * 32; }
template <int N>
__host__ __device__ constexpr int pfft_threads() { return PF_FT + pfft_solvers<N>(); }
// back-sweep inputs per slot (order 4): forward-substituted rows [L][ny]
// (complex) and p, q, r rows [3][L][ny/2 + 2]
template <int ORDER, int N>
__host__ __device__ constexpr bool pfft_back_ring() { return ORDER == 4; }
template <int N>
__host__ __device__ constexpr int pfft_back_slot() { return 2 * 2048 + 3 * (2048 / N) * (N / 2 + 2); }   // doubles
// layout: copy ring (forward rows [2][L][ny], or back-sweep inputs
// [2][slot]) | transform lines [L][ny + ny/8] | hand-over buffers [2][L][ny] |
// band rows [2][L][10] | twiddles [ny] | 4 mbarriers
template <int ORDER, int N>
__host__ __device__ constexpr size_t pfft_ring_bytes()
{
    return pfft_back_ring<ORDER, N>() && 2 * pfft_back_slot<N>() * sizeof(double) > 2 * 2048 * sizeof(double2)
               ? 2 * pfft_back_slot<N>() * sizeof(double)
               : 2 * 2048 * sizeof(double2);
}
template <int ORDER, int N>
constexpr size_t pfft_smem_bytes()
{
    return pfft_ring_bytes<ORDER, N>() + 2304 * sizeof(double2) + 2 * 2048 * sizeof(double2)
         + 2 * (2048 / N) * 10 * sizeof(double) + N * sizeof(double2) + 4 * sizeof(unsigned long long);
}

// named barriers: 1 transform warps (fft_p2_line), 2/3 FULL, 4/5 EMPTY of
// buffer 0/1, 6 solver warps
__device__ __forceinline__ void nbar_sync(int id, int n) { asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void nbar_arrive(int id, int n) { asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(n) : "memory"); }
// barrier id over n threads that also ORs p across them
__device__ __forceinline__ bool nbar_or(int id, int n, bool p)
{
    int r;
    asm volatile("{\n .reg .pred a, b;\n setp.ne.b32 a, %1, 0;\n bar.red.or.pred b, %2, %3, a;\n selp.s32 %0, 1, 0, b;\n}\n"
                 : "=r"(r) : "r"((int) p), "r"(id), "r"(n) : "memory");
    return r != 0;
}

// FILL: the Poisson solve, with the wall ghost rows of the solution; else a
// spectral Helmholtz solve of the fully implicit scheme (band_column without
// FILL): no ghost rows, the xy-average profile from the (0, 0) column when
// A.avg is set, w's top wall face zeroed.
template <int ORDER, int N, bool FILL = true>
__device__ __forceinline__ void poisson_fft_body(const Geo& G, const PoissonFftArgs& F, uint3 bid)
{
    static_assert(N == 256 || N == 512, "groups of 2048 points: 8 or 4 rows");
    constexpr int T = N / 8, L = p2_lines(N), NP = N / 2 + 1, PAD = p2_pad(N);
    constexpr int SW = pfft_solvers<N>(), BT = PF_FT + SW;
    constexpr bool BRING = pfft_back_ring<ORDER, N>();
    constexpr int NPS = NP + 1;                        // pair stride of the multiplier rows (even)
    constexpr int BSLOT = pfft_back_slot<N>();
    constexpr int B_FULL = 2, B_EMPTY = 4, B_SOLVE = 6;
    extern __shared__ double2 pfft_sm[];
    double2* ring = pfft_sm;                                                  // forward copies
    double* bring = reinterpret_cast<double*>(pfft_sm);                       // back-sweep copies (BRING)
    double2* sl = reinterpret_cast<double2*>(reinterpret_cast<char*>(pfft_sm) + pfft_ring_bytes<ORDER, N>());
    double2* xb = sl + L * PAD;                       // [2][L][N] hand-over buffers
    double* cst = reinterpret_cast<double*>(xb + 2 * L * N);   // [2][L][10] band rows of a group
    double2* tws = reinterpret_cast<double2*>(cst + 2 * L * 10);   // stage twiddles (fill_stage_twiddles)
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(tws + N);   // [2] forward, [2] back
    const PoissonArgs& A = F.P;
    const int tid = threadIdx.x;
    const int kx = bid.x;
    const int nkx = G.nkx, n2 = G.n2, n = A.nrows;
    const bool fthr = tid < PF_FT;
    const int t = tid % T, l = tid / T;               // transform lane and line (transform warps)
    const int ky0 = tid - PF_FT;
    const bool solver = !fthr && ky0 < NP;
    const int ky = solver ? ky0 : 0, kyb = (N - ky) & (N - 1);
    const long long ncol = G.splane;
    const long long npair = (long long) nkx * NPS, pair = (long long) kx * NPS + ky;
    double2* sp = A.spec;
    const long long colA = (long long) kx * N + ky, colB = (long long) kx * N + kyb;
    auto SA = [&](int k) -> double2& { return sp[(long long) k * ncol + colA]; };
    auto SB = [&](int k) -> double2& { return sp[(long long) k * ncol + colB]; };
    auto at = [&](double* base, int k) -> double& { return base[(long long) k * npair + pair]; };
    auto row = [&](int k) { return sp + ((long long) k * nkx + kx) * N; };   // spectrum row (k, kx)
    const int var = (kx == 0 && ky == 0) ? 1 : 0;   // pressure.c:331-338
    const PairRows rows{A, A.lamx[kx], A.lamy[ky], var, n};
    const int ngrp = (n + L - 1) / L;
    double* const Pp = A.scratch;                            // order 4: p, q, r; order 2: gamma
    double* const Qp = A.scratch + (long long) n2 * npair;
    double* const Rp = A.scratch + 2 * (long long) n2 * npair;

    auto issue = [&](int g) {   // forward group g's rows into copy slot g & 1
        const int slot = g & 1, r0 = g * L, nr = min(L, n - r0);
        mbar_expect_tx(&bar[slot], (unsigned) (nr * N * sizeof(double2)));
        for (int q = 0; q < nr; q++)
            bulk_g2s(ring + (slot * L + q) * N, row(GZ + r0 + q), N * sizeof(double2), &bar[slot]);
    };
    auto bissue = [&](int j) {   // back group j (forward group ngrp - 1 - j): inputs into slot j & 1
        const int g = ngrp - 1 - j, slot = j & 1, lo = g * L, nr = min(L, n - lo);
        double* b = bring + slot * BSLOT;
        mbar_expect_tx(&bar[2 + slot], (unsigned) (nr * (N * sizeof(double2) + 3 * NPS * sizeof(double))));
        for (int q = 0; q < nr; q++) {
            const long long k = GZ + lo + q;
            bulk_g2s(b + 2 * q * N, row((int) k), N * sizeof(double2), &bar[2 + slot]);
            bulk_g2s(b + 2 * L * N + q * NPS, Pp + (k * nkx + kx) * NPS, NPS * sizeof(double), &bar[2 + slot]);
            bulk_g2s(b + 2 * L * N + (L + q) * NPS, Qp + (k * nkx + kx) * NPS, NPS * sizeof(double), &bar[2 + slot]);
            bulk_g2s(b + 2 * L * N + (2 * L + q) * NPS, Rp + (k * nkx + kx) * NPS, NPS * sizeof(double),
                     &bar[2 + slot]);
        }
    };

    if (tid == 0) {
        for (int q = 0; q < 4; q++) mbar_init(&bar[q], 1);
        mbar_fence_init();
    }
    fill_stage_twiddles<N>(tws, F.twy, tid, BT);
    __syncthreads();
    if (tid == 0 && !F.stall) {
        issue(0);
        if (ngrp > 1) issue(1);
    }

    const double2 z2 = make_double2(0.0, 0.0);
    if (fthr) {
        // ================= transform warps =================
        const double scale = 1.0 / (double) N;
        const bool cthr = tid < 10 * L;
        const int crow = tid / 10, cfld = tid - 10 * (tid / 10);
        bool failed = false;
        for (int g = 0; g < ngrp; g++) {
            const int b = g & 1;
            const int ci = g * L + crow;   // this thread's band-row value of the group
            const double cval = cthr && ci < n ? rows.table(cfld, GZ + ci) : 0.0;
            if (!failed) {
                const bool bad = !mbar_wait_bounded(&bar[b], (g >> 1) & 1);
                if (nbar_or(1, PF_FT, bad)) {
                    failed = true;   // carry on with the hand-overs, without data
                    if (tid == 0) {
                        *F.fault = 1.0;
                        if (!F.stall) {   // the copies of groups g and g + 1 are in flight
                            (void) mbar_wait_bounded(&bar[b], (g >> 1) & 1);
                            if (g + 1 < ngrp) (void) mbar_wait_bounded(&bar[(g + 1) & 1], ((g + 1) >> 1) & 1);
                        }
                    }
                }
            }
            double2 v[8];
            const double2* src = ring + (b * L + l) * N;
#pragma unroll
            for (int q = 0; q < 8; q++) v[q] = src[t + q * T];
            fft_p2_line<N, FftBar256, 1>(v, t, sl + l * PAD, tws, -1, F.c8);
            if (tid == 0 && !failed && g + 2 < ngrp) {   // every transform thread has read slot b
                fence_proxy_async_smem();
                issue(g + 2);
            }
            if (g >= 2) nbar_sync(B_EMPTY + b, BT);
            double2* dst = xb + (b * L + l) * N;
#pragma unroll
            for (int q = 0; q < 8; q++) dst[t + q * T] = make_double2(v[q].x * scale, v[q].y * scale);
            if (cthr) cst[(b * L + crow) * 10 + cfld] = cval;
            nbar_arrive(B_FULL + b, BT);
        }
        __syncthreads();   // forward done (matches the solvers' barrier)
        // back: the groups the solvers hand over, in their order
        const int gt = max(n - 3, 0) / L;
        const int S = FILL ? ngrp + 2 : ngrp;
        for (int s = 0; s < S; s++) {
            const int b = s & 1;
            int target;   // spectrum row of line l, or -1
            if (!FILL) {
                const int g = ngrp - 1 - s;
                target = g * L + l < n ? GZ + g * L + l : -1;
            } else if (s <= ngrp - 1 - gt || (s > ngrp - gt && s <= ngrp)) {
                const int g = s <= ngrp - 1 - gt ? ngrp - 1 - s : ngrp - s;
                target = g * L + l < n ? GZ + g * L + l : -1;
            } else if (s == ngrp - gt) {
                target = l < 3 ? n2 - GZ + l : -1;   // top wall ghost rows
            } else {
                target = l < 3 ? l : -1;             // bottom wall ghost rows
            }
            nbar_sync(B_FULL + b, BT);
            double2 v[8];
            const double2* src = xb + (b * L + l) * N;
#pragma unroll
            for (int q = 0; q < 8; q++) v[q] = src[t + q * T];
            if (s + 2 < S) nbar_arrive(B_EMPTY + b, BT);
            fft_p2_line<N, FftBar256, 1>(v, t, sl + l * PAD, tws, +1, F.c8);
            if (target >= 0) {
                double2* dst = row(target);
#pragma unroll
                for (int q = 0; q < 8; q++) dst[t + q * T] = v[q];
            }
        }
        if (!FILL && GZ + n < n2 - GZ && l == 0) {   // w: the top wall face
            double2* dst = row(GZ + n);
#pragma unroll
            for (int q = 0; q < 8; q++) dst[t + q * T] = make_double2(0.0, 0.0);
        }
        return;
    }

    // ================= solver warps =================
    HeptSweep H;
    double ibet = 0.0, cprev = 0.0;                          // order 2 (tridag.c:4-26)
    double2 uA = z2, uB = z2;
    for (int g = 0; g < ngrp; g++) {
        const int b = g & 1;
        nbar_sync(B_FULL + b, BT);
        if (solver) {
            for (int q = 0; q < L; q++) {
                const int i = g * L + q;
                if (i >= n) break;
                const int k = GZ + i;
                const double2 rA = xb[(b * L + q) * N + ky], rB = xb[(b * L + q) * N + kyb];
                const double* st = cst + (b * L + q) * 10;
                double cf[7];
                rows.coef_from(i, st, cf);
                const double dv = st[9];
                if (ORDER == 2) {
                    if (i == 0) {
                        ibet = 1.0 / cf[3];
                        uA = make_double2(rA.x * dv * ibet, rA.y * dv * ibet);
                        uB = make_double2(rB.x * dv * ibet, rB.y * dv * ibet);
                    } else {
                        const double gm = cprev * ibet;
                        ibet = 1.0 / (cf[3] - cf[0] * gm);
                        at(Pp, k) = gm;
                        uA = make_double2((rA.x * dv - cf[0] * uA.x) * ibet, (rA.y * dv - cf[0] * uA.y) * ibet);
                        uB = make_double2((rB.x * dv - cf[0] * uB.x) * ibet, (rB.y * dv - cf[0] * uB.y) * ibet);
                    }
                    cprev = cf[2];
                    SA(k) = uA;
                    SB(k) = uB;
                } else {
                    double p, qq, r;
                    double2 svA, svB;
                    H.step(cf, make_double2(rA.x * dv, rA.y * dv), make_double2(rB.x * dv, rB.y * dv), p, qq, r,
                           svA, svB);
                    at(Pp, k) = p; at(Qp, k) = qq; at(Rp, k) = r;
                    SA(k) = svA;
                    SB(k) = svB;
                }
            }
        }
        if (g + 2 < ngrp) nbar_arrive(B_EMPTY + b, BT);
    }
    // the forward stores before the bulk copies that read them back
    asm volatile("fence.proxy.async;\n" ::: "memory");
    __syncthreads();
    if (BRING && tid == PF_FT) {   // into the space the transform warps last read as the forward ring
        fence_proxy_async_smem();
        bissue(0);
        if (ngrp > 1) bissue(1);
    }

    // ---- back: groups top down, then the wall ghost rows
    double2 lsA[2], lsB[2];
    double lp[2];
    auto bload = [&](int i) {   // order 2: row i's forward values and gamma, in slot i & 1
        if (BRING || i < 0 || !solver) return;
        const int k = GZ + i;
        const double2 a = SA(k), c = SB(k);
        const double p = i + 1 < n ? at(Pp, k + 1) : 0.0;
        if (i & 1) { lsA[1] = a; lsB[1] = c; lp[1] = p; }
        else { lsA[0] = a; lsB[0] = c; lp[0] = p; }
    };
    bload(n - 1);
    bload(n - 2);
    double2 x1A = z2, x2A = z2, x3A = z2, x1B = z2, x2B = z2, x3B = z2;
    double2 tpA[3] = {z2, z2, z2}, tpB[3] = {z2, z2, z2};   // rows n-1, n-2, n-3
    bool failed = false;
    int s = 0;   // hand-over count
    const bool stats = !FILL && A.avg != nullptr && kx == 0 && ky0 == 0;   // the (0, 0) column
    // back substitution of row i into line i - lo of hand-over buffer `out`
    auto back_row = [&](int i, int lo, double2 svA, double2 svB, double p, double q, double r, double2* out,
                        auto top_tag) {
        constexpr bool TOP = decltype(top_tag)::value;
        double2 xA, xB;
        if (TOP && i == n - 1) {
            xA = svA;
            xB = svB;
        } else if (ORDER == 2) {
            xA = make_double2(svA.x - p * x1A.x, svA.y - p * x1A.y);
            xB = make_double2(svB.x - p * x1B.x, svB.y - p * x1B.y);
        } else {
            xA = hept_back(svA, p, q, r, x1A, x2A, x3A);
            xB = hept_back(svB, p, q, r, x1B, x2B, x3B);
        }
        x3A = x2A; x2A = x1A; x1A = xA;
        x3B = x2B; x2B = x1B; x1B = xB;
        if (TOP) {
            if (i == n - 1) { tpA[0] = xA; tpB[0] = xB; }
            if (i == n - 2) { tpA[1] = xA; tpB[1] = xB; }
            if (i == n - 3) { tpA[2] = xA; tpB[2] = xB; }
        }
        out[(i - lo) * N + ky] = xA;
        out[(i - lo) * N + kyb] = xB;
        if (stats) A.avg[GZ + i] = xA.x;
    };
    auto back_group = [&](int g, auto top_tag) {
        const int b = s & 1;
        double2* out = xb + b * L * N;
        const int lo = g * L, hi = min(n, lo + L) - 1;
        if (s >= 2) nbar_sync(B_EMPTY + b, BT);
        if constexpr (BRING) {
            const int j = ngrp - 1 - g;   // back group j: copies in slot j & 1
            if (!failed) {
                const bool bad = !mbar_wait_bounded(&bar[2 + (j & 1)], (j >> 1) & 1);
                if (nbar_or(B_SOLVE, SW, bad)) {
                    failed = true;   // carry on with the hand-overs, without data
                    if (tid == PF_FT) {
                        *F.fault = 1.0;
                        (void) mbar_wait_bounded(&bar[2 + (j & 1)], (j >> 1) & 1);
                        if (j + 1 < ngrp) (void) mbar_wait_bounded(&bar[2 + ((j + 1) & 1)], ((j + 1) >> 1) & 1);
                    }
                }
            }
            if (solver) {
                const double* bs = bring + (j & 1) * BSLOT;
                const double2* bv = reinterpret_cast<const double2*>(bs);
                const double* bp = bs + 2 * L * N;
                for (int i = hi; i >= lo; i--) {
                    const int q = i - lo;
                    back_row(i, lo, bv[q * N + ky], bv[q * N + kyb], bp[q * NPS + ky], bp[(L + q) * NPS + ky],
                             bp[(2 * L + q) * NPS + ky], out, top_tag);
                }
            }
            nbar_sync(B_SOLVE, SW);   // every solver has read back slot j & 1
            if (tid == PF_FT && !failed && j + 2 < ngrp) {
                fence_proxy_async_smem();
                bissue(j + 2);
            }
        } else if (solver) {
            for (int i1 = hi | 1; i1 >= lo; i1 -= 2) {
#pragma unroll
                for (int u = 1; u >= 0; u--) {
                    const int i = i1 - 1 + u;
                    if (i > hi || i < lo) continue;
                    const double2 svA = lsA[u], svB = lsB[u];
                    const double p = lp[u];
                    bload(i - 2);
                    back_row(i, lo, svA, svB, p, 0.0, 0.0, out, top_tag);
                }
            }
        }
        nbar_arrive(B_FULL + b, BT);
        s++;
    };
    // wall ghost rows (ghost_fill_{bot,top}{2,4}, pressure.c:516-531,
    // 728-769) as one hand-over: lines 0..2 hold gA/gB[0..2]
    auto ghost_group = [&](const double2* gA, const double2* gB) {
        const int b = s & 1;
        double2* out = xb + b * L * N;
        if (s >= 2) nbar_sync(B_EMPTY + b, BT);
        if (solver) {
#pragma unroll
            for (int q = 0; q < 3; q++) {
                out[q * N + ky] = gA[q];
                out[q * N + kyb] = gB[q];
            }
        }
        nbar_arrive(B_FULL + b, BT);
        s++;
    };
    // the groups holding rows n-1 .. max(n-3, 0), the top ghost rows
    // n2-3 .. n2-1 from rows n-1..n-3 (zero where n < 3), the other groups,
    // the bottom ghost rows 0..2 from rows 0..2
    const int gt = max(n - 3, 0) / L;
    for (int g = ngrp - 1; g >= gt; g--) back_group(g, std::true_type{});
    if constexpr (!FILL) {
        for (int g = gt - 1; g >= 0; g--) back_group(g, std::false_type{});
        if (stats) average_walls<ORDER>(A, n2);
        return;
    }
    {
        double2 gA[3], gB[3];
        double g1, g2, g3, h1, h2, h3;
        if (ORDER == 2) {
            fill_top<2>(A.top, tpA[0].x, 0.0, 0.0, g1, g2, g3);
            fill_top<2>(A.top, tpA[0].y, 0.0, 0.0, h1, g2, g3);
            gA[0] = make_double2(g1, h1); gA[1] = gA[2] = z2;
            fill_top<2>(A.top, tpB[0].x, 0.0, 0.0, g1, g2, g3);
            fill_top<2>(A.top, tpB[0].y, 0.0, 0.0, h1, g2, g3);
            gB[0] = make_double2(g1, h1); gB[1] = gB[2] = z2;
        } else {
            fill_top<4>(A.top, tpA[0].x, tpA[1].x, tpA[2].x, g1, g2, g3);
            fill_top<4>(A.top, tpA[0].y, tpA[1].y, tpA[2].y, h1, h2, h3);
            gA[0] = make_double2(g1, h1); gA[1] = make_double2(g2, h2); gA[2] = make_double2(g3, h3);
            fill_top<4>(A.top, tpB[0].x, tpB[1].x, tpB[2].x, g1, g2, g3);
            fill_top<4>(A.top, tpB[0].y, tpB[1].y, tpB[2].y, h1, h2, h3);
            gB[0] = make_double2(g1, h1); gB[1] = make_double2(g2, h2); gB[2] = make_double2(g3, h3);
        }
        ghost_group(gA, gB);
    }
    for (int g = gt - 1; g >= 0; g--) back_group(g, std::false_type{});
    {
        double2 gA[3], gB[3];
        double g1, g2, g3, h1, h2, h3;
        if (ORDER == 2) {
            fill_bot<2>(A.bot[var], x1A.x, 0.0, 0.0, g1, g2, g3);
            fill_bot<2>(A.bot[var], x1A.y, 0.0, 0.0, h1, g2, g3);
            gA[0] = gA[1] = z2; gA[2] = make_double2(g1, h1);
            fill_bot<2>(A.bot[var], x1B.x, 0.0, 0.0, g1, g2, g3);
            fill_bot<2>(A.bot[var], x1B.y, 0.0, 0.0, h1, g2, g3);
            gB[0] = gB[1] = z2; gB[2] = make_double2(g1, h1);
        } else {
            fill_bot<4>(A.bot[var], x1A.x, x2A.x, x3A.x, g1, g2, g3);
            fill_bot<4>(A.bot[var], x1A.y, x2A.y, x3A.y, h1, h2, h3);
            gA[2] = make_double2(g1, h1); gA[1] = make_double2(g2, h2); gA[0] = make_double2(g3, h3);
            fill_bot<4>(A.bot[var], x1B.x, x2B.x, x3B.x, g1, g2, g3);
            fill_bot<4>(A.bot[var], x1B.y, x2B.y, x3B.y, h1, h2, h3);
            gB[2] = make_double2(g1, h1); gB[1] = make_double2(g2, h2); gB[0] = make_double2(g3, h3);
        }
        ghost_group(gA, gB);
    }
}

template <int ORDER, int N>
__global__ void __launch_bounds__(pfft_threads<N>(), 1) k_poisson_fft(Geo G, PoissonFftArgs A)
{
    poisson_fft_body<ORDER, N>(G, A, blockIdx);
}

template <int ORDER, int N, bool FILL = true>
__global__ void __launch_bounds__(pfft_threads<N>(), 1) k_poisson_fft_batch(const BatchRec<PoissonFftArgs>* r, int n)
{
    uint3 b;
    const BatchRec<PoissonFftArgs>& R = batch_locate(r, n, b);
    poisson_fft_body<ORDER, N, FILL>(R.G, R.A, b);
}

// Complex-to-real x transform (fftx_c2d, pressure.c:163-200) as an inverse
// complex transform of half length: with X[0] and X[N/2] taken real (as
// FFTW's c2r does), Z[k] = (X[k] + conj X[M-k]) + i exp(2 pi i k/N)
// (X[k] - conj X[M-k]) for k < M, z = IFFT(Z) unnormalised, and
// x[2m] = Re z[m], x[2m+1] = Im z[m].
template <int N>
__device__ __forceinline__ void k_fftx_c2r_p2_body(const Geo& G, const C2rArgs& A, uint3 bid)
{
    extern __shared__ double2 sbuf[];
    constexpr int M = N / 2, T = M / 8, L = p2_lines(M);
    const int l = threadIdx.x % L, t = threadIdx.x / L;
    const int k = A.kfirst + bid.y;
    const int j = bid.x * L + l;
    const bool valid = j < G.ny;
    const int ny = G.ny;
    const double2* base = A.spec + bid.z * A.fstride + (long long) k * G.nkx * ny + (valid ? j : 0);
    double2 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int kx = t + q * T;
        double2 a = __ldg(base + (long long) kx * ny);
        double2 b = __ldg(base + (long long) (M - kx) * ny);
        if (kx == 0) { a.y = 0.0; b.y = 0.0; }   // imaginary parts of X[0], X[N/2] ignored
        const double sr = a.x + b.x, si = a.y - b.y;   // X[k] + conj X[M-k]
        const double dr = a.x - b.x, di = a.y + b.y;   // X[k] - conj X[M-k]
        const double2 w = __ldg(&A.px.tw[kx]);          // conj of exp(2 pi i kx/N)
        const double tr = w.x * dr + w.y * di, ti = w.x * di - w.y * dr;
        v[q] = make_double2(sr - ti, si + tr);
    }
    fft_p2_line<M>(v, t, sbuf + l * p2_stride_x(M), A.px.tw, +1, A.c8, 2);
    if (!valid) return;
    // the field's pointer picked without indexing the parameter array by a
    // run-time value (which would copy the parameters to the stack)
    double* const pz = bid.z == 0 ? A.p[0] : bid.z == 1 ? A.p[1] : bid.z == 2 ? A.p[2] : A.p[3];
    double* out = pz + (long long) k * G.nx * ny + j;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int m = t + q * T;
        out[(long long) (2 * m) * ny] = v[q].x;
        out[(long long) (2 * m + 1) * ny] = v[q].y;
    }
}

// Four resident blocks per SM, as the forward transform (64 registers, a
// 4-byte spill at N = 512): 0.340 instead of 0.357 ms at 512 x 512 x 384.
template <int N>
__global__ void __launch_bounds__(256, 4) k_fftx_c2r_p2(Geo G, C2rArgs A)
{
    k_fftx_c2r_p2_body<N>(G, A, blockIdx);
}

template <int N>
__global__ void __launch_bounds__(256) k_fftx_c2r_p2_batch(const BatchRec<C2rArgs>* r, int n)
{
    uint3 b;
    const BatchRec<C2rArgs>& R = batch_locate(r, n, b);
    k_fftx_c2r_p2_body<N>(R.G, R.A, b);
}

template <int N>
static size_t p2_smem_x() { return (size_t) p2_lines(N) * p2_stride_x(N) * sizeof(double2); }
template <int N>
static size_t p2_smem_y() { return (size_t) p2_lines(N) * p2_pad(N) * sizeof(double2); }

template <int N>
static void launch_r2c_p2(const Geo& G, const R2cArgs& A, int nrows, int nfields, cudaStream_t st)
{
    constexpr int L = p2_lines(N / 2);
    k_fftx_r2c_p2<N><<<dim3((G.ny + L - 1) / L, nrows, nfields), 256, p2_smem_x<N / 2>(), st>>>(G, A);
}

template <int N>
static void launch_div_fftx_p2(const Geo& G, const DivArgs& A, cudaStream_t st)
{
    dim3 blk(DV_J, DV_I, 1), grd((G.ny + DV_J - 1) / DV_J, (G.nx + DV_I - 1) / DV_I, (G.nz + DV_KC - 1) / DV_KC);
    if (G.order == 2) k_div<2><<<grd, blk, 0, st>>>(G, A);
    else k_div<4><<<grd, blk, 0, st>>>(G, A);
    R2cArgs R{A.dv, A.spec, A.px, A.c8, GZ, 0, 0};
    launch_r2c_p2<N>(G, R, G.nz, 1, st);
}

template <int N>
static void launch_ffty_p2(const Geo& G, const FftyArgs& A, int nrows, int nfields, cudaStream_t st)
{
    constexpr int L = p2_lines(N);
    dim3 grd((G.nkx + L - 1) / L, nrows, nfields);
    k_ffty_p2<N><<<grd, 256, p2_smem_y<N>(), st>>>(G, A);
}

template <int N>
static void launch_c2r_p2(const Geo& G, const C2rArgs& A, int nrows, int nfields, cudaStream_t st)
{
    constexpr int L = p2_lines(N / 2);
    dim3 grd((G.ny + L - 1) / L, nrows, nfields);
    k_fftx_c2r_p2<N><<<grd, 256, p2_smem_x<N / 2>(), st>>>(G, A);
}

template <int N>
static cudaError_t p2_set_smem()
{
    const int sx = (int) p2_smem_x<N / 2>(), sy = (int) p2_smem_y<N>();
    cudaError_t e = cudaFuncSetAttribute(k_fftx_r2c_p2<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sx);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fftx_c2r_p2<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sx);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ffty_p2<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sy);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fftx_r2c_p2_batch<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sx);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fftx_c2r_p2_batch<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sx);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ffty_p2_batch<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sy);
    if constexpr (N == 256 || N == 512) {   // the fused kernel's sizes (poisson_fft_supported)
        const int sp2 = (int) pfft_smem_bytes<2, N>(), sp4 = (int) pfft_smem_bytes<4, N>();
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_poisson_fft<2, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp2);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_poisson_fft<4, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp4);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_poisson_fft_batch<2, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp2);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_poisson_fft_batch<4, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp4);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_poisson_fft_batch<2, N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp2);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_poisson_fft_batch<4, N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp4);
    }
    return e;
}

static bool pow2_kernel_size(int n) { return n == 64 || n == 128 || n == 256 || n == 512; }

// -------------------------------------------------------------- launchers

size_t fft_smem_bytes(int n) { return (size_t) n * FFT_L * sizeof(double2); }

void launch_div_fftx(const Geo& G, const DivArgs& A, cudaStream_t st)
{
    switch (G.nx) {
    case 64: return launch_div_fftx_p2<64>(G, A, st);
    case 128: return launch_div_fftx_p2<128>(G, A, st);
    case 256: return launch_div_fftx_p2<256>(G, A, st);
    case 512: return launch_div_fftx_p2<512>(G, A, st);
    default: break;
    }
    dim3 grd((G.ny + FFT_L - 1) / FFT_L, G.nz);
    size_t sm = fft_smem_bytes(G.nx);
#define CASE_(n_) \
    case n_: \
        if (G.order == 2) k_div_fftx<2, n_><<<grd, FFT_THREADS, sm, st>>>(G, A); \
        else k_div_fftx<4, n_><<<grd, FFT_THREADS, sm, st>>>(G, A); \
        return;
    switch (G.nx) {
    STATIC_FFT_SIZES(CASE_)
    default: break;
    }
#undef CASE_
    if (G.order == 2) k_div_fftx<2, 0><<<grd, FFT_THREADS, sm, st>>>(G, A);
    else k_div_fftx<4, 0><<<grd, FFT_THREADS, sm, st>>>(G, A);
}

void launch_fft2d_field(const Geo& G, const double* field, double2* spec, const FftPlan& px,
                        const FftPlan& py, double c8, cudaStream_t st)
{
    if (pow2_kernel_size(G.nx)) {
        R2cArgs R{field, spec, px, c8, 0, 0, 0};
        launch_fftx_r2c(G, R, G.n2, 1, st);
    } else {
        DivArgs D{};
        D.spec = spec;
        D.px = px;
        D.c8 = c8;
        D.src = field;
        D.kshift = -GZ;
        dim3 grd((G.ny + FFT_L - 1) / FFT_L, G.n2);
        const size_t sm = fft_smem_bytes(G.nx);
#define CASE_(n_) \
    case n_: k_div_fftx<2, n_><<<grd, FFT_THREADS, sm, st>>>(G, D); break;
        switch (G.nx) {
        STATIC_FFT_SIZES(CASE_)
        default: k_div_fftx<2, 0><<<grd, FFT_THREADS, sm, st>>>(G, D); break;
        }
#undef CASE_
    }
    FftyArgs Y{spec, py, -1, 0, c8, 0};
    launch_ffty(G, Y, G.n2, st);
}

bool fftx_batched_supported(int nx)
{
    return nx == 64 || nx == 128 || nx == 256 || nx == 512;
}

void launch_fftx_r2c(const Geo& G, const R2cArgs& A, int nrows, int nfields, cudaStream_t st)
{
    switch (G.nx) {   // power-of-two nx only (fftx_batched_supported)
    case 64: return launch_r2c_p2<64>(G, A, nrows, nfields, st);
    case 128: return launch_r2c_p2<128>(G, A, nrows, nfields, st);
    case 256: return launch_r2c_p2<256>(G, A, nrows, nfields, st);
    case 512: return launch_r2c_p2<512>(G, A, nrows, nfields, st);
    default: break;
    }
}

void launch_ffty(const Geo& G, const FftyArgs& A, int nrows, cudaStream_t st, int nfields)
{
    switch (G.ny) {
    case 64: return launch_ffty_p2<64>(G, A, nrows, nfields, st);
    case 128: return launch_ffty_p2<128>(G, A, nrows, nfields, st);
    case 256: return launch_ffty_p2<256>(G, A, nrows, nfields, st);
    case 512: return launch_ffty_p2<512>(G, A, nrows, nfields, st);
    default: break;
    }
    dim3 grd((G.nkx + FFT_L - 1) / FFT_L, nrows, nfields);
    const size_t sm = fft_generic_smem(G.ny, true);
#define CASE_(n_) \
    case n_: k_ffty<n_><<<grd, FFT_THREADS, sm, st>>>(G, A); return;
    switch (G.ny) {
    STATIC_FFT_SIZES(CASE_)
    default: break;
    }
#undef CASE_
    k_ffty<0><<<grd, FFT_THREADS, sm, st>>>(G, A);
}

void launch_fftx_c2r(const Geo& G, const C2rArgs& A, int nrows, cudaStream_t st, int nfields)
{
    switch (G.nx) {
    case 64: return launch_c2r_p2<64>(G, A, nrows, nfields, st);
    case 128: return launch_c2r_p2<128>(G, A, nrows, nfields, st);
    case 256: return launch_c2r_p2<256>(G, A, nrows, nfields, st);
    case 512: return launch_c2r_p2<512>(G, A, nrows, nfields, st);
    default: break;
    }
    dim3 grd((G.ny + FFT_L - 1) / FFT_L, nrows, nfields);
    const size_t sm = fft_smem_bytes(G.nx);
#define CASE_(n_) \
    case n_: k_fftx_c2r<n_><<<grd, FFT_THREADS, sm, st>>>(G, A); return;
    switch (G.nx) {
    STATIC_FFT_SIZES(CASE_)
    default: break;
    }
#undef CASE_
    k_fftx_c2r<0><<<grd, FFT_THREADS, sm, st>>>(G, A);
}

// ny = 256 or 512: a row group is 2048 points (8 or 4 rows of ny), the
// transform warps' one layout.  Whether an instance takes the fused launch
// by default (one block per kx must give the GPU enough blocks) is decided
// at creation (cf_create).
bool poisson_fft_supported(const Geo& G)
{
    return (G.ny == 256 || G.ny == 512) && (G.order == 2 || G.order == 4);
}

template <int ORDER, int N>
static void launch_poisson_fft_n(const Geo& G, const PoissonFftArgs& A, cudaStream_t st)
{
    k_poisson_fft<ORDER, N><<<G.nkx, pfft_threads<N>(), pfft_smem_bytes<ORDER, N>(), st>>>(G, A);
}

void launch_poisson_fft(const Geo& G, const PoissonFftArgs& A, cudaStream_t st)
{
#define CASE_(n_) \
    case n_: \
        if (G.order == 2) launch_poisson_fft_n<2, n_>(G, A, st); \
        else launch_poisson_fft_n<4, n_>(G, A, st); \
        return;
    switch (G.ny) {   // poisson_fft_supported
    CASE_(256) CASE_(512)
    default: break;
    }
#undef CASE_
}

// The four spectral Helmholtz solves of the fully implicit scheme with their
// y transforms: one record per field (FILL off).
void launch_helmholtz_fft_batch(const BatchLaunch& L, int order, int ny, cudaStream_t st)
{
    auto r = static_cast<const BatchRec<PoissonFftArgs>*>(L.recs);
#define CASE_(n_) \
    case n_: \
        if (order == 2) k_poisson_fft_batch<2, n_, false><<<L.blocks, pfft_threads<n_>(), pfft_smem_bytes<2, n_>(), st>>>(r, L.n); \
        else k_poisson_fft_batch<4, n_, false><<<L.blocks, pfft_threads<n_>(), pfft_smem_bytes<4, n_>(), st>>>(r, L.n); \
        return;
    switch (ny) {
    CASE_(256) CASE_(512)
    default: break;
    }
#undef CASE_
}

void launch_poisson_fft_batch(const BatchLaunch& L, int key, cudaStream_t st)
{
    auto r = static_cast<const BatchRec<PoissonFftArgs>*>(L.recs);
    const int order = key % 8, ny = key / 8;
#define CASE_(n_) \
    case n_: \
        if (order == 2) k_poisson_fft_batch<2, n_><<<L.blocks, pfft_threads<n_>(), pfft_smem_bytes<2, n_>(), st>>>(r, L.n); \
        else k_poisson_fft_batch<4, n_><<<L.blocks, pfft_threads<n_>(), pfft_smem_bytes<4, n_>(), st>>>(r, L.n); \
        return;
    switch (ny) {
    CASE_(256) CASE_(512)
    default: break;
    }
#undef CASE_
}

void launch_poisson(const Geo& G, const PoissonArgs& A, cudaStream_t st)
{
    unsigned nb = grid_poisson(G).x;
    const int nt = G.shape.pois_threads;
    if (G.order == 2) k_poisson<2><<<nb, nt, 0, st>>>(G, A);
    else k_poisson<4><<<nb, nt, pois_smem_bytes(nt), st>>>(G, A);
}

void launch_helmholtz_spectral(const Geo& G, const PoissonArgs& A, cudaStream_t st)
{
    unsigned nb = grid_poisson(G).x;
    const int nt = G.shape.pois_threads;
    if (G.order == 2) k_helmholtz_spectral<2><<<nb, nt, 0, st>>>(G, A);
    else k_helmholtz_spectral<4><<<nb, nt, pois_smem_bytes(nt), st>>>(G, A);
}

void launch_project(const Geo& G, const ProjArgs& A, cudaStream_t st)
{
    dim3 blk(G.shape.proj_bx, G.shape.proj_by, 1);
    dim3 grd = grid_project(G);
    if (G.order == 2) k_project<2><<<grd, blk, 0, st>>>(G, A);
    else k_project<4><<<grd, blk, 0, st>>>(G, A);
}

// ------------------------------------------------------ batched launches
//
// Grids of the single-instance launches above, per stage, and the batched
// launches over records carrying those grids (batch.cuh).  Power-of-two
// transforms are batched per size (their kernels are templates on it); the
// generic transforms of different sizes share one launch with the largest
// instance's shared memory.

dim3 grid_div(const Geo& G)
{
    return dim3((G.ny + DV_J - 1) / DV_J, (G.nx + DV_I - 1) / DV_I, (G.nz + DV_KC - 1) / DV_KC);
}

dim3 grid_r2c(const Geo& G, int nrows, int nfields)
{
    const int L = p2_lines(G.nx / 2);
    return dim3((G.ny + L - 1) / L, nrows, nfields);
}

dim3 grid_div_fftx(const Geo& G) { return dim3((G.ny + FFT_L - 1) / FFT_L, G.nz); }

dim3 grid_ffty(const Geo& G, int nrows, int nfields)
{
    const int L = pow2_kernel_size(G.ny) ? p2_lines(G.ny) : FFT_L;
    return dim3((G.nkx + L - 1) / L, nrows, nfields);
}

dim3 grid_c2r(const Geo& G, int nrows, int nfields)
{
    const int L = pow2_kernel_size(G.nx) ? p2_lines(G.nx / 2) : FFT_L;
    return dim3((G.ny + L - 1) / L, nrows, nfields);
}

// one thread per pair of columns (kx, ky), (kx, ny - ky)
dim3 grid_poisson(const Geo& G)
{
    const long long npair = (long long) G.nkx * (G.ny / 2 + 1);
    const int nt = G.shape.pois_threads;
    return dim3((unsigned) ((npair + nt - 1) / nt));
}

dim3 grid_project(const Geo& G)
{
    const int bx = G.shape.proj_bx, by = G.shape.proj_by;
    return dim3((G.ny + bx - 1) / bx, (G.nx + by - 1) / by, G.n2);
}

template <class Args>
static const BatchRec<Args>* recs_of(const BatchLaunch& L) { return static_cast<const BatchRec<Args>*>(L.recs); }

void launch_div_batch(const BatchLaunch& L, int order, cudaStream_t st)
{
    dim3 blk(DV_J, DV_I, 1);
    if (order == 2) k_div_batch<2><<<L.blocks, blk, 0, st>>>(recs_of<DivArgs>(L), L.n);
    else k_div_batch<4><<<L.blocks, blk, 0, st>>>(recs_of<DivArgs>(L), L.n);
}

void launch_r2c_batch(const BatchLaunch& L, int nx, cudaStream_t st)
{
    switch (nx) {
    case 64: k_fftx_r2c_p2_batch<64><<<L.blocks, 256, p2_smem_x<32>(), st>>>(recs_of<R2cArgs>(L), L.n); break;
    case 128: k_fftx_r2c_p2_batch<128><<<L.blocks, 256, p2_smem_x<64>(), st>>>(recs_of<R2cArgs>(L), L.n); break;
    case 256: k_fftx_r2c_p2_batch<256><<<L.blocks, 256, p2_smem_x<128>(), st>>>(recs_of<R2cArgs>(L), L.n); break;
    default: k_fftx_r2c_p2_batch<512><<<L.blocks, 256, p2_smem_x<256>(), st>>>(recs_of<R2cArgs>(L), L.n); break;
    }
}

void launch_div_fftx_batch(const BatchLaunch& L, int order, int nx, cudaStream_t st)
{
    auto r = recs_of<DivArgs>(L);
#define CASE_(n_) \
    case n_: \
        if (order == 2) k_div_fftx_batch<2, n_><<<L.blocks, FFT_THREADS, L.smem, st>>>(r, L.n); \
        else k_div_fftx_batch<4, n_><<<L.blocks, FFT_THREADS, L.smem, st>>>(r, L.n); \
        return;
    switch (nx) {
    STATIC_FFT_SIZES(CASE_)
    default: break;
    }
#undef CASE_
    if (order == 2) k_div_fftx_batch<2, 0><<<L.blocks, FFT_THREADS, L.smem, st>>>(r, L.n);
    else k_div_fftx_batch<4, 0><<<L.blocks, FFT_THREADS, L.smem, st>>>(r, L.n);
}

void launch_ffty_batch(const BatchLaunch& L, int ny, cudaStream_t st)
{
    switch (ny) {
    case 64: k_ffty_p2_batch<64><<<L.blocks, 256, p2_smem_y<64>(), st>>>(recs_of<FftyArgs>(L), L.n); break;
    case 128: k_ffty_p2_batch<128><<<L.blocks, 256, p2_smem_y<128>(), st>>>(recs_of<FftyArgs>(L), L.n); break;
    case 256: k_ffty_p2_batch<256><<<L.blocks, 256, p2_smem_y<256>(), st>>>(recs_of<FftyArgs>(L), L.n); break;
    case 512: k_ffty_p2_batch<512><<<L.blocks, 256, p2_smem_y<512>(), st>>>(recs_of<FftyArgs>(L), L.n); break;
#define CASE_(n_) \
    case n_: k_ffty_batch<n_><<<L.blocks, FFT_THREADS, L.smem, st>>>(recs_of<FftyArgs>(L), L.n); break;
    STATIC_FFT_SIZES(CASE_)
#undef CASE_
    default: k_ffty_batch<0><<<L.blocks, FFT_THREADS, L.smem, st>>>(recs_of<FftyArgs>(L), L.n); break;
    }
}

void launch_poisson_batch(const BatchLaunch& L, int order, cudaStream_t st)
{
    if (order == 2) k_poisson_batch<2><<<L.blocks, L.block, 0, st>>>(recs_of<PoissonArgs>(L), L.n);
    else k_poisson_batch<4><<<L.blocks, L.block, pois_smem_bytes(L.block.x), st>>>(recs_of<PoissonArgs>(L), L.n);
}

void launch_c2r_batch(const BatchLaunch& L, int nx, cudaStream_t st)
{
    switch (nx) {
    case 64: k_fftx_c2r_p2_batch<64><<<L.blocks, 256, p2_smem_x<32>(), st>>>(recs_of<C2rArgs>(L), L.n); break;
    case 128: k_fftx_c2r_p2_batch<128><<<L.blocks, 256, p2_smem_x<64>(), st>>>(recs_of<C2rArgs>(L), L.n); break;
    case 256: k_fftx_c2r_p2_batch<256><<<L.blocks, 256, p2_smem_x<128>(), st>>>(recs_of<C2rArgs>(L), L.n); break;
    case 512: k_fftx_c2r_p2_batch<512><<<L.blocks, 256, p2_smem_x<256>(), st>>>(recs_of<C2rArgs>(L), L.n); break;
#define CASE_(n_) \
    case n_: k_fftx_c2r_batch<n_><<<L.blocks, FFT_THREADS, L.smem, st>>>(recs_of<C2rArgs>(L), L.n); break;
    STATIC_FFT_SIZES(CASE_)
#undef CASE_
    default: k_fftx_c2r_batch<0><<<L.blocks, FFT_THREADS, L.smem, st>>>(recs_of<C2rArgs>(L), L.n); break;
    }
}

void launch_project_batch(const BatchLaunch& L, int order, cudaStream_t st)
{
    if (order == 2) k_project_batch<2><<<L.blocks, L.block, 0, st>>>(recs_of<ProjArgs>(L), L.n);
    else k_project_batch<4><<<L.blocks, L.block, 0, st>>>(recs_of<ProjArgs>(L), L.n);
}

bool batch_pow2(int n) { return pow2_kernel_size(n); }

int fft_kernel_key(int n) { return pow2_kernel_size(n) || static_fft_size(n) ? n : 0; }

cudaError_t fft_set_smem_limits(int max_n)
{
    size_t sm = fft_smem_bytes(max_n);
    cudaError_t e = p2_set_smem<64>();
    if (e == cudaSuccess) e = p2_set_smem<128>();
    if (e == cudaSuccess) e = p2_set_smem<256>();
    if (e == cudaSuccess) e = p2_set_smem<512>();
    (void) sm;
    // generic transforms (single and batched): room for the largest size
    // handled by the runtime plan and for the padded fixed-size buffers
    const int v = (int) std::max(fft_smem_bytes(FFT_MAX_N), fft_generic_smem(384, true));
    auto set = [&](const void* f) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    };
#define SET_(n_) \
    set((const void*) k_div_fftx<2, n_>); set((const void*) k_div_fftx<4, n_>); \
    set((const void*) k_ffty<n_>); set((const void*) k_fftx_c2r<n_>); \
    set((const void*) k_div_fftx_batch<2, n_>); set((const void*) k_div_fftx_batch<4, n_>); \
    set((const void*) k_ffty_batch<n_>); set((const void*) k_fftx_c2r_batch<n_>);
    SET_(0)
    STATIC_FFT_SIZES(SET_)
#undef SET_
    return e;
}

}  // namespace cf
