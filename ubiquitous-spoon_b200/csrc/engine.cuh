// Device engine of the channel-flow RK3 substep (sm_100a, FP64).
//
// Device layout of every field: [k][i][j], wall-normal index k slowest and
// spanwise index j fastest, no x/y ghost cells (periodicity is modular
// indexing), all n2 = nz + 2*gz wall-normal rows kept.  Column c = i*ny + j.
// One z line is therefore a strided column whose rows are contiguous across
// neighbouring columns, so the per-column line solves run one thread per
// column with coalesced row accesses.  The reference's own layout
// ([i][j][k], k fastest, padded by ghosts in x and y; d3tensor.c:9-42) is
// converted only at the API boundary.
//
// Spectral layout: complex [k][kx][ky], kx in [0, nx/2], ky in [0, ny).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cf {

constexpr int GZ = 3;                // wall-normal ghost rows (reference main.c:13)
constexpr int MAX_FFT_STAGES = 12;
constexpr int LOG_COLS = 10;

// Band coefficient rows of one wall closure (rows k, k-+1, k-+2; a..g).
struct WallRowsD {
    double row[3][7];
};

// Launch shapes of the kernels whose block shape is free: the tuner
// (instance.cu, cf_tune) times the candidates and keeps the fastest; the
// defaults are the hand-picked shapes.  Results do not depend on the choice:
// these kernels index their work from blockDim, one column (pair, point) per
// thread, and the per-warp row sums of k_back4 cover the same 32 columns
// whatever the block size.
struct LaunchShape {
    int solve_threads = 128;           // k_back4: columns per block (64, 128)
    int pois_threads = 128;            // k_poisson / k_helmholtz_spectral: column pairs per block (64, 128)
    int proj_bx = 32, proj_by = 4;     // k_project block: j by i (32x2, 32x4, 32x8, 64x2)
};
// k_back4 is bound to 128 threads: a 256-thread bound costs it 4 registers
// and one resident block per SM (measured 40 % slower)
constexpr int SOLVE_THREADS_MAX = 128;
constexpr int POIS_THREADS_MAX = 128;
constexpr int PROJ_THREADS_MAX = 256;

// Geometry / metric tables shared by all kernels of an instance.
struct Geo {
    LaunchShape shape;    // tuned launch shapes (host side; kernels read blockDim)
    int order, nx, ny, nz, n2, nkx;
    long long plane;      // nx*ny (points per k-plane)
    long long splane;     // nkx*ny (spectral columns per k-plane)
    double dx, dy;
    const double* dz;     // [n2]
    const double* dzp1h;  // 0.5*(dz[k+1]+dz[k])  [n2] (last entry 0)
    const double* dzm1h;  // 0.5*(dz[k-1]+dz[k])  [n2] (first entry 0)
    const double* dzp3h;  // 0.5*(dz[k+2]+dz[k+1])
    const double* dzm3h;  // 0.5*(dz[k-2]+dz[k-1])
    const double* dydz;   // dy*dz[k]
    const double* dxdz;   // dx*dz[k]
    const double* ivol;   // 1 / (dx*dy*dz[k])       cell volume
    const double* ivolw;  // 1 / (dx*dy*dzp1h[k])    w-face volume
    const double* idzp1h; // 1 / dzp1h[k]
    const double* idz;    // 1 / dz[k]
    double dxdy;          // dx*dy
    double idx, idy;      // 1/dx, 1/dy
};

// Line-solve factorisation on device (see host_band.h LineFactor).
struct FactorD {
    int k0, n;
    const double *F1, *F2, *F3, *DEN, *P, *Q, *R;
};

// Back substitution of one implicit solve (its forward sweep runs in k_rhs).
struct SolveArgs {
    double* x;            // field: out, the new value (all n2 rows)
    const double* s;      // forward-substituted vector, rows k0 .. k0+n-1
    FactorD fac;          // back-substitution multipliers P, Q, R; rows k0 .. k0+n-1
    double bc_bot, bc_top;
    WallRowsD bcb, bct;   // apply_bc closure rows for this field
    double* partial;      // per-warp row sums [nwarps][n2] or null
};

struct FftPlan {
    int n, nstages;
    int radix[MAX_FFT_STAGES];
    const double2* tw;    // tw[m] = exp(-2 pi i m / n)
};

struct Fields {
    double *u, *v, *w, *c;
};

struct GhostArgs {
    Fields F;
    WallRowsD ub, ut, wb, wt;   // u-type and w-type closure rows
    double bc_u, bc_v, bc_c_bot, bc_c_top, bc_w;
};

// Forward sweep of one implicit solve, fused into k_rhs (see host_band.h
// fused_rows): s_i = sum cu_m x_{k+m} + cf f_k + cg g_k + c0 - f1 s_{i-1} - ...
struct FwdSweep {
    double* g;             // in: previous-stage RHS g; out: the forward-substituted s (same rows)
    const double* gshift;  // device scalar added to g (mass-flux lazily applied), or null
    const double* rows;    // fused forward rows [n][fused_width]
};

struct RhsArgs {
    const double *u, *v, *w, *c;
    double *fu, *fv, *fw, *fc;
    double nu, kappa;              // nu and nu/prandtl
    double betg_x, betg_y, betg_z;
    FwdSweep sw[4];                // u, v, w, c
    WallRowsD wbot, wtop;          // apply_bc_w closure rows (ghost values of the old w)
    double wbc_bot, wbc_top;
};

struct MassArgs {
    const double* avg;
    const double* dz;
    int order, nz, n2;
    double kappa;
    double green[4];      // statistics of the Green's function column
    int mode;             // uvolavgmode / cvolavgmode
    double target;        // want_uvolavg - uframe, or want_cvolavg
    double fixed;         // -dpdx (u) or 0 (c) when mode != 1
    double* m_out;        // device scalar: mdpdx / dcdt of this substep
    long long* counter;   // device substep counter selecting the log row
    double* log_base;     // log ring buffer [log_cap][LOG_COLS]
    int log_cap;
    int col;              // first column written: m, bottom gradient, top gradient, bulk, centreline
    int advance;          // 1: increment the counter afterwards (last statistics of a substep)
    double* nonfinite;    // device flag: set to 1 when the bulk mean or the control is NaN / Inf
};

struct RowAvgArgs {
    const double* partial;   // per-warp row sums [nwarps][n2]
    long long nwarps;
    int n2;
    double scale;            // 1 / (nx ny)
    double* avg;             // [n2] out
};

struct DivArgs {
    const double *u, *v, *w;
    const double* gu;      // Green's function column of u (n2) or null
    const double* mu;      // device scalar mdpdx or null
    double2* spec;         // [n2][nkx][ny]
    FftPlan px;
    double c8;
    double* dv;            // real divergence field [n2][nx][ny] (power-of-two nx path)
    const double* src;     // non-null: transform this field instead of the divergence
    int kshift;            // rows GZ + kshift ..: 0 for the divergence, -GZ for all n2 rows
};

// Real-to-complex x transform of rows kfirst .. of nfields real fields
// (blockIdx.z = field, fields src_fstride doubles apart) into spectra
// spec_fstride complex values apart.
struct R2cArgs {
    const double* src;
    double2* spec;
    FftPlan px;
    double c8;
    int kfirst;
    long long src_fstride, spec_fstride;
};

struct FftyArgs {
    double2* spec;
    FftPlan py;
    int sign;
    int kfirst;
    double c8;
    long long fstride;    // complex values between the spectra of batched fields
};

// Inverse x transform of spectrum rows kfirst .. of field blockIdx.z into
// the same rows of p[blockIdx.z].
struct C2rArgs {
    const double2* spec;
    double* p[4];
    FftPlan px;
    double c8;
    int kfirst;
    long long fstride;
};

// One per-wavenumber band solve over spectrum rows GZ .. GZ+nrows-1: the
// pressure Poisson equation or the spectral Helmholtz solve of one field.
struct PoissonArgs {
    double2* spec;
    double* scratch;          // width 3: 1 x [n2][ncol]; width 7: 3 x [n2][ncol]
    const double *a, *b, *c, *e, *f, *g, *dpart, *dvol, *lamx, *lamy;
    const double *cx, *cy;    // dvol dt / dx^2, dvol dt / dy^2 per row
    double red[2][6][7];
    double dsub[2][6][3];
    WallRowsD bot[2], top;
    double dt, dxdx, dydy;
    int nrows;                // nz; nz - 1 for the w Helmholtz solve
    double* avg;              // Helmholtz solves of u and c: xy-average profile [n2] out, or null
    WallRowsD abot, atop;     // apply_bc closure rows of that field (its average's ghost rows)
    double abc_bot, abc_top;  // and its wall values
};

// k_poisson block: one thread per (kx, +-ky) column pair, LaunchShape::pois_threads per block
constexpr int POIS_PF = 8;         // forward rows in flight per thread (both columns)
constexpr int POIS_PB = 2;         // back-substitution rows loaded ahead (registers)
inline size_t pois_smem_bytes(int threads) { return (size_t) POIS_PF * 2 * threads * 16; }

// k_poisson_fft: forward y transform + Poisson solve (with the wall ghost
// rows) + inverse y transform, one block per kx, for power-of-two ny
struct PoissonFftArgs {
    PoissonArgs P;
    const double2* twy;   // exp(-2 pi i m / ny)
    double c8;            // cos(pi/4) from the host table
    double* fault;        // set to 1 when a wait for a row copy gave up
    int stall;            // test hook: nonzero leaves the forward row copies unissued,
                          // so that the first wait runs out (cf_debug_stall_copies)
};
bool poisson_fft_supported(const Geo& G);
void launch_poisson_fft(const Geo& G, const PoissonFftArgs& A, cudaStream_t st);

struct ProjArgs {
    double *u, *v, *w, *c;
    const double* p;
    const double *gu, *gc;          // Green's function columns (n2) or null
    const double *mu, *mc;          // device scalars mdpdx, dcdt or null
    double dt;                      // (alpha + beta) dt of the substep
    double dtdx, dtdy;              // dt/dx, dt/dy
};

// ---------------------------------------------------------------- launchers
// extrap: w ghosts as massflux4 leaves them (before the advection);
// otherwise as apply_bc_w leaves them (after the spectral solves)
void launch_ghosts(const Geo& G, const GhostArgs& A, cudaStream_t st, bool extrap = true);
void launch_rhs(const Geo& G, const RhsArgs& A, bool implicit3d, cudaStream_t st);
// k_back4 block: one thread per column, LaunchShape::solve_threads per block
struct SolveBatch {
    SolveArgs a[4];   // u, v, c, w
};
void launch_back4(const Geo& G, const SolveBatch& B, cudaStream_t st);
void launch_mass(const Geo& G, const double* partial, double* avg, const MassArgs& M, cudaStream_t st);
void launch_mass_control(const MassArgs& M, cudaStream_t st);
void launch_div_fftx(const Geo& G, const DivArgs& A, cudaStream_t st);
bool fftx_batched_supported(int nx);
void launch_fftx_r2c(const Geo& G, const R2cArgs& A, int nrows, int nfields, cudaStream_t st);
// forward 2-D transform (x then y, scaled by 1/(nx ny)) of all n2 rows of one field into spec
void launch_fft2d_field(const Geo& G, const double* field, double2* spec, const FftPlan& px,
                        const FftPlan& py, double c8, cudaStream_t st);
void launch_ffty(const Geo& G, const FftyArgs& A, int nrows, cudaStream_t st, int nfields = 1);
void launch_fftx_c2r(const Geo& G, const C2rArgs& A, int nrows, cudaStream_t st, int nfields = 1);
void launch_poisson(const Geo& G, const PoissonArgs& A, cudaStream_t st);
void launch_helmholtz_spectral(const Geo& G, const PoissonArgs& A, cudaStream_t st);
void launch_project(const Geo& G, const ProjArgs& A, cudaStream_t st);
cudaError_t fft_set_smem_limits(int max_n);

// ------------------------------------------------- batched launches (batch.cuh)
struct BatchLaunch;
dim3 grid_ghosts(const Geo& G);
dim3 grid_rhs(const Geo& G);
dim3 grid_back4(const Geo& G);
dim3 grid_div(const Geo& G);                       // power-of-two nx: divergence
dim3 grid_r2c(const Geo& G, int nrows, int nfields);
dim3 grid_div_fftx(const Geo& G);                  // other nx: divergence + x transform
dim3 grid_ffty(const Geo& G, int nrows, int nfields);
dim3 grid_poisson(const Geo& G);
dim3 grid_c2r(const Geo& G, int nrows, int nfields);
dim3 grid_project(const Geo& G);
bool batch_pow2(int n);                            // n has a power-of-two transform kernel
RowAvgArgs row_average_args(const Geo& G, const double* partial, double* avg);
void launch_ghosts_batch(const BatchLaunch& L, int order, cudaStream_t st);
void launch_rhs_batch(const BatchLaunch& L, int order, cudaStream_t st);
void launch_back4_batch(const BatchLaunch& L, int order, cudaStream_t st);
void launch_row_average_batch(const BatchLaunch& L, cudaStream_t st);
void launch_mass_control_batch(const BatchLaunch& L, cudaStream_t st);
void launch_div_batch(const BatchLaunch& L, int order, cudaStream_t st);
void launch_r2c_batch(const BatchLaunch& L, int nx, cudaStream_t st);
void launch_div_fftx_batch(const BatchLaunch& L, int order, int nx, cudaStream_t st);
int fft_kernel_key(int n);                          // n with its own transform kernels, else 0
size_t fft_generic_smem(int n, bool line_major);    // shared memory of the non-power-of-two transforms
void launch_ffty_batch(const BatchLaunch& L, int ny, cudaStream_t st);   // ny: power of two, else generic
void launch_poisson_batch(const BatchLaunch& L, int order, cudaStream_t st);
// key: 8 * ny + order
void launch_poisson_fft_batch(const BatchLaunch& L, int key, cudaStream_t st);
// the four spectral Helmholtz solves of the fully implicit scheme with their y
// transforms, one record per field (ny = 256 or 512)
void launch_helmholtz_fft_batch(const BatchLaunch& L, int order, int ny, cudaStream_t st);
void launch_c2r_batch(const BatchLaunch& L, int nx, cudaStream_t st);    // nx: power of two, else generic
void launch_project_batch(const BatchLaunch& L, int order, cudaStream_t st);
cudaError_t rhs_set_smem_limits();
size_t fft_smem_bytes(int n);
constexpr int FFT_MAX_N = 512;

}  // namespace cf
