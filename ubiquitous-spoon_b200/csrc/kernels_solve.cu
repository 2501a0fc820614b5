// Implicit wall-normal diffusion, second half: one thread per column.
//
// Per column the substep does what chanfast.c:459-482 does for one field
// (order 2; :1383-1406 order 4):
//   h  = helmholtz1d_operator(x, nuadt) + gamdt*f + zetdt*g - hbc
//   x  = solve_helmholtz1d(h, -nubdt)       (tridag.c / heptdag.c)
//   apply_bc(x)
// The band matrix is the same for every column, so its factorisation comes
// precomputed from host_band.cpp; the Helmholtz operator, the RK3 combination,
// the cell volume and the pivot reciprocal are folded into one coefficient
// row per k (fused_rows), and the forward sweep runs inside k_rhs
// (kernels_rhs.cu) right after each row's right-hand side, leaving the
// forward-substituted vector s in the g buffer.  This file does the back
// substitution and apply_bc of the four fields in one launch; with `partial`
// set, each warp also writes the sum of its 32 columns for every row (input
// of get_xy_avg, get.c:281-302).
#include "engine.cuh"
#include "host_band.h"
#include "wall.cuh"
#include "batch.cuh"

namespace cf {

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Back substitution and apply_bc of one column of one field.
template <int ORDER, bool IS_W>
__device__ __forceinline__ void back_column(const Geo& G, const SolveArgs& A, uint3 bid)
{
    const long long col = (long long) bid.x * blockDim.x + threadIdx.x;
    const bool active = col < G.plane;
    const long long P = G.plane;
    const int n2 = G.n2;
    const int kb = GZ - 1;                          // bottom wall ghost row / face
    const int kt = IS_W ? n2 - GZ - 1 : n2 - GZ;    // top wall ghost row / face
    const int n = A.fac.n, k0 = A.fac.k0;
    double* __restrict__ x = A.x;
    const double* __restrict__ sv = A.s;
    const long long cc = active ? col : 0;

    // x_i = s_i - P_i x_{i+1} - Q_i x_{i+2} - R_i x_{i+3}, evaluated with
    // x_{i+1} last (one dependent operation per row on the critical path);
    // s of row i - PD loaded into registers while row i is computed.
    constexpr int PD = 4;
    double ps[PD];
    auto fetch_s = [&](int i, int slot) {
        if (i >= 0) ps[slot] = sv[(long long) (k0 + i) * P + cc];
    };
#pragma unroll
    for (int u = 0; u < PD; u++) fetch_s(n - 1 - u, u);
    double y1 = 0.0, y2 = 0.0, y3 = 0.0;
    double top0 = 0.0, top1 = 0.0, top2 = 0.0, bot0 = 0.0, bot1 = 0.0, bot2 = 0.0;
    const bool stats = A.partial != nullptr;
    const long long wrow = ((long long) bid.x * blockDim.x + threadIdx.x) / 32;
    for (int i0 = n - 1; i0 >= 0; i0 -= PD) {
#pragma unroll
        for (int u = 0; u < PD; u++) {
            const int i = i0 - u;
            if (i >= 0) {
                const int k = k0 + i;
                const double s = ps[u];
                fetch_s(i - PD, u);
                double y;
                if (ORDER == 2) y = s - __ldg(A.fac.P + i) * y1;
                else y = ((s - __ldg(A.fac.R + i) * y3) - __ldg(A.fac.Q + i) * y2) - __ldg(A.fac.P + i) * y1;   // y1 last
                y3 = y2; y2 = y1; y1 = y;
                if (active) x[(long long) k * P + col] = y;
                if (i == n - 1) top0 = y;
                if (i == n - 2) top1 = y;
                if (i == n - 3) top2 = y;
                if (i == 0) bot0 = y;
                if (i == 1) bot1 = y;
                if (i == 2) bot2 = y;
                if (stats) {
                    double t = warp_sum(active ? y : 0.0);
                    if ((threadIdx.x & 31) == 0) A.partial[wrow * n2 + k] = t;
                }
            }
        }
    }

    // apply_bc after the solve (chanfast.c:481-482)
    double b1, b2, b3, t1, t2, t3;
    if (IS_W) {
        bc_w_bot<ORDER>(A.bcb, A.bc_bot, bot0, bot1, b1, b2, b3);
        bc_w_top<ORDER>(A.bct, A.bc_top, top0, top1, t1, t2, t3);
    } else {
        bc_u_bot<ORDER>(A.bcb, A.bc_bot, bot0, bot1, bot2, b1, b2, b3);
        bc_u_top<ORDER>(A.bct, A.bc_top, top0, top1, top2, t1, t2, t3);
    }
    if (active) {
        x[(long long) kb * P + col] = b1;
        x[(long long) kt * P + col] = t1;
        if (ORDER == 4) {
            x[(long long) (kb - 1) * P + col] = b2;
            x[(long long) (kb - 2) * P + col] = b3;
            x[(long long) (kt + 1) * P + col] = t2;
            x[(long long) (kt + 2) * P + col] = t3;
        }
    }
    if (stats) {
        // ghost rows as the reference holds them after apply_bc; rows the
        // second-order closure does not touch are zero there.
        for (int k = 0; k < n2; k++) {
            if (k >= k0 && k < k0 + n) continue;
            double v = 0.0;
            if (k == kb) v = b1;
            else if (k == kt) v = t1;
            else if (ORDER == 4 && k == kb - 1) v = b2;
            else if (ORDER == 4 && k == kb - 2) v = b3;
            else if (ORDER == 4 && k == kt + 1) v = t2;
            else if (ORDER == 4 && k == kt + 2) v = t3;
            double t = warp_sum(active ? v : 0.0);
            if ((threadIdx.x & 31) == 0) A.partial[wrow * n2 + k] = t;
        }
    }
}

// Row sums of the per-warp partials -> xy-average profile avg[k]
// (get_xy_avg, get.c:281-302).  One block per row, fixed summation order.
__device__ __forceinline__ void row_average_body(const RowAvgArgs& A, uint3 bid)
{
    __shared__ double red[256];
    const int k = bid.x, n2 = A.n2;
    const double* __restrict__ partial = A.partial;
    double s = 0.0;
    for (long long w = threadIdx.x; w < A.nwarps; w += blockDim.x) s += partial[w * n2 + k];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) A.avg[k] = red[0] * A.scale;
}

__global__ void k_row_average(RowAvgArgs A) { row_average_body(A, blockIdx); }

__global__ void k_row_average_batch(const BatchRec<RowAvgArgs>* r, int n)
{
    uint3 b;
    const BatchRec<RowAvgArgs>& R = batch_locate(r, n, b);
    row_average_body(R.A, b);
}

// Bulk-mean control of chanfast.c:485-529 (u) / 572-616 (c).  The warp
// stages the profile and the cell heights in shared memory (rows up to
// MASS_MAX_N2, else read in place); one thread then sums them in the
// reference's order.
constexpr int MASS_MAX_N2 = 2048;   // 32 KB of static shared memory
__device__ __forceinline__ void mass_control_body(const MassArgs& A)
{
    __shared__ double s_avg[MASS_MAX_N2], s_dz[MASS_MAX_N2];
    const int g = GZ, n2 = A.n2, nz = A.nz;
    const bool staged = n2 <= MASS_MAX_N2;
    if (staged) {
        for (int k = threadIdx.x; k < n2; k += blockDim.x) {
            s_avg[k] = A.avg[k];
            s_dz[k] = A.dz[k];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double* avg = staged ? s_avg : A.avg;
    const double* dz = staged ? s_dz : A.dz;
    double a = 0.0, l = 0.0;  // get_z_avg (get.c:490-502)
    for (int k = g; k < nz + g; k++) {
        a += avg[k] * dz[k];
        l += dz[k];
    }
    double s[4];
    s[0] = a / l;
    if (A.order == 4) {
        s[1] = A.kappa * (A1 * (avg[g] - avg[g - 1]) + A2 * (avg[g + 1] - avg[g - 2])) / (0.5 * (dz[g] + dz[g - 1]));
        s[2] = A.kappa * (A1 * (avg[n2 - g] - avg[n2 - g - 1]) + A2 * (avg[n2 - g + 1] - avg[n2 - g - 2]))
               / (0.5 * (dz[n2 - g] + dz[n2 - g - 1]));
    } else {
        s[1] = A.kappa * (avg[g] - avg[g - 1]) / (0.5 * (dz[g] + dz[g - 1]));
        s[2] = A.kappa * (avg[n2 - g] - avg[n2 - g - 1]) / (0.5 * (dz[n2 - g] + dz[n2 - g - 1]));
    }
    s[3] = nz % 2 == 0 ? 0.5 * (avg[g + nz / 2 - 1] + avg[g + nz / 2]) : avg[g + nz / 2];
    double m = A.mode == 1 ? (A.target - s[0]) / A.green[0] : A.fixed;
    // The bulk mean sums every interior point of the field, so a NaN or Inf
    // anywhere in it (or in the control) shows here; the flag stays set
    // until the host resets it with new fields.
    if (A.nonfinite && !isfinite(s[0] + m)) *A.nonfinite = 1.0;
    for (int t = 0; t < 4; t++) s[t] += A.green[t] * m;
    *A.m_out = m;
    if (A.log_base) {
        long long cnt = *A.counter;
        double* row = A.log_base + (cnt % A.log_cap) * LOG_COLS + A.col;
        row[0] = m;
        row[1] = s[1];
        row[2] = s[2];
        row[3] = s[0];
        row[4] = s[3];
        if (A.advance) *A.counter = cnt + 1;
    }
}

__global__ void k_mass_control(MassArgs A)
{
    if (blockIdx.x == 0) mass_control_body(A);
}

__global__ void k_mass_control_batch(const BatchRec<MassArgs>* r, int n)
{
    uint3 b;
    const BatchRec<MassArgs>& R = batch_locate(r, n, b);
    mass_control_body(R.A);
}

// The back substitutions of the four implicit solves in one launch; the
// control kernels that read the u and c row sums run after it.  blockIdx.y
// selects the field: 0 u, 1 v, 2 c, 3 w.
template <int ORDER>
__device__ __forceinline__ void back4_body(const Geo& G, const SolveBatch& B, uint3 bid)
{
    switch (bid.y) {
    case 0: back_column<ORDER, false>(G, B.a[0], bid); break;
    case 1: back_column<ORDER, false>(G, B.a[1], bid); break;
    case 2: back_column<ORDER, false>(G, B.a[2], bid); break;
    default: back_column<ORDER, true>(G, B.a[3], bid); break;
    }
}

template <int ORDER>
__global__ void __launch_bounds__(SOLVE_THREADS_MAX) k_back4(Geo G, SolveBatch B)
{
    back4_body<ORDER>(G, B, blockIdx);
}

template <int ORDER>
__global__ void __launch_bounds__(SOLVE_THREADS_MAX) k_back4_batch(const BatchRec<SolveBatch>* r, int n)
{
    uint3 b;
    const BatchRec<SolveBatch>& R = batch_locate(r, n, b);
    back4_body<ORDER>(R.G, R.A, b);
}

dim3 grid_back4(const Geo& G)
{
    const int nt = G.shape.solve_threads;
    return dim3((unsigned) ((G.plane + nt - 1) / nt), 4);
}

void launch_back4(const Geo& G, const SolveBatch& B, cudaStream_t st)
{
    dim3 grd = grid_back4(G);
    const int nt = G.shape.solve_threads;
    if (G.order == 2) k_back4<2><<<grd, nt, 0, st>>>(G, B);
    else k_back4<4><<<grd, nt, 0, st>>>(G, B);
}

RowAvgArgs row_average_args(const Geo& G, const double* partial, double* avg)
{
    RowAvgArgs R;
    R.partial = partial;
    const int nt = G.shape.solve_threads;
    R.nwarps = ((G.plane + nt - 1) / nt) * (nt / 32);
    R.n2 = G.n2;
    R.scale = 1.0 / ((double) G.nx * (double) G.ny);
    R.avg = avg;
    return R;
}

void launch_mass(const Geo& G, const double* partial, double* avg, const MassArgs& M, cudaStream_t st)
{
    k_row_average<<<G.n2, 256, 0, st>>>(row_average_args(G, partial, avg));
    k_mass_control<<<1, 32, 0, st>>>(M);
}

void launch_mass_control(const MassArgs& M, cudaStream_t st)
{
    k_mass_control<<<1, 32, 0, st>>>(M);
}

void launch_back4_batch(const BatchLaunch& L, int order, cudaStream_t st)
{
    auto r = static_cast<const BatchRec<SolveBatch>*>(L.recs);
    if (order == 2) k_back4_batch<2><<<L.blocks, L.block, 0, st>>>(r, L.n);
    else k_back4_batch<4><<<L.blocks, L.block, 0, st>>>(r, L.n);
}

void launch_row_average_batch(const BatchLaunch& L, cudaStream_t st)
{
    k_row_average_batch<<<L.blocks, 256, 0, st>>>(static_cast<const BatchRec<RowAvgArgs>*>(L.recs), L.n);
}

void launch_mass_control_batch(const BatchLaunch& L, cudaStream_t st)
{
    k_mass_control_batch<<<L.blocks, 32, 0, st>>>(static_cast<const BatchRec<MassArgs>*>(L.recs), L.n);
}

}  // namespace cf
