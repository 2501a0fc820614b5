// Implicit wall-normal diffusion: one thread per column.
//
// Per column this kernel does what chanfast.c:459-482 does for one field
// (order 2; :1383-1406 order 4):
//   h  = helmholtz1d_operator(x, nuadt) + gamdt*f + zetdt*g - hbc
//   x  = solve_helmholtz1d(h, -nubdt)       (tridag.c / heptdag.c)
//   apply_bc(x)
// The band matrix is the same for every column, so its factorisation comes
// precomputed from host_band.cpp; the Helmholtz operator, the RK3 combination,
// the cell volume and the pivot reciprocal are folded into one coefficient
// row per k (fused_rows), so the forward sweep is a short dot product per row
// and results agree with the reference to rounding.  The forward-substituted
// vector s is kept in the field's own storage between the two sweeps.  With `partial` set, each warp also writes the sum of its
// 32 columns for every row (input of get_xy_avg, get.c:281-302).
#include "engine.cuh"
#include "host_band.h"

namespace cf {

template <int ORDER>
__device__ __forceinline__ void bcu_bot(const WallRowsD& R, double bc, double x0, double x1, double x2,
                                        double& g1, double& g2, double& g3)
{
    if (ORDER == 2) {
        g1 = (R.row[0][2] * x0 - bc) / -R.row[0][1];
        g2 = g3 = 0.0;
    } else {
        g1 = (R.row[2][6] * x0) / -R.row[2][5];
        g2 = (R.row[1][4] * g1 + R.row[1][5] * x0 + R.row[1][6] * x1 - bc) / -R.row[1][3];
        g3 = (R.row[0][2] * g2 + R.row[0][3] * g1 + R.row[0][4] * x0 + R.row[0][5] * x1
              + R.row[0][6] * x2) / -R.row[0][1];
    }
}

template <int ORDER>
__device__ __forceinline__ void bcu_top(const WallRowsD& R, double bc, double x0, double x1, double x2,
                                        double& g1, double& g2, double& g3)
{
    if (ORDER == 2) {
        g1 = (R.row[0][0] * x0 - bc) / -R.row[0][1];
        g2 = g3 = 0.0;
    } else {
        g1 = (R.row[2][0] * x0) / -R.row[2][1];
        g2 = (R.row[1][0] * x1 + R.row[1][1] * x0 + R.row[1][2] * g1 - bc) / -R.row[1][3];
        g3 = (R.row[0][0] * x2 + R.row[0][1] * x1 + R.row[0][2] * x0 + R.row[0][3] * g1
              + R.row[0][4] * g2) / -R.row[0][5];
    }
}

template <int ORDER>
__device__ __forceinline__ void bcw_bot(const WallRowsD& R, double bc, double x0, double x1,
                                        double& g1, double& g2, double& g3)
{
    if (ORDER == 2) {
        g1 = (-bc) / -R.row[0][1];
        g2 = g3 = 0.0;
    } else {
        g1 = (-bc) / -R.row[2][5];
        g2 = (R.row[1][4] * g1 + R.row[1][5] * x0) / -R.row[1][3];
        g3 = (R.row[0][2] * g2 + R.row[0][3] * g1 + R.row[0][4] * x0 + R.row[0][5] * x1) / -R.row[0][1];
    }
}

template <int ORDER>
__device__ __forceinline__ void bcw_top(const WallRowsD& R, double bc, double x0, double x1,
                                        double& g1, double& g2, double& g3)
{
    if (ORDER == 2) {
        g1 = (-bc) / -R.row[0][1];
        g2 = g3 = 0.0;
    } else {
        g1 = (-bc) / -R.row[2][1];
        g2 = (R.row[1][1] * x0 + R.row[1][2] * g1) / -R.row[1][3];
        g3 = (R.row[0][1] * x1 + R.row[0][2] * x0 + R.row[0][3] * g1 + R.row[0][4] * g2) / -R.row[0][5];
    }
}

// Async 8-byte global -> shared copies whose issue is ordered with the
// thread's other memory accesses ("memory" clobber): the ring slot a copy
// overwrites was read just before.
__device__ __forceinline__ void cp_async8_ordered(double* dst, const double* src)
{
    unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_ordered() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_ordered() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// One column of one field; every thread of the block calls it.
template <int ORDER, bool IS_W, bool SHIFT>
__device__ __forceinline__ void solve_column(const Geo& G, const SolveArgs& A)
{
    const long long col = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = col < G.plane;
    const long long P = G.plane;
    const int n2 = G.n2;
    const int kb = GZ - 1;                          // bottom wall ghost row / face
    const int kt = IS_W ? n2 - GZ - 1 : n2 - GZ;    // top wall ghost row / face
    const int n = A.fac.n, k0 = A.fac.k0;
    double* __restrict__ x = A.x;
    const long long cc = active ? col : 0;
    auto ld = [&](const double* p, int k) { return p[(long long) k * P + cc]; };

    // Old ghost values: cell fields carry apply_bc values already (k_ghosts);
    // face fields recompute apply_bc_w here (k_ghosts stored the massflux4
    // extrapolation there instead).
    double gb0 = 0.0, gb1 = 0.0, gb2 = 0.0, gt0 = 0.0, gt1 = 0.0, gt2 = 0.0;
    if (IS_W) {
        bcw_bot<ORDER>(A.bcb, A.bc_bot, ld(x, kb + 1), ld(x, kb + 2), gb0, gb1, gb2);
        bcw_top<ORDER>(A.bct, A.bc_top, ld(x, kt - 1), ld(x, kt - 2), gt0, gt1, gt2);
    }
    // ghost value d rows beyond the bottom / top wall row
    auto gbot = [&](int d) { return d == 0 ? gb0 : (d == 1 ? gb1 : gb2); };
    auto gtop = [&](int d) { return d == 0 ? gt0 : (d == 1 ? gt1 : gt2); };
    auto old = [&](int k) -> double {
        if (IS_W) {
            if (k <= kb) return gbot(kb - k);
            if (k >= kt) return gtop(k - kt);
        }
        return ld(x, k);
    };

    constexpr int H = ORDER == 2 ? 1 : 3;
    constexpr int W = 2 * H + 1 + 6;   // fused row width (host_band.h fused_rows)
    double win[2 * H + 1];  // old x at rows k-H .. k+H
#pragma unroll
    for (int q = 0; q < 2 * H + 1; q++) win[q] = old(k0 - H + q);

    // Forward sweep: helmholtz1d_operator + RK3 combination + boundary lifting
    // + forward elimination of tridag/heptdag, one fused row per k.  The f, g
    // and next-window values of the coming SOLVE_PF rows are in flight as
    // cp.async copies into this thread's slots of a shared-memory ring (no
    // registers held); none of those rows has been overwritten yet (row i
    // writes only x[k0 + i]).
    extern __shared__ double ring[];   // [SOLVE_PF][3][SOLVE_THREADS]
    auto slot = [&](int i, int fld) { return ring + ((i % SOLVE_PF) * 3 + fld) * SOLVE_THREADS + threadIdx.x; };
    auto fetch = [&](int i) {
        if (i < n) {
            const int k = k0 + i;
            const int kn = min(k + H + 1, n2 - 1);   // window row entering after row i
            cp_async8_ordered(slot(i, 0), A.f + (long long) k * P + cc);
            cp_async8_ordered(slot(i, 1), A.g + (long long) k * P + cc);
            cp_async8_ordered(slot(i, 2), x + (long long) kn * P + cc);
        }
        cp_async_commit_ordered();
    };
    for (int i = 0; i < SOLVE_PF; i++) fetch(i);
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
    const double shift = SHIFT ? *A.gshift : 0.0;
    const double* __restrict__ rows = A.rows;
    for (int i = 0; i < n; i++) {
        const int k = k0 + i;
        const double* r = rows + i * W;
        cp_async_wait_ordered<SOLVE_PF - 1>();   // row i's copies have landed
        const double fk = *slot(i, 0);
        double gk = *slot(i, 1);
        double xn = *slot(i, 2);
        fetch(i + SOLVE_PF);
        if (IS_W && k + H + 1 >= kt) xn = gtop(k + H + 1 - kt);
        if (SHIFT) gk = gk + shift;   // f += mdpdx of the previous substep (chanfast.c:516-519)
        double s = __ldg(r + 2 * H + 3) + __ldg(r + 2 * H + 1) * fk + __ldg(r + 2 * H + 2) * gk;
#pragma unroll
        for (int q = 0; q < 2 * H + 1; q++) s += __ldg(r + q) * win[q];
        s -= __ldg(r + 2 * H + 4) * s1;
        if (ORDER == 4) s -= __ldg(r + 2 * H + 5) * s2 + __ldg(r + 2 * H + 6) * s3;
        s3 = s2; s2 = s1; s1 = s;
        if (active) x[(long long) k * P + col] = s;
#pragma unroll
        for (int q = 0; q < 2 * H; q++) win[q] = win[q + 1];
        win[2 * H] = (i + 1 < n) ? xn : 0.0;
    }
    cp_async_wait_ordered<0>();

    constexpr int PD = 4;   // back-substitution rows loaded ahead
    // Back substitution, reading s PD rows ahead (below) the row being written.
    double ps[PD];
    auto fetch_s = [&](int i, int slot) {
        if (i >= 0) ps[slot] = ld(x, k0 + i);
    };
#pragma unroll
    for (int u = 0; u < PD; u++) fetch_s(n - 1 - u, u);
    double y1 = 0.0, y2 = 0.0, y3 = 0.0;
    double top0 = 0.0, top1 = 0.0, top2 = 0.0, bot0 = 0.0, bot1 = 0.0, bot2 = 0.0;
    const bool stats = A.partial != nullptr;
    const long long wrow = ((long long) blockIdx.x * blockDim.x + threadIdx.x) / 32;
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
                else y = s - __ldg(A.fac.P + i) * y1 - __ldg(A.fac.Q + i) * y2 - __ldg(A.fac.R + i) * y3;
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
        bcw_bot<ORDER>(A.bcb, A.bc_bot, bot0, bot1, b1, b2, b3);
        bcw_top<ORDER>(A.bct, A.bc_top, top0, top1, t1, t2, t3);
    } else {
        bcu_bot<ORDER>(A.bcb, A.bc_bot, bot0, bot1, bot2, b1, b2, b3);
        bcu_top<ORDER>(A.bct, A.bc_top, top0, top1, top2, t1, t2, t3);
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
__global__ void k_row_average(const double* __restrict__ partial, long long nwarps, int n2,
                              double scale, double* __restrict__ avg)
{
    __shared__ double red[256];
    const int k = blockIdx.x;
    double s = 0.0;
    for (long long w = threadIdx.x; w < nwarps; w += blockDim.x) s += partial[w * n2 + k];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) avg[k] = red[0] * scale;
}


// Bulk-mean control of chanfast.c:485-529 (u) / 572-616 (c).
__global__ void k_mass_control(MassArgs A)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double* avg = A.avg;
    const double* dz = A.dz;
    const int g = GZ, n2 = A.n2, nz = A.nz;
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

// The four implicit solves of a substep in one launch (they are independent:
// the mass-flux corrections of u and c are applied lazily, and the control
// kernels that read the u and c row sums run after it).  blockIdx.y selects
// the field: 0 u, 1 v, 2 c (u and c carry the shift of the previous control
// step), 3 w.
template <int ORDER>
__global__ void __launch_bounds__(SOLVE_THREADS, 9) k_solve4(Geo G, SolveBatch B)
{
    switch (blockIdx.y) {
    case 0: solve_column<ORDER, false, true>(G, B.a[0]); break;
    case 1: solve_column<ORDER, false, false>(G, B.a[1]); break;
    case 2: solve_column<ORDER, false, true>(G, B.a[2]); break;
    default: solve_column<ORDER, true, false>(G, B.a[3]); break;
    }
}

void launch_solve4(const Geo& G, const SolveBatch& B, cudaStream_t st)
{
    dim3 grd((unsigned) ((G.plane + SOLVE_THREADS - 1) / SOLVE_THREADS), 4);
    if (G.order == 2) k_solve4<2><<<grd, SOLVE_THREADS, solve_smem_bytes(), st>>>(G, B);
    else k_solve4<4><<<grd, SOLVE_THREADS, solve_smem_bytes(), st>>>(G, B);
}

void launch_mass(const Geo& G, const double* partial, double* avg, const MassArgs& M, cudaStream_t st)
{
    long long nwarps = ((G.plane + SOLVE_THREADS - 1) / SOLVE_THREADS) * (SOLVE_THREADS / 32);
    double scale = 1.0 / ((double) G.nx * (double) G.ny);
    k_row_average<<<G.n2, 256, 0, st>>>(partial, nwarps, G.n2, scale, avg);
    k_mass_control<<<1, 32, 0, st>>>(M);
}

}  // namespace cf
