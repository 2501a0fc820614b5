// Explicit right-hand side of the RK3 substep and the wall ghost refresh.
//
// k_ghosts:  apply_bc_u{2,4} / apply_bc_w{2,4} of chanfast.c:404-418 for
//            every column, plus the in-place wall rewrite that
//            massflux{x,y,z}4 performs before the advection (advect.c:100-131).
// k_rhs:     fused massflux{x,y,z} + advect{u,v,w} + add_laplacexy_operator
//            + flux_quick + advect_scalar + add_buoyancy
//            (chanfast.c:420-452 / 1344-1376) for every interior point; mass
//            fluxes are formed on the fly and never stored.  Expressions keep
//            the reference's evaluation order; this file is compiled with FMA
//            contraction (its kernels are FP64-throughput bound), so results
//            agree with the reference to rounding.
#include "engine.cuh"
#include "host_band.h"
#include "wall.cuh"
#include "batch.cuh"

#include <type_traits>

namespace cf {

__device__ __forceinline__ int wrapi(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }


// ------------------------------------------------------------------ ghosts

// One thread per column: wall ghost rows of u, v, c (apply_bc_u) and w
// (apply_bc_w, then with EXTRAP the massflux4 extrapolation of
// advect.c:100-131).
template <int ORDER, bool EXTRAP>
__device__ __forceinline__ void ghosts_body(const Geo& G, const GhostArgs& A, uint3 bid)
{
    long long col = (long long) bid.x * blockDim.x + threadIdx.x;
    if (col >= G.plane) return;
    const long long P = G.plane;
    const int n2 = G.n2, kb = GZ - 1, kt = n2 - GZ;
    auto at = [&](double* f, int k) -> double& { return f[(long long) k * P + col]; };
    double* uf[3] = {A.F.u, A.F.v, A.F.c};
    double bcb[3] = {A.bc_u, A.bc_v, A.bc_c_bot};
    double bct[3] = {A.bc_u, A.bc_v, A.bc_c_top};
    for (int q = 0; q < 3; q++) {
        double* f = uf[q];
        double g1, g2, g3;
        bc_u_bot<ORDER>(A.ub, bcb[q], at(f, kb + 1), at(f, kb + 2), at(f, kb + 3), g1, g2, g3);
        at(f, kb) = g1;
        if (ORDER == 4) { at(f, kb - 1) = g2; at(f, kb - 2) = g3; }
        bc_u_top<ORDER>(A.ut, bct[q], at(f, kt - 1), at(f, kt - 2), at(f, kt - 3), g1, g2, g3);
        at(f, kt) = g1;
        if (ORDER == 4) { at(f, kt + 1) = g2; at(f, kt + 2) = g3; }
    }
    double* w = A.F.w;
    const int wt = n2 - GZ - 1;
    double g1, g2, g3;
    bc_w_bot<ORDER>(A.wb, A.bc_w, at(w, kb + 1), at(w, kb + 2), g1, g2, g3);
    double top1, top2, top3;
    bc_w_top<ORDER>(A.wt, A.bc_w, at(w, wt - 1), at(w, wt - 2), top1, top2, top3);
    at(w, kb) = g1;
    at(w, wt) = top1;
    if (ORDER == 4 && EXTRAP) {
        // massflux4 wall extrapolation (advect.c:108-109, 124-125)
        at(w, kb - 1) = 2.0 * g1 - at(w, kb + 1);
        at(w, kb - 2) = 2.0 * g1 - at(w, kb + 2);
        at(w, wt + 1) = 2.0 * top1 - at(w, wt - 1);
        at(w, wt + 2) = 2.0 * top1 - at(w, wt - 2);
    } else if (ORDER == 4) {
        at(w, kb - 1) = g2;
        at(w, kb - 2) = g3;
        at(w, wt + 1) = top2;
        at(w, wt + 2) = top3;
    }
    (void) g2; (void) g3; (void) top2; (void) top3;
}

template <int ORDER, bool EXTRAP>
__global__ void k_ghosts(Geo G, GhostArgs A)
{
    ghosts_body<ORDER, EXTRAP>(G, A, blockIdx);
}

template <int ORDER, bool EXTRAP>
__global__ void k_ghosts_batch(const BatchRec<GhostArgs>* r, int n)
{
    uint3 b;
    const BatchRec<GhostArgs>& R = batch_locate(r, n, b);
    ghosts_body<ORDER, EXTRAP>(R.G, R.A, b);
}

// --------------------------------------------------------------------- RHS
//
// One block owns an 8 (x) by 32 (y) column tile and marches up all interior
// rows.  The 7 k-planes a row needs (k-3..k+3) of u, v, w, c, with a
// periodic halo of 3 rows in x and 4 columns in y, sit in a ring of 8
// shared-memory slots; the next plane streams in with cp.async while the
// current row is computed.  Every
// stencil value is read from shared memory.  Divisions by the grid metrics
// are multiplications by their reciprocals (host tables), so results agree
// with the reference to rounding, not bit for bit.
//
// After a row's four right-hand sides the same thread runs that row of the
// forward sweeps of the four implicit solves (chanfast.c:459-482 with the
// forward half of tridag/heptdag): the old field window x_{k-H..k+H} is in
// the ring, f was just computed, g is read and overwritten by s.  The back
// substitution follows in k_back4 (kernels_solve.cu).
//
// IMPL3D (the fully implicit scheme of channel.c): f has no x-y diffusion
// (channel.c:419-438), and in place of the sweep row each thread forms the
// Helmholtz right-hand side h = x + nuadt (Lxy + Lz) x + gamdt f + zetdt g
// - hbc (channel.c:455-467, 531-543, 560-572, 636-648) of its point, which
// overwrites g; A.nu and A.kappa then carry nuadt and nuadt / prandtl.  The
// spectral solves follow (kernels_pressure.cu).

constexpr int RT_I = 8, RT_J = 32;
constexpr int RT_THREADS = RT_I * RT_J;

// Ring geometry per order: the x-y halo and z reach of the stencils (order
// 4: 3, the fourth-order fluxes and Laplacian; order 2: 2, the QUICK scalar
// fluxes), a ring of the 2 ZH + 1 planes a row reads plus the one in flight
// (8 and 6 slots).  Order 2 thus needs 83 KB of ring instead of 136 KB.
// One block per SM for both: capping order 2 at 128 registers for two blocks
// per SM measured 5-9 % slower (less instruction-level parallelism).
// The y halo is rounded up to an even width (XL) so that, for even ny, every
// haloed row segment starts on a 16-byte boundary in global and shared
// memory: planes stream in as 16-byte copies that bypass L1.
template <int ORDER>
struct RhsTile {
    static constexpr int H = ORDER == 2 ? 2 : 3;
    static constexpr int ZH = H;
    static constexpr int XL = (H + 1) & ~1;                      // y halo columns: 4 / 2
    static constexpr int SLOTS = 2 * ZH + 2;
    static constexpr int PI = RT_I + 2 * H, PJ = RT_J + 2 * XL;  // 14 x 40 / 12 x 36
    static constexpr int PLANE = PI * PJ;
    static constexpr int FIELD = SLOTS * PLANE;                  // one field's ring
    static constexpr int LOADS = (PLANE + RT_THREADS - 1) / RT_THREADS;       // 8-byte copies per thread (odd ny)
    static constexpr int PAIRS = PLANE / 2;
    static constexpr int LOADS2 = (PAIRS + RT_THREADS - 1) / RT_THREADS;      // 16-byte copies per thread (even ny)
    static constexpr int BLOCKS = 1;                             // launch bound: blocks per SM
    // plane kk >= 0 (every plane a row reads lies in 0 .. n2-1): an unsigned
    // remainder, a single AND for the 8-slot ring
    __host__ __device__ static constexpr int slot(int kk) { return (int) ((unsigned) kk % (unsigned) SLOTS); }
};
constexpr double B1h = 0.5 * B1, B2h = 0.5 * B2;   // halved interpolation weights (exact)
// 7-point form of the fourth-order staggered second difference:
// A1 (d+1/2 - d-1/2) + A2 (d+3/2 - d-3/2) = L1 (F1+F-1-2F0) + L2 (F2+F-2-2F0) + L3 (F3+F-3-2F0),
// evaluated as L1 (F1+F-1) + L2 (F2+F-2) + L3 (F3+F-3) - 2 (L1+L2+L3) F0
constexpr double L1 = A1 * A1 - 2.0 * A1 * A2, L2 = 2.0 * A1 * A2, L3 = A2 * A2;

constexpr int RT_FWMAX = 14;   // widest fused forward row (order 4: 13), padded to 16-byte pairs
constexpr int RT_MROW = 12;   // per-row grid metrics: dydz[k-1..k+2], dxdz[k-1..k+2], ivol[k], ivolw[k] (+2 pad)
// ring of haloed planes + two rows of each thread's g values + two rows of
// the four fused coefficient rows + two rows of grid metrics
template <int ORDER>
constexpr size_t rhs_smem_bytes()
{
    return (size_t) (4 * RhsTile<ORDER>::FIELD + 2 * 4 * RT_THREADS + 2 * 4 * RT_FWMAX + 2 * RT_MROW) * sizeof(double);
}

// z fluxes of one advected field (order 4), carried up the column.  With
// F1(k) = MZ(k) (Q(k) + Q(k+1)) / 2 and F3(k) = MZ(k+1) (Q(k) + Q(k+3)) / 2,
// row k needs zph = F1(k), zmh = F1(k-1), zp3 = F3(k), zm3 = F3(k-3)
// (advect.c:466-734), so each row forms one new mass flux MZ(k+1) and two
// fluxes and takes the others from earlier rows; prime() forms the earlier
// ones directly for the first row of a chunk.
struct ZQueue {
    double f1m, f3m[3], mzc, mz1, f1, f3;

    // State as if row k-1 had just been processed (called at row k).
    template <class QF, class MF>
    __device__ __forceinline__ void prime(QF Q, MF MZ)
    {
        mz1 = MZ(0, 0, 0);
        f1 = MZ(0, 0, -1) * 0.5 * (Q(0, 0, -1) + Q(0, 0, 0));
        f3m[1] = MZ(0, 0, -2) * 0.5 * (Q(0, 0, -3) + Q(0, 0, 0));
        f3m[2] = MZ(0, 0, -1) * 0.5 * (Q(0, 0, -2) + Q(0, 0, 1));
        f3 = mz1 * 0.5 * (Q(0, 0, -1) + Q(0, 0, 2));
    }

    template <class QF, class MF>
    __device__ __forceinline__ void advance(QF Q, MF MZ)
    {
        f1m = f1;
        f3m[0] = f3m[1];
        f3m[1] = f3m[2];
        f3m[2] = f3;
        mzc = mz1;
        mz1 = MZ(0, 0, 1);
        const double q0 = Q(0, 0, 0);
        f1 = mzc * 0.5 * (q0 + Q(0, 0, 1));
        f3 = mz1 * 0.5 * (q0 + Q(0, 0, 3));
    }
};

__device__ __forceinline__ void cp_async8(double* dst, const double* src)
{
    unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async16(double* dst, const double* src)   // L2 only
{
    unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <int ORDER, bool IMPL3D>
__device__ __forceinline__ void rhs_body(const Geo& G, const RhsArgs& A, uint3 bid)
{
    extern __shared__ double sm[];
    using T = RhsTile<ORDER>;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * RT_J + tx;
    const int j0 = bid.x * RT_J, i0 = bid.y * RT_I;
    const int nx = G.nx, ny = G.ny, n2 = G.n2;
    const long long plane = (long long) nx * ny;
    const int kb = GZ, ke = GZ + G.nz;   // all interior rows: the forward sweeps run in order

    // This thread's points (even ny: pairs of points) of a haloed plane,
    // the same in every plane: their offsets within a field plane, computed
    // once.  For even ny a pair starts at an even y index (j0 and XL are
    // even), so it never straddles the periodic wrap and its global and
    // shared addresses are 16-byte aligned.
    const bool pairs = (ny & 1) == 0;
    int goff[T::LOADS];
#pragma unroll
    for (int m = 0; m < T::LOADS; m++) {
        const int r = tid + m * RT_THREADS;
        int ii, jj;
        if (pairs) { ii = r / (T::PJ / 2); jj = 2 * (r - ii * (T::PJ / 2)); }
        else { ii = r / T::PJ; jj = r - ii * T::PJ; }
        int gi = (i0 + ii - T::H) % nx; if (gi < 0) gi += nx;
        int gj = (j0 + jj - T::XL) % ny; if (gj < 0) gj += ny;
        goff[m] = gi * ny + gj;
    }
    auto load_plane = [&](int kk) {
        const long long base = (long long) kk * plane;   // same for the whole block
        const double* bu = A.u + base;
        const double* bv = A.v + base;
        const double* bw = A.w + base;
        const double* bc = A.c + base;
        double* ps = sm + T::slot(kk) * T::PLANE;
        if (pairs) {
#pragma unroll
            for (int m = 0; m < T::LOADS2; m++) {
                if (tid + m * RT_THREADS < T::PAIRS) {
                    double* d = ps + 2 * (tid + m * RT_THREADS);
                    const int o = goff[m];
                    cp_async16(d, bu + o);
                    cp_async16(d + T::FIELD, bv + o);
                    cp_async16(d + 2 * T::FIELD, bw + o);
                    cp_async16(d + 3 * T::FIELD, bc + o);
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < T::LOADS; m++) {
                if (tid + m * RT_THREADS < T::PLANE) {
                    double* d = ps + tid + m * RT_THREADS;
                    const int o = goff[m];
                    cp_async8(d, bu + o);
                    cp_async8(d + T::FIELD, bv + o);
                    cp_async8(d + 2 * T::FIELD, bw + o);
                    cp_async8(d + 3 * T::FIELD, bc + o);
                }
            }
        }
        cp_async_commit();
    };
    // g values (per thread) and fused coefficient rows (per block) of row kk,
    // staged one row ahead so the sweeps never wait on global memory
    double* gst = sm + 4 * T::FIELD;              // [2][4][RT_THREADS]
    double* cst = gst + 2 * 4 * RT_THREADS;       // [2][4][RT_FWMAX]
    double* mst = cst + 2 * 4 * RT_FWMAX;         // [2][RT_MROW]
    constexpr int FWR = (ORDER == 2 ? 3 : 7) + 6; // fused row width (host_band.h fused_rows)
    const long long gij = (i0 + ty < nx && j0 + tx < ny) ? (long long) (i0 + ty) * ny + (j0 + tx) : 0;
    auto load_extras = [&](int kk) {
        const long long o = (long long) kk * plane + gij;
        double* d = gst + (kk & 1) * 4 * RT_THREADS + tid;
#pragma unroll
        for (int f = 0; f < 4; f++) cp_async8(d + f * RT_THREADS, A.sw[f].g + o);
        if (tid < 4 * FWR) {
            const int f = tid / FWR, e = tid - f * FWR;
            if (!(f == 2 && kk - GZ >= G.nz - 1))   // the w solve has nz - 1 rows
                cp_async8(cst + ((kk & 1) * 4 + f) * RT_FWMAX + e, A.sw[f].rows + (kk - GZ) * FWR + e);
        }
        const int e = tid - 4 * FWR;   // grid metrics of row kk (rows kk-1 .. kk+2 lie within 0 .. n2-1)
        if (e >= 0 && e < 10) {
            const double* src = e < 4 ? G.dydz + kk - 1 + e : e < 8 ? G.dxdz + kk - 5 + e : e == 8 ? G.ivol + kk : G.ivolw + kk;
            cp_async8(mst + (kk & 1) * RT_MROW + e, src);
        }
    };
    load_extras(kb);
    for (int kk = kb - T::ZH; kk <= kb + T::ZH; kk++) load_plane(kk);
    cp_async_wait_all();
    __syncthreads();

    const int i = i0 + ty, j = j0 + tx;
    const bool out = i < nx && j < ny;
    const double dxdy = G.dxdy, idx = G.idx, idy = G.idy;
    const double idx2 = idx * idx, idy2 = idy * idy;
    const double lapc = -2.0 * (L1 + L2 + L3) * (idx2 + idy2);   // centre weight of the sum-form Laplacian
    const int kb_w = GZ - 1, kt_u = n2 - GZ;   // wall ghost rows of cell-centred fields

    int k = kb;
    auto at = [&](int f, int di, int dj, int dk) -> double {
        return sm[f * T::FIELD + T::slot(k + dk) * T::PLANE + (ty + T::H + di) * T::PJ + (tx + T::XL + dj)];
    };
    auto U = [&](int di, int dj, int dk) { return at(0, di, dj, dk); };
    auto V = [&](int di, int dj, int dk) { return at(1, di, dj, dk); };
    auto W = [&](int di, int dj, int dk) { return at(2, di, dj, dk); };
    auto C = [&](int di, int dj, int dk) { return at(3, di, dj, dk); };

    // grid metrics of the current row, staged one row ahead: dydz[k+dk],
    // dxdz[k+dk] for dk = -1 .. 2, 1 / cell volume, 1 / w-face volume
    auto DYDZ = [&](int dk) { return mst[(k & 1) * RT_MROW + 1 + dk]; };
    auto DXDZ = [&](int dk) { return mst[(k & 1) * RT_MROW + 5 + dk]; };
    // massflux{x,y,z}4 (advect.c:88-283): fourth-order interpolation of the
    // w mass fluxes (the u and v ones are formed per face below)
    auto mx_w = [&](int di, int dj, int dk) {
        return B1 * (dxdy * W(di, dj, dk) + dxdy * W(di + 1, dj, dk)) + B2 * (dxdy * W(di - 1, dj, dk) + dxdy * W(di + 2, dj, dk)); };
    auto my_w = [&](int di, int dj, int dk) {
        return B1 * (dxdy * W(di, dj, dk) + dxdy * W(di, dj + 1, dk)) + B2 * (dxdy * W(di, dj - 1, dk) + dxdy * W(di, dj + 2, dk)); };
    auto mz_w = [&](int di, int dj, int dk) {
        return B1 * (dxdy * W(di, dj, dk) + dxdy * W(di, dj, dk + 1)) + B2 * (dxdy * W(di, dj, dk - 1) + dxdy * W(di, dj, dk + 2)); };
    // massflux{x,y,z}2 (advect.c:6-85)
    auto mx_u2 = [&](int di, int dj, int dk) { double d = DYDZ(dk); return 0.5 * (d * U(di, dj, dk) + d * U(di + 1, dj, dk)); };
    auto mx_v2 = [&](int di, int dj, int dk) { double d = DXDZ(dk); return 0.5 * (d * V(di, dj, dk) + d * V(di + 1, dj, dk)); };
    auto mx_w2 = [&](int di, int dj, int dk) { return 0.5 * (dxdy * W(di, dj, dk) + dxdy * W(di + 1, dj, dk)); };
    auto my_u2 = [&](int di, int dj, int dk) { double d = DYDZ(dk); return 0.5 * (d * U(di, dj, dk) + d * U(di, dj + 1, dk)); };
    auto my_v2 = [&](int di, int dj, int dk) { double d = DXDZ(dk); return 0.5 * (d * V(di, dj, dk) + d * V(di, dj + 1, dk)); };
    auto my_w2 = [&](int di, int dj, int dk) { return 0.5 * (dxdy * W(di, dj, dk) + dxdy * W(di, dj + 1, dk)); };
    auto mz_u2 = [&](int di, int dj, int dk) { return 0.5 * (DYDZ(dk) * U(di, dj, dk) + DYDZ(dk + 1) * U(di, dj, dk + 1)); };
    auto mz_v2 = [&](int di, int dj, int dk) { return 0.5 * (DXDZ(dk) * V(di, dj, dk) + DXDZ(dk + 1) * V(di, dj, dk + 1)); };
    auto mz_w2 = [&](int di, int dj, int dk) { return 0.5 * (dxdy * W(di, dj, dk) + dxdy * W(di, dj, dk + 1)); };

    const double qk = -0.125;   // QUICK coefficient (scalar.c:79-162)
    // The face value between cells c0 and c1 takes the upwind curvature
    // x - 2y + z of (c1, c0, c-1) for m > 0, else of (c2, c1, c0): the
    // curvature centred on the upwind cell.  Each point forms the curvatures
    // of cells i-1, i, i+1 once per direction and both faces pick theirs.
    auto curv = [](double x, double y, double z) { return x - 2.0 * y + z; };
    auto quick = [&](double m, double c0, double c1, double kup, double kdn) {
        double cph = 0.5 * (c0 + c1);
        cph += qk * (m > 0.0 ? kup : kdn);
        return m * cph;
    };
    // add_buoyancy is skipped when every betg is zero (adding exact zeros)
    const bool buoyancy = A.betg_x != 0.0 || A.betg_y != 0.0 || A.betg_z != 0.0;

    // z fluxes carried up the column: the queues and the scalar flux
    // through the bottom face, primed for the first row.
    ZQueue zq_u{}, zq_v{}, zq_w{};
    if (ORDER == 4) {
        zq_u.prime(U, mx_w);
        zq_v.prime(V, my_w);
        zq_w.prime(W, mz_w);
    }
    // z curvature of cell k (carried from row to row) and the scalar flux
    // through the bottom face of the first row
    double kz = curv(C(0, 0, 1), C(0, 0, 0), C(0, 0, -1));
    double fzp_prev = quick(dxdy * W(0, 0, -1), C(0, 0, -1), C(0, 0, 0), curv(C(0, 0, 0), C(0, 0, -1), C(0, 0, -2)), kz);

    // Forward-sweep state: s of rows k-1, k-2, k-3 per field, the lazily
    // applied shifts of g (u: mdpdx, c: dcdt of the previous control step),
    // and the ghost values of the old w below / above its wall faces
    // (apply_bc_w; the ring holds the massflux4 extrapolation there instead).
    constexpr int H = ORDER == 2 ? 1 : 3;
    double su1 = 0.0, su2 = 0.0, su3 = 0.0, sv1 = 0.0, sv2 = 0.0, sv3 = 0.0;
    double sw1 = 0.0, sw2 = 0.0, sw3 = 0.0, sc1 = 0.0, sc2 = 0.0, sc3 = 0.0;
    const double shift_u = A.sw[0].gshift ? *A.sw[0].gshift : 0.0;
    const double shift_c = A.sw[3].gshift ? *A.sw[3].gshift : 0.0;
    double gb0, gb1, gb2, gt0 = 0.0, gt1 = 0.0, gt2 = 0.0;
    bc_w_bot<ORDER>(A.wbot, A.wbc_bot, W(0, 0, 0), W(0, 0, 1), gb0, gb1, gb2);
    (void) gb0;
    auto sweep = [&](int f, auto X, double fk, double gk, double lk, double& s1, double& s2, double& s3) {
        // staged coefficient row, read as 16-byte pairs (same value for the
        // whole block: broadcast loads)
        const double2* r2 = reinterpret_cast<const double2*>(cst + ((k & 1) * 4 + f) * RT_FWMAX);
        double r[RT_FWMAX];
#pragma unroll
        for (int q = 0; q < (FWR + 1) / 2; q++) {
            const double2 t = r2[q];
            r[2 * q] = t.x;
            r[2 * q + 1] = t.y;
        }
        double sk = r[2 * H + 3] + r[2 * H + 1] * fk + r[2 * H + 2] * gk;
#pragma unroll
        for (int q = 0; q < 2 * H + 1; q++) sk += r[q] * X(q - H);
        if (IMPL3D) return sk + lk;   // h of this point (channel_rows: no elimination)
        if (ORDER == 4) sk -= r[2 * H + 5] * s2 + r[2 * H + 6] * s3;
        sk -= r[2 * H + 4] * s1;   // the previous row's s enters last
        s3 = s2; s2 = s1; s1 = sk;
        return sk;
    };

    // One row.  WALL: rows within two of a wall, whose z fluxes use the wall
    // closures (and the top row has no w point), and the row whose w-solve
    // window reaches above the top face; other rows take a branch-free path.
    auto row = [&](auto wall_tag) {
        constexpr bool WALL = decltype(wall_tag)::value;
        const double ivol = mst[(k & 1) * RT_MROW + 8], ivolw = mst[(k & 1) * RT_MROW + 9];
        const bool do_w = !WALL || k < n2 - GZ - 1;
        const long long ijk = (long long) k * plane + gij;
        const double* gk = gst + (k & 1) * 4 * RT_THREADS + tid;   // g of this row (staged)
        const double gu = gk[0] + shift_u, gv = gk[RT_THREADS];
        const double gw = gk[2 * RT_THREADS], gc = gk[3 * RT_THREADS] + shift_c;
        double fu, fv, fw = 0.0, fc;
        double lu, lv, lw = 0.0, lc;   // x-y diffusion terms

        if (ORDER == 2) {
            auto adv_cell = [&](auto Q, auto MX, auto MY, auto MZ) {   // advectu2 / advectv2 (advect.c:286-417)
                double q0 = Q(0, 0, 0);
                double xph = MX(0, 0, 0) * 0.5 * (q0 + Q(1, 0, 0));
                double yph = MY(0, 0, 0) * 0.5 * (q0 + Q(0, 1, 0));
                double zph = MZ(0, 0, 0) * 0.5 * (q0 + Q(0, 0, 1));
                double xmh = MX(-1, 0, 0) * 0.5 * (q0 + Q(-1, 0, 0));
                double ymh = MY(0, -1, 0) * 0.5 * (q0 + Q(0, -1, 0));
                double zmh = MZ(0, 0, -1) * 0.5 * (q0 + Q(0, 0, -1));
                if (WALL) {
                    if (k == n2 - GZ - 1) zph = MZ(0, 0, 0) * (0.5 * (Q(0, 0, kt_u - 1 - k) + Q(0, 0, kt_u - k)));
                    if (k == GZ) zmh = MZ(0, 0, -1) * (0.5 * (Q(0, 0, kb_w - k) + Q(0, 0, kb_w + 1 - k)));
                }
                return -((xph - xmh) + (yph - ymh) + (zph - zmh)) * ivol;
            };
            fu = adv_cell(U, mx_u2, mx_v2, mx_w2);
            fv = adv_cell(V, my_u2, my_v2, my_w2);
            if (do_w) {   // advectw2 (advect.c:420-463)
                double q0 = W(0, 0, 0);
                double xph = mz_u2(0, 0, 0) * 0.5 * (q0 + W(1, 0, 0));
                double yph = mz_v2(0, 0, 0) * 0.5 * (q0 + W(0, 1, 0));
                double zph = mz_w2(0, 0, 0) * 0.5 * (q0 + W(0, 0, 1));
                double xmh = mz_u2(-1, 0, 0) * 0.5 * (q0 + W(-1, 0, 0));
                double ymh = mz_v2(0, -1, 0) * 0.5 * (q0 + W(0, -1, 0));
                double zmh = mz_w2(0, 0, -1) * 0.5 * (q0 + W(0, 0, -1));
                fw = -((xph - xmh) + (yph - ymh) + (zph - zmh)) * ivolw;
            }
            // add_laplacexy_operator_{u,w}2 (diffuseu.c:286-313, diffusew.c:290-317)
            auto lap2 = [&](auto F, double nu) {
                double q0 = F(0, 0, 0);
                return nu * (((F(1, 0, 0) - q0) * idx - (q0 - F(-1, 0, 0)) * idx) * idx
                             + ((F(0, 1, 0) - q0) * idy - (q0 - F(0, -1, 0)) * idy) * idy);
            };
            lu = lap2(U, A.nu);
            lv = lap2(V, A.nu);
            if (do_w) lw = lap2(W, A.nu);
            lc = lap2(C, A.kappa);
        } else {
            // advectu4 / advectv4 / advectw4 (advect.c:466-734).  Within one
            // cell every x-direction mass flux carries the same metric
            // (dydz[k] for the u-flux, dxdz[k] for the v-flux), so it is
            // factored out of the x and y flux sums; the halved interpolation
            // weights B1h, B2h absorb the 0.5 of the face value (an exact
            // scaling).  Mathematically the reference's sums; they round
            // differently.  The wall-adjacent z fluxes use the fourth-order
            // wall value qbot / qtop; the z fluxes come from the per-field
            // queue (zph / zp3 of this row, zmh / zm3 = zph of row k-1 / zp3
            // of row k-3).
            auto ix = [&](auto F, int di, int dj) {   // x interpolation to the face i+di+1/2
                return B1h * (F(di, dj, 0) + F(di + 1, dj, 0)) + B2h * (F(di - 1, dj, 0) + F(di + 2, dj, 0));
            };
            auto iy = [&](auto F, int di, int dj) {   // y interpolation to the face j+dj+1/2
                return B1h * (F(di, dj, 0) + F(di, dj + 1, 0)) + B2h * (F(di, dj - 1, 0) + F(di, dj + 2, 0));
            };
            auto xflux = [&](auto Q, auto M, double q0) {   // A1 (xph - xmh) + A2 (xp3 - xm3), metric factored out
                return A1 * (M(0, 0) * (q0 + Q(1, 0, 0)) - M(-1, 0) * (q0 + Q(-1, 0, 0)))
                     + A2 * (M(1, 0) * (q0 + Q(3, 0, 0)) - M(-2, 0) * (q0 + Q(-3, 0, 0)));
            };
            auto yflux = [&](auto Q, auto M, double q0) {
                return A1 * (M(0, 0) * (q0 + Q(0, 1, 0)) - M(0, -1) * (q0 + Q(0, -1, 0)))
                     + A2 * (M(0, 1) * (q0 + Q(0, 3, 0)) - M(0, -2) * (q0 + Q(0, -3, 0)));
            };
            auto zsum = [&](auto Q, auto MZ, double zph, double zmh, double zp3, double zm3) {
                if (WALL) {
                    double qbot = 0.5 * A2 * (Q(0, 0, kb_w - 1 - k) + Q(0, 0, kb_w + 2 - k))
                                + 0.5 * (A1 + 2.0 * A2) * (Q(0, 0, kb_w - k) + Q(0, 0, kb_w + 1 - k));
                    double qtop = 0.5 * A2 * (Q(0, 0, kt_u - 2 - k) + Q(0, 0, kt_u + 1 - k))
                                + 0.5 * (A1 + 2.0 * A2) * (Q(0, 0, kt_u - 1 - k) + Q(0, 0, kt_u - k));
                    if (k == n2 - GZ - 1) {
                        zph = MZ(0, 0, 0) * qtop;
                        zp3 = -MZ(0, 0, -1) * 0.5 * (Q(0, 0, -2) + Q(0, 0, 1)) + 2.0 * MZ(0, 0, 0) * qtop;
                    }
                    if (k == n2 - GZ - 2) zp3 = MZ(0, 0, 1) * qtop;
                    if (k == GZ) {
                        zmh = MZ(0, 0, -1) * qbot;
                        zm3 = -MZ(0, 0, 0) * 0.5 * (Q(0, 0, 2) + Q(0, 0, -1)) + 2.0 * MZ(0, 0, -1) * qbot;
                    }
                    if (k == GZ + 1) zm3 = MZ(0, 0, -2) * qbot;
                }
                return A1 * (zph - zmh) + A2 * (zp3 - zm3);
            };
            const double mdy = DYDZ(0), mdx = DXDZ(0);
            zq_u.advance(U, mx_w);
            zq_v.advance(V, my_w);
            {
                const double q0 = U(0, 0, 0);
                auto mu = [&](int di, int dj) { return ix(U, di, dj); };
                auto mv = [&](int di, int dj) { return ix(V, di, dj); };
                fu = -((mdy * xflux(U, mu, q0) + mdx * yflux(U, mv, q0))
                       + zsum(U, mx_w, zq_u.f1, zq_u.f1m, zq_u.f3, zq_u.f3m[0])) * ivol;
            }
            {
                const double q0 = V(0, 0, 0);
                auto mu = [&](int di, int dj) { return iy(U, di, dj); };
                auto mv = [&](int di, int dj) { return iy(V, di, dj); };
                fv = -((mdy * xflux(V, mu, q0) + mdx * yflux(V, mv, q0))
                       + zsum(V, my_w, zq_v.f1, zq_v.f1m, zq_v.f3, zq_v.f3m[0])) * ivol;
            }
            if (do_w) {
                zq_w.advance(W, mz_w);
                // z interpolation of the u / v mass fluxes to the w face: the
                // metric differs per plane, folded into four row constants
                const double cu0 = B1h * DYDZ(0), cu1 = B1h * DYDZ(1), cum = B2h * DYDZ(-1), cu2 = B2h * DYDZ(2);
                const double cv0 = B1h * DXDZ(0), cv1 = B1h * DXDZ(1), cvm = B2h * DXDZ(-1), cv2 = B2h * DXDZ(2);
                auto mu = [&](int di, int dj) {
                    return (cu0 * U(di, dj, 0) + cu1 * U(di, dj, 1)) + (cum * U(di, dj, -1) + cu2 * U(di, dj, 2));
                };
                auto mv = [&](int di, int dj) {
                    return (cv0 * V(di, dj, 0) + cv1 * V(di, dj, 1)) + (cvm * V(di, dj, -1) + cv2 * V(di, dj, 2));
                };
                const double q0 = W(0, 0, 0);
                fw = -((xflux(W, mu, q0) + yflux(W, mv, q0))
                       + (A1 * (zq_w.f1 - zq_w.f1m) + A2 * (zq_w.f3 - zq_w.f3m[0]))) * ivolw;
            }
            // add_laplacexy_operator_{u,w}4 (diffuseu.c:316-359, diffusew.c:320-363):
            // A1 (d+1/2 - d-1/2) + A2 (d+3/2 - d-3/2) of the staggered first
            // differences is the 7-point stencil L1, L2, L3, here in sum form:
            // the symmetric pairs, then the centre weight -2 (L1 + L2 + L3)
            // folded with both directions (lapc).  Mathematically the same;
            // it rounds differently (the centre term no longer cancels
            // exactly, an error of a few ulps of |u| (1/dx^2 + 1/dy^2) nu).
            auto lap4 = [&](auto F, double nu) {
                const double lx = L3 * (F(3, 0, 0) + F(-3, 0, 0)) + L2 * (F(2, 0, 0) + F(-2, 0, 0))
                                + L1 * (F(1, 0, 0) + F(-1, 0, 0));
                const double ly = L3 * (F(0, 3, 0) + F(0, -3, 0)) + L2 * (F(0, 2, 0) + F(0, -2, 0))
                                + L1 * (F(0, 1, 0) + F(0, -1, 0));
                return nu * ((lx * idx2 + ly * idy2) + lapc * F(0, 0, 0));
            };
            lu = lap4(U, A.nu);
            lv = lap4(V, A.nu);
            if (do_w) lw = lap4(W, A.nu);
            lc = lap4(C, A.kappa);
        }
        if (!IMPL3D) {
            fu += lu;
            fv += lv;
            fw += lw;
        }
        fc = IMPL3D ? 0.0 : lc;

        {   // flux_quick + advect_scalar (scalar.c:79-162), order independent
            const double c0 = C(0, 0, 0);
            const double kx0 = curv(C(1, 0, 0), c0, C(-1, 0, 0)), ky0 = curv(C(0, 1, 0), c0, C(0, -1, 0));
            const double kxm = curv(c0, C(-1, 0, 0), C(-2, 0, 0)), kxp = curv(C(2, 0, 0), C(1, 0, 0), c0);
            const double kym = curv(c0, C(0, -1, 0), C(0, -2, 0)), kyp = curv(C(0, 2, 0), C(0, 1, 0), c0);
            const double kzp = curv(C(0, 0, 2), C(0, 0, 1), c0);
            double fxp = quick(DYDZ(0) * U(0, 0, 0), c0, C(1, 0, 0), kx0, kxp);
            double fxm = quick(DYDZ(0) * U(-1, 0, 0), C(-1, 0, 0), c0, kxm, kx0);
            double fyp = quick(DXDZ(0) * V(0, 0, 0), c0, C(0, 1, 0), ky0, kyp);
            double fym = quick(DXDZ(0) * V(0, -1, 0), C(0, -1, 0), c0, kym, ky0);
            double fzp = quick(dxdy * W(0, 0, 0), c0, C(0, 0, 1), kz, kzp);
            kz = kzp;
            double fzm = fzp_prev;   // the top-face flux of row k-1
            fzp_prev = fzp;
            fc = -((fxp - fxm) + (fyp - fym) + (fzp - fzm)) * ivol + fc;
            // add_buoyancy{2,4} (scalar.c:6-76)
            if (!buoyancy) {
            } else if (ORDER == 2) {
                fu += 0.5 * (c0 + C(1, 0, 0)) * A.betg_x;
                fv += 0.5 * (c0 + C(0, 1, 0)) * A.betg_y;
                if (do_w) fw += 0.5 * (c0 + C(0, 0, 1)) * A.betg_z;
            } else {
                double cphx = B1 * (c0 + C(1, 0, 0)) + B2 * (C(-1, 0, 0) + C(2, 0, 0));
                double cphy = B1 * (c0 + C(0, 1, 0)) + B2 * (C(0, -1, 0) + C(0, 2, 0));
                fu += cphx * A.betg_x;
                fv += cphy * A.betg_y;
                if (do_w) fw += (B1 * (c0 + C(0, 0, 1)) + B2 * (C(0, 0, -1) + C(0, 0, 2))) * A.betg_z;
            }
        }

        // forward sweeps of the implicit solves, rows k0 = GZ .. (u, v, c: nz
        // rows; w: nz - 1 faces)
        if (WALL && k >= n2 - GZ - 3)   // old w above the top face (apply_bc_w)
            bc_w_top<ORDER>(A.wtop, A.wbc_top, W(0, 0, n2 - GZ - 2 - k), W(0, 0, n2 - GZ - 3 - k), gt0, gt1, gt2);
        auto XW = [&](int dk) -> double {
            if (WALL) {
                const int kk = k + dk;
                if (kk < GZ - 1) return kk == GZ - 2 ? gb1 : gb2;
                if (kk > n2 - GZ - 1) return kk == n2 - GZ ? gt1 : gt2;
            }
            return W(0, 0, dk);
        };
        (void) gt0;
        const double s_u = sweep(0, [&](int dk) { return U(0, 0, dk); }, fu, gu, lu, su1, su2, su3);
        const double s_v = sweep(1, [&](int dk) { return V(0, 0, dk); }, fv, gv, lv, sv1, sv2, sv3);
        const double s_w = do_w ? sweep(2, XW, fw, gw, lw, sw1, sw2, sw3) : 0.0;
        const double s_c = sweep(3, [&](int dk) { return C(0, 0, dk); }, fc, gc, lc, sc1, sc2, sc3);
        if (out) {
            A.fu[ijk] = fu;
            A.fv[ijk] = fv;
            A.fc[ijk] = fc;
            A.sw[0].g[ijk] = s_u;
            A.sw[1].g[ijk] = s_v;
            A.sw[3].g[ijk] = s_c;
            if (do_w) {
                A.fw[ijk] = fw;
                A.sw[2].g[ijk] = s_w;
            }
        }
    };

    for (; k < ke; k++) {
        if (k + 1 < ke) load_extras(k + 1);
        if (k + T::ZH + 1 <= ke + T::ZH - 1) load_plane(k + T::ZH + 1);   // the last row reads ke - 1 + ZH
        else cp_async_commit();
        if (k <= GZ + 1 || k >= n2 - GZ - 3) row(std::true_type{});
        else row(std::false_type{});
        cp_async_wait_all();
        __syncthreads();
    }
}

template <int ORDER, bool IMPL3D>
__global__ void __launch_bounds__(RT_THREADS, RhsTile<ORDER>::BLOCKS) k_rhs(Geo G, RhsArgs A)
{
    rhs_body<ORDER, IMPL3D>(G, A, blockIdx);
}

template <int ORDER>
__global__ void __launch_bounds__(RT_THREADS, RhsTile<ORDER>::BLOCKS) k_rhs_batch(const BatchRec<RhsArgs>* r, int n)
{
    uint3 b;
    const BatchRec<RhsArgs>& R = batch_locate(r, n, b);
    rhs_body<ORDER, false>(R.G, R.A, b);
}

// ------------------------------------------------------------- launchers

constexpr int GHOST_THREADS = 256;

dim3 grid_ghosts(const Geo& G) { return dim3((unsigned) ((G.plane + GHOST_THREADS - 1) / GHOST_THREADS)); }

void launch_ghosts(const Geo& G, const GhostArgs& A, cudaStream_t st, bool extrap)
{
    const int th = GHOST_THREADS;
    const unsigned nb = grid_ghosts(G).x;
    if (extrap) {
        if (G.order == 2) k_ghosts<2, true><<<(unsigned) nb, th, 0, st>>>(G, A);
        else k_ghosts<4, true><<<(unsigned) nb, th, 0, st>>>(G, A);
    } else {
        if (G.order == 2) k_ghosts<2, false><<<(unsigned) nb, th, 0, st>>>(G, A);
        else k_ghosts<4, false><<<(unsigned) nb, th, 0, st>>>(G, A);
    }
}

dim3 grid_rhs(const Geo& G) { return dim3((G.ny + RT_J - 1) / RT_J, (G.nx + RT_I - 1) / RT_I, 1); }

void launch_ghosts_batch(const BatchLaunch& L, int order, cudaStream_t st)
{
    auto r = static_cast<const BatchRec<GhostArgs>*>(L.recs);
    if (order == 2) k_ghosts_batch<2, true><<<L.blocks, GHOST_THREADS, 0, st>>>(r, L.n);
    else k_ghosts_batch<4, true><<<L.blocks, GHOST_THREADS, 0, st>>>(r, L.n);
}

void launch_rhs_batch(const BatchLaunch& L, int order, cudaStream_t st)
{
    auto r = static_cast<const BatchRec<RhsArgs>*>(L.recs);
    dim3 blk(RT_J, RT_I, 1);
    if (order == 2) k_rhs_batch<2><<<L.blocks, blk, rhs_smem_bytes<2>(), st>>>(r, L.n);
    else k_rhs_batch<4><<<L.blocks, blk, rhs_smem_bytes<4>(), st>>>(r, L.n);
}

void launch_rhs(const Geo& G, const RhsArgs& A, bool implicit3d, cudaStream_t st)
{
    dim3 blk(RT_J, RT_I, 1);
    dim3 grd = grid_rhs(G);
    if (implicit3d) {
        if (G.order == 2) k_rhs<2, true><<<grd, blk, rhs_smem_bytes<2>(), st>>>(G, A);
        else k_rhs<4, true><<<grd, blk, rhs_smem_bytes<4>(), st>>>(G, A);
    } else {
        if (G.order == 2) k_rhs<2, false><<<grd, blk, rhs_smem_bytes<2>(), st>>>(G, A);
        else k_rhs<4, false><<<grd, blk, rhs_smem_bytes<4>(), st>>>(G, A);
    }
}

cudaError_t rhs_set_smem_limits()
{
    const int v2 = (int) rhs_smem_bytes<2>(), v4 = (int) rhs_smem_bytes<4>();
    cudaError_t e = cudaFuncSetAttribute(k_rhs<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, v2);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_rhs<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, v4);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_rhs<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, v2);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_rhs<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, v4);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_rhs_batch<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, v2);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_rhs_batch<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, v4);
    return e;
}

}  // namespace cf
