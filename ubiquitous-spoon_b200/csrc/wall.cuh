// Wall closures of the cell-centred (u, v, c) and face (w) fields: the ghost
// values that apply_bc_{u,w}{2,4} (diffuseu.c:37-104, diffusew.c:37-104)
// write below / above the walls, from the rows of ghost_stencil_{bot,top}
// (WallRowsD: rows k, k-+1, k-+2, coefficients a..g) and the wall value bc.
// x0, x1, x2 are the first interior values next to the wall, nearest first;
// g1, g2, g3 the ghost values, nearest first.
#pragma once

#include "engine.cuh"

namespace cf {

template <int ORDER>
__device__ __forceinline__ void bc_u_bot(const WallRowsD& R, double bc, double x0, double x1, double x2,
                                         double& g1, double& g2, double& g3)
{
    // ghost_fill_bot{2,4} (diffuseu.c:687-693, 899-918): rows k = gz-1, k-1, k-2
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
__device__ __forceinline__ void bc_u_top(const WallRowsD& R, double bc, double x0, double x1, double x2,
                                         double& g1, double& g2, double& g3)
{
    // ghost_fill_top{2,4} (diffuseu.c:696-702, 921-940); x0 = x[kt-1], x1 = x[kt-2], x2 = x[kt-3]
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
__device__ __forceinline__ void bc_w_bot(const WallRowsD& R, double bc, double x0, double x1,
                                         double& g1, double& g2, double& g3)
{
    // diffusew.c:667-680 (order 2), 849-865 (order 4); x0 = w[gz], x1 = w[gz+1]
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
__device__ __forceinline__ void bc_w_top(const WallRowsD& R, double bc, double x0, double x1,
                                         double& g1, double& g2, double& g3)
{
    // x0 = w[kt-1], x1 = w[kt-2] with kt = n2-gz-1 the top wall face
    if (ORDER == 2) {
        g1 = (-bc) / -R.row[0][1];
        g2 = g3 = 0.0;
    } else {
        g1 = (-bc) / -R.row[2][1];
        g2 = (R.row[1][1] * x0 + R.row[1][2] * g1) / -R.row[1][3];
        g3 = (R.row[0][1] * x1 + R.row[0][2] * x0 + R.row[0][3] * g1 + R.row[0][4] * g2) / -R.row[0][5];
    }
}

}  // namespace cf
