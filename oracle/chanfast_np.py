"""CPU restatement of the reference RK3 substep in numpy -- TEST INFRASTRUCTURE.

This module is the oracle: a from-scratch restatement of the algorithm of the
reference channel-flow code (nasilemakbox/ubiquitous-spoon) for the hot path,
the `chanfast2` / `chanfast4` RK3 substep (chanfast.c:395-656 / 1319-1580).
It is used only by tests/, by ``__graft_entry__.smoke()`` and by bench.py's
CPU-baseline leg, as the checker.  The product never imports it.

Layout is the reference's: every field is a flat C-order array of shape
(n0, n1, n2) = (nx + 2 gx, ny + 2 gy, nz + 2 gz), wall-normal index k fastest
(d3tensor.c:9-42).  Each function below restates the reference function named
in its docstring over the same index ranges with the same floating-point
expression order, so that on x86-64 (no FMA contraction) results agree with
the compiled reference bit for bit except where an FFT or a summation order
differs.  The FFT is numpy's pocketfft, normalised like fft.c:161-208.

Parity of this restatement against the compiled reference (oracle/_ref, built
by oracle/Makefile from the unmodified reference sources) is checked in
tests/test_oracle_vs_ref.py.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# fourth.c:3-6
A1 = 1.125 / 1.0
A2 = -0.125 / 3.0
B1 = 1.125 / 2.0
B2 = -0.125 / 2.0
# rk3.c:3-6
RK3_ALP = (29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0)
RK3_BET = (37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0)
RK3_GAM = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
RK3_ZET = (0.0, -17.0 / 60.0, -5.0 / 12.0)
FILL_VALUE = -999.0  # check.h:13

DIRICHU, NEUMANU = 0, 1  # diffuseu.h:1-2
DIRICHW = 20  # diffusew.h:1
DIRICHP, NEUMANP = 10, 11  # pressure.c:23-24


@dataclass
class Params:
    """Arguments of chanfast2/chanfast4 (chanfast.h:1-21) that the substep uses."""

    order: int
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    dt: float
    nu: float
    prandtl: float = 1.0
    dpdx: float = 0.0
    want_uvolavg: float = 1.0
    uvolavgmode: int = 1
    want_cvolavg: float = 0.0
    cvolavgmode: int = 1
    setuframe: float = 0.0
    setvframe: float = 0.0
    betg_x: float = 0.0
    betg_y: float = 0.0
    betg_z: float = 0.0
    ngx: int = 3
    ngy: int = 3
    ngz: int = 3


class Grid:
    """Grid metrics as chanfast.c:140-192 (dx, dy, stretched dz with mirrored ghosts)."""

    def __init__(self, p: Params):
        self.p = p
        self.n0 = p.nx + 2 * p.ngx
        self.n1 = p.ny + 2 * p.ngy
        self.n2 = p.nz + 2 * p.ngz
        self.dx = p.lx / float(p.nx)
        self.dy = p.ly / float(p.ny)
        dz = np.zeros(self.n2)
        for iz in range(p.nz):
            dz[iz + p.ngz] = p.lz * 0.5 * (math.cos(math.pi * float(iz) / float(p.nz))
                                           - math.cos(math.pi * float(iz + 1) / float(p.nz)))
        ghost_even_z_1d(dz, p.nz, p.ngz)
        self.dz = dz

    @property
    def shape(self):
        return (self.n0, self.n1, self.n2)


def ghost_even_z_1d(u, nz, g):
    """ghost_even_z for one column (ghost.c:31-54)."""
    n2 = nz + 2 * g
    for k in range(g):
        u[k] = u[2 * g - k - 1]
    for k in range(n2 - g, n2):
        u[k] = u[2 * (n2 - g) - k - 1]


def ghostz_periodic(u, g: Grid):
    """Periodic x then y halo of width ngx/ngy (ghostz.c:107-149, one rank)."""
    gx, gy = g.p.ngx, g.p.ngy
    n0, n1 = g.n0, g.n1
    u[0:gx] = u[n0 - 2 * gx:n0 - gx]
    u[n0 - gx:n0] = u[gx:2 * gx]
    u[:, 0:gy] = u[:, n1 - 2 * gy:n1 - gy]
    u[:, n1 - gy:n1] = u[:, gy:2 * gy]


# ---------------------------------------------------------------------------
# Column closures: band rows of the ghost points, their elimination, and their
# recovery.  Band arrays a..g, r are (n2,) coefficient rows; r may be
# (ncol, n2).  One Closure instance per module (diffuseu / diffusew /
# pressure), mirroring the module-static scratch of each .c file.
# ---------------------------------------------------------------------------


class Band:
    def __init__(self, n2, ncol, width):
        self.width = width
        names = "abc" if width == 3 else "abcdefg"
        for nm in names:
            setattr(self, nm, np.zeros(n2))
        self.r = np.zeros((ncol, n2))
        self.x = np.zeros((ncol, n2))


def u_ghost_stencil_bot2(B, dz, k, bc, bctype):
    """diffuseu.c:617-636 (pressure.c:446-465 with NEUMANP/DIRICHP)."""
    dzp1h = 0.5 * (dz[k + 1] + dz[k])
    if bctype in (NEUMANU, NEUMANP):
        B.a[k] = 0.0
        B.b[k] = -1.0 / dzp1h
        B.c[k] = +1.0 / dzp1h
    else:
        B.a[k] = 0.0
        B.b[k] = 0.5
        B.c[k] = 0.5
    B.r[:, k] = bc


def u_ghost_stencil_top2(B, dz, k, bc, bctype):
    """diffuseu.c:639-658 (pressure.c:468-487)."""
    dzm1h = 0.5 * (dz[k - 1] + dz[k])
    if bctype in (NEUMANU, NEUMANP):
        B.a[k] = -1.0 / dzm1h
        B.b[k] = +1.0 / dzm1h
        B.c[k] = 0.0
    else:
        B.a[k] = 0.5
        B.b[k] = 0.5
        B.c[k] = 0.0
    B.r[:, k] = bc


def u_ghost_reduce_bot2(B, k):
    """diffuseu.c:661-671 (pressure.c:490-500)."""
    kp1 = k + 1
    fac = B.a[kp1] / B.b[k]
    B.a[kp1] -= B.b[k] * fac
    B.b[kp1] -= B.c[k] * fac
    B.r[:, kp1] -= B.r[:, k] * fac


def u_ghost_reduce_top2(B, k):
    """diffuseu.c:674-684 (pressure.c:503-513)."""
    km1 = k - 1
    fac = B.c[km1] / B.b[k]
    B.c[km1] -= B.b[k] * fac
    B.b[km1] -= B.a[k] * fac
    B.r[:, km1] -= B.r[:, k] * fac


def u_ghost_fill_bot2(B, k):
    """diffuseu.c:687-693."""
    B.x[:, k] = (B.c[k] * B.x[:, k + 1] - B.r[:, k]) / -B.b[k]


def u_ghost_fill_top2(B, k):
    """diffuseu.c:696-702."""
    B.x[:, k] = (B.a[k] * B.x[:, k - 1] - B.r[:, k]) / -B.b[k]


def u_ghost_stencil_bot4(B, dz, k, bc, bctype):
    """diffuseu.c:705-753 (pressure.c:534-582 with NEUMANP/DIRICHP)."""
    km2, km1 = k - 2, k - 1
    dzp3h = 0.5 * (dz[k + 2] + dz[k + 1])
    dzp1h = 0.5 * (dz[k + 1] + dz[k])
    dzm1h = 0.5 * (dz[k - 1] + dz[k])
    B.a[k] = 0.0
    B.b[k] = - A2 / dzm1h
    B.c[k] = - A1 / dzm1h - 2.0 * - A2 / dzp1h
    B.d[k] = + A1 / dzm1h - 2.0 * - A1 / dzp1h - A2 / dzp3h
    B.e[k] = + A2 / dzm1h - 2.0 * + A1 / dzp1h - A1 / dzp3h
    B.f[k] = - 2.0 * + A2 / dzp1h + A1 / dzp3h
    B.g[k] = + A2 / dzp3h
    B.r[:, k] = 0.0
    B.a[km1] = B.b[km1] = B.c[km1] = 0.0
    if bctype in (NEUMANU, NEUMANP):
        B.d[km1] = - A2 / dzp1h
        B.e[km1] = - A1 / dzp1h
        B.f[km1] = + A1 / dzp1h
        B.g[km1] = + A2 / dzp1h
    else:
        B.d[km1] = 0.5 * A2
        B.e[km1] = 0.5 * (A1 + 2.0 * A2)
        B.f[km1] = 0.5 * (A1 + 2.0 * A2)
        B.g[km1] = 0.5 * A2
    B.r[:, km1] = bc
    B.a[km2] = B.b[km2] = B.c[km2] = B.d[km2] = B.e[km2] = 0.0
    B.f[km2] = -1.0
    B.g[km2] = +1.0
    B.r[:, km2] = 0.0


def u_ghost_stencil_top4(B, dz, k, bc, bctype):
    """diffuseu.c:756-804 (pressure.c:585-633)."""
    kp2, kp1 = k + 2, k + 1
    dzp1h = 0.5 * (dz[k + 1] + dz[k])
    dzm1h = 0.5 * (dz[k - 1] + dz[k])
    dzm3h = 0.5 * (dz[k - 2] + dz[k - 1])
    B.a[k] = - A2 / dzm3h
    B.b[k] = - A1 / dzm3h - 2.0 * - A2 / dzm1h
    B.c[k] = + A1 / dzm3h - 2.0 * - A1 / dzm1h - A2 / dzp1h
    B.d[k] = + A2 / dzm3h - 2.0 * + A1 / dzm1h - A1 / dzp1h
    B.e[k] = - 2.0 * + A2 / dzm1h + A1 / dzp1h
    B.f[k] = + A2 / dzp1h
    B.g[k] = 0.0
    B.r[:, k] = 0.0
    if bctype in (NEUMANU, NEUMANP):
        B.a[kp1] = - A2 / dzm1h
        B.b[kp1] = - A1 / dzm1h
        B.c[kp1] = + A1 / dzm1h
        B.d[kp1] = + A2 / dzm1h
    else:
        B.a[kp1] = 0.5 * A2
        B.b[kp1] = 0.5 * (A1 + 2.0 * A2)
        B.c[kp1] = 0.5 * (A1 + 2.0 * A2)
        B.d[kp1] = 0.5 * A2
    B.e[kp1] = B.f[kp1] = B.g[kp1] = 0.0
    B.r[:, kp1] = bc
    B.a[kp2] = -1.0
    B.b[kp2] = +1.0
    B.c[kp2] = B.d[kp2] = B.e[kp2] = B.f[kp2] = B.g[kp2] = 0.0
    B.r[:, kp2] = 0.0


def u_ghost_reduce_bot4(B, k):
    """diffuseu.c:807-850 (pressure.c:636-679)."""
    a, b, c, d, e, f, g, r = B.a, B.b, B.c, B.d, B.e, B.f, B.g, B.r
    km2, km1, kp1, kp2, kp3 = k - 2, k - 1, k + 1, k + 2, k + 3
    fac = a[kp1] / b[k]
    a[kp1] -= b[k] * fac; b[kp1] -= c[k] * fac; c[kp1] -= d[k] * fac
    d[kp1] -= e[k] * fac; e[kp1] -= f[k] * fac; f[kp1] -= g[k] * fac
    fac = b[kp1] / d[km1]
    b[kp1] -= d[km1] * fac; c[kp1] -= e[km1] * fac; d[kp1] -= f[km1] * fac
    e[kp1] -= g[km1] * fac; r[:, kp1] -= r[:, km1] * fac
    fac = c[kp1] / f[km2]
    c[kp1] -= f[km2] * fac; d[kp1] -= g[km2] * fac
    fac = a[kp2] / d[km1]
    a[kp2] -= d[km1] * fac; b[kp2] -= e[km1] * fac; c[kp2] -= f[km1] * fac
    d[kp2] -= g[km1] * fac; r[:, kp2] -= r[:, km1] * fac
    fac = b[kp2] / f[km2]
    b[kp2] -= f[km2] * fac; c[kp2] -= g[km2] * fac
    fac = a[kp3] / f[km2]
    a[kp3] -= f[km2] * fac; b[kp3] -= g[km2] * fac


def u_ghost_reduce_top4(B, k):
    """diffuseu.c:853-896 (pressure.c:682-725)."""
    a, b, c, d, e, f, g, r = B.a, B.b, B.c, B.d, B.e, B.f, B.g, B.r
    km3, km2, km1, kp1, kp2 = k - 3, k - 2, k - 1, k + 1, k + 2
    fac = g[km1] / f[k]
    g[km1] -= f[k] * fac; f[km1] -= e[k] * fac; e[km1] -= d[k] * fac
    d[km1] -= c[k] * fac; c[km1] -= b[k] * fac; b[km1] -= a[k] * fac
    fac = f[km1] / d[kp1]
    f[km1] -= d[kp1] * fac; e[km1] -= c[kp1] * fac; d[km1] -= b[kp1] * fac
    c[km1] -= a[kp1] * fac; r[:, km1] -= r[:, kp1] * fac
    fac = e[km1] / b[kp2]
    e[km1] -= b[kp2] * fac; d[km1] -= a[kp2] * fac
    fac = g[km2] / d[kp1]
    g[km2] -= d[kp1] * fac; f[km2] -= c[kp1] * fac; e[km2] -= b[kp1] * fac
    d[km2] -= a[kp1] * fac; r[:, km2] -= r[:, kp1] * fac
    fac = f[km2] / b[kp2]
    f[km2] -= b[kp2] * fac; e[km2] -= a[kp2] * fac
    fac = g[km3] / b[kp2]
    g[km3] -= b[kp2] * fac; f[km3] -= a[kp2] * fac


def u_ghost_fill_bot4(B, k):
    """diffuseu.c:899-918 (pressure.c:728-747)."""
    x, r = B.x, B.r
    km2, km1, kp1, kp2, kp3 = k - 2, k - 1, k + 1, k + 2, k + 3
    x[:, k] = (B.g[km2] * x[:, kp1]) / -B.f[km2]
    x[:, km1] = (B.e[km1] * x[:, k] + B.f[km1] * x[:, kp1] + B.g[km1] * x[:, kp2]
                 - r[:, km1]) / -B.d[km1]
    x[:, km2] = (B.c[k] * x[:, km1] + B.d[k] * x[:, k] + B.e[k] * x[:, kp1]
                 + B.f[k] * x[:, kp2] + B.g[k] * x[:, kp3]) / -B.b[k]


def u_ghost_fill_top4(B, k):
    """diffuseu.c:921-940 (pressure.c:750-769)."""
    x, r = B.x, B.r
    km3, km2, km1, kp1, kp2 = k - 3, k - 2, k - 1, k + 1, k + 2
    x[:, k] = (B.a[kp2] * x[:, km1]) / -B.b[kp2]
    x[:, kp1] = (B.a[kp1] * x[:, km2] + B.b[kp1] * x[:, km1] + B.c[kp1] * x[:, k]
                 - r[:, kp1]) / -B.d[kp1]
    x[:, kp2] = (B.a[k] * x[:, km3] + B.b[k] * x[:, km2] + B.c[k] * x[:, km1]
                 + B.d[k] * x[:, k] + B.e[k] * x[:, kp1]) / -B.f[k]


def w_ghost_stencil2(B, k, bc):
    """diffusew.c:617-640 (bottom and top are identical: x[k] = bc)."""
    B.a[k] = 0.0
    B.b[k] = 1.0
    B.c[k] = 0.0
    B.r[:, k] = bc


def w_ghost_reduce_bot2(B, k):
    """diffusew.c:643-652."""
    kp1 = k + 1
    fac = B.a[kp1] / B.b[k]
    B.a[kp1] -= B.b[k] * fac
    B.r[:, kp1] -= B.r[:, k] * fac


def w_ghost_reduce_top2(B, k):
    """diffusew.c:655-664."""
    km1 = k - 1
    fac = B.c[km1] / B.b[k]
    B.c[km1] -= B.b[k] * fac
    B.r[:, km1] -= B.r[:, k] * fac


def w_ghost_fill2(B, k):
    """diffusew.c:667-680."""
    B.x[:, k] = (- B.r[:, k]) / -B.b[k]


def w_ghost_stencil_bot4(B, dz, k, bc):
    """diffusew.c:683-722."""
    km2, km1 = k - 2, k - 1
    dzp0, dzp1 = dz[k], dz[k + 1]
    B.a[k] = 0.0
    B.b[k] = - A2 / dzp0
    B.c[k] = - A1 / dzp0 + A2 / dzp1
    B.d[k] = + A1 / dzp0 + A1 / dzp1
    B.e[k] = + A2 / dzp0 - A1 / dzp1
    B.f[k] = - A2 / dzp1
    B.g[k] = 0.0
    B.r[:, k] = 0.0
    B.a[km1] = B.b[km1] = B.c[km1] = 0.0
    B.d[km1] = -1.0
    B.e[km1] = +2.0
    B.f[km1] = -1.0
    B.g[km1] = 0.0
    B.r[:, km1] = 0.0
    B.a[km2] = B.b[km2] = B.c[km2] = B.d[km2] = B.e[km2] = 0.0
    B.f[km2] = 1.0
    B.g[km2] = 0.0
    B.r[:, km2] = bc


def w_ghost_stencil_top4(B, dz, k, bc):
    """diffusew.c:725-764."""
    kp2, kp1 = k + 2, k + 1
    dzp0, dzp1 = dz[k], dz[k + 1]
    B.a[k] = 0.0
    B.b[k] = - A2 / dzp0
    B.c[k] = - A1 / dzp0 + A2 / dzp1
    B.d[k] = + A1 / dzp0 + A1 / dzp1
    B.e[k] = + A2 / dzp0 - A1 / dzp1
    B.f[k] = - A2 / dzp1
    B.g[k] = 0.0
    B.r[:, k] = 0.0
    B.a[kp1] = 0.0
    B.b[kp1] = -1.0
    B.c[kp1] = +2.0
    B.d[kp1] = -1.0
    B.e[kp1] = B.f[kp1] = B.g[kp1] = 0.0
    B.r[:, kp1] = 0.0
    B.a[kp2] = 0.0
    B.b[kp2] = 1.0
    B.c[kp2] = B.d[kp2] = B.e[kp2] = B.f[kp2] = B.g[kp2] = 0.0
    B.r[:, kp2] = bc


def w_ghost_reduce_bot4(B, k):
    """diffusew.c:767-805."""
    a, b, c, d, e, f, r = B.a, B.b, B.c, B.d, B.e, B.f, B.r
    km2, km1, kp1, kp2, kp3 = k - 2, k - 1, k + 1, k + 2, k + 3
    fac = a[kp1] / b[k]
    a[kp1] -= b[k] * fac; b[kp1] -= c[k] * fac; c[kp1] -= d[k] * fac
    d[kp1] -= e[k] * fac; e[kp1] -= f[k] * fac
    fac = b[kp1] / d[km1]
    b[kp1] -= d[km1] * fac; c[kp1] -= e[km1] * fac; d[kp1] -= f[km1] * fac
    fac = c[kp1] / f[km2]
    c[kp1] -= f[km2] * fac; r[:, kp1] -= r[:, km2] * fac
    fac = a[kp2] / d[km1]
    a[kp2] -= d[km1] * fac; b[kp2] -= e[km1] * fac; c[kp2] -= f[km1] * fac
    fac = b[kp2] / f[km2]
    b[kp2] -= f[km2] * fac; r[:, kp2] -= r[:, km2] * fac
    fac = a[kp3] / f[km2]
    a[kp3] -= f[km2] * fac; r[:, kp3] -= r[:, km2] * fac


def w_ghost_reduce_top4(B, k):
    """diffusew.c:808-846."""
    b, c, d, e, f, g, r = B.b, B.c, B.d, B.e, B.f, B.g, B.r
    km3, km2, km1, kp1, kp2 = k - 3, k - 2, k - 1, k + 1, k + 2
    fac = g[km1] / f[k]
    g[km1] -= f[k] * fac; f[km1] -= e[k] * fac; e[km1] -= d[k] * fac
    d[km1] -= c[k] * fac; c[km1] -= b[k] * fac
    fac = f[km1] / d[kp1]
    f[km1] -= d[kp1] * fac; e[km1] -= c[kp1] * fac; d[km1] -= b[kp1] * fac
    fac = e[km1] / b[kp2]
    e[km1] -= b[kp2] * fac; r[:, km1] -= r[:, kp2] * fac
    fac = g[km2] / d[kp1]
    g[km2] -= d[kp1] * fac; f[km2] -= c[kp1] * fac; e[km2] -= b[kp1] * fac
    fac = f[km2] / b[kp2]
    f[km2] -= b[kp2] * fac; r[:, km2] -= r[:, kp2] * fac
    fac = g[km3] / b[kp2]
    g[km3] -= b[kp2] * fac; r[:, km3] -= r[:, kp2] * fac


def w_ghost_fill_bot4(B, k):
    """diffusew.c:849-865."""
    x, r = B.x, B.r
    km2, km1, kp1, kp2 = k - 2, k - 1, k + 1, k + 2
    x[:, k] = (- r[:, km2]) / -B.f[km2]
    x[:, km1] = (B.e[km1] * x[:, k] + B.f[km1] * x[:, kp1]) / -B.d[km1]
    x[:, km2] = (B.c[k] * x[:, km1] + B.d[k] * x[:, k] + B.e[k] * x[:, kp1]
                 + B.f[k] * x[:, kp2]) / -B.b[k]


def w_ghost_fill_top4(B, k):
    """diffusew.c:868-884."""
    x, r = B.x, B.r
    km2, km1, kp1, kp2 = k - 2, k - 1, k + 1, k + 2
    x[:, k] = (- r[:, kp2]) / -B.b[kp2]
    x[:, kp1] = (B.b[kp1] * x[:, km1] + B.c[kp1] * x[:, k]) / -B.d[kp1]
    x[:, kp2] = (B.b[k] * x[:, km2] + B.c[k] * x[:, km1] + B.d[k] * x[:, k]
                 + B.e[k] * x[:, kp1]) / -B.f[k]


# ---------------------------------------------------------------------------
# Banded solvers, vectorised over columns (rows of r / x).
# ---------------------------------------------------------------------------


def tridag(a, b, c, r, n):
    """Thomas algorithm without pivoting (tridag.c:4-26).  a, b, c: (n,) or
    (ncol, n); r: (ncol, n).  Returns u (ncol, n)."""
    a, b, c = (np.broadcast_to(v, r.shape) for v in (a, b, c))
    u = np.empty_like(r)
    gam = np.empty_like(r)
    bet = b[:, 0].copy()
    if np.any(bet == 0.0):
        raise ZeroDivisionError("tridag: zero pivot")
    u[:, 0] = r[:, 0] / bet
    for j in range(1, n):
        gam[:, j] = c[:, j - 1] / bet
        bet = b[:, j] - a[:, j] * gam[:, j]
        if np.any(bet == 0.0):
            raise ZeroDivisionError("tridag: zero pivot")
        u[:, j] = (r[:, j] - a[:, j] * u[:, j - 1]) / bet
    for j in range(n - 2, -1, -1):
        u[:, j] -= gam[:, j + 1] * u[:, j + 1]
    return u


def heptdag(a, b, c, d, e, f, g, h, n):
    """Banded LU without pivoting, 3 sub- and 3 super-diagonals
    (heptdag.c:5-61).  Coefficients (n,) or (ncol, n); h (ncol, n)."""
    a, b, c, d, e, f, g = (np.broadcast_to(v, h.shape) for v in (a, b, c, d, e, f, g))
    p = np.empty_like(h); q = np.empty_like(h); r = np.empty_like(h); s = np.empty_like(h)
    den = d[:, 0]
    p[:, 0] = e[:, 0] / den; q[:, 0] = f[:, 0] / den; r[:, 0] = g[:, 0] / den; s[:, 0] = h[:, 0] / den
    den = d[:, 1] - c[:, 1] * p[:, 0]
    p[:, 1] = (e[:, 1] - c[:, 1] * q[:, 0]) / den
    q[:, 1] = (f[:, 1] - c[:, 1] * r[:, 0]) / den
    r[:, 1] = (g[:, 1]) / den
    s[:, 1] = (h[:, 1] - c[:, 1] * s[:, 0]) / den
    bet = c[:, 2] - b[:, 2] * p[:, 0]
    den = d[:, 2] - b[:, 2] * q[:, 0] - bet * p[:, 1]
    p[:, 2] = (e[:, 2] - b[:, 2] * r[:, 0] - bet * q[:, 1]) / den
    q[:, 2] = (f[:, 2] - bet * r[:, 1]) / den
    r[:, 2] = (g[:, 2]) / den
    s[:, 2] = (h[:, 2] - b[:, 2] * s[:, 0] - bet * s[:, 1]) / den
    for i in range(3, n):
        alp = b[:, i] - a[:, i] * p[:, i - 3]
        bet = c[:, i] - a[:, i] * q[:, i - 3] - alp * p[:, i - 2]
        den = d[:, i] - a[:, i] * r[:, i - 3] - alp * q[:, i - 2] - bet * p[:, i - 1]
        p[:, i] = (e[:, i] - alp * r[:, i - 2] - bet * q[:, i - 1]) / den
        q[:, i] = (f[:, i] - bet * r[:, i - 1]) / den
        r[:, i] = (g[:, i]) / den
        s[:, i] = (h[:, i] - a[:, i] * s[:, i - 3] - alp * s[:, i - 2] - bet * s[:, i - 1]) / den
    x = s
    x[:, n - 2] = s[:, n - 2] - p[:, n - 2] * s[:, n - 1]
    x[:, n - 3] = s[:, n - 3] - p[:, n - 3] * s[:, n - 2] - q[:, n - 3] * s[:, n - 1]
    for i in range(n - 4, -1, -1):
        x[:, i] = s[:, i] - p[:, i] * x[:, i + 1] - q[:, i] * x[:, i + 2] - r[:, i] * x[:, i + 3]
    return x


# ---------------------------------------------------------------------------
# Per-column boundary conditions, 1-D Helmholtz operator and solve.
# ---------------------------------------------------------------------------


def apply_bc_u(u, g: Grid, bc_bot, bc_top, order):
    """apply_bc_u2 / apply_bc_u4 (diffuseu.c:37-69 / 72-104): set the z ghost
    cells of a cell-centred field from the wall value bc (Dirichlet)."""
    n2, gz = g.n2, g.p.ngz
    cols = u.reshape(-1, n2)
    B = Band(n2, cols.shape[0], 3 if order == 2 else 7)
    B.x[:] = cols
    if order == 2:
        u_ghost_stencil_bot2(B, g.dz, gz - 1, bc_bot, DIRICHU)
        u_ghost_stencil_top2(B, g.dz, n2 - gz, bc_top, DIRICHU)
        u_ghost_fill_bot2(B, gz - 1)
        u_ghost_fill_top2(B, n2 - gz)
    else:
        u_ghost_stencil_bot4(B, g.dz, gz - 1, bc_bot, DIRICHU)
        u_ghost_stencil_top4(B, g.dz, n2 - gz, bc_top, DIRICHU)
        u_ghost_fill_bot4(B, gz - 1)
        u_ghost_fill_top4(B, n2 - gz)
    cols[:] = B.x


def apply_bc_w(w, g: Grid, bc_bot, bc_top, order):
    """apply_bc_w2 / apply_bc_w4 (diffusew.c:37-69 / 72-104): w on z faces."""
    n2, gz = g.n2, g.p.ngz
    cols = w.reshape(-1, n2)
    B = Band(n2, cols.shape[0], 3 if order == 2 else 7)
    B.x[:] = cols
    if order == 2:
        w_ghost_stencil2(B, gz - 1, bc_bot)
        w_ghost_stencil2(B, n2 - gz - 1, bc_top)
        w_ghost_fill2(B, gz - 1)
        w_ghost_fill2(B, n2 - gz - 1)
    else:
        w_ghost_stencil_bot4(B, g.dz, gz - 1, bc_bot)
        w_ghost_stencil_top4(B, g.dz, n2 - gz - 1, bc_top)
        w_ghost_fill_bot4(B, gz - 1)
        w_ghost_fill_top4(B, n2 - gz - 1)
    cols[:] = B.x


def helmholtz1d_operator_u(u, h, g: Grid, nudt, order):
    """h = u + nudt d2u/dz2 on cell centres, interior k only
    (diffuseu.c:107-132 / 135-170)."""
    dz, gz, n2 = g.dz, g.p.ngz, g.n2
    k0, k1 = gz, n2 - gz
    K = slice(k0, k1)
    U = lambda o: u[:, :, k0 + o:k1 + o]
    if order == 2:
        dzp1h = 0.5 * (dz[k0 + 1:k1 + 1] + dz[K])
        dzm1h = 0.5 * (dz[k0 - 1:k1 - 1] + dz[K])
        h[:, :, K] = U(0) + nudt * (((U(1) - U(0)) / dzp1h - (U(0) - U(-1)) / dzm1h) / dz[K])
    else:
        wp3h = A1 * (U(2) - U(1)) + A2 * (U(3) - U(0))
        wp1h = A1 * (U(1) - U(0)) + A2 * (U(2) - U(-1))
        wm1h = A1 * (U(0) - U(-1)) + A2 * (U(1) - U(-2))
        wm3h = A1 * (U(-1) - U(-2)) + A2 * (U(0) - U(-3))
        dzp3h = 0.5 * (dz[k0 + 2:k1 + 2] + dz[k0 + 1:k1 + 1])
        dzp1h = 0.5 * (dz[k0 + 1:k1 + 1] + dz[K])
        dzm1h = 0.5 * (dz[k0 - 1:k1 - 1] + dz[K])
        dzm3h = 0.5 * (dz[k0 - 2:k1 - 2] + dz[k0 - 1:k1 - 1])
        h[:, :, K] = U(0) + nudt * ((A1 * (wp1h / dzp1h - wm1h / dzm1h)
                                     + A2 * (wp3h / dzp3h - wm3h / dzm3h)) / dz[K])


def helmholtz1d_operator_w(w, h, g: Grid, nudt, order):
    """Same for w on z faces (diffusew.c:107-133 / 136-172)."""
    dz, gz, n2 = g.dz, g.p.ngz, g.n2
    k0, k1 = gz, n2 - gz - 1
    K = slice(k0, k1)
    W = lambda o: w[:, :, k0 + o:k1 + o]
    dzp1h = 0.5 * (dz[k0 + 1:k1 + 1] + dz[K])
    if order == 2:
        dzp1 = dz[k0 + 1:k1 + 1]
        dzm0 = dz[K]
        h[:, :, K] = W(0) + nudt * (((W(1) - W(0)) / dzp1 - (W(0) - W(-1)) / dzm0) / dzp1h)
    else:
        wp3h = A1 * (W(2) - W(1)) + A2 * (W(3) - W(0))
        wp1h = A1 * (W(1) - W(0)) + A2 * (W(2) - W(-1))
        wm1h = A1 * (W(0) - W(-1)) + A2 * (W(1) - W(-2))
        wm3h = A1 * (W(-1) - W(-2)) + A2 * (W(0) - W(-3))
        dzp2 = dz[k0 + 2:k1 + 2]
        dzp1 = dz[k0 + 1:k1 + 1]
        dzm0 = dz[K]
        dzm1 = dz[k0 - 1:k1 - 1]
        h[:, :, K] = W(0) + nudt * ((A1 * (wp1h / dzp1 - wm1h / dzm0)
                                     + A2 * (wp3h / dzp2 - wm3h / dzm1)) / dzp1h)


def _band_u(g: Grid, nudt, order, B):
    """Interior band rows of solve_helmholtz1d_u{2,4} (diffuseu.c:190-201 /
    239-268) and of pressure_poisson{2,4} (pressure.c:317-330 / 391-418).
    B.dvol is the cell volume per k; B.diag_fix(k, s) finishes the main
    diagonal from the partial sum s in the reference's evaluation order
    (+ dvol for the Helmholtz solve, - lamx..., - lamy... for the Poisson
    solve, where `nudt` is the pressure coefficient)."""
    dz, gz, n2 = g.dz, g.p.ngz, g.n2
    for k in range(gz, n2 - gz):
        dzp1h = 0.5 * (dz[k + 1] + dz[k])
        dzm1h = 0.5 * (dz[k - 1] + dz[k])
        if order == 2:
            B.a[..., k] = + B.dvol[k] * nudt / (dzm1h * dz[k])
            B.c[..., k] = + B.dvol[k] * nudt / (dzp1h * dz[k])
            B.b[..., k] = B.diag_fix(k, - B.dvol[k] * nudt / (dzm1h * dz[k])
                                     - B.dvol[k] * nudt / (dzp1h * dz[k]))
        else:
            dzp3h = 0.5 * (dz[k + 2] + dz[k + 1])
            dzm3h = 0.5 * (dz[k - 2] + dz[k - 1])
            dv = B.dvol[k]
            B.a[..., k] = + A2 * A2 * dv * nudt / (dzm3h * dz[k])
            B.g[..., k] = + A2 * A2 * dv * nudt / (dzp3h * dz[k])
            B.b[..., k] = (+ A1 * A2 * dv * nudt / (dzm1h * dz[k])
                           + A1 * A2 * dv * nudt / (dzm3h * dz[k]))
            B.f[..., k] = (+ A1 * A2 * dv * nudt / (dzp1h * dz[k])
                           + A1 * A2 * dv * nudt / (dzp3h * dz[k]))
            B.c[..., k] = (- A1 * A2 * dv * nudt / (dzp1h * dz[k])
                           - A1 * A2 * dv * nudt / (dzm3h * dz[k])
                           + A1 * A1 * dv * nudt / (dzm1h * dz[k]))
            B.e[..., k] = (- A1 * A2 * dv * nudt / (dzm1h * dz[k])
                           - A1 * A2 * dv * nudt / (dzp3h * dz[k])
                           + A1 * A1 * dv * nudt / (dzp1h * dz[k]))
            B.d[..., k] = B.diag_fix(k, - A2 * A2 * dv * nudt / (dzm3h * dz[k])
                                     - A2 * A2 * dv * nudt / (dzp3h * dz[k])
                                     - A1 * A1 * dv * nudt / (dzm1h * dz[k])
                                     - A1 * A1 * dv * nudt / (dzp1h * dz[k]))


def solve_helmholtz1d_u(u, h, g: Grid, nudt, order):
    """u = (I + nudt d2/dz2)^-1 h per column with homogeneous Dirichlet
    closures, ghosts recovered (diffuseu.c:173-219 / 222-283).  Every column of
    the padded array is solved, as in the reference."""
    n2, gz, nz = g.n2, g.p.ngz, g.p.nz
    hc = h.reshape(-1, n2)
    B = Band(n2, hc.shape[0], 3 if order == 2 else 7)
    B.dvol = g.dz
    B.diag_fix = lambda k, s: s + g.dz[k]
    _band_u(g, nudt, order, B)
    K = slice(gz, n2 - gz)
    B.r[:, K] = hc[:, K] * g.dz[K]
    if order == 2:
        u_ghost_stencil_bot2(B, g.dz, gz - 1, 0.0, DIRICHU)
        u_ghost_stencil_top2(B, g.dz, n2 - gz, 0.0, DIRICHU)
        u_ghost_reduce_bot2(B, gz - 1)
        u_ghost_reduce_top2(B, n2 - gz)
        B.x[:, K] = tridag(B.a[K], B.b[K], B.c[K], B.r[:, K], nz)
        u_ghost_fill_bot2(B, gz - 1)
        u_ghost_fill_top2(B, n2 - gz)
    else:
        u_ghost_stencil_bot4(B, g.dz, gz - 1, 0.0, DIRICHU)
        u_ghost_stencil_top4(B, g.dz, n2 - gz, 0.0, DIRICHU)
        u_ghost_reduce_bot4(B, gz - 1)
        u_ghost_reduce_top4(B, n2 - gz)
        B.x[:, K] = heptdag(B.a[K], B.b[K], B.c[K], B.d[K], B.e[K], B.f[K], B.g[K], B.r[:, K], nz)
        u_ghost_fill_bot4(B, gz - 1)
        u_ghost_fill_top4(B, n2 - gz)
    u.reshape(-1, n2)[:] = B.x


def solve_helmholtz1d_w(w, h, g: Grid, nudt, order):
    """Same for w: nz-1 unknowns on interior faces (diffusew.c:175-222 /
    225-287)."""
    n2, gz, nz = g.n2, g.p.ngz, g.p.nz
    dz = g.dz
    hc = h.reshape(-1, n2)
    B = Band(n2, hc.shape[0], 3 if order == 2 else 7)
    for k in range(gz, n2 - gz - 1):
        dzp1 = dz[k + 1]
        dzm0 = dz[k]
        dzp1h = 0.5 * (dz[k + 1] + dz[k])
        dvol = dzp1h
        if order == 2:
            B.a[k] = + dvol * nudt / (dzm0 * dzp1h)
            B.c[k] = + dvol * nudt / (dzp1 * dzp1h)
            B.b[k] = - dvol * nudt / (dzm0 * dzp1h) - dvol * nudt / (dzp1 * dzp1h) + dvol
        else:
            dzp2 = dz[k + 2]
            dzm1 = dz[k - 1]
            B.a[k] = + A2 * A2 * dvol * nudt / (dzm1 * dzp1h)
            B.g[k] = + A2 * A2 * dvol * nudt / (dzp2 * dzp1h)
            B.b[k] = + A1 * A2 * dvol * nudt / (dzm0 * dzp1h) + A1 * A2 * dvol * nudt / (dzm1 * dzp1h)
            B.f[k] = + A1 * A2 * dvol * nudt / (dzp1 * dzp1h) + A1 * A2 * dvol * nudt / (dzp2 * dzp1h)
            B.c[k] = (- A1 * A2 * dvol * nudt / (dzp1 * dzp1h) - A1 * A2 * dvol * nudt / (dzm1 * dzp1h)
                      + A1 * A1 * dvol * nudt / (dzm0 * dzp1h))
            B.e[k] = (- A1 * A2 * dvol * nudt / (dzm0 * dzp1h) - A1 * A2 * dvol * nudt / (dzp2 * dzp1h)
                      + A1 * A1 * dvol * nudt / (dzp1 * dzp1h))
            B.d[k] = (- A2 * A2 * dvol * nudt / (dzm1 * dzp1h) - A2 * A2 * dvol * nudt / (dzp2 * dzp1h)
                      - A1 * A1 * dvol * nudt / (dzm0 * dzp1h) - A1 * A1 * dvol * nudt / (dzp1 * dzp1h)
                      + dvol)
        B.r[:, k] = hc[:, k] * dvol
    K = slice(gz, n2 - gz - 1)
    if order == 2:
        w_ghost_stencil2(B, gz - 1, 0.0)
        w_ghost_stencil2(B, n2 - gz - 1, 0.0)
        w_ghost_reduce_bot2(B, gz - 1)
        w_ghost_reduce_top2(B, n2 - gz - 1)
        B.x[:, K] = tridag(B.a[K], B.b[K], B.c[K], B.r[:, K], nz - 1)
        w_ghost_fill2(B, gz - 1)
        w_ghost_fill2(B, n2 - gz - 1)
    else:
        w_ghost_stencil_bot4(B, dz, gz - 1, 0.0)
        w_ghost_stencil_top4(B, dz, n2 - gz - 1, 0.0)
        w_ghost_reduce_bot4(B, gz - 1)
        w_ghost_reduce_top4(B, n2 - gz - 1)
        B.x[:, K] = heptdag(B.a[K], B.b[K], B.c[K], B.d[K], B.e[K], B.f[K], B.g[K], B.r[:, K], nz - 1)
        w_ghost_fill_bot4(B, gz - 1)
        w_ghost_fill_top4(B, n2 - gz - 1)
    w.reshape(-1, n2)[:] = B.x


def add_laplacexy_operator(u, h, g: Grid, nu, order, is_w):
    """h += nu (d2/dx2 + d2/dy2) u on interior k (diffuseu.c:286-313 /
    316-359; diffusew.c:290-317 / 320-363)."""
    gz, n2, n0, n1 = g.p.ngz, g.n2, g.n0, g.n1
    dx, dy = g.dx, g.dy
    k1 = n2 - gz - (1 if is_w else 0)
    m = 1 if order == 2 else 3
    I, J, K = slice(m, n0 - m), slice(m, n1 - m), slice(gz, k1)
    U = lambda di, dj: u[m + di:n0 - m + di, m + dj:n1 - m + dj, gz:k1]
    if order == 2:
        h[I, J, K] += nu * (((U(1, 0) - U(0, 0)) / dx - (U(0, 0) - U(-1, 0)) / dx) / dx
                            + ((U(0, 1) - U(0, 0)) / dy - (U(0, 0) - U(0, -1)) / dy) / dy)
    else:
        up3h = A1 * (U(2, 0) - U(1, 0)) + A2 * (U(3, 0) - U(0, 0))
        up1h = A1 * (U(1, 0) - U(0, 0)) + A2 * (U(2, 0) - U(-1, 0))
        um1h = A1 * (U(0, 0) - U(-1, 0)) + A2 * (U(1, 0) - U(-2, 0))
        um3h = A1 * (U(-1, 0) - U(-2, 0)) + A2 * (U(0, 0) - U(-3, 0))
        vp3h = A1 * (U(0, 2) - U(0, 1)) + A2 * (U(0, 3) - U(0, 0))
        vp1h = A1 * (U(0, 1) - U(0, 0)) + A2 * (U(0, 2) - U(0, -1))
        vm1h = A1 * (U(0, 0) - U(0, -1)) + A2 * (U(0, 1) - U(0, -2))
        vm3h = A1 * (U(0, -1) - U(0, -2)) + A2 * (U(0, 0) - U(0, -3))
        h[I, J, K] += nu * ((A1 * (up1h / dx - um1h / dx) + A2 * (up3h / dx - um3h / dx)) / dx
                            + (A1 * (vp1h / dy - vm1h / dy) + A2 * (vp3h / dy - vm3h / dy)) / dy)


# ---------------------------------------------------------------------------
# Advection, scalar transport, buoyancy.
# ---------------------------------------------------------------------------


def _view(a, i0, i1, j0, j1, k0, k1):
    return lambda di, dj, dk: a[i0 + di:i1 + di, j0 + dj:j1 + dj, k0 + dk:k1 + dk]


def massflux(u, v, w, g: Grid, order, axis):
    """massflux{x,y,z}{2,4} (advect.c:6-283).  Returns (mu, mv, mw); order 4
    first rewrites the wall ghosts of u, v, w in place (advect.c:100-131)."""
    n0, n1, n2, gz = g.n0, g.n1, g.n2, g.p.ngz
    dx, dy, dz = g.dx, g.dy, g.dz
    mu = np.full(g.shape, np.nan); mv = np.full(g.shape, np.nan); mw = np.full(g.shape, np.nan)
    if order == 2:
        i0, i1, j0, j1, k0, k1 = 0, n0 - 1, 0, n1 - 1, 0, n2 - 1
        U, V, W = (_view(a, i0, i1, j0, j1, k0, k1) for a in (u, v, w))
        sh = {0: (1, 0, 0), 1: (0, 1, 0), 2: (0, 0, 1)}[axis]
        dzm0 = dz[k0:k1]
        dzp1 = dz[k0 + 1:k1 + 1] if axis == 2 else dzm0
        S = (slice(i0, i1), slice(j0, j1), slice(k0, k1))
        mu[S] = 0.5 * (dy * dzm0 * U(0, 0, 0) + dy * dzp1 * U(*sh))
        mv[S] = 0.5 * (dx * dzm0 * V(0, 0, 0) + dx * dzp1 * V(*sh))
        mw[S] = 0.5 * (dx * dy * W(0, 0, 0) + dx * dy * W(*sh))
        return mu, mv, mw
    k = gz - 1
    u[:, :, k] = u[:, :, k + 1]
    v[:, :, k] = v[:, :, k + 1]
    w[:, :, k - 1] = 2.0 * w[:, :, k] - w[:, :, k + 1]
    w[:, :, k - 2] = 2.0 * w[:, :, k] - w[:, :, k + 2]
    k = n2 - gz
    u[:, :, k] = u[:, :, k - 1]
    v[:, :, k] = v[:, :, k - 1]
    k = n2 - gz - 1
    w[:, :, k + 1] = 2.0 * w[:, :, k] - w[:, :, k - 1]
    w[:, :, k + 2] = 2.0 * w[:, :, k] - w[:, :, k - 2]
    i0, i1, j0, j1, k0, k1 = 1, n0 - 2, 1, n1 - 2, 1, n2 - 2
    U, V, W = (_view(a, i0, i1, j0, j1, k0, k1) for a in (u, v, w))
    S = (slice(i0, i1), slice(j0, j1), slice(k0, k1))
    dzm0 = dz[k0:k1]
    if axis == 2:
        dzm1, dzp1, dzp2 = dz[k0 - 1:k1 - 1], dz[k0 + 1:k1 + 1], dz[k0 + 2:k1 + 2]
        mu[S] = B1 * (dy * dzm0 * U(0, 0, 0) + dy * dzp1 * U(0, 0, 1)) + B2 * (dy * dzm1 * U(0, 0, -1) + dy * dzp2 * U(0, 0, 2))
        mv[S] = B1 * (dx * dzm0 * V(0, 0, 0) + dx * dzp1 * V(0, 0, 1)) + B2 * (dx * dzm1 * V(0, 0, -1) + dx * dzp2 * V(0, 0, 2))
        mw[S] = B1 * (dx * dy * W(0, 0, 0) + dx * dy * W(0, 0, 1)) + B2 * (dx * dy * W(0, 0, -1) + dx * dy * W(0, 0, 2))
        return mu, mv, mw
    s1 = (1, 0, 0) if axis == 0 else (0, 1, 0)
    sm = tuple(-x for x in s1)
    s2 = tuple(2 * x for x in s1)
    mu[S] = B1 * (dy * dzm0 * U(0, 0, 0) + dy * dzm0 * U(*s1)) + B2 * (dy * dzm0 * U(*sm) + dy * dzm0 * U(*s2))
    mv[S] = B1 * (dx * dzm0 * V(0, 0, 0) + dx * dzm0 * V(*s1)) + B2 * (dx * dzm0 * V(*sm) + dx * dzm0 * V(*s2))
    mw[S] = B1 * (dx * dy * W(0, 0, 0) + dx * dy * W(*s1)) + B2 * (dx * dy * W(*sm) + dx * dy * W(*s2))
    return mu, mv, mw


def advect(q, mu, mv, mw, g: Grid, order, is_w):
    """advect{u,v,w}{2,4} (advect.c:286-734): f = -div(m q) / volume, with the
    wall-closure fluxes of cell-centred fields at the first rows."""
    n0, n1, n2, gz = g.n0, g.n1, g.n2, g.p.ngz
    dx, dy, dz = g.dx, g.dy, g.dz
    f = np.zeros(g.shape)
    m = 1 if order == 2 else 3
    k0, k1 = gz, n2 - gz - (1 if is_w else 0)
    i0, i1, j0, j1 = m, n0 - m, m, n1 - m
    Q = _view(q, i0, i1, j0, j1, k0, k1)
    MU = _view(mu, i0, i1, j0, j1, k0, k1)
    MV = _view(mv, i0, i1, j0, j1, k0, k1)
    MW = _view(mw, i0, i1, j0, j1, k0, k1)
    q0 = Q(0, 0, 0)
    xph = MU(0, 0, 0) * 0.5 * (q0 + Q(1, 0, 0))
    yph = MV(0, 0, 0) * 0.5 * (q0 + Q(0, 1, 0))
    zph = MW(0, 0, 0) * 0.5 * (q0 + Q(0, 0, 1))
    xmh = MU(-1, 0, 0) * 0.5 * (q0 + Q(-1, 0, 0))
    ymh = MV(0, -1, 0) * 0.5 * (q0 + Q(0, -1, 0))
    zmh = MW(0, 0, -1) * 0.5 * (q0 + Q(0, 0, -1))
    if order == 4:
        xp3 = MU(1, 0, 0) * 0.5 * (q0 + Q(3, 0, 0))
        yp3 = MV(0, 1, 0) * 0.5 * (q0 + Q(0, 3, 0))
        zp3 = MW(0, 0, 1) * 0.5 * (q0 + Q(0, 0, 3))
        xm3 = MU(-2, 0, 0) * 0.5 * (q0 + Q(-3, 0, 0))
        ym3 = MV(0, -2, 0) * 0.5 * (q0 + Q(0, -3, 0))
        zm3 = MW(0, 0, -2) * 0.5 * (q0 + Q(0, 0, -3))
    if not is_w:
        I, J = slice(i0, i1), slice(j0, j1)
        kb, kt = gz - 1, n2 - gz
        if order == 2:
            qbot = 0.5 * (q[I, J, kb] + q[I, J, kb + 1])
            qtop = 0.5 * (q[I, J, kt - 1] + q[I, J, kt])
            zph[:, :, -1] = mw[I, J, kt - 1] * qtop
            zmh[:, :, 0] = mw[I, J, kb] * qbot
        else:
            qbot = 0.5 * A2 * (q[I, J, kb - 1] + q[I, J, kb + 2]) + 0.5 * (A1 + 2.0 * A2) * (q[I, J, kb] + q[I, J, kb + 1])
            qtop = 0.5 * A2 * (q[I, J, kt - 2] + q[I, J, kt + 1]) + 0.5 * (A1 + 2.0 * A2) * (q[I, J, kt - 1] + q[I, J, kt])
            kk = kt - 1  # n2 - gz - 1
            zph[:, :, -1] = mw[I, J, kk] * qtop
            zp3[:, :, -1] = - mw[I, J, kk - 1] * 0.5 * (q[I, J, kk - 2] + q[I, J, kk + 1]) + 2.0 * mw[I, J, kk] * qtop
            zp3[:, :, -2] = mw[I, J, kk] * qtop  # k = n2-gz-2: mw[kp1] = mw[n2-gz-1]
            kk = gz
            zmh[:, :, 0] = mw[I, J, kk - 1] * qbot
            zm3[:, :, 0] = - mw[I, J, kk] * 0.5 * (q[I, J, kk + 2] + q[I, J, kk - 1]) + 2.0 * mw[I, J, kk - 1] * qbot
            zm3[:, :, 1] = mw[I, J, kk - 1] * qbot  # k = gz+1: mw[km2] = mw[gz-1]
    dzv = 0.5 * (dz[k0 + 1:k1 + 1] + dz[k0:k1]) if is_w else dz[k0:k1]
    if order == 2:
        f[i0:i1, j0:j1, k0:k1] = - ((xph - xmh) + (yph - ymh) + (zph - zmh)) / (dx * dy * dzv)
    else:
        f[i0:i1, j0:j1, k0:k1] = - ((A1 * (xph - xmh) + A2 * (xp3 - xm3))
                                    + (A1 * (yph - ymh) + A2 * (yp3 - ym3))
                                    + (A1 * (zph - zmh) + A2 * (zp3 - zm3))) / (dx * dy * dzv)
    return f


def flux_quick(u, v, w, c, g: Grid):
    """QUICK face fluxes of the scalar (scalar.c:113-162)."""
    n0, n1, n2 = g.n0, g.n1, g.n2
    dx, dy, dz = g.dx, g.dy, g.dz
    q = -0.125
    i0, i1, j0, j1, k0, k1 = 1, n0 - 2, 1, n1 - 2, 1, n2 - 2
    C = _view(c, i0, i1, j0, j1, k0, k1)
    S = (slice(i0, i1), slice(j0, j1), slice(k0, k1))
    mu = dy * dz[k0:k1] * u[S]
    mv = dx * dz[k0:k1] * v[S]
    mw = dx * dy * w[S]
    c0 = C(0, 0, 0)
    cphx = 0.5 * (c0 + C(1, 0, 0))
    cphy = 0.5 * (c0 + C(0, 1, 0))
    cphz = 0.5 * (c0 + C(0, 0, 1))
    cphx = cphx + np.where(mu > 0.0, q * (C(1, 0, 0) - 2.0 * c0 + C(-1, 0, 0)), q * (C(2, 0, 0) - 2.0 * C(1, 0, 0) + c0))
    cphy = cphy + np.where(mv > 0.0, q * (C(0, 1, 0) - 2.0 * c0 + C(0, -1, 0)), q * (C(0, 2, 0) - 2.0 * C(0, 1, 0) + c0))
    cphz = cphz + np.where(mw > 0.0, q * (C(0, 0, 1) - 2.0 * c0 + C(0, 0, -1)), q * (C(0, 0, 2) - 2.0 * C(0, 0, 1) + c0))
    fx = np.full(g.shape, np.nan); fy = np.full(g.shape, np.nan); fz = np.full(g.shape, np.nan)
    fx[S] = mu * cphx
    fy[S] = mv * cphy
    fz[S] = mw * cphz
    return fx, fy, fz


def advect_scalar(fx, fy, fz, g: Grid):
    """Flux divergence of the scalar (scalar.c:79-110).  Rows i or j >= n-2
    read flux entries the QUICK pass did not write; those land in x/y ghost
    cells that the periodic halo overwrites before use."""
    n0, n1, n2, gz = g.n0, g.n1, g.n2, g.p.ngz
    dx, dy, dz = g.dx, g.dy, g.dz
    f = np.zeros(g.shape)
    i0, i1, j0, j1, k0, k1 = 1, n0 - 2, 1, n1 - 2, gz, n2 - gz
    S = (slice(i0, i1), slice(j0, j1), slice(k0, k1))
    f[S] = - ((fx[S] - fx[i0 - 1:i1 - 1, j0:j1, k0:k1])
              + (fy[S] - fy[i0:i1, j0 - 1:j1 - 1, k0:k1])
              + (fz[S] - fz[i0:i1, j0:j1, k0 - 1:k1 - 1])) / (dx * dy * dz[k0:k1])
    return f


def add_buoyancy(c, fu, fv, fw, g: Grid, betg, order):
    """fu, fv, fw += betg * c interpolated to the faces (scalar.c:6-35 / 38-76)."""
    n0, n1, n2, gz = g.n0, g.n1, g.n2, g.p.ngz
    if order == 2:
        i0, i1, j0, j1 = 0, n0 - 1, 0, n1 - 1
        C = _view(c, i0, i1, j0, j1, gz, n2 - gz)
        S = (slice(i0, i1), slice(j0, j1), slice(gz, n2 - gz))
        fu[S] += 0.5 * (C(0, 0, 0) + C(1, 0, 0)) * betg[0]
        fv[S] += 0.5 * (C(0, 0, 0) + C(0, 1, 0)) * betg[1]
        C = _view(c, i0, i1, j0, j1, gz, n2 - gz - 1)
        S = (slice(i0, i1), slice(j0, j1), slice(gz, n2 - gz - 1))
        fw[S] += 0.5 * (C(0, 0, 0) + C(0, 0, 1)) * betg[2]
    else:
        i0, i1, j0, j1 = 1, n0 - 2, 1, n1 - 2
        C = _view(c, i0, i1, j0, j1, gz, n2 - gz)
        S = (slice(i0, i1), slice(j0, j1), slice(gz, n2 - gz))
        cphx = B1 * (C(0, 0, 0) + C(1, 0, 0)) + B2 * (C(-1, 0, 0) + C(2, 0, 0))
        cphy = B1 * (C(0, 0, 0) + C(0, 1, 0)) + B2 * (C(0, -1, 0) + C(0, 2, 0))
        fu[S] += cphx * betg[0]
        fv[S] += cphy * betg[1]
        C = _view(c, i0, i1, j0, j1, gz, n2 - gz - 1)
        S = (slice(i0, i1), slice(j0, j1), slice(gz, n2 - gz - 1))
        fw[S] += (B1 * (C(0, 0, 0) + C(0, 0, 1)) + B2 * (C(0, 0, -1) + C(0, 0, 2))) * betg[2]


# ---------------------------------------------------------------------------
# Pressure: divergence, FFT, per-wavenumber Poisson line solve, projection.
# ---------------------------------------------------------------------------


def divergence(u, v, w, d, g: Grid, order):
    """divergence{2,4} (pressure.c:40-64 / 67-117).  Order 4 rewrites the w
    ghosts next to the walls in place first."""
    n0, n1, n2, gz = g.n0, g.n1, g.n2, g.p.ngz
    dx, dy, dz = g.dx, g.dy, g.dz
    K = slice(gz, n2 - gz)
    if order == 2:
        i0, j0 = 1, 1
        U, V, W = (_view(a, i0, n0, j0, n1, gz, n2 - gz) for a in (u, v, w))
        d[i0:, j0:, K] = ((U(0, 0, 0) - U(-1, 0, 0)) / dx + (V(0, 0, 0) - V(0, -1, 0)) / dy
                          + (W(0, 0, 0) - W(0, 0, -1)) / dz[K])
        return
    k = gz - 1
    w[:, :, k - 1] = 2.0 * w[:, :, k] - w[:, :, k + 1]
    k = n2 - gz - 1
    w[:, :, k + 1] = 2.0 * w[:, :, k] - w[:, :, k - 1]
    i0, i1, j0, j1 = 2, n0 - 1, 2, n1 - 1
    U, V, W = (_view(a, i0, i1, j0, j1, gz, n2 - gz) for a in (u, v, w))
    d[i0:i1, j0:j1, K] = ((A1 * (U(0, 0, 0) - U(-1, 0, 0)) + A2 * (U(1, 0, 0) - U(-2, 0, 0))) / dx
                          + (A1 * (V(0, 0, 0) - V(0, -1, 0)) + A2 * (V(0, 1, 0) - V(0, -2, 0))) / dy
                          + (A1 * (W(0, 0, 0) - W(0, 0, -1)) + A2 * (W(0, 0, 1) - W(0, 0, -2))) / dz[K])


def project(u, v, w, p, g: Grid, dt, order):
    """u, v, w -= dt grad p on the faces (pressure.c:120-151 / 154-194)."""
    n0, n1, n2, gz = g.n0, g.n1, g.n2, g.p.ngz
    dx, dy, dz = g.dx, g.dy, g.dz
    if order == 2:
        i0, i1, j0, j1 = 0, n0 - 1, 0, n1 - 1
        P = _view(p, i0, i1, j0, j1, gz, n2 - gz)
        S = (slice(i0, i1), slice(j0, j1), slice(gz, n2 - gz))
        u[S] -= (P(1, 0, 0) - P(0, 0, 0)) * dt / dx
        v[S] -= (P(0, 1, 0) - P(0, 0, 0)) * dt / dy
        k0, k1 = gz - 1, n2 - gz
        P = _view(p, i0, i1, j0, j1, k0, k1)
        dzp1h = 0.5 * (dz[k0 + 1:k1 + 1] + dz[k0:k1])
        w[i0:i1, j0:j1, k0:k1] -= (P(0, 0, 1) - P(0, 0, 0)) * dt / dzp1h
        return
    i0, i1, j0, j1 = 1, n0 - 2, 1, n1 - 2
    P = _view(p, i0, i1, j0, j1, gz, n2 - gz)
    S = (slice(i0, i1), slice(j0, j1), slice(gz, n2 - gz))
    up1h = A1 * (P(1, 0, 0) - P(0, 0, 0)) + A2 * (P(2, 0, 0) - P(-1, 0, 0))
    vp1h = A1 * (P(0, 1, 0) - P(0, 0, 0)) + A2 * (P(0, 2, 0) - P(0, -1, 0))
    u[S] -= up1h * dt / dx
    v[S] -= vp1h * dt / dy
    k0, k1 = gz - 1, n2 - gz
    P = _view(p, i0, i1, j0, j1, k0, k1)
    wp1h = A1 * (P(0, 0, 1) - P(0, 0, 0)) + A2 * (P(0, 0, 2) - P(0, 0, -1))
    dzp1h = 0.5 * (dz[k0 + 1:k1 + 1] + dz[k0:k1])
    w[i0:i1, j0:j1, k0:k1] -= wp1h * dt / dzp1h


def modified_wavenumbers(n, order):
    """lamx / lamy of pressure.c:312-315 (order 2) and 376-389 (order 4),
    evaluated with the C library cos like the reference."""
    lam = np.empty(n)
    for i in range(n):
        c1 = math.cos(2.0 * math.pi * 1.0 * float(i) / float(n))
        if order == 2:
            lam[i] = 2.0 - 2.0 * c1
        else:
            c2 = math.cos(2.0 * math.pi * 2.0 * float(i) / float(n))
            c3 = math.cos(2.0 * math.pi * 3.0 * float(i) / float(n))
            lam[i] = ((2.0 * A2 * A2 + 2.0 * A1 * A1) + (4.0 * A1 * A2 - 2.0 * A1 * A1) * c1
                      + (-4.0 * A1 * A2) * c2 + (-2.0 * A2 * A2) * c3)
    return lam


def pressure_poisson(ch, g: Grid, dt, order, kx0=0):
    """Per (kx, ky) line solve of the discrete Poisson equation in z, Re and
    Im parts separately (pressure.c:293-354 / 357-443).  ch: complex array
    (nkx, ny, n2) of the wavenumbers kx0 .. kx0 + nkx - 1 (all nx/2+1 of them
    by default; a range of them for one rank of a kx-slab decomposition),
    modified in place; all n2 entries written.  The mean mode (0, 0) uses
    p = 0 (Dirichlet) at the bottom wall, every other mode Neumann at both
    walls."""
    p = g.p
    n2, gz, nz = g.n2, p.ngz, p.nz
    dx, dy, dz = g.dx, g.dy, g.dz
    nkx = ch.shape[0]
    lamx = modified_wavenumbers(p.nx, order)[kx0:kx0 + nkx]
    lamy = modified_wavenumbers(p.ny, order)
    LX = np.repeat(lamx, p.ny)
    LY = np.tile(lamy, nkx)
    cols = ch.reshape(-1, n2)
    ncol = cols.shape[0]
    out = np.empty_like(cols)
    K = slice(gz, n2 - gz)
    for part in (0, 1):
        B = Band(n2, ncol, 3 if order == 2 else 7)
        for nm in ("abc" if order == 2 else "abcdefg"):
            setattr(B, nm, np.zeros((ncol, n2)))
        B.dvol = dx * dy * dz
        B.diag_fix = lambda k, s: (s - LX * (dx * dy * dz[k]) * dt / (dx * dx)
                                   - LY * (dx * dy * dz[k]) * dt / (dy * dy))
        _band_u(g, dt, order, B)
        src = cols.real if part == 0 else cols.imag
        B.r[:, K] = src[:, K] * B.dvol[K]
        _pressure_closure_and_solve(B, g, order, ncol, kx0 == 0)
        if part == 0:
            out.real = B.x
        else:
            out.imag = B.x
    cols[:] = out


def _pressure_closure_and_solve(B, g, order, ncol, mean_mode=True):
    """ghost_stencil/reduce/solve/fill of pressure_poisson{2,4} with per-column
    coefficient rows (mode (0, 0) is column 0 when mean_mode)."""
    n2, gz, nz = g.n2, g.p.ngz, g.p.nz
    K = slice(gz, n2 - gz)
    # Column 0 is (kx, ky) = (0, 0): Dirichlet bottom; all others Neumann.
    if mean_mode:
        groups = [(np.arange(1), DIRICHP), (np.arange(1, ncol), NEUMANP)]
    else:
        groups = [(np.arange(ncol), NEUMANP)]
    for idx, btype in groups:
        if idx.size == 0:
            continue
        Bs = Band(n2, idx.size, B.width)
        for nm in ("abc" if order == 2 else "abcdefg"):
            setattr(Bs, nm, np.array(getattr(B, nm)[idx].T))  # (n2, ncol)
        Bs.r = B.r[idx].copy()
        Bs.x = np.zeros((idx.size, n2))
        if order == 2:
            u_ghost_stencil_bot2(Bs, g.dz, gz - 1, 0.0, btype)
            u_ghost_stencil_top2(Bs, g.dz, n2 - gz, 0.0, NEUMANP)
            u_ghost_reduce_bot2(Bs, gz - 1)
            u_ghost_reduce_top2(Bs, n2 - gz)
            Bs.x[:, K] = tridag(Bs.a[K].T, Bs.b[K].T, Bs.c[K].T, Bs.r[:, K], nz)
            u_ghost_fill_bot2(Bs, gz - 1)
            u_ghost_fill_top2(Bs, n2 - gz)
        else:
            u_ghost_stencil_bot4(Bs, g.dz, gz - 1, 0.0, btype)
            u_ghost_stencil_top4(Bs, g.dz, n2 - gz, 0.0, NEUMANP)
            u_ghost_reduce_bot4(Bs, gz - 1)
            u_ghost_reduce_top4(Bs, n2 - gz)
            Bs.x[:, K] = heptdag(Bs.a[K].T, Bs.b[K].T, Bs.c[K].T, Bs.d[K].T, Bs.e[K].T,
                                 Bs.f[K].T, Bs.g[K].T, Bs.r[:, K], nz)
            u_ghost_fill_bot4(Bs, gz - 1)
            u_ghost_fill_top4(Bs, n2 - gz)
        B.x = getattr(B, "x", np.zeros((ncol, n2)))
        B.x[idx] = Bs.x


def fft_forward(d, g: Grid):
    """FFT3D_FWD (chanfast.c:21-36): real 2-D DFT over (x, y) of every z plane
    of the interior columns, normalised by 1/nx then 1/ny (fft.c:161-202).
    Returns complex (nx/2+1, ny, n2)."""
    p = g.p
    inner = d[p.ngx:p.ngx + p.nx, p.ngy:p.ngy + p.ny, :]
    xh = np.fft.rfft(inner, axis=0) * (1.0 / float(p.nx))
    return np.fft.fft(xh, axis=1) * (1.0 / float(p.ny))


def fft_backward(ch, g: Grid):
    """FFT3D_BWD (chanfast.c:38-55): unnormalised inverse; returns the real
    (nx, ny, n2) interior."""
    p = g.p
    yh = np.fft.ifft(ch, axis=1, norm="forward")
    return np.fft.irfft(yh, n=p.nx, axis=0, norm="forward")


def pad_interior(a, interior, g: Grid):
    p = g.p
    a[p.ngx:p.ngx + p.nx, p.ngy:p.ngy + p.ny, :] = interior


# ---------------------------------------------------------------------------
# Driver state and the RK3 substep.
# ---------------------------------------------------------------------------


@dataclass
class State:
    """Fields of one instance (padded layout) plus the RK3 history."""

    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    c: np.ndarray
    p: np.ndarray
    f: list = field(default_factory=list)   # current RHS u, v, w, c
    g: list = field(default_factory=list)   # previous-stage RHS
    substep: int = 0
    log: list = field(default_factory=list)  # per substep: mdpdx, ..., dcdt, ...


def new_state(u, v, w, c, grid: Grid) -> State:
    fill = lambda: np.full(grid.shape, FILL_VALUE)
    return State(u=u.copy(), v=v.copy(), w=w.copy(), c=c.copy(), p=fill(),
                 f=[fill() for _ in range(4)], g=[fill() for _ in range(4)])


def _mass_control(x, h, solve, g: Grid, gamdt, kappa, order, comm=None):
    """Bulk-mean statistics of chanfast.c:485-523 / 572-610: xy-average,
    z-average, wall gradients, centreline; for x and for the Green's function
    h = solve(gamdt)."""
    comm = comm or SINGLE_RANK
    p = g.p
    gx, gy, gz, n2, nz = p.ngx, p.ngy, p.ngz, g.n2, p.nz
    dz = g.dz
    out = []
    for pass_ in (0, 1):
        if pass_ == 1:
            h[:] = gamdt
            solve(h, h)
        src = x if pass_ == 0 else h
        avg = comm.xy_avg(src, g)
        vol = get_z_avg(avg, nz, gz, dz)
        if order == 4:
            bot = kappa * (A1 * (avg[gz] - avg[gz - 1]) + A2 * (avg[gz + 1] - avg[gz - 2])) / (0.5 * (dz[gz] + dz[gz - 1]))
            top = kappa * (A1 * (avg[n2 - gz] - avg[n2 - gz - 1]) + A2 * (avg[n2 - gz + 1] - avg[n2 - gz - 2])) / (0.5 * (dz[n2 - gz] + dz[n2 - gz - 1]))
        else:
            bot = kappa * (avg[gz] - avg[gz - 1]) / (0.5 * (dz[gz] + dz[gz - 1]))
            top = kappa * (avg[n2 - gz] - avg[n2 - gz - 1]) / (0.5 * (dz[n2 - gz] + dz[n2 - gz - 1]))
        cl = 0.5 * (avg[gz + nz // 2 - 1] + avg[gz + nz // 2]) if nz % 2 == 0 else avg[gz + nz // 2]
        out.append([vol, bot, top, cl])
    return out


def get_xy_avg(u, g: Grid):
    """get_xy_avg (get.c:281-302): mean over interior x, y for every k."""
    p = g.p
    inner = u[p.ngx:p.ngx + p.nx, p.ngy:p.ngy + p.ny, :]
    return inner.reshape(-1, g.n2).sum(axis=0) * (1.0 / (float(p.nx) * float(p.ny)))


def get_z_avg(avg, nz, gz, dz):
    """get_z_avg (get.c:490-502): dz-weighted mean over interior k."""
    a = 0.0
    lz = 0.0
    for k in range(gz, nz + gz):
        a += avg[k] * dz[k]
        lz += dz[k]
    return a / lz


class SingleRank:
    """The three operations of a substep that need the whole x-y plane, on
    one rank: periodic halos (ghostz_periodic), xy averages (get_xy_avg) and
    the pressure solve (FFT3D_FWD, pressure_poisson, FFT3D_BWD).  A
    decomposed run passes its own object with the same methods to
    substep()."""

    def halo(self, a, g: Grid):
        ghostz_periodic(a, g)

    def xy_avg(self, a, g: Grid):
        return get_xy_avg(a, g)

    def pressure(self, d, g: Grid, dt, order):
        """p (interior, (nx, ny, n2)) from the divergence d (padded)."""
        ch = fft_forward(d, g)
        pressure_poisson(ch, g, dt, order)
        return fft_backward(ch, g)


SINGLE_RANK = SingleRank()


def substep(st: State, prm: Params, g: Grid, comm=None):
    """One RK3 substep of chanfast2/chanfast4 (chanfast.c:395-656 /
    1319-1580), in the reference's order.  comm: the whole-plane operations
    (SingleRank by default)."""
    comm = comm or SINGLE_RANK
    order = prm.order
    step = st.substep % 3
    st.f, st.g = st.g, st.f
    fu, fv, fw, fc = st.f
    gu, gv, gw, gc = st.g
    u, v, w, c = st.u, st.v, st.w, st.c
    uf, vf = prm.setuframe, prm.setvframe
    bcs = {"u": (0.0 - uf, 0.0 - uf), "v": (0.0 - vf, 0.0 - vf), "c": (-0.5, 0.5), "w": (0.0, 0.0)}

    for a, nm in ((u, "u"), (v, "v"), (c, "c")):
        comm.halo(a, g)
        apply_bc_u(a, g, *bcs[nm], order)
    comm.halo(w, g)
    apply_bc_w(w, g, *bcs["w"], order)

    mu, mv, mw = massflux(u, v, w, g, order, 0)
    fu[:] = advect(u, mu, mv, mw, g, order, False)
    mu, mv, mw = massflux(u, v, w, g, order, 1)
    fv[:] = advect(v, mu, mv, mw, g, order, False)
    mu, mv, mw = massflux(u, v, w, g, order, 2)
    fw[:] = advect(w, mu, mv, mw, g, order, True)
    add_laplacexy_operator(u, fu, g, prm.nu, order, False)
    add_laplacexy_operator(v, fv, g, prm.nu, order, False)
    add_laplacexy_operator(w, fw, g, prm.nu, order, True)
    fx, fy, fz = flux_quick(u, v, w, c, g)
    fc[:] = advect_scalar(fx, fy, fz, g)
    add_laplacexy_operator(c, fc, g, prm.nu / prm.prandtl, order, False)
    add_buoyancy(c, fu, fv, fw, g, (prm.betg_x, prm.betg_y, prm.betg_z), order)
    for a in (fu, fv, fw, fc):
        comm.halo(a, g)

    nu, dt, pr = prm.nu, prm.dt, prm.prandtl
    nuadt = nu * RK3_ALP[step] * dt
    nubdt = nu * RK3_BET[step] * dt
    abdt = (RK3_ALP[step] + RK3_BET[step]) * dt
    gamdt = RK3_GAM[step] * dt
    zetdt = RK3_ZET[step] * dt

    h = np.full(g.shape, np.nan)
    row = [0.0] * 10
    for fld, (x, fx_, gx_) in enumerate(((u, fu, gu), (v, fv, gv), (c, fc, gc), (w, fw, gw))):
        name = "uvcw"[fld]
        is_w = name == "w"
        na = nuadt / pr if name == "c" else nuadt
        nb = nubdt / pr if name == "c" else nubdt
        abc = (lambda a: apply_bc_w(a, g, *bcs[name], order)) if is_w else (lambda a: apply_bc_u(a, g, *bcs[name], order))
        hop = helmholtz1d_operator_w if is_w else helmholtz1d_operator_u
        slv_fn = solve_helmholtz1d_w if is_w else solve_helmholtz1d_u
        solve = lambda out, rhs, nb=nb, slv_fn=slv_fn: slv_fn(out, rhs, g, -nb, order)
        abc(x)
        hop(x, h, g, na, order)
        h += gamdt * fx_ + zetdt * gx_
        bc = np.zeros(g.shape)
        abc(bc)
        hbc = np.full(g.shape, np.nan)
        hop(bc, hbc, g, -nb, order)
        h -= hbc
        solve(x, h)
        abc(x)
        if name in ("u", "c"):
            kappa = nu if name == "u" else nu / pr
            s0, s1 = _mass_control(x, h, solve, g, gamdt, kappa, order, comm)
            if name == "u":
                m = (prm.want_uvolavg - uf - s0[0]) / s1[0] if prm.uvolavgmode == 1 else -prm.dpdx
            else:
                m = (prm.want_cvolavg - s0[0]) / s1[0] if prm.cvolavgmode == 1 else 0.0
            s0 = [a + b * m for a, b in zip(s0, s1)]
            x += h * m
            fx_ += m
            o = 0 if name == "u" else 5
            row[o:o + 5] = [m, s0[1], s0[2], s0[0], s0[3]]

    d = np.full(g.shape, np.nan)
    divergence(u, v, w, d, g, order)
    pad_interior(st.p, comm.pressure(d, g, abdt, order), g)
    comm.halo(st.p, g)
    project(u, v, w, st.p, g, abdt, order)
    st.log.append(row)
    st.substep += 1


def run(st: State, prm: Params, g: Grid, nsub: int, comm=None):
    for _ in range(nsub):
        substep(st, prm, g, comm)
    return st


def project_initial(u, v, w, prm: Params, g: Grid, dt=1.0):
    """Make (u, v, w) discretely divergence-free: periodic halos, divergence,
    Poisson solve, projection with time step dt (cases.c:426-470)."""
    for a in (u, v, w):
        ghostz_periodic(a, g)
    d = np.full(g.shape, np.nan)
    divergence(u, v, w, d, g, prm.order)
    ch = fft_forward(d, g)
    pressure_poisson(ch, g, dt, prm.order)
    p = np.full(g.shape, np.nan)
    pad_interior(p, fft_backward(ch, g), g)
    ghostz_periodic(p, g)
    project(u, v, w, p, g, dt, prm.order)
    return p
