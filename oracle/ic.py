"""Seeded initial states and restart files -- TEST INFRASTRUCTURE.

The reference has no initial-condition generator: chanfast reads raw restart
files (chanfast.c:352-368, io.c:259-297).  Tests build the state with the
same counter-based generator the product uses (SplitMix64 of
(seed, field, global interior index)); this module is the numpy statement of
it, used to check the device generator bit for bit and to write restart files
for the unmodified reference driver.

Raw state (before projection), U_cl = 1.5 (laminar centreline, bulk 1):
  u = 1.5 (1 - (z_p - 1)^2) + amp * U_cl * xi_u      on cells
  v = amp * U_cl * xi_v                               on cells
  w = amp * U_cl * xi_w                               on interior z faces, 0 on walls
  c = -0.5 + z_p / 2 + c_amp * xi_c                   on cells
with xi uniform in [-1, 1).  z_p, z_w are the reference grid coordinates
(get.c:458-487).
"""
from __future__ import annotations

import numpy as np

MASK64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15
FIELD_U, FIELD_V, FIELD_W, FIELD_C = 0, 1, 2, 3


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 output function on uint64 arrays (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = x + np.uint64(GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, fld: int, nx: int, ny: int, nz: int) -> np.ndarray:
    """xi in [-1, 1) for every interior point, shape (nx, ny, nz); counter =
    (seed * 4 + fld) << 40 | global index (ix * ny + iy) * nz + iz."""
    idx = np.arange(nx * ny * nz, dtype=np.uint64)
    key = np.uint64(((seed * 4 + fld) << 40) & MASK64)
    r = splitmix64(key | idx)
    m = (r >> np.uint64(11)).astype(np.float64)
    return (m * (2.0 ** -53) * 2.0 - 1.0).reshape(nx, ny, nz)


def z_at_p(dz, nz, gz):
    """get_z_at_p (get.c:458-471)."""
    n2 = nz + 2 * gz
    z = np.empty(n2)
    z[0] = 0.5 * dz[0]
    for k in range(1, n2):
        z[k] = z[k - 1] + 0.5 * (dz[k - 1] + dz[k])
    z0 = 0.5 * (z[gz - 1] + z[gz])
    return z - z0


def z_at_w(dz, nz, gz):
    """get_z_at_w (get.c:474-487)."""
    n2 = nz + 2 * gz
    z = np.empty(n2)
    z[0] = dz[0]
    for k in range(1, n2):
        z[k] = z[k - 1] + dz[k]
    return z - z[gz - 1]


def raw_state(prm, dz, seed: int, amp: float, c_amp: float):
    """Unprojected (u, v, w, c) in the padded layout; x/y ghosts periodic
    copies, z ghosts zero (the drivers recompute them)."""
    nx, ny, nz = prm.nx, prm.ny, prm.nz
    gx, gy, gz = prm.ngx, prm.ngy, prm.ngz
    n0, n1, n2 = nx + 2 * gx, ny + 2 * gy, nz + 2 * gz
    zp = z_at_p(dz, nz, gz)[gz:gz + nz]
    ucl = 1.5
    out = []
    for fld in range(4):
        xi = uniform(seed, fld, nx, ny, nz)
        if fld == FIELD_U:
            a = 1.5 * (1.0 - (zp - 1.0) * (zp - 1.0)) + amp * ucl * xi
        elif fld == FIELD_V:
            a = amp * ucl * xi
        elif fld == FIELD_W:
            a = amp * ucl * xi
            a[:, :, nz - 1] = 0.0  # the face at k = n2 - gz - 1 is the top wall
        else:
            a = -0.5 + zp / 2.0 + c_amp * xi
        full = np.zeros((n0, n1, n2))
        full[gx:gx + nx, gy:gy + ny, gz:gz + nz] = a
        if fld == FIELD_W:
            # interior faces k = gz .. n2-gz-2; walls k = gz-1 and n2-gz-1 are zero
            full[gx:gx + nx, gy:gy + ny, gz:gz + nz - 1] = a[:, :, :nz - 1]
            full[:, :, n2 - gz - 1] = 0.0
            full[:, :, gz - 1] = 0.0
        periodic(full, gx, gy)
        out.append(full)
    return out


def periodic(a, gx, gy):
    n0, n1 = a.shape[:2]
    a[0:gx] = a[n0 - 2 * gx:n0 - gx]
    a[n0 - gx:n0] = a[gx:2 * gx]
    a[:, 0:gy] = a[:, n1 - 2 * gy:n1 - gy]
    a[:, n1 - gy:n1] = a[:, gy:2 * gy]


def write_restart(path, a, prm):
    """Raw native-endian FP64, C order [nx][ny][nz], interior only (io.c:211-257)."""
    gx, gy, gz = prm.ngx, prm.ngy, prm.ngz
    inner = a[gx:gx + prm.nx, gy:gy + prm.ny, gz:gz + prm.nz]
    np.ascontiguousarray(inner).tofile(path)


def read_restart(path, prm):
    """Inverse of write_restart (io.c:259-297): returns the (nx, ny, nz) interior."""
    return np.fromfile(path, dtype=np.float64).reshape(prm.nx, prm.ny, prm.nz)
