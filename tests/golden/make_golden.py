"""Generate the golden fixtures of tests/golden from the compiled reference.

    python tests/golden/make_golden.py        (needs oracle/_ref, built by `make -C oracle`)

For each case the reference (the unmodified sources built against the
single-rank MPI / FFTW shims, driven by oracle/ref_driver.c) is given the
seeded initial state of oracle/ic.py, projected with the reference's own
divergence -> Poisson -> projection (dt = 1), then advanced by NSUB RK3
substeps.  Stored (interior points only, restart-file order [nx][ny][nz]):
the projected initial u, v, w, the initial c, the fields u, v, w, c, p after
NSUB substeps, and the per-substep mass-flux / scalar-mean log.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import chanfast_np as cn  # noqa: E402
import ic  # noqa: E402
import ref  # noqa: E402

NSUB = 6
CASES = {
    "o2_12x8x8": dict(order=2, nx=12, ny=8, nz=8, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                      nu=1 / 2800.0, prandtl=1.0, seed=0, amp=0.1, c_amp=0.0),
    "o4_12x8x10": dict(order=4, nx=12, ny=8, nz=10, lx=2 * np.pi, ly=np.pi, lz=2.0, dt=5e-4,
                       nu=1e-4, prandtl=0.71, seed=1, amp=0.1, c_amp=0.01),
}


def params(case):
    c = dict(case)
    for k in ("seed", "amp", "c_amp"):
        c.pop(k)
    return cn.Params(**c)


def interior(a, p):
    return np.ascontiguousarray(a[p.ngx:p.ngx + p.nx, p.ngy:p.ngy + p.ny, p.ngz:p.ngz + p.nz])


def generate(name, case):
    prm = params(case)
    g = cn.Grid(prm)
    R = ref.RefInstance(prm)
    u, v, w, c = ic.raw_state(prm, g.dz, case["seed"], case["amp"], case["c_amp"])
    for nm, a in zip("uvwc", (u, v, w, c)):
        R.set(nm, a)
    R.project(1.0)
    out = {f"ic_{nm}": interior(R.get(nm), prm) for nm in "uvw"}
    out["ic_c"] = interior(c, prm)
    R.substeps(NSUB)
    for nm in "uvwcp":
        out[nm] = interior(R.get(nm), prm)
    out["log"] = R.log()
    out["dz"] = g.dz
    R.close()
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    for name, case in CASES.items():
        print(generate(name, case))
