"""The oracle's substep replay (oracle/ref_driver.c) equals the unmodified
reference drivers run through restart files, bit for bit: chanfast2/chanfast4
for the z-implicit scheme and channel2/channel4 for the fully implicit one."""
import os

import numpy as np
import pytest

import chanfast_np as cn
import ic


@pytest.mark.parametrize("scheme", ["chanfast", "channel"])
@pytest.mark.parametrize("order", [2, 4])
def test_replay_equals_driver(ref, tmp_path, order, scheme):
    prm = cn.Params(order=order, nx=12, ny=8, nz=10, lx=2 * np.pi, ly=np.pi, lz=2.0, dt=1e-3,
                    nu=1 / 2800.0, prandtl=0.71)
    g = cn.Grid(prm)
    R = ref.RefInstance(prm)
    u, v, w, c = ic.raw_state(prm, g.dz, 5, 0.1, 0.01)
    for nm, a in zip("uvwc", (u, v, w, c)):
        R.set(nm, a)
    R.project(1.0)
    fields = {"u": R.get("u"), "v": R.get("v"), "w": R.get("w"), "c": c}
    os.makedirs(tmp_path / "outputdir")
    for nm, a in fields.items():
        ic.write_restart(str(tmp_path / "outputdir" / f"{nm}_it0.dat"), a, prm)
    nsteps = 2
    ref.run_chanfast(str(tmp_path), prm, 0, nsteps, scheme=scheme)
    R2 = ref.RefInstance(prm)
    for nm, a in fields.items():
        full = np.zeros_like(a)
        full[3:3 + prm.nx, 3:3 + prm.ny, 3:3 + prm.nz] = a[3:3 + prm.nx, 3:3 + prm.ny, 3:3 + prm.nz]
        R2.set(nm, full)
    R2.substeps(3 * nsteps, scheme)
    for nm in "uvwc":
        got = ic.read_restart(str(tmp_path / "outputdir" / f"{nm}_it{nsteps}.dat"), prm)
        mine = R2.get(nm)[3:3 + prm.nx, 3:3 + prm.ny, 3:3 + prm.nz]
        assert np.array_equal(got, mine), nm
    pstat = np.loadtxt(str(tmp_path / "outputdir" / "pstat.dat"))
    log = R2.log()
    assert np.allclose(pstat[:, 1:], log[2::3, 0:5], rtol=1e-6)  # file holds %+e (7 digits)
