"""The numpy restatement (oracle/chanfast_np.py) against the golden fixtures
produced by the compiled reference (tests/golden/make_golden.py), and against
the reference itself when it is built."""
import glob
import os

import numpy as np
import pytest

import chanfast_np as cn
import ic

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
sys_cases = None


def load_cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


MG = load_cases()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("name", sorted(MG.CASES))
def test_oracle_matches_golden(name):
    case = MG.CASES[name]
    gold = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    prm = MG.params(case)
    g = cn.Grid(prm)
    assert np.array_equal(g.dz, gold["dz"]), "grid stretching differs from the reference"
    u, v, w, c = ic.raw_state(prm, g.dz, case["seed"], case["amp"], case["c_amp"])
    # start from the reference-projected state so that only the substep is compared
    I = (slice(prm.ngx, prm.ngx + prm.nx), slice(prm.ngy, prm.ngy + prm.ny), slice(prm.ngz, prm.ngz + prm.nz))
    for a, key in ((u, "ic_u"), (v, "ic_v"), (w, "ic_w")):
        a[I] = gold[key]
        ic.periodic(a, prm.ngx, prm.ngy)
    assert np.array_equal(c[I], gold["ic_c"]), "seeded generator differs"
    st = cn.new_state(u, v, w, c, g)
    cn.run(st, prm, g, MG.NSUB)
    for nm in "uvwc":
        assert rel(getattr(st, nm)[I], gold[nm]) < 1e-13, nm
    assert rel(st.p[I], gold["p"]) < 1e-10
    log = np.array(st.log)
    assert np.allclose(log, gold["log"], rtol=1e-11, atol=1e-13)


@pytest.mark.parametrize("name", sorted(MG.CASES))
def test_oracle_projection_matches_golden(name):
    case = MG.CASES[name]
    gold = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    prm = MG.params(case)
    g = cn.Grid(prm)
    u, v, w, c = ic.raw_state(prm, g.dz, case["seed"], case["amp"], case["c_amp"])
    cn.project_initial(u, v, w, prm, g, 1.0)
    I = (slice(prm.ngx, prm.ngx + prm.nx), slice(prm.ngy, prm.ngy + prm.ny), slice(prm.ngz, prm.ngz + prm.nz))
    for a, key in ((u, "ic_u"), (v, "ic_v"), (w, "ic_w")):
        assert rel(a[I], gold[key]) < 1e-13, key


@pytest.mark.parametrize("order,nx,ny,nz", [(2, 16, 12, 10), (4, 18, 24, 12)])
def test_oracle_matches_reference(ref, order, nx, ny, nz):
    prm = cn.Params(order=order, nx=nx, ny=ny, nz=nz, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                    nu=1 / 2800.0, prandtl=0.71)
    g = cn.Grid(prm)
    R = ref.RefInstance(prm)
    u, v, w, c = ic.raw_state(prm, g.dz, 3, 0.1, 0.01)
    for nm, a in zip("uvwc", (u, v, w, c)):
        R.set(nm, a)
    R.project(1.0)
    u, v, w = R.get("u"), R.get("v"), R.get("w")
    for nm, a in zip("uvwc", (u, v, w, c)):
        R.set(nm, a)
    st = cn.new_state(u, v, w, c, g)
    R.substeps(1)
    cn.run(st, prm, g, 1)
    I = (slice(3, 3 + nx), slice(3, 3 + ny), slice(3, 3 + nz))
    # one substep: identical arithmetic except the FFT inside the projection
    for nm in "uvwc":
        assert rel(getattr(st, nm)[I], R.get(nm)[I]) < 1e-15, nm
    assert np.array_equal(np.array(st.log), R.log())
    R.substeps(29)
    cn.run(st, prm, g, 29)
    for nm in "uvwc":
        assert rel(getattr(st, nm)[I], R.get(nm)[I]) < 1e-13, nm
    assert rel(st.p[I], R.get("p")[I]) < 1e-10
