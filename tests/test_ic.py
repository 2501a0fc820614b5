"""Seeded initial-state generator: pin SplitMix64 and the state formulas."""
import numpy as np

import chanfast_np as cn
import ic


def splitmix_scalar(x):
    M = (1 << 64) - 1
    z = (x + 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return z ^ (z >> 31)


def test_splitmix_known_values():
    # SplitMix64 reference sequence from seed 0: successive states 1*golden, 2*golden, ...
    assert splitmix_scalar(0) == 0xE220A8397B1DCDAF
    xs = np.array([0, 1, 2, 12345, (7 << 40) | 99], dtype=np.uint64)
    got = ic.splitmix64(xs)
    for x, g in zip(xs.tolist(), got.tolist()):
        assert g == splitmix_scalar(x)


def test_uniform_range_and_independence():
    a = ic.uniform(0, 0, 16, 8, 8)
    b = ic.uniform(0, 1, 16, 8, 8)
    c = ic.uniform(1, 0, 16, 8, 8)
    assert a.min() >= -1.0 and a.max() < 1.0
    assert abs(a.mean()) < 0.1
    assert not np.array_equal(a, b) and not np.array_equal(a, c)


def test_raw_state_profiles():
    p = cn.Params(order=2, nx=8, ny=6, nz=10, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3)
    g = cn.Grid(p)
    u, v, w, c = ic.raw_state(p, g.dz, 0, 0.0, 0.0)
    zp = ic.z_at_p(g.dz, p.nz, p.ngz)
    k = slice(p.ngz, p.ngz + p.nz)
    assert np.allclose(u[3, 3, k], 1.5 * (1 - (zp[k] - 1) ** 2))
    assert np.allclose(c[3, 3, k], -0.5 + zp[k] / 2)
    assert np.all(w == 0) and np.all(v == 0)
    # the cosine grid spans the channel height (chanfast.c:184-189)
    assert abs(g.dz[k].sum() - 2.0) < 1e-14
