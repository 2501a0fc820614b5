"""The reference's step functions (include/chanfast_steps.h, computed on the
GPU by libchanfast_steps.so) against the compiled reference CPU functions of
the same name (oracle/_ref), one call each on seeded random padded inputs.

Bar: bit for bit.  The GPU library follows the reference's expressions
operation for operation without FMA contraction, so every output array (and
every input array a function rewrites in place, like the wall ghosts of
massflux*4 and divergence4) must be equal to the last bit.  Grids use the
reference's ghost width 3 (main.c:11-13), plus ghost width 1 for the
second-order functions that allow it."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS_LIB = os.path.join(ROOT, "ubiquitous-spoon_b200", "libchanfast_steps.so")
BC = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double, ctypes.c_double)
DIRICHU, NEUMANU, DIRICHW = 0, 1, 20


@pytest.fixture(scope="module")
def steps(gpu):
    if not os.path.exists(STEPS_LIB):
        pytest.fail(f"{STEPS_LIB} missing: run ubiquitous-spoon_b200/build.py")
    L = ctypes.CDLL(STEPS_LIB)
    L.cf_steps_message.restype = ctypes.c_char_p
    return L


@pytest.fixture(scope="module")
def reflib(ref):
    return ref.lib()


class Grid:
    def __init__(self, lnx, lny, nz, g, seed):
        self.lnx, self.lny, self.nz, self.g = lnx, lny, nz, g
        self.n0, self.n1, self.n2 = lnx + 2 * g, lny + 2 * g, nz + 2 * g
        self.rng = np.random.default_rng(seed)
        self.dz = 0.05 + 0.1 * self.rng.random(self.n2)
        self.dx, self.dy = 0.21, 0.17

    def field(self):
        return self.rng.standard_normal(self.n0 * self.n1 * self.n2)

    def dims(self):
        g = self.g
        return [self.lnx, self.lny, self.nz, g, g, g]


def _arg(a):
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(ctypes.c_void_p)
    if isinstance(a, (bool, int, np.integer)):
        return ctypes.c_int(int(a))
    if isinstance(a, float):
        return ctypes.c_double(a)
    return a   # callbacks


def call_both(steps, reflib, name, args, outputs):
    """Run `name` on copies of args in both libraries; compare the arrays at
    positions `outputs` bit for bit."""
    mine = [a.copy() if isinstance(a, np.ndarray) else a for a in args]
    theirs = [a.copy() if isinstance(a, np.ndarray) else a for a in args]
    getattr(reflib, name)(*[_arg(a) for a in theirs])
    getattr(steps, name)(*[_arg(a) for a in mine])
    assert steps.cf_steps_status() == 0, (name, steps.cf_steps_message().decode())
    for pos in outputs:
        a, b = mine[pos], theirs[pos]
        if not np.array_equal(a, b):
            d = np.abs(a - b)
            pytest.fail(f"{name}: argument {pos} differs, max |diff| {d.max():.3e} at {int(d.argmax())}")


def initialize(lib, order, nz, g):
    for m in ("diffuseu", "diffusew", "pressure"):
        getattr(lib, f"{m}_initialize{order}")(ctypes.c_int(nz), ctypes.c_int(g))


def finalize(lib, order):
    for m in ("diffuseu", "diffusew", "pressure"):
        getattr(lib, f"{m}_finalize{order}")()


@pytest.fixture(params=[(2, 3), (4, 3), (2, 1)], ids=["o2g3", "o4g3", "o2g1"])
def setup(request, steps, reflib):
    order, g = request.param
    G = Grid(7, 6, 10, g, seed=order * 10 + g)
    initialize(steps, order, G.nz, g)
    initialize(reflib, order, G.nz, g)
    yield order, G
    finalize(reflib, order)
    finalize(steps, order)


def test_constants(steps, reflib):
    for name in ("rk3_alp", "rk3_bet", "rk3_gam", "rk3_zet"):
        a = (ctypes.c_double * 3).in_dll(steps, name)
        b = (ctypes.c_double * 3).in_dll(reflib, name)
        assert list(a) == list(b), name
    for name in ("a1", "a2", "b1", "b2"):
        assert ctypes.c_double.in_dll(steps, name).value == ctypes.c_double.in_dll(reflib, name).value, name


def test_advect_family(steps, reflib, setup):
    order, G = setup
    if order == 4 and G.g < 3:
        pytest.skip("fourth order needs 3 ghosts")
    d = G.dims()
    u, v, w = G.field(), G.field(), G.field()
    for axis in "xyz":
        mu, mv, mw = G.field(), G.field(), G.field()
        call_both(steps, reflib, f"massflux{axis}{order}", [u, v, w, mu, mv, mw, *d, G.dx, G.dy, G.dz],
                  [0, 1, 2, 3, 4, 5])
    for comp, q in zip("uvw", (u, v, w)):
        mx, my, mz, f = G.field(), G.field(), G.field(), G.field()
        call_both(steps, reflib, f"advect{comp}{order}", [q, mx, my, mz, f, *d, G.dx, G.dy, G.dz], [4])


def test_scalar_family(steps, reflib, setup):
    order, G = setup
    d = G.dims()
    u, v, w, c = G.field(), G.field(), G.field(), G.field()
    fu, fv, fw = G.field(), G.field(), G.field()
    call_both(steps, reflib, f"add_buoyancy{order}", [c, fu, fv, fw, 0.3, -0.2, 0.7, *d], [1, 2, 3])
    mx, my, mz, fc = G.field(), G.field(), G.field(), G.field()
    call_both(steps, reflib, "flux_quick", [u, v, w, c, mx, my, mz, *d, G.dx, G.dy, G.dz], [4, 5, 6])
    call_both(steps, reflib, "advect_scalar", [mx, my, mz, fc, *d, G.dx, G.dy, G.dz], [3])


def test_pressure_family(steps, reflib, setup):
    order, G = setup
    d = G.dims()
    u, v, w, p, out = G.field(), G.field(), G.field(), G.field(), G.field()
    call_both(steps, reflib, f"divergence{order}", [u, v, w, out, *d, G.dx, G.dy, G.dz], [2, 3])
    call_both(steps, reflib, f"project{order}", [u, v, w, p, *d, G.dx, G.dy, G.dz, 0.013], [0, 1, 2])
    call_both(steps, reflib, f"pressure_laplacian{order}", [p, out, *d, G.dx, G.dy, G.dz, 0.013], [1])
    nx, ny = 8, 6
    for x0, lnx in ((0, nx // 2 + 1), (2, 3)):
        cout = G.rng.standard_normal(lnx * ny * G.n2 * 2)
        call_both(steps, reflib, f"pressure_poisson{order}",
                  [cout, nx, lnx, x0, ny, ny, 0, G.nz, G.g, G.dx, G.dy, G.dz, 0.013], [0])


@pytest.mark.parametrize("kind", ["u", "w"])
def test_diffuse_family(steps, reflib, setup, kind):
    order, G = setup
    d = G.dims()
    bctypes = [(DIRICHW, DIRICHW)] if kind == "w" else [(DIRICHU, DIRICHU), (NEUMANU, DIRICHU), (DIRICHU, NEUMANU)]
    xs = 0.1 * np.arange(G.n0, dtype=float)
    ys = 0.2 * np.arange(G.n1, dtype=float)
    bot = BC(lambda x, y: 0.3 + 0.1 * x - 0.2 * y)
    top = BC(lambda x, y: -0.4 + 0.05 * x * y)
    u, h = G.field(), G.field()
    for bb, bt in bctypes:
        call_both(steps, reflib, f"apply_bc_{kind}{order}", [u, *d, xs, ys, G.dz, bot, top, bb, bt], [0])
        call_both(steps, reflib, f"solve_helmholtz1d_{kind}{order}",
                  [u, h, *d, G.dz, -0.004, 0.25, -0.5, bb, bt], [0])
        nx, ny = 8, 6
        cout = G.rng.standard_normal((nx // 2 + 1) * ny * G.n2 * 2)
        call_both(steps, reflib, f"solve_helmholtz_{kind}{order}",
                  [cout, nx, nx // 2 + 1, 0, ny, ny, 0, G.nz, G.g, G.dx, G.dy, G.dz, -0.004, 0.25, -0.5, bb, bt],
                  [0])
    call_both(steps, reflib, f"helmholtz1d_operator_{kind}{order}", [u, h, *d, G.dz, 0.003], [1])
    call_both(steps, reflib, f"add_laplacexy_operator_{kind}{order}", [u, h, *d, G.dx, G.dy, 0.002], [1])
    call_both(steps, reflib, f"helmholtz_operator_{kind}{order}", [u, h, *d, G.dx, G.dy, G.dz, 0.003], [1])


def test_band_solvers(steps, reflib):
    rng = np.random.default_rng(5)
    n = 23
    a, c = rng.random(n), rng.random(n)
    b = 3.0 + rng.random(n)
    r, x = rng.standard_normal(n), np.zeros(n)
    call_both(steps, reflib, "tridag", [a, b, c, r, x, n], [4])
    bands = [rng.random(n) for _ in range(7)]
    bands[3] += 8.0
    call_both(steps, reflib, "heptdag", [*bands, rng.standard_normal(n), np.zeros(n), n], [8])


def test_order_mismatch_is_reported(steps):
    """Where the reference aborts (check() on the module order), the GPU
    library records CF_STEPS_EORDER and leaves the output untouched."""
    G = Grid(5, 4, 8, 3, seed=1)
    steps.diffuseu_initialize2(ctypes.c_int(G.nz), ctypes.c_int(3))
    u, h = G.field(), G.field()
    before = u.copy()
    steps.solve_helmholtz1d_u4(*[_arg(a) for a in [u, h, *G.dims(), G.dz, -0.01, 0.0, 0.0, DIRICHU, DIRICHU]])
    assert steps.cf_steps_status() == -2
    assert np.array_equal(u, before)
    steps.diffuseu_finalize2()
