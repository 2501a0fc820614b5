"""The C-ABI libraries load and export every entry point include/*.h declares
(no device work: no GPU is needed)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ubiquitous-spoon_b200")


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"^\s*typedef[^;]*;", "", src, flags=re.M)   # function-pointer and struct typedefs
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    names.discard("if")
    return names


def exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


@pytest.fixture(scope="module")
def libs(cf):
    cf.lib()
    cf.driver_lib()
    steps = os.path.join(PKG, "libchanfast_steps.so")
    ctypes.CDLL(steps)   # loads without a device
    return os.path.join(PKG, "libchanfast_cuda.so"), os.path.join(PKG, "libchanfast.so"), steps


def test_every_declared_symbol_is_exported(libs):
    decl = declared_functions()
    assert {"cf_create", "cf_step", "chanfast2", "chanfast4", "channel2", "channel4"} <= decl
    assert {"advectu4", "pressure_poisson4", "solve_helmholtz1d_w4", "heptdag"} <= decl
    have = exported(libs[0]) | exported(libs[1]) | exported(libs[2])
    missing = sorted(decl - have)
    assert not missing, f"declared but not exported: {missing}"


def test_strerror_and_argument_checks(cf):
    L = cf.lib()
    assert L.cf_strerror(0) == b"ok"
    assert b"invalid" in L.cf_strerror(-1)
    # argument validation happens before any device work
    h = ctypes.c_void_p()
    bad = cf.Config.make(order=3, nx=16, ny=16, nz=16, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3)
    assert L.cf_create(ctypes.byref(bad), None, ctypes.byref(h)) == cf.CF_EINVAL
    bad = cf.Config.make(order=4, nx=16, ny=16, nz=16, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3, ngz=2)
    assert L.cf_create(ctypes.byref(bad), None, ctypes.byref(h)) == cf.CF_EINVAL
    bad = cf.Config.make(order=4, nx=14, ny=16, nz=16, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3)
    assert L.cf_create(ctypes.byref(bad), None, ctypes.byref(h)) == cf.CF_EINVAL  # 14 = 2*7: no radix-7 FFT
    # the fully implicit scheme: power-of-two nx of 64..512, nz >= 8 at order 4, known scheme ids
    bad = cf.Config.make(order=2, nx=48, ny=16, nz=16, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3, scheme="channel")
    assert L.cf_create(ctypes.byref(bad), None, ctypes.byref(h)) == cf.CF_EINVAL
    bad = cf.Config.make(order=4, nx=64, ny=16, nz=7, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3, scheme="channel")
    assert L.cf_create(ctypes.byref(bad), None, ctypes.byref(h)) == cf.CF_EINVAL
    bad = cf.Config.make(order=4, nx=64, ny=16, nz=16, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3)
    bad.scheme = 2
    assert L.cf_create(ctypes.byref(bad), None, ctypes.byref(h)) == cf.CF_EINVAL
    assert L.cf_step(None, 1) == cf.CF_EINVAL


def test_config_mirrors_reference_arguments(cf):
    import chanfast_np as cn
    p = cn.Params(order=4, nx=8, ny=8, nz=8, lx=1, ly=1, lz=2, dt=1e-3, nu=1e-3)
    c = cf.Config.from_params(p)
    assert (c.order, c.nx, c.ngz) == (4, 8, 3)


def test_instance_bytes_and_batch_serve_argument_checks(cf):
    """Host-side parts of batching and serving, no device needed: the memory
    estimate used for admission, and argument checks that return before any
    device work."""
    L = cf.lib()
    big = cf.Config.make(order=4, nx=512, ny=512, nz=384, lx=6.28, ly=3.14, lz=2.0, dt=2.5e-4, nu=5e-5)
    small = cf.Config.make(order=2, nx=64, ny=64, nz=64, lx=6.28, ly=3.14, lz=2.0, dt=1e-3, nu=1e-3)
    chan = cf.Config.make(order=4, nx=512, ny=512, nz=384, lx=6.28, ly=3.14, lz=2.0, dt=2.5e-4, nu=5e-5,
                          scheme="channel")
    assert 13e9 < cf.instance_bytes(big) < 15e9          # 13 fields of 818 MB + spectrum + scratch
    assert 30e6 < cf.instance_bytes(small) < 50e6
    assert cf.instance_bytes(chan) > cf.instance_bytes(big)   # four spectra
    bad = cf.Config.make(order=3, nx=64, ny=64, nz=64, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3)
    assert cf.instance_bytes(bad) == 0
    res = (cf.Result * 2)()
    reqs = (cf.Request * 2)()
    for q in range(2):
        reqs[q].cfg = small
        reqs[q].nsteps = 1
    reqs[0].arrival_s, reqs[1].arrival_s = 1.0, 0.5          # not in arrival order
    cb = cf.DONE_FN(lambda i, h, u: None)
    assert L.cf_serve(reqs, 2, 1e9, 4, 1, None, cb, None, res) == cf.CF_EINVAL
    reqs[1].arrival_s = 2.0
    assert L.cf_serve(reqs, 2, 1e9, 0, 1, None, cb, None, res) == cf.CF_EINVAL    # no slots
    assert L.cf_serve(reqs, 2, 1e9, 4, 0, None, cb, None, res) == cf.CF_EINVAL    # empty rounds
    reqs[1].cfg = chan                                          # the fully implicit scheme is not served
    assert L.cf_serve(reqs, 2, 1e9, 4, 1, None, cb, None, res) == cf.CF_EINVAL
    assert L.cf_batch_step(None, 0, 3, None) == cf.CF_EINVAL


def test_ensemble_and_serving_traces_are_deterministic():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    a, b = bench.ensemble_members(), bench.ensemble_members()
    assert a == b and len(a) == 64
    assert {(m["nx"], m["ny"], m["nz"]) for m in a} == set(bench.ENSEMBLE_GRIDS)
    assert all(2800.0 <= m["re"] <= 10000.0 for m in a)
    t = bench.serve_trace(2000, 4.0, 1.0)
    assert t == bench.serve_trace(2000, 4.0, 1.0)
    rate = len(t) / t[-1]["arrival_s"]
    assert 3.6 < rate < 4.4                                     # Poisson arrivals at 4 per second
    assert all(200 <= r["nsteps"] <= 2000 and r["order"] in (2, 4) for r in t)
    assert all(2800.0 <= r["re"] <= 20000.0 for r in t)


def test_tuning_calls_check_arguments(cf):
    """Launch-shape calls: argument checks that return before any device work."""
    import ctypes
    L = cf.lib()
    shape = (ctypes.c_int * 4)(128, 128, 32, 4)
    assert L.cf_get_launch_shape(None, shape) == cf.CF_EINVAL
    assert L.cf_set_launch_shape(None, shape) == cf.CF_EINVAL
    assert L.cf_batch_get_launch_shape(None, shape) == cf.CF_EINVAL
    assert L.cf_set_tuning(1) == cf.CF_OK
