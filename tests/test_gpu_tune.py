"""Launch-shape autotuning (cf_create / cf_batch_create, cf_*_launch_shape).

The tuned kernels index their work from blockDim, one column, column pair or
point per thread, so every candidate shape must give the same results bit
for bit; the tuner may then pick any of them.  Cases include planes that are
not a multiple of the block size (padding warps in the per-warp row sums of
the back substitution) and both orders."""
import os
import subprocess
import sys

import numpy as np
import pytest

import chanfast_np as cn

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOLVE = (64, 128)
POIS = (64, 128)
PROJ = ((32, 2), (32, 4), (32, 8), (64, 2))
SHAPES = [(128, 128, 32, 4), (64, 64, 32, 2), (128, 128, 32, 8), (128, 64, 64, 2), (64, 128, 64, 2)]


def cfg(cf, order, nx, ny, nz, re=2800.0):
    prm = cn.Params(order=order, nx=nx, ny=ny, nz=nz, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                    nu=1.0 / re, prandtl=0.71)
    return cf.Config.from_params(prm)


def valid(shape):
    return shape[0] in SOLVE and shape[1] in POIS and tuple(shape[2:]) in PROJ


def test_tuned_shape_is_a_candidate_and_cached(cf, gpu):
    c = cfg(cf, 4, 128, 96, 32)
    with cf.Instance(c) as a, cf.Instance(c) as b:
        assert valid(a.launch_shape())
        assert a.launch_shape() == b.launch_shape()   # the second creation reads the cache
        with pytest.raises(cf.ChanfastError):
            a.set_launch_shape((256, 128, 32, 4))
        with pytest.raises(cf.ChanfastError):
            a.set_launch_shape((128, 128, 16, 4))


@pytest.mark.parametrize("order,nx,ny,nz", [(2, 48, 40, 16), (4, 96, 72, 24), (4, 128, 128, 32)])
def test_every_shape_gives_identical_results(cf, gpu, order, nx, ny, nz):
    c = cfg(cf, order, nx, ny, nz)
    out = []
    for shape in SHAPES:
        with cf.Instance(c) as inst:
            inst.set_launch_shape(shape)
            assert inst.launch_shape() == shape
            inst.init_fields(5, 0.1, 0.01)
            inst.step(2)          # substeps, eager
            inst.step_graph(3)    # RK3 steps, graph replay with the same shape
            out.append({nm: inst.get_field(nm) for nm in "uvwcp"} | {"log": inst.log()})
    for o in out[1:]:
        for k in o:
            assert np.array_equal(o[k], out[0][k]), k


def test_channel_scheme_shapes_identical(cf, gpu):
    prm = cn.Params(order=4, nx=64, ny=24, nz=16, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                    nu=1 / 100.0, prandtl=0.71)
    c = cf.Config.from_params(prm, scheme="channel")
    out = []
    for shape in SHAPES[:3]:
        with cf.Instance(c) as inst:
            inst.set_launch_shape(shape)
            inst.init_fields(3, 0.1, 0.01)
            inst.step(4)
            out.append({nm: inst.get_field(nm) for nm in "uvwcp"})
    for o in out[1:]:
        for k in o:
            assert np.array_equal(o[k], out[0][k]), k


def test_batch_tuning_keeps_members_and_results(cf, gpu):
    members = [(2, 64, 64, 24), (4, 96, 96, 16), (2, 48, 40, 16), (4, 128, 64, 24)]
    mixed = [cf.Instance(cfg(cf, *m)) for m in members]
    alone = [cf.Instance(cfg(cf, *m)) for m in members]
    for q, (a, b) in enumerate(zip(mixed, alone)):
        a.init_fields(q, 0.1, 0.01)
        b.init_fields(q, 0.1, 0.01)
        a.step(1)   # one substep: members with state (mid RK3 step), which tuning must not touch
        b.step(1)
    own = [m.launch_shape() for m in mixed]
    before = [{nm: m.get_field(nm) for nm in "uvwcp"} for m in mixed]
    with cf.Batch(mixed) as B:
        assert valid(B.launch_shape())
        assert [m.launch_shape() for m in mixed] == own
        for m, snap in zip(mixed, before):   # creating (and tuning) the batch changed no state
            for nm in "uvwcp":
                assert np.array_equal(m.get_field(nm), snap[nm]), nm
        B.run(4)    # RK3 steps
        B.sync()
    for b in alone:
        b.step(12)  # substeps
    for a, b in zip(mixed, alone):
        for nm in "uvwc":
            rel = np.linalg.norm(a.get_field(nm) - b.get_field(nm)) / np.linalg.norm(b.get_field(nm))
            assert rel <= 1e-13, nm
    for inst in mixed + alone:
        inst.close()


def test_cache_file_is_read_and_written(gpu, tmp_path):
    path = tmp_path / "tune.txt"
    prog = (
        "import importlib, numpy as np, sys\n"
        f"sys.path.insert(0, {os.path.join(ROOT, 'oracle')!r}); sys.path.insert(0, {ROOT!r})\n"
        "import chanfast_np as cn\n"
        "cf = importlib.import_module('ubiquitous-spoon_b200')\n"
        "prm = cn.Params(order=2, nx=64, ny=48, nz=16, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3, prandtl=0.71)\n"
        "with cf.Instance(cf.Config.from_params(prm)) as i:\n"
        "    print(*i.launch_shape())\n"
    )
    env = dict(os.environ, CF_TUNE_CACHE=str(path))
    r = subprocess.run([sys.executable, "-c", prog], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = path.read_text().split("\n")
    entry = [ln for ln in lines if "o2s0-64x48x16" in ln]
    assert len(entry) == 1 and entry[0].split()[1:] == r.stdout.split()
    # a cached entry is used as it stands (no timing): plant a different shape
    key = entry[0].split()[0]
    planted = "64 64 64 2" if r.stdout.split() != ["64", "64", "64", "2"] else "128 128 32 8"
    path.write_text(f"{key} {planted}\n")
    r = subprocess.run([sys.executable, "-c", prog], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == planted.split()
