"""The reference's main.c, unchanged, as a program over the drop-in driver
library.

oracle/Makefile (target `dropin`) compiles main.c where it lies in the
reference tree against the single-rank MPI shim and links it with
libchanfast.so.  main.c hard-codes p_row = p_col = 2 (main.c:9-10) and runs
chanfast4 from outputdir/{u,v,w,c}_it17000.dat to step 18000 at 128^3 with
CFL-adaptive dt (main.c:46-60).  The drivers accept that decomposition in a
single process (one GPU holds the whole grid); under an MPI launcher with N
ranks p_row * p_col must be N, rank 0 runs the whole grid and the others
return without touching a GPU or a file."""
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "main_dropin")

# main.c:11-16, 46-53
NX = NY = NZ = 128
LX, LY, LZ = 4.0 * math.pi, 4.0 / 3.0 * math.pi, 2.0
UB = 15.63
IT, NT = 17000, 18000

needs_bin = pytest.mark.skipif(not os.path.exists(BIN), reason="oracle/_ref/main_dropin not built")
LAUNCHER_VARS = ("OMPI_COMM_WORLD_SIZE", "OMPI_COMM_WORLD_RANK", "PMI_SIZE", "PMI_RANK", "PMIX_SIZE",
                 "PMIX_RANK", "SLURM_NTASKS", "SLURM_PROCID")


def clean_env(**kw):
    env = {k: v for k, v in os.environ.items() if k not in LAUNCHER_VARS}
    env.update(kw)
    return env


def run_main(cwd, env):
    return subprocess.run([BIN], cwd=cwd, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                          timeout=600)


@needs_bin
def test_other_ranks_return_without_work(tmp_path):
    """Rank 1 of 4 (Open MPI's environment): nothing is read or written."""
    r = run_main(str(tmp_path), clean_env(OMPI_COMM_WORLD_SIZE="4", OMPI_COMM_WORLD_RANK="1"))
    assert r.returncode == 0
    assert "p_row=2 p_col=2 nx=128" in r.stdout
    assert r.stderr == ""
    assert os.listdir(tmp_path) == []


@needs_bin
@pytest.mark.parametrize("size", ["2", "3", "8"])
def test_decomposition_must_match_rank_count(tmp_path, size):
    """p_row * p_col = 4 under a launcher of another size is rejected, as the
    reference's check at chanfast.c:87 rejects it."""
    r = run_main(str(tmp_path), clean_env(PMI_SIZE=size, PMI_RANK="0"))
    assert r.returncode == 0                 # main.c returns EXIT_SUCCESS; the driver reports
    assert "chanfast4: invalid argument" in r.stderr
    assert os.listdir(tmp_path) == []


@needs_bin
@pytest.mark.gpu
def test_unchanged_main_matches_driver_call(cf, gpu, tmp_path):
    prm_cfg = cf.Config.make(order=4, nx=NX, ny=NY, nz=NZ, lx=LX, ly=LY, lz=LZ, dt=0.002, nu=1.0 / 180.0,
                             prandtl=1.0)
    with cf.Instance(prm_cfg) as inst:   # laminar profile + projected noise, bulk 1
        inst.init_fields(5, 0.1, 0.01)
        fields = {nm: inst.get_field(nm, layout=cf.LAYOUT_INTERIOR) for nm in "uvwc"}
    # the reference keeps u in the frame moving at setuframe = U_b (main.c:50,
    # chanfast.c:61-62): scale to bulk U_b and shift
    fields["u"] = UB * fields["u"] - UB
    fields["v"] = UB * fields["v"]
    fields["w"] = UB * fields["w"]
    dirs = {}
    for who in ("main", "call"):
        d = tmp_path / who
        os.makedirs(d / "outputdir")
        for nm in "uvwc":
            np.ascontiguousarray(fields[nm]).tofile(str(d / "outputdir" / f"{nm}_it{IT}.dat"))
        dirs[who] = d
    r = run_main(str(dirs["main"]), clean_env())
    assert r.returncode == 0, r.stderr
    assert "p_row=2 p_col=2 nx=128 ny=128 nz=128" in r.stdout
    assert r.stderr.strip() == "chanfast4: p_row x p_col = 2 x 2: one GPU holds the whole 128 x 128 x 128 grid"
    cwd = os.getcwd()
    os.chdir(dirs["call"])
    try:   # the same driver called directly with main.c's arguments, at 1 x 1
        rc = cf.chanfast(4, 1, 1, NX, NY, NZ, IT, NT, NT, 3, 3, 3, LX, LY, LZ, 0.002, 1.0, 1, 1.0 / 180.0, 1.0,
                         -1.0, UB, 1, 0.0, 1, UB, 0.0, 0.0, 0.0, 0.0)
    finally:
        os.chdir(cwd)
    assert rc == 0
    a, b = dirs["main"] / "outputdir", dirs["call"] / "outputdir"
    names = sorted(os.listdir(b))
    assert sorted(os.listdir(a)) == names
    assert f"u_it{NT}.dat" in names and "pstat.dat" in names and "uu_specx_it18000.dat" in names
    for n in names:
        assert (a / n).read_bytes() == (b / n).read_bytes(), n
    u = np.fromfile(str(a / f"u_it{NT}.dat"))
    assert u.size == NX * NY * NZ and np.isfinite(u).all()
    cfl = np.loadtxt(str(a / "cfl.dat"))
    assert cfl.shape == (NT - IT, 3) and np.allclose(cfl[:, 2], 1.0)   # cflmode 1: dt keeps CFL at 1
