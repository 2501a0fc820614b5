"""Long reference runs in child processes -- TEST INFRASTRUCTURE.

The compiled reference (oracle/_ref) advances about 1.6 M point-substeps/s on
one core, so a parity case on a production grid needs minutes of it.  Each
case listed in JOBS runs in a child process of its own, started when the
tests that use it are collected (before any GPU work, see conftest.py), so
that those minutes overlap the rest of the GPU suite.  A test reads the
job's results with `JobSet.wait`.

A job (python tests/ref_jobs.py NAME FOLDER) writes into FOLDER:
  init_{u,v,w,c}.npy            the reference-projected initial state
  s<N>_{u,v,w,c,p}.npy, s<N>_log.npy   the reference state after N substeps
  s<N>_div.npy                  max |div u| of that state over the interior,
                                by the reference's own divergence{2,4}
  error.txt                     if the job failed
Every file is written under a temporary name and renamed when complete.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

TWO_PI, PI = 2.0 * np.pi, np.pi

# name -> (Params keywords, seed, amp, c_amp, substep checkpoints, scheme)
JOBS = {
    # order 4 with the scalar, config-1 physics (Re_b 1e4, dt 5e-4, Pr 0.71)
    # on a 64 x 64 x 48 grid: 100 RK3 steps
    "o4_64x64x48_100steps": (dict(order=4, nx=64, ny=64, nz=48, lx=TWO_PI, ly=PI, lz=2.0, dt=5e-4, nu=1e-4,
                                  prandtl=0.71), 1, 0.1, 0.01, [300], "chanfast"),
    # the config-1 grid: 256 x 256 x 192, order 4, Re_b 1e4, dt 5e-4, scalar
    "cfg1_256x256x192": (dict(order=4, nx=256, ny=256, nz=192, lx=TWO_PI, ly=PI, lz=2.0, dt=5e-4, nu=1e-4,
                              prandtl=0.71), 1, 0.1, 0.01, [3, 30], "chanfast"),
    # the config-2 grid: 512 x 512 x 384, order 4, Re_b 2e4, dt 2.5e-4,
    # perturbation 0.05, seed 2
    "cfg2_512x512x384": (dict(order=4, nx=512, ny=512, nz=384, lx=TWO_PI, ly=PI, lz=2.0, dt=2.5e-4, nu=5e-5,
                              prandtl=0.71), 2, 0.05, 0.01, [1], "chanfast"),
}


def params(name):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import chanfast_np as cn
    kw = JOBS[name][0]
    return cn.Params(**kw)


def _save(folder, stem, a):
    tmp = os.path.join(folder, stem + ".part.npy")
    np.save(tmp, a)
    os.replace(tmp, os.path.join(folder, stem + ".npy"))


def run_job(name, folder):
    os.makedirs(folder, exist_ok=True)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import chanfast_np as cn
    import ic
    import ref
    kw, seed, amp, c_amp, checkpoints, scheme = JOBS[name]
    prm = cn.Params(**kw)
    g = cn.Grid(prm)
    R = ref.RefInstance(prm)
    raw = ic.raw_state(prm, g.dz, seed, amp, c_amp)
    for nm, a in zip("uvwc", raw):
        R.set(nm, a)
    R.project(1.0)
    init = {nm: R.get(nm) for nm in "uvw"}
    init["c"] = raw[3]
    del raw
    for nm in "uvwc":
        R.set(nm, init[nm])
        _save(folder, "init_" + nm, init[nm])
    del init
    done = 0
    for n in checkpoints:
        R.substeps(n - done, scheme)
        done = n
        for nm in "uvwcp":
            _save(folder, f"s{n}_{nm}", R.get(nm))
        _save(folder, f"s{n}_log", R.log())
        g3 = prm.ngz
        d = R.divergence()[prm.ngx:prm.ngx + prm.nx, prm.ngy:prm.ngy + prm.ny, g3:g3 + prm.nz]
        _save(folder, f"s{n}_div", np.array([np.abs(d).max()]))
        del d
    R.close()


class JobSet:
    """The child processes of one test session."""

    def __init__(self, folder):
        self.folder = folder
        self.procs = {}

    def start(self, name):
        if name in self.procs:
            return
        d = os.path.join(self.folder, name)
        os.makedirs(d, exist_ok=True)
        log = open(os.path.join(d, "job.log"), "w")
        self.procs[name] = subprocess.Popen([sys.executable, os.path.abspath(__file__), name, d],
                                            stdout=log, stderr=subprocess.STDOUT, cwd=d)
        log.close()

    def wait(self, name, stem, timeout=3600.0):
        """Load <stem>.npy of job `name`, waiting for it to be written."""
        self.start(name)
        d = os.path.join(self.folder, name)
        path = os.path.join(d, stem + ".npy")
        t0 = time.monotonic()
        while not os.path.exists(path):
            p = self.procs[name]
            if p.poll() is not None and not os.path.exists(path):
                msg = open(os.path.join(d, "job.log")).read()[-2000:]
                raise RuntimeError(f"reference job {name} ended (rc {p.returncode}) without {stem}:\n{msg}")
            if time.monotonic() - t0 > timeout:
                raise TimeoutError(f"reference job {name}: {stem} not ready after {timeout:.0f} s")
            time.sleep(0.5)
        return np.load(path)

    def stop(self):
        for p in self.procs.values():
            if p.poll() is None:
                p.kill()
                p.wait()


if __name__ == "__main__":
    job, out = sys.argv[1], sys.argv[2]
    try:
        run_job(job, out)
    except BaseException as e:   # report, then fail the process
        with open(os.path.join(out, "error.txt"), "w") as f:
            f.write(json.dumps({"job": job, "error": repr(e)}))
        raise
