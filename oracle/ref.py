"""ctypes access to the compiled reference (oracle/_ref/libchanref.so) -- TEST
INFRASTRUCTURE.

oracle/Makefile builds the library from the unmodified reference sources plus
the single-rank MPI / FFTW shims and oracle/ref_driver.c.  Used by tests/ and
by bench.py's CPU-baseline leg only.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libchanref.so")
# the reference sources: CHANFAST_REFERENCE_SRC, else a checkout named
# `reference` beside this repository
REFERENCE_SRC = os.environ.get("CHANFAST_REFERENCE_SRC") or os.path.abspath(
    os.path.join(HERE, "..", "..", "reference"))

_lock = threading.Lock()
_lib = None


class RefParams(ctypes.Structure):
    """Mirror of ref_params in oracle/ref_driver.c."""

    _fields_ = [(n, ctypes.c_int) for n in
                ("order", "nx", "ny", "nz", "ngx", "ngy", "ngz", "uvolavgmode", "cvolavgmode")] + \
               [(n, ctypes.c_double) for n in
                ("lx", "ly", "lz", "dt", "nu", "prandtl", "dpdx", "want_uvolavg", "want_cvolavg",
                 "setuframe", "setvframe", "betg_x", "betg_y", "betg_z")]


def build(quiet=True):
    """Compile oracle/_ref from the reference sources (needs the reference tree)."""
    if not os.path.isdir(REFERENCE_SRC):
        raise FileNotFoundError(f"reference sources not found at {REFERENCE_SRC}")
    subprocess.run(["make", "-C", HERE, f"REF={REFERENCE_SRC}", "-j8"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not available():
                raise FileNotFoundError(f"{LIB_PATH} missing; run `make -C oracle`")
            L = ctypes.CDLL(LIB_PATH)
            vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
            L.ref_create.restype = vp
            L.ref_create.argtypes = [ctypes.POINTER(RefParams)]
            L.ref_destroy.argtypes = [vp]
            L.ref_dims.argtypes = [vp, ip]
            L.ref_metrics.argtypes = [vp, dp, dp, dp]
            L.ref_set_field.argtypes = [vp, ctypes.c_int, dp]
            L.ref_get_field.argtypes = [vp, ctypes.c_int, dp]
            L.ref_substeps.argtypes = [vp, ctypes.c_long]
            L.ref_channel_substeps.argtypes = [vp, ctypes.c_long]
            L.ref_project.argtypes = [vp, ctypes.c_double]
            L.ref_divergence.argtypes = [vp, dp]
            L.ref_log.restype = ctypes.c_long
            L.ref_log.argtypes = [vp, dp, ctypes.c_long]
            L.ref_case.argtypes = [ctypes.c_int] * 5
            L.ref_chanfast.argtypes = ([ctypes.c_char_p] + [ctypes.c_int] * 10 + [ctypes.c_double] * 5
                                       + [ctypes.c_int] + [ctypes.c_double] * 4 + [ctypes.c_int]
                                       + [ctypes.c_double, ctypes.c_int] + [ctypes.c_double] * 5)
            L.ref_channel.argtypes = L.ref_chanfast.argtypes
            L.shim_set_exact_dft.argtypes = [ctypes.c_int]
            _lib = L
        return _lib


def set_exact_dft(on: bool):
    """Switch the oracle's FFTW stand-in between its recursive mixed-radix
    FFT (default) and a direct DFT summed in long double (see
    oracle/shim/fftw_shim.c); applies to every later transform."""
    lib().shim_set_exact_dft(1 if on else 0)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


SLOTS = {"u": 0, "v": 1, "w": 2, "c": 3, "p": 4, "h": 5,
         "fu": 6, "fv": 7, "fw": 8, "fc": 9, "gu": 10, "gv": 11, "gw": 12, "gc": 13}


class RefInstance:
    """One reference instance: setup of chanfast.c:85-192 plus the substep
    replay of oracle/ref_driver.c."""

    def __init__(self, prm):
        self.L = lib()
        rp = RefParams()
        for name, _ in RefParams._fields_:
            setattr(rp, name, getattr(prm, name))
        self.ctx = self.L.ref_create(ctypes.byref(rp))
        if not self.ctx:
            raise RuntimeError("ref_create failed")
        d = (ctypes.c_int * 3)()
        self.L.ref_dims(self.ctx, d)
        self.shape = (d[0], d[1], d[2])

    def close(self):
        if self.ctx:
            self.L.ref_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.shape)
        assert self.L.ref_set_field(self.ctx, SLOTS[name], _dp(a)) == 0

    def get(self, name):
        a = np.empty(self.shape)
        assert self.L.ref_get_field(self.ctx, SLOTS[name], _dp(a)) == 0
        return a

    def metrics(self):
        n2 = self.shape[2]
        dz, zp, zw = np.empty(n2), np.empty(n2), np.empty(n2)
        self.L.ref_metrics(self.ctx, _dp(dz), _dp(zp), _dp(zw))
        return dz, zp, zw

    def substeps(self, n, scheme="chanfast"):
        """n RK3 substeps of the chanfast (z-implicit) or channel (fully
        implicit, channel.c) scheme."""
        fn = {"chanfast": self.L.ref_substeps, "channel": self.L.ref_channel_substeps}[scheme]
        if fn(self.ctx, n) != 0:
            raise RuntimeError("reference substep aborted (check() failed)")

    def project(self, dt=1.0):
        if self.L.ref_project(self.ctx, dt) != 0:
            raise RuntimeError("reference projection aborted")

    def divergence(self):
        d = np.empty(self.shape)
        if self.L.ref_divergence(self.ctx, _dp(d)) != 0:
            raise RuntimeError("reference divergence aborted")
        return d

    def log(self):
        n = self.L.ref_log(self.ctx, None, 0)
        out = np.empty((max(n, 1), 10))
        self.L.ref_log(self.ctx, _dp(out), n)
        return out[:n]


def run_chanfast(workdir, prm, it, nt, istat=None, cflmode=0, want_cfl=1.0, scheme="chanfast"):
    """Run the unmodified chanfast2/chanfast4 (or, with scheme="channel",
    channel2/channel4) driver in `workdir` (reads outputdir/{u,v,w,c}_it<it>.dat,
    writes *_it<nt>.dat)."""
    L = lib()
    istat = nt - it if istat is None else istat
    fn = {"chanfast": L.ref_chanfast, "channel": L.ref_channel}[scheme]
    rc = fn(workdir.encode(), prm.order, prm.nx, prm.ny, prm.nz, it, nt, istat,
            prm.ngx, prm.ngy, prm.ngz, prm.lx, prm.ly, prm.lz, prm.dt, want_cfl,
            cflmode, prm.nu, prm.prandtl, prm.dpdx, prm.want_uvolavg, prm.uvolavgmode,
            prm.want_cvolavg, prm.cvolavgmode, prm.setuframe, prm.setvframe,
            prm.betg_x, prm.betg_y, prm.betg_z)
    if rc != 0:
        raise RuntimeError(f"{scheme} driver aborted rc={rc}")
