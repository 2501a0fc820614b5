"""Python host mirror of the chanfast_cuda C ABI (include/chanfast_cuda.h).

The compute path is the CUDA library libchanfast_cuda.so built in this
directory (build.py); this module only binds it with ctypes and mirrors the
reference's driver arguments (chanfast.h:1-21).  There is no CPU fallback:
importing works without a GPU, but every call that needs the engine raises if
the library is missing or no CUDA device is present.

The directory name is not a Python identifier; import it with
``importlib.import_module("ubiquitous-spoon_b200")`` (the repository root on
sys.path).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_CUDA = os.path.join(HERE, "libchanfast_cuda.so")
LIB_DRIVER = os.path.join(HERE, "libchanfast.so")

CF_OK, CF_EINVAL, CF_ENOMEM, CF_ECUDA, CF_EPIVOT, CF_ENONFINITE, CF_EIO, CF_ETIMEOUT = 0, -1, -2, -3, -4, -5, -6, -7
FIELDS = {"u": 0, "v": 1, "w": 2, "c": 3, "p": 4}
LAYOUT_PADDED, LAYOUT_INTERIOR = 0, 1
LOG_COLS = 10
NOALLOC_MAX_ROWS = 8191   # scratch rows of cf_max_divergence_noalloc
KERNEL_GROUPS = ("ghosts", "rhs", "solve", "mass_u", "mass_c", "div_fftx", "ffty_fwd", "poisson", "ffty_bwd",
                 "fftx_c2r", "project")
NKERNEL_GROUPS = len(KERNEL_GROUPS)

_lib = None
_drv = None


class ChanfastError(RuntimeError):
    def __init__(self, status, what):
        super().__init__(f"{what}: status {status} ({strerror(status)})")
        self.status = status


SCHEMES = {"chanfast": 0, "channel": 1}   # CF_SCHEME_CHANFAST, CF_SCHEME_CHANNEL


class Config(ctypes.Structure):
    """Mirror of cf_config."""

    _fields_ = [(n, ctypes.c_int) for n in
                ("order", "nx", "ny", "nz", "ngx", "ngy", "ngz", "uvolavgmode", "cvolavgmode")] + \
               [(n, ctypes.c_double) for n in
                ("lx", "ly", "lz", "dt", "nu", "prandtl", "dpdx", "want_uvolavg", "want_cvolavg",
                 "setuframe", "setvframe", "betg_x", "betg_y", "betg_z")] + \
               [("scheme", ctypes.c_int)]

    @classmethod
    def make(cls, order, nx, ny, nz, lx, ly, lz, dt, nu, prandtl=1.0, dpdx=0.0,
             want_uvolavg=1.0, uvolavgmode=1, want_cvolavg=0.0, cvolavgmode=1,
             setuframe=0.0, setvframe=0.0, betg_x=0.0, betg_y=0.0, betg_z=0.0,
             ngx=3, ngy=3, ngz=3, scheme="chanfast"):
        c = cls()
        for k, v in dict(order=order, nx=nx, ny=ny, nz=nz, ngx=ngx, ngy=ngy, ngz=ngz,
                         uvolavgmode=uvolavgmode, cvolavgmode=cvolavgmode, lx=lx, ly=ly, lz=lz,
                         dt=dt, nu=nu, prandtl=prandtl, dpdx=dpdx, want_uvolavg=want_uvolavg,
                         want_cvolavg=want_cvolavg, setuframe=setuframe, setvframe=setvframe,
                         betg_x=betg_x, betg_y=betg_y, betg_z=betg_z, scheme=SCHEMES[scheme]).items():
            setattr(c, k, v)
        return c

    @classmethod
    def from_params(cls, p, scheme="chanfast"):
        """From any object with the same attribute names (e.g. the oracle's
        Params); `scheme` names the time integration ("chanfast": z-implicit
        diffusion, "channel": fully implicit)."""
        c = cls()
        for name, _ in cls._fields_:
            if name != "scheme":
                setattr(c, name, getattr(p, name))
        c.scheme = SCHEMES[scheme]
        return c

    def padded_shape(self):
        return (self.nx + 2 * self.ngx, self.ny + 2 * self.ngy, self.nz + 2 * self.ngz)

    def interior_shape(self):
        return (self.nx, self.ny, self.nz)


class Request(ctypes.Structure):
    """Mirror of cf_request."""

    _fields_ = [("cfg", Config), ("seed", ctypes.c_ulonglong), ("amp", ctypes.c_double),
                ("c_amp", ctypes.c_double), ("nsteps", ctypes.c_int), ("arrival_s", ctypes.c_double)]


class Result(ctypes.Structure):
    """Mirror of cf_result."""

    _fields_ = [("admit_s", ctypes.c_double), ("finish_s", ctypes.c_double), ("status", ctypes.c_int),
                ("steps_done", ctypes.c_longlong)]


DONE_FN = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p)


def _bind(L):
    vp, ip, dp, ll = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_long
    L.cf_create.argtypes = [ctypes.POINTER(Config), vp, ctypes.POINTER(vp)]
    L.cf_destroy.argtypes = [vp]
    L.cf_set_field.argtypes = [vp, ip, dp, ip]
    L.cf_get_field.argtypes = [vp, ip, dp, ip]
    L.cf_init_fields.argtypes = [vp, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_double]
    L.cf_step.argtypes = [vp, ip]
    L.cf_step_graph.argtypes = [vp, ip]
    L.cf_sync.argtypes = [vp]
    L.cf_get_log.restype = ll
    L.cf_get_log.argtypes = [vp, dp, ll]
    L.cf_substeps_done.restype = ll
    L.cf_substeps_done.argtypes = [vp]
    L.cf_max_divergence.argtypes = [vp, dp]
    L.cf_max_divergence_noalloc.argtypes = [vp, dp]
    L.cf_cfl.argtypes = [vp, ctypes.c_double, dp]
    L.cf_set_dt.argtypes = [vp, ctypes.c_double]
    L.cf_device_field.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_longlong)]
    L.cf_launches_per_substep.argtypes = [vp]
    L.cf_pressure_fused.argtypes = [vp]
    L.cf_debug_stall_copies.argtypes = [vp, ip]
    L.cf_profile.argtypes = [vp, ip, dp]
    L.cf_strerror.restype = ctypes.c_char_p
    L.cf_strerror.argtypes = [ip]
    pvp = ctypes.POINTER(vp)
    L.cf_instance_bytes.restype = ctypes.c_ulonglong
    L.cf_instance_bytes.argtypes = [ctypes.POINTER(Config)]
    L.cf_serve.argtypes = [ctypes.POINTER(Request), ip, ctypes.c_double, ip, ip, vp, DONE_FN, vp,
                           ctypes.POINTER(Result)]
    L.cf_batch_step.argtypes = [pvp, ip, ip, vp]
    L.cf_batch_create.argtypes = [pvp, ip, vp, pvp]
    L.cf_batch_run.argtypes = [vp, ip]
    L.cf_batch_sync.argtypes = [vp]
    L.cf_batch_launches_per_substep.argtypes = [vp]
    L.cf_batch_destroy.argtypes = [vp]
    i4 = ctypes.c_int * 4
    L.cf_set_tuning.argtypes = [ip]
    L.cf_get_launch_shape.argtypes = [vp, i4]
    L.cf_set_launch_shape.argtypes = [vp, i4]
    L.cf_batch_get_launch_shape.argtypes = [vp, i4]
    return L


def lib():
    """The engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_CUDA):
            raise FileNotFoundError(f"{LIB_CUDA} not built; run python ubiquitous-spoon_b200/build.py")
        _lib = _bind(ctypes.CDLL(LIB_CUDA))
    return _lib


def driver_lib():
    """libchanfast.so: the C drop-in drivers chanfast2 / chanfast4 / channel2 / channel4."""
    global _drv
    if _drv is None:
        lib()
        if not os.path.exists(LIB_DRIVER):
            raise FileNotFoundError(f"{LIB_DRIVER} not built")
        D = ctypes.CDLL(LIB_DRIVER)
        args = ([ctypes.c_int] * 11 + [ctypes.c_double] * 5 + [ctypes.c_int] + [ctypes.c_double] * 4
                + [ctypes.c_int] + [ctypes.c_double, ctypes.c_int] + [ctypes.c_double] * 5)
        for name in ("chanfast2_status", "chanfast4_status", "channel2_status", "channel4_status"):
            getattr(D, name).argtypes = args
            getattr(D, name).restype = ctypes.c_int
        _drv = D
    return _drv


def strerror(status):
    try:
        return lib().cf_strerror(status).decode()
    except Exception:
        return "unknown"


def _check(status, what):
    if status != CF_OK:
        raise ChanfastError(status, what)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Instance:
    """One channel-flow state resident on the current CUDA device."""

    def __init__(self, cfg: Config, stream=None):
        self.L = lib()
        self.cfg = cfg
        self.owned = True
        h = ctypes.c_void_p()
        _check(self.L.cf_create(ctypes.byref(cfg), stream, ctypes.byref(h)), "cf_create")
        self.h = h

    @classmethod
    def borrow(cls, handle, cfg):
        """A view of an instance owned elsewhere (the serving loop): usable
        while the owner keeps it alive, never destroyed through the view."""
        v = cls.__new__(cls)
        v.L = lib()
        v.cfg = cfg
        v.owned = False
        v.h = ctypes.c_void_p(handle)
        return v

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            if getattr(self, "owned", True):
                self.L.cf_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_field(self, name, array, layout=LAYOUT_PADDED):
        shape = self.cfg.padded_shape() if layout == LAYOUT_PADDED else self.cfg.interior_shape()
        a = np.ascontiguousarray(array, dtype=np.float64).reshape(shape)
        _check(self.L.cf_set_field(self.h, FIELDS[name], _dp(a), layout), "cf_set_field")

    def get_field(self, name, layout=LAYOUT_PADDED, out=None):
        shape = self.cfg.padded_shape() if layout == LAYOUT_PADDED else self.cfg.interior_shape()
        a = np.empty(shape) if out is None else out
        if a.shape != tuple(shape) or a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of the layout's shape")
        _check(self.L.cf_get_field(self.h, FIELDS[name], _dp(a), layout), "cf_get_field")
        return a

    def init_fields(self, seed, amp, c_amp):
        _check(self.L.cf_init_fields(self.h, seed, amp, c_amp), "cf_init_fields")

    def step(self, nsub):
        _check(self.L.cf_step(self.h, nsub), "cf_step")

    def step_graph(self, nsteps):
        _check(self.L.cf_step_graph(self.h, nsteps), "cf_step_graph")

    def sync(self):
        _check(self.L.cf_sync(self.h), "cf_sync")

    def substeps_done(self):
        return int(self.L.cf_substeps_done(self.h))

    def log(self, max_rows=100000):
        out = np.empty((max_rows, LOG_COLS))
        n = self.L.cf_get_log(self.h, _dp(out), max_rows)
        if n < 0:
            _check(int(n), "cf_get_log")
        return out[:n]

    def max_divergence(self):
        d = ctypes.c_double()
        _check(self.L.cf_max_divergence(self.h, ctypes.byref(d)), "cf_max_divergence")
        return d.value

    def max_divergence_noalloc(self):
        """max |div u| like max_divergence, through the entry point that
        allocates no device memory (fixed scratch; nz <= 8191)."""
        d = ctypes.c_double()
        st = self.L.cf_max_divergence_noalloc(self.h, ctypes.byref(d))
        if st == CF_EINVAL and self.cfg.nz > NOALLOC_MAX_ROWS:
            raise ChanfastError(st, f"cf_max_divergence_noalloc: nz = {self.cfg.nz} exceeds its fixed "
                                    f"scratch of {NOALLOC_MAX_ROWS} wall-normal planes")
        _check(st, "cf_max_divergence_noalloc")
        return d.value

    def cfl(self, dt):
        d = ctypes.c_double()
        _check(self.L.cf_cfl(self.h, dt, ctypes.byref(d)), "cf_cfl")
        return d.value

    def set_dt(self, dt):
        _check(self.L.cf_set_dt(self.h, dt), "cf_set_dt")

    def device_field(self, name):
        p = ctypes.c_void_p()
        n = ctypes.c_longlong()
        _check(self.L.cf_device_field(self.h, FIELDS[name], ctypes.byref(p), ctypes.byref(n)), "cf_device_field")
        return p.value, n.value

    def profile(self, nsub):
        """Per-kernel-group device time (ms, summed over nsub substeps)."""
        ms = np.zeros(NKERNEL_GROUPS)
        _check(self.L.cf_profile(self.h, nsub, _dp(ms)), "cf_profile")
        return dict(zip(KERNEL_GROUPS, ms.tolist()))

    def launches_per_substep(self):
        return int(self.L.cf_launches_per_substep(self.h))

    def debug_stall_copies(self, on):
        """Test hook: the fused pressure launches leave their row copies
        unissued, so their bounded waits run out (cf_sync: CF_ETIMEOUT)."""
        _check(self.L.cf_debug_stall_copies(self.h, int(bool(on))), "cf_debug_stall_copies")

    def pressure_fused(self):
        """True when the y transforms and the Poisson solve run as one launch
        (k_poisson_fft); the profile's y-transform groups are then empty."""
        r = int(self.L.cf_pressure_fused(self.h))
        _check(min(r, 0), "cf_pressure_fused")
        return r == 1

    def launch_shape(self):
        """Tuned launch shape: (back-substitution threads, Poisson threads,
        projection block x, projection block y)."""
        out = (ctypes.c_int * 4)()
        _check(self.L.cf_get_launch_shape(self.h, out), "cf_get_launch_shape")
        return tuple(out)

    def set_launch_shape(self, shape):
        _check(self.L.cf_set_launch_shape(self.h, (ctypes.c_int * 4)(*shape)), "cf_set_launch_shape")


def set_tuning(on):
    """Launch-shape tuning of new instances and batches on (default) or off."""
    _check(lib().cf_set_tuning(1 if on else 0), "cf_set_tuning")


def instance_bytes(cfg):
    """Device bytes an instance of this configuration holds (cf_instance_bytes)."""
    return int(lib().cf_instance_bytes(ctypes.byref(cfg)))


def serve(requests, hbm_budget_bytes, max_active=64, quantum=1, stream=None, on_done=None):
    """Run the serving loop (cf_serve) over `requests`, a list of dicts with
    keys cfg (Config), seed, amp, c_amp, nsteps, arrival_s (seconds after the
    call, non-decreasing).  on_done(index, view) is called as each solve
    retires, with a borrowed Instance view (get_field, log) or None if the
    request failed.  Returns a list of dicts: admit_s, finish_s, status,
    steps_done."""
    L = lib()
    n = len(requests)
    reqs = (Request * n)()
    for q, r in enumerate(requests):
        reqs[q].cfg = r["cfg"]
        reqs[q].seed = r.get("seed", 0)
        reqs[q].amp = r.get("amp", 0.1)
        reqs[q].c_amp = r.get("c_amp", 0.01)
        reqs[q].nsteps = r["nsteps"]
        reqs[q].arrival_s = r.get("arrival_s", 0.0)
    res = (Result * n)()
    errors = []

    def done(index, handle, user):
        if on_done is None:
            return
        try:
            on_done(index, Instance.borrow(handle, requests[index]["cfg"]) if handle else None)
        except Exception as e:   # keep the C loop running; report afterwards
            errors.append(e)

    cb = DONE_FN(done)
    _check(L.cf_serve(reqs, n, float(hbm_budget_bytes), max_active, quantum, stream, cb, None, res), "cf_serve")
    if errors:
        raise errors[0]
    return [dict(admit_s=r.admit_s, finish_s=r.finish_s, status=r.status, steps_done=r.steps_done) for r in res]


def _handles(instances):
    arr = (ctypes.c_void_p * len(instances))()
    for q, inst in enumerate(instances):
        arr[q] = inst.h.value
    return arr


def batch_step(instances, nsub, stream=None):
    """Advance every instance by nsub substeps, one launch per stage of the
    substep for all of them (cf_batch_step)."""
    L = lib()
    _check(L.cf_batch_step(_handles(instances), len(instances), nsub, stream), "cf_batch_step")


class Batch:
    """Instances stepped together by a recorded two-step cycle replayed as
    one CUDA graph (cf_batch_create / cf_batch_run).  The instances stay
    usable for fields and logs; they must not be stepped otherwise while in
    the batch."""

    def __init__(self, instances, stream=None):
        self.L = lib()
        self.instances = list(instances)
        h = ctypes.c_void_p()
        _check(self.L.cf_batch_create(_handles(self.instances), len(self.instances), stream, ctypes.byref(h)),
               "cf_batch_create")
        self.h = h

    def run(self, nsteps):
        _check(self.L.cf_batch_run(self.h, nsteps), "cf_batch_run")

    def sync(self):
        _check(self.L.cf_batch_sync(self.h), "cf_batch_sync")

    def launches_per_substep(self):
        return int(self.L.cf_batch_launches_per_substep(self.h))

    def launch_shape(self):
        out = (ctypes.c_int * 4)()
        _check(self.L.cf_batch_get_launch_shape(self.h, out), "cf_batch_get_launch_shape")
        return tuple(out)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.cf_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def chanfast(order, *args):
    """Call the C drop-in driver chanfast2/chanfast4 (same arguments as the
    reference, chanfast.h:1-21); returns the status instead of aborting."""
    D = driver_lib()
    fn = D.chanfast2_status if order == 2 else D.chanfast4_status
    return fn(*args)


def channel(order, *args):
    """Call the C drop-in driver channel2/channel4 (same arguments as the
    reference, channel.h:1-21); returns the status instead of aborting."""
    D = driver_lib()
    fn = D.channel2_status if order == 2 else D.channel4_status
    return fn(*args)
