"""cf_max_divergence_noalloc: the divergence check that allocates no device
memory, for callers that cannot call cudaMalloc / cudaFree where they check
the flow (a serving loop whose device memory is fully budgeted to resident
instances, or a monitor between the steps of live instances on other
streams, which cudaFree would stall).  Its partial maxima live in a fixed
file-scope device array of 8191 planes.

Checked through the C ABI against the allocating entry point
cf_max_divergence on two calls in a row (the maximum of the same per-point
values, so equal to the last bit; the bar used elsewhere for divergences is
1e-12), and the size limit is checked.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order,nx,ny,nz", [(2, 32, 24, 16), (4, 64, 48, 40)])
def test_noalloc_matches_allocating_entry(cf, gpu, order, nx, ny, nz):
    cfg = cf.Config.make(order=order, nx=nx, ny=ny, nz=nz, lx=2 * np.pi, ly=np.pi, lz=2.0,
                         dt=1e-3, nu=1e-3, prandtl=0.71)
    L = cf.lib()
    with cf.Instance(cfg) as inst:
        inst.init_fields(11, 0.1, 0.01)
        inst.step(2)   # a non-zero, non-trivial divergence field
        for call in range(2):
            a = ctypes.c_double(-1.0)
            b = ctypes.c_double(-2.0)
            assert L.cf_max_divergence(inst.h, ctypes.byref(a)) == cf.CF_OK
            assert L.cf_max_divergence_noalloc(inst.h, ctypes.byref(b)) == cf.CF_OK
            assert a.value >= 0.0
            assert abs(b.value - a.value) <= 1e-12 * max(1.0, a.value)
            assert b.value == a.value
            inst.step(1)


def test_noalloc_rejects_oversized(cf, gpu):
    cfg = cf.Config.make(order=2, nx=4, ny=4, nz=cf.NOALLOC_MAX_ROWS + 1, lx=1.0, ly=1.0, lz=2.0,
                         dt=1e-3, nu=1e-3)
    with cf.Instance(cfg) as inst:
        out = ctypes.c_double(0.0)
        assert cf.lib().cf_max_divergence_noalloc(inst.h, ctypes.byref(out)) == cf.CF_EINVAL
        with pytest.raises(cf.ChanfastError, match="exceeds its fixed scratch"):
            inst.max_divergence_noalloc()
