"""The y-slab exchange plan (ubiquitous-spoon_b200/slabs.py) with 2 and 3
gloo ranks on CPU against the single-instance result: halo ghosts equal the
periodic neighbours, a fourth-order y difference on the slabs equals the
whole field's, the transposes move the half spectrum exactly (so the y
transform on kx slabs equals the 2-D transform of the whole field, and the
way back restores every slab), and the all-reduced xy-average profile equals
the whole field's."""
import importlib
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

A1, A2 = 9.0 / 8.0, -1.0 / 24.0   # fourth-order staggered difference weights (fourth.c:3-6)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nx, ny, n2):
    slabs = importlib.import_module("ubiquitous-spoon_b200.slabs")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        P = slabs.SlabPlan(nx, ny, n2, world, rank)
        h, j0, j1, nyl = P.halo, P.j0, P.j1, P.nyl
        F = np.random.default_rng(7).standard_normal((n2, nx, ny))
        # 1. halo exchange
        a = torch.zeros(P.local_shape(), dtype=torch.float64)
        a[:, :, h:h + nyl] = torch.from_numpy(F[:, :, j0:j1])
        P.exchange_halo(a)
        cols = [(j0 - h + c) % ny for c in range(nyl + 2 * h)]
        assert np.array_equal(a.numpy(), F[:, :, cols]), "halo"
        # 2. a y stencil on the slab with its ghosts (the fourth-order
        # divergence term of pressure.c:67-117) equals the whole field's
        loc = a.numpy()
        mine = A1 * (loc[:, :, h:h + nyl] - loc[:, :, h - 1:h - 1 + nyl]) \
            + A2 * (loc[:, :, h + 1:h + 1 + nyl] - loc[:, :, h - 2:h - 2 + nyl])
        whole = A1 * (F - np.roll(F, 1, axis=2)) + A2 * (np.roll(F, -1, axis=2) - np.roll(F, 2, axis=2))
        assert np.array_equal(mine, whole[:, :, j0:j1]), "stencil"
        # 3. transpose to kx slabs and back
        S_full = np.fft.rfft(F, axis=1)                       # x transform: local to every column
        S = torch.from_numpy(np.ascontiguousarray(S_full[:, :, j0:j1]))
        T = P.to_kx_slabs(S)
        assert np.array_equal(T.numpy(), S_full[:, P.kx0:P.kx1, :]), "to_kx_slabs"
        Y = np.fft.fft(T.numpy(), axis=2)                     # whole ky lines: the same transform per line
        full2d = np.fft.fft(S_full, axis=2)[:, P.kx0:P.kx1, :]
        assert np.array_equal(Y, full2d), "y transform on kx slabs"
        back = P.to_y_slabs(torch.from_numpy(np.fft.ifft(Y, axis=2)))
        assert np.array_equal(P.to_y_slabs(T).numpy(), S.numpy()), "to_y_slabs inverts to_kx_slabs"
        x = np.fft.irfft(back.numpy(), n=nx, axis=1)
        assert np.allclose(x, F[:, :, j0:j1], rtol=0, atol=1e-13), "round trip"
        # 4. profile all-reduce
        prof = P.xy_average(a).numpy()
        assert np.allclose(prof, F.mean(axis=(1, 2)), rtol=0, atol=1e-14), "profile"
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nx,ny,n2", [(2, 16, 12, 6), (2, 18, 11, 5), (3, 16, 13, 4)])
def test_slab_exchanges_match_single_instance(world, nx, ny, n2):
    mp.spawn(_worker, args=(world, _free_port(), nx, ny, n2), nprocs=world, join=True)


def test_split_ranges_cover_exactly():
    slabs = importlib.import_module("ubiquitous-spoon_b200.slabs")
    for n in range(1, 40):
        for parts in range(1, 6):
            rs = [slabs.split_range(n, parts, r) for r in range(parts)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(rs[r][1] == rs[r + 1][0] for r in range(parts - 1))
            assert max(b - a for a, b in rs) - min(b - a for a, b in rs) <= 1


def test_slab_narrower_than_halo_is_rejected():
    slabs = importlib.import_module("ubiquitous-spoon_b200.slabs")
    with pytest.raises(ValueError):
        slabs.SlabPlan(16, 8, 4, 4, 0)
