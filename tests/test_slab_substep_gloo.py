"""One instance decomposed into y slabs over 2 and 3 gloo ranks on CPU, with
the exchange plan of ubiquitous-spoon_b200/slabs.py, against the same
instance on one rank: the numpy oracle's RK3 substep (chanfast.c:395-656 /
1319-1580) runs per rank on the rank's columns, and its three whole-plane
operations go through the plan:

* periodic halos: x stays local, the y ghosts come from the neighbours
  (exchange_halo; ghostz.c:107-149);
* xy averages for the mass-flux and scalar-mean control: per-rank column
  sums, one all-reduce of the n2-long profile (get.c:281-302);
* the pressure solve: x transform of the rank's columns, transpose to kx
  slabs, y transform and per-wavenumber band solve of the rank's kx rows
  (the mean mode on the rank that holds kx = 0), inverse y transform,
  transpose back, inverse x transform (fft.c:161-208, transpose.c:409-448,
  pressure.c:293-443).

The stencils, transforms and line solves then run on exactly the values the
single rank uses; only the all-reduced profile sums its terms in another
order, which moves the control scalars by rounding.  Bars: relative L2
<= 1e-13 on u, v, w, c and <= 1e-10 on p after three substeps (one RK3
step); the log within a relative 1e-10 (the scalar-mean control divides a
bulk mean near zero by its response, which turns rounding of 1e-16 in the
profile into 1e-12 in dcdt).  With the control off (constant pressure
gradient, no scalar-mean forcing) the profile only enters the logged
statistics, and the decomposed fields equal the single rank's bit for
bit."""
import importlib
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class SlabComm:
    """The oracle's whole-plane operations (chanfast_np.SingleRank) on one
    rank of a y-slab decomposition."""

    def __init__(self, cn, plan, gfull):
        self.cn, self.P, self.gfull = cn, plan, gfull

    def halo(self, a, g):
        gx, n0 = g.p.ngx, g.n0
        a[0:gx] = a[n0 - 2 * gx:n0 - gx]        # x: whole lines on every rank
        a[n0 - gx:n0] = a[gx:2 * gx]
        t = torch.from_numpy(np.ascontiguousarray(a.transpose(2, 0, 1)))   # [k][i][j]
        self.P.exchange_halo(t)
        a[...] = t.numpy().transpose(1, 2, 0)

    def xy_avg(self, a, g):
        p = g.p
        inner = a[p.ngx:p.ngx + p.nx, p.ngy:p.ngy + p.ny, :]
        prof = torch.from_numpy(np.ascontiguousarray(inner.reshape(-1, g.n2).sum(axis=0)))
        dist.all_reduce(prof, op=dist.ReduceOp.SUM)
        return prof.numpy() * (1.0 / (float(self.gfull.p.nx) * float(self.gfull.p.ny)))

    def pressure(self, d, g, dt, order):
        p, P, nx, ny = g.p, self.P, self.gfull.p.nx, self.gfull.p.ny
        inner = d[p.ngx:p.ngx + p.nx, p.ngy:p.ngy + p.ny, :]
        xh = np.fft.rfft(inner, axis=0) * (1.0 / float(nx))                     # [kx][j][k]
        T = P.to_kx_slabs(torch.from_numpy(np.ascontiguousarray(xh.transpose(2, 0, 1)))).numpy()
        ch = np.ascontiguousarray((np.fft.fft(T, axis=2) * (1.0 / float(ny))).transpose(1, 2, 0))
        self.cn.pressure_poisson(ch, self.gfull, dt, order, kx0=P.kx0)        # [kx0:kx1][ky][k]
        yh = np.fft.ifft(ch, axis=1, norm="forward")
        back = P.to_y_slabs(torch.from_numpy(np.ascontiguousarray(yh.transpose(2, 0, 1)))).numpy()
        return np.fft.irfft(back.transpose(1, 2, 0), n=nx, axis=0, norm="forward")


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _worker(rank, world, port, order, nx, ny, nz, control, nsub, betg=(0.0, 0.0, 0.0)):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for q in (root, os.path.join(root, "oracle")):
        if q not in sys.path:
            sys.path.insert(0, q)
    import dataclasses
    import chanfast_np as cn
    import ic
    slabs = importlib.import_module("ubiquitous-spoon_b200.slabs")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=120))
    try:
        prm = cn.Params(order=order, nx=nx, ny=ny, nz=nz, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                        nu=1 / 2800.0, prandtl=0.71, uvolavgmode=1 if control else 0,
                        cvolavgmode=1 if control else 0, betg_x=betg[0], betg_y=betg[1], betg_z=betg[2])
        g = cn.Grid(prm)
        u, v, w, c = ic.raw_state(prm, g.dz, 5, 0.1, 0.01)
        cn.project_initial(u, v, w, prm, g, 1.0)
        P = slabs.SlabPlan(nx, ny, g.n2, world, rank, halo=prm.ngy)
        # this rank's instance: its columns j0 .. j1 with ngy ghost columns on each side
        pl = dataclasses.replace(prm, ny=P.nyl)
        gl = cn.Grid(pl)
        gl.dy = g.dy
        gy = prm.ngy
        cols = slice(P.j0, P.j1 + 2 * gy)    # padded columns j0 - gy .. j1 + gy - 1
        loc = [np.ascontiguousarray(a[:, cols, :]) for a in (u, v, w, c)]
        whole = cn.new_state(u, v, w, c, g)
        mine = cn.new_state(*loc, gl)
        cn.run(whole, prm, g, nsub)
        cn.run(mine, pl, gl, nsub, comm=SlabComm(cn, P, g))
        I = slice(prm.ngx, prm.ngx + nx)
        K = slice(prm.ngz, prm.ngz + nz)
        Jw, Jm = slice(gy + P.j0, gy + P.j1), slice(gy, gy + P.nyl)
        err = {nm: rel(getattr(mine, nm)[I, Jm, K], getattr(whole, nm)[I, Jw, K]) for nm in "uvwcp"}
        same = all(np.array_equal(getattr(mine, nm)[I, Jm, K], getattr(whole, nm)[I, Jw, K]) for nm in "uvwcp")
        la, lb = np.array(mine.log), np.array(whole.log)
        print(f"rank {rank}/{world} o{order} {nx}x{ny}x{nz} control={control}:",
              "bitwise" if same else {k: "%.1e" % e for k, e in err.items()}, flush=True)
        if control:
            assert all(err[nm] <= 1e-13 for nm in "uvwc"), err
            assert err["p"] <= 1e-10, err
            assert np.allclose(la, lb, rtol=1e-10, atol=1e-14), (la, lb)
        else:
            assert same, err
            assert np.allclose(la, lb, rtol=1e-10, atol=1e-14), (la, lb)   # the logged statistics use the profile
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,order,nx,ny,nz", [(2, 4, 16, 12, 8), (3, 4, 12, 11, 7), (2, 2, 12, 9, 6),
                                                  (3, 2, 10, 10, 5)])
def test_slab_substeps_match_single_rank(world, order, nx, ny, nz):
    mp.spawn(_worker, args=(world, _free_port(), order, nx, ny, nz, True, 3), nprocs=world, join=True)


@pytest.mark.parametrize("world,order", [(2, 4), (3, 2)])
def test_slab_substeps_without_control_are_bitwise(world, order):
    mp.spawn(_worker, args=(world, _free_port(), order, 12, 12, 6, False, 3), nprocs=world, join=True)


@pytest.mark.parametrize("order", [2, 4])
def test_slab_substeps_with_buoyancy(order):
    """add_buoyancy (scalar.c:6-76) interpolates c to the u, v, w faces,
    in y across the slab edge: the ghosts carry it."""
    mp.spawn(_worker, args=(2, _free_port(), order, 12, 10, 6, True, 3, (0.3, -0.2, 0.5)), nprocs=2, join=True)
