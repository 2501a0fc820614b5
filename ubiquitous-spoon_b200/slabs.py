"""Spanwise (y) slabs: the exchanges of one channel-flow instance spread
over several GPUs, one process per GPU, over torch.distributed (NCCL on
GPUs, gloo on CPU).

The engine runs one instance per GPU.  This module is the exchange plan of
the next step, a single instance on N GPUs; it replaces the reference's MPI
pencil machinery for a y decomposition and runs on any torch.distributed
backend, so its index logic is tested with gloo ranks on CPU
(tests/test_slab_gloo.py).

Rank r owns y columns [j0, j1) of every field in the engine's [k][i][j]
layout (k wall-normal, slowest; x and z whole), with `halo` ghost columns on
both sides.  Per substep:

1. halo exchange -- the stencils reach 3 columns in y (fourth-order
   advection and x-y diffusion, the QUICK scalar fluxes), so each rank sends
   its first and last `halo` interior columns to its y neighbours and
   receives their edge columns into its ghosts; periodic in y.  This is the
   y half of ghostz_periodic / ghost (ghostz.c:107-149); the x half stays a
   modular index inside the kernels.
2. transpose -- the pressure solve transforms x (local: whole x lines), then
   needs whole ky lines for the y transform and whole z columns for the
   per-wavenumber band solve.  One all-to-all moves the half spectrum from
   [k][kx][j0:j1] to [k][kx0:kx1][ky] (kx split into near-equal ranges) and
   one moves it back after the inverse y transform: the reference's
   transpose between pencils (transpose.c:409-448, MPI_Alltoallw).
3. profile all-reduce -- the xy-average profile behind the mass-flux and
   scalar-mean control and the statistics (get_xy_avg, get.c:281-302,
   MPI_Allreduce): each rank sums its columns; one all-reduce of n2 values.

No exchange uses TMA or any other load from a peer's memory: every transfer
is a torch.distributed call into this rank's own buffers.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist


def split_range(n: int, parts: int, index: int) -> tuple[int, int]:
    """[lo, hi) of part `index` of n items split into `parts` contiguous
    ranges whose sizes differ by at most one (the larger ones first)."""
    base, extra = divmod(n, parts)
    lo = index * base + min(index, extra)
    return lo, lo + base + (1 if index < extra else 0)


@dataclass
class SlabPlan:
    """Ownership of one rank: y columns [j0, j1) in physical space, kx rows
    [kx0, kx1) of the half spectrum after the transpose."""
    nx: int
    ny: int
    n2: int
    world: int
    rank: int
    halo: int = 3

    def __post_init__(self):
        self.j0, self.j1 = split_range(self.ny, self.world, self.rank)
        self.nyl = self.j1 - self.j0
        self.nkx = self.nx // 2 + 1
        self.kx0, self.kx1 = split_range(self.nkx, self.world, self.rank)
        if self.nyl < self.halo:
            raise ValueError(f"slab of {self.nyl} columns is narrower than the halo {self.halo}")
        self.left = (self.rank - 1) % self.world
        self.right = (self.rank + 1) % self.world

    # ------------------------------------------------------------ halo
    def local_shape(self):
        """[n2][nx][nyl + 2 halo]: interior columns at halo .. halo + nyl."""
        return (self.n2, self.nx, self.nyl + 2 * self.halo)

    def exchange_halo(self, a: torch.Tensor) -> None:
        """Fill the ghost columns of `a` (local_shape) from the y neighbours'
        edge columns, periodic in y."""
        h, nyl = self.halo, self.nyl
        first = a[:, :, h:2 * h].contiguous()            # -> left neighbour's right ghosts
        last = a[:, :, nyl:nyl + h].contiguous()         # -> right neighbour's left ghosts
        if self.world == 1:
            a[:, :, 0:h] = last
            a[:, :, nyl + h:nyl + 2 * h] = first
            return
        from_left = torch.empty_like(last)
        from_right = torch.empty_like(first)
        # Sends in the order (first, last), receives in the order (from the
        # right, from the left), tagged 1 / 2: with two ranks both
        # neighbours are the same peer, and its `first` must land in the
        # right ghosts, its `last` in the left ones, whether the backend
        # matches by tag (gloo) or by order per peer (NCCL).
        ops = [dist.P2POp(dist.isend, first, self.left, tag=1), dist.P2POp(dist.isend, last, self.right, tag=2),
               dist.P2POp(dist.irecv, from_right, self.right, tag=1),
               dist.P2POp(dist.irecv, from_left, self.left, tag=2)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        a[:, :, 0:h] = from_left
        a[:, :, nyl + h:nyl + 2 * h] = from_right

    # ------------------------------------------------------- transpose
    def _kx_sizes(self):
        return [split_range(self.nkx, self.world, r)[1] - split_range(self.nkx, self.world, r)[0]
                for r in range(self.world)]

    def _y_sizes(self):
        return [split_range(self.ny, self.world, r)[1] - split_range(self.ny, self.world, r)[0]
                for r in range(self.world)]

    def to_kx_slabs(self, s: torch.Tensor) -> torch.Tensor:
        """Half spectrum of this rank's y columns, complex [n2][nkx][nyl]
        (after the x transform), to whole ky lines of this rank's kx rows,
        complex [n2][kx1 - kx0][ny] (for the y transform and the z solve)."""
        ks, ys = self._kx_sizes(), self._y_sizes()
        # send block r: kx rows of rank r, all my columns, packed [r][n2][kx_r][nyl]
        send = torch.cat([s[:, split_range(self.nkx, self.world, r)[0]:split_range(self.nkx, self.world, r)[1], :]
                          .reshape(-1) for r in range(self.world)])
        recv = torch.empty(sum(self.n2 * (self.kx1 - self.kx0) * y for y in ys), dtype=s.dtype, device=s.device)
        self._all_to_all(recv, send, [self.n2 * k * self.nyl for k in ks],
                         [self.n2 * (self.kx1 - self.kx0) * y for y in ys])
        out = torch.empty((self.n2, self.kx1 - self.kx0, self.ny), dtype=s.dtype, device=s.device)
        off = 0
        for r in range(self.world):
            a, b = split_range(self.ny, self.world, r)
            n = self.n2 * (self.kx1 - self.kx0) * (b - a)
            out[:, :, a:b] = recv[off:off + n].reshape(self.n2, self.kx1 - self.kx0, b - a)
            off += n
        return out

    def to_y_slabs(self, t: torch.Tensor) -> torch.Tensor:
        """Inverse of to_kx_slabs: [n2][kx1 - kx0][ny] -> [n2][nkx][nyl]."""
        ks, ys = self._kx_sizes(), self._y_sizes()
        send = torch.cat([t[:, :, split_range(self.ny, self.world, r)[0]:split_range(self.ny, self.world, r)[1]]
                          .reshape(-1) for r in range(self.world)])
        recv = torch.empty(self.n2 * self.nkx * self.nyl, dtype=t.dtype, device=t.device)
        self._all_to_all(recv, send, [self.n2 * (self.kx1 - self.kx0) * y for y in ys],
                         [self.n2 * k * self.nyl for k in ks])
        out = torch.empty((self.n2, self.nkx, self.nyl), dtype=t.dtype, device=t.device)
        off = 0
        for r in range(self.world):
            a, b = split_range(self.nkx, self.world, r)
            n = self.n2 * (b - a) * self.nyl
            out[:, a:b, :] = recv[off:off + n].reshape(self.n2, b - a, self.nyl)
            off += n
        return out

    def _all_to_all(self, recv, send, send_sizes, recv_sizes):
        if self.world == 1:
            recv.copy_(send)
            return
        if send.is_complex():   # exchanged as real pairs
            recv_r, send_r = torch.view_as_real(recv).reshape(-1), torch.view_as_real(send).reshape(-1)
            dist.all_to_all_single(recv_r, send_r, [2 * x for x in recv_sizes], [2 * x for x in send_sizes])
        else:
            dist.all_to_all_single(recv, send, recv_sizes, send_sizes)

    # --------------------------------------------------------- profile
    def xy_average(self, a: torch.Tensor) -> torch.Tensor:
        """get_xy_avg of a field held as this rank's slab (local_shape or
        [n2][nx][nyl]): the n2-long profile, the same on every rank."""
        inner = a[:, :, self.halo:self.halo + self.nyl] if a.shape[2] == self.nyl + 2 * self.halo else a
        prof = inner.sum(dim=(1, 2))
        if self.world > 1:
            dist.all_reduce(prof, op=dist.ReduceOp.SUM)
        return prof / (self.nx * self.ny)
