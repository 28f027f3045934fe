"""Domain decomposition of the cell-centred lens problem into z-slabs: the linearization of a grid
split across ranks (one device each), for grids larger than one GPU.

Rank r owns the cell planes [k0, k1) of the global grid and holds one ghost plane on each side
that has a neighbouring rank. Its device context is the lens problem on the local slab: the same
nx x ny cross-section and cell size, the grid's plane origin (ewg_grid.k_origin) set to the slab's
first global plane so that every cell and face centre, and with them the lens and inlet tests,
are computed from the global plane index exactly as in the whole grid; the permeability of its
planes. A cell's residual row and its Jacobian column depend only on the
cell, its face neighbours and the cached intensive quantities of those, so with the ghost planes
filled from the neighbouring ranks the owned rows of every rank's residual and Jacobian are the
global linearization's rows (the element loop of fvbaselinearizer.hh:401-512 restricted to the
owned elements plus their halo, like the reference's overlapping grid with overlap 1,
parallelbasebackend.hh:511). Rows of ghost cells are not used.

Ghost planes move with point-to-point messages (`exchange_ghosts` over torch.distributed:
NCCL between GPUs, gloo on CPU); `exchange_ghosts_local` does the same between slabs held in one
process. The distributed linear solve (global BiCGStab over the slabs with per-slab ILU(0)) is
not part of this module.
"""
from __future__ import annotations

import copy
import math
from dataclasses import dataclass

import numpy as np

import ewg


@dataclass
class Slab:
    rank: int
    k0: int          # first owned plane (global)
    k1: int          # one past the last owned plane
    ghost_lo: int    # 1 if a lower neighbour rank exists
    ghost_hi: int    # 1 if an upper neighbour rank exists

    @property
    def first(self) -> int:
        """first global plane held (owned or ghost)"""
        return self.k0 - self.ghost_lo

    @property
    def planes(self) -> int:
        return self.k1 - self.k0 + self.ghost_lo + self.ghost_hi


def partition(nz: int, world: int) -> list[Slab]:
    """Balanced z-slabs: the first nz % world ranks own one plane more."""
    if world < 1 or nz < world:
        raise ValueError("need at least one plane per rank")
    base, extra = divmod(nz, world)
    slabs, k = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        slabs.append(Slab(r, k, k + n, 1 if r > 0 else 0, 1 if r < world - 1 else 0))
        k += n
    return slabs


def _slab_extent(hz: float, planes: int) -> float:
    """A z-extent whose cell size (extent / planes, as the library divides) is hz exactly."""
    lz = planes * hz
    for _ in range(64):
        got = lz / planes
        if got == hz:
            return lz
        lz = math.nextafter(lz, math.inf if got < hz else -math.inf)
    raise ValueError("no slab extent reproduces the cell size")


def slab_case(case: ewg.LensCase, slab: Slab) -> ewg.LensCase:
    """The lens problem on one slab (its owned planes and ghost planes): the global problem on a
    grid of slab.planes planes of the global cell size whose plane 0 is global plane slab.first."""
    g = case.grid
    if g.dim != 3 or g.k_origin != 0:
        raise ValueError("slabs split whole 3D grids along z")
    hz = g.lz / g.nz
    grid = ewg.Grid(dim=3, nx=g.nx, ny=g.ny, nz=slab.planes, lx=g.lx, ly=g.ly, lz=_slab_extent(hz, slab.planes),
                    k_origin=slab.first)
    p = copy.deepcopy(case.problem)
    plane = g.nx * g.ny
    perm = np.array(case.perm[slab.first * plane:(slab.first + slab.planes) * plane], copy=True)
    return ewg.LensCase(f"{case.name}_slab{slab.rank}", grid, p, perm, case.dt, case.n_steps)


def local_view(x_global: np.ndarray, grid: ewg.Grid, slab: Slab) -> np.ndarray:
    """A copy of the slab's planes (owned and ghost) of a global natural-order N x 2 field."""
    plane = grid.nx * grid.ny
    return np.array(x_global[slab.first * plane:(slab.first + slab.planes) * plane], copy=True)


def owned_rows(grid: ewg.Grid, slab: Slab) -> slice:
    """Rows of the slab's local natural order that it owns."""
    plane = grid.nx * grid.ny
    return slice(slab.ghost_lo * plane, (slab.ghost_lo + slab.k1 - slab.k0) * plane)


def exchange_ghosts_local(xs: list[np.ndarray], grid: ewg.Grid, slabs: list[Slab]) -> None:
    """Fill every slab's ghost planes from its neighbours' owned planes (slabs in one process)."""
    plane = grid.nx * grid.ny
    for r, s in enumerate(slabs):
        if s.ghost_lo:
            lo = slabs[r - 1]
            src = owned_rows(grid, lo).stop
            xs[r][:plane] = xs[r - 1][src - plane:src]
        if s.ghost_hi:
            hi = slabs[r + 1]
            src = owned_rows(grid, hi).start
            xs[r][-plane:] = xs[r + 1][src:src + plane]


def exchange_ghosts(x_local: np.ndarray, grid: ewg.Grid, slab: Slab, dist) -> None:
    """Fill this rank's ghost planes from the neighbouring ranks: one plane sent and one received
    per neighbour, posted together with torch.distributed.batch_isend_irecv."""
    import torch
    plane = grid.nx * grid.ny
    own = owned_rows(grid, slab)
    t = torch.from_numpy(x_local.reshape(-1, 2))
    ops = []
    if slab.ghost_lo:
        ops.append(dist.P2POp(dist.isend, t[own.start:own.start + plane].contiguous(), slab.rank - 1))
        recv_lo = torch.empty((plane, 2), dtype=t.dtype)
        ops.append(dist.P2POp(dist.irecv, recv_lo, slab.rank - 1))
    if slab.ghost_hi:
        ops.append(dist.P2POp(dist.isend, t[own.stop - plane:own.stop].contiguous(), slab.rank + 1))
        recv_hi = torch.empty((plane, 2), dtype=t.dtype)
        ops.append(dist.P2POp(dist.irecv, recv_hi, slab.rank + 1))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    if slab.ghost_lo:
        x_local[:plane] = recv_lo.numpy()
    if slab.ghost_hi:
        x_local[-plane:] = recv_hi.numpy()


class SlabLinearizer:
    """One rank's slab on its device: set the owned + ghost state, linearize, read the owned rows."""

    def __init__(self, case: ewg.LensCase, slab: Slab):
        self.slab = slab
        self.global_grid = case.grid
        self.case = slab_case(case, slab)
        self.ctx = ewg.Context(self.case)
        self.own = owned_rows(self.case.grid, slab)

    def set_state(self, x_local: np.ndarray, x_old_local: np.ndarray):
        self.ctx.set_solution(1, x_old_local)
        self.ctx.set_solution(0, x_local)

    def linearize(self, dt: float) -> float:
        """Linearizes the slab; returns max |r| over the owned rows (the Newton error's share)."""
        self.ctx.linearize(dt)
        return float(np.max(np.abs(self.owned_residual())))

    def owned_residual(self) -> np.ndarray:
        return self.ctx.residual()[self.own]

    def owned_jacobian(self):
        """(global row of each owned row, BCRS rows of the owned cells with global column indices)."""
        rp, ci, b = self.ctx.jacobian_bcrs()
        plane = self.global_grid.nx * self.global_grid.ny
        shift = self.slab.first * plane
        rows = np.arange(self.own.start, self.own.stop)
        return rows + shift, rp, ci + shift, b

    def close(self):
        self.ctx.close()
