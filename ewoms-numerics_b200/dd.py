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

    def set_reference_pressure(self, p_ref: float):
        """The finite-difference linearizer's reference pressure: pass the whole grid's (p_w of
        global cell 0, known to the bottom slab), so the slab's deflections are the whole
        grid's."""
        self.ctx.set_reference_pressure(p_ref)

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


# ------------------------------------------------------------------------------------------
# Distributed solve over the slabs: BiCGStab with restricted additive Schwarz

DBL_BREAKDOWN = 2.2250738585072014e-308 * 1e10  # DBL_MIN * 1e10, the solver's breakdown threshold
ST_RUNNING, ST_CONVERGED, ST_FAILED, ST_BREAKDOWN, ST_MAXITER = 0, 1, 2, 3, 4


class SplitLayout:
    """Row ranges of a slab's device vectors (the context's red-black storage order: plane k of
    local colour c is the run c*N/2 + k*nx*ny/2 of nx*ny/2 rows). Plane chunks are listed in
    GLOBAL colour order, (i + j + k_global) & 1, so that two slabs whose first planes differ in
    parity still pair the same cells."""

    def __init__(self, grid: ewg.Grid, slab: Slab):
        plane = grid.nx * grid.ny
        self.half = grid.n_cells // 2
        self.planeh = plane // 2
        self.flip = slab.first & 1
        self.owned = [slice(c * self.half + slab.ghost_lo * self.planeh,
                            c * self.half + (slab.ghost_lo + slab.k1 - slab.k0) * self.planeh) for c in (0, 1)]
        self._own = slice(self.owned[0].start, self.owned[0].stop)

    def owned_view(self, a):
        """The owned rows of both colours as one strided view (colour, row, component): the two
        colours' owned runs start at the same offset within their halves."""
        return a.view(2, self.half, 2)[:, self._own]

    def plane(self, k: int) -> list[slice]:
        out = []
        for g in (0, 1):
            s = (g ^ self.flip) * self.half + k * self.planeh
            out.append(slice(s, s + self.planeh))
        return out


class NaturalLayout:
    """Row ranges of a slab vector in natural order (k slowest)."""

    def __init__(self, grid: ewg.Grid, slab: Slab):
        self.planesz = grid.nx * grid.ny
        self.owned = [slice(slab.ghost_lo * self.planesz, (slab.ghost_lo + slab.k1 - slab.k0) * self.planesz)]

    def owned_view(self, a):
        return a[self.owned[0]]

    def plane(self, k: int) -> list[slice]:
        return [slice(k * self.planesz, (k + 1) * self.planesz)]


def _bottom_owned(s: Slab) -> int:
    return s.ghost_lo


def _top_owned(s: Slab) -> int:
    return s.ghost_lo + s.k1 - s.k0 - 1


class LocalComm:
    """All slabs in this process: a ghost exchange copies planes between the slabs' vectors and a
    reduction combines the slabs' partial values. Used to run the distributed algorithm on one
    device. No kernel waits on another: the plane copies run on the current stream after it has
    waited for every slab's stream, and the slabs' streams wait for the copies (a host
    synchronization instead where a slab has no stream)."""

    def exchange(self, parts, vecs):
        import torch
        if not any(sp.slab.ghost_lo or sp.slab.ghost_hi for sp in parts):
            return
        cuda = any(v.is_cuda for v in vecs)
        streams = [getattr(sp, "stream", None) for sp in parts]
        ordered = cuda and all(st is not None for st in streams)
        if ordered:
            cur = torch.cuda.current_stream()
            for st in streams:
                cur.wait_stream(st)
        elif cuda:
            torch.cuda.synchronize()
        for r, (sp, v) in enumerate(zip(parts, vecs)):
            s, L = sp.slab, sp.layout
            if s.ghost_lo:
                lo = parts[r - 1]
                for d, src in zip(L.plane(0), lo.layout.plane(_top_owned(lo.slab))):
                    v[d] = vecs[r - 1][src]
            if s.ghost_hi:
                hi = parts[r + 1]
                for d, src in zip(L.plane(s.planes - 1), hi.layout.plane(_bottom_owned(hi.slab))):
                    v[d] = vecs[r + 1][src]
        if ordered:
            for st in streams:
                st.wait_stream(cur)
        elif cuda:
            torch.cuda.synchronize()

    def reduce_device(self, vals, parts=None):
        """The sum over the slabs of one partial tensor each, left on the device (no host read).
        With several slabs the sum runs on the current stream after it has waited for every
        slab's stream, and the slabs' streams wait for the sum (device synchronizations instead
        where a slab has no stream)."""
        import torch
        if len(vals) == 1:
            return vals[0]
        cuda = any(v.is_cuda for v in vals)
        streams = [getattr(sp, "stream", None) for sp in (parts or [])]
        ordered = cuda and len(streams) == len(vals) and all(st is not None for st in streams)
        if ordered:
            cur = torch.cuda.current_stream()
            for st in streams:
                cur.wait_stream(st)
        elif cuda:
            torch.cuda.synchronize()
        out = torch.stack(vals).sum(0)
        if ordered:
            for st in streams:
                st.wait_stream(cur)
        elif cuda:
            torch.cuda.synchronize()
        return out

    def reduce_device_mixed(self, vals, nsum, parts=None):
        """One 1-D partial tensor per slab combined on the device: the first nsum entries summed
        over the slabs (in slab order), the rest maximised; no host read."""
        import torch
        if len(vals) == 1:
            return vals[0]
        cuda = any(v.is_cuda for v in vals)
        streams = [getattr(sp, "stream", None) for sp in (parts or [])]
        ordered = cuda and len(streams) == len(vals) and all(st is not None for st in streams)
        if ordered:
            cur = torch.cuda.current_stream()
            for st in streams:
                cur.wait_stream(st)
        elif cuda:
            torch.cuda.synchronize()
        g = torch.stack(vals)
        out = torch.cat([g[:, :nsum].sum(0), g[:, nsum:].amax(0)])
        if ordered:
            for st in streams:
                st.wait_stream(cur)
        elif cuda:
            torch.cuda.synchronize()
        return out

    def reduce(self, vals, nsum):
        """vals: one 1-D tensor of partials per slab, the first nsum summed over the slabs and the
        rest maximised. One host read per slab. The partials were computed on the slabs' own
        (non-blocking) streams, so the device is synchronized before they are read."""
        import torch
        if any(v.is_cuda for v in vals):
            torch.cuda.synchronize()
        rows = np.array([v.tolist() for v in vals], dtype=np.float64)
        return _combine(rows, nsum)


def _combine(rows, nsum):
    """Sums of the first nsum columns, maxima of the rest; a NaN maximum reads as infinity, so a
    non-finite residual fails the convergence tests instead of passing them silently."""
    maxes = np.max(rows[:, nsum:], axis=0)
    return ([float(x) for x in np.sum(rows[:, :nsum], axis=0)],
            [math.inf if math.isnan(x) else float(x) for x in maxes])


class TorchComm:
    """One slab per rank of a torch.distributed process group (rank == slab.rank): a ghost
    exchange is one plane per neighbour and direction (batch_isend_irecv), a reduction is one
    all_gather of the ranks' partials. NCCL between GPUs, gloo on CPU."""

    def __init__(self, dist):
        self.dist = dist

    def exchange(self, parts, vecs):
        import torch
        dist = self.dist
        (sp,), (v,) = parts, vecs
        s, L = sp.slab, sp.layout
        ops, recv = [], []
        for flag, peer, send_k, recv_k in ((s.ghost_lo, s.rank - 1, _bottom_owned(s), 0),
                                           (s.ghost_hi, s.rank + 1, _top_owned(s), s.planes - 1)):
            if not flag:
                continue
            buf = torch.cat([v[c] for c in L.plane(send_k)])
            into = torch.empty_like(buf)
            ops.append(dist.P2POp(dist.isend, buf, peer))
            ops.append(dist.P2POp(dist.irecv, into, peer))
            recv.append((recv_k, into))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for k, into in recv:
            o = 0
            for c in L.plane(k):
                n = c.stop - c.start
                v[c] = into[o:o + n]
                o += n

    def reduce_device(self, vals, parts=None):
        """The sum over the ranks of this rank's partial tensor, left on the device: one
        all_gather, summed in rank order, so every rank holds the same bits."""
        import torch
        (x,) = vals
        x = x.to(self._device).reshape(1)
        g = [torch.empty_like(x) for _ in range(self.dist.get_world_size())]
        self.dist.all_gather(g, x)
        return torch.stack(g).sum(0).reshape(())

    def reduce_device_mixed(self, vals, nsum, parts=None):
        """This rank's partials combined over the ranks on the device (one all_gather, combined in
        rank order): the first nsum entries summed, the rest maximised."""
        import torch
        (x,) = vals
        x = x.to(self._device).reshape(-1)
        g = [torch.empty_like(x) for _ in range(self.dist.get_world_size())]
        self.dist.all_gather(g, x)
        st = torch.stack(g)
        return torch.cat([st[:, :nsum].sum(0), st[:, nsum:].amax(0)])

    def reduce(self, vals, nsum):
        """One all_gather of this rank's partials (a 1-D tensor, the first nsum summed and the rest
        maximised over the ranks); every rank combines the same gathered rows in rank order, so
        all ranks take the same branches."""
        import torch
        (x,) = vals
        x = x.to(self._device)
        g = [torch.empty_like(x) for _ in range(self.dist.get_world_size())]
        self.dist.all_gather(g, x)
        return _combine(np.array(torch.stack(g).tolist(), dtype=np.float64), nsum)

    @property
    def _device(self):
        import torch
        backend = self.dist.get_backend()
        return torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")


# Partials over a slab's owned rows as device tensors (no host read); a reduction point stacks
# them into one vector, so a slab reads its partials back once and the ranks combine them in one
# collective.

def _dev_dot(L, a, b):
    return (L.owned_view(a) * L.owned_view(b)).sum()


def _dev_max(L, a):
    """max |a| over the owned rows (NaN propagates; the host reads it as infinity)."""
    import torch
    o = L.owned_view(a)
    return torch.linalg.vector_norm(o, float("inf")) if o.numel() else a.new_zeros(())


def _pack(sums, maxes):
    import torch
    return torch.stack(list(sums) + list(maxes))


class DeviceSlab:
    """One slab's device operators for the distributed solve: SpMV and preconditioner of its
    context on its stream, vectors in the context's storage order."""

    def __init__(self, lin: SlabLinearizer, opts=None):
        import torch
        self.lin = lin
        self.slab = lin.slab
        self.ctx = lin.ctx
        self.layout = SplitLayout(lin.case.grid, lin.slab)
        self.opts = opts or ewg.default_solve_opts()
        self.stream = torch.cuda.ExternalStream(self.ctx.stream)
        self.n = self.ctx.n

    def on(self):
        import torch
        return torch.cuda.stream(self.stream)

    def zeros(self):
        import torch
        return torch.zeros((self.n, 2), dtype=torch.float64, device="cuda")

    def rhs(self):
        return self.ctx.device_buffer(ewg.BUFFER_RESIDUAL)

    def solution(self):
        return self.ctx.device_buffer(ewg.BUFFER_SOLUTION)

    def spmv(self, x, y):
        self.ctx.device_spmv(x, y)

    def precondition(self, b, y):
        self.ctx.device_precondition(b, y, self.opts)

    # the fused kernels of one slab-iteration (ewg_device_bicg_*): vector updates with their
    # owned-row reductions in one pass each, scalars from the device state, results on the device
    def _reduction_slots(self):
        import torch
        if not hasattr(self, "_red"):
            self._red = torch.zeros(16, dtype=torch.float64, device="cuda")
        return self._red, self.layout._own.start, self.layout._own.stop

    def new_state(self):
        import torch
        return torch.zeros(self.ctx.lib.ewg_device_bicg_state_size(), dtype=torch.uint8, device="cuda")

    def dev_p(self, v, state):
        self.ctx.device_bicg_p(v.p, v.r, v.r0, v.v, state)

    def dev_spmv_dot(self, x, y, w, state):
        red, lo, hi = self._reduction_slots()
        out = red[0:1]
        self.ctx.device_bicg_spmv_dot(x, y, w, lo, hi, state, out)
        return out

    def dev_hs(self, v, state):
        red, lo, hi = self._reduction_slots()
        out = red[2:4]
        self.ctx.device_bicg_hs(v.x, v.y, v.r, v.v, lo, hi, state, out)
        return out

    def dev_spmv_dot2(self, z, t, s, state):
        red, lo, hi = self._reduction_slots()
        out = red[4:6]
        self.ctx.device_bicg_spmv_dot2(z, t, s, lo, hi, state, out)
        return out

    def dev_xr(self, v, state):
        red, lo, hi = self._reduction_slots()
        out = red[8:12]
        self.ctx.device_bicg_xr(v.x, v.z, v.r, v.t, v.r0, lo, hi, state, out)
        return out


class _Vecs:
    pass


class _TorchOps:
    """The fused steps of one slab's BiCGStab iteration written with torch operations, for slabs
    without device kernels (the CPU oracle slabs of the tests). DeviceSlab runs the same steps as
    single kernels (ewg_device_bicg_*), each with its owned-row reductions."""

    def __init__(self, p):
        self.p = p

    def bicg_p(self, v, beta, omega, restart):
        if restart:
            v.r0.copy_(v.r)
            v.v.zero_()
            v.p.zero_()
        v.p.sub_(v.v, alpha=omega).mul_(beta).add_(v.r)

    def bicg_spmv_dot(self, x, y, w):
        self.p.spmv(x, y)
        return _dev_dot(self.p.layout, w, y)

    def bicg_hs(self, v, rho_i, denom):
        alpha_dev = rho_i / denom
        v.x.addcmul_(v.y, alpha_dev)
        v.r.addcmul_(v.v, alpha_dev, value=-1.0)
        return [_dev_max(self.p.layout, v.r), _dev_max(self.p.layout, v.y)]

    def bicg_spmv_dot2(self, z, t, s):
        self.p.spmv(z, t)
        return [_dev_dot(self.p.layout, t, t), _dev_dot(self.p.layout, t, s)]

    def bicg_xr(self, v, omega):
        v.x.add_(v.z, alpha=omega)
        m = [_dev_max(self.p.layout, v.r), _dev_max(self.p.layout, v.z)]
        v.r.sub_(v.t, alpha=omega)
        return _pack([_dev_dot(self.p.layout, v.r0, v.r), _dev_dot(self.p.layout, v.r, v.r)], m)


def _ops(p):
    return _TorchOps(p)


def _bicgstab(parts, comm, opts):
    """Solve J dx = b over the slabs, b = the owned rows of each slab's rhs(), dx in the slabs'
    layouts (owned rows meaningful). BiCGStabSolver::apply with CombinedCriterion
    (linear/bicgstabsolver.hh:116-326, linear/combinedcriterion.hh:112-205) in the same steps
    and scalar updates as the single-domain device solver, with every dot product and max-norm
    taken over the owned rows of all slabs and the preconditioner applied
    as restricted additive Schwarz: the ghost planes of the preconditioned vector come from the
    neighbours, each slab applies its own M^-1 (block ILU(0) or Jacobi of the slab matrix,
    ghost rows included), and only the owned rows are kept. Ghost planes of a vector are
    refreshed before every SpMV. The partials of an iteration meet in three reductions, one
    collective each: <r0,v> stays on the device (alpha = rho_i / <r0,v> is formed there); the
    half-step max-norms of s and y together with <t,t>, <t,s> and <r0,v> (z and t are computed
    before the half-step check and left unused when it ends the solve), one host read per slab;
    the full-step max-norms of s and z with <r0,r> and <r,r>, one host read per slab. A zero
    max-norm of y or z is the stagnation test.

    Returns (status, iterations, restarts, final residual, initial residual, [dx per slab])."""
    import contextlib
    import torch
    on = [getattr(p, "on", contextlib.nullcontext) for p in parts]
    V = []
    bb_l, bm_l = [], []
    for p, o in zip(parts, on):
        with o():
            v = _Vecs()
            v.b = p.rhs().clone()
            v.x, v.v, v.p, v.y, v.z, v.t = (p.zeros() for _ in range(6))
            v.r = v.b.clone()
            v.r0 = v.b.clone()
            bb_l.append(_pack([_dev_dot(p.layout, v.b, v.b)], [_dev_max(p.layout, v.b)]))
            V.append(v)
    (bb,), (bmax,) = comm.reduce(bb_l, 1)
    S = dict(resErr=max(bmax, DBL_BREAKDOWN), iter=0, restarts=0, restartPending=0, rho=1.0, alpha=1.0,
             omega=1.0, r0r0=bb, status=ST_RUNNING, replacements=0, beta=0.0, rho_i=0.0)
    S["initResErr"] = S["resErr"]
    relTol, absTol = opts.linear_solver_tolerance, opts.linear_solver_abs_tolerance
    maxRes, maxIter = opts.linear_solver_max_error, opts.linear_solver_max_iterations

    def criterion(stagnates):
        red = S["resErr"] / max(1e-20, S["initResErr"])
        if red <= relTol or S["resErr"] <= absTol:
            S["status"] = ST_CONVERGED
        elif stagnates or S["resErr"] > maxRes:
            S["status"] = ST_FAILED

    def iteration_top(rho_i, rr):
        if S["iter"] >= maxIter:
            S["status"] = ST_MAXITER
            return
        if opts.restart_on_breakdown and abs(rho_i) <= 1e-12 * math.sqrt(S["r0r0"]) * math.sqrt(rr):
            S["restartPending"] = 1
            S["r0r0"] = rr
            rho_i = rr
            S["rho"] = S["alpha"] = S["omega"] = 1.0
            S["restarts"] += 1
        if abs(S["rho"]) <= DBL_BREAKDOWN or abs(S["omega"]) <= DBL_BREAKDOWN:
            S["status"] = ST_BREAKDOWN
            return
        S["beta"] = (rho_i / S["rho"]) * (S["alpha"] / S["omega"])
        S["rho"] = rho_i
        S["rho_i"] = rho_i

    def each(fn):
        out = []
        for p, v, o in zip(parts, V, on):
            with o():
                out.append(fn(p, v))
        return out

    def exchange(name):
        comm.exchange(parts, [getattr(v, name) for v in V])

    if S["resErr"] / max(1e-20, S["initResErr"]) <= relTol or S["resErr"] <= absTol:
        S["status"] = ST_CONVERGED
    else:
        iteration_top(bb, bb)
    while True:
        while S["status"] == ST_RUNNING:
            restart, beta, omega = S["restartPending"], S["beta"], S["omega"]

            each(lambda p, v: _ops(p).bicg_p(v, beta, omega, restart))
            exchange("p")
            each(lambda p, v: p.precondition(v.p, v.y))
            exchange("y")
            # <r0,v> stays on the device: alpha = rho_i / <r0,v> is formed there, and <r0,v> reaches
            # the host with the next read-back, where the breakdown tests run (x and r have moved
            # by then, which a breakdown makes moot)
            d_dev = comm.reduce_device(each(lambda p, v: _ops(p).bicg_spmv_dot(v.y, v.v, v.r0)), parts)
            S["restartPending"] = 0
            rho_i = S["rho_i"]

            def upd_hs(p, v):
                m = _ops(p).bicg_hs(v, rho_i, d_dev)
                # exactly one slab (the bottom one) carries <r0,v> in its sums
                v.half = ([d_dev if p.slab.k0 == 0 else torch.zeros_like(d_dev)], m)
            each(upd_hs)
            # the half-step check travels with <t,t> and <t,s>: z = M^-1 s and t = J z are
            # computed before it is known, and left unused when the half step ends the solve
            exchange("r")
            each(lambda p, v: p.precondition(v.r, v.z))
            exchange("z")
            (tt, ts, d), (smax, ymax) = comm.reduce(
                each(lambda p, v: _pack(_ops(p).bicg_spmv_dot2(v.z, v.t, v.r) + v.half[0], v.half[1])), 3)
            if abs(d) <= DBL_BREAKDOWN:
                S["status"] = ST_BREAKDOWN
                break
            S["alpha"] = rho_i / d
            if abs(S["alpha"]) <= DBL_BREAKDOWN:
                S["status"] = ST_BREAKDOWN
                break
            S["resErr"] = smax
            criterion(ymax == 0.0)  # the update y stagnates when it is all zero
            if S["status"] != ST_RUNNING:
                break
            if abs(tt) <= DBL_BREAKDOWN:
                S["status"] = ST_BREAKDOWN
                break
            S["omega"] = ts / tt
            if abs(S["omega"]) <= DBL_BREAKDOWN:
                S["status"] = ST_BREAKDOWN
                break
            omega = S["omega"]

            (rr0, rr), (smax, zmax) = comm.reduce(each(lambda p, v: _ops(p).bicg_xr(v, omega)), 2)
            S["resErr"] = smax
            criterion(zmax == 0.0)
            if S["status"] != ST_RUNNING:
                break
            S["iter"] += 1
            iteration_top(rr0, rr)
        if not (S["status"] == ST_CONVERGED and opts.verify_true_residual and S["replacements"] < 3):
            break
        # residual replacement: r = r0hat = b - J x; resume if it misses the criterion by 10x
        exchange("x")

        def true_res(p, v):
            p.spmv(v.x, v.t)
            torch.sub(v.b, v.t, out=v.r)
            v.r0.copy_(v.r)
            v.v.zero_()
            v.p.zero_()
            return _pack([_dev_dot(p.layout, v.r, v.r)], [_dev_max(p.layout, v.r)])
        (rr,), (err,) = comm.reduce(each(true_res), 1)
        if err / max(1e-20, S["initResErr"]) <= 10 * relTol or err <= 10 * absTol:
            break
        S["replacements"] += 1
        S["restarts"] += 1
        S["status"] = ST_RUNNING
        S["resErr"] = err
        S["restartPending"] = 0
        S["rho"] = S["alpha"] = S["omega"] = 1.0
        S["r0r0"] = rr
        S["iter"] += 1
        iteration_top(rr, rr)
    return S["status"], S["iter"], S["restarts"], S["resErr"], S["initResErr"], [v.x for v in V]


def _bicgstab_device(parts, comm, opts, check_every=4):
    """_bicgstab with every scalar on the device, for slabs with device kernels (DeviceSlab): the
    fused kernels (ewg_device_bicg_*) update the vectors and reduce over the owned rows, the
    reductions are combined over the slabs on the device (comm.reduce_device_mixed, one collective
    each), and each slab's copy of the BiCGStab state takes the same scalar step on them
    (ewg_device_bicg_state). The host reads the state every check_every iterations; kernels
    launched after the solve has ended return at once. Same steps, tests and results as
    _bicgstab (the dot products are summed in another order)."""
    import torch
    V = []
    for p in parts:
        with p.on():
            v = _Vecs()
            v.b = p.rhs().clone()
            v.x, v.v, v.p, v.y, v.z, v.t = (p.zeros() for _ in range(6))
            v.r = v.b.clone()
            v.r0 = v.b.clone()
            v.state = p.new_state()
            V.append(v)

    def each(fn):
        out = []
        for p, v in zip(parts, V):
            with p.on():
                out.append(fn(p, v))
        return out

    def exchange(name):
        comm.exchange(parts, [getattr(v, name) for v in V])

    def combine(vals, nsum):
        return comm.reduce_device_mixed(vals, nsum, parts)

    def stage(k, red, o=None):
        each(lambda p, v: p.ctx.device_bicg_state(k, v.state, red, o))

    def read():
        return parts[0].ctx.device_bicg_state_read(V[0].state)

    stage(0, combine(each(lambda p, v: _pack([_dev_dot(p.layout, v.b, v.b)], [_dev_max(p.layout, v.b)])), 1), opts)
    replacements = 0
    while True:
        st = read()
        while st[0] == ST_RUNNING:
            for _ in range(check_every):
                each(lambda p, v: p.dev_p(v, v.state))
                exchange("p")
                each(lambda p, v: p.precondition(v.p, v.y))
                exchange("y")
                stage(1, combine(each(lambda p, v: p.dev_spmv_dot(v.y, v.v, v.r0, v.state)), 1))
                each(lambda p, v: setattr(v, "half", p.dev_hs(v, v.state)))
                exchange("r")
                each(lambda p, v: p.precondition(v.r, v.z))
                exchange("z")
                # {t.t, t.s} with the half step's {max|s|, max|y|}, joined on each slab's stream
                stage(2, combine(each(lambda p, v: torch.cat([p.dev_spmv_dot2(v.z, v.t, v.r, v.state), v.half])), 2))
                stage(3, combine(each(lambda p, v: p.dev_xr(v, v.state)), 2))
            st = read()
        if not (st[0] == ST_CONVERGED and opts.verify_true_residual and replacements < 3):
            break
        # residual replacement: r = r0hat = b - J x; resume if it misses the criterion by 10x
        exchange("x")

        def true_res(p, v):
            p.spmv(v.x, v.t)
            torch.sub(v.b, v.t, out=v.r)
            v.r0.copy_(v.r)
            v.v.zero_()
            v.p.zero_()
            return _pack([_dev_dot(p.layout, v.r, v.r)], [_dev_max(p.layout, v.r)])
        stage(4, combine(each(true_res), 1))
        st = read()
        if st[0] != ST_RUNNING:
            break
        replacements += 1
    status, its, restarts, res, init = st
    return status, its, restarts, res, init, [v.x for v in V]


def _single_stream(parts):
    """With one slab in this process, all its work (kernels, torch ops, collectives) runs on its
    context's stream; with several, each slab's work enters its own stream and the exchanges
    synchronize the device."""
    import contextlib
    if len(parts) == 1 and hasattr(parts[0], "on"):
        return parts[0].on()
    return contextlib.nullcontext()


def distributed_bicgstab(parts, comm, opts):
    """Distributed BiCGStab over the slabs in `parts`: device-resident (_bicgstab_device) when
    every slab has device kernels, else with the scalars on the host (_bicgstab)."""
    with _single_stream(parts):
        if parts and all(isinstance(p, DeviceSlab) for p in parts) and hasattr(comm, "reduce_device_mixed"):
            return _bicgstab_device(parts, comm, opts)
        return _bicgstab(parts, comm, opts)


class DistributedNewtonReport:
    def __init__(self):
        self.iterations = 0
        self.linear_iterations = 0
        self.error = 0.0
        self.status = ewg.EWG_OK
        self.converged = False


def distributed_newton(parts, comm, dt, nopts=None, sopts=None) -> DistributedNewtonReport:
    """NewtonMethod::apply (newtonmethod.hh:308-517) over the slabs, after updateBegin (every
    slab takes the whole grid's reference pressure for the finite-difference linearizer): each
    iteration linearizes
    every slab, takes the error as the maximum |r| over all owned rows, solves with
    distributed_bicgstab, subtracts the update from the owned rows of solution(0) and refreshes
    the ghost planes from the neighbours. The stopping rules are the single-domain ones
    (proceed_: at least one iteration, stop when error <= tolerance, past the iteration limit
    continue only while the error shrinks 4x per iteration). Each part is a DeviceSlab whose
    context holds solution(0) with consistent ghost planes and the storage of solution(1)."""
    import torch
    nopts = nopts or ewg.default_newton_opts()
    sopts = sopts or ewg.default_solve_opts()
    rep = DistributedNewtonReport()
    with _single_stream(parts):
        error, last = 1e100, 1e100
        it = 0

        def converged():
            return error <= nopts.newton_tolerance

        def proceed():
            if it < 1:
                return True
            if converged():
                return False
            if it >= nopts.newton_max_iterations:
                return error * 4.0 < last
            return True

        # updateBegin before the solve, as ewg_newton_apply does: every slab takes the whole
        # grid's reference pressure, p_w of global cell 0 (position 0 of the bottom slab's
        # solution(0) in either storage order); only the finite-difference linearizer reads it
        refs = []
        for p in parts:
            with p.on():
                x = p.solution()
                refs.append(_pack([x[0, 0] if p.slab.k0 == 0 else x.new_zeros(())], []))
        (p_ref,), _ = comm.reduce(refs, 1)
        for p in parts:
            p.ctx.set_reference_pressure(p_ref)
        while proceed():
            last = error
            errs = []
            for p in parts:
                with p.on():
                    p.ctx.linearize(dt)
                    errs.append(_pack([], [_dev_max(p.layout, p.rhs())]))
            _, (error,) = comm.reduce(errs, 0)
            if error > nopts.newton_max_error:
                rep.status = ewg.EWG_ERR_MAX_ERROR
                break
            if not proceed():
                it += 1
                break
            st, its, _, _, _, dxs = distributed_bicgstab(parts, comm, sopts)
            rep.linear_iterations += its
            if st != ST_CONVERGED:
                rep.status = ewg.EWG_ERR_BREAKDOWN if st == ST_BREAKDOWN else ewg.EWG_ERR_NOT_CONVERGED
                break
            bad = []
            for p, dx in zip(parts, dxs):
                with p.on():
                    x = p.solution()
                    b = x.new_zeros(())
                    for sl in p.layout.owned:
                        b = torch.maximum(b, (~dx[sl].isfinite()).any().to(x.dtype))
                        x[sl] -= dx[sl]
                    bad.append(_pack([], [b]))
            if comm.reduce(bad, 0)[1][0] != 0.0:
                rep.status = ewg.EWG_ERR_NONFINITE
                break
            comm.exchange(parts, [p.solution() for p in parts])
            it += 1
    rep.iterations = it
    rep.error = error
    if rep.status == ewg.EWG_OK and not converged():
        rep.status = ewg.EWG_ERR_NOT_CONVERGED
    rep.converged = rep.status == ewg.EWG_OK
    return rep


def main(argv=None) -> None:
    """Times one implicit-Euler step of the 3D lens problem on one device: the single-domain
    Newton (ewg_newton_apply) and distributed_newton over 1, 2, ... z-slabs held as separate
    contexts in this process (LocalComm). Both start from the state after one warm-up step, each
    form runs the step once untimed and once timed; the time is host wall clock between device
    synchronizations (the distributed loop is host-orchestrated over several streams). Prints one
    JSON line per form, with the final state's distance from the single-domain step.

    python ewoms-numerics_b200/dd.py --grid 128,128,64 --slabs 1,2,4"""
    import argparse
    import json
    import time
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", default="128,128,64")
    ap.add_argument("--slabs", default="1,2,4")
    ap.add_argument("--dt", type=float, default=250.0)
    ap.add_argument("--linear-tol", type=float, default=1e-3)
    # one ILU(0) order for every form, so that the forms differ only in the decomposition (the
    # box-8 order needs slab plane counts divisible by 4, which ghost planes rarely give)
    ap.add_argument("--ilu-ordering", default="redblack", choices=["redblack", "box8", "auto"])
    a = ap.parse_args(argv)
    nx, ny, nz = (int(v) for v in a.grid.split(","))
    case = ewg.lens3d_case(nx, ny, nz, seed=0)
    order = {"redblack": ewg.ILU_ORDER_REDBLACK, "box8": ewg.ILU_ORDER_BOX8, "auto": ewg.ILU_ORDER_AUTO}[a.ilu_ordering]
    sopts = ewg.default_solve_opts(linear_solver_tolerance=a.linear_tol, ilu_ordering=order)
    ctx = ewg.Context(case)
    ctx.apply_initial_solution()
    st, _ = ctx.newton_apply(a.dt, None, sopts)
    if st:
        raise RuntimeError(f"warm-up step failed: {ewg.STATUS_NAMES.get(st, st)}")
    ctx.advance_time_level()
    x1 = ctx.get_solution(0)
    cfg = {"grid": [nx, ny, nz], "cells": case.grid.n_cells, "dt": a.dt, "linear_tol": a.linear_tol,
           "ilu_ordering": a.ilu_ordering}

    def single():
        ctx.set_solution(1, x1)
        ctx.set_solution(0, x1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st, rep = ctx.newton_apply(a.dt, None, sopts)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, st, rep.iterations, rep.linear_iterations
    single()
    t, st, ni, li = single()
    x_sd = ctx.get_solution(0)
    print(json.dumps({"form": "single-domain", "s_per_step": t, "status": st, "newton_its": ni,
                      "bicgstab_its": li, "ms_per_bicgstab_it": 1e3 * t / max(li, 1), **cfg}), flush=True)
    plane = nx * ny
    for world in (int(w) for w in a.slabs.split(",")):
        parts = [DeviceSlab(SlabLinearizer(case, s), sopts) for s in partition(nz, world)]

        def run():
            for p in parts:
                p.lin.set_state(local_view(x1, case.grid, p.slab), local_view(x1, case.grid, p.slab))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rep = distributed_newton(parts, LocalComm(), a.dt, None, sopts)
            torch.cuda.synchronize()
            return time.perf_counter() - t0, rep
        run()
        t, rep = run()
        x = np.empty_like(x_sd)
        for p in parts:
            x[p.slab.k0 * plane:p.slab.k1 * plane] = p.ctx.get_solution(0)[p.lin.own]
        dp = float(np.max(np.abs(x[:, 0] - x_sd[:, 0])) / np.max(np.abs(x_sd[:, 0])))
        ds = float(np.max(np.abs(x[:, 1] - x_sd[:, 1])))
        print(json.dumps({"form": f"z-slabs x{world}", "s_per_step": t, "status": rep.status,
                          "newton_its": rep.iterations, "bicgstab_its": rep.linear_iterations,
                          "ms_per_bicgstab_it": 1e3 * t / max(rep.linear_iterations, 1),
                          "pw_rel_diff": dp, "sn_abs_diff": ds, **cfg}), flush=True)
        for p in parts:
            p.lin.close()
    ctx.close()


if __name__ == "__main__":
    main()
