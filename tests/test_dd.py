"""Domain decomposition into z-slabs (ewoms-numerics_b200/dd.py), host side: the partition, the
slab problems (same cell size bit for bit, shifted lens and inlet, permeability planes), the
ghost-plane exchange between two and three gloo ranks on CPU, and the distributed BiCGStab and
Newton driven by the oracle as the slabs' operators (in one process and on gloo ranks)."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT


def test_partition_covers_the_grid_once(ewg_mod):
    import dd
    for nz, world in [(10, 1), (10, 3), (128, 8), (7, 7)]:
        slabs = dd.partition(nz, world)
        assert slabs[0].k0 == 0 and slabs[-1].k1 == nz
        assert all(a.k1 == b.k0 for a, b in zip(slabs, slabs[1:]))
        sizes = [s.k1 - s.k0 for s in slabs]
        assert max(sizes) - min(sizes) <= 1
        assert slabs[0].ghost_lo == 0 and slabs[-1].ghost_hi == 0
        assert all(s.ghost_lo == 1 for s in slabs[1:]) and all(s.ghost_hi == 1 for s in slabs[:-1])
    with pytest.raises(ValueError):
        dd.partition(3, 4)


def test_slab_case_keeps_the_cell_and_the_global_geometry(ewg_mod):
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    hz = case.grid.lz / case.grid.nz
    for s in dd.partition(10, 3):
        sc = dd.slab_case(case, s)
        assert sc.grid.lz / sc.grid.nz == hz
        assert sc.grid.k_origin == s.first
        assert list(sc.problem.lens_lo) == list(case.problem.lens_lo)
        assert sc.problem.inlet_z_hi == case.problem.inlet_z_hi
        plane = 16 * 12
        assert np.array_equal(sc.perm, case.perm[s.first * plane:(s.first + s.planes) * plane])


def test_local_ghost_exchange(ewg_mod):
    import dd
    case = ewg_mod.lens3d_case(8, 6, 9, seed=0)
    slabs = dd.partition(9, 3)
    xg = np.arange(case.grid.n_cells * 2, dtype=np.float64).reshape(-1, 2)
    xs = [dd.local_view(xg, case.grid, s) for s in slabs]
    want = [x.copy() for x in xs]
    plane = 8 * 6
    for s, x in zip(slabs, xs):
        if s.ghost_lo:
            x[:plane] = -1
        if s.ghost_hi:
            x[-plane:] = -1
    dd.exchange_ghosts_local(xs, case.grid, slabs)
    assert all(np.array_equal(a, b) for a, b in zip(xs, want))


PROBE = r'''
import os, sys
sys.path.insert(0, os.path.join(sys.argv[1], "ewoms-numerics_b200"))
import numpy as np
import torch.distributed as dist
import dd, ewg
dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
case = ewg.lens3d_case(8, 6, 11, seed=0)
slabs = dd.partition(11, world)
s = slabs[rank]
xg = np.arange(case.grid.n_cells * 2, dtype=np.float64).reshape(-1, 2) * 0.5
x = dd.local_view(xg, case.grid, s)
want = x.copy()
plane = 8 * 6
if s.ghost_lo: x[:plane] = np.nan
if s.ghost_hi: x[-plane:] = np.nan
dd.exchange_ghosts(x, case.grid, s, dist)
assert np.array_equal(x, want), rank
dist.barrier()
dist.destroy_process_group()
print(f"rank {rank} ok", flush=True)
'''


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_ghost_exchange_between_gloo_ranks(tmp_path, world):
    probe = tmp_path / "probe.py"
    probe.write_text(PROBE)
    cmd = ["timeout", "-k", "30", "240", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={world}", "--master-addr=127.0.0.1", f"--master-port={_free_port()}", str(probe), ROOT]
    out = subprocess.run(cmd, capture_output=True, text=True, cwd=ROOT,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stdout + out.stderr
    assert all(f"rank {r} ok" in out.stdout for r in range(world))


@pytest.mark.parametrize("world", [2, 3, 5])
def test_oracle_slab_rows_equal_the_whole_grid(oracle_mod, ewg_mod, world):
    """The oracle linearizes each slab (plane origin at its first plane, ghost planes filled) and
    the owned residual and Jacobian rows equal the whole grid's bit for bit: the decomposition
    changes no operation of a cell's row."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x1 = o.get_solution(0)
    rng = np.random.default_rng(4)
    x0 = x1.copy()
    x0[:, 0] += rng.normal(0, 20.0, len(x0))
    x0[:, 1] = np.clip(x0[:, 1] - np.abs(rng.normal(0, 0.3, len(x0))), 0.2, 1.0)
    o.set_solution(1, x1)
    o.set_solution(0, x0)
    o.linearize(250.0)
    r_g = o.residual()
    rp_g, ci_g, b_g = o.jacobian_bcrs()
    plane = 16 * 12
    for s in dd.partition(10, world):
        sc = dd.slab_case(case, s)
        ol = oracle_mod.Oracle(sc)
        ol.set_solution(1, dd.local_view(x1, case.grid, s))
        ol.set_solution(0, dd.local_view(x0, case.grid, s))
        ol.linearize(250.0)
        own = dd.owned_rows(sc.grid, s)
        assert np.array_equal(ol.residual()[own], r_g[s.k0 * plane:s.k1 * plane])
        rp, ci, b = ol.jacobian_bcrs()
        shift = s.first * plane
        for lr in range(own.start, own.stop):
            gr = lr + shift
            assert np.array_equal(ci[rp[lr]:rp[lr + 1]] + shift, ci_g[rp_g[gr]:rp_g[gr + 1]])
            assert np.array_equal(b[rp[lr]:rp[lr + 1]], b_g[rp_g[gr]:rp_g[gr + 1]])
        ol.close()
    o.close()


@pytest.mark.parametrize("method", [1, 0])
def test_oracle_fd_slab_rows_equal_the_whole_grid(oracle_mod, ewg_mod, method):
    """With the finite-difference linearizer (forward and central differences) the slabs' owned
    rows equal the whole grid's bit for bit once every slab takes the whole grid's reference
    pressure (p_w of global cell 0); with its own (p_w of its first cell) a slab above the first
    deflects the pressure by a different step."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    og, x0, x1 = _perturbed_state(oracle_mod, case)
    o = oracle_mod.Oracle(case)
    o.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, method)
    o.set_solution(1, x1)
    o.set_solution(0, x0)
    o.update_begin()
    o.linearize(250.0)
    r_g = o.residual()
    rp_g, ci_g, b_g = o.jacobian_bcrs()
    plane = 16 * 12
    for given in (True, False):
        same = []
        for s in dd.partition(10, 3):
            sc = dd.slab_case(case, s)
            ol = oracle_mod.Oracle(sc)
            ol.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, method)
            ol.set_solution(1, dd.local_view(x1, case.grid, s))
            ol.set_solution(0, dd.local_view(x0, case.grid, s))
            if given:
                ol.set_reference_pressure(x0[0, 0])
            else:
                ol.update_begin()
            ol.linearize(250.0)
            own = dd.owned_rows(sc.grid, s)
            assert np.array_equal(ol.residual()[own], r_g[s.k0 * plane:s.k1 * plane])
            rp, ci, b = ol.jacobian_bcrs()
            shift = s.first * plane
            same.append(all(np.array_equal(b[rp[lr]:rp[lr + 1]], b_g[rp_g[lr + shift]:rp_g[lr + shift + 1]])
                            for lr in range(own.start, own.stop)))
            ol.close()
        assert all(same) if given else not all(same[1:])
    o.close()


# ---- the distributed BiCGStab's host logic, driven by the oracle as the slabs' operators ----

class OracleSlab:
    """One slab's operators for dd.distributed_bicgstab backed by the oracle (natural-order CPU
    tensors), so the distributed algorithm's host logic runs without a device."""

    def __init__(self, oracle_mod, case, slab, x0, x1, dt, opts):
        import dd
        sc = dd.slab_case(case, slab)
        self.o = oracle_mod.Oracle(sc)
        self.o.set_solution(1, dd.local_view(x1, case.grid, slab))
        self.o.set_solution(0, dd.local_view(x0, case.grid, slab))
        self.o.linearize(dt)
        self.slab, self.layout, self.n, self.opts = slab, dd.NaturalLayout(sc.grid, slab), sc.grid.n_cells, opts

    def zeros(self):
        import torch
        return torch.zeros((self.n, 2), dtype=torch.float64)

    def rhs(self):
        import torch
        return torch.from_numpy(self.o.residual())

    def spmv(self, x, y):
        import torch
        y.copy_(torch.from_numpy(self.o.apply_jacobian(x.numpy())))

    def precondition(self, b, y):
        import torch
        y.copy_(torch.from_numpy(self.o.apply_preconditioner(b.numpy(), self.opts)))


class OracleNewtonSlab(OracleSlab):
    """OracleSlab whose state solution(0) is a CPU tensor in natural order that
    dd.distributed_newton updates in place; linearize() hands it to the oracle first, with the
    Newton iteration number (the oracle takes the old-time-level storage at iteration 0)."""

    def __init__(self, oracle_mod, case, slab, x0, x1, opts):
        import dd
        import torch
        sc = dd.slab_case(case, slab)
        self.o = oracle_mod.Oracle(sc)
        self.o.set_solution(1, dd.local_view(x1, case.grid, slab))
        self.x = torch.from_numpy(np.ascontiguousarray(dd.local_view(x0, case.grid, slab)))
        self.slab, self.layout, self.n, self.opts = slab, dd.NaturalLayout(sc.grid, slab), sc.grid.n_cells, opts
        self.ctx = self
        self.iteration = 0

    def on(self):
        import contextlib
        return contextlib.nullcontext()

    def linearize(self, dt):
        self.o.set_solution(0, self.x.numpy())
        self.o.linearize(dt, self.iteration)
        self.iteration += 1

    def set_reference_pressure(self, p_ref):
        self.o.set_reference_pressure(p_ref)

    def solution(self):
        return self.x


def _stepped_state(oracle_mod, case, steps):
    """The state after `steps` implicit-Euler steps of the single-domain oracle."""
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    o.run(steps, 250.0)
    return o


def _perturbed_state(oracle_mod, case):
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x1 = o.get_solution(0)
    rng = np.random.default_rng(4)
    x0 = x1.copy()
    x0[:, 0] += rng.normal(0, 20.0, len(x0))
    x0[:, 1] = np.clip(x0[:, 1] - np.abs(rng.normal(0, 0.3, len(x0))), 0.2, 1.0)
    o.set_solution(1, x1)
    o.set_solution(0, x0)
    o.linearize(250.0)
    return o, x0, x1


def _solve_opts(ewg_mod):
    opts = ewg_mod.default_solve_opts(linear_solver_tolerance=1e-9)
    opts.verify_true_residual = 1
    return opts


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_distributed_bicgstab_solves_the_whole_grid(oracle_mod, ewg_mod, world):
    """The slabs' distributed BiCGStab (restricted additive Schwarz, global reductions) returns
    an update whose owned rows, put together, solve the whole grid's J dx = r."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    og, x0, x1 = _perturbed_state(oracle_mod, case)
    r_g = og.residual()
    opts = _solve_opts(ewg_mod)
    slabs = dd.partition(10, world)
    parts = [OracleSlab(oracle_mod, case, s, x0, x1, 250.0, opts) for s in slabs]
    st, its, _, res, init, dxs = dd.distributed_bicgstab(parts, dd.LocalComm(), opts)
    assert st == dd.ST_CONVERGED and its > 0
    plane = 16 * 12
    dx = np.concatenate([d.numpy()[p.layout.owned[0]] for d, p in zip(dxs, parts)])
    assert dx.shape == (case.grid.n_cells, 2)
    true = np.max(np.abs(r_g - og.apply_jacobian(dx)))
    assert true <= 10 * 1e-9 * np.max(np.abs(r_g)), (true, np.max(np.abs(r_g)))
    assert init == np.max(np.abs(r_g))


def test_distributed_bicgstab_with_jacobi_does_not_depend_on_the_slabs(oracle_mod, ewg_mod):
    """Block Jacobi acts cell by cell, so its restricted additive Schwarz form is the whole
    grid's preconditioner itself: every slab count, down to one-plane slabs, solves the whole
    grid's system in about the single-domain iteration count (the slabs change only the
    summation order of the dot products) and agrees with the single-domain solve."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    og, x0, x1 = _perturbed_state(oracle_mod, case)
    opts = _solve_opts(ewg_mod)
    opts.precond = ewg_mod.PRECOND_JACOBI
    r_g = og.residual()
    rc, dx_sd, it_sd, _ = og.solve(opts)
    assert rc == 0 and it_sd > 0
    for world in (1, 2, 3, 5, 10):
        parts = [OracleSlab(oracle_mod, case, s, x0, x1, 250.0, opts) for s in dd.partition(10, world)]
        st, its, _, _, _, dxs = dd.distributed_bicgstab(parts, dd.LocalComm(), opts)
        assert st == dd.ST_CONVERGED and abs(its - it_sd) <= 0.1 * it_sd + 2, (world, its, it_sd)
        dx = np.concatenate([d.numpy()[p.layout.owned[0]] for d, p in zip(dxs, parts)])
        assert np.max(np.abs(r_g - og.apply_jacobian(dx))) <= 10 * 1e-9 * np.max(np.abs(r_g))
        assert np.max(np.abs(dx - dx_sd)) <= 1e-5 * np.max(np.abs(dx_sd)), world


class CountingComm:
    """LocalComm that counts the reductions (one collective each between ranks): those read back
    to the host and those left on the device."""

    def __init__(self, dd):
        self.inner, self.reductions, self.device_reductions = dd.LocalComm(), 0, 0

    def exchange(self, parts, vecs):
        self.inner.exchange(parts, vecs)

    def reduce(self, vals, nsum):
        self.reductions += 1
        return self.inner.reduce(vals, nsum)

    def reduce_device(self, vals, parts=None):
        self.device_reductions += 1
        return self.inner.reduce_device(vals, parts)


@pytest.mark.parametrize("verify", [0, 1])
def test_distributed_bicgstab_takes_three_reductions_per_iteration(oracle_mod, ewg_mod, verify):
    """Every BiCGStab iteration's dot products and max-norms meet in three reductions: <r0,v> on
    the device; the half-step check with <t,t>, <t,s> and <r0,v>; the full-step check with
    <r0,r>, <r,r>; only the last two are read back to the host. Besides them: one for ||b|| at
    the start, one per true-residual check."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    og, x0, x1 = _perturbed_state(oracle_mod, case)
    opts = _solve_opts(ewg_mod)
    opts.verify_true_residual = verify
    parts = [OracleSlab(oracle_mod, case, s, x0, x1, 250.0, opts) for s in dd.partition(10, 3)]
    comm = CountingComm(dd)
    st, its, restarts, _, _, _ = dd.distributed_bicgstab(parts, comm, opts)
    assert st == dd.ST_CONVERGED and its > 0
    # the converging iteration ends after its first (half step) or second (full step) host read
    # without adding to the count
    assert comm.reductions - 1 - 2 * its - verify * (1 + restarts) in (1, 2), comm.reductions
    assert comm.device_reductions == its + 1


def _check_newton_state(x_dd, x_sd):
    dp = np.max(np.abs(x_dd[:, 0] - x_sd[:, 0])) / np.max(np.abs(x_sd[:, 0]))
    ds = np.max(np.abs(x_dd[:, 1] - x_sd[:, 1]))
    assert dp <= 1e-7 and ds <= 1e-5, (dp, ds)


@pytest.mark.parametrize("world", [1, 2, 3])
def test_distributed_newton_matches_the_single_domain(oracle_mod, ewg_mod, world):
    """One implicit-Euler step by dd.distributed_newton over oracle slabs: it converges, its
    error is the whole grid's residual max-norm at the final state (the owned rows are the whole
    grid's rows), and the state agrees with the single-domain oracle Newton's (the linear solves
    differ within their tolerance: block ILU(0) of the whole grid against restricted additive
    Schwarz over the slabs)."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    o = _stepped_state(oracle_mod, case, 2)
    x1 = o.get_solution(0)
    sopts = ewg_mod.default_solve_opts()
    parts = [OracleNewtonSlab(oracle_mod, case, s, x1, x1, sopts) for s in dd.partition(10, world)]
    rep = dd.distributed_newton(parts, dd.LocalComm(), 250.0, None, sopts)
    assert rep.converged and rep.iterations >= 1, (rep.status, rep.iterations, rep.error)
    x_dd = np.concatenate([p.x.numpy()[p.layout.owned[0]] for p in parts])
    # the whole grid linearized as the slabs were: old storage recycled at iteration 0 from x1
    ow = oracle_mod.Oracle(case)
    ow.set_solution(1, x1)
    ow.set_solution(0, x1)
    ow.linearize(250.0, 0)
    ow.set_solution(0, x_dd)
    ow.linearize(250.0, 1)
    assert np.max(np.abs(ow.residual())) == rep.error
    ow.close()
    o.set_solution(1, x1)
    o.set_solution(0, x1)
    rc, ni, li, e = o.newton_apply(250.0)
    assert rc == 0
    _check_newton_state(x_dd, o.get_solution(0))


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_fd_newton_matches_the_single_domain(oracle_mod, ewg_mod, world):
    """Newton over slabs that linearize with finite differences (distributed_newton hands every
    slab the whole grid's reference pressure; the row-level tests pin its effect): the step
    converges and agrees with the single-domain oracle's FD Newton."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    o = _stepped_state(oracle_mod, case, 2)
    x1 = o.get_solution(0)
    sopts = ewg_mod.default_solve_opts()
    parts = [OracleNewtonSlab(oracle_mod, case, s, x1, x1, sopts) for s in dd.partition(10, world)]
    for p in parts:
        p.o.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, 1)
    rep = dd.distributed_newton(parts, dd.LocalComm(), 250.0, None, sopts)
    assert rep.converged, (rep.status, rep.iterations, rep.error)
    x_dd = np.concatenate([p.x.numpy()[p.layout.owned[0]] for p in parts])
    o.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, 1)
    o.set_solution(1, x1)
    o.set_solution(0, x1)
    rc, ni, li, e = o.newton_apply(250.0)
    assert rc == 0
    _check_newton_state(x_dd, o.get_solution(0))


def _newton_slabs(oracle_mod, ewg_mod, world):
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    x1 = _stepped_state(oracle_mod, case, 1).get_solution(0)
    sopts = ewg_mod.default_solve_opts()
    return [OracleNewtonSlab(oracle_mod, case, s, x1, x1, sopts) for s in dd.partition(10, world)], sopts


def test_distributed_newton_stops_on_a_nonfinite_update(oracle_mod, ewg_mod, monkeypatch):
    """A solve that reports convergence but leaves a non-finite entry in one slab's update ends
    the distributed Newton with EWG_ERR_NONFINITE (the flag is a maximum over all slabs)."""
    import dd
    parts, sopts = _newton_slabs(oracle_mod, ewg_mod, 3)
    solve = dd.distributed_bicgstab

    def poisoned(parts, comm, opts):
        out = solve(parts, comm, opts)
        out[5][2][parts[2].layout.owned[0].start, 1] = float("nan")
        return out
    monkeypatch.setattr(dd, "distributed_bicgstab", poisoned)
    rep = dd.distributed_newton(parts, dd.LocalComm(), 250.0, None, sopts)
    assert rep.status == ewg_mod.EWG_ERR_NONFINITE and not rep.converged and rep.iterations == 0


def test_distributed_newton_stops_when_a_slab_preconditioner_breaks(oracle_mod, ewg_mod):
    """A NaN out of one slab's preconditioner makes the global residual max-norm infinite, so the
    distributed BiCGStab fails on every slab's side and Newton ends with EWG_ERR_NOT_CONVERGED."""
    import dd
    parts, sopts = _newton_slabs(oracle_mod, ewg_mod, 2)
    bad = parts[1]
    apply = bad.precondition

    def poisoned(b, y):
        apply(b, y)
        y[bad.layout.owned[0].start] = float("nan")
    bad.precondition = poisoned
    rep = dd.distributed_newton(parts, dd.LocalComm(), 250.0, None, sopts)
    assert rep.status == ewg_mod.EWG_ERR_NOT_CONVERGED and not rep.converged


DIST_PROBE = r'''
import os, sys
root = sys.argv[1]
sys.path[:0] = [os.path.join(root, "ewoms-numerics_b200"), os.path.join(root, "oracle"), os.path.join(root, "tests")]
import numpy as np
import torch.distributed as dist
import dd, ewg, oracle
from test_dd import OracleSlab, _perturbed_state, _solve_opts
dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
case = ewg.lens3d_case(16, 12, 10, seed=2)
og, x0, x1 = _perturbed_state(oracle, case)
opts = _solve_opts(ewg)
s = dd.partition(10, world)[rank]
part = OracleSlab(oracle, case, s, x0, x1, 250.0, opts)
st, its, _, res, init, (dx,) = dd.distributed_bicgstab([part], dd.TorchComm(dist), opts)
got = [None] * world
dist.all_gather_object(got, (st, its, dx.numpy()[part.layout.owned[0]]))
assert len({(a, b) for a, b, _ in got}) == 1, got
if rank == 0:
    dxg = np.concatenate([d for _, _, d in got])
    r_g = og.residual()
    true = np.max(np.abs(r_g - og.apply_jacobian(dxg)))
    assert st == dd.ST_CONVERGED and true <= 10 * 1e-9 * np.max(np.abs(r_g)), (st, true)
dist.barrier()
dist.destroy_process_group()
print(f"rank {rank} ok its={its}", flush=True)
'''


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_bicgstab_between_gloo_ranks(tmp_path, world):
    """The same solve with one slab per gloo rank: ghost planes over P2P messages, reductions
    over all_gather; every rank ends with the same status and iteration count."""
    probe = tmp_path / "probe.py"
    probe.write_text(DIST_PROBE)
    cmd = ["timeout", "-k", "30", "300", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={world}", "--master-addr=127.0.0.1", f"--master-port={_free_port()}", str(probe), ROOT]
    out = subprocess.run(cmd, capture_output=True, text=True, cwd=ROOT,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert all(f"rank {r} ok" in out.stdout for r in range(world))


NEWTON_PROBE = r'''
import os, sys
root = sys.argv[1]
sys.path[:0] = [os.path.join(root, "ewoms-numerics_b200"), os.path.join(root, "oracle"), os.path.join(root, "tests")]
import numpy as np
import torch.distributed as dist
import dd, ewg, oracle
from test_dd import OracleNewtonSlab, _stepped_state, _check_newton_state
dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
case = ewg.lens3d_case(16, 12, 10, seed=2)
o = _stepped_state(oracle, case, 2)
x1 = o.get_solution(0)
sopts = ewg.default_solve_opts()
part = OracleNewtonSlab(oracle, case, dd.partition(10, world)[rank], x1, x1, sopts)
rep = dd.distributed_newton([part], dd.TorchComm(dist), 250.0, None, sopts)
got = [None] * world
dist.all_gather_object(got, (rep.status, rep.iterations, rep.linear_iterations, rep.error,
                             part.x.numpy()[part.layout.owned[0]]))
assert len({g[:4] for g in got}) == 1, [g[:4] for g in got]
if rank == 0:
    assert rep.converged, (rep.status, rep.iterations, rep.error)
    o.set_solution(1, x1)
    o.set_solution(0, x1)
    assert o.newton_apply(250.0)[0] == 0
    _check_newton_state(np.concatenate([g[4] for g in got]), o.get_solution(0))
dist.barrier()
dist.destroy_process_group()
print(f"rank {rank} ok newton={rep.iterations} linear={rep.linear_iterations}", flush=True)
'''


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_newton_between_gloo_ranks(tmp_path, world):
    """One implicit-Euler step by Newton with one slab per gloo rank: every rank ends with the
    same status, iteration counts and error, and the gathered state agrees with the
    single-domain oracle Newton's."""
    probe = tmp_path / "probe.py"
    probe.write_text(NEWTON_PROBE)
    cmd = ["timeout", "-k", "30", "300", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={world}", "--master-addr=127.0.0.1", f"--master-port={_free_port()}", str(probe), ROOT]
    out = subprocess.run(cmd, capture_output=True, text=True, cwd=ROOT,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert all(f"rank {r} ok" in out.stdout for r in range(world))


def _to_split(x_nat, grid):
    """Natural -> the device storage order (entry col * N/2 + c/2, col = (i + j + k) & 1)."""
    n = grid.n_cells
    c = np.arange(n)
    i, j, k = c % grid.nx, (c // grid.nx) % grid.ny, c // (grid.nx * grid.ny)
    out = np.empty_like(x_nat)
    out[((i + j + k) & 1) * (n // 2) + (c >> 1)] = x_nat
    return out


def test_split_layout_ghost_exchange(ewg_mod):
    """Ghost planes exchanged in the device storage order (plane chunks in global colour order)
    hold the same cells as an exchange in natural order, also between slabs whose first planes
    differ in parity (there the local colours of a plane are swapped)."""
    import types
    import dd
    import torch
    case = ewg_mod.lens3d_case(8, 6, 11, seed=0)
    xg = np.arange(case.grid.n_cells * 2, dtype=np.float64).reshape(-1, 2) * 0.25
    for world in (2, 3, 4):
        slabs = dd.partition(11, world)
        assert len({s.first & 1 for s in slabs}) == 2 or world == 2
        parts, vecs, want = [], [], []
        for s in slabs:
            g = dd.slab_case(case, s).grid
            nat = dd.local_view(xg, case.grid, s)
            spl = torch.from_numpy(_to_split(nat, g))
            L = dd.SplitLayout(g, s)
            want.append(spl.clone())
            for k in ([0] if s.ghost_lo else []) + ([s.planes - 1] if s.ghost_hi else []):
                for c in L.plane(k):
                    spl[c] = -7.0
            parts.append(types.SimpleNamespace(slab=s, layout=L))
            vecs.append(spl)
        dd.LocalComm().exchange(parts, vecs)
        assert all(torch.equal(a, b) for a, b in zip(vecs, want))


def test_split_layout_owned_view_is_the_owned_rows(ewg_mod):
    """SplitLayout.owned_view covers exactly the rows of both colours' owned runs, so the
    distributed solve's norms and dot products see every owned cell once and no ghost cell."""
    import dd
    import torch
    case = ewg_mod.lens3d_case(8, 6, 11, seed=0)
    for world in (1, 2, 3, 4):
        for s in dd.partition(11, world):
            g = dd.slab_case(case, s).grid
            L = dd.SplitLayout(g, s)
            a = torch.arange(g.n_cells * 2, dtype=torch.float64).reshape(-1, 2)
            want = torch.cat([a[o] for o in L.owned])
            got = L.owned_view(a).reshape(-1, 2)
            assert torch.equal(got, want), (world, s)
            assert got.shape[0] == (s.k1 - s.k0) * 8 * 6
