"""Domain decomposition into z-slabs on the device: every rank's owned residual rows and
Jacobian rows equal the single-domain linearization's bit for bit. The ranks are emulated as
separate contexts in one process (one after the other, no kernel waits on another); on several
GPUs each context sits on its own device and the ghost planes travel with dd.exchange_ghosts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3, 5])
def test_slab_linearization_equals_single_domain(ewg_mod, world):
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    for _ in range(2):
        st, rep = ctx.newton_apply(250.0, None, ewg_mod.default_solve_opts(linear_solver_tolerance=1e-3))
        assert st == 0
        ctx.advance_time_level()
    x1 = ctx.get_solution(0)
    rng = np.random.default_rng(4)
    x0 = x1.copy()
    x0[:, 0] += rng.normal(0, 20.0, len(x0))
    x0[:, 1] = np.clip(x0[:, 1] - np.abs(rng.normal(0, 0.03, len(x0))), 0.4, 1.0)
    ctx.set_solution(1, x1)
    ctx.set_solution(0, x0)
    rep = ctx.linearize(250.0)
    r_g = ctx.residual()
    rp_g, ci_g, b_g = ctx.jacobian_bcrs()
    slabs = dd.partition(case.grid.nz, world)
    # each rank holds its planes; the ghost planes come from the neighbours
    xs = [dd.local_view(x0, case.grid, s) for s in slabs]
    xos = [dd.local_view(x1, case.grid, s) for s in slabs]
    dd.exchange_ghosts_local(xs, case.grid, slabs)
    errs = []
    for s, xl, xol in zip(slabs, xs, xos):
        lin = dd.SlabLinearizer(case, s)
        lin.set_state(xl, xol)
        errs.append(lin.linearize(250.0))
        rows, rp, ci, b = lin.owned_jacobian()
        assert np.array_equal(lin.owned_residual(), r_g[rows])
        for lr, gr in zip(range(lin.own.start, lin.own.stop), rows):
            lcols, gcols = ci[rp[lr]:rp[lr + 1]], ci_g[rp_g[gr]:rp_g[gr + 1]]
            assert np.array_equal(lcols, gcols), gr
            assert np.array_equal(b[rp[lr]:rp[lr + 1]], b_g[rp_g[gr]:rp_g[gr + 1]]), gr
        lin.close()
    # the Newton error is the maximum over the ranks' owned rows
    assert max(errs) == rep.error
    ctx.close()


@pytest.mark.parametrize("method", [1, 0])
def test_fd_slab_linearization_equals_single_domain(ewg_mod, method):
    """The finite-difference linearizer (forward and central) on device slabs: with the whole
    grid's reference pressure (p_w of global cell 0) every slab's owned residual and Jacobian rows
    equal the single-domain FD linearization's bit for bit."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    x1 = ctx.get_solution(0)
    rng = np.random.default_rng(5)
    x0 = x1.copy()
    x0[:, 0] += rng.normal(0, 20.0, len(x0))
    x0[:, 1] = np.clip(x0[:, 1] - np.abs(rng.normal(0, 0.2, len(x0))), 0.3, 1.0)
    ctx.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, method)
    ctx.set_solution(1, x1)
    ctx.set_solution(0, x0)
    ctx.update_begin()
    ctx.linearize(250.0)
    r_g = ctx.residual()
    rp_g, ci_g, b_g = ctx.jacobian_bcrs()
    for s in dd.partition(case.grid.nz, 3):
        lin = dd.SlabLinearizer(case, s)
        lin.ctx.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, method)
        lin.set_state(dd.local_view(x0, case.grid, s), dd.local_view(x1, case.grid, s))
        lin.set_reference_pressure(x0[0, 0])
        lin.linearize(250.0)
        rows, rp, ci, b = lin.owned_jacobian()
        assert np.array_equal(lin.owned_residual(), r_g[rows])
        for lr, gr in zip(range(lin.own.start, lin.own.stop), rows):
            assert np.array_equal(ci[rp[lr]:rp[lr + 1]], ci_g[rp_g[gr]:rp_g[gr + 1]]), gr
            assert np.array_equal(b[rp[lr]:rp[lr + 1]], b_g[rp_g[gr]:rp_g[gr + 1]]), gr
        lin.close()
    ctx.close()


def _state_after_steps(ewg_mod, case, steps):
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    for _ in range(steps):
        st, _ = ctx.newton_apply(250.0, None, ewg_mod.default_solve_opts(linear_solver_tolerance=1e-3))
        assert st == 0
        ctx.advance_time_level()
    return ctx


def _device_slabs(dd, case, x0, x1, world, opts):
    slabs = dd.partition(case.grid.nz, world)
    parts = []
    for s in slabs:
        lin = dd.SlabLinearizer(case, s)
        lin.set_state(dd.local_view(x0, case.grid, s), dd.local_view(x1, case.grid, s))
        parts.append(dd.DeviceSlab(lin, opts))
    return parts


def _gather_owned(dd, case, parts):
    plane = case.grid.nx * case.grid.ny
    out = np.empty((case.grid.n_cells, 2))
    for p in parts:
        s = p.slab
        out[s.k0 * plane:s.k1 * plane] = p.ctx.get_solution(0)[p.lin.own]
    return out


@pytest.mark.parametrize("world", [1, 2, 3])
def test_distributed_bicgstab_on_device_slabs(ewg_mod, world):
    """The distributed BiCGStab over device slabs (device-order vectors, the slabs' own red-black
    ILU(0) as restricted additive Schwarz) returns an update that solves the whole grid's
    J dx = r: checked with the whole-grid context's Jacobian."""
    import dd
    import torch
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    ctx = _state_after_steps(ewg_mod, case, 1)
    x1 = ctx.get_solution(0)
    x0 = x1.copy()
    x0[:, 1] = np.clip(x0[:, 1] - 0.01, 0.0, 1.0)
    ctx.set_solution(1, x1)
    ctx.set_solution(0, x0)
    ctx.linearize(250.0)
    r_g = ctx.residual()
    opts = ewg_mod.default_solve_opts(linear_solver_tolerance=1e-9)
    parts = _device_slabs(dd, case, x0, x1, world, opts)
    for p in parts:
        p.ctx.linearize(250.0)
    st, its, _, res, init, dxs = dd.distributed_bicgstab(parts, dd.LocalComm(), opts)
    torch.cuda.synchronize()
    assert st == dd.ST_CONVERGED and its > 0
    plane = case.grid.nx * case.grid.ny
    dx = np.empty_like(r_g)
    for p, d in zip(parts, dxs):
        # device order -> natural order of the slab, owned planes
        nat = np.empty((p.n, 2))
        L = p.layout
        d = d.cpu().numpy()
        g = p.lin.case.grid
        for k in range(p.slab.planes):
            for gc, sl in zip((0, 1), L.plane(k)):
                cells = np.arange(k * plane, (k + 1) * plane)
                i, j = cells % g.nx, (cells // g.nx) % g.ny
                mine = cells[((i + j + k + p.slab.first) & 1) == gc]
                nat[mine] = d[sl]
        dx[p.slab.k0 * plane:p.slab.k1 * plane] = nat[p.lin.own]
    true = np.max(np.abs(r_g - ctx.apply_jacobian(dx)))
    assert true <= 10 * 1e-9 * np.max(np.abs(r_g)), (true, np.max(np.abs(r_g)), its)
    assert init == np.max(np.abs(r_g))
    for p in parts:
        p.lin.close()
    ctx.close()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("local", ["ad", "fd_forward"])
def test_distributed_newton_step(ewg_mod, world, local):
    """One implicit-Euler step solved by Newton over the slabs: it converges, its final error is
    the whole grid's residual max-norm at the assembled state (owned rows are the whole grid's
    rows; the residual-only evaluation may contract differently, hence 1e-10), and the state
    agrees with the single-domain Newton's. With the forward-difference local linearizer every
    slab must take the whole grid's reference pressure (the updateBegin reduction of
    distributed_newton reads p_w of global cell 0 from the bottom slab's split-order storage) for
    its deflections, and so its Jacobian rows, to be the single domain's."""
    import dd
    case = ewg_mod.lens3d_case(16, 12, 10, seed=2)
    ctx = _state_after_steps(ewg_mod, case, 2)
    x1 = ctx.get_solution(0)
    sopts = ewg_mod.default_solve_opts()
    parts = _device_slabs(dd, case, x1, x1, world, sopts)
    if local == "fd_forward":
        ctx.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, 1)
        for p in parts:
            p.ctx.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, 1)
    rep = dd.distributed_newton(parts, dd.LocalComm(), 250.0, None, sopts)
    assert rep.converged, (rep.status, rep.iterations, rep.error)
    x_dd = _gather_owned(dd, case, parts)
    if local == "ad":
        whole = ctx.residual_norm(x_dd, 250.0)
    else:
        # the finite-difference linearizer's residual comes from its own kernel: linearize the whole
        # grid at the assembled state with the slabs' reference pressure (p_w of global cell 0 at
        # the start of the step) and the same old time level
        ctx.set_reference_pressure(x1[0, 0])
        ctx.set_solution(0, x_dd)
        whole = ctx.linearize(250.0).error
        ctx.set_solution(0, x1)
    assert abs(whole - rep.error) <= 1e-10 * rep.error, (whole, rep.error)
    st, srep = ctx.newton_apply(250.0, None, sopts)
    assert st == 0
    x_sd = ctx.get_solution(0)
    dp = np.max(np.abs(x_dd[:, 0] - x_sd[:, 0])) / np.max(np.abs(x_sd[:, 0]))
    ds = np.max(np.abs(x_dd[:, 1] - x_sd[:, 1]))
    assert dp <= 1e-7 and ds <= 1e-5, (dp, ds, rep.iterations, srep.iterations)
    for p in parts:
        p.lin.close()
    ctx.close()
