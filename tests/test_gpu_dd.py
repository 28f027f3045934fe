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
