"""GPU tests of the box-8-colour block ILU(0) (ewg_box8.cuh) against the oracle's ORDER_BOX8, the
same dune-istl factorization and sweeps on the matrix permuted to that order.

* The preconditioner applied to a vector equals the oracle's within 1e-11 (relaxation 1 and 0.9),
  on 3D lens grids whose dimensions are multiples of 4, at a perturbed state.
* BiCGStab with it converges to the linear tolerance on the oracle's operator, within 1e-5 of the
  oracle's solution and within 15 % of its iteration count (dot products are summed in another
  order), and needs fewer iterations than the red-black order on the same system.
* The mixed-precision solve (FP32 factors and sweeps) reaches the linear tolerance.
* ilu_ordering BOX8 on a grid it does not fit is rejected; AUTO falls back to red-black there.
"""
import numpy as np
import pytest

from conftest import rel_close

pytestmark = pytest.mark.gpu


def _system(ewg, oracle_mod, case, seed):
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x = o.get_solution(0)
    rng = np.random.Generator(np.random.PCG64(seed))
    xc, yc, zc = ewg.cell_centers(case.grid)
    plume = np.exp(-((xc - 0.5 * case.grid.lx) ** 2) / 0.8 - ((yc - 0.8 * case.grid.ly) ** 2) / 0.5)
    x[:, 1] = 1.0 - 0.7 * plume * rng.uniform(0.3, 1.0, size=len(xc))
    x[:, 0] += rng.normal(0.0, 80.0, size=len(xc))
    o.set_solution(0, x)
    o.set_solution(1, x)
    o.linearize(250.0, 0)
    ctx = ewg.Context(case)
    rp, ci, b = o.jacobian_bcrs()
    ctx.set_matrix_bcrs(rp, ci, b)
    ctx.set_residual(o.residual())
    return ctx, o


CASES = [(8, 8, 4), (16, 12, 8), (32, 32, 16)]


@pytest.mark.parametrize("shape", CASES)
@pytest.mark.parametrize("relax", [1.0, 0.9])
def test_box8_preconditioner_matches_oracle(ewg_mod, oracle_mod, shape, relax):
    case = ewg_mod.lens3d_case(*shape, seed=5, corr_cells=3.0)
    ctx, o = _system(ewg_mod, oracle_mod, case, 17)
    rng = np.random.Generator(np.random.PCG64(6))
    v = rng.standard_normal((o.n, 2))
    opts = ewg_mod.default_solve_opts(precond=ewg_mod.PRECOND_ILU0, ilu_ordering=ewg_mod.ILU_ORDER_BOX8,
                                      preconditioner_relaxation=relax)
    y_g = ctx.apply_preconditioner(v, opts)
    y_o = o.apply_preconditioner(v, opts, ordering=oracle_mod.ORDER_BOX8)
    ok, err, scale = rel_close(y_g, y_o, 1e-11)
    assert ok, (err, scale)
    # the red-black order stays available on the same grid
    rb = ewg_mod.default_solve_opts(precond=ewg_mod.PRECOND_ILU0, ilu_ordering=ewg_mod.ILU_ORDER_REDBLACK,
                                    preconditioner_relaxation=relax)
    assert rel_close(ctx.apply_preconditioner(v, rb), o.apply_preconditioner(v, rb, ordering=oracle_mod.ORDER_REDBLACK),
                     1e-11)[0]
    ctx.close()


@pytest.mark.parametrize("shape", CASES)
def test_box8_bicgstab_matches_oracle(ewg_mod, oracle_mod, shape):
    case = ewg_mod.lens3d_case(*shape, seed=5, corr_cells=3.0)
    ctx, o = _system(ewg_mod, oracle_mod, case, 31)
    opts = ewg_mod.default_solve_opts(linear_solver_max_iterations=2000, ilu_ordering=ewg_mod.ILU_ORDER_BOX8)
    rep = ctx.solve(opts, check=True)
    dx_g = ctx.update()
    rc, dx_o, it_o, _ = o.solve(opts, ordering=oracle_mod.ORDER_BOX8)
    assert rc == 0 and rep.converged
    res = o.apply_jacobian(dx_g) - o.residual()
    assert np.max(np.abs(res)) <= 1e-8 * np.max(np.abs(o.residual())) + 1e-9
    assert rel_close(dx_g, dx_o, 1e-5)[0]
    assert abs(rep.iterations - it_o) <= max(3, 0.15 * it_o), (rep.iterations, it_o)
    rb = ctx.solve(ewg_mod.default_solve_opts(linear_solver_max_iterations=2000,
                                              ilu_ordering=ewg_mod.ILU_ORDER_REDBLACK), check=True)
    assert rb.converged and rep.iterations <= rb.iterations, (rep.iterations, rb.iterations)
    ctx.close()


def test_box8_mixed_precision_solve(ewg_mod):
    case = ewg_mod.lens3d_case(32, 32, 16, seed=5, corr_cells=3.0)
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    ctx.run(1, 250.0)
    x = ctx.get_solution(0)
    ctx.set_solution(0, x)
    mixed = ewg_mod.default_solve_opts(precision=ewg_mod.PRECISION_MIXED, ilu_ordering=ewg_mod.ILU_ORDER_BOX8)
    # the mixed solve needs the FP32 Jacobian the linearizer writes in mixed mode
    st, rep = ctx.newton_apply(250.0, ewg_mod.default_newton_opts(), mixed)
    assert st == 0 and rep.converged and rep.error <= 1e-8
    ctx.close()


def test_box8_rejected_where_it_does_not_fit(ewg_mod):
    case = ewg_mod.lens3d_case(16, 12, 10, seed=3, corr_cells=3.0)  # nz = 10
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    ctx.linearize(250.0)
    with pytest.raises(ewg_mod.EwgError) as ei:
        ctx.solve(ewg_mod.default_solve_opts(ilu_ordering=ewg_mod.ILU_ORDER_BOX8), check=True)
    assert ei.value.status == ewg_mod.EWG_ERR_INVALID
    rep = ctx.solve(ewg_mod.default_solve_opts(ilu_ordering=ewg_mod.ILU_ORDER_AUTO))
    assert rep.converged
    ctx.close()
