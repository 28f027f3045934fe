"""GPU parity tests: the CUDA path (through the C ABI of libewg.so) against the CPU oracle.

Tolerances (FP64): residual and every Jacobian entry within 1e-12 relative to the field's maximum
magnitude per (equation, primary variable) component; preconditioner and SpMV within 1e-11;
after 10 implicit-Euler steps p_w within 1e-8 relative and S_w within 1e-8 absolute of the oracle
with identical Newton iteration counts.
"""
import os

import numpy as np
import pytest

from conftest import ROOT, rel_close

pytestmark = pytest.mark.gpu

GOLD = os.path.join(ROOT, "tests", "golden", "lens2d_golden.npz")
LIN_RTOL = 1e-12


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _cases(ewg):
    return {
        "baseline": lambda: ewg.baseline_case(),
        "reference": lambda: ewg.reference_case(),
        "brooks_corey": lambda: ewg.brooks_corey_case(),
        "lens3d_4x3x3": lambda: ewg.lens3d_case(4, 3, 3, seed=1),
        "lens3d_8x6x4": lambda: ewg.lens3d_case(8, 6, 4, seed=2),
        "lens3d_16x12x10": lambda: ewg.lens3d_case(16, 12, 10, seed=3, corr_cells=3.0),
    }


def _perturb(ewg, case, x, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = x.copy()
    xc, yc, zc = ewg.cell_centers(case.grid)
    plume = np.exp(-((xc - 0.5 * case.grid.lx) ** 2) / 0.8 - ((yc - 0.8 * case.grid.ly) ** 2) / 0.5)
    x[:, 1] = 1.0 - 0.7 * plume * rng.uniform(0.3, 1.0, size=len(xc))
    x[:, 1] = np.where(rng.uniform(size=len(xc)) < 0.05, rng.uniform(-0.02, 1.02, size=len(xc)), x[:, 1])
    x[:, 0] += rng.normal(0.0, 80.0, size=len(xc))
    return x


def _compare_linearization(ewg, oracle_mod, case, x, xold=None, dt=250.0):
    xold = x if xold is None else xold
    ctx = ewg.Context(case)
    ctx.set_solution(1, xold)
    ctx.set_solution(0, x)
    rep = ctx.linearize(dt)
    o = oracle_mod.Oracle(case)
    o.set_solution(1, xold)
    o.set_solution(0, x)
    o.set_recycle_first_iteration_storage(False)
    err = o.linearize(dt, 0)
    r_g, r_o = ctx.residual(), o.residual()
    rp_g, ci_g, b_g = ctx.jacobian_bcrs()
    rp_o, ci_o, b_o = o.jacobian_bcrs()
    assert np.array_equal(rp_g, rp_o) and np.array_equal(ci_g, ci_o)
    # the residual is a sum of flux terms that cancel at hydrostatic equilibrium: judge it against
    # the size of those terms (diagonal pressure derivative x one cell's hydrostatic pressure step)
    flux_scale = np.max(np.abs(b_o[:, 0, 0])) * case.problem.rho_w * case.problem.gravity * case.grid.ly / case.grid.ny
    r_scale = max(np.max(np.abs(r_o)), flux_scale)
    for eq in range(2):
        ok, e, s = rel_close(r_g[:, eq], r_o[:, eq], LIN_RTOL, scale=r_scale)
        assert ok, ("residual", eq, e, s)
        for pv in range(2):
            ok, e, s = rel_close(b_g[:, eq, pv], b_o[:, eq, pv], LIN_RTOL)
            assert ok, ("jacobian", eq, pv, e, s)
    assert rep.error == pytest.approx(err, rel=1e-12)
    return ctx, o


@pytest.mark.parametrize("name", ["baseline", "reference", "brooks_corey", "lens3d_4x3x3",
                                  "lens3d_8x6x4", "lens3d_16x12x10"])
@pytest.mark.parametrize("state", ["initial", "perturbed", "old_differs"])
def test_linearization_matches_oracle(ewg_mod, oracle_mod, name, state):
    case = _cases(ewg_mod)[name]()
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x0 = o.get_solution(0)
    if state == "initial":
        _compare_linearization(ewg_mod, oracle_mod, case, x0)
    elif state == "perturbed":
        _compare_linearization(ewg_mod, oracle_mod, case, _perturb(ewg_mod, case, x0, 11))
    else:
        x = _perturb(ewg_mod, case, x0, 12)
        _compare_linearization(ewg_mod, oracle_mod, case, x, xold=_perturb(ewg_mod, case, x0, 13), dt=100.0)


@pytest.mark.parametrize("name", ["baseline", "reference"])
@pytest.mark.parametrize("tag", ["init", "pert"])
def test_linearization_matches_golden(ewg_mod, gold, name, tag):
    case = {"baseline": ewg_mod.baseline_case, "reference": ewg_mod.reference_case}[name]()
    ctx = ewg_mod.Context(case)
    x = gold[f"{name}_{tag}_x"]
    ctx.set_solution(1, x)
    ctx.set_solution(0, x)
    ctx.linearize(250.0)
    _, _, b = ctx.jacobian_bcrs()
    assert rel_close(ctx.residual(), gold[f"{name}_{tag}_r"], LIN_RTOL)[0]
    for eq in range(2):
        for pv in range(2):
            assert rel_close(b[:, eq, pv], gold[f"{name}_{tag}_blocks"][:, eq, pv], LIN_RTOL)[0]


def test_linearization_is_deterministic(ewg_mod):
    case = ewg_mod.lens3d_case(16, 12, 10, seed=5, corr_cells=3.0)
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    x = _perturb(ewg_mod, case, ctx.get_solution(0), 3)
    ctx.set_solution(0, x)
    outs = []
    for _ in range(2):
        ctx.linearize(250.0)
        outs.append((ctx.residual(), ctx.jacobian_bcrs()[2]))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def _system(ewg, oracle_mod, case, seed):
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x = _perturb(ewg, case, o.get_solution(0), seed)
    o.set_solution(0, x)
    o.set_solution(1, x)
    o.linearize(250.0, 0)
    ctx = ewg.Context(case)
    rp, ci, b = o.jacobian_bcrs()
    ctx.set_matrix_bcrs(rp, ci, b)
    ctx.set_residual(o.residual())
    return ctx, o


@pytest.mark.parametrize("name", ["baseline", "lens3d_8x6x4", "lens3d_16x12x10"])
def test_spmv_and_preconditioners_match_oracle(ewg_mod, oracle_mod, name):
    case = _cases(ewg_mod)[name]()
    ctx, o = _system(ewg_mod, oracle_mod, case, 21)
    rng = np.random.Generator(np.random.PCG64(5))
    v = rng.standard_normal((o.n, 2))
    assert rel_close(ctx.apply_jacobian(v), o.apply_jacobian(v), 1e-13)[0]
    ilu = ewg_mod.default_solve_opts(precond=ewg_mod.PRECOND_ILU0)
    y_g = ctx.apply_preconditioner(v, ilu)
    y_o = o.apply_preconditioner(v, ilu, ordering=oracle_mod.ORDER_REDBLACK)
    assert rel_close(y_g, y_o, 1e-11)[0]
    jac = ewg_mod.default_solve_opts(precond=ewg_mod.PRECOND_JACOBI, preconditioner_relaxation=0.9)
    assert rel_close(ctx.apply_preconditioner(v, jac), o.apply_preconditioner(v, jac), 1e-13)[0]


@pytest.mark.parametrize("precond", [0, 1])
@pytest.mark.parametrize("name", ["baseline", "reference", "lens3d_16x12x10"])
def test_bicgstab_matches_oracle(ewg_mod, oracle_mod, name, precond):
    case = _cases(ewg_mod)[name]()
    ctx, o = _system(ewg_mod, oracle_mod, case, 31)
    opts = ewg_mod.default_solve_opts(precond=precond, linear_solver_max_iterations=2000)
    rep = ctx.solve(opts, check=True)
    dx_g = ctx.update()
    rc, dx_o, it_o, fr_o = o.solve(opts, ordering=oracle_mod.ORDER_REDBLACK)
    assert rc == 0 and rep.converged
    # both satisfy the linear tolerance on the oracle's operator (the recursively updated
    # BiCGStab residual and the true residual differ by rounding only)
    res = o.apply_jacobian(dx_g) - o.residual()
    assert np.max(np.abs(res)) <= 1e-8 * np.max(np.abs(o.residual())) + 1e-9
    assert rel_close(dx_g, dx_o, 1e-5)[0]
    # same algorithm and ordering; the dot products are summed in a different order (a fixed
    # tree on the device, sequentially in the oracle), which over hundreds of iterations moves
    # the iteration count by a few percent
    assert abs(rep.iterations - it_o) <= max(3, 0.15 * it_o), (rep.iterations, it_o)


def test_bicgstab_reference_breakdown_is_reported(ewg_mod):
    """Without the shadow restart the reference algorithm breaks down on the initial state; the
    device reports the failure (bicgstabsolver.hh:228-232, combinedcriterion.hh:150) as a status
    instead of hanging or faulting, and with the restart the same system converges."""
    case = ewg_mod.baseline_case()
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    ctx.linearize(250.0)
    rep = ctx.solve(ewg_mod.default_solve_opts(restart_on_breakdown=0))
    # the shadow residual collapses to rounding noise: exact zero -> EWG_ERR_BREAKDOWN, a few
    # ulp of noise -> the iteration diverges and the criterion fails -> EWG_ERR_NOT_CONVERGED
    assert rep.status in (4, 5) and not rep.converged
    rep = ctx.solve(ewg_mod.default_solve_opts(restart_on_breakdown=1))
    assert rep.converged and rep.restarts >= 1


def test_nonfinite_state_is_reported(ewg_mod):
    case = ewg_mod.baseline_case()
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    x = ctx.get_solution(0)
    x[100, 0] = np.nan
    ctx.set_solution(0, x)
    with pytest.raises(ewg_mod.EwgError) as ei:
        ctx.linearize(250.0)
    assert ei.value.status == 3
    assert np.isinf(ctx.residual_norm(x, 250.0))


def test_residual_norm_entry_point(ewg_mod):
    case = ewg_mod.lens3d_case(8, 6, 4, seed=2)
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    x = _perturb(ewg_mod, case, ctx.get_solution(0), 4)
    n = ctx.residual_norm(x, 250.0)
    ctx.set_solution(0, x)
    rep = ctx.linearize(250.0)
    assert n == rep.error
    # the stored iterate was not touched by the residual-only call
    assert np.array_equal(ctx.get_solution(0), x)


@pytest.mark.parametrize("name", ["baseline", "reference"])
def test_ten_steps_match_oracle(ewg_mod, oracle_mod, gold, name):
    """10 implicit-Euler steps, dt = 250 s, Newton tol 1e-8: fields within 1e-8 of the oracle and
    identical Newton iteration counts per step."""
    case = {"baseline": ewg_mod.baseline_case, "reference": ewg_mod.reference_case}[name]()
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    reps = ctx.run(10, 250.0)
    x_g = ctx.get_solution(0)
    x_o = gold[f"{name}_run10_x"]
    steps_o = gold[f"{name}_run10_steps"]
    assert [r.iterations for r in reps] == list(steps_o[:, 0])
    assert rel_close(x_g[:, 0], x_o[:, 0], 1e-8)[0]
    assert np.max(np.abs(x_g[:, 1] - x_o[:, 1])) <= 1e-8


def test_time_step_halving_on_newton_failure(ewg_mod):
    """A Newton failure restores solution(0) from solution(1) (updateFailed) and the step is
    retried with half the size (FvBaseProblem::timeIntegration)."""
    case = ewg_mod.baseline_case()
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    x_init = ctx.get_solution(0)
    nopts = ewg_mod.default_newton_opts(newton_max_iterations=2)
    st, rep = ctx.newton_apply(250.0, nopts)
    assert st == 5 and not rep.converged
    ctx.restore_time_level()
    assert np.array_equal(ctx.get_solution(0), x_init)
    reps = ctx.run(1, 250.0, nopts=ewg_mod.default_newton_opts(newton_max_iterations=4))
    assert reps[0].converged


def test_mixed_precision_newton(ewg_mod):
    """FP32 Jacobian / ILU / BiCGStab inside FP64 defect correction reaches the same Newton
    tolerance; the fields stay within 1e-8 of the FP64 path after 3 steps."""
    case = ewg_mod.baseline_case()
    c64 = ewg_mod.Context(case)
    c64.apply_initial_solution()
    c64.run(3, 250.0)
    c32 = ewg_mod.Context(case)
    c32.apply_initial_solution()
    mixed = ewg_mod.default_solve_opts(precision=ewg_mod.PRECISION_MIXED)
    reps = c32.run(3, 250.0, sopts=mixed)
    assert all(r.converged and r.error <= 1e-8 for r in reps)
    a, b = c64.get_solution(0), c32.get_solution(0)
    assert rel_close(b[:, 0], a[:, 0], 1e-8)[0]
    assert np.max(np.abs(b[:, 1] - a[:, 1])) <= 1e-8


@pytest.mark.parametrize("precond", [0, 1])
def test_repeated_import_and_solve_is_bitwise_reproducible(ewg_mod, oracle_mod, precond):
    """Fresh contexts on recycled device memory: the imported matrix and the whole BiCGStab run
    are stream-ordered and deterministic, so repeated runs agree bit for bit."""
    case = _cases(ewg_mod)["lens3d_16x12x10"]()
    outs = []
    for _ in range(4):
        ctx, o = _system(ewg_mod, oracle_mod, case, 21)
        rep = ctx.solve(ewg_mod.default_solve_opts(precond=precond, linear_solver_max_iterations=2000))
        outs.append((rep.iterations, ctx.update()))
        ctx.close()
    for it, dx in outs[1:]:
        assert it == outs[0][0] and np.array_equal(dx, outs[0][1])
    res = o.apply_jacobian(outs[0][1]) - o.residual()
    assert np.max(np.abs(res)) <= 1e-8 * np.max(np.abs(o.residual())) + 1e-9


# ---- finite-difference local linearizer (FvBaseFdLocalLinearizer) ----------------------------
# A difference quotient divides residual differences by the deflection (0.9123e-11 p_ref for the
# pressure, 0.9123e-10 for the saturation). The two-point gradient is a sum of terms of size
# rho g ~ 1e4 Pa/m while the pressure deflection moves it by ~1e-5 Pa/m, so one rounding
# difference between two evaluation orders (the GPU fuses multiply-adds, the oracle does not)
# moves a pressure derivative by ~1e-7 of its size; the GPU and oracle FD Jacobians are compared
# at FD_RTOL of each component's magnitude. The residual is not differenced and keeps LIN_RTOL.
FD_RTOL = 1e-4


@pytest.mark.parametrize("name", ["baseline", "reference", "brooks_corey", "lens3d_8x6x4", "lens3d_16x12x10"])
@pytest.mark.parametrize("method", [1, 0, -1])
def test_fd_linearizer_matches_oracle(ewg_mod, oracle_mod, name, method):
    case = _cases(ewg_mod)[name]()
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x = _perturb(ewg_mod, case, o.get_solution(0), 21)
    ctx = ewg_mod.Context(case)
    ctx.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, method)
    o.set_local_linearizer(1, method)
    for c in (ctx, o):
        c.set_solution(1, x)
        c.set_solution(0, x)
    o.set_recycle_first_iteration_storage(False)
    ctx.linearize(250.0)
    o.linearize(250.0, 0)
    r_g, r_o = ctx.residual(), o.residual()
    _, _, b_g = ctx.jacobian_bcrs()
    _, _, b_o = o.jacobian_bcrs()
    assert rel_close(r_g, r_o, LIN_RTOL, scale=max(np.max(np.abs(r_o)), 1e-3))[0]
    for eq in range(2):
        for pv in range(2):
            ok, e, s = rel_close(b_g[:, eq, pv], b_o[:, eq, pv], FD_RTOL)
            assert ok, ("fd vs oracle fd", eq, pv, e, s)


@pytest.mark.parametrize("name", ["baseline", "lens3d_8x6x4"])
@pytest.mark.parametrize("method", [1, 0])
def test_fd_linearizer_close_to_ad(ewg_mod, name, method):
    """Away from the laws' kinks and from upwind ties (saturations in (0.3, 1), pressures off
    hydrostatic), the FD Jacobian is the AD Jacobian to the quotient's truncation error."""
    case = _cases(ewg_mod)[name]()
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    x = ctx.get_solution(0)
    rng = np.random.Generator(np.random.PCG64(0))
    x[:, 1] = rng.uniform(0.3, 1.0, size=len(x))
    x[:, 0] += rng.normal(0, 50.0, size=len(x))
    ctx.set_solution(1, x)
    ctx.set_solution(0, x)
    ctx.linearize(250.0)
    _, _, b_ad = ctx.jacobian_bcrs()
    ctx.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, method)
    ctx.linearize(250.0)
    _, _, b_fd = ctx.jacobian_bcrs()
    for eq in range(2):
        for pv in range(2):
            ok, e, s = rel_close(b_fd[:, eq, pv], b_ad[:, eq, pv], 1e-4 if method else 1e-5)
            assert ok, ("fd vs ad", eq, pv, e, s)


@pytest.mark.parametrize("name", ["baseline", "lens3d_8x6x4"])
def test_fd_newton_steps_match_oracle(ewg_mod, oracle_mod, name):
    """Five implicit steps with the FD local linearizer on both sides: identical Newton
    iteration counts and fields within 1e-8 of the oracle."""
    case = _cases(ewg_mod)[name]()
    ctx = ewg_mod.Context(case)
    ctx.set_local_linearizer(ewg_mod.LOCAL_LINEARIZER_FD, 1)
    o = oracle_mod.Oracle(case)
    o.set_local_linearizer(1, 1)
    ctx.apply_initial_solution()
    o.apply_initial_solution()
    so = ewg_mod.default_solve_opts(verify_true_residual=0)
    reps = ctx.run(5, 250.0, sopts=so)
    oreps = o.run(5, 250.0, sopts=so)
    assert [r.iterations for r in reps] == [a for a, _ in oreps]
    xg, xo = ctx.get_solution(0), o.get_solution(0)
    assert rel_close(xg[:, 0], xo[:, 0], 1e-8)[0]
    assert np.max(np.abs(xg[:, 1] - xo[:, 1])) <= 1e-8
