"""GPU parity of the vertex-centred (VCFV, P1 gradient) linearization and Newton solve with the
CPU oracle: residual and Jacobian at perturbed states of 2D presets and 3D lens grids (within
1e-12 of each row's scale: the device sums the same products in the reference's element order),
the same upstream choices (a flipped upwind decision would show as an O(1) Jacobian difference),
and Newton with BiCGStab + block Jacobi taking the same iteration counts and reaching the same
states."""
import numpy as np
import pytest

from conftest import rel_close

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _cases(ewg):
    return {
        "baseline_2d": ewg.vcfv_case(ewg.baseline_case(12, 8)),
        "reference_2d": ewg.vcfv_case(ewg.reference_case(10, 6)),
        "lens3d_small": ewg.vcfv_case(ewg.lens3d_case(6, 5, 4, seed=1)),
        "lens3d_odd": ewg.vcfv_case(ewg.lens3d_case(9, 7, 5, seed=2)),
    }


def _states(oracle, case, steps=2):
    """A stepped state (x1) and a perturbed iterate (x0) from the oracle."""
    o = oracle.VcfvOracle(case)
    o.apply_initial_solution()
    for _ in range(steps):
        st, its, lin, err = o.newton_apply(250.0)
        assert st == 0, o.err()
        o.advance_time_level()
    x1 = o.get_solution(0)
    rng = np.random.default_rng(11)
    x0 = x1.copy()
    x0[:, 0] += rng.normal(0, 20.0, o.n)
    x0[:, 1] = np.clip(x0[:, 1] - np.abs(rng.normal(0, 0.03, o.n)), 0.4, 1.0)
    return o, x1, x0


@pytest.mark.parametrize("name", ["baseline_2d", "reference_2d", "lens3d_small", "lens3d_odd"])
def test_vcfv_linearization_matches_oracle(ewg_mod, oracle_mod, name):
    case = _cases(ewg_mod)[name]
    o, x1, x0 = _states(oracle_mod, case)
    # oracle: storage cache from solution(1) at iteration 0, then the iterate at iteration 1
    o.set_solution(1, x1)
    o.set_solution(0, x1)
    o.linearize(250.0, 0)
    o.set_solution(0, x0)
    e_ref = o.linearize(250.0, 1)
    r_ref = o.residual()
    rp, ci, b_ref = o.jacobian_bcrs()
    g = ewg_mod.VcfvContext(case)
    g.set_solution(1, x1)
    g.set_solution(0, x0)
    e = g.linearize(250.0)
    r = g.residual()
    rp2, ci2, b = g.jacobian_bcrs()
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2)
    ok, err, s = rel_close(r, r_ref, RTOL)
    assert ok, (err, s)
    assert abs(e - e_ref) <= RTOL * e_ref
    # per row: the row's largest block entry is the scale
    for row in range(o.n):
        blk = slice(rp[row], rp[row + 1])
        ok, err, s = rel_close(b[blk], b_ref[blk], RTOL)
        assert ok, (row, err, s)
    g.close()


@pytest.mark.parametrize("name", ["baseline_2d", "lens3d_small"])
def test_vcfv_newton_matches_oracle(ewg_mod, oracle_mod, name):
    case = _cases(ewg_mod)[name]
    so = ewg_mod.default_solve_opts(precond=ewg_mod.PRECOND_JACOBI, linear_solver_tolerance=1e-10,
                                    linear_solver_max_iterations=5000)
    o = oracle_mod.VcfvOracle(case)
    o.apply_initial_solution()
    g = ewg_mod.VcfvContext(case)
    g.apply_initial_solution()
    assert np.array_equal(g.get_solution(0), o.get_solution(0))
    for step in range(3):
        st_o, its_o, lin_o, err_o = o.newton_apply(250.0, None, so)
        st_g, its_g, lin_g, err_g = g.newton_apply(250.0, None, so)
        assert st_o == 0 and st_g == 0, (st_o, st_g)
        assert its_g == its_o, (step, its_g, its_o)
        xo, xg = o.get_solution(0), g.get_solution(0)
        assert np.max(np.abs(xg[:, 0] - xo[:, 0])) <= 1e-9 * np.max(np.abs(xo[:, 0]))
        assert np.max(np.abs(xg[:, 1] - xo[:, 1])) <= 1e-9
        o.advance_time_level()
        g.advance_time_level()
    assert g.launches > 0
    g.close()


# finite-difference quotients amplify the last-bit differences of the two evaluations by 1/eps
FD_RTOL = 1e-4


@pytest.mark.parametrize("name", ["baseline_2d", "lens3d_small"])
@pytest.mark.parametrize("method", [1, 0])
def test_vcfv_fd_linearization_matches_oracle(ewg_mod, oracle_mod, name, method):
    """lens_immiscible_vcfv_fd: the FD local linearizer on the device against the oracle's, same
    deflections (BaseEpsilon / primaryVarWeight with the updateBegin reference pressure)."""
    case = _cases(ewg_mod)[name]
    o, x1, x0 = _states(oracle_mod, case)
    o.set_local_linearizer(1, method)
    o.set_solution(1, x1)
    o.set_solution(0, x1)
    o.linearize(250.0, 0)
    o.set_solution(0, x0)
    o.update_begin()
    o.linearize(250.0, 1)
    r_ref = o.residual()
    rp, ci, b_ref = o.jacobian_bcrs()
    g = ewg_mod.VcfvContext(case)
    g.set_local_linearizer(1, method)
    g.set_solution(1, x1)
    g.set_solution(0, x0)
    g.update_begin()
    g.linearize(250.0)
    ok, err, s = rel_close(g.residual(), r_ref, RTOL)
    assert ok, (err, s)
    _, _, b = g.jacobian_bcrs()
    for row in range(o.n):
        blk = slice(rp[row], rp[row + 1])
        ok, err, s = rel_close(b[blk], b_ref[blk], FD_RTOL)
        assert ok, (row, err, s)
    g.close()


def test_vcfv_fd_newton_matches_oracle(ewg_mod, oracle_mod):
    case = _cases(ewg_mod)["baseline_2d"]
    so = ewg_mod.default_solve_opts(precond=ewg_mod.PRECOND_JACOBI, linear_solver_tolerance=1e-10,
                                    linear_solver_max_iterations=5000)
    o = oracle_mod.VcfvOracle(case)
    o.set_local_linearizer(1, 1)
    o.apply_initial_solution()
    g = ewg_mod.VcfvContext(case)
    g.set_local_linearizer(1, 1)
    g.apply_initial_solution()
    for step in range(2):
        st_o, its_o, _, _ = o.newton_apply(250.0, None, so)
        st_g, its_g, _, _ = g.newton_apply(250.0, None, so)
        assert st_o == 0 and st_g == 0 and its_g == its_o, (step, its_g, its_o)
        xo, xg = o.get_solution(0), g.get_solution(0)
        assert np.max(np.abs(xg[:, 1] - xo[:, 1])) <= 1e-8
        o.advance_time_level()
        g.advance_time_level()
    g.close()


@pytest.mark.parametrize("name", ["baseline_2d", "lens3d_small", "lens3d_odd"])
def test_vcfv_ilu_newton_matches_oracle(ewg_mod, oracle_mod, name):
    """Newton with BiCGStab + block ILU(0) in the parity-colour order (the device's) against the
    oracle's bilu0 on the same permuted matrix: same Newton iteration counts, same states."""
    case = _cases(ewg_mod)[name]
    so = ewg_mod.default_solve_opts(precond=ewg_mod.PRECOND_ILU0, linear_solver_tolerance=1e-10,
                                    linear_solver_max_iterations=5000)
    o = oracle_mod.VcfvOracle(case)
    o.apply_initial_solution()
    g = ewg_mod.VcfvContext(case)
    g.apply_initial_solution()
    for step in range(3):
        st_o, its_o, lin_o, _ = o.newton_apply(250.0, None, so, oracle_mod.ORDER_COLOURS)
        st_g, its_g, lin_g, _ = g.newton_apply(250.0, None, so)
        assert st_o == 0 and st_g == 0, (st_o, st_g)
        assert its_g == its_o, (step, its_g, its_o)
        assert abs(lin_g - lin_o) <= max(2, 0.1 * lin_o), (step, lin_g, lin_o)
        xo, xg = o.get_solution(0), g.get_solution(0)
        assert np.max(np.abs(xg[:, 0] - xo[:, 0])) <= 1e-9 * np.max(np.abs(xo[:, 0]))
        assert np.max(np.abs(xg[:, 1] - xo[:, 1])) <= 1e-9
        o.advance_time_level()
        g.advance_time_level()
    g.close()


@pytest.mark.parametrize("shape", [(1, 1), (2, 1), (1, 1, 1), (2, 1, 3)])
def test_vcfv_minimal_grids_match_oracle(ewg_mod, oracle_mod, shape):
    """Grids of one or a few elements: every vertex is a corner or edge vertex, every element
    touches the boundary on most faces."""
    if len(shape) == 2:
        base = ewg_mod.baseline_case(*shape)
    else:
        base = ewg_mod.lens3d_case(*shape, seed=3)
    case = ewg_mod.vcfv_case(base)
    o = oracle_mod.VcfvOracle(case)
    o.apply_initial_solution()
    x1 = o.get_solution(0)
    x0 = x1.copy()
    x0[:, 1] = np.linspace(0.6, 1.0, len(x0))
    o.set_solution(1, x1); o.set_solution(0, x1); o.linearize(250.0, 0)
    o.set_solution(0, x0); e_ref = o.linearize(250.0, 1)
    rp, ci, b_ref = o.jacobian_bcrs()
    g = ewg_mod.VcfvContext(case)
    g.set_solution(1, x1)
    g.set_solution(0, x0)
    e = g.linearize(250.0)
    ok, err, s = rel_close(g.residual(), o.residual(), RTOL)
    assert ok, (err, s)
    _, _, b = g.jacobian_bcrs()
    for row in range(o.n):
        blk = slice(rp[row], rp[row + 1])
        ok, err, s = rel_close(b[blk], b_ref[blk], RTOL)
        assert ok, (row, err, s)
    assert abs(e - e_ref) <= RTOL * e_ref
    g.close()


@pytest.mark.parametrize("precond", ["ilu0", "jacobi"])
def test_vcfv_solve_entry_point(ewg_mod, oracle_mod, precond):
    """ewg_vcfv_solve (the LinearSolverBackend::solve contract): after a linearization, the update
    it returns satisfies J dx = r to the requested relative tolerance, checked with the exported
    BCRS Jacobian."""
    case = _cases(ewg_mod)["lens3d_small"]
    _, x1, x0 = _states(oracle_mod, case)
    g = ewg_mod.VcfvContext(case)
    g.set_solution(1, x1)
    g.set_solution(0, x0)
    g.linearize(250.0)
    r = g.residual().ravel()
    rp, ci, b = g.jacobian_bcrs()
    pc = ewg_mod.PRECOND_ILU0 if precond == "ilu0" else ewg_mod.PRECOND_JACOBI
    so = ewg_mod.default_solve_opts(precond=pc, linear_solver_tolerance=1e-10, linear_solver_max_iterations=5000)
    st, its, dx = g.solve(so)
    assert st == 0 and its > 0
    dxf = dx.ravel()
    Jdx = np.zeros_like(r)
    for row in range(g.n):
        for q in range(rp[row], rp[row + 1]):
            Jdx[2 * row:2 * row + 2] += b[q] @ dxf[2 * ci[q]:2 * ci[q] + 2]
    assert np.max(np.abs(Jdx - r)) <= 1e-8 * np.max(np.abs(r))
    g.close()


def test_vcfv_jacobian_export_rejects_foreign_pattern(ewg_mod):
    """A BCRS pattern with a block outside the vertex stencil is an error, not a read of a band the
    device does not store."""
    import ctypes as C
    case = ewg_mod.vcfv_case(ewg_mod.baseline_case(6, 4))
    g = ewg_mod.VcfvContext(case)
    g.apply_initial_solution()
    g.linearize(250.0)
    rp, ci = ewg_mod.vcfv_pattern(case.grid)
    bad = ci.copy()
    bad[0] = g.n - 1  # row 0 coupled to the far corner
    blocks = np.zeros((len(ci), 2, 2))
    st = g.lib.ewg_vcfv_get_jacobian_bcrs(g.h, ewg_mod._ptr(rp, C.c_int32), ewg_mod._ptr(bad, C.c_int32), len(ci),
                                          ewg_mod._ptr(blocks))
    assert st == 1
    g.close()
