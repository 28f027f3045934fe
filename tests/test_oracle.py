"""CPU pins of the oracle (the parity checker).

The reference cannot be built here and ships no golden vectors (parity unpinned at the
ewoms-material / dune-istl boundary), so the oracle is pinned by properties the reference's own
algorithms guarantee: the AD Jacobian equals a finite-difference Jacobian of the residual
(fvbasefdlocallinearizer.hh), discrete mass conservation (checkConservativeness,
fvbasediscretization.hh:969-1080), the hydrostatic initial state of LensProblem::initial has a zero
residual away from the inlet, the material laws are continuous across their regularisation
thresholds, BiCGStab with r0hat = b breaks down exactly on the initial state as the reference's
algorithm does, and the committed golden fixtures.
"""
import os

import numpy as np
import pytest

from conftest import ROOT, rel_close

GOLD = os.path.join(ROOT, "tests", "golden", "lens2d_golden.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _oracle_lin(oracle_mod, case, x, dt=250.0):
    o = oracle_mod.Oracle(case)
    o.set_solution(0, x)
    o.set_solution(1, x)
    e = o.linearize(dt, 0)
    return o, e


@pytest.mark.parametrize("name", ["baseline", "reference"])
@pytest.mark.parametrize("tag", ["init", "pert"])
def test_oracle_reproduces_golden_linearization(oracle_mod, ewg_mod, gold, name, tag):
    case = {"baseline": ewg_mod.baseline_case, "reference": ewg_mod.reference_case}[name]()
    x = gold[f"{name}_{tag}_x"]
    o, e = _oracle_lin(oracle_mod, case, x)
    rp, ci, b = o.jacobian_bcrs()
    assert np.array_equal(rp, gold[f"{name}_{tag}_row_ptr"])
    assert np.array_equal(ci, gold[f"{name}_{tag}_col_idx"])
    assert rel_close(o.residual(), gold[f"{name}_{tag}_r"], 1e-14)[0]
    assert rel_close(b, gold[f"{name}_{tag}_blocks"], 1e-14)[0]
    assert e == pytest.approx(float(gold[f"{name}_{tag}_error"]), rel=1e-14)


def test_oracle_reproduces_golden_run(oracle_mod, ewg_mod, gold):
    case = ewg_mod.baseline_case()
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    steps = o.run(10, 250.0)
    assert np.array_equal(np.array(steps), gold["baseline_run10_steps"])
    x = o.get_solution(0)
    assert rel_close(x[:, 0], gold["baseline_run10_x"][:, 0], 1e-12)[0]
    assert rel_close(x[:, 1], gold["baseline_run10_x"][:, 1], 1e-12, scale=1.0)[0]


def test_material_golden_and_continuity(oracle_mod, ewg_mod, gold):
    sws = gold["mat_sw"]
    for mname, mat in (("vg_outer", ewg_mod.baseline_case().problem.outer),
                       ("vg_lens", ewg_mod.baseline_case().problem.lens),
                       ("bc_outer", ewg_mod.brooks_corey_case().problem.outer)):
        got = np.array([oracle_mod.material_eval(mat, s) for s in sws])
        assert np.allclose(got, gold[f"mat_{mname}"], rtol=1e-14, atol=0)
        # continuity of p_c at the regularisation thresholds (absolute saturations)
        den = 1.0 - (mat.swr + mat.snr)
        # (a jump that shrinks in proportion to the probe distance is a slope, not a jump)
        for se in (0.01, 0.99, 1.0):
            sw = mat.swr + se * den
            jumps = []
            for h in (1e-7, 1e-9):
                lo = oracle_mod.material_eval(mat, sw - h)[0]
                hi = oracle_mod.material_eval(mat, sw + h)[0]
                jumps.append(abs(hi - lo))
            assert jumps[1] <= jumps[0] / 20 + 1e-9 * abs(lo), (mname, se, jumps)
        # AD derivative equals a central difference of the value inside each smooth piece
        for sw in (mat.swr + 0.3 * den, mat.swr + 0.995 * den, mat.swr + 0.005 * den):
            h = 1e-7
            v = oracle_mod.material_eval(mat, sw)
            vp = oracle_mod.material_eval(mat, sw + h)
            vm = oracle_mod.material_eval(mat, sw - h)
            for k in (0, 2, 4):
                fd = (vp[k] - vm[k]) / (2 * h)
                assert abs(fd - v[k + 1]) <= 1e-5 * max(1.0, abs(v[k + 1])), (mname, sw, k, fd, v[k + 1])


def test_hydrostatic_initial_residual(oracle_mod, ewg_mod):
    """LensProblem::initial is in hydrostatic equilibrium: only the inlet cells carry a residual
    (the DNAPL inflow 0.04 kg/(m^2 s) x face area / cell volume on the non-wetting equation)."""
    case = ewg_mod.baseline_case()
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    o.linearize(250.0, 0)
    r = o.residual()
    xc, yc, _ = ewg_mod.cell_centers(case.grid)
    inlet = (yc > 4.0 - 0.125) & (xc > 2.25) & (xc < 3.75)
    assert np.max(np.abs(r[~inlet])) < 1e-12
    assert np.allclose(r[inlet, 1], -0.04 * 0.125 / (0.125 * 0.125), rtol=1e-12)
    assert np.max(np.abs(r[inlet, 0])) < 1e-12


def test_ad_jacobian_matches_finite_differences(oracle_mod, ewg_mod):
    case = ewg_mod.baseline_case(nx=8, ny=6)
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x = o.get_solution(0)
    rng = np.random.Generator(np.random.PCG64(7))
    x[:, 1] = rng.uniform(0.3, 0.9, size=len(x))
    x[:, 0] += rng.normal(0, 300.0, size=len(x))
    o.set_solution(0, x)
    o.set_solution(1, x)
    o.linearize(250.0, 0)
    _, _, J = o.jacobian_bcrs()
    Jfd = o.fd_jacobian(250.0)
    for pv in (0, 1):
        a, b = J[:, :, pv], Jfd[:, :, pv]
        scale = np.max(np.abs(a))
        assert np.max(np.abs(a - b)) <= 2e-5 * scale, (pv, np.max(np.abs(a - b)), scale)


@pytest.mark.parametrize("method", [1, 0, -1])
def test_fd_local_linearizer_matches_ad(oracle_mod, ewg_mod, method):
    """FvBaseFdLocalLinearizer restated: same residual as the AD linearizer, Jacobian within the
    difference quotient's error (forward / backward first order, central second order)."""
    case = ewg_mod.baseline_case()
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x = o.get_solution(0)
    rng = np.random.Generator(np.random.PCG64(0))
    x[:, 1] = rng.uniform(0.3, 1.0, size=len(x))
    x[:, 0] += rng.normal(0, 50.0, size=len(x))
    o.set_solution(1, x)
    o.set_solution(0, x)
    o.linearize(250.0)
    r_ad = o.residual()
    _, _, J_ad = o.jacobian_bcrs()
    o.set_local_linearizer(1, method)
    o.linearize(250.0)
    assert np.array_equal(o.residual(), r_ad)
    _, _, J_fd = o.jacobian_bcrs()
    tol = 5e-5 if method else 5e-6
    for eq in range(2):
        for pv in range(2):
            a, b = J_fd[:, eq, pv], J_ad[:, eq, pv]
            assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(b)), (eq, pv)


def test_mass_conservation(oracle_mod, ewg_mod):
    """sum_i R_i V_i = storage change / dt + boundary outflow: interior face fluxes cancel."""
    case = ewg_mod.baseline_case()
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    o.run(3, 250.0)
    x1 = o.get_solution(0)
    # take a non-converged iterate so the residual is far from zero
    x = x1.copy()
    x[:, 1] = np.clip(x[:, 1] - 0.01, 0.0, 1.0)
    o.set_solution(1, x1)
    o.set_solution(0, x)
    # with the storage cache recycling the first iterate the old storage would be taken from x;
    # take it from solution(1) explicitly
    o.set_recycle_first_iteration_storage(False)
    o.linearize(250.0, 0)
    V = (6.0 / 48) * (4.0 / 32)
    total = o.residual().sum(axis=0) * V
    s_new = o.global_storage(0)
    s_old = o.global_storage(1)
    bnd = o.boundary_rates()
    expect = (s_new - s_old) / 250.0 + bnd
    assert np.allclose(total, expect, rtol=1e-9, atol=1e-12 * np.max(np.abs(s_new)))


def test_bicgstab_reference_breakdown_and_restart(oracle_mod, ewg_mod):
    """On the initial state r0hat = b lives only in decoupled non-wetting rows, so the reference
    algorithm in FP64 breaks down exactly; the shadow-residual restart recovers."""
    case = ewg_mod.baseline_case()
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    o.linearize(250.0, 0)
    rc, _, _, _ = o.solve(ewg_mod.default_solve_opts(restart_on_breakdown=0))
    assert rc == 4  # EWG_ERR_BREAKDOWN
    rc, dx, it, fr = o.solve(ewg_mod.default_solve_opts(restart_on_breakdown=1))
    assert rc == 0 and fr <= 1e-10
    rcb, dxb, itb, frb = o.solve(ewg_mod.default_solve_opts(), ordering=oracle_mod.ORDER_REDBLACK)
    assert rcb == 0
    # both orderings solve the same system to the linear tolerance
    Ax = o.apply_jacobian(dxb)
    assert np.max(np.abs(Ax - o.residual())) <= 1e-9


def test_ilu_exact_where_no_fill_is_dropped(oracle_mod, ewg_mod):
    """Block ILU(0) is an exact factorisation when the elimination creates no fill outside the
    pattern: a single grid row (block-tridiagonal) in natural order, and a block-diagonal matrix in
    either order. Then M^-1 A v = v."""
    rng = np.random.Generator(np.random.PCG64(3))
    case = ewg_mod.baseline_case(nx=8, ny=1)
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x = o.get_solution(0)
    x[:, 1] = rng.uniform(0.4, 0.9, size=len(x))
    o.set_solution(0, x)
    o.set_solution(1, x)
    o.linearize(250.0, 0)
    v = rng.standard_normal((o.n, 2))
    y = o.apply_preconditioner(o.apply_jacobian(v), ordering=oracle_mod.ORDER_NATURAL)
    assert np.max(np.abs(y - v)) <= 1e-9 * np.max(np.abs(v))
    rp, ci, b = o.jacobian_bcrs()
    rows = np.repeat(np.arange(o.n), np.diff(rp))
    b = b.copy()
    b[ci != rows] = 0.0
    o.set_jacobian_blocks(b)
    for ordering in (oracle_mod.ORDER_NATURAL, oracle_mod.ORDER_REDBLACK):
        y = o.apply_preconditioner(o.apply_jacobian(v), ordering=ordering)
        assert np.max(np.abs(y - v)) <= 1e-9 * np.max(np.abs(v))  # 2x2 blocks with condition ~1e4


def test_newton_run_mass_balance(oracle_mod, ewg_mod):
    """Over 10 steps the DNAPL mass in the domain equals the injected mass minus the outflow."""
    case = ewg_mod.baseline_case()
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    m0 = o.global_storage(1)
    steps = o.run(10, 250.0)
    assert all(1 <= ni <= 18 for ni, _ in steps)
    m1 = o.global_storage(0)
    # inflow through the inlet faces: 12 faces x 0.125 m x 0.04 kg/(m^2 s) x 2500 s; no DNAPL
    # leaves through the hydrostatic side boundaries while they stay water-saturated
    injected = 12 * 0.125 * 0.04 * 2500.0
    assert m1[1] - m0[1] == pytest.approx(injected, rel=1e-6)


def test_oracle_rejects_bad_reference_pressure(oracle_mod):
    """orc_set_reference_pressure rejects a value that is not positive and finite, like the
    device's ewg_set_reference_pressure (EWG_ERR_INVALID), and keeps the stored value."""
    import ewg
    o = oracle_mod.Oracle(ewg.baseline_case())
    o.apply_initial_solution()
    o.set_reference_pressure(1.2e5)
    for bad in (0.0, -1e5, float("nan"), float("inf")):
        with pytest.raises(ValueError):
            o.set_reference_pressure(bad)
    o.set_local_linearizer(1, 1)
    o.linearize(250.0, 0)  # still linearizes with the stored 1.2e5


def test_box8_ordering_is_a_permutation_and_converges_faster(oracle_mod):
    """ORC_ORDER_BOX8 (2x2x2 boxes in eight colours, natural order inside a box) factorizes the
    same matrix as the other orders: its preconditioned BiCGStab solves the system, and on the 3D
    lens it needs fewer iterations than the red-black order (the reference's natural order needs
    the fewest)."""
    import ewg
    case = ewg.lens3d_case(16, 16, 8, seed=4, corr_cells=4.0)
    o = oracle_mod.Oracle(case)
    o.apply_initial_solution()
    x = o.get_solution(0)
    rng = np.random.Generator(np.random.PCG64(3))
    x[:, 1] = 1.0 - 0.5 * rng.uniform(size=len(x)) * (np.arange(len(x)) % 7 == 0)
    o.set_solution(0, x)
    o.set_solution(1, x)
    o.linearize(250.0, 0)
    opts = ewg.default_solve_opts(linear_solver_max_iterations=2000)
    its = {}
    for name, order in (("natural", oracle_mod.ORDER_NATURAL), ("redblack", oracle_mod.ORDER_REDBLACK),
                        ("box8", oracle_mod.ORDER_BOX8)):
        rc, dx, it, _ = o.solve(opts, ordering=order)
        assert rc == 0, name
        res = o.apply_jacobian(dx) - o.residual()
        assert np.max(np.abs(res)) <= 1e-8 * np.max(np.abs(o.residual())) + 1e-9, name
        its[name] = it
    assert its["natural"] <= its["box8"] < its["redblack"], its
