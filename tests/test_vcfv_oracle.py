"""CPU pins of the vertex-centred (VCFV, P1 gradients) oracle.

As for the cell-centred path there is no reference binary and no golden vector: the oracle is held
to properties the reference's algorithms guarantee. The AD Jacobian equals a central finite
difference of the residual; fluxes over interior sub-control-volume faces cancel, so the residual
weighted by the control volumes sums to the storage change plus the boundary rates; the
hydrostatic initial state has a zero residual away from the inlet; the structured element's
geometry is that of the box method (areas, normals from i to j, P1 gradients that sum to zero and
reproduce linear fields).
"""
import numpy as np
import pytest


def _cases(ewg):
    return [ewg.vcfv_case(ewg.baseline_case(12, 8)), ewg.vcfv_case(ewg.reference_case(10, 6)),
            ewg.vcfv_case(ewg.lens3d_case(6, 5, 4, seed=1))]


def _stepped(oracle, case, steps=2):
    o = oracle.VcfvOracle(case)
    o.apply_initial_solution()
    for _ in range(steps):
        st, its, lin, err = o.newton_apply(250.0)
        assert st == 0, o.err()
        o.advance_time_level()
    return o


def test_geometry_is_the_box_method(oracle_mod, ewg_mod):
    for case in _cases(ewg_mod):
        o = oracle_mod.VcfvOracle(case)
        g = o.geometry()
        dim = case.grid.dim
        h = np.array([case.grid.lx / case.grid.nx, case.grid.ly / case.grid.ny,
                      case.grid.lz / case.grid.nz if dim == 3 else 1.0])
        vb = np.array([[(v >> d) & 1 for d in range(3)] for v in range(8)], dtype=float)
        for k in range(len(g["area"])):
            i, j = g["ij"][k]
            dx = (vb[j] - vb[i])[:dim] * h[:dim]
            # the normal points from i to j along the edge, and the face is a quarter (3D) or
            # half (2D) of the element's cross-section
            assert np.allclose(g["nrm"][k][:dim], dx / np.linalg.norm(dx))
            axis = int(np.argmax(np.abs(dx)))
            cross = np.prod([h[d] for d in range(dim) if d != axis])
            assert np.isclose(g["area"][k], cross / (4.0 if dim == 3 else 2.0))
            G = g["G"][k][: 1 << dim, :dim]
            assert np.allclose(G.sum(axis=0), 0.0, atol=1e-12)
            # a linear field a . x is reproduced exactly by the P1 gradient
            a = np.array([0.3, -1.7, 2.2])[:dim]
            vals = (vb[: 1 << dim, :dim] * h[:dim]) @ a
            assert np.allclose(vals @ G, a)
        assert np.isclose(o.total_volumes().sum(), np.prod(h[:dim]) * np.prod(
            [case.grid.nx, case.grid.ny] + ([case.grid.nz] if dim == 3 else [])))


def test_vcfv_ad_jacobian_matches_finite_differences(oracle_mod, ewg_mod):
    for case in _cases(ewg_mod):
        o = _stepped(oracle_mod, case)
        x0 = o.get_solution(0)
        o.set_solution(1, x0)
        o.linearize(250.0, 0)  # storage cache from solution(1)
        rng = np.random.default_rng(3)
        x = x0.copy()
        x[:, 0] += rng.normal(0, 50.0, o.n)
        x[:, 1] = np.clip(x[:, 1] - np.abs(rng.normal(0, 0.05, o.n)), 0.3, 1.0)
        o.set_solution(0, x)
        o.linearize(250.0, 1)
        rp, ci, B = o.jacobian_bcrs()
        J = np.zeros((2 * o.n, 2 * o.n))
        for r in range(o.n):
            for q in range(rp[r], rp[r + 1]):
                J[2 * r:2 * r + 2, 2 * ci[q]:2 * ci[q] + 2] = B[q]
        cols = rng.choice(o.n, size=min(o.n, 12), replace=False)
        for c in cols:
            for pv, eps in ((0, 1e-2), (1, 1e-7)):
                xp, xm = x.copy(), x.copy()
                xp[c, pv] += eps
                xm[c, pv] -= eps
                o.set_solution(0, xp); o.linearize(250.0, 1); rp_ = o.residual().ravel()
                o.set_solution(0, xm); o.linearize(250.0, 1); rm_ = o.residual().ravel()
                fd = (rp_ - rm_) / (2 * eps)
                ad = J[:, 2 * c + pv]
                scale = np.max(np.abs(ad)) + 1e-30
                assert np.max(np.abs(fd - ad)) <= 2e-5 * scale, (case.name, c, pv)
        o.set_solution(0, x)


def test_vcfv_mass_conservation(oracle_mod, ewg_mod):
    for case in _cases(ewg_mod):
        o = _stepped(oracle_mod, case, steps=1)
        x1 = o.get_solution(0)
        o.set_solution(1, x1)
        o.linearize(250.0, 0)
        rng = np.random.default_rng(5)
        x = x1.copy()
        x[:, 0] += rng.normal(0, 30.0, o.n)
        x[:, 1] = np.clip(x[:, 1] - np.abs(rng.normal(0, 0.02, o.n)), 0.5, 1.0)
        o.set_solution(0, x)
        o.linearize(250.0, 1)
        r = o.residual()
        V = o.total_volumes()
        total = (r * V[:, None]).sum(axis=0)
        m0, m1 = o.global_storage(0), o.global_storage(1)
        expect = (m0 - m1) / 250.0 + o.boundary_rates()
        scale = np.abs(r * V[:, None]).max()
        assert np.allclose(total, expect, rtol=0, atol=1e-9 * scale), (case.name, total, expect)


def test_vcfv_hydrostatic_initial_residual(oracle_mod, ewg_mod):
    case = ewg_mod.vcfv_case(ewg_mod.baseline_case(24, 16))
    o = oracle_mod.VcfvOracle(case)
    o.apply_initial_solution()
    o.linearize(250.0, 0)
    r = o.residual()
    x, y, _ = ewg_mod.vertex_positions(case.grid)
    hx, hy = 6.0 / 24, 4.0 / 16
    away = (y < 4.0 - 1.5 * hy) | (x < 2.25 - 1.5 * hx) | (x > 3.75 + 1.5 * hx)
    # a vertex on the left / right boundary sees the free-flow state at the integration points of
    # its boundary sub-faces, a quarter cell above and below it, through a horizontal two-point
    # gradient from its SCV centre: the two hydrostatic differences cancel except at the corners,
    # where the vertex has one sub-face on that boundary
    corner = ((x == 0.0) | (x == 6.0)) & ((y == 0.0) | (y == 4.0))
    assert np.all(np.abs(r[corner][:, 0]) > 0)
    keep = away & ~corner
    assert np.max(np.abs(r[keep])) < 1e-9 * np.max(np.abs(r))
    assert np.max(np.abs(r[~away])) > 0


@pytest.mark.parametrize("method", [1, 0, -1])
def test_vcfv_fd_local_linearizer_matches_ad(oracle_mod, ewg_mod, method):
    """lens_immiscible_vcfv_fd: FvBaseFdLocalLinearizer on the vertex-centred stencil gives the AD
    linearizer's residual and its Jacobian within the difference quotient's error (forward /
    backward first order, central second order)."""
    for case in (ewg_mod.vcfv_case(ewg_mod.baseline_case(12, 8)), ewg_mod.vcfv_case(ewg_mod.lens3d_case(6, 5, 4, seed=1))):
        o = oracle_mod.VcfvOracle(case)
        o.apply_initial_solution()
        x = o.get_solution(0)
        rng = np.random.Generator(np.random.PCG64(0))
        x[:, 1] = rng.uniform(0.3, 1.0, size=len(x))
        x[:, 0] += rng.normal(0, 50.0, size=len(x))
        o.set_solution(1, x)
        o.set_solution(0, x)
        o.linearize(250.0, 0)
        r_ad = o.residual()
        _, _, J_ad = o.jacobian_bcrs()
        o.set_local_linearizer(1, method)
        o.linearize(250.0, 0)
        assert np.array_equal(o.residual(), r_ad)
        _, _, J_fd = o.jacobian_bcrs()
        # central differences are limited by rounding: the element's local residual sums more
        # flux terms than a cell's (12 SCVFs), divided by 2 eps (eps = 9e-7 Pa for p_w)
        tol = 5e-5 if method else 2e-5
        for eq in range(2):
            for pv in range(2):
                a, b = J_fd[:, eq, pv], J_ad[:, eq, pv]
                assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(b)), (case.name, eq, pv)


def test_vcfv_pattern_matches_oracle(oracle_mod, ewg_mod):
    """The BCRS pattern callers pass to ewg_vcfv_get_jacobian_bcrs (ewg.vcfv_pattern) is the
    oracle's createMatrix_ pattern: each vertex row holds the vertices of its adjacent elements,
    columns ascending."""
    for case in (ewg_mod.vcfv_case(ewg_mod.baseline_case(5, 3)), ewg_mod.vcfv_case(ewg_mod.lens3d_case(3, 4, 2, seed=0))):
        o = oracle_mod.VcfvOracle(case)
        rp, ci, _ = o.jacobian_bcrs()
        rp2, ci2 = ewg_mod.vcfv_pattern(case.grid)
        assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2)
        assert all(np.all(np.diff(ci[rp[r]:rp[r + 1]]) > 0) for r in range(o.n))
