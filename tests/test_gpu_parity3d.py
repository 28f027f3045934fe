"""3D parity of the CUDA path against the CPU oracle on grids shaped like the 256 x 256 x 128
benchmark problem (y vertical, lens box of 40 % of each extent, seeded log-normal permeability,
inlet patch on the top face), small enough for the oracle.

* Linearization on 64 x 64 x 32 (131 072 cells, 913 408 blocks) at the hydrostatic initial state,
  a perturbed state and a mid-run state (after three implicit steps, old time level = the state one
  step earlier): residual and every Jacobian component within 1e-12 of the field's maximum
  magnitude (the bound the path is held to), and the entrywise relative error, each entry against
  its own size, recorded beside it and bounded too (ENTRY_RTOL).
* Ten implicit-Euler AD steps (dt 250 s, Newton tolerance 1e-8, BiCGStab + block ILU(0), linear
  tolerance 1e-10) on 32 x 32 x 16 and 64 x 64 x 32 against the oracle's natural-order run stored in
  tests/golden/lens3d_golden.npz: identical Newton iteration counts in every step, p_w within 1e-8
  relative and S_w within 1e-8 absolute after ten steps.
* The mixed-precision form (FP32 Jacobian, ILU(0) and inner BiCGStab in FP64 defect correction,
  FP64 residual and Newton update, same Newton tolerance) against the same fixtures to the same
  1e-8 field tolerance.

Set EWG_PARITY_REPORT=<file> to collect the measured errors as JSON lines.
"""
import os

import numpy as np
import pytest

from conftest import ROOT, parity_errors, record_parity, rel_close

pytestmark = pytest.mark.gpu

GOLD3 = os.path.join(ROOT, "tests", "golden", "lens3d_golden.npz")
LIN_RTOL = 1e-12
# entrywise relative error of Jacobian entries and residual entries that are at least 1e-6 of
# their field's maximum (smaller entries are cancellations of much larger terms). Measured on a
# B200: at most 3e-13 (a few ulps of the FP64 products that differ in fused multiply-adds)
ENTRY_RTOL = 1e-11
FIELD_TOL = 1e-8

# (tag, grid shape, permeability seed, correlation length in cells): as make_golden.CASES_3D
CASES_3D = {"g32x32x16": ((32, 32, 16), 7, 4.0), "g64x64x32": ((64, 64, 32), 8, 8.0)}


@pytest.fixture(scope="module")
def gold3():
    return np.load(GOLD3)


def _case(ewg, gold3, tag):
    shape, seed, corr = CASES_3D[tag]
    case = ewg.lens3d_case(*shape, seed=seed, corr_cells=corr)
    perm = gold3[f"{tag}_perm"]
    # the fixture's permeability is the one the oracle ran with; numpy's exp may round the field
    # differently on another CPU, so the device takes the stored bits
    assert np.allclose(case.perm, perm, rtol=1e-13, atol=0)
    case.perm = np.ascontiguousarray(perm)
    return case


def _perturbed(ewg, case, x, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = x.copy()
    xc, yc, zc = ewg.cell_centers(case.grid)
    g = case.grid
    plume = np.exp(-((xc - 0.5 * g.lx) ** 2) / 0.8 - ((yc - 0.8 * g.ly) ** 2) / 0.5 - ((zc - 0.5 * g.lz) ** 2) / 0.6)
    x[:, 1] = 1.0 - 0.7 * plume * rng.uniform(0.3, 1.0, size=len(xc))
    x[:, 1] = np.where(rng.uniform(size=len(xc)) < 0.05, rng.uniform(-0.02, 1.02, size=len(xc)), x[:, 1])
    x[:, 0] += rng.normal(0.0, 80.0, size=len(xc))
    return x


@pytest.mark.parametrize("state", ["initial", "perturbed", "mid_run"])
def test_linearization_64x64x32_matches_oracle(ewg_mod, oracle_mod, gold3, state):
    case = _case(ewg_mod, gold3, "g64x64x32")
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    x0 = ctx.get_solution(0)
    if state == "initial":
        x, xold = x0, x0
    elif state == "perturbed":
        x, xold = _perturbed(ewg_mod, case, x0, 41), _perturbed(ewg_mod, case, x0, 42)
    else:
        ctx.run(2, 250.0)
        xold = ctx.get_solution(0)
        ctx.run(1, 250.0)
        x = ctx.get_solution(0)
    ctx.set_solution(1, xold)
    ctx.set_solution(0, x)
    rep = ctx.linearize(250.0)
    o = oracle_mod.Oracle(case, nthreads=os.cpu_count() or 1)
    o.set_solution(1, xold)
    o.set_solution(0, x)
    o.set_recycle_first_iteration_storage(False)
    err = o.linearize(250.0, 0)
    r_g, r_o = ctx.residual(), o.residual()
    rp_g, ci_g, b_g = ctx.jacobian_bcrs()
    rp_o, ci_o, b_o = o.jacobian_bcrs()
    assert np.array_equal(rp_g, rp_o) and np.array_equal(ci_g, ci_o)
    # the residual is a sum of flux terms that cancel at hydrostatic equilibrium: it is judged
    # against the size of those terms (diagonal pressure derivative x one cell's hydrostatic step)
    flux_scale = np.max(np.abs(b_o[:, 0, 0])) * case.problem.rho_w * case.problem.gravity * case.grid.ly / case.grid.ny
    r_scale = max(np.max(np.abs(r_o)), flux_scale)
    report = {}
    for eq in range(2):
        ok, e, s = rel_close(r_g[:, eq], r_o[:, eq], LIN_RTOL, scale=r_scale)
        assert ok, ("residual", eq, e, s)
        # entrywise: each residual entry against its own size, for entries above 1e-6 of the scale
        d = np.abs(r_g[:, eq] - r_o[:, eq])
        m = np.abs(r_o[:, eq]) >= 1e-6 * r_scale
        ent = float(np.max(d[m] / np.abs(r_o[m, eq]))) if np.any(m) else 0.0
        report[f"r{eq}_field"], report[f"r{eq}_entry"] = e / r_scale, ent
        assert ent <= ENTRY_RTOL, ("residual entrywise", eq, ent)
        for pv in range(2):
            field, entry = parity_errors(b_g[:, eq, pv], b_o[:, eq, pv])
            report[f"J{eq}{pv}_field"], report[f"J{eq}{pv}_entry"] = field, entry
            assert field <= LIN_RTOL, ("jacobian", eq, pv, field)
            assert entry <= ENTRY_RTOL, ("jacobian entrywise", eq, pv, entry)
    assert rep.error == pytest.approx(err, rel=1e-12)
    record_parity(f"linearization_64x64x32_{state}", **report)
    ctx.close()
    o.close()


def _run_and_compare(ewg_mod, gold3, tag, sopts, name, check_counts):
    case = _case(ewg_mod, gold3, tag)
    ctx = ewg_mod.Context(case)
    ctx.apply_initial_solution()
    reps = ctx.run(10, 250.0, sopts=sopts)
    x_g = ctx.get_solution(0)
    x_o = gold3[f"{tag}_run10_x"]
    steps_o = gold3[f"{tag}_run10_steps"]
    its = [r.iterations for r in reps]
    assert all(r.converged and r.error <= 1e-8 for r in reps)
    dp = float(np.max(np.abs(x_g[:, 0] - x_o[:, 0])) / np.max(np.abs(x_o[:, 0])))
    ds = float(np.max(np.abs(x_g[:, 1] - x_o[:, 1])))
    record_parity(name, p_w_rel=dp, s_w_abs=ds, newton=its, newton_oracle=[int(a) for a in steps_o[:, 0]])
    if check_counts:
        assert its == list(steps_o[:, 0]), (its, list(steps_o[:, 0]))
    assert dp <= FIELD_TOL, ("p_w", dp)
    assert ds <= FIELD_TOL, ("S_w", ds)
    ctx.close()
    return its


@pytest.mark.parametrize("tag", ["g32x32x16", "g64x64x32"])
def test_ten_steps_3d_match_oracle(ewg_mod, gold3, tag):
    """Identical Newton iteration counts per step and fields within 1e-8 after ten steps."""
    _run_and_compare(ewg_mod, gold3, tag, ewg_mod.default_solve_opts(), f"run10_fp64_{tag}", True)


@pytest.mark.parametrize("tag", ["g32x32x16", "g64x64x32"])
def test_ten_steps_3d_mixed_precision_match_oracle(ewg_mod, gold3, tag):
    """The FP32-inner / FP64-outer form reaches the same Newton tolerance and the same fields
    (within 1e-8 of the FP64 oracle) after ten steps."""
    mixed = ewg_mod.default_solve_opts(precision=ewg_mod.PRECISION_MIXED)
    _run_and_compare(ewg_mod, gold3, tag, mixed, f"run10_mixed_{tag}", False)
