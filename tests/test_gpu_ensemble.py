"""GPU tests of the batched ensemble (ewg_ensemble_*): every member of an ensemble of uneven 3D
lens problems gets the same results as the same problem run alone through ewg_ctx.

  * linearization: each member's residual equals the single-problem residual bit for bit (both
    evaluate the same per-cell code);
  * FP64 Newton steps: identical Newton iteration counts per step, p_w within 1e-8 relative and
    S_w within 1e-8 absolute of the single-problem run (BiCGStab's reductions are grouped per
    tile instead of per grid, so the linear iterates differ at rounding level);
  * the launch-shape autotuner changes no result bit;
  * mixed precision (FP32 inner solve) reaches the Newton tolerance 1e-8 with fields within 1e-6;
  * a member whose step fails is restored and retries with half the step size; the accepted
    step equals the single-problem Newton solve at that size.
"""
import numpy as np
import pytest

from conftest import rel_close

pytestmark = pytest.mark.gpu

SIZES = [(8, 6, 4), (12, 8, 6), (16, 10, 8)]
DTS = [100.0, 250.0, 500.0]


def _cases(ewg):
    return [ewg.lens3d_case(nx, ny, nz, seed=10 + k, sigma=0.5 + 0.5 * k, corr_cells=2.0 + k)
            for k, (nx, ny, nz) in enumerate(SIZES)]


def _perturbed(ewg, case, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    ctx = ewg.Context(case)
    ctx.apply_initial_solution()
    x = ctx.get_solution(0)
    ctx.close()
    x[:, 1] = np.clip(1.0 - 0.6 * rng.uniform(0, 1, len(x)) ** 3, -0.01, 1.01)
    x[:, 0] += rng.normal(0.0, 50.0, len(x))
    return x


def _fp64_opts(ewg, **kw):
    # the ensemble has no true-residual replacement pass; the reference does not either
    return ewg.default_solve_opts(verify_true_residual=0, **kw)


def test_ensemble_linearization_bitwise(ewg_mod):
    cases = _cases(ewg_mod)
    ens = ewg_mod.Ensemble(cases, precision=ewg_mod.PRECISION_FP64)
    xs, olds = [], []
    for m, c in enumerate(cases):
        x = _perturbed(ewg_mod, c, 100 + m)
        xo = _perturbed(ewg_mod, c, 200 + m)
        ens.set_solution(m, 1, xo)
        ens.set_solution(m, 0, x)
        xs.append(x)
        olds.append(xo)
    norms = ens.linearize(DTS)
    for m, c in enumerate(cases):
        ctx = ewg_mod.Context(c)
        ctx.set_solution(1, olds[m])
        ctx.set_solution(0, xs[m])
        rep = ctx.linearize(DTS[m])
        assert np.array_equal(ens.residual(m), ctx.residual()), m
        assert norms[m] == rep.error
        assert np.array_equal(ens.get_solution(m, 0), xs[m])
        ctx.close()
    ens.close()


def _run_single(ewg, case, dt, steps, sopts, nopts=None):
    ctx = ewg.Context(case)
    ctx.apply_initial_solution()
    reps = ctx.run(steps, dt, nopts=nopts, sopts=sopts)
    x = ctx.get_solution(0)
    ctx.close()
    return reps, x


@pytest.mark.parametrize("use_graph", [True, False])
def test_ensemble_fp64_steps_match_single_problems(ewg_mod, use_graph):
    cases = _cases(ewg_mod)
    so = _fp64_opts(ewg_mod)
    ens = ewg_mod.Ensemble(cases, precision=ewg_mod.PRECISION_FP64, use_graph=use_graph, check_interval=4)
    ens.apply_initial_solution()
    steps = 3
    ens_its = [[] for _ in cases]
    for _ in range(steps):
        st, reps, stats = ens.step(DTS, sopts=so)
        assert st == 0 and stats.rounds >= 1
        for m, r in enumerate(reps):
            assert r.status == 0 and r.halvings == 0 and r.error <= 1e-8
            ens_its[m].append(r.newton_iterations)
    # the same steps at each member's own pace
    ens2 = ewg_mod.Ensemble(cases, precision=ewg_mod.PRECISION_FP64, use_graph=use_graph, check_interval=4)
    ens2.apply_initial_solution()
    st, reps2, _ = ens2.advance(steps, DTS, sopts=so)
    assert st == 0
    for m, c in enumerate(cases):
        reps, x = _run_single(ewg_mod, c, DTS[m], steps, so)
        assert ens_its[m] == [r.iterations for r in reps], (m, ens_its[m], [r.iterations for r in reps])
        assert reps2[m].newton_iterations == sum(r.iterations for r in reps)
        for e in (ens, ens2):
            xe = e.get_solution(m, 0)
            assert np.array_equal(xe, e.get_solution(m, 1))
            assert rel_close(xe[:, 0], x[:, 0], 1e-8)[0]
            assert np.max(np.abs(xe[:, 1] - x[:, 1])) <= 1e-8
    ens.close()
    ens2.close()


def test_autotune_changes_no_bit(ewg_mod):
    cases = _cases(ewg_mod)
    so = _fp64_opts(ewg_mod)
    outs = []
    for tune in (False, True):
        ens = ewg_mod.Ensemble(cases, precision=ewg_mod.PRECISION_FP64)
        ens.apply_initial_solution()
        if tune:
            shapes = ens.autotune(DTS, so)
            assert all(v >= 1 for v in shapes.values())
            ens.apply_initial_solution()
        for _ in range(2):
            ens.step(DTS, sopts=so)
        outs.append([ens.get_solution(m, 0) for m in range(len(cases))])
        ens.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_ensemble_mixed_precision(ewg_mod):
    cases = _cases(ewg_mod)
    ens = ewg_mod.Ensemble(cases, precision=ewg_mod.PRECISION_MIXED)
    ens.apply_initial_solution()
    so = ewg_mod.default_solve_opts(precision=ewg_mod.PRECISION_MIXED, linear_solver_tolerance=1e-3,
                                    verify_true_residual=0)
    for _ in range(3):
        st, reps, _ = ens.step(DTS, sopts=so)
        assert st == 0 and all(r.status == 0 and r.error <= 1e-8 for r in reps)
    for m, c in enumerate(cases):
        _, x = _run_single(ewg_mod, c, DTS[m], 3, _fp64_opts(ewg_mod))
        xe = ens.get_solution(m, 0)
        assert rel_close(xe[:, 0], x[:, 0], 1e-8)[0]
        assert np.max(np.abs(xe[:, 1] - x[:, 1])) <= 1e-6
    ens.close()


def test_ensemble_step_halving(ewg_mod):
    """With Newton limited to 2 iterations the 4000 s step of member 0 fails and is halved until
    it is accepted. The accepted size is dt / 2^halvings, the failed attempts left no trace (the
    single-problem path started from the same state at the accepted size gives the same Newton
    iteration count and fields), and the other member is unaffected."""
    cases = _cases(ewg_mod)[:2]
    so = _fp64_opts(ewg_mod)
    no = ewg_mod.default_newton_opts(newton_max_iterations=2)
    dts = [4000.0, 250.0]
    ens = ewg_mod.Ensemble(cases, precision=ewg_mod.PRECISION_FP64)
    ens.apply_initial_solution()
    st, reps, _ = ens.step(dts, nopts=no, sopts=so)
    assert st == 0
    assert reps[0].halvings >= 1
    for m, c in enumerate(cases):
        r = reps[m]
        assert r.status == 0 and r.dt == dts[m] / 2 ** r.halvings
        ctx = ewg_mod.Context(c)
        ctx.apply_initial_solution()
        s, rep = ctx.newton_apply(r.dt, no, so)
        assert s == 0 and rep.iterations == r.newton_iterations
        x = ctx.get_solution(0)
        xe = ens.get_solution(m, 0)
        assert rel_close(xe[:, 0], x[:, 0], 1e-8)[0]
        assert np.max(np.abs(xe[:, 1] - x[:, 1])) <= 1e-8
        ctx.close()
    ens.close()


def _advance_pair(ewg, cases, dts, steps, precision, so, no=None, max_divisions=10, check_interval=4):
    out = []
    for device in (False, True):
        ens = ewg.Ensemble(cases, precision=precision, check_interval=check_interval, max_divisions=max_divisions)
        ens.apply_initial_solution()
        st, reps, stats = ens.advance(steps, dts, nopts=no, sopts=so, check=False, device=device)
        xs = [(ens.get_solution(m, 0), ens.get_solution(m, 1)) for m in range(len(cases))]
        ens.close()
        out.append((st, reps, stats, xs))
    return out


def _same_run(a, b):
    (sa, ra, ta, xa), (sb, rb, tb, xb) = a, b
    assert sa == sb
    for p, q in zip(ra, rb):
        assert (p.status, p.newton_iterations, p.linear_iterations, p.halvings) == \
               (q.status, q.newton_iterations, q.linear_iterations, q.halvings)
        assert p.dt == q.dt and p.error == q.error
    assert (ta.rounds, ta.linear_iterations, ta.cell_iterations, ta.supersteps) == \
           (tb.rounds, tb.linear_iterations, tb.cell_iterations, tb.supersteps)
    for (a0, a1), (b0, b1) in zip(xa, xb):
        assert np.array_equal(a0.view(np.uint64), b0.view(np.uint64))
        assert np.array_equal(a1.view(np.uint64), b1.view(np.uint64))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_scheduled_advance_is_bit_identical(ewg_mod, precision):
    """ewg_ensemble_advance_device (every decision on the device, supersteps inside one CUDA graph
    WHILE node) gives the host-scheduled advance's reports, stats and fields bit for bit."""
    cases = _cases(ewg_mod)
    if precision == "fp64":
        prec, so = ewg_mod.PRECISION_FP64, _fp64_opts(ewg_mod)
    else:
        prec = ewg_mod.PRECISION_MIXED
        so = ewg_mod.default_solve_opts(precision=prec, linear_solver_tolerance=1e-3, verify_true_residual=0)
    host, dev = _advance_pair(ewg_mod, cases, DTS, 3, prec, so)
    assert host[0] == 0 and all(r.status == 0 for r in host[1])
    assert host[2].supersteps > 3
    _same_run(host, dev)


def test_device_scheduled_halving_and_failure(ewg_mod):
    """Step halving and a member that fails after its allowed halvings take the same course on the
    device: with Newton limited to 2 iterations the 4000 s step of member 0 is halved until it is
    accepted (10 divisions allowed), or the advance fails with that member's status (1 allowed)."""
    cases = _cases(ewg_mod)[:2]
    so = _fp64_opts(ewg_mod)
    no = ewg_mod.default_newton_opts(newton_max_iterations=2)
    dts = [4000.0, 250.0]
    host, dev = _advance_pair(ewg_mod, cases, dts, 2, ewg_mod.PRECISION_FP64, so, no=no)
    assert host[0] == 0 and host[1][0].halvings >= 1
    _same_run(host, dev)
    host, dev = _advance_pair(ewg_mod, cases, dts, 2, ewg_mod.PRECISION_FP64, so, no=no, max_divisions=1)
    assert host[0] == ewg_mod.EWG_ERR_NOT_CONVERGED and host[1][0].status != 0 and host[1][1].status == 0
    _same_run(host, dev)


SIZES8 = [(8, 8, 4), (12, 8, 8), (16, 12, 8)]  # every extent a multiple of 4: box-8-colour ILU(0)


def _cases8(ewg):
    return [ewg.lens3d_case(nx, ny, nz, seed=20 + k, sigma=0.5 + 0.5 * k, corr_cells=2.0 + k)
            for k, (nx, ny, nz) in enumerate(SIZES8)]


@pytest.mark.parametrize("device", [False, True])
def test_box8_ensemble_matches_single_problems(ewg_mod, device):
    """With every member's grid in box-8 order the ensemble solves with the box-8-colour ILU(0)
    (ilu_ordering AUTO), as the single problem does on those grids: three FP64 steps give the same
    Newton iteration counts per member as the single-problem runs, BiCGStab counts within 15 %, and
    fields within 1e-8; the red-black order stays selectable and needs more BiCGStab iterations."""
    cases = _cases8(ewg_mod)
    so = _fp64_opts(ewg_mod)
    ens = ewg_mod.Ensemble(cases, precision=ewg_mod.PRECISION_FP64, check_interval=4)
    ens.apply_initial_solution()
    st, reps, _ = ens.advance(3, DTS, sopts=so, device=device)
    assert st == 0
    rb = ewg_mod.Ensemble(cases, precision=ewg_mod.PRECISION_FP64, check_interval=4)
    rb.apply_initial_solution()
    st2, reps_rb, _ = rb.advance(3, DTS, sopts=_fp64_opts(ewg_mod, ilu_ordering=ewg_mod.ILU_ORDER_REDBLACK),
                                 device=device)
    assert st2 == 0
    for m, c in enumerate(cases):
        sreps, x = _run_single(ewg_mod, c, DTS[m], 3, so)
        assert reps[m].newton_iterations == sum(r.iterations for r in sreps), m
        lin = sum(r.linear_iterations for r in sreps)
        assert abs(reps[m].linear_iterations - lin) <= max(3, 0.15 * lin), (reps[m].linear_iterations, lin)
        xe = ens.get_solution(m, 0)
        assert rel_close(xe[:, 0], x[:, 0], 1e-8)[0]
        assert np.max(np.abs(xe[:, 1] - x[:, 1])) <= 1e-8
        assert reps[m].linear_iterations < reps_rb[m].linear_iterations, (m, reps[m].linear_iterations,
                                                                          reps_rb[m].linear_iterations)
    ens.close()
    rb.close()


def test_box8_ensemble_mixed_and_rejection(ewg_mod):
    """The mixed-precision box-8 ensemble reaches the Newton tolerance with S_w within 1e-6 of the
    FP64 single problem, the host and device schedulers give the same bits, and requesting the box-8
    order on an ensemble with a member that lacks it is rejected."""
    cases = _cases8(ewg_mod)
    so = ewg_mod.default_solve_opts(precision=ewg_mod.PRECISION_MIXED, linear_solver_tolerance=1e-3,
                                    verify_true_residual=0)
    host, dev = _advance_pair(ewg_mod, cases, DTS, 3, ewg_mod.PRECISION_MIXED, so)
    assert host[0] == 0 and all(r.status == 0 and r.error <= 1e-8 for r in host[1])
    _same_run(host, dev)
    for m, c in enumerate(cases):
        _, x = _run_single(ewg_mod, c, DTS[m], 3, _fp64_opts(ewg_mod))
        xe = host[3][m][0]
        assert rel_close(xe[:, 0], x[:, 0], 1e-8)[0]
        assert np.max(np.abs(xe[:, 1] - x[:, 1])) <= 1e-6
    mixed_cases = _cases8(ewg_mod)[:2] + [_cases(ewg_mod)[1]]  # 12x8x6 lacks the order
    ens = ewg_mod.Ensemble(mixed_cases, precision=ewg_mod.PRECISION_FP64)
    ens.apply_initial_solution()
    st, _, _ = ens.advance(1, DTS, sopts=_fp64_opts(ewg_mod, ilu_ordering=ewg_mod.ILU_ORDER_BOX8), check=False)
    assert st == ewg_mod.EWG_ERR_INVALID
    st, reps, _ = ens.advance(1, DTS, sopts=_fp64_opts(ewg_mod))  # AUTO: red-black for all
    assert st == 0 and all(r.status == 0 for r in reps)
    ens.close()
