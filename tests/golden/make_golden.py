"""Generate the committed golden fixtures of the lens problem from the CPU oracle.

lens2d_golden.npz: the 2D lens problem (48 x 32), linearizations and 10-step runs of both presets,
material-law values. lens3d_golden.npz: 10 implicit-Euler steps (dt 250 s, Newton tolerance 1e-8,
BiCGStab + natural-order block ILU(0), linear tolerance 1e-10) of the 3D lens problem on
32 x 32 x 16 and 64 x 64 x 32 grids with seeded log-normal permeability; each entry stores the
permeability field it was run with, so the GPU test runs on the same bits wherever numpy's
transcendental functions round differently.

The reference itself cannot be built here (DUNE / ewoms-material are absent) and ships no golden
vectors, so these fixtures pin the oracle restatement against regressions and give the GPU tests
inputs and outputs that do not need the oracle at run time.
Run:  python tests/golden/make_golden.py [--2d] [--3d]   (both when no flag is given)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ewoms-numerics_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ewg  # noqa: E402
import oracle  # noqa: E402


def perturbed_state(case, seed=1):
    """Hydrostatic state with a DNAPL plume below the inlet and pressure noise: away from the
    exact upwind ties of the initial state, so every Jacobian entry is exercised."""
    o = oracle.Oracle(case)
    o.apply_initial_solution()
    x = o.get_solution(0)
    rng = np.random.Generator(np.random.PCG64(seed))
    xc, yc, _ = ewg.cell_centers(case.grid)
    plume = np.exp(-((xc - 3.0) ** 2) / 0.8 - ((yc - 3.2) ** 2) / 0.5)
    x[:, 1] = 1.0 - 0.6 * plume * rng.uniform(0.5, 1.0, size=len(xc))
    x[:, 0] += rng.normal(0.0, 50.0, size=len(xc))
    return x


def linearization(case, x, dt=250.0):
    o = oracle.Oracle(case)
    o.set_solution(0, x)
    o.set_solution(1, x)
    err = o.linearize(dt, 0)
    rp, ci, b = o.jacobian_bcrs()
    return dict(x=x, r=o.residual(), row_ptr=rp, col_idx=ci, blocks=b, error=np.array(err))


def run10(case, ordering):
    o = oracle.Oracle(case)
    o.apply_initial_solution()
    steps = o.run(10, 250.0, ordering=ordering)
    return o.get_solution(0), np.array(steps, dtype=np.int32)


# (tag, grid shape, permeability seed, correlation length in cells) of the 3D fixtures
CASES_3D = (("g32x32x16", (32, 32, 16), 7, 4.0), ("g64x64x32", (64, 64, 32), 8, 8.0))


def case_3d(shape, seed, corr_cells):
    return ewg.lens3d_case(*shape, seed=seed, corr_cells=corr_cells)


def main_3d():
    out = {}
    for tag, shape, seed, corr in CASES_3D:
        case = case_3d(shape, seed, corr)
        o = oracle.Oracle(case, nthreads=os.cpu_count() or 1)
        o.apply_initial_solution()
        steps = o.run(10, 250.0, ordering=oracle.ORDER_NATURAL)
        out[f"{tag}_perm"] = case.perm
        out[f"{tag}_run10_x"] = o.get_solution(0)
        out[f"{tag}_run10_steps"] = np.array(steps, dtype=np.int32)
        print(tag, steps)
    path = os.path.join(HERE, "lens3d_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


def main():
    out = {}
    for name, mk in (("baseline", ewg.baseline_case), ("reference", ewg.reference_case)):
        case = mk()
        o = oracle.Oracle(case)
        o.apply_initial_solution()
        x0 = o.get_solution(0)
        for tag, x in (("init", x0), ("pert", perturbed_state(case))):
            for k, v in linearization(case, x).items():
                out[f"{name}_{tag}_{k}"] = v
        xf, steps = run10(case, oracle.ORDER_NATURAL)
        out[f"{name}_run10_x"] = xf
        out[f"{name}_run10_steps"] = steps
    sws = np.array([-0.05, 0.0, 0.005, 0.04, 0.0999, 0.18, 0.2, 0.5, 0.9, 0.989, 0.99, 0.995, 1.0, 1.02])
    for mname, mat in (("vg_outer", ewg.baseline_case().problem.outer), ("vg_lens", ewg.baseline_case().problem.lens),
                       ("bc_outer", ewg.brooks_corey_case().problem.outer)):
        out[f"mat_{mname}"] = np.array([oracle.material_eval(mat, s) for s in sws])
    out["mat_sw"] = sws
    np.savez_compressed(os.path.join(HERE, "lens2d_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "lens2d_golden.npz"), len(out), "arrays")


if __name__ == "__main__":
    flags = set(sys.argv[1:])
    if not flags or "--2d" in flags:
        main()
    if not flags or "--3d" in flags:
        main_3d()
