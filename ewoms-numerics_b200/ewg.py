"""ctypes plumbing for the C ABI in include/ewg.h (libewg.so) and the lens-problem presets.

The product is the CUDA library; this module only declares the ABI structs, loads the in-tree
``libewg.so`` and builds problem definitions (grid, material regions, permeability fields) on the
host. There is no CPU fallback: ``load()`` raises if the library is missing and ``Context``
raises if no sm_100 device is usable.

Problem presets follow ``tests/problems/lensproblem.hh``:
  * ``reference``  -- the reference's own parameters (lensproblem.hh:248-288, 464-533)
  * ``baseline``   -- the graded 2D parameter set (48x32, K 9.05e-12 / 9.05e-13, VG alpha
                      3.7e-4 / 4.5e-4, inlet x in (2.25, 3.75), hydrostatic left and right)
  * ``lens3d``     -- the 3D extrusion (256x256x128 at full size, any even nx) with a seeded
                      log-normal permeability field
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libewg.so")

EWG_OK = 0
(EWG_ERR_INVALID, EWG_ERR_CUDA, EWG_ERR_NONFINITE, EWG_ERR_BREAKDOWN, EWG_ERR_NOT_CONVERGED, EWG_ERR_TIMEOUT,
 EWG_ERR_NO_DEVICE, EWG_ERR_MAX_ERROR) = range(1, 9)
STATUS_NAMES = {0: "EWG_OK", 1: "EWG_ERR_INVALID", 2: "EWG_ERR_CUDA", 3: "EWG_ERR_NONFINITE",
                4: "EWG_ERR_BREAKDOWN", 5: "EWG_ERR_NOT_CONVERGED", 6: "EWG_ERR_TIMEOUT",
                7: "EWG_ERR_NO_DEVICE", 8: "EWG_ERR_MAX_ERROR"}

LAW_VG, LAW_BC = 0, 1
PRECOND_ILU0, PRECOND_JACOBI = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
# ewg_ilu_ordering: row order of the block ILU(0) (BOX8 needs a 3D grid with dimensions divisible by 4)
ILU_ORDER_AUTO, ILU_ORDER_REDBLACK, ILU_ORDER_BOX8 = 0, 1, 2
LOCAL_LINEARIZER_AD, LOCAL_LINEARIZER_FD = 0, 1


class Grid(C.Structure):
    _fields_ = [("dim", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double), ("k_origin", C.c_int32)]

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * (self.nz if self.dim == 3 else 1)

    @property
    def shape(self):
        """numpy shape of a natural-order cell field (x fastest): (nz, ny, nx)."""
        return (self.nz if self.dim == 3 else 1, self.ny, self.nx)


class Material(C.Structure):
    _fields_ = [("law", C.c_int32), ("swr", C.c_double), ("snr", C.c_double),
                ("vg_alpha", C.c_double), ("vg_n", C.c_double),
                ("bc_entry_pressure", C.c_double), ("bc_lambda", C.c_double)]


class Problem(C.Structure):
    _fields_ = [("lens_lo", C.c_double * 3), ("lens_hi", C.c_double * 3), ("eps", C.c_double),
                ("porosity", C.c_double), ("temperature", C.c_double),
                ("rho_w", C.c_double), ("mu_w", C.c_double), ("rho_n", C.c_double),
                ("mu_n", C.c_double), ("gravity", C.c_double), ("p_ref", C.c_double),
                ("left_pressure_scale", C.c_double),
                ("inlet_x_lo", C.c_double), ("inlet_x_hi", C.c_double),
                ("inlet_z_lo", C.c_double), ("inlet_z_hi", C.c_double),
                ("inlet_rate", C.c_double), ("outer", Material), ("lens", Material)]


class SolveOpts(C.Structure):
    _fields_ = [("precond", C.c_int32), ("precision", C.c_int32),
                ("linear_solver_tolerance", C.c_double),
                ("linear_solver_abs_tolerance", C.c_double),
                ("linear_solver_max_error", C.c_double),
                ("linear_solver_max_iterations", C.c_int32),
                ("preconditioner_relaxation", C.c_double),
                ("defect_tolerance", C.c_double), ("inner_tolerance", C.c_double),
                ("max_defect_iterations", C.c_int32), ("check_interval", C.c_int32),
                ("restart_on_breakdown", C.c_int32), ("verify_true_residual", C.c_int32),
                ("ilu_ordering", C.c_int32)]


class SolveReport(C.Structure):
    _fields_ = [("converged", C.c_int32), ("restarts", C.c_int32), ("iterations", C.c_int32),
                ("outer_iterations", C.c_int32), ("status", C.c_int32),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("seconds", C.c_double)]


class LinReport(C.Structure):
    _fields_ = [("error", C.c_double), ("nonfinite", C.c_int32), ("seconds", C.c_double)]


class NewtonOpts(C.Structure):
    _fields_ = [("newton_tolerance", C.c_double), ("newton_max_error", C.c_double),
                ("newton_max_iterations", C.c_int32), ("newton_target_iterations", C.c_int32),
                ("verbose", C.c_int32)]


class NewtonReport(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32),
                ("linear_iterations", C.c_int32), ("status", C.c_int32), ("error", C.c_double),
                ("t_linearize", C.c_double), ("t_solve", C.c_double), ("t_update", C.c_double)]


class EnsembleOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("use_graph", C.c_int32), ("check_interval", C.c_int32),
                ("max_divisions", C.c_int32)]


class EnsembleReport(C.Structure):
    _fields_ = [("status", C.c_int32), ("newton_iterations", C.c_int32),
                ("linear_iterations", C.c_int32), ("halvings", C.c_int32), ("dt", C.c_double),
                ("error", C.c_double)]


class EnsembleStats(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("linear_iterations", C.c_int32), ("t_linearize", C.c_double),
                ("t_solve", C.c_double), ("t_update", C.c_double), ("cell_iterations", C.c_double),
                ("supersteps", C.c_int32)]


ENSEMBLE_KERNEL_CLASSES = ("intensive", "assemble", "factor", "cell", "ilu_black", "ilu_red",
                           "spmv_alpha", "spmv_omega", "bicg_p", "bicg_hs", "bicg_xr")


def default_solve_opts(**kw) -> SolveOpts:
    """Reference defaults (fvbasediscretization.hh:249-252, parallelbicgstabbackend.hh:48,
    parallelbasebackend.hh:514) with the graded linear tolerance 1e-10 unless overridden."""
    o = SolveOpts(precond=PRECOND_ILU0, precision=PRECISION_FP64,
                  linear_solver_tolerance=1e-10, linear_solver_abs_tolerance=1e-10,
                  linear_solver_max_error=1e7, linear_solver_max_iterations=1000,
                  preconditioner_relaxation=1.0, defect_tolerance=0.0, inner_tolerance=1e-4,
                  max_defect_iterations=50, check_interval=0, restart_on_breakdown=1,
                  verify_true_residual=1, ilu_ordering=ILU_ORDER_AUTO)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def default_newton_opts(**kw) -> NewtonOpts:
    """NewtonTolerance 1e-8, NewtonMaxError 1e100, max 18, target 10 (newtonmethod.hh:150-155)."""
    o = NewtonOpts(newton_tolerance=1e-8, newton_max_error=1e100, newton_max_iterations=18,
                   newton_target_iterations=10, verbose=0)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


# ------------------------------------------------------------------------------------------
# problem presets


def _vg(swr, snr, alpha, n) -> Material:
    return Material(law=LAW_VG, swr=swr, snr=snr, vg_alpha=alpha, vg_n=n,
                    bc_entry_pressure=0.0, bc_lambda=0.0)


def _bc(swr, snr, pe, lam) -> Material:
    return Material(law=LAW_BC, swr=swr, snr=snr, vg_alpha=0.0, vg_n=0.0,
                    bc_entry_pressure=pe, bc_lambda=lam)


@dataclass
class LensCase:
    """A complete lens-problem definition: grid, problem constants and permeability field."""
    name: str
    grid: Grid
    problem: Problem
    perm: np.ndarray          # natural order, float64, N
    dt: float = 250.0
    n_steps: int = 10

    @property
    def n_cells(self) -> int:
        return self.grid.n_cells


def cell_centers(grid: Grid):
    """Cell centres (x, y, z) as natural-order flat arrays: (i + 0.5) * h per axis."""
    nz = grid.nz if grid.dim == 3 else 1
    hx, hy = grid.lx / grid.nx, grid.ly / grid.ny
    hz = grid.lz / nz if grid.dim == 3 else 0.0
    k, j, i = np.meshgrid(np.arange(nz), np.arange(grid.ny), np.arange(grid.nx), indexing="ij")
    x = (i + 0.5) * hx
    y = (j + 0.5) * hy
    z = (k + 0.5) * hz if grid.dim == 3 else np.zeros_like(x, dtype=float)
    return x.ravel(), y.ravel(), z.ravel()


def in_lens(grid: Grid, problem: Problem) -> np.ndarray:
    """isInLens_ (lensproblem.hh:596-604) at the cell centres."""
    x, y, z = cell_centers(grid)
    pos = [x, y, z]
    m = np.ones(grid.n_cells, dtype=bool)
    for a in range(grid.dim):
        m &= (pos[a] >= problem.lens_lo[a] - problem.eps) & (pos[a] <= problem.lens_hi[a] + problem.eps)
    return m


def _base_problem() -> Problem:
    p = Problem()
    p.eps = 3e-6
    p.porosity = 0.4
    p.temperature = 293.15
    p.rho_w, p.mu_w = 1000.0, 1e-3      # SimpleH2O as a liquid
    p.rho_n, p.mu_n = 1460.0, 5.7e-4    # DNAPL (TCE)
    p.gravity = 9.81
    p.p_ref = 1e5
    p.inlet_rate = -0.04
    p.inlet_z_lo, p.inlet_z_hi = -1e30, 1e30
    return p


def reference_case(nx=48, ny=32) -> LensCase:
    """The reference's lensproblem.hh parameters in 2D (6 m x 4 m)."""
    g = Grid(dim=2, nx=nx, ny=ny, nz=1, lx=6.0, ly=4.0, lz=1.0)
    p = _base_problem()
    p.lens_lo[:] = [1.0, 2.0, 0.0]
    p.lens_hi[:] = [4.0, 3.0, 1.0]
    p.outer = _vg(0.05, 0.0, 0.0037, 4.7)
    p.lens = _vg(0.18, 0.0, 0.00045, 7.3)
    p.left_pressure_scale = 1.0 + 1.5 / 4.0
    p.inlet_x_lo, p.inlet_x_hi = 2.0, 3.0     # 0.5 < (xmax - x)/width < 2/3
    lens = in_lens(g, p)
    perm = np.where(lens, 9.05e-12, 4.6e-10).astype(np.float64)
    return LensCase("reference", g, p, perm)


def baseline_case(nx=48, ny=32) -> LensCase:
    """The graded 2D lens preset (Dirichlet-like hydrostatic free flow on left and right)."""
    g = Grid(dim=2, nx=nx, ny=ny, nz=1, lx=6.0, ly=4.0, lz=1.0)
    p = _base_problem()
    p.lens_lo[:] = [1.0, 2.0, 0.0]
    p.lens_hi[:] = [4.0, 3.0, 1.0]
    p.outer = _vg(0.05, 0.0, 3.7e-4, 4.7)
    p.lens = _vg(0.18, 0.0, 4.5e-4, 7.3)
    p.left_pressure_scale = 1.0
    p.inlet_x_lo, p.inlet_x_hi = 2.25, 3.75
    lens = in_lens(g, p)
    perm = np.where(lens, 9.05e-13, 9.05e-12).astype(np.float64)
    return LensCase("baseline", g, p, perm)


def brooks_corey_case(nx=48, ny=32) -> LensCase:
    """The baseline geometry with EffToAbsLaw<RegularizedBrooksCorey> (entry pressure 500 Pa,
    lambda 2 as in tutorial/tutorial1problem.hh:182-183; lens entry pressure 1500 Pa)."""
    c = baseline_case(nx, ny)
    c.problem.outer = _bc(0.05, 0.0, 500.0, 2.0)
    c.problem.lens = _bc(0.18, 0.0, 1500.0, 2.0)
    c.name = "brooks_corey"
    return c


def gaussian_log_field(shape, sigma=1.0, corr_cells=8.0, seed=0) -> np.ndarray:
    """Seeded stationary Gaussian field with exponential covariance exp(-r / corr_cells), zero
    mean and standard deviation sigma, by spectral synthesis on the periodic grid: white noise
    filtered with the square root of the covariance's discrete spectrum, then rescaled so the
    sample standard deviation is exactly sigma."""
    rng = np.random.Generator(np.random.PCG64(seed))
    axes = [np.fft.fftfreq(s) * s for s in shape]  # integer lags on the torus
    grids = np.meshgrid(*[np.minimum(np.abs(a), s - np.abs(a)) for a, s in zip(axes, shape)],
                        indexing="ij")
    r = np.sqrt(sum(g.astype(np.float64) ** 2 for g in grids))
    cov = np.exp(-r / corr_cells)
    axes = tuple(range(len(shape)))
    spec = np.fft.rfftn(cov, axes=axes).real
    spec = np.maximum(spec, 0.0)
    noise = rng.standard_normal(shape)
    f = np.fft.irfftn(np.fft.rfftn(noise, axes=axes) * np.sqrt(spec), s=shape, axes=axes)
    f -= f.mean()
    sd = f.std()
    if sd > 0:  # a one-cell field has no variation to scale
        f *= sigma / sd
    return f


def lens3d_case(nx=256, ny=256, nz=128, seed=0, sigma=1.0, corr_cells=8.0,
                extents=(6.0, 4.0, 3.0)) -> LensCase:
    """3D extrusion of the graded lens problem: centred lens box of 40 % of each extent, ln K a
    seeded Gaussian field (mean ln 9.05e-12, exponential covariance), K x 0.1 in the lens,
    DNAPL inlet on the top face over x in (2.25, 3.75) m and the middle 40 % in z."""
    lx, ly, lz = extents
    g = Grid(dim=3, nx=nx, ny=ny, nz=nz, lx=lx, ly=ly, lz=lz)
    p = _base_problem()
    p.lens_lo[:] = [0.3 * lx, 0.3 * ly, 0.3 * lz]
    p.lens_hi[:] = [0.7 * lx, 0.7 * ly, 0.7 * lz]
    p.outer = _vg(0.05, 0.0, 3.7e-4, 4.7)
    p.lens = _vg(0.18, 0.0, 4.5e-4, 7.3)
    p.left_pressure_scale = 1.0
    p.inlet_x_lo, p.inlet_x_hi = 2.25 * lx / 6.0, 3.75 * lx / 6.0
    p.inlet_z_lo, p.inlet_z_hi = 0.3 * lz, 0.7 * lz
    f = gaussian_log_field((nz, ny, nx), sigma=sigma, corr_cells=corr_cells, seed=seed).ravel()
    lnk = np.log(9.05e-12) + f
    lens = in_lens(g, p)
    lnk = np.where(lens, lnk + np.log(0.1), lnk)
    return LensCase("lens3d", g, p, np.exp(lnk).astype(np.float64))


# ------------------------------------------------------------------------------------------
# vertex-centred (VCFV) cases: the same problems with one DOF and one permeability per grid vertex


def vertex_positions(grid: Grid):
    """Vertex coordinates (x, y, z) as flat arrays, x fastest: index * h per axis."""
    nz = grid.nz if grid.dim == 3 else 0
    hx, hy = grid.lx / grid.nx, grid.ly / grid.ny
    hz = grid.lz / grid.nz if grid.dim == 3 else 0.0
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(grid.ny + 1), np.arange(grid.nx + 1), indexing="ij")
    return (i * hx).ravel(), (j * hy).ravel(), (k * hz).ravel()


def n_vertices(grid: Grid) -> int:
    return (grid.nx + 1) * (grid.ny + 1) * ((grid.nz + 1) if grid.dim == 3 else 1)


def in_lens_vertices(grid: Grid, problem: Problem) -> np.ndarray:
    """isInLens_ (lensproblem.hh:596-604) at the vertex positions."""
    pos = vertex_positions(grid)
    m = np.ones(n_vertices(grid), dtype=bool)
    for a in range(grid.dim):
        m &= (pos[a] >= problem.lens_lo[a] - problem.eps) & (pos[a] <= problem.lens_hi[a] + problem.eps)
    return m


def vcfv_case(case: LensCase, seed: int | None = None, sigma: float = 1.0, corr_cells: float = 8.0) -> LensCase:
    """The vertex-centred version of a lens case: permeability per vertex. The 2D presets take
    their lens / outer values by vertex position; lens3d draws its log-normal field on the vertex
    grid (seed defaults to 0)."""
    g, p = case.grid, case.problem
    lens = in_lens_vertices(g, p)
    if case.name == "lens3d":
        shape = (g.nz + 1, g.ny + 1, g.nx + 1)
        f = gaussian_log_field(shape, sigma=sigma, corr_cells=corr_cells, seed=0 if seed is None else seed).ravel()
        lnk = np.log(9.05e-12) + f
        perm = np.exp(np.where(lens, lnk + np.log(0.1), lnk))
    else:
        # (K in the lens, K outside) of the 2D presets
        k_lens, k_out = {"reference": (9.05e-12, 4.6e-10), "baseline": (9.05e-13, 9.05e-12),
                         "brooks_corey": (9.05e-13, 9.05e-12)}[case.name]
        perm = np.where(lens, k_lens, k_out)
    return LensCase("vcfv_" + case.name, g, p, np.ascontiguousarray(perm, dtype=np.float64), case.dt, case.n_steps)


# ------------------------------------------------------------------------------------------
# library loading

_lib = None


def _ptr(a: np.ndarray, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


def load(path: str = LIB_PATH):
    """Load the in-tree libewg.so and declare its signatures. Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libewg.so not built at {path}: run __graft_entry__.build()")
    lib = C.CDLL(path)
    P = C.POINTER
    d = C.c_double
    sig = {
        "ewg_create": (C.c_int, [P(Grid), P(Problem), P(d), P(C.c_void_p)]),
        "ewg_destroy": (None, [C.c_void_p]),
        "ewg_last_error": (C.c_char_p, [C.c_void_p]),
        "ewg_create_error": (C.c_char_p, []),
        "ewg_num_cells": (C.c_int64, [C.c_void_p]),
        "ewg_num_blocks": (C.c_int64, [C.c_void_p]),
        "ewg_abi_version": (C.c_int32, []),
        "ewg_set_solution": (C.c_int, [C.c_void_p, C.c_int32, P(d)]),
        "ewg_get_solution": (C.c_int, [C.c_void_p, C.c_int32, P(d)]),
        "ewg_apply_initial_solution": (C.c_int, [C.c_void_p]),
        "ewg_advance_time_level": (C.c_int, [C.c_void_p]),
        "ewg_restore_time_level": (C.c_int, [C.c_void_p]),
        "ewg_linearize": (C.c_int, [C.c_void_p, d, P(LinReport)]),
        "ewg_set_local_linearizer": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
        "ewg_update_begin": (C.c_int, [C.c_void_p]),
        "ewg_set_reference_pressure": (C.c_int, [C.c_void_p, C.c_double]),
        "ewg_get_intensive_quantities": (C.c_int, [C.c_void_p, P(d)]),
        "ewg_get_residual": (C.c_int, [C.c_void_p, P(d)]),
        "ewg_get_jacobian_bcrs": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int32), P(d)]),
        "ewg_residual_norm": (C.c_int, [C.c_void_p, P(d), d, P(d)]),
        "ewg_set_matrix_bcrs": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int32), P(d)]),
        "ewg_set_residual": (C.c_int, [C.c_void_p, P(d)]),
        "ewg_solve": (C.c_int, [C.c_void_p, P(SolveOpts), P(SolveReport)]),
        "ewg_get_update": (C.c_int, [C.c_void_p, P(d)]),
        "ewg_apply_preconditioner": (C.c_int, [C.c_void_p, P(SolveOpts), P(d), P(d)]),
        "ewg_apply_jacobian": (C.c_int, [C.c_void_p, P(d), P(d)]),
        "ewg_newton_update": (C.c_int, [C.c_void_p]),
        "ewg_newton_apply": (C.c_int, [C.c_void_p, d, P(NewtonOpts), P(SolveOpts), P(NewtonReport)]),
        "ewg_default_solve_opts": (None, [P(SolveOpts)]),
        "ewg_default_newton_opts": (None, [P(NewtonOpts)]),
        "ewg_get_stream": (C.c_void_p, [C.c_void_p]),
        "ewg_device_buffer": (C.c_int, [C.c_void_p, C.c_int32, P(C.c_void_p)]),
        "ewg_device_spmv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "ewg_device_precondition": (C.c_int, [C.c_void_p, P(SolveOpts), C.c_void_p, C.c_void_p]),
        "ewg_device_bicg_p": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ewg_device_bicg_spmv_dot": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                               C.c_int64, C.c_void_p, C.c_void_p]),
        "ewg_device_bicg_hs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                         C.c_int64, C.c_void_p, C.c_void_p]),
        "ewg_device_bicg_spmv_dot2": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                                C.c_int64, C.c_void_p, C.c_void_p]),
        "ewg_device_bicg_xr": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]),
        "ewg_device_bicg_state_size": (C.c_int32, []),
        "ewg_device_bicg_state": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, P(SolveOpts)]),
        "ewg_device_bicg_state_read": (C.c_int, [C.c_void_p, C.c_void_p, P(C.c_int32), P(C.c_int32),
                                                 P(C.c_int32), P(C.c_double), P(C.c_double)]),
        "ewg_transfer_counters": (C.c_int, [C.c_void_p, C.c_int32, P(C.c_uint64), P(C.c_uint64)]),
        "ewg_profile_num_kernels": (C.c_int32, []),
        "ewg_profile_kernel_name": (C.c_char_p, [C.c_int32]),
        "ewg_profile_enable": (C.c_int, [C.c_void_p, C.c_int32]),
        "ewg_profile_reset": (C.c_int, [C.c_void_p]),
        "ewg_profile_get": (C.c_int, [C.c_void_p, C.c_int32, P(d), P(C.c_int64)]),
        "ewg_vcfv_create": (C.c_int, [P(Grid), P(Problem), P(d), P(C.c_void_p)]),
        "ewg_vcfv_destroy": (None, [C.c_void_p]),
        "ewg_vcfv_last_error": (C.c_char_p, [C.c_void_p]),
        "ewg_vcfv_num_dofs": (C.c_int64, [C.c_void_p]),
        "ewg_vcfv_launches": (C.c_int64, [C.c_void_p]),
        "ewg_vcfv_set_solution": (C.c_int, [C.c_void_p, C.c_int32, P(d)]),
        "ewg_vcfv_get_solution": (C.c_int, [C.c_void_p, C.c_int32, P(d)]),
        "ewg_vcfv_apply_initial_solution": (C.c_int, [C.c_void_p]),
        "ewg_vcfv_advance_time_level": (C.c_int, [C.c_void_p]),
        "ewg_vcfv_restore_time_level": (C.c_int, [C.c_void_p]),
        "ewg_vcfv_set_local_linearizer": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
        "ewg_vcfv_update_begin": (C.c_int, [C.c_void_p]),
        "ewg_vcfv_linearize": (C.c_int, [C.c_void_p, d, P(d)]),
        "ewg_vcfv_get_residual": (C.c_int, [C.c_void_p, P(d)]),
        "ewg_vcfv_get_jacobian_bcrs": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int32), C.c_int64, P(d)]),
        "ewg_vcfv_solve": (C.c_int, [C.c_void_p, P(SolveOpts), P(d), P(C.c_int32)]),
        "ewg_vcfv_newton_apply": (C.c_int, [C.c_void_p, d, P(NewtonOpts), P(SolveOpts), P(C.c_int32),
                                            P(C.c_int32), P(d)]),
        "ewg_net_num_params": (C.c_int64, []),
        "ewg_net_create": (C.c_int, [C.c_uint64, P(C.c_void_p)]),
        "ewg_net_destroy": (None, [C.c_void_p]),
        "ewg_net_last_error": (C.c_char_p, [C.c_void_p]),
        "ewg_net_get_params": (C.c_int, [C.c_void_p, P(C.c_float), C.c_int64]),
        "ewg_net_set_params": (C.c_int, [C.c_void_p, P(C.c_float), C.c_int64]),
        "ewg_net_set_scales": (C.c_int, [C.c_void_p, P(d)]),
        "ewg_net_get_scales": (C.c_int, [C.c_void_p, P(d)]),
        "ewg_net_set_options": (C.c_int, [C.c_void_p, C.c_float, C.c_float, C.c_int32, d]),
        "ewg_net_eval_host": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                        P(C.c_float), P(C.c_float), P(C.c_float), P(C.c_float), P(C.c_float)]),
        "ewg_net_record_sample": (C.c_int, [C.c_void_p, C.c_void_p, d]),
        "ewg_net_num_samples": (C.c_int64, [C.c_void_p]),
        "ewg_net_train": (C.c_int, [C.c_void_p, P(C.c_int64), C.c_int32, C.c_float, P(C.c_float)]),
        "ewg_net_eval_samples": (C.c_int, [C.c_void_p, P(C.c_int64), C.c_int32, P(C.c_float)]),
        "ewg_predict_guess": (C.c_int, [C.c_void_p, C.c_void_p, d, P(C.c_int32), P(d), P(d)]),
        "ewg_default_ensemble_opts": (None, [P(EnsembleOpts)]),
        "ewg_ensemble_create": (C.c_int, [C.c_int32, P(Grid), P(Problem), P(P(d)), P(EnsembleOpts),
                                          P(C.c_void_p)]),
        "ewg_ensemble_destroy": (None, [C.c_void_p]),
        "ewg_ensemble_last_error": (C.c_char_p, [C.c_void_p]),
        "ewg_ensemble_create_error": (C.c_char_p, []),
        "ewg_ensemble_num_members": (C.c_int32, [C.c_void_p]),
        "ewg_ensemble_num_cells": (C.c_int64, [C.c_void_p, C.c_int32]),
        "ewg_ensemble_get_stream": (C.c_void_p, [C.c_void_p]),
        "ewg_ensemble_apply_initial_solution": (C.c_int, [C.c_void_p]),
        "ewg_ensemble_set_solution": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, P(d)]),
        "ewg_ensemble_get_solution": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, P(d)]),
        "ewg_ensemble_linearize": (C.c_int, [C.c_void_p, P(d), P(d)]),
        "ewg_ensemble_get_residual": (C.c_int, [C.c_void_p, C.c_int32, P(d)]),
        "ewg_ensemble_autotune": (C.c_int, [C.c_void_p, P(d), P(SolveOpts)]),
        "ewg_ensemble_get_launch_shapes": (C.c_int, [C.c_void_p, P(C.c_int32), C.c_int32, P(C.c_int32)]),
        "ewg_ensemble_step": (C.c_int, [C.c_void_p, P(d), P(NewtonOpts), P(SolveOpts), P(EnsembleReport),
                                        P(EnsembleStats)]),
        "ewg_ensemble_advance": (C.c_int, [C.c_void_p, C.c_int32, P(d), P(NewtonOpts), P(SolveOpts),
                                           P(EnsembleReport), P(EnsembleStats)]),
        "ewg_ensemble_advance_device": (C.c_int, [C.c_void_p, C.c_int32, P(d), P(NewtonOpts), P(SolveOpts),
                                                  P(EnsembleReport), P(EnsembleStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class EwgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


BUFFER_SOLUTION, BUFFER_RESIDUAL = 0, 1


class _DeviceVector:
    """__cuda_array_interface__ of an N x 2 float64 device vector owned by a context."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n, 2), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


class Context:
    """One device problem (ewg_ctx). Host arrays are natural order, N x 2 float64."""

    def __init__(self, case: LensCase):
        lib = load()
        self.lib = lib
        self.case = case
        self.n = case.grid.n_cells
        h = C.c_void_p()
        perm = np.ascontiguousarray(case.perm, dtype=np.float64)
        st = lib.ewg_create(C.byref(case.grid), C.byref(case.problem), _ptr(perm), C.byref(h))
        if st != EWG_OK:
            raise EwgError(st, lib.ewg_create_error().decode())
        self.h = h
        self.nnzb = lib.ewg_num_blocks(h)

    def _check(self, st, what=""):
        if st != EWG_OK:
            raise EwgError(st, f"{what}: {self.lib.ewg_last_error(self.h).decode()}")
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.ewg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def vec(self):
        return np.zeros((self.n, 2), dtype=np.float64)

    def set_solution(self, time_idx, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 2)
        self._check(self.lib.ewg_set_solution(self.h, time_idx, _ptr(x)), "set_solution")

    def get_solution(self, time_idx=0, out=None):
        x = self.vec() if out is None else out
        assert x.dtype == np.float64 and x.shape == (self.n, 2) and x.flags.c_contiguous
        self._check(self.lib.ewg_get_solution(self.h, time_idx, _ptr(x)), "get_solution")
        return x

    def apply_initial_solution(self):
        self._check(self.lib.ewg_apply_initial_solution(self.h), "apply_initial_solution")

    def advance_time_level(self):
        self._check(self.lib.ewg_advance_time_level(self.h), "advance_time_level")

    def restore_time_level(self):
        self._check(self.lib.ewg_restore_time_level(self.h), "restore_time_level")

    def set_local_linearizer(self, kind: int, method: int = 1):
        """LOCAL_LINEARIZER_AD (default) or LOCAL_LINEARIZER_FD with NumericDifferenceMethod
        `method` (-1 backward, 0 central, +1 forward)."""
        self._check(self.lib.ewg_set_local_linearizer(self.h, kind, method), "set_local_linearizer")

    def update_begin(self):
        """ImmiscibleModel::updateBegin: records the FD linearizer's reference pressure."""
        self._check(self.lib.ewg_update_begin(self.h), "update_begin")

    def set_reference_pressure(self, p_ref: float):
        """updateBegin with the caller's reference pressure (a slab takes the whole grid's)."""
        self._check(self.lib.ewg_set_reference_pressure(self.h, float(p_ref)), "set_reference_pressure")

    def intensive_quantities(self):
        """N x {p_cnw, lambda_w, lambda_n} of solution(0), natural order."""
        out = np.zeros((self.n, 3))
        self._check(self.lib.ewg_get_intensive_quantities(self.h, _ptr(out)), "intensive_quantities")
        return out

    def linearize(self, dt) -> LinReport:
        rep = LinReport()
        self._check(self.lib.ewg_linearize(self.h, dt, C.byref(rep)), "linearize")
        return rep

    def residual(self):
        r = self.vec()
        self._check(self.lib.ewg_get_residual(self.h, _ptr(r)), "get_residual")
        return r

    def jacobian_bcrs(self):
        rp = np.zeros(self.n + 1, dtype=np.int32)
        ci = np.zeros(self.nnzb, dtype=np.int32)
        b = np.zeros((self.nnzb, 2, 2), dtype=np.float64)
        self._check(self.lib.ewg_get_jacobian_bcrs(self.h, _ptr(rp, C.c_int32), _ptr(ci, C.c_int32),
                                                   _ptr(b)), "get_jacobian_bcrs")
        return rp, ci, b

    def set_matrix_bcrs(self, rp, ci, b):
        rp = np.ascontiguousarray(rp, dtype=np.int32)
        ci = np.ascontiguousarray(ci, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self._check(self.lib.ewg_set_matrix_bcrs(self.h, _ptr(rp, C.c_int32), _ptr(ci, C.c_int32),
                                                 _ptr(b)), "set_matrix_bcrs")

    def set_residual(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(self.n, 2)
        self._check(self.lib.ewg_set_residual(self.h, _ptr(r)), "set_residual")

    def residual_norm(self, x, dt):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 2)
        out = C.c_double()
        self._check(self.lib.ewg_residual_norm(self.h, _ptr(x), dt, C.byref(out)), "residual_norm")
        return out.value

    def solve(self, opts: SolveOpts | None = None, check=False) -> SolveReport:
        opts = opts or default_solve_opts()
        rep = SolveReport()
        st = self.lib.ewg_solve(self.h, C.byref(opts), C.byref(rep))
        if check:
            self._check(st, "solve")
        return rep

    def update(self):
        dx = self.vec()
        self._check(self.lib.ewg_get_update(self.h, _ptr(dx)), "get_update")
        return dx

    def apply_preconditioner(self, b, opts: SolveOpts | None = None):
        opts = opts or default_solve_opts()
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(self.n, 2)
        y = self.vec()
        self._check(self.lib.ewg_apply_preconditioner(self.h, C.byref(opts), _ptr(b), _ptr(y)),
                    "apply_preconditioner")
        return y

    def apply_jacobian(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 2)
        y = self.vec()
        self._check(self.lib.ewg_apply_jacobian(self.h, _ptr(x), _ptr(y)), "apply_jacobian")
        return y

    def newton_update(self):
        self._check(self.lib.ewg_newton_update(self.h), "newton_update")

    def newton_apply(self, dt, nopts=None, sopts=None) -> tuple[int, NewtonReport]:
        nopts = nopts or default_newton_opts()
        sopts = sopts or default_solve_opts()
        rep = NewtonReport()
        st = self.lib.ewg_newton_apply(self.h, dt, C.byref(nopts), C.byref(sopts), C.byref(rep))
        return st, rep

    @property
    def stream(self) -> int:
        """The cudaStream_t (as an integer handle) all work of this context runs on."""
        return self.lib.ewg_get_stream(self.h)

    # ---- device-order vectors (N x 2 float64 torch tensors in the context's storage order) ----

    def device_buffer(self, which: int):
        """A torch view of the solution(0) (BUFFER_SOLUTION) or residual (BUFFER_RESIDUAL) device
        vector; it aliases the context's memory and is valid until close()."""
        import torch
        p = C.c_void_p()
        self._check(self.lib.ewg_device_buffer(self.h, which, C.byref(p)), "device_buffer")
        return torch.as_tensor(_DeviceVector(p.value, self.n), device="cuda")

    def _device_args(self, *ts):
        for t in ts:
            if not (t.is_cuda and t.dtype.is_floating_point and t.element_size() == 8 and t.is_contiguous()
                    and tuple(t.shape) == (self.n, 2)):
                raise ValueError("device vectors are contiguous N x 2 float64 CUDA tensors")
        return [C.c_void_p(t.data_ptr()) for t in ts]

    def device_spmv(self, x, y):
        """y = J x on the context's stream (device storage order)."""
        xp, yp = self._device_args(x, y)
        self._check(self.lib.ewg_device_spmv(self.h, xp, yp), "device_spmv")

    def device_precondition(self, b, y, opts: SolveOpts | None = None):
        """y = M^-1 b on the context's stream (device storage order)."""
        opts = opts or default_solve_opts()
        bp, yp = self._device_args(b, y)
        self._check(self.lib.ewg_device_precondition(self.h, C.byref(opts), bp, yp), "device_precondition")

    # fused kernels of one slab's BiCGStab iteration (dd.distributed_bicgstab); device tensors
    # (N x 2 float64), owned rows [lo, hi) of each colour half, `out` a float64 device tensor,
    # `state` the device state (a uint8 tensor of ewg_device_bicg_state_size() bytes)

    @staticmethod
    def _ptr_of(t):
        return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(None)

    def device_bicg_p(self, p, r, r0, v, state):
        a = self._device_args(p, r, r0, v)
        self._check(self.lib.ewg_device_bicg_p(self.h, *a, self._ptr_of(state)), "device_bicg_p")

    def device_bicg_spmv_dot(self, x, y, w, lo, hi, state, out):
        a = self._device_args(x, y, w)
        self._check(self.lib.ewg_device_bicg_spmv_dot(self.h, *a, int(lo), int(hi), self._ptr_of(state),
                                                      self._ptr_of(out)), "device_bicg_spmv_dot")

    def device_bicg_hs(self, x, y, r, v, lo, hi, state, out):
        a = self._device_args(x, y, r, v)
        self._check(self.lib.ewg_device_bicg_hs(self.h, *a, int(lo), int(hi), self._ptr_of(state), self._ptr_of(out)),
                    "device_bicg_hs")

    def device_bicg_spmv_dot2(self, z, t, s, lo, hi, state, out):
        a = self._device_args(z, t, s)
        self._check(self.lib.ewg_device_bicg_spmv_dot2(self.h, *a, int(lo), int(hi), self._ptr_of(state),
                                                       self._ptr_of(out)), "device_bicg_spmv_dot2")

    def device_bicg_xr(self, x, z, r, t, r0, lo, hi, state, out):
        a = self._device_args(x, z, r, t, r0)
        self._check(self.lib.ewg_device_bicg_xr(self.h, *a, int(lo), int(hi), self._ptr_of(state), self._ptr_of(out)),
                    "device_bicg_xr")

    def device_bicg_state(self, stage, state, red, opts=None):
        o = C.byref(opts) if opts is not None else None
        self._check(self.lib.ewg_device_bicg_state(self.h, int(stage), self._ptr_of(state), self._ptr_of(red), o),
                    "device_bicg_state")

    def device_bicg_state_read(self, state):
        """(status, iterations, restarts, residual, initial residual) of a distributed solve's state."""
        st, it, rs = C.c_int32(), C.c_int32(), C.c_int32()
        res, ini = C.c_double(), C.c_double()
        self._check(self.lib.ewg_device_bicg_state_read(self.h, self._ptr_of(state), C.byref(st), C.byref(it),
                                                        C.byref(rs), C.byref(res), C.byref(ini)),
                    "device_bicg_state_read")
        return st.value, it.value, rs.value, res.value, ini.value

    def transfer_counters(self, reset=False):
        """(host->device, device->host) bytes of this context's entry points (ewg_transfer_counters)."""
        h2d, d2h = C.c_uint64(), C.c_uint64()
        self._check(self.lib.ewg_transfer_counters(self.h, int(reset), C.byref(h2d), C.byref(d2h)), "transfer_counters")
        return h2d.value, d2h.value

    def profile_enable(self, on=True, period=1):
        """Time kernel launches with CUDA events: every `period`-th launch of each class."""
        self._check(self.lib.ewg_profile_enable(self.h, int(period) if on else 0), "profile_enable")

    def profile_reset(self):
        self._check(self.lib.ewg_profile_reset(self.h), "profile_reset")

    def profile(self) -> dict:
        """{kernel class: (milliseconds, launches)} accumulated since the last reset."""
        out = {}
        ms = C.c_double()
        n = C.c_int64()
        for k in range(self.lib.ewg_profile_num_kernels()):
            self._check(self.lib.ewg_profile_get(self.h, k, C.byref(ms), C.byref(n)), "profile_get")
            if n.value:
                out[self.lib.ewg_profile_kernel_name(k).decode()] = (ms.value, n.value)
        return out

    def save_restart(self, output_dir: str, sim_name: str, sim: "SimulatorState") -> str:
        """Simulator::serialize of this context's solution(0) (restart file name returned)."""
        return write_restart(output_dir, sim_name, self.case.grid, self.get_solution(0), sim)

    def load_restart(self, output_dir: str, sim_name: str, t: float) -> "SimulatorState":
        """Restart from the file written at time t: solution(0) from the file and solution(1) =
        solution(0) (EcfvDiscretization::deserialize); returns the simulator state."""
        sim, x, _ = read_restart(output_dir, sim_name, t, self.case.grid)
        self.set_solution(0, x)
        self.set_solution(1, x)
        return sim

    def run(self, n_steps, dt, nopts=None, sopts=None, max_divisions=10):
        """Simulator time loop at a fixed step size with FvBaseProblem::timeIntegration's halving
        retry (fvbaseproblem.hh:507-550). Returns the per-step Newton reports."""
        reports = []
        for _ in range(n_steps):
            h = dt
            for _attempt in range(max_divisions):
                st, rep = self.newton_apply(h, nopts, sopts)
                if st == EWG_OK:
                    break
                self.restore_time_level()
                h /= 2.0
            else:
                raise EwgError(st, "time integration did not converge")
            self.advance_time_level()
            reports.append(rep)
        return reports


# ------------------------------------------------------------------------------------------
# restart files (io/restart.hh:36-271; the C++ driver's host/restart.hh writes the same files)


@dataclass
class SimulatorState:
    """Simulator's serialized state (utils/simulator.hh:944-952)."""
    episode_idx: int = 0
    episode_start_time: float = 0.0
    episode_length: float = 1e100
    start_time: float = 0.0
    time: float = 0.0
    time_step_idx: int = 0


def _g20(v: float) -> str:
    """A double as an ostream with precision 20 prints it (%.20g)."""
    return "%.20g" % v


def _ostream_default(v: float) -> str:
    """A double as an ostream with its default precision (6) prints it (%g)."""
    return "%g" % v


def restart_grid_counts(grid: Grid):
    """(elements, codim dim-1 entities, vertices) of the structured grid."""
    nx, ny = grid.nx, grid.ny
    if grid.dim == 2:
        return nx * ny, nx * (ny + 1) + (nx + 1) * ny, (nx + 1) * (ny + 1)
    nz = grid.nz
    return (nx * ny * nz, nx * (ny + 1) * (nz + 1) + (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz,
            (nx + 1) * (ny + 1) * (nz + 1))


def restart_cookie(grid: Grid, num_cpus: int = 1, rank: int = 0) -> str:
    """magicRestartCookie_ (restart.hh:42-62); the grid name is the reference's literal 'blubb'."""
    ne, ned, nv = restart_grid_counts(grid)
    return (f"eWoms restart file: gridName='blubb' numCPUs={num_cpus} myRank={rank} "
            f"numElements={ne} numEdges={ned} numVertices={nv}")


def restart_file_name(output_dir: str, sim_name: str, t: float, rank: int = 0) -> str:
    """restartFileName_ (restart.hh:67-83): <dir>/<simName>_time=<t>_rank=<rank>.ers."""
    d = "" if output_dir == "." else (output_dir if not output_dir or output_dir.endswith("/") else output_dir + "/")
    return f"{d}{sim_name}_time={_ostream_default(t)}_rank={rank}.ers"


def write_restart(output_dir: str, sim_name: str, grid: Grid, x: np.ndarray, sim: SimulatorState,
                  vtk: tuple | None = None, num_cpus: int = 1, rank: int = 0) -> str:
    """Simulator::serialize: cookie, Simulator section, the VTK writer's section when given
    (writer index, collection text, write position), and solution(0) of every cell (natural order).
    Returns the file name."""
    x = np.asarray(x, dtype=np.float64).reshape(-1, 2)
    path = restart_file_name(output_dir, sim_name, sim.time, rank)
    parts = [restart_cookie(grid, num_cpus, rank), "\n", "\n", "Simulator\n",
             f"{sim.episode_idx} {_g20(sim.episode_start_time)} {_g20(sim.episode_length)} "
             f"{_g20(sim.start_time)} {_g20(sim.time)} {sim.time_step_idx} ", "\n"]
    if vtk is not None:
        num, coll, pos = vtk
        parts += ["VTKMultiWriter\n", f"{num}\n", f"{len(coll.encode())}  {pos}\n", coll, "\n"]
    parts.append("Entities: Codim 0\n")
    parts.append("".join(f"{_g20(a)} {_g20(b)} \n" for a, b in x))
    parts.append("\n")
    with open(path, "w") as f:
        f.write("".join(parts))
    return path


def read_restart(output_dir: str, sim_name: str, t: float, grid: Grid, vtk: bool = False,
                 num_cpus: int = 1, rank: int = 0):
    """Simulator::run with RestartTime = t: (SimulatorState, solution(0) as N x 2, the VTK
    section (index, collection, write position) or None). Raises like Restart::deserialize* on a
    missing or empty file, a wrong cookie, a short section or unread values."""
    path = restart_file_name(output_dir, sim_name, t, rank)
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError as e:
        raise RuntimeError(f"Restart file '{path}' could not be opened properly") from e
    if not data:
        raise RuntimeError(f"Restart file '{path}' is empty")
    pos = 0

    def line():
        nonlocal pos
        if pos >= len(data):
            raise RuntimeError("Encountered unexpected EOF in restart file.")
        e = data.find(b"\n", pos)
        e = len(data) if e < 0 else e
        ln = data[pos:e].decode()
        pos = e + 1
        return ln

    def section_begin(cookie):
        if line() != cookie:
            raise RuntimeError(f"Could not start section '{cookie}'")

    def section_end():
        if line().strip():
            raise RuntimeError("Encountered unread values while deserializing")

    section_begin(restart_cookie(grid, num_cpus, rank))
    section_end()
    section_begin("Simulator")
    vals = line().split()
    if len(vals) != 6:
        raise RuntimeError("Encountered unread values while deserializing" if len(vals) > 6 else
                           "Restart file is corrupted (Simulator section)")
    # the values and the section's end share one line (the writer ends the section right after them)
    sim = SimulatorState(int(vals[0]), float(vals[1]), float(vals[2]), float(vals[3]), float(vals[4]), int(vals[5]))
    vtk_state = None
    if vtk:
        section_begin("VTKMultiWriter")
        num = int(line().split()[0])
        ln, wpos = (int(v) for v in line().split())
        coll = data[pos:pos + ln].decode()
        pos += ln
        section_end()
        vtk_state = (num, coll, wpos)
    section_begin("Entities: Codim 0")
    n = grid.n_cells
    x = np.empty((n, 2))
    for c in range(n):
        v = line().split()
        if len(v) < 2:
            raise RuntimeError(f"Could not deserialize degree of freedom {c}")
        x[c, 0], x[c, 1] = float(v[0]), float(v[1])
    section_end()
    return sim, x, vtk_state


# ------------------------------------------------------------------------------------------
# learned Newton initial guess

NET_CIN = (16, 32, 32, 32)
NET_COUT = (32, 32, 32, 8)
NET_CIN_REAL = (5, 32, 32, 32)
NET_COUT_REAL = (32, 32, 32, 2)


def net_layout():
    """[(w_offset, b_offset, cin_pad, cout_pad)] of the flat FP32 parameter vector."""
    out, off = [], 0
    for ci, co in zip(NET_CIN, NET_COUT):
        w = off
        off += 27 * co * ci
        out.append((w, off, ci, co))
        off += co
    return out


class GuessNet:
    """The learned initial-guess network (ewg_net): device training and inference."""

    def __init__(self, seed: int = 0):
        lib = load()
        self.lib = lib
        h = C.c_void_p()
        st = lib.ewg_net_create(seed, C.byref(h))
        if st != EWG_OK:
            raise EwgError(st, "ewg_net_create")
        self.h = h
        self.n_params = lib.ewg_net_num_params()

    def _check(self, st, what):
        if st != EWG_OK:
            raise EwgError(st, f"{what}: {self.lib.ewg_net_last_error(self.h).decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.ewg_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        self._check(self.lib.ewg_net_get_params(self.h, _ptr(p, C.c_float), self.n_params), "get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self.lib.ewg_net_set_params(self.h, _ptr(p, C.c_float), self.n_params), "set_params")

    def scales(self) -> np.ndarray:
        s = np.zeros(8)
        self._check(self.lib.ewg_net_get_scales(self.h, _ptr(s)), "get_scales")
        return s

    def set_scales(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64)
        self._check(self.lib.ewg_net_set_scales(self.h, _ptr(s)), "set_scales")

    def set_options(self, loss_weight_p=1.0, loss_weight_s=1.0, apply_pressure=False, sn_threshold=0.0):
        self._check(self.lib.ewg_net_set_options(self.h, loss_weight_p, loss_weight_s, int(apply_pressure),
                                                 sn_threshold), "set_options")

    def eval_host(self, feats, targets=None, grads=False):
        """feats [B, D, H, W, 5] float32 -> (outputs [B, D, H, W, 2], loss, grads or None)."""
        feats = np.ascontiguousarray(feats, dtype=np.float32)
        B, D, H, W, _ = feats.shape
        out = np.zeros((B, D, H, W, 2), dtype=np.float32)
        loss = C.c_float()
        g = np.zeros(self.n_params, dtype=np.float32) if grads else None
        t = None if targets is None else np.ascontiguousarray(targets, dtype=np.float32)
        st = self.lib.ewg_net_eval_host(self.h, B, D, H, W, _ptr(feats, C.c_float),
                                        None if t is None else _ptr(t, C.c_float), _ptr(out, C.c_float),
                                        C.byref(loss), None if g is None else _ptr(g, C.c_float))
        self._check(st, "eval_host")
        return out, loss.value, g

    def record(self, ctx: "Context", dt: float):
        self._check(self.lib.ewg_net_record_sample(self.h, ctx.h, dt), "record_sample")

    @property
    def n_samples(self) -> int:
        return self.lib.ewg_net_num_samples(self.h)

    def train(self, idx, lr=1e-3) -> float:
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        loss = C.c_float()
        self._check(self.lib.ewg_net_train(self.h, _ptr(idx, C.c_int64), len(idx), lr, C.byref(loss)), "train")
        return loss.value

    def eval_samples(self, idx) -> float:
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        loss = C.c_float()
        self._check(self.lib.ewg_net_eval_samples(self.h, _ptr(idx, C.c_int64), len(idx), C.byref(loss)), "eval")
        return loss.value

    def save(self, path, options=None):
        np.savez_compressed(path, params=self.params(), scales=self.scales(),
                            options=np.array(options if options is not None else [0.1, 1.0, 0.0, 0.0]))

    def load_file(self, path):
        z = np.load(path)
        self.set_scales(z["scales"])
        self.set_params(z["params"])
        if "options" in z:
            o = z["options"]
            self.set_options(float(o[0]), float(o[1]), bool(o[2]), float(o[3]))

    def predict_guess(self, ctx: "Context", dt: float):
        """Writes solution(0) of ctx; returns (used_guess, residual of guess, residual of previous)."""
        used = C.c_int32()
        rg, rp = C.c_double(), C.c_double()
        st = self.lib.ewg_predict_guess(ctx.h, self.h, dt, C.byref(used), C.byref(rg), C.byref(rp))
        ctx._check(st, "predict_guess")
        return bool(used.value), rg.value, rp.value


# ------------------------------------------------------------------------------------------
# vertex-centred discretization


def vcfv_pattern(grid: Grid):
    """BCRS pattern of the vertex stencil: row v holds the vertices of its adjacent elements,
    columns ascending (the order FvBaseLinearizer::createMatrix_ produces with std::set)."""
    nvx, nvy = grid.nx + 1, grid.ny + 1
    nvz = grid.nz + 1 if grid.dim == 3 else 1
    rows, cols = [0], []
    for k in range(nvz):
        for j in range(nvy):
            for i in range(nvx):
                for dk in ((-1, 0, 1) if grid.dim == 3 else (0,)):
                    for dj in (-1, 0, 1):
                        for di in (-1, 0, 1):
                            ii, jj, kk = i + di, j + dj, k + dk
                            if 0 <= ii < nvx and 0 <= jj < nvy and 0 <= kk < nvz:
                                cols.append(ii + nvx * (jj + nvy * kk))
                rows.append(len(cols))
    return np.array(rows, dtype=np.int32), np.array(cols, dtype=np.int32)


class VcfvContext:
    """One vertex-centred lens problem on the device (ewg_vcfv_* in include/ewg.h). Host arrays
    are natural vertex order, NV x 2 float64."""

    def __init__(self, case: LensCase):
        self.lib = load()
        self.case = case
        self._perm = np.ascontiguousarray(case.perm, dtype=np.float64)
        h = C.c_void_p()
        st = self.lib.ewg_vcfv_create(C.byref(case.grid), C.byref(case.problem), _ptr(self._perm), C.byref(h))
        if st != EWG_OK:
            raise EwgError(st, "ewg_vcfv_create failed")
        self.h = h
        self.n = self.lib.ewg_vcfv_num_dofs(h)

    def _check(self, st, what=""):
        if st != EWG_OK:
            raise EwgError(st, f"{what}: {self.lib.ewg_vcfv_last_error(self.h).decode()}")
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.ewg_vcfv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(self.lib.ewg_vcfv_launches(self.h))

    def vec(self):
        return np.zeros((self.n, 2), dtype=np.float64)

    def set_solution(self, t, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 2)
        self._check(self.lib.ewg_vcfv_set_solution(self.h, t, _ptr(x)), "set_solution")

    def get_solution(self, t=0):
        x = self.vec()
        self._check(self.lib.ewg_vcfv_get_solution(self.h, t, _ptr(x)), "get_solution")
        return x

    def apply_initial_solution(self):
        self._check(self.lib.ewg_vcfv_apply_initial_solution(self.h), "apply_initial_solution")

    def advance_time_level(self):
        self._check(self.lib.ewg_vcfv_advance_time_level(self.h), "advance_time_level")

    def restore_time_level(self):
        self._check(self.lib.ewg_vcfv_restore_time_level(self.h), "restore_time_level")

    def set_local_linearizer(self, kind: int, method: int = 1):
        self._check(self.lib.ewg_vcfv_set_local_linearizer(self.h, kind, method), "set_local_linearizer")

    def update_begin(self):
        self._check(self.lib.ewg_vcfv_update_begin(self.h), "update_begin")

    def linearize(self, dt) -> float:
        e = C.c_double()
        self._check(self.lib.ewg_vcfv_linearize(self.h, dt, C.byref(e)), "linearize")
        return e.value

    def residual(self):
        r = self.vec()
        self._check(self.lib.ewg_vcfv_get_residual(self.h, _ptr(r)), "get_residual")
        return r

    def jacobian_bcrs(self):
        rp, ci = vcfv_pattern(self.case.grid)
        b = np.zeros((len(ci), 2, 2), dtype=np.float64)
        self._check(self.lib.ewg_vcfv_get_jacobian_bcrs(self.h, _ptr(rp, C.c_int32), _ptr(ci, C.c_int32), len(ci),
                                                        _ptr(b)), "get_jacobian_bcrs")
        return rp, ci, b

    def solve(self, sopts=None):
        """BiCGStab on the last linearization: (status, iterations, dx)."""
        sopts = sopts or default_solve_opts()
        dx = self.vec()
        its = C.c_int32()
        st = self.lib.ewg_vcfv_solve(self.h, C.byref(sopts), _ptr(dx), C.byref(its))
        return st, its.value, dx

    def newton_apply(self, dt, nopts=None, sopts=None):
        nopts = nopts or default_newton_opts()
        sopts = sopts or default_solve_opts(precond=PRECOND_JACOBI)
        its, lin, err = C.c_int32(), C.c_int32(), C.c_double()
        st = self.lib.ewg_vcfv_newton_apply(self.h, dt, C.byref(nopts), C.byref(sopts), C.byref(its), C.byref(lin),
                                            C.byref(err))
        return st, its.value, lin.value, err.value


# ------------------------------------------------------------------------------------------
# batched ensemble


class Ensemble:
    """Many lens problems (3D, even nx) in one device context, advanced together
    (ewg_ensemble_* in include/ewg.h). Host arrays are natural order, N_m x 2 float64."""

    def __init__(self, cases, precision=PRECISION_MIXED, use_graph=True, check_interval=8,
                 max_divisions=10):
        lib = load()
        self.lib = lib
        self.cases = list(cases)
        M = len(self.cases)
        grids = (Grid * M)(*[c.grid for c in self.cases])
        probs = (Problem * M)(*[c.problem for c in self.cases])
        self._perms = [np.ascontiguousarray(c.perm, dtype=np.float64) for c in self.cases]
        parr = (C.POINTER(C.c_double) * M)(*[_ptr(p) for p in self._perms])
        o = EnsembleOpts()
        lib.ewg_default_ensemble_opts(C.byref(o))
        o.precision, o.use_graph, o.check_interval = precision, int(use_graph), check_interval
        o.max_divisions = max_divisions
        h = C.c_void_p()
        st = lib.ewg_ensemble_create(M, grids, probs, parr, C.byref(o), C.byref(h))
        if st != EWG_OK:
            raise EwgError(st, lib.ewg_ensemble_create_error().decode())
        self.h = h
        self.M = M
        self.n = [c.grid.n_cells for c in self.cases]

    def _check(self, st, what=""):
        if st != EWG_OK:
            raise EwgError(st, f"{what}: {self.lib.ewg_ensemble_last_error(self.h).decode()}")
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.ewg_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def total_cells(self) -> int:
        return int(self.lib.ewg_ensemble_num_cells(self.h, -1))

    @property
    def stream(self) -> int:
        return self.lib.ewg_ensemble_get_stream(self.h)

    def _dt(self, dt):
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.M,)))
        return a

    def apply_initial_solution(self):
        self._check(self.lib.ewg_ensemble_apply_initial_solution(self.h), "apply_initial_solution")

    def set_solution(self, member, time_idx, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n[member], 2)
        self._check(self.lib.ewg_ensemble_set_solution(self.h, member, time_idx, _ptr(x)), "set_solution")

    def get_solution(self, member, time_idx=0, out=None):
        x = np.zeros((self.n[member], 2)) if out is None else out
        self._check(self.lib.ewg_ensemble_get_solution(self.h, member, time_idx, _ptr(x)), "get_solution")
        return x

    def linearize(self, dt):
        d = self._dt(dt)
        norms = np.zeros(self.M)
        self._check(self.lib.ewg_ensemble_linearize(self.h, _ptr(d), _ptr(norms)), "linearize")
        return norms

    def residual(self, member):
        r = np.zeros((self.n[member], 2))
        self._check(self.lib.ewg_ensemble_get_residual(self.h, member, _ptr(r)), "get_residual")
        return r

    def autotune(self, dt, sopts=None):
        d = self._dt(dt)
        sopts = sopts or default_solve_opts()
        self._check(self.lib.ewg_ensemble_autotune(self.h, _ptr(d), C.byref(sopts)), "autotune")
        return self.launch_shapes()

    def launch_shapes(self):
        g = np.zeros(len(ENSEMBLE_KERNEL_CLASSES), dtype=np.int32)
        v = C.c_int32()
        self._check(self.lib.ewg_ensemble_get_launch_shapes(self.h, _ptr(g, C.c_int32), len(g), C.byref(v)),
                    "launch_shapes")
        out = dict(zip(ENSEMBLE_KERNEL_CLASSES, (int(x) for x in g)))
        out["assemble_variant"] = v.value
        return out

    def step(self, dt, nopts=None, sopts=None, check=True):
        """One implicit step of every member (own dt each). Returns (status, reports, stats)."""
        return self.advance(1, dt, nopts, sopts, check)

    def advance(self, steps, dt, nopts=None, sopts=None, check=True, device=False):
        """`steps` implicit steps of every member, each at its own pace. Returns (status, reports,
        stats); reports sum the iterations over each member's accepted steps. device=True takes
        every decision on the device (ewg_ensemble_advance_device: the supersteps run inside one
        CUDA graph WHILE node); the results are the same bits."""
        d = self._dt(dt)
        nopts = nopts or default_newton_opts()
        sopts = sopts or default_solve_opts()
        reps = (EnsembleReport * self.M)()
        stats = EnsembleStats()
        fn = self.lib.ewg_ensemble_advance_device if device else self.lib.ewg_ensemble_advance
        st = fn(self.h, int(steps), _ptr(d), C.byref(nopts), C.byref(sopts), reps, C.byref(stats))
        if check:
            self._check(st, "advance")
        return st, list(reps), stats

