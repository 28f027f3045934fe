"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (liboracle.so).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm as the checker / the
timed CPU restatement of the reference. PARITY UNPINNED at the third-party boundary (material
laws, DenseAd, dune-istl ILU): see ewoms_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "ewoms-numerics_b200"))
import ewg  # noqa: E402  (ABI structs only)

ORDER_NATURAL, ORDER_REDBLACK, ORDER_COLOURS, ORDER_BOX8 = 0, 1, 2, 3


def build(force=False):
    """Compile the oracle restatement with g++ (a few seconds)."""
    src = os.path.join(HERE, "ewoms_oracle.cc")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "ewoms_oracle.h"))):
        return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", LIB, src, "-lpthread"]
    subprocess.check_call(cmd)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    P = C.POINTER
    d = C.c_double
    i32 = C.c_int32
    sig = {
        "orc_create": (C.c_void_p, [P(ewg.Grid), P(ewg.Problem), P(d), C.c_int]),
        "orc_destroy": (None, [C.c_void_p]),
        "orc_last_error": (C.c_char_p, [C.c_void_p]),
        "orc_num_cells": (C.c_int64, [C.c_void_p]),
        "orc_num_blocks": (C.c_int64, [C.c_void_p]),
        "orc_set_recycle_first_iteration_storage": (None, [C.c_void_p, C.c_int]),
        "orc_set_local_linearizer": (None, [C.c_void_p, C.c_int, C.c_int]),
        "orc_update_begin": (None, [C.c_void_p]),
        "orc_set_reference_pressure": (C.c_int, [C.c_void_p, C.c_double]),
        "orc_set_solution": (None, [C.c_void_p, C.c_int, P(d)]),
        "orc_get_solution": (None, [C.c_void_p, C.c_int, P(d)]),
        "orc_apply_initial_solution": (None, [C.c_void_p]),
        "orc_advance_time_level": (None, [C.c_void_p]),
        "orc_linearize": (C.c_int, [C.c_void_p, d, C.c_int, P(d)]),
        "orc_get_residual": (None, [C.c_void_p, P(d)]),
        "orc_get_jacobian_bcrs": (None, [C.c_void_p, P(i32), P(i32), P(d)]),
        "orc_set_jacobian_blocks": (None, [C.c_void_p, P(d)]),
        "orc_set_residual": (None, [C.c_void_p, P(d)]),
        "orc_fd_jacobian": (C.c_int, [C.c_void_p, d, P(d)]),
        "orc_solve": (C.c_int, [C.c_void_p, P(ewg.SolveOpts), C.c_int, P(d), P(C.c_int), P(d)]),
        "orc_apply_preconditioner": (C.c_int, [C.c_void_p, P(ewg.SolveOpts), C.c_int, P(d), P(d)]),
        "orc_apply_jacobian": (None, [C.c_void_p, P(d), P(d)]),
        "orc_newton_apply": (C.c_int, [C.c_void_p, d, P(ewg.NewtonOpts), P(ewg.SolveOpts), C.c_int,
                                       P(C.c_int), P(C.c_int), P(d)]),
        "orc_residual_norm": (d, [C.c_void_p, P(d), d]),
        "orc_material_eval": (None, [P(ewg.Material), d, P(d)]),
        "orc_global_storage": (None, [C.c_void_p, C.c_int, P(d)]),
        "orc_boundary_rates": (None, [C.c_void_p, P(d)]),
        "orc_vcfv_create": (C.c_void_p, [P(ewg.Grid), P(ewg.Problem), P(d), C.c_int]),
        "orc_vcfv_destroy": (None, [C.c_void_p]),
        "orc_vcfv_last_error": (C.c_char_p, [C.c_void_p]),
        "orc_vcfv_num_dofs": (C.c_int64, [C.c_void_p]),
        "orc_vcfv_num_blocks": (C.c_int64, [C.c_void_p]),
        "orc_vcfv_set_solution": (None, [C.c_void_p, C.c_int, P(d)]),
        "orc_vcfv_get_solution": (None, [C.c_void_p, C.c_int, P(d)]),
        "orc_vcfv_apply_initial_solution": (None, [C.c_void_p]),
        "orc_vcfv_advance_time_level": (None, [C.c_void_p]),
        "orc_vcfv_set_local_linearizer": (None, [C.c_void_p, C.c_int, C.c_int]),
        "orc_vcfv_update_begin": (None, [C.c_void_p]),
        "orc_vcfv_total_volumes": (None, [C.c_void_p, P(d)]),
        "orc_vcfv_linearize": (C.c_int, [C.c_void_p, d, C.c_int, P(d)]),
        "orc_vcfv_get_residual": (None, [C.c_void_p, P(d)]),
        "orc_vcfv_get_jacobian_bcrs": (None, [C.c_void_p, P(i32), P(i32), P(d)]),
        "orc_vcfv_newton_apply": (C.c_int, [C.c_void_p, d, P(ewg.NewtonOpts), P(ewg.SolveOpts), C.c_int,
                                            P(C.c_int), P(C.c_int), P(d)]),
        "orc_vcfv_global_storage": (None, [C.c_void_p, C.c_int, P(d)]),
        "orc_vcfv_boundary_rates": (None, [C.c_void_p, P(d)]),
        "orc_vcfv_geometry": (None, [C.c_void_p, P(i32), P(d), P(d), P(d), P(d), P(d)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


class Oracle:
    """CPU restatement of the reference's linearizer + solver on one lens case."""

    def __init__(self, case: "ewg.LensCase", nthreads: int = 1):
        self.lib = load()
        self.case = case
        perm = np.ascontiguousarray(case.perm, dtype=np.float64)
        self.h = self.lib.orc_create(C.byref(case.grid), C.byref(case.problem), _p(perm), nthreads)
        self.n = self.lib.orc_num_cells(self.h)
        self.nnzb = self.lib.orc_num_blocks(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def err(self):
        return self.lib.orc_last_error(self.h).decode()

    def vec(self):
        return np.zeros((self.n, 2), dtype=np.float64)

    def set_recycle_first_iteration_storage(self, on: bool):
        self.lib.orc_set_recycle_first_iteration_storage(self.h, int(on))

    def set_local_linearizer(self, kind: int, method: int = 1):
        """kind 0: AutoDiffLocalLinearizer; 1: FiniteDifferenceLocalLinearizer with
        NumericDifferenceMethod `method` (-1 backward, 0 central, +1 forward)."""
        self.lib.orc_set_local_linearizer(self.h, int(kind), int(method))

    def update_begin(self):
        """ImmiscibleModel::updateBegin: the reference pressure for the FD pressure weight."""
        self.lib.orc_update_begin(self.h)

    def set_reference_pressure(self, p_ref):
        """updateBegin with the caller's reference pressure (a z-slab takes the whole grid's)."""
        if self.lib.orc_set_reference_pressure(self.h, float(p_ref)):
            raise ValueError(self.err())

    def set_solution(self, t, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 2)
        self.lib.orc_set_solution(self.h, t, _p(x))

    def get_solution(self, t=0):
        x = self.vec()
        self.lib.orc_get_solution(self.h, t, _p(x))
        return x

    def apply_initial_solution(self):
        self.lib.orc_apply_initial_solution(self.h)

    def advance_time_level(self):
        self.lib.orc_advance_time_level(self.h)

    def linearize(self, dt, newton_iteration=0):
        e = C.c_double()
        rc = self.lib.orc_linearize(self.h, dt, newton_iteration, C.byref(e))
        if rc:
            raise RuntimeError(self.err())
        return e.value

    def residual(self):
        r = self.vec()
        self.lib.orc_get_residual(self.h, _p(r))
        return r

    def jacobian_bcrs(self):
        rp = np.zeros(self.n + 1, dtype=np.int32)
        ci = np.zeros(self.nnzb, dtype=np.int32)
        b = np.zeros((self.nnzb, 2, 2), dtype=np.float64)
        self.lib.orc_get_jacobian_bcrs(self.h, _p(rp, C.c_int32), _p(ci, C.c_int32), _p(b))
        return rp, ci, b

    def set_jacobian_blocks(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.lib.orc_set_jacobian_blocks(self.h, _p(b))

    def set_residual(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(self.n, 2)
        self.lib.orc_set_residual(self.h, _p(r))

    def fd_jacobian(self, dt):
        b = np.zeros((self.nnzb, 2, 2), dtype=np.float64)
        if self.lib.orc_fd_jacobian(self.h, dt, _p(b)):
            raise RuntimeError(self.err())
        return b

    def solve(self, opts=None, ordering=ORDER_NATURAL):
        opts = opts or ewg.default_solve_opts()
        dx = self.vec()
        it = C.c_int()
        fr = C.c_double()
        rc = self.lib.orc_solve(self.h, C.byref(opts), ordering, _p(dx), C.byref(it), C.byref(fr))
        return rc, dx, it.value, fr.value

    def apply_preconditioner(self, b, opts=None, ordering=ORDER_NATURAL):
        opts = opts or ewg.default_solve_opts()
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(self.n, 2)
        y = self.vec()
        if self.lib.orc_apply_preconditioner(self.h, C.byref(opts), ordering, _p(b), _p(y)):
            raise RuntimeError(self.err())
        return y

    def apply_jacobian(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 2)
        y = self.vec()
        self.lib.orc_apply_jacobian(self.h, _p(x), _p(y))
        return y

    def newton_apply(self, dt, nopts=None, sopts=None, ordering=ORDER_NATURAL):
        nopts = nopts or ewg.default_newton_opts()
        sopts = sopts or ewg.default_solve_opts()
        ni, li, e = C.c_int(), C.c_int(), C.c_double()
        rc = self.lib.orc_newton_apply(self.h, dt, C.byref(nopts), C.byref(sopts), ordering,
                                       C.byref(ni), C.byref(li), C.byref(e))
        return rc, ni.value, li.value, e.value

    def run(self, n_steps, dt, nopts=None, sopts=None, ordering=ORDER_NATURAL):
        """Fixed-step time loop; returns [(newton_iterations, linear_iterations)] per step."""
        out = []
        for _ in range(n_steps):
            rc, ni, li, e = self.newton_apply(dt, nopts, sopts, ordering)
            if rc:
                raise RuntimeError(f"oracle Newton failed ({rc}): {self.err()}")
            self.advance_time_level()
            out.append((ni, li))
        return out

    def residual_norm(self, x, dt):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 2)
        return self.lib.orc_residual_norm(self.h, _p(x), dt)

    def global_storage(self, t):
        out = np.zeros(2)
        self.lib.orc_global_storage(self.h, t, _p(out))
        return out

    def boundary_rates(self):
        out = np.zeros(2)
        self.lib.orc_boundary_rates(self.h, _p(out))
        return out


def material_eval(mat: "ewg.Material", sw: float) -> np.ndarray:
    """{pcnw, dpcnw/dSw, krw, dkrw/dSw, krn, dkrn/dSw} at absolute S_w through the AD type."""
    out = np.zeros(6)
    load().orc_material_eval(C.byref(mat), sw, _p(out))
    return out


class VcfvOracle:
    """CPU restatement of the vertex-centred (VCFV, P1 gradients) linearizer and Newton on one lens
    case whose permeability is given per vertex (VcfvCase)."""

    def __init__(self, case, nthreads: int = 1):
        self.lib = load()
        self.case = case
        perm = np.ascontiguousarray(case.perm, dtype=np.float64)
        self.h = self.lib.orc_vcfv_create(C.byref(case.grid), C.byref(case.problem), _p(perm), nthreads)
        self.n = self.lib.orc_vcfv_num_dofs(self.h)
        self.nnzb = self.lib.orc_vcfv_num_blocks(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_vcfv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def err(self):
        return self.lib.orc_vcfv_last_error(self.h).decode()

    def vec(self):
        return np.zeros((self.n, 2), dtype=np.float64)

    def set_solution(self, t, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 2)
        self.lib.orc_vcfv_set_solution(self.h, t, _p(x))

    def get_solution(self, t=0):
        x = self.vec()
        self.lib.orc_vcfv_get_solution(self.h, t, _p(x))
        return x

    def apply_initial_solution(self):
        self.lib.orc_vcfv_apply_initial_solution(self.h)

    def advance_time_level(self):
        self.lib.orc_vcfv_advance_time_level(self.h)

    def set_local_linearizer(self, kind: int, method: int = 1):
        self.lib.orc_vcfv_set_local_linearizer(self.h, kind, method)

    def update_begin(self):
        self.lib.orc_vcfv_update_begin(self.h)

    def total_volumes(self):
        v = np.zeros(self.n, dtype=np.float64)
        self.lib.orc_vcfv_total_volumes(self.h, _p(v))
        return v

    def linearize(self, dt, newton_iteration=0):
        e = C.c_double()
        if self.lib.orc_vcfv_linearize(self.h, dt, newton_iteration, C.byref(e)) != 0:
            raise RuntimeError(self.err())
        return e.value

    def residual(self):
        r = self.vec()
        self.lib.orc_vcfv_get_residual(self.h, _p(r))
        return r

    def jacobian_bcrs(self):
        rp = np.zeros(self.n + 1, dtype=np.int32)
        ci = np.zeros(self.nnzb, dtype=np.int32)
        b = np.zeros((self.nnzb, 2, 2), dtype=np.float64)
        self.lib.orc_vcfv_get_jacobian_bcrs(self.h, _p(rp, C.c_int32), _p(ci, C.c_int32), _p(b))
        return rp, ci, b

    def newton_apply(self, dt, nopts=None, sopts=None, ordering=ORDER_NATURAL):
        nopts = nopts or ewg.default_newton_opts()
        sopts = sopts or ewg.default_solve_opts()
        its, lin, err = C.c_int(), C.c_int(), C.c_double()
        st = self.lib.orc_vcfv_newton_apply(self.h, dt, C.byref(nopts), C.byref(sopts), ordering, C.byref(its),
                                            C.byref(lin), C.byref(err))
        return st, its.value, lin.value, err.value

    def global_storage(self, t=0):
        out = np.zeros(2)
        self.lib.orc_vcfv_global_storage(self.h, t, _p(out))
        return out

    def boundary_rates(self):
        out = np.zeros(2)
        self.lib.orc_vcfv_boundary_rates(self.h, _p(out))
        return out

    def geometry(self):
        ne = 4 if self.case.grid.dim == 2 else 12
        ij = np.zeros((ne, 2), dtype=np.int32)
        ip = np.zeros((ne, 3)); nrm = np.zeros((ne, 3)); area = np.zeros(ne)
        G = np.zeros((ne, 8, 3)); sv = C.c_double()
        self.lib.orc_vcfv_geometry(self.h, _p(ij, C.c_int32), _p(ip), _p(nrm), _p(area), _p(G), C.byref(sv))
        return {"ij": ij, "ip": ip, "nrm": nrm, "area": area, "G": G, "scv_volume": sv.value}
