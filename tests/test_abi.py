"""CPU checks of the C-ABI library: it loads, exports every entry point include/ewg.h declares,
its structs have the C layout, and it fails loudly (no CPU fallback) without a device."""
import ctypes as C
import os
import re
import subprocess
import sys

import pytest

from conftest import ROOT, PKG

HEADER = os.path.join(ROOT, "include", "ewg.h")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ewg_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    import ewg
    if not os.path.exists(ewg.LIB_PATH):
        sys.path.insert(0, PKG)
        import build
        build.build()
    return ewg.load()


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version(lib):
    assert lib.ewg_abi_version() == 1


def test_struct_layout_matches_c(tmp_path):
    """sizeof/offsetof of the ABI structs from a C compiler equal the ctypes mirrors."""
    import ewg
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ewg.h"\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
                   'sizeof(ewg_grid),sizeof(ewg_material),sizeof(ewg_problem),sizeof(ewg_solve_opts),'
                   'sizeof(ewg_solve_report),sizeof(ewg_lin_report),sizeof(ewg_newton_opts),'
                   'sizeof(ewg_newton_report),offsetof(ewg_problem,lens),offsetof(ewg_solve_opts,restart_on_breakdown));'
                   'printf("%zu %zu %zu %zu\\n",sizeof(ewg_ensemble_opts),sizeof(ewg_ensemble_report),'
                   'sizeof(ewg_ensemble_stats),offsetof(ewg_ensemble_stats,t_linearize));}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = [int(v) for v in subprocess.check_output([str(exe)]).split()]
    want = [C.sizeof(ewg.Grid), C.sizeof(ewg.Material), C.sizeof(ewg.Problem), C.sizeof(ewg.SolveOpts),
            C.sizeof(ewg.SolveReport), C.sizeof(ewg.LinReport), C.sizeof(ewg.NewtonOpts),
            C.sizeof(ewg.NewtonReport), ewg.Problem.lens.offset, ewg.SolveOpts.restart_on_breakdown.offset,
            C.sizeof(ewg.EnsembleOpts), C.sizeof(ewg.EnsembleReport), C.sizeof(ewg.EnsembleStats),
            ewg.EnsembleStats.t_linearize.offset]
    assert got == want


def test_create_without_device_fails_loudly(lib):
    """On a machine without a usable B200 ewg_create reports EWG_ERR_NO_DEVICE instead of
    falling back to the CPU."""
    import ewg
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    case = ewg.baseline_case()
    with pytest.raises(ewg.EwgError) as ei:
        ewg.Context(case)
    assert ei.value.status == 7


def test_invalid_grid_rejected(lib):
    import ewg
    case = ewg.baseline_case(nx=47, ny=32)
    with pytest.raises(ewg.EwgError) as ei:
        ewg.Context(case)
    assert ei.value.status in (1, 7)


def test_ensemble_without_device_or_bad_grid_fails_loudly(lib):
    """Ensembles take 3D grids with even nx and a device; anything else is an error status."""
    import ewg
    import torch
    bad = ewg.lens3d_case(7, 4, 4, seed=0)
    with pytest.raises(ewg.EwgError) as ei:
        ewg.Ensemble([bad])
    assert ei.value.status == 1
    if not torch.cuda.is_available():
        with pytest.raises(ewg.EwgError) as ei:
            ewg.Ensemble([ewg.lens3d_case(8, 4, 4, seed=0)])
        assert ei.value.status == 7


def test_vcfv_bad_arguments_and_no_device_fail_loudly(lib):
    """The vertex-centred context rejects an empty grid with EWG_ERR_INVALID before touching a
    device and, without a usable B200, reports EWG_ERR_NO_DEVICE instead of running on the CPU;
    its calls reject a null context."""
    import ctypes as C
    import ewg
    import torch
    case = ewg.vcfv_case(ewg.baseline_case(4, 4))
    case.grid.nx = 0
    with pytest.raises(ewg.EwgError) as ei:
        ewg.VcfvContext(case)
    assert ei.value.status == 1
    e = C.c_double()
    assert lib.ewg_vcfv_linearize(None, 250.0, C.byref(e)) == 1
    assert lib.ewg_vcfv_set_local_linearizer(None, 1, 1) == 1
    if not torch.cuda.is_available():
        with pytest.raises(ewg.EwgError) as ei:
            ewg.VcfvContext(ewg.vcfv_case(ewg.baseline_case(4, 4)))
        assert ei.value.status == 7


def test_device_vector_calls_reject_bad_arguments(lib):
    """The device-order vector calls reject a null context, an unknown buffer and null vectors
    with EWG_ERR_INVALID before touching a device."""
    import ctypes as C
    import ewg
    p = C.c_void_p()
    assert lib.ewg_device_buffer(None, ewg.BUFFER_SOLUTION, C.byref(p)) == 1
    assert lib.ewg_device_spmv(None, None, None) == 1
    opts = ewg.default_solve_opts()
    assert lib.ewg_device_precondition(None, C.byref(opts), None, None) == 1
