"""The GPU drop-in headers (host/gpuecfvlinearizer.hh, host/gpubicgstabbackend.hh,
host/gpusparsematrixadapter.hh) compiled with g++ against stand-ins of the eWoms property system
(tests/dropin/ewoms/common/) and driven by NewtonMethod::apply's call sequence
(tests/dropin/newton_dropin.cc).

CPU: the headers and the test program compile (-Wall -Wextra -Werror) and link against libewg.so.
GPU: per mode, two implicit steps of a 16 x 12 x 8 lens through the drop-in sequence give the same
Newton iteration counts and the same fields bit for bit as ewg_newton_apply; with
GpuSparseMatrixAdapter the Jacobian never crosses PCIe and each Newton iteration moves exactly
solution(0) to the device and the residual and the update back (3 x N x 16 bytes; the first
iteration of a step also uploads solution(1)); a host consumer's block reads export the matrix once
and its block change is uploaded by setMatrix and solved.
"""
import os
import subprocess

import pytest

from conftest import PKG, ROOT

SRC = os.path.join(ROOT, "tests", "dropin", "newton_dropin.cc")
CELLS = 16 * 12 * 8


def _compile(out_dir):
    exe = os.path.join(str(out_dir), "newton_dropin")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "tests", "dropin"), "-I", os.path.join(PKG, "host"),
           "-o", exe, SRC, "-L", PKG, "-lewg", f"-Wl,-rpath,{PKG}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_dropin_headers_compile(tmp_path):
    if not os.path.exists(os.path.join(PKG, "libewg.so")):
        import build
        build.build()
    _compile(tmp_path)


def _run(exe, mode):
    r = subprocess.run([exe, mode], capture_output=True, text=True, timeout=300)
    out = r.stdout
    assert r.returncode == 0 and out.strip().endswith("OK"), out[-4000:] + r.stderr[-2000:]
    vals = {}
    for line in out.splitlines():
        parts = line.split()
        if len(parts) == 2:
            vals[parts[0]] = parts[1]
    return vals


@pytest.mark.gpu
def test_dropin_newton_keeps_jacobian_on_device(tmp_path):
    exe = _compile(tmp_path)
    v = _run(exe, "device")
    assert int(v["device_matrix_exports"]) == 0 and int(v["device_matrix_uploads"]) == 0
    n16 = CELLS * 16
    for step in (0, 1):
        assert float(v[f"device_step{step}_max_field_difference"]) == 0.0
        k = 0
        while f"device_step{step}_it{k}_h2d_bytes" in v:
            h2d = int(v[f"device_step{step}_it{k}_h2d_bytes"])
            d2h = int(v[f"device_step{step}_it{k}_d2h_bytes"])
            assert h2d == (2 if k == 0 else 1) * n16 and d2h == 2 * n16, (step, k, h2d, d2h)
            k += 1
        assert k >= 2


@pytest.mark.gpu
def test_dropin_newton_with_host_matrix_adapter(tmp_path):
    """An IstlSparseMatrixAdapter-like SparseMatrixAdapter: same results, the matrix crosses twice
    per iteration (export by jacobian(), upload by setMatrix)."""
    exe = _compile(tmp_path)
    v = _run(exe, "istl")
    n16 = CELLS * 16
    for step in (0, 1):
        assert float(v[f"istl_step{step}_max_field_difference"]) == 0.0
        d2h = int(v[f"istl_step{step}_it1_d2h_bytes"])
        assert d2h > 2 * n16 + 32 * CELLS  # the blocks came back to the host


@pytest.mark.gpu
def test_dropin_host_consumer_reads_and_changes_blocks(tmp_path):
    exe = _compile(tmp_path)
    v = _run(exe, "host")
    assert int(v["host_consumer_matrix_exports"]) == 1
    assert int(v["host_consumer_matrix_uploads"]) == 1
    assert float(v["host_consumer_max_update_difference"]) == 0.0
