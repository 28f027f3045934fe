"""The C++ host driver (ewoms-numerics_b200/lens_gpu) over the C ABI: parameter handling on CPU,
and the 10-step lens simulation on the GPU against the oracle's golden run."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_close

DRIVER = os.path.join(ROOT, "ewoms-numerics_b200", "lens_gpu")


@pytest.fixture(scope="module")
def driver():
    if not os.path.exists(DRIVER):
        import build
        build.build()
    return DRIVER


def test_unknown_parameter_rejected(driver):
    out = subprocess.run([driver, "--no-such-parameter=1"], capture_output=True, text=True)
    assert out.returncode == 1 and "unknown parameter" in out.stderr


def test_duplicate_parameter_rejected(driver, tmp_path):
    ini = tmp_path / "p.ini"
    ini.write_text("EndTime = 500\n")
    out = subprocess.run([driver, f"--parameter-file={ini}", "--end-time=250"], capture_output=True, text=True)
    assert out.returncode == 1 and "given twice" in out.stderr


def test_missing_parameter_file_rejected(driver, tmp_path):
    out = subprocess.run([driver, f"--parameter-file={tmp_path / 'none.ini'}"], capture_output=True, text=True)
    assert out.returncode == 1 and "does not exist" in out.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("preset", ["baseline", "reference"])
def test_driver_ten_steps_match_oracle(driver, tmp_path, preset):
    gold = np.load(os.path.join(ROOT, "tests", "golden", "lens2d_golden.npz"))
    outf = tmp_path / "x.bin"
    # the golden run uses a fixed dt = 250 s; with NewtonTargetIterations = 18 the reference's
    # suggestTimeStepSize never shrinks the step below MaxTimeStepSize (newtonmethod.hh:527-544)
    out = subprocess.run([driver, f"--preset={preset}", "--end-time=2500", "--initial-time-step-size=250",
                          "--max-time-step-size=250", "--newton-target-iterations=18", f"--output={outf}"],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    steps = [ln for ln in out.stdout.splitlines() if ln.startswith("Time step")]
    assert len(steps) == 10
    its = [int(ln.split("Newton iterations")[1].split(",")[0]) for ln in steps]
    assert its == list(gold[f"{preset}_run10_steps"][:, 0])
    x = np.fromfile(outf, dtype=np.float64).reshape(-1, 2)
    xo = gold[f"{preset}_run10_x"]
    assert rel_close(x[:, 0], xo[:, 0], 1e-8)[0]
    assert np.max(np.abs(x[:, 1] - xo[:, 1])) <= 1e-8
