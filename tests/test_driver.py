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
                          "--max-time-step-size=250", "--newton-target-iterations=18", f"--output={outf}",
                          f"--output-dir={tmp_path}"],
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


def _vtu_fields(path):
    import xml.etree.ElementTree as ET
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    fields = {a.get("Name"): np.array(a.text.split(), dtype=np.float64)
              for a in piece.find("CellData").findall("DataArray")}
    return piece, fields


def test_vtk_writer_layout(tmp_path):
    """The VTK writer on its own (host code, no device): point / cell counts, connectivity of a
    hexahedron, field lengths, and the collection file listing every step."""
    src = tmp_path / "vtk.cc"
    src.write_text(r'''
#include "vtkwriter.hh"
int main(int argc, char** argv) {
    ewg_grid g{}; g.dim = 3; g.nx = 3; g.ny = 2; g.nz = 2; g.lx = 3.0; g.ly = 1.0; g.lz = 2.0;
    ewg::VtkMultiWriter w(argv[1], "probe");
    for (int s = 0; s < 2; ++s) {
        std::vector<ewg::VtkMultiWriter::Field> f = {{"saturation_w", 1, {}}, {"intrinsicPerm", 9, {}}};
        for (int c = 0; c < 12; ++c) {
            f[0].values.push_back(c + 0.5 * s);
            for (int k = 0; k < 9; ++k) f[1].values.push_back(k % 4 == 0 ? 1e-12 * (c + 1) : 0.0);
        }
        w.write(250.0 * s, g, f);
    }
    return 0;
}
''')
    exe = tmp_path / "vtk"
    subprocess.check_call(["g++", "-std=c++17", "-I", os.path.join(ROOT, "ewoms-numerics_b200", "host"),
                           str(src), "-o", str(exe)])
    subprocess.check_call([str(exe), str(tmp_path)])
    piece, f = _vtu_fields(tmp_path / "probe-00001.vtu")
    assert piece.get("NumberOfPoints") == str(4 * 3 * 3) and piece.get("NumberOfCells") == "12"
    assert np.array_equal(f["saturation_w"], np.arange(12) + 0.5)
    assert f["intrinsicPerm"].shape == (108,) and f["intrinsicPerm"][9] == 2e-12
    conn = np.array(piece.find("Cells/DataArray[@Name='connectivity']").text.split(), dtype=np.int64)
    # first hexahedron: points (0,0,0) (1,0,0) (1,1,0) (0,1,0) and the same one layer up
    assert list(conn[:8]) == [0, 1, 5, 4, 12, 13, 17, 16]
    pvd = (tmp_path / "probe.pvd").read_text()
    assert 'timestep="0"' in pvd and 'timestep="250"' in pvd and "probe-00001.vtu" in pvd


@pytest.mark.gpu
def test_driver_vtk_output(driver, tmp_path):
    """VtkMultiWriter output of the driver: one .vtu per step plus the initial state, listed in the
    .pvd, with the final fields equal to the solution the driver writes."""
    outf = tmp_path / "x.bin"
    out = subprocess.run([driver, "--preset=baseline", "--end-time=500", "--initial-time-step-size=250",
                          "--max-time-step-size=250", f"--output={outf}", f"--output-dir={tmp_path}"],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    names = sorted(p.name for p in tmp_path.glob("lens_immiscible_ecfv_ad-*.vtu"))
    assert names == ["lens_immiscible_ecfv_ad-00000.vtu", "lens_immiscible_ecfv_ad-00001.vtu",
                     "lens_immiscible_ecfv_ad-00002.vtu"]
    piece, f = _vtu_fields(tmp_path / names[-1])
    x = np.fromfile(outf, dtype=np.float64).reshape(-1, 2)
    assert np.array_equal(f["pressure_w"], x[:, 0]) and np.array_equal(f["saturation_w"], x[:, 1])
    assert np.allclose(f["saturation_n"], 1.0 - x[:, 1])
    assert np.all(f["pressure_n"] >= f["pressure_w"])
    assert np.all((f["relativePerm_w"] >= 0) & (f["relativePerm_w"] <= 1))
    assert "lens_immiscible_ecfv_ad-00002.vtu" in (tmp_path / "lens_immiscible_ecfv_ad.pvd").read_text()


@pytest.mark.gpu
def test_driver_fd_linearizer_runs(driver, tmp_path):
    """LocalLinearizerSplice = FiniteDifferenceLocalLinearizer through the driver's parameters."""
    out = subprocess.run([driver, "--preset=baseline", "--end-time=500", "--initial-time-step-size=250",
                          "--max-time-step-size=250", "--local-linearizer=fd", "--numeric-difference-method=0",
                          "--enable-vtk-output=0"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert len([ln for ln in out.stdout.splitlines() if ln.startswith("Time step")]) == 2


def test_driver_rejects_unknown_discretization(driver):
    out = subprocess.run([driver, "--discretization=box"], capture_output=True, text=True)
    assert out.returncode == 2 and "Discretization" in out.stderr


@pytest.mark.gpu
def test_driver_vcfv_runs_and_matches_oracle(driver, tmp_path, oracle_mod, ewg_mod):
    """lens_immiscible_vcfv_ad through the driver: two steps of the baseline preset on the vertex
    grid with block Jacobi; the final state equals the oracle's VCFV Newton run to the solver
    tolerance's effect, and the VTK output carries the vertex fields as point data."""
    outf = tmp_path / "x.bin"
    out = subprocess.run([driver, "--discretization=vcfv", "--preconditioner=jacobi", "--preset=baseline",
                          "--cells-x=24", "--cells-y=16", "--end-time=500", "--initial-time-step-size=250",
                          "--max-time-step-size=250", f"--output={outf}", f"--output-dir={tmp_path}"],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    x = np.fromfile(outf, dtype=np.float64).reshape(-1, 2)
    case = ewg_mod.vcfv_case(ewg_mod.baseline_case(24, 16))
    o = oracle_mod.VcfvOracle(case)
    o.apply_initial_solution()
    so = ewg_mod.default_solve_opts(precond=ewg_mod.PRECOND_JACOBI)
    for _ in range(2):
        st, its, lin, err = o.newton_apply(250.0, None, so)
        assert st == 0
        o.advance_time_level()
    xo = o.get_solution(0)
    assert np.max(np.abs(x[:, 0] - xo[:, 0])) <= 1e-8 * np.max(np.abs(xo[:, 0]))
    assert np.max(np.abs(x[:, 1] - xo[:, 1])) <= 1e-8
    vtu = (tmp_path / "lens_immiscible_vcfv_ad-00002.vtu").read_text()
    assert "<PointData>" in vtu and 'Name="saturation_n"' in vtu


@pytest.mark.gpu
def test_driver_vcfv_fd_runs(driver, tmp_path):
    """lens_immiscible_vcfv_fd through the driver: the finite-difference local linearizer on the
    vertex-centred stencil, two steps, VTK output under the finite-difference name."""
    out = subprocess.run([driver, "--discretization=vcfv", "--preconditioner=jacobi", "--preset=baseline",
                          "--cells-x=24", "--cells-y=16", "--end-time=500", "--initial-time-step-size=250",
                          "--max-time-step-size=250", "--local-linearizer=fd", f"--output-dir={tmp_path}"],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert len([ln for ln in out.stdout.splitlines() if ln.startswith("Time step")]) == 2
    assert (tmp_path / "lens_immiscible_vcfv-00002.vtu").exists()
