"""Restart files in the reference's format (io/restart.hh:36-271, Simulator::serialize /
deserialize utils/simulator.hh:923-979, EcfvDiscretization::serialize ecfvdiscretization.hh:186-202).

CPU: the Python writer and the C++ header (host/restart.hh) write byte-identical files for the same
state, each reads the other's back to the bit, the file name and magic cookie follow the reference,
and reading rejects a missing or empty file, a file of another grid and a section with extra
values. GPU: a run checkpointed after 5 of 10 implicit steps and resumed from the file (Python API
and the C++ driver with RestartTime) ends bit-identical to the uninterrupted run, and the driver's
VTK collection lists every step after the resumed run.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

import ewg


def _state(n, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = np.empty((n, 2))
    x[:, 0] = 1e5 + rng.normal(0, 3e4, n)
    x[:, 1] = rng.uniform(0, 1, n)
    x[0] = [1e5 / 3.0, 1.0 - 1e-17]     # values that need all 17 significant digits
    x[1] = [5e-324, -0.0]               # a subnormal and a negative zero
    return x


def test_file_name_and_cookie():
    g = ewg.Grid(dim=3, nx=4, ny=3, nz=2, lx=6.0, ly=4.0, lz=3.0)
    assert ewg.restart_file_name(".", "lens_immiscible_ecfv_ad", 1250.0) == "lens_immiscible_ecfv_ad_time=1250_rank=0.ers"
    assert ewg.restart_file_name("out", "s", 2.5e6, 3) == "out/s_time=2.5e+06_rank=3.ers"
    # 24 elements; edges 4*4*3 + 5*3*3 + 5*4*2 = 48 + 45 + 40; 5*4*3 vertices
    assert ewg.restart_cookie(g) == ("eWoms restart file: gridName='blubb' numCPUs=1 myRank=0 numElements=24 "
                                     "numEdges=133 numVertices=60")
    g2 = ewg.Grid(dim=2, nx=48, ny=32, nz=1, lx=6.0, ly=4.0, lz=1.0)
    assert ewg.restart_grid_counts(g2) == (1536, 48 * 33 + 49 * 32, 49 * 33)


def test_python_round_trip_and_errors(tmp_path):
    g = ewg.Grid(dim=3, nx=4, ny=3, nz=2, lx=6.0, ly=4.0, lz=3.0)
    x = _state(g.n_cells)
    sim = ewg.SimulatorState(episode_idx=2, episode_start_time=0.0, episode_length=1e100, start_time=0.0,
                             time=1250.0, time_step_idx=5)
    path = ewg.write_restart(str(tmp_path), "lens", g, x, sim)
    sim2, x2, _ = ewg.read_restart(str(tmp_path), "lens", 1250.0, g)
    assert sim2 == sim
    assert np.array_equal(x2.view(np.uint64), x.view(np.uint64))
    text = open(path).read().splitlines()
    # cookie, end; Simulator, values (ending the section); cells; end
    assert text[1] == "" and text[2] == "Simulator" and text[4] == "Entities: Codim 0" and text[-1] == ""
    # errors the reference raises
    with pytest.raises(RuntimeError, match="could not be opened"):
        ewg.read_restart(str(tmp_path), "lens", 999.0, g)
    open(ewg.restart_file_name(str(tmp_path), "empty", 1.0), "w").close()
    with pytest.raises(RuntimeError, match="is empty"):
        ewg.read_restart(str(tmp_path), "empty", 1.0, g)
    other = ewg.Grid(dim=3, nx=4, ny=3, nz=3, lx=6.0, ly=4.0, lz=3.0)
    with pytest.raises(RuntimeError, match="Could not start section"):
        ewg.read_restart(str(tmp_path), "lens", 1250.0, other)
    lines = open(path).read().split("\n")
    lines[3] = lines[3] + " 7.0"  # a seventh value in the Simulator section
    open(path, "w").write("\n".join(lines))
    with pytest.raises(RuntimeError, match="unread values"):
        ewg.read_restart(str(tmp_path), "lens", 1250.0, g)


CPP = r'''
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>
#include "restart.hh"
// usage: restart_io write <dir> <name> <x.bin> | read <dir> <name> <time> <x.bin>
int main(int argc, char** argv) {
    ewg_grid g{}; g.dim = 3; g.nx = 4; g.ny = 3; g.nz = 2; g.lx = 6.0; g.ly = 4.0; g.lz = 3.0;
    const int64_t n = 24;
    std::vector<double> x(2 * n);
    std::string mode = argv[1];
    try {
        if (mode == "write") {
            std::ifstream f(argv[4], std::ios::binary);
            f.read(reinterpret_cast<char*>(x.data()), sizeof(double) * x.size());
            ewg::SimulatorState s; s.episodeIdx = 2; s.time = 1250.0; s.timeStepIdx = 5;
            ewg::Restart r;
            r.serializeBegin(argv[2], argv[3], s.time, g);
            r.serializeSimulator(s);
            r.serializeCells(x.data(), n);
            r.serializeEnd();
        } else {
            ewg::Restart r;
            r.deserializeBegin(argv[2], argv[3], std::stod(argv[4]), g);
            ewg::SimulatorState s;
            r.deserializeSimulator(s);
            r.deserializeCells(x.data(), n);
            r.deserializeEnd();
            std::ofstream f(argv[5], std::ios::binary);
            f.write(reinterpret_cast<const char*>(x.data()), sizeof(double) * x.size());
            std::printf("%d %.17g %d\n", s.episodeIdx, s.time, s.timeStepIdx);
        }
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
        return 3;
    }
    return 0;
}
'''


def test_cpp_header_matches_python(tmp_path):
    src = tmp_path / "restart_io.cc"
    src.write_text(CPP)
    exe = tmp_path / "restart_io"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(PKG, "host"), "-o", str(exe),
                        str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    g = ewg.Grid(dim=3, nx=4, ny=3, nz=2, lx=6.0, ly=4.0, lz=3.0)
    x = _state(g.n_cells, seed=4)
    xb = tmp_path / "x.bin"
    x.tofile(xb)
    # the C++ writer and the Python writer produce the same bytes
    (tmp_path / "cpp").mkdir()
    (tmp_path / "py").mkdir()
    r = subprocess.run([str(exe), "write", str(tmp_path / "cpp"), "lens", str(xb)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    sim = ewg.SimulatorState(episode_idx=2, time=1250.0, time_step_idx=5)
    pp = ewg.write_restart(str(tmp_path / "py"), "lens", g, x, sim)
    cp = ewg.restart_file_name(str(tmp_path / "cpp"), "lens", 1250.0)
    assert open(cp, "rb").read() == open(pp, "rb").read()
    # each reads the other's file back to the bit
    _, xpy, _ = ewg.read_restart(str(tmp_path / "cpp"), "lens", 1250.0, g)
    assert np.array_equal(xpy.view(np.uint64), x.view(np.uint64))
    out = tmp_path / "back.bin"
    r = subprocess.run([str(exe), "read", str(tmp_path / "py"), "lens", "1250", str(out)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.split() == ["2", "1250", "5"], r.stdout
    assert np.array_equal(np.fromfile(out, dtype=np.uint64), x.view(np.uint64).ravel())
    # a short entity section is an error of the C++ reader too
    txt = open(pp).read().split("\n")
    open(pp, "w").write("\n".join(txt[:10]) + "\n")
    r = subprocess.run([str(exe), "read", str(tmp_path / "py"), "lens", "1250", str(out)], capture_output=True, text=True)
    assert r.returncode == 3 and "error" in r.stdout


@pytest.mark.gpu
def test_restarted_run_is_bit_identical(tmp_path):
    case = ewg.lens3d_case(16, 16, 8, seed=3, corr_cells=4.0)
    full = ewg.Context(case)
    full.apply_initial_solution()
    full.run(10, 250.0)
    x_full = full.get_solution(0)
    first = ewg.Context(case)
    first.apply_initial_solution()
    first.run(5, 250.0)
    first.save_restart(str(tmp_path), "lens3d", ewg.SimulatorState(time=1250.0, time_step_idx=5))
    first.close()
    resumed = ewg.Context(case)
    sim = resumed.load_restart(str(tmp_path), "lens3d", 1250.0)
    assert sim.time_step_idx == 5 and sim.time == 1250.0
    resumed.run(5, 250.0)
    assert np.array_equal(resumed.get_solution(0).view(np.uint64), x_full.view(np.uint64))
    full.close()
    resumed.close()


@pytest.mark.gpu
def test_driver_restart_is_bit_identical(tmp_path):
    driver = os.path.join(PKG, "lens_gpu")
    args = ["--preset=baseline", "--end-time=2500", "--initial-time-step-size=250", "--max-time-step-size=250",
            "--newton-target-iterations=18", "--restart-file-interval=5"]
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    r = subprocess.run([driver] + args + [f"--output={a / 'x.bin'}", f"--output-dir={a}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert (a / "lens_immiscible_ecfv_ad_time=1250_rank=0.ers").exists()
    assert (a / "lens_immiscible_ecfv_ad_time=2500_rank=0.ers").exists()
    # resume from the step-5 file of run a in directory b
    (b / "lens_immiscible_ecfv_ad_time=1250_rank=0.ers").write_bytes(
        (a / "lens_immiscible_ecfv_ad_time=1250_rank=0.ers").read_bytes())
    for k in range(6):
        (b / f"lens_immiscible_ecfv_ad-{k:05d}.vtu").write_bytes((a / f"lens_immiscible_ecfv_ad-{k:05d}.vtu").read_bytes())
    r = subprocess.run([driver] + args + ["--restart-time=1250", f"--output={b / 'x.bin'}", f"--output-dir={b}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    steps = [ln for ln in r.stdout.splitlines() if ln.startswith("Time step")]
    assert len(steps) == 5 and steps[0].startswith("Time step 6 ")
    assert (a / "x.bin").read_bytes() == (b / "x.bin").read_bytes()
    # the collection of the resumed run lists all eleven outputs, like the uninterrupted one
    assert (b / "lens_immiscible_ecfv_ad.pvd").read_text() == (a / "lens_immiscible_ecfv_ad.pvd").read_text()
