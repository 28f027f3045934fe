"""The N > 1 path of bench.py on CPU: two ranks over gloo (the GPU runs use NCCL with the same
calls). Each rank takes its own permeability realization and its own ensemble (weak scaling, no
data-path collective); timings are combined as the max over ranks and work as the sum. The
reference arm runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

PROBE = r'''
import os, sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, os.path.join(sys.argv[1], "ewoms-numerics_b200"))
import numpy as np
import bench, ewg
rank, world, local, pg = bench.dist_init(None)
assert world == 2 and pg is not None
assert bench.max_over_ranks(pg, float(rank) * 3.0) == 3.0
assert bench.sum_over_ranks(pg, 1.5) == 3.0
bench.barrier(pg)
# the units of each rank: its own realization of the 3D lens problem and its own ensemble
case = ewg.lens3d_case(8, 6, 4, seed=rank)
cases, dts = bench.ensemble_cases(ewg, 3, seed=3 + rank)
mine = float(np.sum(np.log(case.perm))) + sum(float(np.sum(np.log(c.perm))) for c in cases)
import torch
t = torch.tensor([mine, -mine], dtype=torch.float64)
pg.all_reduce(t, op=pg.ReduceOp.MAX)
assert t[0].item() != -t[1].item(), "the ranks drew the same realizations"
bench.barrier(pg)
pg.destroy_process_group()
print(f"rank {rank} ok", flush=True)
'''


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, timeout=240):
    cmd = ["timeout", "-k", "30", str(timeout), sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node=2", "--master-addr=127.0.0.1", f"--master-port={_free_port()}"] + args
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    return subprocess.run(cmd, capture_output=True, text=True, cwd=ROOT, env=env)


def test_two_rank_plumbing_gloo(tmp_path):
    probe = tmp_path / "probe.py"
    probe.write_text(PROBE)
    out = _torchrun([str(probe), ROOT])
    assert out.returncode == 0, out.stdout + out.stderr
    assert "rank 0 ok" in out.stdout and "rank 1 ok" in out.stdout


def test_reference_arm_runs_on_rank_zero_only():
    out = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"], timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["cpu_baseline"]["kind"] == "port" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
