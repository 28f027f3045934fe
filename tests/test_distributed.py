"""The N > 1 path of bench.py on CPU: two ranks over gloo (the GPU runs use NCCL with the same
calls). Each rank takes its own permeability realization of the single problem (weak scaling) and
its cost-balanced share of one ensemble (shard.py), with no data-path collective; timings are
combined as the max over ranks and work as the sum. The reference arm runs on rank 0 alone."""
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
# the units of each rank: its own realization of the 3D lens problem (weak scaling) ...
case = ewg.lens3d_case(8, 6, 4, seed=rank)
mine = float(np.sum(case.perm))  # the log field has zero mean, its exponential does not
import torch
t = torch.tensor([mine, -mine], dtype=torch.float64)
pg.all_reduce(t, op=pg.ReduceOp.MAX)
assert t[0].item() != -t[1].item(), "the ranks drew the same realizations"
# ... and its share of one ensemble that every rank draws identically (sharded by cost)
cases, dts = bench.ensemble_cases(ewg, 3, seed=3)
ens = float(sum(float(np.sum(np.log(c.perm))) for c in cases)) + sum(dts)
t = torch.tensor([ens, -ens], dtype=torch.float64)
pg.all_reduce(t, op=pg.ReduceOp.MAX)
assert t[0].item() == -t[1].item(), "the ranks drew different ensembles"
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


def test_member_assignment_is_balanced_and_complete():
    """Greedy cost balance over the 64-member bench ensemble: every member on exactly one rank,
    the same assignment on every call, and the heaviest rank within the mean plus one member."""
    sys.path.insert(0, os.path.join(ROOT, "ewoms-numerics_b200"))
    import numpy as np
    import bench
    import ewg
    import shard
    rng = np.random.default_rng(3)
    sizes = rng.choice([32, 48, 64, 96, 128], size=64)
    dts = [float(rng.choice([100.0, 250.0, 500.0])) for _ in range(64)]
    costs = [shard.member_cost(int(n) ** 3, dt) for n, dt in zip(sizes, dts)]
    for world in (1, 2, 4, 8):
        members = shard.assign_members(costs, world)
        assert sorted(m for ms in members for m in ms) == list(range(64))
        assert members == shard.assign_members(costs, world)
        loads = shard.rank_loads(costs, members)
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-6 * sum(costs)
    assert shard.imbalance(costs, shard.assign_members(costs, 2)) < 1.02
    # the bench draws its member list through the same generator
    cases, bdts = bench.ensemble_cases(ewg, 4, seed=3)
    assert len(cases) == 4 and len(bdts) == 4


SHARD_PROBE = r'''
import os, sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, os.path.join(sys.argv[1], "ewoms-numerics_b200"))
sys.path.insert(0, os.path.join(sys.argv[1], "oracle"))
import numpy as np
import torch.distributed as dist
import bench, ewg, oracle, shard
rank, world, local, pg = bench.dist_init(None)
# one ensemble of small members, the same list on both ranks; each rank advances its own members
# (the oracle stands in for the device ensemble on CPU) and rank 0 gathers reports and fields
cases, dts = bench.ensemble_cases(ewg, 5, seed=11, sizes=(4, 6, 8))
costs = [shard.member_cost(c.n_cells, dt) for c, dt in zip(cases, dts)]
members = shard.assign_members(costs, world)
mine = {}
for m in members[rank]:
    o = oracle.Oracle(cases[m])
    o.apply_initial_solution()
    its = o.run(1, dts[m], sopts=ewg.default_solve_opts(linear_solver_tolerance=1e-8))
    mine[m] = {"rank": rank, "newton": its[0][0], "x": o.get_solution(0)}
got = shard.gather_results(dist, rank, world, mine)
if rank == 0:
    assert sorted(got) == list(range(5)), sorted(got)
    assert {got[m]["rank"] for m in got} == {0, 1}
    for m in range(5):
        o = oracle.Oracle(cases[m])
        o.apply_initial_solution()
        its = o.run(1, dts[m], sopts=ewg.default_solve_opts(linear_solver_tolerance=1e-8))
        assert its[0][0] == got[m]["newton"]
        assert np.array_equal(o.get_solution(0), got[m]["x"])
bench.barrier(pg)
pg.destroy_process_group()
print(f"rank {rank} ok", flush=True)
'''


def test_sharded_ensemble_gathers_every_member_gloo(tmp_path):
    """Two gloo ranks split one ensemble by cost, advance their members and gather: rank 0 holds
    every member once, with the same Newton counts and bit-identical fields as a single process."""
    probe = tmp_path / "shard_probe.py"
    probe.write_text(SHARD_PROBE)
    out = _torchrun([str(probe), ROOT])
    assert out.returncode == 0, out.stdout + out.stderr
    assert "rank 0 ok" in out.stdout and "rank 1 ok" in out.stdout
