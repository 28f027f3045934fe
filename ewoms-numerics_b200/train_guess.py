"""Train the learned Newton initial-guess network on states the simulator itself generates.

Data: 3D lens realizations (seeded log-normal permeability, sigma 0.5-1.5, correlation length
4-12 cells, dt drawn from {100, 250, 500} s) stepped with the GPU path; every converged step
solution(1) -> solution(0) is recorded on the device as one sample. Seeds 1000+ train, seeds
2000+ are held out. Training: Adam on whole volumes with the device forward / backward kernels.
Evaluation: Newton iterations per step with and without the guess on held-out realizations.

    python ewoms-numerics_b200/train_guess.py [--n 48] [--members 24] [--steps 12] [--iters 3000]
        [--out ewoms-numerics_b200/data/guess_net_lens3d.npz] [--report out.json]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ewg  # noqa: E402

DT_CHOICES = (100.0, 250.0, 500.0)


def mixed_opts():
    return ewg.default_solve_opts(precision=ewg.PRECISION_MIXED, linear_solver_tolerance=1e-3,
                                  inner_tolerance=1e-3, max_defect_iterations=3)


SHAPE = None  # (nx, ny, nz): train on the 3D lens problem at this size (sigma 1, length 8, dt 250)


def member(seed: int, n: int):
    if SHAPE is not None:
        # the benchmark's problem family: same grid, field statistics and step size, other seeds
        return ewg.lens3d_case(*SHAPE, seed=seed), 250.0
    rng = np.random.default_rng(seed)
    sigma = float(rng.uniform(0.5, 1.5))
    corr = float(rng.uniform(4.0, 12.0))
    dt = float(rng.choice(DT_CHOICES))
    case = ewg.lens3d_case(n, n, n, seed=seed, sigma=sigma, corr_cells=corr)
    return case, dt


def step(ctx, dt, sopts, net=None):
    """One implicit step with the reference's halving retry; returns (report, dt used, used guess)."""
    h, used = dt, None
    for _ in range(8):
        if net is not None:
            used, _, _ = net.predict_guess(ctx, h)
        st, rep = ctx.newton_apply(h, None, sopts)
        if st == ewg.EWG_OK:
            return rep, h, used
        ctx.restore_time_level()
        h /= 2
    raise RuntimeError("time step failed")


def generate(net, seeds, n, steps, sopts, log):
    counts = []
    for s in seeds:
        case, dt = member(s, n)
        ctx = ewg.Context(case)
        ctx.apply_initial_solution()
        for k in range(steps):
            rep, h, _ = step(ctx, dt, sopts)
            net.record(ctx, h)
            ctx.advance_time_level()
        counts.append(net.n_samples)
        ctx.close()
        log(f"member {s}: {net.n_samples} samples")
    return counts


def estimate_scales(n, sopts):
    """Output scales from two steps of one training member: the std of dp_w and dS_n."""
    case, dt = member(999, n)
    ctx = ewg.Context(case)
    ctx.apply_initial_solution()
    dps, dss = [], []
    for _ in range(3):
        rep, h, _ = step(ctx, dt, sopts)
        x1, x0 = ctx.get_solution(1), ctx.get_solution(0)
        dps.append(x0[:, 0] - x1[:, 0])
        dss.append(x1[:, 1] - x0[:, 1])
        ctx.advance_time_level()
    dp = np.concatenate(dps)
    ds = np.concatenate(dss)
    return max(float(np.std(dp)), 1.0), max(float(np.max(np.abs(ds))) / 4, 1e-3)


def evaluate(net, seeds, n, steps, sopts):
    """Newton iterations per step with and without the learned guess, same member and steps."""
    out = []
    for s in seeds:
        case, dt = member(s, n)
        res = {}
        for mode in ("previous", "learned"):
            ctx = ewg.Context(case)
            ctx.apply_initial_solution()
            its, lins, used, t0 = [], [], [], time.perf_counter()
            for k in range(steps):
                rep, h, u = step(ctx, dt, sopts, net if mode == "learned" else None)
                its.append(rep.iterations)
                lins.append(rep.linear_iterations)
                used.append(u)
                ctx.advance_time_level()
            res[mode] = {"newton": its, "linear": lins, "used_guess": used, "seconds": time.perf_counter() - t0}
            ctx.close()
        out.append({"seed": s, "dt": dt, **res})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--members", type=int, default=24)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-members", type=int, default=3)
    ap.add_argument("--out", default=os.path.join(HERE, "data", "guess_net_lens3d.npz"))
    ap.add_argument("--report", default=None)
    ap.add_argument("--loss-weight-p", type=float, default=0.05)
    ap.add_argument("--sn-threshold", type=float, default=0.002)
    ap.add_argument("--front-weight", type=float, default=20.0)
    ap.add_argument("--shape", default=None, help="nx,ny,nz of the lens problem to train on instead of cubes")
    ap.add_argument("--train-seeds", default=None, help="first,count of the training realizations")
    ap.add_argument("--hold-seeds", default=None, help="first,count of the held-out realizations")
    ap.add_argument("--apply-pressure", type=int, default=0)
    args = ap.parse_args()
    global SHAPE
    if args.shape:
        SHAPE = tuple(int(v) for v in args.shape.split(","))
    t0 = time.perf_counter()

    def log(msg):
        print(f"[{time.perf_counter() - t0:7.1f}s] {msg}", flush=True)

    sopts = mixed_opts()
    net = ewg.GuessNet(seed=0)
    options = [args.loss_weight_p, args.front_weight, float(args.apply_pressure), args.sn_threshold]
    net.set_options(options[0], options[1], bool(args.apply_pressure), options[3])
    tp, ts = estimate_scales(args.n, sopts)
    sc = net.scales()
    sc[6], sc[7] = tp, ts
    net.set_scales(sc)
    log(f"output scales dp {tp:.3g} Pa, dSn {ts:.3g}")
    train_seeds = list(range(1000, 1000 + args.members))
    hold_seeds = list(range(2000, 2000 + max(2, args.members // 6)))
    if args.train_seeds:
        a, b = (int(v) for v in args.train_seeds.split(","))
        train_seeds = list(range(a, a + b))
    if args.hold_seeds:
        a, b = (int(v) for v in args.hold_seeds.split(","))
        hold_seeds = list(range(a, a + b))
    generate(net, train_seeds, args.n, args.steps, sopts, log)
    n_train = net.n_samples
    generate(net, hold_seeds, args.n, args.steps, sopts, log)
    train_idx = np.arange(n_train)
    hold_idx = np.arange(n_train, net.n_samples)
    rng = np.random.default_rng(0)
    hist = []
    l_tr0, l_ho0 = net.eval_samples(train_idx), net.eval_samples(hold_idx)
    log(f"initial loss train {l_tr0:.4g} held-out {l_ho0:.4g}")
    chunk = 250
    for it in range(0, args.iters, chunk):
        lr = args.lr * (0.3 if it > 0.7 * args.iters else 1.0)
        idx = rng.choice(train_idx, size=min(chunk, args.iters - it))
        ltr = net.train(idx, lr=lr)
        lho = net.eval_samples(hold_idx)
        hist.append((it + len(idx), ltr, lho))
        log(f"iter {it + len(idx)}: train {ltr:.4g} held-out {lho:.4g}")
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    net.save(args.out, options)
    log(f"saved {args.out}")
    ev = evaluate(net, hold_seeds[:args.eval_members], args.n, args.steps, sopts)
    for e in ev:
        log(f"seed {e['seed']} dt {e['dt']}: newton previous {sum(e['previous']['newton'])} "
            f"learned {sum(e['learned']['newton'])}, used {sum(1 for u in e['learned']['used_guess'] if u)}"
            f"/{len(e['learned']['used_guess'])}")
    report = {"n": args.n, "members": args.members, "steps": args.steps, "samples_train": int(n_train),
              "samples_held_out": int(len(hold_idx)), "scales": net.scales().tolist(),
              "loss_initial": [l_tr0, l_ho0], "history": hist, "evaluation": ev}
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f)


if __name__ == "__main__":
    main()
