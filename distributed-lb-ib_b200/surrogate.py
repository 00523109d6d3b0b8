"""A learned screen for parameter sweeps: an MLP surrogate trained on
trajectories the batched solver generates, with the plain solver as its
fallback and judge.

Workload (the learned-sweep benchmark): problems on a 96 x 48 x 48 lattice
with a 32 x 32 sheet (spacing 0.5, plane x = 16, centred, free as in the
reference), parameters (Ks, Kb, tau, u_x) drawn as in the batched sweep
(log-uniform Ks in [1e-3, 1e-1], Kb in [1e-4, 1e-2], tau in [0.55, 0.9],
u_x in [0.005, 0.03]); training runs from default_rng(2), held-out sweep
points from default_rng(3); T = 3000 steps.

Model: inputs (log10 Ks, log10 Kb, tau, u_x, t/T), affinely scaled to about
[-1, 1]; 4 hidden layers of 256 with GELU; outputs the x, y, z displacement
of an 8 x 8 subsample of the sheet's nodes (rows and columns 0, 4, 9, 13,
18, 22, 27, 31) since t = 0, scaled by 1/20; trained on the snapshots of
runs that are still going, three members, each on its own bootstrap of the
training runs.  Many runs of
this parameter range stop (their sheet leaves the grid or blows up), so a
second, small net (4 parameters -> 2 x 64 -> 1) learns whether a run
reaches T.  Both are trained by the library's own GPU kernels (lbib_mlp_*:
BF16 tensor-core GEMMs, Adam).

Screen: the nets predict every point at t = T.  A point is re-run by the
batched solver (FP16 flow-shifted storage by default, FP64 on request) when
its stop output is undecided, when it is among the
top 5% of the points predicted to reach T by tip displacement (the points a
sweep is after), or when the members disagree on its tip by more than a
threshold; every other point is reported from the surrogate: "stops", or
its tip.  The two thresholds are calibrated on the last eighth of the
training runs, which the nets do not train on: the loosest settings at which
98% of the points the surrogate would report there are right.  The referee:
the plain FP64 solver on every point, which the report compares against --
tip displacement = mean x-displacement of the subsample's last row.
"""
from __future__ import annotations

import time
from typing import Dict, List

import numpy as np

import lbib
import sweep

NX, NY, NZ, SIDE = 96, 48, 48, 32
SUB = np.round(np.arange(8) * (SIDE - 1) / 7.0).astype(int)  # 0 4 9 13 18 22 27 31
DISP_SCALE = 20.0


def draw(n: int, seed: int, pinned: bool = False) -> List[lbib.Problem]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ks = float(10 ** rng.uniform(-3, -1))
        kb = float(10 ** rng.uniform(-4, -2))
        tau = float(rng.uniform(0.55, 0.9))
        u = float(rng.uniform(0.005, 0.03))
        out.append(sweep.make_problem(NX, NY, NZ, SIDE, ks, kb, tau, u, pinned))
    return out


def subsample(sheet: np.ndarray) -> np.ndarray:
    return sheet[SUB][:, SUB, :3].reshape(64, 3)


AUTOTUNE_MIN_STEPS = 1000


def simulate(problems, steps: int, every: int, precision: str, chunk: int = 1024):
    """Run the problems in batches of `chunk`; returns the subsample
    displacement [n, snaps, 64, 3] at t = every, 2 every, ..., steps, the
    alive flag [n, snaps], each problem's stop step (0 = completed) and the
    wall-clock seconds (set-up included)."""
    n = len(problems)
    snaps = steps // every
    disp = np.zeros((n, snaps, 64, 3), dtype=np.float32)
    alive = np.ones((n, snaps), dtype=bool)
    stop = np.zeros(n, dtype=np.int64)
    t0 = time.perf_counter()
    for c0 in range(0, n, chunk):
        part = problems[c0:c0 + chunk]
        with lbib.Batch(part, precision, compat=0) as b:
            # the kernel-variant trial costs a few dozen steps per size
            # class: worth it for long runs only
            if b.variants() > 1 and steps >= AUTOTUNE_MIN_STEPS:
                b.autotune(4)
            x0 = [subsample(b.sheet(k)) for k in range(len(part))]
            for s in range(snaps):
                b.run(every)
                codes, at = b.status()
                for k in range(len(part)):
                    disp[c0 + k, s] = subsample(b.sheet(k)) - x0[k]
                    if codes[k]:
                        alive[c0 + k, s] = False
                        stop[c0 + k] = at[k]
    return disp, alive, stop, time.perf_counter() - t0


def features(problems, tfrac) -> np.ndarray:
    p = np.array([[np.log10(q.Ks_l), np.log10(q.Kb_l), q.tau, q.u_l] for q in problems])
    x = np.empty((len(problems), 5), dtype=np.float32)
    x[:, 0] = (p[:, 0] + 2.0)          # [-1, 1]
    x[:, 1] = (p[:, 1] + 3.0)
    x[:, 2] = (p[:, 2] - 0.725) / 0.175
    x[:, 3] = (p[:, 3] - 0.0175) / 0.0125
    x[:, 4] = 2.0 * np.asarray(tfrac) - 1.0
    return x


MAX_DISP = 60.0   # a node further than this from its start is counted as a stopped run


def clean(disp, alive):
    """A snapshot is valid while its run is going and its displacements are
    finite and bounded (a diverging run blows up before its sheet leaves the
    grid).  After the last valid snapshot the displacement target is held at
    that snapshot's value and the stop output is 0."""
    ok = alive & np.isfinite(disp).all(axis=(2, 3)) & (np.abs(np.nan_to_num(disp, nan=1e9)).max(axis=(2, 3)) <= MAX_DISP)
    ok = np.cumprod(ok, axis=1).astype(bool)        # once stopped, stays stopped
    d = np.where(ok[..., None, None], disp, 0.0).astype(np.float32)
    last = np.maximum(ok.sum(axis=1) - 1, 0)
    for i in np.nonzero(~ok.all(axis=1))[0]:
        hold = d[i, last[i]] if ok[i, last[i]] else np.zeros((64, 3), np.float32)
        d[i, ~ok[i]] = hold
    return d, ok


def training_set(problems, disp, alive):
    n, snaps = alive.shape
    d, ok = clean(disp, alive)
    tf = np.repeat(((np.arange(snaps) + 1) / snaps)[None, :], n, axis=0).ravel()
    X = features([problems[i] for i in range(n) for _ in range(snaps)], tf)
    Y = np.concatenate([d.reshape(n * snaps, 192) / DISP_SCALE, ok.reshape(n * snaps, 1)], axis=1)
    return X, Y.astype(np.float32)


WIDTHS = [5, 256, 256, 256, 256, 192]      # the displacement surrogate
STOP_WIDTHS = [4, 64, 64, 1]              # does the run reach T? (parameters only)


def _fit(net, Xd, Yd, iters, batch, lr, seed):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    n = Xd.shape[0]
    curve = []
    for it in range(iters):
        idx = torch.randint(0, n, (batch,), device="cuda", generator=g)
        want = it % 500 == 0 or it == iters - 1
        loss = net.train_step(Xd[idx].contiguous(), Yd[idx].contiguous(), lr * (0.1 ** (it / iters)),
                              want_loss=want)
        if want:
            curve.append((it, loss))
    net.synchronize()
    return curve


def train(X, Y, members: int = 3, iters: int = 6000, batch: int = 1024, lr: float = 1e-3):
    """Train on the GPU: `members` displacement nets on the snapshots of runs
    still going, and one stop net on each run's fate at T.  X, Y as made by
    training_set (Y's last column: the run is still going)."""
    import torch
    final = X[:, 4] > 1.0 - 1e-6                   # t = T rows, one per run
    runs = int(final.sum())
    run_of_row = np.arange(X.shape[0]) // (X.shape[0] // runs)
    going = Y[:, 192] > 0.5
    nets, curves = [], []
    for m in range(members):
        # each member sees its own bootstrap of the runs, so that their
        # disagreement tracks how well the data pins a point down
        pick = np.zeros(runs, dtype=bool)
        pick[np.random.default_rng(500 + m).integers(0, runs, runs)] = True
        rows = going & pick[run_of_row]
        Xd = torch.from_numpy(np.ascontiguousarray(X[rows])).cuda()
        Yd = torch.from_numpy(np.ascontiguousarray(Y[rows, :192])).cuda()
        net = lbib.MLP(WIDTHS, max_batch=batch, seed=100 + m)
        curves.append(_fit(net, Xd, Yd, iters, batch, lr, 1000 + m))
        nets.append(net)
    Xs = torch.from_numpy(np.ascontiguousarray(X[final, :4])).cuda()
    Ys = torch.from_numpy(np.ascontiguousarray(Y[final, 192:193])).cuda()
    stop = lbib.MLP(STOP_WIDTHS, max_batch=min(batch, Xs.shape[0]), seed=7)
    curves.append(_fit(stop, Xs, Ys, iters // 2, min(batch, Xs.shape[0]), lr, 77))
    return (nets, stop), curves


def predict(model, problems):
    """Per member the tip displacement at T, and the probability-like stop
    output (1: reaches T)."""
    import torch
    nets, stop = model
    X = torch.from_numpy(features(problems, np.ones(len(problems)))).cuda()
    def run(net, X):
        return torch.cat([net.forward(X[c0:c0 + net.max_batch].contiguous())
                          for c0 in range(0, X.shape[0], net.max_batch)]).cpu().numpy()
    outs = np.stack([run(net, X) for net in nets])          # [members, n, 192]
    disp = outs.reshape(len(nets), len(problems), 64, 3) * DISP_SCALE
    tip = disp[..., 56:64, 0].mean(axis=-1)                  # last subsample row, x
    alive = run(stop, X[:, :4].contiguous())[:, 0]
    return tip, alive


def tip_of(disp_final: np.ndarray) -> np.ndarray:
    return disp_final[:, 56:64, 0].mean(axis=-1)


def calibrate(model, problems, disp_final, going, target: float = 0.98) -> Dict:
    """Re-run thresholds from runs the nets did not train on: the widest
    stop band edge and the largest member disagreement at which the points
    the surrogate would report are still right at `target` rate (stop
    right; tip within 2%)."""
    tip, alive = predict(model, problems)
    m_tip = tip.mean(axis=0)
    spread = np.abs(tip.max(axis=0) - tip.min(axis=0)) / np.maximum(np.abs(m_tip), 1e-3)
    true_tip = tip_of(disp_final)
    tip_ok = np.abs(m_tip - true_tip) <= np.maximum(0.02 * np.abs(true_tip), 0.02)
    band = 0.3
    for b in (0.05, 0.1, 0.15, 0.2, 0.25, 0.3, 0.35, 0.4, 0.45):
        decided = np.abs(alive - 0.5) >= b
        if decided.any() and ((alive[decided] > 0.5) == going[decided]).mean() >= target:
            band = b
            break
    goes = (alive - 0.5 >= band) & going
    disagree = 0.0
    for d in np.sort(spread[goes]):
        kept = goes & (spread <= d)
        if tip_ok[kept].mean() >= target:
            disagree = float(d)
    return {"stop_band": band, "disagree": disagree}


def screen(model, problems, top: float = 0.05, disagree: float = 0.01, band: float = 0.3):
    """Which points the surrogate reports and which go to the plain solver:
    stop outputs within `band` of 0.5, the top `top` by predicted tip, and
    points whose members disagree by more than `disagree` (relative) are
    re-run."""
    t0 = time.perf_counter()
    tip, alive = predict(model, problems)
    m_tip = tip.mean(axis=0)
    spread = np.abs(tip.max(axis=0) - tip.min(axis=0)) / np.maximum(np.abs(m_tip), 1e-3)
    goes = alive > 0.5
    undecided = np.abs(alive - 0.5) < band
    disagreeing = goes & ~undecided & (spread > disagree)
    k = max(1, int(round(top * len(problems))))
    cand = np.where(goes, np.abs(m_tip), -1.0)
    topk = np.zeros(len(problems), dtype=bool)
    topk[np.argsort(-cand)[:k]] = True
    rerun = undecided | disagreeing | topk
    return {"tip": m_tip, "alive": goes, "spread": spread, "rerun": rerun, "seconds": time.perf_counter() - t0,
            "why": {"undecided_stop": int(undecided.sum()), "disagreement": int(disagreeing.sum()),
                    "top": int(topk.sum())}}


def evaluate(model, problems, steps: int, truth=None, thresholds=None, rerun_precision: str = "f16-flow") -> Dict:
    """Screen `problems`, re-run the flagged ones with the batched solver in
    `rerun_precision`, and judge every point -- reported or re-run --
    against the plain FP64 solver's own run."""
    th = thresholds or {}
    s = screen(model, problems, disagree=th.get("disagree", 0.01), band=th.get("stop_band", 0.3))
    idx = np.nonzero(s["rerun"])[0]
    tip, goes = s["tip"].copy(), s["alive"].copy()
    rerun_s = 0.0
    if len(idx):
        d, a, _, rerun_s = simulate([problems[i] for i in idx], steps, steps, rerun_precision)
        d, a = clean(d, a)
        tip[idx], goes[idx] = tip_of(d[:, -1]), a[:, -1]
    if truth is None:
        truth = simulate(problems, steps, steps, "f64")
    tdisp, talive, _, plain_s = truth
    tdisp, talive = clean(tdisp, talive)
    true_tip = tip_of(tdisp[:, -1])
    true_alive = talive[:, -1]
    rep = ~s["rerun"]
    # a point is right when it gets "stopped" right, and, for a run that
    # completes, its tip within 2% (or 0.02 lattice units for tiny tips)
    tip_ok = np.abs(tip - true_tip) <= np.maximum(0.02 * np.abs(true_tip), 0.02)
    rel = np.abs(s["tip"] - true_tip) / np.maximum(np.abs(true_tip), 1e-3)
    right = (goes == true_alive) & (~true_alive | tip_ok)
    rr = s["rerun"]
    sur_s = s["seconds"] + rerun_s
    return {"points": len(problems), "reported_by_surrogate": int(rep.sum()), "rerun": int(len(idx)), "rerun_why": s["why"],
            "rerun_precision": rerun_precision, "rerun_s": rerun_s, "screen_s": s["seconds"],
            "plain_fp64_s": plain_s, "plain_points_per_s": len(problems) / plain_s,
            "surrogate_s": sur_s, "surrogate_points_per_s": len(problems) / sur_s,
            "speedup": plain_s / sur_s,
            "right": int(right.sum()), "right_frac": float(right.mean()),
            "reported_right": int(right[rep].sum()), "reported_right_frac": float(right[rep].mean()) if rep.any() else 1.0,
            "rerun_right": int(right[rr].sum()),
            "completed": int(true_alive.sum()), "completed_tip_within_2pct": int((true_alive & tip_ok & (goes == true_alive)).sum()),
            "reported_completed": int((rep & true_alive).sum()),
            "reported_completed_tip_within_2pct": int((rep & true_alive & tip_ok).sum()),
            "stop_prediction_accuracy": float((s["alive"] == true_alive).mean()),
            "all_completed_tip_rel_err_median": float(np.median(rel[true_alive])) if true_alive.any() else None,
            "all_completed_tip_within_2pct_frac": float((rel[true_alive] <= 0.02).mean()) if true_alive.any() else None}


def pipeline(train_n: int = 4096, eval_n: int = 2048, steps: int = 3000, every: int = 100, iters: int = 10000,
             members: int = 3, calib_frac: float = 0.125, target: float = 0.98,
             rerun_precision: str = "f16-flow", data: str = None) -> Dict:
    """The whole learned sweep: training runs (batched, FP16 storage), GPU
    training, calibration of the re-run thresholds on the last `calib_frac`
    of the training runs, the plain FP64 batched sweep of the held-out points
    (the referee, and the baseline rate), and the screen of the same points.
    With `data`, simulated runs are kept there and reused."""
    import os
    out = {"config": {"train_n": train_n, "eval_n": eval_n, "steps": steps, "every": every, "iters": iters,
                      "members": members, "calib_frac": calib_frac, "target": target,
                      "rerun_precision": rerun_precision}}
    tr = draw(train_n, 2)
    ev = draw(eval_n, 3)
    ftr = os.path.join(data, f"train_{train_n}_{steps}_{every}.npz") if data else None
    fev = os.path.join(data, f"truth_{eval_n}_{steps}.npz") if data else None
    if ftr and os.path.exists(ftr):
        z = np.load(ftr)
        disp, alive, gen_s = z["disp"].astype(np.float32), z["alive"], float(z["seconds"])
    else:
        disp, alive, _, gen_s = simulate(tr, steps, every, "f16-flow")
        if ftr:
            os.makedirs(data, exist_ok=True)
            np.savez(ftr, disp=disp.astype(np.float16), alive=alive, seconds=gen_s)
    out["training_runs"] = {"n": train_n, "seconds": gen_s, "completed": int(clean(disp, alive)[1][:, -1].sum())}
    nval = max(1, int(round(train_n * calib_frac)))      # the last runs calibrate the screen
    ntr = train_n - nval
    X, Y = training_set(tr[:ntr], disp[:ntr], alive[:ntr])
    t0 = time.perf_counter()
    model, curves = train(X, Y, members=members, iters=iters)
    out["training"] = {"runs": ntr, "samples": int(X.shape[0]), "seconds": time.perf_counter() - t0,
                       "loss_curves": curves}
    dv, okv = clean(disp[ntr:], alive[ntr:])
    th = calibrate(model, tr[ntr:], dv[:, -1], okv[:, -1], target=target)
    out["calibration"] = dict(th, runs=nval)
    if fev and os.path.exists(fev):
        z = np.load(fev)
        truth = (z["disp"], z["alive"], z["stop"], float(z["seconds"]))
    else:
        truth = simulate(ev, steps, steps, "f64")
        if fev:
            np.savez(fev, disp=truth[0], alive=truth[1], stop=truth[2], seconds=truth[3])
    out["evaluation"] = evaluate(model, ev, steps, truth=truth, thresholds=th, rerun_precision=rerun_precision)
    for n in model[0] + [model[1]]:
        n.close()
    return out


def main(argv=None) -> int:
    import argparse
    import json

    ap = argparse.ArgumentParser(description="learned sweep screen")
    ap.add_argument("--train-n", type=int, default=4096)
    ap.add_argument("--eval-n", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--iters", type=int, default=10000)
    ap.add_argument("--members", type=int, default=3)
    ap.add_argument("--calib-frac", type=float, default=0.125,
                    help="fraction of the training runs held back to calibrate the re-run thresholds")
    ap.add_argument("--target", type=float, default=0.98,
                    help="rate of right points the calibration asks of the points the surrogate reports")
    ap.add_argument("--rerun-precision", default="f16-flow",
                    help="storage of the batched solver that re-runs the flagged points (f64: the plain solver)")
    ap.add_argument("--data", default=None,
                    help="directory to keep the simulated runs in (reused when present: only the "
                         "training and the screen run again)")
    a = ap.parse_args(argv)
    out = pipeline(a.train_n, a.eval_n, a.steps, a.every, a.iters, a.members, a.calib_frac, a.target,
                   a.rerun_precision, a.data)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
