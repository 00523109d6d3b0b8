"""The learned sweep screen end to end at a small size, judged on the
quantity the learned-sweep benchmark states: the screen's sweep points per
second over the plain batched FP64 sweep's, on held-out points, at a stated
tip-error bound.

Batched runs (FP16 storage) make the training set, the GPU MLP learns it
(tcgen05 kernels), and the screen reports points from the surrogate or
re-runs them with the batched solver; every point, reported or re-run, is
judged against the plain FP64 batched solver's own run of it.  A point is
right when its stop / complete outcome matches the FP64 run and, if it
completes, its tip displacement (mean x-displacement of the last fiber row)
is within 2% of the FP64 run's (or 0.02 lattice units for a tiny tip).

Size: 256 training runs and 128 held-out points of the 96 x 48 x 48 /
32 x 32-sheet workload over 500 steps (the benchmark's are 4096 / 2048 over
3000 steps); the re-run thresholds are fixed here (member disagreement 2%,
stop band 0.2) instead of calibrated, which needs more runs than this test
makes.  Measured at this size, alone: ~7x the plain sweep's points/s with
~95% of the points right.  At this size the screen's few re-runs are
dominated by the batch's fixed set-up cost, so the wall-clock ratio moves
with the process's state (after the rest of the suite it has measured 1.7x
with the same 28 re-runs); the test therefore bounds the ratio loosely and
the screen's share of re-run points -- the work it leaves to the solver --
tightly.  The bars leave room for the run-to-run spread of the training
data (the batch autotuner's variant choice moves its last bits).
"""
import numpy as np
import pytest

import lbib
import surrogate

pytestmark = pytest.mark.gpu

TRAIN, EVAL, STEPS, EVERY, ITERS = 256, 128, 500, 50, 1500
MIN_SPEEDUP = 1.5        # screen points/s over plain batched FP64 points/s (wall clock)
MAX_RERUN = 0.35         # share of the held-out points the screen sends to the solver
MIN_RIGHT = 0.85         # fraction of held-out points right at the 2% tip bound


def test_surrogate_screen_beats_the_plain_sweep(gpu):
    tr = surrogate.draw(TRAIN, 2)
    disp, alive, stop, _ = surrogate.simulate(tr, STEPS, EVERY, "f16-flow")
    assert disp.shape == (TRAIN, STEPS // EVERY, 64, 3) and np.abs(disp[:, -1]).max() > 0
    X, Y = surrogate.training_set(tr, disp, alive)
    assert np.isfinite(X).all() and np.isfinite(Y).all()
    model, curves = surrogate.train(X, Y, members=2, iters=ITERS, batch=256)
    for c in curves[:2]:
        assert c[-1][1] < 0.2 * c[0][1], c          # both members learned

    ev = surrogate.draw(EVAL, 3)
    truth = surrogate.simulate(ev, STEPS, STEPS, "f64")
    rep = surrogate.evaluate(model, ev, STEPS, truth=truth, thresholds={"disagree": 0.02, "stop_band": 0.2})
    assert rep["points"] == EVAL and rep["rerun"] + rep["reported_by_surrogate"] == EVAL
    assert rep["rerun"] >= round(0.05 * EVAL)       # the top 5% always go to the solver
    assert rep["rerun"] <= MAX_RERUN * EVAL, rep
    # the benchmark's quantity: points/s over the plain FP64 batched sweep, at the 2% bound
    assert rep["speedup"] >= MIN_SPEEDUP, rep
    assert rep["right_frac"] >= MIN_RIGHT, rep
    assert rep["rerun_right"] >= 0.9 * rep["rerun"]            # FP16 re-runs judged by FP64

    # what training gains: the same nets untrained are far off on the same points
    d, ok = surrogate.clean(truth[0], truth[1])
    true_tip = surrogate.tip_of(d[:, -1])
    done = ok[:, -1]
    tip, _ = surrogate.predict(model, ev)
    untrained = ([lbib.MLP(surrogate.WIDTHS, max_batch=256, seed=100 + m) for m in range(2)],
                 lbib.MLP(surrogate.STOP_WIDTHS, max_batch=256, seed=7))
    tip0, _ = surrogate.predict(untrained, ev)
    err = np.abs(tip.mean(axis=0) - true_tip)[done].mean()
    err0 = np.abs(tip0.mean(axis=0) - true_tip)[done].mean()
    assert err < 0.5 * err0, (err, err0)

    # re-running in FP64 makes every re-run point right by definition
    rep64 = surrogate.evaluate(model, ev, STEPS, truth=truth, thresholds={"disagree": 0.02, "stop_band": 0.2},
                               rerun_precision="f64")
    assert rep64["rerun"] == rep["rerun"] and rep64["rerun_right"] == rep64["rerun"]
    for n in model[0] + [model[1]] + untrained[0] + [untrained[1]]:
        n.close()
