"""The learned sweep screen end to end, at a small size: batched runs make
the training set, the GPU MLP learns it, and every point of the screen (reported
or re-run) is judged against the plain FP64 solver.  The trained network must beat
the same network untrained on the held-out points (what training gains),
and the screen must be cheaper than running every point."""
import numpy as np
import pytest

import lbib
import surrogate

pytestmark = pytest.mark.gpu


def test_surrogate_learns_and_screens(gpu):
    steps, every = 200, 50
    tr = surrogate.draw(96, 2)
    disp, alive, stop, _ = surrogate.simulate(tr, steps, every, "f16-flow")
    assert disp.shape == (96, 4, 64, 3) and np.abs(disp[:, -1]).max() > 0
    X, Y = surrogate.training_set(tr, disp, alive)
    assert np.isfinite(X).all() and np.isfinite(Y).all()
    model, curves = surrogate.train(X, Y, members=2, iters=600, batch=256)
    for c in curves[:2]:
        assert c[-1][1] < 0.2 * c[0][1], c
    ev = surrogate.draw(32, 3)
    truth = surrogate.simulate(ev, steps, steps, "f64")
    d, ok = surrogate.clean(truth[0], truth[1])
    true_tip = surrogate.tip_of(d[:, -1])
    done = ok[:, -1]
    tip, _ = surrogate.predict(model, ev)
    err_trained = np.abs(tip.mean(axis=0) - true_tip)[done].mean()
    untrained = ([lbib.MLP(surrogate.WIDTHS, max_batch=256, seed=100 + m) for m in range(2)],
                 lbib.MLP(surrogate.STOP_WIDTHS, max_batch=256, seed=7))
    tip0, _ = surrogate.predict(untrained, ev)
    err_untrained = np.abs(tip0.mean(axis=0) - true_tip)[done].mean()
    assert err_trained < 0.5 * err_untrained, (err_trained, err_untrained)
    rep = surrogate.evaluate(model, ev, steps, truth=truth)
    assert rep["points"] == 32 and rep["rerun"] + rep["reported_by_surrogate"] == 32
    assert rep["rerun"] >= 2                      # the top 5% always go to the solver
    assert 0.0 <= rep["reported_right_frac"] <= 1.0
    assert rep["rerun_right"] >= 0.9 * rep["rerun"]          # FP16 re-runs judged by FP64
    rep64 = surrogate.evaluate(model, ev, steps, truth=truth, rerun_precision="f64")
    assert rep64["rerun"] == rep["rerun"]
    assert rep64["rerun_right"] == rep64["rerun"]           # the plain solver is its own judge
    for n in model[0] + [model[1]] + untrained[0] + [untrained[1]]:
        n.close()
