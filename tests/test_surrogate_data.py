"""Training-set hygiene of the sweep surrogate (no GPU)."""
import numpy as np

import surrogate


def test_clean_holds_targets_after_a_stop_and_drops_blowups():
    disp = np.zeros((3, 4, 64, 3), dtype=np.float32)
    disp[:, :, :, 0] = np.arange(4)[None, :, None]
    alive = np.ones((3, 4), dtype=bool)
    alive[1, 2:] = False                       # stopped after snapshot 1
    disp[2, 2] = np.nan                        # blew up at snapshot 2
    disp[2, 3] = 1e6
    d, ok = surrogate.clean(disp, alive)
    assert ok[0].all() and list(ok[1]) == [True, True, False, False] and list(ok[2]) == [True, True, False, False]
    assert np.isfinite(d).all()
    assert (d[1, 2:, :, 0] == 1).all() and (d[2, 2:, :, 0] == 1).all()
    X, Y = surrogate.training_set(surrogate.draw(3, 2), disp, alive)
    assert X.shape == (12, 5) and Y.shape == (12, 193) and np.isfinite(Y).all()
    assert np.abs(X).max() <= 1.0 + 1e-6
