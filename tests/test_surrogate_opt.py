"""Surrogate-assisted optimisation loop (surrogate_opt.py) on a small problem:
the FDTD-run budget holds, a step counts only after its simulation (the best
value is monotone and always a simulated one), and both the surrogate and the
adjoint-only variants run end to end."""
from __future__ import annotations

import importlib

import numpy as np
import pytest


@pytest.mark.gpu
def test_optimisation_loop_small(fd, gpu):
    O = importlib.import_module("3d_fdtd_b200.surrogate_opt")
    nz, steps = 96, 4000
    widths = [O.random_widths(1000 + i) for i in range(16)]
    t, _ = O.simulate(fd, widths, nz, steps)
    assert t.shape == (16, 11) and np.all(np.isfinite(t))
    X, Y = O.norm_x(np.array(widths)), O.to_y(t)
    net = O.Net(fd)
    try:
        first = net.train(X, Y, 1)
        last = net.train(X, Y, 80)
        assert last < first
        w0 = np.array(widths[int(np.argmax(O.mean_T_of_y(Y)))])
        for use_net in (True, False):
            r = O.optimise(fd, w0, nz, steps, budget=8, net=net if use_net else None, data=(X.copy(), Y.copy()),
                           finetune_epochs=5)
            assert r["runs"] <= 8
            sims = [h["T"] for h in r["history"]]
            bests = [h.get("best", h["T"]) for h in r["history"]]
            assert all(b2 >= b1 for b1, b2 in zip(bests, bests[1:]))
            assert r["best"] in sims
            assert all(O.W_LO <= w <= O.W_HI for w in r["widths"])
    finally:
        net.close()
