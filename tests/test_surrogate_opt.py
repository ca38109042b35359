"""Surrogate-assisted optimisation loop (surrogate_opt.py) on a small problem:
the FDTD-run budget holds, a step counts only after its simulation (the best
value is monotone and always a simulated one), widths stay in bounds, the
surrogate's proposals stay in their trust region, and both arms run end to
end."""
from __future__ import annotations

import importlib

import numpy as np
import pytest


def check_arm(O, r, budget):
    assert r["runs"] <= budget
    bests = [h["best"] for h in r["history"]]
    assert all(b2 >= b1 for b1, b2 in zip(bests, bests[1:]))
    assert r["best"] in [h["T"] for h in r["history"]]
    assert all(O.W_LO <= w <= O.W_HI for w in r["widths"])
    assert all(h2["seconds"] >= h1["seconds"] for h1, h2 in zip(r["history"], r["history"][1:]))


@pytest.mark.gpu
def test_optimisation_loop_small(fd, gpu):
    O = importlib.import_module("3d_fdtd_b200.surrogate_opt")
    nz, steps = 96, 4000
    widths, t, gen = O.training_data(fd, 16, nz, steps, None)
    assert t.shape == (16, 11) and np.all(np.isfinite(t)) and not gen["cached"]
    X, Y = O.norm_x(widths), O.to_y(t)
    net = O.Net(fd)
    try:
        first = net.train(X, Y, 1)
        last = net.train(X, Y, 80, lr=1e-3, lr_end=1e-5)
        assert last < first
        start = int(np.argmax(O.mean_T_of_y(Y)))
        w0 = widths[start]
        props = O.surrogate_proposals(net, w0, 0.2, 3, np.random.default_rng(0), starts=16, substeps=5)
        assert 1 <= len(props) <= 3 and props.shape[1] == O.NCTRL and np.abs(props - w0).max() <= 0.2 + 1e-12
        sur = O.optimise_surrogate(fd, net, (X.copy(), Y.copy()), w0, float(O.mean_T_of_y(Y)[start]), nz, steps,
                                   budget=6, k=3, finetune_epochs=5)
        check_arm(O, sur, 6)
        adj = O.optimise_adjoint(fd, w0, nz, steps, budget=6)
        check_arm(O, adj, 6)
        p = net.get_params()
        net.set_params(p)
        assert np.array_equal(net.get_params(), p)
        hyb = O.optimise_hybrid(fd, net, (X.copy(), Y.copy()), w0, nz, steps, budget=6, finetune_epochs=5)
        check_arm(O, hyb, 6)
        assert O.time_to(adj, adj["best"]) is not None
    finally:
        net.close()
