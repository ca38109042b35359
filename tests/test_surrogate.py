"""Surrogate network (surrogate.cu) against the FP64 restatement in
oracle/surrogate.py.  CPU: the restatement's backward against central finite
differences.  GPU: forward, weight gradients, input gradient and one Adam step
against the restatement with the same BF16 rounding points (the GPU
accumulates in FP32, the restatement in FP64)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import surrogate as S

FP = C.POINTER(C.c_float)


def test_restatement_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    n_in, hid, n_out, B = 3, 8, 2, 4
    count = hid * n_in + hid + 2 * (hid * hid + hid) + n_out * hid + n_out
    flat = rng.normal(0, 0.5, count)
    x, t = rng.normal(size=(B, n_in)), rng.normal(size=(B, n_out))
    loss, grads, dx = S.gradients(S.unflatten(flat, n_in, hid, n_out), x, t, bf=False)
    g = S.flatten(grads)
    eps = 1e-6
    for idx in rng.choice(count, 12, replace=False):
        fp, fm = flat.copy(), flat.copy()
        fp[idx] += eps
        fm[idx] -= eps
        lp = S.gradients(S.unflatten(fp, n_in, hid, n_out), x, t, bf=False)[0]
        lm = S.gradients(S.unflatten(fm, n_in, hid, n_out), x, t, bf=False)[0]
        assert abs((lp - lm) / (2 * eps) - g[idx]) < 1e-7 * max(1.0, abs(g[idx]))
    for c in range(n_in):
        xp, xm = x.copy(), x.copy()
        xp[0, c] += eps
        xm[0, c] -= eps
        fd_ = (S.gradients(S.unflatten(flat, n_in, hid, n_out), xp, t, bf=False)[0]
               - S.gradients(S.unflatten(flat, n_in, hid, n_out), xm, t, bf=False)[0]) / (2 * eps)
        assert abs(fd_ - dx[0, c]) < 1e-7


@pytest.fixture()
def net(fd, gpu):
    h = fd.lib.fdtd_mlp_new(20, 256, 22, 123)
    assert h, fd.lib.fdtd_last_error_message()
    yield h
    fd.lib.fdtd_mlp_free(h)


def params_of(fd, h):
    n = fd.lib.fdtd_mlp_param_count(h)
    p = np.zeros(n, np.float32)
    fd.call("fdtd_mlp_get_params", h, p.ctypes.data_as(FP))
    return p


def data(B, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.5, 3.0, (B, 20)).astype(np.float32)
    t = np.concatenate([np.sin(x[:, :11] * 1.3), np.cos(x[:, 9:] * 0.7)], axis=1).astype(np.float32)
    return x, t


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.gpu
def test_param_count(fd, net):
    assert fd.lib.fdtd_mlp_param_count(net) == 142_614


@pytest.mark.gpu
def test_forward_and_gradients_match_restatement(fd, net):
    B = 256
    x, t = data(B)
    flat = params_of(fd, net)
    P = S.unflatten(flat.astype(np.float64), 20, 256, 22)
    y = np.zeros((B, 22), np.float32)
    fd.call("fdtd_mlp_forward", net, x.ctypes.data_as(FP), B, y.ctypes.data_as(FP))
    y_ref = S.forward(P, x.astype(np.float64))[0]
    assert rel(y, y_ref) < 2e-3
    g = np.zeros_like(flat)
    loss = C.c_double()
    fd.call("fdtd_mlp_gradients", net, x.ctypes.data_as(FP), t.ctypes.data_as(FP), B, g.ctypes.data_as(FP),
            C.byref(loss))
    loss_ref, grads_ref, _ = S.gradients(P, x.astype(np.float64), t.astype(np.float64))
    assert abs(loss.value - loss_ref) < 1e-3 * loss_ref
    got = S.unflatten(g.astype(np.float64), 20, 256, 22)
    for (gw, gb), (rw, rb) in zip(got, grads_ref):
        assert rel(gw, rw) < 2e-2 and rel(gb, rb) < 2e-2
        assert np.dot(gw.ravel(), rw.ravel()) / np.linalg.norm(gw) / np.linalg.norm(rw) > 0.9999


@pytest.mark.gpu
def test_input_gradient_matches_restatement(fd, net):
    B = 64
    x, _ = data(B, seed=2)
    dy = np.random.default_rng(3).normal(size=(B, 22)).astype(np.float32)
    dx = np.zeros((B, 20), np.float32)
    fd.call("fdtd_mlp_input_gradient", net, x.ctypes.data_as(FP), dy.ctypes.data_as(FP), B, dx.ctypes.data_as(FP))
    P = S.unflatten(params_of(fd, net).astype(np.float64), 20, 256, 22)
    ref = S.input_gradient(P, x.astype(np.float64), dy.astype(np.float64))
    assert rel(dx, ref) < 2e-2


@pytest.mark.gpu
def test_adam_step_matches_restatement_and_training_converges(fd, net):
    B = 512
    x, t = data(B, seed=4)
    flat = params_of(fd, net).astype(np.float64)
    P = S.unflatten(flat, 20, 256, 22)
    lr = 1e-3
    loss = C.c_double()
    fd.call("fdtd_mlp_train_step", net, x.ctypes.data_as(FP), t.ctypes.data_as(FP), B, C.c_float(lr), C.byref(loss))
    _, g, _ = S.gradients(P, x.astype(np.float64), t.astype(np.float64))
    zeros = [(np.zeros_like(W), np.zeros_like(b)) for W, b in P]
    P1, _, _ = S.adam(P, g, zeros, zeros, 1, lr)
    new = params_of(fd, net).astype(np.float64)
    # first Adam step moves every parameter by ~lr * sign(g): compare the moves
    step_gpu, step_ref = new - flat, S.flatten(P1) - flat
    big = np.abs(step_ref) > 0.5 * lr
    assert np.mean(np.sign(step_gpu[big]) == np.sign(step_ref[big])) > 0.99
    assert np.abs(step_gpu - step_ref).max() < 1.01 * lr
    first = loss.value
    for _ in range(300):
        fd.call("fdtd_mlp_train_step", net, x.ctypes.data_as(FP), t.ctypes.data_as(FP), B, C.c_float(lr),
                C.byref(loss))
    assert loss.value < 0.05 * first
