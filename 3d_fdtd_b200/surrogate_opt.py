"""Surrogate-assisted taper optimisation: a tensor-core MLP trained on
simulations from the candidate sweep proposes design steps; every step is
confirmed by an FDTD run, and the adjoint gradient takes over when the
surrogate's prediction misses the simulation.

Design: the spline taper of batch.py (20 control widths in [0.5, 3.0] um,
natural cubic spline, sub-pixel fill) on one fixed grid of the candidate
family (256 x 128 x nz, 25 nm, 12-cell CPML).  Outputs: the complex
transmission t(lambda) = O_out / O_in at the 11 monitor wavelengths
1.50..1.60 um as (Re, Im) -> 22 network outputs; T = |t|^2.
Objective: mean T over the 11 wavelengths.

Surrogate step: ascend the predicted objective along the network's input
gradient (normalised, fixed step in um, clipped to the width bounds);
simulate the proposal; if |T_pred - T_fdtd| > 1e-2 discard the surrogate's
direction for this step and take an adjoint step instead (forward + CW
adjoint run as the reference driver does, 3d_fdtd.c:97-165, spline-weighted
edge gradient of |O_out| at 1.55 um); add the simulated point to the training
set and fine-tune; accept a step only if the simulated objective improves,
else halve the step.  Baseline: the same loop with adjoint steps only, given
the same number of FDTD runs.

    python -m 3d_fdtd_b200.surrogate_opt [--train 1024] [--iters 12]
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import math
import time

import numpy as np

B = importlib.import_module("3d_fdtd_b200.batch")
DP = C.POINTER(C.c_double)
FP = C.POINTER(C.c_float)
NCTRL, NLAM, LAM0_INDEX = 20, 11, 5
W_LO, W_HI = 0.5, 3.0


def norm_x(w: np.ndarray) -> np.ndarray:
    return ((np.asarray(w, np.float64) - 1.75) / 1.25).astype(np.float32)


def design(widths, index: int, nz: int, steps: int) -> dict:
    return dict(index=index, L=0.0, nz=nz, steps=steps, widths=np.asarray(widths, float))


def random_widths(seed: int) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).uniform(W_LO, W_HI, NCTRL))


def simulate(fd, widths_list, nz: int, steps: int, slots: int = 4):
    """FDTD of every design (concurrent); returns complex t [n, 11]."""
    cands = [design(w, i, nz, steps) for i, w in enumerate(widths_list)]
    r = B.sweep(fd, cands, slots=slots, variant=fd.YEE_FLAT4)
    return np.array([r["amplitudes"][i] for i in range(len(cands))]), r


class Net:
    """The MLP of csrc/surrogate.cu through the C ABI."""

    def __init__(self, fd, seed: int = 7):
        self.fd = fd
        self.h = fd.lib.fdtd_mlp_new(NCTRL, 256, 2 * NLAM, seed)
        if not self.h:
            raise RuntimeError(fd.lib.fdtd_last_error_message())

    def close(self):
        if self.h:
            self.fd.lib.fdtd_mlp_free(self.h)
            self.h = None

    @staticmethod
    def _pad(x: np.ndarray):
        n = len(x)
        m = (n + 7) // 8 * 8
        if m == n:
            return np.ascontiguousarray(x, np.float32), n
        return np.ascontiguousarray(np.concatenate([x, np.repeat(x[-1:], m - n, axis=0)]), np.float32), n

    def predict(self, x: np.ndarray) -> np.ndarray:
        xp, n = self._pad(x)
        y = np.zeros((len(xp), 2 * NLAM), np.float32)
        self.fd.call("fdtd_mlp_forward", self.h, xp.ctypes.data_as(FP), len(xp), y.ctypes.data_as(FP))
        return y[:n]

    def input_gradient(self, x: np.ndarray, dy: np.ndarray) -> np.ndarray:
        xp, n = self._pad(x)
        dyp, _ = self._pad(dy)
        dx = np.zeros((len(xp), NCTRL), np.float32)
        self.fd.call("fdtd_mlp_input_gradient", self.h, xp.ctypes.data_as(FP), dyp.ctypes.data_as(FP), len(xp),
                     dx.ctypes.data_as(FP))
        return dx[:n]

    def train(self, x: np.ndarray, y: np.ndarray, epochs: int, batch: int = 128, lr: float = 1e-3,
              seed: int = 0) -> float:
        rng = np.random.default_rng(seed)
        n = len(x)
        bs = min(batch, n // 8 * 8)
        loss = C.c_double()
        last = float("nan")
        for _ in range(epochs):
            order = rng.permutation(n)
            for s in range(0, n - bs + 1, bs):
                idx = order[s:s + bs]
                xb, yb = np.ascontiguousarray(x[idx], np.float32), np.ascontiguousarray(y[idx], np.float32)
                self.fd.call("fdtd_mlp_train_step", self.h, xb.ctypes.data_as(FP), yb.ctypes.data_as(FP), bs,
                             C.c_float(lr), C.byref(loss))
                last = loss.value
        return last


def to_y(t: np.ndarray) -> np.ndarray:
    return np.concatenate([t.real, t.imag], axis=-1).astype(np.float32)


def mean_T_of_y(y: np.ndarray) -> np.ndarray:
    return (y[..., :NLAM] ** 2 + y[..., NLAM:] ** 2).mean(axis=-1)


def adjoint_gradient(fd, widths: np.ndarray, nz: int, steps: int) -> np.ndarray:
    """Spline-weighted adjoint gradient of |O_out(1.55 um)| with respect to
    the widths (direction; the reference's formula omits a global constant)."""
    s = B.SPEC
    cand = design(widths, 0, nz, steps)
    slot = B.Slot(fd)
    slot.prepare(cand, fd.YEE_FLAT4)
    t = slot.grid.t
    b, top = s["core_y"]
    z0, z1 = s["margin"], nz - s["margin"]
    w = np.ascontiguousarray(widths, float)
    store = fd.lib.fdtd_spline_store_new(t, NCTRL, w.ctypes.data_as(DP), float(s["cx"]), z0, z1, b, top, steps)
    if not store:
        raise RuntimeError(fd.lib.fdtd_last_error_message())
    try:
        fd.call("fdtd_spline_store_bind", store, t, 0, 0, 1)
        slot.start()
        n = len(slot.omega)
        out = (fd.Complex * n)()
        fd.call("timefield3d_read_overlap_monitor", t, slot.mon_out, out)
        fd.call("fdtd_spline_store_unbind", store, t)
        O = complex(out[LAM0_INDEX].re, out[LAM0_INDEX].im)
        tph = math.atan2(O.imag, O.real) % (2 * B.REF_PI)
        mode = slot.mode_out.copy()
        mode.fields *= complex(math.cos(tph + B.REF_PI / 2), math.sin(tph + B.REF_PI / 2))
        fd.lib.timefield3d_zero_fields(t)
        fd.call("timefield3d_clear_monitors", t)
        omega = slot.omega[LAM0_INDEX]
        aph = np.array([(steps - k) * slot.dt * omega for k in range(steps)])
        ones = np.ones(steps)
        fd.call("timefield3d_set_source_schedule", t, s["cx"], s["cy"], nz - s["out_back"], mode.struct, 0, 1, steps,
                ones.ctypes.data_as(DP), aph.ctypes.data_as(DP))
        fd.call("fdtd_spline_store_bind", store, t, 1, steps - 1, -1)
        fd.call("timefield3d_run", t, slot.dt, steps)
        fd.call("fdtd_spline_store_unbind", store, t)
        grad = np.zeros(NCTRL)
        fd.call("fdtd_spline_store_gradient", store, s["ep_core"] - s["ep_clad"], grad.ctypes.data_as(DP), None)
    finally:
        fd.lib.fdtd_spline_store_free(store)
        slot.close()
    return grad


def optimise(fd, w0: np.ndarray, nz: int, steps: int, budget: int, step_um: float = 0.15, net: Net | None = None,
             data: tuple | None = None, finetune_epochs: int = 20, log=None) -> dict:
    """Ascend mean T from w0 within `budget` FDTD runs; surrogate steps when a
    network is given, adjoint steps otherwise (and as the fallback)."""
    w = np.asarray(w0, float).copy()
    t0 = simulate(fd, [w], nz, steps, slots=1)[0][0]
    best = float(np.mean(np.abs(t0) ** 2))
    runs = 1
    hist = [dict(run=runs, T=best, kind="start")]
    X, Y = data if data is not None else (None, None)
    fallbacks = 0
    while runs < budget:
        kind = "adjoint"
        proposal = None
        if net is not None:
            x = norm_x(w)[None]
            y = net.predict(x)
            dy = np.concatenate([2 * y[:, :NLAM], 2 * y[:, NLAM:]], axis=1) / NLAM
            g = net.input_gradient(x, dy.astype(np.float32))[0].astype(np.float64) / 1.25
            if np.abs(g).max() > 0:
                proposal = np.clip(w + step_um * g / np.abs(g).max(), W_LO, W_HI)
                t_p = simulate(fd, [proposal], nz, steps, slots=1)[0][0]
                runs += 1
                T_fd = float(np.mean(np.abs(t_p) ** 2))
                T_pred = float(mean_T_of_y(net.predict(norm_x(proposal)[None]))[0])
                X = np.concatenate([X, norm_x(proposal)[None]])
                Y = np.concatenate([Y, to_y(t_p[None])])
                net.train(X, Y, finetune_epochs, batch=min(128, len(X) // 8 * 8), seed=runs)
                kind = "surrogate"
                if abs(T_pred - T_fd) > 1e-2:
                    fallbacks += 1
                    proposal = None
                    kind = "surrogate miss -> adjoint"
        if proposal is None:
            if runs + 3 > budget:     # an adjoint step costs forward + adjoint + confirmation
                break
            g = adjoint_gradient(fd, w, nz, steps)
            runs += 2
            proposal = np.clip(w + step_um * g / max(np.abs(g).max(), 1e-30), W_LO, W_HI)
            t_p = simulate(fd, [proposal], nz, steps, slots=1)[0][0]
            runs += 1
            T_fd = float(np.mean(np.abs(t_p) ** 2))
            if X is not None:
                X = np.concatenate([X, norm_x(proposal)[None]])
                Y = np.concatenate([Y, to_y(t_p[None])])
        if T_fd > best:
            w, best = proposal, T_fd
        else:
            step_um *= 0.5
        hist.append(dict(run=runs, T=T_fd, best=best, kind=kind, step=step_um))
        if log:
            log(hist[-1])
    return dict(widths=w.tolist(), best=best, runs=runs, fallbacks=fallbacks, history=hist)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1024)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--steps", type=int, default=4451)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--budget", type=int, default=30)
    args = ap.parse_args()
    fd = importlib.import_module("3d_fdtd_b200")
    t0 = time.perf_counter()
    n_all = args.train + max(8, args.train // 8)
    widths = [random_widths(1000 + i) for i in range(n_all)]
    t, sweep = simulate(fd, widths, args.nz, args.steps)
    t_data = time.perf_counter() - t0
    X, Y = norm_x(np.array(widths)), to_y(t)
    Xtr, Ytr, Xva, Yva = X[:args.train], Y[:args.train], X[args.train:], Y[args.train:]
    net = Net(fd)
    t1 = time.perf_counter()
    loss = net.train(Xtr, Ytr, args.epochs)
    t_train = time.perf_counter() - t1
    pred = net.predict(Xva)
    T_va, T_pred = mean_T_of_y(Yva), mean_T_of_y(pred)
    start = int(np.argmax(mean_T_of_y(Ytr)))
    w0 = np.array(widths[start])
    sur = optimise(fd, w0, args.nz, args.steps, args.budget, net=net, data=(Xtr.copy(), Ytr.copy()))
    adj = optimise(fd, w0, args.nz, args.steps, args.budget)
    net.close()
    print(json.dumps(dict(
        problem=dict(grid=[256, 128, args.nz], steps=args.steps, controls=NCTRL, wavelengths=NLAM),
        data=dict(runs=n_all, seconds=t_data, mcell_updates_per_s=sweep["cell_steps"] / sweep["seconds"] / 1e6),
        training=dict(samples=args.train, epochs=args.epochs, final_loss=loss, seconds=t_train,
                      val_rmse_t=float(np.sqrt(np.mean((pred - Yva) ** 2))),
                      val_mae_meanT=float(np.mean(np.abs(T_pred - T_va)))),
        start=dict(index=start, meanT=float(mean_T_of_y(Ytr)[start])),
        surrogate=dict(best_meanT=sur["best"], fdtd_runs=sur["runs"], fallbacks=sur["fallbacks"]),
        adjoint_only=dict(best_meanT=adj["best"], fdtd_runs=adj["runs"]),
        target_meanT=0.95)), flush=True)


if __name__ == "__main__":
    main()
