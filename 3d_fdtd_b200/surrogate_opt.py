"""Surrogate-assisted taper optimisation: a tensor-core MLP trained on
simulations from the candidate runner proposes designs, every proposal is
confirmed by an FDTD run, against an adjoint-only optimiser with the same
budget of FDTD runs.

Design: the spline taper of batch.py (20 control widths in [0.5, 3.0] um,
natural cubic spline, sub-pixel fill) on one fixed grid of the candidate
family (256 x 128 x nz, 25 nm, 12-cell CPML).  Outputs: the complex
transmission t(lambda) = O_out / O_in at the 11 monitor wavelengths
1.50..1.60 um as (Re, Im) -> 22 network outputs; T = |t|^2.
Objective: mean T over the 11 wavelengths.

The arms start from the best design of the training set, share the budget of
FDTD runs and are timed by the host clock:
- adjoint-only, the reference driver's method (3d_fdtd.c:97-187): a forward
  run with the taper's edge store bound, the phase-reversed CW adjoint at
  1.55 um, the spline-weighted edge gradient of |O_out|
  (fdtd_spline_store_gradient), a step of fixed length along it; the forward
  run at the proposal confirms the step and gives the next gradient, so a
  step costs two runs; a step that does not improve is retried at half length.
- surrogate: ascent of the predicted objective on the network from 64 starts
  in a trust region around the current design (batched forward and input
  gradient calls), the k best distinct proposals simulated concurrently on k
  slots of the candidate runner, the simulated points added to the training
  set and the network fine-tuned; the region grows after an improvement and
  shrinks after a miss.
- adjoint steps sized by the surrogate: the adjoint arm's directions, with the
  step length along each chosen by the network's prediction (the network
  fine-tuned on every simulated point).
Reported: best objective against FDTD runs and wall time per arm, the time
each arm takes to reach the adjoint arm's final best, the validation error of
t against the training-set size, and the data-generation time (the fixed cost
the surrogate pays once per design family).

    python -m 3d_fdtd_b200.surrogate_opt [--train 1024] [--budget 32] [--k 4]
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import math
import os
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
    """FDTD of every design (concurrent, default kernel design); returns
    complex t [n, 11] and the runner's record."""
    cands = [design(w, i, nz, steps) for i, w in enumerate(widths_list)]
    r = B.sweep(fd, cands, slots=max(1, min(slots, len(cands))), variant=fd.YEE_AUTO)
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

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.fd.lib.fdtd_mlp_param_count(self.h), np.float32)
        self.fd.call("fdtd_mlp_get_params", self.h, p.ctypes.data_as(FP))
        return p

    def set_params(self, p: np.ndarray) -> None:
        """Weights from get_params (the optimiser state restarts)."""
        p = np.ascontiguousarray(p, np.float32)
        self.fd.call("fdtd_mlp_set_params", self.h, p.ctypes.data_as(FP))

    def train(self, x: np.ndarray, y: np.ndarray, epochs: int, batch: int = 128, lr: float = 1e-3,
              lr_end: float | None = None, seed: int = 0) -> float:
        """Adam over shuffled minibatches; with lr_end the rate follows a
        cosine from lr to lr_end over the epochs."""
        rng = np.random.default_rng(seed)
        n = len(x)
        bs = min(batch, n // 8 * 8)
        loss = C.c_double()
        last = float("nan")
        for ep in range(epochs):
            rate = lr if lr_end is None else lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * ep / epochs))
            order = rng.permutation(n)
            for s in range(0, n - bs + 1, bs):
                idx = order[s:s + bs]
                xb, yb = np.ascontiguousarray(x[idx], np.float32), np.ascontiguousarray(y[idx], np.float32)
                self.fd.call("fdtd_mlp_train_step", self.h, xb.ctypes.data_as(FP), yb.ctypes.data_as(FP), bs,
                             C.c_float(rate), C.byref(loss))
                last = loss.value
        return last


def to_y(t: np.ndarray) -> np.ndarray:
    return np.concatenate([t.real, t.imag], axis=-1).astype(np.float32)


def mean_T_of_y(y: np.ndarray) -> np.ndarray:
    return (y[..., :NLAM] ** 2 + y[..., NLAM:] ** 2).mean(axis=-1)


def mean_T(t: np.ndarray) -> float:
    return float(np.mean(np.abs(t) ** 2))


def adjoint_gradient(fd, widths: np.ndarray, nz: int, steps: int):
    """(gradient, t): the spline-weighted adjoint gradient of |O_out(1.55 um)|
    with respect to the widths (a direction: the reference's formula omits a
    global constant), and the forward run's complex t(lambda)."""
    s = B.SPEC
    cand = design(widths, 0, nz, steps)
    slot = B.Slot(fd)
    slot.prepare(cand, fd.YEE_AUTO)
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
        amp = slot.amplitudes()
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
    return grad, amp


def optimise_adjoint(fd, w0: np.ndarray, nz: int, steps: int, budget: int, step_um: float = 0.15,
                     log=None) -> dict:
    """Adjoint-only ascent from w0 within `budget` FDTD runs (2 per step)."""
    clock = time.perf_counter()
    w = np.asarray(w0, float).copy()
    g, t = adjoint_gradient(fd, w, nz, steps)
    runs, best = 2, mean_T(t)
    hist = [dict(run=runs, T=best, best=best, seconds=time.perf_counter() - clock, kind="start")]
    while runs + 2 <= budget:
        proposal = np.clip(w + step_um * g / max(np.abs(g).max(), 1e-30), W_LO, W_HI)
        g_p, t_p = adjoint_gradient(fd, proposal, nz, steps)
        runs += 2
        T_p = mean_T(t_p)
        if T_p > best:
            w, best, g = proposal, T_p, g_p
        else:
            step_um *= 0.5
        hist.append(dict(run=runs, T=T_p, best=best, seconds=time.perf_counter() - clock, kind="adjoint",
                         step=step_um))
        if log:
            log(hist[-1])
    return dict(widths=w.tolist(), best=best, runs=runs, seconds=time.perf_counter() - clock, history=hist)


STEP_LENGTHS = (0.025, 0.05, 0.1, 0.15, 0.2, 0.3, 0.45, 0.6)


def optimise_hybrid(fd, net: Net, data: tuple, w0: np.ndarray, nz: int, steps: int, budget: int,
                    finetune_epochs: int = 20, log=None) -> dict:
    """Adjoint directions, step lengths chosen by the network: along each
    adjoint direction the network predicts mean T at STEP_LENGTHS (times a
    trust factor, halved after a step that does not improve) and the best is
    simulated; the simulated point joins the training set.  2 runs a step, as
    the adjoint-only arm."""
    clock = time.perf_counter()
    X, Y = data
    w = np.asarray(w0, float).copy()
    g, t = adjoint_gradient(fd, w, nz, steps)
    runs, best, trust = 2, mean_T(t), 1.0
    hist = [dict(run=runs, T=best, best=best, seconds=time.perf_counter() - clock, kind="start")]
    while runs + 2 <= budget:
        d = g / max(np.abs(g).max(), 1e-30)
        cands = np.array([np.clip(w + trust * s * d, W_LO, W_HI) for s in STEP_LENGTHS])
        pred = mean_T_of_y(net.predict(norm_x(cands)))
        proposal = cands[int(np.argmax(pred))]
        g_p, t_p = adjoint_gradient(fd, proposal, nz, steps)
        runs += 2
        T_p = mean_T(t_p)
        X = np.concatenate([X, norm_x(proposal)[None]])
        Y = np.concatenate([Y, to_y(t_p[None])])
        net.train(X, Y, finetune_epochs, batch=min(128, len(X) // 8 * 8), lr=3e-4, seed=runs)
        if T_p > best:
            w, best, g = proposal, T_p, g_p
        else:
            trust *= 0.5
        hist.append(dict(run=runs, T=T_p, pred=float(pred.max()), best=best, seconds=time.perf_counter() - clock,
                         kind="hybrid", trust=trust))
        if log:
            log(hist[-1])
    return dict(widths=w.tolist(), best=best, runs=runs, seconds=time.perf_counter() - clock, history=hist)


def surrogate_proposals(net: Net, w: np.ndarray, radius: float, k: int, rng, starts: int = 64,
                        substeps: int = 20) -> np.ndarray:
    """Up to k distinct designs (apart by more than radius/10 in some width)
    of highest predicted mean T, found by ascending the network's prediction
    from `starts` points of the box |x - w| <= radius (per width, within the
    bounds); the first start is w itself."""
    lo, hi = np.maximum(w - radius, W_LO), np.minimum(w + radius, W_HI)
    x = np.clip(w + rng.uniform(-radius, radius, (starts, NCTRL)), lo, hi)
    x[0] = w
    step = radius / substeps
    for _ in range(substeps):
        y = net.predict(norm_x(x))
        dy = np.concatenate([2 * y[:, :NLAM], 2 * y[:, NLAM:]], axis=1) / NLAM
        g = net.input_gradient(norm_x(x), dy.astype(np.float32)).astype(np.float64)
        g /= np.maximum(np.abs(g).max(axis=1, keepdims=True), 1e-30)
        x = np.clip(x + step * g, lo, hi)
    pred = mean_T_of_y(net.predict(norm_x(x)))
    chosen = []
    for i in np.argsort(-pred):
        if all(np.abs(x[i] - x[c]).max() > radius / 10 for c in chosen):
            chosen.append(i)
        if len(chosen) == k:
            break
    return x[chosen]


def optimise_surrogate(fd, net: Net, data: tuple, w0: np.ndarray, T0: float, nz: int, steps: int, budget: int,
                       k: int = 4, radius: float = 0.3, finetune_epochs: int = 20, seed: int = 0, log=None) -> dict:
    """Surrogate-proposal ascent from w0 (mean T T0, already simulated: a
    training design) within `budget` FDTD runs, k concurrent runs a round."""
    clock = time.perf_counter()
    rng = np.random.default_rng(seed)
    X, Y = data
    w, best, runs = np.asarray(w0, float).copy(), float(T0), 0
    hist = [dict(run=0, T=best, best=best, seconds=0.0, kind="start")]
    while runs + k <= budget:
        props = surrogate_proposals(net, w, radius, k, rng)
        pred = mean_T_of_y(net.predict(norm_x(props)))
        t_p, _ = simulate(fd, list(props), nz, steps, slots=len(props))
        runs += len(props)
        T_p = np.mean(np.abs(t_p) ** 2, axis=1)
        X = np.concatenate([X, norm_x(props)])
        Y = np.concatenate([Y, to_y(t_p)])
        net.train(X, Y, finetune_epochs, batch=min(128, len(X) // 8 * 8), lr=3e-4, seed=runs)
        i = int(np.argmax(T_p))
        if T_p[i] > best:
            w, best = props[i].copy(), float(T_p[i])
            radius = min(1.5 * radius, 0.6)
        else:
            radius *= 0.5
        hist.append(dict(run=runs, T=float(T_p[i]), pred=float(pred[i]), best=best, radius=radius,
                         seconds=time.perf_counter() - clock, kind="surrogate"))
        if log:
            log(hist[-1])
    return dict(widths=w.tolist(), best=best, runs=runs, seconds=time.perf_counter() - clock, history=hist)


def time_to(result: dict, target: float):
    """(seconds, FDTD runs) at which an arm's best first reached `target`, or None."""
    for h in result["history"]:
        if h["best"] >= target - 1e-12:
            return h["seconds"], h["run"]
    return None


def training_data(fd, n: int, nz: int, steps: int, cache: str | None):
    """n seeded designs (seeds 1000..) and their simulated t, from the cache
    file when it holds the same problem."""
    widths = np.array([random_widths(1000 + i) for i in range(n)])
    if cache and os.path.exists(cache):
        z = np.load(cache)
        if int(z["nz"]) == nz and int(z["steps"]) == steps and len(z["t"]) >= n and \
                np.array_equal(z["widths"][:n], widths):
            return widths, z["t"][:n], dict(seconds=float(z["seconds"]) * n / len(z["t"]), cached=True,
                                            mcell_updates_per_s=float(z["rate"]))
    t0 = time.perf_counter()
    t, sweep = simulate(fd, list(widths), nz, steps)
    seconds = time.perf_counter() - t0
    rate = sweep["cell_steps"] / sweep["seconds"] / 1e6
    if cache:
        np.savez(cache, widths=widths, t=t, nz=nz, steps=steps, seconds=seconds, rate=rate)
    return widths, t, dict(seconds=seconds, cached=False, mcell_updates_per_s=rate)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1024)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--steps", type=int, default=4451)
    ap.add_argument("--epochs", type=int, default=1000)
    ap.add_argument("--budget", type=int, default=32)
    ap.add_argument("--k", type=int, default=4, help="surrogate proposals simulated together per round")
    ap.add_argument("--sizes", default="128,256,512", help="smaller training sets for the accuracy curve")
    ap.add_argument("--data", default=None, help="npz cache of the training simulations")
    args = ap.parse_args()
    fd = importlib.import_module("3d_fdtd_b200")
    n_val = max(8, args.train // 8)
    widths, t, gen = training_data(fd, args.train + n_val, args.nz, args.steps, args.data)
    X, Y = norm_x(widths), to_y(t)
    Xtr, Ytr, Xva, Yva = X[:args.train], Y[:args.train], X[args.train:], Y[args.train:]

    def fit(n):
        net = Net(fd)
        t1 = time.perf_counter()
        loss = net.train(Xtr[:n], Ytr[:n], args.epochs, lr=1e-3, lr_end=1e-5)
        pred = net.predict(Xva)
        return net, dict(samples=n, final_loss=loss, seconds=time.perf_counter() - t1,
                         val_rmse_t=float(np.sqrt(np.mean((pred - Yva) ** 2))),
                         val_mae_meanT=float(np.mean(np.abs(mean_T_of_y(pred) - mean_T_of_y(Yva)))))

    by_size = []
    for n in sorted({int(v) for v in args.sizes.split(",") if v} - {args.train}):
        if 8 <= n < args.train:
            net_n, rec = fit(n)
            net_n.close()
            by_size.append(rec)
    net, rec = fit(args.train)
    by_size.append(rec)
    start = int(np.argmax(mean_T_of_y(Ytr)))
    w0, T0 = widths[start], float(mean_T_of_y(Ytr)[start])
    params = net.get_params()
    adj = optimise_adjoint(fd, w0, args.nz, args.steps, args.budget)
    sur = optimise_surrogate(fd, net, (Xtr.copy(), Ytr.copy()), w0, T0, args.nz, args.steps, args.budget, k=args.k)
    net.set_params(params)
    hyb = optimise_hybrid(fd, net, (Xtr.copy(), Ytr.copy()), w0, args.nz, args.steps, args.budget)
    net.close()
    target = adj["best"]

    def arm(r, **extra):
        return dict(best_meanT=r["best"], fdtd_runs=r["runs"], seconds=r["seconds"], **extra,
                    curve=[(h["run"], round(h["seconds"], 3), h["best"]) for h in r["history"]])

    def reach(r):
        x = time_to(r, target)
        return None if x is None else dict(seconds=x[0], runs=x[1])
    print(json.dumps(dict(
        problem=dict(grid=[256, 128, args.nz], steps=args.steps, controls=NCTRL, wavelengths=NLAM),
        data=dict(runs=len(widths), **gen),
        training=dict(epochs=args.epochs, by_size=by_size),
        start=dict(index=start, meanT=T0),
        adjoint_only=arm(adj),
        surrogate=arm(sur, k=args.k),
        adjoint_steps_sized_by_surrogate=arm(hyb),
        time_to_adjoint_best=dict(target_meanT=target, adjoint_only=reach(adj), surrogate=reach(sur),
                                  adjoint_steps_sized_by_surrogate=reach(hyb)),
        target_meanT=0.95)), flush=True)


if __name__ == "__main__":
    main()
