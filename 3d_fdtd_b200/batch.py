"""Candidate sweeps: many independent taper simulations, concurrently on one
GPU and split over GPUs.

A candidate is the Si strip taper of the single-run workload (SiO2 2.085, Si
12.1, 9-row (225 nm) core, 25 nm grid, 12-cell CPML, TE0 source and 11
wavelength overlap monitors) with its own length and shape:
  L ~ U(5, 20) um, widths: 20 values ~ U(0.5, 3.0) um sorted ascending (seed 2);
  grid (256, 128, nz), nz = 96 + round(288 (L - 5) / 15);
  time steps 4000 + round(4000 (L - 5) / 15);
  input waveguide 0.5 um for z < 30, spline taper (natural cubic spline
  through the widths, sub-pixel fill) on z in [30, nz - 30), output waveguide
  3.0 um after; source plane z = 20, launch monitor z = 25, output monitor
  z = nz - 20.
The physical taper is shorter than L (nz - 60 cells of 25 nm): the grid size
and step count follow L, the geometry is scaled to fit, like the single-run
workload.

Runner: `slots` candidates are resident at a time, each with its own grid,
CUDA stream and captured graphs; their runs are queued and overlap on the GPU
while the host prepares the next candidate of a finished slot (grids are
reused when the shape repeats).  Every candidate's result is the same, bit for
bit, as running it alone.  An autotuner times the Yee kernel designs
(streaming, flat4, flat, fused) on each grid shape with the in-graph kernel
timers and keeps the fastest.  Across GPUs the candidates are split by replicas.Ranks (rank r runs
r, r + N, ...) and the transmissions gathered to every rank.

    python -m 3d_fdtd_b200.batch [--candidates 64] [--slots 4]
    torchrun --nproc-per-node N -m 3d_fdtd_b200.batch ...
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

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_PI = 3.141592652
DP = C.POINTER(C.c_double)

SPEC = dict(nx=256, ny=128, dx=0.025, ep_clad=2.085, ep_core=12.1, core_y=(60, 69), cx=128, cy=64,
            w_in=(118, 138), w_out=(68, 188), cpml=12, src_z=20, launch_z=25, margin=30, out_back=20,
            lam0=1.55, bw=0.3, lams=[round(1.50 + 0.01 * i, 2) for i in range(11)])


def candidates(n: int = 64, seed: int = 2, ncontrol: int = 20, steps_scale: float = 1.0) -> list[dict]:
    """The seeded candidate list (index, L, nz, steps, widths)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L = float(rng.uniform(5.0, 20.0))
        widths = np.sort(rng.uniform(0.5, 3.0, ncontrol))
        nz = 96 + int(round(288 * (L - 5) / 15))
        steps = 4000 + int(round(4000 * (L - 5) / 15))
        out.append(dict(index=i, L=L, nz=nz, steps=max(1, int(round(steps * steps_scale))), widths=widths))
    return out


def algorithmic_bytes(nx: int, ny: int, nz: int, L: int) -> int:
    """Per time step: 60 B per cell + 32 B per (cell, CPML axis), FP32."""
    return 60 * nx * ny * nz + 32 * (2 * L * ny * nz + nx * 2 * L * nz + nx * ny * 2 * L)


def source_tables(T: int, dt: float):
    w0 = 2 * REF_PI / SPEC["lam0"]
    dw = 2 * math.pi * SPEC["bw"] / SPEC["lam0"] ** 2
    sigma_n = (2 * math.sqrt(2 * math.log(2)) / dw) / dt
    n = np.arange(T, dtype=np.float64)
    return np.exp(-((n - 3 * sigma_n) ** 2) / (2 * sigma_n ** 2)), n * dt * w0


_MODES = {}


def candidate_modes(fd):
    """TE0 modes of the 0.5 um input and 3.0 um output strips on the candidates'
    256 x 128 cross-section, from the library's GPU mode solver (once per process)."""
    if "c" not in _MODES:
        modes = importlib.import_module("3d_fdtd_b200.modes")
        s = SPEC
        b, top = s["core_y"]
        _MODES["c"] = tuple(modes.strip_mode(fd, s["nx"], s["ny"], s["dx"], (x0, x1, b, top), s["ep_clad"],
                                             s["ep_core"], s["lam0"], 20, 1e-8)[0]
                            for x0, x1 in (s["w_in"], s["w_out"]))
    return tuple(m.copy() for m in _MODES["c"])


class Slot:
    """One resident simulation: a grid, its modes, monitors and source schedule."""

    def __init__(self, fd):
        self.fd = fd
        self.grid = None
        self.shape = None
        self.cand = None
        self.variant = 0
        self.mode_in, self.mode_out = candidate_modes(fd)
        self.omega = np.array([2 * REF_PI / l for l in SPEC["lams"]])

    def prepare(self, cand: dict, variant: int = 0, retire: list | None = None) -> None:
        """Set the slot up for `cand`.  A grid of another shape is handed to
        `retire` (closed later by the caller) instead of being freed here:
        freeing device memory waits for the whole GPU, which would stall the
        other slots' runs."""
        fd, s = self.fd, SPEC
        shape = (s["nx"], s["ny"], cand["nz"])
        if self.shape != shape:
            if self.grid is not None:
                if retire is None:
                    self.grid.close()
                else:
                    retire.append(self.grid)
            self.grid = fd.Grid(*shape, s["dx"], fd.F32)
            self.shape = shape
        t, lib, nz = self.grid.t, fd.lib, cand["nz"]
        b, top = s["core_y"]
        z0, z1 = s["margin"], nz - s["margin"]
        lib.timefield3d_set_background(t, s["ep_clad"], 1.0)
        lib.timefield3d_set_waveguide(t, s["ep_core"], s["w_in"][0], s["w_in"][1], 0, z0, b, top)
        lib.timefield3d_set_waveguide(t, s["ep_core"], s["w_out"][0], s["w_out"][1], z1, nz, b, top)
        w = np.ascontiguousarray(cand["widths"], float)
        fd.call("timefield3d_set_spline_taper", t, s["ep_core"], 1.0, len(w), w.ctypes.data_as(DP), float(s["cx"]),
                z0, z1, b, top)
        fd.call("timefield3d_set_cpml", t, s["cpml"], 3, -1.0, 1.0, 0.0)
        fd.call("timefield3d_set_yee_variant", t, variant)
        self.variant = variant
        self.dt = 0.99 * s["dx"] / math.sqrt(3)
        self.T = cand["steps"]
        self.amp, self.phase = source_tables(self.T, self.dt)
        fd.call("timefield3d_clear_monitors", t)
        self.mon_in = fd.call("timefield3d_add_overlap_monitor", t, s["cx"], s["cy"], s["launch_z"],
                              self.mode_in.copy().struct, 0, len(self.omega), self.omega.ctypes.data_as(DP))
        self.mon_out = fd.call("timefield3d_add_overlap_monitor", t, s["cx"], s["cy"], nz - s["out_back"],
                               self.mode_out.copy().struct, 0, len(self.omega), self.omega.ctypes.data_as(DP))
        fd.call("timefield3d_set_source_schedule", t, s["cx"], s["cy"], s["src_z"], self.mode_in.copy().struct, 0, 0,
                self.T, self.amp.ctypes.data_as(DP), self.phase.ctypes.data_as(DP))
        fd.call("timefield3d_upload_materials", t)
        self.cand = cand

    def start(self) -> None:
        """Queue the whole run on this slot's stream; returns at once."""
        self.fd.lib.timefield3d_zero_fields(self.grid.t)
        self.fd.call("timefield3d_run", self.grid.t, self.dt, self.T)

    def amplitudes(self) -> np.ndarray:
        """Waits for this slot's run; complex t(lambda) = O_out / O_in."""
        fd, n = self.fd, len(self.omega)
        a, b = (fd.Complex * n)(), (fd.Complex * n)()
        fd.call("timefield3d_read_overlap_monitor", self.grid.t, self.mon_in, a)
        fd.call("timefield3d_read_overlap_monitor", self.grid.t, self.mon_out, b)
        oi = np.array([complex(x.re, x.im) for x in a])
        oo = np.array([complex(x.re, x.im) for x in b])
        return oo / oi

    def transmission(self) -> np.ndarray:
        """Waits for this slot's run; T(lambda) = |O_out / O_in|^2."""
        return np.abs(self.amplitudes()) ** 2

    def close(self):
        if self.grid is not None:
            self.grid.close()
            self.grid = None


def autotune(fd, cand: dict, steps: int = 64) -> tuple[int, dict]:
    """Fastest Yee kernel design for this candidate's grid shape (in-graph
    kernel timers over `steps` steps after a warm-up run)."""
    slot = Slot(fd)
    times = {}
    short = dict(cand, steps=steps)
    for variant in (fd.YEE_STREAM, fd.YEE_FLAT4, fd.YEE_FLAT, fd.YEE_FUSED):
        slot.prepare(short, variant)
        slot.start()
        slot.transmission()
        fd.call("timefield3d_set_kernel_timing", slot.grid.t, 1)
        slot.start()
        slot.transmission()
        ms, cnt = C.c_double(), C.c_longlong()
        fd.call("timefield3d_read_kernel_timing", slot.grid.t, C.byref(ms), C.byref(cnt))
        fd.call("timefield3d_set_kernel_timing", slot.grid.t, 0)
        if cnt.value > 0:
            times[variant] = ms.value / cnt.value
    slot.close()
    best = min(times, key=times.get)
    return best, times


def sweep(fd, cands: list[dict], slots: int = 4, variant: int | None = None, retire_gb: float = 100.0) -> dict:
    """Run every candidate, `slots` at a time; returns index -> T(lambda) and timing.
    Finished grids are kept (not freed) until about `retire_gb` of device
    memory is held by them, then freed together."""
    if not cands:
        return dict(results={}, amplitudes={}, seconds=0.0, cell_steps=0, bytes=0, variant=variant, tuning={})
    tuning = {}
    if variant is None:
        variant, tuning = autotune(fd, cands[0])
    pool = [Slot(fd) for _ in range(min(slots, len(cands)))]
    queue = list(cands)
    busy = []
    retired = []

    def prepare(slot, cand):
        slot.prepare(cand, variant, retired)
        held = sum(g.nx * g.ny * g.nz for g in retired) * 100   # ~100 B of device memory per cell
        if held > retire_gb * 1e9:
            for g in retired:
                g.close()
            retired.clear()

    results = {}
    amplitudes = {}
    cell_steps = 0
    nbytes = 0
    t0 = time.perf_counter()
    for slot in pool:
        if not queue:
            break
        prepare(slot, queue.pop(0))
        slot.start()
        busy.append(slot)
    while busy:
        slot = busy.pop(0)
        c = slot.cand
        t = slot.amplitudes()
        amplitudes[c["index"]] = t
        results[c["index"]] = (np.abs(t) ** 2).tolist()
        nx, ny, nz = slot.shape
        cell_steps += nx * ny * nz * c["steps"]
        nbytes += algorithmic_bytes(nx, ny, nz, SPEC["cpml"]) * c["steps"]
        if queue:
            prepare(slot, queue.pop(0))
            slot.start()
            busy.append(slot)
    seconds = time.perf_counter() - t0
    for slot in pool:
        slot.close()
    for g in retired:
        g.close()
    return dict(results=results, amplitudes=amplitudes, seconds=seconds, cell_steps=cell_steps, bytes=nbytes,
                variant=variant, tuning={int(k): v for k, v in tuning.items()})


def _sweep_call(fd, slots, nsteps, steps_per_launch, band_rows, tiles_per_sm):
    grids = (fd.Timefield3d * len(slots))(*[s.grid.t for s in slots])
    n = (C.c_int * len(slots))(*nsteps)
    fd.call("fdtd_sweep_run", grids, len(slots), slots[0].dt, n, steps_per_launch, band_rows, tiles_per_sm)


def autotune_tiles(fd, cands: list[dict], steps: int = 128, steps_per_launch: int = 64,
                   shapes=((0, 2.0), (0, 4.0), (0, 8.0), (4, 4.0), (3, 4.0))) -> tuple[tuple[int, float], dict]:
    """Tile shape of the persistent sweep: for each (band rows cap, tiles per
    SM) the sweep of these candidates runs `steps` steps after a warm-up, timed
    on the host around a synchronised call; the fastest shape is returned."""
    slots = []
    for c in cands:
        s = Slot(fd)
        s.prepare(dict(c, steps=max(c["steps"], steps)), fd.YEE_STREAM)
        slots.append(s)
    times = {}
    for shape in shapes:
        for s in slots:
            fd.lib.timefield3d_zero_fields(s.grid.t)
        _sweep_call(fd, slots, [steps_per_launch] * len(slots), steps_per_launch, *shape)   # warm-up (graph, plan)
        for s in slots:
            fd.call("timefield3d_synchronize", s.grid.t)
        t0 = time.perf_counter()
        _sweep_call(fd, slots, [steps] * len(slots), steps_per_launch, *shape)
        for s in slots:
            fd.call("timefield3d_synchronize", s.grid.t)
        times[shape] = (time.perf_counter() - t0) / steps * 1e3
    for s in slots:
        s.close()
    best = min(times, key=times.get)
    return best, times


def sweep_persistent(fd, cands: list[dict], group: int = 8, steps_per_launch: int = 64,
                     shape: tuple[int, float] | None = None) -> dict:
    """Every candidate through persistent sweep launches: candidates sorted by
    step count, `group` at a time advance together (uneven lengths inside the
    launches); the next group is set up on the host while the current one runs."""
    if not cands:
        return dict(results={}, amplitudes={}, seconds=0.0, cell_steps=0, bytes=0, shape=None, tuning={})
    order = sorted(cands, key=lambda c: c["steps"])
    groups = [order[i:i + group] for i in range(0, len(order), group)]
    tuning = {}
    if shape is None:
        shape, tuning = autotune_tiles(fd, groups[-1][:group])
    results, amplitudes = {}, {}
    cell_steps = nbytes = 0
    t0 = time.perf_counter()
    current = []
    for c in groups[0]:
        s = Slot(fd)
        s.prepare(c, fd.YEE_STREAM)
        fd.lib.timefield3d_zero_fields(s.grid.t)
        current.append(s)
    for gi in range(len(groups)):
        _sweep_call(fd, current, [s.cand["steps"] for s in current], steps_per_launch, *shape)
        nxt = []
        if gi + 1 < len(groups):
            for c in groups[gi + 1]:
                s = Slot(fd)
                s.prepare(c, fd.YEE_STREAM)
                fd.lib.timefield3d_zero_fields(s.grid.t)
                nxt.append(s)
        for s in current:
            c = s.cand
            t = s.amplitudes()
            amplitudes[c["index"]] = t
            results[c["index"]] = (np.abs(t) ** 2).tolist()
            nx, ny, nz = s.shape
            cell_steps += nx * ny * nz * c["steps"]
            nbytes += algorithmic_bytes(nx, ny, nz, SPEC["cpml"]) * c["steps"]
        for s in current:
            s.close()
        current = nxt
    seconds = time.perf_counter() - t0
    return dict(results=results, amplitudes=amplitudes, seconds=seconds, cell_steps=cell_steps, bytes=nbytes,
                shape=list(shape), tuning={f"{k[0]}x{k[1]}": v for k, v in tuning.items()})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--candidates", type=int, default=64)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--steps-scale", type=float, default=1.0)
    ap.add_argument("--mode", choices=["persistent", "slots"], default="persistent",
                    help="persistent: groups of candidates in persistent sweep launches; slots: one run per slot")
    ap.add_argument("--group", type=int, default=8)
    args = ap.parse_args()
    import torch

    fd = importlib.import_module("3d_fdtd_b200")
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local_rank)
    fd.call("fdtd_set_device", local_rank)
    Ranks = importlib.import_module("3d_fdtd_b200.replicas").Ranks
    ranks = Ranks("nccl" if int(os.environ.get("WORLD_SIZE", 1)) > 1 else "gloo")
    cands = candidates(args.candidates, args.seed, steps_scale=args.steps_scale)
    mine = [cands[i] for i in ranks.shard(len(cands))]
    ranks.barrier()
    if args.mode == "persistent":
        r = sweep_persistent(fd, mine, args.group)
        r["variant"] = "persistent sweep"
    else:
        r = sweep(fd, mine, args.slots)
    seconds = ranks.max(r["seconds"])
    per_rank = ranks.gather(dict(cell_steps=r["cell_steps"], bytes=r["bytes"]))
    T = ranks.gather_shards(len(cands), r["results"])
    if ranks.rank == 0:
        cell_steps = sum(p["cell_steps"] for p in per_rank)
        nbytes = sum(p["bytes"] for p in per_rank)
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"] \
            if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0
        line = dict(metric="candidate sweep Yee Mcell-updates/s", value=cell_steps / seconds / 1e6,
                    unit="Mcell-updates/s", n_gpus=ranks.world, candidates=len(cands), seconds=seconds,
                    hbm_frac=nbytes / seconds / 1e9 / (peak * ranks.world), slots=args.slots,
                    mode=args.mode, group=args.group, tile_shape=r.get("shape"),
                    variant=r["variant"], tuning_ms_per_step=r["tuning"],
                    T_mean_1550=float(np.mean([t[5] for t in T])),
                    T_best_1550=float(np.max([t[5] for t in T])))
        print(json.dumps(line), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
