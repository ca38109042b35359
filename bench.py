"""Benchmark of the FDTD hot path: the 200x160x400 Si taper (FP32, 12-cell CPML,
mode source, 11-wavelength mode-overlap monitors), one bench step = one full
6000-time-step forward simulation, through libfdtd_b200.so's C ABI.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    torchrun --nproc-per-node N bench.py --gpus N ...   (N > 1: one replica per GPU)

Prints one JSON line (rank 0).  Metric: Yee Mcell-updates/s = nx*ny*nz*time_steps
per second, whole job (all ranks).  Device timing: CUDA events on the engine's
own stream, barrier + synchronize on both sides, max over ranks.  `e2e` repeats
the step through the public API with the geometry re-rasterised on the host and
uploaded (pinned host mirrors), the mode profiles uploaded and the monitor
results read back, timed on the host clock.  `roofline` uses the Yee-update
time measured live with event pairs inside the captured graphs of the timed
runs.  `--impl reference` times the reference's own C/OpenMP step (built from
its sources into oracle/_ref) on the host cores on the same grid.
"""
from __future__ import annotations

import argparse
import ctypes as C
import gzip
import importlib
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# modes written by the reference's own solver (test fixtures): used only by the
# reference's CPU arm, which loads modes through its own mode_file_load
REF_MODES = os.path.join(ROOT, "tests", "golden", "modes")
REF_PI = 3.141592652

# ---------------------------------------------------------------------------
# the workload: Si strip taper 0.5 -> 3.0 um, 220 nm core, SiO2 cladding
# ---------------------------------------------------------------------------
W = dict(nx=200, ny=160, nz=400, dx=0.025, ep_clad=2.085, ep_core=12.1, core_y=(76, 85), cx=100, cy=80,
         w_in=(90, 110), w_out=(40, 160), taper_z=(30, 370), cpml=12, src_z=20, launch_z=25, out_z=380,
         lam0=1.55, bw=0.3, lams=[round(1.50 + 0.01 * l, 2) for l in range(11)], time_steps=6000)
KTIME_PERIOD = 8
WORKLOAD_NAME = "si_taper_200x160x400_dx25nm_cpml12_fp32_11lambda"


def cell_axes_in_pml(nx, ny, nz, L):
    return 2 * L * ny * nz + nx * 2 * L * nz + nx * ny * 2 * L


def algorithmic_bytes_per_step(nx, ny, nz, L):
    """60 B per cell (6 field components read + written, 3 E coefficients) and
    32 B per (cell, CPML axis) (4 auxiliaries read + written), FP32."""
    return 60 * nx * ny * nz + 32 * cell_axes_in_pml(nx, ny, nz, L)


def source_tables(T, dt):
    w0 = 2 * REF_PI / W["lam0"]
    dw = 2 * math.pi * W["bw"] / W["lam0"] ** 2
    sigma_n = (2 * math.sqrt(2 * math.log(2)) / dw) / dt
    n0 = 3 * sigma_n
    n = np.arange(T, dtype=np.float64)
    amp = np.exp(-((n - n0) ** 2) / (2 * sigma_n ** 2))
    phase = n * dt * w0
    return amp, phase


def rasterise(lib, t):
    """Geometry through the reference's rasterisers (timefield3d.c:1356-1535)."""
    b, top = W["core_y"]
    z0, z1 = W["taper_z"]
    lib.timefield3d_set_background(t, W["ep_clad"], 1.0)
    lib.timefield3d_set_waveguide(t, W["ep_core"], W["w_in"][0], W["w_in"][1], 0, z0, b, top)
    lib.timefield3d_set_taper(t, W["ep_core"], 1.0, W["w_in"][0], W["w_in"][1], W["w_out"][0], W["w_out"][1],
                              z0, z1, b, top)
    lib.timefield3d_set_waveguide(t, W["ep_core"], W["w_out"][0], W["w_out"][1], z1, W["nz"], b, top)


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


_MODES = {}


def taper_modes(fd):
    """TE0 modes of the taper's input (0.5 um) and output (3.0 um) strips on the
    full 200 x 160 cross-section, from the library's GPU mode solver (solved once
    per process, outside every timed region)."""
    if "taper" not in _MODES:
        modes = importlib.import_module("3d_fdtd_b200.modes")
        b, top = W["core_y"]
        out = []
        for x0, x1 in (W["w_in"], W["w_out"]):
            m, _ = modes.strip_mode(fd, W["nx"], W["ny"], W["dx"], (x0, x1, b, top), W["ep_clad"], W["ep_core"],
                                    W["lam0"], 20, 1e-8)
            out.append(m)
        _MODES["taper"] = tuple(out)
    return tuple(m.copy() for m in _MODES["taper"])


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")
        if shutil.which("nvidia-smi") is None:
            return
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if gpu_id:
            cmd += ["-i", gpu_id]
        self.fh = open(self.path, "w")
        self.proc = subprocess.Popen(cmd, stdout=self.fh, stderr=subprocess.DEVNULL)

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, v in zip(self.NAMES, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# the reference's own C (CPU baseline and --impl reference)
# ---------------------------------------------------------------------------
class ReferenceRun:
    """The reference's step + mode source + two mode overlaps per time step on the
    same grid (Mur boundary: the reference has no CPML), on `threads` cores.  The
    grid and the modes are set up once; `sample(n)` times n further time steps."""

    def __init__(self, threads: int):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from bindings import Complex, Reference
        self.R = R = Reference()
        R.set_threads(threads)
        self.threads = threads
        nx, ny, nz, dx = W["nx"], W["ny"], W["nz"], W["dx"]
        self.dt = 0.99 * dx / math.sqrt(3)
        self.tf = R.timefield3d_new(nx, ny, nz, dx)
        rasterise(R.lib, self.tf)
        tmp = tempfile.mkdtemp()
        self.modes = []
        for name in ("c1_in_te0", "c1_out_te0"):
            txt = os.path.join(tmp, name + ".txt")
            with gzip.open(os.path.join(REF_MODES, name + ".txt.gz"), "rb") as fi, open(txt, "wb") as fo:
                shutil.copyfileobj(fi, fo)
            self.modes.append(R.load_mode(txt))
        shutil.rmtree(tmp)
        self.amp, self.phase = source_tables(W["time_steps"], self.dt)
        self.acc = [Complex(), Complex()]
        self.n = 0

    def sample(self, steps: int) -> dict:
        R, tf, m = self.R, self.tf, self.modes
        t0 = time.perf_counter()
        for _ in range(steps):
            n = self.n % W["time_steps"]
            R.timefield3d_mode_source(tf, W["cx"], W["cy"], W["src_z"], m[0], self.phase[n], self.amp[n], 0)
            R.timefield3d_apply_timestep_omp_full(tf, self.dt)
            R.timefield3d_mode_overlap(tf, W["cx"], W["cy"], W["launch_z"], m[0], self.phase[n], 0,
                                       C.byref(self.acc[0]))
            R.timefield3d_mode_overlap(tf, W["cx"], W["cy"], W["out_z"], m[1], self.phase[n], 0, C.byref(self.acc[1]))
            self.n += 1
        el = time.perf_counter() - t0
        cells = W["nx"] * W["ny"] * W["nz"]
        return {"mcells": cells * steps / el / 1e6, "steps": steps, "seconds": el, "threads": self.threads}

    def close(self):
        self.R.timefield3d_free(self.tf)


REF_SAMPLE_STEPS = 50      # time steps per bench step of the reference arm
CPU_BASELINE_STEPS = 150   # time steps of the cpu_baseline leg (about 15 s on 16 cores)


def reference_threads() -> int:
    # the reference's OpenMP z-slabs must hold >= 2 planes each (timefield3d.c:2794-2848)
    return max(1, min(os.cpu_count() or 1, W["nz"] // 2))


def reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    run = ReferenceRun(reference_threads())
    run.sample(2)   # first touch of the grid's pages
    vals = []
    for s in range(args.warmup + args.steps):
        r = run.sample(REF_SAMPLE_STEPS if s >= args.warmup else 5)
        if s >= args.warmup:
            vals.append(r)
    run.close()
    v = statistics.median([r["mcells"] for r in vals])
    ms = statistics.median([r["seconds"] * 1e3 for r in vals])
    sample = f"{REF_SAMPLE_STEPS} consecutive of {W['time_steps']} time steps per bench step (grid " \
             f"{W['nx']}x{W['ny']}x{W['nz']}, reference Mur boundary, mode source + 2 overlaps per time step, " \
             "FP64 as the reference computes); ms_per_step is that sample's wall time"
    line = {"impl": "reference", "metric": "Yee Mcell-updates/s", "value": v, "unit": "Mcell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_block(args),
            "cpu_baseline": {"value": v, "unit": "Mcell-updates/s", "cores": run.threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_block(args) -> dict:
    return {"workload": WORKLOAD_NAME, "grid": [W["nx"], W["ny"], W["nz"]], "dx_um": W["dx"],
            "time_steps": args.time_steps,
            "cpml_cells": (getattr(args, "cpml_cells", None) or W["cpml"]) if getattr(args, "boundary", "cpml") == "cpml" else 0,
            "n_lambda": len(W["lams"]),
            "lambda_um": [W["lams"][0], W["lams"][-1]], "fields": "f32", "monitors": "f64 compensated",
            "taper_um": [0.5, 3.0], "taper_length_um": (W["taper_z"][1] - W["taper_z"][0]) * W["dx"],
            "l2": "inputs larger than L2 (fields 307 MB, no flush needed)",
            "parallelism": f"replicas x{args.gpus}"}


# ---------------------------------------------------------------------------
# our engine
# ---------------------------------------------------------------------------
class Taper:
    """One simulation of the workload on one GPU."""

    def __init__(self, fd, time_steps: int, variant: int = 0, precision: int | None = None, boundary: str = "cpml",
                 cpml_cells: int | None = None):
        self.fd, self.T = fd, time_steps
        lib = fd.lib
        nx, ny, nz, dx = W["nx"], W["ny"], W["nz"], W["dx"]
        self.dt = 0.99 * dx / math.sqrt(3)
        self.grid = fd.Grid(nx, ny, nz, dx, fd.F32 if precision is None else precision)
        self.t = self.grid.t
        rasterise(lib, self.t)
        self.L = W["cpml"] if cpml_cells is None else cpml_cells
        if boundary == "cpml":
            fd.call("timefield3d_set_cpml", self.t, self.L, 3, -1.0, 1.0, 0.0)
        else:   # analysis only: the same grid with PEC walls (no CPML terms)
            fd.call("timefield3d_set_boundary", self.t, fd.PEC)
        fd.call("timefield3d_set_yee_variant", self.t, variant)
        self.mode_in, self.mode_out = taper_modes(fd)
        self.amp, self.phase = source_tables(time_steps, self.dt)
        self.omega = np.array([2 * REF_PI / l for l in W["lams"]])
        fd.call("timefield3d_upload_materials", self.t)
        self.set_inputs()

    def set_inputs(self):
        fd, t = self.fd, self.t
        fd.call("timefield3d_clear_monitors", t)
        self.mon_in = fd.call("timefield3d_add_overlap_monitor", t, W["cx"], W["cy"], W["launch_z"],
                              self.mode_in.copy().struct, 0, len(self.omega), dptr(self.omega))
        self.mon_out = fd.call("timefield3d_add_overlap_monitor", t, W["cx"], W["cy"], W["out_z"],
                               self.mode_out.copy().struct, 0, len(self.omega), dptr(self.omega))
        fd.call("timefield3d_set_source_schedule", t, W["cx"], W["cy"], W["src_z"], self.mode_in.copy().struct, 0, 0,
                self.T, dptr(self.amp), dptr(self.phase))

    def h2d_bytes(self):
        n = W["nx"] * W["ny"] * W["nz"]
        # ep + mu (the rasterisers touch both), the input mode twice (source schedule,
        # launch monitor), the output mode once, the source table, the frequencies
        modes = 2 * 6 * 16 * self.mode_in.mi * self.mode_in.mj + 6 * 16 * self.mode_out.mi * self.mode_out.mj
        return 2 * 3 * 4 * n + modes + 3 * 8 * self.T + 2 * 8 * len(self.omega)

    def d2h_bytes(self):
        return 2 * 2 * 16 * len(self.omega)

    def run(self):
        self.fd.lib.timefield3d_zero_fields(self.t)
        self.fd.call("timefield3d_run", self.t, self.dt, self.T)

    def amplitude_ratio(self):
        """t(lambda) = O_out / O_in, the complex ratio the reference driver prints
        the magnitude of (3d_fdtd.c:139-142)."""
        a, b = (self.fd.Complex * len(self.omega))(), (self.fd.Complex * len(self.omega))()
        self.fd.call("timefield3d_read_overlap_monitor", self.t, self.mon_in, a)
        self.fd.call("timefield3d_read_overlap_monitor", self.t, self.mon_out, b)
        oi = np.array([complex(x.re, x.im) for x in a])
        oo = np.array([complex(x.re, x.im) for x in b])
        return oo / oi

    def transmission(self):
        return np.abs(self.amplitude_ratio()) ** 2

    def close(self):
        self.grid.close()

    def e2e_step(self):
        """Design evaluation through the public API: re-rasterise, upload, run, read."""
        rasterise(self.fd.lib, self.t)
        self.fd.call("timefield3d_upload_materials", self.t)
        self.set_inputs()
        self.run()
        return self.transmission()


def read_traffic(kernel_tag: str):
    """DRAM bytes per Yee step from the committed ncu summary of this workload, or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel_tag}.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_step:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        p = json.load(open(path))
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def our_arm(args, rank: int, world: int, local_rank: int) -> None:
    import torch
    fd = importlib.import_module("3d_fdtd_b200")
    if fd.lib.fdtd_device_count() <= 0:
        raise SystemExit("bench: no CUDA device")
    torch.cuda.set_device(local_rank)
    fd.call("fdtd_set_device", local_rank)
    ranks = importlib.import_module("3d_fdtd_b200.replicas").Ranks("nccl", timeout_s=120)
    barrier, max_over_ranks = ranks.barrier, ranks.max

    sim = Taper(fd, args.time_steps, {"auto": 0, "flat": 1, "fused": 2, "flat4": 3, "wave": 4, "stream": 5}[args.yee_variant],
                boundary=args.boundary, cpml_cells=args.cpml_cells)
    stream = torch.cuda.ExternalStream(fd.lib.timefield3d_get_stream(sim.t))
    cells = W["nx"] * W["ny"] * W["nz"]
    # warm-up: full runs (graph capture, clocks)
    for _ in range(args.warmup):
        sim.run()
    barrier()
    # timed: K full runs on the engine's stream
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    # Yee-update event pairs on one 32-step graph replay in KTIME_PERIOD (the
    # records stand between a step's kernels, so timing every replay would slow
    # the run being measured); the rest run the plain graph
    fd.call("timefield3d_set_kernel_timing", sim.t, KTIME_PERIOD)
    l0 = fd.lib.fdtd_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        sim.run()
    ev1.record(stream)
    ev1.synchronize()
    barrier()
    launches = fd.lib.fdtd_launch_count() - l0
    clk = clocks.stop()
    ktot, kcnt = C.c_double(), C.c_longlong()
    fd.call("timefield3d_read_kernel_timing", sim.t, C.byref(ktot), C.byref(kcnt))
    fd.call("timefield3d_set_kernel_timing", sim.t, 0)
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = world * cells * args.time_steps * args.steps / (ms / 1e3) / 1e6
    trans = sim.transmission()
    # roofline of the Yee update (E + H kernels with CPML), measured inside the timed runs
    kms = ktot.value / max(kcnt.value, 1)
    bytes_step = algorithmic_bytes_per_step(W["nx"], W["ny"], W["nz"], sim.L if args.boundary == "cpml" else 0)
    achieved = bytes_step / (kms / 1e3) / 1e9
    peak, peak_kind = peaks()
    wave = args.yee_variant == "wave"
    stream_kernel = args.yee_variant in ("auto", "stream")
    kernel_tag = ("yee_wave_si_taper_200x160x400_fp32" if wave else
                  "yee_stream_si_taper_200x160x400_fp32" if stream_kernel else "yee_step_si_taper_200x160x400_fp32")
    traffic = read_traffic(kernel_tag)
    # end to end through the public API, host clock
    barrier()
    sim.e2e_step()   # warm
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        trans_e2e = sim.e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = world * cells * args.time_steps * args.steps / e2e_s / 1e6
    # candidate sweep (64-candidate taper family, seeded subset): persistent
    # multi-grid launches with the tile-shape autotuner, host clock around it
    sweep = None
    if rank == 0 and world == 1 and args.sweep_candidates > 0:
        batch = importlib.import_module("3d_fdtd_b200.batch")
        cands = batch.candidates(64, seed=2)[:args.sweep_candidates]
        r = batch.sweep_persistent(fd, cands, group=len(cands))
        peak_gbs, _ = peaks()
        sweep = {"candidates": len(cands), "of": "64-candidate taper family (seed 2), first candidates",
                 "value": r["cell_steps"] / r["seconds"] / 1e6, "unit": "Mcell-updates/s",
                 "hbm_frac": r["bytes"] / r["seconds"] / 1e9 / peak_gbs, "seconds": r["seconds"],
                 "tile_shape": r["shape"], "autotune_ms_per_step": r["tuning"],
                 "launch": "persistent cooperative launches of 64 steps over all candidates, one CUDA graph"}
    # FP32 against FP64: the same workload once on the engine's FP64 path (bit-exact
    # to the CPU restatement on CPML grids), outside every timed region
    t32 = sim.amplitude_ratio()
    f64_check = None
    if not args.no_f64_check:
        ref64 = Taper(fd, args.time_steps, 0, fd.F64, boundary=args.boundary)
        ref64.run()
        t64 = ref64.amplitude_ratio()
        ref64.close()
        rel = np.abs(t32 - t64) / np.abs(t64)
        f64_check = {"rel_err_vs_f64": float(rel.max()), "per_lambda": [float(x) for x in rel],
                     "tolerance": 1e-3, "quantity": "complex t = O_out/O_in per wavelength"}
    # CPU baseline: the reference on this host's cores (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        run = ReferenceRun(reference_threads())
        run.sample(2)
        r = run.sample(CPU_BASELINE_STEPS)
        run.close()
        cpu = {"value": r["mcells"], "unit": "Mcell-updates/s", "cores": r["threads"], "kind": "reference",
               "sample": f"{r['steps']} consecutive of {W['time_steps']} time steps of the same grid in "
                         f"{r['seconds']:.1f} s (reference step with its Mur boundary, mode source and 2 overlaps "
                         "per time step, FP64)"}
    if rank == 0:
        line = {"metric": "Yee Mcell-updates/s", "value": value, "unit": "Mcell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded geometry; TE0 modes from the library's GPU mode solver on the 200x160 cross-section)",
                "config": config_block(args),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "kernel": ("wavefront launch (E, H, CPML, source, monitor partials), per step"
                                        if wave else
                                        "one-pass streaming Yee kernel (E, H, CPML terms, scheduled source), per step"
                                        if stream_kernel else "Yee step (E and H update kernels, CPML terms)"),
                             "bytes_per_launch": bytes_step, "avg_launch_ms": kms,
                             "timed_launches": kcnt.value,
                             "timed_sample": (f"one wavefront launch in {KTIME_PERIOD}" if wave else
                                              f"Yee E+H of every step of one 32-step graph replay in {KTIME_PERIOD}")},
                "cpu_baseline": cpu,
                "e2e": {"value": e2e, "unit": "Mcell-updates/s", "h2d_bytes_per_step": sim.h2d_bytes(),
                        "d2h_bytes_per_step": sim.d2h_bytes()},
                "gpu_launches": launches, "clocks": clk, "sweep": sweep,
                "transmission": {"lambda_um": W["lams"], "T": [round(float(x), 6) for x in trans],
                                 "T_e2e_equal": bool(np.allclose(trans, trans_e2e, rtol=1e-6)),
                                 **(f64_check or {})}}
        print(json.dumps(line), flush=True)
    ranks.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--time-steps", type=int, default=W["time_steps"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-f64-check", action="store_true", help="skip the FP64 run that checks the FP32 transmission")
    ap.add_argument("--sweep-candidates", type=int, default=8,
                    help="candidates of the taper family in the sweep measurement (0: skip)")
    ap.add_argument("--cpml-cells", type=int, default=None,
                    help="analysis only: CPML thickness other than the workload's 12 cells")
    ap.add_argument("--boundary", choices=["cpml", "pec"], default="cpml",
                    help="pec: analysis of the update without CPML terms (not the bench workload)")
    ap.add_argument("--yee-variant", choices=["auto", "flat", "flat4", "fused", "wave", "stream"], default="auto")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.gpus != world and world > 1:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE {world}")
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    our_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
