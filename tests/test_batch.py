"""Candidate sweeps (3d_fdtd_b200/batch.py): seeded candidate list, and on the
GPU: every candidate's transmission from a concurrent sweep equals the same
candidate simulated alone, bit for bit; the autotuner times every design."""
from __future__ import annotations

import importlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def B():
    return importlib.import_module("3d_fdtd_b200.batch")


def test_candidates_follow_the_spec(B):
    cands = B.candidates(64, seed=2)
    again = B.candidates(64, seed=2)
    assert all(a["L"] == b["L"] and np.array_equal(a["widths"], b["widths"]) for a, b in zip(cands, again))
    for c in cands:
        assert 5.0 <= c["L"] <= 20.0
        assert c["nz"] == 96 + round(288 * (c["L"] - 5) / 15)
        assert c["steps"] == 4000 + round(4000 * (c["L"] - 5) / 15)
        w = c["widths"]
        assert len(w) == 20 and np.all(np.diff(w) >= 0) and w[0] >= 0.5 and w[-1] <= 3.0
    assert len({c["nz"] for c in cands}) > 10


def test_algorithmic_bytes_formula(B):
    # 60 B per cell + 32 B per (cell, CPML axis); the single-run workload's 903.2 MB
    assert B.algorithmic_bytes(200, 160, 400, 12) == 903_168_000


@pytest.mark.gpu
def test_sweep_equals_single_runs(fd, gpu, B):
    cands = B.candidates(3, seed=2)      # full step counts: the pulse must reach the output
    r = B.sweep(fd, cands, slots=3, variant=fd.YEE_FLAT4)
    assert sorted(r["results"]) == [0, 1, 2]
    for c in cands:
        s = B.Slot(fd)
        s.prepare(c, fd.YEE_FLAT4)
        s.start()
        alone = s.transmission()
        s.close()
        got = np.array(r["results"][c["index"]])
        assert np.all(np.isfinite(got)) and 0.05 < got.max() < 1.5
        assert np.array_equal(got, alone)
    assert r["cell_steps"] == sum(256 * 128 * c["nz"] * c["steps"] for c in cands)


@pytest.mark.gpu
def test_autotune_times_each_design(fd, gpu, B):
    c = B.candidates(1, seed=2)[0]
    best, times = B.autotune(fd, c, steps=32)
    assert set(times) == {fd.YEE_STREAM, fd.YEE_FLAT4, fd.YEE_FLAT, fd.YEE_FUSED}
    assert best == min(times, key=times.get) and all(v > 0 for v in times.values())


@pytest.mark.gpu
def test_persistent_sweep_equals_single_runs(fd, gpu, B):
    # three candidates of different lengths advance together in persistent
    # launches; each equals the same candidate run alone on the one-pass kernel
    cands = B.candidates(3, seed=2)
    r = B.sweep_persistent(fd, cands, group=3, shape=(0, 1.0))
    assert sorted(r["results"]) == [0, 1, 2]
    for c in cands:
        s = B.Slot(fd)
        s.prepare(c, fd.YEE_STREAM)
        s.start()
        alone = s.amplitudes()
        s.close()
        got = r["amplitudes"][c["index"]]
        assert np.all(np.isfinite(got)) and 0.05 < np.abs(got).max() ** 2 < 1.5
        assert np.array_equal(got, alone)
    assert r["cell_steps"] == sum(256 * 128 * c["nz"] * c["steps"] for c in cands)


@pytest.mark.gpu
def test_tile_autotuner_times_each_shape(fd, gpu, B):
    cands = B.candidates(2, seed=2)
    shapes = ((0, 1.0), (3, 2.0))
    best, times = B.autotune_tiles(fd, cands, steps=64, shapes=shapes)
    assert set(times) == set(shapes) and best == min(times, key=times.get) and all(v > 0 for v in times.values())
