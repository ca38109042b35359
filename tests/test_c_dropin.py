"""The drop-in checked by a C compiler and linker: tests/c_dropin/taper_driver.c
(the reference driver's call sequence, 3d_fdtd.c:97-187, on the small taper)
compiled against the reference's own headers, once linked with the reference's
timefield3d.o / adjoint3d.o and once with libfdtd_b200.so in their place
(`make -C oracle dropin`, which needs the reference's sources; the binaries
land in oracle/_ref/).  Both run here and their outputs are compared: the
library is in its default FP64 mode, so the fields equal the reference's to
rounding of the plane reductions, and the gradients and edge updates agree.
"""
from __future__ import annotations

import gzip
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "taper_driver_ref")
B200_BIN = os.path.join(ROOT, "oracle", "_ref", "taper_driver_b200")
MODE = os.path.join(ROOT, "tests", "golden", "modes", "small_te0.txt.gz")

NX, NY, H, LEN, SEG = 40, 28, 5, 24, 5


def parse(path):
    raw = open(path, "rb").read()
    d = np.frombuffer(raw, dtype=np.float64, count=6)
    off = 48
    plane = NX * NY * 6
    fwd = np.frombuffer(raw, dtype=np.float64, count=plane, offset=off); off += 8 * plane
    adj = np.frombuffer(raw, dtype=np.float64, count=plane, offset=off); off += 8 * plane
    epg = np.frombuffer(raw, dtype=np.float64, count=2 * H * LEN, offset=off); off += 8 * 2 * H * LEN
    lg = np.frombuffer(raw, dtype=np.float64, count=SEG, offset=off); off += 8 * SEG
    rg = np.frombuffer(raw, dtype=np.float64, count=SEG, offset=off); off += 8 * SEG
    edges = np.frombuffer(raw, dtype=np.int32, count=2 * SEG + 1, offset=off); off += 4 * (2 * SEG + 1)
    assert off == len(raw)
    return dict(overlaps=d.view(np.complex128), fwd=fwd, adj=adj, epg=epg, lg=lg, rg=rg, edges=edges)


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.gpu
def test_c_program_links_library_in_place_of_reference_objects(gpu, tmp_path):
    if not (os.path.exists(REF_BIN) and os.path.exists(B200_BIN)):
        pytest.skip("drop-in drivers not built (make -C oracle dropin needs the reference's sources)")
    mode = tmp_path / "small_te0.txt"
    with gzip.open(MODE, "rb") as fi, open(mode, "wb") as fo:
        shutil.copyfileobj(fi, fo)
    env = dict(os.environ, OMP_NUM_THREADS="8")   # every reference z-slab keeps >= 2 planes
    outs = {}
    for name, exe in (("ref", REF_BIN), ("b200", B200_BIN)):
        out = tmp_path / f"{name}.bin"
        p = subprocess.run([exe, str(mode), str(out)], env=env, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, (name, p.stdout[-2000:], p.stderr[-2000:])
        outs[name] = parse(out)
    a, b = outs["b200"], outs["ref"]
    assert np.abs(b["overlaps"]).min() > 0
    assert rel(a["overlaps"], b["overlaps"]) < 1e-10
    assert rel(a["fwd"], b["fwd"]) < 1e-10 and rel(a["adj"], b["adj"]) < 1e-10
    assert rel(a["epg"], b["epg"]) < 1e-9
    assert rel(a["lg"], b["lg"]) < 1e-9 and rel(a["rg"], b["rg"]) < 1e-9
    assert np.array_equal(a["edges"], b["edges"])
