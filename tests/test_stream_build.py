"""The streaming kernel runs 16 warps a block at the 128-register cap, with no
headroom: a build in which the lossless kernels spill ran the 200 x 160 x 400
CPML workload 18 % slower.  Compiles yee_stream.cu as the library build does
(sm_100a, nvcc only, no GPU) and checks ptxas' report: no spill stores or
loads in k_yee_stream<CPML, lossless, rows> and k_yee_stream<PEC, lossless,
rows> for every instantiated row count.
"""
from __future__ import annotations

import importlib.util
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_module():
    spec = importlib.util.spec_from_file_location("fdtd_build", os.path.join(ROOT, "3d_fdtd_b200", "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not available")
def test_streaming_kernels_do_not_spill(tmp_path):
    b = build_module()
    src = os.path.join(b.CSRC, "yee_stream.cu")
    cmd = [b.nvcc(), *b.ARCH, *b.NVCC_FLAGS, "-Xptxas", "-v", "-c", src, "-o", str(tmp_path / "ys.o")]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    report = {}
    name = None
    for line in p.stderr.splitlines():
        m = re.search(r"Function properties for (\S+)", line)
        if m:
            name = m.group(1)
            continue
        m = re.search(r"(\d+) bytes spill stores, (\d+) bytes spill loads", line)
        if m and name:
            report[name] = (int(m.group(1)), int(m.group(2)))
            name = None
    # _ZN4fdtd12k_yee_streamILb<CPML>ELb<LOSSY>ELi<rows>EEEvNS_10StreamArgsE,
    # rows 0 (known at run time) or 2..8
    for cpml in (1, 0):
        for tp in (0, 2, 3, 4, 5, 6, 7, 8):
            key = f"_ZN4fdtd12k_yee_streamILb{cpml}ELb0ELi{tp}EEEvNS_10StreamArgsE"
            assert key in report, sorted(report)
            assert report[key] == (0, 0), (key, report[key])
