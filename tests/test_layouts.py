"""The host level layouts (build_layout in nricp_b200/csrc/host.cpp): the
usable bindings, gather lists, node-pair groups, off-diagonal blocks (one per
coupled node pair) and rows, and warm-start bindings the device kernels walk, each checked against a direct
restatement (tests/layout_check.cpp) on seeded graphs with planted repeated
nodes, zero weights and out-of-range nodes."""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_layouts_hold_what_the_kernels_walk(tmp_path):
    exe = tmp_path / "layout_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off",
                    str(ROOT / "tests" / "layout_check.cpp"), str(ROOT / "nricp_b200" / "csrc" / "host.cpp"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and out.stdout.strip().endswith("ok"), out.stdout + out.stderr
