"""The one-launch four-step's work list (crd_b200/csrc/chain_list.hpp), checked on the host: every tile once, and
every wait on a tile earlier in the list (so the list drains whatever CTAs are resident), at the bench's and the
parity tests' shapes (tests/cpp/chain_list_check.cpp, compiled with g++)."""

from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_chain_work_list_drains(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    exe = str(tmp_path / "chain_list_check")
    r = subprocess.run(["g++", "-std=c++20", "-O1", "-Wall", "-I", os.path.join(ROOT, "crd_b200", "csrc"),
                        os.path.join(ROOT, "tests", "cpp", "chain_list_check.cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "chain list ok" in r.stdout, r.stdout + r.stderr
