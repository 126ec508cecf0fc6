"""The C++20 binding (include/crdfft.hpp) compiled with g++ against libcrdfft.so: the device-free paths on the CPU,
and (GPU) a transform, a real transform, a Welch PSD and a lowered CEIR tensor.fft on split-complex planes from C++
host code checked against the FP64 oracle."""

from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "crd_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(LIBDIR, "libcrdfft.so")):
        pytest.skip("g++ or libcrdfft.so missing")
    exe = str(tmp_path / "abi_demo")
    cmd = ["g++", "-std=c++20", "-O1", os.path.join(ROOT, "tests", "cpp", "abi_demo.cpp"), "-I",
           os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"), "-L", LIBDIR, "-lcrdfft",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath,{CUDA}/lib64",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def test_cpp_binding_host_paths(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, "host"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "host ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_binding_device(tmp_path):
    from oracle import spectral as S

    exe = _build(tmp_path)
    n = 4096
    x = oracle.lcg_complex64(0xC0DE, n)
    inp, out = tmp_path / "x.bin", tmp_path / "y.bin"
    x.tofile(inp)
    r = subprocess.run([exe, "device", str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "device ok" in r.stdout, r.stdout + r.stderr
    raw = np.fromfile(out, dtype=np.uint8)
    y = raw[: 8 * n].view(np.complex64)
    sp = raw[8 * n: 8 * n + 8 * (n // 2 + 1)].view(np.complex64)
    off = 8 * n + 8 * (n // 2 + 1)
    psd = raw[off: off + 4 * 33].view(np.float32)
    planes = raw[off + 4 * 33:].view(np.float32)
    got = planes[:n].astype(np.float64) + 1j * planes[n:].astype(np.float64)
    assert oracle.rel_l2(got, oracle.fft64(x[None, :])[0]) <= 1e-6  # the lowered tensor.fft on split planes
    assert oracle.rel_l2(y, oracle.fft64(x[None, :])[0]) <= 1e-6
    assert oracle.rel_l2(sp, oracle.rfft64(x.real.astype(np.float64))) <= 1e-6
    want = S.welch(x.real[:128].astype(np.float64), 1.0, 64, 32)
    assert np.linalg.norm(psd - want) / np.linalg.norm(want) <= 1e-6
