"""The C++ facade (include/mps_b200.hpp) on a GPU: the ClcMPS-style loop of tests/cpp runs
its per-method and fused steps, two steps of the corrected-matrix gradient, and writes the
reference's output files through mps_b200::Output."""
from __future__ import annotations

import os
import subprocess

import pytest

from mps_cuda_b200 import _lib as L

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_facade_runs_on_the_gpu(tmp_path):
    lib = L.library_path()
    exe = tmp_path / "clcmps_loop"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "clcmps_loop.cpp"), "-L", os.path.dirname(lib),
                    "-lmps_b200", "-Wl,-rpath," + os.path.dirname(lib), "-o", str(exe)],
                   check=True, capture_output=True)
    res = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "alive 480" in res.stdout, res.stdout
    for name in ("output00001.csv", "outputMRR00001.csv", "outputwall00000.csv", "seitei.txt"):
        assert (tmp_path / "out" / name).exists(), name
