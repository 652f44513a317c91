"""The bit-sliced byte classifier of the index kernel (csrc/classify.cuh),
compiled for the host: every byte value at every position of a 32-byte
group, plus random groups, against a per-byte classification."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_bit_sliced_classifier_matches_per_byte(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "classify_test"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", str(ROOT / "15418-project_b200" / "csrc"),
                    str(ROOT / "tests" / "cpp_host" / "classify_test.cpp"), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.startswith("OK"), out.stdout
