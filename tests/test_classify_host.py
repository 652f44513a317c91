"""Host builds of index-kernel building blocks: the bit-sliced byte
classifier (csrc/classify.cuh: every byte value at every position of a
32-byte group, plus random groups, against a per-byte classification) and
the look-back descriptor algebra (csrc/descriptor.cuh: packed composition
equals the field-wise one; associativity; identity)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _run_host_test(tmp_path, name):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / name
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", str(ROOT / "15418-project_b200" / "csrc"),
                    str(ROOT / "tests" / "cpp_host" / f"{name}.cpp"), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.startswith("OK"), out.stdout


def test_bit_sliced_classifier_matches_per_byte(tmp_path):
    _run_host_test(tmp_path, "classify_test")


def test_lookback_descriptor_algebra(tmp_path):
    _run_host_test(tmp_path, "descriptor_test")
