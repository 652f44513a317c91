"""The C ABI library loads and exports every symbol include/gpjson_b200.h
declares (CPU only: no compute calls)."""
import re
from pathlib import Path

import pytest

HEADER = Path(__file__).resolve().parent.parent / "include" / "gpjson_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gpj_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "gpj_index_build" in names and "gpj_query_run" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol(gpj):
    lib = gpj.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert set(declared_functions()) == set(gpj.EXPORTED_SYMBOLS)


def test_version(gpj):
    assert gpj.load_library().gpj_version() >= 100


def test_no_cpu_path_without_device(gpj):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(gpj.CudaError, match="no CPU path"):
        gpj.Context(0)


def test_server_needs_a_device(gpj):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(gpj.CudaError):
        gpj.Server(0, hbm_budget_bytes=1 << 20)
