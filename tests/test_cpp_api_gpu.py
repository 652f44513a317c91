"""The reference-shaped C++ API (Engine, IndexBuilder for every builder type,
QueryCompiler, QueryExecutor, FileReader, DeviceArray) over the B200 engine,
and gpjson_driver end to end."""
import importlib.util
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def _build():
    spec = importlib.util.spec_from_file_location("_b", ROOT / "15418-project_b200" / "build.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    m.build_cpp()
    return m


def test_cpp_api_suite(tmp_path):
    m = _build()
    exe = m.build_cpp_test(ROOT / "tests" / "cpp", ROOT / "tests" / "cpp" / "_build" / "api_test")
    ld = tmp_path / "ld.json"
    ld.write_text(KATS["ld_json_fixture"]["data"])
    book = tmp_path / "book.json"
    book.write_text(KATS["query_executor"]["json_text"])
    p = subprocess.run([str(exe), str(ld), str(book), str(tmp_path)], capture_output=True,
                       text=True, timeout=300)
    print(p.stdout, p.stderr)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "ALL PASSED 0" in p.stdout


def test_driver_end_to_end_counts(tmp_path):
    from gpjson_b200 import datagen
    m = _build()
    data = datagen.tweets(31, 3 << 20)
    path = tmp_path / "tweets.ldjson"
    path.write_bytes(bytes(data))
    cfg = tmp_path / "run.toml"
    cfg.write_text(f'dataset_path = "{path}"\nrun_name = "e2e"\n'
                   'queries = ["$.user.lang", "$.place.country_code"]\n'
                   '[file_reader]\ntype = "MMAP"\n[index_builder]\ntype = "B200"\n'
                   'file_partition_size = 1000000\n')
    p = subprocess.run([str(m.DRIVER), "-c", str(cfg)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    # the partitions are newline-aligned, so per-line results equal one
    # whole-file oracle run
    want = oracle.OracleIndex(data, 3)
    import gpjson_b200 as gpj
    for q in ["$.user.lang", "$.place.country_code"]:
        c = gpj.compile(q)
        res = want.query(c.ir_bytes, c.num_result_slots)
        lines = int((res[:, :, 0] >= 0).any(axis=1).sum())
        matches = int((res[:, :, 0] >= 0).sum())
        assert f"Query '{q}' has {lines} lines of result, and {matches} matched values" in p.stdout
    assert "Engine::query profiler:" in p.stdout and "### RUN END run_name=e2e ###" in p.stdout
