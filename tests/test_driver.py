"""gpjson_driver configuration surface (CPU only): TOML keys, command-line
overrides and aliases, validation errors -- the cases of the reference's
tests/app/driver_config_test.cpp.  The driver prints its resolved
configuration (GPJSON_RUN_CONFIG) before touching the dataset, so a missing
dataset file lets these run without a GPU."""
import importlib.util
import json
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def driver():
    spec = importlib.util.spec_from_file_location("_b", ROOT / "15418-project_b200" / "build.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    m.build_cpp()
    return m.DRIVER


def run(driver, *args):
    p = subprocess.run([str(driver), *map(str, args)], capture_output=True, text=True, timeout=60)
    cfg = None
    for line in p.stdout.splitlines():
        if line.startswith("GPJSON_RUN_CONFIG "):
            cfg = json.loads(line[len("GPJSON_RUN_CONFIG "):])
    return p, cfg


def test_parses_toml_config(driver, tmp_path):
    toml = tmp_path / "c.toml"
    toml.write_text('dataset_path = "missing/input.json"\nrun_name = "toml_run"\n'
                    'queries = ["$.user.lang", "$.user.id"]\n\n[file_reader]\ntype = "MMAP"\n\n'
                    '[index_builder]\ntype = "COMBINED"\nfile_partition_size = 65536\n'
                    'grid_size = 16384\nblock_size = 1024\nreduction_grid_size = 32\n'
                    'reduction_block_size = 16\n\n[query_executor]\ngrid_size = 99\n'
                    'block_size = 128\n')
    p, cfg = run(driver, "--config", toml)
    assert cfg["run_name"] == "toml_run" and cfg["dataset_path"] == "missing/input.json"
    assert cfg["queries"] == ["$.user.lang", "$.user.id"]
    eo = cfg["engine_options"]
    assert eo["file_reader"]["type"] == "MMAP"
    assert eo["index_builder"] == {"type": "COMBINED", "file_partition_size": 65536,
                                   "grid_size": 16384, "block_size": 1024,
                                   "reduction_grid_size": 32, "reduction_block_size": 16}
    assert eo["query_executor"] == {"grid_size": 99, "block_size": 128}
    assert p.returncode == 1 and "Failed to get size for file" in p.stderr
    assert "### RUN BEGIN run_name=toml_run ###" in p.stdout


def test_cli_overrides_toml(driver, tmp_path):
    toml = tmp_path / "c.toml"
    toml.write_text('dataset_path = "from_toml.json"\nrun_name = "toml_run"\nqueries = ["$.toml"]\n'
                    '[file_reader]\ntype = "COPIED"\n[index_builder]\ntype = "UNCOMBINED"\n'
                    'grid_size = 1\nblock_size = 2\n[query_executor]\ngrid_size = 3\nblock_size = 4\n')
    p, cfg = run(driver, "--config", toml, "--dataset", "from_cli.json", "--query", "$.cli.one",
                 "--query", "$.cli.two", "--run-name", "cli_run", "--index-builder.type",
                 "COMBINED", "--file-reader.type", "MMAP", "--index-builder.grid-size", "16384",
                 "--query-executor.grid-size", "55", "--query-executor.block-size", "64")
    assert cfg["run_name"] == "cli_run" and cfg["dataset_path"] == "from_cli.json"
    assert cfg["queries"] == ["$.cli.one", "$.cli.two"]
    eo = cfg["engine_options"]
    assert eo["file_reader"]["type"] == "MMAP"
    assert eo["index_builder"]["type"] == "COMBINED"
    assert eo["index_builder"]["grid_size"] == 16384 and eo["index_builder"]["block_size"] == 2
    assert eo["query_executor"] == {"grid_size": 55, "block_size": 64}


def test_defaults_and_required_dataset(driver):
    p, cfg = run(driver, "-q", "$.a")
    assert p.returncode == 1 and "dataset_path is required" in p.stderr
    p, cfg = run(driver, "--dataset", "x.json")
    assert p.returncode == 1 and "At least one query is required" in p.stderr
    p, cfg = run(driver, "--dataset", "x.json", "-q", "$.a")
    assert cfg["run_name"].startswith("run_")
    eo = cfg["engine_options"]
    assert eo["file_reader"]["type"] == "COPIED" and eo["index_builder"]["type"] == "UNCOMBINED"
    assert eo["query_executor"] == {"grid_size": 512, "block_size": 1024}


def test_rejects_negative_sizes_and_bad_enums(driver, tmp_path):
    p, _ = run(driver, "--dataset", "x", "-q", "$.a", "--query-executor.grid-size", "-1")
    assert p.returncode == 1 and "must be non-negative" in p.stderr
    p, _ = run(driver, "--dataset", "x", "-q", "$.a", "--file-reader.type", "BAD_READER")
    assert p.returncode == 1 and "Invalid enum value 'BAD_READER'" in p.stderr
    p, _ = run(driver, "--dataset", "x", "-q", "$.a", "--index-builder.type", "BAD_BUILDER")
    assert p.returncode == 1 and "Invalid enum value 'BAD_BUILDER'" in p.stderr
    toml = tmp_path / "bad.toml"
    toml.write_text('[index_builder]\ngrid_size = "many"\n')
    p, _ = run(driver, "--config", toml, "--dataset", "x", "-q", "$.a")
    assert p.returncode == 1 and "must be an integer" in p.stderr
    p, cfg = run(driver, "--dataset", "x", "-q", "$.a", "--index-builder.type", "B200")
    assert cfg["engine_options"]["index_builder"]["type"] == "B200"
