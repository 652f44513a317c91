import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _load(name: str, path: Path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, path / "__init__.py", submodule_search_locations=[str(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    parent, _, child = name.rpartition(".")
    if parent in sys.modules:
        setattr(sys.modules[parent], child, mod)
    return mod


# the package directory name is not an identifier; expose it as gpjson_b200
gpjson_b200 = _load("gpjson_b200", ROOT / "15418-project_b200")
_load("gpjson_b200.datagen", ROOT / "15418-project_b200" / "datagen")


@pytest.fixture(scope="session")
def gpj():
    gpjson_b200.load_library(build_if_missing=True)
    return gpjson_b200


@pytest.fixture(scope="session")
def cuda_ctx(gpj):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    torch.cuda.init()
    ctx = gpj.Context(0)
    yield ctx
    ctx.close()
