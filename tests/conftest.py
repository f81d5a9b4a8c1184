import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _load_package():
    name = "cgmli_slam_b200"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            name, ROOT / "cgmli-slam_b200" / "__init__.py", submodule_search_locations=[str(ROOT / "cgmli-slam_b200")])
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)


_load_package()
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.lib()
    return O
