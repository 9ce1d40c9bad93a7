import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    """Import vortexpasta.jl_b200/ (a directory whose name is not an identifier) as vortexpasta_b200."""
    name = "vortexpasta_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = ROOT / "vortexpasta.jl_b200"
    spec = importlib.util.spec_from_file_location(name, pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def vp():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.load()
    return O


@pytest.fixture(scope="session")
def built_lib(vp):
    from importlib import import_module
    build = import_module("vortexpasta_b200.build")
    return build.build_library()
