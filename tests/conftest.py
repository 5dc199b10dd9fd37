import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_package():
    """Import ``geodynamo.jl_b200/`` (a directory name Python cannot spell) as ``gdb200``."""
    if "gdb200" in sys.modules:
        return sys.modules["gdb200"]
    pkg_dir = os.path.join(ROOT, "geodynamo.jl_b200")
    spec = importlib.util.spec_from_file_location("gdb200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gdb200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libgdb200.so")


@pytest.fixture(scope="session")
def gdb():
    return load_package()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as o
    o.build()
    return o
