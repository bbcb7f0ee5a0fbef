"""Shared fixtures: the CPU oracle (checker) and the sm_100a library's Python host mirror."""
import importlib.util
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "combinatorialspaces.jl_b200"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def load_package():
    """Import the package directory (its name holds a dot) under the module name ``dec_b200``."""
    if "dec_b200" in sys.modules:
        return sys.modules["dec_b200"]
    spec = importlib.util.spec_from_file_location(
        "dec_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dec_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def O():
    import oracle
    return oracle.load()


@pytest.fixture(scope="session")
def dec():
    return load_package()


def csc(t):
    """Oracle CSC tuple -> scipy.sparse.csc_matrix."""
    import scipy.sparse as sp
    colptr, rowval, nzval, shape = t
    return sp.csc_matrix((nzval, rowval, colptr), shape=shape)


def uniform(seed, n, dtype=np.float64):
    """The project's input generator: splitmix64 -> uniform[-1, 1)."""
    state = np.uint64(seed)
    out = np.empty(n, dtype=np.float64)
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = state + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    out[:] = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) * 2.0 - 1.0
    return out.astype(dtype)
