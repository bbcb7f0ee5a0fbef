"""TEST INFRASTRUCTURE ONLY.

The CPU oracle: a C++ (FP64) restatement of the CombinatorialSpaces.jl DEC hot path
(dec_oracle.cpp cites the reference file:line of every function).  It is the checker for the
sm_100a library.  Only the test suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline legs may load it; the product library never does.

Parity of the oracle itself is pinned by the reference's own known-answer tests, restated in
``tests/test_oracle_*.py``; the reference (Julia) cannot run in this environment.
"""
import importlib
import pathlib
import subprocess
import sys

_HERE = pathlib.Path(__file__).resolve().parent
_BUILD = _HERE / "_build"


def build() -> None:
    """Compile the oracle module (g++ and pybind11; a few seconds)."""
    subprocess.run(["make", "-s", "-C", str(_HERE), f"PY={sys.executable}"], check=True)


def load():
    """Return the compiled ``dec_oracle`` module, building it first if needed."""
    if str(_BUILD) not in sys.path:
        sys.path.insert(0, str(_BUILD))
    try:
        return importlib.import_module("dec_oracle")
    except ImportError:
        build()
        return importlib.import_module("dec_oracle")
