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


def level_lmax(md, level, steps=30, safety=1.05):
    """λmax(D⁻¹A) of level `level` of an oracle hierarchy by `steps` power iterations from a fixed
    smooth start vector, times `safety`: the Chebyshev interval bound of the oracle's own FP64
    solves (the library estimates its bound on the device; the two need not agree to the bit)."""
    import numpy as np
    import scipy.sparse as sp
    cp, rv, nz, shape = md.op(level)
    A = sp.csc_matrix((nz, rv, cp), shape=shape).tocsr()
    d = A.diagonal()
    x = np.cos(np.arange(A.shape[0]) * 0.7 + 0.3)
    lam = 1.0
    for _ in range(steps):
        y = (A @ x) / d
        lam = np.linalg.norm(y) / np.linalg.norm(x)
        x = y / np.linalg.norm(y)
    return float(lam * safety)


def fp64_solve(md, b, rtol=1e-13, max_cycles=40, pre=3, post=3, ratio=4.0, lmax=None):
    """An FP64-only solve on the CPU: the oracle's plain V(pre, post)-cycles (Chebyshev-Jacobi on
    [λ/ratio, λ], dense solve on the coarsest level, every SpMV in SparseArrays' column order)
    from u = 0, cycled until ‖b - A u‖ / ‖b‖ ≤ rtol or the residual stops falling.  The
    reference's own Krylov-CG-smoothed cycle cannot serve here: its CG calls stop at √eps of their
    initial residual, and the cycle stalls near 1e-9.  Returns (u, relative residual, cycles,
    lmax list)."""
    import numpy as np
    import scipy.sparse as sp
    O = load()
    if lmax is None:
        lmax = [level_lmax(md, l) for l in range(md.nlevels)]
    cp, rv, nz, shape = md.op(0)
    A = sp.csc_matrix((nz, rv, cp), shape=shape).tocsr()
    b = np.ascontiguousarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    u = np.zeros_like(b)
    if nb == 0.0:
        return u, 0.0, 0, lmax
    best, stall, cycles, rel = np.inf, 0, 0, 1.0
    while cycles < max_cycles:
        u = O.plain_vcycles(md, u, b, 1, 1, pre, post, 0.8, ratio, lmax)
        cycles += 1
        rel = float(np.linalg.norm(b - A @ u) / nb)
        if rel <= rtol:
            break
        if rel >= 0.5 * best:
            stall += 1
            if stall >= 2:
                break
        else:
            stall = 0
        best = min(best, rel)
    return u, rel, cycles, lmax
