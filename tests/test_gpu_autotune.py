"""The autotuner's variants on the GPU.

* The ELL apply's rows-per-thread variants (1, 2, 4) give the same bits; dec_op_autotune records
  one of them for the operator's (dtype, width, size bucket) and later applies use it.
* The FP32 sweep's lanes-per-row variants (vector width 4 or 2 on panels of 8 or more) give the same
  cycles bit for bit; dec_mg_autotune records one per level.
"""
import json

import numpy as np
import pytest

from conftest import uniform

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_ell_rows_variants_same_bits(dec, dtype):
    m = dec.meshes.icosphere(6)
    g = dec.Mesh(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation, m.tri_orientation,
                 center="circumcenter")
    L = dec.laplace_beltrami(g, dtype)
    tdt = torch.float64 if dtype == "float64" else torch.float32
    x = torch.tensor(uniform(3, g.nv), dtype=tdt, device="cuda")
    key = f"ell/{'f64' if dtype == 'float64' else 'f32'}/W7/n{int(np.log2(g.nv))}"
    outs = []
    for rows in (1, 2, 4):
        dec.tune_set(key, rows)
        outs.append(L.apply(x).cpu().numpy())
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])
    choice = L.autotune(reps=5)
    assert choice in (1, 2, 4) and dec.tune_get(key) == choice
    np.testing.assert_array_equal(L.apply(x).cpu().numpy(), outs[0])
    d0 = dec.dec_differential(0, g, dtype)
    assert d0.autotune(reps=2) == 0


def _sweep_keys(K, levels):
    """The FP32 sweep's tuning keys of an icosphere hierarchy (level k: 10·4^k + 2 vertices, rows of
    5 off-diagonal slots on the icosahedron, 6 above it)."""
    return [f"sweep/f32/K{K}/W{5 if k == 0 else 6}/n{int(np.log2(10 * 4 ** k + 2))}" for k in range(levels + 1)]


def test_sweep_lane_variants_same_cycles(dec, tmp_path):
    dec.tune_clear()
    ico = dec.meshes.icosahedron()
    kw = dict(shift=1.0, center="circumcenter", project_radius=1.0, precision=1, pre=0, post=2, cheb_ratio=3.0,
              inner_cycles=2)
    mg = dec.MultigridData(ico, 6, **kw)
    K = mg.autotune(32, reps=2)
    if K >= 8:   # the variant of every level at the chosen width is recorded
        assert all(dec.tune_get(k) in (2, 4) for k in _sweep_keys(K, 6))
    B = torch.tensor(np.stack([uniform(70 + j, mg.n) for j in range(32)]), device="cuda")
    res = []
    for v in (4, 2):
        for k in _sweep_keys(32, 6):
            dec.tune_set(k, v)
        h = dec.MultigridData(ico, 6, rhs_block=32, **kw)   # its graphs are captured with variant v
        U, rep = h.solve(torch.zeros_like(B), B, rtol=1e-9, use_initial_guess=False)
        assert rep.converged == 1
        res.append((U.cpu().numpy(), rep.iterations))
    np.testing.assert_array_equal(res[0][0], res[1][0])
    assert res[0][1] == res[1][1]
    dec.tune_clear()


def _cheb2_keys(levels, K=32):
    return [f"cheb2/f32/K{K}/W6/n{int(np.log2(10 * 4 ** k + 2))}" for k in range(levels + 1)
            if 10 * 4 ** k + 2 >= 1 << 14]


def test_two_step_chebyshev_pair_same_bits(dec):
    """The temporal-blocked post-smoothing pair (k_cheb2: both Chebyshev steps in one pass over patches
    with their halos in shared memory) gives the two sweeps' results bit for bit: V-cycles from a
    given iterate, and the refined solve whose last sweep adds into the FP64 iterate.  The two sweeps
    here follow a stored prolongation (tuning key "pfuse" 0), as the pair does."""
    dec.tune_clear()
    dec.tune_set("pfuse", 0)
    ico = dec.meshes.icosahedron()
    kw = dict(shift=1.0, center="circumcenter", project_radius=1.0, precision=1, pre=0, post=2, cheb_ratio=3.0,
              inner_cycles=3, rhs_block=32)
    n = 10 * 4 ** 7 + 2
    B = torch.tensor(np.stack([uniform(90 + j, n) for j in range(32)]), device="cuda")
    U0 = torch.tensor(np.stack([uniform(190 + j, n) for j in range(32)]) * 0.1, device="cuda")
    out = []
    for v in (0, 512, 128):   # two sweeps; the pair over patches of 512 and of 128 rows
        for k in _cheb2_keys(7):
            dec.tune_set(k, v)
        h = dec.MultigridData(ico, 7, **kw)
        U = h.cycles(U0.clone(), B, 2).cpu().numpy()
        X, rep = h.solve(torch.zeros_like(B), B, rtol=1e-9, use_initial_guess=False)
        assert rep.converged == 1
        out.append((U, X.cpu().numpy(), rep.iterations))
    for o in out[1:]:
        np.testing.assert_array_equal(out[0][0], o[0])
        np.testing.assert_array_equal(out[0][1], o[1])
        assert out[0][2] == o[2]
    dec.tune_clear()
    mg = dec.MultigridData(ico, 7, **kw)
    mg.autotune(32, reps=2)
    assert all(dec.tune_get(k) in (0, 128, 256, 512) for k in _cheb2_keys(7))
    dec.tune_clear()


def test_batched_wedge11_pairs_variants_same_bits(dec):
    """The batched FP32 ∧(1,1) with 1, 2, 4, 8 and 16 form pairs per thread (a count that no variant
    divides) equals the single applications bit for bit; dec_wedge_autotune records one of them."""
    m = dec.meshes.icosphere(4)
    g = dec.Mesh(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation, m.tri_orientation,
                 center="circumcenter")
    w = dec.dec_wedge_product(1, 1, g, "float32")
    count = 37
    a = torch.tensor(np.stack([uniform(700 + j, w.len_a) for j in range(count)]), dtype=torch.float32, device="cuda")
    b = torch.tensor(np.stack([uniform(800 + j, w.len_b) for j in range(count)]), dtype=torch.float32, device="cuda")
    single = np.stack([w(a[j], b[j]).cpu().numpy() for j in range(count)])
    key = f"w11pairs/f32/n{int(np.log2(g.nt))}"
    for pairs in (1, 2, 4, 8, 16):
        dec.tune_set(key, pairs)
        out = torch.full((count, w.len_out), float("nan"), dtype=torch.float32, device="cuda")
        w.batched(a, b, out)
        np.testing.assert_array_equal(out.cpu().numpy(), single)
    choice = w.autotune(count, reps=2)
    assert choice in (1, 2, 4, 8, 16) and dec.tune_get(key) == choice
    assert dec.dec_wedge_product(0, 1, g, "float32").autotune(count) == 0
