"""dec_c_wedge_apply (dec_c_wedge_product!, FastDEC.jl:217-232): every wedge kernel on caller
caches in the reference's layout, the 3D (0,3) and (2,1) kernels included, bit for bit with the
oracle's restatement in FP64 and FP32, with 0- and 1-based indices."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SHAPES = {(0, 1): (2, None), (0, 2): (6, 6), (0, 3): (24, 24), (1, 1): (3, 3), (2, 1): (10, 12)}


def _caches(rng, j, k, n, na):
    rp, rc = SHAPES[(j, k)]
    if (j, k) == (2, 1):
        p = np.concatenate([rng.integers(0, na[1], (n, 6)), rng.integers(0, na[0], (n, 4))], axis=1)
    elif (j, k) == (0, 1):
        p = rng.integers(0, na[0], (2, n))  # n x 2 column-major: the two endpoint columns
    else:
        p = rng.integers(0, na[0], (n, rp))
    c = rng.uniform(-1, 1, (n, rc)) if rc else np.zeros(0)
    return p.astype(np.int32), c


@pytest.mark.parametrize("jk", list(SHAPES))
@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_cached_wedges_match_oracle(O, dec, jk, dt):
    j, k = jk
    rng = np.random.default_rng(100 + 10 * j + k)
    n = 100003
    sizes = {"nv": 30011, "ne": 90007, "nt": 60013}
    # α's length: vertices for j = 0, edges for (1,1), triangles for (2,1); β's: the output
    # simplices for j = 0, edges otherwise
    la = {0: sizes["nv"], 1: sizes["ne"], 2: sizes["nt"]}[j]
    lb = n if j == 0 else sizes["ne"]
    p, c = _caches(rng, j, k, n, (la, sizes["ne"]) if jk == (2, 1) else (la if jk != (1, 1) else sizes["ne"],))
    npdt = np.float64 if dt == "float64" else np.float32
    a = rng.uniform(-1, 1, la).astype(npdt)
    b = rng.uniform(-1, 1, lb).astype(npdt)
    c = c.astype(npdt)
    ref = (O.c_wedge if dt == "float64" else O.c_wedge_f32)(j, k, n, p, c, a, b)
    tc = torch.tensor(c, device="cuda") if c.size else None
    got = dec.dec_c_wedge_product(j, k, torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda"),
                                  torch.tensor(p, device="cuda"), tc, n).cpu().numpy()
    np.testing.assert_array_equal(got, ref)
    got1 = dec.dec_c_wedge_product(j, k, torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda"),
                                   torch.tensor(p + 1, device="cuda"), tc, n, index_base=1).cpu().numpy()
    np.testing.assert_array_equal(got1, ref)
    assert got.dtype == npdt


def test_cached_wedge_rejects_unsupported(dec):
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = torch.zeros(8, dtype=torch.int32, device="cuda")
    with pytest.raises(dec.DecError, match="Unsupported combination"):
        dec.dec_c_wedge_product(1, 2, x, x, p, x, 4)
