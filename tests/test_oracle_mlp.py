"""The oracle's statement of the learned smoother's MLP (CPU only).

* Its backward pass is the exact gradient of its forward pass: with the BF16 roundings switched
  off (FP64 throughout) central differences agree with mlp_backward.
* A hand-built network that computes damped Jacobi (y = ω f0 through two ReLU units) returns
  ω · bf16(f0) exactly, so the network family contains the plain smoother.
* The BF16 forward stays close to the FP64 one.
"""
import numpy as np
import pytest

from conftest import uniform

NP = 5313
OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3 = 0, 1024, 1088, 5184, 5248, 5312


def xavier(seed=4):
    u = uniform(seed, 1024 + 4096 + 64)
    p = np.zeros(NP, np.float32)
    p[OFF_W1:OFF_B1] = (u[:1024] * np.sqrt(6.0 / 80)).astype(np.float32)
    p[OFF_W2:OFF_B2] = (u[1024:5120] * np.sqrt(6.0 / 128)).astype(np.float32)
    p[OFF_W3:OFF_B3] = (u[5120:] * np.sqrt(6.0 / 65)).astype(np.float32)
    return p


def jacobi_net(omega):
    p = np.zeros(NP, np.float32)
    p[OFF_W1 + 0 * 16 + 0] = 1.0    # h1_0 = relu(f0)
    p[OFF_W1 + 1 * 16 + 0] = -1.0   # h1_1 = relu(-f0)
    p[OFF_W2 + 0 * 64 + 0] = 1.0    # z2_0 = h1_0
    p[OFF_W2 + 1 * 64 + 1] = 1.0    # z2_1 = h1_1
    p[OFF_W3 + 0] = omega
    p[OFF_W3 + 1] = -omega
    return p


def test_backward_matches_finite_differences(O):
    rng = np.random.default_rng(0)
    p = xavier(7)
    p[OFF_B1:OFF_W2] = rng.uniform(-0.1, 0.1, 64)
    p[OFF_B2:OFF_W3] = rng.uniform(-0.1, 0.1, 64)
    p[OFF_B3] = 0.05
    S = 6
    x = rng.uniform(-1, 1, (S, 16)).astype(np.float32)
    dy = rng.uniform(-1, 1, S)
    g = O.mlp_backward(p, x, dy, bf16=False)
    f = lambda q: float(np.dot(dy, O.mlp_forward(q, x, bf16=False)))
    idx = np.concatenate([rng.choice(np.arange(a, b), 6, replace=False)
                          for a, b in ((OFF_W1, OFF_B1), (OFF_B1, OFF_W2), (OFF_W2, OFF_B2), (OFF_B2, OFF_W3),
                                       (OFF_W3, OFF_B3))] + [np.array([OFF_B3])])
    for i in idx:
        h = 1e-3
        qp, qm = p.copy(), p.copy()
        qp[i] = np.float32(p[i] + h)
        qm[i] = np.float32(p[i] - h)
        fd = (f(qp) - f(qm)) / (float(qp[i]) - float(qm[i]))
        assert fd == pytest.approx(g[i], rel=2e-3, abs=2e-5), i


def test_jacobi_network_is_damped_jacobi(O):
    x = np.zeros((64, 16), np.float32)
    x[:, 0] = np.linspace(-1, 1, 64, dtype=np.float32) * np.float32(0.987654)
    x[:, 1:7] = 0.3
    omega = np.float32(0.8)
    y = O.mlp_forward(jacobi_net(omega), x)
    bf = x[:, 0].astype(np.float32).view(np.uint32).astype(np.uint64)
    bf = ((bf + 0x7FFF + ((bf >> 16) & 1)) & 0xFFFF0000).astype(np.uint32).view(np.float32)
    np.testing.assert_array_equal(y, float(omega) * bf.astype(np.float64))


def test_bf16_forward_close_to_fp64(O):
    rng = np.random.default_rng(1)
    p = xavier(4)
    x = rng.uniform(-1, 1, (500, 16)).astype(np.float32)
    y16 = O.mlp_forward(p, x)
    y64 = O.mlp_forward(p, x, bf16=False)
    assert np.max(np.abs(y16 - y64)) < 2e-2 * np.max(np.abs(y64))
