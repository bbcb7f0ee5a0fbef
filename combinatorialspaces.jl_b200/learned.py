"""Training pipeline of the learned multigrid smoother (no counterpart in the reference).

Data: (residual, error) pairs that the plain FP64 V-cycle itself produces on icospheres L5-L7
(unit sphere, circumcentric duals, A = L + shift I).  The V-cycle runs on A u = 0 from an initial
guess u0 ~ U[-1, 1] (the project's splitmix64 generator), so after k cycles the error is
e_k = -u_k and the residual r_k = -A u_k; fields cycle over k in `cycles`.  The k = 0 pairs are
rough (white-noise) errors, the error a smoother exists to remove; the later ones are what the
plain cycle leaves behind.  Each pair enters the energy-norm loss through its residual alone (the
loss differs from ||e_k - δ||²_{⋆0 A} by a constant), so the errors are never formed.

Schedule: Adam steps cycle over the meshes in blocks of `block` steps; a step on L5 uses 6 fields
(61,452 vertex samples, all in the batch), on L6 2 fields and on L7 one field, with a batch of
65,536 vertex samples drawn from them.
"""
import numpy as np

from . import MultigridData, SmootherMLP, meshes


def residual_fields(level, count, shift=1.0, seed=100, cycles=(0,)):
    """(hierarchy, operator, residual fields (count, n) float64 CUDA) on icosphere L_level."""
    import torch
    mg = MultigridData(meshes.icosahedron(), level, shift=shift, center="circumcenter", project_radius=1.0,
                       smoother=1, precision=0)
    n = mg.n
    op = mg.level_op(0)
    out = torch.empty((count, n), dtype=torch.float64, device="cuda")
    zero = torch.zeros(n, dtype=torch.float64, device="cuda")
    for j in range(count):
        u = torch.tensor(meshes.uniform(seed + 1000 * level + j, n), device="cuda")
        k = cycles[j % len(cycles)]
        if k:
            mg.cycles(u, zero, k)
        out[j] = -op.apply(u)
    return mg, op, out


def train_smoother(steps=20000, lr=1e-3, batch=65536, seed=4, shift=1.0, levels=(5, 6, 7), block=10,
                   fields=None, cycles=(0,), log_every=0):
    """Trains a fresh SmootherMLP(seed); returns (mlp, losses), losses a list of
    (step, level, loss before that step's update) at the first step of every block."""
    fields = fields or {5: 48, 6: 16, 7: 8}
    per_step = {5: 6, 6: 2, 7: 1}
    data = {}
    for lv in levels:
        data[lv] = residual_fields(lv, fields[lv], shift=shift, cycles=cycles)
    mlp = SmootherMLP(seed)
    losses = []
    rng = np.random.default_rng(seed)
    t = 0
    while t < steps:
        for lv in levels:
            if t >= steps:
                break
            _, op, r = data[lv]
            S = per_step.get(lv, 1)
            j = int(rng.integers(0, r.shape[0] - S + 1))
            nb = min(block, steps - t)
            rec = mlp.train(op, r[j:j + S], 1, lr=lr, batch=batch, seed=seed, record_loss=True)
            losses.append((t, lv, float(rec[0])))
            if nb > 1:
                mlp.train(op, r[j:j + S], nb - 1, lr=lr, batch=batch, seed=seed)
            t += nb
            if log_every and (t // block) % log_every == 0:
                print(f"step {t} L{lv} loss {rec[0]:.5f}")
    return mlp, losses
