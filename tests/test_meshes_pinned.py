"""The package's mesh generators (the inputs of every bench workload) equal the oracle's.

`meshes.triangulated_grid` (src/CombMeshes.jl:79-133), `meshes.icosahedron` and the vectorised
`meshes.refine_binary` (refine(::BinarySubdivision) + propagate_points, src/Multigrid.jl:111-183,
with the unit-sphere projection of the icosphere workloads) must give the oracle's arrays bit for
bit: topology (∂v0, ∂v1, ∂e0..∂e2), points, and the orientations the generator sets.  CPU only.
"""
import numpy as np
import pytest


def _same_topology_and_points(m, om):
    for a, b in (("ev0", "ev0"), ("ev1", "ev1"), ("te0", "te0"), ("te1", "te1"), ("te2", "te2")):
        np.testing.assert_array_equal(np.asarray(getattr(m, a), np.int64), np.asarray(getattr(om, b), np.int64),
                                      err_msg=a)
    np.testing.assert_array_equal(np.asarray(m.points, np.float64), om.points)


@pytest.mark.parametrize("args", [(127, 127, 1.0, 1.0, False), (1, 1, 0.25, np.sqrt(3) / 8, False),
                                  (8, 5, 1.0, 1.0, True), (511, 511, 1.0, 1.0, False)])
def test_triangulated_grid_equals_oracle(O, dec, args):
    m = dec.meshes.triangulated_grid(*args)
    om = O.triangulated_grid(*args[:4], compress=args[4])
    _same_topology_and_points(m, om)
    np.testing.assert_array_equal(np.asarray(m.tri_orientation, np.int64), om.tri_orientation.astype(np.int64))
    assert m.nv == om.nv and m.ne == om.ne and m.nt == om.nt


def test_grid_128_counts(dec):
    """The 128 x 128 operator workload: 16,384 vertices, 48,641 edges, 32,258 triangles."""
    m = dec.meshes.triangulated_grid(127, 127, 1.0, 1.0, False)
    assert (m.nv, m.ne, m.nt) == (16384, 48641, 32258)


def test_icosahedron_equals_oracle(O, dec):
    m = dec.meshes.icosahedron()
    _same_topology_and_points(m, O.icosahedron())


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6])
def test_icosphere_equals_oracle_refinement(O, dec, k):
    """Icosphere L_k (unit-sphere projection) against k oracle refinements of its icosahedron;
    L6 is the 40,962-vertex multigrid workload."""
    m = dec.meshes.icosphere(k)
    om = O.icosahedron()
    for _ in range(k):
        om = O.refine_binary(om, 1.0)
    _same_topology_and_points(m, om)
    assert (m.nv, m.ne, m.nt) == (10 * 4 ** k + 2, 30 * 4 ** k, 20 * 4 ** k)


def test_planar_refinement_equals_oracle(O, dec):
    """Binary refinement without projection (the batched grid workloads: a coarse grid refined)."""
    m = dec.meshes.triangulated_grid(8, 8, 1.0, 1.0, False)
    om = O.triangulated_grid(8, 8, 1.0, 1.0, compress=False)
    for _ in range(3):
        m = dec.meshes.refine_binary(m, 0.0)
        om = O.refine_binary(om, 0.0)
    _same_topology_and_points(m, om)
