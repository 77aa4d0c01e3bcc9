"""Host C++ of the product (Mesh normal / tangent generators, BVH build and
flatten, sample table) against the oracle, bit for bit.  No GPU needed."""
import numpy as np
import pytest

from fornos_b200 import api
from fornos_b200 import workloads as W
from tests.cases import same_bits

MESHES = {
    "sphere": lambda: W.sphere_pair(seed=1, lo_seg=(32, 16), hi_seg=(64, 32)),
    "plane": lambda: W.plane_pair(seed=2, lo_quads=8, hi_quads=48, bumps=20),
    "icosphere": lambda: W.icosphere_pair(seed=3, lo_subdiv=1, hi_subdiv=3),
}


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("which", ["face", "vertex", "welded"])
def test_normals(lib, oracle, name, which):
    lo, hi = MESHES[name]()
    for m in (lo, hi):
        pm = api.Mesh(m)
        {"face": pm.compute_face_normals, "vertex": pm.compute_vertex_normals,
         "welded": pm.compute_vertex_normals_aggressive}[which]()
        a = pm.arrays()
        ov, on = oracle.normals(m, which)
        assert np.array_equal(a.vertices, ov)
        assert same_bits(a.normals, on)


@pytest.mark.parametrize("name", list(MESHES))
def test_tangent_space(lib, oracle, name):
    lo, _ = MESHES[name]()
    pm = api.Mesh(lo)
    pm.compute_tangent_space()
    a = pm.arrays()
    t, b = oracle.tangent_space(lo)
    assert same_bits(a.tangents, t) and same_bits(a.bitangents, b)


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("max_tris", [1, 4, 8, 32])
def test_bvh_matches_oracle(lib, oracle, name, max_tris):
    _, hi = MESHES[name]()
    pm = api.Mesh(hi)
    pm.compute_vertex_normals()
    a = pm.arrays()
    nodes, p4, n4 = api.BVH.create_binary(pm, max_tris).flatten(pm)
    on, op, onr = oracle.scene(a, max_tris)
    assert nodes.tobytes() == on.tobytes()
    assert same_bits(p4, op) and same_bits(n4, onr)
    # structural invariants of the skip-pointer layout
    i = np.arange(len(nodes))
    assert np.all(nodes["jump"] > i) and nodes["jump"][0] == len(nodes)
    leaf = nodes["jump"] == i + 1
    assert np.all((nodes["end"] > nodes["start"]) == leaf)
    assert np.all(nodes["end"][leaf] - nodes["start"][leaf] <= 3 * max_tris) or max_tris == 1


def test_bvh_depth_limit(lib, oracle):
    _, hi = MESHES["plane"]()
    pm = api.Mesh(hi)
    pm.compute_vertex_normals()
    nodes, _, _ = api.BVH.create_binary(pm, 8, 3).flatten(pm)
    on, _, _ = oracle.scene(pm.arrays(), 8, 3)
    assert nodes.tobytes() == on.tobytes() and len(nodes) <= 15


def test_degenerate_meshes(lib, oracle):
    # all triangles with one centroid: the split gives up, one leaf
    p = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    tris = np.zeros((20, 3), np.uint32) + np.array([0, 1, 2], np.uint32)
    m = W.MeshArrays(p, np.zeros((1, 2)), np.array([[0, 0, 1]]), np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0]]), tris)
    pm = api.Mesh(m)
    nodes, p4, _ = api.BVH.create_binary(pm, 8).flatten(pm)
    on, op, _ = oracle.scene(m, 8)
    assert nodes.tobytes() == on.tobytes() and len(nodes) == 1 and nodes["end"][0] == 60
    # invalid indices are refused
    bad = W.MeshArrays(p, np.zeros((1, 2)), np.array([[0, 0, 1]]), np.array([[5, 0, 0]]), np.array([[0, 0, 0]]))
    with pytest.raises(api.FornosError):
        api.Mesh(bad)


@pytest.mark.parametrize("spp,seed", [(1, 0), (16, 7), (64, 12345), (256, 3)])
def test_sample_table(lib, oracle, spp, seed):
    s = api.samples_cosine(spp, 4096, seed)
    assert same_bits(s, oracle.samples(spp, 4096, seed))
    r2 = s[:, 0] ** 2 + s[:, 1] ** 2 + s[:, 2] ** 2
    assert np.allclose(r2, 1.0, atol=1e-5) and (s[:, 2] >= 0).all()
