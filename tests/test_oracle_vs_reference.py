"""Pins the oracle restatement to the reference's own code: Src/*.cpp and the
Shaders/*.comp sources compiled on the host by oracle/build_ref.py.  Skipped
where the reference tree (and so oracle/_ref) is absent; tests/golden holds
fixtures generated from the same build for that case."""
import numpy as np
import pytest

from fornos_b200 import workloads as W
from tests.cases import pix8, same_bits

MESHES = {
    "sphere": lambda: W.sphere_pair(seed=1, lo_seg=(32, 16), hi_seg=(64, 32)),
    "plane": lambda: W.plane_pair(seed=2, lo_quads=8, hi_quads=48, bumps=20),
    "icosphere": lambda: W.icosphere_pair(seed=3, lo_subdiv=1, hi_subdiv=3),
}


def prepared(oracle, name):
    lo, hi = MESHES[name]()
    v, n = oracle.normals(hi, "vertex")
    hi.vertices, hi.normals = v, n
    lo.tangents, lo.bitangents = oracle.tangent_space(lo)
    dirs = oracle.normals(lo, "welded")
    return lo, hi, dirs


@pytest.mark.parametrize("name", list(MESHES))
def test_host_preprocessing(oracle, reference, name):
    lo, hi = MESHES[name]()
    for m in (lo, hi):
        for which in ("face", "vertex", "welded"):
            a, b = oracle.normals(m, which), reference.normals(m, which)
            assert np.array_equal(a[0], b[0]) and same_bits(a[1], b[1])
    v, n = oracle.normals(lo, "vertex")
    lo.vertices, lo.normals = v, n
    ta, tb = oracle.tangent_space(lo), reference.tangent_space(lo)
    assert same_bits(ta[0], tb[0]) and same_bits(ta[1], tb[1])


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("max_tris", [1, 8])
def test_bvh(oracle, reference, name, max_tris):
    _, hi, _ = prepared(oracle, name)
    a, b = oracle.scene(hi, max_tris), reference.scene(hi, max_tris)
    assert a[0].tobytes() == b[0].tobytes()
    assert same_bits(a[1], b[1]) and same_bits(a[2], b[2])


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_raster(oracle, reference, name, mode):
    lo, _, dirs = prepared(oracle, name)
    for w, h in ((64, 64), (100, 70)):
        a = oracle.raster(lo, w, h, mode, dirs)
        b = reference.raster(lo, w, h, mode, dirs)
        assert len(a["indices"]) == len(b["indices"]) > 0
        for k in a:
            assert np.array_equal(np.asarray(a[k]).view(np.uint32), np.asarray(b[k]).view(np.uint32)), k


def test_raster_drops_triangles_touching_uv_zero(oracle, reference):
    """Src/compute.cpp:136-139: a negative rounded bound wraps to 0xFFFFFFFF
    and is clamped to the width, so the loop never runs."""
    p = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    for inset, expect in ((0.0, 0), (0.01, 256)):
        uv = np.array([[inset, inset], [1 - inset, inset], [1 - inset, 1 - inset], [inset, 1 - inset]], np.float32)
        m = W.MeshArrays(p, uv, np.array([[0, 0, 1]]), np.array([[i, i, 0] for i in range(4)]),
                         np.array([[0, 1, 2], [0, 2, 3]]))
        a = oracle.raster(m, 16, 16, 1)
        b = reference.raster(m, 16, 16, 1)
        assert len(a["indices"]) == len(b["indices"]) == expect


@pytest.mark.parametrize("spp,seed", [(4, 1), (64, 99)])
def test_samples(oracle, reference, spp, seed):
    assert same_bits(oracle.samples(spp, 4096, seed), reference.samples(spp, 4096, seed))


@pytest.mark.parametrize("name", list(MESHES))
def test_shaders(oracle, reference, name):
    lo, hi, dirs = prepared(oracle, name)
    nodes, p4, n4 = oracle.scene(hi)
    cm = oracle.raster(lo, 48, 48, 0, dirs)
    px = pix8(cm)
    for cull in (True, False):
        a = oracle.meshmap(nodes, p4, px, cull)
        b = reference.meshmap(nodes, p4, px, cull)
        assert same_bits(a[0], b[0]) and np.array_equal(a[1], b[1])
    coords, tidx = oracle.meshmap(nodes, p4, px, True)
    hit = tidx != 0xFFFFFFFF
    s = oracle.samples(24, 4096, 5)
    for kind in (0, 1, 2):
        a, _ = oracle.hemisphere(kind, nodes, p4, n4, coords, tidx, s, 24, 0.001, 0.3)
        b = reference.hemisphere(kind, nodes, p4, n4, coords, tidx, s, 24, 0.001, 0.3)
        assert same_bits(a[hit], b[hit]), kind
    for what in (0, 1, 2):
        a = oracle.gather(what, p4, n4, coords, tidx)
        b = reference.gather(what, p4, n4, coords, tidx)
        assert same_bits(a[hit], b[hit])
    g = oracle.gather(2, p4, n4, coords, tidx)
    a = oracle.tangent_transform(cm["normals"], cm["tangents"], cm["bitangents"], g)
    b = reference.tangent_transform(cm["normals"], cm["tangents"], cm["bitangents"], g)
    assert same_bits(a, b)


@pytest.mark.parametrize("max_tris,max_depth", [(8, 8192), (1, 3)])
def test_host_bvh_build_of_a_large_mesh(oracle, reference, max_tris, max_depth):
    """The library's host build (fk_bvh_build + fk_bvh_flatten), whose top
    levels run their passes over chunks on several threads from 2^18
    triangles up, against the reference's own BVH::createBinary +
    fillMeshData on a 627k-triangle heightfield: the same nodes and corner
    arrays, bit for bit (also with the depth limit reached while the splits
    still run in chunks)."""
    from fornos_b200 import api
    _, hi = W.plane_pair(seed=4, lo_quads=8, hi_quads=560, bumps=40)
    assert hi.triangle_count > 1 << 19  # chunked passes at the root and at its children
    v, n = oracle.normals(hi, "vertex")
    hi.vertices, hi.normals = v, n
    mesh = api.Mesh(hi)
    mine = api.BVH.create_binary(mesh, max_tris, max_depth).flatten(mesh)
    ref = reference.scene(hi, max_tris, max_depth)
    assert mine[0].tobytes() == ref[0].tobytes()
    assert same_bits(mine[1], ref[1]) and same_bits(mine[2], ref[2])
