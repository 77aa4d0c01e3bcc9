"""BVH::createBinary + fillMeshData built on the device (fk_bvh_build_flat,
fk_scene_build) against the host build (fk_bvh_build + fk_bvh_flatten, itself
pinned to the reference's Src/bvh.cpp and Src/meshmapping.cpp compiled from
source): nodes and corner arrays bit for bit.

Cases: the test scenes; a larger plane whose top levels run the level passes
with many blocks per node; triangle soups built to reach the rules' corners
(identical triangles that cannot be split, at the top levels and inside the
one-thread subtrees; signed zeros; a NaN vertex; unreferenced positions that
widen the root box); depth and leaf-size limits; tiny meshes.
"""
import numpy as np
import pytest

from fornos_b200 import api
from fornos_b200 import workloads as W
from tests import cases

pytestmark = pytest.mark.gpu


def soup(points, rng=None, extra_positions=None):
    """Triangle soup: triangle f uses points 3f, 3f + 1, 3f + 2."""
    pts = np.asarray(points, np.float32).reshape(-1, 3)
    n = len(pts)
    pos = pts if extra_positions is None else np.concatenate([pts, np.asarray(extra_positions, np.float32)])
    rng = rng or np.random.default_rng(0)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    verts = np.stack([np.arange(n), np.zeros(n, np.int64), np.arange(n)], 1)
    tris = np.arange(n).reshape(-1, 3)
    return W.MeshArrays(pos, np.zeros((1, 2), np.float32), nrm, verts, tris)


def host_flat(mesh, max_tris, max_depth):
    return api.BVH.create_binary(mesh, max_tris, max_depth).flatten(mesh)


def same(ctx, mesh, max_tris=8, max_depth=8192):
    hn, hp, hq = host_flat(mesh, max_tris, max_depth)
    dn, dp, dq = api.BVH.build_flat_device(ctx, mesh, max_tris, max_depth)
    assert len(dn) == len(hn)
    assert np.array_equal(dn.view(np.uint8), hn.view(np.uint8)), "nodes differ"
    assert np.array_equal(dp.view(np.uint32), hp.view(np.uint32)), "positions differ"
    assert np.array_equal(dq.view(np.uint32), hq.view(np.uint32)), "normals differ"
    return hn


@pytest.mark.parametrize("name", ["sphere", "plane", "icosphere"])
def test_device_build_equals_host_on_cases(ctx, name):
    c = getattr(cases, name)()
    same(ctx, c.hm)


def test_device_build_equals_host_large_plane(ctx):
    lo, hi = W.plane_pair(seed=5, lo_quads=8, hi_quads=256, bumps=40)
    m = api.Mesh(hi)
    m.compute_vertex_normals()
    nodes = same(ctx, m)
    assert len(nodes) > 20000


@pytest.mark.parametrize("max_tris,max_depth", [(1, 8192), (3, 8192), (16, 8192), (8, 0), (8, 2), (8, 5), (2, 11)])
def test_device_build_equals_host_limits(ctx, max_tris, max_depth):
    c = cases.sphere()
    same(ctx, c.hm, max_tris, max_depth)


def _random_soup(rng, n, spread=1.0, size=0.05):
    c = rng.uniform(-spread, spread, (n, 1, 3))
    return (c + rng.uniform(-size, size, (n, 3, 3))).astype(np.float32)


def test_device_build_identical_triangles(ctx):
    # 3000 copies of one triangle: no split ever separates them (leaves at the
    # top levels), then 300 copies (inside a one-thread subtree)
    t = np.array([[0.1, 0.2, 0.3], [0.5, 0.2, 0.3], [0.1, 0.9, 0.3]], np.float32)
    same(ctx, api.Mesh(soup(np.tile(t, (3000, 1)))))
    rng = np.random.default_rng(3)
    pts = np.concatenate([np.tile(t, (300, 1)), _random_soup(rng, 200).reshape(-1, 3)])
    same(ctx, api.Mesh(soup(pts)))


def test_device_build_signed_zeros(ctx):
    rng = np.random.default_rng(4)
    pts = _random_soup(rng, 5000, spread=0.5).reshape(-1, 3)
    pick = rng.random(pts.shape) < 0.2
    pts[pick] = np.where(rng.random(pick.sum()) < 0.5, 0.0, -0.0).astype(np.float32)
    same(ctx, api.Mesh(soup(pts)))


def test_device_build_nan_vertex_and_unreferenced_positions(ctx):
    rng = np.random.default_rng(5)
    pts = _random_soup(rng, 2000).reshape(-1, 3)
    pts[17] = np.nan
    extra = np.array([[40.0, -3.0, 7.0], [-25.0, 60.0, -0.0]], np.float32)
    same(ctx, api.Mesh(soup(pts, extra_positions=extra)))


@pytest.mark.parametrize("n", [1, 2, 9, 513, 4097])
def test_device_build_small_meshes(ctx, n):
    rng = np.random.default_rng(n)
    same(ctx, api.Mesh(soup(_random_soup(rng, n).reshape(-1, 3))))


def test_scene_build_equals_uploaded_scene(ctx):
    c = cases.plane()
    up = api.Scene(ctx, c.nodes, c.pos4, c.nrm4)
    built = api.Scene.build(ctx, c.hm, 8, 8192)
    assert built.info() == up.info()
    for tree in (api.TREE_REFERENCE, api.TREE_SAH):
        a, da = up.tree(tree)
        b, db = built.tree(tree)
        assert da == db and np.array_equal(a.view(np.uint32), b.view(np.uint32))
