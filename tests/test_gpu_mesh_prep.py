"""Mesh preprocessing on the device (fk_mesh_compute_normals_device,
fk_mesh_compute_tangent_space_device) against the host generators
(fk_mesh_compute_*, themselves pinned to the reference's Src/mesh.cpp compiled
from source) and the oracle: vertex tables exactly, normals / tangents /
bitangents bit for bit (NaN payloads aside).

Cases: the test scenes' low- and high-poly meshes; the same meshes with
shuffled triangle and vertex order (the sums must follow triangle order, not
storage order); welds across position indices, signed zeros included; a fan
of 20,000 triangles round one position; unreferenced positions and vertices;
degenerate triangles; a NaN coordinate; a 300k-triangle soup on a coarse
lattice (many welds, several tiles and digit passes per sort); no triangles;
index errors, which leave the mesh as it was.
"""
import numpy as np
import pytest

from fornos_b200 import api
from fornos_b200 import workloads as W
from tests.cases import same_bits

pytestmark = pytest.mark.gpu

METHODS = {"face": api.NORMALS_FACE, "vertex": api.NORMALS_VERTEX, "welded": api.NORMALS_WELDED}
HOST = {"face": "compute_face_normals", "vertex": "compute_vertex_normals",
        "welded": "compute_vertex_normals_aggressive"}

SCENES = {
    "sphere": lambda: W.sphere_pair(seed=1, lo_seg=(32, 16), hi_seg=(64, 32)),
    "plane": lambda: W.plane_pair(seed=2, lo_quads=8, hi_quads=64, bumps=20),
    "icosphere": lambda: W.icosphere_pair(seed=3, lo_subdiv=1, hi_subdiv=4),
}


def host_normals(m, which):
    h = api.Mesh(m)
    getattr(h, HOST[which])()
    return h.arrays()


def device_normals(ctx, m, which):
    d = api.Mesh(m)
    d.compute_normals_device(ctx, METHODS[which])
    return d.arrays()


def same_normals(ctx, m, which):
    h, d = host_normals(m, which), device_normals(ctx, m, which)
    assert np.array_equal(h.vertices, d.vertices)
    assert same_bits(h.normals, d.normals)
    return d


def same_tangents(ctx, m):
    h, d = api.Mesh(m), api.Mesh(m)
    h.compute_tangent_space()
    d.compute_tangent_space_device(ctx)
    a, b = h.arrays(), d.arrays()
    assert same_bits(a.tangents, b.tangents) and same_bits(a.bitangents, b.bitangents)
    return b


def shuffled(m, seed):
    """The same surface with triangles and vertices stored in another order
    (and each triangle's corners rotated)."""
    rng = np.random.default_rng(seed)
    nv = len(m.vertices)
    vperm = rng.permutation(nv)
    inv = np.empty(nv, np.int64)
    inv[vperm] = np.arange(nv)
    tris = inv[m.triangles.astype(np.int64)][rng.permutation(m.triangle_count)]
    rot = rng.integers(0, 3, len(tris))
    tris = np.stack([tris[np.arange(len(tris)), (rot + k) % 3] for k in range(3)], 1)
    return W.MeshArrays(m.positions, m.texcoords, m.normals, m.vertices[vperm], tris)


def soup(pos, tris, uv=None, nrm=None):
    """One vertex per position: vertex i = (position i, texcoord i, normal i)."""
    pos = np.asarray(pos, np.float32).reshape(-1, 3)
    n = len(pos)
    uv = np.zeros((n, 2), np.float32) if uv is None else np.asarray(uv, np.float32)
    nrm = np.zeros((n, 3), np.float32) if nrm is None else np.asarray(nrm, np.float32)
    verts = np.stack([np.arange(n)] * 3, 1)
    return W.MeshArrays(pos, uv, nrm, verts, np.asarray(tris, np.int64).reshape(-1, 3))


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("which", list(METHODS))
def test_scene_normals(ctx, oracle, name, which):
    for m in SCENES[name]():
        d = same_normals(ctx, m, which)
        ov, on = oracle.normals(m, which)
        assert np.array_equal(d.vertices, ov) and same_bits(d.normals, on)


@pytest.mark.parametrize("name", list(SCENES))
def test_scene_tangents(ctx, oracle, name):
    lo, _ = SCENES[name]()
    d = same_tangents(ctx, lo)
    t, b = oracle.tangent_space(lo)
    assert same_bits(d.tangents, t) and same_bits(d.bitangents, b)


@pytest.mark.parametrize("which", list(METHODS))
@pytest.mark.parametrize("seed", [5, 6])
def test_shuffled_order(ctx, which, seed):
    lo, hi = SCENES["icosphere"]()
    same_normals(ctx, shuffled(hi, seed), which)
    same_tangents(ctx, shuffled(lo, seed))


def test_weld_across_indices_and_signed_zeros(ctx):
    # a grid stored as a triangle soup: every triangle has its own positions,
    # equal values repeat at many indices; half the zero coordinates are -0
    rng = np.random.default_rng(11)
    g = 40
    xs = np.linspace(-1, 1, g + 1, dtype=np.float32)
    pts = []
    for i in range(g):
        for j in range(g):
            a, b, c, d = (xs[i], xs[j]), (xs[i + 1], xs[j]), (xs[i + 1], xs[j + 1]), (xs[i], xs[j + 1])
            for tri in ((a, b, c), (a, c, d)):
                for (x, y) in tri:
                    pts.append((x, y, np.float32(0.05) * np.float32(np.sin(3 * x + 2 * y))))
    pos = np.asarray(pts, np.float32)
    zero = pos == 0
    pos[zero & (rng.random(pos.shape) < 0.5)] = np.float32(-0.0)
    m = soup(pos, np.arange(len(pos)))
    d = same_normals(ctx, m, "welded")
    assert len(d.normals) == (g + 1) ** 2  # every lattice point welded once
    for which in ("face", "vertex"):
        same_normals(ctx, m, which)


def test_fan(ctx):
    # 20,000 triangles round one centre position: one long group per sort
    n = 20000
    ang = np.linspace(0, 2 * np.pi, n, endpoint=False)
    rim = np.stack([np.cos(ang), np.sin(ang), 0.1 * np.sin(7 * ang)], 1).astype(np.float32)
    pos = np.concatenate([np.zeros((1, 3), np.float32), rim])
    tris = np.stack([np.zeros(n, np.int64), 1 + np.arange(n), 1 + (np.arange(n) + 1) % n], 1)
    uv = np.concatenate([[[0.5, 0.5]], 0.5 + 0.5 * rim[:, :2]]).astype(np.float32)
    m = soup(pos, tris, uv=uv)
    for which in METHODS:
        same_normals(ctx, m, which)
    h = host_normals(m, "vertex")
    same_tangents(ctx, h)


def test_unreferenced_and_degenerate(ctx):
    rng = np.random.default_rng(12)
    pos = rng.normal(size=(60, 3)).astype(np.float32)
    pos[50:] = pos[0]            # duplicates of a used position, never referenced themselves
    tris = rng.integers(0, 40, (80, 3))
    tris[:5, 1] = tris[:5, 0]    # zero-area triangles: NaN face normals
    tris[5] = (7, 7, 7)
    m = soup(pos, tris, uv=rng.random((60, 2)))
    for which in METHODS:
        same_normals(ctx, m, which)
    same_tangents(ctx, host_normals(m, "vertex"))


def test_nan_coordinate(ctx):
    lo, _ = SCENES["plane"]()
    m = lo.copy()
    m.positions[3, 1] = np.float32(np.nan)
    for which in METHODS:
        same_normals(ctx, m, which)
    same_tangents(ctx, m)


def test_large_soup(ctx):
    # 300k triangles on a 64^3 lattice: many welds, ids above 2^16, several
    # tiles and digit passes in every sort
    rng = np.random.default_rng(13)
    nf = 300_000
    lattice = rng.integers(0, 64, (nf * 3, 3)).astype(np.float32) / np.float32(8) - np.float32(4)
    m = soup(lattice, np.arange(3 * nf), uv=rng.random((3 * nf, 2)))
    for which in METHODS:
        same_normals(ctx, m, which)
    same_tangents(ctx, host_normals(m, "vertex"))


def test_no_triangles(ctx):
    m = W.MeshArrays(np.ones((4, 3), np.float32), np.zeros((4, 2), np.float32), np.zeros((4, 3), np.float32),
                     np.stack([np.arange(4)] * 3, 1), np.zeros((0, 3), np.uint32))
    for which in METHODS:
        same_normals(ctx, m, which)
    same_tangents(ctx, m)


def test_index_errors_leave_mesh(ctx):
    lo, _ = SCENES["sphere"]()
    bad = lo.copy()
    bad.vertices[3, 1] = len(bad.texcoords)  # texcoord index out of range
    d = api.Mesh(bad)
    with pytest.raises(api.FornosError) as e:
        d.compute_tangent_space_device(ctx)
    assert e.value.code == -1  # FK_ERR_INVALID
    a = d.arrays()
    assert a.tangents is None and np.array_equal(a.vertices, bad.vertices)
    with pytest.raises(api.FornosError):
        d.compute_normals_device(ctx, 7)
