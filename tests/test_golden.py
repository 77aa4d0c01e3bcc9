"""Replays the committed golden fixtures (tests/golden/*.npz, generated by
tests/golden/make_golden.py from the reference's own code compiled on the
host) against the oracle, the product's host code and, on a GPU, the
product's kernels.  Comparisons are bit for bit (NaN payloads canonical)."""
import hashlib
import os

import numpy as np
import pytest

from fornos_b200 import api
from fornos_b200 import workloads as W
from tests.cases import same_bits

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["sphere", "plane", "icosphere"]


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    return {k: z[k] for k in z.files}


def mesh(g, prefix, normals=None):
    v = g[prefix + "vertices"] if normals is None else g["%s%s_vertices" % (prefix, normals)]
    n = g[prefix + "normals"] if normals is None else g["%s%s_normals" % (prefix, normals)]
    return W.MeshArrays(g[prefix + "positions"], g[prefix + "texcoords"], n, v, g[prefix + "triangles"])


def params(g):
    tex, spp, seed, lo, hi = g["params"]
    return int(tex), int(spp), int(seed), float(np.float32(lo)), float(np.float32(hi))


def nodes_of(g):
    return np.ascontiguousarray(g["nodes"]).view(api.NODE_DTYPE).reshape(-1)


def pix8(g):
    n = len(g["map0_indices"])
    out = np.zeros((n, 8), np.float32)
    out[:, 0:3], out[:, 4:7] = g["map0_positions"], g["map0_directions"]
    return out


def pixt12(g):
    n = len(g["map0_indices"])
    out = np.zeros((n, 12), np.float32)
    out[:, 0:3], out[:, 4:7], out[:, 8:11] = g["map0_normals"], g["map0_tangents"], g["map0_bitangents"]
    return out


# ------------------------------------------------------------------ oracle
@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_golden(oracle, name):
    g = load(name)
    tex, spp, seed, lo_d, hi_d = params(g)
    lo, hi = mesh(g, "lo_"), mesh(g, "hi_")
    for which in ("face", "vertex", "welded"):
        for m, p in ((lo, "lo_"), (hi, "hi_")):
            v, n = oracle.normals(m, which)
            assert np.array_equal(v, g[p + which + "_vertices"]) and same_bits(n, g[p + which + "_normals"])
    t, b = oracle.tangent_space(lo)
    assert same_bits(t, g["lo_tangents"]) and same_bits(b, g["lo_bitangents"])
    hv = mesh(g, "hi_", "vertex")
    nodes, p4, n4 = oracle.scene(hv, 8)
    assert nodes.tobytes() == nodes_of(g).tobytes() and same_bits(p4, g["pos4"]) and same_bits(n4, g["nrm4"])
    lo.tangents, lo.bitangents = t, b
    dirs = (g["lo_welded_vertices"], g["lo_welded_normals"])
    for mode in (0, 1, 2):
        cm = oracle.raster(lo, tex, tex, mode, dirs)
        for k, v in cm.items():
            assert same_bits(v, g["map%d_%s" % (mode, k)]) if v.dtype == np.float32 else np.array_equal(
                v, g["map%d_%s" % (mode, k)])
    s = oracle.samples(spp, 4096, seed)
    assert hashlib.sha256(s.tobytes()).digest() == g["samples_sha256"].tobytes()
    for cull in (0, 1):
        c, ti = oracle.meshmap(nodes, p4, pix8(g), bool(cull))
        assert same_bits(c, g["coords%d" % cull]) and np.array_equal(ti, g["tidx%d" % cull])
    coords, tidx = g["coords1"], g["tidx1"]
    hit = tidx != api.MISS
    assert hit.mean() > 0.3
    for kind, label in ((0, "ao"), (1, "bn"), (2, "thick")):
        out, _ = oracle.hemisphere(kind, nodes, p4, n4, coords, tidx, s, spp, lo_d, hi_d)
        assert same_bits(out[hit], g[label][hit]), label
    for what, label in ((0, "height"), (1, "position"), (2, "normal")):
        assert same_bits(oracle.gather(what, p4, n4, coords, tidx)[hit], g[label][hit])
    ts = oracle.tangent_transform(g["map0_normals"], g["map0_tangents"], g["map0_bitangents"], g["normal"])
    assert same_bits(ts, g["normal_ts"])


# ------------------------------------------------------------------ product host code
@pytest.mark.parametrize("name", NAMES)
def test_product_host_matches_golden(lib, name):
    g = load(name)
    tex, spp, seed, _, _ = params(g)
    for prefix in ("lo_", "hi_"):
        for which, fn in (("face", "compute_face_normals"), ("vertex", "compute_vertex_normals"),
                          ("welded", "compute_vertex_normals_aggressive")):
            m = api.Mesh(mesh(g, prefix))
            getattr(m, fn)()
            a = m.arrays()
            assert np.array_equal(a.vertices, g[prefix + which + "_vertices"])
            assert same_bits(a.normals, g[prefix + which + "_normals"])
    lm = api.Mesh(mesh(g, "lo_"))
    lm.compute_tangent_space()
    a = lm.arrays()
    assert same_bits(a.tangents, g["lo_tangents"]) and same_bits(a.bitangents, g["lo_bitangents"])
    hm = api.Mesh(mesh(g, "hi_", "vertex"))
    nodes, p4, n4 = api.BVH.create_binary(hm, 8).flatten(hm)
    assert nodes.tobytes() == nodes_of(g).tobytes() and same_bits(p4, g["pos4"]) and same_bits(n4, g["nrm4"])
    s = api.samples_cosine(spp, api.PERMS, seed)
    assert hashlib.sha256(s.tobytes()).digest() == g["samples_sha256"].tobytes()


# ------------------------------------------------------------------ product kernels
@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_kernels_match_golden(ctx, name):
    g = load(name)
    tex, spp, seed, lo_d, hi_d = params(g)
    lo = mesh(g, "lo_")
    lo.tangents, lo.bitangents = g["lo_tangents"], g["lo_bitangents"]
    lm = api.Mesh(lo)
    dm = api.Mesh(W.MeshArrays(lo.positions, lo.texcoords, g["lo_welded_normals"], g["lo_welded_vertices"],
                               lo.triangles))
    for mode in (0, 1, 2):
        tm = api.TexelMap.rasterize(ctx, lm, tex, tex, mode, None if mode == 1 else dm)
        got = tm.download()
        for k, v in got.items():
            ref = g["map%d_%s" % (mode, k)]
            assert (same_bits(v, ref) if v.dtype == np.float32 else np.array_equal(v, ref)), (mode, k)
    tm = api.TexelMap.from_host(ctx, tex, tex, pix8(g), pixt12(g), g["map0_indices"])
    scene = api.Scene(ctx, nodes_of(g), g["pos4"], g["nrm4"])
    n = tm.count
    coords, tidx = ctx.buffer(16 * n), ctx.buffer(4 * n)
    for cull in (0, 1):
        api.meshmap(ctx, scene, tm, bool(cull), coords, tidx)
        assert same_bits(coords.download(np.float32, (n, 4)), g["coords%d" % cull])
        assert np.array_equal(tidx.download(np.uint32, n), g["tidx%d" % cull])
    hit = g["tidx1"] != api.MISS
    sbuf = ctx.upload(api.samples_cosine(spp, api.PERMS, seed))
    for kind, label, width in ((api.AO, "ao", 1), (api.BN, "bn", 3), (api.THICK, "thick", 1)):
        for trav in (api.TRAVERSE_SKIP | api.SCHEDULE_STATIC, api.TRAVERSE_SKIP | api.SCHEDULE_DYNAMIC):
            out = ctx.buffer(4 * width * n)
            api.hemisphere(ctx, scene, coords, tidx, kind, spp, lo_d, hi_d, sbuf, out, count=n, traverse=trav)
            got = out.download(np.float32, n if width == 1 else (n, 3))
            assert same_bits(got[hit], g[label][hit]), (label, trav)
    for what, label, width in ((api.GATHER_HEIGHT, "height", 1), (api.GATHER_POSITION, "position", 3),
                               (api.GATHER_NORMAL, "normal", 3)):
        out = ctx.buffer(4 * width * n)
        api.gather(ctx, scene, what, coords, tidx, out, 0, n)
        got = out.download(np.float32, n if width == 1 else (n, 3))
        assert same_bits(got[hit], g[label][hit]), label
        if what == api.GATHER_NORMAL:
            api.tangent_space(ctx, tm, out)
            assert same_bits(out.download(np.float32, (n, 3)), g["normal_ts"])
