"""Parity at the benchmarked sizes, through the C ABI, against the
reference's own code compiled on the host (oracle/_ref; the oracle
restatement where that build is absent).

* The 512x512 sphere bake (512x256 perturbed UV sphere, 261,120 triangles;
  height, tangent-space normals, AO 64 spp, min 0.001, max 0.5) in full,
  with the product's default traversal and tuning.  The reference rasterises
  the texel map and builds and flattens the BVH itself, so those arrays are
  compared too.  The mapping runs twice: without a limit against the
  reference's mapping shader, and with the 0.1 maximum distance the
  workload names against the oracle fed the same initial distance; the
  sampling and the gathers run over the limited mapping.
* The 2048x2048 plane bake (1024x1024-quad heightfield, 2,097,152
  triangles; AO + bent normals fused and thickness, 256 spp, min 0.001,
  max 0.3) on every 256th texel.

Bar: texel map, BVH arrays, hit indices, barycentrics and gathers bit-exact;
sampled outputs bit-exact except on at most 0.01 % of texels, each occluder
count within one sample.  The measured fractions are recorded
(tests/.out/records.jsonl).
"""
import numpy as np
import pytest

from fornos_b200 import api
from fornos_b200 import workloads as W
from oracle import parity
from tests.cases import record, same_bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cpu(oracle):
    from oracle.pyoracle import Reference
    try:
        return Reference()
    except OSError:
        return oracle


def _prepare(cpu, lo, hi, tex):
    """Src/fornos.cpp:53-157 on the CPU side: vertex normals of the
    high-poly, tangents and welded directions of the low-poly, raster and
    BVH."""
    v, nrm = cpu.normals(hi, "vertex")
    hi_c = hi.copy()
    hi_c.vertices, hi_c.normals = v, nrm
    lo_c = lo.copy()
    lo_c.tangents, lo_c.bitangents = cpu.tangent_space(lo_c)
    cmap = cpu.raster(lo_c, tex, tex, 0, cpu.normals(lo_c, "welded"))
    nodes, pos4, nrm4 = cpu.scene(hi_c)
    return cmap, nodes, pos4, nrm4


def _gpu_prepare(ctx, lo, hi, tex):
    hm = api.Mesh(hi)
    hm.compute_vertex_normals()
    lm = api.Mesh(lo)
    lm.compute_tangent_space()
    dm = lm.copy()
    dm.compute_vertex_normals_aggressive()
    bvh = api.BVH.create_binary(hm, 8, 8192)
    nodes, pos4, nrm4 = bvh.flatten(hm)
    tmap = api.TexelMap.from_meshes(ctx, lm, dm, tex, tex)
    scene = api.Scene(ctx, nodes, pos4, nrm4)
    return tmap, scene, nodes, pos4, nrm4


def _pix8(cmap, sel=None):
    p, d = cmap["positions"], cmap["directions"]
    if sel is not None:
        p, d = p[sel], d[sel]
    out = np.zeros((len(p), 8), np.float32)
    out[:, 0:3], out[:, 4:7] = p, d
    return out


def _same_scene(nodes, pos4, nrm4, r_nodes, r_pos4, r_nrm4):
    return (nodes.tobytes() == r_nodes.tobytes() and same_bits(pos4, r_pos4) and same_bits(nrm4, r_nrm4))


def test_sphere512_in_full(ctx, oracle, cpu):
    tex, spp, lo_d, hi_d, map_max = 512, 64, 0.001, 0.5, 0.1
    lo, hi = W.sphere_pair(seed=1)
    cmap, r_nodes, r_pos4, r_nrm4 = _prepare(cpu, lo, hi, tex)
    tmap, scene, nodes, pos4, nrm4 = _gpu_prepare(ctx, lo, hi, tex)
    got_map = tmap.download()
    n = tmap.count
    assert np.array_equal(got_map["indices"], cmap["indices"])
    for k in ("positions", "directions", "normals", "tangents", "bitangents"):
        assert same_bits(got_map[k], cmap[k]), k
    assert _same_scene(nodes, pos4, nrm4, r_nodes, r_pos4, r_nrm4)

    pix8 = _pix8(cmap)
    coords, tidx = ctx.buffer(16 * n), ctx.buffer(4 * n)
    # without a limit: the reference's mapping shader
    api.meshmap(ctx, scene, tmap, True, coords, tidx)
    rc, rt = cpu.meshmap(r_nodes, r_pos4, pix8, True)
    m_full = parity.mapping(rc, rt, coords.download(np.float32, (n, 4)), tidx.download(np.uint32, n))
    # with the workload's 0.1 limit: the oracle fed the same initial distance
    api.meshmap(ctx, scene, tmap, True, coords, tidx, max_dist=map_max)
    oc, ot = oracle.meshmap(r_nodes, r_pos4, pix8, True, max_dist=map_max)
    gc, gt = coords.download(np.float32, (n, 4)), tidx.download(np.uint32, n)
    m_lim = parity.mapping(oc, ot, gc, gt)

    samples = api.samples_cosine(spp, api.PERMS, 1)
    sbuf = ctx.upload(samples)
    ao, occ = ctx.buffer(4 * n), ctx.buffer(4 * n)
    api.hemisphere(ctx, scene, coords, tidx, api.AO, spp, lo_d, hi_d, sbuf, ao, None, occ, None, 0, n)
    height, nrm = ctx.buffer(4 * n), ctx.buffer(12 * n)
    api.gather(ctx, scene, api.GATHER_HEIGHT, coords, tidx, height, 0, n)
    api.gather(ctx, scene, api.GATHER_NORMAL, coords, tidx, nrm, 0, n)
    api.tangent_space(ctx, tmap, nrm)
    ctx.check()
    r_ao = cpu.hemisphere(0, r_nodes, r_pos4, r_nrm4, oc, ot, samples, spp, lo_d, hi_d)
    if isinstance(r_ao, tuple):
        r_ao = r_ao[0]
    hit = ot != api.MISS
    ao_fig = parity.sampled(r_ao, ao.download(np.float32, n), hit, spp, gpu_hits=occ.download(np.uint32, n))
    r_height = cpu.gather(0, r_pos4, r_nrm4, oc, ot)
    r_nrm = cpu.tangent_transform(cmap["normals"], cmap["tangents"], cmap["bitangents"],
                                  cpu.gather(2, r_pos4, r_nrm4, oc, ot))
    record("scale:sphere512", texels=n, map_tidx_diff=m_full["tidx_diff_frac"], map_limited_tidx_diff=m_lim[
        "tidx_diff_frac"], ao_out_diff=ao_fig["out_diff_frac"], ao_hits_diff=ao_fig["hits_diff_frac"],
        ao_max_hits_delta=ao_fig["max_hits_delta"])
    assert m_full["tidx_diff_frac"] == 0 and m_full["coords_bits_diff_frac"] == 0
    assert m_lim["tidx_diff_frac"] == 0 and m_lim["coords_bits_diff_frac"] == 0
    assert 0.3 < hit.mean() < (rt != api.MISS).mean()  # the limit drops some hits
    assert same_bits(height.download(np.float32, n)[hit], r_height[hit])
    assert same_bits(nrm.download(np.float32, (n, 3))[hit], r_nrm[hit])
    assert parity.meets_bar({"ao": ao_fig}), ao_fig
    assert 0.0 < r_ao[hit].mean() < 1.0


def test_plane2048_every_256th_texel(ctx, cpu):
    tex, spp, lo_d, hi_d = 2048, 256, 0.001, 0.3
    lo, hi = W.plane_pair(seed=1, lo_quads=64, hi_quads=1024, bumps=200)
    cmap, r_nodes, r_pos4, r_nrm4 = _prepare(cpu, lo, hi, tex)
    tmap, scene, nodes, pos4, nrm4 = _gpu_prepare(ctx, lo, hi, tex)
    n = tmap.count
    assert np.array_equal(tmap.download()["indices"], cmap["indices"])
    assert _same_scene(nodes, pos4, nrm4, r_nodes, r_pos4, r_nrm4)
    coords, tidx = ctx.buffer(16 * n), ctx.buffer(4 * n)
    api.meshmap(ctx, scene, tmap, True, coords, tidx)
    samples = api.samples_cosine(spp, api.PERMS, 1)
    sbuf = ctx.upload(samples)
    ao, bn, th = ctx.buffer(4 * n), ctx.buffer(12 * n), ctx.buffer(4 * n)
    occ, anyhit, th_hits = ctx.buffer(4 * n), ctx.buffer(4 * n), ctx.buffer(4 * n)
    api.hemisphere(ctx, scene, coords, tidx, api.AO_BN, spp, lo_d, hi_d, sbuf, ao, bn, occ, anyhit, 0, n)
    api.hemisphere(ctx, scene, coords, tidx, api.THICK, spp, lo_d, hi_d, sbuf, th, None, th_hits, None, 0, n)
    ctx.check()
    sel = np.arange(0, n, 256, dtype=np.uint32)
    rc, rt = cpu.meshmap(r_nodes, r_pos4, _pix8(cmap, sel), True)
    m = parity.mapping(rc, rt, coords.download(np.float32, (n, 4))[sel], tidx.download(np.uint32, n)[sel])
    full_c = np.zeros((n, 4), np.float32)
    full_t = np.full(n, api.MISS, np.uint32)
    full_c[sel], full_t[sel] = rc, rt
    hit = rt != api.MISS
    figs = {"mapping": m}
    for kind, name, buf, w in ((0, "ao", ao, 1), (1, "bn", bn, 3), (2, "thick", th, 1)):
        r = cpu.hemisphere(kind, r_nodes, r_pos4, r_nrm4, full_c, full_t, samples, spp, lo_d, hi_d, texels=sel)
        if isinstance(r, tuple):
            r = r[0]
        g = buf.download(np.float32, n if w == 1 else (n, 3))[sel]
        figs[name] = parity.sampled(r, g, hit, spp if kind == 0 else None,
                                    gpu_hits=occ.download(np.uint32, n)[sel] if kind == 0 else None)
    record("scale:plane2048:1/256", texels=len(sel), hit_texels=hit.sum(), map_tidx_diff=m["tidx_diff_frac"],
           **{"%s_out_diff" % k: figs[k]["out_diff_frac"] for k in ("ao", "bn", "thick")},
           ao_hits_diff=figs["ao"]["hits_diff_frac"], ao_max_hits_delta=figs["ao"]["max_hits_delta"])
    assert hit.mean() > 0.9
    assert parity.meets_bar(figs), figs
