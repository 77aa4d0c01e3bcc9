"""CUDA path vs the CPU oracle, through the C ABI, on seeded small cases.

Bar: bit-exact for the texel map, hit indices, barycentrics, distances,
occluder counts and every aggregated output of the skip-pointer traversal
(the reference's own visit order).  The ordered traversal may differ only
where a hit distance rounds below its leaf box's entry distance; the tests
bound those texels at 0.01 % and their occluder counts at one sample, and
record the measured fractions (tests/.out/records.jsonl).
"""
import numpy as np
import pytest

from fornos_b200 import api
from tests import cases
from tests.cases import bits, record, same_bits

pytestmark = pytest.mark.gpu

CASES = {"sphere": cases.sphere, "plane": cases.plane, "icosphere": cases.icosphere}
_cache = {}


def case(name):
    if name not in _cache:
        _cache[name] = CASES[name]()
    return _cache[name]


def oracle_map(oracle, c, w, h, mode):
    return oracle.raster(c.lo, w, h, mode, None if mode == 1 else c.dirs)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("size", [(64, 64), (100, 70)])
def test_raster_matches_oracle(ctx, oracle, name, mode, size):
    c = case(name)
    w, h = size
    ref = oracle_map(oracle, c, w, h, mode)
    tm = api.TexelMap.rasterize(ctx, c.lm, w, h, mode, None if mode == 1 else c.dm, 0.05)
    got = tm.download()
    assert tm.count == len(ref["indices"]) and tm.count > 0
    assert np.array_equal(got["indices"], ref["indices"])
    for k in ("positions", "directions", "normals", "tangents", "bitangents"):
        assert same_bits(got[k], ref[k]), k


def mapped(ctx, oracle, c, w=64, h=64, cull=True):
    ref = oracle_map(oracle, c, w, h, 0)
    tm = api.TexelMap.from_host(ctx, w, h, cases.pix8(ref), cases.pixt12(ref), ref["indices"])
    mm = api.MeshMapping(ctx)
    mm.init(tm, c.hm, c.bvh, cull)
    mm.run()
    return ref, tm, mm


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("cull", [True, False])
def test_meshmap_matches_oracle(ctx, oracle, name, cull):
    c = case(name)
    ref, tm, mm = mapped(ctx, oracle, c, cull=cull)
    coords, tidx = mm.results()
    n = tm.count
    oc, ot = oracle.meshmap(c.nodes, c.pos4, cases.pix8(ref), cull)
    assert np.array_equal(tidx[:n], ot)
    assert same_bits(coords[:n], oc)
    assert (tidx[n:] == api.MISS).all()
    assert (ot != api.MISS).mean() > 0.5


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("cull", [True, False])
@pytest.mark.parametrize("max_dist", [0.1, 0.02])
def test_meshmap_max_distance_matches_oracle(ctx, oracle, name, cull, max_dist):
    """fk_meshmap with a maximum distance (the walks' initial closest
    distance) against the oracle fed the same initial distance: hits at or
    beyond it are dropped, misses write FLT_MAX, and some texels of every case
    lose their hit."""
    c = case(name)
    ref, tm, mm = mapped(ctx, oracle, c, cull=cull)
    n = tm.count
    coords, tidx = ctx.buffer(16 * n), ctx.buffer(4 * n)
    api.meshmap(ctx, mm.scene, tm, cull, coords, tidx, max_dist=max_dist)
    oc, ot = oracle.meshmap(c.nodes, c.pos4, cases.pix8(ref), cull, max_dist=max_dist)
    got_t = tidx.download(np.uint32, n)
    assert np.array_equal(got_t, ot)
    assert same_bits(coords.download(np.float32, (n, 4)), oc)
    full_t = mm.results()[1][:n]
    hit = ot != api.MISS
    assert (oc[hit, 0] < np.float32(max_dist)).all() and (oc[~hit, 0] == api.FLT_MAX).all()
    assert hit.sum() <= (full_t != api.MISS).sum()
    if max_dist < 0.05:  # every case has mapping distances beyond 0.02
        assert hit.sum() < (full_t != api.MISS).sum()
    # a hit under the limit is the unlimited walk's hit (grazing hits on box faces aside)
    assert (ot[hit] == full_t[hit]).mean() >= 0.999


def test_meshmap_chunked_equals_whole(ctx, oracle):
    c = case("sphere")
    ref, tm, mm = mapped(ctx, oracle, c)
    whole = mm.results()
    mm2 = api.MeshMapping(ctx)
    mm2.init(tm, c.hm, c.bvh, True)
    mm2.set_work_per_step(333)
    steps = 0
    while not mm2.run_step():
        steps += 1
        assert 0.0 < mm2.progress() < 1.0
    assert steps == (tm.count - 1) // 333
    part = mm2.results()
    assert same_bits(whole[0], part[0]) and np.array_equal(whole[1], part[1])


def run_hemi(ctx, mm, kind, spp, lo, hi, traverse, seed=7):
    samples = api.samples_cosine(spp, api.PERMS, seed)
    sbuf = ctx.upload(samples)
    n = mm.tmap.count
    out0 = ctx.buffer(12 * n)
    out1 = ctx.buffer(12 * n)
    h0, h1 = ctx.buffer(4 * n), ctx.buffer(4 * n)
    api.hemisphere(ctx, mm.scene, mm.coords, mm.coords_tidx, kind, spp, lo, hi, sbuf, out0,
                   out1 if kind == api.AO_BN else None, h0, h1 if kind == api.AO_BN else None, 0, n,
                   traverse=traverse)
    w0 = 3 if kind == api.BN else 1
    r = [out0.download(np.float32, (n, w0) if w0 == 3 else n), h0.download(np.uint32, n)]
    if kind == api.AO_BN:
        r += [out1.download(np.float32, (n, 3)), h1.download(np.uint32, n)]
    return samples, r


def oracle_hemi(oracle, c, mm, kind, samples, spp, lo, hi):
    coords, tidx = mm.results()
    n = mm.tmap.count
    out, hits = oracle.hemisphere(kind, c.nodes, c.pos4, c.nrm4, coords[:n], tidx[:n], samples, spp, lo, hi)
    return out, hits, tidx[:n]


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kind", [api.AO, api.BN, api.THICK])
@pytest.mark.parametrize("spp", [16, 40])
@pytest.mark.parametrize("sched", [api.SCHEDULE_STATIC, api.SCHEDULE_DYNAMIC,
                                   api.SCHEDULE_DYNAMIC | api.EXACT_BOX_TESTS])
def test_hemisphere_skip_is_bit_exact(ctx, oracle, name, kind, spp, sched):
    c = case(name)
    _, _, mm = mapped(ctx, oracle, c)
    lo, hi = 0.001, 0.3
    samples, (out, hits) = run_hemi(ctx, mm, kind, spp, lo, hi, api.TRAVERSE_SKIP | sched)
    ref, rhits, tidx = oracle_hemi(oracle, c, mm, kind, samples, spp, lo, hi)
    hit = tidx != api.MISS
    assert hit.mean() > 0.5
    assert np.array_equal(hits[hit], rhits[hit])
    assert same_bits(out[hit], ref[hit])
    miss_val = {api.AO: 1.0, api.BN: 0.0, api.THICK: hi}[kind]
    assert np.all(out[~hit] == miss_val) and np.all(hits[~hit] == 0)
    assert 0 < hits[hit].sum() < spp * hit.sum()


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kind", [api.AO, api.BN, api.THICK])
@pytest.mark.parametrize("sched", [api.SCHEDULE_STATIC, api.SCHEDULE_DYNAMIC,
                                   api.SCHEDULE_DYNAMIC | api.EXACT_BOX_TESTS])
def test_hemisphere_ordered_matches(ctx, oracle, name, kind, sched):
    c = case(name)
    _, _, mm = mapped(ctx, oracle, c)
    spp, lo, hi = 32, 0.001, 0.3
    samples, (out, hits) = run_hemi(ctx, mm, kind, spp, lo, hi, api.TRAVERSE_ORDERED | sched)
    ref, rhits, tidx = oracle_hemi(oracle, c, mm, kind, samples, spp, lo, hi)
    hit = tidx != api.MISS
    exact_hits = hits[hit] == rhits[hit]
    if kind == api.BN:
        ok = np.all(bits(out[hit]) == bits(ref[hit]), axis=1)
    else:
        ok = bits(out[hit]) == bits(ref[hit])
    record("ordered:%s:%d:%d" % (name, kind, sched), texels=hit.sum(), hit_diff=(~exact_hits).mean(),
           out_diff=(~ok).mean())
    assert np.abs(hits[hit].astype(np.int64) - rhits[hit]).max() <= 1
    assert (~exact_hits).mean() <= 1e-4  # at most 0.01 % of texels
    assert (~ok).mean() <= 1e-4


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kind", [api.AO, api.BN, api.THICK, api.AO_BN])
@pytest.mark.parametrize("exact", [False, True])
def test_hemisphere_ordered4_matches(ctx, oracle, name, kind, exact):
    """The collapsed 4-wide layout holds the same leaves and leaf boxes, so it
    meets the ordered traversal's bar against the reference order."""
    c = case(name)
    _, _, mm = mapped(ctx, oracle, c)
    spp, lo, hi = 32, 0.001, 0.3
    flags = api.TRAVERSE_ORDERED4 | api.SCHEDULE_DYNAMIC | (api.EXACT_BOX_TESTS if exact else 0)
    samples, got = run_hemi(ctx, mm, kind, spp, lo, hi, flags)
    k = api.AO if kind == api.AO_BN else kind
    ref, rhits, tidx = oracle_hemi(oracle, c, mm, k, samples, spp, lo, hi)
    hit = tidx != api.MISS
    out, hits = got[0], got[1]
    ok = bits(out[hit]) == bits(ref[hit])
    if kind == api.BN:
        ok = np.all(ok, axis=1)
    record("ordered4:%s:%d:%d" % (name, kind, exact), texels=hit.sum(), hit_diff=(hits[hit] != rhits[hit]).mean(),
           out_diff=(~ok).mean())
    assert np.abs(hits[hit].astype(np.int64) - rhits[hit]).max() <= 1
    assert (hits[hit] != rhits[hit]).mean() <= 1e-4  # at most 0.01 % of texels
    assert (~ok).mean() <= 1e-4
    if kind == api.AO_BN:
        bref, bhits, _ = oracle_hemi(oracle, c, mm, api.BN, samples, spp, lo, hi)
        bok = np.all(bits(got[2][hit]) == bits(bref[hit]), axis=1)
        record("ordered4_bn_half:%s:%d" % (name, exact), texels=hit.sum(),
               hit_diff=(got[3][hit] != bhits[hit]).mean(), out_diff=(~bok).mean())
        assert np.abs(got[3][hit].astype(np.int64) - bhits[hit]).max() <= 1
        assert (got[3][hit] != bhits[hit]).mean() <= 1e-4  # at most 0.01 % of texels
        assert (~bok).mean() <= 1e-4


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kind", [api.AO, api.BN, api.THICK])
@pytest.mark.parametrize("trav", [api.TRAVERSE_ORDERED, api.TRAVERSE_ORDERED4, api.TRAVERSE_SKIP])
@pytest.mark.parametrize("tree", [api.TREE_REFERENCE, api.TREE_SAH])
def test_either_inner_tree_matches(ctx, oracle, name, kind, trav, tree):
    """The reference's inner tree or one rebuilt over the same leaves (the
    default): the ordered traversals meet their bar against the reference
    order, the skip walk stays bit-exact."""
    c = case(name)
    _, _, mm = mapped(ctx, oracle, c)
    mm.scene.set_tree(tree)
    try:
        spp, lo, hi = 32, 0.001, 0.3
        samples, (out, hits) = run_hemi(ctx, mm, kind, spp, lo, hi, trav | api.SCHEDULE_DYNAMIC)
        ctx.check()
    finally:
        mm.scene.set_tree(api.TREE_SAH)
    ref, rhits, tidx = oracle_hemi(oracle, c, mm, kind, samples, spp, lo, hi)
    hit = tidx != api.MISS
    if trav == api.TRAVERSE_SKIP:
        assert np.array_equal(hits[hit], rhits[hit]) and same_bits(out[hit], ref[hit])
        return
    ok = bits(out[hit]) == bits(ref[hit])
    if kind == api.BN:
        ok = np.all(ok, axis=1)
    record("tree:%s:%d:%d:%d" % (name, kind, trav, tree), texels=hit.sum(),
           hit_diff=(hits[hit] != rhits[hit]).mean(), out_diff=(~ok).mean())
    assert np.abs(hits[hit].astype(np.int64) - rhits[hit]).max() <= 1
    assert (hits[hit] != rhits[hit]).mean() <= 1e-4  # at most 0.01 % of texels
    assert (~ok).mean() <= 1e-4


@pytest.mark.parametrize("knobs", [dict(ray_order=0), dict(ray_order=1), dict(top_records=64),
                                   dict(top_records=1024), dict(l2_persist=1), dict(l2_persist=2),
                                   dict(ray_order=1, top_records=256, l2_persist=1)])
@pytest.mark.parametrize("trav", [api.TRAVERSE_ORDERED, api.TRAVERSE_ORDERED4, api.TRAVERSE_SKIP])
def test_tuning_knobs_leave_results_unchanged(ctx, oracle, knobs, trav):
    """Ray order, staged top records and L2 windows change only where and when
    work runs: every output and count equals the context defaults' bit for
    bit, on both trees, for spp a multiple of 32 (where the sector order
    applies) and not."""
    c = case("plane")
    _, _, mm = mapped(ctx, oracle, c)
    base = ctx.get_tuning()
    for tree in (api.TREE_SAH, api.TREE_REFERENCE):
        mm.scene.set_tree(tree)
        for kind, spp in ((api.AO_BN, 64), (api.THICK, 40)):
            ctx.set_tuning(**dict(base, ray_order=0, top_records=0, l2_persist=0))
            _, want = run_hemi(ctx, mm, kind, spp, 0.001, 0.3, trav | api.SCHEDULE_DYNAMIC)
            ctx.set_tuning(**dict(base, **knobs))
            try:
                _, got = run_hemi(ctx, mm, kind, spp, 0.001, 0.3, trav | api.SCHEDULE_DYNAMIC)
                ctx.check()
            finally:
                ctx.set_tuning(**base)
            for a, b in zip(got, want):
                assert (same_bits(a, b) if a.dtype == np.float32 else np.array_equal(a, b)), (tree, kind)
    mm.scene.set_tree(api.TREE_SAH)


def test_ordered4_needs_the_dynamic_schedule(ctx, oracle):
    _, _, mm = mapped(ctx, oracle, case("sphere"))
    with pytest.raises(api.FornosError):
        run_hemi(ctx, mm, api.AO, 8, 0.0, 0.3, api.TRAVERSE_ORDERED4 | api.SCHEDULE_STATIC)


def test_ao_bn_fused_equals_separate(ctx, oracle):
    c = case("plane")
    _, _, mm = mapped(ctx, oracle, c)
    spp, lo, hi = 48, 0.001, 0.3
    for sched in (api.SCHEDULE_STATIC, api.SCHEDULE_DYNAMIC):
        _, (ao, aoh) = run_hemi(ctx, mm, api.AO, spp, lo, hi, api.TRAVERSE_SKIP | sched)
        _, (bn, bnh) = run_hemi(ctx, mm, api.BN, spp, lo, hi, api.TRAVERSE_SKIP | sched)
        _, (fa, fah, fb, fbh) = run_hemi(ctx, mm, api.AO_BN, spp, lo, hi, api.TRAVERSE_SKIP | sched)
        assert same_bits(ao, fa) and np.array_equal(aoh, fah)
        assert same_bits(bn, fb) and np.array_equal(bnh, fbh)


@pytest.mark.parametrize("name", list(CASES))
def test_gathers_match_oracle(ctx, oracle, name):
    c = case(name)
    ref, tm, mm = mapped(ctx, oracle, c)
    coords, tidx = mm.results()
    n = tm.count
    hit = tidx[:n] != api.MISS
    for what, width in ((api.GATHER_HEIGHT, 1), (api.GATHER_POSITION, 3), (api.GATHER_NORMAL, 3)):
        out = ctx.buffer(4 * width * n)
        api.gather(ctx, mm.scene, what, mm.coords, mm.coords_tidx, out, 0, n)
        got = out.download(np.float32, n if width == 1 else (n, 3))
        exp = oracle.gather(what, c.pos4, c.nrm4, coords[:n], tidx[:n])
        assert same_bits(got[hit], exp[hit]), what
        if width == 3:
            assert np.all(got[~hit] == 0)
    out = ctx.buffer(12 * n)
    api.gather(ctx, mm.scene, api.GATHER_NORMAL, mm.coords, mm.coords_tidx, out, 0, n)
    api.tangent_space(ctx, tm, out)
    got = out.download(np.float32, (n, 3))
    nrm = oracle.gather(2, c.pos4, c.nrm4, coords[:n], tidx[:n])
    exp = oracle.tangent_transform(ref["normals"], ref["tangents"], ref["bitangents"], nrm)
    assert same_bits(got[hit], exp[hit])


def test_solver_api_end_to_end(ctx, oracle):
    """MeshMapping + the six solvers as the runner drives them (Src/fornos.cpp:162-237)."""
    c = case("sphere")
    tm = api.TexelMap.from_meshes(ctx, c.lm, c.dm, 64, 64)
    mm = api.MeshMapping(ctx)
    mm.init(tm, c.hm, c.bvh, True)
    mm.run()
    n = tm.count
    coords, tidx = mm.results()
    ref = tm.download()
    hit = tidx[:n] != api.MISS
    spp, lo, hi = 32, 0.01, 0.5
    samples = api.samples_cosine(spp, api.PERMS, 11)
    solvers = {
        "height": api.HeightSolver(ctx),
        "position": api.PositionSolver(ctx),
        "normals": api.NormalsSolver(ctx, tangent_space=True),
        "ao": api.AmbientOcclusionSolver(ctx, spp, lo, hi, seed=11),
        "bn": api.BentNormalsSolver(ctx, spp, lo, hi, tangent_space=True, seed=11),
        "thick": api.ThicknessSolver(ctx, spp, lo, hi, seed=11),
    }
    res = {}
    for k, s in solvers.items():
        s.init(tm, mm)
        s.set_work_per_step(500)
        while not s.run_step():
            pass
        assert s.progress() == 1.0
        r = s.get_results()
        assert len(r) == (n + 63) // 64 * 64
        res[k] = r[:n]
    cc, ct = coords[:n], tidx[:n]
    assert same_bits(res["height"][hit], oracle.gather(0, c.pos4, c.nrm4, cc, ct)[hit])
    assert same_bits(res["position"][hit], oracle.gather(1, c.pos4, c.nrm4, cc, ct)[hit])
    nrm = oracle.tangent_transform(ref["normals"], ref["tangents"], ref["bitangents"],
                                   oracle.gather(2, c.pos4, c.nrm4, cc, ct))
    assert same_bits(res["normals"][hit], nrm[hit])
    # sampling solvers use AUTO traversal (ordered, with the default tuning):
    # compare with the skip-exact oracle at the ordered traversal's bar
    for k, kind in (("ao", 0), ("bn", 1), ("thick", 2)):
        exp, ehits = oracle.hemisphere(kind, c.nodes, c.pos4, c.nrm4, cc, ct, samples, spp, lo, hi)
        if kind == 1:
            exp = oracle.tangent_transform(ref["normals"], ref["tangents"], ref["bitangents"], exp)
            ok = np.all(bits(res[k][hit]) == bits(exp[hit]), axis=1)
        else:
            ok = bits(res[k][hit]) == bits(exp[hit])
        hits = solvers[k].hits()[:n]
        record("solver_auto:%s" % k, texels=hit.sum(), hit_diff=(hits[hit] != ehits[hit]).mean(),
               out_diff=(~ok).mean())
        assert np.abs(hits[hit].astype(np.int64) - ehits[hit]).max() <= 1, k
        assert (hits[hit] != ehits[hit]).mean() <= 1e-4, k  # at most 0.01 % of texels
        assert (~ok).mean() <= 1e-4, k


def test_errors_are_reported_not_fatal(ctx):
    c = case("sphere")
    tm = api.TexelMap.from_meshes(ctx, c.lm, c.dm, 32, 32)
    mm = api.MeshMapping(ctx)
    with pytest.raises(api.FornosError):
        mm.run_step()  # before init
    mm.init(tm, c.hm, c.bvh, True)
    small = ctx.buffer(16)
    with pytest.raises(api.FornosError):
        api.meshmap(ctx, mm.scene, tm, True, small, small)
    s = api.AmbientOcclusionSolver(ctx, 8, 0.0, 1.0)
    s.init(tm, mm)
    with pytest.raises(api.FornosError):
        s.run_step()  # mapping not run yet
    mm.run()
    s.run()
    assert np.isfinite(s.get_results()[: tm.count]).all()


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kind", [api.AO, api.BN, api.THICK, api.AO_BN])
@pytest.mark.parametrize("trav", [api.TRAVERSE_ORDERED, api.TRAVERSE_ORDERED4, api.TRAVERSE_SKIP])
def test_filtered_box_tests_equal_exact(ctx, oracle, name, kind, trav):
    """The reciprocal-filtered box test must take every decision the divided
    one takes: outputs and counts are identical bit for bit."""
    c = case(name)
    _, _, mm = mapped(ctx, oracle, c)
    spp, lo, hi = 24, 0.001, 0.3
    _, a = run_hemi(ctx, mm, kind, spp, lo, hi, trav | api.SCHEDULE_DYNAMIC)
    _, b = run_hemi(ctx, mm, kind, spp, lo, hi, trav | api.SCHEDULE_DYNAMIC | api.EXACT_BOX_TESTS)
    for x, y in zip(a, b):
        assert same_bits(x, y) if x.dtype == np.float32 else np.array_equal(x, y)
