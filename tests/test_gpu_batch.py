"""Batched bakes (fk_batch_*) and the autotuner: several jobs with their own
scenes, texels, sample tables and parameters in one persistent launch must
give each job exactly what fk_hemisphere gives it alone, also when the run is
recorded into a CUDA graph and replayed."""
import numpy as np
import pytest

from fornos_b200 import api
from tests import cases
from tests.cases import same_bits

pytestmark = pytest.mark.gpu

JOBS = [("sphere", 48, 0.001, 0.5, 64), ("plane", 32, 0.001, 0.3, 48), ("icosphere", 16, 0.01, 0.8, 40),
        ("plane", 5, 0.0, 0.2, 32)]


@pytest.fixture(scope="module")
def setup(ctx, oracle):
    made = {"sphere": cases.sphere(), "plane": cases.plane(), "icosphere": cases.icosphere()}
    jobs = []
    for name, spp, lo, hi, tex in JOBS:
        c = made[name]
        ref = oracle.raster(c.lo, tex, tex, 0, c.dirs)
        tm = api.TexelMap.from_host(ctx, tex, tex, cases.pix8(ref), cases.pixt12(ref), ref["indices"])
        mm = api.MeshMapping(ctx)
        mm.init(tm, c.hm, c.bvh, True)
        mm.run()
        n = tm.count
        jobs.append(dict(tm=tm, mm=mm, scene=mm.scene, coords=mm.coords, tidx=mm.coords_tidx, texel_count=n,
                         spp=spp, min_distance=lo, max_distance=hi,
                         samples=ctx.upload(api.samples_cosine(spp, api.PERMS, 100 + spp))))
    return jobs


def alone(ctx, j, kind, trav):
    n = j["texel_count"]
    o0, o1, h0, h1 = ctx.buffer(12 * n), ctx.buffer(12 * n), ctx.buffer(4 * n), ctx.buffer(4 * n)
    api.hemisphere(ctx, j["scene"], j["coords"], j["tidx"], kind, j["spp"], j["min_distance"], j["max_distance"],
                   j["samples"], o0, o1 if kind == api.AO_BN else None, h0, h1 if kind == api.AO_BN else None, 0, n,
                   traverse=trav | api.SCHEDULE_DYNAMIC)
    return read(o0, o1, h0, h1, n, kind)


def read(o0, o1, h0, h1, n, kind):
    w = 3 if kind == api.BN else 1
    r = [o0.download(np.float32, (n, 3) if w == 3 else n), h0.download(np.uint32, n)]
    if kind == api.AO_BN:
        r += [o1.download(np.float32, (n, 3)), h1.download(np.uint32, n)]
    return r


def make_batch(ctx, jobs, kind):
    outs, specs = [], []
    for j in jobs:
        n = j["texel_count"]
        o = [ctx.buffer(12 * n), ctx.buffer(12 * n), ctx.buffer(4 * n), ctx.buffer(4 * n)]
        outs.append(o)
        specs.append(dict(j, out0=o[0], out1=o[1], hits0=o[2], hits1=o[3]))
    return api.Batch(ctx, specs, kind), outs


def check(jobs, outs, kind, want):
    for j, o, w in zip(jobs, outs, want):
        got = read(o[0], o[1], o[2], o[3], j["texel_count"], kind)
        for a, b in zip(got, w):
            assert same_bits(a, b) if a.dtype == np.float32 else np.array_equal(a, b)


@pytest.mark.parametrize("kind", [api.AO, api.BN, api.THICK, api.AO_BN])
@pytest.mark.parametrize("trav", [api.TRAVERSE_ORDERED, api.TRAVERSE_ORDERED4, api.TRAVERSE_SKIP])
def test_batch_equals_jobs_alone(ctx, setup, kind, trav):
    want = [alone(ctx, j, kind, trav) for j in setup]
    b, outs = make_batch(ctx, setup, kind)
    info = b.info()
    assert info["rays"] == sum(j["texel_count"] * j["spp"] for j in setup)
    b.run(trav)
    ctx.sync()
    check(setup, outs, kind, want)


def test_batch_graph_replay(ctx, setup):
    kind = api.AO_BN
    want = [alone(ctx, j, kind, api.TRAVERSE_ORDERED) for j in setup]
    b, outs = make_batch(ctx, setup, kind)
    b.capture(api.TRAVERSE_ORDERED)
    for _ in range(2):
        for o in outs:
            for buf in o:
                buf.upload(np.zeros(buf.nbytes, np.uint8))
        b.replay()
        ctx.sync()
        check(setup, outs, kind, want)


def test_autotuner_choice_gives_same_results(ctx, setup):
    kind = api.THICK
    b, outs = make_batch(ctx, setup, kind)
    best = b.tune(sample_rays=1 << 16)
    assert best["traverse"] & 0x0F in (api.TRAVERSE_ORDERED, api.TRAVERSE_ORDERED4, api.TRAVERSE_SKIP)
    assert 1 <= best["refill"] <= 32 and 1 <= best["leaf_batch"] <= 32
    want = [alone(ctx, j, kind, best["traverse"] & 0x0F) for j in setup]
    b.run()
    ctx.sync()
    check(setup, outs, kind, want)
    j = setup[1]
    tun, trav = api.tune_hemisphere(ctx, j["scene"], j["coords"], j["tidx"], api.AO, j["spp"], j["min_distance"],
                                    j["max_distance"], j["samples"], 0, j["texel_count"], sample_rays=1 << 15)
    ctx.set_tuning(**tun)
    assert trav & api.SCHEDULE_DYNAMIC
    ctx.set_tuning(refill=8, leaf_batch=8, speculate=0)


def test_batch_with_a_job_run_alone(ctx, setup):
    """A job of at least 2^21 rays runs alone through the single-job path in
    the batch's run (and in its graph), beside jobs that share launches; every
    job still gets what fk_hemisphere gives it alone."""
    big = dict(setup[0], spp=1 << 16, perms=8)
    big["samples"] = ctx.upload(api.samples_cosine(big["spp"], 8, 7))
    assert big["texel_count"] * big["spp"] >= 1 << 27  # more than one chunk of scratch too
    jobs = [setup[1], big, setup[3]]
    kind = api.AO_BN

    def alone_p(j):
        n = j["texel_count"]
        o0, o1, h0, h1 = ctx.buffer(12 * n), ctx.buffer(12 * n), ctx.buffer(4 * n), ctx.buffer(4 * n)
        api.hemisphere(ctx, j["scene"], j["coords"], j["tidx"], kind, j["spp"], j["min_distance"],
                       j["max_distance"], j["samples"], o0, o1, h0, h1, 0, n, perms=j.get("perms", api.PERMS),
                       traverse=api.TRAVERSE_ORDERED | api.SCHEDULE_DYNAMIC)
        return read(o0, o1, h0, h1, n, kind)

    want = [alone_p(j) for j in jobs]
    b, outs = make_batch(ctx, jobs, kind)
    launches = b.info()["launches_per_run"]
    before = ctx.launches
    b.run(api.TRAVERSE_ORDERED)
    ctx.sync()
    assert ctx.launches - before == launches
    check(jobs, outs, kind, want)
    b.capture(api.TRAVERSE_ORDERED)
    for o in outs:
        for buf in o:
            buf.upload(np.zeros(buf.nbytes, np.uint8))
    b.replay()
    ctx.sync()
    ctx.check()
    check(jobs, outs, kind, want)
