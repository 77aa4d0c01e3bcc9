"""fk_hemisphere_texels: a texel-list pass writes, at every listed texel, the
bits a whole-map fk_hemisphere pass writes there, and leaves other texels
alone.  Ids beyond texel_count are skipped and reported by fk_ctx_check."""
import numpy as np
import pytest

from fornos_b200 import api
from tests import cases
from tests.cases import same_bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mapped_sphere(ctx, oracle):
    c = cases.sphere()
    ref = oracle.raster(c.lo, 64, 64, 0, c.dirs)
    tm = api.TexelMap.from_host(ctx, 64, 64, cases.pix8(ref), cases.pixt12(ref), ref["indices"])
    mm = api.MeshMapping(ctx)
    mm.init(tm, c.hm, c.bvh, True)
    mm.run()
    try:
        ctx.check()  # start from clear flags whatever ran before on this context
    except api.FornosError:
        pass
    return mm


def outputs(ctx, n, fill):
    bufs = [ctx.buffer(12 * n), ctx.buffer(12 * n), ctx.buffer(4 * n), ctx.buffer(4 * n)]
    for b in bufs:
        b.upload(np.full(b.nbytes // 4, fill, np.uint32))
    return bufs


def read(bufs, n, kind):
    o0 = bufs[0].download(np.float32, (n, 3) if kind == api.BN else n)
    r = [o0, bufs[2].download(np.uint32, n)]
    if kind == api.AO_BN:
        r += [bufs[1].download(np.float32, (n, 3)), bufs[3].download(np.uint32, n)]
    return r


@pytest.mark.parametrize("kind", [api.AO, api.BN, api.THICK, api.AO_BN])
@pytest.mark.parametrize("trav", [api.TRAVERSE_ORDERED, api.TRAVERSE_ORDERED4, api.TRAVERSE_SKIP])
def test_texel_list_equals_whole_map(ctx, mapped_sphere, kind, trav):
    mm = mapped_sphere
    n = mm.tmap.count
    spp = 24
    samples = ctx.upload(api.samples_cosine(spp, api.PERMS, 5))
    whole = outputs(ctx, n, 0)
    api.hemisphere(ctx, mm.scene, mm.coords, mm.coords_tidx, kind, spp, 0.001, 0.4, samples, whole[0],
                   whole[1] if kind == api.AO_BN else None, whole[2], whole[3] if kind == api.AO_BN else None, 0, n,
                   traverse=trav)
    want = read(whole, n, kind)
    rng = np.random.default_rng(3)
    ids = np.sort(rng.choice(n, size=n // 3, replace=False)).astype(np.uint32)[::-1].copy()  # any order
    sentinel = 0x7FBADBAD
    part = outputs(ctx, n, sentinel)
    api.hemisphere_texels(ctx, mm.scene, mm.coords, mm.coords_tidx, n, kind, spp, 0.001, 0.4, samples,
                          ctx.upload(ids), part[0], part[1] if kind == api.AO_BN else None, part[2],
                          part[3] if kind == api.AO_BN else None, traverse=trav)
    ctx.check()
    got = read(part, n, kind)
    listed = np.zeros(n, bool)
    listed[ids] = True
    for g, w in zip(got, want):
        assert same_bits(g[listed], w[listed]) if g.dtype == np.float32 else np.array_equal(g[listed], w[listed])
        assert np.all(g[~listed].view(np.uint32) == sentinel)


def test_texel_list_offset_count_and_bad_ids(ctx, mapped_sphere):
    mm = mapped_sphere
    n = mm.tmap.count
    spp = 8
    samples = ctx.upload(api.samples_cosine(spp, api.PERMS, 9))
    whole = outputs(ctx, n, 0)
    api.hemisphere(ctx, mm.scene, mm.coords, mm.coords_tidx, api.AO, spp, 0.0, 0.5, samples, whole[0], None,
                   whole[2], None, 0, n)
    want = read(whole, n, api.AO)
    # a window of the list, with ids beyond texel_count inside it
    ids = np.array([5, n + 7, 11, 0xFFFFFFFF, 2, 40, n], np.uint32)
    part = outputs(ctx, n, 0x7FBADBAD)
    api.hemisphere_texels(ctx, mm.scene, mm.coords, mm.coords_tidx, n, api.AO, spp, 0.0, 0.5, samples,
                          ctx.upload(ids), part[0], None, part[2], None, offset=1, count=5)
    with pytest.raises(api.FornosError, match="texel list"):
        ctx.check()
    ctx.check()  # flags were cleared
    got = read(part, n, api.AO)
    for t in (11, 2, 40):
        assert got[0][t].view(np.uint32) == want[0][t].view(np.uint32) and got[1][t] == want[1][t]
    assert got[0][5].view(np.uint32) == 0x7FBADBAD  # before the window
    # host-side validation
    with pytest.raises(api.FornosError):
        api.hemisphere_texels(ctx, mm.scene, mm.coords, mm.coords_tidx, 1 << 30, api.AO, spp, 0.0, 0.5, samples,
                              ctx.upload(ids), part[0], None, part[2], None)
    with pytest.raises(api.FornosError):
        api.hemisphere_texels(ctx, mm.scene, mm.coords, mm.coords_tidx, n, api.AO, spp, 0.0, 0.5, samples,
                              ctx.upload(ids), part[0], None, part[2], None, traverse=api.SCHEDULE_STATIC)
