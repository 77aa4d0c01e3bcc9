"""fk_hemisphere_noalloc, the entry point for callers that must not allocate
device memory during a bake (a host running one bake chunk per interactive
frame, or one that budgets GPU memory through its own allocator).  Through
the C ABI, two calls in a row must reproduce fk_hemisphere's outputs bit for
bit (the tolerance these tests use for hemisphere outputs), although the
second call starts from the first call's leftovers in the shared fixed
scratch array, also over a sub-range of the texels.  A warmed-up call leaves
the device's free memory unchanged, device errors reach fk_ctx_check, and
oversized requests are refused.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

from fornos_b200 import _lib as L
from fornos_b200 import api
from tests import cases
from tests.cases import same_bits

pytestmark = pytest.mark.gpu


def _setup(ctx, oracle):
    c = cases.plane()
    ref = oracle.raster(c.lo, 64, 64, 0, c.dirs)
    tm = api.TexelMap.from_host(ctx, 64, 64, cases.pix8(ref), cases.pixt12(ref), ref["indices"])
    mm = api.MeshMapping(ctx)
    mm.init(tm, c.hm, c.bvh, True)
    mm.run()
    return tm, mm


def _noalloc(ctx, mm, kind, spp, lo, hi, sbuf, out0, out1, h0, h1, n, trav, offset=0, tidx=None):
    p = L.SampleParams(spp, api.PERMS, lo, hi)
    dp = lambda b: b.device_ptr if b is not None else None
    tidx = mm.coords_tidx if tidx is None else tidx
    ctx.sync()
    rc = ctx.lib.fk_hemisphere_noalloc(mm.scene.handle, mm.coords.device_ptr, tidx.device_ptr, kind,
                                       ctypes.byref(p), sbuf.device_ptr, offset, n, trav, dp(out0), dp(out1), dp(h0),
                                       dp(h1), ctx.lib.fk_ctx_stream(ctx.handle))
    ctx.sync()
    return rc


@pytest.mark.parametrize("kind", [api.AO_BN, api.THICK])
@pytest.mark.parametrize("trav", [api.TRAVERSE_ORDERED, api.TRAVERSE_SKIP])
def test_noalloc_matches_fk_hemisphere_twice(ctx, oracle, kind, trav):
    tm, mm = _setup(ctx, oracle)
    n, spp, lo, hi = tm.count, 40, 0.001, 0.3
    sbuf = ctx.upload(api.samples_cosine(spp, api.PERMS, 3))
    want = [ctx.buffer(12 * n), ctx.buffer(12 * n), ctx.buffer(4 * n), ctx.buffer(4 * n)]
    api.hemisphere(ctx, mm.scene, mm.coords, mm.coords_tidx, kind, spp, lo, hi, sbuf, want[0],
                   want[1] if kind == api.AO_BN else None, want[2], want[3] if kind == api.AO_BN else None, 0, n,
                   traverse=trav | api.SCHEDULE_DYNAMIC)
    w0 = 1
    exp = [want[0].download(np.float32, n * w0), want[2].download(np.uint32, n)]
    if kind == api.AO_BN:
        exp += [want[1].download(np.float32, (n, 3)), want[3].download(np.uint32, n)]
    for call in range(2):
        got = [ctx.buffer(12 * n), ctx.buffer(12 * n), ctx.buffer(4 * n), ctx.buffer(4 * n)]
        rc = _noalloc(ctx, mm, kind, spp, lo, hi, sbuf, got[0], got[1] if kind == api.AO_BN else None, got[2],
                      got[3] if kind == api.AO_BN else None, n, trav)
        assert rc == 0, ctx.lib.fk_last_error(ctx.handle)
        res = [got[0].download(np.float32, n * w0), got[2].download(np.uint32, n)]
        if kind == api.AO_BN:
            res += [got[1].download(np.float32, (n, 3)), got[3].download(np.uint32, n)]
        for a, b in zip(res, exp):
            assert (same_bits(a, b) if a.dtype == np.float32 else np.array_equal(a, b)), call


def test_noalloc_refuses_oversized_requests(ctx, oracle):
    tm, mm = _setup(ctx, oracle)
    spp = 1024
    n = (1 << 22) // spp + 1  # one texel more than the fixed scratch holds
    sbuf = ctx.upload(api.samples_cosine(spp, api.PERMS, 3))
    out = ctx.buffer(12 * n)
    rc = _noalloc(ctx, mm, api.AO, spp, 0.001, 0.3, sbuf, out, None, None, None, n, 0)
    assert rc == -1
    assert b"exceeds the fixed scratch" in ctx.lib.fk_last_error(ctx.handle)


def test_noalloc_sub_range_and_no_device_allocation(ctx, oracle):
    """A texel range that starts past 0 and stops before the end, against
    fk_hemisphere over the same range; a warmed-up call changes neither the
    device's free memory nor the context's pool."""
    import torch
    tm, mm = _setup(ctx, oracle)
    n, spp, lo, hi = tm.count, 64, 0.001, 0.3
    off, cnt = n // 3, n // 2
    sbuf = ctx.upload(api.samples_cosine(spp, api.PERMS, 9))
    want_ao, want_bn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    api.hemisphere(ctx, mm.scene, mm.coords, mm.coords_tidx, api.AO_BN, spp, lo, hi, sbuf, want_ao, want_bn, None,
                   None, off, cnt)
    got_ao, got_bn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    assert _noalloc(ctx, mm, api.AO_BN, spp, lo, hi, sbuf, got_ao, got_bn, None, None, cnt, 0, off) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert _noalloc(ctx, mm, api.AO_BN, spp, lo, hi, sbuf, got_ao, got_bn, None, None, cnt, 0, off) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    ctx.check()
    sl = slice(off, off + cnt)
    assert same_bits(got_ao.download(np.float32, n)[sl], want_ao.download(np.float32, n)[sl])
    assert same_bits(got_bn.download(np.float32, (n, 3))[sl], want_bn.download(np.float32, (n, 3))[sl])


def test_noalloc_reports_device_errors(ctx, oracle):
    """A texel whose hit index names a triangle past the end of the scene is
    skipped by the kernels (no access is made for it) and flagged; the flag
    reaches fk_ctx_check as FK_ERR_DEVICE, as it does for fk_hemisphere."""
    tm, mm = _setup(ctx, oracle)
    n, spp = tm.count, 32
    sbuf = ctx.upload(api.samples_cosine(spp, api.PERMS, 4))
    ids = mm.coords_tidx.download(np.uint32, n).copy()
    hit = np.nonzero(ids != api.MISS)[0]
    ids[hit[len(hit) // 2]] = mm.scene.info()["corner_count"]  # first corner of a triangle past the last one
    bad = ctx.upload(ids)
    ctx.check()  # nothing pending before the call
    out = ctx.buffer(4 * n)
    assert _noalloc(ctx, mm, api.AO, spp, 0.001, 0.3, sbuf, out, None, None, None, n, 0, tidx=bad) == 0
    with pytest.raises(api.FornosError) as e:
        ctx.check()
    assert e.value.code == -5 and "outside the scene" in str(e.value)
    ctx.check()  # the flag is cleared once reported
