"""Denoiser inference on tcgen05 (tensor memory accumulators) against the CPU
oracle and against the mma.sync kernel: the same BF16 network with FP32
accumulation, so outputs agree up to accumulation order (and the rare bf16
rounding flip of a hidden activation that order can cause)."""
import numpy as np
import pytest

from fornos_b200 import api
from oracle import denoise as D
from tests import cases

pytestmark = pytest.mark.gpu

HI = 0.3


def close(got, want):
    d = np.abs(np.asarray(got, np.float64) - np.asarray(want, np.float64))
    assert np.quantile(d, 0.99) < 1e-5 and d.max() < 2e-3, (np.quantile(d, 0.99), d.max())


def params(seed):
    rng = np.random.default_rng(seed)
    p = D.init_params(seed)
    q = D.unpack(p)
    q["b1"][:] = rng.normal(0, 0.2, 64)
    q["b2"][:] = rng.normal(0, 0.2, 64)
    q["b3"][:] = rng.normal(0, 0.05, 4)
    q["w3"][:] *= 5
    return p


def test_forward_rows_matches_oracle(ctx):
    rng = np.random.default_rng(0)
    m = 300  # two full 128-row tiles and a partial one
    x = np.zeros((m, 256), np.float32)
    x[:, :250] = rng.normal(0, 0.7, (m, 250))
    x = D.bf16(x)
    rows = ctx.upload((x.view(np.uint32) >> 16).astype(np.uint16))
    p = params(1)
    dn = api.Denoiser(ctx, p)
    dn.set_engine(api.DN_ENGINE_TCGEN05)
    y = dn.forward(rows, m).download(np.float32, (m, 4))
    ctx.check()
    want, _ = D.forward(p, x)
    assert np.abs(want).max() > 0.1
    close(y, want)
    dn.set_engine(api.DN_ENGINE_MMA_SYNC)
    close(dn.forward(rows, m).download(np.float32, (m, 4)), y)


def test_apply_matches_mma_sync(ctx, oracle):
    c = cases.plane()
    w, h = 96, 80
    ref = oracle.raster(c.lo, w, h, 0, c.dirs)
    tm = api.TexelMap.from_host(ctx, w, h, cases.pix8(ref), cases.pixt12(ref), ref["indices"])
    mm = api.MeshMapping(ctx)
    mm.init(tm, c.hm, c.bvh, True)
    mm.run()
    n = tm.count
    samples = ctx.upload(api.samples_cosine(16, api.PERMS, 21))
    ao, bn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    api.hemisphere(ctx, mm.scene, mm.coords, mm.coords_tidx, api.AO_BN, 16, 0.001, HI, samples, ao, bn, None, None,
                   0, n)
    pos, nrm = ctx.buffer(12 * n), ctx.buffer(12 * n)
    api.gather(ctx, mm.scene, api.GATHER_POSITION, mm.coords, mm.coords_tidx, pos, 0, n)
    api.gather(ctx, mm.scene, api.GATHER_NORMAL, mm.coords, mm.coords_tidx, nrm, 0, n)
    image = api.denoise_features(ctx, tm, mm.coords, mm.coords_tidx, ao, bn, pos, nrm, HI)
    dn = api.Denoiser(ctx, params(2))
    out = {}
    for eng in (api.DN_ENGINE_TCGEN05, api.DN_ENGINE_MMA_SYNC):
        dn.set_engine(eng)
        a2, b2 = ctx.buffer(4 * n), ctx.buffer(12 * n)
        dn.apply(tm, image, mm.coords_tidx, ao, bn, a2, b2)
        ctx.check()
        out[eng] = (a2.download(np.float32, n), b2.download(np.float32, (n, 3)))
    close(out[api.DN_ENGINE_TCGEN05][0], out[api.DN_ENGINE_MMA_SYNC][0])
    close(out[api.DN_ENGINE_TCGEN05][1], out[api.DN_ENGINE_MMA_SYNC][1])
    # a window of the texels (offset / count) gives the same values there
    dn.set_engine(api.DN_ENGINE_TCGEN05)
    a3, b3 = ctx.buffer(4 * n), ctx.buffer(12 * n)
    dn.apply(tm, image, mm.coords_tidx, ao, bn, a3, b3, offset=37, count=n - 100)
    got = a3.download(np.float32, n)
    close(got[37:n - 63], out[api.DN_ENGINE_TCGEN05][0][37:n - 63])
    assert np.all(got[:37] == 0) and np.all(got[n - 63:] == 0)


def test_engine_choice_is_validated(ctx):
    dn = api.Denoiser(ctx)
    with pytest.raises(api.FornosError):
        dn.set_engine(7)
