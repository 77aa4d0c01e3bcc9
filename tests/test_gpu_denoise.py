"""Learned denoiser kernels against the CPU oracle (oracle/denoise.py).

Bars: the feature image and the input rows are bit-exact; the forward pass
and the gradient agree to float32 accumulation-order rounding (the oracle
rounds to bf16 at the same points as the kernels); one Adam step from the
kernels' own gradient is bit-exact.  The verified bake equals the plain
full-sample bake exactly where it falls back, and equals features + network
where it does not."""
import numpy as np
import pytest

from fornos_b200 import api
from oracle import denoise as D
from tests import cases
from tests.cases import same_bits

pytestmark = pytest.mark.gpu

LO, HI = 0.001, 0.3


@pytest.fixture(scope="module")
def baked(ctx, oracle):
    """The plane case at 96 x 80 texels: mapping, AO + BN at 16 spp, gathers."""
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
    api.hemisphere(ctx, mm.scene, mm.coords, mm.coords_tidx, api.AO_BN, 16, LO, HI, samples, ao, bn, None, None, 0, n)
    pos, nrm = ctx.buffer(12 * n), ctx.buffer(12 * n)
    api.gather(ctx, mm.scene, api.GATHER_POSITION, mm.coords, mm.coords_tidx, pos, 0, n)
    api.gather(ctx, mm.scene, api.GATHER_NORMAL, mm.coords, mm.coords_tidx, nrm, 0, n)
    coords, tidx = mm.results()
    host = dict(indices=np.asarray(ref["indices"], np.uint32), tidx=tidx[:n], coords=coords[:n],
                ao=ao.download(np.float32, n), bn=bn.download(np.float32, (n, 3)),
                pos=pos.download(np.float32, (n, 3)), nrm=nrm.download(np.float32, (n, 3)))
    image = api.denoise_features(ctx, tm, mm.coords, mm.coords_tidx, ao, bn, pos, nrm, HI)
    return dict(c=c, tm=tm, mm=mm, w=w, h=h, n=n, ao=ao, bn=bn, image=image, host=host, samples=samples)


def close(got, want):
    """Float32 accumulation order aside, the kernels and the oracle round the
    same values to bf16; a value that lands within an ulp of a bf16 rounding
    boundary can round the other way and move an output by up to ~1e-3.  So:
    almost every output agrees to 1e-5, and none by more than 2e-3."""
    d = np.abs(np.asarray(got, np.float64) - np.asarray(want, np.float64))
    assert np.quantile(d, 0.99) < 1e-5 and d.max() < 2e-3, (np.quantile(d, 0.99), d.max())


def random_params(seed):
    rng = np.random.default_rng(seed)
    p = D.init_params(seed)
    q = D.unpack(p)
    q["b1"][:] = rng.normal(0, 0.2, 64)
    q["b2"][:] = rng.normal(0, 0.2, 64)
    q["b3"][:] = rng.normal(0, 0.05, 4)
    q["w3"][:] *= 5
    return p


def test_features_and_rows_bit_exact(ctx, baked):
    b, hs = baked, baked["host"]
    want = D.features(b["w"], b["h"], hs["indices"], hs["tidx"], hs["coords"], hs["ao"], hs["bn"], hs["pos"],
                      hs["nrm"], HI)
    got = b["image"].download(np.float32, (3, b["w"] * b["h"], 4))
    assert same_bits(got, want)
    assert (want[0, :, 3] == 1).sum() > 0.5 * b["n"]
    pixels = np.concatenate([hs["indices"], np.array([0xFFFFFFFF, b["w"] * b["h"]], np.uint32)])
    rows = api.denoise_rows(ctx, b["image"], b["w"], b["h"], ctx.upload(pixels), len(pixels))
    got_rows = rows.download(np.uint16, (len(pixels), 256))
    want_rows = (D.rows(want, b["w"], b["h"], pixels).view(np.uint32) >> 16).astype(np.uint16)
    assert np.array_equal(got_rows, want_rows)
    assert np.all(got_rows[-2:] == 0)


def rows_and_targets(ctx, baked, m, seed):
    b, hs = baked, baked["host"]
    rng = np.random.default_rng(seed)
    hit = np.nonzero(hs["tidx"] != api.MISS)[0]
    pick = rng.choice(hit, m, replace=len(hit) < m)
    pixels = hs["indices"][pick].astype(np.uint32)
    f = D.features(b["w"], b["h"], hs["indices"], hs["tidx"], hs["coords"], hs["ao"], hs["bn"], hs["pos"], hs["nrm"],
                   HI)
    x = D.rows(f, b["w"], b["h"], pixels)
    t = rng.normal(0, 0.2, (m, 4)).astype(np.float32)
    rows = api.denoise_rows(ctx, b["image"], b["w"], b["h"], ctx.upload(pixels), m)
    return x, t, rows, ctx.upload(t)


def test_forward_matches_oracle(ctx, baked):
    x, _, rows, _ = rows_and_targets(ctx, baked, 300, 1)
    p = random_params(3)
    dn = api.Denoiser(ctx, p)
    y = dn.forward(rows, 300).download(np.float32, (300, 4))
    want, _ = D.forward(p, x)
    assert np.abs(want).max() > 0.1
    close(y, want)


@pytest.mark.parametrize("with_ids", [False, True])
def test_gradient_matches_oracle(ctx, baked, with_ids):
    m = 384
    x, t, rows, tbuf = rows_and_targets(ctx, baked, m, 2)
    p = random_params(4)
    dn = api.Denoiser(ctx, p)
    ids = None
    if with_ids:
        perm = np.random.default_rng(5).permutation(m).astype(np.uint32)
        ids = ctx.upload(perm)
        x, t = x[perm], t[perm]
    g, loss = dn.gradient(rows, tbuf, m, m, row_ids=ids)
    want, wloss = D.backward(p, x, t)
    assert abs(loss - wloss) <= 1e-4 * wloss
    for name, (off, shape) in D.LAYOUT.items():
        sl = slice(off, off + int(np.prod(shape)))
        a, b = g[sl], want[sl]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 3e-3, (name, rel)
    assert np.all(g[:16384].reshape(64, 256)[:, 250:] == 0)


def test_adam_steps_bit_exact(ctx, baked):
    m = 256
    x, t, rows, tbuf = rows_and_targets(ctx, baked, m, 6)
    p = random_params(7)
    dn = api.Denoiser(ctx, p)
    mo, vo = np.zeros_like(p), np.zeros_like(p)
    for step in (1, 2, 3):
        g, _ = dn.gradient(rows, tbuf, m, m)
        dn.train_step(rows, tbuf, m, m, lr=1e-3)
        p, mo, vo = D.adam(p, mo, vo, g, step, 1e-3)
        got = dn.get_params()
        assert np.array_equal(got.view(np.uint32), p.view(np.uint32)), step


def test_training_reduces_loss(ctx, baked):
    m = 2048
    x, t, rows, _ = rows_and_targets(ctx, baked, m, 8)
    # a learnable target: a fixed smooth function of the inputs
    t = np.tanh(x[:, :250] @ np.random.default_rng(9).normal(0, 0.05, (250, 4))).astype(np.float32)
    tbuf = ctx.upload(t)
    dn = api.Denoiser(ctx, D.init_params(10))
    dn.train_step(rows, tbuf, m, m, lr=0.0)
    first = dn.last_loss()
    for _ in range(300):
        dn.train_step(rows, tbuf, m, 1024, offset=0, lr=3e-3)
        dn.train_step(rows, tbuf, m, 1024, offset=1024, lr=3e-3)
    dn.train_step(rows, tbuf, m, m, lr=0.0)
    assert dn.last_loss() < 0.1 * first


def test_apply_matches_oracle(ctx, baked):
    b, hs = baked, baked["host"]
    p = random_params(11)
    dn = api.Denoiser(ctx, p)
    n = b["n"]
    ao, bn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    dn.apply(b["tm"], b["image"], b["mm"].coords_tidx, b["ao"], b["bn"], ao, bn)
    f = b["image"].download(np.float32, (3, b["w"] * b["h"], 4))
    wao, wbn = D.apply(p, f, b["w"], b["h"], hs["indices"], hs["tidx"], hs["ao"], hs["bn"])
    gao, gbn = ao.download(np.float32, n), bn.download(np.float32, (n, 3))
    close(gao, wao)
    close(gbn, wbn)
    miss = hs["tidx"] == api.MISS
    assert np.all(gao[miss] == 1) and np.all(gbn[miss] == 0)
    # in place over the inputs gives the same values
    ao2 = ctx.upload(hs["ao"])
    bn2 = ctx.upload(hs["bn"])
    dn.apply(b["tm"], b["image"], b["mm"].coords_tidx, ao2, bn2, ao2, bn2)
    assert same_bits(ao2.download(np.float32, n), gao) and same_bits(bn2.download(np.float32, (n, 3)), gbn)


def test_bake_falls_back_to_the_plain_bake(ctx, baked):
    b = baked
    n, mm = b["n"], b["mm"]
    full = ctx.upload(api.samples_cosine(64, api.PERMS, 22))
    plain_ao, plain_bn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    api.hemisphere(ctx, mm.scene, mm.coords, mm.coords_tidx, api.AO_BN, 64, LO, HI, full, plain_ao, plain_bn, None,
                   None, 0, n)
    dn = api.Denoiser(ctx, random_params(12))
    ao, bn = ctx.buffer(4 * n), ctx.buffer(12 * n)
    # every tile fails: the result is the plain 64-sample bake, bit for bit
    st = dn.bake(mm.scene, b["tm"], mm.coords, mm.coords_tidx, b["samples"], full, ao, bn, low_samples=16,
                 full_samples=64, min_distance=LO, max_distance=HI, tile=32, verify_cells=4, max_tile_error=-1.0)
    ctx.check()
    hit = b["host"]["tidx"] != api.MISS
    assert st["tiles"] == st["tiles_failed"] > 0 and st["texels_rebaked"] == hit.sum()
    assert st["rays"] == n * 16 + (st["spot_checks"] + st["texels_rebaked"]) * 64
    assert same_bits(ao.download(np.float32, n)[hit], plain_ao.download(np.float32, n)[hit])
    assert same_bits(bn.download(np.float32, (n, 3))[hit], plain_bn.download(np.float32, (n, 3))[hit])
    # no tile fails: the result is features + network over the 16-sample bake
    st = dn.bake(mm.scene, b["tm"], mm.coords, mm.coords_tidx, b["samples"], full, ao, bn, low_samples=16,
                 full_samples=64, min_distance=LO, max_distance=HI, tile=32, verify_cells=4,
                 max_tile_error=float("inf"))
    assert st["tiles_failed"] == 0 and st["texels_rebaked"] == 0 and 0 < st["spot_checks"] <= 9 * 16
    ao2, bn2 = ctx.buffer(4 * n), ctx.buffer(12 * n)
    dn.apply(b["tm"], b["image"], mm.coords_tidx, b["ao"], b["bn"], ao2, bn2)
    assert same_bits(ao.download(np.float32, n), ao2.download(np.float32, n))
    assert same_bits(bn.download(np.float32, (n, 3)), bn2.download(np.float32, (n, 3)))
