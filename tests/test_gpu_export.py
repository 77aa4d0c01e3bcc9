"""Image export on the device (fk_export_image) against the oracle
restatement of Src/image.cpp:22-405 (itself pinned to the reference's export
functions, tests/test_export_oracle.py): every mode, filter / normalisation
settings and dilation depths, bit for bit, on chart-shaped texel maps with
isolated holes (dilation sources that are themselves uncovered, which the
row-order scan fills first)."""
import numpy as np
import pytest

from fornos_b200 import api
from tests.cases import same_bits
from tests.test_export_oracle import chart_map, unit_vectors, values

pytestmark = pytest.mark.gpu


def tmap_of(ctx, w, h, idx):
    n = len(idx)
    return api.TexelMap.from_host(ctx, w, h, np.zeros((n, 8), np.float32), np.zeros((n, 12), np.float32),
                                  np.asarray(idx, np.uint32))


@pytest.mark.parametrize("w,h", [(64, 64), (80, 48), (257, 129)])
@pytest.mark.parametrize("normalize,flo,fhi", [(True, 0.0, 0.0), (False, 0.0, 0.0), (True, 0.2, 0.7), (False, 0.1, 0.9)])
@pytest.mark.parametrize("dilate", [0, 3, 16])
def test_float_rgb8(ctx, oracle, w, h, normalize, flo, fhi, dilate):
    idx = chart_map(w, h, 11 + w)
    data = values(len(idx), 12)
    img, mm = api.export_image(ctx, tmap_of(ctx, w, h, idx), ctx.upload(data), api.EXPORT_FLOAT_RGB8, (flo, fhi),
                               normalize, dilate)
    want, wmm = oracle.export_float(w, h, idx, data, flo, fhi, normalize, dilate, rgb8=True)
    assert np.array_equal(img, want)
    assert np.array_equal(np.float32(mm), np.float32(wmm))


@pytest.mark.parametrize("normalize,flo,fhi", [(True, 0.0, 0.0), (False, 0.0, 0.0), (True, 0.2, 0.7)])
def test_float_f32(ctx, oracle, normalize, flo, fhi):
    w, h = 96, 72
    idx = chart_map(w, h, 31)
    data = values(len(idx), 32)
    img, mm = api.export_image(ctx, tmap_of(ctx, w, h, idx), ctx.upload(data), api.EXPORT_FLOAT_F32, (flo, fhi),
                               normalize)
    want, wmm = oracle.export_float(w, h, idx, data, flo, fhi, normalize, 0, rgb8=False)
    # bit for bit, NaN payloads aside (the NaN texel's arithmetic: x86 keeps the payload, CUDA does not)
    assert same_bits(img, want)
    assert np.array_equal(np.float32(mm), np.float32(wmm))


@pytest.mark.parametrize("w,h,dilate", [(64, 64, 0), (64, 64, 5), (48, 64, 4), (128, 128, 24)])
def test_normal_rgb8(ctx, oracle, w, h, dilate):
    idx = chart_map(w, h, 41 + w)
    data3 = unit_vectors(len(idx), 42)
    img, _ = api.export_image(ctx, tmap_of(ctx, w, h, idx), ctx.upload(data3), api.EXPORT_NORMAL_RGB8,
                              dilate=dilate)
    assert np.array_equal(img, oracle.export_normal(w, h, idx, data3, dilate))


def test_vector_f32(ctx, oracle):
    w, h = 50, 70
    idx = chart_map(w, h, 51)
    data3 = unit_vectors(len(idx), 52) * np.float32(-2.5)
    img, _ = api.export_image(ctx, tmap_of(ctx, w, h, idx), ctx.upload(data3), api.EXPORT_VECTOR_F32)
    want = oracle.export_vector(w, h, idx, data3)
    assert same_bits(img, want)


def test_dilation_chains(ctx, oracle):
    # dense holes inside a chart: many uncovered pixels whose chosen source
    # centre is itself uncovered and earlier in the scan
    w = h = 96
    rng = np.random.default_rng(7)
    yy, xx = np.mgrid[0:h, 0:w]
    m = ((xx - 48) ** 2 + (yy - 48) ** 2 < 40 ** 2) & (rng.random((h, w)) > 0.12)
    idx = np.nonzero(m.ravel())[0].astype(np.uint32)
    data = rng.uniform(0, 1, len(idx)).astype(np.float32)
    img, _ = api.export_image(ctx, tmap_of(ctx, w, h, idx), ctx.upload(data), api.EXPORT_FLOAT_RGB8, dilate=30)
    want, _ = oracle.export_float(w, h, idx, data, 0.0, 0.0, True, 30, rgb8=True)
    assert np.array_equal(img, want)


def test_export_rejects_bad_arguments(ctx):
    idx = chart_map(32, 32, 1)
    tm = tmap_of(ctx, 32, 32, idx)
    with pytest.raises(api.FornosError):
        api.export_image(ctx, tm, ctx.upload(np.zeros(len(idx) // 2, np.float32)), api.EXPORT_FLOAT_RGB8)
    with pytest.raises(api.FornosError):
        api.export_image(ctx, tm, ctx.upload(np.zeros(len(idx), np.float32)), api.EXPORT_FLOAT_F32, dilate=3)
