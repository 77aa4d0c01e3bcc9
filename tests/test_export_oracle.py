"""The image export of Src/image.cpp:22-405 (scatter with flipped rows,
filtering and normalisation, 8-bit quantisation, dilation, EXR planes): the
oracle restatement against the reference's own functions compiled from
source (oracle/_ref), which write PNG / TGA / EXR files that these tests
decode.  The reference's dilation runs on one thread here (row order), the
order the restatement follows.
"""
import os
import shutil

import numpy as np
import pytest

from tests.imagefiles import half_bits, read_exr, read_png, read_tga

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture
def outdir(request):
    d = os.path.join(ROOT, "tests", ".out", request.node.name.replace("[", "_").replace("]", ""))
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(d)
    yield d
    shutil.rmtree(d, ignore_errors=True)


def chart_map(w, h, seed, blobs=12):
    """Covered texels: a union of disks (charts) with a few holes; ascending ids."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    m = np.zeros((h, w), bool)
    for _ in range(blobs):
        cx, cy, r = rng.uniform(0, w), rng.uniform(0, h), rng.uniform(3, max(4, min(w, h) / 4))
        m |= (xx - cx) ** 2 + (yy - cy) ** 2 < r * r
    hole = rng.random((h, w)) < 0.02
    m &= ~hole
    return np.nonzero(m.ravel())[0].astype(np.uint32)


def values(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(-0.3, 1.4, n).astype(np.float32)
    if n > 10:
        v[7] = np.nan
    return v


@pytest.mark.parametrize("fmt", ["png", "tga"])
@pytest.mark.parametrize("normalize,flo,fhi", [(True, 0.0, 0.0), (False, 0.0, 0.0), (True, 0.2, 0.7), (False, 0.1, 0.9)])
@pytest.mark.parametrize("dilate", [0, 3, 16])
def test_float_rgb8_matches_reference(oracle, reference, outdir, fmt, normalize, flo, fhi, dilate):
    w, h = 64, 64
    idx = chart_map(w, h, 11)
    data = values(len(idx), 12)
    path = os.path.join(outdir, "f." + fmt)
    mm_ref = reference.export_float(path, w, h, idx, data, flo, fhi, normalize, dilate)
    img, mm = oracle.export_float(w, h, idx, data, flo, fhi, normalize, dilate, rgb8=True)
    got = read_png(path) if fmt == "png" else read_tga(path)
    assert np.array_equal(got, img)
    assert np.array_equal(np.float32(mm), np.float32(mm_ref))


def test_float_rgb8_non_square(oracle, reference, outdir):
    w, h = 80, 48
    idx = chart_map(w, h, 21)
    data = values(len(idx), 22)
    path = os.path.join(outdir, "f.png")
    reference.export_float(path, w, h, idx, data, 0.0, 0.0, True, 8)
    img, _ = oracle.export_float(w, h, idx, data, 0.0, 0.0, True, 8, rgb8=True)
    assert np.array_equal(read_png(path), img)


@pytest.mark.parametrize("normalize,flo,fhi", [(True, 0.0, 0.0), (False, 0.0, 0.0), (True, 0.2, 0.7)])
def test_float_exr_matches_reference(oracle, reference, outdir, normalize, flo, fhi):
    w, h = 48, 40
    idx = chart_map(w, h, 31)
    data = values(len(idx), 32)
    path = os.path.join(outdir, "f.exr")
    reference.export_float(path, w, h, idx, data, flo, fhi, normalize, 0)
    img, _ = oracle.export_float(w, h, idx, data, flo, fhi, normalize, 0, rgb8=False)
    names, planes = read_exr(path)
    assert names == ["B"]
    # the file holds HALF values (tinyexr converts on write, rounding ties up)
    assert np.array_equal(planes[0].astype(np.float16).view(np.uint16), half_bits(img))


def unit_vectors(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v = v.astype(np.float32)
    v[::17] = -1.0  # all three bytes 0: counts as uncovered for the normal map's dilation
    return v


@pytest.mark.parametrize("fmt", ["png", "tga"])
@pytest.mark.parametrize("w,h,dilate", [(64, 64, 0), (64, 64, 5), (48, 64, 4)])
def test_normal_rgb8_matches_reference(oracle, reference, outdir, fmt, w, h, dilate):
    idx = chart_map(w, h, 41)
    data3 = unit_vectors(len(idx), 42)
    path = os.path.join(outdir, "n." + fmt)
    reference.export_normal(path, w, h, idx, data3, dilate)
    img = oracle.export_normal(w, h, idx, data3, dilate)
    got = read_png(path) if fmt == "png" else read_tga(path)
    assert np.array_equal(got, img)


def test_vector_exr_matches_reference(oracle, reference, outdir):
    w, h = 40, 40
    idx = chart_map(w, h, 51)
    data3 = unit_vectors(len(idx), 52) * np.float32(3.5)
    path = os.path.join(outdir, "v.exr")
    reference.export_vector(path, w, h, idx, data3)
    planes = oracle.export_vector(w, h, idx, data3)
    names, got = read_exr(path)
    assert names == ["B", "G", "R"]
    for k in range(3):
        assert np.array_equal(got[k].astype(np.float16).view(np.uint16), half_bits(planes[k]))
