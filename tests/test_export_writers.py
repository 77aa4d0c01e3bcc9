"""Host image writers (fk_image_write_rgb8 / fk_image_write_exr): PNG and TGA
decode to the RGB8 buffer written; EXR decodes to the HALF values tinyexr's
conversion gives (ties rounded up, float denormals to zero, NaN quiet,
overflow to infinity)."""
import os
import shutil

import numpy as np
import pytest

from fornos_b200 import api
from tests.imagefiles import half_bits, read_exr, read_png, read_tga

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture
def outdir(request):
    d = os.path.join(ROOT, "tests", ".out", request.node.name.replace("[", "_").replace("]", ""))
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(d)
    yield d
    shutil.rmtree(d, ignore_errors=True)


@pytest.mark.parametrize("w,h", [(1, 1), (37, 23), (300, 260)])
@pytest.mark.parametrize("fmt", ["png", "tga"])
def test_rgb8_round_trip(lib, outdir, w, h, fmt):
    img = np.random.default_rng(w * h).integers(0, 256, (h, w, 3), dtype=np.uint8)
    path = os.path.join(outdir, "i." + fmt)
    api.write_image(path, img)
    got = read_png(path) if fmt == "png" else read_tga(path)
    assert np.array_equal(got, img)


def test_exr_round_trip(lib, outdir):
    rng = np.random.default_rng(3)
    planes = rng.normal(scale=100.0, size=(3, 19, 29)).astype(np.float32)
    special = np.array([0.0, -0.0, 1e-40, -1e-42, 70000.0, -1e9, np.inf, -np.inf, np.nan, 6.0e-8, 3.0e-5,
                        0.00030481815, 1.0009766, 2049.0], np.float32)
    planes.reshape(-1)[:len(special)] = special
    for img, names in ((planes[0], ["B"]), (planes, ["B", "G", "R"])):
        path = os.path.join(outdir, "i.exr")
        api.write_image(path, img)
        got_names, got = read_exr(path)
        assert got_names == names
        want = img.reshape(-1, *img.shape[-2:])
        for k in range(len(names)):
            assert np.array_equal(got[k].astype(np.float16).view(np.uint16), half_bits(want[k]))


def test_writers_refuse_bad_arguments(lib, outdir):
    with pytest.raises(api.FornosError):
        api.write_image(os.path.join(outdir, "x.bmp"), np.zeros((2, 2, 3), np.uint8))
    with pytest.raises(api.FornosError):
        api.write_image(os.path.join(outdir, "x.exr"), np.zeros((2, 4, 4), np.float32))


def baked_like(h, w, seed):
    """An image with the structure of a baked map: flat regions, gradients,
    hard edges and some noise (rows compress very differently)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    img = np.stack([xx * 255 // max(w - 1, 1), yy * 255 // max(h - 1, 1), np.full_like(xx, 128)], -1)
    img[(xx // 7 + yy // 5) % 3 == 0] = (255, 255, 255)
    noisy = rng.random((h, w)) < 0.1
    img[noisy] = rng.integers(0, 256, (int(noisy.sum()), 3))
    return img.astype(np.uint8)


@pytest.mark.parametrize("level", [0, 1, 6, 9])
@pytest.mark.parametrize("w,h", [(1, 1), (5000, 1), (1, 3000), (301, 259), (1500, 1000)])
def test_png_levels_round_trip(lib, outdir, w, h, level):
    """fk_image_write_png at every kind of level: stored rows, or rows filtered
    as stb_image_write filters them and deflated (in bands on several threads
    from 4 MB of rows, as 1500 x 1000 has).  Decoded by Pillow where it is
    installed, and by the tests' own reader up to 100k pixels."""
    img = baked_like(h, w, w + h + level)
    path = os.path.join(outdir, "l.png")
    api.write_image(path, img, png_level=level)
    try:
        from PIL import Image
        with Image.open(path) as im:
            assert np.array_equal(np.asarray(im.convert("RGB")), img)
    except ImportError:
        pass
    if w * h <= 100_000:
        assert np.array_equal(read_png(path), img)
    if level and w * h > 1000:
        assert os.path.getsize(path) < 3 * w * h  # the filtered rows compressed
    with open(path, "rb") as fh:
        data = fh.read()
    assert data.count(b"IDAT") >= 1 and data.endswith(b"IEND\xaeB`\x82")


def test_png_level_out_of_range(lib, outdir):
    img = np.zeros((4, 4, 3), np.uint8)
    for level in (-1, 10):
        with pytest.raises(api.FornosError):
            api.write_image(os.path.join(outdir, "x.png"), img, png_level=level)


def test_tga_run_lengths(lib, outdir):
    """Run packets longer than 128 pixels, single pixels between runs,
    alternating pixels (raw packets), uniform rows, one-pixel rows."""
    w, h = 300, 6
    img = np.zeros((h, w, 3), np.uint8)
    img[0] = (10, 20, 30)                                   # one run of 300: 128 + 128 + 44
    img[1, ::2] = (1, 2, 3)                                 # alternating: raw packets
    img[2, :150] = (9, 9, 9); img[2, 150] = (1, 1, 1); img[2, 151:] = (9, 9, 9)
    img[3] = np.random.default_rng(1).integers(0, 256, (w, 3))
    img[4, 127:131] = (200, 100, 0)                         # runs around a packet boundary
    img[5, -2:] = (7, 7, 7)
    path = os.path.join(outdir, "r.tga")
    api.write_image(path, img)
    assert np.array_equal(read_tga(path), img)
    try:
        from PIL import Image
        with Image.open(path) as im:
            assert np.array_equal(np.asarray(im.convert("RGB")), img)
    except ImportError:
        pass
    with open(path, "rb") as fh:
        data = fh.read()
    assert data[2] == 10  # run-length-coded true colour
    for shape in ((1, 1), (1, 129), (129, 1)):
        one = np.random.default_rng(sum(shape)).integers(0, 3, (*shape, 3)).astype(np.uint8)
        api.write_image(path, one)
        assert np.array_equal(read_tga(path), one)
