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
