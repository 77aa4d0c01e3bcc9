"""fk_run (FornosRunner::start + run, Src/fornos.cpp:53-251): mesh files in,
image files out.  Each written image must equal, bit for bit, the image the
library's separately pinned steps give when composed by hand the way the
reference's runner composes them: Mesh::loadFile, normals per NormalImport,
tangent space, the welded direction copy, the texel map of the mapping
method, the BVH, mesh mapping, the solvers and each task's export
(Src/solver_*.cpp finish()).  Also: the runner's errors, and output paths the
reference writes nothing to."""
import os

import numpy as np
import pytest

from fornos_b200 import api
from fornos_b200 import workloads as W
from tests import imagefiles as IF
from tests import meshfiles as MF
from tests.cases import same_bits

pytestmark = pytest.mark.gpu

TEX, SPP, SEED = 96, 16, 7


def write_pair(tmp_path, seed=2):
    lo, hi = W.plane_pair(seed=seed, lo_quads=6, hi_quads=40, bumps=12)
    lp, hp = tmp_path / "lo.obj", tmp_path / "hi.obj"
    lp.write_text(MF.obj_of(lo))
    hp.write_text(MF.obj_of(hi))
    return str(lp), str(hp)


def composed(ctx, lo_path, hi_path, mapping, lo_normal, hi_normal, solvers, dilation, backfaces=True,
             traverse=api.TRAVERSE_AUTO):
    """The runner's images, step by step through the pinned entry points."""
    lo = api.Mesh.load(lo_path)
    hi = api.Mesh.load(hi_path) if hi_path else lo
    how = {api.NORMAL_COMPUTE_PER_FACE: "compute_face_normals", api.NORMAL_COMPUTE_PER_VERTEX: "compute_vertex_normals"}
    if lo_normal in how:
        getattr(lo, how[lo_normal])()
    if hi_path and hi_normal in how:
        getattr(hi, how[hi_normal])()
    if any(solvers.get(k, {}).get("tangent_space", True) for k in ("normals", "bent_normals") if k in solvers):
        lo.compute_tangent_space()
    dirs = None
    if mapping != api.MAP_LOWPOLY_NORMALS:
        if lo_normal != api.NORMAL_COMPUTE_PER_VERTEX:
            dirs = lo.copy()
            dirs.compute_vertex_normals_aggressive()
        else:
            dirs = lo
    tmap = api.TexelMap.rasterize(ctx, lo, TEX, TEX, mapping, dirs, 0.05)
    scene = api.Scene.build(ctx, hi, 8, 8192)
    n = tmap.count
    coords, tidx = ctx.buffer(16 * n), ctx.buffer(4 * n)
    api.meshmap(ctx, scene, tmap, backfaces, coords, tidx)
    samples = ctx.upload(api.samples_cosine(SPP, api.PERMS, SEED))
    out = {}

    def fmt(path):
        return "rgb8" if path.endswith((".png", ".tga")) else "exr"

    def float_img(buf, path, lo_f, hi_f, normalize):
        rgb = fmt(path) == "rgb8"
        img, _ = api.export_image(ctx, tmap, buf, api.EXPORT_FLOAT_RGB8 if rgb else api.EXPORT_FLOAT_F32,
                                  (lo_f, hi_f), normalize, dilation if rgb else 0)
        return img

    def normal_img(buf, path):
        rgb = fmt(path) == "rgb8"
        img, _ = api.export_image(ctx, tmap, buf, api.EXPORT_NORMAL_RGB8 if rgb else api.EXPORT_VECTOR_F32,
                                  (0.0, 0.0), False, dilation if rgb else 0)
        return img

    if "height" in solvers:
        b = ctx.buffer(4 * n)
        api.gather(ctx, scene, api.GATHER_HEIGHT, coords, tidx, b, 0, n)
        s = solvers["height"]
        out["height"] = float_img(b, s["output_path"], 0.0, s.get("max_distance", 0.0), s.get("normalize_output", 1))
    if "positions" in solvers:
        b = ctx.buffer(12 * n)
        api.gather(ctx, scene, api.GATHER_POSITION, coords, tidx, b, 0, n)
        out["positions"] = api.export_image(ctx, tmap, b, api.EXPORT_VECTOR_F32, (0.0, 0.0), False, 0)[0]
    if "normals" in solvers:
        b = ctx.buffer(12 * n)
        api.gather(ctx, scene, api.GATHER_NORMAL, coords, tidx, b, 0, n)
        if solvers["normals"].get("tangent_space", 1):
            api.tangent_space(ctx, tmap, b)
        out["normals"] = normal_img(b, solvers["normals"]["output_path"])
    for kind, key in ((api.AO, "ao"), (api.BN, "bent_normals"), (api.THICK, "thickness")):
        if key not in solvers:
            continue
        s = solvers[key]
        b = ctx.buffer((12 if kind == api.BN else 4) * n)
        api.hemisphere(ctx, scene, coords, tidx, kind, SPP, s["min_distance"], s["max_distance"], samples, b,
                       count=n, traverse=traverse)
        if kind == api.BN:
            if s.get("tangent_space", 1):
                api.tangent_space(ctx, tmap, b)
            out[key] = normal_img(b, s["output_path"])
        else:
            out[key] = float_img(b, s["output_path"], 0.0, 0.0, True)
    return out


def read(path):
    if path.endswith(".png"):
        return IF.read_png(path)
    if path.endswith(".tga"):
        return IF.read_tga(path)
    names, planes = IF.read_exr(path)
    return names, planes


def same_file(path, img):
    got = read(path)
    if isinstance(got, np.ndarray):
        return np.array_equal(got, img)
    names, planes = got
    want = img.reshape(-1, *img.shape[-2:])
    return len(planes) == len(want) and all(
        np.array_equal(IF.half_bits(p), IF.half_bits(q)) for p, q in zip(planes, want))


def solver_set(tmp_path, exts):
    d = str(tmp_path)
    return {
        "height": dict(enabled=1, output_path=os.path.join(d, "height" + exts[0]), max_distance=0.3,
                       normalize_output=1),
        "positions": dict(enabled=1, output_path=os.path.join(d, "positions.exr")),
        "normals": dict(enabled=1, output_path=os.path.join(d, "normals" + exts[1]), tangent_space=1),
        "ao": dict(enabled=1, output_path=os.path.join(d, "ao" + exts[2]), sample_count=SPP, min_distance=0.001,
                   max_distance=0.3),
        "bent_normals": dict(enabled=1, output_path=os.path.join(d, "bn" + exts[3]), sample_count=SPP,
                             min_distance=0.001, max_distance=0.3, tangent_space=1),
        "thickness": dict(enabled=1, output_path=os.path.join(d, "thick" + exts[4]), sample_count=SPP,
                          min_distance=0.001, max_distance=0.3),
    }


@pytest.mark.parametrize("mapping,lo_normal,exts", [
    (api.MAP_SMOOTH, api.NORMAL_IMPORT, (".png", ".png", ".png", ".png", ".tga")),
    (api.MAP_HYBRID, api.NORMAL_COMPUTE_PER_VERTEX, (".exr", ".exr", ".tga", ".exr", ".exr")),
    (api.MAP_LOWPOLY_NORMALS, api.NORMAL_COMPUTE_PER_FACE, (".tga", ".png", ".exr", ".png", ".png")),
])
def test_runner_images(ctx, tmp_path, mapping, lo_normal, exts):
    lo_path, hi_path = write_pair(tmp_path)
    solvers = solver_set(tmp_path, exts)
    api.run(ctx, lo_poly_mesh_path=lo_path, hi_poly_mesh_path=hi_path, lo_poly_mesh_normal=lo_normal,
            hi_poly_mesh_normal=api.NORMAL_COMPUTE_PER_VERTEX, tex_width=TEX, tex_height=TEX, tex_dilation=4,
            mapping=mapping, seed=SEED, traverse=api.TRAVERSE_SKIP, **solvers)
    # the runner traces AO and bent normals in one fused pass, the composition in two: compared on the
    # bit-exact skip walk, where the fused pass is known to equal the separate ones
    want = composed(ctx, lo_path, hi_path, mapping, lo_normal, api.NORMAL_COMPUTE_PER_VERTEX, solvers, 4,
                    traverse=api.TRAVERSE_SKIP)
    for key, img in want.items():
        path = solvers[key]["output_path"]
        assert os.path.exists(path), key
        if key in ("height", "positions", "normals"):  # maps with content on any covered texel
            assert np.count_nonzero(img) > img.size // 4, key
        assert same_file(path, img), key


def test_runner_single_mesh_and_skipped_outputs(ctx, tmp_path):
    lo_path, _ = write_pair(tmp_path, seed=3)
    d = str(tmp_path)
    solvers = {"positions": dict(enabled=1, output_path=os.path.join(d, "pos.png")),   # EXR only: nothing
               "height": dict(enabled=1, output_path=os.path.join(d, "height.bmp")),  # unknown: nothing
               "ao": dict(enabled=1, output_path=os.path.join(d, "ao.png"), sample_count=SPP, min_distance=0.001,
                          max_distance=0.3)}
    api.run(ctx, lo_poly_mesh_path=lo_path, tex_width=TEX, tex_height=TEX, seed=SEED, **solvers)
    assert not os.path.exists(solvers["positions"]["output_path"])
    assert not os.path.exists(solvers["height"]["output_path"])
    want = composed(ctx, lo_path, None, api.MAP_SMOOTH, api.NORMAL_IMPORT, api.NORMAL_IMPORT,
                    {"ao": solvers["ao"]}, 16)
    assert same_file(solvers["ao"]["output_path"], want["ao"])


def test_runner_errors(ctx, tmp_path):
    with pytest.raises(api.FornosError) as e:
        api.run(ctx, lo_poly_mesh_path=str(tmp_path / "none.ply"))
    assert "Missing low poly mesh" in str(e.value)
    bare = tmp_path / "bare.obj"
    bare.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")  # no texture coordinates
    with pytest.raises(api.FornosError) as e:
        api.run(ctx, lo_poly_mesh_path=str(bare), lo_poly_mesh_normal=api.NORMAL_COMPUTE_PER_FACE,
                mapping=api.MAP_LOWPOLY_NORMALS, tex_width=TEX, tex_height=TEX)
    assert "missing texture coordinates or normals" in str(e.value)
