"""Mesh files (fk_mesh_load) against the reference's own loaders
(Mesh::loadFile, Src/mesh.cpp:235-617, and tinyply 2.0, compiled from source
in oracle/_ref): positions, texcoords and normals bit for bit, vertex and
triangle tables exactly, and the same files rejected.  Without the reference
build the committed golden fixtures (tests/golden/meshio.npz, made by
tests/golden/make_meshio.py from the same loader) stand in.  No GPU needed.

OBJ cases: every corner format, polygons (fans), faces of 0-2 corners, w
components, CRLF, tabs, comments and unknown statements, -0, syntax errors,
range errors, inconsistent corner formats, indices that do not resolve, an
unreadable file.  PLY cases: ASCII, binary little / big endian, float and
double values, uint and ushort index lists with uchar / int counts, vertex
and face normals, properties in another order, unrequested scalar and list
properties, the face element first, type aliases, CRLF header lines, missing
elements, truncated data; and the cases this loader defines where the
reference's result is unusable (no s / t or no normals, int index lists).
"""
import os
import re

import numpy as np
import pytest

from fornos_b200 import api
from tests import meshfiles as MF
from tests.cases import same_bits

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "meshio.npz")


def load(path):
    """fk_mesh_load's arrays, or None when it rejects the file."""
    try:
        m = api.Mesh.load(path)
    except api.FornosError as e:
        assert e.code == -1
        return None
    a = m.arrays()
    return a.positions, a.texcoords, a.normals, a.vertices, a.triangles


def same_mesh(a, b):
    if a is None or b is None:
        return a is None and b is None
    return (same_bits(a[0], b[0]) and same_bits(a[1], b[1]) and same_bits(a[2], b[2])
            and np.array_equal(a[3], b[3]) and np.array_equal(a[4], b[4]))


def resolves(ref):
    """The reference's mesh names only positions it has (else this loader
    rejects the file)."""
    return ref is not None and (len(ref[3]) == 0 or int(ref[3][:, 0].max()) < len(ref[0]))


def write(tmp_path, name, data):
    p = tmp_path / name
    p.write_bytes(data if isinstance(data, bytes) else data.encode())
    return str(p)


# ------------------------------------------------------------------ OBJ
@pytest.mark.parametrize("corners", ["v", "vt", "vn", "vtn"])
@pytest.mark.parametrize("seed", range(4))
def test_obj_matches_reference(reference, tmp_path, corners, seed):
    p = write(tmp_path, "m.obj", MF.obj_text(100 * seed + len(corners), corners))
    ref = reference.load_mesh(p)
    assert resolves(ref)
    assert same_mesh(load(p), ref)


def test_obj_plain_triangles(reference, tmp_path):
    p = write(tmp_path, "t.obj", MF.obj_text(7, "vtn", polygons=False, quirks=False, n_pos=500, n_faces=2000))
    ref = reference.load_mesh(p)
    assert len(ref[4]) == 2000 and same_mesh(load(p), ref)


OBJ_CASES = {
    "missing z": "v 1 2\nf 1 1 1\n",
    "extra value": "v 1 2 3 4 5\n",
    "vt one value": "vt 0.5\n",
    "vn two values": "vn 0 1\n",
    "trailing text": "v 1 2 3 x\n",
    "bad corner": "v 0 0 0\nf 1a 1 1\n",
    "mixed corner formats": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nf 1/1 2/1 3/1\nf 1 2 3\n",
    "missing normal index": "v 0 0 0\nf 1// 1// 1//\n",
    "overflow": "v 1e39 0 0\n",
    "double overflow": "v 1e400 0 0\n",
    "underflow": "v 1e-400 0 0\n",
    "inf and nan": "v inf -inf nan\nv 0x1p3 1 2\nf 1 2 1\n",
    "denormal float": "v 1e-40 0 0\nv 1 1 1\nv 2 2 2\nf 1 2 3\n",
    "texcoord w and spacing": "v 0 0 0\n\tv 1 0 0\nv 0 1 0 \r\nvt 0 0 0\nvt 1 0\nf  1/1  2/2\t3/1  \n",
    "no trailing newline": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3",
    "short faces": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf\nf 1\nf 1 2\nf 1 2 3\n",
    "texcoord index 0": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nf 1/0 2/0 3/0\nf 1/1 2/1 3/1\n",
    "index beyond texcoords": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nf 1/9 2/9 3/9\n",
    "unknown statements": "v 0 0 0\nvx 1 2 3\nv 1 0 0\nvp 1\nv 0 1 0\nfo 1 2 3\nf 1 2 3\n#v 9 9 9\n",
    "empty": "",
    "blank lines": "\n\n   \n\t\n",
    "embedded nul": "v 0 0 0\x00 junk\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
    "int wraps": "v 0 0 0\nf 4294967297 4294967297 4294967297\n",
}


@pytest.mark.parametrize("name", list(OBJ_CASES))
def test_obj_cases(reference, tmp_path, name):
    p = write(tmp_path, "c.obj", OBJ_CASES[name])
    ref = reference.load_mesh(p)
    mine = load(p)
    if ref is not None and not resolves(ref):
        assert mine is None  # the reference's mesh names positions it lacks
    else:
        assert same_mesh(mine, ref), (mine, ref)


@pytest.mark.parametrize("text", ["v 0 0 0\nv 1 0 0\nv 0 1 0\nf -3 -2 -1\n", "v 0 0 0\nf 0 1 1\n",
                                  "v 0 0 0\nf 1 2 1\n"])
def test_obj_unresolved_indices(reference, tmp_path, text):
    p = write(tmp_path, "u.obj", text)
    ref = reference.load_mesh(p)
    assert ref is not None and not resolves(ref)
    assert load(p) is None


def test_obj_unreadable(reference, tmp_path):
    p = str(tmp_path / "missing.obj")
    ref = reference.load_mesh(p)
    mine = load(p)
    assert ref is not None and len(ref[0]) == 0 and same_mesh(mine, ref)


def test_other_extension(tmp_path):
    p = write(tmp_path, "m.stl", "v 0 0 0\n")
    assert load(p) is None
    assert load(write(tmp_path, "m.OBJ", "v 0 0 0\n")) is None  # the extension test is case-sensitive


# ------------------------------------------------------------------ PLY
PLY_VARIANTS = {
    "binary le": {},
    "binary be": {"fmt": "binary_big_endian"},
    "ascii": {"fmt": "ascii"},
    "double values": {"pos_type": "double", "uv_type": "double", "nrm_type": "double"},
    "ascii double": {"fmt": "ascii", "pos_type": "double", "nrm_type": "double"},
    "ushort indices": {"index_type": "ushort"},
    "int counts": {"count_type": "int", "fmt": "binary_big_endian"},
    "zxy order": {"vertex_order": "zxy"},
    "no extras": {"extra": False, "comments": False},
    "face element first": {"face_first": True},
    "aliases": {"aliases": True},
    "crlf ascii": {"fmt": "ascii", "crlf": True},
    "face normals": {"normals": "face"},
    "face normals ascii": {"normals": "face", "fmt": "ascii"},
}


def ply_case(seed, opts):
    pos, uv, nrm, fnrm, faces = MF.random_ply_mesh(seed)
    opts = dict(opts)
    where = opts.pop("normals", "vertex")
    return MF.ply_bytes(pos, faces, uv=uv, nrm=nrm if where == "vertex" else None,
                        face_nrm=fnrm if where == "face" else None, **opts)


@pytest.mark.parametrize("name", list(PLY_VARIANTS))
def test_ply_matches_reference(reference, tmp_path, name):
    p = write(tmp_path, "m.ply", ply_case(len(name), PLY_VARIANTS[name]))
    ref = reference.load_mesh(p)
    assert resolves(ref)
    mine = load(p)
    assert same_mesh(mine, ref)
    if "face normals" in name:
        assert list(mine[3][3:6, 2]) == [3, 3, 3]  # face i's corners name normal 3 i


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian"])
@pytest.mark.parametrize("count_type,index_type", [("uchar", "uint"), ("int", "ushort"), ("ushort", "uint")])
@pytest.mark.parametrize("lengths", ["triangles", "quads", "mixed"])
def test_ply_face_lists_of_one_length(reference, tmp_path, fmt, count_type, index_type, lengths):
    """A face element holding only the index list: when every face has the
    first one's length the loader copies the records in bulk, otherwise face
    by face; both read what the reference reads."""
    pos, uv, nrm, _, faces = MF.random_ply_mesh(5, n=40, m=60)
    if lengths == "quads":
        faces = [f + [int((f[0] + 1) % 40)] for f in faces]
    elif lengths == "mixed":
        faces[17] = faces[17] + [int((faces[17][0] + 1) % 40)]
    p = write(tmp_path, "u.ply", MF.ply_bytes(pos, faces, fmt=fmt, uv=uv, nrm=nrm, count_type=count_type,
                                               index_type=index_type, extra=False))
    ref = reference.load_mesh(p)
    assert resolves(ref)
    assert same_mesh(load(p), ref)


def test_ply_polygons_read_as_triples(reference, tmp_path):
    # quads: the reference reads the flattened index list three at a time
    pos, uv, nrm, _, _ = MF.random_ply_mesh(3, n=30, m=4)
    faces = [[0, 1, 2, 3], [4, 5, 6, 7], [8, 9, 10, 11], [12, 13, 14, 15]]
    p = write(tmp_path, "q.ply", MF.ply_bytes(pos, faces, uv=uv, nrm=nrm))
    ref = reference.load_mesh(p)
    assert same_mesh(load(p), ref)
    assert list(ref[3][3:6, 0]) == [3, 4, 5]


def test_ply_rejected_like_reference(reference, tmp_path):
    pos, uv, nrm, _, faces = MF.random_ply_mesh(4)
    good = MF.ply_bytes(pos, faces, uv=uv, nrm=nrm, extra=False)
    cases = {
        "no vertex element": good.replace(b"element vertex", b"element points"),
        "no x": good.replace(b"property float x", b"property float q"),
        "no faces": good.replace(b"vertex_indices", b"vertex_index"),
        "unknown value type": good.replace(b"property float x", b"property half x"),
        "missing file": None,
    }
    for name, data in cases.items():
        p = str(tmp_path / "missing.ply") if data is None else write(tmp_path, name.replace(" ", "_") + ".ply", data)
        assert reference.load_mesh(p) is None, name
        assert load(p) is None, name


def test_ply_truncated_and_unparsable(tmp_path):
    # the reference goes on with zeros or uninitialised memory here; this loader rejects the file
    pos, uv, nrm, _, faces = MF.random_ply_mesh(5)
    good = MF.ply_bytes(pos, faces, uv=uv, nrm=nrm)
    assert load(write(tmp_path, "cut.ply", good[:-7])) is None
    asc = MF.ply_bytes(pos, faces, uv=uv, nrm=nrm, fmt="ascii")
    assert load(write(tmp_path, "cut_ascii.ply", asc[:len(asc) // 2])) is None
    assert load(write(tmp_path, "word.ply", asc.replace(b"end_header\n", b"end_header\nabc ", 1))) is None


def test_ply_defined_where_reference_fails(tmp_path):
    """No s / t, no normals, int index lists: the reference's loader
    dereferences a null buffer or reads every index as UINT32_MAX; this
    loader gives the arrays its vertex loop intends."""
    pos, uv, nrm, _, faces = MF.random_ply_mesh(6)
    flat = np.asarray(faces, np.uint32).reshape(-1)
    none = 0xFFFFFFFF
    m = load(write(tmp_path, "bare.ply", MF.ply_bytes(pos, faces)))
    assert same_bits(m[0], pos) and len(m[1]) == 0 and len(m[2]) == 0
    assert np.array_equal(m[3][:, 0], flat) and (m[3][:, 1] == none).all() and (m[3][:, 2] == none).all()
    assert np.array_equal(m[4].reshape(-1), np.arange(len(flat)))
    for it in ("int", "short", "uchar"):
        m = load(write(tmp_path, "i.ply", MF.ply_bytes(pos, faces, uv=uv, nrm=nrm, index_type=it, fmt="ascii")))
        assert np.array_equal(m[3][:, 0], flat) and np.array_equal(m[3][:, 1], flat)
        assert np.array_equal(m[3][:, 2], flat) and same_bits(m[1], uv) and same_bits(m[2], nrm)


# ------------------------------------------------------------------ golden fixtures
def test_golden_fixtures(tmp_path):
    g = np.load(GOLDEN, allow_pickle=False)
    names = [str(n) for n in g["names"]]
    assert names
    for i, name in enumerate(names):
        p = write(tmp_path, name, g["file_%d" % i].tobytes())
        mine = load(p)
        if int(g["ok_%d" % i]) == 0:
            assert mine is None, name
            continue
        ref = tuple(g["arr_%d_%d" % (i, k)] for k in range(5))
        assert same_mesh(mine, ref), name


def test_run_params_defaults():
    """fk_run_params_default carries FornosParameters' defaults (Src/fornos.h)."""
    p = api.run_params()
    assert (p.bvh_tris_per_node, p.tex_width, p.tex_height, p.tex_dilation, p.ignore_backfaces) == (8, 2048, 2048, 16, 1)
    assert p.mapping == api.MAP_SMOOTH and abs(p.mapping_edge - 0.05) < 1e-7
    assert p.lo_poly_mesh_normal == p.hi_poly_mesh_normal == api.NORMAL_IMPORT
    for s in (p.ao, p.bent_normals, p.thickness):
        assert s.sample_count == 256 and abs(s.min_distance - 0.01) < 1e-7 and s.max_distance == 10.0
    assert p.height.normalize_output == 1 and p.normals.tangent_space == 1 and p.bent_normals.tangent_space == 1
    assert not any(getattr(p, k).enabled for k in api.RUN_SOLVERS)


def test_ply_zero_width_data_is_not_looped(tmp_path):
    """Binary elements or lists whose items have an unknown type hold no bytes:
    skipped at once however large the count, rejected when requested."""
    import struct
    import time
    hdr = lambda body: ("ply\nformat binary_little_endian 1.0\n" + body + "end_header\n").encode()
    v = "".join("property float %s\n" % k for k in ("x", "y", "z", "s", "t", "nx", "ny", "nz"))
    vdata = b"".join(struct.pack("<8f", i, 0, 0, 0, 0, 0, 0, 1) for i in range(3))
    fdata = struct.pack("<B3I", 3, 0, 1, 2)
    files = {
        "element": hdr("element vertex 3\n" + v + "element face 1\nproperty list uchar uint vertex_indices\n"
                       "element junk 999999999999\nproperty half q\n") + vdata + fdata,
        "list": hdr("element vertex 3\n" + v + "element face 1\nproperty list uint half junk\n"
                    "property list uchar uint vertex_indices\n") + vdata + struct.pack("<I", 4000000000) + fdata,
    }
    for name, data in files.items():
        t = time.time()
        m = load(write(tmp_path, name + ".ply", data))
        assert time.time() - t < 5 and m is not None and len(m[4]) == 1, name
    requested = hdr("element vertex 3\n" + v.replace("float x", "half x") + "element face 1\n"
                    "property list uchar uint vertex_indices\n") + vdata + fdata
    assert load(write(tmp_path, "req.ply", requested)) is None


def test_mutated_files_load_or_reject(tmp_path):
    """Seeded byte mutations, truncations and splices of valid OBJ / PLY files:
    each loads into a valid mesh or is rejected, never more."""
    rng = np.random.default_rng(2024)
    pos, uv, nrm, fnrm, faces = MF.random_ply_mesh(1, n=12, m=10)
    bases = [(".ply", MF.ply_bytes(pos, faces, fmt=f, uv=uv, nrm=nrm)) for f in
             ("binary_little_endian", "binary_big_endian", "ascii")]
    bases += [(".obj", MF.obj_text(3, c, n_pos=8, n_faces=6).encode()) for c in ("v", "vt", "vn", "vtn")]
    loaded = 0
    for it in range(400):
        ext, data = bases[it % len(bases)]
        b = bytearray(data)
        for _ in range(int(rng.integers(1, 4))):
            k = int(rng.integers(3))
            if k == 0:
                b[int(rng.integers(len(b)))] = int(rng.integers(256))
            elif k == 1:
                b = b[:int(rng.integers(1, len(b)))]
            else:
                i = int(rng.integers(len(b) + 1))
                b[i:i] = bytes(rng.integers(0, 256, int(rng.integers(1, 9)), dtype=np.uint8))
        m = load(write(tmp_path, "f" + ext, bytes(b)))
        if m is not None:
            loaded += 1
            assert len(m[3]) == 0 or int(m[3][:, 0].max()) < len(m[0])
    assert loaded > 0


def test_bench_ply_layout(reference, tmp_path):
    """The binary PLY the benchmark's files-to-images step writes reads the same
    through both loaders, with the mesh's own positions and texcoords."""
    import bench
    from fornos_b200 import workloads as W
    lo, _ = W.plane_pair(seed=2, lo_quads=6, hi_quads=8, bumps=3)
    p = str(tmp_path / "lo.ply")
    bench.write_ply(p, lo)
    mine, ref = load(p), reference.load_mesh(p)
    assert same_mesh(mine, ref)
    v = lo.vertices.astype(np.int64)
    assert same_bits(mine[0], lo.positions[v[:, 0]]) and same_bits(mine[1], lo.texcoords[v[:, 1]])


def test_obj_large_file_in_ranges(reference, tmp_path):
    """Files of more than a few MB are parsed in ranges of whole lines on
    several threads and merged in file order: the same mesh as the reference's
    loader, and the same rejections, including errors and a corner format that
    only a later range sees, and a first range without faces."""
    block = MF.obj_text(31, "vtn", n_pos=4000, n_faces=6000)
    if not block.endswith("\n"):
        block += "\n"
    text = block * 12  # about 11 MB, every quirk in every range; indices are absolute, so they still resolve
    rng = np.random.default_rng(8)
    verts = "".join("v %.9g %.9g %.9g\n" % tuple(p) for p in rng.normal(size=(150000, 3)).astype(np.float32))
    cases = {"blocks": text, "late syntax error": text + "v 1 2\n", "late corner format": text + "f 1 2 3\n",
             "faceless first range": verts + text}
    for name, body in cases.items():
        p = write(tmp_path, "big.obj", body)
        ref = reference.load_mesh(p)
        mine = load(p)
        assert same_mesh(mine, ref), name
        assert (ref is None) == name.startswith("late"), name


def test_loaders_under_sanitizers(tmp_path):
    """fk_meshio.cpp built alone under AddressSanitizer / UBSan
    (tests/meshio_check/load_files.cpp) over seeded mutations of valid PLY files
    (ASCII and both binary orders; uchar / ushort / int counts; triangles,
    quads and extra properties) and OBJ files: no read or write outside a
    buffer, no undefined behaviour, whatever the bytes."""
    import subprocess

    from fornos_b200 import build as fk_build
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "load_files")
    p = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-pthread", "-fno-omit-frame-pointer",
                        "-fsanitize=address,undefined", "-I" + os.path.join(fk_build.CUDA, "include"),
                        os.path.join(root, "tests", "meshio_check", "load_files.cpp"),
                        os.path.join(root, "fornos_b200", "csrc", "fk_meshio.cpp"),
                        os.path.join(root, "fornos_b200", "csrc", "fk_mesh.cpp"), "-o", exe],
                       capture_output=True, text=True)
    if p.returncode != 0:
        pytest.skip("no sanitizer build: %s" % p.stderr.strip().splitlines()[-1:])
    rng = np.random.default_rng(31)
    pos, uv, nrm, _, faces = MF.random_ply_mesh(1, n=12, m=10)
    quads = [f + [int((f[0] + 1) % 12)] for f in faces]
    bases = []
    for fmt in ("binary_little_endian", "binary_big_endian", "ascii"):
        for ct, it in (("uchar", "uint"), ("ushort", "uint"), ("int", "ushort")):
            for fc in (faces, quads):
                bases.append((".ply", MF.ply_bytes(pos, fc, fmt=fmt, uv=uv, nrm=nrm, count_type=ct, index_type=it,
                                                   extra=False)))
        bases.append((".ply", MF.ply_bytes(pos, faces, fmt=fmt, uv=uv, nrm=nrm)))
    bases += [(".obj", MF.obj_text(3, c, n_pos=8, n_faces=6).encode()) for c in ("v", "vt", "vn", "vtn")]
    files = []
    for i in range(4000):
        ext, data = bases[i % len(bases)]
        b = bytearray(data)
        for _ in range(int(rng.integers(1, 4))):
            k = int(rng.integers(3))
            if k == 0:
                b[int(rng.integers(len(b)))] = int(rng.integers(256))
            elif k == 1 and len(b) > 2:
                b = b[:int(rng.integers(1, len(b)))]
            else:
                j = int(rng.integers(len(b) + 1))
                b[j:j] = bytes(rng.integers(0, 256, int(rng.integers(1, 9)), dtype=np.uint8))
        files.append(write(tmp_path, "m%04d%s" % (i, ext), bytes(b)))
    files += [write(tmp_path, "base%02d%s" % (i, ext), data) for i, (ext, data) in enumerate(bases)]
    r = subprocess.run([exe] + files, capture_output=True, text=True)
    assert r.returncode == 0 and "runtime error" not in r.stderr and "ERROR" not in r.stderr, r.stderr[-2000:]
    counts = dict(re.findall(r"(\w+) (\d+)", r.stdout))
    assert int(counts["loaded"]) >= len(bases)  # every valid base file loads
