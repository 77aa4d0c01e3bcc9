"""Writers of OBJ and PLY test files (test infrastructure): seeded random
meshes in the syntax variants the loaders must read alike."""
import struct

import numpy as np

PLY_TYPES = {"char": ("b", 1), "uchar": ("B", 1), "short": ("h", 2), "ushort": ("H", 2), "int": ("i", 4),
             "uint": ("I", 4), "float": ("f", 4), "double": ("d", 8)}
ALIASES = {"char": "int8", "uchar": "uint8", "short": "int16", "ushort": "uint16", "int": "int32", "uint": "uint32",
           "float": "float32", "double": "float64"}


def _num(rng, x):
    """A float written in one of several decimal spellings."""
    k = rng.integers(0, 5)
    if k == 0:
        return repr(float(x))
    if k == 1:
        return "%.9g" % x
    if k == 2:
        return "%.6e" % x
    if k == 3:
        return "%+.7f" % x
    return "%.3f" % x


def obj_text(seed, corners="vtn", polygons=True, quirks=True, n_pos=40, n_faces=60):
    """A random OBJ file.  corners: 'v', 'vt', 'vn' or 'vtn' (the corner
    format of every face).  Positions, texcoords and normals are referenced at
    random, so shared and unreferenced ones both occur."""
    rng = np.random.default_rng(seed)
    nl = "\r\n" if quirks and rng.random() < 0.3 else "\n"
    out = []
    pos = rng.normal(size=(n_pos, 3)).astype(np.float32)
    if quirks:
        pos[0, 0] = np.float32(-0.0)
    uv = rng.random((n_pos, 2)).astype(np.float32)
    nrm = rng.normal(size=(n_pos // 2, 3)).astype(np.float32)
    sp = (lambda: rng.choice([" ", "  ", "\t", " \t "])) if quirks else (lambda: " ")
    if quirks:
        out += ["# generated", "mtllib none.mtl", "o thing", "", "   ", "g group1"]
    for p in pos:
        w = (sp() + _num(rng, 1.0)) if quirks and rng.random() < 0.2 else ""
        out.append("v" + sp() + sp().join(_num(rng, x) for x in p) + w + (sp() if quirks and rng.random() < 0.1 else ""))
    for t in uv:
        w = (sp() + "0") if quirks and rng.random() < 0.2 else ""
        out.append("vt" + sp() + sp().join(_num(rng, x) for x in t) + w)
    for n in nrm:
        out.append("vn" + sp() + sp().join(_num(rng, x) for x in n))
    if quirks:
        out += ["s off", "usemtl m", "vp 0.5 0.5", "l 1 2", "p 3", "#f 1 2 3"]
    for _ in range(n_faces):
        k = int(rng.integers(3, 7)) if polygons else 3
        if quirks and rng.random() < 0.05:
            k = int(rng.integers(0, 3))  # a face too short to make triangles
        cs = []
        for _ in range(k):
            p = int(rng.integers(1, n_pos + 1))
            t = int(rng.integers(1, n_pos + 1))
            n = int(rng.integers(1, len(nrm) + 1))
            cs.append({"v": "%d" % p, "vt": "%d/%d" % (p, t), "vn": "%d//%d" % (p, n), "vtn": "%d/%d/%d" % (p, t, n)}[corners])
        out.append("f" + ("" if not cs else sp() + sp().join(cs)))
        if quirks and rng.random() < 0.05:
            out.append("# comment between faces")
    return nl.join(out) + (nl if rng.random() < 0.8 else "")


def ply_bytes(pos, faces, fmt="binary_little_endian", uv=None, nrm=None, face_nrm=None, pos_type="float",
              uv_type="float", nrm_type="float", index_type="uint", count_type="uchar", vertex_order="xyz",
              extra=True, face_first=False, comments=True, aliases=False, crlf=False):
    """A PLY file.  faces: list of index lists (any lengths).  vertex_order:
    the order of x y z in the header (e.g. 'zxy'); extra: add unrequested
    scalar and list properties."""
    n, m = len(pos), len(faces)
    tname = (lambda t: ALIASES[t]) if aliases else (lambda t: t)
    vprops = []  # (name, type, values per vertex)
    for c in vertex_order:
        vprops.append((c, pos_type, pos[:, "xyz".index(c)]))
    if extra:
        vprops.append(("quality", "uchar", np.arange(n) % 251))
    if uv is not None:
        vprops += [("s", uv_type, uv[:, 0]), ("t", uv_type, uv[:, 1])]
    if nrm is not None:
        vprops += [("nx", nrm_type, nrm[:, 0]), ("ny", nrm_type, nrm[:, 1]), ("nz", nrm_type, nrm[:, 2])]
    if extra:
        vprops.append(("red", "short", (np.arange(n) * 7) % 300 - 150))
    fprops = [("vertex_indices", "list")]
    if face_nrm is not None:
        fprops += [("nx", nrm_type, face_nrm[:, 0]), ("ny", nrm_type, face_nrm[:, 1]), ("nz", nrm_type, face_nrm[:, 2])]
    if extra:
        fprops += [("flags", "int", np.arange(m) - 3), ("tags", "list_extra")]
    eol = "\r\n" if crlf else "\n"
    head = ["ply", "format %s 1.0" % fmt]
    if comments:
        head += ["comment made by the test writer", "obj_info seeded"]

    def vert_block():
        h = ["element vertex %d" % n]
        h += ["property %s %s" % (tname(t), name) for name, t, _ in vprops]
        return h

    def face_block():
        h = ["element face %d" % m]
        for p in fprops:
            if p[1] == "list":
                h.append("property list %s %s vertex_indices" % (tname(count_type), tname(index_type)))
            elif p[1] == "list_extra":
                h.append("property list uchar float tags")
            else:
                h.append("property %s %s" % (tname(p[1]), p[0]))
        return h

    head += (face_block() + vert_block()) if face_first else (vert_block() + face_block())
    head.append("end_header")
    data = bytearray((eol.join(head) + eol).encode())
    if fmt == "ascii":
        def num(t, x):
            return repr(float(np.float32(x) if t == "float" else x)) if t in ("float", "double") else str(int(x))
        vlines = [" ".join(num(t, vals[i]) for _, t, vals in vprops) for i in range(n)]
        flines = []
        for i, f in enumerate(faces):
            parts = []
            for p in fprops:
                if p[1] == "list":
                    parts += [str(len(f))] + [str(int(v)) for v in f]
                elif p[1] == "list_extra":
                    parts += ["2", "0.5", "-1.25"]
                else:
                    parts.append(num(p[1], p[2][i]))
            flines.append(" ".join(parts))
        body = (flines + vlines) if face_first else (vlines + flines)
        data += (eol.join(body) + eol).encode()
        return bytes(data)
    e = ">" if fmt == "binary_big_endian" else "<"

    def pack(t, x):
        c = PLY_TYPES[t][0]
        return struct.pack(e + c, float(x) if c in "fd" else int(x))

    vbytes = bytearray()
    for i in range(n):
        for _, t, vals in vprops:
            vbytes += pack(t, vals[i])
    fbytes = bytearray()
    for i, f in enumerate(faces):
        for p in fprops:
            if p[1] == "list":
                fbytes += pack(count_type, len(f))
                for v in f:
                    fbytes += pack(index_type, v)
            elif p[1] == "list_extra":
                fbytes += pack("uchar", 2) + pack("float", 0.5) + pack("float", -1.25)
            else:
                fbytes += pack(p[1], p[2][i])
    data += (fbytes + vbytes) if face_first else (vbytes + fbytes)
    return bytes(data)


def random_ply_mesh(seed, n=30, m=40):
    rng = np.random.default_rng(seed)
    pos = rng.normal(size=(n, 3)).astype(np.float32)
    pos[1, 2] = np.float32(-0.0)
    uv = rng.random((n, 2)).astype(np.float32)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    fnrm = rng.normal(size=(m, 3)).astype(np.float32)
    faces = [list(rng.integers(0, n, 3)) for _ in range(m)]
    return pos, uv, nrm, fnrm, faces


def obj_of(mesh):
    """An OBJ file of a MeshArrays mesh: v / vt / vn with the mesh's own
    values ('%.9g' round-trips binary32), one v/t/n corner per vertex index.
    Loading it gives one vertex per face corner with the mesh's positions,
    texcoords and normals."""
    out = ["v %.9g %.9g %.9g" % tuple(p) for p in mesh.positions]
    out += ["vt %.9g %.9g" % tuple(t) for t in mesh.texcoords]
    out += ["vn %.9g %.9g %.9g" % tuple(n) for n in mesh.normals]
    v = mesh.vertices.astype(np.int64) + 1
    for tri in mesh.triangles:
        out.append("f " + " ".join("%d/%d/%d" % tuple(v[k]) for k in tri))
    return "\n".join(out) + "\n"
