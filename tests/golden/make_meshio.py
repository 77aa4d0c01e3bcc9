"""Generates tests/golden/meshio.npz: mesh files and what the reference's own
loader (Mesh::loadFile with tinyply 2.0, compiled on the host into oracle/_ref
by oracle/build_ref.py) makes of them.

    python tests/golden/make_meshio.py

Each entry holds the file's bytes (name_i gives its extension), ok_i (0 when
the loader rejects the file) and the five arrays the loader returned:
positions, texcoords, normals, vertices, triangles.  tests/test_meshio.py
replays them against fk_mesh_load.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.pyoracle import Reference  # noqa: E402
from tests import meshfiles as MF  # noqa: E402


def files():
    out = []
    for k, corners in enumerate(("v", "vt", "vn", "vtn")):
        out.append(("q%d.obj" % k, MF.obj_text(900 + k, corners, n_pos=12, n_faces=10).encode()))
    out.append(("bad.obj", b"v 0 0 0\nf 1/1 1 1\n"))
    out.append(("range.obj", b"v 1e-400 0 0\n"))
    pos, uv, nrm, fnrm, faces = MF.random_ply_mesh(77, n=10, m=8)
    out.append(("le.ply", MF.ply_bytes(pos, faces, uv=uv, nrm=nrm)))
    out.append(("be.ply", MF.ply_bytes(pos, faces, uv=uv, nrm=nrm, fmt="binary_big_endian", vertex_order="yzx")))
    out.append(("ascii.ply", MF.ply_bytes(pos, faces, uv=uv, face_nrm=fnrm, fmt="ascii", pos_type="double")))
    out.append(("ushort.ply", MF.ply_bytes(pos, faces, uv=uv, nrm=nrm, index_type="ushort", face_first=True)))
    out.append(("nox.ply", MF.ply_bytes(pos, faces, uv=uv, nrm=nrm, vertex_order="xy")))
    return out


def main():
    ref = Reference()
    blob = {}
    names = []
    with tempfile.TemporaryDirectory() as d:
        for i, (name, data) in enumerate(files()):
            p = os.path.join(d, name)
            with open(p, "wb") as fh:
                fh.write(data)
            arrs = ref.load_mesh(p)
            names.append(name)
            blob["file_%d" % i] = np.frombuffer(data, np.uint8)
            blob["ok_%d" % i] = np.int32(arrs is not None)
            for k, a in enumerate(arrs or ()):
                blob["arr_%d_%d" % (i, k)] = a
    blob["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "meshio.npz"), **blob)
    print("wrote", os.path.join(HERE, "meshio.npz"), len(names), "files")


if __name__ == "__main__":
    main()
