"""Generates tests/golden/*.npz from the reference's own code compiled on the
host (oracle/_ref, built by oracle/build_ref.py from the reference tree).

    python tests/golden/make_golden.py

Each fixture holds the input meshes (so the fixtures do not depend on the
mesh generators) and the reference's outputs for them: normal and tangent
generators, the BVH build + flatten, the UV raster + compaction (32x32, the
three mapping modes), the seeded sample table, both mesh-mapping shaders,
ambient occlusion / bent normals / thickness (8 spp), the gathers and the
tangent-space transform.  tests/test_golden.py replays them against the
oracle, the product's host code and (on a GPU) the product's kernels.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fornos_b200 import workloads as W  # noqa: E402
from oracle.pyoracle import Reference, pixels8  # noqa: E402

CASES = {
    "sphere": lambda: W.sphere_pair(seed=1, lo_seg=(16, 8), hi_seg=(48, 24)),
    "plane": lambda: W.plane_pair(seed=2, lo_quads=4, hi_quads=40, bumps=10),
    "icosphere": lambda: W.icosphere_pair(seed=3, lo_subdiv=1, hi_subdiv=3),
}
TEX, SPP, SEED, MIN_D, MAX_D = 32, 8, 7, 0.001, 0.3


def mesh_fields(prefix, m):
    return {prefix + "positions": m.positions, prefix + "texcoords": m.texcoords, prefix + "normals": m.normals,
            prefix + "vertices": m.vertices, prefix + "triangles": m.triangles}


def make(name, R):
    lo, hi = CASES[name]()
    out = {}
    out.update(mesh_fields("lo_", lo))
    out.update(mesh_fields("hi_", hi))
    for which in ("face", "vertex", "welded"):
        v, n = R.normals(hi, which)
        out["hi_%s_vertices" % which], out["hi_%s_normals" % which] = v, n
        v, n = R.normals(lo, which)
        out["lo_%s_vertices" % which], out["lo_%s_normals" % which] = v, n
    hi.vertices, hi.normals = out["hi_vertex_vertices"], out["hi_vertex_normals"]
    t, b = R.tangent_space(lo)
    out["lo_tangents"], out["lo_bitangents"] = t, b
    lo.tangents, lo.bitangents = t, b
    dirs = (out["lo_welded_vertices"], out["lo_welded_normals"])
    nodes, p4, n4 = R.scene(hi, 8)
    out["nodes"], out["pos4"], out["nrm4"] = nodes.view(np.uint32).reshape(-1, 9), p4, n4
    for mode in (0, 1, 2):
        cm = R.raster(lo, TEX, TEX, mode, dirs)
        for k, v in cm.items():
            out["map%d_%s" % (mode, k)] = v
    samples = R.samples(SPP, 4096, SEED)
    # the table is regenerated by the code under test and checked by digest
    out["samples_sha256"] = np.frombuffer(hashlib.sha256(samples.tobytes()).digest(), np.uint8)
    out["samples_head"] = samples[:64]
    px = pixels8(out["map0_positions"], out["map0_directions"])
    for cull in (0, 1):
        c, t = R.meshmap(nodes, p4, px, bool(cull))
        out["coords%d" % cull], out["tidx%d" % cull] = c, t
    coords, tidx = out["coords1"], out["tidx1"]
    for kind, label in ((0, "ao"), (1, "bn"), (2, "thick")):
        out[label] = R.hemisphere(kind, nodes, p4, n4, coords, tidx, samples, SPP, MIN_D, MAX_D)
    for what, label in ((0, "height"), (1, "position"), (2, "normal")):
        out[label] = R.gather(what, p4, n4, coords, tidx)
    out["normal_ts"] = R.tangent_transform(out["map0_normals"], out["map0_tangents"], out["map0_bitangents"],
                                           out["normal"])
    out["params"] = np.array([TEX, SPP, SEED, MIN_D, MAX_D], np.float64)
    np.savez_compressed(os.path.join(HERE, "%s.npz" % name), **out)
    return sum(v.nbytes for v in out.values())


if __name__ == "__main__":
    R = Reference()
    for name in CASES:
        print(name, make(name, R), "bytes before compression")
