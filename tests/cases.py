"""Small seeded bake cases shared by the tests (product host preprocessing +
the oracle's view of the same arrays)."""
import numpy as np

from fornos_b200 import api
from fornos_b200 import workloads as W


class Case:
    """A low-/high-poly pair prepared as Src/fornos.cpp:53-157 prepares it:
    high-poly normals per vertex, low-poly tangent space, welded-normal copy
    of the low-poly for Smooth mapping directions, BVH with 8 triangles per
    leaf."""

    def __init__(self, lo, hi, max_tris=8, hi_normals=True):
        self.hm = api.Mesh(hi)
        if hi_normals:
            self.hm.compute_vertex_normals()
        self.hi = self.hm.arrays()
        self.lm = api.Mesh(lo)
        self.lm.compute_tangent_space()
        self.lo = self.lm.arrays()
        self.dm = self.lm.copy()
        self.dm.compute_vertex_normals_aggressive()
        d = self.dm.arrays()
        self.dirs = (d.vertices, d.normals)
        self.bvh = api.BVH.create_binary(self.hm, max_tris)
        self.nodes, self.pos4, self.nrm4 = self.bvh.flatten(self.hm)


def sphere(seed=1, lo=(32, 16), hi=(64, 32)):
    return Case(*W.sphere_pair(seed=seed, lo_seg=lo, hi_seg=hi))


def plane(seed=2, lo=8, hi=64, bumps=20):
    return Case(*W.plane_pair(seed=seed, lo_quads=lo, hi_quads=hi, bumps=bumps))


def icosphere(seed=3, lo=1, hi=4):
    return Case(*W.icosphere_pair(seed=seed, lo_subdiv=lo, hi_subdiv=hi))


def pix8(cmap):
    n = len(cmap["indices"])
    out = np.zeros((n, 8), np.float32)
    out[:, 0:3] = cmap["positions"]
    out[:, 4:7] = cmap["directions"]
    return out


def pixt12(cmap):
    n = len(cmap["indices"])
    out = np.zeros((n, 12), np.float32)
    out[:, 0:3] = cmap["normals"]
    out[:, 4:7] = cmap["tangents"]
    out[:, 8:11] = cmap["bitangents"]
    return out


def bits(a):
    """Bit patterns with every NaN mapped to one value: x86 and CUDA produce
    different NaN payloads for the same invalid operation (e.g. 0 * inf in
    normalize of a zero tangent), which carries no information."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).copy()
    u[np.isnan(np.asarray(a, np.float32))] = 0x7FC00000
    return u


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(bits(a), bits(b))


def record(test, **values):
    """Appends one JSON line of measured values to tests/.out/records.jsonl
    (ignored by git): figures a test bounds, kept for reading after a run."""
    import json
    import os
    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), ".out")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "records.jsonl"), "a") as fh:
        fh.write(json.dumps(dict(test=test, **{k: float(v) for k, v in values.items()})) + "\n")
