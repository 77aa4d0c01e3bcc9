"""ctypes front-end for the CPU oracle (oracle/oracle.cpp) and for the
reference's own code compiled into oracle/_ref (oracle/build_ref.py).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfornos_ref.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_f32 = ctypes.c_float
_int = ctypes.c_int

NODE_DTYPE = np.dtype([("lo", np.float32, 3), ("hi", np.float32, 3), ("start", np.uint32), ("end", np.uint32),
                       ("jump", np.uint32)])
assert NODE_DTYPE.itemsize == 36
FLT_MAX = float(np.finfo(np.float32).max)


def build_oracle(force=False):
    """Compiles oracle/liboracle.so with g++ (IEEE, no contraction, OpenMP)."""
    src = os.path.join(HERE, "oracle.cpp")
    if not force and os.path.exists(ORACLE_SO) and os.path.getmtime(ORACLE_SO) >= os.path.getmtime(src):
        return ORACLE_SO
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           src, "-o", ORACLE_SO]
    subprocess.run(cmd, check=True)
    return ORACLE_SO


def build_ref(force=False):
    """Builds oracle/_ref from the reference tree when it is present (force:
    rebuild even when a build exists; without the tree an existing build is
    kept)."""
    if os.path.exists(REF_SO) and not force:
        return REF_SO
    p = subprocess.run(["python", os.path.join(HERE, "build_ref.py")], capture_output=True, text=True)
    return REF_SO if os.path.exists(REF_SO) else None


def ptr(a, t=_f32p):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _mesh_args(m):
    return [m.positions.shape[0], ptr(m.positions)]


class Oracle:
    """Restated reference algorithm (oracle/oracle.cpp)."""

    def __init__(self, path=None):
        self.lib = ctypes.CDLL(path or build_oracle())
        L = self.lib
        L.orc_scene_build.restype = _vp
        L.orc_raster.restype = _vp
        L.orc_threads.restype = _int

    def threads(self, n=0):
        return self.lib.orc_threads(n)

    # ---- host preprocessing (Src/mesh.cpp:627-768)
    def normals(self, m, which):
        """which: 'face' | 'vertex' | 'welded'.  Returns (vertices, normals)."""
        vtx = np.zeros_like(m.vertices)
        if which == "face":
            nrm = np.zeros((m.triangle_count, 3), np.float32)
            self.lib.orc_face_normals(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.vertices)),
                                      ptr(m.vertices, _u32p), _u32(m.triangle_count), ptr(m.triangles, _u32p),
                                      ptr(vtx, _u32p), ptr(nrm))
        elif which == "vertex":
            nrm = np.zeros((len(m.positions), 3), np.float32)
            self.lib.orc_vertex_normals(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.vertices)),
                                        ptr(m.vertices, _u32p), _u32(m.triangle_count), ptr(m.triangles, _u32p),
                                        ptr(vtx, _u32p), ptr(nrm))
        else:
            nrm = np.zeros((3 * m.triangle_count + 1, 3), np.float32)
            n = self.lib.orc_welded_normals(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.vertices)),
                                            ptr(m.vertices, _u32p), _u32(m.triangle_count), ptr(m.triangles, _u32p),
                                            ptr(vtx, _u32p), ptr(nrm))
            nrm = nrm[:n].copy()
        return vtx, nrm

    def tangent_space(self, m):
        t = np.zeros((len(m.vertices), 3), np.float32)
        b = np.zeros_like(t)
        self.lib.orc_tangent_space(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.texcoords)),
                                   ptr(m.texcoords), _u32(len(m.normals)), ptr(m.normals), _u32(len(m.vertices)),
                                   ptr(m.vertices, _u32p), _u32(m.triangle_count), ptr(m.triangles, _u32p),
                                   ptr(t), ptr(b))
        return t, b

    # ---- BVH build + flatten (Src/bvh.cpp, Src/meshmapping.cpp:62-125)
    def scene(self, m, max_tris=8, max_depth=8192):
        h = self.lib.orc_scene_build(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.normals)),
                                     ptr(m.normals), _u32(len(m.vertices)), ptr(m.vertices, _u32p),
                                     _u32(m.triangle_count), ptr(m.triangles, _u32p), _u32(max_tris),
                                     _u32(max_depth))
        nn, nc = _u32(), _u32()
        self.lib.orc_scene_sizes(_vp(h), ctypes.byref(nn), ctypes.byref(nc))
        nodes = np.zeros(nn.value, NODE_DTYPE)
        pos4 = np.zeros((nc.value, 4), np.float32)
        nrm4 = np.zeros((nc.value, 4), np.float32)
        self.lib.orc_scene_copy(_vp(h), nodes.ctypes.data_as(_vp), ptr(pos4), ptr(nrm4))
        self.lib.orc_scene_free(_vp(h))
        return nodes, pos4, nrm4

    # ---- raster + compaction (Src/compute.cpp)
    def raster(self, m, w, h, mode=0, dirs=None, edge=0.05):
        """mode 0 Smooth (dirs = (vertices, normals) of the welded copy), 1
        LowPolyNormals, 2 Hybrid.  Returns dict of compressed arrays or None."""
        dv, dn = (None, None) if dirs is None else dirs
        hm = self.lib.orc_raster(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.texcoords)), ptr(m.texcoords),
                                 _u32(len(m.normals)), ptr(m.normals), _u32(len(m.vertices)), ptr(m.vertices, _u32p),
                                 _u32(m.triangle_count), ptr(m.triangles, _u32p), ptr(m.tangents),
                                 ptr(m.bitangents), ptr(dv, _u32p), ptr(dn), _u32(w), _u32(h), _int(mode), _f32(edge))
        if not hm:
            return None
        c = _u32()
        self.lib.orc_compress(_vp(hm), ctypes.byref(c), None, None, None, None, None, None)
        n = c.value
        out = {k: np.zeros((n, 3), np.float32) for k in ("positions", "directions", "normals", "tangents",
                                                          "bitangents")}
        out["indices"] = np.zeros(n, np.uint32)
        self.lib.orc_compress(_vp(hm), ctypes.byref(c), ptr(out["indices"], _u32p), ptr(out["positions"]),
                              ptr(out["directions"]), ptr(out["normals"]), ptr(out["tangents"]),
                              ptr(out["bitangents"]))
        self.lib.orc_map_free(_vp(hm))
        return out

    # ---- sample table (Src/math.h:314-382)
    def samples(self, spp, perms=4096, seed=0):
        out = np.zeros((perms * spp, 4), np.float32)
        self.lib.orc_samples(_u32(spp), _u32(perms), _u32(seed), ptr(out))
        return out

    # ---- shaders
    def meshmap(self, nodes, pos4, pix8, cull=True, counters=False, max_dist=FLT_MAX):
        """max_dist: the walks' initial closest distance (FLT_MAX in the
        shaders)."""
        n = pix8.shape[0]
        coords = np.zeros((n, 4), np.float32)
        tidx = np.zeros(n, np.uint32)
        ctr = np.zeros(2, np.uint64) if counters else None
        self.lib.orc_meshmap(nodes.ctypes.data_as(_vp), _u32(len(nodes)), ptr(pos4), ptr(pix8), _u32(n), _int(int(cull)),
                             ctypes.c_float(max_dist), ptr(coords), ptr(tidx, _u32p), ptr(ctr, _u64p))
        return (coords, tidx, ctr) if counters else (coords, tidx)

    def hemisphere(self, kind, nodes, pos4, nrm4, coords, tidx, samples4, spp, min_d, max_d, texels=None,
                   perms=4096, counters=False):
        """kind 0 AO, 1 bent normals, 2 thickness.  Returns (out, hits[, ctr])
        for the listed texels (all texels when `texels` is None)."""
        n = len(tidx) if texels is None else len(texels)
        out = np.zeros((n, 3) if kind == 1 else n, np.float32)
        hits = np.zeros(n, np.uint32)
        ctr = np.zeros(2, np.uint64) if counters else None
        tx = None if texels is None else np.ascontiguousarray(texels, np.uint32)
        self.lib.orc_hemisphere(_int(kind), nodes.ctypes.data_as(_vp), _u32(len(nodes)), ptr(pos4), ptr(nrm4),
                                ptr(coords), ptr(tidx, _u32p), ptr(samples4), _u32(spp), _u32(perms), _f32(min_d),
                                _f32(max_d), ptr(tx, _u32p), _u32(n), ptr(out), ptr(hits, _u32p), ptr(ctr, _u64p))
        return (out, hits, ctr) if counters else (out, hits)

    def sample_rays(self, kind, nodes, pos4, nrm4, coords, tidx, samples4, spp, min_d, max_d, texel, perms=4096):
        t = np.zeros(spp, np.float32)
        r = self.lib.orc_sample_rays(_int(kind), nodes.ctypes.data_as(_vp), _u32(len(nodes)), ptr(pos4), ptr(nrm4),
                                     ptr(coords), ptr(tidx, _u32p), ptr(samples4), _u32(spp), _u32(perms),
                                     _f32(min_d), _f32(max_d), _u32(texel), ptr(t))
        return t if r == 0 else None

    def gather(self, what, pos4, nrm4, coords, tidx):
        n = len(tidx)
        out = np.zeros(n if what == 0 else (n, 3), np.float32)
        self.lib.orc_gather(_int(what), ptr(pos4), ptr(nrm4), ptr(coords), ptr(tidx, _u32p), _u32(n), ptr(out))
        return out

    def tangent_transform(self, n3, t3, b3, v3):
        io = np.ascontiguousarray(v3, np.float32).copy()
        self.lib.orc_tangent_transform(ptr(n3), ptr(t3), ptr(b3), _u32(len(io)), ptr(io))
        return io

    # ---- image export (Src/image.cpp:22-405)
    def export_float(self, w, h, idx, data, flo=0.0, fhi=0.0, normalize=True, dilate=0, rgb8=True):
        """(image, (min, max)): h x w x 3 uint8 (rgb8) or h x w float32, file row order."""
        idx = np.ascontiguousarray(idx, np.uint32)
        data = np.ascontiguousarray(data, np.float32)
        out = np.zeros((h, w, 3), np.uint8) if rgb8 else np.zeros((h, w), np.float32)
        mm = np.zeros(2, np.float32)
        self.lib.orc_export_float(_u32(w), _u32(h), _u32(len(idx)), ptr(idx, _u32p), ptr(data), ctypes.c_float(flo),
                                  ctypes.c_float(fhi), _int(int(normalize)), _int(dilate), _int(int(rgb8)),
                                  out.ctypes.data_as(_vp), ptr(mm))
        return out, (float(mm[0]), float(mm[1]))

    def export_normal(self, w, h, idx, data3, dilate=0):
        idx = np.ascontiguousarray(idx, np.uint32)
        data3 = np.ascontiguousarray(data3, np.float32)
        out = np.zeros((h, w, 3), np.uint8)
        self.lib.orc_export_normal(_u32(w), _u32(h), _u32(len(idx)), ptr(idx, _u32p), ptr(data3), _int(dilate),
                                   out.ctypes.data_as(_vp))
        return out

    def export_vector(self, w, h, idx, data3):
        """3 x h x w float32: planes B (z), G (y), R (x)."""
        idx = np.ascontiguousarray(idx, np.uint32)
        data3 = np.ascontiguousarray(data3, np.float32)
        out = np.zeros((3, h, w), np.float32)
        self.lib.orc_export_vector(_u32(w), _u32(h), _u32(len(idx)), ptr(idx, _u32p), ptr(data3), ptr(out))
        return out


class Reference:
    """The reference's own sources compiled on the host (oracle/_ref)."""

    def __init__(self, path=None):
        path = path or build_ref()
        if not path or not os.path.exists(path):
            raise OSError("oracle/_ref/libfornos_ref.so is not built (reference tree absent)")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_scene_build.restype = _vp
        L.ref_raster.restype = _vp
        L.ref_mesh_load.restype = _vp
        L.ref_mesh_load.argtypes = [ctypes.c_char_p]
        L.ref_mesh_sizes.argtypes = [_vp, ctypes.POINTER(ctypes.c_uint64)]
        L.ref_mesh_arrays.argtypes = [_vp] + [_vp] * 5
        L.ref_mesh_free.argtypes = [_vp]

    def load_mesh(self, path):
        """Mesh::loadFile (Src/mesh.cpp:612-617): the loaded arrays as
        (positions, texcoords, normals, vertices, triangles), or None when the
        loader returns null.  Never call it on a PLY file without s / t or
        without normals: the reference's loader dereferences a null buffer
        there."""
        h = self.lib.ref_mesh_load(os.fsencode(path))
        if not h:
            return None
        n = (ctypes.c_uint64 * 5)()
        self.lib.ref_mesh_sizes(h, n)
        arrs = [np.zeros((n[0], 3), np.float32), np.zeros((n[1], 2), np.float32), np.zeros((n[2], 3), np.float32),
                np.zeros((n[3], 3), np.uint32), np.zeros((n[4], 3), np.uint32)]
        self.lib.ref_mesh_arrays(h, *[a.ctypes.data_as(_vp) for a in arrs])
        self.lib.ref_mesh_free(h)
        return tuple(arrs)

    def normals(self, m, which):
        code = {"face": 0, "vertex": 1, "welded": 2}[which]
        vtx = np.zeros_like(m.vertices)
        nrm = np.zeros((max(3 * m.triangle_count, len(m.positions)) + 1, 3), np.float32)
        n = self.lib.ref_normals(_int(code), _u32(len(m.positions)), ptr(m.positions), _u32(len(m.vertices)),
                                 ptr(m.vertices, _u32p), _u32(m.triangle_count), ptr(m.triangles, _u32p),
                                 ptr(vtx, _u32p), ptr(nrm))
        return vtx, nrm[:n].copy()

    def tangent_space(self, m):
        t = np.zeros((len(m.vertices), 3), np.float32)
        b = np.zeros_like(t)
        self.lib.ref_tangent_space(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.texcoords)),
                                   ptr(m.texcoords), _u32(len(m.normals)), ptr(m.normals), _u32(len(m.vertices)),
                                   ptr(m.vertices, _u32p), _u32(m.triangle_count), ptr(m.triangles, _u32p),
                                   ptr(t), ptr(b))
        return t, b

    def scene(self, m, max_tris=8, max_depth=8192):
        h = self.lib.ref_scene_build(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.normals)),
                                     ptr(m.normals), _u32(len(m.vertices)), ptr(m.vertices, _u32p),
                                     _u32(m.triangle_count), ptr(m.triangles, _u32p), _u32(max_tris),
                                     _u32(max_depth))
        nn, nc = _u32(), _u32()
        self.lib.ref_scene_sizes(_vp(h), ctypes.byref(nn), ctypes.byref(nc))
        nodes = np.zeros(nn.value, NODE_DTYPE)
        pos4 = np.zeros((nc.value, 4), np.float32)
        nrm4 = np.zeros((nc.value, 4), np.float32)
        self.lib.ref_scene_copy(_vp(h), nodes.ctypes.data_as(_vp), ptr(pos4), ptr(nrm4))
        self.lib.ref_scene_free(_vp(h))
        return nodes, pos4, nrm4

    def raster(self, m, w, h, mode=0, dirs=None, edge=0.05):
        dv, dn = (None, None) if dirs is None else dirs
        hm = self.lib.ref_raster(_u32(len(m.positions)), ptr(m.positions), _u32(len(m.texcoords)), ptr(m.texcoords),
                                 _u32(len(m.normals)), ptr(m.normals), _u32(len(m.vertices)), ptr(m.vertices, _u32p),
                                 _u32(m.triangle_count), ptr(m.triangles, _u32p), ptr(m.tangents),
                                 ptr(m.bitangents), ptr(dv, _u32p), _u32(0 if dn is None else len(dn)), ptr(dn),
                                 _u32(w), _u32(h), _int(mode), _f32(edge))
        if not hm:
            return None
        c = _u32()
        self.lib.ref_cmap_copy(_vp(hm), ctypes.byref(c), None, None, None, None, None, None)
        n = c.value
        out = {k: np.zeros((n, 3), np.float32) for k in ("positions", "directions", "normals", "tangents",
                                                          "bitangents")}
        out["indices"] = np.zeros(n, np.uint32)
        self.lib.ref_cmap_copy(_vp(hm), ctypes.byref(c), ptr(out["indices"], _u32p), ptr(out["positions"]),
                               ptr(out["directions"]), ptr(out["normals"]), ptr(out["tangents"]),
                               ptr(out["bitangents"]))
        self.lib.ref_cmap_free(_vp(hm))
        return out

    def samples(self, spp, perms=4096, seed=0):
        out = np.zeros((perms * spp, 4), np.float32)
        self.lib.ref_samples(_u32(spp), _u32(perms), _u32(seed), ptr(out))
        return out

    def meshmap(self, nodes, pos4, pix8, cull=True):
        n = pix8.shape[0]
        coords = np.zeros((n, 4), np.float32)
        tidx = np.zeros(n, np.uint32)
        self.lib.ref_shader_meshmap(_int(int(cull)), ptr(pix8), ptr(pos4), nodes.ctypes.data_as(_vp),
                                    _u32(len(nodes)), _u32(n), ptr(coords), ptr(tidx, _u32p))
        return coords, tidx

    def hemisphere(self, kind, nodes, pos4, nrm4, coords, tidx, samples4, spp, min_d, max_d, texels=None,
                   perms=4096):
        """Reference shaders for the listed texels (all when None); one row per
        listed texel."""
        n = len(tidx) if texels is None else len(texels)
        out = np.zeros((n, 3) if kind == 1 else n, np.float32)
        tx = None if texels is None else np.ascontiguousarray(texels, np.uint32)
        self.lib.ref_shader_hemisphere(_int(kind), nodes.ctypes.data_as(_vp), _u32(len(nodes)), ptr(pos4), ptr(nrm4),
                                       ptr(coords), ptr(tidx, _u32p), ptr(samples4), _u32(spp), _u32(perms),
                                       _f32(min_d), _f32(max_d), ptr(tx, _u32p), _u32(n), ptr(out))
        return out

    def gather(self, what, pos4, nrm4, coords, tidx):
        n = len(tidx)
        out = np.zeros(n if what == 0 else (n, 3), np.float32)
        self.lib.ref_shader_gather(_int(what), ptr(pos4), ptr(nrm4), ptr(coords), ptr(tidx, _u32p), _u32(n), ptr(out))
        return out

    def tangent_transform(self, n3, t3, b3, v3):
        n = len(v3)
        pixt = np.zeros((n, 12), np.float32)
        pixt[:, 0:3], pixt[:, 4:7], pixt[:, 8:11] = n3, t3, b3
        io = np.ascontiguousarray(v3, np.float32).copy()
        self.lib.ref_shader_tangentspace(ptr(pixt), _u32(n), ptr(io))
        return io

    # ---- image export: the reference writes the file (extension picks the format)
    def export_float(self, path, w, h, idx, data, flo=0.0, fhi=0.0, normalize=True, dilate=0):
        idx = np.ascontiguousarray(idx, np.uint32)
        data = np.ascontiguousarray(data, np.float32)
        mm = np.zeros(2, np.float32)
        rc = self.lib.ref_export_float(_u32(w), _u32(h), _u32(len(idx)), ptr(idx, _u32p), ptr(data),
                                       ctypes.c_char_p(path.encode()), ctypes.c_float(flo), ctypes.c_float(fhi),
                                       _int(int(normalize)), _int(dilate), ptr(mm))
        assert rc == 0
        return float(mm[0]), float(mm[1])

    def export_normal(self, path, w, h, idx, data3, dilate=0):
        idx = np.ascontiguousarray(idx, np.uint32)
        data3 = np.ascontiguousarray(data3, np.float32)
        assert self.lib.ref_export_normal(_u32(w), _u32(h), _u32(len(idx)), ptr(idx, _u32p), ptr(data3),
                                          ctypes.c_char_p(path.encode()), _int(dilate)) == 0

    def export_vector(self, path, w, h, idx, data3):
        idx = np.ascontiguousarray(idx, np.uint32)
        data3 = np.ascontiguousarray(data3, np.float32)
        assert self.lib.ref_export_vector(_u32(w), _u32(h), _u32(len(idx)), ptr(idx, _u32p), ptr(data3),
                                          ctypes.c_char_p(path.encode())) == 0


def pixels8(positions, directions):
    """Pix_GPUData rows (Src/meshmapping.h:15-20): p.xyz, pad, d.xyz, pad."""
    n = len(positions)
    out = np.zeros((n, 8), np.float32)
    out[:, 0:3] = positions
    out[:, 4:7] = directions
    return out
