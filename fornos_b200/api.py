"""Python front-end of the bake path, over the C ABI (include/fornos_gpu.h).

Names follow the reference's host API: Mesh (Src/mesh.h), BVH.create_binary
(Src/bvh.h), TexelMap = MapUV + CompressedMapUV (Src/compute.h), MeshMapping
(Src/meshmapping.h) and the six solvers (Src/solver_*.h) with init /
run_step / get_results / progress.  Mesh.load is Mesh::loadFile (OBJ / PLY).
FornosRunner::start + run (Src/fornos.cpp:53-251) is run(ctx, **fields),
with the fields of FornosParameters (Src/fornos.h:35-123): mesh files in,
image files out (fk_run); bake() is the same bake from host arrays.
"""
import ctypes
import os

import numpy as np

from . import _lib as L
from .workloads import MeshArrays

OK = 0
MISS = 0xFFFFFFFF
FLT_MAX = float(np.finfo(np.float32).max)

# kinds (include/fornos_gpu.h)
AO, BN, THICK, AO_BN = 0, 1, 2, 3
TRAVERSE_AUTO, TRAVERSE_ORDERED, TRAVERSE_SKIP, TRAVERSE_ORDERED4 = 0, 1, 2, 3
TREE_REFERENCE, TREE_SAH = 0, 1
NORMALS_FACE, NORMALS_VERTEX, NORMALS_WELDED = 0, 1, 2
SCHEDULE_STATIC, SCHEDULE_DYNAMIC = 0x10, 0x20  # or-ed into `traverse`
EXACT_BOX_TESTS = 0x100  # or-ed into `traverse`: divide in every box test
GATHER_HEIGHT, GATHER_POSITION, GATHER_NORMAL = 0, 1, 2
MAP_SMOOTH, MAP_LOWPOLY_NORMALS, MAP_HYBRID = 0, 1, 2
SOLVER_HEIGHT, SOLVER_POSITION, SOLVER_NORMALS, SOLVER_AO, SOLVER_BENT_NORMALS, SOLVER_THICKNESS = range(6)
PERMS = 4096  # k_samplePermCount (Src/solver_ao.cpp:34)

NODE_DTYPE = np.dtype([("lo", np.float32, 3), ("hi", np.float32, 3), ("start", np.uint32), ("end", np.uint32),
                       ("jump", np.uint32)])


class FornosError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("fornos error %d: %s" % (code, msg))
        self.code = code


def _f32(a):
    return a.ctypes.data_as(L.f32p)


def _u32(a):
    return a.ctypes.data_as(L.u32p)


def _check(rc, ctx=None, what=""):
    if rc != OK:
        msg = what
        if ctx is not None and ctx.handle:
            msg = (what + ": " if what else "") + L.load().fk_last_error(ctx.handle).decode()
        raise FornosError(rc, msg)


def _tuning_dict(t):
    return {name: int(getattr(t, name)) for name, _ in L.Tuning._fields_}


# ------------------------------------------------------------------ context
class Context:
    """One device context (fk_ctx); device work runs on its stream."""

    def __init__(self, device=0):
        self.lib = L.load()
        h = L.c_vp()
        rc = self.lib.fk_ctx_create(device, ctypes.byref(h))
        if rc != OK:
            raise FornosError(rc, "fk_ctx_create(%d) failed (needs a compute capability 10.x GPU)" % device)
        self.handle = h.value

    def close(self):
        if self.handle:
            self.lib.fk_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, cuda_stream_ptr):
        _check(self.lib.fk_ctx_set_stream(self.handle, cuda_stream_ptr), self)

    def sync(self):
        _check(self.lib.fk_sync(self.handle), self)

    def trim(self):
        """Release the context pool's unused device memory (fk_ctx_trim)."""
        _check(self.lib.fk_ctx_trim(self.handle), self)

    def check(self):
        """Waits for the stream; raises FornosError when a kernel flagged an
        error since the last check (fk_ctx_check)."""
        _check(self.lib.fk_ctx_check(self.handle), self, "fk_ctx_check")

    @property
    def launches(self):
        return int(self.lib.fk_launch_count(self.handle))

    def set_tuning(self, **knobs):
        """fk_ctx_set_tuning: the given knobs (fk_tuning field names), the
        others as they are now."""
        t = L.Tuning(**dict(self.get_tuning(), **knobs))
        _check(self.lib.fk_ctx_set_tuning(self.handle, ctypes.byref(t)), self, "fk_ctx_set_tuning")

    def get_tuning(self):
        t = L.Tuning()
        _check(self.lib.fk_ctx_get_tuning(self.handle, ctypes.byref(t)), self)
        return _tuning_dict(t)

    def buffer(self, nbytes):
        return Buffer(self, nbytes)

    def upload(self, arr):
        arr = np.ascontiguousarray(arr)
        b = Buffer(self, max(arr.nbytes, 4))
        b.upload(arr)
        return b


class Buffer:
    """Device allocation (fk_buf), zero-filled on creation."""

    def __init__(self, ctx, nbytes):
        self.ctx = ctx
        h = L.c_vp()
        _check(ctx.lib.fk_buf_alloc(ctx.handle, nbytes, ctypes.byref(h)), ctx, "fk_buf_alloc")
        self.handle = h.value
        self.nbytes = nbytes
        self.owned = True

    @classmethod
    def borrowed(cls, ctx, handle):
        b = cls.__new__(cls)
        b.ctx, b.handle, b.owned = ctx, handle, False
        b.nbytes = ctx.lib.fk_buf_size(handle)
        return b

    def upload(self, arr, offset=0):
        arr = np.ascontiguousarray(arr)
        _check(self.ctx.lib.fk_buf_upload(self.ctx.handle, self.handle, offset, arr.ctypes.data, arr.nbytes), self.ctx)

    def download(self, dtype, shape, offset=0):
        out = np.empty(shape, dtype)
        _check(self.ctx.lib.fk_buf_download(self.ctx.handle, self.handle, offset, out.ctypes.data, out.nbytes), self.ctx)
        return out

    @property
    def device_ptr(self):
        return self.ctx.lib.fk_buf_device_ptr(self.handle)

    def free(self):
        if self.owned and self.handle and self.ctx.handle:
            self.ctx.lib.fk_buf_free(self.ctx.handle, self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ------------------------------------------------------------------ mesh / BVH
class Mesh:
    """Host indexed mesh (fk_mesh, Src/mesh.h:35-63)."""

    def __init__(self, arrays=None, handle=None):
        self.lib = L.load()
        if handle is not None:
            self.handle = handle
            return
        a = arrays
        self._keep = [a.positions, a.texcoords, a.normals, a.vertices, a.triangles, a.tangents, a.bitangents]
        d = L.MeshDesc(len(a.positions), _f32(a.positions), len(a.texcoords), _f32(a.texcoords), len(a.normals),
                       _f32(a.normals), len(a.vertices), _u32(a.vertices), a.triangle_count, _u32(a.triangles),
                       _f32(a.tangents) if a.tangents is not None else None,
                       _f32(a.bitangents) if a.bitangents is not None else None)
        h = L.c_vp()
        _check(self.lib.fk_mesh_create(ctypes.byref(d), ctypes.byref(h)), None, "fk_mesh_create: invalid mesh")
        self.handle = h.value
        self._keep = None

    def __del__(self):
        try:
            if self.handle:
                self.lib.fk_mesh_free(self.handle)
        except Exception:
            pass

    @classmethod
    def load(cls, path):
        """Mesh::loadFile: an .obj or .ply file as the reference's loader reads it."""
        h = L.c_vp()
        _check(L.load().fk_mesh_load(os.fsencode(path), ctypes.byref(h)), what="fk_mesh_load(%s)" % path)
        return cls(handle=h.value)

    def copy(self):
        h = L.c_vp()
        _check(self.lib.fk_mesh_copy(self.handle, ctypes.byref(h)))
        return Mesh(handle=h.value)

    def compute_face_normals(self):
        _check(self.lib.fk_mesh_compute_face_normals(self.handle))

    def compute_vertex_normals(self):
        _check(self.lib.fk_mesh_compute_vertex_normals(self.handle))

    def compute_vertex_normals_aggressive(self):
        _check(self.lib.fk_mesh_compute_vertex_normals_welded(self.handle))

    def compute_tangent_space(self):
        _check(self.lib.fk_mesh_compute_tangent_space(self.handle))

    def compute_normals_device(self, ctx, method):
        """The normal generator `method` (NORMALS_FACE / NORMALS_VERTEX /
        NORMALS_WELDED) run on the device; the mesh ends as the host
        generator leaves it."""
        _check(self.lib.fk_mesh_compute_normals_device(ctx.handle, self.handle, int(method)), ctx)

    def compute_tangent_space_device(self, ctx):
        _check(self.lib.fk_mesh_compute_tangent_space_device(ctx.handle, self.handle), ctx)

    def arrays(self):
        d = L.MeshDesc()
        _check(self.lib.fk_mesh_describe(self.handle, ctypes.byref(d)))

        def grab(p, n, w, dt):
            if n == 0 or not p:
                return np.zeros((0, w), dt)
            return np.ctypeslib.as_array(p, shape=(n * w,)).reshape(n, w).astype(dt, copy=True)

        tan = grab(d.tangents, d.vertex_count, 3, np.float32) if d.tangents else None
        bit = grab(d.bitangents, d.vertex_count, 3, np.float32) if d.bitangents else None
        return MeshArrays(grab(d.positions, d.position_count, 3, np.float32),
                          grab(d.texcoords, d.texcoord_count, 2, np.float32),
                          grab(d.normals, d.normal_count, 3, np.float32),
                          grab(d.vertices, d.vertex_count, 3, np.uint32),
                          grab(d.triangles, d.triangle_count, 3, np.uint32), tan, bit)


class BVH:
    """Host BVH (fk_bvh): BVH::createBinary (Src/bvh.cpp:283-314)."""

    def __init__(self, handle):
        self.lib = L.load()
        self.handle = handle

    @classmethod
    def create_binary(cls, mesh, max_triangle_count=8, max_tree_depth=8192):
        h = L.c_vp()
        _check(L.load().fk_bvh_build(mesh.handle, max_triangle_count, max_tree_depth, ctypes.byref(h)))
        return cls(h.value)

    def flatten(self, mesh):
        """fillMeshData (Src/meshmapping.cpp:62-125): (nodes, positions4, normals4)."""
        nn, nc = L.c_u32(), L.c_u32()
        _check(self.lib.fk_bvh_flatten_sizes(self.handle, ctypes.byref(nn), ctypes.byref(nc)))
        nodes = np.zeros(nn.value, NODE_DTYPE)
        pos4 = np.zeros((nc.value, 4), np.float32)
        nrm4 = np.zeros((nc.value, 4), np.float32)
        _check(self.lib.fk_bvh_flatten(self.handle, mesh.handle, nodes.ctypes.data, _f32(pos4), _f32(nrm4)))
        return nodes, pos4, nrm4

    def __del__(self):
        try:
            if self.handle:
                self.lib.fk_bvh_free(self.handle)
        except Exception:
            pass

    @staticmethod
    def build_flat_device(ctx, mesh, max_triangle_count=8, max_tree_depth=8192):
        """createBinary + fillMeshData on the device (fk_bvh_build_flat):
        (nodes, positions4, normals4), equal to create_binary(...).flatten(mesh)."""
        nf = mesh.arrays().triangle_count
        nodes = np.zeros(max(2 * nf - 1, 1), NODE_DTYPE)
        pos4 = np.zeros((3 * nf, 4), np.float32)
        nrm4 = np.zeros((3 * nf, 4), np.float32)
        nn = L.c_u32()
        _check(ctx.lib.fk_bvh_build_flat(ctx.handle, mesh.handle, max_triangle_count, max_tree_depth, nodes.ctypes.data,
                                         len(nodes), ctypes.byref(nn), _f32(pos4), _f32(nrm4)), ctx,
               "fk_bvh_build_flat")
        return nodes[:nn.value].copy(), pos4, nrm4


class Scene:
    """High-poly mesh + BVH resident on the device (fk_scene)."""

    def __init__(self, ctx, nodes, pos4, nrm4):
        self.ctx = ctx
        nodes = np.ascontiguousarray(nodes)
        pos4 = np.ascontiguousarray(pos4, np.float32)
        nrm4 = np.ascontiguousarray(nrm4, np.float32)
        h = L.c_vp()
        _check(ctx.lib.fk_scene_upload(ctx.handle, nodes.ctypes.data, len(nodes), _f32(pos4), _f32(nrm4), len(pos4),
                                       ctypes.byref(h)), ctx, "fk_scene_upload")
        self.handle = h.value
        self.owned = True

    @classmethod
    def borrowed(cls, ctx, handle):
        s = cls.__new__(cls)
        s.ctx, s.handle, s.owned = ctx, handle, False
        return s

    @classmethod
    def build(cls, ctx, mesh, max_triangle_count=8, max_tree_depth=8192):
        """BVH built on the device straight into a scene (fk_scene_build)."""
        h = L.c_vp()
        _check(ctx.lib.fk_scene_build(ctx.handle, mesh.handle, max_triangle_count, max_tree_depth, ctypes.byref(h)),
               ctx, "fk_scene_build")
        s = cls.__new__(cls)
        s.ctx, s.handle, s.owned = ctx, h.value, True
        return s

    def info(self):
        i = L.SceneInfo()
        _check(self.ctx.lib.fk_scene_get_info(self.handle, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in L.SceneInfo._fields_}

    def set_tree(self, tree):
        """Inner tree of the ordered traversals: TREE_REFERENCE or TREE_SAH."""
        _check(self.ctx.lib.fk_scene_set_tree(self.handle, tree), self.ctx, "fk_scene_set_tree")

    def tree(self, tree):
        """(records, depth) of an inner tree as resident on the device
        (fk_diag_scene_tree): records is (count, 16) float32, count 0 when that
        tree was not built."""
        n, d = L.c_u32(), L.c_u32()
        _check(self.ctx.lib.fk_diag_scene_tree(self.ctx.handle, self.handle, tree, None, 0, ctypes.byref(n),
                                               ctypes.byref(d)), self.ctx, "fk_diag_scene_tree")
        out = np.zeros((n.value, 16), np.float32)
        if n.value:
            _check(self.ctx.lib.fk_diag_scene_tree(self.ctx.handle, self.handle, tree, _f32(out), n.value,
                                                   ctypes.byref(n), ctypes.byref(d)), self.ctx, "fk_diag_scene_tree")
        return out, d.value

    def free(self):
        if self.owned and self.handle and self.ctx.handle:
            self.ctx.lib.fk_scene_free(self.ctx.handle, self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class TexelMap:
    """Compressed texel map on the device: MapUV::from* + CompressedMapUV."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.handle = handle
        w, h, c = L.c_u32(), L.c_u32(), L.c_u32()
        _check(ctx.lib.fk_texel_map_info(handle, ctypes.byref(w), ctypes.byref(h), ctypes.byref(c)))
        self.width, self.height, self.count = w.value, h.value, c.value

    @classmethod
    def rasterize(cls, ctx, mesh, width, height, mode=MAP_SMOOTH, dirs=None, edge=0.05):
        h = L.c_vp()
        _check(ctx.lib.fk_raster_uv(ctx.handle, mesh.handle, dirs.handle if dirs is not None else None, width, height,
                                    mode, edge, ctypes.byref(h)), ctx, "fk_raster_uv")
        return cls(ctx, h.value)

    @classmethod
    def from_mesh(cls, ctx, mesh, width, height):
        return cls.rasterize(ctx, mesh, width, height, MAP_LOWPOLY_NORMALS)

    @classmethod
    def from_meshes(cls, ctx, mesh, mesh_dirs, width, height):
        return cls.rasterize(ctx, mesh, width, height, MAP_SMOOTH, mesh_dirs)

    @classmethod
    def from_meshes_hybrid(cls, ctx, mesh, mesh_dirs, width, height, edge):
        return cls.rasterize(ctx, mesh, width, height, MAP_HYBRID, mesh_dirs, edge)

    @classmethod
    def from_host(cls, ctx, width, height, pix8, pixt12, indices):
        pix8 = np.ascontiguousarray(pix8, np.float32)
        pixt12 = np.ascontiguousarray(pixt12, np.float32)
        indices = np.ascontiguousarray(indices, np.uint32)
        h = L.c_vp()
        _check(ctx.lib.fk_texel_map_from_host(ctx.handle, width, height, len(indices), _f32(pix8), _f32(pixt12),
                                              _u32(indices), ctypes.byref(h)), ctx, "fk_texel_map_from_host")
        return cls(ctx, h.value)

    def download(self):
        n = self.count
        pix = np.zeros((n, 8), np.float32)
        pixt = np.zeros((n, 12), np.float32)
        idx = np.zeros(n, np.uint32)
        _check(self.ctx.lib.fk_texel_map_download(self.ctx.handle, self.handle, _f32(pix), _f32(pixt), _u32(idx)), self.ctx)
        return {"positions": pix[:, 0:3].copy(), "directions": pix[:, 4:7].copy(), "normals": pixt[:, 0:3].copy(),
                "tangents": pixt[:, 4:7].copy(), "bitangents": pixt[:, 8:11].copy(), "indices": idx}

    def free(self):
        if self.handle and self.ctx.handle:
            self.ctx.lib.fk_texel_map_free(self.ctx.handle, self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


EXPORT_FLOAT_RGB8, EXPORT_FLOAT_F32, EXPORT_NORMAL_RGB8, EXPORT_VECTOR_F32 = 0, 1, 2, 3


def export_image(ctx, tmap, data, mode, filter_range=(0.0, 0.0), normalize=True, dilate=0):
    """Image export of Src/image.cpp:22-405 on the device (fk_export_image):
    `data` holds 1 float per texel (FLOAT modes) or 3 (NORMAL / VECTOR), in the
    map's order.  Returns (image, (min, max)): h x w x 3 uint8 for the RGB8
    modes, h x w float32 (FLOAT_F32) or 3 x h x w float32 (VECTOR_F32, planes B,
    G, R), rows as written to the file; (min, max) for the FLOAT modes."""
    w, h = tmap.width, tmap.height
    shape, dt = {EXPORT_FLOAT_RGB8: ((h, w, 3), np.uint8), EXPORT_NORMAL_RGB8: ((h, w, 3), np.uint8),
                 EXPORT_FLOAT_F32: ((h, w), np.float32), EXPORT_VECTOR_F32: ((3, h, w), np.float32)}[mode]
    img = ctx.buffer(int(np.prod(shape)) * np.dtype(dt).itemsize)
    p = L.ExportParams(mode, filter_range[0], filter_range[1], int(normalize), dilate)
    mm = np.zeros(2, np.float32)
    _check(ctx.lib.fk_export_image(ctx.handle, tmap.handle, data.handle, ctypes.byref(p), img.handle, _f32(mm)), ctx,
           "fk_export_image")
    out = img.download(dt, shape)
    img.free()
    return out, (float(mm[0]), float(mm[1]))


def write_image(path, image, png_level=None):
    """Writes an exported image: h x w x 3 uint8 as .png (filtered and deflated;
    png_level 0-9 picks the zlib level, 0 = stored) / .tga (run-length coded),
    h x w or 3 x h x w float32 as .exr (HALF channels B, or B, G, R)."""
    image = np.ascontiguousarray(image)
    lib = L.load()
    if image.dtype == np.uint8:
        h, w, _ = image.shape
        if png_level is not None and path.endswith(".png"):
            _check(lib.fk_image_write_png(path.encode(), w, h, image.ctypes.data, int(png_level)))
        else:
            _check(lib.fk_image_write_rgb8(path.encode(), w, h, image.ctypes.data))
    else:
        planes = np.ascontiguousarray(image.astype(np.float32).reshape(-1, *image.shape[-2:]))
        _check(lib.fk_image_write_exr(path.encode(), planes.shape[2], planes.shape[1], planes.shape[0],
                                      _f32(planes)))


def sah_tree_host(nodes):
    """(records, depth) of the surface-area inner tree computed on the host
    (fk_diag_sah_host), the records fk_scene_upload builds on the device."""
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    lib = L.load()
    n, d = L.c_u32(), L.c_u32()
    _check(lib.fk_diag_sah_host(nodes.ctypes.data, len(nodes), None, 0, ctypes.byref(n), ctypes.byref(d)))
    out = np.zeros((n.value, 16), np.float32)
    if n.value:
        _check(lib.fk_diag_sah_host(nodes.ctypes.data, len(nodes), _f32(out), n.value, ctypes.byref(n),
                                    ctypes.byref(d)))
    return out, d.value


def samples_cosine(spp, perms=PERMS, seed=0):
    """computeSamplesImportanceCosDir (Src/math.h:363-382), seeded."""
    out = np.zeros((perms * spp, 4), np.float32)
    _check(L.load().fk_samples_cosine(spp, perms, seed, _f32(out)))
    return out


# ------------------------------------------------------------------ kernels
def meshmap(ctx, scene, tmap, cull_backfaces, coords, tidx, offset=0, count=None, max_dist=FLT_MAX):
    """fk_meshmap: the mapping shaders over texels [offset, offset + count).
    max_dist is the walks' initial closest distance (FLT_MAX reproduces the
    reference); hits at or beyond it are not taken."""
    count = tmap.count - offset if count is None else count
    _check(ctx.lib.fk_meshmap(ctx.handle, scene.handle, tmap.handle, int(cull_backfaces), max_dist, offset, count,
                              coords.handle, tidx.handle), ctx, "fk_meshmap")


def hemisphere(ctx, scene, coords, tidx, kind, spp, min_d, max_d, samples, out0, out1=None, hits0=None, hits1=None,
               offset=0, count=0, perms=PERMS, traverse=TRAVERSE_AUTO):
    p = L.SampleParams(spp, perms, min_d, max_d)
    hv = lambda b: b.handle if b is not None else None
    _check(ctx.lib.fk_hemisphere(ctx.handle, scene.handle, coords.handle, tidx.handle, kind, ctypes.byref(p),
                                 samples.handle, offset, count, traverse, out0.handle, hv(out1), hv(hits0), hv(hits1)),
           ctx, "fk_hemisphere")


def hemisphere_texels(ctx, scene, coords, tidx, texel_count, kind, spp, min_d, max_d, samples, ids, out0, out1=None,
                      hits0=None, hits1=None, offset=0, count=None, perms=PERMS, traverse=TRAVERSE_AUTO):
    """fk_hemisphere over the texels listed in `ids` (u32 buffer); each listed
    texel gets exactly the value a whole-map pass gives it."""
    count = ids.nbytes // 4 - offset if count is None else count
    p = L.SampleParams(spp, perms, min_d, max_d)
    hv = lambda b: b.handle if b is not None else None
    _check(ctx.lib.fk_hemisphere_texels(ctx.handle, scene.handle, coords.handle, tidx.handle, texel_count, kind,
                                        ctypes.byref(p), samples.handle, ids.handle, offset, count, traverse,
                                        out0.handle, hv(out1), hv(hits0), hv(hits1)), ctx, "fk_hemisphere_texels")


def gather(ctx, scene, kind, coords, tidx, out, offset=0, count=0):
    _check(ctx.lib.fk_gather(ctx.handle, scene.handle, kind, coords.handle, tidx.handle, offset, count, out.handle),
           ctx, "fk_gather")


def tangent_space(ctx, tmap, io3, offset=0, count=None):
    count = tmap.count - offset if count is None else count
    _check(ctx.lib.fk_tangent_space(ctx.handle, tmap.handle, offset, count, io3.handle), ctx, "fk_tangent_space")


# ------------------------------------------------------------------ solvers
class MeshMapping:
    """MeshMapping (Src/meshmapping.h:42-75)."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = L.c_vp()
        _check(ctx.lib.fk_meshmapping_create(ctx.handle, ctypes.byref(h)), ctx)
        self.handle = h.value

    def init(self, tmap, mesh, bvh, cull_backfaces=True):
        _check(self.ctx.lib.fk_meshmapping_init(self.handle, tmap.handle, mesh.handle, bvh.handle, int(cull_backfaces)),
               self.ctx, "MeshMapping.init")
        self.tmap = tmap

    def init_scene(self, tmap, scene, cull_backfaces=True):
        _check(self.ctx.lib.fk_meshmapping_init_scene(self.handle, tmap.handle, scene.handle, int(cull_backfaces)),
               self.ctx, "MeshMapping.init")
        self.tmap = tmap

    def set_work_per_step(self, texels):
        _check(self.ctx.lib.fk_meshmapping_set_work_per_step(self.handle, texels))

    def run_step(self):
        done = L.c_int()
        _check(self.ctx.lib.fk_meshmapping_run_step(self.handle, ctypes.byref(done)), self.ctx, "MeshMapping.runStep")
        return bool(done.value)

    def run(self):
        while not self.run_step():
            pass

    def progress(self):
        return float(self.ctx.lib.fk_meshmapping_progress(self.handle))

    def results(self):
        n = (self.tmap.count + 63) // 64 * 64 or 64
        coords = np.zeros((n, 4), np.float32)
        tidx = np.zeros(n, np.uint32)
        _check(self.ctx.lib.fk_meshmapping_results(self.handle, _f32(coords), _u32(tidx)), self.ctx)
        return coords, tidx

    @property
    def coords(self):
        return Buffer.borrowed(self.ctx, self.ctx.lib.fk_meshmapping_coords(self.handle))

    @property
    def coords_tidx(self):
        return Buffer.borrowed(self.ctx, self.ctx.lib.fk_meshmapping_tidx(self.handle))

    @property
    def scene(self):
        return Scene.borrowed(self.ctx, self.ctx.lib.fk_meshmapping_scene(self.handle))

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                self.ctx.lib.fk_meshmapping_free(self.handle)
        except Exception:
            pass


class _Solver:
    KIND = None
    WIDTH = 1

    def __init__(self, ctx, sample_count=0, min_distance=0.0, max_distance=0.0, tangent_space=False,
                 normalize_output=False, seed=0, traverse=TRAVERSE_AUTO):
        self.ctx = ctx
        p = L.SolverParams(self.KIND, sample_count, min_distance, max_distance, int(tangent_space),
                           int(normalize_output), seed, traverse)
        h = L.c_vp()
        _check(ctx.lib.fk_solver_create(ctx.handle, ctypes.byref(p), ctypes.byref(h)), ctx, "solver create")
        self.handle = h.value

    def init(self, tmap, mesh_mapping):
        _check(self.ctx.lib.fk_solver_init(self.handle, tmap.handle, mesh_mapping.handle), self.ctx, "solver init")
        self.tmap = tmap

    def set_work_per_step(self, texels):
        _check(self.ctx.lib.fk_solver_set_work_per_step(self.handle, texels))

    def run_step(self):
        done = L.c_int()
        _check(self.ctx.lib.fk_solver_run_step(self.handle, ctypes.byref(done)), self.ctx, "solver runStep")
        return bool(done.value)

    def run(self):
        while not self.run_step():
            pass

    def progress(self):
        return float(self.ctx.lib.fk_solver_progress(self.handle))

    def get_results(self):
        n = int(self.ctx.lib.fk_solver_result_count(self.handle))
        out = np.zeros(n, np.float32)
        _check(self.ctx.lib.fk_solver_results(self.handle, _f32(out), n), self.ctx, "getResults")
        return out.reshape(-1, 3) if self.WIDTH == 3 else out

    def hits(self):
        n = int(self.ctx.lib.fk_solver_result_count(self.handle)) // self.WIDTH
        out = np.zeros(n, np.uint32)
        _check(self.ctx.lib.fk_solver_hits(self.handle, _u32(out), n), self.ctx, "hits")
        return out

    @property
    def result_buffer(self):
        return Buffer.borrowed(self.ctx, self.ctx.lib.fk_solver_result_buffer(self.handle))

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                self.ctx.lib.fk_solver_free(self.handle)
        except Exception:
            pass


class HeightSolver(_Solver):
    KIND = SOLVER_HEIGHT

    def __init__(self, ctx, normalize_output=True, max_distance=0.0):
        super().__init__(ctx, max_distance=max_distance, normalize_output=normalize_output)


class PositionSolver(_Solver):
    KIND = SOLVER_POSITION
    WIDTH = 3

    def __init__(self, ctx):
        super().__init__(ctx)


class NormalsSolver(_Solver):
    KIND = SOLVER_NORMALS
    WIDTH = 3

    def __init__(self, ctx, tangent_space=True):
        super().__init__(ctx, tangent_space=tangent_space)


class AmbientOcclusionSolver(_Solver):
    KIND = SOLVER_AO


class BentNormalsSolver(_Solver):
    KIND = SOLVER_BENT_NORMALS
    WIDTH = 3


class ThicknessSolver(_Solver):
    KIND = SOLVER_THICKNESS


# ------------------------------------------------------------------ runner
def fp32_peak(ctx):
    """Measured FP32 add/mul/min instruction throughput (ops/s) of the device."""
    v = ctypes.c_double()
    _check(ctx.lib.fk_diag_fp32_peak(ctx.handle, ctypes.byref(v)), ctx, "fk_diag_fp32_peak")
    return v.value


def traversal_counts(ctx, scene, coords, tidx, kind, spp, min_d, max_d, samples, offset=0, count=0, perms=PERMS,
                     traverse=TRAVERSE_AUTO):
    """Box and triangle tests the GPU traversal executes for these rays."""
    p = L.SampleParams(spp, perms, min_d, max_d)
    out = (L.c_u64 * 2)()
    _check(ctx.lib.fk_diag_traversal_counts(ctx.handle, scene.handle, coords.handle, tidx.handle, kind, ctypes.byref(p),
                                            samples.handle, offset, count, traverse, out), ctx, "traversal counts")
    return int(out[0]), int(out[1])


PROFILE_KEYS = ("box_tests", "tri_tests", "iterations", "leaf_iterations", "inner_lanes", "leaf_lanes",
                "ray_lanes", "refills")


def traversal_profile(ctx, scene, coords, tidx, kind, spp, min_d, max_d, samples, offset=0, count=0, perms=PERMS,
                      traverse=TRAVERSE_AUTO):
    """Lane-utilisation profile of the dynamic schedule (fk_diag_traversal_profile)."""
    p = L.SampleParams(spp, perms, min_d, max_d)
    out = (L.c_u64 * 8)()
    _check(ctx.lib.fk_diag_traversal_profile(ctx.handle, scene.handle, coords.handle, tidx.handle, kind,
                                             ctypes.byref(p), samples.handle, offset, count, traverse, out), ctx,
           "traversal profile")
    return dict(zip(PROFILE_KEYS, (int(v) for v in out)))


def _sampler(cfg):
    if not cfg:
        return L.BakeSampler(0, 0, 0.0, 0.0, 0, 0)
    return L.BakeSampler(1, cfg["sample_count"], cfg["min_distance"], cfg["max_distance"], cfg.get("seed", 0),
                         int(cfg.get("tangent_space", False)))


def bake(ctx, nodes, pos4, nrm4, width, height, pix8, pixt12, indices, outputs, cull_backfaces=True,
         height_map=False, position_map=False, normals_map=False, normals_tangent_space=True, ao=None,
         bent_normals=None, thickness=None, traverse=TRAVERSE_AUTO, mapping_max_distance=0.0):
    """fk_bake: one call from host arrays to host results.  `outputs` maps
    'coords4', 'tidx', 'height', 'position3', 'normals3', 'ao',
    'bent_normals3', 'thickness' to preallocated host arrays (pinned memory
    gives the fastest copies).  ao / bent_normals / thickness: dicts with
    sample_count, min_distance, max_distance, seed (and tangent_space).
    mapping_max_distance: fk_meshmap's max_dist (0: no limit)."""
    n = len(indices)
    d = L.BakeDesc(nodes.ctypes.data, len(nodes), _f32(pos4), _f32(nrm4), len(pos4), width, height, n, _f32(pix8),
                   _f32(pixt12), _u32(indices), int(cull_backfaces), int(height_map), int(position_map),
                   int(normals_map), int(normals_tangent_space), _sampler(ao), _sampler(bent_normals),
                   _sampler(thickness), traverse, mapping_max_distance)
    o = L.BakeOut()
    for name, ctype in (("coords4", L.f32p), ("tidx", L.u32p), ("height", L.f32p), ("position3", L.f32p),
                        ("normals3", L.f32p), ("ao", L.f32p), ("bent_normals3", L.f32p), ("thickness", L.f32p)):
        a = outputs.get(name)
        if a is not None:
            setattr(o, name, a.ctypes.data_as(ctype))
    _check(ctx.lib.fk_bake(ctx.handle, ctypes.byref(d), ctypes.byref(o)), ctx, "fk_bake")


NORMAL_IMPORT, NORMAL_COMPUTE_PER_FACE, NORMAL_COMPUTE_PER_VERTEX = 0, 1, 2
RUN_SOLVERS = ("height", "positions", "normals", "ao", "bent_normals", "thickness")


def run_params(**fields):
    """FornosParameters (Src/fornos.h:35-123) as fk_run_params: the
    reference's defaults, overridden by `fields`.  Shared fields by name
    (lo_poly_mesh_path, hi_poly_mesh_path, lo_poly_mesh_normal,
    hi_poly_mesh_normal, bvh_tris_per_node, tex_width, tex_height,
    tex_dilation, ignore_backfaces, mapping, mapping_edge, seed, traverse);
    solvers (height, positions, normals, ao, bent_normals, thickness) as dicts
    of enabled, output_path, sample_count, min_distance, max_distance,
    tangent_space, normalize_output."""
    p = L.RunParams()
    L.load().fk_run_params_default(ctypes.byref(p))
    keep = []
    for k, v in fields.items():
        if k in RUN_SOLVERS:
            sv = getattr(p, k)
            for sk, x in v.items():
                if sk == "output_path":
                    x = os.fsencode(x) if x is not None else None
                    keep.append(x)
                setattr(sv, sk, x)
        elif k.endswith("_path"):
            x = os.fsencode(v) if v is not None else None
            keep.append(x)
            setattr(p, k, x)
        else:
            setattr(p, k, v)
    p._keep = keep
    return p


def run(ctx, **fields):
    """fk_run: FornosRunner::start + run to completion, mesh files in, image
    files out (fields as run_params)."""
    p = run_params(**fields)
    _check(ctx.lib.fk_run(ctx.handle, ctypes.byref(p)), ctx, "fk_run")


# ------------------------------------------------------------------ batches and tuning
class Batch:
    """Batched hemisphere jobs in one persistent launch (fk_batch_*).
    jobs: list of dicts with scene, coords, tidx, texel_count, spp, min_distance, max_distance, samples, out0
    (and out1, hits0, hits1); perms defaults to 4096."""

    def __init__(self, ctx, jobs, kind=AO):
        self.ctx = ctx
        arr = (L.BatchJob * len(jobs))()
        hv = lambda b: b.handle if b is not None else None
        for i, j in enumerate(jobs):
            arr[i] = L.BatchJob(j["scene"].handle, j["coords"].handle, j["tidx"].handle, j["texel_count"],
                                L.SampleParams(j["spp"], j.get("perms", PERMS), j["min_distance"], j["max_distance"]),
                                j["samples"].handle, j["out0"].handle, hv(j.get("out1")), hv(j.get("hits0")),
                                hv(j.get("hits1")))
        h = L.c_vp()
        _check(ctx.lib.fk_batch_create(ctx.handle, arr, len(jobs), kind, ctypes.byref(h)), ctx, "fk_batch_create")
        self.handle = h.value

    def info(self):
        rays, texels, launches = L.c_u64(), L.c_u32(), L.c_u32()
        _check(self.ctx.lib.fk_batch_info(self.handle, ctypes.byref(rays), ctypes.byref(texels),
                                          ctypes.byref(launches)))
        return {"rays": rays.value, "texels": texels.value, "launches_per_run": launches.value}

    def tune(self, sample_rays=0):
        t, trav = L.Tuning(), L.c_int()
        _check(self.ctx.lib.fk_batch_tune(self.handle, sample_rays, ctypes.byref(t), ctypes.byref(trav)), self.ctx,
               "fk_batch_tune")
        return dict(_tuning_dict(t), traverse=trav.value)

    def run(self, traverse=0):
        _check(self.ctx.lib.fk_batch_run(self.handle, traverse), self.ctx, "fk_batch_run")

    def capture(self, traverse=0):
        _check(self.ctx.lib.fk_batch_capture(self.handle, traverse), self.ctx, "fk_batch_capture")

    def replay(self):
        _check(self.ctx.lib.fk_batch_replay(self.handle), self.ctx, "fk_batch_replay")

    def free(self):
        if self.handle and self.ctx.handle:
            self.ctx.lib.fk_batch_free(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def tune_hemisphere(ctx, scene, coords, tidx, kind, spp, min_d, max_d, samples, offset=0, count=0, perms=PERMS,
                    sample_rays=0):
    """Autotunes the dynamic traversal for one fk_hemisphere call; returns
    (tuning dict, traverse flags).  Apply with ctx.set_tuning(**...)."""
    p = L.SampleParams(spp, perms, min_d, max_d)
    t, trav = L.Tuning(), L.c_int()
    _check(ctx.lib.fk_tune_hemisphere(ctx.handle, scene.handle, coords.handle, tidx.handle, kind, ctypes.byref(p),
                                      samples.handle, offset, count, sample_rays, ctypes.byref(t),
                                      ctypes.byref(trav)), ctx, "fk_tune_hemisphere")
    return _tuning_dict(t), trav.value


# ------------------------------------------------------------------ learned denoiser
DN_INPUTS = 250
DN_PARAMS = 20868
DN_ROW_BYTES = 512
DN_TILE_ROWS = 128
DN_ENGINE_MMA_SYNC, DN_ENGINE_TCGEN05 = 0, 1
DN_HIDDEN = 64
DN_OUT = 4
# parameter blocks: name -> (offset, shape)
DN_LAYOUT = {"w1": (0, (64, 256)), "b1": (16384, (64,)), "w2": (16448, (64, 64)), "b2": (20544, (64,)),
             "w3": (20608, (4, 64)), "b3": (20864, (4,))}


def denoise_features(ctx, tmap, coords, tidx, ao, bn3, pos3, nrm3, max_distance, image=None):
    """Dense feature image (3 planes of W x H float4) of a texel map."""
    if image is None:
        image = ctx.buffer(48 * tmap.width * tmap.height)
    _check(ctx.lib.fk_denoise_features(ctx.handle, tmap.handle, coords.handle, tidx.handle, ao.handle, bn3.handle,
                                       pos3.handle, nrm3.handle, max_distance, image.handle), ctx,
           "fk_denoise_features")
    return image


def denoise_rows(ctx, image, width, height, pixels, count, rows=None):
    """Network input rows (256 bf16 each) for `count` pixel indices."""
    if rows is None:
        rows = ctx.buffer(max(count, 1) * DN_ROW_BYTES)
    _check(ctx.lib.fk_denoise_rows(ctx.handle, image.handle, width, height, pixels.handle, count, rows.handle), ctx,
           "fk_denoise_rows")
    return rows


class Denoiser:
    """The learned AO + bent-normal denoiser (fk_denoiser)."""

    def __init__(self, ctx, params=None):
        self.ctx = ctx
        h = L.c_vp()
        _check(ctx.lib.fk_denoiser_create(ctx.handle, ctypes.byref(h)), ctx, "fk_denoiser_create")
        self.handle = h.value
        if params is not None:
            self.set_params(params)

    def set_engine(self, engine):
        """Inference kernel: DN_ENGINE_TCGEN05 (default) or DN_ENGINE_MMA_SYNC."""
        _check(self.ctx.lib.fk_denoiser_set_engine(self.handle, engine), self.ctx, "fk_denoiser_set_engine")

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        _check(self.ctx.lib.fk_denoiser_set_params(self.handle, _f32(p), p.size), self.ctx, "fk_denoiser_set_params")

    def get_params(self):
        p = np.empty(DN_PARAMS, np.float32)
        _check(self.ctx.lib.fk_denoiser_get_params(self.handle, _f32(p), p.size), self.ctx, "fk_denoiser_get_params")
        return p

    def train_step(self, rows, targets, n_rows, batch, row_ids=None, offset=0, lr=1e-3, beta1=0.9, beta2=0.999,
                   eps=1e-8):
        a = L.Adam(lr, beta1, beta2, eps)
        _check(self.ctx.lib.fk_denoiser_train_step(self.handle, rows.handle, targets.handle, n_rows,
                                                   row_ids.handle if row_ids is not None else None, offset, batch,
                                                   ctypes.byref(a)), self.ctx, "fk_denoiser_train_step")

    def last_loss(self):
        v = ctypes.c_double()
        _check(self.ctx.lib.fk_denoiser_last_loss(self.handle, ctypes.byref(v)), self.ctx, "fk_denoiser_last_loss")
        return v.value

    def gradient(self, rows, targets, n_rows, batch, row_ids=None, offset=0):
        g = np.empty(DN_PARAMS, np.float32)
        v = ctypes.c_double()
        _check(self.ctx.lib.fk_denoiser_gradient(self.handle, rows.handle, targets.handle, n_rows,
                                                 row_ids.handle if row_ids is not None else None, offset, batch,
                                                 _f32(g), ctypes.byref(v)), self.ctx, "fk_denoiser_gradient")
        return g, v.value

    def forward(self, rows, count, y4=None):
        if y4 is None:
            y4 = self.ctx.buffer(max(count, 1) * 16)
        _check(self.ctx.lib.fk_denoiser_forward(self.handle, rows.handle, count, y4.handle), self.ctx,
               "fk_denoiser_forward")
        return y4

    def apply(self, tmap, image, tidx, ao_in, bn_in, ao_out, bn_out, offset=0, count=None):
        count = tmap.count - offset if count is None else count
        _check(self.ctx.lib.fk_denoise_apply(self.handle, tmap.handle, image.handle, tidx.handle, ao_in.handle,
                                             bn_in.handle, offset, count, ao_out.handle, bn_out.handle), self.ctx,
               "fk_denoise_apply")

    def bake(self, scene, tmap, coords, tidx, samples_low, samples_full, ao_out, bn_out, low_samples=16,
             full_samples=1024, min_distance=0.001, max_distance=0.3, perms=PERMS, tile=64, verify_cells=4,
             max_tile_error=0.02, traverse=TRAVERSE_AUTO):
        """The verified denoised AO + bent-normal bake; returns its statistics."""
        p = L.DenoiseParams(low_samples, full_samples, perms, min_distance, max_distance, tile, verify_cells,
                            max_tile_error, traverse)
        st = L.DenoiseStats()
        _check(self.ctx.lib.fk_denoise_bake(self.handle, scene.handle, tmap.handle, coords.handle, tidx.handle,
                                            ctypes.byref(p), samples_low.handle, samples_full.handle, ao_out.handle,
                                            bn_out.handle, ctypes.byref(st)), self.ctx, "fk_denoise_bake")
        return {k: getattr(st, k) for k, _ in L.DenoiseStats._fields_}

    def free(self):
        if self.handle and self.ctx.handle:
            self.ctx.lib.fk_denoiser_free(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
