"""ctypes binding of libfornos_b200.so (declarations in include/fornos_gpu.h).

The library is built in-tree by fornos_b200/build.py.  Importing this module
fails loudly when the library is missing: there is no fallback path.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfornos_b200.so")

c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_int = ctypes.c_int
c_float = ctypes.c_float
c_size = ctypes.c_size_t
c_vp = ctypes.c_void_p
f32p = ctypes.POINTER(ctypes.c_float)
u32p = ctypes.POINTER(ctypes.c_uint32)


class MeshDesc(ctypes.Structure):
    _fields_ = [("position_count", c_u32), ("positions", f32p),
                ("texcoord_count", c_u32), ("texcoords", f32p),
                ("normal_count", c_u32), ("normals", f32p),
                ("vertex_count", c_u32), ("vertices", u32p),
                ("triangle_count", c_u32), ("triangles", u32p),
                ("tangents", f32p), ("bitangents", f32p)]


class SampleParams(ctypes.Structure):
    _fields_ = [("sample_count", c_u32), ("perm_count", c_u32), ("min_distance", c_float),
                ("max_distance", c_float)]


class SolverParams(ctypes.Structure):
    _fields_ = [("kind", c_int), ("sample_count", c_u32), ("min_distance", c_float), ("max_distance", c_float),
                ("tangent_space", c_int), ("normalize_output", c_int), ("seed", c_u32), ("traverse", c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("refill", c_u32), ("leaf_batch", c_u32), ("speculate", c_u32), ("ray_order", c_u32),
                ("top_records", c_u32), ("l2_persist", c_u32), ("block_threads", c_u32), ("stack_depth", c_u32)]


class ExportParams(ctypes.Structure):
    _fields_ = [("mode", c_int), ("filter_lo", c_float), ("filter_hi", c_float), ("normalize", c_int),
                ("dilate", c_int)]


class RunSolver(ctypes.Structure):
    _fields_ = [("enabled", c_int), ("output_path", ctypes.c_char_p), ("sample_count", c_u32),
                ("min_distance", c_float), ("max_distance", c_float), ("tangent_space", c_int),
                ("normalize_output", c_int)]


class RunParams(ctypes.Structure):
    _fields_ = [("lo_poly_mesh_path", ctypes.c_char_p), ("hi_poly_mesh_path", ctypes.c_char_p),
                ("lo_poly_mesh_normal", c_int), ("hi_poly_mesh_normal", c_int), ("bvh_tris_per_node", c_u32),
                ("tex_width", c_u32), ("tex_height", c_u32), ("tex_dilation", c_int), ("ignore_backfaces", c_int),
                ("mapping", c_int), ("mapping_edge", c_float), ("height", RunSolver), ("positions", RunSolver),
                ("normals", RunSolver), ("ao", RunSolver), ("bent_normals", RunSolver), ("thickness", RunSolver),
                ("seed", c_u32), ("traverse", c_int)]


class SceneInfo(ctypes.Structure):
    _fields_ = [("node_count", c_u32), ("corner_count", c_u32), ("depth", c_u32), ("leaf_count", c_u32),
                ("device_bytes", c_u64)]


class BakeSampler(ctypes.Structure):
    _fields_ = [("enabled", c_int), ("sample_count", c_u32), ("min_distance", c_float), ("max_distance", c_float),
                ("seed", c_u32), ("tangent_space", c_int)]


class BakeDesc(ctypes.Structure):
    _fields_ = [("nodes", c_vp), ("node_count", c_u32), ("positions4", f32p), ("normals4", f32p),
                ("corner_count", c_u32), ("width", c_u32), ("height", c_u32), ("texel_count", c_u32),
                ("pix8", f32p), ("pixt12", f32p), ("indices", u32p), ("cull_backfaces", c_int),
                ("height_enabled", c_int), ("position_enabled", c_int), ("normals_enabled", c_int),
                ("normals_tangent_space", c_int), ("ao", BakeSampler), ("bent_normals", BakeSampler),
                ("thickness", BakeSampler), ("traverse", c_int), ("mapping_max_distance", c_float)]


class BatchJob(ctypes.Structure):
    _fields_ = [("scene", c_vp), ("coords", c_vp), ("tidx", c_vp), ("texel_count", c_u32),
                ("params", SampleParams), ("samples", c_vp), ("out0", c_vp), ("out1", c_vp), ("hits0", c_vp),
                ("hits1", c_vp)]


class BakeOut(ctypes.Structure):
    _fields_ = [("coords4", f32p), ("tidx", u32p), ("height", f32p), ("position3", f32p), ("normals3", f32p),
                ("ao", f32p), ("bent_normals3", f32p), ("thickness", f32p)]


class Adam(ctypes.Structure):
    _fields_ = [("learning_rate", c_float), ("beta1", c_float), ("beta2", c_float), ("eps", c_float)]


class DenoiseParams(ctypes.Structure):
    _fields_ = [("low_samples", c_u32), ("full_samples", c_u32), ("perm_count", c_u32), ("min_distance", c_float),
                ("max_distance", c_float), ("tile", c_u32), ("verify_cells", c_u32), ("max_tile_error", c_float),
                ("traverse", c_int)]


class DenoiseStats(ctypes.Structure):
    _fields_ = [("tiles", c_u32), ("tiles_failed", c_u32), ("spot_checks", c_u32), ("texels_rebaked", c_u32),
                ("rays", c_u64), ("worst_tile_error", c_float)]


# name: (restype, argtypes)
_SIGS = {
    "fk_ctx_create": (c_int, [c_int, ctypes.POINTER(c_vp)]),
    "fk_ctx_destroy": (c_int, [c_vp]),
    "fk_last_error": (ctypes.c_char_p, [c_vp]),
    "fk_ctx_set_stream": (c_int, [c_vp, c_vp]),
    "fk_ctx_stream": (c_vp, [c_vp]),
    "fk_sync": (c_int, [c_vp]),
    "fk_ctx_trim": (c_int, [c_vp]),
    "fk_launch_count": (c_u64, [c_vp]),
    "fk_ctx_set_tuning": (c_int, [c_vp, ctypes.POINTER(Tuning)]),
    "fk_ctx_get_tuning": (c_int, [c_vp, ctypes.POINTER(Tuning)]),
    "fk_buf_alloc": (c_int, [c_vp, c_size, ctypes.POINTER(c_vp)]),
    "fk_buf_upload": (c_int, [c_vp, c_vp, c_size, c_vp, c_size]),
    "fk_buf_download": (c_int, [c_vp, c_vp, c_size, c_vp, c_size]),
    "fk_buf_free": (c_int, [c_vp, c_vp]),
    "fk_buf_size": (c_size, [c_vp]),
    "fk_buf_device_ptr": (c_vp, [c_vp]),
    "fk_mesh_create": (c_int, [ctypes.POINTER(MeshDesc), ctypes.POINTER(c_vp)]),
    "fk_mesh_describe": (c_int, [c_vp, ctypes.POINTER(MeshDesc)]),
    "fk_mesh_copy": (c_int, [c_vp, ctypes.POINTER(c_vp)]),
    "fk_mesh_load": (c_int, [ctypes.c_char_p, ctypes.POINTER(c_vp)]),
    "fk_mesh_free": (c_int, [c_vp]),
    "fk_mesh_compute_face_normals": (c_int, [c_vp]),
    "fk_mesh_compute_vertex_normals": (c_int, [c_vp]),
    "fk_mesh_compute_vertex_normals_welded": (c_int, [c_vp]),
    "fk_mesh_compute_tangent_space": (c_int, [c_vp]),
    "fk_mesh_compute_normals_device": (c_int, [c_vp, c_vp, c_int]),
    "fk_mesh_compute_tangent_space_device": (c_int, [c_vp, c_vp]),
    "fk_bvh_build": (c_int, [c_vp, c_u32, c_u32, ctypes.POINTER(c_vp)]),
    "fk_bvh_free": (c_int, [c_vp]),
    "fk_bvh_flatten_sizes": (c_int, [c_vp, u32p, u32p]),
    "fk_bvh_flatten": (c_int, [c_vp, c_vp, c_vp, f32p, f32p]),
    "fk_scene_upload": (c_int, [c_vp, c_vp, c_u32, f32p, f32p, c_u32, ctypes.POINTER(c_vp)]),
    "fk_scene_free": (c_int, [c_vp, c_vp]),
    "fk_scene_get_info": (c_int, [c_vp, ctypes.POINTER(SceneInfo)]),
    "fk_scene_set_tree": (c_int, [c_vp, c_int]),
    "fk_raster_uv": (c_int, [c_vp, c_vp, c_vp, c_u32, c_u32, c_int, c_float, ctypes.POINTER(c_vp)]),
    "fk_texel_map_from_host": (c_int, [c_vp, c_u32, c_u32, c_u32, f32p, f32p, u32p, ctypes.POINTER(c_vp)]),
    "fk_texel_map_info": (c_int, [c_vp, u32p, u32p, u32p]),
    "fk_texel_map_download": (c_int, [c_vp, c_vp, f32p, f32p, u32p]),
    "fk_texel_map_free": (c_int, [c_vp, c_vp]),
    "fk_samples_cosine": (c_int, [c_u32, c_u32, c_u32, f32p]),
    "fk_meshmap": (c_int, [c_vp, c_vp, c_vp, c_int, c_float, c_u32, c_u32, c_vp, c_vp]),
    "fk_hemisphere": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, ctypes.POINTER(SampleParams), c_vp, c_u32, c_u32,
                              c_int, c_vp, c_vp, c_vp, c_vp]),
    "fk_hemisphere_texels": (c_int, [c_vp, c_vp, c_vp, c_vp, c_u32, c_int, ctypes.POINTER(SampleParams), c_vp, c_vp,
                                     c_u32, c_u32, c_int, c_vp, c_vp, c_vp, c_vp]),
    "fk_ctx_check": (c_int, [c_vp]),
    "fk_gather": (c_int, [c_vp, c_vp, c_int, c_vp, c_vp, c_u32, c_u32, c_vp]),
    "fk_tangent_space": (c_int, [c_vp, c_vp, c_u32, c_u32, c_vp]),
    "fk_hemisphere_noalloc": (c_int, [c_vp, c_vp, c_vp, c_int, ctypes.POINTER(SampleParams), c_vp, c_u32, c_u32,
                                      c_int, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "fk_meshmapping_create": (c_int, [c_vp, ctypes.POINTER(c_vp)]),
    "fk_meshmapping_init": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int]),
    "fk_meshmapping_init_scene": (c_int, [c_vp, c_vp, c_vp, c_int]),
    "fk_meshmapping_set_work_per_step": (c_int, [c_vp, c_u32]),
    "fk_meshmapping_run_step": (c_int, [c_vp, ctypes.POINTER(c_int)]),
    "fk_meshmapping_progress": (c_float, [c_vp]),
    "fk_meshmapping_results": (c_int, [c_vp, f32p, u32p]),
    "fk_meshmapping_coords": (c_vp, [c_vp]),
    "fk_meshmapping_tidx": (c_vp, [c_vp]),
    "fk_meshmapping_scene": (c_vp, [c_vp]),
    "fk_meshmapping_free": (c_int, [c_vp]),
    "fk_solver_create": (c_int, [c_vp, ctypes.POINTER(SolverParams), ctypes.POINTER(c_vp)]),
    "fk_solver_init": (c_int, [c_vp, c_vp, c_vp]),
    "fk_solver_set_work_per_step": (c_int, [c_vp, c_u32]),
    "fk_solver_run_step": (c_int, [c_vp, ctypes.POINTER(c_int)]),
    "fk_solver_progress": (c_float, [c_vp]),
    "fk_solver_result_count": (c_size, [c_vp]),
    "fk_solver_results": (c_int, [c_vp, f32p, c_size]),
    "fk_solver_hits": (c_int, [c_vp, u32p, c_size]),
    "fk_solver_result_buffer": (c_vp, [c_vp]),
    "fk_solver_free": (c_int, [c_vp]),
    "fk_bake": (c_int, [c_vp, ctypes.POINTER(BakeDesc), ctypes.POINTER(BakeOut)]),
    "fk_run_params_default": (None, [ctypes.POINTER(RunParams)]),
    "fk_run": (c_int, [c_vp, ctypes.POINTER(RunParams)]),
    "fk_batch_create": (c_int, [c_vp, ctypes.POINTER(BatchJob), c_u32, c_int, ctypes.POINTER(c_vp)]),
    "fk_batch_info": (c_int, [c_vp, ctypes.POINTER(c_u64), u32p, u32p]),
    "fk_batch_tune": (c_int, [c_vp, c_u64, ctypes.POINTER(Tuning), ctypes.POINTER(c_int)]),
    "fk_batch_run": (c_int, [c_vp, c_int]),
    "fk_batch_capture": (c_int, [c_vp, c_int]),
    "fk_batch_replay": (c_int, [c_vp]),
    "fk_batch_free": (c_int, [c_vp]),
    "fk_tune_hemisphere": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, ctypes.POINTER(SampleParams), c_vp, c_u32, c_u32,
                                   c_u64, ctypes.POINTER(Tuning), ctypes.POINTER(c_int)]),
    "fk_diag_fp32_peak": (c_int, [c_vp, ctypes.POINTER(ctypes.c_double)]),
    "fk_diag_traversal_counts": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, ctypes.POINTER(SampleParams), c_vp, c_u32,
                                         c_u32, c_int, ctypes.POINTER(c_u64)]),
    "fk_diag_traversal_profile": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, ctypes.POINTER(SampleParams), c_vp, c_u32,
                                          c_u32, c_int, ctypes.POINTER(c_u64)]),
    "fk_bvh_build_flat": (c_int, [c_vp, c_vp, c_u32, c_u32, c_vp, c_u32, ctypes.POINTER(c_u32), f32p, f32p]),
    "fk_scene_build": (c_int, [c_vp, c_vp, c_u32, c_u32, ctypes.POINTER(c_vp)]),
    "fk_export_image": (c_int, [c_vp, c_vp, c_vp, ctypes.POINTER(ExportParams), c_vp, f32p]),
    "fk_image_write_rgb8": (c_int, [ctypes.c_char_p, c_u32, c_u32, c_vp]),
    "fk_image_write_png": (c_int, [ctypes.c_char_p, c_u32, c_u32, c_vp, c_int]),
    "fk_image_write_exr": (c_int, [ctypes.c_char_p, c_u32, c_u32, c_u32, f32p]),
    "fk_diag_scene_tree": (c_int, [c_vp, c_vp, c_int, f32p, c_u32, ctypes.POINTER(c_u32), ctypes.POINTER(c_u32)]),
    "fk_diag_sah_host": (c_int, [c_vp, c_u32, f32p, c_u32, ctypes.POINTER(c_u32), ctypes.POINTER(c_u32)]),
    "fk_denoiser_create": (c_int, [c_vp, ctypes.POINTER(c_vp)]),
    "fk_denoiser_free": (c_int, [c_vp]),
    "fk_denoiser_set_engine": (c_int, [c_vp, c_int]),
    "fk_denoiser_set_params": (c_int, [c_vp, f32p, c_u32]),
    "fk_denoiser_get_params": (c_int, [c_vp, f32p, c_u32]),
    "fk_denoise_features": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_float, c_vp]),
    "fk_denoise_rows": (c_int, [c_vp, c_vp, c_u32, c_u32, c_vp, c_u32, c_vp]),
    "fk_denoiser_train_step": (c_int, [c_vp, c_vp, c_vp, c_u32, c_vp, c_u32, c_u32, ctypes.POINTER(Adam)]),
    "fk_denoiser_last_loss": (c_int, [c_vp, ctypes.POINTER(ctypes.c_double)]),
    "fk_denoiser_gradient": (c_int, [c_vp, c_vp, c_vp, c_u32, c_vp, c_u32, c_u32, f32p,
                                     ctypes.POINTER(ctypes.c_double)]),
    "fk_denoiser_forward": (c_int, [c_vp, c_vp, c_u32, c_vp]),
    "fk_denoise_apply": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_u32, c_u32, c_vp, c_vp]),
    "fk_denoise_bake": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(DenoiseParams), c_vp, c_vp, c_vp, c_vp,
                                ctypes.POINTER(DenoiseStats)]),
}

_lib = None


def load():
    """Loads the in-tree library (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("libfornos_b200.so is not built; run `python -m fornos_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGS)
