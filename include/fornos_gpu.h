/*
 * fornos_gpu.h - C ABI of the B200 (sm_100a) texture-baking path.
 *
 * This ABI replaces the OpenGL buffer-and-dispatch layer of Fornos:
 *   ComputeBuffer<T>            Src/compute.h:37-87     -> fk_buf_*
 *   LoadComputeShader_*()       Src/computeshaders.h:28-46
 *   + glDispatchCompute in every runStep (e.g. Src/solver_ao.cpp:91-118)
 *                                                       -> fk_meshmap, fk_hemisphere,
 *                                                          fk_gather, fk_tangent_space
 * and exposes the host solver API that sits on top of it:
 *   MeshMapping                 Src/meshmapping.h:42-75 -> fk_meshmapping_*
 *   Height/Position/Normals/AmbientOcclusion/BentNormals/Thickness solvers
 *                               Src/solver_*.h          -> fk_solver_*
 *   Mesh, normal / tangent generators
 *                               Src/mesh.h:35-63, Src/mesh.cpp:619-768 -> fk_mesh_*
 *   BVH::createBinary + fillMeshData
 *                               Src/bvh.h:32-46, Src/meshmapping.cpp:62-125 -> fk_bvh_*
 *   MapUV::from* + CompressedMapUV
 *                               Src/compute.h:214-259   -> fk_raster_uv, fk_texel_map_*
 *   computeSamplesImportanceCosDir
 *                               Src/math.h:363-382      -> fk_samples_cosine
 *
 * Conventions.  Every function returns FK_OK (0) or a negative FK_ERR_* code;
 * nothing aborts or throws across the ABI.  fk_last_error(ctx) describes the
 * last failure of that context.  Device work is ordered on the context's
 * stream (fk_ctx_set_stream); functions that return host data synchronise it.
 * Handles belong to the context that made them and are freed by their *_free
 * call or by fk_ctx_destroy.  One context per host thread.
 */
#ifndef FORNOS_GPU_H
#define FORNOS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define FK_OK 0
#define FK_ERR_INVALID (-1)     /* bad argument: null handle, size, range, kind */
#define FK_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define FK_ERR_NOMEM (-3)       /* device or host allocation failed */
#define FK_ERR_STATE (-4)       /* call out of order (e.g. run_step before init) */
#define FK_ERR_DEVICE (-5)      /* a kernel reported a limit it could not honour */
#define FK_ERR_UNSUPPORTED (-6) /* no sm_100 device, or feature not built */

/* ------------------------------------------------------------ handles */
typedef struct fk_ctx fk_ctx;
typedef struct fk_buf fk_buf;               /* device allocation */
typedef struct fk_mesh fk_mesh;             /* host indexed mesh (Src/mesh.h) */
typedef struct fk_bvh fk_bvh;               /* host BVH tree (Src/bvh.h) */
typedef struct fk_scene fk_scene;           /* high-poly mesh + BVH resident on the device */
typedef struct fk_texel_map fk_texel_map;   /* compressed texel map on the device */
typedef struct fk_meshmapping fk_meshmapping;
typedef struct fk_solver fk_solver;

/* ------------------------------------------------------------ context */
/* Opens `device` (must be compute capability 10.x).  No graphics context.
 * Device memory of the context (buffers, scenes, texel maps, scratch) comes
 * from a stream-ordered pool of its own that keeps what is freed for reuse;
 * fk_ctx_trim returns the unused part to the device. */
int fk_ctx_create(int device, fk_ctx** out);
int fk_ctx_destroy(fk_ctx* ctx);
const char* fk_last_error(const fk_ctx* ctx);
/* cudaStream_t to order work on; NULL = the context's own stream.  Waits for
 * the work queued on the previous stream. */
int fk_ctx_set_stream(fk_ctx* ctx, void* cuda_stream);
void* fk_ctx_stream(const fk_ctx* ctx);
int fk_sync(fk_ctx* ctx);
/* No counterpart in the reference.  Waits for the context's stream and
 * releases the pool memory no live object uses and the scene uploads' pinned
 * host staging. */
int fk_ctx_trim(fk_ctx* ctx);
/* Kernel launches issued by this context so far. */
uint64_t fk_launch_count(const fk_ctx* ctx);

/* Knobs of the dynamically scheduled hemisphere traversal (defaults 20, 8,
 * 1, FK_RAY_ORDER_SECTOR, from full-size sweeps of the plane workload);
 * fk_tune_hemisphere picks them by measurement.  No knob changes a result:
 * each ray still writes the slot of its own sample, and the per-texel sums
 * run in sample order. */
#define FK_RAY_ORDER_SAMPLE 0 /* a texel's rays are taken in sample order */
#define FK_RAY_ORDER_SECTOR 1 /* sample k = (q % 32) * (spp / 32) + q / 32 for queue slot q: the 32
                                 rays a warp takes share one azimuth sector of the sample table
                                 (Src/math.h:339-382 puts the low bits of k into the azimuth's high
                                 bits); spp a multiple of 32, else sample order */
typedef struct fk_tuning {
  uint32_t refill;      /* idle lanes of a warp that trigger a batch fetch (1..32) */
  uint32_t leaf_batch;  /* lanes holding a postponed leaf that start a leaf phase (1..32) */
  uint32_t speculate;   /* lanes holding a leaf keep visiting inner records (0 / 1) */
  uint32_t ray_order;   /* FK_RAY_ORDER_* */
  uint32_t top_records; /* 2-wide ordered traversal: the first top_records inner records of the tree in
                           breadth-first order (its top levels) are staged in each block's shared
                           memory (0 = none, at most FK_MAX_TOP_RECORDS; 64 bytes each) */
  uint32_t l2_persist;  /* FK_L2_*: records read through a persisting L2 access-policy window.  The
                           window is a launch attribute of the trace kernel (the stream's attributes
                           are untouched); the context sets the device's persisting L2 set-aside
                           while a window is in use and restores it when the knob is turned off or
                           the context is destroyed */
  uint32_t block_threads; /* threads per block of the trace kernel: 128, 256 or 512 */
  uint32_t stack_depth;   /* deferred entries per lane of the ordered traversals: 32 or 64; 32 serves
                             trees of at most 24 levels (4-wide: 10), deeper trees use 64 */
} fk_tuning;
#define FK_MAX_TOP_RECORDS 1024
#define FK_L2_NONE 0
#define FK_L2_TREE 1      /* the inner records of the tree being walked */
#define FK_L2_TRIANGLES 2 /* the triangle records (hit ratio: set-aside / their size) */
int fk_ctx_set_tuning(fk_ctx* ctx, const fk_tuning* tuning);
int fk_ctx_get_tuning(const fk_ctx* ctx, fk_tuning* tuning);

/* ------------------------------------------------------------ buffers
 * Replaces ComputeBuffer<T> (Src/compute.h:37-87).  New buffers are
 * zero-filled like ComputeBuffer(count, usage) (Src/compute.h:57-65). */
int fk_buf_alloc(fk_ctx* ctx, size_t bytes, fk_buf** out);
int fk_buf_upload(fk_ctx* ctx, fk_buf* buf, size_t offset, const void* src, size_t bytes);
int fk_buf_download(fk_ctx* ctx, const fk_buf* buf, size_t offset, void* dst, size_t bytes);
int fk_buf_free(fk_ctx* ctx, fk_buf* buf);
size_t fk_buf_size(const fk_buf* buf);
void* fk_buf_device_ptr(const fk_buf* buf);

/* ------------------------------------------------------------ host mesh
 * Indexed mesh exactly as Src/mesh.h:35-63: per-vertex (position, texcoord,
 * normal) indices, per-triangle vertex indices; tangents / bitangents per
 * vertex (may be absent).  Arrays are copied on create. */
typedef struct fk_mesh_desc {
  uint32_t position_count;
  const float* positions;   /* 3 floats each */
  uint32_t texcoord_count;
  const float* texcoords;   /* 2 floats each */
  uint32_t normal_count;
  const float* normals;     /* 3 floats each */
  uint32_t vertex_count;
  const uint32_t* vertices; /* 3 u32 each: position, texcoord, normal index */
  uint32_t triangle_count;
  const uint32_t* triangles;/* 3 u32 each: vertex indices */
  const float* tangents;    /* 3 floats per vertex, or NULL */
  const float* bitangents;  /* 3 floats per vertex, or NULL */
} fk_mesh_desc;

int fk_mesh_create(const fk_mesh_desc* desc, fk_mesh** out);
/* Fills `out` with pointers into the mesh's own arrays (valid until the
 * mesh changes or is freed). */
int fk_mesh_describe(const fk_mesh* mesh, fk_mesh_desc* out);
int fk_mesh_copy(const fk_mesh* mesh, fk_mesh** out);                 /* Mesh::createCopy */
/* Mesh::loadFile (Src/mesh.cpp:612-617): ".obj" through the Wavefront reader
 * (:235-456), ".ply" through the PLY reader (:515-601, tinyply 2.0); the mesh
 * the reference's loader returns, array for array.  FK_ERR_INVALID for a file
 * the reference rejects, another extension, or a mesh whose corners name
 * positions the file lacks; an OBJ file that cannot be opened gives an empty
 * mesh, as in the reference. */
int fk_mesh_load(const char* path, fk_mesh** out);
int fk_mesh_free(fk_mesh* mesh);
int fk_mesh_compute_face_normals(fk_mesh* mesh);                      /* Src/mesh.cpp:627 */
int fk_mesh_compute_vertex_normals(fk_mesh* mesh);                    /* Src/mesh.cpp:650 */
int fk_mesh_compute_vertex_normals_welded(fk_mesh* mesh);             /* Src/mesh.cpp:680 (Aggressive) */
int fk_mesh_compute_tangent_space(fk_mesh* mesh);                     /* Src/mesh.cpp:724 */

/* The same generators on the device (sort-and-reduce kernels on ctx's
 * stream): the mesh's arrays are uploaded, processed and written back, with
 * results equal to the host calls above bit for bit (NaN payloads aside).
 * method: FK_NORMALS_FACE (Mesh::computeFaceNormals, Src/mesh.cpp:627),
 * FK_NORMALS_VERTEX (computeVertexNormals, :650) or FK_NORMALS_WELDED
 * (computeVertexNormalsAggressive, :680).  Index errors: FK_ERR_INVALID,
 * mesh unchanged. */
#define FK_NORMALS_FACE 0
#define FK_NORMALS_VERTEX 1
#define FK_NORMALS_WELDED 2
int fk_mesh_compute_normals_device(fk_ctx* ctx, fk_mesh* mesh, int method);
int fk_mesh_compute_tangent_space_device(fk_ctx* ctx, fk_mesh* mesh);  /* Mesh::computeTangentSpace, :724 */

/* ------------------------------------------------------------ BVH (host)
 * BVH::createBinary (Src/bvh.cpp:283-314): 16-bucket split, leaves of at
 * most max_tris_per_node triangles, depth limit max_depth (8192 in
 * Src/fornos.cpp:157).  Multi-threaded; the tree is identical to the
 * single-threaded build. */
int fk_bvh_build(const fk_mesh* mesh, uint32_t max_tris_per_node, uint32_t max_depth, fk_bvh** out);
int fk_bvh_free(fk_bvh* bvh);

/* Flattened skip-pointer node (BVHGPUData, Src/meshmapping.h:33-40), 36 B. */
typedef struct fk_bvh_node {
  float aabb_min[3];
  float aabb_max[3];
  uint32_t start; /* first triangle corner (multiple of 3) */
  uint32_t end;   /* one past the last corner; start == end for inner nodes */
  uint32_t jump;  /* index of the node after this subtree */
} fk_bvh_node;

/* fillMeshData (Src/meshmapping.cpp:62-125): node and corner counts, then the
 * arrays (positions / normals as 4 floats per corner, w = 0). */
int fk_bvh_flatten_sizes(const fk_bvh* bvh, uint32_t* node_count, uint32_t* corner_count);
int fk_bvh_flatten(const fk_bvh* bvh, const fk_mesh* mesh, fk_bvh_node* nodes, float* positions4, float* normals4);
/* BVH::createBinary (Src/bvh.cpp:128-314) + fillMeshData
 * (Src/meshmapping.cpp:62-125) built on the device: the nodes and corner
 * arrays of fk_bvh_build + fk_bvh_flatten, bit for bit.  *node_count gets the
 * node count (at most 2 x triangles - 1); nodes (capacity in entries),
 * positions4 and normals4 (3 x triangles x 4 floats) may each be NULL. */
int fk_bvh_build_flat(fk_ctx* ctx, const fk_mesh* mesh, uint32_t max_tris, uint32_t max_depth, fk_bvh_node* nodes,
                      uint32_t node_capacity, uint32_t* node_count, float* positions4, float* normals4);

/* ------------------------------------------------------------ device scene */
/* Checks the node array (FK_ERR_INVALID names the first defective node) and
 * lays it out for the device on host threads, in pinned host memory that the
 * context keeps for later uploads (72 bytes per node; fk_ctx_trim
 * releases it).  Returns once the scene is on the device. */
int fk_scene_upload(fk_ctx* ctx, const fk_bvh_node* nodes, uint32_t node_count, const float* positions4,
                    const float* normals4, uint32_t corner_count, fk_scene** out);
int fk_scene_free(fk_ctx* ctx, fk_scene* scene);
/* fk_bvh_build_flat + fk_scene_upload without the round trip: the device-built
 * nodes and corners become the scene's arrays. */
int fk_scene_build(fk_ctx* ctx, const fk_mesh* mesh, uint32_t max_tris, uint32_t max_depth, fk_scene** out);
typedef struct fk_scene_info {
  uint32_t node_count;
  uint32_t corner_count;
  uint32_t depth;        /* levels from the root to the deepest leaf */
  uint32_t leaf_count;
  uint64_t device_bytes;
} fk_scene_info;
int fk_scene_get_info(const fk_scene* scene, fk_scene_info* out);
/* No counterpart in the reference.  The inner tree the ordered traversals
 * (FK_TRAVERSE_ORDERED / ORDERED4) walk: FK_TREE_SAH (the default whenever it
 * was built), an inner tree rebuilt on the device at upload over the same
 * leaves with a binned surface-area split on all three box faces (the
 * reference's split cost, Src/bvh.cpp:63-68, counts x*y twice and y*z never),
 * or FK_TREE_REFERENCE, the inner nodes of BVH::createBinary as uploaded.
 * Leaves, leaf boxes and the skip-pointer walk are untouched, and the outcome
 * is that of any inner tree over these leaves (an inner box only prunes what
 * its leaves' own tests reject), so results stay within the ordered
 * traversal's bar.  Both trees stay resident.  The rebuilt tree is not built
 * when a leaf box coordinate is not finite or not below 1e30 in magnitude, nor
 * kept when it is deeper than 48 levels. */
#define FK_TREE_REFERENCE 0
#define FK_TREE_SAH 1
int fk_scene_set_tree(fk_scene* scene, int tree);

/* ------------------------------------------------------------ texel map
 * MapUV::fromMesh / fromMeshes / fromMeshes_Hybrid (Src/compute.cpp:352-370)
 * followed by CompressedMapUV (Src/compute.cpp:372-416), on the device.
 * Pixel rows: Pix_GPUData {p, pad, d, pad} (32 B) and PixT_GPUData
 * {n, pad, t, pad, b, pad} (48 B) (Src/meshmapping.h:15-31), plus the texel
 * index in the full map. */
#define FK_MAP_SMOOTH 0           /* directions from `dirs` (welded normals) */
#define FK_MAP_LOWPOLY_NORMALS 1  /* directions = the mesh's own normals */
#define FK_MAP_HYBRID 2           /* blend by edge distance (mappingEdge) */
int fk_raster_uv(fk_ctx* ctx, const fk_mesh* lowpoly, const fk_mesh* dirs, uint32_t width, uint32_t height,
                 int mode, float edge, fk_texel_map** out);
int fk_texel_map_from_host(fk_ctx* ctx, uint32_t width, uint32_t height, uint32_t count, const float* pix8,
                           const float* pixt12, const uint32_t* indices, fk_texel_map** out);
int fk_texel_map_info(const fk_texel_map* map, uint32_t* width, uint32_t* height, uint32_t* count);
int fk_texel_map_download(fk_ctx* ctx, const fk_texel_map* map, float* pix8, float* pixt12, uint32_t* indices);
int fk_texel_map_free(fk_ctx* ctx, fk_texel_map* map);

/* ------------------------------------------------------------ sample table
 * computeSamplesImportanceCosDir(spp, perms) (Src/math.h:363-382) with a
 * seeded std::mt19937 in place of std::random_device; 4 floats per sample
 * (w = 0), perms rows of spp samples.  Host function. */
int fk_samples_cosine(uint32_t spp, uint32_t perms, uint32_t seed, float* out4);

/* ------------------------------------------------------------ kernels
 * Mesh mapping, Shaders/meshmapping_nobackfaces.comp (cull_backfaces = 1,
 * the default of Src/fornos.h:48) or Shaders/meshmapping.comp, over texels
 * [offset, offset + count) of `map`.  coords: float4 (t, b0, b1, b2) per
 * texel; tidx: u32 per texel, 0xFFFFFFFF on a miss.  max_dist is the walks'
 * initial closest distance (curdist / mint of the shaders, FLT_MAX there):
 * only hits at t < max_dist are taken, and boxes are pruned against it.
 * FLT_MAX gives the reference's mapping; a miss writes t = FLT_MAX either
 * way.  Must be positive (FK_ERR_INVALID otherwise). */
int fk_meshmap(fk_ctx* ctx, const fk_scene* scene, const fk_texel_map* map, int cull_backfaces, float max_dist,
               uint32_t offset, uint32_t count, fk_buf* coords, fk_buf* tidx);

/* ShaderParams of Src/solver_ao.h:67-73. */
typedef struct fk_sample_params {
  uint32_t sample_count;
  uint32_t perm_count;   /* rows of the sample table; 4096 in the reference */
  float min_distance;
  float max_distance;
} fk_sample_params;

#define FK_AO 0     /* ao_step0/1/2: 1 - occluded / spp */
#define FK_BN 1     /* bentnormals_step1/2: normalize(sum of free directions) */
#define FK_THICK 2  /* thick_step1/2: mean hit distance around -normal */
#define FK_AO_BN 3  /* AO and bent normals from one traversal (same params) */

/* Traversal strategy. */
#define FK_TRAVERSE_AUTO 0    /* tuned choice for the scene */
#define FK_TRAVERSE_ORDERED 1 /* near-first stack traversal over the BVH2 layout */
#define FK_TRAVERSE_SKIP 2    /* the reference's skip-pointer walk, node order */
#define FK_TRAVERSE_ORDERED4 3 /* near-first stack traversal over the collapsed 4-wide layout */
#define FK_TRAVERSE_MASK 0x0F
/* Ray scheduling, or-ed into the traversal argument (0 = tuned choice). */
#define FK_SCHEDULE_STATIC 0x10  /* one warp per texel, lanes = samples */
#define FK_SCHEDULE_DYNAMIC 0x20 /* lanes refilled with rays from a queue */
#define FK_SCHEDULE_MASK 0xF0
/* Divide for every ray-box slab instead of the filtered reciprocal form (the
 * dynamic schedule's default), which takes the same decisions. */
#define FK_EXACT_BOX_TESTS 0x100

/* Hemisphere sampling for texels [offset, offset + count) (global indices
 * into coords / tidx).  Outputs, indexed by texel:
 *   FK_AO    out0: float            out_hits0: occluded samples (t < max)
 *   FK_BN    out0: 3 floats (V3)    out_hits0: samples with any hit
 *   FK_THICK out0: float            out_hits0: samples with any hit
 *   FK_AO_BN out0: AO, out1: BN     out_hits0 / out_hits1 as above
 * hits buffers may be NULL.  Texels whose mapping missed get AO 1, BN (0,0,0),
 * thickness max_distance and 0 hits. */
int fk_hemisphere(fk_ctx* ctx, const fk_scene* scene, const fk_buf* coords, const fk_buf* tidx, int kind,
                  const fk_sample_params* params, const fk_buf* samples4, uint32_t offset, uint32_t count,
                  int traverse, fk_buf* out0, fk_buf* out1, fk_buf* out_hits0, fk_buf* out_hits1);

/* No counterpart in the reference.  fk_hemisphere over a texel list: the
 * texels ids[offset .. offset + count) (u32 indices into coords / tidx and
 * the outputs), each traced and written exactly as a whole-map fk_hemisphere
 * call traces and writes it (same sample permutation: texel index modulo
 * perm_count), other texels untouched.  Used for spot checks at full sample
 * count and for re-baking selected tiles.  `texel_count` bounds the ids:
 * coords / tidx / outputs must hold that many texels; the kernels skip ids
 * at or above it and flag the context, so the next fk_ctx_check reports
 * FK_ERR_DEVICE.  Dynamic schedule only (FK_SCHEDULE_STATIC is refused). */
int fk_hemisphere_texels(fk_ctx* ctx, const fk_scene* scene, const fk_buf* coords, const fk_buf* tidx,
                         uint32_t texel_count, int kind, const fk_sample_params* params, const fk_buf* samples4,
                         const fk_buf* ids, uint32_t offset, uint32_t count, int traverse, fk_buf* out0,
                         fk_buf* out1, fk_buf* out_hits0, fk_buf* out_hits1);

/* Waits for the context's stream and reads the kernels' error flags (then
 * clears them): FK_ERR_DEVICE with a message when a traversal overflowed its
 * stack, a texel named an invalid triangle or a texel list held an id out of
 * range; FK_OK otherwise. */
int fk_ctx_check(fk_ctx* ctx);

/* Gathers, Shaders/heights.comp, positions.comp, normals.comp, over texels
 * [offset, offset + count).  HEIGHT: float; POSITION / NORMAL: 3 floats.
 * Missed texels: height 0 (the shader's rule), position / normal (0,0,0). */
#define FK_GATHER_HEIGHT 0
#define FK_GATHER_POSITION 1
#define FK_GATHER_NORMAL 2
int fk_gather(fk_ctx* ctx, const fk_scene* scene, int kind, const fk_buf* coords, const fk_buf* tidx,
              uint32_t offset, uint32_t count, fk_buf* out);

/* No counterpart in the reference.  fk_hemisphere for callers that must not
 * allocate device memory during a bake (a host running one bake chunk per
 * interactive frame, or one that budgets all GPU memory through its own
 * allocator): cudaMalloc / cudaFree would stall such a caller's frame and can
 * fail under memory pressure.  It allocates nothing; its per-ray scratch is a
 * fixed array compiled into the library, held by every GPU that loads it
 * until the process exits, so one call takes at most FK_NOALLOC_MAX_RAYS
 * texels x samples (16 MiB of distances); larger requests are refused with
 * FK_ERR_INVALID and should be split over calls.  All pointers are device
 * pointers owned by the caller (coords4 / tidx as fk_meshmap writes them,
 * samples4 as fk_samples_cosine fills them, outputs as fk_hemisphere writes
 * them); `stream` is a cudaStream_t (NULL = default stream).  The scene's
 * device must be current.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and keeps it for the process, so make
 * that first call before any stream capture, and do not reset the device
 * after it.  Every call reuses the same array: calls whose work may overlap on
 * the GPU race on it and must be serialised by the caller.  Device errors (a
 * traversal that overflowed its stack, a texel naming a triangle outside the
 * scene) are recorded in the context's status word, as fk_hemisphere records
 * them: synchronise `stream`, then call fk_ctx_check, which reports them as
 * FK_ERR_DEVICE. */
#define FK_NOALLOC_MAX_RAYS (1u << 22)
int fk_hemisphere_noalloc(const fk_scene* scene, const float* coords4, const uint32_t* tidx, int kind,
                          const fk_sample_params* params, const float* samples4, uint32_t offset, uint32_t count,
                          int traverse, float* out0, float* out1, uint32_t* hits0, uint32_t* hits1, void* stream);

/* Shaders/tangentspace.comp in place over 3-float values [offset, offset+count). */
int fk_tangent_space(fk_ctx* ctx, const fk_texel_map* map, uint32_t offset, uint32_t count, fk_buf* io3);

/* ------------------------------------------------------------ MeshMapping
 * Src/meshmapping.h:42-75.  init flattens the BVH (fillMeshData), uploads the
 * pixels, mesh and nodes, and sizes the result buffers to the texel count
 * rounded up to 64 (Src/meshmapping.cpp:165).  run_step maps the next chunk
 * of work_per_step texels (0 = all remaining); *done = 1 when finished. */
int fk_meshmapping_create(fk_ctx* ctx, fk_meshmapping** out);
int fk_meshmapping_init(fk_meshmapping* mm, const fk_texel_map* map, const fk_mesh* hipoly, const fk_bvh* bvh,
                        int cull_backfaces);
int fk_meshmapping_init_scene(fk_meshmapping* mm, const fk_texel_map* map, const fk_scene* scene,
                              int cull_backfaces);
int fk_meshmapping_set_work_per_step(fk_meshmapping* mm, uint32_t texels);
int fk_meshmapping_run_step(fk_meshmapping* mm, int* done);
float fk_meshmapping_progress(const fk_meshmapping* mm);
int fk_meshmapping_results(fk_meshmapping* mm, float* coords4, uint32_t* tidx);
const fk_buf* fk_meshmapping_coords(const fk_meshmapping* mm);
const fk_buf* fk_meshmapping_tidx(const fk_meshmapping* mm);
const fk_scene* fk_meshmapping_scene(const fk_meshmapping* mm);
int fk_meshmapping_free(fk_meshmapping* mm);

/* ------------------------------------------------------------ solvers
 * One handle type for the six solvers of Src/solver_*.h.  Params mirror
 * FornosParameters_Solver* (Src/fornos.h:57-112). */
#define FK_SOLVER_HEIGHT 0
#define FK_SOLVER_POSITION 1
#define FK_SOLVER_NORMALS 2
#define FK_SOLVER_AO 3
#define FK_SOLVER_BENT_NORMALS 4
#define FK_SOLVER_THICKNESS 5

typedef struct fk_solver_params {
  int kind;                /* FK_SOLVER_* */
  uint32_t sample_count;   /* AO / BN / thickness */
  float min_distance;      /* AO / BN / thickness */
  float max_distance;      /* AO / BN / thickness; height: export range */
  int tangent_space;       /* normals / bent normals */
  int normalize_output;    /* height (export option, carried only) */
  uint32_t seed;           /* sample-table seed (std::random_device in the reference) */
  int traverse;            /* FK_TRAVERSE_* */
} fk_solver_params;

int fk_solver_create(fk_ctx* ctx, const fk_solver_params* params, fk_solver** out);
int fk_solver_init(fk_solver* s, const fk_texel_map* map, fk_meshmapping* mm);
/* Texels per run_step (0 = all remaining).  Progress is kept, so a long bake
 * advances (and can be resumed) chunk by chunk. */
int fk_solver_set_work_per_step(fk_solver* s, uint32_t texels);
int fk_solver_run_step(fk_solver* s, int* done);
float fk_solver_progress(const fk_solver* s);
/* getResults(): floats per texel (1 or 3) times the texel count rounded up to
 * 64, as the reference's result buffers are sized. */
size_t fk_solver_result_count(const fk_solver* s);
int fk_solver_results(fk_solver* s, float* host_out, size_t floats);
/* Occluder / hit counts per texel (sampling solvers only). */
int fk_solver_hits(fk_solver* s, uint32_t* host_out, size_t count);
const fk_buf* fk_solver_result_buffer(const fk_solver* s);
int fk_solver_free(fk_solver* s);

/* ------------------------------------------------------------ batched bakes
 * No counterpart in the reference (which bakes one mesh pair at a time, one
 * chunk per UI frame).  Up to 64 hemisphere jobs, each with its own scene,
 * mapped texels, sample table, parameters and outputs.  Jobs of fewer than
 * 2^21 rays share persistent launches: their rays are laid end to end and
 * every lane maps its ray back to its job, so small jobs keep the whole GPU
 * busy together.  A job of 2^21 rays or more runs alone through the
 * single-job path within the same run (and the same graph), on the batch's
 * scratch.  Results are those fk_hemisphere gives per job. */
typedef struct fk_batch fk_batch;
typedef struct fk_batch_job {
  const fk_scene* scene;
  const fk_buf* coords;      /* fk_meshmap output for the job's texels 0 .. texel_count-1 */
  const fk_buf* tidx;
  uint32_t texel_count;
  fk_sample_params params;
  const fk_buf* samples;     /* perm_count x sample_count table (fk_samples_cosine) */
  fk_buf* out0;              /* outputs as fk_hemisphere writes them for the batch's kind */
  fk_buf* out1;
  fk_buf* hits0;
  fk_buf* hits1;
} fk_batch_job;

int fk_batch_create(fk_ctx* ctx, const fk_batch_job* jobs, uint32_t job_count, int kind, fk_batch** out);
int fk_batch_info(const fk_batch* batch, uint64_t* rays, uint32_t* texels, uint32_t* launches_per_run);
/* Autotuner: times a strided sample of about sample_rays rays of every job
 * (0 = 4M) under each candidate schedule (ordered over the 2-wide or the
 * collapsed 4-wide layout vs the skip-pointer walk, filtered vs divided box
 * tests, refill threshold, postponed-leaf batch, speculation) and keeps the
 * fastest for later runs; reports it.  The ray order is the context's (a
 * strided sample has no per-texel order to time); the batch kernel runs
 * 256-thread blocks with 64-entry stacks. */
int fk_batch_tune(fk_batch* batch, uint64_t sample_rays, fk_tuning* best_tuning, int* best_traverse);
/* One run on the context's stream; traverse 0 = the tuned schedule. */
int fk_batch_run(fk_batch* batch, int traverse);
/* Records fk_batch_run into a CUDA graph; fk_batch_replay launches it. */
int fk_batch_capture(fk_batch* batch, int traverse);
int fk_batch_replay(fk_batch* batch);
int fk_batch_free(fk_batch* batch);

/* The autotuner for one fk_hemisphere call (same arguments; sample_rays 0 =
 * 16M).  It times the call's own trace kernel on eight windows of consecutive
 * texels spread over the range (about sample_rays rays, traced as the whole
 * pass traces them) and searches the knobs one group at a time from the
 * context's tuning, keeping each group's fastest: traversal layout (2-wide,
 * 4-wide, skip walk), refill x leaf batch, speculation, ray order, block
 * shape x stack depth, staged top records, L2 window.  Rays per lane follow
 * from the persistent schedule: a lane takes its next ray as soon as it
 * finishes one, and `refill` sets how many lanes a warp refills at once.
 * Apply the result with fk_ctx_set_tuning and the returned traverse flags;
 * the context's tuning is left unchanged. */
int fk_tune_hemisphere(fk_ctx* ctx, const fk_scene* scene, const fk_buf* coords, const fk_buf* tidx, int kind,
                       const fk_sample_params* params, const fk_buf* samples4, uint32_t offset, uint32_t count,
                       uint64_t sample_rays, fk_tuning* best_tuning, int* best_traverse);

/* ------------------------------------------------------------ one-shot bake
 * FornosRunner::start + run (Src/fornos.cpp:53-251) from host arrays, after
 * the host preprocessing (mesh loading, normals, BVH build, texel map): uploads
 * the flattened scene and the texel rows, runs mesh mapping and every enabled
 * solver, and copies the results back.  AO and bent normals with equal
 * sample parameters share one traversal. */
typedef struct fk_bake_sampler {
  int enabled;
  uint32_t sample_count;
  float min_distance;
  float max_distance;
  uint32_t seed;
  int tangent_space; /* bent normals only */
} fk_bake_sampler;

typedef struct fk_bake_desc {
  const fk_bvh_node* nodes;
  uint32_t node_count;
  const float* positions4;
  const float* normals4;
  uint32_t corner_count;
  uint32_t width, height, texel_count;
  const float* pix8;        /* Pix_GPUData rows */
  const float* pixt12;      /* PixT_GPUData rows */
  const uint32_t* indices;  /* texel index in the full map */
  int cull_backfaces;
  int height_enabled;
  int position_enabled;
  int normals_enabled;
  int normals_tangent_space;
  fk_bake_sampler ao;
  fk_bake_sampler bent_normals;
  fk_bake_sampler thickness;
  int traverse;             /* FK_TRAVERSE_* */
  float mapping_max_distance; /* fk_meshmap's max_dist; 0 = no limit (the reference's mapping) */
} fk_bake_desc;

/* Host outputs, texel_count rows each; NULL skips the copy. */
typedef struct fk_bake_out {
  float* coords4;
  uint32_t* tidx;
  float* height;
  float* position3;
  float* normals3;
  float* ao;
  float* bent_normals3;
  float* thickness;
} fk_bake_out;

int fk_bake(fk_ctx* ctx, const fk_bake_desc* desc, fk_bake_out* out);

/* ------------------------------------------------------------ runner
 * FornosRunner::start, then FornosRunner::run until every task has finished
 * (Src/fornos.cpp:53-251), with the fields of FornosParameters
 * (Src/fornos.h:35-123): mesh files in, image files out.  Meshes load with
 * fk_mesh_load, normals / tangents / the welded direction copy are computed
 * on the device, the texel map by fk_raster_uv, the BVH by fk_scene_build
 * (bvh_tris_per_node, depth 8192); each enabled solver's result is exported
 * as its task's finish() exports it (height: filter [0, max_distance],
 * normalize_output, dilation; positions: EXR only; normals and bent normals:
 * normal image, EXR as a vector image; AO and thickness: normalised,
 * dilation) and written by the path's extension (.png, .tga, .exr; other
 * extensions write nothing, as in the reference).  Sample tables come from
 * `seed`.  Errors: "Missing low poly mesh", "Low poly mesh is missing
 * texture coordinates or normals information" (fk_last_error). */
#define FK_NORMAL_IMPORT 0             /* NormalImport::Import */
#define FK_NORMAL_COMPUTE_PER_FACE 1   /* NormalImport::ComputePerFace */
#define FK_NORMAL_COMPUTE_PER_VERTEX 2 /* NormalImport::ComputePerVertex */
typedef struct fk_run_solver {
  int enabled;
  const char* output_path;
  uint32_t sample_count;   /* AO, bent normals, thickness */
  float min_distance;      /* AO, bent normals, thickness */
  float max_distance;      /* AO, bent normals, thickness; height: the filter's upper end */
  int tangent_space;       /* normals, bent normals */
  int normalize_output;    /* height */
} fk_run_solver;
typedef struct fk_run_params {
  const char* lo_poly_mesh_path;
  const char* hi_poly_mesh_path;  /* NULL or "": the low-poly mesh */
  int lo_poly_mesh_normal;        /* FK_NORMAL_* */
  int hi_poly_mesh_normal;
  uint32_t bvh_tris_per_node;
  uint32_t tex_width, tex_height;
  int tex_dilation;
  int ignore_backfaces;
  int mapping;                    /* FK_MAP_* (MeshMappingMethod) */
  float mapping_edge;
  fk_run_solver height, positions, normals, ao, bent_normals, thickness;
  uint32_t seed;
  int traverse;                   /* FK_TRAVERSE_* */
} fk_run_params;
/* The defaults of FornosParameters (8 triangles per node, 2048 x 2048,
 * dilation 16, back faces ignored, Smooth mapping with edge 0.05, 256
 * samples in [0.01, 10], tangent space on, height normalised). */
void fk_run_params_default(fk_run_params* params);
int fk_run(fk_ctx* ctx, const fk_run_params* params);

/* ------------------------------------------------------------ image export
 * exportFloatImage / exportNormalImage / exportVectorImage (Src/image.cpp:22-405)
 * on the device: the texel map's values (1 float per texel, or 3 for the
 * NORMAL / VECTOR modes, in the map's order) scattered into the W x H image
 * the reference writes, rows flipped (texel (x, y) in row H - y - 1):
 *   FK_EXPORT_FLOAT_RGB8   PNG / TGA path: min / max over the values, the
 *                          filter range (filter_hi > filter_lo: values outside
 *                          become 0, the range clamps the min / max), optional
 *                          normalisation, (uint8)(clamp(t, 0, 1) * 255) in all
 *                          three channels; W x H x 3 bytes;
 *   FK_EXPORT_FLOAT_F32    EXR path: clamped to the filter range, optionally
 *                          normalised; W x H floats;
 *   FK_EXPORT_NORMAL_RGB8  PNG / TGA path of normal maps: (uint8)((n * 0.5 +
 *                          0.5) * 255) per channel; W x H x 3 bytes;
 *   FK_EXPORT_VECTOR_F32   EXR path of vector maps: planes B (z), G (y), R (x);
 *                          3 x W x H floats.
 * dilate > 0 (RGB8 modes): dilateRGB's fill of uncovered pixels from the
 * nearest centre (distance < dilate, 8 directions) whose 8 neighbours are
 * covered, with the result of its row-order scan.  minmax (FLOAT modes, may be
 * NULL) gets the range used.  `image` holds at least the bytes above. */
#define FK_EXPORT_FLOAT_RGB8 0
#define FK_EXPORT_FLOAT_F32 1
#define FK_EXPORT_NORMAL_RGB8 2
#define FK_EXPORT_VECTOR_F32 3
typedef struct fk_export_params {
  int mode;
  float filter_lo, filter_hi;
  int normalize;
  int dilate;
} fk_export_params;
int fk_export_image(fk_ctx* ctx, const fk_texel_map* map, const fk_buf* data, const fk_export_params* params,
                    fk_buf* image, float* minmax);

/* Host writers of exported images (stbi_write_png / stbi_write_tga /
 * tinyexr's SaveEXRImageToFile in Src/image.cpp): an RGB8 image (rows in
 * buffer order) as PNG (".png", rows filtered and deflated at zlib level 6)
 * or TGA (".tga", run-length coded, bottom-left origin), the kinds of file
 * stb_image_write writes; float planes as a scanline EXR without
 * compression, channels "B" (1 plane) or "B", "G", "R" (3 planes), stored as
 * HALF with tinyexr's conversion (rounded up in magnitude on the first dropped
 * bit).  The decoded pixels equal the reference's files'. */
int fk_image_write_rgb8(const char* path, uint32_t width, uint32_t height, const uint8_t* rgb);
/* PNG at a chosen zlib level: 0 stores the rows unfiltered (fastest, largest),
 * 1-9 filter each row as stb_image_write does and deflate them
 * (fk_image_write_rgb8 uses 6). */
int fk_image_write_png(const char* path, uint32_t width, uint32_t height, const uint8_t* rgb, int level);
int fk_image_write_exr(const char* path, uint32_t width, uint32_t height, uint32_t planes, const float* data);

/* ------------------------------------------------------------ diagnostics
 * FP32 throughput of independent add / multiply / min chains on this device
 * (one operation counted per instruction), the denominator of the traversal
 * roofline. */
int fk_diag_fp32_peak(fk_ctx* ctx, double* ops_per_second);

/* Runs fk_hemisphere's counting variant over the same arguments (outputs go
 * to scratch) and returns the ray-box and ray-triangle tests it executed:
 * tests[0] = box tests, tests[1] = triangle tests. */
int fk_diag_traversal_counts(fk_ctx* ctx, const fk_scene* scene, const fk_buf* coords, const fk_buf* tidx, int kind,
                             const fk_sample_params* params, const fk_buf* samples4, uint32_t offset, uint32_t count,
                             int traverse, uint64_t* tests);
/* The same run's lane-utilisation profile of the dynamic schedule (8
 * counters): box tests, triangle tests, warp iterations, iterations in a leaf
 * phase, lanes doing inner work summed over inner-phase iterations, lanes
 * holding a leaf summed over leaf-phase iterations, lanes holding a ray summed
 * over all iterations, refills. */
int fk_diag_traversal_profile(fk_ctx* ctx, const fk_scene* scene, const fk_buf* coords, const fk_buf* tidx, int kind,
                              const fk_sample_params* params, const fk_buf* samples4, uint32_t offset, uint32_t count,
                              int traverse, uint64_t* counters);

/* No counterpart in the reference.  An inner tree of the scene as resident on
 * the device (FK_TREE_REFERENCE or FK_TREE_SAH): its 2-wide records, 16 words
 * each (floats 0-3 / 4-7: the left / right child's x and y bounds, 8-9 /
 * 10-11: their z bounds; ints 12 / 13: the children's refs, a record index or
 * -(flattened leaf index + 1); ints 14 / 15: leaf triangle counts), root
 * record 0, and its depth (root = 1, counting the leaf level).  records may be
 * NULL to query count and depth, else capacity (in records) must hold them
 * all.  count 0: that tree was not built for this scene. */
int fk_diag_scene_tree(fk_ctx* ctx, const fk_scene* scene, int tree, float* records, uint32_t capacity,
                       uint32_t* count, uint32_t* depth);
/* The surface-area inner tree computed on the host from a flattened node
 * array, no device needed: when its depth is at most 48 these are, bit for
 * bit, the FK_TREE_SAH records fk_scene_upload builds on the device.  count 0
 * and depth 0: a leaf box coordinate is not finite or not below 1e30 in
 * magnitude (no rebuilt tree); count 0 and depth 1: a single leaf. */
int fk_diag_sah_host(const fk_bvh_node* nodes, uint32_t node_count, float* records, uint32_t capacity,
                     uint32_t* count, uint32_t* depth);

/* ------------------------------------------------------------ learned denoiser
 * No counterpart in the reference.  A per-texel MLP that turns a low-sample
 * AO + bent-normal bake into an estimate of the full-sample one, from a 5 x 5
 * texel neighbourhood of 10 features per texel: AO, bent normal (2-D
 * octahedral), position relative to the centre texel in units of the centre's
 * texel spacing (3, clamped to +-4), interpolated normal (octahedral, 2),
 * mapping hit distance / max distance and coverage (mapping hit).  Network 250 -> 64 -> 64 -> 4 with tanh-form GELU,
 * BF16 weights and activations, FP32 accumulation; outputs are residuals: AO =
 * clamp(AO_low + y0, 0, 1), BN = normalize(BN_low + y1..3).
 *
 * Parameters (FK_DN_PARAMS fp32, row-major): W1 [64][256] (input columns
 * 250..255 are padding and held at zero), b1 [64], W2 [64 out][64 in], b2
 * [64], W3 [4][64], b3 [4].
 *
 * The feature image is 3 planes of W x H float4 (48 bytes per pixel); an input
 * row is 256 bf16 (512 bytes).  Training runs the project's own kernels:
 * forward, MSE loss on the residual targets (dAO, dBN.xyz), backward, and Adam
 * with FP32 master weights and moments. */
#define FK_DN_INPUTS 250
#define FK_DN_ROW_BYTES 512
#define FK_DN_PARAMS 20868
#define FK_DN_TILE_ROWS 128 /* training batches are multiples of this */

typedef struct fk_denoiser fk_denoiser;

int fk_denoiser_create(fk_ctx* ctx, fk_denoiser** out);
int fk_denoiser_free(fk_denoiser* d);
/* Inference kernel: FK_DN_ENGINE_TCGEN05 (the default; tcgen05.mma with
 * accumulators in tensor memory, sm_100a) or FK_DN_ENGINE_MMA_SYNC
 * (mma.sync.m16n8k16); both compute the same network in BF16 with FP32
 * accumulation, differing only in accumulation order.  Training always runs
 * the mma.sync kernels. */
#define FK_DN_ENGINE_MMA_SYNC 0
#define FK_DN_ENGINE_TCGEN05 1
int fk_denoiser_set_engine(fk_denoiser* d, int engine);
/* Host fp32 parameters in the layout above (count = FK_DN_PARAMS); setting
 * them zeroes W1's padding columns and resets the optimiser state. */
int fk_denoiser_set_params(fk_denoiser* d, const float* params, uint32_t count);
int fk_denoiser_get_params(fk_denoiser* d, float* params, uint32_t count);

/* Dense feature image (48 x W x H bytes) of a texel map's texels from a
 * low-sample AO (float) + bent normal (3 floats) bake, world positions and
 * normals (fk_gather POSITION / NORMAL) and the mapping (coords / tidx);
 * pixels without a mapping hit stay zero.  Planes: (AO, octahedral BN, 1),
 * (position / max distance, mapping distance / max distance), (octahedral
 * normal, texel spacing, 0); the spacing is the mean distance to the covered
 * 4-neighbours. */
int fk_denoise_features(fk_ctx* ctx, const fk_texel_map* map, const fk_buf* coords, const fk_buf* tidx,
                        const fk_buf* ao, const fk_buf* bn3, const fk_buf* pos3, const fk_buf* nrm3,
                        float max_distance, fk_buf* image);
/* Network input rows for `count` pixels (u32 pixel indices y * W + x). */
int fk_denoise_rows(fk_ctx* ctx, const fk_buf* image, uint32_t width, uint32_t height, const fk_buf* pixels,
                    uint32_t count, fk_buf* rows);

typedef struct {
  float learning_rate, beta1, beta2, eps;
} fk_adam;
/* One optimiser step over `batch` rows (a multiple of FK_DN_TILE_ROWS):
 * dataset rows row_ids[offset .. offset + batch) (row_ids NULL: rows offset ..
 * offset + batch) of `rows` (n_rows input rows) with float4 targets. */
int fk_denoiser_train_step(fk_denoiser* d, const fk_buf* rows, const fk_buf* targets4, uint32_t n_rows,
                           const fk_buf* row_ids, uint32_t offset, uint32_t batch, const fk_adam* adam);
/* Mean squared error over the last train step's batch (waits for it). */
int fk_denoiser_last_loss(fk_denoiser* d, double* loss);
/* The gradient of the batch's mean squared error with respect to the
 * parameters (FK_DN_PARAMS floats to the host) without updating them. */
int fk_denoiser_gradient(fk_denoiser* d, const fk_buf* rows, const fk_buf* targets4, uint32_t n_rows,
                         const fk_buf* row_ids, uint32_t offset, uint32_t batch, float* grad, double* loss);
/* Raw network outputs (float4 per row) for `count` input rows. */
int fk_denoiser_forward(fk_denoiser* d, const fk_buf* rows, uint32_t count, fk_buf* y4);
/* Denoised AO / bent normals of texels [offset, offset + count) of `map`:
 * reads the feature image and the low-sample values ao_in / bn_in (which may
 * be the output buffers themselves); texels without a mapping hit get AO 1 and
 * BN (0,0,0). */
int fk_denoise_apply(fk_denoiser* d, const fk_texel_map* map, const fk_buf* image, const fk_buf* tidx,
                     const fk_buf* ao_in, const fk_buf* bn_in, uint32_t offset, uint32_t count, fk_buf* ao_out,
                     fk_buf* bn_out);

/* The denoised AO + bent-normal bake, checked against the plain bake:
 *   1. AO + BN at low_samples over every texel;
 *   2. features, network;
 *   3. per tile of tile x tile texels, verify_cells^2 spot checks (the first
 *      texel with a mapping hit of each cell) traced at full_samples exactly
 *      as the plain bake traces them;
 *   4. tiles whose error (the larger of the AO mean absolute error and the
 *      bent normals' per-component one over the spot checks) exceeds
 *      max_tile_error are re-baked at full_samples (the plain path's values).
 * Samples tables: low_samples x perm_count and full_samples x perm_count. */
typedef struct {
  uint32_t low_samples, full_samples, perm_count;
  float min_distance, max_distance;
  uint32_t tile, verify_cells;
  float max_tile_error;
  int traverse;
} fk_denoise_params;
typedef struct {
  uint32_t tiles;           /* tiles with at least one spot check */
  uint32_t tiles_failed;    /* re-baked at full_samples */
  uint32_t spot_checks;     /* texels traced at full_samples to verify */
  uint32_t texels_rebaked;  /* texels of failed tiles */
  uint64_t rays;            /* all rays traced */
  float worst_tile_error;
} fk_denoise_stats;
int fk_denoise_bake(fk_denoiser* d, const fk_scene* scene, const fk_texel_map* map, const fk_buf* coords,
                    const fk_buf* tidx, const fk_denoise_params* params, const fk_buf* samples_low,
                    const fk_buf* samples_full, fk_buf* ao_out, fk_buf* bn_out, fk_denoise_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* FORNOS_GPU_H */
