/*
 * A compiled consumer of include/fornos_gpu.h, built as C (C11) and as C++
 * by tests/test_abi_consumer.py: the way the reference's C++ solvers would
 * bind the library, through the header alone.
 *
 *   consumer layout             sizes and field offsets of the ABI structs
 *                               (one "name size offsets..." line each); the
 *                               test also compiles in static assertions that
 *                               the ctypes binding's layouts agree
 *   consumer host OUT           host-side calls on a generated heightfield:
 *                               mesh, vertex normals, BVH build + flatten,
 *                               sample table; arrays written to OUT
 *   consumer bake IN OUT        fk_bake on the arrays of IN (nodes, corners,
 *                               texel map), every output written to OUT
 */
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fornos_gpu.h"

#ifdef FK_LAYOUT_ASSERTS
#include FK_LAYOUT_ASSERTS
#endif

#define FIELD(T, f) (unsigned long)offsetof(T, f)

static int layout(void) {
  printf("fk_tuning %lu %lu %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_tuning),
         FIELD(fk_tuning, refill), FIELD(fk_tuning, leaf_batch), FIELD(fk_tuning, speculate),
         FIELD(fk_tuning, ray_order), FIELD(fk_tuning, top_records), FIELD(fk_tuning, l2_persist),
         FIELD(fk_tuning, block_threads), FIELD(fk_tuning, stack_depth));
  printf("fk_mesh_desc %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_mesh_desc),
         FIELD(fk_mesh_desc, position_count), FIELD(fk_mesh_desc, positions), FIELD(fk_mesh_desc, texcoord_count),
         FIELD(fk_mesh_desc, texcoords), FIELD(fk_mesh_desc, normal_count), FIELD(fk_mesh_desc, normals),
         FIELD(fk_mesh_desc, vertex_count), FIELD(fk_mesh_desc, vertices), FIELD(fk_mesh_desc, triangle_count),
         FIELD(fk_mesh_desc, triangles), FIELD(fk_mesh_desc, tangents), FIELD(fk_mesh_desc, bitangents));
  printf("fk_bvh_node %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_bvh_node), FIELD(fk_bvh_node, aabb_min),
         FIELD(fk_bvh_node, aabb_max), FIELD(fk_bvh_node, start), FIELD(fk_bvh_node, end), FIELD(fk_bvh_node, jump));
  printf("fk_scene_info %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_scene_info),
         FIELD(fk_scene_info, node_count), FIELD(fk_scene_info, corner_count), FIELD(fk_scene_info, depth),
         FIELD(fk_scene_info, leaf_count), FIELD(fk_scene_info, device_bytes));
  printf("fk_sample_params %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_sample_params),
         FIELD(fk_sample_params, sample_count), FIELD(fk_sample_params, perm_count),
         FIELD(fk_sample_params, min_distance), FIELD(fk_sample_params, max_distance));
  printf("fk_solver_params %lu %lu %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_solver_params),
         FIELD(fk_solver_params, kind), FIELD(fk_solver_params, sample_count), FIELD(fk_solver_params, min_distance),
         FIELD(fk_solver_params, max_distance), FIELD(fk_solver_params, tangent_space),
         FIELD(fk_solver_params, normalize_output), FIELD(fk_solver_params, seed), FIELD(fk_solver_params, traverse));
  printf("fk_batch_job %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_batch_job),
         FIELD(fk_batch_job, scene), FIELD(fk_batch_job, coords), FIELD(fk_batch_job, tidx),
         FIELD(fk_batch_job, texel_count), FIELD(fk_batch_job, params), FIELD(fk_batch_job, samples),
         FIELD(fk_batch_job, out0), FIELD(fk_batch_job, out1), FIELD(fk_batch_job, hits0), FIELD(fk_batch_job, hits1));
  printf("fk_bake_sampler %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_bake_sampler),
         FIELD(fk_bake_sampler, enabled), FIELD(fk_bake_sampler, sample_count), FIELD(fk_bake_sampler, min_distance),
         FIELD(fk_bake_sampler, max_distance), FIELD(fk_bake_sampler, seed), FIELD(fk_bake_sampler, tangent_space));
  printf("fk_bake_desc %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu\n",
         (unsigned long)sizeof(fk_bake_desc), FIELD(fk_bake_desc, nodes), FIELD(fk_bake_desc, node_count),
         FIELD(fk_bake_desc, positions4), FIELD(fk_bake_desc, normals4), FIELD(fk_bake_desc, corner_count),
         FIELD(fk_bake_desc, width), FIELD(fk_bake_desc, height), FIELD(fk_bake_desc, texel_count),
         FIELD(fk_bake_desc, pix8), FIELD(fk_bake_desc, pixt12), FIELD(fk_bake_desc, indices),
         FIELD(fk_bake_desc, cull_backfaces), FIELD(fk_bake_desc, height_enabled),
         FIELD(fk_bake_desc, position_enabled), FIELD(fk_bake_desc, normals_enabled),
         FIELD(fk_bake_desc, normals_tangent_space), FIELD(fk_bake_desc, ao), FIELD(fk_bake_desc, bent_normals),
         FIELD(fk_bake_desc, thickness), FIELD(fk_bake_desc, traverse), FIELD(fk_bake_desc, mapping_max_distance));
  printf("fk_bake_out %lu %lu %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_bake_out),
         FIELD(fk_bake_out, coords4), FIELD(fk_bake_out, tidx), FIELD(fk_bake_out, height),
         FIELD(fk_bake_out, position3), FIELD(fk_bake_out, normals3), FIELD(fk_bake_out, ao),
         FIELD(fk_bake_out, bent_normals3), FIELD(fk_bake_out, thickness));
  printf("fk_export_params %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_export_params),
         FIELD(fk_export_params, mode), FIELD(fk_export_params, filter_lo), FIELD(fk_export_params, filter_hi),
         FIELD(fk_export_params, normalize), FIELD(fk_export_params, dilate));
  printf("fk_run_solver %lu %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_run_solver),
         FIELD(fk_run_solver, enabled), FIELD(fk_run_solver, output_path), FIELD(fk_run_solver, sample_count),
         FIELD(fk_run_solver, min_distance), FIELD(fk_run_solver, max_distance), FIELD(fk_run_solver, tangent_space),
         FIELD(fk_run_solver, normalize_output));
  printf("fk_run_params %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu\n",
         (unsigned long)sizeof(fk_run_params), FIELD(fk_run_params, lo_poly_mesh_path),
         FIELD(fk_run_params, hi_poly_mesh_path), FIELD(fk_run_params, lo_poly_mesh_normal),
         FIELD(fk_run_params, hi_poly_mesh_normal), FIELD(fk_run_params, bvh_tris_per_node),
         FIELD(fk_run_params, tex_width), FIELD(fk_run_params, tex_height), FIELD(fk_run_params, tex_dilation),
         FIELD(fk_run_params, ignore_backfaces), FIELD(fk_run_params, mapping), FIELD(fk_run_params, mapping_edge),
         FIELD(fk_run_params, height), FIELD(fk_run_params, positions), FIELD(fk_run_params, normals),
         FIELD(fk_run_params, ao), FIELD(fk_run_params, bent_normals), FIELD(fk_run_params, thickness),
         FIELD(fk_run_params, seed), FIELD(fk_run_params, traverse));
  printf("fk_adam %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_adam), FIELD(fk_adam, learning_rate),
         FIELD(fk_adam, beta1), FIELD(fk_adam, beta2), FIELD(fk_adam, eps));
  printf("fk_denoise_params %lu %lu %lu %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_denoise_params),
         FIELD(fk_denoise_params, low_samples), FIELD(fk_denoise_params, full_samples),
         FIELD(fk_denoise_params, perm_count), FIELD(fk_denoise_params, min_distance),
         FIELD(fk_denoise_params, max_distance), FIELD(fk_denoise_params, tile), FIELD(fk_denoise_params, verify_cells),
         FIELD(fk_denoise_params, max_tile_error), FIELD(fk_denoise_params, traverse));
  printf("fk_denoise_stats %lu %lu %lu %lu %lu %lu %lu\n", (unsigned long)sizeof(fk_denoise_stats),
         FIELD(fk_denoise_stats, tiles), FIELD(fk_denoise_stats, tiles_failed), FIELD(fk_denoise_stats, spot_checks),
         FIELD(fk_denoise_stats, texels_rebaked), FIELD(fk_denoise_stats, rays),
         FIELD(fk_denoise_stats, worst_tile_error));
  return 0;
}

static int put(FILE* f, const void* p, size_t bytes) { return fwrite(p, 1, bytes, f) == bytes ? 0 : -1; }

/* A (q + 1)^2-vertex heightfield of 2 q^2 triangles over [0, 1]^2 with
 * z = ((7 i + 13 j) mod 11) / 100: exact in binary32 on every host. */
static int host(const char* out_path) {
  enum { Q = 24 };
  const uint32_t nv = (Q + 1) * (Q + 1), nt = 2 * Q * Q;
  float* pos = (float*)malloc(sizeof(float) * 3 * nv);
  float* uv = (float*)malloc(sizeof(float) * 2 * nv);
  uint32_t* vtx = (uint32_t*)malloc(sizeof(uint32_t) * 3 * nv);
  uint32_t* tri = (uint32_t*)malloc(sizeof(uint32_t) * 3 * nt);
  fk_mesh* mesh = NULL;
  fk_bvh* bvh = NULL;
  fk_bvh_node* nodes = NULL;
  float *p4 = NULL, *n4 = NULL, *samples = NULL;
  uint32_t node_count = 0, corner_count = 0, i, j, k = 0;
  int rc = -1;
  FILE* f = NULL;
  fk_mesh_desc d;
  for (j = 0; j <= Q; ++j)
    for (i = 0; i <= Q; ++i) {
      const uint32_t v = j * (Q + 1) + i;
      pos[3 * v] = (float)i / (float)Q;
      pos[3 * v + 1] = (float)j / (float)Q;
      pos[3 * v + 2] = (float)((7 * i + 13 * j) % 11) / 100.0f;
      uv[2 * v] = pos[3 * v];
      uv[2 * v + 1] = pos[3 * v + 1];
      vtx[3 * v] = v;
      vtx[3 * v + 1] = v;
      vtx[3 * v + 2] = 0;
    }
  for (j = 0; j < Q; ++j)
    for (i = 0; i < Q; ++i) {
      const uint32_t a = j * (Q + 1) + i, b = a + 1, c = a + Q + 1, e = c + 1;
      tri[k++] = a; tri[k++] = b; tri[k++] = e;
      tri[k++] = a; tri[k++] = e; tri[k++] = c;
    }
  memset(&d, 0, sizeof d);
  d.position_count = nv;
  d.positions = pos;
  d.texcoord_count = nv;
  d.texcoords = uv;
  d.normal_count = 1;
  {
    static const float up[3] = {0.0f, 0.0f, 1.0f};
    d.normals = up;
  }
  d.vertex_count = nv;
  d.vertices = vtx;
  d.triangle_count = nt;
  d.triangles = tri;
  if (fk_mesh_create(&d, &mesh) != FK_OK) goto done;
  if (fk_mesh_compute_vertex_normals(mesh) != FK_OK) goto done;
  if (fk_bvh_build(mesh, 8, 8192, &bvh) != FK_OK) goto done;
  if (fk_bvh_flatten_sizes(bvh, &node_count, &corner_count) != FK_OK) goto done;
  nodes = (fk_bvh_node*)malloc(sizeof(fk_bvh_node) * node_count);
  p4 = (float*)malloc(sizeof(float) * 4 * corner_count);
  n4 = (float*)malloc(sizeof(float) * 4 * corner_count);
  samples = (float*)malloc(sizeof(float) * 4 * 32 * 16);
  if (fk_bvh_flatten(bvh, mesh, nodes, p4, n4) != FK_OK) goto done;
  if (fk_samples_cosine(32, 16, 5, samples) != FK_OK) goto done;
  f = fopen(out_path, "wb");
  if (!f) goto done;
  if (put(f, &node_count, 4) || put(f, &corner_count, 4) || put(f, nodes, sizeof(fk_bvh_node) * node_count) ||
      put(f, p4, 16 * (size_t)corner_count) || put(f, n4, 16 * (size_t)corner_count) ||
      put(f, samples, sizeof(float) * 4 * 32 * 16))
    goto done;
  rc = 0;
done:
  if (f) fclose(f);
  if (bvh) fk_bvh_free(bvh);
  if (mesh) fk_mesh_free(mesh);
  free(pos); free(uv); free(vtx); free(tri); free(nodes); free(p4); free(n4); free(samples);
  return rc;
}

static void* grab(FILE* f, size_t bytes) {
  void* p = malloc(bytes ? bytes : 1);
  if (p && fread(p, 1, bytes, f) != bytes) {
    free(p);
    return NULL;
  }
  return p;
}

/* IN: u32 node_count, corner_count, width, height, texel_count; nodes;
 * positions4; normals4; pix8; pixt12; indices.  OUT: coords4, tidx, height,
 * position3, normals3, ao, bent_normals3, thickness. */
static int bake(const char* in_path, const char* out_path) {
  uint32_t h[5];
  fk_ctx* ctx = NULL;
  fk_bake_desc d;
  fk_bake_out o;
  int rc = -1;
  FILE* f = fopen(in_path, "rb");
  void *nodes = NULL, *p4 = NULL, *n4 = NULL, *pix8 = NULL, *pixt = NULL, *idx = NULL, *res = NULL;
  size_t n, per = 4 * 4 + 4 + 4 + 3 * 4 + 3 * 4 + 4 + 3 * 4 + 4;
  if (!f || fread(h, 4, 5, f) != 5) goto done;
  n = h[4];
  nodes = grab(f, sizeof(fk_bvh_node) * h[0]);
  p4 = grab(f, 16 * (size_t)h[1]);
  n4 = grab(f, 16 * (size_t)h[1]);
  pix8 = grab(f, 32 * n);
  pixt = grab(f, 48 * n);
  idx = grab(f, 4 * n);
  res = calloc(n ? n : 1, per);
  if (!nodes || !p4 || !n4 || !pix8 || !pixt || !idx || !res) goto done;
  memset(&d, 0, sizeof d);
  d.nodes = (const fk_bvh_node*)nodes;
  d.node_count = h[0];
  d.positions4 = (const float*)p4;
  d.normals4 = (const float*)n4;
  d.corner_count = h[1];
  d.width = h[2];
  d.height = h[3];
  d.texel_count = h[4];
  d.pix8 = (const float*)pix8;
  d.pixt12 = (const float*)pixt;
  d.indices = (const uint32_t*)idx;
  d.cull_backfaces = 1;
  d.height_enabled = d.position_enabled = d.normals_enabled = d.normals_tangent_space = 1;
  d.ao.enabled = d.bent_normals.enabled = d.thickness.enabled = 1;
  d.ao.sample_count = d.bent_normals.sample_count = d.thickness.sample_count = 64;
  d.ao.min_distance = d.bent_normals.min_distance = d.thickness.min_distance = 0.001f;
  d.ao.max_distance = d.bent_normals.max_distance = d.thickness.max_distance = 0.3f;
  d.ao.seed = d.bent_normals.seed = d.thickness.seed = 7;
  d.bent_normals.tangent_space = 1;
  d.traverse = FK_TRAVERSE_AUTO;
  {
    char* r = (char*)res;
    o.coords4 = (float*)r; r += 16 * n;
    o.tidx = (uint32_t*)r; r += 4 * n;
    o.height = (float*)r; r += 4 * n;
    o.position3 = (float*)r; r += 12 * n;
    o.normals3 = (float*)r; r += 12 * n;
    o.ao = (float*)r; r += 4 * n;
    o.bent_normals3 = (float*)r; r += 12 * n;
    o.thickness = (float*)r;
  }
  if (fk_ctx_create(0, &ctx) != FK_OK) {
    fprintf(stderr, "fk_ctx_create failed\n");
    goto done;
  }
  if (fk_bake(ctx, &d, &o) != FK_OK) {
    fprintf(stderr, "fk_bake: %s\n", fk_last_error(ctx));
    goto done;
  }
  fclose(f);
  f = fopen(out_path, "wb");
  if (!f || put(f, res, per * n)) goto done;
  rc = 0;
done:
  if (f) fclose(f);
  if (ctx) fk_ctx_destroy(ctx);
  free(nodes); free(p4); free(n4); free(pix8); free(pixt); free(idx); free(res);
  return rc;
}

int main(int argc, char** argv) {
  if (argc >= 2 && !strcmp(argv[1], "layout")) return layout();
  if (argc >= 3 && !strcmp(argv[1], "host")) return host(argv[2]) ? 1 : 0;
  if (argc >= 4 && !strcmp(argv[1], "bake")) return bake(argv[2], argv[3]) ? 1 : 0;
  fprintf(stderr, "usage: consumer layout | host OUT | bake IN OUT\n");
  return 2;
}
