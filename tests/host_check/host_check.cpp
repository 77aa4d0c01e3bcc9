// Runs the library's host preprocessing and writers on a seeded random mesh,
// for the sanitizer builds of the CPU tests: the mesh generators
// (fk_mesh.cpp), the BVH build with its threaded top levels and the flatten
// (fk_bvh.cpp), the surface-area inner tree built on the host (fk_tree.cpp),
// the scene upload's node checks and layout (fk_layout.cpp), the sample table
// (fk_samples_cosine) and the PNG / TGA / EXR writers with their threaded
// bands (fk_image.cpp).
//
//   host_check <seed> <triangles> <output directory>
//
// Prints "ok" and exits 0 when every call returns FK_OK; a call that fails
// prints its name and the run exits 1.
#include <cstdio>
#include <random>
#include <string>
#include <vector>

#include "../../fornos_b200/csrc/fk_internal.h"
#include "../../fornos_b200/csrc/fk_layout.h"

namespace {

bool ok(int rc, const char* what) {
  if (rc != FK_OK) std::printf("%s failed: %d\n", what, rc);
  return rc == FK_OK;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) return 2;
  std::mt19937 rng((uint32_t)std::stoul(argv[1]));
  const uint32_t nt = (uint32_t)std::stoul(argv[2]);
  const std::string dir = argv[3];
  std::uniform_real_distribution<float> u(-1.0f, 1.0f);
  // positions on a bumpy sheet, some repeated exactly (welding), a few far out
  const uint32_t np = nt / 2 + 3, nuv = np, nn = np;
  std::vector<float> pos(3 * (size_t)np), uv(2 * (size_t)nuv), nrm(3 * (size_t)nn);
  for (uint32_t i = 0; i < np; ++i) {
    pos[3 * i] = u(rng) * 10.0f, pos[3 * i + 1] = u(rng) * 10.0f, pos[3 * i + 2] = u(rng) * 0.5f;
    if (i % 97 == 5) pos[3 * i] = pos[3 * (i - 1)], pos[3 * i + 1] = pos[3 * (i - 1) + 1], pos[3 * i + 2] = pos[3 * (i - 1) + 2];
    if (i % 1009 == 7) pos[3 * i + 2] = 1e4f;
  }
  for (auto& x : uv) x = 0.5f + 0.5f * u(rng);
  for (auto& x : nrm) x = u(rng);
  std::vector<uint32_t> verts(9 * (size_t)nt), tris(3 * (size_t)nt);
  for (uint32_t t = 0; t < nt; ++t)
    for (int k = 0; k < 3; ++k) {
      const uint32_t p = (t % 53 == 1 && k == 2) ? verts[9 * (size_t)t] : rng() % np;  // some degenerate faces
      verts[9 * (size_t)t + 3 * k] = p, verts[9 * (size_t)t + 3 * k + 1] = p % nuv, verts[9 * (size_t)t + 3 * k + 2] = p % nn;
      tris[3 * (size_t)t + k] = 3 * t + k;
    }
  fk_mesh_desc d = {};
  d.position_count = np, d.positions = pos.data(), d.texcoord_count = nuv, d.texcoords = uv.data();
  d.normal_count = nn, d.normals = nrm.data(), d.vertex_count = 3 * nt, d.vertices = verts.data();
  d.triangle_count = nt, d.triangles = tris.data();
  fk_mesh* mesh = nullptr;
  if (!ok(fk_mesh_create(&d, &mesh), "fk_mesh_create")) return 1;
  int (*generators[])(fk_mesh*) = {fk_mesh_compute_face_normals, fk_mesh_compute_vertex_normals,
                                   fk_mesh_compute_vertex_normals_welded, fk_mesh_compute_tangent_space};
  for (auto g : generators) {
    fk_mesh* c = nullptr;
    if (!ok(fk_mesh_copy(mesh, &c), "fk_mesh_copy") || !ok(g(c), "mesh generator")) return 1;
    fk_mesh_free(c);
  }
  std::vector<float> samples(4 * 256 * 512);  // enough rows for the threaded fill
  if (!ok(fk_samples_cosine(256, 512, 3, samples.data()), "fk_samples_cosine")) return 1;
  for (uint32_t max_tris : {1u, 8u}) {
    fk_bvh* bvh = nullptr;
    if (!ok(fk_bvh_build(mesh, max_tris, max_tris == 1 ? 16u : 8192u, &bvh), "fk_bvh_build")) return 1;
    uint32_t nodes_n = 0, corners = 0;
    if (!ok(fk_bvh_flatten_sizes(bvh, &nodes_n, &corners), "fk_bvh_flatten_sizes")) return 1;
    std::vector<fk_bvh_node> nodes(nodes_n);
    std::vector<float> p4(4 * (size_t)corners), n4(4 * (size_t)corners);
    if (!ok(fk_bvh_flatten(bvh, mesh, nodes.data(), p4.data(), n4.data()), "fk_bvh_flatten")) return 1;
    uint32_t count = 0, depth = 0;
    if (!ok(fk_diag_sah_host(nodes.data(), nodes_n, nullptr, 0, &count, &depth), "fk_diag_sah_host")) return 1;
    std::vector<float> records(16 * (size_t)(count ? count : 1));
    if (!ok(fk_diag_sah_host(nodes.data(), nodes_n, records.data(), count, &count, &depth), "fk_diag_sah_host")) return 1;
    struct alignas(16) W { unsigned char b[16]; };
    std::vector<W> arena(fk::layout_bytes(nodes_n) / 16);
    fk::NodeLayout lay;
    const std::string bad = fk::layout_nodes(nodes.data(), nodes_n, corners, arena.data(), lay);
    if (!bad.empty()) {
      std::printf("layout_nodes failed: %s\n", bad.c_str());
      return 1;
    }
    fk_bvh_free(bvh);
  }
  fk_mesh_free(mesh);
  const uint32_t sizes[][2] = {{1, 1}, {7, 3}, {300, 41}, {1024, 700}};
  for (const auto& s : sizes) {
    const size_t px = (size_t)s[0] * s[1];
    std::vector<uint8_t> rgb(3 * px);
    std::vector<float> planes(3 * px);
    for (size_t i = 0; i < rgb.size(); ++i) rgb[i] = (uint8_t)((i * 7 + (i / 97) * 13) ^ (rng() & 3));
    for (auto& x : planes) x = u(rng) * 1000.0f;
    const std::string base = dir + "/img" + std::to_string(s[0]) + "x" + std::to_string(s[1]);
    if (!ok(fk_image_write_rgb8((base + ".png").c_str(), s[0], s[1], rgb.data()), "png") ||
        !ok(fk_image_write_png((base + "_0.png").c_str(), s[0], s[1], rgb.data(), 0), "png level 0") ||
        !ok(fk_image_write_rgb8((base + ".tga").c_str(), s[0], s[1], rgb.data()), "tga") ||
        !ok(fk_image_write_exr((base + "_1.exr").c_str(), s[0], s[1], 1, planes.data()), "exr 1") ||
        !ok(fk_image_write_exr((base + "_3.exr").c_str(), s[0], s[1], 3, planes.data()), "exr 3"))
      return 1;
  }
  std::printf("ok\n");
  return 0;
}
