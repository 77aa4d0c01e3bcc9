// Host side of the scene upload over a flattened node array (fk_bvh_node, the
// layout of fillMeshData, Src/meshmapping.cpp:62-125): the checks that keep
// every kernel inside the skip-pointer structure, the device node arrays and
// the reference tree's 2-wide inner records, split over host threads.  Plain
// C++ (no CUDA types), so the CPU tests compile it on its own.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/fornos_gpu.h"

namespace fk {

struct NodeLayout {
  // In the caller's arena (layout_bytes):
  // per node, 4 floats each: the box minimum (maximum), then the node's first
  // (one-past-last) triangle corner as bits: the device's node_lo / node_hi
  float* lo = nullptr;
  float* hi = nullptr;
  uint32_t* jump = nullptr;  // skip pointers: the node after the subtree
  // per inner node, 16 floats: the boxes of its two children as
  // (lx, hx, ly, hy) x2 and (lz, hz) x2, then the children's refs and triangle
  // counts as bits (an inner child: its record index, count 0; a leaf child:
  // -(node index + 1), its triangle count)
  float* wide = nullptr;
  std::vector<uint32_t> leaf_ids;  // flattened indices of the leaves, ascending
  uint32_t leaves = 0;
  uint32_t wide_count = 0;  // inner nodes
  uint32_t depth = 1;       // nodes on the longest root-to-leaf path
  bool sah_ok = true;       // every leaf box within the surface-area tree's coordinate range
  bool coords_ok = true;    // every box within +-2^24 with its faces in order (the filtered box tests)
};

// Bytes of the arena layout_nodes lays nn nodes out in (16-byte aligned): the
// node arrays, the inner records (a checked tree of nn nodes has (nn - 1) / 2
// inner nodes) and the pass's own record numbering.
size_t layout_bytes(uint32_t nn);

// Checks and lays out nodes[0 .. nn) over nc triangle corners into `arena`
// (layout_bytes(nn) bytes, 16-byte aligned; the scene upload passes pinned
// memory, so that the copies to the device need no staging).  Returns an
// empty string on success, else the message of the defect that a scan in
// node order meets first: a node outside the array or with a corner range
// not in whole triangles, a node with both children and triangles, node 0
// not spanning the array, then an inner node whose children do not split its
// subtree.  threads 0: as many as the host has, up to 16 (one below 2^16
// nodes); the result does not depend on it.
std::string layout_nodes(const fk_bvh_node* nodes, uint32_t nn, uint32_t nc, void* arena, NodeLayout& out,
                         unsigned threads = 0);

}  // namespace fk
