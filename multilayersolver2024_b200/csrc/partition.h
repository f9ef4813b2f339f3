// partition.h -- vertex-connected mesh parts for the cluster kernel.
#pragma once

#include <cstdint>
#include <vector>

namespace mlx {

struct MeshPartition {
  int parts = 0;
  std::vector<int> vowner;   // [N] part owning each vertex
  std::vector<int> vslot;    // [N] index of the vertex among its owner's vertices
  std::vector<int> tpart;    // [T] part of each element (element order)
  std::vector<int> own;      // [N] vertices grouped by part, ascending inside a part
  std::vector<int> own_off;  // [parts + 1]
  int max_owned = 0;
};

// Splits a tet mesh (t: T x 4, column-major, 1-based) into `parts` pieces.
void partition_mesh(int N, int T, const int32_t* t, int parts, MeshPartition& out);

}  // namespace mlx
