// partition.cpp -- vertex-connected mesh parts for the cluster kernel.
//
// The parts only decide which CTA of a cluster holds which vertex record and
// projects which tets of a colour; any split gives the same results, a
// compact one keeps most corner accesses inside the CTA's own shared memory.
// No geometry is needed: vertices are ordered breadth-first over the
// vertex-tet incidence graph from a pseudo-peripheral vertex (the last vertex
// reached by a first sweep), which lays a beam or a block out in level-set
// slabs, and that order is cut into `parts` runs of equal incident-tet count.
// A tet belongs to the part that owns most of its corners (ties: the lower
// part).
#include "partition.h"

#include <algorithm>

namespace mlx {

namespace {

// Breadth-first order of the component containing `start`; returns the
// last vertex reached.
int bfs(int start, const std::vector<int>& vt_off, const std::vector<int>& vt, const int32_t* t, int T,
        std::vector<char>& seen, std::vector<int>& order) {
  size_t head = order.size();
  order.push_back(start);
  seen[start] = 1;
  int last = start;
  while (head < order.size()) {
    int v = order[head++];
    last = v;
    for (int q = vt_off[v]; q < vt_off[v + 1]; ++q) {
      int e = vt[q];
      for (int k = 0; k < 4; ++k) {
        int u = t[e + (size_t)T * k] - 1;
        if (!seen[u]) {
          seen[u] = 1;
          order.push_back(u);
        }
      }
    }
  }
  return last;
}

}  // namespace

void partition_mesh(int N, int T, const int32_t* t, int parts, MeshPartition& out) {
  out.parts = parts;
  // vertex -> tets incidence (CSR)
  std::vector<int> vt_off(N + 1, 0), vt(4 * (size_t)T);
  for (int e = 0; e < T; ++e)
    for (int k = 0; k < 4; ++k) ++vt_off[t[e + (size_t)T * k]];
  for (int v = 0; v < N; ++v) vt_off[v + 1] += vt_off[v];
  {
    std::vector<int> fill(vt_off.begin(), vt_off.end() - 1);
    for (int e = 0; e < T; ++e)
      for (int k = 0; k < 4; ++k) vt[fill[t[e + (size_t)T * k] - 1]++] = e;
  }
  // breadth-first order, component by component
  std::vector<int> order;
  order.reserve(N);
  std::vector<char> seen(N, 0), probe(N, 0);
  for (int v0 = 0; v0 < N; ++v0) {
    if (seen[v0]) continue;
    std::vector<int> tmp;
    int far = bfs(v0, vt_off, vt, t, T, probe, tmp);
    bfs(far, vt_off, vt, t, T, seen, order);
  }
  // cut into runs of equal incident-tet weight (isolated vertices weigh 1)
  long long W = 0;
  for (int v = 0; v < N; ++v) W += std::max(vt_off[v + 1] - vt_off[v], 1);
  out.vowner.assign(N, 0);
  long long acc = 0;
  for (int v : order) {
    int p = (int)((acc * parts) / std::max<long long>(W, 1));
    out.vowner[v] = std::min(p, parts - 1);
    acc += std::max(vt_off[v + 1] - vt_off[v], 1);
  }
  // owned lists and slots
  out.own_off.assign(parts + 1, 0);
  for (int v = 0; v < N; ++v) ++out.own_off[out.vowner[v] + 1];
  for (int p = 0; p < parts; ++p) out.own_off[p + 1] += out.own_off[p];
  out.own.assign(N, 0);
  out.vslot.assign(N, 0);
  {
    std::vector<int> fill(out.own_off.begin(), out.own_off.end() - 1);
    for (int v = 0; v < N; ++v) {
      int p = out.vowner[v];
      out.vslot[v] = fill[p] - out.own_off[p];
      out.own[fill[p]++] = v;
    }
  }
  out.max_owned = 0;
  for (int p = 0; p < parts; ++p) out.max_owned = std::max(out.max_owned, out.own_off[p + 1] - out.own_off[p]);
  // element parts: majority owner of the corners
  out.tpart.assign(T, 0);
  for (int e = 0; e < T; ++e) {
    int o[4];
    for (int k = 0; k < 4; ++k) o[k] = out.vowner[t[e + (size_t)T * k] - 1];
    int best = o[0], bestn = 0;
    for (int a = 0; a < 4; ++a) {
      int n = 0;
      for (int b = 0; b < 4; ++b) n += o[b] == o[a];
      if (n > bestn || (n == bestn && o[a] < best)) {
        best = o[a];
        bestn = n;
      }
    }
    out.tpart[e] = best;
  }
}

}  // namespace mlx
