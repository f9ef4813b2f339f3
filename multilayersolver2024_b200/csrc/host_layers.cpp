// host_layers.cpp -- CPU helpers of the step that the reference also runs on
// the host: greedy colouring (mesh setup), the strain-rate layer ordering and
// union-find layer builder (per step), and the per-layer vertex masks.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/mlxpbd.h"
#include "solver.h"

using mlx::set_error;

extern "C" {

// naiveGraphColoring (2d/tools/functionalities/naiveGraphColoring.m:1-19): the
// smallest colour not yet used by any of the tet's four vertices, tets in
// index order.  Used colours are kept as a per-vertex bitset.
int mlx_greedy_coloring(const int32_t* t, int32_t T, int32_t N, int32_t* color, int32_t* num_colors) {
  return mlx::guarded([&]() -> int {
    if (!t || !color || T < 0 || N < 0) return set_error(MLX_ERR_ARGUMENT, "bad coloring arguments");
    int words = 1;
    std::vector<uint64_t> used((size_t)N * words, 0);
    int maxc = 0;
    for (int e = 0; e < T; ++e) {
      int v[4];
      for (int k = 0; k < 4; ++k) {
        v[k] = t[e + (size_t)T * k] - 1;
        if (v[k] < 0 || v[k] >= N) return set_error(MLX_ERR_ARGUMENT, "tet vertex index out of range");
      }
      int c = -1;
      for (int w = 0; w < words && c < 0; ++w) {
        uint64_t m = used[(size_t)v[0] * words + w] | used[(size_t)v[1] * words + w] |
                     used[(size_t)v[2] * words + w] | used[(size_t)v[3] * words + w];
        if (~m) c = 64 * w + __builtin_ctzll(~m);
      }
      if (c < 0) {  // all words full: widen every vertex's bitset
        std::vector<uint64_t> wider((size_t)N * (words + 1), 0);
        for (int i = 0; i < N; ++i)
          std::memcpy(&wider[(size_t)i * (words + 1)], &used[(size_t)i * words], sizeof(uint64_t) * words);
        used.swap(wider);
        c = 64 * words;
        ++words;
      }
      for (int k = 0; k < 4; ++k) used[(size_t)v[k] * words + c / 64] |= 1ull << (c % 64);
      color[e] = c + 1;
      maxc = std::max(maxc, c + 1);
    }
    if (num_colors) *num_colors = maxc;
    return MLX_OK;
  });
}

// Per-tet strain-rate measure of buildLayers (xpbdLayer3D.m:606-608): F = B*p
// with computeB3D's row layout (entry 3*(d-1)+(j-1) of a tet's 9 rows holds
// F(d,j), computeB3D.m:26-41), read by mexEdiffNorm3D.cpp:35-61 as a
// column-major 3x3 G; the measure is ||(G'G)_a - (G'G)_b||^2 / (4 h^2) with the
// off-diagonal terms counted twice.
int mlx_strain_rate_norms(const int32_t* t, int32_t T, const double* DmInv, const double* p,
                          const double* oldp, double h, double* norms) {
  return mlx::guarded([&]() -> int {
    if (!t || !DmInv || !p || !oldp || !norms || T < 0 || !(h > 0))
      return set_error(MLX_ERR_ARGUMENT, "bad strain-rate arguments");
    const double inv_h2 = 1.0 / (h * h);
    for (int e = 0; e < T; ++e) {
      const double* g = DmInv + 9 * (size_t)e;
      int ids[4];
      for (int k = 0; k < 4; ++k) ids[k] = t[e + (size_t)T * k] - 1;
      // weights of the four vertices in column j of F
      double wgt[4][3];
      for (int j = 0; j < 3; ++j) {
        wgt[0][j] = -(g[3 * j] + g[3 * j + 1] + g[3 * j + 2]);
        wgt[1][j] = g[3 * j];
        wgt[2][j] = g[3 * j + 1];
        wgt[3][j] = g[3 * j + 2];
      }
      double Ga[9], Gb[9];  // G(i, c) at [i + 3c] = F(c, i)
      for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 3; ++i) {
          double a = 0, b = 0;
          for (int k = 0; k < 4; ++k) {
            a += wgt[k][i] * p[3 * ids[k] + c];
            b += wgt[k][i] * oldp[3 * ids[k] + c];
          }
          Ga[i + 3 * c] = a;
          Gb[i + 3 * c] = b;
        }
      auto half_gram = [](const double* G, int a, int b) {
        return (G[3 * a] * G[3 * b]) / 2.0 + (G[3 * a + 1] * G[3 * b + 1]) / 2.0 + (G[3 * a + 2] * G[3 * b + 2]) / 2.0;
      };
      static const int ca[6] = {0, 0, 1, 0, 1, 2}, cb[6] = {1, 2, 2, 0, 1, 2};
      double acc = 0;
      for (int q = 0; q < 6; ++q) {
        double d = half_gram(Ga, ca[q], cb[q]) - half_gram(Gb, ca[q], cb[q]);
        double term = inv_h2 * (d * d);
        acc += q < 3 ? term * 2.0 : term;
      }
      norms[e] = acc;
    }
    return MLX_OK;
  });
}

// mexUnionFindByVertice (2d/mex/mexUnionFindByVertice.cpp:117-178): tets are
// made rigid in `order` up to floor(pct/100*T) for each ascending layer
// percentage; rigid tets sharing a vertex form one body.  Body IDs are
// numbered 1.. by the smallest element of each body; counts per layer.
int mlx_union_find_layers(const int32_t* order, int32_t T, const double* sorted_layers, int32_t L,
                          const uint8_t* forced_elastic, const int32_t* t, int32_t N,
                          int32_t* sets, int32_t* num_rigids) {
  return mlx::guarded([&]() -> int {
    if (!order || !sorted_layers || !forced_elastic || !t || !sets || !num_rigids || T < 0 || N < 0 || L < 1)
      return set_error(MLX_ERR_ARGUMENT, "bad union-find arguments");
    std::vector<int> parent(T, -1), size(T, 1), owner(N, -1);
    int components = 0;
    auto root = [&](int x) {
      int r = x;
      while (parent[r] != r) r = parent[r];
      while (parent[x] != r) { int n = parent[x]; parent[x] = r; x = n; }
      return r;
    };
    auto unite = [&](int a, int b) {
      int ra = root(a), rb = root(b);
      if (ra == rb) return;
      if (size[ra] < size[rb]) std::swap(ra, rb);
      parent[rb] = ra;
      size[ra] += size[rb];
      --components;
    };
    std::vector<int> label(T);
    int done = 0;
    for (int l = 0; l < L; ++l) {
      if (l > 0 && sorted_layers[l] < sorted_layers[l - 1])
        return set_error(MLX_ERR_ARGUMENT, "layers must be ascending");
      int end = (int)std::floor((sorted_layers[l] / 100.0) * T);
      end = std::min(end, T);
      for (int q = done; q < end; ++q) {
        int e = order[q] - 1;
        if (e < 0 || e >= T) return set_error(MLX_ERR_ARGUMENT, "order entry out of range");
        if (forced_elastic[e] || parent[e] != -1) continue;
        parent[e] = e;
        ++components;
        for (int k = 0; k < 4; ++k) {
          int v = t[e + (size_t)T * k] - 1;
          if (v < 0 || v >= N) return set_error(MLX_ERR_ARGUMENT, "tet vertex index out of range");
          if (owner[v] >= 0) unite(e, owner[v]);
          owner[v] = e;
        }
      }
      done = std::max(done, end);
      std::fill(label.begin(), label.end(), 0);
      int next = 1;
      for (int e = 0; e < T; ++e) {
        if (parent[e] == -1) { sets[e + (size_t)T * l] = 0; continue; }
        int r = root(e);
        if (label[r] == 0) label[r] = next++;
        sets[e + (size_t)T * l] = label[r];
      }
      num_rigids[l] = components;
    }
    return MLX_OK;
  });
}

// xpbdLayer2D.findBoundaryVertices (2d/integrator/xpbdLayer2D.m:551-569): a
// vertex is rigid if it belongs to a rigid tet (its body is the last such tet
// in (corner, element) order), and a boundary vertex if it is rigid and also
// belongs to an elastic tet.
int mlx_find_boundary_vertices(const int32_t* t, int32_t T, int32_t N, const int32_t* sets, int32_t L,
                               uint8_t* is_boundary, uint8_t* is_elastic_element, uint8_t* is_rigid_vertex,
                               int32_t* vertex_rigid_body) {
  return mlx::guarded([&]() -> int {
    if (!t || !sets || !is_boundary || !is_elastic_element || !is_rigid_vertex || !vertex_rigid_body || L < 1)
      return set_error(MLX_ERR_ARGUMENT, "bad boundary arguments");
    std::vector<uint8_t> touches_elastic(N);
    for (int l = 0; l < L; ++l) {
      const int32_t* s = sets + (size_t)T * l;
      uint8_t* rig = is_rigid_vertex + (size_t)N * l;
      int32_t* body = vertex_rigid_body + (size_t)N * l;
      std::fill(rig, rig + N, 0);
      std::fill(body, body + N, 0);
      std::fill(touches_elastic.begin(), touches_elastic.end(), 0);
      for (int e = 0; e < T; ++e) is_elastic_element[e + (size_t)T * l] = s[e] == 0;
      for (int k = 0; k < 4; ++k)
        for (int e = 0; e < T; ++e) {
          int v = t[e + (size_t)T * k] - 1;
          if (v < 0 || v >= N) return set_error(MLX_ERR_ARGUMENT, "tet vertex index out of range");
          if (s[e] != 0) { rig[v] = 1; body[v] = s[e]; }
          else touches_elastic[v] = 1;
        }
      for (int v = 0; v < N; ++v) is_boundary[v + (size_t)N * l] = rig[v] && touches_elastic[v];
    }
    return MLX_OK;
  });
}

}  // extern "C"
