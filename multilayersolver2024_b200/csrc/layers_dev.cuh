// layers_dev.cuh -- buildLayers and findBoundaryVertices on the device.
//
// xpbdLayer3D.buildLayers (xpbdLayer3D.m:601-619) orders the tets by a
// strain-rate measure (mexEdiffNorm3D, sort ascending, stable) and
// mexUnionFindByVertice makes the first floor(pct/100*T) tets of that order
// rigid for each ascending layer percentage, rigid tets that share a vertex
// forming one body, bodies numbered 1.. by their smallest element;
// xpbdLayer2D.findBoundaryVertices (xpbdLayer2D.m:551-569) then derives the
// per-layer vertex masks.  Here:
//
//  * the strain-rate measure uses explicitly rounded FP64 operations in the
//    order of the host restatement, so the measures (and hence the order)
//    are the same bits;
//  * the stable ascending sort is a radix sort of (measure, element) pairs;
//  * the components are found by lock-free union-find over the tets: every
//    vertex names its smallest incident rigid tet and each rigid tet is
//    united with the representative of each of its corners, a union always
//    hooking the larger root under the smaller, so every root is the
//    smallest element of its body; an exclusive scan of the roots in element
//    order gives the reference's numbering;
//  * a vertex's body is the set of its last rigid tet in (corner, element)
//    order (an atomic max over corner*T + element).
//
// Tets are visited in colour-sorted order (s), identified by their element
// id e = s2e[s]; corners come from the sorted vertex-id array.
#pragma once

#include "common.cuh"

namespace mlx {

constexpr int kUfMaxSteps = 1 << 22;  // bound of every union-find loop (never reached by a valid forest)

__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }

// mexEdiffNorm3D's measure of one tet (xpbdLayer3D.m:606-608,
// 3d/mex/mexEdiffNorm3D.cpp:35-61): F = B p for the current and the
// step-start positions, ||(F'F)/2 differences||^2 / h^2 with the off-diagonal
// entries counted twice.  dminv is the mesh's DmInv, 9 values per element.
__global__ void k_strain_rate_norms(const int4* __restrict__ vid, const int* __restrict__ s2e, int T,
                                    const double* __restrict__ dminv, const double* __restrict__ p,
                                    const double* __restrict__ oldp, double inv_h2, double* __restrict__ norms,
                                    int* __restrict__ elems) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= T) return;
  const int e = s2e[s];
  const int4 v4 = vid[s];
  const int ids[4] = {v4.x, v4.y, v4.z, v4.w};
  const double* g = dminv + 9 * (size_t)e;
  double wgt[4][3];
  for (int j = 0; j < 3; ++j) {
    wgt[0][j] = -rn_add(rn_add(g[3 * j], g[3 * j + 1]), g[3 * j + 2]);
    wgt[1][j] = g[3 * j];
    wgt[2][j] = g[3 * j + 1];
    wgt[3][j] = g[3 * j + 2];
  }
  double Ga[9], Gb[9];
  for (int c = 0; c < 3; ++c)
    for (int i = 0; i < 3; ++i) {
      double a = 0, b = 0;
      for (int k = 0; k < 4; ++k) {
        a = rn_add(a, rn_mul(wgt[k][i], p[3 * ids[k] + c]));
        b = rn_add(b, rn_mul(wgt[k][i], oldp[3 * ids[k] + c]));
      }
      Ga[i + 3 * c] = a;
      Gb[i + 3 * c] = b;
    }
  auto half_gram = [](const double* G, int a, int b) {
    return rn_add(rn_add(__ddiv_rn(rn_mul(G[3 * a], G[3 * b]), 2.0), __ddiv_rn(rn_mul(G[3 * a + 1], G[3 * b + 1]), 2.0)),
                  __ddiv_rn(rn_mul(G[3 * a + 2], G[3 * b + 2]), 2.0));
  };
  const int ca[6] = {0, 0, 1, 0, 1, 2}, cb[6] = {1, 2, 2, 0, 1, 2};
  double acc = 0;
  for (int q = 0; q < 6; ++q) {
    const double d = rn_sub(half_gram(Ga, ca[q], cb[q]), half_gram(Gb, ca[q], cb[q]));
    const double term = rn_mul(inv_h2, rn_mul(d, d));
    acc = rn_add(acc, q < 3 ? rn_mul(term, 2.0) : term);
  }
  norms[e] = acc;
  elems[e] = e;
}

// Position of every element in the order (0-based).
__global__ void k_order_rank(const int* __restrict__ order, int T, int* __restrict__ rank) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < T) rank[order[q]] = q;
}

// A layer's rigid tets: the first `end` of the order that are not forced
// elastic.  parent = e for a rigid tet, -1 otherwise; rep[v] = INT_MAX.
__global__ void k_uf_init(const int* __restrict__ rank, const uint8_t* __restrict__ forced, int T, int end,
                          int* __restrict__ parent) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < T) parent[e] = (rank[e] < end && !forced[e]) ? e : -1;
}

// Smallest rigid tet at every vertex.
__global__ void k_uf_rep(const int4* __restrict__ vid, const int* __restrict__ s2e, int T,
                         const int* __restrict__ parent, int* __restrict__ rep) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= T) return;
  const int e = s2e[s];
  if (parent[e] < 0) return;
  const int4 v = vid[s];
  atomicMin(rep + v.x, e);
  atomicMin(rep + v.y, e);
  atomicMin(rep + v.z, e);
  atomicMin(rep + v.w, e);
}

__device__ __forceinline__ int uf_find(volatile int* parent, int x, int* err) {
  for (int n = 0; n < kUfMaxSteps; ++n) {
    const int p = parent[x];
    if (p == x) return x;
    const int gp = parent[p];
    if (gp != p) parent[x] = gp;  // path halving (values only move towards the root)
    x = p;
  }
  atomicExch(err, 1);
  return x;
}

__global__ void k_uf_unite(const int4* __restrict__ vid, const int* __restrict__ s2e, int T, int* parent,
                           const int* __restrict__ rep, int* err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= T) return;
  const int e = s2e[s];
  if (((volatile int*)parent)[e] < 0) return;
  const int4 v4 = vid[s];
  const int vs[4] = {v4.x, v4.y, v4.z, v4.w};
  for (int k = 0; k < 4; ++k) {
    int a = e, b = rep[vs[k]];
    for (int n = 0; n < kUfMaxSteps; ++n) {
      a = uf_find((volatile int*)parent, a, err);
      b = uf_find((volatile int*)parent, b, err);
      if (a == b) break;
      if (a < b) {
        const int t = a;
        a = b;
        b = t;
      }
      // hook the larger root under the smaller one
      if (atomicCAS(parent + a, a, b) == a) break;
      if (n + 1 == kUfMaxSteps) atomicExch(err, 1);
    }
  }
}

// Roots (the smallest element of each body) flagged for the scan.
__global__ void k_uf_roots(int T, int* parent, int* __restrict__ root, int* __restrict__ flag, int* err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= T) return;
  if (parent[e] < 0) {
    root[e] = -1;
    flag[e] = 0;
    return;
  }
  const int r = uf_find((volatile int*)parent, e, err);
  root[e] = r;
  flag[e] = r == e;
}

// sets(:, l) of mexUnionFindByVertice: body number of every rigid tet.
__global__ void k_uf_label(int T, const int* __restrict__ root, const int* __restrict__ scan,
                           int32_t* __restrict__ sets) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= T) return;
  const int r = root[e];
  sets[e] = r < 0 ? 0 : scan[r] + 1;
}

// findBoundaryVertices of one layer: key[v] = max corner*T + element over the
// rigid tets of v (-1: none); touch[v] = 1 when an elastic tet has v.
__global__ void k_bv_keys(const int4* __restrict__ vid, const int* __restrict__ s2e, int T,
                          const int32_t* __restrict__ sets, int* __restrict__ key, int* __restrict__ touch) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= T) return;
  const int e = s2e[s];
  const int4 v4 = vid[s];
  const int vs[4] = {v4.x, v4.y, v4.z, v4.w};
  if (sets[e] != 0) {
    for (int k = 0; k < 4; ++k) atomicMax(key + vs[k], k * T + e);
  } else {
    for (int k = 0; k < 4; ++k) touch[vs[k]] = 1;
  }
}

__global__ void k_bv_masks(int N, int T, const int32_t* __restrict__ sets, const int* __restrict__ key,
                           const int* __restrict__ touch, uint8_t* __restrict__ is_boundary,
                           uint8_t* __restrict__ is_rigid, int32_t* __restrict__ body) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const int k = key[v];
  const bool rig = k >= 0;
  is_rigid[v] = rig;
  body[v] = rig ? sets[k % T] : 0;
  is_boundary[v] = rig && touch[v];
}

__global__ void k_elastic_mask(int T, const int32_t* __restrict__ sets, uint8_t* __restrict__ is_elastic) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < T) is_elastic[e] = sets[e] == 0;
}

}  // namespace mlx
