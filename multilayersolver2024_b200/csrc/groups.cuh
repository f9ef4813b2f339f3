// groups.cuh -- the projectGS loop of a body-free layer, one CTA per group of
// independent mesh components, vertex records in shared memory.
//
// A mesh made of several vertex-disconnected components (the scenes of a
// batch merged as Mesh3D.mergeMesh merges them, or separate objects of one
// scene) needs no ordering between components: the Gauss-Seidel order of the
// reference only orders the colours of each component.  The colour launches
// still synchronise every component at every colour.  Here a layer with a
// fixed iteration count and no rigid body (xpbdLayer3D.m:315-341: colour
// sweep, contact phase, pinning) runs as one launch in which CTA g owns the
// consecutive components of group g:
//
//  * the group's vertices are a contiguous range [v0, v1); their records
//    (x, y, z, 1/m) are copied into shared memory at the start and back at
//    the end, so a tet's four corners are gathered from and scattered to
//    shared memory (corner slots v - v0 are precomputed per tet);
//  * the tets of (colour c, group g) are a contiguous range of the layer's
//    elastic list; the colours of the group are separated by __syncthreads;
//  * each tet's rest data and multipliers (the only per-tet HBM traffic:
//    slots, DmInv, material, lambda read and write) are loaded before the
//    barrier that precedes its colour when every colour of the group fits in
//    one pass of the CTA;
//  * the contact phase (device-detected contacts of the group's vertices, or
//    the vertex groups of a host contact list) and the pinning phase run on
//    the same records.
//
// The per-tet arithmetic is tet_update of the other paths and every vertex
// sees the same sequence of updates, so results are bit-identical to the
// colour launches.
#pragma once

#include "cluster.cuh"
#include "common.cuh"
#include "contacts.cuh"
#include "persistent.cuh"
#include "tet_kernels.cuh"

namespace mlx {

constexpr int kGroupThreads = 512;

struct GroupArgs {
  const int* list;       // layer's elastic tets (sorted ids), NULL = identity
  const int* off;        // [C*G + 1] start of (colour c, group g) in list / in sorted order
  const int* gv0;        // [G + 1] vertex range of each group
  const int4* tloc;      // [T] corner slots (vertex - v0 of its group), sorted order
  const int* pin_off;    // [G + 1] range of each group in the pinned-DOF list
  const int* pin_dofs;   // 0-based DOFs, ascending
  int C, G, iterations;
  int one_per_thread;    // no (colour, group) range exceeds blockDim.x
};

// The elastic contacts of a host contact list grouped by vertex, groups in
// ascending vertex order (off / ids as elastic_contact_list_group takes them,
// vert[g] the vertex of group g).
struct HostContactGroups {
  ContactData cd;
  const int* off;
  const int* ids;
  const int* vert;
  int n;
};

// The records of one group, addressed by vertex id.
template <typename R> struct SharedPos {
  R4<R>* rec;
  int v0;
  __device__ __forceinline__ R4<R> ld(int v) const { return rec[v - v0]; }
  __device__ __forceinline__ void st(int v, R4<R> x) const { rec[v - v0] = x; }
  __device__ __forceinline__ void st_comp(int v, int c, R val) const {
    reinterpret_cast<R*>(rec + (v - v0))[c] = val;
  }
  __device__ __forceinline__ void fence() const {}
};

template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void load_group_rest(const TetData<R>& td, const GroupArgs& ga, int i,
                                                TetRest<R, MAT>& r, int4& slot) {
  const int s = ga.list ? ga.list[i] : i;
  const int T = td.T;
  r.s = s;
  if (DAMP) r.v = td.vid[s];
  slot = ga.tloc[s];
#pragma unroll
  for (int k = 0; k < 9; ++k) r.G[k] = td.dminv[(size_t)k * T + s];
  if (MAT != MAT_NH) r.vol = td.vol[s];
#pragma unroll
  for (int k = 0; k < mat_stride(MAT); ++k) r.mat[k] = td.mat[(size_t)k * T + s];
#pragma unroll
  for (int k = 0; k < num_lambda<MAT>(); ++k) r.lam[k] = td.lambda[(size_t)k * T + s];
}

template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void project_group(const TetData<R>& td, const TetRest<R, MAT>& r, int4 l,
                                              R4<R>* rec, const R4<R>* __restrict__ oldp, R inv_h2, R inv_h) {
  const R4<R> p0 = rec[l.x], p1 = rec[l.y], p2 = rec[l.z], p3 = rec[l.w];
  V3<R> X[4] = {{p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}, {p3.x, p3.y, p3.z}};
  R minv[4] = {p0.w, p1.w, p2.w, p3.w};
  R lnew[num_lambda<MAT>()];
  tet_update<R, MAT, DAMP>(r, X, minv, oldp, inv_h2, inv_h, lnew);
#pragma unroll
  for (int q = 0; q < num_lambda<MAT>(); ++q) td.lambda[(size_t)q * td.T + r.s] = lnew[q];
  rec[l.x] = make_r4<R>(X[0].x, X[0].y, X[0].z, minv[0]);
  rec[l.y] = make_r4<R>(X[1].x, X[1].y, X[1].z, minv[1]);
  rec[l.z] = make_r4<R>(X[2].x, X[2].y, X[2].z, minv[2]);
  rec[l.w] = make_r4<R>(X[3].x, X[3].y, X[3].z, minv[3]);
}

// First index in the ascending list a[0, n) whose value is >= x.
__device__ __forceinline__ int lower_bound_dev(const int* a, int n, int x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// One launch = the whole projectGS loop of one body-free layer; CTA g owns
// group g.  Dynamic shared memory: the records of the largest group.  CMODE
// (each a separate instantiation, so the reference-order kernel carries none
// of the other code): 0 = no contacts or device-detected contacts after the
// sweep; 1 = device contacts coloured with the elastic constraints; 2 = a
// host contact list (`hc`) after the sweep.
template <typename R, int MAT, bool DAMP, int CMODE = 0>
__global__ void __launch_bounds__(kGroupThreads, 1)
    k_layer_groups(TetData<R> td, GroupArgs ga, R4<R>* __restrict__ pos, const R4<R>* __restrict__ oldp,
                   R inv_h2, R inv_h, DevContacts dc, const R4<R>* __restrict__ x0, double h,
                   double contact_resistance, const R* __restrict__ pin_vals, HostContactGroups hc) {
  constexpr bool CC = CMODE == 1, HC = CMODE == 2;
  extern __shared__ __align__(32) unsigned char gr_smem[];
  R4<R>* rec = reinterpret_cast<R4<R>*>(gr_smem);
  __shared__ int crange[2];
  const int g = blockIdx.x, tid = threadIdx.x, nthr = blockDim.x;
  const int v0 = ga.gv0[g], nv = ga.gv0[g + 1] - v0;
  const SharedPos<R> sp{rec, v0};
  for (int i = tid; i < nv; i += nthr) rec[i] = ldcg_r4(pos + v0 + i);
  if (dc.nobs && tid == 0) {
    // the contact list is ascending by vertex: the group's contacts are one range
    const int n = *dc.count;
    crange[0] = lower_bound_dev(dc.verts, n, v0);
    crange[1] = lower_bound_dev(dc.verts, n, v0 + nv);
  }
  if (HC && tid == 0) {
    // the host list's vertex groups are ascending by vertex: the group's are one range
    crange[0] = lower_bound_dev(hc.vert, hc.n, v0);
    crange[1] = lower_bound_dev(hc.vert, hc.n, v0 + nv);
  }
  TetRest<R, MAT> cur;
  int4 slot = make_int4(0, 0, 0, 0);
  bool have = false;
  auto fetch = [&](int c) {
    have = false;
    if (c >= ga.C) return;
    const int beg = ga.off[c * ga.G + g], cnt = ga.off[c * ga.G + g + 1] - beg;
    if (tid < cnt) {
      load_group_rest<R, MAT, DAMP>(td, ga, beg + tid, cur, slot);
      have = true;
    }
  };
  // colours with no tet of this group are skipped, unless contact colouring
  // may have put contacts in them
  auto next_colour = [&](int c) {
    ++c;
    while (c < ga.C && !CC && ga.off[c * ga.G + g + 1] == ga.off[c * ga.G + g]) ++c;
    return c;
  };
  if (ga.one_per_thread) fetch(next_colour(-1));
  __syncthreads();
  for (int it = 0; it < ga.iterations; ++it) {
    for (int c = next_colour(-1); c < ga.C; c = next_colour(c)) {
      if (ga.one_per_thread) {
        if (have) project_group<R, MAT, DAMP>(td, cur, slot, rec, oldp, inv_h2, inv_h);
        // the next colour's rest data does not depend on positions; at the
        // last colour of an iteration the first colour of the next one
        const int nc = next_colour(c);
        fetch(nc < ga.C ? nc : (it + 1 < ga.iterations ? next_colour(-1) : ga.C));
      } else {
        const int beg = ga.off[c * ga.G + g], end = ga.off[c * ga.G + g + 1];
        for (int i = beg + tid; i < end; i += nthr) {
          TetRest<R, MAT> t;
          int4 l;
          load_group_rest<R, MAT, DAMP>(td, ga, i, t, l);
          project_group<R, MAT, DAMP>(td, t, l, rec, oldp, inv_h2, inv_h);
        }
      }
      if (CC) {
        // contact_coloring: the contacts of this colour phase touch no tet of
        // the colour, so they join its phase
        for (int i = crange[0] + tid; i < crange[1]; i += nthr)
          if (dc.vcc[dc.verts[i]] == c) elastic_contacts_of_vertex<R>(dc, i, sp, x0, h, contact_resistance);
      }
      __syncthreads();
    }
    if (dc.nobs) {
      for (int i = crange[0] + tid; i < crange[1]; i += nthr)
        if (!CC || dc.vcc[dc.verts[i]] == dc.C) elastic_contacts_of_vertex<R>(dc, i, sp, x0, h, contact_resistance);
      __syncthreads();
    }
    if (HC) {
      for (int q = crange[0] + tid; q < crange[1]; q += nthr)
        elastic_contact_list_group<R>(hc.off, hc.ids, q, sp, hc.cd, h, contact_resistance);
      __syncthreads();
    }
    const int p0 = ga.pin_off[g], p1 = ga.pin_off[g + 1];
    if (p1 > p0) {
      for (int i = p0 + tid; i < p1; i += nthr) {
        const int d = ga.pin_dofs[i];
        sp.st_comp(d / 3, d % 3, pin_vals[i]);
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < nv; i += nthr) stcg_r4(pos + v0 + i, rec[i]);
}

// ---------------------------------------------------------------------------
// The same loop when a group is too large for one CTA's pass of a colour:
// group g runs on thread-block cluster g of CS CTAs.  The group's vertex
// range [v0, v1) is split into CS contiguous spans of ceil(nv / CS) records,
// span r in the shared memory of rank r; a tet's corners are addressed by
// code (rank << 24 | slot, in GroupArgs.tloc) through distributed shared
// memory (mapa), the
// tets of (colour, group) are split across the ranks, and colours are
// separated by the hardware cluster barrier (release on arrive, acquire on
// wait), between whose two halves every thread loads its tet of the next
// colour.  Body-free layers without contacts (the batch of independent
// scenes).  Every vertex sees the same sequence of updates as with the colour
// launches, so results are bit-identical.
template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void project_cgroup(const TetData<R>& td, const TetRest<R, MAT>& r, const uint32_t a[4],
                                               const R4<R>* __restrict__ oldp, R inv_h2, R inv_h) {
  R4<R> p[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) dsm_ld(a[k], p[k]);
  V3<R> X[4] = {{p[0].x, p[0].y, p[0].z}, {p[1].x, p[1].y, p[1].z}, {p[2].x, p[2].y, p[2].z},
                {p[3].x, p[3].y, p[3].z}};
  R minv[4] = {p[0].w, p[1].w, p[2].w, p[3].w};
  R lnew[num_lambda<MAT>()];
  tet_update<R, MAT, DAMP>(r, X, minv, oldp, inv_h2, inv_h, lnew);
#pragma unroll
  for (int q = 0; q < num_lambda<MAT>(); ++q) td.lambda[(size_t)q * td.T + r.s] = lnew[q];
#pragma unroll
  for (int k = 0; k < 4; ++k) dsm_st(a[k], make_r4<R>(X[k].x, X[k].y, X[k].z, minv[k]));
}

template <typename R, int MAT, bool DAMP>
__global__ void __launch_bounds__(kGroupThreads, 1)
    k_layer_cgroups(TetData<R> td, GroupArgs ga, R4<R>* __restrict__ pos, const R4<R>* __restrict__ oldp,
                    R inv_h2, R inv_h, const R* __restrict__ pin_vals) {
  extern __shared__ __align__(32) unsigned char cg_smem[];
  R4<R>* rec = reinterpret_cast<R4<R>*>(cg_smem);
  const int rank = (int)cluster_rank(), CS = (int)cluster_size();
  const int g = (int)blockIdx.x / CS;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int v0 = ga.gv0[g], nv = ga.gv0[g + 1] - v0;
  const int span = (nv + CS - 1) / CS;
  const int my0 = min(nv, rank * span), my1 = min(nv, (rank + 1) * span);
  for (int i = my0 + tid; i < my1; i += nthr) rec[i - my0] = ldcg_r4(pos + v0 + i);
  const uint32_t base = smem_u32(rec), rb = (uint32_t)sizeof(R4<R>);
  TetRest<R, MAT> cur;
  uint32_t ca[4] = {0, 0, 0, 0};
  bool have = false;
  // ga.tloc holds the corner codes (rank << 24 | slot) on this path
  auto load = [&](int i, TetRest<R, MAT>& t, uint32_t* a) {
    int4 c;
    load_group_rest<R, MAT, DAMP>(td, ga, i, t, c);
    a[0] = vcode_addr(base, c.x, rb);
    a[1] = vcode_addr(base, c.y, rb);
    a[2] = vcode_addr(base, c.z, rb);
    a[3] = vcode_addr(base, c.w, rb);
  };
  auto fetch = [&](int c) {
    have = false;
    if (c >= ga.C) return;
    const int beg = ga.off[c * ga.G + g], cnt = ga.off[c * ga.G + g + 1] - beg;
    const int q = rank * nthr + tid;
    if (q < cnt) {
      load(beg + q, cur, ca);
      have = true;
    }
  };
  // colours with no tet of this group are skipped (the same for every rank)
  auto next_colour = [&](int c) {
    ++c;
    while (c < ga.C && ga.off[c * ga.G + g + 1] == ga.off[c * ga.G + g]) ++c;
    return c;
  };
  __syncthreads();
  cluster_arrive();
  if (ga.one_per_thread) fetch(next_colour(-1));
  cluster_wait();
  for (int it = 0; it < ga.iterations; ++it) {
    for (int c = next_colour(-1); c < ga.C; c = next_colour(c)) {
      if (ga.one_per_thread) {
        if (have) project_cgroup<R, MAT, DAMP>(td, cur, ca, oldp, inv_h2, inv_h);
      } else {
        const int beg = ga.off[c * ga.G + g], end = ga.off[c * ga.G + g + 1];
        for (int i = beg + rank * nthr + tid; i < end; i += CS * nthr) {
          TetRest<R, MAT> t;
          uint32_t a[4];
          load(i, t, a);
          project_cgroup<R, MAT, DAMP>(td, t, a, oldp, inv_h2, inv_h);
        }
      }
      cluster_arrive();
      if (ga.one_per_thread) {
        const int nc = next_colour(c);
        fetch(nc < ga.C ? nc : (it + 1 < ga.iterations ? next_colour(-1) : ga.C));
      }
      cluster_wait();
    }
    const int p0 = ga.pin_off[g], p1 = ga.pin_off[g + 1];
    if (p1 > p0) {
      for (int i = p0 + rank * nthr + tid; i < p1; i += CS * nthr) {
        const int d = ga.pin_dofs[i];
        const int off = d / 3 - v0;
        const uint32_t a = mapa_rank(base + (uint32_t)(off % span) * rb + (uint32_t)((d % 3) * sizeof(R)),
                                     (unsigned)(off / span));
        dsm_st1(a, pin_vals[i]);
      }
      cluster_arrive();
      cluster_wait();
    }
  }
  // every remote access ended at the last barrier: write this rank's span back
  for (int i = my0 + tid; i < my1; i += nthr) stcg_r4(pos + v0 + i, rec[i - my0]);
}

}  // namespace mlx
