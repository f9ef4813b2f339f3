// cluster.cuh -- the projectGS loop of one layer inside one thread-block
// cluster, vertex records in distributed shared memory.
//
// A layer with a fixed iteration count (xpbdLayer3D.m:315-341 without residual
// monitoring) is a chain of short dependent phases: every colour of the
// Gauss-Seidel sweep, the boundary/contact phase, pinning.  On B200 a kernel
// boundary or a software grid barrier between two phases costs more than the
// phase itself for a mesh of ~1e5 tets.  Here one cluster of up to 16 CTAs
// (one per SM) runs the whole loop:
//
//  * the mesh is split into `CS` vertex-connected parts (one per CTA rank) and
//    tets are sorted by (colour, part), so the tets a CTA projects in a
//    colour are a contiguous range;
//  * every CTA keeps, in its shared memory, a record (x, y, z, 1/m) for each
//    vertex its tets touch.  A tet writes its corners into its own CTA's
//    records only and reads each corner from the record of the vertex's
//    previous writer in colour order, wherever that is (ld.shared::cluster
//    through mapa); the slots are fixed per layer on the host.  No CTA ever
//    stores into another CTA's shared memory during the sweep, so a barrier's
//    release waits only for local stores;
//  * the multipliers of a CTA's tets stay in its shared memory for the whole
//    launch;
//  * phases are separated by the hardware cluster barrier
//    (barrier.cluster.arrive.release / wait.acquire) -- no spin loop;
//  * between the arrive and the wait of a barrier every thread loads the
//    read-only data of its tet of the next colour (ids, DmInv, volume,
//    material, multipliers), so those loads overlap the barrier.
//
// Positions are copied from global memory into the cluster at the start of
// the launch and back at the end.  Results are bit-identical to the colour
// launches: the order of tets inside a colour does not change any value.
#pragma once

#include "body_kernels.cuh"
#include "common.cuh"
#include "persistent.cuh"
#include "tet_kernels.cuh"

namespace mlx {

constexpr int kClusterMaxThreads = 384;

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// Every thread of every CTA of the cluster executes the same sequence of
// arrive/wait pairs (the loops below are uniform across the cluster).
__device__ __forceinline__ void cluster_arrive() {
  __syncwarp();
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  __syncwarp();
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// address of the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t mapa_rank(uint32_t a, unsigned rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}

__device__ __forceinline__ void dsm_ld(uint32_t a, float4& v) {
  asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a) : "memory");
}
__device__ __forceinline__ void dsm_ld(uint32_t a, double4& v) {
  asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a) : "memory");
  asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.z), "=d"(v.w) : "r"(a + 16) : "memory");
}
__device__ __forceinline__ void dsm_st(uint32_t a, float4 v) {
  asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};"
               ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
}
__device__ __forceinline__ void dsm_st(uint32_t a, double4 v) {
  asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x), "d"(v.y) : "memory");
  asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(a + 16), "d"(v.z), "d"(v.w) : "memory");
}
__device__ __forceinline__ void dsm_st1(uint32_t a, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void dsm_st1(uint32_t a, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}

// Vertex code: (rank << 24) | slot in that CTA's record array.
__device__ __forceinline__ uint32_t vcode_addr(uint32_t base, int code, uint32_t rec_bytes) {
  return mapa_rank(base + (uint32_t)(code & 0xffffff) * rec_bytes, (unsigned)code >> 24);
}

// Vertex records of the cluster addressed by vertex id, at each vertex's
// home slot (body, contact and pinning phases).
template <typename R> struct ClusterPos {
  const int* vcode;  // [N] home codes
  uint32_t base;     // shared address of the record array (same offset in every CTA)
  __device__ __forceinline__ uint32_t addr(int v) const {
    return vcode_addr(base, __ldg(vcode + v), (uint32_t)sizeof(R4<R>));
  }
  __device__ __forceinline__ R4<R> ld(int v) const {
    R4<R> x;
    dsm_ld(addr(v), x);
    return x;
  }
  __device__ __forceinline__ void st(int v, R4<R> x) const { dsm_st(addr(v), x); }
  __device__ __forceinline__ void st_comp(int v, int c, R val) const {
    dsm_st1(addr(v) + (uint32_t)(c * sizeof(R)), val);
  }
  // records may live in another CTA: make the stores visible at cluster
  // scope before the CTA barrier that precedes their readers
  __device__ __forceinline__ void fence() const { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }
};

__device__ __forceinline__ void sm_st(uint32_t a, float4 v) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}
__device__ __forceinline__ void sm_st(uint32_t a, double4 v) {
  asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x), "d"(v.y) : "memory");
  asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a + 16), "d"(v.z), "d"(v.w) : "memory");
}

struct ClusterArgs {
  const int* list;      // layer's elastic tets (sorted ids) in (colour, part) order; NULL = identity
  const int* off;       // [C*CS + 1] start of (colour c, rank r) in list / in sorted order
  const int* lbase;     // [C*CS] first shared-memory multiplier slot of (colour c, rank r)
  const int* colours;   // [nC] colours with at least one elastic tet in this layer
  int nC;
  const int4* tsrc;     // [list] codes of the slots each corner is read from (previous writer)
  const int2* tdst;     // [list] own-CTA slots the corners are written to (16 bits each)
  const int* vhome;     // [N] home codes
  const int* home_v;    // vertices grouped by the rank of their home slot
  const int* home_s;    // their home slots
  const int* home_off;  // [CS + 1]
  int rec_slots;        // vertex slots per CTA (the multipliers follow them)
  int lam_slots;        // multiplier slots per component; 0 = multipliers stay in global memory
  int iterations;
  int body_work;
  const int* pin_dofs;  // 0-based DOFs
  int npin;
  int one_per_thread;   // no (colour, rank) range exceeds blockDim.x: prefetch the next colour
};

template <typename R, int MAT> struct ClRest {
  TetRest<R, MAT> r;
  uint32_t a[4];  // cluster addresses the corners are read from
  uint32_t d[4];  // shared (CTA) addresses the corners are written to
};

// Rest data of the tet at list position i (sorted id s, multiplier slot j),
// its multipliers and the addresses of its corner records.
template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void load_cl_rest(const TetData<R>& td, const ClusterArgs& ca, int i, int s, int j,
                                             uint32_t base, const R* lam_s, ClRest<R, MAT>& q) {
  const int T = td.T;
  q.r.s = s;
  q.r.j = j;
  if (DAMP) q.r.v = td.vid[s];
#pragma unroll
  for (int k = 0; k < 9; ++k) q.r.G[k] = td.dminv[(size_t)k * T + s];
  if (MAT != MAT_NH) q.r.vol = td.vol[s];
#pragma unroll
  for (int k = 0; k < mat_stride(MAT); ++k) q.r.mat[k] = td.mat[(size_t)k * T + s];
  if (ca.lam_slots) {
#pragma unroll
    for (int k = 0; k < num_lambda<MAT>(); ++k) q.r.lam[k] = lam_s[k * ca.lam_slots + j];
  } else {
#pragma unroll
    for (int k = 0; k < num_lambda<MAT>(); ++k) q.r.lam[k] = td.lambda[(size_t)k * T + s];
  }
  const int4 c = ca.tsrc[i];
  const int2 w = ca.tdst[i];
  const uint32_t rb = (uint32_t)sizeof(R4<R>);
  q.a[0] = vcode_addr(base, c.x, rb);
  q.a[1] = vcode_addr(base, c.y, rb);
  q.a[2] = vcode_addr(base, c.z, rb);
  q.a[3] = vcode_addr(base, c.w, rb);
  q.d[0] = base + (uint32_t)(w.x & 0xffff) * rb;
  q.d[1] = base + (uint32_t)((unsigned)w.x >> 16) * rb;
  q.d[2] = base + (uint32_t)(w.y & 0xffff) * rb;
  q.d[3] = base + (uint32_t)((unsigned)w.y >> 16) * rb;
}

template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void project_cl(const TetData<R>& td, const ClusterArgs& ca, const ClRest<R, MAT>& q,
                                           R* lam_s, const R4<R>* __restrict__ oldp, R inv_h2, R inv_h) {
  R4<R> p[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) dsm_ld(q.a[k], p[k]);
  V3<R> X[4] = {{p[0].x, p[0].y, p[0].z}, {p[1].x, p[1].y, p[1].z}, {p[2].x, p[2].y, p[2].z},
                {p[3].x, p[3].y, p[3].z}};
  R minv[4] = {p[0].w, p[1].w, p[2].w, p[3].w};
  R lnew[num_lambda<MAT>()];
  tet_update<R, MAT, DAMP>(q.r, X, minv, oldp, inv_h2, inv_h, lnew);
#pragma unroll
  for (int k = 0; k < 4; ++k) sm_st(q.d[k], make_r4<R>(X[k].x, X[k].y, X[k].z, minv[k]));
  if (ca.lam_slots) {
#pragma unroll
    for (int k = 0; k < num_lambda<MAT>(); ++k) lam_s[k * ca.lam_slots + q.r.j] = lnew[k];
  } else {
#pragma unroll
    for (int k = 0; k < num_lambda<MAT>(); ++k) td.lambda[(size_t)k * td.T + q.r.s] = lnew[k];
  }
}

// One launch = one cluster = the whole projectGS loop of one layer.
// Dynamic shared memory of every CTA: rec_slots vertex records, then (when
// lam_slots > 0) num_lambda x lam_slots multipliers of the CTA's own tets.
template <typename R, int MAT, bool DAMP>
__global__ void __launch_bounds__(kClusterMaxThreads, 1)
    k_layer_cluster(TetData<R> td, ClusterArgs ca, R4<R>* __restrict__ pos, const R4<R>* __restrict__ oldp,
                    R inv_h2, R inv_h, LayerDev L, Body* __restrict__ bodies, const double4* __restrict__ ri,
                    const double* __restrict__ vmass, double* __restrict__ lamB, ContactData cd, double h,
                    double boundary_compliance, double contact_resistance, int use_rigid_contacts,
                    const R* __restrict__ pin_vals) {
  extern __shared__ __align__(32) unsigned char cl_smem[];
  __shared__ Body sb;
  __shared__ double invI[9];
  R4<R>* rec = reinterpret_cast<R4<R>*>(cl_smem);
  R* lam_s = reinterpret_cast<R*>(rec + ca.rec_slots);
  const unsigned rank = cluster_rank(), CS = cluster_size();
  const int tid = threadIdx.x, nthr = blockDim.x;
  const uint32_t base = smem_u32(rec);
  const ClusterPos<R> cp{ca.vhome, base};
  constexpr int NL = num_lambda<MAT>();

  // fill this CTA's home slots and multipliers from global memory
  const int h0 = ca.home_off[rank], h1 = ca.home_off[rank + 1];
  for (int i = h0 + tid; i < h1; i += nthr) rec[ca.home_s[i]] = ldcg_r4(pos + ca.home_v[i]);
  if (ca.lam_slots) {
    for (int q = 0; q < ca.nC; ++q) {
      const int c = ca.colours[q];
      const int beg = ca.off[c * CS + rank], end = ca.off[c * CS + rank + 1], lb = ca.lbase[c * CS + rank];
      for (int i = beg + tid; i < end; i += nthr) {
        const int s = ca.list ? ca.list[i] : i;
#pragma unroll
        for (int k = 0; k < NL; ++k) lam_s[k * ca.lam_slots + lb + (i - beg)] = td.lambda[(size_t)k * td.T + s];
      }
    }
  }
  __syncthreads();

  ClRest<R, MAT> cur;
  bool have = false;
  // phase k of the sweep sequence (iteration k / nC, colour ca.colours[k % nC])
  auto fetch = [&](int k) {
    have = false;
    if (k >= ca.iterations * ca.nC) return;
    const int c = ca.colours[k % ca.nC];
    const int beg = ca.off[c * CS + rank], cnt = ca.off[c * CS + rank + 1] - beg;
    if (tid < cnt) {
      const int i = beg + tid;
      load_cl_rest<R, MAT, DAMP>(td, ca, i, ca.list ? ca.list[i] : i, ca.lbase[c * CS + rank] + tid, base, lam_s,
                                 cur);
      have = true;
    }
  };
  cluster_arrive();
  if (ca.one_per_thread) fetch(0);
  cluster_wait();

  int k = 0;
  for (int it = 0; it < ca.iterations; ++it) {
    for (int q = 0; q < ca.nC; ++q, ++k) {
      if (ca.one_per_thread) {
        if (have) project_cl<R, MAT, DAMP>(td, ca, cur, lam_s, oldp, inv_h2, inv_h);
      } else {
        const int c = ca.colours[q];
        const int beg = ca.off[c * CS + rank], end = ca.off[c * CS + rank + 1], lb = ca.lbase[c * CS + rank];
        for (int i = beg + tid; i < end; i += nthr) {
          ClRest<R, MAT> t;
          load_cl_rest<R, MAT, DAMP>(td, ca, i, ca.list ? ca.list[i] : i, lb + (i - beg), base, lam_s, t);
          project_cl<R, MAT, DAMP>(td, ca, t, lam_s, oldp, inv_h2, inv_h);
        }
      }
      cluster_arrive();
      if (ca.one_per_thread) fetch(k + 1);
      cluster_wait();
    }
    if (ca.body_work) {
      for (int b = (int)rank; b < L.nb; b += (int)CS)
        body_iteration<R>(L, b, bodies, cp, ri, vmass, lamB, cd, h, boundary_compliance, contact_resistance,
                          use_rigid_contacts, sb, invI);
      for (int g = (int)rank * nthr + tid; g < L.n_ec_groups; g += (int)CS * nthr)
        elastic_contact_group<R>(L, g, cp, cd, h, contact_resistance);
      cluster_arrive();
      cluster_wait();
    }
    if (ca.npin) {
      for (int i = (int)rank * nthr + tid; i < ca.npin; i += (int)CS * nthr) {
        const int d = ca.pin_dofs[i];
        cp.st_comp(d / 3, d % 3, pin_vals[i]);
      }
      cluster_arrive();
      cluster_wait();
    }
  }
  // every remote access ended at the last barrier: write the home slots and
  // the multipliers back
  for (int i = h0 + tid; i < h1; i += nthr) stcg_r4(pos + ca.home_v[i], rec[ca.home_s[i]]);
  if (ca.lam_slots) {
    for (int q = 0; q < ca.nC; ++q) {
      const int c = ca.colours[q];
      const int beg = ca.off[c * CS + rank], end = ca.off[c * CS + rank + 1], lb = ca.lbase[c * CS + rank];
      for (int i = beg + tid; i < end; i += nthr) {
        const int s = ca.list ? ca.list[i] : i;
#pragma unroll
        for (int k = 0; k < NL; ++k) td.lambda[(size_t)k * td.T + s] = lam_s[k * ca.lam_slots + lb + (i - beg)];
      }
    }
  }
}

}  // namespace mlx
