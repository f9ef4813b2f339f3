// persistent.cuh -- one cooperative launch per layer.
//
// The projectGS loop of a layer with a fixed iteration count
// (xpbdLayer3D.m:315-341 without residual monitoring) runs inside a single
// kernel: every colour of the Gauss-Seidel sweep, then the body / contact
// phase, then pinning, each separated by a grid-wide barrier.  This replaces
// ~34 dependent launches per iteration by barriers on an L2-resident counter.
// All CTAs are co-resident (cooperative launch), and every wait gives up after
// kWaitNs, setting an error flag that the host reads after the step.
#pragma once

#include "body_kernels.cuh"
#include "common.cuh"
#include "tet_kernels.cuh"

namespace mlx {

constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s per barrier wait

struct GridSync {
  unsigned int* count;  // arrivals since the launch started (monotonic)
  int* error;           // 1 when a wait gave up; the launch then returns
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add_gpu(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits until *count >= target (acquire), giving up after limit_ns or when
// another waiter has set *error (which a timeout here sets).  Returns false
// when it gave up.
__device__ __forceinline__ bool wait_count_ge(const unsigned* count, unsigned target, int* error,
                                              unsigned long long limit_ns) {
  if (ld_acquire_gpu(count) >= target) return true;
  const unsigned long long t0 = global_ns();
  unsigned spins = 0;
  while (ld_acquire_gpu(count) < target) {
    if ((++spins & 255u) == 0) {
      if (*reinterpret_cast<volatile int*>(error)) return false;
      if (global_ns() - t0 > limit_ns) {
        atomicExch(error, 1);
        return false;
      }
    }
  }
  return true;
}

// Grid-wide counting barrier with a bounded wait.  Barrier number `k`
// (1, 2, ... within the launch) completes when the monotonic arrival counter
// reaches k * gridDim.x.  The CTA barrier orders this CTA's writes before the
// release-add of its arrival; the acquire load that observes the target
// orders every CTA's earlier writes before this CTA's later reads.  Returns
// false when the wait gave up (kWaitNs) or another CTA already did.
__device__ __forceinline__ bool grid_sync(const GridSync& g, unsigned& k) {
  __shared__ int ok;
  ++k;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned target = k * gridDim.x;
    red_release_add_gpu(g.count, 1u);
    ok = wait_count_ge(g.count, target, g.error, kWaitNs) ? 1 : 0;
  }
  __syncthreads();
  return ok != 0;
}

// Read-only data of one tet plus its multipliers, loaded ahead of the
// barrier that precedes its colour (nothing here depends on positions).
template <typename R, int MAT> struct TetRest {
  int s;
  int4 v;
  R G[9];
  R vol;
  R mat[mat_stride(MAT)];
  R lam[MAT == MAT_NH ? 2 : 6];
  int j;  // slot of the multipliers in shared memory (cluster kernel)
};

template <typename R, int MAT>
__device__ __forceinline__ void load_rest(const TetData<R>& td, int s, TetRest<R, MAT>& r) {
  const int T = td.T;
  r.s = s;
  r.v = td.vid[s];
#pragma unroll
  for (int j = 0; j < 9; ++j) r.G[j] = td.dminv[(size_t)j * T + s];
  if (MAT != MAT_NH) r.vol = td.vol[s];
#pragma unroll
  for (int q = 0; q < mat_stride(MAT); ++q) r.mat[q] = td.mat[(size_t)q * T + s];
#pragma unroll
  for (int q = 0; q < (MAT == MAT_NH ? 2 : 6); ++q) r.lam[q] = td.lambda[(size_t)q * T + s];
}

template <int MAT> __host__ __device__ constexpr int num_lambda() { return MAT == MAT_NH ? 2 : 6; }

// The projection of one tet whose rest data is in registers and whose four
// corner records have been gathered into X / minv: X is updated in place and
// lnew receives lambda + dlambda (xpbdLayer3D.m:358-377 for one element).
template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void tet_update(const TetRest<R, MAT>& r, V3<R> X[4], const R minv[4],
                                           const R4<R>* __restrict__ oldp, R inv_h2, R inv_h,
                                           R (&lnew)[num_lambda<MAT>()]) {
  if constexpr (MAT == MAT_NH) {
    double lam[2] = {(double)r.lam[0], (double)r.lam[1]}, dl[2];
    nh_project<R>(X, minv, r.G, (double)r.mat[0], (double)r.mat[1], (double)inv_h2, lam, dl);
    lnew[0] = (R)(lam[0] + dl[0]);
    lnew[1] = (R)(lam[1] + dl[1]);
  } else {
    Compliance<R> cm;
    load_compliance<R, MAT>(r.mat, 0, 1, inv_h2, inv_h, cm, DAMP);
    R dl[6];
    V3<R> Xo[4];
    if (DAMP) {
      const int4 v = r.v;
      R4<R> o0 = oldp[v.x], o1 = oldp[v.y], o2 = oldp[v.z], o3 = oldp[v.w];
      Xo[0] = {o0.x, o0.y, o0.z}; Xo[1] = {o1.x, o1.y, o1.z};
      Xo[2] = {o2.x, o2.y, o2.z}; Xo[3] = {o3.x, o3.y, o3.z};
    }
    stvk_project<R, MAT, DAMP>(X, Xo, minv, r.G, r.vol, cm, r.lam, dl);
#pragma unroll
    for (int q = 0; q < 6; ++q) lnew[q] = r.lam[q] + dl[q];
  }
}

// project_tet with the rest data already in registers.
template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void project_loaded(const TetData<R>& td, const TetRest<R, MAT>& r,
                                               R4<R>* __restrict__ pos, const R4<R>* __restrict__ oldp,
                                               R inv_h2, R inv_h) {
  const int4 v = r.v;
  R4<R> p0 = ldcg_r4(pos + v.x), p1 = ldcg_r4(pos + v.y), p2 = ldcg_r4(pos + v.z), p3 = ldcg_r4(pos + v.w);
  V3<R> X[4] = {{p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}, {p3.x, p3.y, p3.z}};
  R minv[4] = {p0.w, p1.w, p2.w, p3.w};
  R lnew[num_lambda<MAT>()];
  tet_update<R, MAT, DAMP>(r, X, minv, oldp, inv_h2, inv_h, lnew);
#pragma unroll
  for (int q = 0; q < num_lambda<MAT>(); ++q) td.lambda[(size_t)q * td.T + r.s] = lnew[q];
  stcg_r4(pos + v.x, make_r4<R>(X[0].x, X[0].y, X[0].z, minv[0]));
  stcg_r4(pos + v.y, make_r4<R>(X[1].x, X[1].y, X[1].z, minv[1]));
  stcg_r4(pos + v.z, make_r4<R>(X[2].x, X[2].y, X[2].z, minv[2]));
  stcg_r4(pos + v.w, make_r4<R>(X[3].x, X[3].y, X[3].z, minv[3]));
}

struct PersistArgs {
  const int* list;        // elastic tets of the layer (colour-sorted ids), NULL = identity
  const int* cstart;      // [C] start of each colour in `list` (or in sorted order)
  const int* ccount;      // [C] tets of each colour in this layer
  int C;
  int iterations;
  int body_work;          // run the body / elastic-contact phase
  const int* pin_dofs;    // 0-based DOFs
  int npin;
  int one_per_thread;     // every colour fits in the grid (enables the prefetch)
};

template <typename R, int MAT, bool DAMP>
__global__ void __launch_bounds__(128) k_layer_persistent(TetData<R> td, PersistArgs pa, R4<R>* __restrict__ pos,
                                                          const R4<R>* __restrict__ oldp, R inv_h2, R inv_h,
                                                          LayerDev L, Body* __restrict__ bodies,
                                                          const double4* __restrict__ ri,
                                                          const double* __restrict__ vmass,
                                                          double* __restrict__ lamB, ContactData cd, double h,
                                                          double boundary_compliance, double contact_resistance,
                                                          int use_rigid_contacts, const R* __restrict__ pin_vals,
                                                          GridSync gs) {
  __shared__ Body sb;
  __shared__ double invI[9];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  unsigned k = 0;  // barriers passed
  // With at most one tet of a colour per thread (pa.one_per_thread) the next
  // colour's rest data is loaded before the barrier that precedes it.
  TetRest<R, MAT> cur;
  bool have = false;
  auto fetch = [&](int c) {
    have = false;
    if (c < pa.C && tid < pa.ccount[c]) {
      int i = pa.cstart[c] + tid;
      load_rest<R, MAT>(td, pa.list ? pa.list[i] : i, cur);
      have = true;
    }
  };
  for (int it = 0; it < pa.iterations; ++it) {
    if (pa.one_per_thread) fetch(0);
    for (int c = 0; c < pa.C; ++c) {
      const int count = pa.ccount[c];
      if (count == 0) continue;
      if (pa.one_per_thread) {
        if (have) project_loaded<R, MAT, DAMP>(td, cur, pos, oldp, inv_h2, inv_h);
        int nc = c + 1;
        while (nc < pa.C && pa.ccount[nc] == 0) ++nc;
        fetch(nc);
      } else {
        const int begin = pa.cstart[c];
        for (int i = tid; i < count; i += nthreads) {
          int s = pa.list ? pa.list[begin + i] : begin + i;
          project_tet<R, MAT, DAMP>(td, s, pos, oldp, inv_h2, inv_h);
        }
      }
      if (!grid_sync(gs, k)) return;
    }
    if (pa.body_work) {
      for (int b = blockIdx.x; b < L.nb; b += gridDim.x)
        body_iteration<R>(L, b, bodies, GlobalPos<R>{pos}, ri, vmass, lamB, cd, h, boundary_compliance, contact_resistance,
                          use_rigid_contacts, sb, invI);
      for (int g = tid; g < L.n_ec_groups; g += nthreads) elastic_contact_group<R>(L, g, GlobalPos<R>{pos}, cd, h, contact_resistance);
      if (!grid_sync(gs, k)) return;
    }
    if (pa.npin) {
      for (int i = tid; i < pa.npin; i += nthreads) {
        int d = pa.pin_dofs[i];
        GlobalPos<R>{pos}.st_comp(d / 3, d % 3, pin_vals[i]);
      }
      if (!grid_sync(gs, k)) return;
    }
  }
}

}  // namespace mlx
