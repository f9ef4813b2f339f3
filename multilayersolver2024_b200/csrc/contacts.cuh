// contacts.cuh -- analytic obstacles on the device: contact detection
// (simulate3D's finder loop, 3d/simulate3D.m:156-171) and the per-vertex
// contact representation of the resident stepper.
//
// A finder reports at most one contact per vertex, and simulate3D
// concatenates the finders' lists in finder order, each in ascending vertex
// order.  The device keeps, per vertex, a bit mask of the finders whose
// obstacle contains it at step start; a contact's normal and collider point
// are recomputed from the vertex's step-start position with the finder's own
// arithmetic (explicitly rounded operations, so FP64 results are the bits the
// CPU finders produce).  The contact list of the reference is the
// finder-major, order-preserving compaction of those masks.
#pragma once

#include "common.cuh"
#include "tet_kernels.cuh"

namespace mlx {

enum ObstacleType : int { OBS_PLANE = 1, OBS_SPHERE = 2, OBS_BOX = 3 };

// An obstacle prepared on the host (normalised plane normal and offset, box
// directions and half extents) exactly as the finder's constructor does.
struct Obstacle {
  int type;
  double n[3];        // plane: unit normal
  double D;           // plane: dot(raw normal, position)
  double c[3];        // sphere / box: centre
  double radius;      // sphere
  double dir[9];      // box: DirectionX, DirectionY, DirectionZ (rows)
  double half[3];     // box: HalfWidth, HalfDepth, HalfHeight
  double compliance;  // contactInfo3D.xpbdContactCompliance
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddot3(double a0, double a1, double a2, double b0, double b1, double b2) {
  return dadd(dadd(dmul(a0, b0), dmul(a1, b1)), dmul(a2, b2));
}

// contactInfo3D.xpbdContactCompliance of an obstacle's contacts: one value
// per finder (the sphere finder leaves contactInfo3D's default).
__device__ __forceinline__ double obstacle_compliance(const Obstacle& o) {
  return o.type == OBS_SPHERE ? 1e-4 : o.compliance;
}

// Contact of a point with one obstacle: PlaneContactFinder3D.findContacts
// (3d/contact/PlaneContactFinder3D.m:34-75), SphereContactFinder.findContacts
// (3d/contact/SphereContactFinder.m:24-71), PlatformContactDetector.findContacts
// (3d/contact/PlatformContactDetector.m:65-119); pointCollider = x - n phi
// (3d/contact/contactInfo3D.m:44).  Returns false when there is no contact.
__device__ __forceinline__ bool obstacle_contact(const Obstacle& o, double x, double y, double z, D3& n, D3& pt,
                                                 double& comp) {
  double phi;
  if (o.type == OBS_PLANE) {
    phi = dsub(ddot3(x, y, z, o.n[0], o.n[1], o.n[2]), o.D);
    if (!(phi <= 0.0)) return false;
    n = d3(o.n[0], o.n[1], o.n[2]);
    comp = obstacle_compliance(o);
  } else if (o.type == OBS_SPHERE) {
    const double dx = dsub(o.c[0], x), dy = dsub(o.c[1], y), dz = dsub(o.c[2], z);
    const double d = __dsqrt_rn(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)));
    if (!(d <= o.radius)) return false;
    phi = dsub(d, o.radius);
    n = d3(__ddiv_rn(dsub(x, o.c[0]), d), __ddiv_rn(dsub(y, o.c[1]), d), __ddiv_rn(dsub(z, o.c[2]), d));
    comp = obstacle_compliance(o);
  } else {
    const double ex = dsub(x, o.c[0]), ey = dsub(y, o.c[1]), ez = dsub(z, o.c[2]);
    double dots[3], ad[3];
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dots[a] = ddot3(ex, ey, ez, o.dir[3 * a], o.dir[3 * a + 1], o.dir[3 * a + 2]);
      inside = inside && fabs(dots[a]) <= o.half[a];
      ad[a] = dsub(o.half[a], fabs(dots[a]));
    }
    if (!inside) return false;
    int k = 0;  // min over the axes, first on ties
    if (ad[1] < ad[k]) k = 1;
    if (ad[2] < ad[k]) k = 2;
    phi = -ad[k];
    const double s = dots[k] > 0 ? 1.0 : (dots[k] < 0 ? -1.0 : 0.0);
    n = d3(s * o.dir[3 * k], s * o.dir[3 * k + 1], s * o.dir[3 * k + 2]);
    comp = obstacle_compliance(o);
  }
  pt = d3(dsub(x, dmul(n.x, phi)), dsub(y, dmul(n.y, phi)), dsub(z, dmul(n.z, phi)));
  return true;
}

// Elastic contacts of one vertex from a host contact list (contactConstraints
// elastic branch, xpbdLayer3D.m:426-438 + penaltyConstraint.projectElastic
// :4-28): contacts ids[off[g] .. off[g+1]) all touch one vertex; every one
// reads the same step-start position, each updates its multiplier, and the
// last one's position is kept (MATLAB's scatter).
template <typename R, typename P>
__device__ __forceinline__ void elastic_contact_list_group(const int* __restrict__ off, const int* __restrict__ ids,
                                                           int g, const P& pos, const ContactData& cd, double h,
                                                           double contact_resistance) {
  double h2 = h * h;
  int k0 = off[g], k1 = off[g + 1];
  int v = cd.vid[ids[k0]];
  R4<R> p = pos.ld(v);
  D3 x = d3((double)p.x, (double)p.y, (double)p.z);
  double minv = (double)p.w;
  D3 xn = x;
  for (int q = k0; q < k1; ++q) {
    int k = ids[q];
    D3 n = d3(cd.normal[k], cd.normal[cd.K + k], cd.normal[2 * cd.K + k]);
    D3 c = d3(cd.point[k], cd.point[cd.K + k], cd.point[2 * cd.K + k]);
    double phi = dot(n, x - c);
    if (phi > 0) phi = 0;
    double C = contact_resistance * phi;
    double aT = cd.compliance[k] / h2;
    double dl = (-C - aT * cd.lambda[k]) / (2 * minv + aT);
    cd.lambda[k] += dl;
    xn = d3(x.x + minv * (dl * n.x), x.y + minv * (dl * n.y), x.z + minv * (dl * n.z));
  }
  pos.st(v, make_r4<R>((R)xn.x, (R)xn.y, (R)xn.z, p.w));
}

// Contacts of the resident stepper for the current step.
struct DevContacts {
  int nobs;                // 0: no obstacles
  const Obstacle* obs;     // [nobs]
  const unsigned* mask;    // [N] bit f: inside obstacle f at step start
  const int* verts;        // contact vertices, ascending (compact)
  const int* cidx;         // [N] index of the vertex in verts, or -1
  const int* count;        // [1] number of contact vertices
  double* lambda;          // [count * nobs] contact multipliers of the current layer
  const int* obs_count;    // [nobs] contacts of each obstacle (its finder's list length)
  // contact_coloring: vertex v's elastic contacts run in colour phase vcc[v]
  // (C: after the sweep); cbucket lists the step's contact vertices by that
  // colour, colour c at [coff[c], coff[c + 1])
  int colored;
  int C;
  const int* vcc;          // [N]
  const int* cbucket;      // [count]
  const int* coff;         // [C + 2]
};

// Bit masks of every vertex at the step-start positions.
template <typename R>
__global__ void k_contact_mask(const R4<R>* __restrict__ x0, int N, const Obstacle* __restrict__ obs, int nobs,
                               unsigned* __restrict__ mask) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const R4<R> p = x0[v];
  unsigned m = 0;
  for (int f = 0; f < nobs; ++f) {
    D3 n, pt;
    double comp;
    if (obstacle_contact(obs[f], (double)p.x, (double)p.y, (double)p.z, n, pt, comp)) m |= 1u << f;
  }
  mask[v] = m;
}

// Order-preserving compaction, pass 1: per-block counts of the selected
// vertices (bit `f` of the mask, or any bit when f < 0).
__global__ void __launch_bounds__(256) k_compact_count(const unsigned* __restrict__ mask, int N, int f,
                                                       int* __restrict__ block_counts) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const bool sel = v < N && (f < 0 ? mask[v] != 0 : ((mask[v] >> f) & 1u));
  const int c = __syncthreads_count(sel);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = c;
}

// Pass 2 (one CTA of 1024 threads): exclusive prefix sum of the block
// counts, in place, starting at *base (0 when base is NULL); base + the sum
// lands in *total.
__global__ void __launch_bounds__(1024) k_compact_scan(int* __restrict__ block_counts, int nblocks,
                                                       const int* __restrict__ base_ptr, int* __restrict__ total) {
  __shared__ int part[1024];
  const int base = base_ptr ? *base_ptr : 0;
  const int t = threadIdx.x, per = (nblocks + blockDim.x - 1) / blockDim.x;
  const int b0 = min(t * per, nblocks), b1 = min(b0 + per, nblocks);
  int s = 0;
  for (int b = b0; b < b1; ++b) s += block_counts[b];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    const int add = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += add;
    __syncthreads();
  }
  int run = base + part[t] - s;
  for (int b = b0; b < b1; ++b) {
    const int c = block_counts[b];
    block_counts[b] = run;
    run += c;
  }
  if (t == blockDim.x - 1) *total = base + part[t];
}

// Pass 3: every selected vertex writes its rank.  out_vert[rank] = v and
// (optionally) rank_of[v] = rank, -1 for the others.
__global__ void __launch_bounds__(256) k_compact_scatter(const unsigned* __restrict__ mask, int N, int f,
                                                         const int* __restrict__ block_offsets,
                                                         int* __restrict__ out_vert, int* __restrict__ rank_of) {
  __shared__ int warp_tot[8];
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const bool sel = v < N && (f < 0 ? mask[v] != 0 : ((mask[v] >> f) & 1u));
  const unsigned bal = __ballot_sync(0xffffffffu, sel);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_tot[w] = __popc(bal);
  __syncthreads();
  int before = 0;
  for (int q = 0; q < w; ++q) before += warp_tot[q];
  const int rank = block_offsets[blockIdx.x] + before + __popc(bal & ((1u << lane) - 1u));
  if (v < N) {
    if (sel) out_vert[rank] = v;
    if (rank_of) rank_of[v] = sel ? rank : -1;
  }
}

// The reference-format contact list of finder f (contacts [off, off + K_f)):
// 1-based vertex ids, normals and collider points (K x 3, column-major with
// leading dimension ld) and compliances.
template <typename R>
__global__ void k_contact_list(const R4<R>* __restrict__ x0, const Obstacle* __restrict__ obs, int f,
                               const int* __restrict__ verts, const int* __restrict__ begin,
                               const int* __restrict__ end, int ld, int* __restrict__ vid,
                               double* __restrict__ normal, double* __restrict__ point,
                               double* __restrict__ comp) {
  const int k = *begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *end || k >= ld) return;
  const int v = verts[k];
  const R4<R> p = x0[v];
  D3 n, pt;
  double c = 0;
  obstacle_contact(obs[f], (double)p.x, (double)p.y, (double)p.z, n, pt, c);
  vid[k] = v + 1;
  normal[k] = n.x; normal[k + ld] = n.y; normal[k + 2 * ld] = n.z;
  point[k] = pt.x; point[k + ld] = pt.y; point[k + 2 * ld] = pt.z;
  comp[k] = c;
}

// Elastic contacts of one vertex (penaltyConstraint.projectElastic,
// 3d/constraints/penaltyConstraint.m:4-28, applied in contactConstraints'
// order, xpbdLayer3D.m:426-438): every contact reads the same position, each
// updates its multiplier, and the last one's position is kept.
template <typename R, typename P>
__device__ __forceinline__ void elastic_contacts_of_vertex(const DevContacts& dc, int i, const P& pos,
                                                           const R4<R>* __restrict__ x0, double h,
                                                           double contact_resistance) {
  const int v = dc.verts[i];
  const unsigned m = dc.mask[v];
  const R4<R> p = pos.ld(v);
  const R4<R> s = x0[v];
  const D3 x = d3((double)p.x, (double)p.y, (double)p.z);
  const double minv = (double)p.w, h2 = h * h;
  D3 xn = x;
  for (int f = 0; f < dc.nobs; ++f) {
    if (!((m >> f) & 1u)) continue;
    D3 n, c;
    double comp;
    obstacle_contact(dc.obs[f], (double)s.x, (double)s.y, (double)s.z, n, c, comp);
    double phi = dot(n, x - c);
    if (phi > 0) phi = 0;
    const double C = contact_resistance * phi;
    const double aT = comp / h2;
    double& lam = dc.lambda[(size_t)i * dc.nobs + f];
    const double dl = (-C - aT * lam) / (2 * minv + aT);
    lam += dl;
    xn = d3(x.x + minv * (dl * n.x), x.y + minv * (dl * n.y), x.z + minv * (dl * n.z));
  }
  pos.st(v, make_r4<R>((R)xn.x, (R)xn.y, (R)xn.z, p.w));
}

// contactVelocityUpdate (2d/integrator/xpbdLayer2D.m:577-603 as called by
// xpbdLayer3D.m:740) on the device: all contacts read the velocity after the
// step and the vertex keeps the last contact's result (MATLAB's vectorised
// v(dofs) = ...), so only the highest finder bit of a vertex matters.
template <typename R>
__global__ void k_contact_velocity(const DevContacts dc, const R4<R>* __restrict__ x0, R4<R>* __restrict__ vel,
                                   double h, double gravity, double e) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *dc.count) return;
  const int v = dc.verts[i];
  const unsigned m = dc.mask[v];
  const int f = 31 - __clz(m);
  const R4<R> s = x0[v];
  D3 n, c;
  double comp;
  obstacle_contact(dc.obs[f], (double)s.x, (double)s.y, (double)s.z, n, c, comp);
  const R4<R> u = vel[v];
  const D3 vn = d3((double)u.x, (double)u.y, (double)u.z);
  double ek = e;
  if (sqrt(dot(vn, vn)) <= 2 * gravity * h) ek = 0;
  const double vt = dot(n, vn);
  const double mn = fmin(-ek * vt, 0.0);
  vel[v] = make_r4<R>((R)(vn.x + n.x * (-vn.x + mn)), (R)(vn.y + n.y * (-vn.y + mn)), (R)(vn.z + n.z * (-vn.z + mn)),
                      u.w);
}

// Length of each finder's contact list: the vertices whose mask has bit f
// (integer atomics, so the counts are exact).  `counts` is zeroed before.
__global__ void __launch_bounds__(256) k_obstacle_counts(const unsigned* __restrict__ mask, int N, int nobs,
                                                         int* __restrict__ counts) {
  __shared__ int s[32];
  if (threadIdx.x < 32) s[threadIdx.x] = 0;
  __syncthreads();
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) {
    unsigned m = mask[v];
    while (m) {
      atomicAdd(&s[__ffs(m) - 1], 1);
      m &= m - 1;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < nobs && s[threadIdx.x]) atomicAdd(&counts[threadIdx.x], s[threadIdx.x]);
}

// The contact part of simpleEvaluateAllConstraintResiduals
// (xpbdLayer3D.m:546-586) for the device contacts, one partial sum per
// block.  The reference's correction term is the K x 1 x K implicit expansion
// of (compliance/h^2) (1x1xK) times lambda (Kx1) (xpbdLayer3D.m:581-583), so
// contact k meets the compliance of every contact j of the step; the
// compliances are one value per obstacle, so contact k's K terms are
// obs_count[g] copies of its term with obstacle g's compliance.
template <typename R>
__global__ void __launch_bounds__(256) k_contact_residual_partials(const DevContacts dc, const R4<R>* __restrict__ pos,
                                                                   const R4<R>* __restrict__ x0,
                                                                   double contact_resistance, double inv_h2_d,
                                                                   double* __restrict__ partials) {
  __shared__ double comp[32];
  __shared__ int cnt[32];
  if ((int)threadIdx.x < dc.nobs) {
    comp[threadIdx.x] = obstacle_compliance(dc.obs[threadIdx.x]);
    cnt[threadIdx.x] = dc.obs_count[threadIdx.x];
  }
  __syncthreads();
  const int K = *dc.count;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < K; i += gridDim.x * blockDim.x) {
    const int v = dc.verts[i];
    const unsigned m = dc.mask[v];
    const R4<R> p = ldcg_r4(pos + v);
    const R4<R> s0 = x0[v];
    for (int f = 0; f < dc.nobs; ++f) {
      if (!((m >> f) & 1u)) continue;
      D3 n, c;
      double cf;
      obstacle_contact(dc.obs[f], (double)s0.x, (double)s0.y, (double)s0.z, n, c, cf);
      double phi = n.x * ((double)p.x - c.x) + n.y * ((double)p.y - c.y) + n.z * ((double)p.z - c.z);
      if (phi > 0) phi = 0;
      const double a = fabs(contact_resistance * phi);
      const double lk = dc.lambda[(size_t)i * dc.nobs + f];
      for (int g = 0; g < dc.nobs; ++g) {
        if (!cnt[g]) continue;
        const double r = a - fmin(a, fabs((comp[g] * inv_h2_d) * lk));
        acc[0] += (double)cnt[g] * (r * r);
      }
    }
  }
  block_sum<1>(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

// contact_coloring, per step: the contact vertices bucketed by their colour
// phase (counts, offsets, scatter).  The order inside a bucket is free: a
// bucket holds distinct vertices, each projected by one thread.
__global__ void k_cc_hist(const DevContacts dc, int* __restrict__ hist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < *dc.count) atomicAdd(hist + dc.vcc[dc.verts[i]], 1);
}
__global__ void k_cc_offsets(const int* __restrict__ hist, int nb, int* __restrict__ off, int* __restrict__ cur) {
  if (blockIdx.x || threadIdx.x) return;
  int run = 0;
  for (int c = 0; c < nb; ++c) {
    off[c] = run;
    cur[c] = run;
    run += hist[c];
  }
  off[nb] = run;
}
__global__ void k_cc_scatter(const DevContacts dc, int* __restrict__ cur, int* __restrict__ bucket) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < *dc.count) {
    const int v = dc.verts[i];
    bucket[atomicAdd(cur + dc.vcc[v], 1)] = v;
  }
}

// One colour of the sweep with the elastic contacts of that colour phase
// (contact_coloring): CTAs [0, tet_blocks) project the colour's tets exactly
// as k_project_color, the remaining CTAs the contacts of the vertices in
// bucket `colour` (no tet of this colour touches them) that are elastic in
// this layer.
template <typename R, int MAT, bool DAMP>
__global__ void __launch_bounds__(kMaxColorTile) k_project_color_cc(TetData<R> td, const int* __restrict__ list,
                                                          int begin, int count, R4<R>* __restrict__ pos,
                                                          const R4<R>* __restrict__ oldp, R inv_h2, R inv_h,
                                                          int tet_blocks, DevContacts dc, int colour,
                                                          const int* __restrict__ vert_body,
                                                          const R4<R>* __restrict__ x0, double h,
                                                          double contact_resistance) {
  pdl_launch_dependents();
  if ((int)blockIdx.x < tet_blocks) {
    project_color_tet<R, MAT, DAMP>(td, list, begin, count, blockIdx.x * blockDim.x + threadIdx.x, pos, oldp, inv_h2,
                                    inv_h);
    return;
  }
  pdl_wait();
  const GlobalPos<R> gp{pos};
  const int b = (int)blockIdx.x - tet_blocks, stride = ((int)gridDim.x - tet_blocks) * blockDim.x;
  const int end = dc.coff[colour + 1];
  for (int q = dc.coff[colour] + b * blockDim.x + threadIdx.x; q < end; q += stride) {
    const int v = dc.cbucket[q];
    if (vert_body[v] == 0) elastic_contacts_of_vertex<R>(dc, dc.cidx[v], gp, x0, h, contact_resistance);
  }
}

}  // namespace mlx
