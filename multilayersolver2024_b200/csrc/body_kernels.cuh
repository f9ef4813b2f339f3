// body_kernels.cuh -- rigid-layer kernels (FP64 body state on every path).
//
// One thread group owns one rigid body: its vertex, boundary-vertex and
// rigid-contact lists are contiguous CSR ranges, the per-body sums of the
// reference's accumarray calls become fixed-order reductions over the group
// (deterministic), and the body update (expRodrigues, R <- dR R,
// I <- R I0 R') runs on the group's first thread between two barriers.  In
// the per-body kernels the group is a whole CTA for a body of more than
// kSmallBody vertices and one warp otherwise (eight bodies per 256-thread
// CTA), chosen per body from its own size, so a body's arithmetic never
// depends on the other bodies of the layer (a scene steps bit-identically
// alone or inside a batch).  Elastic contacts, which touch no body, ride in
// the extra CTAs of the same launch.
#pragma once

#include "common.cuh"
#include "contacts.cuh"
#include "tet_kernels.cuh"

namespace mlx {

// Device description of one layer (built on the host from the layer masks).
struct LayerDev {
  int nb;                   // bodies in this layer
  const int* body_vert_off; // [nb+1] CSR over body_verts
  const int* body_verts;    // rigid vertices grouped by body, ascending
  const int* bnd_off;       // [nb+1] CSR over bnd_verts
  const int* bnd_verts;     // boundary vertices grouped by body, ascending
  const int* rc_off;        // [nb+1] CSR over rc_ids
  const int* rc_ids;        // rigid contact ids grouped by body, ascending
  int any_boundary;         // the layer has at least one boundary vertex
  int any_rigid_contact;    // the layer has at least one rigid contact
  const int* vert_body;     // [N] 1-based body of each vertex, 0 = elastic
  const unsigned char* vert_rigid;  // [N] isRigidVertex
  int n_ec_groups;          // elastic contacts grouped by vertex, ascending vertex
  const int* ec_off;        // [n_ec_groups+1]
  const int* ec_ids;        // contact ids, ascending inside a group
  const int* ec_vert;       // [n_ec_groups] the vertex of each group
  int n_items;              // CTAs of the per-body kernels
  const int* items;         // [n_items][kItemInts]: see body_of_item
};

// Bodies of at most kSmallBody vertices are owned by one warp.
constexpr int kSmallBody = 128;
constexpr int kBodyThreads = 256;                 // CTA size of the per-body kernels
constexpr int kItemInts = kBodyThreads / 32;      // one body per warp, or one large body
constexpr int kLargeItem = -2;                    // item[1] marking a CTA-wide body

// Deterministic sum of NV doubles over a warp (xor butterfly: at every stage
// both lanes of a pair add the same two operands, so all lanes hold the same
// bits).
template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
  for (int q = 0; q < NV; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
}

// The thread group that owns a body.
struct CtaGroup {
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int size() const { return blockDim.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  template <int NV> __device__ __forceinline__ void sum(double (&v)[NV]) const { block_sum<NV>(v); }
};
struct WarpGroup {
  __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
  __device__ __forceinline__ int size() const { return 32; }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
  template <int NV> __device__ __forceinline__ void sum(double (&v)[NV]) const { warp_sum<NV>(v); }
};

// Body of this thread in a per-body kernel (kBodyThreads threads per CTA):
// item[1] == kLargeItem gives body item[0] to the whole CTA (returns 1);
// otherwise warp w owns body item[w] (returns 0; -1 = no body).
__device__ __forceinline__ int body_of_item(const LayerDev& L, int& b) {
  const int* it = L.items + (size_t)kItemInts * blockIdx.x;
  if (it[1] == kLargeItem) {
    b = it[0];
    return 1;
  }
  b = it[threadIdx.x >> 5];
  return 0;
}

__device__ __forceinline__ D3 solve3_piv(const double* Mcm, D3 b) {
  double A[3][3], bb[3] = {b.x, b.y, b.z}, x[3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) A[r][c] = Mcm[r + 3 * c];
  solve3x3<double>(A, bb, x);
  return d3(x[0], x[1], x[2]);
}

__device__ __forceinline__ void mm3(const double* A, const double* B, double* C) {  // C = A*B
  double t[9];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) t[r + 3 * c] = A[r] * B[3 * c] + A[r + 3] * B[1 + 3 * c] + A[r + 6] * B[2 + 3 * c];
#pragma unroll
  for (int i = 0; i < 9; ++i) C[i] = t[i];
}
__device__ __forceinline__ void mm3_bt(const double* A, const double* B, double* C) {  // C = A*B'
  double t[9];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) t[r + 3 * c] = A[r] * B[c] + A[r + 3] * B[c + 3] + A[r + 6] * B[c + 6];
#pragma unroll
  for (int i = 0; i < 9; ++i) C[i] = t[i];
}

// expRodrigues (3d/tools/math/expRodrigues.m:1-15)
__device__ __forceinline__ void exp_rodrigues(D3 w, double h, double* R) {
  double mag = sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
  double u[3] = {w.x / mag, w.y / mag, w.z / mag};
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (isnan(u[i])) u[i] = 0;
  double th = h * mag;
  double K[9] = {0, u[2], -u[1], -u[2], 0, u[0], u[1], -u[0], 0}, K2[9];
  mm3(K, K, K2);
  double s = sin(th), c1 = 1 - cos(th);
#pragma unroll
  for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0 ? 1.0 : 0.0) + s * K[i] + c1 * K2[i];
}

__device__ __forceinline__ D3 body_point(const Body& b, const double4& r) {
  return mv3(b.R, d3(r.x, r.y, r.z)) + d3(b.com[0], b.com[1], b.com[2]);
}

template <typename R, typename P>
__device__ __forceinline__ void store_xyz(const P& pos, int v, D3 x) {
  R4<R> p = pos.ld(v);
  pos.st(v, make_r4<R>((R)x.x, (R)x.y, (R)x.z, p.w));
}
template <typename R>
__device__ __forceinline__ void store_xyz(R4<R>* pos, int v, D3 x) {
  store_xyz<R>(GlobalPos<R>{pos}, v, x);
}

// AdaptiveMesh3D.makeRigidsFromConnectivity (AdaptiveMesh3D.m:32-43) ->
// RigidBody3D.matComputeRigidBodyProperties3D (RigidBody3D.m:198-247):
// mass, COM, COM velocity, inertia, angular momentum and omega = I \ L, with
// the residual velocity as vertex velocity; writes ri = p - COM.
template <typename R, typename G>
__device__ __forceinline__ void make_rigid(const LayerDev& L, int b, Body* __restrict__ bodies,
                                           const R4<R>* __restrict__ pos, const R4<R>* __restrict__ resv,
                                           const double* __restrict__ vmass, double4* __restrict__ ri, const G& g) {
  int beg = L.body_vert_off[b], end = L.body_vert_off[b + 1];
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = beg + g.rank(); i < end; i += g.size()) {
    int v = L.body_verts[i];
    double m = vmass[v];
    R4<R> p = pos[v], u = resv[v];
    s[0] += m;
    s[1] += (double)p.x * m; s[2] += (double)p.y * m; s[3] += (double)p.z * m;
    s[4] += (double)u.x * m; s[5] += (double)u.y * m; s[6] += (double)u.z * m;
  }
  g.template sum<7>(s);
  double M = s[0];
  D3 com = d3(s[1] / M, s[2] / M, s[3] / M), cdot = d3(s[4] / M, s[5] / M, s[6] / M);
  double t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // Ixx Iyy Izz Ixy Ixz Iyz Lx Ly Lz
  for (int i = beg + g.rank(); i < end; i += g.size()) {
    int v = L.body_verts[i];
    double m = vmass[v];
    R4<R> p = pos[v], u = resv[v];
    D3 r = d3((double)p.x, (double)p.y, (double)p.z) - com;
    D3 vd = d3((double)u.x, (double)u.y, (double)u.z) - cdot;
    ri[v] = make_double4(r.x, r.y, r.z, 0.0);
    double nm = -m;  // -m .* ([r]x [r]x)  (RigidBody3D.m:251)
    t[0] += nm * (-(r.z * r.z) - r.y * r.y);
    t[1] += nm * (-(r.z * r.z) - r.x * r.x);
    t[2] += nm * (-(r.y * r.y) - r.x * r.x);
    t[3] += nm * (r.y * r.x);
    t[4] += nm * (r.z * r.x);
    t[5] += nm * (r.z * r.y);
    D3 c = cross(r, vd);
    t[6] += m * c.x; t[7] += m * c.y; t[8] += m * c.z;
  }
  g.template sum<9>(t);
  if (g.rank() == 0) {
    Body& B = bodies[b];
    double I0[9] = {t[0], t[3], t[4], t[3], t[1], t[5], t[4], t[5], t[2]};
    D3 w = solve3_piv(I0, d3(t[6], t[7], t[8]));
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      B.I0[i] = I0[i];
      B.I[i] = I0[i];
      B.R[i] = (i % 4 == 0) ? 1.0 : 0.0;
      B.Rstep[i] = B.R[i];
    }
    B.com[0] = com.x; B.com[1] = com.y; B.com[2] = com.z;
    B.comdot[0] = cdot.x; B.comdot[1] = cdot.y; B.comdot[2] = cdot.z;
    B.omega[0] = w.x; B.omega[1] = w.y; B.omega[2] = w.z;
    B.mass = M;
  }
}

template <typename R>
__global__ void __launch_bounds__(kBodyThreads) k_make_rigids(LayerDev L, Body* __restrict__ bodies,
                                                              const R4<R>* __restrict__ pos,
                                                              const R4<R>* __restrict__ resv,
                                                              const double* __restrict__ vmass,
                                                              double4* __restrict__ ri) {
  int b;
  if (body_of_item(L, b)) make_rigid<R>(L, b, bodies, pos, resv, vmass, ri, CtaGroup{});
  else if (b >= 0) make_rigid<R>(L, b, bodies, pos, resv, vmass, ri, WarpGroup{});
}

// Release all elastic residual (xpbdLayer3D.m:138-139).
template <typename R>
__global__ void k_release_elastic(R4<R>* __restrict__ pos, R4<R>* __restrict__ resv,
                                  const unsigned char* __restrict__ vert_rigid, int N, R h) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N || vert_rigid[v]) return;
  R4<R> p = pos[v], u = resv[v];
  pos[v] = make_r4<R>(p.x + h * u.x, p.y + h * u.y, p.z + h * u.z, p.w);
  resv[v] = make_r4<R>(0, 0, 0, 0);
}

// RigidBody3D.rigidSymplecticImperativeStep (RigidBody3D.m:174-179), the
// re-placement of rigid vertices (xpbdLayer3D.m:147) and the residual rebase
// resv = R_step resv - (x - xprev)/h (xpbdLayer3D.m:149-158).
template <typename R, typename G>
__device__ __forceinline__ void rigid_step(const LayerDev& L, int b, Body* __restrict__ bodies, R4<R>* __restrict__ pos,
                                           const R4<R>* __restrict__ xprev, R4<R>* __restrict__ resv,
                                           const double4* __restrict__ ri, double h, Body& sb, const G& g) {
  if (g.rank() == 0) {
    Body B = bodies[b];
    for (int d = 0; d < 3; ++d) B.com[d] += h * B.comdot[d];
    double dR[9], tmp[9];
    exp_rodrigues(d3(B.omega[0], B.omega[1], B.omega[2]), h, dR);
    mm3(dR, B.R, B.R);
    mm3(B.R, B.I0, tmp);
    mm3_bt(tmp, B.R, B.I);
    for (int i = 0; i < 9; ++i) B.Rstep[i] = B.R[i];
    bodies[b] = B;
    sb = B;
  }
  g.sync();
  int beg = L.body_vert_off[b], end = L.body_vert_off[b + 1];
  for (int i = beg + g.rank(); i < end; i += g.size()) {
    int v = L.body_verts[i];
    D3 x = body_point(sb, ri[v]);
    R4<R> p = pos[v];
    R4<R> q = make_r4<R>((R)x.x, (R)x.y, (R)x.z, p.w);
    pos[v] = q;
    R4<R> u = resv[v], xp = xprev[v];
    D3 rot = mv3(sb.Rstep, d3((double)u.x, (double)u.y, (double)u.z));
    double rx = ((double)q.x - (double)xp.x) / h;
    double ry = ((double)q.y - (double)xp.y) / h;
    double rz = ((double)q.z - (double)xp.z) / h;
    resv[v] = make_r4<R>((R)(rot.x - rx), (R)(rot.y - ry), (R)(rot.z - rz), 0);
  }
}

template <typename R>
__global__ void __launch_bounds__(kBodyThreads) k_rigid_step(LayerDev L, Body* __restrict__ bodies,
                                                             R4<R>* __restrict__ pos,
                                                             const R4<R>* __restrict__ xprev,
                                                             R4<R>* __restrict__ resv,
                                                             const double4* __restrict__ ri, double h) {
  __shared__ Body sb[kItemInts];
  int b;
  if (body_of_item(L, b)) rigid_step<R>(L, b, bodies, pos, xprev, resv, ri, h, sb[0], CtaGroup{});
  else if (b >= 0) rigid_step<R>(L, b, bodies, pos, xprev, resv, ri, h, sb[threadIdx.x >> 5], WarpGroup{});
}

// rigidGeneralizedInverseMass (3d/constraints/rigidGeneralizedInverseMass.m):
// w = 1/M + (r x n)' I^-1 (r x n), with I^-1 formed once per body update
// (the reference solves I \ axis per vertex; the results agree to rounding).
__device__ __forceinline__ double gen_inv_mass(double invM, D3 r, const double* invI, D3 n) {
  D3 axis = cross(r, n);
  return invM + dot(axis, mv3(invI, axis));
}

// inverse of a 3x3 column-major matrix by columns of a pivoted solve
__device__ __forceinline__ void inverse3(const double* A, double* inv) {
  for (int c = 0; c < 3; ++c) {
    D3 e = d3(c == 0, c == 1, c == 2);
    D3 col = solve3_piv(A, e);
    inv[3 * c] = col.x; inv[3 * c + 1] = col.y; inv[3 * c + 2] = col.z;
  }
}

// Inverse of a body's world inertia (column-major) by its adjugate: one
// division and independent products, a short dependent chain for the thread
// that updates the body (the inertia of a cluster is well conditioned; the
// results agree with a pivoted solve to rounding).
__device__ __forceinline__ void inertia_inverse(const double* A, double* inv) {
  const double a00 = A[0], a10 = A[1], a20 = A[2], a01 = A[3], a11 = A[4], a21 = A[5], a02 = A[6], a12 = A[7],
               a22 = A[8];
  const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
  const double c10 = a02 * a21 - a01 * a22, c11 = a00 * a22 - a02 * a20, c12 = a01 * a20 - a00 * a21;
  const double c20 = a01 * a12 - a02 * a11, c21 = a02 * a10 - a00 * a12, c22 = a00 * a11 - a01 * a10;
  const double r = 1.0 / (a00 * c00 + a01 * c01 + a02 * c02);
  // inv(row, col) = C(col, row) / det, column-major
  inv[0] = c00 * r; inv[1] = c01 * r; inv[2] = c02 * r;
  inv[3] = c10 * r; inv[4] = c11 * r; inv[5] = c12 * r;
  inv[6] = c20 * r; inv[7] = c21 * r; inv[8] = c22 * r;
}

// Per-body update after an accumulation (xpbdLayer3D.m:401-414, 466-479):
// omega = I \ dL with I's inverse `invI` (the reference's solve, to rounding).
__device__ __forceinline__ void apply_increments(Body& B, const double* s, double h, const double* invI) {
  for (int d = 0; d < 3; ++d) B.com[d] += s[d];
  D3 w = mv3(invI, d3(s[3], s[4], s[5]));
  double dR[9], tmp[9];
  exp_rodrigues(w, h, dR);
  mm3(dR, B.R, B.R);
  mm3_bt(B.I0, B.R, tmp);
  mm3(B.R, tmp, B.I);
}

// Elastic contacts of one vertex of the layer's host contact list
// (elastic_contact_list_group over the layer's vertex groups).
template <typename R, typename P>
__device__ __forceinline__ void elastic_contact_group(const LayerDev& L, int g, const P& pos,
                                                      const ContactData& cd, double h, double contact_resistance) {
  elastic_contact_list_group<R>(L.ec_off, L.ec_ids, g, pos, cd, h, contact_resistance);
}

// One iteration of one rigid body, run by a whole CTA: the rigid-elastic glue
// of its boundary vertices (rigidElasticBoundaryAccumulationConstraints,
// xpbdLayer3D.m:381-420 + rigidBoundaryConstraint.m:4-35) and then its rigid
// contacts (contactConstraints rigid branch, xpbdLayer3D.m:440-484 +
// penaltyConstraint.projectRigid :30-63), Jacobi style as in the reference.
// All bodies are updated whenever the layer has any boundary vertex / rigid
// contact, as the reference's vectorised update does.
template <typename R, typename P, typename G = CtaGroup>
__device__ __forceinline__ void body_iteration(const LayerDev& L, int b, Body* __restrict__ bodies,
                                               const P& pos, const double4* __restrict__ ri,
                                               const double* __restrict__ vmass, double* __restrict__ lamB,
                                               const ContactData& cd, double h, double boundary_compliance,
                                               double contact_resistance, int use_rigid_contacts, Body& sb,
                                               double* invI, const DevContacts& dc = DevContacts{},
                                               const R4<R>* __restrict__ x0 = nullptr, const G g = G{}) {
  if (g.rank() == 0) {
    sb = bodies[b];
    inertia_inverse(sb.I, invI);
  }
  g.sync();
  bool dirty = false;
  if (L.any_boundary) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    int beg = L.bnd_off[b], end = L.bnd_off[b + 1];
    double invM = 1.0 / sb.mass;
    D3 com = d3(sb.com[0], sb.com[1], sb.com[2]);
    for (int i = beg + g.rank(); i < end; i += g.size()) {
      int v = L.bnd_verts[i];
      R4<R> p = pos.ld(v);
      D3 pE = d3((double)p.x, (double)p.y, (double)p.z);
      double minvE = 1.0 / vmass[v];
      D3 pR = body_point(sb, ri[v]);
      D3 r = pR - com;
      D3 dir = pR - pE;
      double C = sqrt(dot(dir, dir));
      D3 n = d3(dir.x / C, dir.y / C, dir.z / C);
      if (isnan(n.x)) n.x = 0;
      if (isnan(n.y)) n.y = 0;
      if (isnan(n.z)) n.z = 0;
      double w = gen_inv_mass(invM, r, invI, n);
      double dl = (-C - boundary_compliance * lamB[i]) / ((minvE + w) + boundary_compliance);
      lamB[i] += dl;
      D3 pp = dl * n;
      s[0] += pp.x * invM; s[1] += pp.y * invM; s[2] += pp.z * invM;
      D3 dw = cross(r, d3(pp.x / h, pp.y / h, pp.z / h));
      s[3] += dw.x; s[4] += dw.y; s[5] += dw.z;
    }
    g.template sum<6>(s);
    if (g.rank() == 0) {
      apply_increments(sb, s, h, invI);
      inertia_inverse(sb.I, invI);
    }
    g.sync();
    for (int i = beg + g.rank(); i < end; i += g.size()) {
      int v = L.bnd_verts[i];
      store_xyz<R>(pos, v, body_point(sb, ri[v]));
    }
    dirty = true;
  }
  if (use_rigid_contacts && L.any_rigid_contact) {
    pos.fence();
    g.sync();
    double s[6] = {0, 0, 0, 0, 0, 0};
    int beg = L.rc_off[b], end = L.rc_off[b + 1];
    double invM = 1.0 / sb.mass, h2 = h * h;
    D3 com = d3(sb.com[0], sb.com[1], sb.com[2]);
    for (int i = beg + g.rank(); i < end; i += g.size()) {
      int k = L.rc_ids[i];
      int v = cd.vid[k];
      R4<R> p = pos.ld(v);
      D3 x = d3((double)p.x, (double)p.y, (double)p.z);
      D3 pR = body_point(sb, ri[v]);
      D3 r = pR - com;
      D3 n = d3(cd.normal[k], cd.normal[cd.K + k], cd.normal[2 * cd.K + k]);
      D3 c = d3(cd.point[k], cd.point[cd.K + k], cd.point[2 * cd.K + k]);
      double phi = dot(n, x - c);
      if (phi > 0) phi = 0;
      double C = contact_resistance * phi;
      double w = gen_inv_mass(invM, r, invI, n);
      double aT = (2 * cd.compliance[k]) / h2;
      double dl = (-C - aT * cd.lambda[k]) / (2 * w + aT);
      cd.lambda[k] += dl;
      D3 pp = dl * n;
      s[0] += pp.x * invM; s[1] += pp.y * invM; s[2] += pp.z * invM;
      D3 cr = cross(r, pp);
      s[3] += (1 / h) * cr.x; s[4] += (1 / h) * cr.y; s[5] += (1 / h) * cr.z;
    }
    g.template sum<6>(s);
    if (g.rank() == 0) apply_increments(sb, s, h, invI);
    g.sync();
    for (int i = beg + g.rank(); i < end; i += g.size()) {
      int v = cd.vid[L.rc_ids[i]];
      store_xyz<R>(pos, v, body_point(sb, ri[v]));
    }
    dirty = true;
  }
  if (use_rigid_contacts && dc.nobs) {
    // contacts detected on the device: the body's vertices carry finder masks
    pos.fence();
    g.sync();
    double s[6] = {0, 0, 0, 0, 0, 0};
    const int beg = L.body_vert_off[b], end = L.body_vert_off[b + 1];
    const double invM = 1.0 / sb.mass, h2 = h * h;
    const D3 com = d3(sb.com[0], sb.com[1], sb.com[2]);
    for (int i = beg + g.rank(); i < end; i += g.size()) {
      const int v = L.body_verts[i];
      const unsigned m = dc.mask[v];
      if (!m) continue;
      const R4<R> p = pos.ld(v);
      const R4<R> s0 = x0[v];
      const D3 x = d3((double)p.x, (double)p.y, (double)p.z);
      const D3 r = body_point(sb, ri[v]) - com;
      const int ci = dc.cidx[v];
      for (int f = 0; f < dc.nobs; ++f) {
        if (!((m >> f) & 1u)) continue;
        D3 n, c;
        double comp;
        obstacle_contact(dc.obs[f], (double)s0.x, (double)s0.y, (double)s0.z, n, c, comp);
        double phi = dot(n, x - c);
        if (phi > 0) phi = 0;
        const double C = contact_resistance * phi;
        const double w = gen_inv_mass(invM, r, invI, n);
        const double aT = (2 * comp) / h2;
        double& lam = dc.lambda[(size_t)ci * dc.nobs + f];
        const double dl = (-C - aT * lam) / (2 * w + aT);
        lam += dl;
        const D3 pp = dl * n;
        s[0] += pp.x * invM; s[1] += pp.y * invM; s[2] += pp.z * invM;
        const D3 cr = cross(r, pp);
        s[3] += (1 / h) * cr.x; s[4] += (1 / h) * cr.y; s[5] += (1 / h) * cr.z;
      }
    }
    g.template sum<6>(s);
    if (g.rank() == 0) apply_increments(sb, s, h, invI);
    g.sync();
    for (int i = beg + g.rank(); i < end; i += g.size()) {
      const int v = L.body_verts[i];
      if (dc.mask[v]) store_xyz<R>(pos, v, body_point(sb, ri[v]));
    }
    dirty = true;
  }
  if (dirty && g.rank() == 0) bodies[b] = sb;
  pos.fence();
  g.sync();
}

// One iteration's body phase as its own launch: CTAs [0, nb) run one body
// each, the remaining CTAs the elastic contact groups.
// Three CTAs per SM (80 registers, a few spilled FP64 values): with many
// small bodies a layer's CTAs then run in fewer waves, which measured faster
// than the spill-free 126-register build (configs 2-4, 1-2 %).
template <typename R>
__global__ void __launch_bounds__(kBodyThreads, 3) k_iterate_bodies(LayerDev L, Body* __restrict__ bodies,
                                                                 R4<R>* __restrict__ pos,
                                                                 const double4* __restrict__ ri,
                                                                 const double* __restrict__ vmass,
                                                                 double* __restrict__ lamB, ContactData cd,
                                                                 double h, double boundary_compliance,
                                                                 double contact_resistance, int use_rigid_contacts,
                                                                 DevContacts dc, const R4<R>* __restrict__ x0) {
  __shared__ Body sb[kItemInts];
  __shared__ double invI[kItemInts][9];
  pdl_launch_dependents();
  pdl_wait();
  const int nbc = L.nb > 0 ? L.n_items : 0;  // CTAs [0, nbc) work on bodies
  if ((int)blockIdx.x >= nbc) {
    const GlobalPos<R> gp{pos};
    const int e = (int)blockIdx.x - nbc;
    if (dc.nobs) {
      // device-detected contacts: elastic ones are those of non-rigid vertices
      const int n = *dc.count, stride = (gridDim.x - nbc) * blockDim.x;
      for (int i = e * blockDim.x + threadIdx.x; i < n; i += stride)
        // (with contact_coloring only the vertices no colour phase took)
        if (L.vert_body[dc.verts[i]] == 0 && (!dc.colored || dc.vcc[dc.verts[i]] == dc.C))
          elastic_contacts_of_vertex<R>(dc, i, gp, x0, h, contact_resistance);
      return;
    }
    int g = e * blockDim.x + threadIdx.x;
    if (g < L.n_ec_groups) elastic_contact_group<R>(L, g, gp, cd, h, contact_resistance);
    return;
  }
  int b;
  if (body_of_item(L, b)) {
    body_iteration<R>(L, b, bodies, GlobalPos<R>{pos}, ri, vmass, lamB, cd, h, boundary_compliance,
                      contact_resistance, use_rigid_contacts, sb[0], invI[0], dc, x0, CtaGroup{});
  } else if (b >= 0) {
    const int w = threadIdx.x >> 5;
    body_iteration<R>(L, b, bodies, GlobalPos<R>{pos}, ri, vmass, lamB, cd, h, boundary_compliance,
                      contact_resistance, use_rigid_contacts, sb[w], invI[w], dc, x0, WarpGroup{});
  }
}

// xi(pinnedDOFs) = pinnedx (xpbdLayer3D.m:333)
template <typename R>
__global__ void k_pin(R4<R>* __restrict__ pos, const int* __restrict__ dofs,
                      const R* __restrict__ vals, int n) {
  pdl_launch_dependents();
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int d = dofs[i];
  GlobalPos<R>{pos}.st_comp(d / 3, d % 3, vals[i]);
}

// End of projectGS / layer: rotateAllVerts (xpbdLayer3D.m:344, 508-513) and,
// for a rigid layer, rotateResidual by dR = R_proj R_step' (:217-221, 234-241).
template <typename R, typename G>
__device__ __forceinline__ void finish_layer(const LayerDev& L, int b, const Body* __restrict__ bodies,
                                             R4<R>* __restrict__ pos, R4<R>* __restrict__ resv,
                                             const double4* __restrict__ ri, int rigid_layer, Body& sb, double* dR,
                                             const G& g) {
  if (g.rank() == 0) {
    sb = bodies[b];
    mm3_bt(sb.R, sb.Rstep, dR);
  }
  g.sync();
  int beg = L.body_vert_off[b], end = L.body_vert_off[b + 1];
  for (int i = beg + g.rank(); i < end; i += g.size()) {
    int v = L.body_verts[i];
    store_xyz<R>(pos, v, body_point(sb, ri[v]));
    if (rigid_layer) {
      R4<R> u = resv[v];
      D3 r = mv3(dR, d3((double)u.x, (double)u.y, (double)u.z));
      resv[v] = make_r4<R>((R)r.x, (R)r.y, (R)r.z, 0);
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(kBodyThreads) k_finish_layer(LayerDev L, const Body* __restrict__ bodies,
                                                               R4<R>* __restrict__ pos, R4<R>* __restrict__ resv,
                                                               const double4* __restrict__ ri, int rigid_layer) {
  __shared__ Body sb[kItemInts];
  __shared__ double dR[kItemInts][9];
  int b;
  if (body_of_item(L, b)) {
    finish_layer<R>(L, b, bodies, pos, resv, ri, rigid_layer, sb[0], dR[0], CtaGroup{});
  } else if (b >= 0) {
    const int w = threadIdx.x >> 5;
    finish_layer<R>(L, b, bodies, pos, resv, ri, rigid_layer, sb[w], dR[w], WarpGroup{});
  }
}

// ||residualv|| partial sums (xpbdLayer3D.m:161), FP64.
template <typename R>
__global__ void __launch_bounds__(256) k_norm3_partials(const R4<R>* __restrict__ v, int N,
                                                        double* __restrict__ partials) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    R4<R> u = v[i];
    acc[0] += (double)u.x * u.x + (double)u.y * u.y + (double)u.z * u.z;
  }
  block_sum<1>(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

}  // namespace mlx
