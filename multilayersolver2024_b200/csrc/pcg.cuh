// pcg.cuh -- preconditioned conjugate gradients on the device.
//
// The iteration of the reference's solvePCG.m (2d/tools/solver/solvePCG.m:
// x = x0, r = b - A x, z = P r, d = z, rTz = r'z; per iteration Ap = A d,
// alpha = rTz / d'Ap (0 when d'Ap = 0), x += alpha d, r -= alpha Ap,
// z = P r, beta = r'z / rTz, d = z + beta d, and resvec(i) = ||A x - b||),
// here for the linearly implicit system of a tet mesh
//     A = M + h^2 K0
// (lumped masses; K0 the linear-elasticity stiffness at the rest shape from
// each tet's DmInv, volume and Lame parameters) restricted to the unpinned
// DOFs, with the 3x3 block-Jacobi preconditioner P = blockdiag(A)^-1.  This
// is the system the reference's quick solve hands to solvePCG
// (3d/tools/solve/quickSolve3D.m:170, Afun = M v + h Md v - B' (h alpha1 C B v
// + h^2 C B v), qspcgHelper3D.m) without damping, at the rest tangent.
//
// Vectors are FP64 [N] double4 (w unused).  A x is a per-vertex gather over
// the vertex's tets in a fixed order (deterministic, one launch); the dot
// products are fixed-order block reductions; alpha and beta never leave the
// device.
#pragma once

#include "common.cuh"
#include "tet_kernels.cuh"

namespace mlx {

struct PcgOp {
  int N;
  const int* vt_off;        // [N+1] CSR over vt
  const int2* vt;           // (sorted tet id, corner 0..3)
  const int4* vid;          // [T] corners (sorted)
  const double* G;          // [T*9] DmInv, column-major per tet (element (r, c) at 9 s + r + 3 c)
  const double* vol;        // [T]
  const double* lame;       // [T*2] mu, lambda
  const double* vmass;      // [N]
  const unsigned char* pin; // [N] bit d: DOF d of the vertex is pinned
  double h2;
};

// Gradient of the linear shape function of corner k (k = 0..3) of tet s:
// rows of DmInv for corners 1..3, minus their sum for corner 0.
__device__ __forceinline__ D3 shape_grad(const double* G, int k) {
  if (k == 0)
    return d3(-(G[0] + G[1] + G[2]), -(G[3] + G[4] + G[5]), -(G[6] + G[7] + G[8]));
  return d3(G[k - 1], G[k - 1 + 3], G[k - 1 + 6]);
}

// Linear elastic force on corner k of tet s for displacements u:
// -vol sigma grad N_k, sigma = lambda tr(eps) I + 2 mu eps, eps = sym(grad u).
__device__ __forceinline__ D3 tet_force(const PcgOp& op, int s, int k, const double4* __restrict__ u) {
  const double* G = op.G + 9 * (size_t)s;
  const int4 v = op.vid[s];
  const int ids[4] = {v.x, v.y, v.z, v.w};
  double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // grad u, H[i + 3 j] = d u_i / d X_j
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const double4 ua = u[ids[a]];
    const D3 g = shape_grad(G, a);
    H[0] += ua.x * g.x; H[1] += ua.y * g.x; H[2] += ua.z * g.x;
    H[3] += ua.x * g.y; H[4] += ua.y * g.y; H[5] += ua.z * g.y;
    H[6] += ua.x * g.z; H[7] += ua.y * g.z; H[8] += ua.z * g.z;
  }
  const double mu = op.lame[2 * s], lm = op.lame[2 * s + 1];
  const double tr = H[0] + H[4] + H[8];
  double S[9];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) S[i + 3 * j] = mu * (H[i + 3 * j] + H[j + 3 * i]) + (i == j ? lm * tr : 0.0);
  const D3 g = shape_grad(G, k);
  const double V = op.vol[s];
  return d3(-V * (S[0] * g.x + S[3] * g.y + S[6] * g.z), -V * (S[1] * g.x + S[4] * g.y + S[7] * g.z),
            -V * (S[2] * g.x + S[5] * g.y + S[8] * g.z));
}

// y = A u on the unpinned DOFs (pinned DOFs: y = 0, u ignored).  The
// pinned components of u must be zero on entry.
__global__ void k_pcg_apply(PcgOp op, const double4* __restrict__ u, double4* __restrict__ y) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= op.N) return;
  const double4 uv = u[v];
  const double m = op.vmass[v];
  D3 acc = d3(m * uv.x, m * uv.y, m * uv.z);
  for (int q = op.vt_off[v]; q < op.vt_off[v + 1]; ++q) {
    const int2 e = op.vt[q];
    const D3 f = tet_force(op, e.x, e.y, u);
    acc = acc - op.h2 * f;  // K0 u = -f
  }
  const unsigned char pm = op.pin[v];
  y[v] = make_double4((pm & 1) ? 0.0 : acc.x, (pm & 2) ? 0.0 : acc.y, (pm & 4) ? 0.0 : acc.z, 0.0);
}

// Inverse of the 3x3 diagonal block of A at every vertex (pinned rows and
// columns replaced by the identity); column-major, 9 doubles per vertex.
__global__ void k_pcg_block_jacobi(PcgOp op, double* __restrict__ Pinv) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= op.N) return;
  const double m = op.vmass[v];
  double B[9] = {m, 0, 0, 0, m, 0, 0, 0, m};
  for (int q = op.vt_off[v]; q < op.vt_off[v + 1]; ++q) {
    const int2 e = op.vt[q];
    const double* G = op.G + 9 * (size_t)e.x;
    const D3 g = shape_grad(G, e.y);
    const double mu = op.lame[2 * e.x], lm = op.lame[2 * e.x + 1], V = op.vol[e.x];
    const double gg[3] = {g.x, g.y, g.z};
    const double n2 = g.x * g.x + g.y * g.y + g.z * g.z;
    // d(-f_k)/du_k = vol (mu |g|^2 I + (mu + lambda) g g^T)
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        B[i + 3 * j] += op.h2 * V * ((i == j ? mu * n2 : 0.0) + (mu + lm) * gg[i] * gg[j]);
  }
  const unsigned char pm = op.pin[v];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (pm & (1 << d)) {
      for (int k = 0; k < 3; ++k) B[d + 3 * k] = B[k + 3 * d] = 0.0;
      B[d + 3 * d] = 1.0;
    }
  double inv[9];
  inverse3(B, inv);
  for (int i = 0; i < 9; ++i) Pinv[9 * (size_t)v + i] = inv[i];
}

// z = P r (block Jacobi; pinned components 0)
__global__ void k_pcg_precond(int N, const double* __restrict__ Pinv, const unsigned char* __restrict__ pin,
                              const double4* __restrict__ r, double4* __restrict__ z) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const double* P = Pinv + 9 * (size_t)v;
  const double4 a = r[v];
  const D3 b = mv3(P, d3(a.x, a.y, a.z));
  const unsigned char pm = pin[v];
  z[v] = make_double4((pm & 1) ? 0.0 : b.x, (pm & 2) ? 0.0 : b.y, (pm & 4) ? 0.0 : b.z, 0.0);
}

// Partial dot products of up to two vector pairs, fixed order.
__global__ void __launch_bounds__(256) k_pcg_dot2(int N, const double4* __restrict__ a, const double4* __restrict__ b,
                                                  const double4* __restrict__ c, const double4* __restrict__ d,
                                                  double* __restrict__ partials) {
  double s[2] = {0.0, 0.0};
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) {
    const double4 x = a[v], y = b[v];
    s[0] += x.x * y.x + x.y * y.y + x.z * y.z;
    if (c) {
      const double4 p = c[v], q = d[v];
      s[1] += p.x * q.x + p.y * q.y + p.z * q.z;
    }
  }
  block_sum<2>(s);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = s[0];
    partials[2 * blockIdx.x + 1] = s[1];
  }
}

// Scalars of the iteration, in device memory.
struct PcgScalars {
  double rTz;    // r'z
  double alpha;
  double beta;
  double dAp;    // d'Ap
  double rTz_new;
  double res;    // ||A x - b||
};

// Sums the partials (one block of 256) and updates the scalars:
// mode 0: rTz = sum0 (set-up); mode 1: dAp = sum0, alpha = rTz / dAp
// (0 when dAp == 0); mode 2: rTz_new = sum0, beta = rTz_new / rTz,
// rTz = rTz_new; mode 3: res = sqrt(sum0); mode 4: mode 2 with beta = 0
// when the previous r'z is 0.
__global__ void __launch_bounds__(256) k_pcg_scalars(const double* __restrict__ partials, int n, int mode,
                                                     PcgScalars* __restrict__ sc, double* __restrict__ resvec, int it) {
  double s[1] = {0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) s[0] += partials[2 * i];
  block_sum<1>(s);
  if (threadIdx.x != 0) return;
  if (mode == 0) {
    sc->rTz = s[0];
  } else if (mode == 1) {
    sc->dAp = s[0];
    sc->alpha = s[0] == 0.0 ? 0.0 : sc->rTz / s[0];
  } else if (mode == 2) {
    sc->rTz_new = s[0];
    sc->beta = s[0] / sc->rTz;
    sc->rTz = s[0];
  } else if (mode == 4) {  // mode 2 with beta = 0 once r'z is 0 (a converged or zero system)
    sc->rTz_new = s[0];
    sc->beta = sc->rTz == 0.0 ? 0.0 : s[0] / sc->rTz;
    sc->rTz = s[0];
  } else {
    sc->res = sqrt(s[0]);
    if (resvec) resvec[it] = sc->res;
  }
}

// x += alpha d, r -= alpha Ap
__global__ void k_pcg_step(int N, const PcgScalars* __restrict__ sc, const double4* __restrict__ d,
                           const double4* __restrict__ Ap, double4* __restrict__ x, double4* __restrict__ r) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const double a = sc->alpha;
  const double4 dv = d[v], av = Ap[v], xv = x[v], rv = r[v];
  x[v] = make_double4(xv.x + a * dv.x, xv.y + a * dv.y, xv.z + a * dv.z, 0.0);
  r[v] = make_double4(rv.x - a * av.x, rv.y - a * av.y, rv.z - a * av.z, 0.0);
}

// d = z + beta d
__global__ void k_pcg_direction(int N, const PcgScalars* __restrict__ sc, const double4* __restrict__ z,
                                double4* __restrict__ d) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const double b = sc->beta;
  const double4 zv = z[v], dv = d[v];
  d[v] = make_double4(zv.x + b * dv.x, zv.y + b * dv.y, zv.z + b * dv.z, 0.0);
}

// out = a with the pinned components zeroed
__global__ void k_pcg_mask(int N, const unsigned char* __restrict__ pin, const double4* __restrict__ a,
                           double4* __restrict__ out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const double4 p = a[v];
  const unsigned char pm = pin[v];
  out[v] = make_double4((pm & 1) ? 0.0 : p.x, (pm & 2) ? 0.0 : p.y, (pm & 4) ? 0.0 : p.z, 0.0);
}

// out = a - b (componentwise)
__global__ void k_pcg_sub(int N, const double4* __restrict__ a, const double4* __restrict__ b,
                          double4* __restrict__ out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const double4 p = a[v], q = b[v];
  out[v] = make_double4(p.x - q.x, p.y - q.y, p.z - q.z, 0.0);
}

// ---------------------------------------------------------------------------
// Newton-PCG correction of a Neo-Hookean layer (the PCG used in the layer
// solve).  The XPBD projection of a layer solves, constraint by constraint,
//     C(x) + alpha~ lambda = 0,   M (x - x_c) = J^T (lambda - lambda_c),
// (x_c, lambda_c: the state the layer started from).  Linearised at the
// current x with J = dC/dx and W = alpha~^-1 this is
//     (M + J^T W J) dx = -J^T (W C + lambda),   lambda' = -W (C + J dx),
// a symmetric positive definite system on the free DOFs, solved here by the
// iteration of solvePCG (2d/tools/solver/solvePCG.m) with the 3x3
// block-Jacobi preconditioner; x += dx and lambda = lambda' give a state that
// keeps M dx = J^T (lambda' - lambda) to the PCG's residual.  The
// Gauss-Seidel sweeps of projectGS then continue from it.  C = (C_D, C_H) is
// the library's stable Neo-Hookean pair (tet_kernels.cuh nh_eval), W =
// (h^2 vol mu, h^2 vol (lambda - mu)) from the stored compliances.
//
// Storage.  The Jacobian is kept twice: structure of arrays jt[24][T] (row
// 6a + k: corner a, k < 3 dC_D/dx_a, k >= 3 dC_H/dx_a) for the per-tet
// products, whose warps then read consecutive words, and in the order of the
// vertex -> (tet, corner) CSR, jv[pairs][6], for the per-vertex gathers (each
// vertex then reads its pairs contiguously).  vtpos[4 s + a] is
// the CSR position of corner a of tet s.  Per tet, double2: w = (W_D, W_H),
// c = (C_D, C_H), q = W C + lambda (the right-hand side's factor), s scratch.

template <typename R>
__global__ void __launch_bounds__(256) k_ns_jacobian(TetData<R> td, const R4<R>* __restrict__ pos, double h2,
                                                     const int* __restrict__ vtpos, R* __restrict__ jt,
                                                     R* __restrict__ jv, double2* __restrict__ w,
                                                     double2* __restrict__ c, double2* __restrict__ q) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int T = td.T;
  if (s >= T) return;
  int4 v;
  R G[9], minv[4];
  V3<R> X[4];
  load_tet<R>(td, s, pos, v, G, X, minv);
  const double cD = (double)td.mat[s], cH = (double)td.mat[(size_t)T + s];
  NHEval<R> e;
  nh_eval<R>(X, G, cD, cH, 0.0, e);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const R g[6] = {e.gD[a].x, e.gD[a].y, e.gD[a].z, e.gH[a].x, e.gH[a].y, e.gH[a].z};
    R* u = jv + (size_t)6 * vtpos[4 * (size_t)s + a];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      jt[(size_t)(6 * a + k) * T + s] = g[k];
      u[k] = g[k];
    }
  }
  const double wD = cD > 0.0 ? h2 / cD : 0.0, wH = e.hasH ? h2 / cH : 0.0;
  w[s] = make_double2(wD, wH);
  c[s] = make_double2(e.CD, e.CH);
  q[s] = make_double2(wD * e.CD + (double)td.lambda[s],
                      e.hasH ? wH * e.CH + (double)td.lambda[(size_t)T + s] : 0.0);
}

// (J_t u) for tet s: the two constraint rows against the corners' u.
template <typename R>
__device__ __forceinline__ double2 ns_ju(const R* __restrict__ jt, int T, int s, int4 v,
                                         const double4* __restrict__ u) {
  const int vv[4] = {v.x, v.y, v.z, v.w};
  double d0 = 0.0, d1 = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const double4 ua = u[vv[a]];
    const R* t = jt + (size_t)(6 * a) * T + s;
    d0 += (double)t[0] * ua.x + (double)t[(size_t)T] * ua.y + (double)t[2 * (size_t)T] * ua.z;
    d1 += (double)t[3 * (size_t)T] * ua.x + (double)t[4 * (size_t)T] * ua.y + (double)t[5 * (size_t)T] * ua.z;
  }
  return make_double2(d0, d1);
}

// s_t = W_t (J_t u) for every tet.
template <typename R>
__global__ void __launch_bounds__(256) k_ns_tet_apply(int T, const int4* __restrict__ vid, const R* __restrict__ jt,
                                                      const double2* __restrict__ w, const double4* __restrict__ u,
                                                      double2* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= T) return;
  const double2 ju = ns_ju<R>(jt, T, s, vid[s], u);
  const double2 ws = w[s];
  out[s] = make_double2(ws.x * ju.x, ws.y * ju.y);
}

// sum over the vertex's (tet, corner) pairs of J_{t,corner}^T f_t, in the
// CSR's fixed order.
// Pairs go four at a time with their loads issued together (the sum keeps
// the CSR order).
template <typename R>
__device__ __forceinline__ D3 ns_jtf(const PcgOp& op, const R* __restrict__ jv, const double2* __restrict__ f,
                                     int v) {
  D3 acc = d3(0.0, 0.0, 0.0);
  const int k0 = op.vt_off[v], k1 = op.vt_off[v + 1];
  int k = k0;
  for (; k + 4 <= k1; k += 4) {
    double2 fk[4];
    R g[4][6];
#pragma unroll
    for (int q = 0; q < 4; ++q) fk[q] = f[op.vt[k + q].x];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 6; ++c) g[q][c] = jv[(size_t)6 * (k + q) + c];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      acc = acc + d3(fk[q].x * (double)g[q][0] + fk[q].y * (double)g[q][3],
                     fk[q].x * (double)g[q][1] + fk[q].y * (double)g[q][4],
                     fk[q].x * (double)g[q][2] + fk[q].y * (double)g[q][5]);
  }
  for (; k < k1; ++k) {
    const double2 fk = f[op.vt[k].x];
    const R* g = jv + (size_t)6 * k;
    acc = acc + d3(fk.x * (double)g[0] + fk.y * (double)g[3], fk.x * (double)g[1] + fk.y * (double)g[4],
                   fk.x * (double)g[2] + fk.y * (double)g[5]);
  }
  return acc;
}

// y = -J^T q on the unpinned DOFs (the right-hand side).
template <typename R>
__global__ void k_ns_rhs(PcgOp op, const R* __restrict__ jv, const double2* __restrict__ q, double4* __restrict__ y) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= op.N) return;
  const D3 a = ns_jtf<R>(op, jv, q, v);
  const unsigned char pm = op.pin[v];
  y[v] = make_double4((pm & 1) ? 0.0 : -a.x, (pm & 2) ? 0.0 : -a.y, (pm & 4) ? 0.0 : -a.z, 0.0);
}

// y = M u + J^T f on the unpinned DOFs, and the partial sums of u'y (one per
// block, at partials[2 b]; grid-stride over the vertices, fixed order).
template <typename R>
__global__ void __launch_bounds__(256) k_ns_vertex_apply(PcgOp op, const R* __restrict__ jv,
                                                         const double2* __restrict__ f, const double4* __restrict__ u,
                                                         double4* __restrict__ y, double* __restrict__ partials) {
  double dot[1] = {0.0};
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < op.N; v += gridDim.x * blockDim.x) {
    const D3 a = ns_jtf<R>(op, jv, f, v);
    const double m = op.vmass[v];
    const double4 uv = u[v];
    const unsigned char pm = op.pin[v];
    const double4 yv = make_double4((pm & 1) ? 0.0 : a.x + m * uv.x, (pm & 2) ? 0.0 : a.y + m * uv.y,
                                    (pm & 4) ? 0.0 : a.z + m * uv.z, 0.0);
    y[v] = yv;
    dot[0] += uv.x * yv.x + uv.y * yv.y + uv.z * yv.z;
  }
  block_sum<1>(dot);
  if (threadIdx.x == 0) partials[2 * blockIdx.x] = dot[0];
}

// Sum of the n partials of a fixed-order reduction (the same order in every
// block, so every block obtains the same value).
__device__ __forceinline__ double ns_sum_partials(const double* __restrict__ partials, int n) {
  double s[1] = {0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) s[0] += partials[2 * i];
  block_sum<1>(s);
  return s[0];
}

// alpha = rTz[cur] / d'Ap (0 when d'Ap = 0) from the partials of d'Ap; then
// x += alpha d, r -= alpha Ap, z = P r, and the partial sums of r'z (one per
// block at partials2[2 b]; grid-stride, fixed order).
__global__ void __launch_bounds__(256) k_ns_step(int N, const double* __restrict__ rTz, int cur,
                                                 const double* __restrict__ partials, int nparts,
                                                 const double4* __restrict__ d, const double4* __restrict__ Ap,
                                                 double4* __restrict__ x, double4* __restrict__ r,
                                                 const double* __restrict__ Pinv,
                                                 const unsigned char* __restrict__ pin, double4* __restrict__ z,
                                                 double* __restrict__ partials2) {
  const double dAp = ns_sum_partials(partials, nparts);
  const double alpha = dAp == 0.0 ? 0.0 : rTz[cur] / dAp;
  double dot[1] = {0.0};
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) {
    const double4 dv = d[v], av = Ap[v], xv = x[v], rv = r[v];
    x[v] = make_double4(xv.x + alpha * dv.x, xv.y + alpha * dv.y, xv.z + alpha * dv.z, 0.0);
    const D3 rn = d3(rv.x - alpha * av.x, rv.y - alpha * av.y, rv.z - alpha * av.z);
    r[v] = make_double4(rn.x, rn.y, rn.z, 0.0);
    const D3 b = mv3(Pinv + 9 * (size_t)v, rn);
    const unsigned char pm = pin[v];
    const D3 zn = d3((pm & 1) ? 0.0 : b.x, (pm & 2) ? 0.0 : b.y, (pm & 4) ? 0.0 : b.z);
    z[v] = make_double4(zn.x, zn.y, zn.z, 0.0);
    dot[0] += rn.x * zn.x + rn.y * zn.y + rn.z * zn.z;
  }
  block_sum<1>(dot);
  if (threadIdx.x == 0) partials2[2 * blockIdx.x] = dot[0];
}

// rTz_new from the partials of r'z; beta = rTz_new / rTz[cur] (0 when
// rTz[cur] = 0); d = z + beta d; block 0 stores rTz_new in rTz[1 - cur] for
// the next iteration (r'z is double-buffered: every block reads rTz[cur]).
__global__ void __launch_bounds__(256) k_ns_direction(int N, double* __restrict__ rTz, int cur,
                                                      const double* __restrict__ partials, int nparts,
                                                      const double4* __restrict__ z, double4* __restrict__ d) {
  const double rtz_new = ns_sum_partials(partials, nparts);
  const double old = rTz[cur];
  const double beta = old == 0.0 ? 0.0 : rtz_new / old;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) {
    const double4 zv = z[v], dv = d[v];
    d[v] = make_double4(zv.x + beta * dv.x, zv.y + beta * dv.y, zv.z + beta * dv.z, 0.0);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) rTz[1 - cur] = rtz_new;
}

// Inverse of the 3x3 diagonal block of M + J^T W J at every vertex (pinned
// rows and columns replaced by the identity).
template <typename R>
__global__ void k_ns_block_jacobi(PcgOp op, const R* __restrict__ jv, const double2* __restrict__ w,
                                  double* __restrict__ Pinv) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= op.N) return;
  const double m = op.vmass[v];
  double B[9] = {m, 0, 0, 0, m, 0, 0, 0, m};
  for (int k = op.vt_off[v]; k < op.vt_off[v + 1]; ++k) {
    const double2 wk = w[op.vt[k].x];
    const R* g = jv + (size_t)6 * k;
    const double gD[3] = {(double)g[0], (double)g[1], (double)g[2]};
    const double gH[3] = {(double)g[3], (double)g[4], (double)g[5]};
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) B[i + 3 * j] += wk.x * gD[i] * gD[j] + wk.y * gH[i] * gH[j];
  }
  const unsigned char pm = op.pin[v];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (pm & (1 << d)) {
      for (int k = 0; k < 3; ++k) B[d + 3 * k] = B[k + 3 * d] = 0.0;
      B[d + 3 * d] = 1.0;
    }
  double inv[9];
  inverse3(B, inv);
  for (int i = 0; i < 9; ++i) Pinv[9 * (size_t)v + i] = inv[i];
}

// lambda = -W (C + J dx) for every tet (rows 0 and 1; an absent C_H keeps 0).
template <typename R>
__global__ void __launch_bounds__(256) k_ns_lambda(int T, const int4* __restrict__ vid, const R* __restrict__ jt,
                                                   const double2* __restrict__ w, const double2* __restrict__ c,
                                                   const double4* __restrict__ dx, R* __restrict__ lambda) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= T) return;
  const double2 jd = ns_ju<R>(jt, T, s, vid[s], dx);
  const double2 ws = w[s], cs = c[s];
  lambda[s] = (R)(-ws.x * (cs.x + jd.x));
  lambda[(size_t)T + s] = ws.y > 0.0 ? (R)(-ws.y * (cs.y + jd.y)) : R(0);
}

// x += dx on every vertex (dx is 0 on the pinned DOFs).
template <typename R>
__global__ void k_ns_move(int N, const double4* __restrict__ dx, R4<R>* __restrict__ pos) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const double4 d = dx[v];
  R4<R> p = pos[v];
  pos[v] = make_r4<R>((R)((double)p.x + d.x), (R)((double)p.y + d.y), (R)((double)p.z + d.z), p.w);
}

}  // namespace mlx
