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
  unsigned int count[2];  // last-block counts of the Newton-PCG grid reductions (0 between launches)
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
// product of the new multipliers, whose warps then read consecutive words,
// and in the order of the vertex -> (tet, corner) CSR, jv[pairs][6], for the
// right-hand side and the assembly (each vertex then reads its pairs
// contiguously).  vtpos[4 s + a] is the CSR position of corner a of tet s.
// Per tet, double2: w = (W_D, W_H), c = (C_D, C_H), q = W C + lambda (the
// right-hand side's factor).  The PCG iterations read neither: J^T W J is
// assembled once per correction into 3x3 blocks per (vertex, neighbour)
// (k_ns_assemble), and an iteration is one blocked product (k_ns_spmv) and
// one vector step (k_ns_step).

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

// The search direction at vertex v for this iteration: d_k = z_k + beta d_{k-1}
// (beta from the previous iteration's r'z; beta = 0 and d = 0 at the start).
// Every row that reads vertex v evaluates it with the same fused
// multiply-add, so all see the bits that v's own row stores.
__device__ __forceinline__ double4 ns_dir(const double4 z, const double4 d, double beta) {
  return make_double4(__fma_rn(beta, d.x, z.x), __fma_rn(beta, d.y, z.y), __fma_rn(beta, d.z, z.z), 0.0);
}

// Lanes per row in the blocked product: a vertex of a tet mesh shares tets
// with ~14 others; four lanes take ~4 blocks each, eight rows to a warp.
constexpr int kNsTeam = 4;
// Largest grid of a Newton-PCG grid reduction (one partial sum per block).
constexpr int kNsMaxPartials = 2048;

// y = -J^T q on the unpinned DOFs (the right-hand side): kNsTeam lanes per
// vertex, each lane every kNsTeam-th (tet, corner) pair of the vertex's CSR
// range, a fixed butterfly over the team (lane 0 stores).
template <typename R>
__global__ void __launch_bounds__(256) k_ns_rhs(PcgOp op, const R* __restrict__ jv, const double2* __restrict__ q,
                                                double4* __restrict__ y) {
  const int lane = threadIdx.x & (kNsTeam - 1);
  const unsigned mask = ((1u << kNsTeam) - 1u) << ((threadIdx.x & 31) & ~(kNsTeam - 1));
  const int v = (blockIdx.x * blockDim.x + threadIdx.x) / kNsTeam;
  if (v >= op.N) return;  // whole teams leave together
  double ax = 0.0, ay = 0.0, az = 0.0;
  const int k1 = op.vt_off[v + 1];
  for (int k = op.vt_off[v] + lane; k < k1; k += kNsTeam) {
    const double2 fk = q[op.vt[k].x];
    const R* g = jv + (size_t)6 * k;
    ax += fk.x * (double)g[0] + fk.y * (double)g[3];
    ay += fk.x * (double)g[1] + fk.y * (double)g[4];
    az += fk.x * (double)g[2] + fk.y * (double)g[5];
  }
#pragma unroll
  for (int o = kNsTeam / 2; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(mask, ax, o);
    ay += __shfl_xor_sync(mask, ay, o);
    az += __shfl_xor_sync(mask, az, o);
  }
  if (lane == 0) {
    const unsigned char pm = op.pin[v];
    y[v] = make_double4((pm & 1) ? 0.0 : -ax, (pm & 2) ? 0.0 : -ay, (pm & 4) ? 0.0 : -az, 0.0);
  }
}

// The block's partial sum of a grid reduction goes to partials[blockIdx.x];
// the last block to finish (an atomic count, after a fence) sums all of them
// in index order, which does not depend on which block that is, and resets
// the count for the next launch.  Returns true in that block, with the sum in
// `total` (all its threads).
__device__ __forceinline__ bool ns_last_block(double mine, double* __restrict__ partials,
                                              unsigned int* __restrict__ count, double& total) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = mine;
    __threadfence();
    last = atomicAdd(count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double s[1] = {0.0};
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s[0] += __ldcg(partials + i);
  block_sum<1>(s);
  total = s[0];
  if (threadIdx.x == 0) *count = 0u;
  return true;
}

// J^T W J assembled into 3x3 blocks per (vertex, neighbour) once per
// correction, so that each PCG iteration reads one blocked sparse matrix
// (~15 blocks per vertex) instead of passing twice over the Jacobian.
// Row v lists the vertices sharing a tet with v (itself included), in
// increasing order: nb_off[N+1], nb_col[nnz]; block j of the matrix is
// K[9 j + r + 3 c] (column-major) = sum over the tets t holding v (corner a)
// and nb_col[j] (corner b) of wD gD_a gD_b' + wH gH_a gH_b'.
// pslot[k] holds, for pair k = (t, a) of the vertex CSR, the row slot of each
// corner b of t (byte b).
struct NsBlocks {
  const int* nb_off;         // [N+1]
  const int* nb_col;         // [nnz]
  const unsigned int* pslot; // [pairs] four row slots, one byte per corner
  const int* vtpos;          // [4T] CSR position of pair (t, b)
};

// One warp per row (grid-stride over the rows), 32 pairs at a time: lane p
// stages pair p (its tet's four corner gradients from the CSR-order
// Jacobian, the tet's weights, the corners' row slots) in shared memory;
// then lane l, the owner of slots l, l + 32, ..., sums the staged pairs'
// contributions to its slots in CSR order -- the same order every run, no
// atomics.  The owner of the row's diagonal block also writes the inverse of
// M + K_vv (pinned rows and columns replaced by the identity): the
// block-Jacobi preconditioner.
constexpr int kNsAsmWarps = 4;

struct NsStage {
  double g[32][4][6];     // corner b's two gradient rows (D: 0..2, H: 3..5)
  double2 w[32];          // (wD, wH)
  unsigned int slot[32];  // byte b: row slot of corner b
  int corner[32];         // the row's own corner a
};

template <typename R>
__global__ void __launch_bounds__(32 * kNsAsmWarps) k_ns_assemble(PcgOp op, NsBlocks nb, const R* __restrict__ jv,
                                                                  const double2* __restrict__ w,
                                                                  R* __restrict__ K, double* __restrict__ Pinv) {
  __shared__ NsStage stage[kNsAsmWarps];
  NsStage& st = stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * kNsAsmWarps;
  for (int v = blockIdx.x * kNsAsmWarps + (threadIdx.x >> 5); v < op.N; v += nwarps) {
    const int k0 = op.vt_off[v], k1 = op.vt_off[v + 1];
    const int r0 = nb.nb_off[v], rn = nb.nb_off[v + 1] - r0;
    if (rn == 0) {  // a vertex of no tet: the preconditioner block is M alone
      if (lane == 0) {
        const double m = op.vmass[v];
        const unsigned char pm = op.pin[v];
        double* pv = Pinv + 9 * (size_t)v;
#pragma unroll
        for (int q = 0; q < 9; ++q) pv[q] = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) pv[4 * d] = (pm & (1 << d)) ? 1.0 : 1.0 / m;
      }
      continue;
    }
    // the row's diagonal slot (the vertex itself)
    int dslot = -1;
    for (int b0 = 0; b0 < rn; b0 += 32) {
      const unsigned bal = __ballot_sync(0xffffffffu, b0 + lane < rn && nb.nb_col[r0 + b0 + lane] == v);
      if (bal) dslot = b0 + __ffs(bal) - 1;
    }
    for (int base = 0; base < rn; base += 32) {
      const int mine = base + lane;
      // every pair adds one product to the diagonal block (its own corner),
      // ~22 against ~6 for the other blocks: when this round has two or
      // more lanes without a slot, they split the diagonal's pairs (helper
      // h takes the pairs p = h mod nh) and the diagonal's owner sums their
      // parts in helper order
      const int nh = base + 32 > rn ? base + 32 - rn : 0;
      const bool split = nh >= 2 && dslot >= base && dslot < base + 32;
      const int hi = mine - rn;  // helper index (split rounds, lanes without a slot)
      // every byte of the pattern is this lane's slot (slots are < 255); no
      // match for lanes without a slot and for a split diagonal's owner
      const unsigned int rep =
          (mine < rn && !(split && mine == dslot)) ? (unsigned int)mine * 0x01010101u : 0xffffffffu;
      double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int p0 = k0; p0 < k1; p0 += 32) {
        const int np = min(32, k1 - p0);
        __syncwarp();
        if (lane < np) {
          const int k = p0 + lane;
          const int2 tk = op.vt[k];
          const int4 pos4 = *reinterpret_cast<const int4*>(nb.vtpos + 4 * (size_t)tk.x);
          const int pk[4] = {pos4.x, pos4.y, pos4.z, pos4.w};
#pragma unroll
          for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 6; ++c) st.g[lane][b][c] = (double)jv[(size_t)6 * pk[b] + c];
          st.w[lane] = w[tk.x];
          st.slot[lane] = nb.pslot[k];
          st.corner[lane] = tk.y;
        }
        __syncwarp();
        // bit 4 q + b of word wd: corner b of staged pair 8 wd + q lies in
        // this lane's slot (a byte compare, then the four match bits of a
        // word gathered by one multiply: byte b's bit lands on bit 24 + b)
        unsigned int mw[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int wd = 0; wd < 4; ++wd)
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int p = 8 * wd + q;
            if (p < np) {
              const unsigned int x = __vcmpeq4(st.slot[p], rep) & 0x01010101u;
              mw[wd] |= ((x * 0x01020408u) >> 24) << (4 * q);
            }
          }
        // a helper's diagonal pairs of this chunk
        if (split && hi >= 0) {
          for (int p = ((hi - (p0 - k0)) % nh + nh) % nh; p < np; p += nh) {
            const int b = st.corner[p];
            mw[p >> 3] |= 1u << (4 * (p & 7) + b);
          }
        }
        // the matches in pair order, then corner order
#pragma unroll
        for (int wd = 0; wd < 4; ++wd) {
          unsigned int m = mw[wd];
          while (m) {
            const int bit = __ffs(m) - 1;
            m &= m - 1u;
            const int p = 8 * wd + (bit >> 2), b = bit & 3;
            const double* ga = st.g[p][st.corner[p]];
            const double* gb = st.g[p][b];
            const double2 wk = st.w[p];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const double bD = wk.x * gb[c], bH = wk.y * gb[3 + c];
#pragma unroll
              for (int r = 0; r < 3; ++r) acc[r + 3 * c] += ga[r] * bD + ga[3 + r] * bH;
            }
          }
        }
      }
      if (split) {
#pragma unroll 1
        for (int hh = 0; hh < nh; ++hh) {
#pragma unroll
          for (int q = 0; q < 9; ++q) {
            const double t = __shfl_sync(0xffffffffu, acc[q], rn - base + hh);
            if (mine == dslot) acc[q] += t;
          }
        }
      }
      if (mine < rn) {
        R* kb = K + (size_t)9 * (r0 + mine);
#pragma unroll
        for (int q = 0; q < 9; ++q) kb[q] = (R)acc[q];
        if (mine == dslot) {
          const double m = op.vmass[v];
          double B[9];
#pragma unroll
          for (int q = 0; q < 9; ++q) B[q] = acc[q];
          B[0] += m;
          B[4] += m;
          B[8] += m;
          const unsigned char pm = op.pin[v];
#pragma unroll
          for (int d = 0; d < 3; ++d)
            if (pm & (1 << d)) {
              for (int k = 0; k < 3; ++k) B[d + 3 * k] = B[k + 3 * d] = 0.0;
              B[d + 3 * d] = 1.0;
            }
          double inv[9];
          inverse3(B, inv);
#pragma unroll
          for (int q = 0; q < 9; ++q) Pinv[9 * (size_t)v + q] = inv[q];
        }
      }
    }
  }
}

// Ap = M d_k + K d_k on the unpinned DOFs, with d_k = z + beta d_{k-1} formed
// at every column (d_{k-1} from `dprev`) and stored for the row in `dnext`
// (the two direction buffers alternate between iterations, so no row reads a
// direction another row has already replaced).  A team of kNsTeam lanes per
// row, each lane every kNsTeam-th block, a fixed butterfly over the team
// (lane 0's sum), d_k'Ap summed per block; the last block sets alpha.
template <typename R>
__global__ void __launch_bounds__(256) k_ns_spmv(PcgOp op, NsBlocks nb, const R* __restrict__ K,
                                                 const double4* __restrict__ z, const double4* __restrict__ dprev,
                                                 double4* __restrict__ dnext, double4* __restrict__ Ap,
                                                 PcgScalars* __restrict__ sc, double* __restrict__ partials,
                                                 unsigned int* __restrict__ count) {
  const double beta = sc->beta;
  const int lane = threadIdx.x & (kNsTeam - 1);
  const unsigned mask = ((1u << kNsTeam) - 1u) << ((threadIdx.x & 31) & ~(kNsTeam - 1));
  const int nteams = gridDim.x * (blockDim.x / kNsTeam);
  double dot[1] = {0.0};
  for (int v = blockIdx.x * (blockDim.x / kNsTeam) + threadIdx.x / kNsTeam; v < op.N; v += nteams) {
    double ax = 0.0, ay = 0.0, az = 0.0;
    // the row's own data, loaded while the blocks are gathered
    double4 zv = make_double4(0, 0, 0, 0), dv = zv;
    double m = 0.0;
    unsigned char pm = 0;
    if (lane == 0) {
      zv = z[v];
      dv = dprev[v];
      m = op.vmass[v];
      pm = op.pin[v];
    }
    const int j1 = nb.nb_off[v + 1];
    for (int j = nb.nb_off[v] + lane; j < j1; j += kNsTeam) {
      const int c = nb.nb_col[j];
      const double4 u = ns_dir(z[c], dprev[c], beta);
      const R* kb = K + (size_t)9 * j;
      ax += (double)kb[0] * u.x + (double)kb[3] * u.y + (double)kb[6] * u.z;
      ay += (double)kb[1] * u.x + (double)kb[4] * u.y + (double)kb[7] * u.z;
      az += (double)kb[2] * u.x + (double)kb[5] * u.y + (double)kb[8] * u.z;
    }
#pragma unroll
    for (int o = kNsTeam / 2; o > 0; o >>= 1) {
      ax += __shfl_xor_sync(mask, ax, o);
      ay += __shfl_xor_sync(mask, ay, o);
      az += __shfl_xor_sync(mask, az, o);
    }
    if (lane == 0) {
      const double4 dk = ns_dir(zv, dv, beta);
      dnext[v] = dk;
      const double4 yv = make_double4((pm & 1) ? 0.0 : ax + m * dk.x, (pm & 2) ? 0.0 : ay + m * dk.y,
                                      (pm & 4) ? 0.0 : az + m * dk.z, 0.0);
      Ap[v] = yv;
      dot[0] += dk.x * yv.x + dk.y * yv.y + dk.z * yv.z;
    }
  }
  block_sum<1>(dot);
  double dAp;
  if (ns_last_block(dot[0], partials, count, dAp) && threadIdx.x == 0) {
    sc->dAp = dAp;
    sc->alpha = dAp == 0.0 ? 0.0 : sc->rTz / dAp;
  }
}

// x += alpha d_k, r -= alpha Ap, z = P r (grid-stride, fixed order), and r'z:
// the last block sets beta = r'z / rTz (0 when rTz = 0) and rTz = r'z for the
// next iteration.
__global__ void __launch_bounds__(256) k_ns_step(int N, PcgScalars* __restrict__ sc, const double4* __restrict__ d,
                                                 const double4* __restrict__ Ap, double4* __restrict__ x,
                                                 double4* __restrict__ r, const double* __restrict__ Pinv,
                                                 const unsigned char* __restrict__ pin, double4* __restrict__ z,
                                                 double* __restrict__ partials, unsigned int* __restrict__ count) {
  const double alpha = sc->alpha;
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
  double rtz;
  if (ns_last_block(dot[0], partials, count, rtz) && threadIdx.x == 0) {
    sc->rTz_new = rtz;
    sc->beta = sc->rTz == 0.0 ? 0.0 : rtz / sc->rTz;
    sc->rTz = rtz;
  }
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
