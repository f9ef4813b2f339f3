// warmstart.cuh -- features, corrections and training targets of the learned
// warm start of the coarse (rigid-cluster) layer.
//
// For every cluster (rigid body of the first layer), right after
// makeRigidsFromConnectivity (AdaptiveMesh3D.m:32-43):
//   features (44): own state (12) -- COM velocity, angular velocity, COM
//     displacement from the rest configuration, rotation vector of the
//     cluster's deformation from rest (polar decomposition, FP64); and for
//     the 4 clusters nearest at rest (8 each) their COM and angular velocity
//     relative to this cluster's, the change of their COM distance, and their
//     mass ratio;
//   outputs (8): a COM-velocity and angular-velocity correction applied
//     before the symplectic rigid step (6), the cluster's starting boundary
//     multiplier (rigidElasticBoundaryAccumulationConstraints' lambda, 0 in
//     the reference) (1), and the predicted residual of the cluster's rigid
//     fit, log10 of the RMS distance (m) of its vertices' final positions from
//     the best-fit rigid motion of the step (1).  A cluster whose predicted
//     residual exceeds the gate (1e-3 m by default) is not corrected: it falls
//     back to the plain start.
// Targets come from the converged step: the best-fit rigid motion of each
// cluster from its step-start to its final positions (Kabsch: the polar
// factor of sum m (x* - c*)(x0 - c0)^T), expressed as the velocities that make
// the rigid step land there, the mean final boundary multiplier, and the
// log10 RMS residual of that fit.  The
// polar decomposition restates the reference's polarDecomposition.m
// (2d/tools/math/polarDecomposition.m: C = F'F, eig(C),
// U^-1 = Q diag(1/sqrt(lambda)) Q', R = F U^-1) in 3D with a cyclic Jacobi
// eigen-solver, in FP64.
#pragma once

#include "body_kernels.cuh"
#include "common.cuh"
#include "tet_kernels.cuh"

namespace mlx {

constexpr int kWsOwn = 12;
constexpr int kWsNbr = 4;
constexpr int kWsFeat = kWsOwn + 8 * kWsNbr;  // 44
constexpr int kWsOut = 8;
constexpr int kWsResidualCol = 7;  // log10 of the predicted rigid-fit residual (m)
constexpr int kWsRec = 9;  // COM, COM velocity, angular velocity at makeRigids

// Eigen-decomposition of a symmetric 3x3 matrix (column-major) by cyclic
// Jacobi rotations: A = Q diag(w) Q^T.
__device__ __forceinline__ void sym_eig3(const double* Ain, double* w, double* Q) {
  double A[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    A[i] = Ain[i];
    Q[i] = (i % 4 == 0) ? 1.0 : 0.0;
  }
  for (int sweep = 0; sweep < 12; ++sweep) {
    const double off = A[3] * A[3] + A[6] * A[6] + A[7] * A[7];
    if (off < 1e-30 * (A[0] * A[0] + A[4] * A[4] + A[8] * A[8]) + 1e-300) break;
#pragma unroll
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      const double apq = A[p + 3 * q];
      if (fabs(apq) < 1e-300) continue;
      const double app = A[p + 3 * p], aqq = A[q + 3 * q];
      const double theta = (aqq - app) / (2.0 * apq);
      const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
      // A <- J^T A J, Q <- Q J with J the rotation in the (p, q) plane
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double akp = A[k + 3 * p], akq = A[k + 3 * q];
        A[k + 3 * p] = c * akp - s * akq;
        A[k + 3 * q] = s * akp + c * akq;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double apk = A[p + 3 * k], aqk = A[q + 3 * k];
        A[p + 3 * k] = c * apk - s * aqk;
        A[q + 3 * k] = s * apk + c * aqk;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double qkp = Q[k + 3 * p], qkq = Q[k + 3 * q];
        Q[k + 3 * p] = c * qkp - s * qkq;
        Q[k + 3 * q] = s * qkp + c * qkq;
      }
    }
  }
  w[0] = A[0];
  w[1] = A[4];
  w[2] = A[8];
}

// Rotation factor of F = R U (column-major): R = F Q diag(1/sqrt(w)) Q^T
// with F^T F = Q diag(w) Q^T.
__device__ __forceinline__ void polar_rotation(const double* F, double* R) {
  double C[9], w[3], Q[9], Ui[9];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      C[r + 3 * c] = F[3 * r] * F[3 * c] + F[3 * r + 1] * F[3 * c + 1] + F[3 * r + 2] * F[3 * c + 2];
  sym_eig3(C, w, Q);
  double inv[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) inv[i] = w[i] > 1e-300 ? 1.0 / sqrt(w[i]) : 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      Ui[r + 3 * c] = Q[r] * inv[0] * Q[c] + Q[r + 3] * inv[1] * Q[c + 3] + Q[r + 6] * inv[2] * Q[c + 6];
  mm3(F, Ui, R);
}

// Rotation vector (axis * angle) of a rotation matrix (column-major).
__device__ __forceinline__ D3 rotation_log(const double* R) {
  const double c = fmin(fmax(0.5 * (R[0] + R[4] + R[8] - 1.0), -1.0), 1.0);
  const double th = acos(c);
  const D3 v = d3(R[5] - R[7], R[6] - R[2], R[1] - R[3]);  // 2 sin(th) * axis
  const double k = th < 1e-6 ? 0.5 : 0.5 * th / sin(th);
  return k * v;
}

// Per-cluster data of the warm-started layer, fixed at set-up.
struct WsStatic {
  int nb;
  const int* body_vert_off;  // [nb+1]
  const int* body_verts;
  const int* bnd_off;        // [nb+1] CSR over the layer's boundary vertices
  const int* nbr;            // [nb * 4] nearest clusters at rest (-1: none)
  const double* rest_com;    // [nb * 3]
  const double* rest_cinv;   // [nb * 9] inverse of sum m (X-C)(X-C)^T
  const double* mass;        // [nb] cluster mass
  const double4* rest;       // [N] rest positions
  const double* vmass;       // [N]
};

// Rest data of every cluster: COM, inverse rest covariance, mass (one CTA per cluster).
__global__ void __launch_bounds__(256) k_ws_rest(WsStatic S, double* rest_com, double* rest_cinv, double* mass) {
  const int b = blockIdx.x;
  const int beg = S.body_vert_off[b], end = S.body_vert_off[b + 1];
  double s[4] = {0, 0, 0, 0};
  for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int v = S.body_verts[i];
    const double m = S.vmass[v];
    const double4 X = S.rest[v];
    s[0] += m; s[1] += m * X.x; s[2] += m * X.y; s[3] += m * X.z;
  }
  block_sum<4>(s);
  const D3 C = d3(s[1] / s[0], s[2] / s[0], s[3] / s[0]);
  double cv[6] = {0, 0, 0, 0, 0, 0};
  for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int v = S.body_verts[i];
    const double m = S.vmass[v];
    const double4 X = S.rest[v];
    const D3 d = d3(X.x, X.y, X.z) - C;
    cv[0] += m * d.x * d.x; cv[1] += m * d.y * d.y; cv[2] += m * d.z * d.z;
    cv[3] += m * d.x * d.y; cv[4] += m * d.x * d.z; cv[5] += m * d.y * d.z;
  }
  block_sum<6>(cv);
  if (threadIdx.x == 0) {
    const double Cm[9] = {cv[0], cv[3], cv[4], cv[3], cv[1], cv[5], cv[4], cv[5], cv[2]};
    double inv[9];
    inverse3(Cm, inv);
    for (int i = 0; i < 9; ++i) rest_cinv[9 * b + i] = inv[i];
    rest_com[3 * b] = C.x; rest_com[3 * b + 1] = C.y; rest_com[3 * b + 2] = C.z;
    mass[b] = s[0];
  }
}

// Own features of every cluster after makeRigids (one CTA per cluster);
// also records COM, COM velocity and angular velocity for the targets.
template <typename R>
__global__ void __launch_bounds__(256) k_ws_own(WsStatic S, const Body* __restrict__ bodies,
                                                const R4<R>* __restrict__ pos, float* __restrict__ own,
                                                double* __restrict__ rec) {
  const int b = blockIdx.x;
  const Body& B = bodies[b];
  const D3 com = d3(B.com[0], B.com[1], B.com[2]);
  const D3 C = d3(S.rest_com[3 * b], S.rest_com[3 * b + 1], S.rest_com[3 * b + 2]);
  const int beg = S.body_vert_off[b], end = S.body_vert_off[b + 1];
  double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // sum m (x - com)(X - C)^T, column-major
  for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int v = S.body_verts[i];
    const double m = S.vmass[v];
    const R4<R> p = pos[v];
    const double4 X = S.rest[v];
    const D3 x = d3((double)p.x, (double)p.y, (double)p.z) - com;
    const D3 y = d3(X.x, X.y, X.z) - C;
    a[0] += m * x.x * y.x; a[1] += m * x.y * y.x; a[2] += m * x.z * y.x;
    a[3] += m * x.x * y.y; a[4] += m * x.y * y.y; a[5] += m * x.z * y.y;
    a[6] += m * x.x * y.z; a[7] += m * x.y * y.z; a[8] += m * x.z * y.z;
  }
  block_sum<9>(a);
  if (threadIdx.x == 0) {
    double F[9], Rm[9];
    mm3(a, S.rest_cinv + 9 * b, F);  // the cluster's deformation from rest
    polar_rotation(F, Rm);
    const D3 th = rotation_log(Rm);
    float* o = own + (size_t)kWsOwn * b;
    o[0] = (float)B.comdot[0]; o[1] = (float)B.comdot[1]; o[2] = (float)B.comdot[2];
    o[3] = (float)B.omega[0]; o[4] = (float)B.omega[1]; o[5] = (float)B.omega[2];
    o[6] = (float)(com.x - C.x); o[7] = (float)(com.y - C.y); o[8] = (float)(com.z - C.z);
    o[9] = (float)th.x; o[10] = (float)th.y; o[11] = (float)th.z;
    double* r = rec + (size_t)kWsRec * b;
    for (int d = 0; d < 3; ++d) {
      r[d] = B.com[d];
      r[3 + d] = B.comdot[d];
      r[6 + d] = B.omega[d];
    }
  }
}

// Full feature rows (own + neighbours), raw and, when `norm` is given,
// normalised ((f - mean) / std).
__global__ void k_ws_features(WsStatic S, const float* __restrict__ own, const float* __restrict__ fmean,
                              const float* __restrict__ fstd, float* __restrict__ raw, float* __restrict__ norm) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= S.nb) return;
  float f[kWsFeat];
  const float* o = own + (size_t)kWsOwn * b;
#pragma unroll
  for (int i = 0; i < kWsOwn; ++i) f[i] = o[i];
  const D3 Cb = d3(S.rest_com[3 * b], S.rest_com[3 * b + 1], S.rest_com[3 * b + 2]);
  for (int k = 0; k < kWsNbr; ++k) {
    float* g = f + kWsOwn + 8 * k;
    const int n = S.nbr[kWsNbr * b + k];
    if (n < 0) {
#pragma unroll
      for (int i = 0; i < 8; ++i) g[i] = 0.f;
      continue;
    }
    const float* on = own + (size_t)kWsOwn * n;
#pragma unroll
    for (int i = 0; i < 6; ++i) g[i] = on[i] - o[i];
    const D3 Cn = d3(S.rest_com[3 * n], S.rest_com[3 * n + 1], S.rest_com[3 * n + 2]);
    const D3 r0 = Cn - Cb;
    const D3 r1 = d3(r0.x + on[6] - o[6], r0.y + on[7] - o[7], r0.z + on[8] - o[8]);
    g[6] = (float)(sqrt(dot(r1, r1)) - sqrt(dot(r0, r0)));
    g[7] = (float)(S.mass[n] / S.mass[b]);
  }
  for (int i = 0; i < kWsFeat; ++i) {
    raw[(size_t)kWsFeat * b + i] = f[i];
    if (norm) norm[(size_t)kWsFeat * b + i] = (f[i] - fmean[i]) / fstd[i];
  }
}

// Whether cluster b falls back to the plain start: its predicted rigid-fit
// residual (output column kWsResidualCol, denormalised) is above `gate` (m);
// gate <= 0 applies every correction.
__device__ __forceinline__ bool ws_gated(const float* __restrict__ y, int ld, int b, const float* __restrict__ omean,
                                         const float* __restrict__ ostd, double gate) {
  if (!(gate > 0.0)) return false;
  const double lg = (double)(y[(size_t)ld * b + kWsResidualCol] * ostd[kWsResidualCol] + omean[kWsResidualCol]);
  return !(lg <= log10(gate));  // NaN predictions fall back too
}

// Velocity correction of every cluster from output rows y (stride ld),
// denormalised as y * std + mean; gated clusters are left alone and counted.
__global__ void k_ws_apply_velocity(int nb, Body* __restrict__ bodies, const float* __restrict__ y, int ld,
                                    const float* __restrict__ omean, const float* __restrict__ ostd, double gate,
                                    int* __restrict__ fallbacks) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  if (ws_gated(y, ld, b, omean, ostd, gate)) {
    atomicAdd(fallbacks, 1);
    return;
  }
  Body& B = bodies[b];
  for (int d = 0; d < 3; ++d) {
    B.comdot[d] += (double)(y[(size_t)ld * b + d] * ostd[d] + omean[d]);
    B.omega[d] += (double)(y[(size_t)ld * b + 3 + d] * ostd[3 + d] + omean[3 + d]);
  }
}

// Starting boundary multipliers: every boundary vertex of cluster b starts
// at the cluster's predicted multiplier (one CTA per cluster).
__global__ void k_ws_apply_lambda(WsStatic S, double* __restrict__ lamB, const float* __restrict__ y, int ld,
                                  const float* __restrict__ omean, const float* __restrict__ ostd, double gate) {
  const int b = blockIdx.x;
  if (ws_gated(y, ld, b, omean, ostd, gate)) return;
  const double l = (double)(y[(size_t)ld * b + 6] * ostd[6] + omean[6]);
  for (int i = S.bnd_off[b] + threadIdx.x; i < S.bnd_off[b + 1]; i += blockDim.x) lamB[i] = l;
}

// Targets of every cluster from the converged step (one CTA per cluster):
// the velocity corrections that make the rigid step land on the best-fit
// rigid motion from the step-start positions x0 to the final positions, and
// the mean final boundary multiplier of the layer.
template <typename R>
__global__ void __launch_bounds__(256) k_ws_targets(WsStatic S, const R4<R>* __restrict__ pos,
                                                    const R4<R>* __restrict__ x0, const double* __restrict__ rec,
                                                    const double* __restrict__ lamB, double h,
                                                    float* __restrict__ target) {
  const int b = blockIdx.x;
  const double* r = rec + (size_t)kWsRec * b;
  const D3 c0 = d3(r[0], r[1], r[2]);
  const int beg = S.body_vert_off[b], end = S.body_vert_off[b + 1];
  double s[4] = {0, 0, 0, 0};
  for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int v = S.body_verts[i];
    const double m = S.vmass[v];
    const R4<R> p = pos[v];
    s[0] += m; s[1] += m * (double)p.x; s[2] += m * (double)p.y; s[3] += m * (double)p.z;
  }
  block_sum<4>(s);
  const D3 c1 = d3(s[1] / s[0], s[2] / s[0], s[3] / s[0]);
  double a[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int v = S.body_verts[i];
    const double m = S.vmass[v];
    const R4<R> p = pos[v], q = x0[v];
    const D3 x = d3((double)p.x, (double)p.y, (double)p.z) - c1;
    const D3 y = d3((double)q.x, (double)q.y, (double)q.z) - c0;
    a[0] += m * x.x * y.x; a[1] += m * x.y * y.x; a[2] += m * x.z * y.x;
    a[3] += m * x.x * y.y; a[4] += m * x.y * y.y; a[5] += m * x.z * y.y;
    a[6] += m * x.x * y.z; a[7] += m * x.y * y.z; a[8] += m * x.z * y.z;
  }
  for (int i = S.bnd_off[b] + threadIdx.x; i < S.bnd_off[b + 1]; i += blockDim.x) a[9] += lamB[i];
  block_sum<10>(a);
  __shared__ double sR[9];
  if (threadIdx.x == 0) polar_rotation(a, sR);
  __syncthreads();
  // residual of the fit: sum m |(x - c1) - R (x0 - c0)|^2
  double q[1] = {0.0};
  for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int v = S.body_verts[i];
    const double m = S.vmass[v];
    const R4<R> p = pos[v], o = x0[v];
    const D3 x = d3((double)p.x, (double)p.y, (double)p.z) - c1;
    const D3 y = d3((double)o.x, (double)o.y, (double)o.z) - c0;
    const D3 e = d3(x.x - (sR[0] * y.x + sR[3] * y.y + sR[6] * y.z), x.y - (sR[1] * y.x + sR[4] * y.y + sR[7] * y.z),
                    x.z - (sR[2] * y.x + sR[5] * y.y + sR[8] * y.z));
    q[0] += m * dot(e, e);
  }
  block_sum<1>(q);
  if (threadIdx.x == 0) {
    const double* Rm = sR;
    const D3 w = (1.0 / h) * rotation_log(Rm);
    float* t = target + (size_t)kWsOut * b;
    t[0] = (float)((c1.x - c0.x) / h - r[3]);
    t[1] = (float)((c1.y - c0.y) / h - r[4]);
    t[2] = (float)((c1.z - c0.z) / h - r[5]);
    t[3] = (float)(w.x - r[6]);
    t[4] = (float)(w.y - r[7]);
    t[5] = (float)(w.z - r[8]);
    const int nbv = S.bnd_off[b + 1] - S.bnd_off[b];
    t[6] = (float)(nbv > 0 ? a[9] / nbv : 0.0);
    t[kWsResidualCol] = (float)log10(fmax(sqrt(q[0] / s[0]), 1e-9));
  }
}

// ---------------------------------------------------------------------------
// Multiplier warm start of the last layer.  The reference zeroes every tet's
// multipliers at the start of a step (xpbdLayer3D.m:666), so projectGS
// rebuilds them from zero and the stiff tets need most of the iterations to
// the residual.  Here the last layer (the fine layer, where every tet is
// elastic) may start from the previous steps' converged multipliers,
//   lambda0 = a lambda_{n-1} + b (lambda_{n-1} - lambda_{n-2}).
// Within one layer XPBD keeps x - x_c = M^-1 grad C^T (lambda -
// lambda_c) along its iterations (x_c, lambda_c: the state the layer starts
// from), so replacing lambda_c by lambda0 moves the positions by
// M^-1 grad C(x)^T (lambda0 - lambda_c): the layer then converges to the same
// fixed point from a nearer start.  (The coarse layers are not warm-started:
// they snap boundary vertices to their rigid bodies, which breaks that
// relation.)  The stop rules decide convergence exactly as in the plain solve.
// Measured on B200: on the Neo-Hookean blocks the layer needs <= 5 % fewer
// iterations to the residual, and the positions it converges to differ from
// the plain solve's by 3e-4 to 6e-4 of the bounding-box diagonal after one
// step (the plain solve's own positions at residual 1e-4 and 1e-5 differ by
// ~1e-6): the constraints' gradients turn along the iterations, so the
// fixed point depends on the path.  It is an option, off by default.

// lambda0 for the tets of one colour (they share no vertex) and the position
// shift it implies, on the unpinned DOFs.  Rows: 2 for the Neo-Hookean pair, 6
// for StVK.  `seen` = steps already saved: lambda_{n-1} and lambda_{n-2}
// exist only after one and two steps.
template <typename R, int MAT>
__global__ void __launch_bounds__(256) k_ws_lambda_shift(TetData<R> td, int begin, int count,
                                                         R4<R>* __restrict__ pos,
                                                         const unsigned char* __restrict__ pin_mask,
                                                         const R* __restrict__ lam1, const R* __restrict__ lam2,
                                                         double a, double b, const int* __restrict__ seen) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int s = begin + i, T = td.T;
  const int n = *seen;
  if (n < 1) return;  // nothing saved yet: the plain start
  if (n < 2) b = 0.0;
  constexpr int kRows = MAT == MAT_NH ? 2 : 6;
  R dl[kRows];
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const size_t k = (size_t)q * T + s;
    const double l1 = (double)lam1[k], l2 = (double)lam2[k];
    const R l0 = (R)(a * l1 + b * (l1 - l2));
    dl[q] = l0 - td.lambda[k];
    td.lambda[k] = l0;
  }
  int4 v;
  R G[9], minv[4];
  V3<R> X[4];
  load_tet<R>(td, s, pos, v, G, X, minv);
  V3<R> dx[4];
  if (MAT == MAT_NH) {
    NHEval<R> e;
    nh_eval<R>(X, G, (double)td.mat[s], (double)td.mat[(size_t)T + s], 0.0, e);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const R m = minv[k];
      dx[k] = {m * (dl[0] * e.gD[k].x + dl[1] * e.gH[k].x), m * (dl[0] * e.gD[k].y + dl[1] * e.gH[k].y),
               m * (dl[0] * e.gD[k].z + dl[1] * e.gH[k].z)};
    }
  } else {
    StrainKin<R> kin;
    strain_kin<R>(X, G, kin);
    const R half = R(0.5), vol = td.vol[s];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const R c0 = dl[0] * kin.d[k][0] + half * (dl[3] * kin.d[k][1] + dl[4] * kin.d[k][2]);
      const R c1 = dl[1] * kin.d[k][1] + half * (dl[3] * kin.d[k][0] + dl[5] * kin.d[k][2]);
      const R c2 = dl[2] * kin.d[k][2] + half * (dl[4] * kin.d[k][0] + dl[5] * kin.d[k][1]);
      const R sc = minv[k] * vol;
      const V3<R> d = vaxpy3(c0, kin.f[0], c1, kin.f[1], c2, kin.f[2]);
      dx[k] = {sc * d.x, sc * d.y, sc * d.z};
    }
  }
  const int vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const unsigned char pm = pin_mask[vv[k]];
    R4<R> r = pos[vv[k]];
    if (!(pm & 1)) r.x += dx[k].x;
    if (!(pm & 2)) r.y += dx[k].y;
    if (!(pm & 4)) r.z += dx[k].z;
    pos[vv[k]] = r;
  }
}

// End of a step: lambda_{n-2} <- lambda_{n-1} <- lambda (rows x T), and one
// more step seen (counted up to 2).
template <typename R>
__global__ void k_ws_lambda_save(long long n, const R* __restrict__ lam, R* __restrict__ lam1, R* __restrict__ lam2,
                                 int* __restrict__ seen) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && *seen < 2) *seen += 1;
  if (i >= n) return;
  lam2[i] = lam1[i];
  lam1[i] = lam[i];
}

}  // namespace mlx
