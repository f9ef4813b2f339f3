// tet_kernels.cuh -- per-tet constraint projection and residual kernels.
//
// One thread projects one tet of the current colour (tets of one colour share
// no vertex, xpbdLayer3D.m:374-377).  Tet rest data is stored structure-of-
// arrays in colour-sorted order, so the threads of a warp read consecutive
// words of every field; the four vertex records are gathered with one vector
// load each (position + inverse mass).
#pragma once

#include "common.cuh"

namespace mlx {

// material encodings of the per-tet compliance block
enum MatKind : int {
  MAT_STVK_BLOCKS = 0,  // alpha and alpha*beta blocks, 24 values per tet
  MAT_STVK_LAME = 1,    // mu, lambda, alpha1 -> blocks formed in registers
  MAT_NH = 2            // 1/(vol mu), 1/(vol (lambda - mu)) or 0 (stable Neo-Hookean D/H pair)
};
__host__ __device__ constexpr int mat_stride(int kind) {
  return kind == MAT_STVK_BLOCKS ? 24 : (kind == MAT_STVK_LAME ? 3 : 2);
}

template <typename R> struct V3 { R x, y, z; };
template <typename R> __device__ __forceinline__ V3<R> v3r(R x, R y, R z) { return {x, y, z}; }
template <typename R> __device__ __forceinline__ V3<R> vsub(V3<R> a, V3<R> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename R> __device__ __forceinline__ R vdot(V3<R> a, V3<R> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename R> __device__ __forceinline__ V3<R> vcross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename R> __device__ __forceinline__ V3<R> vaxpy3(R a, V3<R> u, R b, V3<R> v, R c, V3<R> w) {
  return {a * u.x + b * v.x + c * w.x, a * u.y + b * v.y + c * w.y, a * u.z + b * v.z + c * w.z};
}

// 3x3 solve A x = b by Gaussian elimination with partial pivoting (the
// pagemldivide of matStvkVoigtConstraint3D.m:42).  A is row-major here.
template <typename R> __device__ __forceinline__ void solve3x3(R A[3][3], R b[3], R x[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    int p = k;
    R best = fabs(A[k][k]);
#pragma unroll
    for (int r = k + 1; r < 3; ++r) {
      R v = fabs(A[r][k]);
      if (v > best) { best = v; p = r; }
    }
    // swap rows k and p with compile-time indices only (keeps A in registers)
#pragma unroll
    for (int r = k + 1; r < 3; ++r) {
      if (p == r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) { R t = A[k][c]; A[k][c] = A[r][c]; A[r][c] = t; }
        R t = b[k]; b[k] = b[r]; b[r] = t;
      }
    }
#pragma unroll
    for (int r = k + 1; r < 3; ++r) {
      R f = A[r][k] / A[k][k];
#pragma unroll
      for (int c = k; c < 3; ++c) A[r][c] -= f * A[k][c];
      b[r] -= f * b[k];
    }
  }
#pragma unroll
  for (int k = 2; k >= 0; --k) {
    R s = b[k];
#pragma unroll
    for (int c = k + 1; c < 3; ++c) s -= A[k][c] * x[c];
    x[k] = s / A[k][k];
  }
}

// Compliance of one tet in the form the projection needs:
// alphaTilde top block (3x3, row-major), alphaTilde shear diagonal,
// gamma = alphaTilde*betaTilde/h top block and shear diagonal.
template <typename R> struct Compliance {
  R aT[3][3];
  R aS[3];
  R gT[3][3];
  R gS[3];
};

template <typename R, int MAT>
__device__ __forceinline__ void load_compliance(const R* __restrict__ mat, int s, int T, R inv_h2,
                                                R inv_h, Compliance<R>& c, bool need_gamma) {
  if (MAT == MAT_STVK_BLOCKS) {
#pragma unroll
    for (int col = 0; col < 3; ++col)
#pragma unroll
      for (int row = 0; row < 3; ++row) c.aT[row][col] = mat[(size_t)(row + 3 * col) * T + s] * inv_h2;
#pragma unroll
    for (int q = 0; q < 3; ++q) c.aS[q] = mat[(size_t)(9 + q) * T + s] * inv_h2;
    if (need_gamma) {
#pragma unroll
      for (int col = 0; col < 3; ++col)
#pragma unroll
        for (int row = 0; row < 3; ++row) c.gT[row][col] = mat[(size_t)(12 + row + 3 * col) * T + s] * inv_h;
#pragma unroll
      for (int q = 0; q < 3; ++q) c.gS[q] = mat[(size_t)(21 + q) * T + s] * inv_h;
    } else {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        c.gS[i] = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j) c.gT[i][j] = 0;
      }
    }
  } else {  // MAT_STVK_LAME: K = [lam+4mu lam lam; ...] (+) 2mu I (Mesh3D.m:449-456)
    R mu = mat[s], lam = mat[(size_t)T + s], a1 = mat[(size_t)2 * T + s];
    R inv4mu = R(1) / (R(4) * mu);
    R den = R(1) / (R(4) * mu + R(3) * lam);
    R dg = inv4mu * (R(4) * mu + R(2) * lam) * den;
    R off = -inv4mu * lam * den;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) c.aT[i][j] = (i == j ? dg : off) * inv_h2;
    R sh = R(1) / (R(2) * mu) * inv_h2;
    c.aS[0] = c.aS[1] = c.aS[2] = sh;
    // beta = alpha1*K and alpha = inv(K) give alpha*beta = alpha1*I
    R g = a1 * inv_h;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      c.gS[i] = g;
#pragma unroll
      for (int j = 0; j < 3; ++j) c.gT[i][j] = (i == j ? g : R(0));
    }
  }
}

// Green-strain kinematics shared by projection and residual
// (StVKconstraintGrad3D.m:1-70 in analytic form): f_i = sum_k (x0-x_k)
// DmInv(k,i), d[a][i] = coefficient of x_a in f_i.
template <typename R> struct StrainKin {
  V3<R> f[3];
  R d[4][3];
};
template <typename R>
__device__ __forceinline__ void strain_kin(const V3<R> X[4], const R G[9], StrainKin<R>& k) {
  V3<R> e1 = vsub(X[0], X[1]), e2 = vsub(X[0], X[2]), e3 = vsub(X[0], X[3]);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    k.f[i] = vaxpy3(G[0 + 3 * i], e1, G[1 + 3 * i], e2, G[2 + 3 * i], e3);
    k.d[0][i] = G[0 + 3 * i] + G[1 + 3 * i] + G[2 + 3 * i];
    k.d[1][i] = -G[0 + 3 * i];
    k.d[2][i] = -G[1 + 3 * i];
    k.d[3][i] = -G[2 + 3 * i];
  }
}

// ---------------------------------------------------------------------------
// StVK "Voigt" projection of one tet: matStvkVoigtConstraint3D.m:1-22 with the
// block-decoupled solve of decomposeSolve (:31-45).  Returns dx (in X) and
// dlambda.
template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void stvk_project(V3<R> X[4], const V3<R>* Xold, const R minv[4],
                                             const R G[9], R vol, const Compliance<R>& cm,
                                             const R lam[6], R dl[6]) {
  StrainKin<R> k;
  strain_kin<R>(X, G, k);
  R FF[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i; j < 3; ++j) { FF[i][j] = vdot(k.f[i], k.f[j]); FF[j][i] = FF[i][j]; }
  R W[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i; j < 3; ++j) {
      R s = 0;
#pragma unroll
      for (int a = 0; a < 4; ++a) s += minv[a] * k.d[a][i] * k.d[a][j];
      W[i][j] = s; W[j][i] = s;
    }
  const R half = R(0.5);
  R C[6] = {vol * (half * FF[0][0] - half), vol * (half * FF[1][1] - half), vol * (half * FF[2][2] - half),
            vol * (half * FF[0][1]), vol * (half * FF[0][2]), vol * (half * FF[1][2])};
  R v2 = vol * vol;
  // numGamma = gamma * (gradC * (x - xprev))
  R ng[6] = {0, 0, 0, 0, 0, 0};
  if (DAMP) {
    V3<R> dX[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) dX[a] = vsub(X[a], Xold[a]);
    V3<R> e1 = vsub(dX[0], dX[1]), e2 = vsub(dX[0], dX[2]), e3 = vsub(dX[0], dX[3]);
    V3<R> D[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) D[i] = vaxpy3(G[0 + 3 * i], e1, G[1 + 3 * i], e2, G[2 + 3 * i], e3);
    R gdx[6];
    gdx[0] = vol * vdot(k.f[0], D[0]);
    gdx[1] = vol * vdot(k.f[1], D[1]);
    gdx[2] = vol * vdot(k.f[2], D[2]);
    gdx[3] = vol * half * (vdot(k.f[0], D[1]) + vdot(k.f[1], D[0]));
    gdx[4] = vol * half * (vdot(k.f[0], D[2]) + vdot(k.f[2], D[0]));
    gdx[5] = vol * half * (vdot(k.f[1], D[2]) + vdot(k.f[2], D[1]));
#pragma unroll
    for (int r = 0; r < 3; ++r) ng[r] = cm.gT[r][0] * gdx[0] + cm.gT[r][1] * gdx[1] + cm.gT[r][2] * gdx[2];
#pragma unroll
    for (int q = 0; q < 3; ++q) ng[3 + q] = cm.gS[q] * gdx[3 + q];
  }
  // top block: ((I + gammaTop) * (gradCM gradC')_top + alphaTop) dl = b
  R GM[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) GM[i][j] = v2 * W[i][j] * FF[i][j];
  R A[3][3], b[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      R s = GM[r][c];
#pragma unroll
      for (int q = 0; q < 3; ++q) s += cm.gT[r][q] * GM[q][c];
      A[r][c] = s + cm.aT[r][c];
    }
    b[r] = -C[r] - (cm.aT[r][0] * lam[0] + cm.aT[r][1] * lam[1] + cm.aT[r][2] * lam[2]) - ng[r];
  }
  solve3x3<R>(A, b, dl);
  // shear rows: scalar solves with alphaTilde(4,4), DenomGamma(4,4)
  const int si[3] = {0, 0, 1}, sj[3] = {1, 2, 2};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    int i = si[q], j = sj[q];
    R S = v2 * R(0.25) * (W[i][i] * FF[j][j] + R(2) * W[i][j] * FF[i][j] + W[j][j] * FF[i][i]);
    dl[3 + q] = (-C[3 + q] - cm.aS[0] * lam[3 + q] - ng[3 + q]) / ((R(1) + cm.gS[0]) * S + cm.aS[0]);
  }
  // dx_a = minv_a vol sum_i c_i(a) f_i
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    R c0 = dl[0] * k.d[a][0] + half * (dl[3] * k.d[a][1] + dl[4] * k.d[a][2]);
    R c1 = dl[1] * k.d[a][1] + half * (dl[3] * k.d[a][0] + dl[5] * k.d[a][2]);
    R c2 = dl[2] * k.d[a][2] + half * (dl[4] * k.d[a][0] + dl[5] * k.d[a][1]);
    R s = minv[a] * vol;
    V3<R> dx = vaxpy3(c0, k.f[0], c1, k.f[1], c2, k.f[2]);
    X[a].x += s * dx.x;
    X[a].y += s * dx.y;
    X[a].z += s * dx.z;
  }
}

// StVK residual terms of one tet (simpleEvaluateAllConstraintResiduals,
// xpbdLayer3D.m:555-568): sum over components of (|C| - min(|C|, |aT*lambda|))^2
template <typename R>
__device__ __forceinline__ double stvk_residual(const V3<R> X[4], const R G[9], R vol,
                                                const Compliance<R>& cm, const R lam[6]) {
  StrainKin<R> k;
  strain_kin<R>(X, G, k);
  const R half = R(0.5);
  R C[6] = {vol * (half * vdot(k.f[0], k.f[0]) - half), vol * (half * vdot(k.f[1], k.f[1]) - half),
            vol * (half * vdot(k.f[2], k.f[2]) - half), vol * (half * vdot(k.f[0], k.f[1])),
            vol * (half * vdot(k.f[0], k.f[2])), vol * (half * vdot(k.f[1], k.f[2]))};
  R corr[6];
#pragma unroll
  for (int r = 0; r < 3; ++r) corr[r] = cm.aT[r][0] * lam[0] + cm.aT[r][1] * lam[1] + cm.aT[r][2] * lam[2];
#pragma unroll
  for (int q = 0; q < 3; ++q) corr[3 + q] = cm.aS[q] * lam[3 + q];
  double acc = 0;
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    double a = fabs((double)C[r]), c = fabs((double)corr[r]);
    double v = a - fmin(a, c);
    acc += v * v;
  }
  return acc;
}

// ---------------------------------------------------------------------------
// Stable Neo-Hookean tet, psi = mu/2 (I_C - 3) + lambda/2 (J - 1 - mu/lambda)^2
// (the energy of the 2D pair 2d/mex/mexNeoHookeanDConstraint.cpp /
// mexNeoHookeanHConstraint.cpp), written as two constraints that vanish at
// rest: psi = mu/2 B + (lambda - mu)/2 (J - 1)^2 + const with
// B = ||F||^2 + J^2 - 4J >= 0, so C_D = sqrt(B) (compliance 1/(vol mu)) and
// C_H = J - 1 (compliance 1/(vol (lambda - mu)), absent when lambda <= mu),
// solved as one 2x2 block.  The per-tet compliances cD = 1/(vol mu) and
// cH = 1/(vol (lambda - mu)) (0 = no C_H) are precomputed; alpha~ = c / h^2.
//
// Precision: F = Ds DmInv, the gradients G' [dC/dF] and the position update
// run in the storage precision R.  B, sqrt(B), J and the numerator
// F + (J - 2) cof(F) of dC_D/dF cancel to O(strain) near rest, so they are
// formed in FP64 from F; since B is stationary at rotations, rounding F to R
// moves B only by O(strain * eps_R).  The 2x2 solve is FP64.
template <typename R> struct NHEval {
  double CD, CH, aD, aH;
  bool hasH;
  V3<R> gD[4], gH[4];
};
template <typename R>
__device__ __forceinline__ void nh_eval(const V3<R> X[4], const R G[9], double cD, double cH, double inv_h2,
                                        NHEval<R>& e) {
  const V3<R> u1 = vsub(X[1], X[0]), u2 = vsub(X[2], X[0]), u3 = vsub(X[3], X[0]);
  D3 f[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    V3<R> fc = vaxpy3(G[0 + 3 * c], u1, G[1 + 3 * c], u2, G[2 + 3 * c], u3);
    f[c] = d3(fc.x, fc.y, fc.z);
  }
  D3 cf[3] = {cross(f[1], f[2]), cross(f[2], f[0]), cross(f[0], f[1])};
  double J = dot(f[0], cf[0]);
  double IC = dot(f[0], f[0]) + dot(f[1], f[1]) + dot(f[2], f[2]);
  double B = IC + J * J - 4.0 * J;
  e.CD = sqrt(fmax(B, 0.0));
  e.hasH = cH > 0.0;
  e.CH = e.hasH ? J - 1.0 : 0.0;
  e.aD = inv_h2 * cD;
  e.aH = e.hasH ? inv_h2 * cH : 0.0;
  const double invCD = e.CD > 1e-12 ? 1.0 / e.CD : 0.0;
  V3<R> pd[3], cr[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    D3 n = invCD * (f[c] + (J - 2.0) * cf[c]);
    pd[c] = {(R)n.x, (R)n.y, (R)n.z};
    cr[c] = {(R)cf[c].x, (R)cf[c].y, (R)cf[c].z};
  }
  V3<R> sD = {0, 0, 0}, sH = {0, 0, 0};
#pragma unroll
  for (int k = 1; k <= 3; ++k) {
    const R g0 = G[(k - 1) + 0], g1 = G[(k - 1) + 3], g2 = G[(k - 1) + 6];
    e.gD[k] = vaxpy3(g0, pd[0], g1, pd[1], g2, pd[2]);
    e.gH[k] = vaxpy3(g0, cr[0], g1, cr[1], g2, cr[2]);
    sD = {sD.x + e.gD[k].x, sD.y + e.gD[k].y, sD.z + e.gD[k].z};
    sH = {sH.x + e.gH[k].x, sH.y + e.gH[k].y, sH.z + e.gH[k].z};
  }
  e.gD[0] = {-sD.x, -sD.y, -sD.z};
  e.gH[0] = {-sH.x, -sH.y, -sH.z};
}

template <typename R>
__device__ __forceinline__ void nh_project(V3<R> X[4], const R minv[4], const R G[9], double cD, double cH,
                                           double inv_h2, const double lam[2], double dl[2]) {
  NHEval<R> e;
  nh_eval<R>(X, G, cD, cH, inv_h2, e);
  R wD = 0, wH = 0, wDH = 0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const R m = minv[a];
    wD += m * vdot(e.gD[a], e.gD[a]);
    wH += m * vdot(e.gH[a], e.gH[a]);
    wDH += m * vdot(e.gD[a], e.gH[a]);
  }
  const double b1 = -e.CD - e.aD * lam[0];
  if (e.hasH) {
    const double a11 = (double)wD + e.aD, a22 = (double)wH + e.aH, a12 = (double)wDH;
    const double b2 = -e.CH - e.aH * lam[1];
    const double rdet = 1.0 / (a11 * a22 - a12 * a12);
    dl[0] = (b1 * a22 - a12 * b2) * rdet;
    dl[1] = (a11 * b2 - a12 * b1) * rdet;
  } else {
    dl[0] = b1 / ((double)wD + e.aD);
    dl[1] = 0.0;
  }
  const R d0 = (R)dl[0], d1 = (R)dl[1];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const R m = minv[a];
    X[a].x += m * (d0 * e.gD[a].x + d1 * e.gH[a].x);
    X[a].y += m * (d0 * e.gD[a].y + d1 * e.gH[a].y);
    X[a].z += m * (d0 * e.gD[a].z + d1 * e.gH[a].z);
  }
}

// ---------------------------------------------------------------------------
// Rest data of the mesh in colour-sorted order.
template <typename R> struct TetData {
  const int4* vid;     // [T] 0-based vertex ids
  const R* dminv;      // [9][T] DmInv, column-major entry j of tet s at dminv[j*T+s]
  const R* vol;        // [T]
  const R* mat;        // [stride][T]
  R* lambda;           // [6][T]
  int T;
};

template <typename R>
__device__ __forceinline__ void load_tet(const TetData<R>& td, int s, const R4<R>* __restrict__ pos,
                                         int4& v, R G[9], V3<R> X[4], R minv[4]) {
  v = td.vid[s];
#pragma unroll
  for (int j = 0; j < 9; ++j) G[j] = td.dminv[(size_t)j * td.T + s];
  R4<R> p0 = ldcg_r4(pos + v.x), p1 = ldcg_r4(pos + v.y), p2 = ldcg_r4(pos + v.z), p3 = ldcg_r4(pos + v.w);
  X[0] = {p0.x, p0.y, p0.z}; X[1] = {p1.x, p1.y, p1.z};
  X[2] = {p2.x, p2.y, p2.z}; X[3] = {p3.x, p3.y, p3.z};
  minv[0] = p0.w; minv[1] = p1.w; minv[2] = p2.w; minv[3] = p3.w;
}

// Projection of one tet (colour-sorted id s) in place: gather, project,
// scatter, lambda += dlambda (xpbdLayer3D.m:358-377 for one element).
template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void project_tet(const TetData<R>& td, int s, R4<R>* __restrict__ pos,
                                            const R4<R>* __restrict__ oldp, R inv_h2, R inv_h) {
  int4 v;
  R G[9], minv[4];
  V3<R> X[4];
  load_tet<R>(td, s, pos, v, G, X, minv);
  R vol = td.vol[s];
  const int T = td.T;
  if (MAT == MAT_NH) {
    double cD = td.mat[s], cH = td.mat[(size_t)T + s];
    double lam[2] = {(double)td.lambda[s], (double)td.lambda[(size_t)T + s]}, dl[2];
    nh_project<R>(X, minv, G, cD, cH, (double)inv_h2, lam, dl);
    td.lambda[s] = (R)(lam[0] + dl[0]);
    td.lambda[(size_t)T + s] = (R)(lam[1] + dl[1]);
  } else {
    Compliance<R> cm;
    load_compliance<R, MAT>(td.mat, s, T, inv_h2, inv_h, cm, DAMP);
    R lam[6], dl[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) lam[q] = td.lambda[(size_t)q * T + s];
    V3<R> Xo[4];
    if (DAMP) {
      R4<R> o0 = oldp[v.x], o1 = oldp[v.y], o2 = oldp[v.z], o3 = oldp[v.w];
      Xo[0] = {o0.x, o0.y, o0.z}; Xo[1] = {o1.x, o1.y, o1.z};
      Xo[2] = {o2.x, o2.y, o2.z}; Xo[3] = {o3.x, o3.y, o3.z};
    }
    stvk_project<R, MAT, DAMP>(X, Xo, minv, G, vol, cm, lam, dl);
#pragma unroll
    for (int q = 0; q < 6; ++q) td.lambda[(size_t)q * T + s] = lam[q] + dl[q];
  }
  stcg_r4(pos + v.x, make_r4<R>(X[0].x, X[0].y, X[0].z, minv[0]));
  stcg_r4(pos + v.y, make_r4<R>(X[1].x, X[1].y, X[1].z, minv[1]));
  stcg_r4(pos + v.z, make_r4<R>(X[2].x, X[2].y, X[2].z, minv[2]));
  stcg_r4(pos + v.w, make_r4<R>(X[3].x, X[3].y, X[3].z, minv[3]));
}

// Largest block of a colour kernel (the tile autotuner's candidates stay
// within it; FP64 variants need up to ~220 registers per thread).
constexpr int kMaxColorTile = 256;

// Programmatic dependent launch: a colour kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization starts while the previous
// kernel of the stream still runs; griddepcontrol.wait blocks until that
// kernel has completed and its writes are visible (a no-op without the
// attribute).  launch_dependents lets the next colour start early in turn.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

// One colour of the Gauss-Seidel sweep (xpbdLayer3D.m:357-378).  `list` holds
// the colour-sorted ids of this layer's elastic tets of this colour; NULL
// means the identity over [begin, begin+count).  The tet's read-only data
// (ids, DmInv, volume, material) is loaded before waiting on the previous
// colour; positions and multipliers after.
template <typename R, int MAT, bool DAMP>
__device__ __forceinline__ void project_color_tet(const TetData<R>& td, const int* __restrict__ list, int begin,
                                                  int count, int i, R4<R>* __restrict__ pos,
                                                  const R4<R>* __restrict__ oldp, R inv_h2, R inv_h) {
  const bool active = i < count;
  const int T = td.T;
  int s = 0;
  int4 v = make_int4(0, 0, 0, 0);
  R G[9], vol = 0, mat[mat_stride(MAT)];
  if (active) {
    s = list ? list[begin + i] : begin + i;
    v = td.vid[s];
#pragma unroll
    for (int j = 0; j < 9; ++j) G[j] = td.dminv[(size_t)j * T + s];
    vol = td.vol[s];
#pragma unroll
    for (int q = 0; q < mat_stride(MAT); ++q) mat[q] = td.mat[(size_t)q * T + s];
  }
  pdl_wait();
  if (!active) return;
  R4<R> p0 = ldcg_r4(pos + v.x), p1 = ldcg_r4(pos + v.y), p2 = ldcg_r4(pos + v.z), p3 = ldcg_r4(pos + v.w);
  V3<R> X[4] = {{p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}, {p3.x, p3.y, p3.z}};
  R minv[4] = {p0.w, p1.w, p2.w, p3.w};
  if (MAT == MAT_NH) {
    double lam[2] = {(double)td.lambda[s], (double)td.lambda[(size_t)T + s]}, dl[2];
    nh_project<R>(X, minv, G, (double)mat[0], (double)mat[1], (double)inv_h2, lam, dl);
    td.lambda[s] = (R)(lam[0] + dl[0]);
    td.lambda[(size_t)T + s] = (R)(lam[1] + dl[1]);
  } else {
    Compliance<R> cm;
    load_compliance<R, MAT>(mat, 0, 1, inv_h2, inv_h, cm, DAMP);
    R lam[6], dl[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) lam[q] = td.lambda[(size_t)q * T + s];
    V3<R> Xo[4];
    if (DAMP) {
      R4<R> o0 = oldp[v.x], o1 = oldp[v.y], o2 = oldp[v.z], o3 = oldp[v.w];
      Xo[0] = {o0.x, o0.y, o0.z}; Xo[1] = {o1.x, o1.y, o1.z};
      Xo[2] = {o2.x, o2.y, o2.z}; Xo[3] = {o3.x, o3.y, o3.z};
    }
    stvk_project<R, MAT, DAMP>(X, Xo, minv, G, vol, cm, lam, dl);
#pragma unroll
    for (int q = 0; q < 6; ++q) td.lambda[(size_t)q * T + s] = lam[q] + dl[q];
  }
  stcg_r4(pos + v.x, make_r4<R>(X[0].x, X[0].y, X[0].z, minv[0]));
  stcg_r4(pos + v.y, make_r4<R>(X[1].x, X[1].y, X[1].z, minv[1]));
  stcg_r4(pos + v.z, make_r4<R>(X[2].x, X[2].y, X[2].z, minv[2]));
  stcg_r4(pos + v.w, make_r4<R>(X[3].x, X[3].y, X[3].z, minv[3]));
}

template <typename R, int MAT, bool DAMP>
__global__ void __launch_bounds__(kMaxColorTile) k_project_color(TetData<R> td, const int* __restrict__ list,
                                                       int begin, int count, R4<R>* __restrict__ pos,
                                                       const R4<R>* __restrict__ oldp, R inv_h2, R inv_h) {
  pdl_launch_dependents();
  project_color_tet<R, MAT, DAMP>(td, list, begin, count, blockIdx.x * blockDim.x + threadIdx.x, pos, oldp, inv_h2,
                                  inv_h);
}

// ---------------------------------------------------------------------------
// Deterministic block sum of NV doubles (fixed shuffle tree + fixed warp
// order).  All threads get the result.  blockDim.x must be a multiple of 32.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[32][NV];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) sh[warp][q] = v[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double x = lane < nw ? sh[lane][q] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) sh[0][q] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = sh[0][q];
  __syncthreads();
}

struct ContactData {
  int K;
  const double* normal;     // [3][K]
  const double* point;      // [3][K]
  const double* compliance; // [K]
  const int* vid;           // [K] 0-based
  double* lambda;           // [K]
  // the distinct compliance values and how many contacts carry each (first
  // occurrence order; ncomp = 0 when there are more than kMaxCompliances)
  int ncomp;
  const double* comp_vals;  // [ncomp]
  const int* comp_counts;   // [ncomp]
};
constexpr int kMaxCompliances = 32;

// Residual partial sums over all tets (blocks [0, tetBlocks)) and all
// contacts (the remaining blocks), one double per block
// (simpleEvaluateAllConstraintResiduals, xpbdLayer3D.m:546-586).
// This thread's sum of the tets' residual terms over the grid-stride range
// starting at `first` (stride `stride`).
template <typename R, int MAT>
__device__ __forceinline__ double residual_tets(const TetData<R>& td, const R4<R>* __restrict__ pos, R inv_h2,
                                                R inv_h, double inv_h2_d, int first, int stride) {
  double acc[1] = {0.0};
  {
    for (int s = first; s < td.T; s += stride) {
      int4 v;
      R G[9], minv[4];
      V3<R> X[4];
      load_tet<R>(td, s, pos, v, G, X, minv);
      R vol = td.vol[s];
      const int T = td.T;
      if (MAT == MAT_NH) {
        NHEval<R> e;
        nh_eval<R>(X, G, (double)td.mat[s], (double)td.mat[(size_t)T + s], inv_h2_d, e);
        double l0 = td.lambda[s], l1 = td.lambda[(size_t)T + s];
        double a = fabs(e.CD), c = fabs(e.aD * l0);
        double r0 = a - fmin(a, c);
        a = fabs(e.CH); c = fabs(e.aH * l1);
        double r1 = a - fmin(a, c);
        acc[0] += r0 * r0 + r1 * r1;
      } else {
        Compliance<R> cm;
        load_compliance<R, MAT>(td.mat, s, T, inv_h2, inv_h, cm, false);
        R lam[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) lam[q] = td.lambda[(size_t)q * T + s];
        acc[0] += stvk_residual<R>(X, G, vol, cm, lam);
      }
    }
  }
  return acc[0];
}

template <typename R, int MAT>
__global__ void __launch_bounds__(256) k_residual_partials(TetData<R> td, const R4<R>* __restrict__ pos,
                                                           ContactData cd, double contact_resistance,
                                                           R inv_h2, R inv_h, double inv_h2_d,
                                                           int tetBlocks, double* __restrict__ partials) {
  double acc[1] = {0.0};
  if ((int)blockIdx.x < tetBlocks) {
    acc[0] = residual_tets<R, MAT>(td, pos, inv_h2, inv_h, inv_h2_d, blockIdx.x * blockDim.x + threadIdx.x,
                                   tetBlocks * blockDim.x);
  } else {
    // contacts: the reference's correction term is the K x 1 x K implicit
    // expansion of (compliance/h^2) (1x1xK) times lambda (Kx1)
    // (xpbdLayer3D.m:581-583), so contact k meets every compliance j; the
    // contacts sharing a compliance give equal terms, so with few distinct
    // compliances each is taken once, times its count (O(K) instead of
    // O(K^2))
    int cb = blockIdx.x - tetBlocks, ncb = gridDim.x - tetBlocks;
    for (int k = cb * blockDim.x + threadIdx.x; k < cd.K; k += ncb * blockDim.x) {
      R4<R> p = ldcg_r4(pos + cd.vid[k]);
      double n0 = cd.normal[k], n1 = cd.normal[cd.K + k], n2 = cd.normal[2 * cd.K + k];
      double phi = n0 * ((double)p.x - cd.point[k]) + n1 * ((double)p.y - cd.point[cd.K + k]) +
                   n2 * ((double)p.z - cd.point[2 * cd.K + k]);
      if (phi > 0) phi = 0;
      double a = fabs(contact_resistance * phi);
      double lk = cd.lambda[k];
      if (cd.ncomp > 0) {
        for (int g = 0; g < cd.ncomp; ++g) {
          const double r = a - fmin(a, fabs((cd.comp_vals[g] * inv_h2_d) * lk));
          acc[0] += (double)cd.comp_counts[g] * (r * r);
        }
      } else {
        for (int j = 0; j < cd.K; ++j) {
          double c = fabs((cd.compliance[j] * inv_h2_d) * lk);
          double r = a - fmin(a, c);
          acc[0] += r * r;
        }
      }
    }
  }
  block_sum<1>(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

// Sums `n` partials in index order (one block) and writes sqrt of the sum.
// (A template so that every translation unit can instantiate it.)
template <int kBlock = 256>
__global__ void __launch_bounds__(kBlock) k_finish_norm(const double* __restrict__ partials, int n,
                                                     double* __restrict__ out) {
  double acc[1] = {0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc[0] += partials[i];
  block_sum<1>(acc);
  if (threadIdx.x == 0) *out = sqrt(acc[0]);
}

}  // namespace mlx
