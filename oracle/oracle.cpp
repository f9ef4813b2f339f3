// oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A plain, single-threaded-by-default FP64 C++ restatement of the reference's
// multi-layer XPBD step (AlexandreMercierAubin/MultiLayerSolver2024).  It is the
// parity checker for the CUDA product path and the timed CPU baseline; the
// product never links, loads or calls it.  Each function names the reference
// file:line it restates.  Vectorised MATLAB page operations are written as
// plain loops in the same order of evaluation where the order matters
// (gather -> compute -> scatter per colour, accumarray sums in index order).
//
// Parity pins: the Green-strain constraint and gradient are checked against
// values evaluated from the reference's own symbolic expressions
// (3d/constraints/StVKconstraintGrad3D.m), and the layer builder against the
// reference's mexUnionFindByVertice.cpp / mexEdiffNorm3D.cpp compiled unchanged
// (oracle/_ref).  The 3D Neo-Hookean constraint has no 3D reference (the 2D
// pair 2d/mex/mexNeoHookean{D,H}Constraint.cpp defines its energy); it is
// parity unpinned.
//
// Optional OpenMP: the per-colour tet loop and the residual loop run in
// parallel when compiled with -fopenmp and orc_set_threads(n>1) is called;
// tets of one colour share no vertex, so the result is identical.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <string>
#include <vector>
#include <algorithm>
#include <unordered_map>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/mlxpbd.h"

namespace {

int g_threads = 1;
thread_local std::string g_err;

int fail(int code, const std::string& msg) { g_err = msg; return code; }

// ---- small dense helpers (column-major 3x3: m[r + 3c]) --------------------
struct V3 { double x, y, z; };
inline V3 v3(double a, double b, double c) { return {a, b, c}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// MATLAB cross(a,b,2)
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 matvec(const double* M, V3 v) {  // M (3x3 col-major) * v
  return {M[0] * v.x + M[3] * v.y + M[6] * v.z,
          M[1] * v.x + M[4] * v.y + M[7] * v.z,
          M[2] * v.x + M[5] * v.y + M[8] * v.z};
}
inline void matmul3(const double* A, const double* B, double* C) {  // C = A*B
  double t[9];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += A[r + 3 * k] * B[k + 3 * c];
      t[r + 3 * c] = s;
    }
  std::memcpy(C, t, sizeof(t));
}
inline void matmul3_bt(const double* A, const double* B, double* C) {  // A*B'
  double t[9];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += A[r + 3 * k] * B[c + 3 * k];
      t[r + 3 * c] = s;
    }
  std::memcpy(C, t, sizeof(t));
}
// Gaussian elimination with partial pivoting (pagemldivide on an n x n page).
void mldivide(int n, const double* Ain, const double* bin, double* x) {
  double A[36], b[6];
  std::memcpy(A, Ain, sizeof(double) * n * n);
  std::memcpy(b, bin, sizeof(double) * n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::fabs(A[k + n * k]);
    for (int r = k + 1; r < n; ++r)
      if (std::fabs(A[r + n * k]) > best) { best = std::fabs(A[r + n * k]); p = r; }
    if (p != k) {
      for (int c = 0; c < n; ++c) std::swap(A[k + n * c], A[p + n * c]);
      std::swap(b[k], b[p]);
    }
    for (int r = k + 1; r < n; ++r) {
      double f = A[r + n * k] / A[k + n * k];
      for (int c = k; c < n; ++c) A[r + n * c] -= f * A[k + n * c];
      b[r] -= f * b[k];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    double s = b[k];
    for (int c = k + 1; c < n; ++c) s -= A[k + n * c] * x[c];
    x[k] = s / A[k + n * k];
  }
}
inline V3 solve3(const double* M, V3 b) {
  double bb[3] = {b.x, b.y, b.z}, x[3];
  mldivide(3, M, bb, x);
  return {x[0], x[1], x[2]};
}

// expRodrigues (3d/tools/math/expRodrigues.m:1-15) with crossProductMatrix
// (3d/tools/math/crossProductMatrix.m:1-8).
void exp_rodrigues(V3 omega, double h, double* R) {
  double mag = std::sqrt(omega.x * omega.x + omega.y * omega.y + omega.z * omega.z);
  double w[3] = {omega.x / mag, omega.y / mag, omega.z / mag};
  for (double& c : w) if (std::isnan(c)) c = 0;  // "can happen when there is no rotation"
  double theta = h * mag;
  double K[9] = {0, w[2], -w[1], -w[2], 0, w[0], w[1], -w[0], 0};
  double K2[9];
  matmul3(K, K, K2);
  double s = std::sin(theta), c1 = 1 - std::cos(theta);
  for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0 ? 1.0 : 0.0) + s * K[i] + c1 * K2[i];
}

// Green-strain constraint and gradient of StVKconstraintGrad3D.m:1-70 in
// analytic form.  f_i = sum_k (x0 - x_k) DmInv(k,i) (the file's t50..t58),
// C = [E11 E22 E33 E12 E13 E23] with E = (F'F - I)/2 (off-diagonals not
// doubled), gradC 6 x 12 column-major.
void stvk_grad(const double* DmInv, const double* x, double* gradC, double* C) {
  V3 X[4];
  for (int a = 0; a < 4; ++a) X[a] = v3(x[3 * a], x[3 * a + 1], x[3 * a + 2]);
  V3 f[3];
  for (int i = 0; i < 3; ++i) {
    V3 s = v3(0, 0, 0);
    for (int k = 1; k <= 3; ++k) {
      V3 d = sub(X[0], X[k]);
      double g = DmInv[(k - 1) + 3 * i];
      s = add(s, v3(g * d.x, g * d.y, g * d.z));
    }
    f[i] = s;
  }
  // d(a,i): coefficient of x_a in f_i
  double d[4][3];
  for (int i = 0; i < 3; ++i) {
    d[0][i] = DmInv[0 + 3 * i] + DmInv[1 + 3 * i] + DmInv[2 + 3 * i];
    for (int k = 1; k <= 3; ++k) d[k][i] = -DmInv[(k - 1) + 3 * i];
  }
  C[0] = 0.5 * dot(f[0], f[0]) - 0.5;
  C[1] = 0.5 * dot(f[1], f[1]) - 0.5;
  C[2] = 0.5 * dot(f[2], f[2]) - 0.5;
  C[3] = 0.5 * dot(f[0], f[1]);
  C[4] = 0.5 * dot(f[0], f[2]);
  C[5] = 0.5 * dot(f[1], f[2]);
  const int pi[6] = {0, 1, 2, 0, 0, 1}, pj[6] = {0, 1, 2, 1, 2, 2};
  for (int r = 0; r < 6; ++r)
    for (int a = 0; a < 4; ++a) {
      V3 g;
      if (r < 3) {
        double c = d[a][r];
        g = v3(c * f[r].x, c * f[r].y, c * f[r].z);
      } else {
        int i = pi[r], j = pj[r];
        double ci = 0.5 * d[a][i], cj = 0.5 * d[a][j];
        g = v3(ci * f[j].x + cj * f[i].x, ci * f[j].y + cj * f[i].y, ci * f[j].z + cj * f[i].z);
      }
      gradC[r + 6 * (3 * a + 0)] = g.x;
      gradC[r + 6 * (3 * a + 1)] = g.y;
      gradC[r + 6 * (3 * a + 2)] = g.z;
    }
}

// matStvkVoigtConstraint3D (3d/constraints/matStvkVoigtConstraint3D.m:1-22)
// with decomposeSolve (:31-45).
void stvk_voigt_project(const double* x, const double* xprev, const double* DmInv,
                        const double* aT, const double* lambda, const double* minv,
                        double vol, const double* bT, double h, double* dx,
                        double* dlambda, double* Cout) {
  double gC[72], Ce[6];
  stvk_grad(DmInv, x, gC, Ce);
  double C[6], G[72], GM[72];
  for (int r = 0; r < 6; ++r) C[r] = Ce[r] * vol;
  for (int i = 0; i < 72; ++i) G[i] = gC[i] * vol;
  for (int c = 0; c < 12; ++c)
    for (int r = 0; r < 6; ++r) GM[r + 6 * c] = G[r + 6 * c] * minv[c];
  if (Cout) std::memcpy(Cout, C, sizeof(C));
  // gamma = alphaTilde*betaTilde ./ h
  double gamma[36];
  for (int c = 0; c < 6; ++c)
    for (int r = 0; r < 6; ++r) {
      double s = 0;
      for (int k = 0; k < 6; ++k) s += aT[r + 6 * k] * bT[k + 6 * c];
      gamma[r + 6 * c] = s / h;
    }
  // numGamma = (gamma * gradC) * (x - xprev), in that association order
  double gG[72];
  for (int c = 0; c < 12; ++c)
    for (int r = 0; r < 6; ++r) {
      double s = 0;
      for (int k = 0; k < 6; ++k) s += gamma[r + 6 * k] * G[k + 6 * c];
      gG[r + 6 * c] = s;
    }
  double numGamma[6];
  for (int r = 0; r < 6; ++r) {
    double s = 0;
    for (int c = 0; c < 12; ++c) s += gG[r + 6 * c] * (x[c] - xprev[c]);
    numGamma[r] = s;
  }
  double Den[36];
  for (int i = 0; i < 36; ++i) Den[i] = gamma[i] + ((i % 7 == 0) ? 1.0 : 0.0);
  // top 3x3 block
  double GMGt[9];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 12; ++k) s += GM[r + 6 * k] * G[c + 6 * k];
      GMGt[r + 3 * c] = s;
    }
  double A[9], b[3];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += Den[r + 6 * k] * GMGt[k + 3 * c];
      A[r + 3 * c] = s + aT[r + 6 * c];
    }
  for (int r = 0; r < 3; ++r) {
    double s = 0;
    for (int k = 0; k < 3; ++k) s += aT[r + 6 * k] * lambda[k];
    b[r] = -C[r] - s - numGamma[r];
  }
  double top[3];
  mldivide(3, A, b, top);
  for (int r = 0; r < 3; ++r) dlambda[r] = top[r];
  // shear rows: scalar solves with alphaTilde(4,4) and DenomGamma(4,4)
  for (int r = 3; r < 6; ++r) {
    double num = -C[r] - aT[3 + 6 * 3] * lambda[r] - numGamma[r];
    double bottom = 0;
    for (int k = 0; k < 12; ++k) bottom += GM[r + 6 * k] * G[r + 6 * k];
    dlambda[r] = num / (Den[3 + 6 * 3] * bottom + aT[3 + 6 * 3]);
  }
  for (int c = 0; c < 12; ++c) {
    double s = 0;
    for (int r = 0; r < 6; ++r) s += GM[r + 6 * c] * dlambda[r];
    dx[c] = s;
  }
}

// 3D stable Neo-Hookean constraint pair.  The 2D reference
// (2d/mex/mexNeoHookeanDConstraint.cpp, mexNeoHookeanHConstraint.cpp, gamma =
// 1 + mu/lambda at 2d/@Mesh/Mesh.m:244) projects C_D = ||F|| (compliance
// 1/mu) and C_H = det F - gamma (1/lambda), whose energy is the stable
// Neo-Hookean psi = mu/2 (I_C - 3) + lambda/2 (J - gamma)^2 + const.  In 3D the
// pair needs large multipliers at rest (C_D = sqrt 3 there) that XPBD rebuilds
// from zero every step, which drifts from rest for stiff tets.  The same
// energy is written here as two constraints that both vanish at rest:
//   psi = mu/2 B + (lambda - mu)/2 (J - 1)^2 + const,  B = ||F||^2 + J^2 - 4J,
// B >= 0 with B = 0 exactly for rotations, so
//   C_D = sqrt(B),  compliance 1/(vol mu);   C_H = J - 1, compliance
//   1/(vol (lambda - mu)) (dropped when lambda <= mu, i.e. nu <= 0.25);
// the pair is solved as one 2x2 block per tet (the block-solve style of
// matStvkVoigtConstraint3D.m:31-45).  F = Ds * DmInv, Ds = [x1-x0 x2-x0 x3-x0].
void nh_project(const double* x, const double* DmInv, double mu, double lam, double vol,
                double h, const double* lambda, const double* minv, double* dx,
                double* dlambda, double* Cout, double* alphaTildeOut) {
  V3 X[4];
  for (int a = 0; a < 4; ++a) X[a] = v3(x[3 * a], x[3 * a + 1], x[3 * a + 2]);
  double Ds[9];
  for (int k = 0; k < 3; ++k) {
    V3 d = sub(X[k + 1], X[0]);
    Ds[0 + 3 * k] = d.x; Ds[1 + 3 * k] = d.y; Ds[2 + 3 * k] = d.z;
  }
  double F[9];
  matmul3(Ds, DmInv, F);
  V3 f1 = v3(F[0], F[1], F[2]), f2 = v3(F[3], F[4], F[5]), f3 = v3(F[6], F[7], F[8]);
  V3 c1 = cross(f2, f3), c2 = cross(f3, f1), c3 = cross(f1, f2);
  double J = dot(f1, c1);
  double IC = 0;
  for (int i = 0; i < 9; ++i) IC += F[i] * F[i];
  double B = IC + J * J - 4 * J;
  double CD = std::sqrt(std::max(B, 0.0));
  double CH = J - 1;
  const bool hasH = lam > mu;
  double h2 = h * h;
  double aD = 1.0 / (vol * mu * h2);
  double aH = hasH ? 1.0 / (vol * (lam - mu) * h2) : 0.0;
  if (Cout) { Cout[0] = CD; Cout[1] = hasH ? CH : 0.0; }
  if (alphaTildeOut) { alphaTildeOut[0] = aD; alphaTildeOut[1] = aH; }
  // dC/dF: D -> (F + (J - 2) cof F) / C_D (zero at C_D = 0), H -> cof F
  double PD[9] = {0}, PH[9];
  PH[0] = c1.x; PH[1] = c1.y; PH[2] = c1.z;
  PH[3] = c2.x; PH[4] = c2.y; PH[5] = c2.z;
  PH[6] = c3.x; PH[7] = c3.y; PH[8] = c3.z;
  if (CD > 1e-12)
    for (int i = 0; i < 9; ++i) PD[i] = (F[i] + (J - 2) * PH[i]) / CD;
  // gradient wrt x_k (k=1..3) = column k of P * DmInv'; x0 gets minus the sum
  double GD[9], GH[9];
  matmul3_bt(PD, DmInv, GD);
  matmul3_bt(PH, DmInv, GH);
  double gD[12], gH[12];
  for (int k = 1; k <= 3; ++k)
    for (int a = 0; a < 3; ++a) {
      gD[3 * k + a] = GD[a + 3 * (k - 1)];
      gH[3 * k + a] = GH[a + 3 * (k - 1)];
    }
  for (int a = 0; a < 3; ++a) {
    gD[a] = -(gD[3 + a] + gD[6 + a] + gD[9 + a]);
    gH[a] = -(gH[3 + a] + gH[6 + a] + gH[9 + a]);
  }
  double wD = 0, wH = 0, wDH = 0;
  for (int c = 0; c < 12; ++c) {
    wD += minv[c] * gD[c] * gD[c];
    wH += minv[c] * gH[c] * gH[c];
    wDH += minv[c] * gD[c] * gH[c];
  }
  double b1 = -CD - aD * lambda[0];
  double dlD, dlH;
  if (hasH) {
    double a11 = wD + aD, a22 = wH + aH, a12 = wDH;
    double b2 = -CH - aH * lambda[1];
    double det = a11 * a22 - a12 * a12;
    dlD = (b1 * a22 - a12 * b2) / det;
    dlH = (a11 * b2 - a12 * b1) / det;
  } else {
    dlD = b1 / (wD + aD);
    dlH = 0;
  }
  dlambda[0] = dlD;
  dlambda[1] = dlH;
  for (int c = 0; c < 12; ++c) dx[c] = minv[c] * (gD[c] * dlD + gH[c] * dlH);
}

// Mesh arrays in MATLAB layout.
struct Mesh {
  int N, T, numColors;
  const int32_t* t;        // T x 4, 1-based
  const double* mass;      // 3N
  const double* DmInv;     // 3x3xT
  const double* vol;       // T
  const int32_t* color;    // T, 1-based
  const int32_t* pinned;   // 1-based DOFs
  int numPinned;
  int energy;
  std::vector<double> alpha, beta;   // 6x6xT
  std::vector<double> mu, lam;       // T
  int vid(int e, int k) const { return t[e + (size_t)T * k] - 1; }
};

// Mesh3D.updateMaterials compliance blocks (Mesh3D.m:445-460): K =
// [lam+4mu lam lam; ...] (+) 2mu*I, alpha = inv(K), beta = alpha1*K.
void material_blocks(double mu, double lam, double a1, double* alpha, double* alphaInv,
                     double* beta) {
  double K[36] = {0};
  double diagMu = 2 * mu, diagVal = lam + 2 * diagMu;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) K[r + 6 * c] = (r == c) ? diagVal : lam;
  for (int r = 3; r < 6; ++r) K[r + 6 * r] = diagMu;
  if (alphaInv) std::memcpy(alphaInv, K, sizeof(K));
  if (beta) for (int i = 0; i < 36; ++i) beta[i] = K[i] * a1;
  if (alpha) {
    // pageinv: solve K X = I column by column
    for (int c = 0; c < 6; ++c) {
      double e[6] = {0}, col[6];
      e[c] = 1;
      mldivide(6, K, e, col);
      for (int r = 0; r < 6; ++r) alpha[r + 6 * c] = col[r];
    }
  }
}

struct Bodies {
  int n = 0;
  std::vector<double> R, I0, I, COM, COMDOT, omega, M;  // 9n, 9n, 9n, 3n, 3n, 3n, n
};

// RigidBody3D.matComputeRigidBodyProperties3D (RigidBody3D.m:198-247) and
// buildInertiaTensor (:249-258), called from
// AdaptiveMesh3D.makeRigidsFromConnectivity (AdaptiveMesh3D.m:32-43).
void make_rigids(int nb, const int32_t* rigidIDbyVert, int N, const std::vector<double>& p,
                 const std::vector<double>& v, const double* mass, Bodies& B,
                 std::vector<double>& ri) {
  B.n = nb;
  B.R.assign(9 * nb, 0); B.I0.assign(9 * nb, 0); B.COM.assign(3 * nb, 0);
  B.COMDOT.assign(3 * nb, 0); B.omega.assign(3 * nb, 0); B.M.assign(nb, 0);
  for (int b = 0; b < nb; ++b) B.R[9 * b] = B.R[9 * b + 4] = B.R[9 * b + 8] = 1;
  std::vector<double> mp(3 * nb, 0), mv(3 * nb, 0);
  for (int i = 0; i < N; ++i) {
    int b = rigidIDbyVert[i];
    if (b == 0) continue;
    --b;
    double m = mass[3 * i];
    B.M[b] += m;
    for (int d = 0; d < 3; ++d) {
      mp[3 * b + d] += p[3 * i + d] * m;
      mv[3 * b + d] += v[3 * i + d] * m;
    }
  }
  for (int b = 0; b < nb; ++b)
    for (int d = 0; d < 3; ++d) {
      B.COM[3 * b + d] = mp[3 * b + d] / B.M[b];
      B.COMDOT[3 * b + d] = mv[3 * b + d] / B.M[b];
    }
  std::vector<double> Lm(3 * nb, 0);
  ri.assign(3 * (size_t)N, 0);
  for (int i = 0; i < N; ++i) {
    int b = rigidIDbyVert[i];
    if (b == 0) continue;
    --b;
    double m = mass[3 * i];
    V3 r = v3(p[3 * i] - B.COM[3 * b], p[3 * i + 1] - B.COM[3 * b + 1], p[3 * i + 2] - B.COM[3 * b + 2]);
    V3 vd = v3(v[3 * i] - B.COMDOT[3 * b], v[3 * i + 1] - B.COMDOT[3 * b + 1], v[3 * i + 2] - B.COMDOT[3 * b + 2]);
    ri[3 * i] = r.x; ri[3 * i + 1] = r.y; ri[3 * i + 2] = r.z;
    double K[9] = {0, r.z, -r.y, -r.z, 0, r.x, r.y, -r.x, 0}, K2[9];
    matmul3(K, K, K2);
    for (int k = 0; k < 9; ++k) B.I0[9 * b + k] += -m * K2[k];
    V3 c = cross(r, vd);
    Lm[3 * b] += m * c.x; Lm[3 * b + 1] += m * c.y; Lm[3 * b + 2] += m * c.z;
  }
  for (int b = 0; b < nb; ++b) {
    V3 w = solve3(&B.I0[9 * b], v3(Lm[3 * b], Lm[3 * b + 1], Lm[3 * b + 2]));
    B.omega[3 * b] = w.x; B.omega[3 * b + 1] = w.y; B.omega[3 * b + 2] = w.z;
  }
  B.I = B.I0;
}

// RigidBody3D.pageRelativeVertexPosition (RigidBody3D.m:193-196)
inline V3 rigid_pos(const Bodies& B, int b, const std::vector<double>& ri, int v) {
  V3 r = matvec(&B.R[9 * b], v3(ri[3 * v], ri[3 * v + 1], ri[3 * v + 2]));
  return add(r, v3(B.COM[3 * b], B.COM[3 * b + 1], B.COM[3 * b + 2]));
}

// xpbdLayer3D.rotateAllVerts (xpbdLayer3D.m:508-513)
void rotate_all_verts(const int32_t* rid, int N, const std::vector<double>& ri, const Bodies& B,
                      std::vector<double>& xi) {
  for (int v = 0; v < N; ++v) {
    if (rid[v] == 0) continue;
    V3 q = rigid_pos(B, rid[v] - 1, ri, v);
    xi[3 * v] = q.x; xi[3 * v + 1] = q.y; xi[3 * v + 2] = q.z;
  }
}

// per-body update after an accumulation (xpbdLayer3D.m:401-414 / 466-479)
void apply_body_increments(Bodies& B, const std::vector<double>& dCOM,
                           const std::vector<double>& dW, double h) {
  for (int b = 0; b < B.n; ++b) {
    for (int d = 0; d < 3; ++d) B.COM[3 * b + d] += dCOM[3 * b + d];
    V3 w = solve3(&B.I[9 * b], v3(dW[3 * b], dW[3 * b + 1], dW[3 * b + 2]));
    double dR[9];
    exp_rodrigues(w, h, dR);
    matmul3(dR, &B.R[9 * b], &B.R[9 * b]);
    double tmp[9];
    matmul3_bt(&B.I0[9 * b], &B.R[9 * b], tmp);  // I0 * R'
    matmul3(&B.R[9 * b], tmp, &B.I[9 * b]);
  }
}

// rigidGeneralizedInverseMass (3d/constraints/rigidGeneralizedInverseMass.m:1-13)
inline double gen_inv_mass(double minvBody, V3 r, const double* I, V3 n) {
  V3 axis = cross(r, n);
  V3 ic = solve3(I, axis);
  return minvBody + dot(axis, ic);
}

struct Solve {
  const Mesh& m;
  const mlx_solve_params& P;
  std::vector<double> xi, lambdai, resv, oldp, minv, contactLambdas;
  std::vector<double> residualArray;
  double runUntil, sumNonMon;
  bool errorChangeDecreased = false;
  int totalIterations = 0;
  // contacts
  int K = 0;
  const double *cn = nullptr, *cp = nullptr, *ccomp = nullptr;
  const int32_t* cv = nullptr;
  // contact_coloring: the colour phase of each vertex's elastic contacts --
  // the first colour none of its tets has, numColors when every colour does
  std::vector<int> ccol;
  Solve(const Mesh& mm, const mlx_solve_params& pp) : m(mm), P(pp) {}

  void contact_colours() {
    if (!ccol.empty()) return;
    const int words = (m.numColors + 64) / 64;
    std::vector<uint64_t> used((size_t)m.N * words, 0);
    for (int e = 0; e < m.T; ++e)
      for (int k = 0; k < 4; ++k) {
        const int c = m.color[e] - 1;
        used[(size_t)m.vid(e, k) * words + c / 64] |= 1ull << (c % 64);
      }
    ccol.assign(m.N, m.numColors);
    for (int v = 0; v < m.N; ++v)
      for (int c = 0; c < m.numColors; ++c)
        if (!((used[(size_t)v * words + c / 64] >> (c % 64)) & 1ull)) {
          ccol[v] = c;
          break;
        }
  }

  void tet_gather(int e, const std::vector<double>& src, double* out) const {
    for (int k = 0; k < 4; ++k)
      for (int d = 0; d < 3; ++d) out[3 * k + d] = src[3 * (size_t)m.vid(e, k) + d];
  }

  // xpbdLayer3D.stvkVoigtConstraints (xpbdLayer3D.m:347-379); the NH branch is
  // the per-colour loop of xpbdLayer2D.neoHookeanConstraints (:260-294).
  void color_sweep(const std::vector<int>& elastic, const int32_t* rid) {
    if (elastic.empty() && !(P.contact_coloring && K > 0)) return;
    double h = P.h, h2 = h * h;
    std::vector<std::vector<int>> byColor(m.numColors);
    for (int e : elastic) byColor[m.color[e] - 1].push_back(e);
    for (int c = 0; c < m.numColors; ++c) {
      const std::vector<int>& es = byColor[c];
      int ne = (int)es.size();
      std::vector<double> newx(12 * (size_t)ne), newl(6 * (size_t)ne);
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
      for (int q = 0; q < ne; ++q) {
        int e = es[q];
        double x[12], xo[12], mi[12], lam[6], dx[12], dl[6] = {0};
        tet_gather(e, xi, x);
        for (int k = 0; k < 6; ++k) lam[k] = lambdai[e + (size_t)m.T * k];
        for (int k = 0; k < 4; ++k)
          for (int d = 0; d < 3; ++d) mi[3 * k + d] = minv[3 * (size_t)m.vid(e, k) + d];
        if (m.energy == MLX_ENERGY_STVK_VOIGT) {
          tet_gather(e, oldp, xo);
          double aT[36], bT[36];
          for (int i = 0; i < 36; ++i) {
            aT[i] = m.alpha[36 * (size_t)e + i] / h2;
            bT[i] = m.beta[36 * (size_t)e + i] * h2;
          }
          stvk_voigt_project(x, xo, &m.DmInv[9 * (size_t)e], aT, lam, mi, m.vol[e], bT, h, dx, dl, nullptr);
          for (int k = 0; k < 6; ++k) lam[k] += dl[k];
        } else {
          nh_project(x, &m.DmInv[9 * (size_t)e], m.mu[e], m.lam[e], m.vol[e], h, lam, mi, dx, dl, nullptr, nullptr);
          lam[0] += dl[0];
          lam[1] += dl[1];
        }
        for (int i = 0; i < 12; ++i) newx[12 * (size_t)q + i] = x[i] + dx[i];
        for (int k = 0; k < 6; ++k) newl[6 * (size_t)q + k] = lam[k];
      }
      // scatter in element order (xpbdLayer3D.m:376-377)
      for (int q = 0; q < ne; ++q) {
        int e = es[q];
        for (int k = 0; k < 6; ++k) lambdai[e + (size_t)m.T * k] = newl[6 * (size_t)q + k];
        for (int k = 0; k < 4; ++k)
          for (int d = 0; d < 3; ++d) xi[3 * (size_t)m.vid(e, k) + d] = newx[12 * (size_t)q + 3 * k + d];
      }
      // contact_coloring: the elastic contacts of this colour's free vertices
      if (P.contact_coloring && K > 0) elastic_contacts(rid, c);
    }
  }

  // xpbdLayer3D.rigidElasticBoundaryAccumulationConstraints (:381-420) with
  // rigidBoundaryConstraint.project (rigidBoundaryConstraint.m:4-35).
  void boundary(const std::vector<int>& bverts, std::vector<double>& lamB, const int32_t* rid,
                Bodies& B, const std::vector<double>& ri) {
    if (bverts.empty() || B.n == 0) return;
    double h = P.h, alpha = P.boundary_compliance;
    std::vector<double> dCOM(3 * B.n, 0), dW(3 * B.n, 0);
    for (size_t i = 0; i < bverts.size(); ++i) {
      int v = bverts[i], b = rid[v] - 1;
      V3 pE = v3(xi[3 * v], xi[3 * v + 1], xi[3 * v + 2]);
      double minvE = 1.0 / m.mass[3 * v + 2];
      V3 pR = rigid_pos(B, b, ri, v);
      V3 com = v3(B.COM[3 * b], B.COM[3 * b + 1], B.COM[3 * b + 2]);
      V3 r = sub(pR, com);
      V3 dir = sub(pR, pE);
      double C = std::sqrt(dot(dir, dir));
      V3 n = v3(dir.x / C, dir.y / C, dir.z / C);
      if (std::isnan(n.x)) n.x = 0;
      if (std::isnan(n.y)) n.y = 0;
      if (std::isnan(n.z)) n.z = 0;
      double invM = 1.0 / B.M[b];
      double w = gen_inv_mass(invM, r, &B.I[9 * b], n);
      double dl = (-C - alpha * lamB[i]) / ((minvE + w) + alpha);
      V3 p = v3(dl * n.x, dl * n.y, dl * n.z);
      lamB[i] += dl;
      dCOM[3 * b] += p.x * invM; dCOM[3 * b + 1] += p.y * invM; dCOM[3 * b + 2] += p.z * invM;
      V3 dw = cross(r, v3(p.x / h, p.y / h, p.z / h));
      dW[3 * b] += dw.x; dW[3 * b + 1] += dw.y; dW[3 * b + 2] += dw.z;
    }
    apply_body_increments(B, dCOM, dW, h);
    for (int v : bverts) {
      V3 q = rigid_pos(B, rid[v] - 1, ri, v);
      xi[3 * v] = q.x; xi[3 * v + 1] = q.y; xi[3 * v + 2] = q.z;
    }
  }

  // The elastic branch of contactConstraints (xpbdLayer3D.m:426-438,
  // penaltyConstraint.projectElastic): gather, project, scatter (last write
  // wins).  colour < 0: every elastic contact; otherwise (contact_coloring)
  // those whose vertex has that contact colour.
  void elastic_contacts(const int32_t* rid, int colour) {
    double h = P.h, h2 = h * h, res = P.contact_resistance;
    if (colour >= 0) contact_colours();  // (colour == numColors: the vertices no phase took)
    auto mine = [&](int k) {
      const int v = cv[k] - 1;
      return rid[v] == 0 && (colour < 0 || ccol[v] == colour);
    };
    std::vector<double> newx;
    std::vector<int> ev;
    std::vector<double> dls;
    for (int k = 0; k < K; ++k) {
      int v = cv[k] - 1;
      if (!mine(k)) continue;
      V3 x = v3(xi[3 * v], xi[3 * v + 1], xi[3 * v + 2]);
      V3 n = v3(cn[k], cn[k + K], cn[k + 2 * K]);
      V3 c = v3(cp[k], cp[k + K], cp[k + 2 * K]);
      double phi = dot(n, sub(x, c));
      if (phi > 0) phi = 0;
      double C = res * phi;
      double aT = ccomp[k] / h2;
      double dl = (-C - aT * contactLambdas[k]) / (2 * minv[3 * v] + aT);
      V3 p = v3(dl * n.x, dl * n.y, dl * n.z);
      ev.push_back(v);
      newx.push_back(x.x + minv[3 * v] * p.x);
      newx.push_back(x.y + minv[3 * v + 1] * p.y);
      newx.push_back(x.z + minv[3 * v + 2] * p.z);
      dls.push_back(dl);
    }
    for (size_t i = 0; i < ev.size(); ++i)
      for (int d = 0; d < 3; ++d) xi[3 * ev[i] + d] = newx[3 * i + d];
    {
      size_t i = 0;
      for (int k = 0; k < K; ++k)
        if (mine(k)) contactLambdas[k] += dls[i++];
    }
  }

  // xpbdLayer3D.contactConstraints (:422-485) with penaltyConstraint
  // projectElastic / projectRigid (penaltyConstraint.m:4-63).
  void contacts(const int32_t* rid, Bodies& B, const std::vector<double>& ri) {
    if (K == 0) return;
    double h = P.h, h2 = h * h, res = P.contact_resistance;
    // elastic contacts (with contact_coloring only those no colour phase took)
    elastic_contacts(rid, P.contact_coloring ? m.numColors : -1);
    if (!P.use_rigid_contacts) return;
    std::vector<int> rk;
    for (int k = 0; k < K; ++k)
      if (rid[cv[k] - 1] != 0) rk.push_back(k);
    if (rk.empty() || B.n == 0) return;
    std::vector<double> dCOM(3 * B.n, 0), dW(3 * B.n, 0);
    for (int k : rk) {
      int v = cv[k] - 1, b = rid[v] - 1;
      V3 x = v3(xi[3 * v], xi[3 * v + 1], xi[3 * v + 2]);
      V3 pR = rigid_pos(B, b, ri, v);
      V3 com = v3(B.COM[3 * b], B.COM[3 * b + 1], B.COM[3 * b + 2]);
      V3 r = sub(pR, com);
      V3 n = v3(cn[k], cn[k + K], cn[k + 2 * K]);
      V3 c = v3(cp[k], cp[k + K], cp[k + 2 * K]);
      double phi = dot(n, sub(x, c));
      if (phi > 0) phi = 0;
      double C = res * phi;
      double invM = 1.0 / B.M[b];
      double w = gen_inv_mass(invM, r, &B.I[9 * b], n);
      double aT = (2 * ccomp[k]) / h2;
      double dl = (-C - aT * contactLambdas[k]) / (2 * w + aT);
      V3 p = v3(dl * n.x, dl * n.y, dl * n.z);
      contactLambdas[k] += dl;
      dCOM[3 * b] += p.x * invM; dCOM[3 * b + 1] += p.y * invM; dCOM[3 * b + 2] += p.z * invM;
      V3 cr = cross(r, p);
      dW[3 * b] += (1 / h) * cr.x; dW[3 * b + 1] += (1 / h) * cr.y; dW[3 * b + 2] += (1 / h) * cr.z;
    }
    apply_body_increments(B, dCOM, dW, h);
    for (int k : rk) {
      int v = cv[k] - 1;
      V3 q = rigid_pos(B, rid[v] - 1, ri, v);
      xi[3 * v] = q.x; xi[3 * v + 1] = q.y; xi[3 * v + 2] = q.z;
    }
  }

  // xpbdLayer3D.simpleEvaluateAllConstraintResiduals (:546-586)
  double residual() {
    double h = P.h, h2 = h * h;
    double acc = 0;
#pragma omp parallel for reduction(+ : acc) schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (int e = 0; e < m.T; ++e) {
      double x[12], xo[12], mi[12], lam[6], dx[12], dl[6], C[6];
      tet_gather(e, xi, x);
      for (int k = 0; k < 6; ++k) lam[k] = lambdai[e + (size_t)m.T * k];
      for (int k = 0; k < 4; ++k)
        for (int d = 0; d < 3; ++d) mi[3 * k + d] = minv[3 * (size_t)m.vid(e, k) + d];
      if (m.energy == MLX_ENERGY_STVK_VOIGT) {
        tet_gather(e, oldp, xo);
        double aT[36], bT[36];
        for (int i = 0; i < 36; ++i) {
          aT[i] = m.alpha[36 * (size_t)e + i] / h2;
          bT[i] = m.beta[36 * (size_t)e + i] * h2;
        }
        stvk_voigt_project(x, xo, &m.DmInv[9 * (size_t)e], aT, lam, mi, m.vol[e], bT, h, dx, dl, C);
        for (int r = 0; r < 6; ++r) {
          double s = 0;
          for (int k = 0; k < 6; ++k) s += aT[r + 6 * k] * lam[k];
          double a = std::fabs(C[r]), cr = std::fabs(s);
          double v = a - std::min(a, cr);
          acc += v * v;
        }
      } else {
        double aT[2];
        nh_project(x, &m.DmInv[9 * (size_t)e], m.mu[e], m.lam[e], m.vol[e], h, lam, mi, dx, dl, C, aT);
        for (int r = 0; r < 2; ++r) {
          double a = std::fabs(C[r]), cr = std::fabs(aT[r] * lam[r]);
          double v = a - std::min(a, cr);
          acc += v * v;
        }
      }
    }
    // contacts: (contactCompliance/h2) is 1x1xK and contactLambdas(:) is Kx1,
    // so implicit expansion makes the correction term K x 1 x K
    // (xpbdLayer3D.m:581-583): every |C_k| is compared with every
    // |compliance_j / h^2 * lambda_k|, K^2 terms in all
    std::vector<double> absC(K);
    for (int k = 0; k < K; ++k) {
      int v = cv[k] - 1;
      V3 x = v3(xi[3 * v], xi[3 * v + 1], xi[3 * v + 2]);
      V3 n = v3(cn[k], cn[k + K], cn[k + 2 * K]);
      V3 c = v3(cp[k], cp[k + K], cp[k + 2 * K]);
      double phi = dot(n, sub(x, c));
      if (phi > 0) phi = 0;
      absC[k] = std::fabs(P.contact_resistance * phi);
    }
    for (int j = 0; j < K; ++j)
      for (int k = 0; k < K; ++k) {
        double cr = std::fabs((ccomp[j] / h2) * contactLambdas[k]);
        double vv = absC[k] - std::min(absC[k], cr);
        acc += vv * vv;
      }
    return std::sqrt(acc);
  }
};

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_stvk_constraint_grad(const double* DmInv, const double* x, double* gradC, double* C) {
  stvk_grad(DmInv, x, gradC, C);
}

void orc_stvk_voigt_project(const double* x, const double* xprev, const double* DmInv,
                            const double* alphaTilde, const double* lambda, const double* minv,
                            double vol, const double* betaTilde, double h, double* dx,
                            double* dlambda, double* C) {
  stvk_voigt_project(x, xprev, DmInv, alphaTilde, lambda, minv, vol, betaTilde, h, dx, dlambda, C);
}

void orc_nh_project(const double* x, const double* DmInv, double mu, double lam, double vol,
                    double h, const double* lambda, const double* minv, double* dx,
                    double* dlambda, double* C, double* alphaTilde) {
  nh_project(x, DmInv, mu, lam, vol, h, lambda, minv, dx, dlambda, C, alphaTilde);
}

void orc_exp_rodrigues(const double* omega, double h, double* R) {
  exp_rodrigues(v3(omega[0], omega[1], omega[2]), h, R);
}

// naiveGraphColoring (2d/tools/functionalities/naiveGraphColoring.m:1-19)
int orc_greedy_coloring(const int32_t* t, int32_t T, int32_t N, int32_t* color) {
  std::vector<std::vector<int>> used(N);
  int maxc = 0;
  for (int e = 0; e < T; ++e) {
    int c = 1;
    for (;;) {
      bool clash = false;
      for (int k = 0; k < 4 && !clash; ++k) {
        const std::vector<int>& u = used[t[e + (size_t)T * k] - 1];
        clash = std::find(u.begin(), u.end(), c) != u.end();
      }
      if (!clash) break;
      ++c;
    }
    for (int k = 0; k < 4; ++k) used[t[e + (size_t)T * k] - 1].push_back(c);
    color[e] = c;
    maxc = std::max(maxc, c);
  }
  return maxc;
}

// computeB3D (3d/tools/functionalities/computeB3D.m:23-24) and the signed
// volume of makeElements3D.m:11 (gptoolbox volume = det(Dm)/6).
void orc_rest_state(const double* p, const int32_t* t, int32_t T, double* DmInv, double* vol) {
  for (int e = 0; e < T; ++e) {
    int id[4];
    for (int k = 0; k < 4; ++k) id[k] = t[e + (size_t)T * k] - 1;
    double Dm[9];
    for (int k = 0; k < 3; ++k)
      for (int d = 0; d < 3; ++d) Dm[d + 3 * k] = p[3 * id[k + 1] + d] - p[3 * id[0] + d];
    for (int c = 0; c < 3; ++c) {
      double ec[3] = {0, 0, 0}, col[3];
      ec[c] = 1;
      mldivide(3, Dm, ec, col);
      for (int r = 0; r < 3; ++r) DmInv[9 * (size_t)e + r + 3 * c] = col[r];
    }
    V3 a = v3(Dm[0], Dm[1], Dm[2]), b = v3(Dm[3], Dm[4], Dm[5]), c = v3(Dm[6], Dm[7], Dm[8]);
    vol[e] = dot(a, cross(b, c)) / 6.0;
  }
}

// Mesh3D.updateMaterials (Mesh3D.m:445-460)
void orc_update_materials(const double* mu, const double* lam, const double* a1, int32_t T,
                          double* alpha, double* alphaInv, double* beta) {
  for (int e = 0; e < T; ++e)
    material_blocks(mu[e], lam[e], a1 ? a1[e] : 0.0, alpha ? alpha + 36 * (size_t)e : nullptr,
                    alphaInv ? alphaInv + 36 * (size_t)e : nullptr,
                    beta ? beta + 36 * (size_t)e : nullptr);
}

// computeMass, density branch (3d/@Mesh3D/computeMass.m:20-37)
void orc_compute_mass(const int32_t* t, int32_t T, int32_t N, const double* vol,
                      const double* rho, double* mass) {
  for (int i = 0; i < 3 * N; ++i) mass[i] = 0;
  for (int e = 0; e < T; ++e)
    for (int k = 0; k < 4; ++k) {
      int v = t[e + (size_t)T * k] - 1;
      for (int d = 0; d < 3; ++d) mass[3 * v + d] += (vol[e] * rho[e]) / 4;
    }
}

// F = B*p in the B layout of computeB3D.m:26-41 (per tet 9 entries,
// entry 3*(d-1)+(j-1) = F(d,j)), then the formula of mexEdiffNorm3D.cpp:35-61.
void orc_strain_rate_norms(const int32_t* t, int32_t T, const double* DmInv, const double* p,
                           const double* oldp, double h, double* norms) {
  for (int e = 0; e < T; ++e) {
    int id[4];
    for (int k = 0; k < 4; ++k) id[k] = t[e + (size_t)T * k] - 1;
    const double* G = DmInv + 9 * (size_t)e;
    double D[4][3];  // D = [-sum(DmInv,1); DmInv]
    for (int j = 0; j < 3; ++j) {
      D[0][j] = -(G[0 + 3 * j] + G[1 + 3 * j] + G[2 + 3 * j]);
      for (int k = 1; k <= 3; ++k) D[k][j] = G[(k - 1) + 3 * j];
    }
    double Fa[9], Fb[9];
    for (int d = 0; d < 3; ++d)
      for (int j = 0; j < 3; ++j) {
        double sa = 0, sb = 0;
        for (int k = 0; k < 4; ++k) {
          sa += D[k][j] * p[3 * id[k] + d];
          sb += D[k][j] * oldp[3 * id[k] + d];
        }
        Fa[3 * d + j] = sa;
        Fb[3 * d + j] = sb;
      }
    // columns as the mex reads them: col c = entries 3c..3c+2
    auto e2 = [&](const double* F, int a, int b) {
      return (F[3 * a] * F[3 * b]) / 2.0 + (F[3 * a + 1] * F[3 * b + 1]) / 2.0 + (F[3 * a + 2] * F[3 * b + 2]) / 2.0;
    };
    double t2 = 1.0 / (h * h);
    double s = 0;
    const int pa[6] = {0, 0, 1, 0, 1, 2}, pb[6] = {1, 2, 2, 0, 1, 2};
    for (int q = 0; q < 6; ++q) {
      double dd = e2(Fa, pa[q], pb[q]) - e2(Fb, pa[q], pb[q]);
      s += t2 * dd * dd * (q < 3 ? 2.0 : 1.0);
    }
    norms[e] = s;
  }
}

// mexUnionFindByVertice (2d/mex/mexUnionFindByVertice.cpp:11-178),
// restated: union by size over shared vertices, IDs numbered in element order.
int orc_union_find_layers(const int32_t* order, int32_t T, const double* layers, int32_t L,
                          const uint8_t* forced, const int32_t* t, int32_t N,
                          int32_t* sets, int32_t* numRigids) {
  std::vector<int> id(T, -1), sz(T, 1), claimed(N, -1);
  int count = 0;
  auto find = [&](int p) -> int {
    if (p == -1 || id[p] == -1) return -1;
    int root = p;
    while (root != id[root]) root = id[root];
    while (p != root) { int np = id[p]; id[p] = root; p = np; }
    return root;
  };
  auto merge = [&](int x, int y) {
    int i = find(x), j = find(y);
    if (i == j || i == -1 || j == -1) return;
    if (sz[i] < sz[j]) { id[i] = j; sz[j] += sz[i]; } else { id[j] = i; sz[i] += sz[j]; }
    --count;
  };
  auto copy_layer = [&](int col) {
    std::unordered_map<int, int> map;
    int counter = 1;
    numRigids[col] = count;
    for (int e = 0; e < T; ++e) {
      if (id[e] == -1) { sets[e + (size_t)T * col] = 0; continue; }
      int r = find(e);
      auto it = map.find(r);
      if (it != map.end()) sets[e + (size_t)T * col] = it->second;
      else { map.emplace(r, counter); sets[e + (size_t)T * col] = counter++; }
    }
  };
  copy_layer(0);
  int start = 0;
  for (int l = 0; l < L; ++l) {
    int end = (int)std::floor((layers[l] / 100.0) * T);
    for (int q = start; q < end; ++q) {
      int e = order[q] - 1;
      if (forced[e]) continue;
      id[e] = e;
      ++count;
      for (int k = 0; k < 4; ++k) {
        int v = t[e + (size_t)T * k] - 1;
        merge(e, claimed[v]);
        claimed[v] = e;
      }
    }
    copy_layer(l);
    start = end;
  }
  return 0;
}

// xpbdLayer2D.findBoundaryVertices (2d/integrator/xpbdLayer2D.m:551-569)
void orc_find_boundary_vertices(const int32_t* t, int32_t T, int32_t N, const int32_t* sets,
                                int32_t L, uint8_t* isBoundary, uint8_t* isElastic,
                                uint8_t* isRigidVertex, int32_t* vertexRigidBody) {
  std::vector<uint8_t> ofElastic((size_t)N * L, 0);
  for (size_t i = 0; i < (size_t)N * L; ++i) { isRigidVertex[i] = 0; vertexRigidBody[i] = 0; }
  for (size_t i = 0; i < (size_t)T * L; ++i) isElastic[i] = sets[i] == 0;
  for (int l = 0; l < L; ++l)
    for (int k = 0; k < 4; ++k)
      for (int e = 0; e < T; ++e) {
        int v = t[e + (size_t)T * k] - 1;
        size_t vi = v + (size_t)N * l;
        int s = sets[e + (size_t)T * l];
        if (s != 0) { isRigidVertex[vi] = 1; vertexRigidBody[vi] = s; }
        else ofElastic[vi] = 1;
      }
  for (size_t i = 0; i < (size_t)N * L; ++i) isBoundary[i] = ofElastic[i] && isRigidVertex[i];
}

// xpbdLayer3D.layerSolve (xpbdLayer3D.m:44-232) with projectGS (:243-345) and
// simpleMonitorError (:515-544).
int orc_layer_solve(const mlx_mesh_desc* md, const mlx_layer_desc* ld, const mlx_solve_params* P,
                    const mlx_contacts* cts, const mlx_solve_inputs* in, mlx_solve_outputs* out) {
  if (!md || !ld || !P || !in || !out) return fail(MLX_ERR_ARGUMENT, "null argument");
  Mesh m;
  m.N = md->num_vertices; m.T = md->num_tets; m.numColors = md->num_colors;
  m.t = md->t; m.mass = md->mass; m.DmInv = md->DmInv; m.vol = md->volume;
  m.color = md->element_color; m.pinned = md->pinned_dofs; m.numPinned = md->num_pinned_dofs;
  m.energy = md->energy_type;
  if (m.energy == MLX_ENERGY_STVK_VOIGT) {
    if (md->alpha && md->beta) {
      m.alpha.assign(md->alpha, md->alpha + 36 * (size_t)m.T);
      m.beta.assign(md->beta, md->beta + 36 * (size_t)m.T);
    } else if (md->mu && md->lambda) {
      m.alpha.resize(36 * (size_t)m.T); m.beta.resize(36 * (size_t)m.T);
      orc_update_materials(md->mu, md->lambda, md->alpha1, m.T, m.alpha.data(), nullptr, m.beta.data());
    } else return fail(MLX_ERR_ARGUMENT, "StVK mesh needs alpha/beta or mu/lambda");
  } else if (m.energy == MLX_ENERGY_NEOHOOKEAN) {
    if (!md->mu || !md->lambda) return fail(MLX_ERR_ARGUMENT, "Neo-Hookean mesh needs mu/lambda");
    m.mu.assign(md->mu, md->mu + m.T);
    m.lam.assign(md->lambda, md->lambda + m.T);
  } else return fail(MLX_ERR_ARGUMENT, "unknown energy type");
  if (P->run_until >= 0 && !P->compute_residuals)
    return fail(MLX_ERR_ARGUMENT, "run_until >= 0 needs compute_residuals (the reference loops forever)");

  const int N = m.N, T = m.T;
  Solve S(m, *P);
  S.xi.assign(in->xi, in->xi + 3 * (size_t)N);
  S.lambdai.assign(in->lambdai, in->lambdai + 6 * (size_t)T);
  S.resv.assign(in->residualv, in->residualv + 3 * (size_t)N);
  S.oldp.assign(in->oldp, in->oldp + 3 * (size_t)N);
  S.minv.resize(3 * (size_t)N);
  for (int i = 0; i < 3 * N; ++i) S.minv[i] = 1.0 / m.mass[i];
  S.residualArray.assign(in->residual_in, in->residual_in + in->residual_in_len);
  S.runUntil = P->run_until;
  S.sumNonMon = in->sum_non_monitored_time;
  if (cts && cts->num_contacts > 0) {
    S.K = cts->num_contacts; S.cn = cts->normals; S.cp = cts->point_colliders;
    S.cv = cts->vertex_ids; S.ccomp = cts->compliance;
  }
  S.contactLambdas.assign(S.K, 0.0);
  const double h = P->h;
  const long long kSafetyIterations = 100000000LL;

  for (int layer = 0; layer < ld->num_layers; ++layer) {
    double setPercentStop = layer == 0 ? P->stop_at_improvement_percent : 0;
    std::vector<double> xprev = S.xi;
    bool isLast = layer == ld->num_layers - 1;
    int col = ld->layers_map[layer] - 1;
    const uint8_t* isE = ld->is_elastic_element + (size_t)T * col;
    const uint8_t* isR = ld->is_rigid_element + (size_t)T * col;
    const int32_t* rid = ld->vertex_rigid_body + (size_t)N * col;
    const uint8_t* isBV = ld->is_boundary_vertex + (size_t)N * col;
    const uint8_t* isRV = ld->is_rigid_vertex + (size_t)N * col;
    int nb = ld->num_rigids[col];
    std::vector<int> elastic;
    int nRigidElements = 0;
    for (int e = 0; e < T; ++e) { if (isE[e]) elastic.push_back(e); if (isR[e]) ++nRigidElements; }

    Bodies B;
    std::vector<double> ri;
    make_rigids(nb, rid, N, S.xi, S.resv, m.mass, B, ri);
    // release all elastic residual (xpbdLayer3D.m:138-139)
    for (int v = 0; v < N; ++v)
      if (!isRV[v])
        for (int d = 0; d < 3; ++d) { S.xi[3 * v + d] += h * S.resv[3 * v + d]; S.resv[3 * v + d] = 0; }
    std::vector<double> steppedR = B.R;
    bool rigidLayer = nRigidElements > 0;
    if (rigidLayer) {
      // RigidBody3D.rigidSymplecticImperativeStep (RigidBody3D.m:174-179)
      for (int b = 0; b < nb; ++b) {
        for (int d = 0; d < 3; ++d) B.COM[3 * b + d] += h * B.COMDOT[3 * b + d];
        double dR[9];
        exp_rodrigues(v3(B.omega[3 * b], B.omega[3 * b + 1], B.omega[3 * b + 2]), h, dR);
        matmul3(dR, &B.R[9 * b], &B.R[9 * b]);
        double tmp[9];
        matmul3(&B.R[9 * b], &B.I0[9 * b], tmp);
        matmul3_bt(tmp, &B.R[9 * b], &B.I[9 * b]);
      }
      steppedR = B.R;
      rotate_all_verts(rid, N, ri, B, S.xi);
      for (int v = 0; v < N; ++v) {
        if (rid[v] <= 0) continue;
        const double* Rb = &B.R[9 * (rid[v] - 1)];
        V3 rot = matvec(Rb, v3(S.resv[3 * v], S.resv[3 * v + 1], S.resv[3 * v + 2]));
        double rr[3] = {rot.x, rot.y, rot.z};
        for (int d = 0; d < 3; ++d) {
          double rigidResv = (S.xi[3 * v + d] - xprev[3 * v + d]) / h;  // BDF.BDF1
          S.resv[3 * v + d] = rr[d] - rigidResv;
        }
      }
    }
    double normresv = 0;
    for (double r : S.resv) normresv += r * r;
    normresv = std::sqrt(normresv);

    // ---- projectGS ----
    // projectGS does not return contactLambdas (xpbdLayer3D.m:163): every
    // layer starts from the zeros layerSolve created (xpbdLayer3D.m:99-102)
    std::fill(S.contactLambdas.begin(), S.contactLambdas.end(), 0.0);
    std::vector<int> bverts;
    for (int v = 0; v < N; ++v) if (isBV[v]) bverts.push_back(v);
    std::vector<double> lamB(bverts.size(), 0.0);
    bool stopSolve = false;
    long long it = 1;
    while (it <= ld->iterations[layer] || (!stopSolve && S.runUntil >= 0 && isLast)) {
      ++it;
      if (it > kSafetyIterations) return fail(MLX_ERR_LIMIT, "iteration safety limit reached");
      ++S.totalIterations;
      S.color_sweep(elastic, rid);
      S.boundary(bverts, lamB, rid, B, ri);
      S.contacts(rid, B, ri);
      for (int q = 0; q < m.numPinned; ++q) S.xi[m.pinned[q] - 1] = in->pinnedx[q];
      bool endLayer = false;
      if (P->compute_residuals) {
        double newRes = S.residual();
        S.residualArray.push_back(newRes);
        double lastResidual = std::fabs(S.residualArray[S.residualArray.size() - 2]);
        double newResidual = std::fabs(newRes);
        double errorChange = newResidual - lastResidual;
        if (setPercentStop > 0) {
          S.runUntil = std::max((1 - setPercentStop / 100.0) * newResidual, 1e-8);
          setPercentStop = 0;
        }
        if (errorChange < 0) S.errorChangeDecreased = true;
        if (P->give_up_enabled && errorChange > P->give_up_threshold && S.errorChangeDecreased &&
            (!isLast || P->last_layer_give_up_enabled))
          endLayer = true;
        bool stopHanging = (long long)S.residualArray.size() > P->hanging_stop && P->hanging_stop >= 0;
        if (stopHanging || (S.runUntil >= 0 && (S.runUntil >= newResidual && (isLast || normresv < S.runUntil))))
          stopSolve = true;
      }
      if (endLayer || stopSolve) break;
    }
    rotate_all_verts(rid, N, ri, B, S.xi);
    // ---- end projectGS ----
    if (rigidLayer) {
      for (int v = 0; v < N; ++v) {
        if (rid[v] == 0) continue;
        int b = rid[v] - 1;
        double dR[9];
        matmul3_bt(&B.R[9 * b], &steppedR[9 * b], dR);
        V3 r = matvec(dR, v3(S.resv[3 * v], S.resv[3 * v + 1], S.resv[3 * v + 2]));
        S.resv[3 * v] = r.x; S.resv[3 * v + 1] = r.y; S.resv[3 * v + 2] = r.z;
      }
    }
    if (stopSolve) break;
  }
  std::memcpy(out->xi, S.xi.data(), sizeof(double) * 3 * (size_t)N);
  if (out->lambdai) std::memcpy(out->lambdai, S.lambdai.data(), sizeof(double) * 6 * (size_t)T);
  int n = (int)S.residualArray.size();
  if (out->residual) {
    if (n > out->residual_capacity) return fail(MLX_ERR_ARGUMENT, "residual capacity too small");
    std::memcpy(out->residual, S.residualArray.data(), sizeof(double) * n);
  }
  out->residual_len = n;
  out->run_until = S.runUntil;
  out->sum_non_monitored_time = S.sumNonMon;
  out->total_iterations = S.totalIterations;
  return MLX_OK;
}

// xpbdLayer2D.contactVelocityUpdate (2d/integrator/xpbdLayer2D.m:577-603),
// dim = 3.  Duplicate vertices: last write wins, as MATLAB's v(dofs) = ...
void orc_contact_velocity_update(const double* normals, const int32_t* vids, int32_t K,
                                 double* v, double h, double gravity, double e) {
  std::vector<double> nv(3 * (size_t)K);
  for (int k = 0; k < K; ++k) {
    int i = vids[k] - 1;
    V3 vn = v3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    V3 n = v3(normals[k], normals[k + K], normals[k + 2 * K]);
    double ek = e;
    if (std::sqrt(dot(vn, vn)) <= 2 * gravity * h) ek = 0;
    double vt = dot(n, vn);
    double mn = std::min(-ek * vt, 0.0);
    nv[3 * k] = vn.x + n.x * (-vn.x + mn);
    nv[3 * k + 1] = vn.y + n.y * (-vn.y + mn);
    nv[3 * k + 2] = vn.z + n.z * (-vn.z + mn);
  }
  for (int k = 0; k < K; ++k) {
    int i = vids[k] - 1;
    for (int d = 0; d < 3; ++d) v[3 * i + d] = nv[3 * k + d];
  }
}

// PlaneContactFinder3D.findContacts (3d/contact/PlaneContactFinder3D.m:34-75):
// returns the number of contacts; outputs (vertex ids 1-based, normal K x 3,
// point collider K x 3, in vertex order) sized for N.
int orc_find_contacts_plane(const double* p, int32_t N, const double* normal_raw,
                            const double* position, double compliance, int32_t* vids,
                            double* normals, double* points, double* comp) {
  double nn = std::sqrt(dot(v3(normal_raw[0], normal_raw[1], normal_raw[2]),
                            v3(normal_raw[0], normal_raw[1], normal_raw[2])));
  V3 n = v3(normal_raw[0] / nn, normal_raw[1] / nn, normal_raw[2] / nn);
  double D = normal_raw[0] * position[0] + normal_raw[1] * position[1] + normal_raw[2] * position[2];
  std::vector<int> idx;
  std::vector<double> phis;
  for (int i = 0; i < N; ++i) {
    double dist = (p[3 * i] * n.x + p[3 * i + 1] * n.y + p[3 * i + 2] * n.z) - D;
    if (dist <= 0) { idx.push_back(i); phis.push_back(dist); }
  }
  int K = (int)idx.size();
  for (int k = 0; k < K; ++k) {
    int i = idx[k];
    vids[k] = i + 1;
    normals[k] = n.x; normals[k + K] = n.y; normals[k + 2 * K] = n.z;
    points[k] = p[3 * i] - n.x * phis[k];
    points[k + K] = p[3 * i + 1] - n.y * phis[k];
    points[k + 2 * K] = p[3 * i + 2] - n.z * phis[k];
    comp[k] = compliance;
  }
  return K;
}

// SphereContactFinder.findContacts (3d/contact/SphereContactFinder.m:24-71);
// contactInfo3D keeps its default compliance 1e-4 for this finder.
int orc_find_contacts_sphere(const double* p, int32_t N, double radius, const double* center,
                             int32_t* vids, double* normals, double* points, double* comp) {
  std::vector<int> idx;
  std::vector<double> dist;
  for (int i = 0; i < N; ++i) {
    double dx = center[0] - p[3 * i], dy = center[1] - p[3 * i + 1], dz = center[2] - p[3 * i + 2];
    double d = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (d <= radius) { idx.push_back(i); dist.push_back(d); }
  }
  int K = (int)idx.size();
  for (int k = 0; k < K; ++k) {
    int i = idx[k];
    double phi = dist[k] - radius;
    V3 n = v3((p[3 * i] - center[0]) / dist[k], (p[3 * i + 1] - center[1]) / dist[k],
              (p[3 * i + 2] - center[2]) / dist[k]);
    vids[k] = i + 1;
    normals[k] = n.x; normals[k + K] = n.y; normals[k + 2 * K] = n.z;
    points[k] = p[3 * i] - n.x * phi;
    points[k + K] = p[3 * i + 1] - n.y * phi;
    points[k + 2 * K] = p[3 * i + 2] - n.z * phi;
    comp[k] = 1e-4;
  }
  return K;
}

// PlatformContactDetector.findContacts (3d/contact/PlatformContactDetector.m:65-119)
// for a box with rotation R (row-major, RotationMatrixDegrees), full extents
// scale = [width depth height] and centre: contacts of the vertices inside
// the box, pushed out through the nearest face (first axis on ties),
// normal = sign(dot) * direction of that axis, phi = -(half - |dot|).
int orc_find_contacts_platform(const double* p, int32_t N, const double* R, const double* scale,
                               const double* center, double compliance, int32_t* vids, double* normals,
                               double* points, double* comp) {
  double dir[9], half[3];
  for (int r = 0; r < 3; ++r) {
    const double* row = R + 3 * r;
    double nr = std::sqrt(row[0] * row[0] + row[1] * row[1] + row[2] * row[2]);
    for (int d = 0; d < 3; ++d) dir[3 * r + d] = row[d] / nr;
    half[r] = scale[r] / 2;
  }
  std::vector<int> idx;
  std::vector<V3> nrm;
  std::vector<double> phis;
  for (int i = 0; i < N; ++i) {
    double e[3] = {p[3 * i] - center[0], p[3 * i + 1] - center[1], p[3 * i + 2] - center[2]};
    double dots[3], ad[3];
    bool inside = true;
    for (int a = 0; a < 3; ++a) {
      dots[a] = e[0] * dir[3 * a] + e[1] * dir[3 * a + 1] + e[2] * dir[3 * a + 2];
      inside = inside && std::fabs(dots[a]) <= half[a];
      ad[a] = half[a] - std::fabs(dots[a]);
    }
    if (!inside) continue;
    int k = 0;
    if (ad[1] < ad[k]) k = 1;
    if (ad[2] < ad[k]) k = 2;
    double sgn = dots[k] > 0 ? 1.0 : (dots[k] < 0 ? -1.0 : 0.0);
    idx.push_back(i);
    nrm.push_back(v3(sgn * dir[3 * k], sgn * dir[3 * k + 1], sgn * dir[3 * k + 2]));
    phis.push_back(-ad[k]);
  }
  int K = (int)idx.size();
  for (int k = 0; k < K; ++k) {
    int i = idx[k];
    V3 n = nrm[k];
    vids[k] = i + 1;
    normals[k] = n.x; normals[k + K] = n.y; normals[k + 2 * K] = n.z;
    points[k] = p[3 * i] - n.x * phis[k];
    points[k + K] = p[3 * i + 1] - n.y * phis[k];
    points[k + 2 * K] = p[3 * i + 2] - n.z * phis[k];
    comp[k] = compliance;
  }
  return K;
}

}  // extern "C"
