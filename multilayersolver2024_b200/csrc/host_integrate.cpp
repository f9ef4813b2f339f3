// host_integrate.cpp -- the per-step vector arithmetic of
// xpbdLayer3D.integrate around layerSolve (xpbdLayer3D.m:621-745) on the host:
// the NaN check of the step-start positions, forces and residual velocity
// before the solve, the velocity update after it.  Each is one fused pass
// over the DOFs with the reference's operation order (the same doubles as
// its element-wise expressions); meshes of more than 2^16 DOFs are split
// over the host threads.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/mlxpbd.h"
#include "solver.h"

using mlx::set_error;

namespace {

constexpr long long kGrain = 1 << 16;  // DOFs per thread at least

// fn(begin, end) over [0, n), on up to hardware_concurrency() threads.
template <typename F>
void parallel_ranges(long long n, F fn) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const long long nt = std::min<long long>(hw, (n + kGrain - 1) / kGrain);
  if (nt <= 1) {
    if (n > 0) fn(0LL, n);
    return;
  }
  const long long chunk = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  th.reserve((size_t)nt - 1);
  for (long long t = 1; t < nt; ++t) {
    const long long a = t * chunk, b = std::min(n, a + chunk);
    if (a < b) th.emplace_back(fn, a, b);
  }
  fn(0LL, std::min(n, chunk));
  for (std::thread& x : th) x.join();
}

}  // namespace

extern "C" {

int32_t mlx_any_nan(int64_t n, const double* x) {
  if (n <= 0) return 0;
  if (!x) return -set_error(MLX_ERR_ARGUMENT, "x is NULL");  // negative: 1 means found
  std::atomic<int> found{0};
  parallel_ranges(n, [&](long long a, long long b) {
    for (long long i = a; i < b; i += 4096) {
      if (found.load(std::memory_order_relaxed)) return;
      const long long e = std::min(b, i + 4096);
      bool nan = false;
      for (long long j = i; j < e; ++j) nan |= std::isnan(x[j]);
      if (nan) {
        found.store(1, std::memory_order_relaxed);
        return;
      }
    }
  });
  return found.load();
}

// f(3:3:end) = f(3:3:end) + mass(3:3:end) * Gravity on a reset force, then
// f = f + CustomForce (xpbdLayer3D.m:638-643); residualVelocity = v, plus
// h * f ./ mass on the unpinned DOFs, times (1 - airDrag) (:662-664).
int mlx_integrate_begin(int32_t num_dofs, double h, double gravity, double air_drag, double custom_force,
                        const double* custom_force_vec, const double* mass, const double* v,
                        const int32_t* pinned_dofs, int32_t num_pinned, double* f, double* residualv) {
  if (num_dofs < 0 || num_pinned < 0) return set_error(MLX_ERR_ARGUMENT, "negative size");
  if (num_dofs % 3) return set_error(MLX_ERR_ARGUMENT, "num_dofs is not a multiple of 3");
  if (num_dofs == 0) return MLX_OK;
  if (!mass || !v || !f || !residualv) return set_error(MLX_ERR_ARGUMENT, "mass, v, f and residualv are required");
  if (num_pinned > 0 && !pinned_dofs) return set_error(MLX_ERR_ARGUMENT, "pinned_dofs is NULL");
  for (int32_t i = 0; i < num_pinned; ++i)
    if (pinned_dofs[i] < 1 || pinned_dofs[i] > num_dofs) return set_error(MLX_ERR_ARGUMENT, "pinned DOF out of range");
  const double keep = 1.0 - air_drag;
  parallel_ranges(num_dofs, [&](long long a, long long b) {
    for (long long i = a; i < b; ++i) {
      const double g = (i % 3 == 2) ? 0.0 + mass[i] * gravity : 0.0;
      const double fi = g + (custom_force_vec ? custom_force_vec[i] : custom_force);
      f[i] = fi;
      residualv[i] = keep * (v[i] + h * fi / mass[i]);
    }
  });
  // pinned DOFs: the velocity alone (the reference adds h f / m on the
  // unpinned ones only)
  for (int32_t i = 0; i < num_pinned; ++i) {
    const int32_t d = pinned_dofs[i] - 1;
    residualv[d] = keep * v[d];
  }
  return MLX_OK;
}

// mesh3D.v = (xi - cache.oldp) ./ h (xpbdLayer3D.m:737).
int mlx_integrate_end(int32_t num_dofs, double h, const double* xi, const double* oldp, double* v) {
  if (num_dofs < 0) return set_error(MLX_ERR_ARGUMENT, "negative size");
  if (num_dofs == 0) return MLX_OK;
  if (!xi || !oldp || !v) return set_error(MLX_ERR_ARGUMENT, "xi, oldp and v are required");
  parallel_ranges(num_dofs, [&](long long a, long long b) {
    for (long long i = a; i < b; ++i) v[i] = (xi[i] - oldp[i]) / h;
  });
  return MLX_OK;
}

}  // extern "C"
