// host_integrate.cpp -- the per-step vector arithmetic of
// xpbdLayer3D.integrate around layerSolve (xpbdLayer3D.m:621-745) on the host:
// the NaN check of the step-start positions, forces and residual velocity
// before the solve, the velocity update and contactVelocityUpdate after it.  Each is one fused pass
// over the DOFs with the reference's operation order (the same doubles as
// its element-wise expressions); meshes of more than 2^16 DOFs are split
// over the host threads.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/mlxpbd.h"
#include "solver.h"

using mlx::set_error;

namespace {

constexpr long long kGrain = 1 << 16;  // DOFs per thread at least

// fn(begin, end) over [0, n), on up to hardware_concurrency() threads of at
// least `grain` items each.
template <typename F>
void parallel_ranges(long long n, F fn, long long grain = kGrain) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const long long nt = std::min<long long>(hw, (n + grain - 1) / grain);
  if (nt <= 1) {
    if (n > 0) fn(0LL, n);
    return;
  }
  const long long chunk = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  th.reserve((size_t)nt - 1);
  for (long long t = 1; t < nt; ++t) {
    const long long a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) continue;
    try {
      th.emplace_back(fn, a, b);
    } catch (const std::system_error&) {
      fn(a, b);  // no thread to be had: this one runs the range
    }
  }
  fn(0LL, std::min(n, chunk));
  for (std::thread& x : th) x.join();
}

// The element-wise loops, written so the compiler vectorises them (the
// library's host code is built at -O2, which does not).  IEEE operations in
// the same order either way: the results are the same doubles.
#pragma GCC push_options
#pragma GCC optimize("O3")

int nan_in(long long a, long long b, const double* __restrict__ x) {
  int nan = 0;
  for (long long j = a; j < b; ++j) nan |= x[j] != x[j];
  return nan;
}

// f of vertices [a, b): 0 + custom force on x and y, (0 + m g) + custom force on z
void forces(long long a, long long b, double gravity, double cf, const double* __restrict__ cfv,
            const double* __restrict__ mass, double* __restrict__ f) {
  if (cfv) {
    for (long long k = a; k < b; ++k) {
      f[3 * k] = 0.0 + cfv[3 * k];
      f[3 * k + 1] = 0.0 + cfv[3 * k + 1];
      f[3 * k + 2] = (0.0 + mass[3 * k + 2] * gravity) + cfv[3 * k + 2];
    }
  } else {
    for (long long k = a; k < b; ++k) {
      f[3 * k] = 0.0 + cf;
      f[3 * k + 1] = 0.0 + cf;
      f[3 * k + 2] = (0.0 + mass[3 * k + 2] * gravity) + cf;
    }
  }
}

// residual velocity of DOFs [a, b): (1 - airDrag) (v + h f / m)
void residual_velocity(long long a, long long b, double h, double keep, const double* __restrict__ mass,
                       const double* __restrict__ v, const double* __restrict__ f, double* __restrict__ rv) {
  for (long long i = a; i < b; ++i) rv[i] = keep * (v[i] + h * f[i] / mass[i]);
}

void velocity(long long a, long long b, double h, const double* __restrict__ xi, const double* __restrict__ oldp,
              double* __restrict__ v) {
  for (long long i = a; i < b; ++i) v[i] = (xi[i] - oldp[i]) / h;
}

#pragma GCC pop_options

// any(isnan(x)) over n > 0 values: 1 or 0.
int any_nan_impl(long long n, const double* x) {
  std::atomic<int> found{0};
  parallel_ranges(n, [&](long long a, long long b) {
    for (long long i = a; i < b; i += 4096) {
      if (found.load(std::memory_order_relaxed)) return;
      if (nan_in(i, std::min(b, i + 4096), x)) {
        found.store(1, std::memory_order_relaxed);
        return;
      }
    }
  });
  return found.load();
}

}  // namespace

extern "C" {

int32_t mlx_any_nan(int64_t n, const double* x) {
  if (n <= 0) return 0;
  if (!x) return -set_error(MLX_ERR_ARGUMENT, "x is NULL");  // negative: 1 means found
  try {
    return any_nan_impl(n, x);
  } catch (...) {
    return -set_error(MLX_ERR_ALLOC, "host resource exhausted");
  }
}

// f(3:3:end) = f(3:3:end) + mass(3:3:end) * Gravity on a reset force, then
// f = f + CustomForce (xpbdLayer3D.m:638-643); residualVelocity = v, plus
// h * f ./ mass on the unpinned DOFs, times (1 - airDrag) (:662-664).
int mlx_integrate_begin(int32_t num_dofs, double h, double gravity, double air_drag, double custom_force,
                        const double* custom_force_vec, const double* mass, const double* v,
                        const int32_t* pinned_dofs, int32_t num_pinned, double* f, double* residualv) {
  return mlx::guarded([&]() -> int {
    if (num_dofs < 0 || num_pinned < 0) return set_error(MLX_ERR_ARGUMENT, "negative size");
    if (num_dofs % 3) return set_error(MLX_ERR_ARGUMENT, "num_dofs is not a multiple of 3");
    if (num_dofs == 0) return MLX_OK;
    if (!mass || !v || !f || !residualv) return set_error(MLX_ERR_ARGUMENT, "mass, v, f and residualv are required");
    if (num_pinned > 0 && !pinned_dofs) return set_error(MLX_ERR_ARGUMENT, "pinned_dofs is NULL");
    for (int32_t i = 0; i < num_pinned; ++i)
      if (pinned_dofs[i] < 1 || pinned_dofs[i] > num_dofs) return set_error(MLX_ERR_ARGUMENT, "pinned DOF out of range");
    const double keep = 1.0 - air_drag;
    parallel_ranges(num_dofs / 3, [&](long long a, long long b) {
      forces(a, b, gravity, custom_force, custom_force_vec, mass, f);
      residual_velocity(3 * a, 3 * b, h, keep, mass, v, f, residualv);
    }, kGrain / 3);
    // pinned DOFs: the velocity alone (the reference adds h f / m on the
    // unpinned ones only)
    for (int32_t i = 0; i < num_pinned; ++i) {
      const int32_t d = pinned_dofs[i] - 1;
      residualv[d] = keep * v[d];
    }
    return MLX_OK;
  });
}

// mesh3D.v = (xi - cache.oldp) ./ h (xpbdLayer3D.m:737).
int mlx_integrate_end(int32_t num_dofs, double h, const double* xi, const double* oldp, double* v) {
  return mlx::guarded([&]() -> int {
    if (num_dofs < 0) return set_error(MLX_ERR_ARGUMENT, "negative size");
    if (num_dofs == 0) return MLX_OK;
    if (!xi || !oldp || !v) return set_error(MLX_ERR_ARGUMENT, "xi, oldp and v are required");
    parallel_ranges(num_dofs, [&](long long a, long long b) { velocity(a, b, h, xi, oldp, v); });
    return MLX_OK;
  });
}

// xpbdLayer2D.contactVelocityUpdate (2d/integrator/xpbdLayer2D.m:577-603):
// per contact, the vertex's velocity vn (read before any write), e = 0 when
// |vn| <= 2 gravity h, else the restitution; vn + n .* (-vn + min(-e (n . vn), 0))
// written back in contact order, so a repeated vertex keeps its last contact's
// value as MATLAB's v(dofs) = ... does.
int mlx_contact_velocity_update(int32_t num_contacts, const double* normals, const int32_t* vertex_ids, int32_t dim,
                                int64_t num_dofs, const double* v, double h, double gravity, double restitution,
                                double* v_out) {
  return mlx::guarded([&]() -> int {
    if (num_contacts < 0 || num_dofs < 0) return set_error(MLX_ERR_ARGUMENT, "negative size");
    if (dim != 2 && dim != 3) return set_error(MLX_ERR_ARGUMENT, "dim must be 2 or 3");
    if (num_dofs % dim) return set_error(MLX_ERR_ARGUMENT, "num_dofs is not a multiple of dim");
    if (num_dofs > 0 && (!v || !v_out)) return set_error(MLX_ERR_ARGUMENT, "v and v_out are required");
    if (num_contacts > 0 && (!normals || !vertex_ids)) return set_error(MLX_ERR_ARGUMENT, "normals and vertex_ids are required");
    const long long nv = num_dofs / dim, K = num_contacts;
    for (long long k = 0; k < K; ++k)
      if (vertex_ids[k] < 1 || vertex_ids[k] > nv) return set_error(MLX_ERR_ARGUMENT, "contact vertex id out of range");
    std::unique_ptr<double[]> nvel(new double[(size_t)K * dim]);
    const double thresh = 2 * gravity * h;
    const bool can_stop = thresh >= 0;  // |vn| <= a negative threshold never holds
    parallel_ranges(K, [&](long long a, long long b) {
      for (long long k = a; k < b; ++k) {
        const double* vk = v + (size_t)(vertex_ids[k] - 1) * dim;
        double sq = vk[0] * vk[0], vt = normals[k] * vk[0];
        for (int c = 1; c < dim; ++c) {
          sq = sq + vk[c] * vk[c];
          vt = vt + normals[k + c * K] * vk[c];
        }
        const double e = can_stop && std::sqrt(sq) <= thresh ? 0.0 : restitution;
        const double m = std::min(-e * vt, 0.0);
        for (int c = 0; c < dim; ++c) nvel[(size_t)k * dim + c] = vk[c] + normals[k + c * K] * (-vk[c] + m);
      }
    }, kGrain / 8);  // scattered reads: threads pay off sooner
    if (v_out != v) std::memcpy(v_out, v, sizeof(double) * (size_t)num_dofs);
    for (long long k = 0; k < K; ++k) {
      double* o = v_out + (size_t)(vertex_ids[k] - 1) * dim;
      for (int c = 0; c < dim; ++c) o[c] = nvel[(size_t)k * dim + c];
    }
    return MLX_OK;
  });
}

}  // extern "C"
