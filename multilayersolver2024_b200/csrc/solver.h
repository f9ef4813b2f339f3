// solver.h -- internal interface between the C ABI and the precision-typed
// solver implementations.
#pragma once

#include <cuda_runtime.h>
#include <exception>
#include <new>
#include <string>
#include <system_error>
#include "../../include/mlxpbd.h"

namespace mlx {

extern thread_local std::string g_err;
int set_error(int code, const std::string& msg);

// The body of a C ABI entry point: a C++ exception (a failed host
// allocation, a host thread that could not start) becomes a status instead
// of crossing the C boundary.
template <typename F>
int guarded(F&& body) {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    return set_error(MLX_ERR_ALLOC, "host allocation failed");
  } catch (const std::system_error& e) {
    return set_error(MLX_ERR_ALLOC, std::string("host resource: ") + e.what());
  } catch (const std::exception& e) {
    return set_error(MLX_ERR_ARGUMENT, e.what());
  } catch (...) {
    return set_error(MLX_ERR_ARGUMENT, "unexpected C++ exception");
  }
}

struct SolverBase {
  virtual ~SolverBase() {}
  virtual int layer_solve(const mlx_layer_desc* ld, const mlx_solve_params* P, const mlx_contacts* K,
                          const mlx_solve_inputs* in, mlx_solve_outputs* out) = 0;
  virtual int sim_init(const mlx_layer_desc* ld, const mlx_solve_params* P, const double* p0, const double* v0,
                       double air_drag) = 0;
  virtual int sim_step(int nsteps, int use_graph, double* device_ms) = 0;
  virtual int sim_add_velocity(const int32_t* dofs, const double* dv, int n) = 0;
  virtual int sim_get_state(double* p, double* v) = 0;
  virtual long long sim_launches_per_step() const = 0;
  virtual long long launches_last_call() const = 0;
  virtual int enable_sweep_timing(int on) = 0;
  virtual int sweep_stats(double* ms, double* bytes, long long* launches, int reset) = 0;
  virtual std::string launch_path() const = 0;
  virtual int sim_autotune(int reps, double* before_ms, double* after_ms) = 0;
  virtual int find_contacts(const mlx_obstacle* obs, int nobs, const double* p, int max_contacts, int32_t* vids,
                            double* normals, double* points, double* comp, int32_t* K) = 0;
  virtual int sim_set_obstacles(const mlx_obstacle* obs, int nobs, double restitution) = 0;
  virtual int sim_contact_count(int32_t* n) = 0;
  virtual int sim_monitor(double* ra, int cap, int32_t* len, int32_t* total_it, double* run_until,
                          int32_t* status) = 0;
  virtual int ws_configure(int record, int mode, mlx_mlp* net, double gate, const float* fmean, const float* fstd,
                           const float* omean, const float* ostd, const float* corrections, int32_t* nb) = 0;
  virtual int ws_fetch(float* features, float* targets, int cap, int32_t* nb, int32_t* fallbacks) = 0;
  virtual int mws_configure(int on, double a, double b) = 0;
  virtual int ns_configure(int pcg_iterations, int every) = 0;
  virtual int pcg_solve(double h, const double* b, int iterations, double* x, double* resvec) = 0;
  virtual int build_layers(const double* p, const double* oldp, double h, int ordering, const int32_t* order,
                           const double* dminv, const double* sorted_layers, int L, const uint8_t* forced,
                           int32_t* sets, int32_t* num_rigids, uint8_t* is_elastic, uint8_t* is_boundary,
                           uint8_t* is_rigid_vertex, int32_t* vertex_body) = 0;
};

SolverBase* make_solver(const mlx_mesh_desc* md, int* rc);

int mlp_forward_on_stream(mlx_mlp* m, const float* d_x, int batch, cudaStream_t s, const float** y, int* ld);
int mlp_dims(const mlx_mlp* m, int* n_in, int* n_out, int* max_batch);
int mlp_wait_probe(int device, long long limit_ns, int* timed_out);

}  // namespace mlx
