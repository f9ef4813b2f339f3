// noalloc.cu -- constraint residual on caller-owned device arrays, without
// allocating any memory.
//
// Some callers of this library cannot allocate device memory themselves:
// a MATLAB mexcuda function whose arrays belong to MATLAB's gpuArray
// allocator, or a fixed-rate control loop where a cudaMalloc/cudaFree would
// stall the whole device.  mlx_stvk_residual_noalloc serves them: they pass
// device pointers to inputs and to the output, and the per-block partial sums
// of the reduction live in one file-scope device array of fixed size that the
// library image carries (every GPU that loads the library holds it until the
// process exits).
//
// Sharing rules of that array: every call uses the same array, and it keeps
// the partial sums of the last call.  Each call overwrites every partial it
// reads, so nothing has to be cleared between calls; two calls whose kernels
// overlap on the GPU (different streams, or another thread) race on it and
// must be serialised by the caller.
//
// Set-up: the first call on a device looks the array's device address up
// with cudaGetSymbolAddress while that device is current and caches it; make
// that first call outside any stream capture.
#include "../../include/mlxpbd.h"
#include "common.cuh"
#include "tet_kernels.cuh"
#include "solver.h"

#include <mutex>
#include <string>

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = MLX_NOALLOC_MAX_TETS / kThreads;

static __device__ __align__(256) double g_partials[kMaxBlocks];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_partials_addr[kMaxDevices] = {nullptr};

// Residual terms of the tets (simpleEvaluateAllConstraintResiduals,
// xpbdLayer3D.m:546-568) read from the MATLAB layout: x 3N interleaved,
// t T x 4 column-major 1-based, DmInv 3x3xT and alpha 6x6xT column-major
// pages, lambda T x 6 column-major.  One partial per block.
__global__ void __launch_bounds__(kThreads) k_residual_partials_matlab(
    const double* __restrict__ x, const int32_t* __restrict__ t, const double* __restrict__ DmInv,
    const double* __restrict__ alpha, const double* __restrict__ lambda, const double* __restrict__ vol, int T,
    double inv_h2, double* __restrict__ partials) {
  double acc[1] = {0.0};
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < T) {
    mlx::V3<double> X[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      int v = t[e + (size_t)T * k] - 1;
      X[k] = {x[3 * (size_t)v], x[3 * (size_t)v + 1], x[3 * (size_t)v + 2]};
    }
    double G[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) G[j] = DmInv[9 * (size_t)e + j];
    const double* a = alpha + 36 * (size_t)e;
    mlx::Compliance<double> cm;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) cm.aT[r][c] = a[r + 6 * c] * inv_h2;
#pragma unroll
    for (int q = 0; q < 3; ++q) cm.aS[q] = a[(3 + q) + 6 * (3 + q)] * inv_h2;
    double lam[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) lam[q] = lambda[e + (size_t)T * q];
    acc[0] = mlx::stvk_residual<double>(X, G, vol[e], cm, lam);
  }
  mlx::block_sum<1>(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

// Device address of g_partials on the current device (looked up once).
int partials_on_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return mlx::set_error(MLX_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return mlx::set_error(MLX_ERR_UNSUPPORTED, "device ordinal beyond 63");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_partials_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess)
      return mlx::set_error(MLX_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_partials_addr[dev] = static_cast<double*>(p);
  }
  *out = g_partials_addr[dev];
  return MLX_OK;
}

}  // namespace

extern "C" int mlx_stvk_residual_noalloc(int32_t num_vertices, int32_t num_tets, const double* d_x,
                                         const int32_t* d_t, const double* d_DmInv, const double* d_alpha,
                                         const double* d_lambda, const double* d_volume, double h,
                                         double* d_residual, void* stream) {
  if (num_tets < 0 || num_vertices < 0) return mlx::set_error(MLX_ERR_ARGUMENT, "negative size");
  if (num_tets > MLX_NOALLOC_MAX_TETS)
    return mlx::set_error(MLX_ERR_ARGUMENT, "mlx_stvk_residual_noalloc handles at most " +
                                                std::to_string(MLX_NOALLOC_MAX_TETS) + " tets, got " +
                                                std::to_string(num_tets));
  if (!(h > 0)) return mlx::set_error(MLX_ERR_ARGUMENT, "h must be > 0");
  if (!d_residual || (num_tets > 0 && (!d_x || !d_t || !d_DmInv || !d_alpha || !d_lambda || !d_volume)))
    return mlx::set_error(MLX_ERR_ARGUMENT, "null device pointer");
  double* partials = nullptr;
  int rc = partials_on_current_device(&partials);
  if (rc != MLX_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int blocks = num_tets > 0 ? (num_tets + kThreads - 1) / kThreads : 0;
  if (blocks > 0)
    k_residual_partials_matlab<<<blocks, kThreads, 0, s>>>(d_x, d_t, d_DmInv, d_alpha, d_lambda, d_volume, num_tets,
                                                           1.0 / (h * h), partials);
  mlx::k_finish_norm<256><<<1, kThreads, 0, s>>>(partials, blocks, d_residual);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mlx::set_error(MLX_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return MLX_OK;
}
