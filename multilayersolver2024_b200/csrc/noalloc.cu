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
// Set-up: the first call in a CUDA context (the first call on a device, and
// the first call after a cudaDeviceReset -- MATLAB's reset(gpuDevice) --
// which reloads the library image at a new address) looks the array's device
// address up with cudaGetSymbolAddress while that device is current and
// caches it per context; make that first call outside any stream capture.
//
// Indices: t is read as int32, 1-based.  A tet with a vertex index outside
// [1, num_vertices] is not read; its block's partial becomes NaN, so the
// residual written to d_residual is NaN and no memory outside the caller's
// arrays is touched.
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
// per device ordinal: the context the address was looked up in, and the address
unsigned long long g_partials_ctx[kMaxDevices] = {0};
double* g_partials_addr[kMaxDevices] = {nullptr};

// Unique id of the current CUDA context (cuCtxGetCurrent + cuCtxGetId through
// the runtime's driver entry points, so nothing links libcuda); 0 if unknown.
unsigned long long current_context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
    resolved = true;
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

// Residual terms of the tets (simpleEvaluateAllConstraintResiduals,
// xpbdLayer3D.m:546-568) read from the MATLAB layout: x 3N interleaved,
// t T x 4 column-major 1-based, DmInv 3x3xT and alpha 6x6xT column-major
// pages, lambda T x 6 column-major.  One partial per block.
__global__ void __launch_bounds__(kThreads) k_residual_partials_matlab(
    const double* __restrict__ x, const int32_t* __restrict__ t, const double* __restrict__ DmInv,
    const double* __restrict__ alpha, const double* __restrict__ lambda, const double* __restrict__ vol, int T,
    int N, double inv_h2, double* __restrict__ partials) {
  double acc[1] = {0.0};
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  int vid[4] = {0, 0, 0, 0};
  bool bad = false;
  if (e < T) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      vid[k] = t[e + (size_t)T * k] - 1;
      bad |= (unsigned)vid[k] >= (unsigned)N;
    }
  }
  if (e < T && !bad) {
    mlx::V3<double> X[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t v = (size_t)vid[k];
      X[k] = {x[3 * v], x[3 * v + 1], x[3 * v + 2]};
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
  if (bad) acc[0] = __longlong_as_double(0x7ff8000000000000LL);  // NaN marks an index outside the mesh
  mlx::block_sum<1>(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

// Device address of g_partials in the current context (looked up once per
// context; a context id of 0, when the driver cannot report it, looks it up
// on every call).
int partials_on_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return mlx::set_error(MLX_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return mlx::set_error(MLX_ERR_UNSUPPORTED, "device ordinal beyond 63");
  std::lock_guard<std::mutex> lock(g_mutex);
  const unsigned long long ctx = current_context_id();
  if (!g_partials_addr[dev] || ctx == 0 || ctx != g_partials_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess)
      return mlx::set_error(MLX_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_partials_addr[dev] = static_cast<double*>(p);
    g_partials_ctx[dev] = ctx;
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
  if (num_tets > 0 && num_vertices == 0) return mlx::set_error(MLX_ERR_ARGUMENT, "tets given without vertices");
  // an error left pending by earlier work belongs to the caller: report it
  // as such, without clearing it or launching anything
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return mlx::set_error(MLX_ERR_CUDA, std::string("a CUDA error was pending before this call: ") +
                                            cudaGetErrorString(e));
  double* partials = nullptr;
  int rc = partials_on_current_device(&partials);
  if (rc != MLX_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int blocks = num_tets > 0 ? (num_tets + kThreads - 1) / kThreads : 0;
  if (blocks > 0) {
    k_residual_partials_matlab<<<blocks, kThreads, 0, s>>>(d_x, d_t, d_DmInv, d_alpha, d_lambda, d_volume, num_tets,
                                                           num_vertices, 1.0 / (h * h), partials);
    e = cudaGetLastError();
    if (e != cudaSuccess)
      return mlx::set_error(MLX_ERR_CUDA, std::string("residual launch: ") + cudaGetErrorString(e));
  }
  mlx::k_finish_norm<256><<<1, kThreads, 0, s>>>(partials, blocks, d_residual);
  e = cudaGetLastError();
  if (e != cudaSuccess) return mlx::set_error(MLX_ERR_CUDA, std::string("norm launch: ") + cudaGetErrorString(e));
  return MLX_OK;
}
