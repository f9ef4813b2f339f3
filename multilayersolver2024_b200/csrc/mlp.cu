// mlp.cu -- the learned warm start's multilayer perceptron on the 5th-gen
// tensor cores: BF16 operands, FP32 accumulation in tensor memory.
//
// Every product of training and inference is written as one "TN" GEMM
//     C[M x N] = A[M x K] . B[N x K]^T        (both operands K-contiguous)
// by keeping transposed copies where needed (W^T for dX, activations^T and
// dZ^T for dW).  One CTA (4 warps) computes a 128 x N tile:
//   * the K loop stages a 128 x 64 slice of A and an N x 64 slice of B into
//     shared memory in the canonical K-major layout of tcgen05 (8-row x 16 B
//     core matrices; the two K halves of one K=16 instruction LBO = 128 B
//     apart, 8-row groups SBO = 1024 B apart), makes them visible to the
//     async proxy and has one thread issue four tcgen05.mma (K = 16 each) into
//     the FP32 accumulator in tensor memory, completed through an mbarrier;
//   * the epilogue reads the accumulator with tcgen05.ld (warp w owns rows
//     32w..32w+31, one row per thread) and applies the layer's epilogue
//     (bias, GELU, GELU', BF16 rounding, transposed stores).
// Every mbarrier wait is bounded; a wait that gives up sets an error flag,
// and the kernel still releases its tensor memory.
#include "../../include/mlxpbd.h"
#include "solver.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace mlx {

namespace {

constexpr int kTileM = 128;
constexpr int kTileK = 64;
constexpr int kMaxN = 128;
constexpr unsigned long long kWaitNs = 1000000000ull;  // bounded mbarrier wait: 1 s

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, K-major, no swizzle (sm_100 version 1)
__device__ __forceinline__ uint64_t umma_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for phase `parity` of the barrier; false when the wait gave up
// after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned long long limit_ns = kWaitNs) {
  const uint32_t a = smem_addr(bar);
  const unsigned long long t0 = now_ns();
  for (unsigned spin = 0;; ++spin) {
    if ((spin & 1023u) == 1023u && now_ns() - t0 > limit_ns) return false;
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// GELU, x Phi(x) with Phi the standard normal CDF (Hendrycks & Gimpel,
// "Gaussian Error Linear Units (GELUs)", arXiv:1606.08415, 2016), in the
// tanh approximation given in that paper:
//   0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))),
// which stays within 1e-3 of x Phi(x) = 0.5 x (1 + erf(x / sqrt 2)) for every
// x (tested against erf on the host and on the device).
__device__ __forceinline__ float gelu(float x) {
  const float k = 0.7978845608028654f;  // sqrt(2 / pi)
  return 0.5f * x * (1.f + tanhf(k * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float k = 0.7978845608028654f;
  const float u = k * (x + 0.044715f * x * x * x);
  const float t = tanhf(u);
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * k * (1.f + 3.f * 0.044715f * x * x);
}

enum Epilogue : int {
  EPI_STORE_F32 = 0,   // C (FP32, row-major ldc)
  EPI_BIAS_GELU = 1,   // Z = C + bias (FP32), H = GELU(Z) as BF16 row-major and transposed
  EPI_BIAS = 2,        // Y = C + bias (FP32)
  EPI_GELU_GRAD = 3,   // dZ = C * GELU'(Z) as BF16 row-major and transposed
  EPI_BIAS_GELU_FWD = 4,  // inference: H = GELU(C + bias) as BF16 row-major only
};

struct GemmArgs {
  const __nv_bfloat16* A;  // [M x K], row stride lda (elements)
  const __nv_bfloat16* B;  // [N x K], row stride ldb
  int M, N, K, lda, ldb;
  int epi;
  const float* bias;       // [N]
  const float* Z;          // EPI_GELU_GRAD: pre-activation [M x N] (ldz)
  float* outF;             // FP32 output [M x N] (ldo)
  __nv_bfloat16* outH;     // BF16 output [M x N] (ldo)
  __nv_bfloat16* outHT;    // BF16 transposed output [N x M] (ldt)
  int ldo, ldt, ldz;
  int n_valid;             // columns >= n_valid are written as 0 (padding)
  int* error;              // set to 1 when a wait gives up
};

// One 128 x N tile (N a multiple of 16, at most 128).  128 threads.
__global__ void __launch_bounds__(128, 1) k_umma_gemm(GemmArgs g) {
  __shared__ __align__(1024) __nv_bfloat16 sA[kTileM * kTileK];
  __shared__ __align__(1024) __nv_bfloat16 sB[kMaxN * kTileK];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTileM;
  const int N = g.N;
  const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : 128u);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    failed = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = umma_idesc_bf16(N);
  unsigned phase = 0;

  for (int k0 = 0; k0 < g.K; k0 += kTileK) {
    // stage A (128 x 64) and B (N x 64) in the canonical K-major layout:
    // element (r, k) at (r/8)*1024 + (k/8)*128 + (r%8)*16 + (k%8)*2 bytes
    for (int c = tid; c < kTileM * (kTileK / 8); c += blockDim.x) {
      const int r = c / (kTileK / 8), kc = c % (kTileK / 8);
      const int gm = m0 + r, gk = k0 + kc * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (gm < g.M && gk < g.K) v = *reinterpret_cast<const uint4*>(g.A + (size_t)gm * g.lda + gk);
      *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sA) + (r >> 3) * 1024 + kc * 128 + (r & 7) * 16) = v;
    }
    for (int c = tid; c < N * (kTileK / 8); c += blockDim.x) {
      const int r = c / (kTileK / 8), kc = c % (kTileK / 8);
      const int gk = k0 + kc * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (gk < g.K) v = *reinterpret_cast<const uint4*>(g.B + (size_t)r * g.ldb + gk);
      *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sB) + (r >> 3) * 1024 + kc * 128 + (r & 7) * 16) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
#pragma unroll
      for (int kk = 0; kk < kTileK / 16; ++kk) {
        const uint64_t da = umma_desc(a0 + kk * 256, 128, 1024);
        const uint64_t db = umma_desc(b0 + kk * 256, 128, 1024);
        const uint32_t acc = (k0 > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&bar))
                   : "memory");
    }
    // the slices are reused by the next k step only after the MMAs read them
    if (!mbar_wait(&bar, phase)) failed = 1;
    phase ^= 1u;
    __syncthreads();
    if (failed) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;");

  if (!failed) {
    // epilogue: thread (warp w, lane l) owns row 32w + l
    const int row = m0 + warp * 32 + lane;
    const bool live = row < g.M;
    for (int n0 = 0; n0 < N; n0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)n0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (!live) continue;
      if (g.epi == EPI_BIAS || g.epi == EPI_BIAS_GELU_FWD) {
        // the thread's 16 consecutive columns of its row, in 16-byte stores
        // (ldo and n0 are multiples of 16)
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; j += 4) {
          const float4 b4 = *reinterpret_cast<const float4*>(g.bias + n0 + j);
          const float bb[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
          for (int i = 0; i < 4; ++i)
            v[j + i] = n0 + j + i >= g.n_valid ? 0.f : __uint_as_float(r[j + i]) + bb[i];
        }
        if (g.epi == EPI_BIAS) {
          float4* o = reinterpret_cast<float4*>(g.outF + (size_t)row * g.ldo + n0);
#pragma unroll
          for (int j = 0; j < 4; ++j) o[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        } else {
          uint4 h[2];
          __nv_bfloat162* hp = reinterpret_cast<__nv_bfloat162*>(h);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int a = 2 * j, b = 2 * j + 1;
            hp[j] = __floats2bfloat162_rn(n0 + a >= g.n_valid ? 0.f : gelu(v[a]),
                                          n0 + b >= g.n_valid ? 0.f : gelu(v[b]));
          }
          uint4* o = reinterpret_cast<uint4*>(g.outH + (size_t)row * g.ldo + n0);
          o[0] = h[0];
          o[1] = h[1];
        }
        continue;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + j;
        float v = __uint_as_float(r[j]);
        const bool pad = n >= g.n_valid;
        switch (g.epi) {
          case EPI_STORE_F32:
            g.outF[(size_t)row * g.ldo + n] = pad ? 0.f : v;
            break;
          case EPI_BIAS_GELU: {
            const float z = pad ? 0.f : v + g.bias[n];
            const __nv_bfloat16 hb = __float2bfloat16_rn(pad ? 0.f : gelu(z));
            g.outF[(size_t)row * g.ldo + n] = z;
            g.outH[(size_t)row * g.ldo + n] = hb;
            g.outHT[(size_t)n * g.ldt + row] = hb;
            break;
          }
          default: {  // EPI_GELU_GRAD
            const float dz = pad ? 0.f : v * gelu_grad(g.Z[(size_t)row * g.ldz + n]);
            const __nv_bfloat16 b = __float2bfloat16_rn(dz);
            g.outH[(size_t)row * g.ldo + n] = b;
            g.outHT[(size_t)n * g.ldt + row] = b;
          }
        }
      }
    }
  }
  if (failed) {
    // give the committed MMAs a second bounded chance to finish before the
    // tensor memory they write is released
    mbar_wait(&bar, phase ^ 1u);
    if (tid == 0) atomicExch(g.error, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}


// FP32 rows [B x n_in] -> BF16 [Bp x K] (zero padded) and its transpose [K x Bp]
__global__ void k_stage_input(const float* __restrict__ x, int B, int n_in, int Bp, int K,
                              __nv_bfloat16* __restrict__ xb, __nv_bfloat16* __restrict__ xt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Bp * K) return;
  const int r = i / K, c = i % K;
  const float v = (r < B && c < n_in) ? x[(size_t)r * n_in + c] : 0.f;
  const __nv_bfloat16 b = __float2bfloat16_rn(v);
  xb[(size_t)r * K + c] = b;
  xt[(size_t)c * Bp + r] = b;
}

// Mean-squared error over the valid outputs, L = sum (y - t)^2 / (B n_out):
// dY = 2 (y - t) / (B n_out) as BF16 [Bp x No] and transposed, and the
// squared error of every row (summed in fixed order afterwards).
__global__ void k_mse_grad(const float* __restrict__ y, int ldy, const float* __restrict__ t, int B, int n_out,
                           int Bp, int No, __nv_bfloat16* __restrict__ dy, __nv_bfloat16* __restrict__ dyt,
                           float* __restrict__ row_err) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Bp) return;
  float e = 0.f;
  const float scale = 2.f / ((float)B * (float)n_out);
  for (int c = 0; c < No; ++c) {
    float g = 0.f;
    if (r < B && c < n_out) {
      const float d = y[(size_t)r * ldy + c] - t[(size_t)r * n_out + c];
      e += d * d;
      g = scale * d;
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(g);
    dy[(size_t)r * No + c] = b;
    dyt[(size_t)c * Bp + r] = b;
  }
  row_err[r] = e;
}

// Row sums of a BF16 matrix [rows x cols] in FP32, one warp per row, fixed
// order (bias gradients from dZ^T).
__global__ void k_row_sums(const __nv_bfloat16* __restrict__ a, int rows, int cols, float* __restrict__ out) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= rows) return;
  float s = 0.f;
  for (int c = lane; c < cols; c += 32) s += __bfloat162float(a[(size_t)w * cols + c]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) out[w] = s;
}

// Sum of n floats in fixed order (one block of 256).
__global__ void k_sum(const float* __restrict__ a, int n, float* __restrict__ out) {
  __shared__ float sh[256];
  float s = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += a[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// Adam on the flat FP32 parameters (Kingma & Ba, bias-corrected moments).
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// FP32 layer parameters (W [n_out x n_in] row-major, then b) -> padded BF16
// W [No x Ki] and W^T [Ki x No], FP32 bias [No].
__global__ void k_refresh_layer(const float* __restrict__ W, const float* __restrict__ b, int n_out, int n_in, int No,
                                int Ki, __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wt,
                                float* __restrict__ bias) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= No * Ki) return;
  const int r = i / Ki, c = i % Ki;
  const float v = (r < n_out && c < n_in) ? W[(size_t)r * n_in + c] : 0.f;
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  wb[(size_t)r * Ki + c] = h;
  wt[(size_t)c * No + r] = h;
  if (c == 0) bias[r] = r < n_out ? b[r] : 0.f;
}

// Gradient tiles (FP32 [No x Ki] padded, bias [No]) -> flat gradient layout.
__global__ void k_gather_grad(const float* __restrict__ dw, const float* __restrict__ db, int n_out, int n_in, int Ki,
                              float* __restrict__ flat) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_out * n_in) {
    const int r = i / n_in, c = i % n_in;
    flat[i] = dw[(size_t)r * Ki + c];
  } else if (i < n_out * n_in + n_out) {
    flat[i] = db[i - n_out * n_in];
  }
}

inline int pad_to(int x, int m) { return (x + m - 1) / m * m; }

// Diagnostic of the bounded mbarrier wait the GEMM uses: thread 0 waits on a
// barrier no thread arrives at, so the wait runs out after limit_ns.
__global__ void k_probe_mbar_wait(unsigned long long limit_ns, int* timed_out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  *timed_out = mbar_wait(&bar, 0, limit_ns) ? 0 : 1;
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&bar)) : "memory");
}

}  // namespace

// The perceptron: n_in -> n_hidden (GELU) x n_layers_hidden -> n_out.
struct Mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n_in = 0, n_hidden = 0, n_hl = 0, n_out = 0, max_batch = 0;
  std::vector<int> din, dout, Kp, Np;   // per layer: true and padded dims
  std::vector<long long> poff;          // flat offset of each layer's W
  long long nparams = 0;
  int step = 0;
  // device buffers
  std::vector<void*> bufs;
  float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  std::vector<__nv_bfloat16*> wb, wt;    // per layer
  std::vector<float*> bias, dwf, dbf;    // per layer
  std::vector<float*> Z;                 // per hidden layer [Bp x Np]
  std::vector<__nv_bfloat16*> H, HT;     // layer inputs: [0] = X, [l] = output of hidden layer l-1
  std::vector<__nv_bfloat16*> dZ, dZT;   // per layer (last = dY)
  float *Y = nullptr, *row_err = nullptr, *scalar = nullptr, *xin = nullptr, *tin = nullptr;
  int* err = nullptr;

  ~Mlp() {
    for (void* p : bufs) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
  template <typename T> int alloc(T** p, size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess)
      return set_error(MLX_ERR_ALLOC, "cudaMalloc failed for the perceptron");
    cudaMemset(q, 0, sizeof(T) * std::max<size_t>(n, 1));
    bufs.push_back(q);
    *p = reinterpret_cast<T*>(q);
    return MLX_OK;
  }
  int layers() const { return n_hl + 1; }

  int create(int in, int hidden, int nhl, int out, int maxb, unsigned long long seed, int dev) {
    // a hidden layer's padded output width must equal the next layer's
    // padded input width (multiples of 64), hence n_hidden in {64, 128}
    if (in < 1 || (hidden != 64 && hidden != 128) || nhl < 1 || out < 1 || out > kMaxN || maxb < 1)
      return set_error(MLX_ERR_ARGUMENT, "perceptron sizes: n_hidden 64 or 128, n_out in [1, 128]");
    if (cudaSetDevice(dev) != cudaSuccess) return set_error(MLX_ERR_NO_DEVICE, "cudaSetDevice failed");
    device = dev;
    n_in = in; n_hidden = hidden; n_hl = nhl; n_out = out;
    max_batch = pad_to(maxb, kTileM);
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
      return set_error(MLX_ERR_CUDA, "cudaStreamCreate failed");
    const int L = layers();
    for (int l = 0; l < L; ++l) {
      const int a = l == 0 ? n_in : n_hidden, b = l == L - 1 ? n_out : n_hidden;
      din.push_back(a);
      dout.push_back(b);
      Kp.push_back(pad_to(a, kTileK));
      Np.push_back(pad_to(b, 16));
      poff.push_back(nparams);
      nparams += (long long)a * b + b;
    }
    int rc;
    if ((rc = alloc(&params, nparams)) || (rc = alloc(&grad, nparams)) || (rc = alloc(&adam_m, nparams)) ||
        (rc = alloc(&adam_v, nparams)))
      return rc;
    const int Bp = max_batch;
    wb.resize(L); wt.resize(L); bias.resize(L); dwf.resize(L); dbf.resize(L);
    H.resize(L); HT.resize(L); dZ.resize(L); dZT.resize(L); Z.resize(L);
    for (int l = 0; l < L; ++l) {
      if ((rc = alloc(&wb[l], (size_t)Np[l] * Kp[l])) || (rc = alloc(&wt[l], (size_t)Kp[l] * Np[l])) ||
          (rc = alloc(&bias[l], Np[l])) || (rc = alloc(&dwf[l], (size_t)Np[l] * Kp[l])) ||
          (rc = alloc(&dbf[l], Np[l])) || (rc = alloc(&H[l], (size_t)Bp * Kp[l])) ||
          (rc = alloc(&HT[l], (size_t)Kp[l] * Bp)) || (rc = alloc(&dZ[l], (size_t)Bp * Np[l])) ||
          (rc = alloc(&dZT[l], (size_t)Np[l] * Bp)) || (rc = alloc(&Z[l], (size_t)Bp * Np[l])))
        return rc;
    }
    if ((rc = alloc(&Y, (size_t)Bp * Np[L - 1])) || (rc = alloc(&row_err, Bp)) || (rc = alloc(&scalar, 4)) ||
        (rc = alloc(&xin, (size_t)Bp * n_in)) || (rc = alloc(&tin, (size_t)Bp * n_out)) || (rc = alloc(&err, 1)))
      return rc;
    // He-style initialisation from a fixed-seed generator (host), biases 0
    std::vector<float> h(nparams, 0.f);
    unsigned long long st = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto uni = [&]() {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      return ((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
    };
    for (int l = 0; l < L; ++l) {
      const double a = std::sqrt(6.0 / din[l]) * (l == L - 1 ? 0.1 : 1.0);
      for (long long i = 0; i < (long long)din[l] * dout[l]; ++i) h[poff[l] + i] = (float)(a * uni());
    }
    return set_params(h.data(), nparams);
  }

  int refresh() {
    for (int l = 0; l < layers(); ++l) {
      const int n = Np[l] * Kp[l];
      k_refresh_layer<<<(n + 255) / 256, 256, 0, stream>>>(params + poff[l], params + poff[l] + (long long)din[l] * dout[l],
                                                           dout[l], din[l], Np[l], Kp[l], wb[l], wt[l], bias[l]);
    }
    return cudaGetLastError() == cudaSuccess ? MLX_OK : set_error(MLX_ERR_CUDA, "refresh launch failed");
  }
  int set_params(const float* h, long long n) {
    if (n != nparams) return set_error(MLX_ERR_ARGUMENT, "parameter count mismatch");
    if (cudaMemcpyAsync(params, h, sizeof(float) * n, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return set_error(MLX_ERR_CUDA, "parameter upload failed");
    cudaMemsetAsync(adam_m, 0, sizeof(float) * n, stream);
    cudaMemsetAsync(adam_v, 0, sizeof(float) * n, stream);
    step = 0;
    int rc = refresh();
    if (rc) return rc;
    return cudaStreamSynchronize(stream) == cudaSuccess ? MLX_OK : set_error(MLX_ERR_CUDA, "sync failed");
  }

  int gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K, int epi,
           const float* bias_, const float* Zin, int ldz, float* outF, __nv_bfloat16* outH, __nv_bfloat16* outHT,
           int ldo, int ldt, int n_valid) {
    GemmArgs g{A, B, M, N, K, lda, ldb, epi, bias_, Zin, outF, outH, outHT, ldo, ldt, ldz, n_valid, err};
    k_umma_gemm<<<(M + kTileM - 1) / kTileM, 128, 0, stream>>>(g);
    return cudaGetLastError() == cudaSuccess ? MLX_OK : set_error(MLX_ERR_CUDA, "tensor-core GEMM launch failed");
  }

  // forward on device inputs x [B x n_in] (FP32); output Y [Bp x Np_last].
  // `train` keeps what the backward pass reads (pre-activations, transposed
  // activations); inference writes the activations only.
  int forward_dev(const float* x, int B, bool train = true) {
    if (B < 1 || B > max_batch) return set_error(MLX_ERR_ARGUMENT, "batch size out of [1, max_batch]");
    const int Bp = pad_to(B, kTileM), L = layers();
    const int n0 = Bp * Kp[0];
    k_stage_input<<<(n0 + 255) / 256, 256, 0, stream>>>(x, B, n_in, Bp, Kp[0], H[0], HT[0]);
    int rc;
    for (int l = 0; l < L; ++l) {
      if (l < L - 1 && !train) {
        rc = gemm(H[l], Kp[l], wb[l], Kp[l], Bp, Np[l], Kp[l], EPI_BIAS_GELU_FWD, bias[l], nullptr, 0, nullptr,
                  H[l + 1], nullptr, Np[l], 0, dout[l]);
      } else if (l < L - 1) {
        rc = gemm(H[l], Kp[l], wb[l], Kp[l], Bp, Np[l], Kp[l], EPI_BIAS_GELU, bias[l], nullptr, 0, Z[l], H[l + 1],
                  HT[l + 1], Np[l], Bp, dout[l]);
      } else {
        rc = gemm(H[l], Kp[l], wb[l], Kp[l], Bp, Np[l], Kp[l], EPI_BIAS, bias[l], nullptr, 0, Y, nullptr, nullptr,
                  Np[l], 0, dout[l]);
      }
      if (rc) return rc;
    }
    return MLX_OK;
  }

  // loss and flat gradient (device) for inputs x / targets t already on the device
  int backward_dev(const float* t, int B) {
    const int Bp = pad_to(B, kTileM), L = layers();
    k_mse_grad<<<(Bp + 127) / 128, 128, 0, stream>>>(Y, Np[L - 1], t, B, n_out, Bp, Np[L - 1], dZ[L - 1], dZT[L - 1],
                                                     row_err);
    k_sum<<<1, 256, 0, stream>>>(row_err, Bp, scalar);
    int rc;
    for (int l = L - 1; l >= 0; --l) {
      // dW_l = dZ_l^T . H_l  (M = Np[l], N = Kp[l], reduction over the batch)
      rc = gemm(dZT[l], Bp, HT[l], Bp, Np[l], Kp[l], Bp, EPI_STORE_F32, nullptr, nullptr, 0, dwf[l], nullptr,
                nullptr, Kp[l], 0, Kp[l]);
      if (rc) return rc;
      k_row_sums<<<(Np[l] * 32 + 255) / 256, 256, 0, stream>>>(dZT[l], Np[l], Bp, dbf[l]);
      const int ng = dout[l] * din[l] + dout[l];
      k_gather_grad<<<(ng + 255) / 256, 256, 0, stream>>>(dwf[l], dbf[l], dout[l], din[l], Kp[l], grad + poff[l]);
      if (l > 0) {
        // dH_{l} = dZ_l . W_l, then dZ_{l-1} = dH * GELU'(Z_{l-1})
        rc = gemm(dZ[l], Np[l], wt[l], Np[l], Bp, Np[l - 1], Np[l], EPI_GELU_GRAD, nullptr, Z[l - 1], Np[l - 1],
                  nullptr, dZ[l - 1], dZT[l - 1], Np[l - 1], Bp, dout[l - 1]);
        if (rc) return rc;
      }
    }
    return cudaGetLastError() == cudaSuccess ? MLX_OK : set_error(MLX_ERR_CUDA, "backward launch failed");
  }

  int check_error() {
    int e = 0;
    cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return set_error(MLX_ERR_CUDA, "perceptron stream failed");
    if (e) return set_error(MLX_ERR_LIMIT, "a tensor-core GEMM waited more than 1 s for its MMAs");
    return MLX_OK;
  }

  int upload(const float* x, const float* t, int B) {
    if (B < 1 || B > max_batch) return set_error(MLX_ERR_ARGUMENT, "batch size out of [1, max_batch]");
    if (x && cudaMemcpyAsync(xin, x, sizeof(float) * B * n_in, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return set_error(MLX_ERR_CUDA, "input upload failed");
    if (t && cudaMemcpyAsync(tin, t, sizeof(float) * B * n_out, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return set_error(MLX_ERR_CUDA, "target upload failed");
    return MLX_OK;
  }

  int adam(float lr) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    k_adam<<<(int)((nparams + 255) / 256), 256, 0, stream>>>(params, grad, adam_m, adam_v, nparams, lr, b1, b2, 1e-8f,
                                                             c1, c2);
    return refresh();
  }
};

}  // namespace mlx

using mlx::Mlp;

struct mlx_mlp {
  Mlp impl;
};

namespace mlx {
// Forward of `batch` device rows on stream `s` (which may be capturing);
// *y / *ld receive the device output rows and their stride.
int mlp_forward_on_stream(mlx_mlp* m, const float* d_x, int batch, cudaStream_t s, const float** y, int* ld) {
  if (!m) return set_error(MLX_ERR_ARGUMENT, "null perceptron");
  Mlp& p = m->impl;
  cudaStream_t own = p.stream;
  p.stream = s;
  const int rc = p.forward_dev(d_x, batch, false);
  p.stream = own;
  if (y) *y = p.Y;
  if (ld) *ld = p.Np.back();
  return rc;
}
int mlp_dims(const mlx_mlp* m, int* n_in, int* n_out, int* max_batch) {
  if (!m) return set_error(MLX_ERR_ARGUMENT, "null perceptron");
  *n_in = m->impl.n_in;
  *n_out = m->impl.n_out;
  *max_batch = m->impl.max_batch;
  return MLX_OK;
}
}  // namespace mlx

namespace mlx {
int mlp_wait_probe(int device, long long limit_ns, int* timed_out) {
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return set_error(MLX_ERR_ARGUMENT, "bad device");
  int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(int));
  if (e == cudaSuccess) {
    k_probe_mbar_wait<<<1, 32>>>((unsigned long long)limit_ns, d);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(timed_out, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
  }
  cudaSetDevice(prev);
  if (e != cudaSuccess) return set_error(MLX_ERR_CUDA, std::string("mbarrier wait probe: ") + cudaGetErrorString(e));
  return MLX_OK;
}
}  // namespace mlx

extern "C" {

int mlx_mlp_create(int32_t n_in, int32_t n_hidden, int32_t n_hidden_layers, int32_t n_out, int32_t max_batch,
                   uint64_t seed, int32_t device, mlx_mlp** out) {
  return mlx::guarded([&]() -> int {
    if (!out) return mlx::set_error(MLX_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    mlx_mlp* m = new mlx_mlp();
    int rc = m->impl.create(n_in, n_hidden, n_hidden_layers, n_out, max_batch, seed, device);
    if (rc != MLX_OK) {
      delete m;
      return rc;
    }
    *out = m;
    return MLX_OK;
  });
}

int mlx_mlp_destroy(mlx_mlp* m) {
  return mlx::guarded([&]() -> int {
    delete m;
    return MLX_OK;
  });
}

long long mlx_mlp_num_params(const mlx_mlp* m) { return m ? m->impl.nparams : 0; }

int mlx_mlp_set_params(mlx_mlp* m, const float* params, long long n) {
  return mlx::guarded([&]() -> int {
    if (!m || !params) return mlx::set_error(MLX_ERR_ARGUMENT, "null argument");
    cudaSetDevice(m->impl.device);
    return m->impl.set_params(params, n);
  });
}

int mlx_mlp_get_params(mlx_mlp* m, float* params, long long n) {
  return mlx::guarded([&]() -> int {
    if (!m || !params) return mlx::set_error(MLX_ERR_ARGUMENT, "null argument");
    if (n != m->impl.nparams) return mlx::set_error(MLX_ERR_ARGUMENT, "parameter count mismatch");
    cudaSetDevice(m->impl.device);
    cudaMemcpyAsync(params, m->impl.params, sizeof(float) * n, cudaMemcpyDeviceToHost, m->impl.stream);
    return cudaStreamSynchronize(m->impl.stream) == cudaSuccess ? MLX_OK : mlx::set_error(MLX_ERR_CUDA, "copy failed");
  });
}

int mlx_mlp_forward(mlx_mlp* m, const float* x, int32_t batch, float* y) {
  return mlx::guarded([&]() -> int {
    if (!m || !x || !y) return mlx::set_error(MLX_ERR_ARGUMENT, "null argument");
    Mlp& p = m->impl;
    cudaSetDevice(p.device);
    int rc;
    if ((rc = p.upload(x, nullptr, batch)) || (rc = p.forward_dev(p.xin, batch, false)) || (rc = p.check_error()))
      return rc;
    const int No = p.Np.back();
    std::vector<float> h((size_t)batch * No);
    cudaMemcpyAsync(h.data(), p.Y, sizeof(float) * batch * No, cudaMemcpyDeviceToHost, p.stream);
    if (cudaStreamSynchronize(p.stream) != cudaSuccess) return mlx::set_error(MLX_ERR_CUDA, "copy failed");
    for (int r = 0; r < batch; ++r)
      for (int c = 0; c < p.n_out; ++c) y[(size_t)r * p.n_out + c] = h[(size_t)r * No + c];
    return MLX_OK;
  });
}

int mlx_mlp_loss_grad(mlx_mlp* m, const float* x, const float* target, int32_t batch, float* loss, float* grad) {
  return mlx::guarded([&]() -> int {
    if (!m || !x || !target) return mlx::set_error(MLX_ERR_ARGUMENT, "null argument");
    Mlp& p = m->impl;
    cudaSetDevice(p.device);
    int rc;
    if ((rc = p.upload(x, target, batch)) || (rc = p.forward_dev(p.xin, batch)) || (rc = p.backward_dev(p.tin, batch)) ||
        (rc = p.check_error()))
      return rc;
    float h[1];
    cudaMemcpyAsync(h, p.scalar, sizeof(float), cudaMemcpyDeviceToHost, p.stream);
    if (grad) cudaMemcpyAsync(grad, p.grad, sizeof(float) * p.nparams, cudaMemcpyDeviceToHost, p.stream);
    if (cudaStreamSynchronize(p.stream) != cudaSuccess) return mlx::set_error(MLX_ERR_CUDA, "copy failed");
    if (loss) *loss = h[0] / ((float)batch * (float)p.n_out);
    return MLX_OK;
  });
}

int mlx_mlp_train(mlx_mlp* m, const float* x, const float* target, int32_t n_samples, int32_t batch, int32_t epochs,
                  float lr, uint64_t seed, float* losses) {
  return mlx::guarded([&]() -> int {
    if (!m || !x || !target) return mlx::set_error(MLX_ERR_ARGUMENT, "null argument");
    Mlp& p = m->impl;
    if (batch < 1 || batch > p.max_batch || n_samples < batch)
      return mlx::set_error(MLX_ERR_ARGUMENT, "need 1 <= batch <= max_batch and batch <= n_samples");
    cudaSetDevice(p.device);
    // mini-batches are gathered by a host-side permutation per epoch (fixed seed)
    std::vector<int> order(n_samples);
    for (int i = 0; i < n_samples; ++i) order[i] = i;
    unsigned long long st = seed * 2862933555777941757ull + 3037000493ull;
    std::vector<float> bx((size_t)batch * p.n_in), bt((size_t)batch * p.n_out);
    int rc = MLX_OK;
    const int nb = n_samples / batch;
    for (int e = 0; e < epochs && rc == MLX_OK; ++e) {
      for (int i = n_samples - 1; i > 0; --i) {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        const int j = (int)((st >> 33) % (unsigned long long)(i + 1));
        std::swap(order[i], order[j]);
      }
      double esum = 0;
      for (int b = 0; b < nb && rc == MLX_OK; ++b) {
        for (int r = 0; r < batch; ++r) {
          const int k = order[b * batch + r];
          std::memcpy(&bx[(size_t)r * p.n_in], x + (size_t)k * p.n_in, sizeof(float) * p.n_in);
          std::memcpy(&bt[(size_t)r * p.n_out], target + (size_t)k * p.n_out, sizeof(float) * p.n_out);
        }
        if ((rc = p.upload(bx.data(), bt.data(), batch)) || (rc = p.forward_dev(p.xin, batch)) ||
            (rc = p.backward_dev(p.tin, batch)) || (rc = p.adam(lr)))
          break;
        float h = 0;
        cudaMemcpyAsync(&h, p.scalar, sizeof(float), cudaMemcpyDeviceToHost, p.stream);
        if (cudaStreamSynchronize(p.stream) != cudaSuccess) rc = mlx::set_error(MLX_ERR_CUDA, "training step failed");
        esum += h / ((double)batch * p.n_out);
      }
      if (losses) losses[e] = (float)(esum / nb);
    }
    if (rc == MLX_OK) rc = p.check_error();
    return rc;
  });
}

}  // extern "C"
