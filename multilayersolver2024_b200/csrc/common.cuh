// common.cuh -- shared device types and helpers of the B200 XPBD kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mlx {

// Vertex record: position and inverse mass in one 16 B (FP32) or 32 B (FP64)
// load, so a tet gathers its four vertices with four vector loads.
template <typename R> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };
template <typename R> using R4 = typename Vec4<R>::type;

template <typename R> __host__ __device__ inline R4<R> make_r4(R x, R y, R z, R w);
template <> __host__ __device__ inline float4 make_r4<float>(float x, float y, float z, float w) {
  return make_float4(x, y, z, w);
}
template <> __host__ __device__ inline double4 make_r4<double>(double x, double y, double z, double w) {
  return make_double4(x, y, z, w);
}

// Vertex records are read and written through L2 (.cg): inside one
// persistent launch another SM may have written the record since this SM
// last cached it, and a tet's corners are never reused by the same SM within
// a colour, so L1 would only hold stale lines.
__device__ __forceinline__ float4 ldcg_r4(const float4* p) { return __ldcg(p); }
__device__ __forceinline__ double4 ldcg_r4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldcg(q), b = __ldcg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void stcg_r4(float4* p, float4 v) { __stcg(p, v); }
__device__ __forceinline__ void stcg_r4(double4* p, double4 v) {
  double2* q = reinterpret_cast<double2*>(p);
  __stcg(q, make_double2(v.x, v.y));
  __stcg(q + 1, make_double2(v.z, v.w));
}

// Vertex records addressed by vertex id in global memory.  The body, contact
// and pinning phases are written against this interface so the cluster
// kernel can run them on records held in distributed shared memory.
template <typename R> struct GlobalPos {
  R4<R>* p;
  __device__ __forceinline__ R4<R> ld(int v) const { return ldcg_r4(p + v); }
  __device__ __forceinline__ void st(int v, R4<R> x) const { stcg_r4(p + v, x); }
  __device__ __forceinline__ void st_comp(int v, int c, R val) const {
    __stcg(reinterpret_cast<R*>(p + v) + c, val);
  }
  // orders this thread's record stores before a following CTA barrier
  // (__syncthreads already does so for global memory)
  __device__ __forceinline__ void fence() const {}
};

struct D3 { double x, y, z; };
__host__ __device__ inline D3 d3(double x, double y, double z) { return {x, y, z}; }
__host__ __device__ inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline D3 cross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// M is a 3x3 column-major matrix
__host__ __device__ inline D3 mv3(const double* M, D3 v) {
  return {M[0] * v.x + M[3] * v.y + M[6] * v.z, M[1] * v.x + M[4] * v.y + M[7] * v.z,
          M[2] * v.x + M[5] * v.y + M[8] * v.z};
}

// Rigid body state, FP64 (the momentum and rotation accumulation stays in
// double on every precision path).  One record per body, 256 B aligned so a
// body's CTA reads it with few sectors.
struct __align__(16) Body {
  double R[9];      // current rotation
  double Rstep[9];  // rotation after the symplectic step (steppedVelocityR)
  double I0[9];     // body-frame inertia at construction
  double I[9];      // world inertia R I0 R'
  double com[3];
  double comdot[3];
  double omega[3];
  double mass;
  double pad[2];
};

}  // namespace mlx
