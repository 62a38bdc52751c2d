// Shared helpers of the sm_100a PF-FLIP library: error state, launch
// accounting, storage-type conversion, index helpers and deterministic block
// reductions.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>

#include "pfflip.h"

namespace pf {

// ---------------------------------------------------------------- errors
void set_error(int code, const char* fmt, ...);
void set_cuda_error(cudaError_t e, const char* where);
void count_launch(uint64_t n = 1);

#define PF_REQUIRE(cond, ...)                    \
  do {                                           \
    if (!(cond)) {                               \
      ::pf::set_error(PF_ERR_ARG, __VA_ARGS__);  \
      return PF_ERR_ARG;                         \
    }                                            \
  } while (0)

#define PF_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t e_ = (expr);                                \
    if (e_ != cudaSuccess) {                                \
      ::pf::set_cuda_error(e_, #expr);                      \
      return PF_ERR_CUDA;                                   \
    }                                                       \
  } while (0)

// after a kernel launch
#define PF_LAUNCHED()                                       \
  do {                                                      \
    cudaError_t e_ = cudaGetLastError();                    \
    if (e_ != cudaSuccess) {                                \
      ::pf::set_cuda_error(e_, "kernel launch");            \
      return PF_ERR_CUDA;                                   \
    }                                                       \
    ::pf::count_launch();                                   \
  } while (0)

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kNumSMs = 148;

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// ---------------------------------------------------------------- storage types
template <class T> struct Store;
template <> struct Store<float> {
  static __device__ __forceinline__ float ld(const float* p) { return *p; }
  static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
};
template <> struct Store<__half> {
  static __device__ __forceinline__ float ld(const __half* p) { return __half2float(*p); }
  static __device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
};
template <> struct Store<__nv_bfloat16> {
  static __device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};

template <class T> __device__ __forceinline__ float ldT(const T* p) { return Store<T>::ld(p); }
// the value a float becomes when stored as T and read back
template <class T> __device__ __forceinline__ float roundT(float v) {
  T t;
  Store<T>::st(&t, v);
  return Store<T>::ld(&t);
}
template <class T> __device__ __forceinline__ void stT(T* p, float v) { Store<T>::st(p, v); }

// ---------------------------------------------------------------- particle sort keys
// linear index of the cell floor(x/dx) (IEEE binary32 division, clamped to the grid)
__device__ __forceinline__ int cell_key(float x, float y, float z, float dx, int nx, int ny, int nz) {
  int i = (int)floorf(x / dx), j = (int)floorf(y / dx), k = (int)floorf(z / dx);
  i = min(max(i, 0), nx - 1);
  j = min(max(j, 0), ny - 1);
  k = min(max(k, 0), nz - 1);
  return (i * ny + j) * nz + k;
}

// warp-aggregated atomicAdd(&ctr[key], 1) over the lanes in `active`: returns this lane's slot
__device__ __forceinline__ int agg_inc(int* ctr, int key, unsigned active) {
  const unsigned grp = __match_any_sync(active, key);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(grp) - 1;
  const int rank = __popc(grp & ((1u << lane) - 1u));
  int base = 0;
  if (lane == leader) base = atomicAdd(ctr + key, __popc(grp));
  base = __shfl_sync(grp, base, leader);
  return base + rank;
}

// ---------------------------------------------------------------- index helpers
struct Dim3i {
  int n0, n1, n2;
  __host__ __device__ __forceinline__ long long at(int i, int j, int k) const {
    return ((long long)i * n1 + j) * n2 + k;
  }
  __host__ __device__ __forceinline__ long long size() const { return (long long)n0 * n1 * n2; }
};

__host__ __device__ __forceinline__ Dim3i face_dims(int nx, int ny, int nz, int axis) {
  return Dim3i{nx + (axis == 0), ny + (axis == 1), nz + (axis == 2)};
}

// ---------------------------------------------------------------- reductions
// Block-wide sum of a double; result valid in thread 0.  blockDim.x must be a
// multiple of 32 and <= 1024.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <int NT> __device__ __forceinline__ double block_sum(double v, double* sh /*>= 32*/) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = (l < NT / 32) ? sh[l] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

template <int NT> __device__ __forceinline__ float block_max(float v, float* sh /*>= 32*/) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  float r = 0.f;
  if (w == 0) {
    r = (l < NT / 32) ? sh[l] : 0.f;
    r = warp_max(r);
  }
  __syncthreads();
  return r;
}

// Deterministic grid reduction over a grid of any shape: every block writes
// its partial at its linear block id, the last block to arrive (ticket on
// *counter) sums the partials in block order with a fixed tree and resets the
// counter.  Returns true in the last block (all threads), with *result valid
// in every thread of that block.  The partials are read from L2 (__ldcg):
// they were written by other blocks before their fenced ticket.
// [c0, c1) of this warp's contiguous share of n items (a 1-D launch), in
// multiples of 32: lane l takes items c0 + l, c0 + l + 32, ...  Over the
// cell-sorted particle streams a warp's successive items lie in neighbouring
// cells, so the grid values it gathers stay in L1 from one step to the next.
__device__ __forceinline__ void warp_chunk(long long n, long long& c0, long long& c1) {
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  const long long chunk = ((n + warps - 1) / warps + 31) & ~31LL;
  c0 = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * chunk;
  c1 = c0 + chunk < n ? c0 + chunk : n;
}

__device__ __forceinline__ unsigned lin_block() { return (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x; }
__device__ __forceinline__ unsigned num_blocks() { return gridDim.x * gridDim.y * gridDim.z; }

template <int NT>
__device__ __forceinline__ bool grid_sum_last(double partial_in_t0, double* partials, unsigned* counter,
                                              double* result, double* sh) {
  __shared__ bool s_last;
  const unsigned nb = num_blocks();
  if (threadIdx.x == 0) {
    partials[lin_block()] = partial_in_t0;
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    s_last = (t == nb - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double v = 0.0;
#pragma unroll 8
  for (unsigned b = threadIdx.x; b < nb; b += NT) v += __ldcg(partials + b);
  v = block_sum<NT>(v, sh);
  if (threadIdx.x == 0) {
    sh[32] = v;
    *counter = 0u;
  }
  __syncthreads();
  *result = sh[32];
  return true;
}

// Two sums at once (same protocol; partials holds 2 * blocks doubles).
template <int NT>
__device__ __forceinline__ bool grid_sum2_last(double a_t0, double b_t0, double* partials, unsigned* counter,
                                               double* ra, double* rb, double* sh) {
  __shared__ bool s_last;
  const unsigned nb = num_blocks();
  if (threadIdx.x == 0) {
    const unsigned id = lin_block();
    partials[2 * id] = a_t0;
    partials[2 * id + 1] = b_t0;
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    s_last = (t == nb - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double va = 0.0, vb = 0.0;
#pragma unroll 8
  for (unsigned b = threadIdx.x; b < nb; b += NT) {
    va += __ldcg(partials + 2 * b);
    vb += __ldcg(partials + 2 * b + 1);
  }
  va = block_sum<NT>(va, sh);
  vb = block_sum<NT>(vb, sh);
  if (threadIdx.x == 0) {
    sh[32] = va;
    sh[33] = vb;
    *counter = 0u;
  }
  __syncthreads();
  *ra = sh[32];
  *rb = sh[33];
  return true;
}

template <int NT>
__device__ __forceinline__ bool grid_max_last(float partial_in_t0, double* partials, unsigned* counter,
                                              float* result, float* shf) {
  __shared__ bool s_last;
  const unsigned nb = num_blocks();
  if (threadIdx.x == 0) {
    partials[lin_block()] = (double)partial_in_t0;
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    s_last = (t == nb - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  float v = 0.f;
#pragma unroll 8
  for (unsigned b = threadIdx.x; b < nb; b += NT) v = fmaxf(v, (float)__ldcg(partials + b));
  v = block_max<NT>(v, shf);
  if (threadIdx.x == 0) {
    shf[32] = v;
    *counter = 0u;
  }
  __syncthreads();
  *result = shf[32];
  return true;
}

// 3D launch shape for cell-wise kernels: 256 threads = 8 rows (j) of 32 cells
// (k), blockIdx.z = i.  Index math is shifts and adds only.
constexpr int C3_TK = 32, C3_TJ = 8, C3_NT = 256;
inline dim3 grid_cells(int n0, int n1, int n2) {
  return dim3((unsigned)((n2 + C3_TK - 1) / C3_TK), (unsigned)((n1 + C3_TJ - 1) / C3_TJ), (unsigned)n0);
}
struct Cell3 {
  int i, j, k;
};
__device__ __forceinline__ Cell3 cell_here() {
  return Cell3{(int)blockIdx.z, (int)(blockIdx.y * C3_TJ + (threadIdx.x >> 5)),
               (int)(blockIdx.x * C3_TK + (threadIdx.x & 31))};
}

// float max via integer atomics (valid for non-negative floats)
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

inline int grid_for(long long n, int nt, int max_blocks) {
  long long b = (n + nt - 1) / nt;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

}  // namespace pf
