// common.cuh -- shared device helpers for the monolis B200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dev.h"

#define MB_CUDA_OK(expr)                                         \
  do {                                                           \
    cudaError_t _e = (expr);                                     \
    if (_e != cudaSuccess) return mb::report_cuda(_e, #expr, __FILE__, __LINE__); \
  } while (0)

namespace mb {

int report_cuda(cudaError_t e, const char* what, const char* file, int line);

constexpr int kWarp = 32;
constexpr int kSlice = 32;  // rows per sliced-ELL slice (one warp)

// ---- arithmetic without contraction: a*b + c evaluated as two roundings,
// the order the reference's Fortran loops use (gfortran emits no FMA on the
// x86-64 baseline ISA). Used wherever the FP64 path mirrors the reference.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
// FP32 inner loops have no reference order to follow: let the compiler fuse.
__device__ __forceinline__ float mul_rn(float a, float b) { return a * b; }
__device__ __forceinline__ float add_rn(float a, float b) { return a + b; }
__device__ __forceinline__ float sub_rn(float a, float b) { return a - b; }
__device__ __forceinline__ double axpy_rn(double a, double x, double y) { return __dadd_rn(__dmul_rn(a, x), y); }
__device__ __forceinline__ float axpy_rn(float a, float x, float y) { return fmaf(a, x, y); }

// ---- streaming loads: matrix values and column ids are read once per SpMV,
// so they are loaded with the evict-first hint to keep x resident in L1/L2.
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }

// ---- deterministic one-pass grid reduction of K doubles.
// Every block writes its K partial sums to partials[block*K + k]; the last
// block to arrive (atomic ticket) sums all partials in a fixed order and
// runs `fin` on thread 0. The ticket is reset by the last block, so the same
// scratch is reusable by the next stream-ordered launch.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* smem /* >= 32*K */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    double s = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) smem[wid * K + k] = s;
  }
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s = lane < nw ? smem[lane * K + k] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      v[k] = s;  // valid in thread 0
    }
  }
  __syncthreads();
}

template <int K, class Fin>
__device__ __forceinline__ void grid_reduce(double (&v)[K], double* partials, unsigned int* ticket, Fin fin) {
  __shared__ double smem[32 * K];
  __shared__ bool am_last;
  block_sum<K>(v, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) partials[(size_t)blockIdx.x * K + k] = v[k];
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] += __ldcg(partials + (size_t)b * K + k);
  }
  block_sum<K>(acc, smem);
  if (threadIdx.x == 0) {
    fin(acc);
    *ticket = 0u;
  }
}

}  // namespace mb
