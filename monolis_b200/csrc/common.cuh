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
__device__ __forceinline__ short ld_stream(const short* p) { return __ldcs(p); }

// ---- deterministic one-pass grid reduction of K doubles, two levels.
// Every block writes its K partial sums to partials[block*K + k]. Blocks are
// grouped by kReduceGroup consecutive indices; the last block of a group to
// arrive (atomic ticket[1 + group]) sums that group's partials in index order
// into partials[(gridDim.x + group)*K + k], and the last group to finish
// (atomic ticket[0]) sums the group sums in index order and runs `fin` on
// thread 0. Each finishing block reads at most kReduceGroup values, one per
// thread, so the tail of the reduction stays short at any grid size, and the
// result does not depend on the order in which blocks arrive. The tickets
// are reset by the blocks that consumed them, so the same scratch serves the
// next stream-ordered launch.
//   partials: >= (gridDim.x + ceil(gridDim.x / kReduceGroup)) * K doubles
//   ticket:   >= 1 + ceil(gridDim.x / kReduceGroup) zero-initialised words
constexpr int kReduceGroup = 256;
constexpr int kTicketWords = 1 + 65536 / kReduceGroup;  // grids up to 65536 blocks

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
  const unsigned int G = gridDim.x;
  const unsigned int ngroups = (G + kReduceGroup - 1) / kReduceGroup;
  const unsigned int g = blockIdx.x / kReduceGroup;
  const unsigned int g0 = g * kReduceGroup;
  const unsigned int gsize = min((unsigned int)kReduceGroup, G - g0);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) partials[(size_t)blockIdx.x * K + k] = v[k];
    __threadfence();
    const unsigned int t = atomicAdd(ticket + 1 + g, 1u);
    am_last = (t == gsize - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  for (unsigned int b = threadIdx.x; b < gsize; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] += __ldcg(partials + (size_t)(g0 + b) * K + k);
  }
  block_sum<K>(acc, smem);
  double* top = partials + (size_t)G * K;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) top[(size_t)g * K + k] = acc[k];
    ticket[1 + g] = 0u;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    am_last = (t == ngroups - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  for (unsigned int b = threadIdx.x; b < ngroups; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] += __ldcg(top + (size_t)b * K + k);
  }
  block_sum<K>(acc, smem);
  if (threadIdx.x == 0) {
    fin(acc);
    *ticket = 0u;
  }
}

}  // namespace mb
