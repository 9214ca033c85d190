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

// ---- order-robust dot products (FP64 solver path) ----
// The reference's serial inner product rounds after every addition, so its
// value depends on the order of the sum; an OpenMP build with another thread
// count, or any parallel reduction, gets other roundings, and BiCGSTAB's
// iteration count drifts with them. The FP64 kernels here therefore sum
// the products in double-double, the arithmetic of the reference's own
// pseudo-quadruple inner product (src/linalg/inner_product.f90:219-258:
// each product X(i)*Y(i) rounded to double, accumulated in a two-double
// sum, converted back to double at the end). Knuth's TwoSum gives the
// rounding error of each addition exactly; every addition, of a product to
// a thread's sum or of one partial sum to another, is a double-double
// addition renormalised after each step (Dekker 1971), so no error term
// outgrows half an ulp of its leading part. The result is within a small
// multiple of n eps^2 sum|x_i y_i| of the exact sum of the rounded
// products, so it is the same double whatever the grouping (the oracle's
// serial and threaded sums included) unless the exact sum lies that close
// to a rounding boundary.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
// (hi, lo) += p as a double-double addition, renormalised so that
// hi = fl(hi + lo) (the low part never grows past half an ulp of hi)
__device__ __forceinline__ void dd_add(double& hi, double& lo, double p) {
  double s, e;
  two_sum(hi, p, s, e);
  e = __dadd_rn(e, lo);
  hi = __dadd_rn(s, e);
  lo = __dsub_rn(e, __dsub_rn(hi, s));
}
// (hi, lo) += (h2, l2), renormalised so that hi = fl(hi + lo)
__device__ __forceinline__ void dd_merge(double& hi, double& lo, double h2, double l2) {
  double s, e;
  two_sum(hi, h2, s, e);
  e = __dadd_rn(e, __dadd_rn(lo, l2));
  hi = __dadd_rn(s, e);
  lo = __dsub_rn(e, __dsub_rn(hi, s));
}

// Accumulator of K dot products: plain FP64 sums (operands of FP32 loops,
// whose products are exact in FP64), or double-double (FP64 operands).
template <int K>
struct PlainAcc {
  double s[K];
  __device__ __forceinline__ PlainAcc() {
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = 0.0;
  }
  template <class T>
  __device__ __forceinline__ void add(int k, T a, T b) { s[k] += (double)a * (double)b; }
};
template <int K>
struct DDAcc {
  double hi[K], lo[K];
  __device__ __forceinline__ DDAcc() {
#pragma unroll
    for (int k = 0; k < K; k++) { hi[k] = 0.0; lo[k] = 0.0; }
  }
  __device__ __forceinline__ void add(int k, double a, double b) { dd_add(hi[k], lo[k], __dmul_rn(a, b)); }
};
template <int K, class T>
struct DotAccOf { using type = PlainAcc<K>; };
template <int K>
struct DotAccOf<K, double> { using type = DDAcc<K>; };
template <int K, class T>
using DotAcc = typename DotAccOf<K, T>::type;

template <int K, class Fin>
__device__ __forceinline__ void grid_reduce(PlainAcc<K>& v, double* partials, unsigned int* ticket, Fin fin) {
  grid_reduce<K>(v.s, partials, ticket, fin);
}

template <int K>
__device__ __forceinline__ void block_sum_dd(double (&h)[K], double (&l)[K], double* smem /* >= 64*K */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    double a = h[k], b = l[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double a2 = __shfl_down_sync(0xffffffffu, a, o);
      const double b2 = __shfl_down_sync(0xffffffffu, b, o);
      dd_merge(a, b, a2, b2);
    }
    if (lane == 0) {
      smem[wid * 2 * K + k] = a;
      smem[wid * 2 * K + K + k] = b;
    }
  }
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double a = lane < nw ? smem[lane * 2 * K + k] : 0.0;
      double b = lane < nw ? smem[lane * 2 * K + K + k] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double a2 = __shfl_down_sync(0xffffffffu, a, o);
        const double b2 = __shfl_down_sync(0xffffffffu, b, o);
        dd_merge(a, b, a2, b2);
      }
      h[k] = a;  // valid in thread 0
      l[k] = b;
    }
  }
  __syncthreads();
}

// grid_reduce of double-double partials: the same two-level scheme, each
// partial stored as 2K doubles (K high parts, then K low parts); fin gets
// the K sums rounded to double.
template <int K, class Fin>
__device__ __forceinline__ void grid_reduce(DDAcc<K>& v, double* partials, unsigned int* ticket, Fin fin) {
  __shared__ double smem[64 * K];
  __shared__ bool am_last;
  block_sum_dd<K>(v.hi, v.lo, smem);
  const unsigned int G = gridDim.x;
  const unsigned int ngroups = (G + kReduceGroup - 1) / kReduceGroup;
  const unsigned int g = blockIdx.x / kReduceGroup;
  const unsigned int g0 = g * kReduceGroup;
  const unsigned int gsize = min((unsigned int)kReduceGroup, G - g0);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      partials[(size_t)blockIdx.x * 2 * K + k] = v.hi[k];
      partials[(size_t)blockIdx.x * 2 * K + K + k] = v.lo[k];
    }
    __threadfence();
    const unsigned int t = atomicAdd(ticket + 1 + g, 1u);
    am_last = (t == gsize - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double h[K], l[K];
#pragma unroll
  for (int k = 0; k < K; k++) { h[k] = 0.0; l[k] = 0.0; }
  for (unsigned int b = threadIdx.x; b < gsize; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; k++)
      dd_merge(h[k], l[k], __ldcg(partials + (size_t)(g0 + b) * 2 * K + k),
               __ldcg(partials + (size_t)(g0 + b) * 2 * K + K + k));
  }
  block_sum_dd<K>(h, l, smem);
  double* top = partials + (size_t)G * 2 * K;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      top[(size_t)g * 2 * K + k] = h[k];
      top[(size_t)g * 2 * K + K + k] = l[k];
    }
    ticket[1 + g] = 0u;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    am_last = (t == ngroups - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; k++) { h[k] = 0.0; l[k] = 0.0; }
  for (unsigned int b = threadIdx.x; b < ngroups; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; k++)
      dd_merge(h[k], l[k], __ldcg(top + (size_t)b * 2 * K + k), __ldcg(top + (size_t)b * 2 * K + K + k));
  }
  block_sum_dd<K>(h, l, smem);
  if (threadIdx.x == 0) {
    double tot[K];
#pragma unroll
    for (int k = 0; k < K; k++) tot[k] = __dadd_rn(h[k], l[k]);
    fin(tot);
    *ticket = 0u;
  }
}

}  // namespace mb
