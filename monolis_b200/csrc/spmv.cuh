// spmv.cuh -- sliced-ELL block SpMV row kernel and the DIAG block solve,
// shared by the standalone kernels and the fused solver kernels.
#pragma once

#include "common.cuh"
#include "dev.h"

namespace mb {

template <class V>
struct SellView {
  const int* __restrict__ rowptr;
  const long long* __restrict__ slptr;
  const int* __restrict__ col;
  const V* __restrict__ val;
  int N;
};

template <class V>
inline SellView<V> view_of(const SellMatrix& m);
template <>
inline SellView<double> view_of<double>(const SellMatrix& m) {
  return {m.d_rowptr, m.d_slptr, m.d_col, m.d_val64, m.N};
}
template <>
inline SellView<float> view_of<float>(const SellMatrix& m) {
  return {m.d_rowptr, m.d_slptr, m.d_col, m.d_val32, m.N};
}

// y = (A x)[row] for one block row, blocks visited in CSR order. Within a
// block the reference evaluates Y_r = ((Y_r + a_r0*x0) + a_r1*x1) + a_r2*x2
// (src/linalg/matvec.f90:805-823); the FP64 instantiation keeps exactly that
// sequence of roundings. U slots are loaded before any is consumed so that
// each thread keeps U*(B*B + 1) independent loads in flight.
template <int B, int U, class V, class T>
__device__ __forceinline__ void sell_row(const SellView<V>& A, const T* __restrict__ x, int row, T (&y)[B]) {
  constexpr int B2 = B * B;
  const int lane = row & (kSlice - 1);
  const long long base = A.slptr[row >> 5];
  const int len = A.rowptr[row + 1] - A.rowptr[row];
  const int* __restrict__ c = A.col + base + lane;
  const V* __restrict__ v = A.val + base * B2 + lane;
#pragma unroll
  for (int r = 0; r < B; r++) y[r] = T(0);
  int k = 0;
  for (; k + U <= len; k += U) {
    int j[U];
    V a[U][B2];
#pragma unroll
    for (int u = 0; u < U; u++) j[u] = ld_stream(c + (long long)(k + u) * kSlice);
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int e = 0; e < B2; e++) a[u][e] = ld_stream(v + ((long long)(k + u) * B2 + e) * kSlice);
#pragma unroll
    for (int u = 0; u < U; u++) {
      T xs[B];
#pragma unroll
      for (int l = 0; l < B; l++) xs[l] = __ldg(x + (long long)j[u] * B + l);
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int l = 0; l < B; l++) y[r] = add_rn(y[r], mul_rn(T(a[u][r * B + l]), xs[l]));
    }
  }
  for (; k < len; k++) {
    const int jj = ld_stream(c + (long long)k * kSlice);
    V a[B2];
#pragma unroll
    for (int e = 0; e < B2; e++) a[e] = ld_stream(v + ((long long)k * B2 + e) * kSlice);
    T xs[B];
#pragma unroll
    for (int l = 0; l < B; l++) xs[l] = __ldg(x + (long long)jj * B + l);
#pragma unroll
    for (int r = 0; r < B; r++)
#pragma unroll
      for (int l = 0; l < B; l++) y[r] = add_rn(y[r], mul_rn(T(a[r * B + l]), xs[l]));
  }
}

// z = M^-1 v for one block row with the in-place LU factors of the diagonal
// block (entry-major: alu[e*N + row]); order of src/prec/diag/diag_nn.f90:
// 195-229, which for B = 3 is the unrolled sequence of diag_33.f90:121-131.
template <int B, class T>
__device__ __forceinline__ void diag_row(const T* __restrict__ alu, int N, int row, T (&t)[B]) {
  auto L = [&](int j, int k) { return alu[(long long)(j * B + k) * N + row]; };
#pragma unroll
  for (int j = 1; j < B; j++)
#pragma unroll
    for (int k = 0; k < j; k++) t[j] = sub_rn(t[j], mul_rn(L(j, k), t[k]));
#pragma unroll
  for (int j = B - 1; j >= 0; j--) {
#pragma unroll
    for (int k = B - 1; k > j; k--) t[j] = sub_rn(t[j], mul_rn(L(j, k), t[k]));
    t[j] = mul_rn(L(j, j), t[j]);
  }
}

}  // namespace mb
