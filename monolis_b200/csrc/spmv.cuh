// spmv.cuh -- sliced-ELL block SpMV row kernel and the DIAG block solve,
// shared by the standalone kernels and the fused solver kernels.
#pragma once

#include <cstdio>
#include <type_traits>

#include "common.cuh"
#include "dev.h"

namespace mb {

// Gather of the multiplied vector. Kernels that read a vector written by
// other blocks of the same launch (persistent kernels, between barriers)
// must not use the non-coherent read-only path: kCoherent reads through L2.
template <bool kCoherent, class T>
__device__ __forceinline__ T ldx(const T* p) {
  if constexpr (kCoherent) return __ldcg(p);
  else return __ldg(p);
}

template <class V>
struct SellView {
  const int* __restrict__ rowptr;
  const long long* __restrict__ slc;  // slice offset, bit 0 set: 32-bit column ids
  const int* __restrict__ col;
  const short* __restrict__ col16;
  const int* __restrict__ cbase;
  const V* __restrict__ val;
  int N;
};

template <class V>
inline SellView<V> view_of(const SellMatrix& m);
template <>
inline SellView<double> view_of<double>(const SellMatrix& m) {
  return {m.d_rowptr, m.d_slc, m.d_col, m.d_col16, m.d_cbase, m.d_val64, m.N};
}

// Column ids of slots k .. k+n-1 (n <= U) of one lane: 32-bit ids (wide
// slice), base + lane (uniform slice: every difference is zero and the
// difference stream is not read) or base + lane + 16-bit difference. The
// branch is uniform over the warp (one slice).
template <int U>
__device__ __forceinline__ void load_cols(bool wide, bool uniform, const int* __restrict__ c,
                                          const short* __restrict__ c16, const int* __restrict__ cb, int lane, int k,
                                          int n, int (&j)[U]) {
  if (wide) {
#pragma unroll
    for (int u = 0; u < U; u++) j[u] = u < n ? ld_stream(c + (long long)(k + u) * kSlice) : 0;
  } else if (uniform) {
#pragma unroll
    for (int u = 0; u < U; u++) j[u] = u < n ? __ldg(cb + k + u) + lane : 0;
  } else {
#pragma unroll
    for (int u = 0; u < U; u++)
      j[u] = u < n ? __ldg(cb + k + u) + lane + (int)ld_stream(c16 + (long long)(k + u) * kSlice) : 0;
  }
}

// y = (A x)[row] for one block row, blocks visited in CSR order. Within a
// block the reference evaluates Y_r = ((Y_r + a_r0*x0) + a_r1*x1) + a_r2*x2
// (src/linalg/matvec.f90:805-823); the FP64 instantiation keeps exactly that
// sequence of roundings. U slots are loaded before any is consumed so that
// each thread keeps U*(B*B + 1) independent loads in flight.
// xf(i) gives entry i = column*B + l of the multiplied vector. kCols16 =
// false reads the 32-bit column ids of every slice.
template <int B, int U, class V, class T, bool kCols16 = true, class XF>
__device__ __forceinline__ void sell_row_f(const SellView<V>& A, const XF xf, int row, T (&y)[B]) {
  constexpr int B2 = B * B;
  const int lane = row & (kSlice - 1);
  const long long sc = A.slc[row >> 5];
  const long long base = sc & ~3LL;
  const bool wide = !kCols16 || (sc & 1);
  const bool uni = (sc & 2) != 0;
  const int len = A.rowptr[row + 1] - A.rowptr[row];
  const int* __restrict__ c = A.col + base + lane;
  const short* __restrict__ c16 = A.col16 + base + lane;
  const int* __restrict__ cb = A.cbase + (base >> 5);
  const V* __restrict__ v = A.val + base * B2 + lane;
#pragma unroll
  for (int r = 0; r < B; r++) y[r] = T(0);
  int k = 0;
  for (; k + U <= len; k += U) {
    int j[U];
    V a[U][B2];
    load_cols<U>(wide, uni, c, c16, cb, lane, k, U, j);
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int e = 0; e < B2; e++) a[u][e] = ld_stream(v + ((long long)(k + u) * B2 + e) * kSlice);
#pragma unroll
    for (int u = 0; u < U; u++) {
      T xs[B];
#pragma unroll
      for (int l = 0; l < B; l++) xs[l] = xf((long long)j[u] * B + l);
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int l = 0; l < B; l++) y[r] = add_rn(y[r], mul_rn(T(a[u][r * B + l]), xs[l]));
    }
  }
  // the last, partial chunk: its loads are issued together (predicated; slots
  // past the row end are not read) and only the row's slots are added, in order
  const int rem = len - k;
  if (U > 1 && rem > 0) {
    int j[U];
    V a[U][B2];
    load_cols<U>(wide, uni, c, c16, cb, lane, k, rem, j);
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int e = 0; e < B2; e++) a[u][e] = u < rem ? ld_stream(v + ((long long)(k + u) * B2 + e) * kSlice) : V(0);
    T xs[U][B];
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int l = 0; l < B; l++) xs[u][l] = u < rem ? xf((long long)j[u] * B + l) : T(0);
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (u >= rem) break;
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int l = 0; l < B; l++) y[r] = add_rn(y[r], mul_rn(T(a[u][r * B + l]), xs[u][l]));
    }
  }
}

template <int B, int U, class V, class T, bool kCoherent = false>
__device__ __forceinline__ void sell_row(const SellView<V>& A, const T* __restrict__ x, int row, T (&y)[B]) {
  sell_row_f<B, U, V, T>(A, [&](long long i) { return ldx<kCoherent>(x + i); }, row, y);
}

// Paired FP32 layout (see SellMatrix::d_col2): thread t owns rows 2t and
// 2t+1 of the matrix; slot k of its pair is at block slptr2[t/32] + 64k + 2(t%32).
struct SellView2 {
  const int* __restrict__ rowptr;
  const long long* __restrict__ slc2;  // slice offset, bit 0 set: 32-bit column ids
  const int* __restrict__ col2;
  const short* __restrict__ col16p;
  const int* __restrict__ cbase2;
  const float* __restrict__ val;
  int N;
};

inline SellView2 view2_of(const SellMatrix& m) {
  return {m.d_rowptr, m.d_slc2, m.d_col2, m.d_col16p, m.d_cbase2, m.d_val32, m.N};
}

__device__ __forceinline__ float2 ld_stream2(const float2* p) { return __ldcs(p); }
__device__ __forceinline__ int2 ld_stream2(const int2* p) { return __ldcs(p); }
__device__ __forceinline__ short2 ld_stream2(const short2* p) { return __ldcs(p); }

// Column ids of slots k .. k+n-1 of a row pair (paired layout).
template <int U>
__device__ __forceinline__ void load_cols2(bool wide, bool uniform, const int2* __restrict__ c,
                                           const short2* __restrict__ c16, const int* __restrict__ cb, int lane2,
                                           int k, int n, int2 (&j)[U]) {
  if (wide) {
#pragma unroll
    for (int u = 0; u < U; u++) j[u] = u < n ? ld_stream2(c + (long long)(k + u) * 32) : make_int2(0, 0);
  } else if (uniform) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int b = u < n ? __ldg(cb + k + u) + lane2 : 0;
      j[u] = make_int2(b, b + 1);
    }
  } else {
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (u < n) {
        const int b = __ldg(cb + k + u) + lane2;
        const short2 d = ld_stream2(c16 + (long long)(k + u) * 32);
        j[u] = make_int2(b + d.x, b + 1 + d.y);
      } else {
        j[u] = make_int2(0, 0);
      }
    }
  }
}

// y0/y1 = (A x) of rows 2t and 2t+1 in FP32 (fused multiply-add). Slots past
// a row's length hold zero values and a valid column, so both rows run to the
// longer length.
// The entries of the multiplied vector come from xf(i) (i = column*B + l):
// a plain gather, or a value computed from other vectors (see sell_row2).
template <int B, int U, bool kCols16 = true, class XF>
__device__ __forceinline__ void sell_row2_f(const SellView2& A, const XF xf, int t, float (&y0)[B], float (&y1)[B]) {
  constexpr int B2 = B * B;
  const int r0 = 2 * t;
  const int lane2 = 2 * (t & 31);
  const long long sc = A.slc2[t >> 5];
  const long long base = sc & ~3LL;
  const bool wide = !kCols16 || (sc & 1);
  const bool uni = (sc & 2) != 0;
  const int len0 = A.rowptr[r0 + 1] - A.rowptr[r0];
  const int len1 = (r0 + 1 < A.N) ? A.rowptr[r0 + 2] - A.rowptr[r0 + 1] : 0;
  const int len = len0 > len1 ? len0 : len1;
  const int2* __restrict__ c = reinterpret_cast<const int2*>(A.col2 + base + lane2);
  const short2* __restrict__ c16 = reinterpret_cast<const short2*>(A.col16p + base + lane2);
  const int* __restrict__ cb = A.cbase2 + (base >> 6);
  const float2* __restrict__ v = reinterpret_cast<const float2*>(A.val + base * B2 + lane2);
#pragma unroll
  for (int r = 0; r < B; r++) { y0[r] = 0.f; y1[r] = 0.f; }
  int k = 0;
  for (; k + U <= len; k += U) {
    int2 j[U];
    float2 a[U][B2];
    load_cols2<U>(wide, uni, c, c16, cb, lane2, k, U, j);
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int e = 0; e < B2; e++) a[u][e] = ld_stream2(v + ((long long)(k + u) * B2 + e) * 32);
#pragma unroll
    for (int u = 0; u < U; u++) {
      float x0[B], x1[B];
#pragma unroll
      for (int l = 0; l < B; l++) {
        x0[l] = xf((long long)j[u].x * B + l);
        x1[l] = xf((long long)j[u].y * B + l);
      }
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int l = 0; l < B; l++) {
          y0[r] = fmaf(a[u][r * B + l].x, x0[l], y0[r]);
          y1[r] = fmaf(a[u][r * B + l].y, x1[l], y1[r]);
        }
    }
  }
  // the last, partial chunk: loads issued together, slots past the end not read
  const int rem = len - k;
  if (rem > 0) {
    int2 j[U];
    float2 a[U][B2];
    load_cols2<U>(wide, uni, c, c16, cb, lane2, k, rem, j);
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int e = 0; e < B2; e++)
        a[u][e] = u < rem ? ld_stream2(v + ((long long)(k + u) * B2 + e) * 32) : make_float2(0.f, 0.f);
    float x0[U][B], x1[U][B];
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int l = 0; l < B; l++) {
        x0[u][l] = u < rem ? xf((long long)j[u].x * B + l) : 0.f;
        x1[u][l] = u < rem ? xf((long long)j[u].y * B + l) : 0.f;
      }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (u >= rem) break;
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int l = 0; l < B; l++) {
          y0[r] = fmaf(a[u][r * B + l].x, x0[u][l], y0[r]);
          y1[r] = fmaf(a[u][r * B + l].y, x1[u][l], y1[r]);
        }
    }
  }
}

// Two row pairs of the paired layout at once (1x1 blocks): pairs ta and tb
// (tb skipped when !hb) advance slot by slot together, U slots of each in
// flight, so a thread keeps both pairs' loads in flight at once. Each row
// adds its slots in the order of sell_row2_f, with the same results.
template <int U, bool kCols16, class XF>
__device__ __forceinline__ void sell_row2_two(const SellView2& A, const XF xf, int ta, int tb, bool hb,
                                              float (&ya)[2], float (&yb)[2]) {
  const int tt[2] = {ta, tb};
  const int2* __restrict__ c[2];
  const short2* __restrict__ c16[2];
  const int* __restrict__ cb[2];
  const float2* __restrict__ v[2];
  bool wide[2], uni[2];
  int len[2], lane2[2];
#pragma unroll
  for (int p = 0; p < 2; p++) {
    const int t = tt[p];
    const long long sc = A.slc2[t >> 5];
    const long long base = sc & ~3LL;
    wide[p] = !kCols16 || (sc & 1);
    uni[p] = (sc & 2) != 0;
    lane2[p] = 2 * (t & 31);
    const int r0 = 2 * t;
    const int l0 = A.rowptr[r0 + 1] - A.rowptr[r0];
    const int l1 = (r0 + 1 < A.N) ? A.rowptr[r0 + 2] - A.rowptr[r0 + 1] : 0;
    len[p] = (p == 0 || hb) ? (l0 > l1 ? l0 : l1) : 0;
    c[p] = reinterpret_cast<const int2*>(A.col2 + base + lane2[p]);
    c16[p] = reinterpret_cast<const short2*>(A.col16p + base + lane2[p]);
    cb[p] = A.cbase2 + (base >> 6);
    v[p] = reinterpret_cast<const float2*>(A.val + base + lane2[p]);
  }
  float y[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
  const int lmax = len[0] > len[1] ? len[0] : len[1];
  for (int k = 0; k < lmax; k += U) {
    int2 j[2][U];
    float2 a[2][U];
    float x0[2][U], x1[2][U];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      const int n = len[p] - k;
      load_cols2<U>(wide[p], uni[p], c[p], c16[p], cb[p], lane2[p], k, n, j[p]);
#pragma unroll
      for (int u = 0; u < U; u++) a[p][u] = u < n ? ld_stream2(v[p] + (long long)(k + u) * 32) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int p = 0; p < 2; p++)
#pragma unroll
      for (int u = 0; u < U; u++) {
        const bool in = u < len[p] - k;
        x0[p][u] = in ? xf((long long)j[p][u].x) : 0.f;
        x1[p][u] = in ? xf((long long)j[p][u].y) : 0.f;
      }
#pragma unroll
    for (int p = 0; p < 2; p++)
#pragma unroll
      for (int u = 0; u < U; u++)
        if (u < len[p] - k) {
          y[p][0] = fmaf(a[p][u].x, x0[p][u], y[p][0]);
          y[p][1] = fmaf(a[p][u].y, x1[p][u], y[p][1]);
        }
  }
  ya[0] = y[0][0];
  ya[1] = y[0][1];
  yb[0] = y[1][0];
  yb[1] = y[1][1];
}

template <int B, int U, bool kCoherent = false, bool kCols16 = true>
__device__ __forceinline__ void sell_row2(const SellView2& A, const float* __restrict__ x, int t, float (&y0)[B],
                                          float (&y1)[B]) {
  sell_row2_f<B, U, kCols16>(A, [&](long long i) { return ldx<kCoherent>(x + i); }, t, y0, y1);
}

// 16-byte vector type of an element type.
template <class T>
struct Vec16T;
template <>
struct Vec16T<float> {
  using type = float4;
  static constexpr int n = 4;
};
template <>
struct Vec16T<double> {
  using type = double2;
  static constexpr int n = 2;
};

constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }

// Register blocking of an interleaved vector x[row*B + c]: a thread owns R
// consecutive block rows, E = R*B elements, a whole number of 16-byte words
// (R = W / gcd(B, W) with W elements per word), so it moves them with E/W
// aligned vector accesses.
template <class T, int B>
struct RowGroup {
  static constexpr int W = Vec16T<T>::n;
  static constexpr int R = W / gcd_c(B, W);
  static constexpr int E = R * B;
};

template <class T, int E>
__device__ __forceinline__ void vload(const T* __restrict__ p, T (&v)[E]) {
  using V = typename Vec16T<T>::type;
  constexpr int W = Vec16T<T>::n;
#pragma unroll
  for (int i = 0; i < E / W; i++) {
    const V t = reinterpret_cast<const V*>(p)[i];
    const T* e = reinterpret_cast<const T*>(&t);
#pragma unroll
    for (int k = 0; k < W; k++) v[i * W + k] = e[k];
  }
}
template <class T, int E>
__device__ __forceinline__ void vstore(T* __restrict__ p, const T (&v)[E]) {
  using V = typename Vec16T<T>::type;
  constexpr int W = Vec16T<T>::n;
#pragma unroll
  for (int i = 0; i < E / W; i++) {
    V t;
    T* e = reinterpret_cast<T*>(&t);
#pragma unroll
    for (int k = 0; k < W; k++) e[k] = v[i * W + k];
    reinterpret_cast<V*>(p)[i] = t;
  }
}

// In-place LU solve of one B x B diagonal block with the factors in L
// (row-major), order of src/prec/diag/diag_nn.f90:195-229 (for B = 3 the
// unrolled sequence of diag_33.f90:121-131).
template <int B, class T, class F>
__device__ __forceinline__ void diag_solve(F L, T (&t)[B]) {
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

// Factors of R consecutive rows, entry-major storage alu[e*N + row]: one
// vector load per entry when R words fill 16 bytes and N keeps them aligned.
template <class T, int B, int R>
__device__ __forceinline__ void load_alu_rows(const T* __restrict__ alu, int N, long long row0, bool vec_ok,
                                              T (&L)[B * B][R]) {
#pragma unroll
  for (int e = 0; e < B * B; e++) {
    const T* src = alu + (long long)e * N + row0;
    if constexpr (R * sizeof(T) == 16) {
      if (vec_ok) {
        T v[R];
        vload<T, R>(src, v);
#pragma unroll
        for (int k = 0; k < R; k++) L[e][k] = v[k];
        continue;
      }
    }
#pragma unroll
    for (int k = 0; k < R; k++) L[e][k] = src[k];
  }
}

// z = M^-1 v for one block row with the in-place LU factors of the diagonal
// block (entry-major: alu[e*N + row]); order of src/prec/diag/diag_nn.f90:
// 195-229, which for B = 3 is the unrolled sequence of diag_33.f90:121-131.
template <int B, class T>
__device__ __forceinline__ void diag_row(const T* __restrict__ alu, int N, int row, T (&t)[B]) {
  diag_solve<B, T>([&](int j, int k) { return alu[(long long)(j * B + k) * N + row]; }, t);
}

// Per-row DIAG apply of E = R*B values held in registers (R rows of B).
template <int B, class T, int R>
__device__ __forceinline__ void diag_rows(const T* __restrict__ alu, int N, long long row0, bool alu_vec,
                                          T (&w)[R * B]) {
  T L[B * B][R];
  load_alu_rows<T, B, R>(alu, N, row0, alu_vec, L);
#pragma unroll
  for (int k = 0; k < R; k++) {
    T t[B];
#pragma unroll
    for (int c = 0; c < B; c++) t[c] = w[k * B + c];
    diag_solve<B, T>([&](int j, int kk) { return L[j * B + kk][k]; }, t);
#pragma unroll
    for (int c = 0; c < B; c++) w[k * B + c] = t[c];
  }
}

// Resident blocks of 256 threads per SM that the SpMV kernels are compiled
// for. With 1x1 blocks a row has few slots and the kernels are bound by
// memory latency, not bandwidth: at 256^3 (7 entries a row) six blocks per
// SM (40 registers) stream the FP64 SELL matrix at 5.7 TB/s where four
// (56-64 registers) reach 4.9 TB/s, with the same per-row order and bits.
// Larger blocks keep the compiler's choice.
template <int B>
struct SpmvMinBlocks {
  static constexpr int value = B == 1 ? 6 : 1;
};
// The same for the FP32 kernels of the paired layout, where a thread carries
// two rows: at 1x1 blocks five resident blocks (48 registers, no spills)
// beat six (40, about 100 bytes of spills a thread at 8 slots in flight) in
// BiCGSTAB at 256^3: V = A PT 172 -> 167 us, T = A ST 177 -> 168 us; four
// (64 registers) were slower (184 us).
template <int B>
struct SpmvMinBlocks2 {
  static constexpr int value = B == 1 ? 5 : 1;
};

// Compile-time block size and unroll depth from their runtime values.
template <class F>
inline int dispatch_ndof(int ndof, F&& f) {
  switch (ndof) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    default:
      fprintf(stderr, "** monolis_b200: NDOF=%d is not supported on the device (1..6)\n", ndof);
      return kBadInput;
  }
}

template <class F>
inline int dispatch_u(int u, F&& f) {
  switch (u) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 8: return f(std::integral_constant<int, 8>{});
    default: return f(std::integral_constant<int, 2>{});
  }
}

// Unroll depth actually used for block size B: deep unrolls (4, 8 slots in
// flight) only for 1x1 blocks, where a row has few slots and registers are
// plentiful; 2x2 and 3x3 blocks stop at 3, larger blocks at 1.
constexpr int eff_u(int B, int u) { return B >= 4 ? 1 : (B >= 2 && u > 3 ? 3 : u); }

}  // namespace mb
