// multi.cu -- many right-hand sides on one matrix: CG (+ DIAG) for up to 32
// right-hand sides at once in one persistent kernel.
//
// Layout: the right-hand sides of a block row are interleaved, v[(row*B + c)*K
// + k] for right-hand side k < K <= 32, so that a warp owns one block row and
// lane k works on right-hand side k: every vector access of the warp is one
// contiguous line, and the matrix row (CSR, read once for all K) is loaded
// cooperatively by the lanes and broadcast with shuffles. One warp keeps the
// same rows in every phase, so a thread only ever reads back the entries it
// wrote itself; values of other rows (the SpMV gathers) are read through L2.
//
// The kernel is launched cooperatively (all blocks resident) and separates
// its phases with a grid barrier whose last arriving block also sums the
// per-block partial dot products (block order: deterministic) and updates the
// per-right-hand-side scalars before releasing the others. Each barrier wait
// is bounded: past the limit a block records an error and every block leaves.
// Two barriers per iteration: the search direction p = z + beta p is formed
// inside the SpMV (own rows written to the other p buffer, neighbours' values
// recomputed from z and the old p), so no separate pass and barrier for p.
//
// Right-hand sides converge independently: a converged one is masked out
// (its lane idles), the others continue. FP32 (refine = 1): FP32 matrix and
// vectors in the loop, FP64 dots and scalars, FP64 solution x + y with
// reliable updates r = b - A (x + y) in FP64; FP64: the same loop in double.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "monolis_b200.h"
#include "spmv.cuh"

namespace mb {
namespace {

constexpr int kMultiK = 32;
constexpr int kMultiThreads = 256;
// default bound of every barrier wait: polls of an L2 round trip + 32 ns each, seconds in all
constexpr unsigned long long kSpinLimit = 1ull << 22;

constexpr int kBarrierGroup = 32;  // blocks per first-level group of the barrier
constexpr int kMaxGroups = 128;

constexpr int kLine = 32;  // words per 128-byte line: every counter and flag gets its own

struct MultiCtl {
  alignas(128) unsigned int count;  // groups finished (global arrival)
  alignas(128) unsigned int gen;    // global release generation
  alignas(128) int err;
  int all_done, any_refresh, it;
  alignas(128) unsigned int gcount[kMaxGroups * kLine];  // blocks arrived, per group
  alignas(128) unsigned int grel[kMaxGroups * kLine];    // release generation, per group
  double rho[kMultiK], rho1[kMultiK], alpha[kMultiK], beta[kMultiK], B2[kMultiK], rmax[kMultiK], resid[kMultiK];
  int iter[kMultiK], done[kMultiK], status[kMultiK], refresh[kMultiK], fold[kMultiK], nref[kMultiK];
};

template <class T>
struct MultiArgs {
  int N, K, prec, refine, max_iter;
  double tol, delta;
  const int* rowptr;
  const int* col;      // 0-based
  const T* val;        // CSR values in the loop precision
  const double* val64;  // CSR values, FP64 (residual refresh)
  const T* alu;        // DIAG factors, entry-major alu[e*N + row]
  const double* b;
  double* x;
  T *y, *r, *z, *p0, *p1, *q;
  double* partials;    // [gridDim.x][2][32]
  MultiCtl* ctl;
  unsigned long long spin_limit;  // polls before a barrier wait gives up
  unsigned int delay_ns;          // testing: block 0 arrives this much later at the first barrier
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier of a cooperative launch, with an optional reduction of the
// per-block partial sums (2 x 32 doubles per block, partials[block][64]).
// Blocks arrive in groups of kBarrierGroup: the last block of a group sums
// the group's partials in block order (group sums after the block partials),
// the last group finisher sums the group sums in group order into tot and
// runs `last` (with all its threads) before releasing everyone. Each block
// adds at most one group's worth of values, so the barrier's tail stays short.
// Waits are bounded; returns false once any block has given up.
template <class F>
__device__ bool grid_sync(MultiCtl* c, double* partials, bool reduce, double (*tot)[kMultiK],
                          unsigned long long limit, F&& last) {
  __shared__ unsigned int s_grel, s_gen;
  __shared__ int s_role, s_ok;  // 0: wait for the group, 1: group finisher, 2: last block
  const unsigned int G = gridDim.x, g = blockIdx.x / kBarrierGroup;
  const unsigned int ngroups = (G + kBarrierGroup - 1) / kBarrierGroup;
  const unsigned int g0 = g * kBarrierGroup, gsize = min((unsigned int)kBarrierGroup, G - g0);
  unsigned int* gcount = c->gcount + g * kLine;
  unsigned int* grel = c->grel + g * kLine;
  double* gpart = partials + (size_t)G * 2 * kMultiK;
  __syncthreads();
  if (threadIdx.x == 0) {
    s_grel = ld_acquire(grel);
    s_gen = ld_acquire(&c->gen);
    __threadfence();
    s_role = atomicAdd(gcount, 1u) == gsize - 1 ? 1 : 0;
  }
  __syncthreads();
  if (s_role == 1) {
    __threadfence();
    if (reduce && threadIdx.x < 2 * kMultiK) {
      double s = 0.0;
#pragma unroll 8
      for (unsigned int b = 0; b < gsize; b++) s += __ldcg(partials + (size_t)(g0 + b) * 2 * kMultiK + threadIdx.x);
      gpart[(size_t)g * 2 * kMultiK + threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      *gcount = 0u;
      __threadfence();
      if (atomicAdd(&c->count, 1u) == ngroups - 1) s_role = 2;
    }
    __syncthreads();
    if (s_role == 2) {
      __threadfence();
      if (reduce) {
        if (threadIdx.x < 2 * kMultiK) {
          double t = 0.0;
#pragma unroll 8
          for (unsigned int q = 0; q < ngroups; q++) t += __ldcg(gpart + (size_t)q * 2 * kMultiK + threadIdx.x);
          tot[threadIdx.x >> 5][threadIdx.x & 31] = t;
        }
        __syncthreads();
      }
      last();
      __syncthreads();
      if (threadIdx.x == 0) {
        c->count = 0u;
        __threadfence();
        st_release(&c->gen, s_gen + 1u);
      }
    } else if (threadIdx.x == 0) {
      // group finisher: wait for the global release (at most ngroups pollers)
      unsigned long long n = 0;
      while (ld_acquire(&c->gen) == s_gen) {
        if (++n > limit) {
          atomicExch(&c->err, 1);
          break;
        }
        __nanosleep(32);
      }
      __threadfence();
    }
    if (threadIdx.x == 0) st_release(grel, s_grel + 1u);  // release this group
  } else if (threadIdx.x == 0) {
    // wait for this group's release (at most kBarrierGroup pollers per line)
    unsigned long long n = 0;
    while (ld_acquire(grel) == s_grel) {
      if (++n > limit) {
        atomicExch(&c->err, 1);
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
  }
  if (threadIdx.x == 0) s_ok = __ldcg(&c->err) == 0;
  __syncthreads();
  return s_ok != 0;
}

template <class T>
__device__ __forceinline__ T fmat(T a, T b, T c);
template <>
__device__ __forceinline__ float fmat<float>(float a, float b, float c) { return fmaf(a, b, c); }
template <>
__device__ __forceinline__ double fmat<double>(double a, double b, double c) { return fma(a, b, c); }

// Four consecutive right-hand sides of one vector entry: one 16-byte access
// for FP32, two for FP64; kCoherent reads through L2 (values written by other
// blocks of this launch).
template <bool kCoherent, class T>
__device__ __forceinline__ void ld4(const T* p, T (&o)[4]);
template <bool kCoherent>
__device__ __forceinline__ void ld4(const float* p, float (&o)[4]) {
  const float4 v = kCoherent ? __ldcg(reinterpret_cast<const float4*>(p)) : *reinterpret_cast<const float4*>(p);
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <bool kCoherent>
__device__ __forceinline__ void ld4(const double* p, double (&o)[4]) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 a = kCoherent ? __ldcg(q) : q[0];
  const double2 b = kCoherent ? __ldcg(q + 1) : q[1];
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const float (&o)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&o)[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(o[0], o[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(o[2], o[3]);
}

// The kernel. A group of Q lanes owns one block row (a warp works on 32/Q rows
// at once) and lane q of the group carries right-hand sides 4q..4q+3, so every
// vector access of a thread is 16 bytes (K is padded to Kp = 4Q; padded
// right-hand sides are zero and start converged). The row's matrix entries are
// loaded by the group's lanes, Q at a time, and broadcast with width-Q
// shuffles; all loops that contain shuffles run to warp-uniform bounds.
// Small blocks are held to few registers (4 blocks of FP32, 3 of FP64 per
// SM) so that enough loads are in flight for HBM bandwidth.
template <int B, class T, int Q>
__global__ void __launch_bounds__(kMultiThreads, B <= 2 ? (sizeof(T) == 4 ? 4 : 3) : 1)
    multi_cg_kernel(const MultiArgs<T> a) {
  constexpr int B2 = B * B;
  constexpr int Kp = 4 * Q;
  constexpr int RPW = 32 / Q;  // rows per warp
  const int* __restrict__ rowptr = a.rowptr;
  const int* __restrict__ colv = a.col;
  const T* __restrict__ val = a.val;
  const double* __restrict__ val64 = a.val64;
  const T* __restrict__ alu = a.alu;
  const double* __restrict__ bv = a.b;
  double* __restrict__ xv = a.x;
  T* __restrict__ yv = a.y;
  T* __restrict__ rv = a.r;
  T* __restrict__ zv = a.z;
  T* __restrict__ qv = a.q;
  __shared__ double s_red[kMultiThreads / 32][2][kMultiK];
  __shared__ double s_tot[2][kMultiK];
  __shared__ int s_flag[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int qd = lane & (Q - 1);  // quad of right-hand sides
  const int g = lane / Q;         // row slot within the warp
  const long long wrow0 = ((long long)blockIdx.x * nw + warp) * RPW;  // first row of this warp
  const long long sweep = (long long)gridDim.x * nw * RPW;
  const long long N = a.N;
  const int K = a.K;
  MultiCtl* c = a.ctl;
  // the last block of a barrier reads and writes the scalars through a
  // volatile view (L1 is not coherent across SMs); the others use __ldcg
  volatile MultiCtl* vc = c;
  auto at = [&](long long row, int comp) { return (row * B + comp) * Kp + 4 * qd; };
  auto warp_max = [](int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
  };
  // per-thread sums of its 4 right-hand sides -> partials of the block
  auto reduce_write = [&](const double (&v0)[4], const double (&v1)[4]) {
    double w0[4], w1[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      w0[j] = v0[j];
      w1[j] = v1[j];
#pragma unroll
      for (int o = Q; o < 32; o <<= 1) {
        w0[j] += __shfl_xor_sync(0xffffffffu, w0[j], o);
        w1[j] += __shfl_xor_sync(0xffffffffu, w1[j], o);
      }
    }
    if (lane < Q)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        s_red[warp][0][4 * lane + j] = w0[j];
        s_red[warp][1][4 * lane + j] = w1[j];
      }
    __syncthreads();
    if (threadIdx.x < 2 * kMultiK) {
      const int which = threadIdx.x >> 5, kk = threadIdx.x & 31;
      double sum = 0.0;
      if (kk < Kp)
        for (int i = 0; i < nw; i++) sum += s_red[i][which][kk];
      a.partials[((size_t)blockIdx.x * 2 + which) * kMultiK + kk] = sum;
    }
  };
  auto live4 = [&](bool (&lv)[4]) {
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = 4 * qd + j;
      lv[j] = k < K && __ldcg(&c->done[k]) == 0;
    }
  };

  // x = y = 0 on the own rows
  for (long long rb = wrow0; rb < N; rb += sweep) {
    const long long row = rb + g;
    if (row < N)
#pragma unroll
      for (int cc = 0; cc < B; cc++) {
        const double z4[4] = {0.0, 0.0, 0.0, 0.0};
        const T t4[4] = {T(0), T(0), T(0), T(0)};
        st4(xv + at(row, cc), z4);
        st4(yv + at(row, cc), t4);
      }
  }

  // r = b - A (x + y) in FP64, z = M^-1 r, for the right-hand sides with
  // mine[j]; partial sums <r,r>, <r,z> written per block
  auto refresh = [&](const bool (&mine)[4]) {
    double v0[4] = {0.0, 0.0, 0.0, 0.0}, v1[4] = {0.0, 0.0, 0.0, 0.0};
    const bool any = mine[0] || mine[1] || mine[2] || mine[3];
    for (long long rb = wrow0; rb < N; rb += sweep) {
      const long long row = rb + g;
      const bool valid = row < N;
      const int k0 = valid ? rowptr[row] : 0;
      const int len = valid ? rowptr[row + 1] - k0 : 0;
      const int mlen = warp_max(len);
      double ax[B][4];
#pragma unroll
      for (int cc = 0; cc < B; cc++)
#pragma unroll
        for (int j = 0; j < 4; j++) ax[cc][j] = 0.0;
      for (int base = 0; base < mlen; base += Q) {
        const bool has = base + qd < len;
        const int cj = has ? colv[k0 + base + qd] : 0;
        double vv[B2];
#pragma unroll
        for (int e = 0; e < B2; e++) vv[e] = has ? val64[(long long)(k0 + base + qd) * B2 + e] : 0.0;
#pragma unroll
        for (int u = 0; u < Q; u++) {
          const int j = __shfl_sync(0xffffffffu, cj, u, Q);
          double ae[B2];
#pragma unroll
          for (int e = 0; e < B2; e++) ae[e] = __shfl_sync(0xffffffffu, vv[e], u, Q);
          if (base + u < len && any) {
#pragma unroll
            for (int l = 0; l < B; l++) {
              const long long ij = ((long long)j * B + l) * Kp + 4 * qd;
              double x4[4];
              T y4[4];
              ld4<true>(xv + ij, x4);
              ld4<true>(yv + ij, y4);
#pragma unroll
              for (int rr = 0; rr < B; rr++)
#pragma unroll
                for (int jj = 0; jj < 4; jj++) ax[rr][jj] = fma(ae[rr * B + l], x4[jj] + (double)y4[jj], ax[rr][jj]);
            }
          }
        }
      }
      if (valid && any) {
        double b4[B][4];
        T t[B][4], w[B][4];
#pragma unroll
        for (int cc = 0; cc < B; cc++) {
          const long long i = at(row, cc);
          double bb[4];
          ld4<false>(bv + i, bb);
          T r4[4], z4[4];
          ld4<false>(rv + i, r4);
          ld4<false>(zv + i, z4);
#pragma unroll
          for (int j = 0; j < 4; j++) {
            b4[cc][j] = bb[j] - ax[cc][j];
            t[cc][j] = mine[j] ? (T)b4[cc][j] : r4[j];
            w[cc][j] = mine[j] ? t[cc][j] : z4[j];
          }
        }
        if (a.prec) {
#pragma unroll
          for (int j = 0; j < 4; j++) {
            if (!mine[j]) continue;
            T wj[B];
#pragma unroll
            for (int cc = 0; cc < B; cc++) wj[cc] = t[cc][j];
            diag_row<B, T>(alu, a.N, (int)row, wj);
#pragma unroll
            for (int cc = 0; cc < B; cc++) w[cc][j] = wj[cc];
          }
        }
#pragma unroll
        for (int cc = 0; cc < B; cc++) {
          st4(rv + at(row, cc), t[cc]);
          st4(zv + at(row, cc), w[cc]);
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (mine[j]) {
              v0[j] += b4[cc][j] * b4[cc][j];
              v1[j] += (double)t[cc][j] * (double)w[cc][j];
            }
        }
      }
    }
    reduce_write(v0, v1);
  };

  // testing: block 0 late at the first barrier (bounded sleep), so that the
  // other blocks' waits run out when the limit is shorter
  if (a.delay_ns && blockIdx.x == 0 && threadIdx.x == 0) {
    for (unsigned int t = 0; t < a.delay_ns; t += 1000) __nanosleep(1000);
  }
  // the whole grid has zeroed its x and y before any residual reads them
  if (!grid_sync(c, a.partials, false, s_tot, a.spin_limit, [] {})) return;
  {
    bool all[4];
#pragma unroll
    for (int j = 0; j < 4; j++) all[j] = 4 * qd + j < K;
    refresh(all);
  }
  if (!grid_sync(c, a.partials, true, s_tot, a.spin_limit, [&] {
        if (threadIdx.x < kMultiK) {
          const int kk = threadIdx.x;
          const double rr = s_tot[0][kk], rz = s_tot[1][kk];
          vc->B2[kk] = rr;
          vc->iter[kk] = 0;
          vc->nref[kk] = 0;
          vc->fold[kk] = 0;
          vc->refresh[kk] = 0;
          vc->resid[kk] = 0.0;
          if (kk >= K || !(rr > 0.0) || !isfinite(rr)) {
            vc->done[kk] = 1;  // B2 == 0: x = 0 solves it (also the padding)
            vc->status[kk] = (kk >= K || isfinite(rr)) ? MONOLIS_B200_OK : MONOLIS_B200_NONFINITE;
          } else {
            vc->done[kk] = 0;
            vc->status[kk] = MONOLIS_B200_OK;
            vc->rho[kk] = rz;
            vc->rmax[kk] = sqrt(rr);
          }
        }
        if (threadIdx.x == 0) vc->it = 1;
      }))
    return;

  T* pold = a.p0;
  T* pnew = a.p1;
  for (;;) {
    bool live[4];
    live4(live);
    const bool any = live[0] || live[1] || live[2] || live[3];
    const bool first = __ldcg(&c->it) == 1;
    T beta[4];
    bool fold[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = 4 * qd + j;
      beta[j] = k < K ? (T)__ldcg(&c->beta[k]) : T(0);
      fold[j] = k < K && __ldcg(&c->fold[k]) != 0;
    }
    // P = Z + beta P (own rows, to pnew); Q = A P with the neighbours' P
    // recomputed from Z and the old P; <P,Q>
    double pq[4] = {0.0, 0.0, 0.0, 0.0}, zero4[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long rb = wrow0; rb < N; rb += sweep) {
      const long long row = rb + g;
      const bool valid = row < N;
      const int k0 = valid ? rowptr[row] : 0;
      const int len = valid ? rowptr[row + 1] - k0 : 0;
      const int mlen = warp_max(len);
      T acc[B][4];
#pragma unroll
      for (int cc = 0; cc < B; cc++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[cc][j] = T(0);
      for (int base = 0; base < mlen; base += Q) {
        const bool has = base + qd < len;
        const int cj = has ? colv[k0 + base + qd] : 0;
        T vv[B2];
#pragma unroll
        for (int e = 0; e < B2; e++) vv[e] = has ? val[(long long)(k0 + base + qd) * B2 + e] : T(0);
#pragma unroll
        for (int u = 0; u < Q; u++) {
          const int j = __shfl_sync(0xffffffffu, cj, u, Q);
          T ae[B2];
#pragma unroll
          for (int e = 0; e < B2; e++) ae[e] = __shfl_sync(0xffffffffu, vv[e], u, Q);
          if (base + u < len && any) {
#pragma unroll
            for (int l = 0; l < B; l++) {
              const long long ij = ((long long)j * B + l) * Kp + 4 * qd;
              T z4[4], p4[4];
              ld4<true>(zv + ij, z4);
              if (!first) ld4<true>(pold + ij, p4);
#pragma unroll
              for (int jj = 0; jj < 4; jj++) {
                const T pl = first ? z4[jj] : fmat<T>(beta[jj], p4[jj], z4[jj]);
#pragma unroll
                for (int rr = 0; rr < B; rr++) acc[rr][jj] = fmat<T>(ae[rr * B + l], pl, acc[rr][jj]);
              }
            }
          }
        }
      }
      if (valid && any) {
#pragma unroll
        for (int cc = 0; cc < B; cc++) {
          const long long i = at(row, cc);
          T z4[4], p4[4], pn[4];
          ld4<false>(zv + i, z4);
          if (!first) ld4<false>(pold + i, p4);
#pragma unroll
          for (int jj = 0; jj < 4; jj++) {
            pn[jj] = first ? z4[jj] : fmat<T>(beta[jj], p4[jj], z4[jj]);
            if (live[jj]) pq[jj] += (double)pn[jj] * (double)acc[cc][jj];
          }
          st4(pnew + i, pn);
          st4(qv + i, acc[cc]);
          if (fold[0] || fold[1] || fold[2] || fold[3]) {
            double x4[4];
            T y4[4];
            ld4<false>(xv + i, x4);
            ld4<false>(yv + i, y4);
#pragma unroll
            for (int jj = 0; jj < 4; jj++)
              if (fold[jj] && live[jj]) {
                x4[jj] += (double)y4[jj];
                y4[jj] = T(0);
              }
            st4(xv + i, x4);
            st4(yv + i, y4);
          }
        }
      }
    }
    reduce_write(pq, zero4);
    if (!grid_sync(c, a.partials, true, s_tot, a.spin_limit, [&] {
          if (threadIdx.x < K && !vc->done[threadIdx.x]) {
            const int kk = threadIdx.x;
            const double w = s_tot[0][kk];
            vc->fold[kk] = 0;
            if (w == 0.0 || !isfinite(w)) {
              vc->done[kk] = 1;
              vc->status[kk] = isfinite(w) ? MONOLIS_B200_BREAKDOWN : MONOLIS_B200_NONFINITE;
            } else {
              vc->alpha[kk] = vc->rho[kk] / w;
            }
          }
        }))
      return;
    // Y += alpha P, R -= alpha Q, Z = M^-1 R; <R,R>, <R,Z>
    {
      bool lv[4];
      live4(lv);
      const bool anyl = lv[0] || lv[1] || lv[2] || lv[3];
      T alpha[4];
#pragma unroll
      for (int j = 0; j < 4; j++) alpha[j] = lv[j] ? (T)__ldcg(&c->alpha[4 * qd + j]) : T(0);
      double v0[4] = {0.0, 0.0, 0.0, 0.0}, v1[4] = {0.0, 0.0, 0.0, 0.0};
      // z is rewritten for the live right-hand sides; it is read only to keep
      // a stopped one's entries when this thread has one
      const bool keep_z = !(lv[0] && lv[1] && lv[2] && lv[3]);
      for (long long rb = wrow0; anyl && rb < N; rb += sweep) {
        const long long row = rb + g;
        if (row >= N) continue;
        T t[B][4], w[B][4];
#pragma unroll
        for (int cc = 0; cc < B; cc++) {
          const long long i = at(row, cc);
          T p4[4], q4[4], r4[4], y4[4], z4[4] = {T(0), T(0), T(0), T(0)};
          ld4<false>(pnew + i, p4);
          ld4<false>(qv + i, q4);
          ld4<false>(rv + i, r4);
          ld4<false>(yv + i, y4);
          if (keep_z) ld4<false>(zv + i, z4);
#pragma unroll
          for (int j = 0; j < 4; j++) {
            y4[j] = lv[j] ? fmat<T>(alpha[j], p4[j], y4[j]) : y4[j];
            t[cc][j] = lv[j] ? fmat<T>(-alpha[j], q4[j], r4[j]) : r4[j];
            w[cc][j] = lv[j] ? t[cc][j] : z4[j];
          }
          st4(yv + i, y4);
        }
        if (a.prec) {
#pragma unroll
          for (int j = 0; j < 4; j++) {
            if (!lv[j]) continue;
            T wj[B];
#pragma unroll
            for (int cc = 0; cc < B; cc++) wj[cc] = t[cc][j];
            diag_row<B, T>(alu, a.N, (int)row, wj);
#pragma unroll
            for (int cc = 0; cc < B; cc++) w[cc][j] = wj[cc];
          }
        }
#pragma unroll
        for (int cc = 0; cc < B; cc++) {
          st4(rv + at(row, cc), t[cc]);
          st4(zv + at(row, cc), w[cc]);
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (lv[j]) {
              v0[j] += (double)t[cc][j] * (double)t[cc][j];
              v1[j] += (double)t[cc][j] * (double)w[cc][j];
            }
        }
      }
      reduce_write(v0, v1);
    }
    if (!grid_sync(c, a.partials, true, s_tot, a.spin_limit, [&] {
          int any_r = 0;
          if (threadIdx.x < K && !vc->done[threadIdx.x]) {
            const int kk = threadIdx.x;
            const double rr = s_tot[0][kk], rz = s_tot[1][kk];
            const int it = vc->iter[kk] + 1;
            vc->iter[kk] = it;
            const double rn = sqrt(rr), resid = sqrt(rr / vc->B2[kk]);
            vc->resid[kk] = resid;
            if (!isfinite(resid)) {
              vc->done[kk] = 1;
              vc->status[kk] = MONOLIS_B200_NONFINITE;
            } else {
              vc->rmax[kk] = fmax(vc->rmax[kk], rn);
              const bool stop = resid < a.tol || it >= a.max_iter;
              if (stop || (a.refine && rn < a.delta * vc->rmax[kk])) {
                vc->refresh[kk] = 1;  // FP64 residual: convergence test (refine) or the reported residual
                any_r = 1;
              } else {
                vc->rho1[kk] = vc->rho[kk];
                vc->rho[kk] = rz;
                vc->beta[kk] = vc->rho[kk] / vc->rho1[kk];
              }
            }
          }
          if (threadIdx.x < 32) any_r = __any_sync(0xffffffffu, any_r);
          if (threadIdx.x == 0) {
            vc->any_refresh = any_r;
            vc->it += 1;
          }
        }))
      return;
    if (__ldcg(&c->any_refresh)) {
      bool mine[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int k = 4 * qd + j;
        mine[j] = k < K && __ldcg(&c->refresh[k]) != 0;
      }
      refresh(mine);
      if (!grid_sync(c, a.partials, true, s_tot, a.spin_limit, [&] {
            if (threadIdx.x < K && vc->refresh[threadIdx.x]) {
              const int kk = threadIdx.x;
              const double rr = s_tot[0][kk], rz = s_tot[1][kk];
              const double resid = sqrt(rr / vc->B2[kk]);
              vc->refresh[kk] = 0;
              vc->fold[kk] = 1;
              vc->nref[kk] += 1;
              vc->resid[kk] = resid;
              if (!isfinite(resid)) {
                vc->done[kk] = 1;
                vc->status[kk] = MONOLIS_B200_NONFINITE;
              } else if (resid < a.tol || !a.refine) {
                // refine: converged on the FP64 residual; FP32-only: the
                // iterated residual met tol, this is the reported one
                vc->done[kk] = 1;
                vc->status[kk] = (resid < a.tol || vc->iter[kk] < a.max_iter) ? MONOLIS_B200_OK : MONOLIS_B200_MAXITER;
              } else if (vc->iter[kk] >= a.max_iter) {
                vc->done[kk] = 1;
                vc->status[kk] = MONOLIS_B200_MAXITER;
              } else {
                vc->rmax[kk] = sqrt(rr);
                vc->rho1[kk] = vc->rho[kk];
                vc->rho[kk] = rz;
                vc->beta[kk] = vc->rho[kk] / vc->rho1[kk];
              }
            }
          }))
        return;
    }
    // every right-hand side done (or the iteration cap, as a backstop)
    if (threadIdx.x == 0) {
      int all = 1;
      for (int kk = 0; kk < K; kk++) all &= __ldcg(&c->done[kk]) != 0;
      s_flag[0] = all || __ldcg(&c->it) > a.max_iter + 1;
    }
    __syncthreads();
    if (s_flag[0]) break;
    T* tmp = pold;
    pold = pnew;
    pnew = tmp;
  }
  // fold the last corrections (every block has passed its last reads of x, y)
  bool fold[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int k = 4 * qd + j;
    fold[j] = k < K && __ldcg(&c->fold[k]) != 0;
  }
  if (fold[0] || fold[1] || fold[2] || fold[3])
    for (long long rb = wrow0; rb < N; rb += sweep) {
      const long long row = rb + g;
      if (row >= N) continue;
#pragma unroll
      for (int cc = 0; cc < B; cc++) {
        const long long i = at(row, cc);
        double x4[4];
        T y4[4];
        ld4<false>(xv + i, x4);
        ld4<false>(yv + i, y4);
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (fold[j]) {
            x4[j] += (double)y4[j];
            y4[j] = T(0);
          }
        st4(xv + i, x4);
        st4(yv + i, y4);
      }
    }
}

// column-major (k slowest) <-> interleaved (k fastest, stride Kp >= K;
// the padding right-hand sides are zero)
__global__ void to_interleaved(const double* __restrict__ src, double* __restrict__ dst, long long n, int K, int Kp,
                               long long ld) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * Kp; i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / Kp;
    const int k = (int)(i - e * Kp);
    dst[i] = k < K ? src[(long long)k * ld + e] : 0.0;
  }
}
__global__ void from_interleaved(const double* __restrict__ src, double* __restrict__ dst, long long n, int K, int Kp,
                                 long long ld) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * Kp; i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / Kp;
    const int k = (int)(i - e * Kp);
    if (k < K) dst[(long long)k * ld + e] = src[i];
  }
}
__global__ void csr_to_solver(const int* __restrict__ item, const double* __restrict__ val, long long nz, int B2,
                              int* __restrict__ col, float* __restrict__ val32) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nz * B2; i += (long long)gridDim.x * blockDim.x) {
    if (i < nz) col[i] = item[i] - 1;
    val32[i] = (float)val[i];
  }
}

template <class P>
cudaError_t grow_m(P** p, size_t& cap, size_t need) {
  if (*p && cap >= need) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void**)p, need * sizeof(P) + 16);
  if (e == cudaSuccess) cap = need;
  return e;
}

// The chunk's work as one CUDA graph: right-hand sides to the interleaved
// layout, control block cleared, the persistent kernel (cooperative launch:
// every block resident), solutions back to the caller's layout.
template <int B, class T, int Q>
int capture_multi(const MultiArgs<T>& args, const double* d_B, double* b_dst, double* d_X, long long ld, int Kc,
                  cudaStream_t s, cudaGraph_t* graph) {
  auto kernel = multi_cg_kernel<B, T, Q>;
  constexpr int Kp = 4 * Q;
  int per_sm = 0, dev = 0, sms = 0;
  MB_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kMultiThreads, 0));
  MB_CUDA_OK(cudaGetDevice(&dev));
  MB_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm < 1) return kBadInput;
  // every block resident (cooperative launch), within the barrier's group table
  const int grid = std::min(per_sm * sms, kMaxGroups * kBarrierGroup);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kMultiThreads);
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MB_CUDA_OK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  to_interleaved<<<148 * 8, 256, 0, s>>>(d_B, b_dst, ld, Kc, Kp, ld);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemsetAsync(args.ctl, 0, sizeof(MultiCtl), s);
  if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, kernel, args);
  if (e == cudaSuccess) {
    from_interleaved<<<148 * 8, 256, 0, s>>>(args.x, d_X, ld, Kc, Kp, ld);
    e = cudaGetLastError();
  }
  // the capture is always ended, so the stream stays usable after an error
  const cudaError_t e2 = cudaStreamEndCapture(s, graph);
  if (e != cudaSuccess) {
    if (*graph) cudaGraphDestroy(*graph);
    *graph = nullptr;
    return report_cuda(e, "multi-RHS launch sequence (stream capture)", __FILE__, __LINE__);
  }
  if (e2 != cudaSuccess) return report_cuda(e2, "cudaStreamEndCapture (multi-RHS graph)", __FILE__, __LINE__);
  return kOk;
}

}  // namespace

struct MultiState {
  int* col = nullptr;
  float* val32 = nullptr;
  size_t cap_col = 0, cap_val = 0;
  double *b = nullptr, *x = nullptr, *partials = nullptr;
  void* vec = nullptr;  // y r z p0 p1 q (loop precision)
  MultiCtl* ctl = nullptr;
  size_t cap_b = 0, cap_x = 0, cap_vec = 0, cap_part = 0;
  long long built_for = -1;
  // instantiated graphs of recent chunk launches, keyed by every argument
  // of the launch sequence (a repeated solve relaunches its graph)
  struct Slot {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<Slot> graphs;
};

MultiState* multi_new() { return new MultiState(); }
void multi_free(MultiState* ms) {
  if (!ms) return;
  for (auto& g : ms->graphs) cudaGraphExecDestroy(g.exec);
  cudaFree(ms->col);
  cudaFree(ms->val32);
  cudaFree(ms->b);
  cudaFree(ms->x);
  cudaFree(ms->partials);
  cudaFree(ms->vec);
  cudaFree(ms->ctl);
  delete ms;
}

// Solve A X_k = B_k for n_rhs right-hand sides stored one after another
// (B + k*ld, ld = N*ndof), in chunks of up to 32.
namespace {
template <class P>
void append_bytes(std::vector<unsigned char>& k, const P& v) {
  const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
  k.insert(k.end(), p, p + sizeof(P));
}
}  // namespace

int multi_solve(SellMatrix& m, MultiState& ms, long long build_id, int n_rhs, const double* d_B, double* d_X,
                int precision, int prec, double tol, int max_iter, double delta, unsigned long long wait_limit,
                unsigned int delay_ns, int* iter, double* resid, int* status, cudaStream_t s) {
  if (n_rhs < 1 || max_iter < 1 || !(tol >= 0.0)) return kBadInput;
  if (wait_limit == 0) wait_limit = kSpinLimit;
  if (prec && !m.have_alu) return kBadInput;
  if (precision == 1 && prec && !m.have_alu32) return kBadInput;
  const int N = m.N, nd = m.ndof, B2 = nd * nd;
  const long long ld = (long long)N * nd;
  if (ms.built_for != build_id) {
    MB_CUDA_OK(grow_m(&ms.col, ms.cap_col, (size_t)m.nz));
    MB_CUDA_OK(grow_m(&ms.val32, ms.cap_val, (size_t)m.nz * B2));
    csr_to_solver<<<148 * 8, 256, 0, s>>>(m.d_item, m.d_csrval, m.nz, B2, ms.col, ms.val32);
    MB_CUDA_OK(cudaGetLastError());
    ms.built_for = build_id;
  }
  const size_t nv = (size_t)ld * kMultiK;  // capacity for the widest chunk
  const size_t tsize = precision == 1 ? sizeof(float) : sizeof(double);
  MB_CUDA_OK(grow_m(&ms.b, ms.cap_b, nv));
  MB_CUDA_OK(grow_m(&ms.x, ms.cap_x, nv));
  const size_t vec_bytes = (nv * tsize + 255) / 256 * 256;
  if (!ms.vec || ms.cap_vec < 6 * vec_bytes) {
    cudaFree(ms.vec);
    ms.vec = nullptr;
    MB_CUDA_OK(cudaMalloc(&ms.vec, 6 * vec_bytes));
    ms.cap_vec = 6 * vec_bytes;
  }
  int dev = 0, sms = 0;
  MB_CUDA_OK(cudaGetDevice(&dev));
  MB_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // resident blocks x partials, then one row of group sums per group
  const size_t part = ((size_t)sms * (2048 / kMultiThreads) + kMaxGroups) * 2 * kMultiK;
  MB_CUDA_OK(grow_m(&ms.partials, ms.cap_part, part));
  if (!ms.ctl) MB_CUDA_OK(cudaMalloc((void**)&ms.ctl, sizeof(MultiCtl)));
  std::vector<MultiCtl> h(1);
  for (int k0 = 0; k0 < n_rhs; k0 += kMultiK) {
    const int Kc = std::min(kMultiK, n_rhs - k0);
    const int Q = Kc <= 8 ? 2 : 8;  // lanes per row; right-hand sides padded to 4Q
    const double* Bk = d_B + (long long)k0 * ld;
    double* Xk = d_X + (long long)k0 * ld;
    char* v = static_cast<char*>(ms.vec);
    // the launch arguments, zero-filled first so that padding bytes compare equal in the key
    std::vector<unsigned char> key;
    cudaGraph_t graph = nullptr;
    int rc = dispatch_ndof(nd, [&](auto Bc) -> int {
      constexpr int Bn = decltype(Bc)::value;
      append_bytes(key, Bn);
      append_bytes(key, Q);
      append_bytes(key, precision);
      append_bytes(key, Bk);
      append_bytes(key, Xk);
      append_bytes(key, ld);
      append_bytes(key, s);
      if (precision == 1) {
        MultiArgs<float> a;
        memset(&a, 0, sizeof(a));
        a.N = N; a.K = Kc; a.prec = prec; a.refine = 1; a.max_iter = max_iter; a.tol = tol;
        a.delta = delta > 0 ? delta : 0.1;
        a.rowptr = m.d_rowptr; a.col = ms.col; a.val = ms.val32; a.val64 = m.d_csrval; a.alu = m.d_alu32;
        a.b = ms.b; a.x = ms.x;
        a.y = (float*)(v); a.r = (float*)(v + vec_bytes); a.z = (float*)(v + 2 * vec_bytes);
        a.p0 = (float*)(v + 3 * vec_bytes); a.p1 = (float*)(v + 4 * vec_bytes); a.q = (float*)(v + 5 * vec_bytes);
        a.partials = ms.partials; a.ctl = ms.ctl; a.spin_limit = wait_limit; a.delay_ns = delay_ns;
        append_bytes(key, a);
        for (auto& g : ms.graphs)
          if (g.key == key) return kOk;
        return Q == 2 ? capture_multi<Bn, float, 2>(a, Bk, ms.b, Xk, ld, Kc, s, &graph)
                      : capture_multi<Bn, float, 8>(a, Bk, ms.b, Xk, ld, Kc, s, &graph);
      }
      MultiArgs<double> a;
      memset(&a, 0, sizeof(a));
      a.N = N; a.K = Kc; a.prec = prec; a.refine = 0; a.max_iter = max_iter; a.tol = tol; a.delta = 0.1;
      a.rowptr = m.d_rowptr; a.col = ms.col; a.val = m.d_csrval; a.val64 = m.d_csrval; a.alu = m.d_alu64;
      a.b = ms.b; a.x = ms.x;
      a.y = (double*)(v); a.r = (double*)(v + vec_bytes); a.z = (double*)(v + 2 * vec_bytes);
      a.p0 = (double*)(v + 3 * vec_bytes); a.p1 = (double*)(v + 4 * vec_bytes); a.q = (double*)(v + 5 * vec_bytes);
      a.partials = ms.partials; a.ctl = ms.ctl; a.spin_limit = wait_limit; a.delay_ns = delay_ns;
      append_bytes(key, a);
      for (auto& g : ms.graphs)
        if (g.key == key) return kOk;
      return Q == 2 ? capture_multi<Bn, double, 2>(a, Bk, ms.b, Xk, ld, Kc, s, &graph)
                    : capture_multi<Bn, double, 8>(a, Bk, ms.b, Xk, ld, Kc, s, &graph);
    });
    if (rc) return rc;
    cudaGraphExec_t exec = nullptr;
    for (auto& g : ms.graphs)
      if (g.key == key) exec = g.exec;
    if (!exec) {
      const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return report_cuda(e, "cudaGraphInstantiate (multi-RHS graph)", __FILE__, __LINE__);
      if (ms.graphs.size() >= 8) {
        cudaGraphExecDestroy(ms.graphs.front().exec);
        ms.graphs.erase(ms.graphs.begin());
      }
      ms.graphs.push_back({key, exec});
    }
    MB_CUDA_OK(cudaGraphLaunch(exec, s));
    MB_CUDA_OK(cudaMemcpyAsync(h.data(), ms.ctl, sizeof(MultiCtl), cudaMemcpyDeviceToHost, s));
    MB_CUDA_OK(cudaStreamSynchronize(s));
    if (h[0].err) {
      fprintf(stderr, "** monolis_b200: multi-RHS kernel gave up waiting at a grid barrier\n");
      return kTimeout;
    }
    for (int k = 0; k < Kc; k++) {
      if (iter) iter[k0 + k] = h[0].iter[k];
      if (resid) resid[k0 + k] = h[0].resid[k];
      if (status) status[k0 + k] = h[0].status[k];
    }
  }
  return kOk;
}

}  // namespace mb
