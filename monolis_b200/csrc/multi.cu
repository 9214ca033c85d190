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
#include <vector>

#include "monolis_b200.h"
#include "spmv.cuh"

namespace mb {
namespace {

constexpr int kMultiK = 32;
constexpr int kMultiThreads = 256;
constexpr unsigned long long kSpinLimit = 1ull << 22;  // polls (an L2 round trip + 32 ns each): seconds

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
__device__ bool grid_sync(MultiCtl* c, double* partials, bool reduce, double (*tot)[kMultiK], F&& last) {
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
        if (++n > kSpinLimit) {
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
      if (++n > kSpinLimit) {
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

// This block's partial sums (v0, v1 per lane = right-hand side) into partials.
__device__ __forceinline__ void write_partials(double v0, double v1, double (*s_red)[2][kMultiK], double* partials) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  s_red[w][0][lane] = v0;
  s_red[w][1][lane] = v1;
  __syncthreads();
  if (threadIdx.x < 2 * kMultiK) {
    const int which = threadIdx.x >> 5, kk = threadIdx.x & 31;
    double s = 0.0;
    for (int i = 0; i < nw; i++) s += s_red[i][which][kk];
    partials[((size_t)blockIdx.x * 2 + which) * kMultiK + kk] = s;
  }
}

template <class T>
__device__ __forceinline__ T fmat(T a, T b, T c);
template <>
__device__ __forceinline__ float fmat<float>(float a, float b, float c) { return fmaf(a, b, c); }
template <>
__device__ __forceinline__ double fmat<double>(double a, double b, double c) { return fma(a, b, c); }

// Small blocks: at most 64 registers, so that 4 blocks (32 warps) per SM
// keep enough loads in flight for HBM bandwidth.
template <int B, class T>
__global__ void __launch_bounds__(kMultiThreads, B <= 2 ? 4 : 1) multi_cg_kernel(const MultiArgs<T> a) {
  constexpr int B2 = B * B;
  constexpr int kCh = B == 1 ? 8 : (B == 2 ? 4 : (B == 3 ? 2 : 1));  // row entries gathered together
  constexpr int kRows = B == 1 ? 4 : (B <= 3 ? 2 : 1);                // rows per step of the update
  constexpr int kChR = kCh > 1 ? kCh / 2 : 1;  // the (rare) FP64 refresh: fewer registers
  // the arrays never alias: tell the compiler, so that loads of the next
  // rows may move above the stores of the current ones
  const int* __restrict__ rowptr = a.rowptr;
  const int* __restrict__ colv = a.col;
  const T* __restrict__ val = a.val;
  const double* __restrict__ val64 = a.val64;
  const T* __restrict__ alu = a.alu;
  const double* __restrict__ bv = a.b;
  double* __restrict__ xv = a.x;
  T* __restrict__ yv_ = a.y;
  T* __restrict__ rv_ = a.r;
  T* __restrict__ zv = a.z;
  T* __restrict__ qv_ = a.q;
  __shared__ double s_red[kMultiThreads / 32][2][kMultiK];
  __shared__ double s_tot[2][kMultiK];
  __shared__ int s_flag[2];
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const long long W = (long long)gridDim.x * nw;
  const long long gw = (long long)blockIdx.x * nw + (threadIdx.x >> 5);
  const int K = a.K;
  const bool act = lane < K;
  const int k = lane;
  MultiCtl* c = a.ctl;
  // the last block of a barrier reads and writes the scalars through a
  // volatile view (L1 is not coherent across SMs); the others use __ldcg
  volatile MultiCtl* vc = c;
  auto at = [&](long long row, int comp) { return (row * B + comp) * K + k; };

  // x = y = 0 on the own rows
  for (long long row = gw; row < a.N; row += W)
    if (act)
#pragma unroll
      for (int cc = 0; cc < B; cc++) {
        xv[at(row, cc)] = 0.0;
        yv_[at(row, cc)] = T(0);
      }

  // r = b - A (x + y) in FP64, z = M^-1 r, for the lanes with `mine` set
  // (all lanes at the start); partial sums <r,r>, <r,z> written per block
  auto refresh = [&](bool mine) {
    double v0 = 0.0, v1 = 0.0;
    for (long long row = gw; row < a.N; row += W) {
      const int k0 = rowptr[row], len = rowptr[row + 1] - k0;
      double ax[B];
#pragma unroll
      for (int cc = 0; cc < B; cc++) ax[cc] = 0.0;
      for (int base = 0; base < len; base += 32) {
        const int m = min(32, len - base);
        int cj = 0;
        double vv[B2];
#pragma unroll
        for (int e = 0; e < B2; e++) vv[e] = 0.0;
        if (lane < m) {
          cj = colv[k0 + base + lane];
#pragma unroll
          for (int e = 0; e < B2; e++) vv[e] = val64[(long long)(k0 + base + lane) * B2 + e];
        }
        for (int t0 = 0; t0 < m; t0 += kChR) {
          int jj[kChR];
          double ae[kChR][B2];
#pragma unroll
          for (int u = 0; u < kChR; u++) {
            jj[u] = __shfl_sync(0xffffffffu, cj, (t0 + u) & 31);
#pragma unroll
            for (int e = 0; e < B2; e++) ae[u][e] = __shfl_sync(0xffffffffu, vv[e], (t0 + u) & 31);
          }
          if (act && mine) {
            double xs[kChR][B];
#pragma unroll
            for (int u = 0; u < kChR; u++)
#pragma unroll
              for (int l = 0; l < B; l++) {
                const long long ij = ((long long)jj[u] * B + l) * K + k;
                xs[u][l] = __ldcg(xv + ij) + (double)__ldcg(yv_ + ij);
              }
#pragma unroll
            for (int u = 0; u < kChR; u++)
              if (t0 + u < m)
#pragma unroll
                for (int rr = 0; rr < B; rr++)
#pragma unroll
                  for (int l = 0; l < B; l++) ax[rr] = fma(ae[u][rr * B + l], xs[u][l], ax[rr]);
          }
        }
      }
      if (act && mine) {
        T t[B], w[B];
#pragma unroll
        for (int cc = 0; cc < B; cc++) {
          const double rv = bv[at(row, cc)] - ax[cc];
          v0 += rv * rv;
          t[cc] = (T)rv;
          w[cc] = t[cc];
          rv_[at(row, cc)] = t[cc];
        }
        if (a.prec) diag_row<B, T>(alu, a.N, (int)row, w);
#pragma unroll
        for (int cc = 0; cc < B; cc++) {
          zv[at(row, cc)] = w[cc];
          v1 += (double)t[cc] * (double)w[cc];
        }
      }
    }
    write_partials(v0, v1, s_red, a.partials);
  };

  // the whole grid has zeroed its x and y before any residual reads them
  if (!grid_sync(c, a.partials, false, s_tot, [] {})) return;
  refresh(true);
  if (!grid_sync(c, a.partials, true, s_tot, [&] {
        if (threadIdx.x < K) {
          const int kk = threadIdx.x;
          const double rr = s_tot[0][kk], rz = s_tot[1][kk];
          vc->B2[kk] = rr;
          vc->iter[kk] = 0;
          vc->nref[kk] = 0;
          vc->fold[kk] = 0;
          vc->refresh[kk] = 0;
          vc->resid[kk] = 0.0;
          if (!(rr > 0.0) || !isfinite(rr)) {
            vc->done[kk] = 1;  // B2 == 0: x = 0 solves it
            vc->status[kk] = isfinite(rr) ? MONOLIS_B200_OK : MONOLIS_B200_NONFINITE;
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
    const bool done_k = !act || __ldcg(&c->done[k]) != 0;
    const bool first = __ldcg(&c->it) == 1;
    const T beta = act ? (T)__ldcg(&c->beta[k]) : T(0);
    const bool fold = act && __ldcg(&c->fold[k]) != 0;
    // P = Z + beta P (own rows, to pnew); Q = A P with P recomputed from Z
    // and the old P at the neighbours; <P,Q>
    double pq = 0.0;
    for (long long row = gw; row < a.N; row += W) {
      const int k0 = rowptr[row], len = rowptr[row + 1] - k0;
      T acc[B];
#pragma unroll
      for (int cc = 0; cc < B; cc++) acc[cc] = T(0);
      for (int base = 0; base < len; base += 32) {
        const int m = min(32, len - base);
        int cj = 0;
        T vv[B2];
#pragma unroll
        for (int e = 0; e < B2; e++) vv[e] = T(0);
        if (lane < m) {
          cj = colv[k0 + base + lane];
#pragma unroll
          for (int e = 0; e < B2; e++) vv[e] = val[(long long)(k0 + base + lane) * B2 + e];
        }
        // kCh entries at a time: all their gathers are issued before any is
        // used (lanes past the row end hold column 0 and value 0)
        for (int t0 = 0; t0 < m; t0 += kCh) {
          int jj[kCh];
          T ae[kCh][B2];
#pragma unroll
          for (int u = 0; u < kCh; u++) {
            jj[u] = __shfl_sync(0xffffffffu, cj, (t0 + u) & 31);
#pragma unroll
            for (int e = 0; e < B2; e++) ae[u][e] = __shfl_sync(0xffffffffu, vv[e], (t0 + u) & 31);
          }
          if (!done_k) {
            T zs[kCh][B], po[kCh][B];
#pragma unroll
            for (int u = 0; u < kCh; u++)
#pragma unroll
              for (int l = 0; l < B; l++) {
                const long long ij = ((long long)jj[u] * B + l) * K + k;
                zs[u][l] = __ldcg(zv + ij);
                po[u][l] = first ? T(0) : __ldcg(pold + ij);
              }
#pragma unroll
            for (int u = 0; u < kCh; u++) {
              if (t0 + u < m) {
#pragma unroll
                for (int l = 0; l < B; l++) {
                  const T pl = first ? zs[u][l] : fmat<T>(beta, po[u][l], zs[u][l]);
#pragma unroll
                  for (int rr = 0; rr < B; rr++) acc[rr] = fmat<T>(ae[u][rr * B + l], pl, acc[rr]);
                }
              }
            }
          }
        }
      }
      if (!done_k) {
#pragma unroll
        for (int cc = 0; cc < B; cc++) {
          const long long i = at(row, cc);
          const T pv = first ? zv[i] : fmat<T>(beta, pold[i], zv[i]);
          pnew[i] = pv;
          qv_[i] = acc[cc];
          pq += (double)pv * (double)acc[cc];
          if (fold) {
            xv[i] += (double)yv_[i];
            yv_[i] = T(0);
          }
        }
      }
    }
    write_partials(pq, 0.0, s_red, a.partials);
    if (!grid_sync(c, a.partials, true, s_tot, [&] {
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
      const bool live = act && __ldcg(&c->done[k]) == 0;
      const T alpha = live ? (T)__ldcg(&c->alpha[k]) : T(0);
      double v0 = 0.0, v1 = 0.0;
      // kRows rows per step: the loads of all of them are in flight together
      for (long long row = gw; live && row < a.N; row += kRows * W) {
        const int nr = (int)min((long long)kRows, (a.N - row + W - 1) / W);
        T pv[kRows][B], qv[kRows][B], rv[kRows][B], yv[kRows][B];
#pragma unroll
        for (int h = 0; h < kRows; h++)
          if (h < nr)
#pragma unroll
            for (int cc = 0; cc < B; cc++) {
              const long long i = at(row + h * W, cc);
              pv[h][cc] = pnew[i];
              qv[h][cc] = qv_[i];
              rv[h][cc] = rv_[i];
              yv[h][cc] = yv_[i];
            }
#pragma unroll
        for (int h = 0; h < kRows; h++) {
          if (h >= nr) break;
          const long long rw = row + h * W;
          T t[B], w[B];
#pragma unroll
          for (int cc = 0; cc < B; cc++) {
            const long long i = at(rw, cc);
            yv_[i] = fmat<T>(alpha, pv[h][cc], yv[h][cc]);
            t[cc] = fmat<T>(-alpha, qv[h][cc], rv[h][cc]);
            rv_[i] = t[cc];
            w[cc] = t[cc];
          }
          if (a.prec) diag_row<B, T>(alu, a.N, (int)rw, w);
#pragma unroll
          for (int cc = 0; cc < B; cc++) {
            zv[at(rw, cc)] = w[cc];
            v0 += (double)t[cc] * (double)t[cc];
            v1 += (double)t[cc] * (double)w[cc];
          }
        }
      }
      write_partials(v0, v1, s_red, a.partials);
    }
    if (!grid_sync(c, a.partials, true, s_tot, [&] {
            int any = 0;
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
                any = 1;
              } else {
                vc->rho1[kk] = vc->rho[kk];
                vc->rho[kk] = rz;
                vc->beta[kk] = vc->rho[kk] / vc->rho1[kk];
              }
            }
          }
          if (threadIdx.x < 32) any = __any_sync(0xffffffffu, any);
          if (threadIdx.x == 0) {
            vc->any_refresh = any;
            vc->it += 1;
          }
        }))
      return;
    if (__ldcg(&c->any_refresh)) {
      const bool mine = act && __ldcg(&c->refresh[k]) != 0;
      refresh(mine);
      if (!grid_sync(c, a.partials, true, s_tot, [&] {
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
  const bool fold = act && __ldcg(&c->fold[k]) != 0;
  if (fold)
    for (long long row = gw; row < a.N; row += W)
#pragma unroll
      for (int cc = 0; cc < B; cc++) {
        const long long i = at(row, cc);
        xv[i] += (double)yv_[i];
        yv_[i] = T(0);
      }
}

// column-major (k slowest) <-> interleaved (k fastest) copies
__global__ void to_interleaved(const double* __restrict__ src, double* __restrict__ dst, long long n, int K,
                               long long ld) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * K; i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / K;
    const int k = (int)(i - e * K);
    dst[i] = src[(long long)k * ld + e];
  }
}
__global__ void from_interleaved(const double* __restrict__ src, double* __restrict__ dst, long long n, int K,
                                 long long ld) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * K; i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / K;
    const int k = (int)(i - e * K);
    dst[(long long)k * ld + e] = src[i];
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

template <int B, class T>
int launch_multi(const MultiArgs<T>& args, cudaStream_t s) {
  auto kernel = multi_cg_kernel<B, T>;
  int per_sm = 0, dev = 0, sms = 0;
  MB_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kMultiThreads, 0));
  MB_CUDA_OK(cudaGetDevice(&dev));
  MB_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (per_sm < 1) return kBadInput;
  // every block resident (cooperative launch), within the barrier's group table
  const int grid = std::min(per_sm * sms, kMaxGroups * kBarrierGroup);
  MultiArgs<T> a = args;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kMultiThreads);
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MB_CUDA_OK(cudaMemsetAsync(a.ctl, 0, sizeof(MultiCtl), s));
  MB_CUDA_OK(cudaLaunchKernelEx(&cfg, kernel, a));
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
};

MultiState* multi_new() { return new MultiState(); }
void multi_free(MultiState* ms) {
  if (!ms) return;
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
int multi_solve(SellMatrix& m, MultiState& ms, long long build_id, int n_rhs, const double* d_B, double* d_X,
                int precision, int prec, double tol, int max_iter, double delta, int* iter, double* resid, int* status,
                cudaStream_t s) {
  if (n_rhs < 1 || max_iter < 1 || !(tol >= 0.0)) return kBadInput;
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
  const int K = std::min(n_rhs, kMultiK);
  const size_t nv = (size_t)ld * K;
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
    to_interleaved<<<148 * 8, 256, 0, s>>>(d_B + (long long)k0 * ld, ms.b, ld, Kc, ld);
    char* v = static_cast<char*>(ms.vec);
    int rc = dispatch_ndof(nd, [&](auto Bc) -> int {
      constexpr int Bn = decltype(Bc)::value;
      if (precision == 1) {
        MultiArgs<float> a{};
        a.N = N; a.K = Kc; a.prec = prec; a.refine = 1; a.max_iter = max_iter; a.tol = tol;
        a.delta = delta > 0 ? delta : 0.1;
        a.rowptr = m.d_rowptr; a.col = ms.col; a.val = ms.val32; a.val64 = m.d_csrval; a.alu = m.d_alu32;
        a.b = ms.b; a.x = ms.x;
        a.y = (float*)(v); a.r = (float*)(v + vec_bytes); a.z = (float*)(v + 2 * vec_bytes);
        a.p0 = (float*)(v + 3 * vec_bytes); a.p1 = (float*)(v + 4 * vec_bytes); a.q = (float*)(v + 5 * vec_bytes);
        a.partials = ms.partials; a.ctl = ms.ctl;
        return launch_multi<Bn, float>(a, s);
      }
      MultiArgs<double> a{};
      a.N = N; a.K = Kc; a.prec = prec; a.refine = 0; a.max_iter = max_iter; a.tol = tol; a.delta = 0.1;
      a.rowptr = m.d_rowptr; a.col = ms.col; a.val = m.d_csrval; a.val64 = m.d_csrval; a.alu = m.d_alu64;
      a.b = ms.b; a.x = ms.x;
      a.y = (double*)(v); a.r = (double*)(v + vec_bytes); a.z = (double*)(v + 2 * vec_bytes);
      a.p0 = (double*)(v + 3 * vec_bytes); a.p1 = (double*)(v + 4 * vec_bytes); a.q = (double*)(v + 5 * vec_bytes);
      a.partials = ms.partials; a.ctl = ms.ctl;
      return launch_multi<Bn, double>(a, s);
    });
    if (rc) return rc;
    from_interleaved<<<148 * 8, 256, 0, s>>>(ms.x, d_X + (long long)k0 * ld, ld, Kc, ld);
    MB_CUDA_OK(cudaGetLastError());
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
