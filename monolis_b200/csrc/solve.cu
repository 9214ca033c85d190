// solve.cu -- device-resident CG and BiCGSTAB (FP64, and FP32-inner with
// FP64 refinement) built from fused kernels.
//
// Every scalar of the recurrences (rho, alpha, beta, omega, B2, the
// residual) lives in SolverState on the device. Each reduction is a one-pass
// grid reduction (common.cuh) whose last block also evaluates the scalar
// update, so an iteration is a fixed sequence of kernels with no host round
// trip. Kernels that reduce run on a persistent grid (as many blocks as fit
// on the GPU at once) and grid-stride over rows: at ndof 1 (7 blocks a row)
// a block per 256 rows spends more time entering, reducing and leaving than
// on its rows.
//
// A batch of iterations is captured as the body of a CUDA graph while node
// whose last kernel lets the body run again until the state word says done,
// so the whole solve is one graph launch with no host thread in the loop;
// kernels return immediately once `done` is set. The true residual every
// iter_RR iterations of FP64 CG/BiCGSTAB falls on the last iteration of a
// batch (the batch divides iter_RR), whose residual kernel returns at entry
// unless a replacement is due. Several ranks keep a host-driven loop of batch
// graphs (every rank must enqueue the same collectives). The FP64 refresh of
// the mixed solver is decided on the device from the residual history; its
// kernel sits in every iteration on a small grid and returns at once when
// there is nothing to do.
//
// FP64 CG follows src/iterative/CG.f90:74-101 and BiCGSTAB follows
// src/iterative/BiCGSTAB.f90:87-170 operation by operation (same vector
// update expressions and roundings, true residual every 200 iterations,
// convergence relative to the initial residual); only the order in which the
// dot products are summed differs (tree instead of serial).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <functional>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "spmv.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

int num_sms() {
  static int n = 0;
  if (!n) {
    int d = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
    if (n <= 0) n = 148;
  }
  return n;
}

// Persistent grid of a kernel: resident blocks per SM x SMs.
template <class K>
int pgrid(K kernel) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  std::lock_guard<std::mutex> lk(mu);
  const void* key = reinterpret_cast<const void*>(kernel);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kThreads, 0) != cudaSuccess || b < 1) b = 1;
  const int g = b * num_sms();
  cache[key] = g;
  return g;
}

// Rows a matrix kernel visits: all N (slices == nullptr), or the 32-row
// slices listed (multi-rank: interior or boundary slices). Returns the row
// of work item i, or -1 past the matrix end.
struct RowSet {
  const int* __restrict__ slices;
  int nsl;
  __device__ __forceinline__ long long count(int N) const { return slices ? (long long)nsl * kSlice : N; }
  __device__ __forceinline__ int row(long long i, int N) const {
    const long long r = slices ? (long long)slices[i >> 5] * kSlice + (i & (kSlice - 1)) : i;
    return r < N ? (int)r : -1;
  }
};

// body(row) for this thread's rows of a grid-stride loop: all N rows, or
// (kSet) the rows of the listed slices.
template <bool kSet, class F>
__device__ __forceinline__ void for_rows(const RowSet& rs, int N, F&& body) {
  if constexpr (kSet) {
    const long long nit = rs.count(N);
    for (long long it = blockIdx.x * (long long)blockDim.x + threadIdx.x; it < nit;
         it += (long long)gridDim.x * blockDim.x) {
      const int row = rs.row(it, N);
      if (row >= 0) body(row);
    }
  } else {
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < N; row += gridDim.x * blockDim.x) body(row);
  }
}

// ---------------------------------------------------------------------------
// Scalar updates run by the last block of a grid reduction.
// ---------------------------------------------------------------------------
__device__ void record(SolverState* st, double* hist, double resid) {
  st->resid = resid;
  if (hist) hist[st->iter] = resid;
}

// end of CG iteration `iter` (or the initial residual when iter == 0):
// rr = <r,r>, rz = <r,z> (= rho of the next iteration).
__device__ void fin_cg(SolverState* st, double rr, double rz, double* hist) {
  if (st->iter == 0) {
    st->B2 = rr;
    if (rr == 0.0) { st->done = 1; st->status = kZeroRhs; return; }
    st->rho = rz;
    st->iter = 1;
    return;
  }
  const double resid = sqrt(rr / st->B2);  // src/linalg/mat_converge.f90:120
  record(st, hist, resid);
  if (resid < st->tol) { st->done = 1; st->status = kOk; return; }
  if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
  if (st->iter >= st->max_iter) { st->done = 1; st->status = kMaxIter; return; }
  st->rho1 = st->rho;
  st->rho = rz;
  st->beta = st->rho / st->rho1;  // src/iterative/CG.f90:79
  st->iter += 1;
}

// end of BiCGSTAB iteration: rr = <R,R>, rrt = <R,RT> (= rho of the next one)
__device__ void fin_bicg(SolverState* st, double rr, double rrt, double* hist) {
  if (st->iter == 0) {
    st->B2 = rr;
    if (rr == 0.0) { st->done = 1; st->status = kZeroRhs; return; }
    st->rho = rrt;
    st->iter = 1;
    return;
  }
  const double resid = sqrt(rr / st->B2);
  record(st, hist, resid);
  if (resid < st->tol) { st->done = 1; st->status = kOk; return; }
  if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
  if (st->iter >= st->max_iter) { st->done = 1; st->status = kMaxIter; return; }
  st->rho1 = st->rho;
  st->rho = rrt;
  if (rrt == 0.0) { st->done = 1; st->status = kBreakdown; return; }
  st->beta = (st->rho / st->rho1) * (st->alpha / st->omega);  // src/iterative/BiCGSTAB.f90:96
  st->iter += 1;
}

// PipeCG (src/iterative/PipeCG.f90:93-149). Convergence check of an
// iteration (or the initial residual when iter == 0): rr = <R,R>.
__device__ void fin_pipe_check(SolverState* st, double rr, double* hist) {
  if (st->iter == 0) {
    st->B2 = rr;
    if (rr == 0.0) { st->done = 1; st->status = kZeroRhs; return; }
    st->rho = 1.0;    // gamma (PipeCG.f90:85)
    st->alpha = 1.0;  // alpha (PipeCG.f90:86)
    st->iter = 1;
    return;
  }
  const double resid = sqrt(rr / st->B2);
  record(st, hist, resid);
  if (resid < st->tol) { st->done = 1; st->status = kOk; return; }
  if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
  if (st->iter >= st->max_iter) { st->done = 1; st->status = kMaxIter; return; }
  st->iter += 1;
}

// PipeCG scalars from gamma = <R,U>, delta = <V,U> (PipeCG.f90:100-113);
// rho holds gamma, c2 delta.
__device__ void fin_pipe_dots(SolverState* st, double g, double d) {
  const double gamma1 = 1.0 / st->rho;
  const double alpha1 = 1.0 / st->alpha;
  st->rho = g;
  st->c2 = d;
  if (1 < st->iter) {
    st->beta = g * gamma1;
    // two roundings, left to right, as the reference's Fortran (no FMA)
    st->alpha = g / __dsub_rn(d, __dmul_rn(__dmul_rn(st->beta, g), alpha1));
  } else {
    st->alpha = g / d;
    st->beta = 0.0;
  }
}

// GropCG (src/iterative/GropCG.f90:88-125); rho holds gamma, c2 delta.
__device__ void fin_grop_alpha(SolverState* st, double d) {
  st->c2 = d;
  st->alpha = st->rho / d;  // GropCG.f90:93
}
// gamma1 = <R,U>, rr = <R,R>: beta, gamma (GropCG.f90:111-112), then the
// convergence check of the iteration
__device__ void fin_grop(SolverState* st, double g1, double rr, double* hist) {
  st->beta = g1 / st->rho;
  st->rho = g1;
  const double resid = sqrt(rr / st->B2);
  record(st, hist, resid);
  if (resid < st->tol) { st->done = 1; st->status = kOk; return; }
  if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
  if (st->iter >= st->max_iter) { st->done = 1; st->status = kMaxIter; return; }
  st->iter += 1;
}

// ---------------------------------------------------------------------------
// FP64 residual kernel: r = b - A x, then z = M^-1 r (CG) and the two dots.
// mode 0: CG (dots <r,r>, <r,z>); mode 1: BiCGSTAB (dots <r,r>, <r,rt>;
// at iter 0 also rt = r); mode 2: PipeCG (z is U = M^-1 r; <r,r> decides
// convergence). Runs for the initial residual and, on iterations
// with iter % iter_RR == 0, after the update kernel has raised rr_flag.
// ---------------------------------------------------------------------------
template <int B, int U, class V, class T>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks<B>::value)
    resid_kernel(SellView<V> A, const T* __restrict__ x, const T* __restrict__ b, T* __restrict__ r,
                 T* __restrict__ z, T* __restrict__ rt, const T* __restrict__ alu, int prec, int mode,
                 double* partials, unsigned int* ticket, SolverState* st, double* hist) {
  if (st->done) return;
  const bool init = st->iter == 0;
  if (!init && !st->rr_flag) return;
  DotAcc<2, T> v;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < A.N; row += gridDim.x * blockDim.x) {
    T y[B];
    sell_row<B, U, V, T>(A, x, row, y);
    T t[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      t[c] = sub_rn(b[i], y[c]);  // src/linalg/matvec.f90:902  R = 1.0*B + (-1.0)*R
      r[i] = t[c];
      v.add(0, t[c], t[c]);
    }
    if (mode != 1) {  // CG and PipeCG: z (PipeCG: U) = M^-1 r
      T w[B];
#pragma unroll
      for (int c = 0; c < B; c++) w[c] = t[c];
      if (prec) diag_row<B, T>(alu, A.N, row, w);
#pragma unroll
      for (int c = 0; c < B; c++) {
        z[(long long)row * B + c] = w[c];
        v.add(1, t[c], w[c]);
      }
    } else {
#pragma unroll
      for (int c = 0; c < B; c++) {
        const long long i = (long long)row * B + c;
        T rtv;
        if (init) { rt[i] = t[c]; rtv = t[c]; } else { rtv = rt[i]; }
        v.add(1, t[c], rtv);
      }
    }
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // the global sums and the update come after the all-reduce
      st->red[0] = tot[0];
      st->red[1] = tot[1];
      return;
    }
    st->rr_flag = 0;
    if (mode == 0) fin_cg(st, tot[0], tot[1], hist);
    else if (mode == 2) fin_pipe_check(st, tot[0], hist);
    else fin_bicg(st, tot[0], tot[1], hist);
  });
}

// ---------------------------------------------------------------------------
// CG kernels
// ---------------------------------------------------------------------------
// P = beta*P + 1.0*Z (src/iterative/CG.f90:78-83); P = Z on iteration 1.
// 16-byte vector accesses (work vectors are allocation-aligned), scalar tail.
template <class T>
__global__ void cg_p_kernel(long long n, T* __restrict__ p, const T* __restrict__ z, const SolverState* st) {
  using V = typename Vec16T<T>::type;
  constexpr int W = Vec16T<T>::n;
  if (st->done) return;
  const bool first = st->iter == 1;
  const T beta = (T)st->beta;
  const long long nv = n / W;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += stride) {
    V zv = reinterpret_cast<const V*>(z)[i];
    if (!first) {
      V pv = reinterpret_cast<const V*>(p)[i];
      T* pe = reinterpret_cast<T*>(&pv);
      T* ze = reinterpret_cast<T*>(&zv);
#pragma unroll
      for (int k = 0; k < W; k++) ze[k] = axpy_rn(beta, pe[k], ze[k]);
    }
    reinterpret_cast<V*>(p)[i] = zv;
  }
  for (long long i = nv * W + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
    p[i] = first ? z[i] : axpy_rn(beta, p[i], z[i]);
}

// Q = A P fused with omega = <P,Q>, alpha = rho/omega (CG.f90:85-87).
template <int B, int U, class V, class T, bool kSet = false>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks<B>::value)
    cg_spmv_kernel(SellView<V> A, const T* __restrict__ p, T* __restrict__ q, double* partials,
                   unsigned int* ticket, SolverState* st, RowSet rs, int acc) {
  if (st->done) return;
  DotAcc<1, T> v;
  for_rows<kSet>(rs, A.N, [&](int row) {
    T y[B];
    sell_row<B, U, V, T>(A, p, row, y);
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      q[i] = y[c];
      v.add(0, p[i], y[c]);
    }
  });
  grid_reduce<1>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // acc: the boundary slices add to the interior ones' sum
      st->red[0] = acc ? st->red[0] + tot[0] : tot[0];
      return;
    }
    st->omega = tot[0];
    st->alpha = st->rho / tot[0];
  });
}

// X = alpha*P + X; R = -alpha*Q + R; Z = M^-1 R; <R,R>, <R,Z>
// (CG.f90:89-97 + the next iteration's precond apply and rho).
// On iterations with iter % iter_RR == 0 only X is updated here and the
// residual kernel recomputes R = B - A X. Each thread owns R consecutive rows
// (RowGroup) and moves them with 16-byte accesses; rows past the last full
// group, or all rows when x is not 16-byte aligned, take the per-row path.
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    cg_update_kernel(int N, T* __restrict__ x, const T* __restrict__ p, T* __restrict__ r,
                     const T* __restrict__ q, T* __restrict__ z, const T* __restrict__ alu, int prec,
                     double* partials, unsigned int* ticket, SolverState* st, double* hist) {
  using RG = RowGroup<T, B>;
  constexpr int R = RG::R, E = RG::E;
  if (st->done) return;
  const bool rr_iter = (st->iter % st->iter_rr) == 0;
  const T alpha = (T)st->alpha;
  const bool alu_vec = (N % R) == 0;
  const long long ngroups = ((reinterpret_cast<uintptr_t>(x) & 15) == 0) ? N / R : 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  DotAcc<2, T> v;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ngroups; g += stride) {
    const long long row0 = g * R, e0 = row0 * B;
    T xv[E], pv[E];
    vload<T, E>(x + e0, xv);
    vload<T, E>(p + e0, pv);
#pragma unroll
    for (int i = 0; i < E; i++) xv[i] = axpy_rn(alpha, pv[i], xv[i]);
    vstore<T, E>(x + e0, xv);
    if (!rr_iter) {
      T rv[E], qv[E], zv[E];
      vload<T, E>(r + e0, rv);
      vload<T, E>(q + e0, qv);
#pragma unroll
      for (int i = 0; i < E; i++) rv[i] = axpy_rn(-alpha, qv[i], rv[i]);
#pragma unroll
      for (int i = 0; i < E; i++) zv[i] = rv[i];
      if (prec) {
        T L[B * B][R];
        load_alu_rows<T, B, R>(alu, N, row0, alu_vec, L);
#pragma unroll
        for (int k = 0; k < R; k++) {
          T t[B];
#pragma unroll
          for (int c = 0; c < B; c++) t[c] = rv[k * B + c];
          diag_solve<B, T>([&](int j, int kk) { return L[j * B + kk][k]; }, t);
#pragma unroll
          for (int c = 0; c < B; c++) zv[k * B + c] = t[c];
        }
      }
#pragma unroll
      for (int i = 0; i < E; i++) {
        v.add(0, rv[i], rv[i]);
        v.add(1, rv[i], zv[i]);
      }
      vstore<T, E>(r + e0, rv);
      vstore<T, E>(z + e0, zv);
    }
  }
  for (long long row = ngroups * R + blockIdx.x * (long long)blockDim.x + threadIdx.x; row < N; row += stride) {
    T t[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = row * B + c;
      x[i] = axpy_rn(alpha, p[i], x[i]);
      if (!rr_iter) {
        t[c] = axpy_rn(-alpha, q[i], r[i]);
        r[i] = t[c];
      }
    }
    if (!rr_iter) {
      T w[B];
#pragma unroll
      for (int c = 0; c < B; c++) w[c] = t[c];
      if (prec) diag_row<B, T>(alu, N, (int)row, w);
#pragma unroll
      for (int c = 0; c < B; c++) {
        z[row * B + c] = w[c];
        v.add(0, t[c], t[c]);
        v.add(1, t[c], w[c]);
      }
    }
  }
  if (rr_iter) {
    // the counter is not advanced here: the residual kernel that follows
    // recomputes R = B - A X and finishes the iteration
    if (blockIdx.x == 0 && threadIdx.x == 0) st->rr_flag = 1;
    return;
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {
      st->red[0] = tot[0];
      st->red[1] = tot[1];
      return;
    }
    fin_cg(st, tot[0], tot[1], hist);
  });
}

// Device-side loop control: the last kernel of the body of a while node
// (one graph for the whole solve) lets the body run again until the solve has
// a verdict; the iteration cap bounds it even without one.
__global__ void loop_continue_kernel(cudaGraphConditionalHandle h, SolverState* st, int cap) {
  st->loops += 1;
  cudaGraphSetConditional(h, (st->done || st->iter > cap) ? 0u : 1u);
}

// Multi-rank CG: the scalar updates, with the sums all-reduced over the ranks
// (red[] holds them); one thread. Each kernel returns when the phase it
// follows did not reduce (solve finished, or residual not due).
__global__ void shard_alpha_kernel(SolverState* st) {
  if (st->done) return;
  st->omega = st->red[0];
  st->alpha = st->rho / st->red[0];
}
__global__ void shard_cg_kernel(SolverState* st, double* hist) {
  if (st->done || (st->iter % st->iter_rr) == 0) return;
  fin_cg(st, st->red[0], st->red[1], hist);
}
__global__ void shard_resid_kernel(SolverState* st, double* hist, int mode) {
  if (st->done || !(st->iter == 0 || st->rr_flag)) return;
  st->rr_flag = 0;
  if (mode == 0) fin_cg(st, st->red[0], st->red[1], hist);
  else if (mode == 2) fin_pipe_check(st, st->red[0], hist);
  else fin_bicg(st, st->red[0], st->red[1], hist);
}

// ---------------------------------------------------------------------------
// PipeCG kernels (src/iterative/PipeCG.f90:87-149). One iteration: the two
// dots and M = M^-1 V in one pass, L = A M, then every vector update with
// <R,R> in one pass; the replacement iteration (iter % iter_RR == 0)
// recomputes R = B - A X, U = M^-1 R and V = A U instead of the R, U, V
// recurrences.
// ---------------------------------------------------------------------------
// gamma = <R,U>, delta = <V,U>; M = M^-1 V
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    pipe_dots_kernel(int N, const T* __restrict__ r, const T* __restrict__ u, const T* __restrict__ vv,
                     T* __restrict__ mm, const T* __restrict__ alu, int prec, double* partials, unsigned int* ticket,
                     SolverState* st) {
  if (st->done) return;
  DotAcc<2, T> v;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < N; row += gridDim.x * blockDim.x) {
    T w[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      const T uv = u[i];
      w[c] = vv[i];
      v.add(0, r[i], uv);
      v.add(1, w[c], uv);
    }
    if (prec) diag_row<B, T>(alu, N, row, w);
#pragma unroll
    for (int c = 0; c < B; c++) mm[(long long)row * B + c] = w[c];
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // the scalars after the all-reduce (shard_pipe_dots_kernel)
      st->red[0] = tot[0];
      st->red[1] = tot[1];
      return;
    }
    fin_pipe_dots(st, tot[0], tot[1]);
  });
}

// out = A in (no dot)
template <int B, int U, class V, class T>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks<B>::value)
    pipe_spmv_kernel(SellView<V> A, const T* __restrict__ in, T* __restrict__ out, const SolverState* st) {
  if (st->done) return;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < A.N; row += gridDim.x * blockDim.x) {
    T y[B];
    sell_row<B, U, V, T>(A, in, row, y);
#pragma unroll
    for (int c = 0; c < B; c++) out[(long long)row * B + c] = y[c];
  }
}

// Z = beta Z + L, Q = beta Q + M, S = beta S + V, P = beta P + U; then
// R -= alpha S, U -= alpha Q, V -= alpha Z, X += alpha P and <R,R>, or on a
// replacement iteration X += alpha P only (the residual kernel follows).
// Each update is the reference's AXPBY with a unit second factor: two
// roundings.
template <class T>
__global__ void __launch_bounds__(kThreads)
    pipe_update_kernel(long long n, T* __restrict__ x, T* __restrict__ r, T* __restrict__ u, T* __restrict__ vv,
                       T* __restrict__ q, T* __restrict__ p, T* __restrict__ z, const T* __restrict__ l,
                       const T* __restrict__ mm, T* __restrict__ s, double* partials, unsigned int* ticket,
                       SolverState* st, double* hist) {
  if (st->done) return;
  const bool rr_iter = (st->iter % st->iter_rr) == 0;
  const T alpha = (T)st->alpha, beta = (T)st->beta;
  DotAcc<1, T> v;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const T zi = add_rn(mul_rn(beta, z[i]), l[i]);
    const T qi = add_rn(mul_rn(beta, q[i]), mm[i]);
    const T vi = vv[i];
    const T si = add_rn(mul_rn(beta, s[i]), vi);
    const T pi = add_rn(mul_rn(beta, p[i]), u[i]);
    z[i] = zi;
    q[i] = qi;
    s[i] = si;
    p[i] = pi;
    if (!rr_iter) {
      const T ri = add_rn(mul_rn(-alpha, si), r[i]);
      r[i] = ri;
      u[i] = add_rn(mul_rn(-alpha, qi), u[i]);
      vv[i] = add_rn(mul_rn(-alpha, zi), vi);
      v.add(0, ri, ri);
    }
    x[i] = add_rn(mul_rn(alpha, pi), x[i]);
  }
  if (rr_iter) {
    if (blockIdx.x == 0 && threadIdx.x == 0) st->rr_flag = 1;
    return;
  }
  grid_reduce<1>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // the check after the all-reduce (shard_pipe_check_kernel)
      st->red[0] = tot[0];
      return;
    }
    fin_pipe_check(st, tot[0], hist);
  });
}

// Multi-rank PipeCG: the scalar steps with the all-reduced sums in red[].
__global__ void shard_pipe_dots_kernel(SolverState* st) {
  if (st->done) return;
  fin_pipe_dots(st, st->red[0], st->red[1]);
}
__global__ void shard_pipe_check_kernel(SolverState* st, double* hist) {
  if (st->done || (st->iter % st->iter_rr) == 0) return;
  fin_pipe_check(st, st->red[0], hist);
}

// ---------------------------------------------------------------------------
// GropCG kernels (src/iterative/GropCG.f90:88-125): delta = <P,S> with
// Q = M^-1 S; the X, R, U updates with <R,U> and <R,R>; V = A U with the P and
// S updates (one rank: fused; several: V stored while the sums of the
// previous pass are all-reduced, then the P, S pass).
// ---------------------------------------------------------------------------
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    grop_q_kernel(int N, const T* __restrict__ p, const T* __restrict__ s, T* __restrict__ q,
                  const T* __restrict__ alu, int prec, double* partials, unsigned int* ticket, SolverState* st) {
  if (st->done) return;
  DotAcc<1, T> v;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < N; row += gridDim.x * blockDim.x) {
    T w[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      w[c] = s[i];
      v.add(0, p[i], w[c]);
    }
    if (prec) diag_row<B, T>(alu, N, row, w);
#pragma unroll
    for (int c = 0; c < B; c++) q[(long long)row * B + c] = w[c];
  }
  grid_reduce<1>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {
      st->red[0] = tot[0];
      return;
    }
    fin_grop_alpha(st, tot[0]);
  });
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    grop_update_kernel(long long n, T* __restrict__ x, T* __restrict__ r, T* __restrict__ u,
                       const T* __restrict__ p, const T* __restrict__ s, const T* __restrict__ q, double* partials,
                       unsigned int* ticket, SolverState* st, double* hist) {
  if (st->done) return;
  const T alpha = (T)st->alpha;
  DotAcc<2, T> v;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] = add_rn(mul_rn(alpha, p[i]), x[i]);
    const T ri = add_rn(mul_rn(-alpha, s[i]), r[i]);
    const T ui = add_rn(mul_rn(-alpha, q[i]), u[i]);
    r[i] = ri;
    u[i] = ui;
    v.add(0, ri, ui);
    v.add(1, ri, ri);
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {
      st->red[0] = tot[0];
      st->red[1] = tot[1];
      return;
    }
    fin_grop(st, tot[0], tot[1], hist);
  });
}

// V = A U, P = beta P + U, S = beta S + V (one rank: V is not stored)
template <int B, int U, class V, class T>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks<B>::value)
    grop_spmv_kernel(SellView<V> A, const T* __restrict__ u, T* __restrict__ p, T* __restrict__ s,
                     const SolverState* st) {
  if (st->done) return;
  const T beta = (T)st->beta;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < A.N; row += gridDim.x * blockDim.x) {
    T y[B];
    sell_row<B, U, V, T>(A, u, row, y);
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      p[i] = add_rn(mul_rn(beta, p[i]), u[i]);
      s[i] = add_rn(mul_rn(beta, s[i]), y[c]);
    }
  }
}

// P = beta P + U, S = beta S + V (several ranks, after the all-reduce)
template <class T>
__global__ void grop_ps_kernel(long long n, T* __restrict__ p, T* __restrict__ s, const T* __restrict__ u,
                               const T* __restrict__ vv, const SolverState* st) {
  if (st->done) return;
  const T beta = (T)st->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    p[i] = add_rn(mul_rn(beta, p[i]), u[i]);
    s[i] = add_rn(mul_rn(beta, s[i]), vv[i]);
  }
}

__global__ void shard_grop_alpha_kernel(SolverState* st) {
  if (st->done) return;
  fin_grop_alpha(st, st->red[0]);
}
__global__ void shard_grop_kernel(SolverState* st, double* hist) {
  if (st->done) return;
  fin_grop(st, st->red[0], st->red[1], hist);
}

// ---------------------------------------------------------------------------
// BiCGSTAB kernels (src/iterative/BiCGSTAB.f90:87-170)
// ---------------------------------------------------------------------------
// P = R + beta*(P - omega*V) (or P = R on iteration 1); PT = M^-1 P.
// Mixed precision (x64 != null): after a refresh it also folds the FP32
// correction into the FP64 solution, X += Y, Y = 0, on the ghost entries
// [N*B, n_ext) as well (several ranks: the owners' arithmetic, so the
// refresh can multiply x + y there). Register-blocked like cg_update_kernel
// (the work vectors are the solver's own, 16-byte aligned).
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    bicg_p_kernel(int N, T* __restrict__ p, const T* __restrict__ r, const T* __restrict__ vv,
                  T* __restrict__ pt, const T* __restrict__ alu, int prec, const SolverState* st,
                  double* __restrict__ x64 = nullptr, T* __restrict__ yacc = nullptr, long long n_ext = 0) {
  using RG = RowGroup<T, B>;
  constexpr int R = RG::R, E = RG::E;
  if (st->done) return;
  const bool first = st->iter == 1;
  const bool fold = x64 && st->fold;
  const T beta = (T)st->beta, omega = (T)st->omega;
  const bool alu_vec = (N % R) == 0;
  const long long ngroups = N / R;
  const long long stride = (long long)gridDim.x * blockDim.x;
  auto pval = [&](T rv, T pv, T vv_) { return first ? rv : add_rn(rv, mul_rn(beta, sub_rn(pv, mul_rn(omega, vv_)))); };
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ngroups; g += stride) {
    const long long row0 = g * R, e0 = row0 * B;
    T rv[E], pv[E], w[E];
    vload<T, E>(r + e0, rv);
    if (!first) {
      T vvv[E];
      vload<T, E>(p + e0, pv);
      vload<T, E>(vv + e0, vvv);
#pragma unroll
      for (int i = 0; i < E; i++) pv[i] = pval(rv[i], pv[i], vvv[i]);
    } else {
#pragma unroll
      for (int i = 0; i < E; i++) pv[i] = rv[i];
    }
    vstore<T, E>(p + e0, pv);
#pragma unroll
    for (int i = 0; i < E; i++) w[i] = pv[i];
    if (prec) diag_rows<B, T, R>(alu, N, row0, alu_vec, w);
    vstore<T, E>(pt + e0, w);
    if (fold) {
#pragma unroll
      for (int i = 0; i < E; i++) {
        x64[e0 + i] += (double)yacc[e0 + i];
        yacc[e0 + i] = (T)0;
      }
    }
  }
  for (long long row = ngroups * R + blockIdx.x * (long long)blockDim.x + threadIdx.x; row < N; row += stride) {
    T w[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = row * B + c;
      const T pv = first ? r[i] : pval(r[i], p[i], vv[i]);
      p[i] = pv;
      w[c] = pv;
      if (fold) {
        x64[i] += (double)yacc[i];
        yacc[i] = (T)0;
      }
    }
    if (prec) diag_row<B, T>(alu, N, (int)row, w);
#pragma unroll
    for (int c = 0; c < B; c++) pt[row * B + c] = w[c];
  }
  if (fold)
    for (long long i = (long long)N * B + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_ext; i += stride) {
      x64[i] += (double)yacc[i];
      yacc[i] = (T)0;
    }
}

// V = A PT; c2 = <RT,V>; alpha = rho/c2 (BiCGSTAB.f90:113-123)
template <int B, int U, class V, class T, bool kSet = false>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks<B>::value)
    bicg_v_kernel(SellView<V> A, const T* __restrict__ pt, T* __restrict__ vv, const T* __restrict__ rt,
                  double* partials, unsigned int* ticket, SolverState* st, RowSet rs, int acc) {
  if (st->done) return;
  DotAcc<1, T> v;
  for_rows<kSet>(rs, A.N, [&](int row) {
    T y[B];
    sell_row<B, U, V, T>(A, pt, row, y);
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      vv[i] = y[c];
      v.add(0, rt[i], y[c]);
    }
  });
  grid_reduce<1>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // alpha after the all-reduce (shard_bicg_alpha_kernel); acc as cg_spmv
      st->red[0] = acc ? st->red[0] + tot[0] : tot[0];
      return;
    }
    st->c2 = tot[0];
    if (tot[0] == 0.0) { st->done = 1; st->status = kBreakdown; return; }
    st->alpha = st->rho / tot[0];
  });
}

// S = -alpha*V + R; ST = M^-1 S (BiCGSTAB.f90:124-126). Register-blocked.
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    bicg_s_kernel(int N, T* __restrict__ s, const T* __restrict__ r, const T* __restrict__ vv,
                  T* __restrict__ stv, const T* __restrict__ alu, int prec, const SolverState* st) {
  using RG = RowGroup<T, B>;
  constexpr int R = RG::R, E = RG::E;
  if (st->done) return;
  const T alpha = (T)st->alpha;
  const bool alu_vec = (N % R) == 0;
  const long long ngroups = N / R;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ngroups; g += stride) {
    const long long row0 = g * R, e0 = row0 * B;
    T rv[E], vvv[E], w[E];
    vload<T, E>(r + e0, rv);
    vload<T, E>(vv + e0, vvv);
#pragma unroll
    for (int i = 0; i < E; i++) rv[i] = axpy_rn(-alpha, vvv[i], rv[i]);
    vstore<T, E>(s + e0, rv);
#pragma unroll
    for (int i = 0; i < E; i++) w[i] = rv[i];
    if (prec) diag_rows<B, T, R>(alu, N, row0, alu_vec, w);
    vstore<T, E>(stv + e0, w);
  }
  for (long long row = ngroups * R + blockIdx.x * (long long)blockDim.x + threadIdx.x; row < N; row += stride) {
    T w[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = row * B + c;
      w[c] = axpy_rn(-alpha, vv[i], r[i]);
      s[i] = w[c];
    }
    if (prec) diag_row<B, T>(alu, N, (int)row, w);
#pragma unroll
    for (int c = 0; c < B; c++) stv[row * B + c] = w[c];
  }
}

// T = A ST; (T,S), (T,T); omega = (T,S)/(T,T) or 0 (BiCGSTAB.f90:128-146)
template <int B, int U, class V, class T, bool kSet = false>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks<B>::value)
    bicg_t_kernel(SellView<V> A, const T* __restrict__ stv, T* __restrict__ t, const T* __restrict__ s,
                  double* partials, unsigned int* ticket, SolverState* st, RowSet rs, int acc) {
  if (st->done) return;
  DotAcc<2, T> v;
  for_rows<kSet>(rs, A.N, [&](int row) {
    T y[B];
    sell_row<B, U, V, T>(A, stv, row, y);
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      t[i] = y[c];
      v.add(0, y[c], s[i]);
      v.add(1, y[c], y[c]);
    }
  });
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // omega after the all-reduce (shard_bicg_omega_kernel); acc as cg_spmv
      st->red[0] = acc ? st->red[0] + tot[0] : tot[0];
      st->red[1] = acc ? st->red[1] + tot[1] : tot[1];
      return;
    }
    st->ts = tot[0];
    st->tt = tot[1];
    st->omega = tot[1] == 0.0 ? 0.0 : tot[0] / tot[1];
  });
}

// X = X + alpha*PT + omega*ST; R = -omega*T + S; <R,R>, <R,RT>
// (BiCGSTAB.f90:148-164). On iter % iter_RR == 0 only X is updated here.
// n_ghost entries after the owned ones get the X update too (the FP32
// correction of the multi-rank refined solve, kept with the owners'
// arithmetic; PT and ST hold their ghost entries after the halo updates).
__device__ void fin_mixed_bicg(SolverState* st, double rr, double rrt, double* hist);

template <int B, class T, bool Mixed = false>
__global__ void __launch_bounds__(kThreads)
    bicg_xr_kernel(int N, T* __restrict__ x, const T* __restrict__ pt, const T* __restrict__ stv,
                   T* __restrict__ r, const T* __restrict__ s, const T* __restrict__ t, const T* __restrict__ rt,
                   double* partials, unsigned int* ticket, SolverState* st, double* hist, long long n_ghost) {
  constexpr int W = Vec16T<T>::n;  // elements per 16-byte access
  if (st->done) return;
  const bool rr_iter = (st->iter % st->iter_rr) == 0;
  const T alpha = (T)st->alpha, omega = (T)st->omega;
  const long long n = (long long)N * B;
  // x is the caller's vector: 16-byte accesses only when it is aligned
  const long long nv = ((reinterpret_cast<uintptr_t>(x) & 15) == 0) ? n / W : 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  DotAcc<2, T> v;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nv; q += stride) {
    const long long i0 = q * W;
    T xv[W], ptv[W], sv_[W];
    vload<T, W>(x + i0, xv);
    vload<T, W>(pt + i0, ptv);
    vload<T, W>(stv + i0, sv_);
#pragma unroll
    for (int k = 0; k < W; k++) xv[k] = add_rn(add_rn(xv[k], mul_rn(alpha, ptv[k])), mul_rn(omega, sv_[k]));
    vstore<T, W>(x + i0, xv);
    if (!rr_iter) {
      T tv[W], ssv[W], rtv[W];
      vload<T, W>(t + i0, tv);
      vload<T, W>(s + i0, ssv);
      vload<T, W>(rt + i0, rtv);
#pragma unroll
      for (int k = 0; k < W; k++) {
        tv[k] = axpy_rn(-omega, tv[k], ssv[k]);
        v.add(0, tv[k], tv[k]);
        v.add(1, tv[k], rtv[k]);
      }
      vstore<T, W>(r + i0, tv);
    }
  }
  for (long long i = n + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n + n_ghost; i += stride)
    x[i] = add_rn(add_rn(x[i], mul_rn(alpha, pt[i])), mul_rn(omega, stv[i]));
  for (long long i = nv * W + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    x[i] = add_rn(add_rn(x[i], mul_rn(alpha, pt[i])), mul_rn(omega, stv[i]));
    if (!rr_iter) {
      const T rv = axpy_rn(-omega, t[i], s[i]);
      r[i] = rv;
      v.add(0, rv, rv);
      v.add(1, rv, rt[i]);
    }
  }
  if (rr_iter) {
    if (blockIdx.x == 0 && threadIdx.x == 0) st->rr_flag = 1;
    return;
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // fin_bicg / fin_mixed_bicg after the all-reduce (shard_bicg_kernel, shard_mbicg_kernel)
      st->red[0] = tot[0];
      st->red[1] = tot[1];
      return;
    }
    if (Mixed) fin_mixed_bicg(st, tot[0], tot[1], hist);
    else fin_bicg(st, tot[0], tot[1], hist);
  });
}

// Multi-rank BiCGSTAB: the scalar steps with the all-reduced sums in red[].
__global__ void shard_bicg_alpha_kernel(SolverState* st) {
  if (st->done) return;
  st->c2 = st->red[0];
  if (st->red[0] == 0.0) { st->done = 1; st->status = kBreakdown; return; }
  st->alpha = st->rho / st->red[0];
}
__global__ void shard_bicg_omega_kernel(SolverState* st) {
  if (st->done) return;
  st->ts = st->red[0];
  st->tt = st->red[1];
  st->omega = st->red[1] == 0.0 ? 0.0 : st->red[0] / st->red[1];
}
__global__ void shard_bicg_kernel(SolverState* st, double* hist) {
  if (st->done || (st->iter % st->iter_rr) == 0) return;
  fin_bicg(st, st->red[0], st->red[1], hist);
}

// ---------------------------------------------------------------------------
// Mixed precision CG: FP32 matrix (paired layout), vectors and arithmetic in
// the loop; FP64 accumulation of every dot product and FP64 scalars. The
// FP64 solution is x + y, with y the FP32 correction accumulated since the
// last refresh. When the iterated residual norm has dropped below `delta`
// times its largest value since the last refresh (which bounds the range
// that y and the FP32 recursion must carry), when `period` iterations have
// passed without one, or when it looks converged, the solver recomputes
// r = b - A (x + y) with the FP64 matrix and continues from it with the same
// search direction p ("reliable update", Sleijpen & van der Vorst 1996).
// Convergence is decided only on that FP64 residual. The fold x += y, y = 0
// is done by the next p update (or after the loop).
// ---------------------------------------------------------------------------
__device__ void fin_mixed_inner(SolverState* st, double rr, double rz, double* hist) {
  const double rn = sqrt(rr);
  const double resid = sqrt(rr / st->B2);
  record(st, hist, resid);
  st->rho1 = st->rho;
  if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
  if (rn > st->rmax) st->rmax = rn;
  if (rn < st->delta * st->rmax || resid < st->tol || st->iter >= st->max_iter ||
      (st->period > 0 && st->iter - st->last_refresh >= st->period)) {
    st->refresh = 1;  // the refresh kernel of this iteration finishes it
    return;
  }
  st->rho = rz;
  st->beta = st->rho / st->rho1;
  st->iter += 1;
}

// Mixed precision BiCGSTAB: the same scheme on src/iterative/BiCGSTAB.f90's
// recurrences. X + Y is the solution (Y accumulates alpha*PT + omega*ST in
// FP32); a refresh recomputes R = B - A (X + Y) in FP64 and continues with
// rho = <R,RT> of that residual, the shadow residual RT and P, V unchanged
// (the reference's own true-residual replacement, made adaptive).
__device__ void fin_mixed_bicg(SolverState* st, double rr, double rrt, double* hist) {
  const double rn = sqrt(rr);
  const double resid = sqrt(rr / st->B2);
  record(st, hist, resid);
  st->rho1 = st->rho;
  if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
  if (rn > st->rmax) st->rmax = rn;
  if (rn < st->delta * st->rmax || resid < st->tol || st->iter >= st->max_iter ||
      (st->period > 0 && st->iter - st->last_refresh >= st->period)) {
    st->refresh = 1;
    return;
  }
  st->rho = rrt;
  if (rrt == 0.0) { st->done = 1; st->status = kBreakdown; return; }
  st->beta = (st->rho / st->rho1) * (st->alpha / st->omega);
  st->iter += 1;
}

// V = A PT (FP32 paired layout); c2 = <RT,V>; alpha = rho/c2.
template <int B, int U>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks2<B>::value)
    mbicg_v_kernel(SellView2 A, const float* __restrict__ pt, float* __restrict__ vv, const float* __restrict__ rt,
                   double* partials, unsigned int* ticket, SolverState* st) {
  if (st->done) return;
  PlainAcc<1> v;
  const int npairs = (A.N + 1) / 2;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npairs; t += gridDim.x * blockDim.x) {
    float y0[B], y1[B];
    sell_row2<B, U>(A, pt, t, y0, y1);
    const int nr = (2 * t + 1 < A.N) ? 2 : 1;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (h >= nr) break;
#pragma unroll
      for (int c = 0; c < B; c++) {
        const long long i = (long long)(2 * t + h) * B + c;
        const float yv = h ? y1[c] : y0[c];
        vv[i] = yv;
        v.add(0, rt[i], yv);
      }
    }
  }
  grid_reduce<1>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // alpha after the all-reduce (shard_mbicg_alpha_kernel)
      st->red[0] = tot[0];
      return;
    }
    st->c2 = tot[0];
    st->fold = 0;  // the p kernel of this iteration has folded y
    if (tot[0] == 0.0) { st->done = 1; st->status = kBreakdown; return; }
    st->alpha = st->rho / tot[0];
  });
}

// T = A ST (FP32 paired layout); (T,S), (T,T); omega.
template <int B, int U>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks2<B>::value)
    mbicg_t_kernel(SellView2 A, const float* __restrict__ stv, float* __restrict__ t, const float* __restrict__ s,
                   double* partials, unsigned int* ticket, SolverState* st) {
  if (st->done) return;
  PlainAcc<2> v;
  const int npairs = (A.N + 1) / 2;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npairs; q += gridDim.x * blockDim.x) {
    float y0[B], y1[B];
    sell_row2<B, U>(A, stv, q, y0, y1);
    const int nr = (2 * q + 1 < A.N) ? 2 : 1;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (h >= nr) break;
#pragma unroll
      for (int c = 0; c < B; c++) {
        const long long i = (long long)(2 * q + h) * B + c;
        const float yv = h ? y1[c] : y0[c];
        t[i] = yv;
        v.add(0, yv, s[i]);
        v.add(1, yv, yv);
      }
    }
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // omega after the all-reduce (shard_bicg_omega_kernel)
      st->red[0] = tot[0];
      st->red[1] = tot[1];
      return;
    }
    st->ts = tot[0];
    st->tt = tot[1];
    st->omega = tot[1] == 0.0 ? 0.0 : tot[0] / tot[1];
  });
}

// Multi-rank FP32-refined BiCGSTAB: the scalar steps with the all-reduced
// sums in red[] (omega: shard_bicg_omega_kernel).
__global__ void shard_mbicg_alpha_kernel(SolverState* st) {
  if (st->done) return;
  st->c2 = st->red[0];
  st->fold = 0;
  if (st->red[0] == 0.0) { st->done = 1; st->status = kBreakdown; return; }
  st->alpha = st->rho / st->red[0];
}
__global__ void shard_mbicg_kernel(SolverState* st, double* hist) {
  if (st->done) return;
  fin_mixed_bicg(st, st->red[0], st->red[1], hist);
}

// P = Z + beta*P in FP32 (P = Z on iteration 1), and after a refresh the
// fold of the FP32 correction into the FP64 solution: X += Y, Y = 0.
__global__ void mixed_p_kernel(long long n, float* __restrict__ p, const float* __restrict__ z,
                               double* __restrict__ x, float* __restrict__ y, const SolverState* st,
                               long long n_fold = 0) {
  if (st->done) return;
  const bool first = st->iter == 1;
  const bool fold = st->fold != 0;
  const float beta = (float)st->beta;
  const bool xal = (reinterpret_cast<uintptr_t>(x) & 15) == 0;
  const long long nv = n / 4;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += stride) {
    float4 zv = reinterpret_cast<const float4*>(z)[i];
    if (!first) {
      const float4 pv = reinterpret_cast<const float4*>(p)[i];
      zv.x = fmaf(beta, pv.x, zv.x);
      zv.y = fmaf(beta, pv.y, zv.y);
      zv.z = fmaf(beta, pv.z, zv.z);
      zv.w = fmaf(beta, pv.w, zv.w);
    }
    reinterpret_cast<float4*>(p)[i] = zv;
    if (fold) {
      const float4 yv = reinterpret_cast<const float4*>(y)[i];
      if (xal) {
        double2 a = reinterpret_cast<double2*>(x)[2 * i];
        double2 b = reinterpret_cast<double2*>(x)[2 * i + 1];
        a.x += (double)yv.x;
        a.y += (double)yv.y;
        b.x += (double)yv.z;
        b.y += (double)yv.w;
        reinterpret_cast<double2*>(x)[2 * i] = a;
        reinterpret_cast<double2*>(x)[2 * i + 1] = b;
      } else {
        x[4 * i] += (double)yv.x;
        x[4 * i + 1] += (double)yv.y;
        x[4 * i + 2] += (double)yv.z;
        x[4 * i + 3] += (double)yv.w;
      }
      reinterpret_cast<float4*>(y)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  for (long long i = nv * 4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    p[i] = first ? z[i] : fmaf(beta, p[i], z[i]);
    if (fold) {
      x[i] += (double)y[i];
      y[i] = 0.0f;
    }
  }
  // several ranks: the ghost rows of x and y follow their owners' (same fold)
  if (fold)
    for (long long i = n + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_fold; i += stride) {
      x[i] += (double)y[i];
      y[i] = 0.0f;
    }
}

// FP32 paired-layout SpMV fused with <P,Q> (mixed precision inner loop).
template <int B, int U>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks2<B>::value)
    cg_spmv2_kernel(SellView2 A, const float* __restrict__ p, float* __restrict__ q, double* partials,
                    unsigned int* ticket, SolverState* st) {
  if (st->done) return;
  PlainAcc<1> v;
  const int npairs = (A.N + 1) / 2;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npairs; t += gridDim.x * blockDim.x) {
    float y0[B], y1[B];
    sell_row2<B, U>(A, p, t, y0, y1);
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)2 * t * B + c;
      q[i] = y0[c];
      v.add(0, p[i], y0[c]);
    }
    if (2 * t + 1 < A.N) {
#pragma unroll
      for (int c = 0; c < B; c++) {
        const long long i = (long long)(2 * t + 1) * B + c;
        q[i] = y1[c];
        v.add(0, p[i], y1[c]);
      }
    }
  }
  grid_reduce<1>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // alpha after the all-reduce (shard_mixed_alpha_kernel)
      st->red[0] = tot[0];
      return;
    }
    st->omega = tot[0];
    st->alpha = st->rho / tot[0];
    st->fold = 0;  // the p kernel of this iteration has folded y
  });
}

// y += alpha*p; r -= alpha*q; z = M^-1 r; dots (FP32 vectors, FP64 sums).
// Register-blocked like cg_update_kernel (all vectors are the solver's own,
// allocation-aligned).
template <int B>
__global__ void __launch_bounds__(kThreads)
    mixed_update_kernel(int N, float* __restrict__ y, const float* __restrict__ p, float* __restrict__ r,
                        const float* __restrict__ q, float* __restrict__ z, const float* __restrict__ alu, int prec,
                        double* partials, unsigned int* ticket, SolverState* st, double* hist, int n_ext_rows = 0) {
  using RG = RowGroup<float, B>;
  constexpr int R = RG::R, E = RG::E;
  if (st->done) return;
  const float alpha = (float)st->alpha;
  const bool alu_vec = (N % R) == 0;
  const long long ngroups = N / R;
  const long long stride = (long long)gridDim.x * blockDim.x;
  PlainAcc<2> v;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ngroups; g += stride) {
    const long long row0 = g * R, e0 = row0 * B;
    float yv[E], pv[E], rv[E], qv[E], zv[E];
    vload<float, E>(y + e0, yv);
    vload<float, E>(p + e0, pv);
    vload<float, E>(r + e0, rv);
    vload<float, E>(q + e0, qv);
#pragma unroll
    for (int i = 0; i < E; i++) {
      yv[i] = fmaf(alpha, pv[i], yv[i]);
      rv[i] = fmaf(-alpha, qv[i], rv[i]);
      zv[i] = rv[i];
    }
    if (prec) {
      float L[B * B][R];
      load_alu_rows<float, B, R>(alu, N, row0, alu_vec, L);
#pragma unroll
      for (int k = 0; k < R; k++) {
        float t[B];
#pragma unroll
        for (int c = 0; c < B; c++) t[c] = rv[k * B + c];
        diag_solve<B, float>([&](int j, int kk) { return L[j * B + kk][k]; }, t);
#pragma unroll
        for (int c = 0; c < B; c++) zv[k * B + c] = t[c];
      }
    }
#pragma unroll
    for (int i = 0; i < E; i++) {
      v.add(0, rv[i], rv[i]);
      v.add(1, rv[i], zv[i]);
    }
    vstore<float, E>(y + e0, yv);
    vstore<float, E>(r + e0, rv);
    vstore<float, E>(z + e0, zv);
  }
  for (long long row = ngroups * R + blockIdx.x * (long long)blockDim.x + threadIdx.x; row < N; row += stride) {
    float t[B], w[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = row * B + c;
      y[i] = fmaf(alpha, p[i], y[i]);
      t[c] = fmaf(-alpha, q[i], r[i]);
      r[i] = t[c];
      w[c] = t[c];
    }
    if (prec) diag_row<B, float>(alu, N, (int)row, w);
#pragma unroll
    for (int c = 0; c < B; c++) {
      z[row * B + c] = w[c];
      v.add(0, t[c], t[c]);
      v.add(1, t[c], w[c]);
    }
  }
  // several ranks: y of the ghost rows follows its owner's (p's ghost entries
  // hold the owner's values after this iteration's halo update), so x + y is
  // valid on the ghost rows whenever the FP64 refresh multiplies it
  for (long long i = (long long)N * B + blockIdx.x * (long long)blockDim.x + threadIdx.x;
       i < (long long)n_ext_rows * B; i += stride)
    y[i] = fmaf(alpha, p[i], y[i]);
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // fin_mixed_inner after the all-reduce (shard_mixed_inner_kernel)
      st->red[0] = tot[0];
      st->red[1] = tot[1];
      return;
    }
    fin_mixed_inner(st, tot[0], tot[1], hist);
  });
}

// End of a refresh (or of the initial residual when iter == 0): rr = <r64,r64>,
// rz = <r,z> (CG) or <r,rt> (BiCGSTAB).
template <bool Bicg>
__device__ void fin_mixed_refresh(SolverState* st, double rr, double rz, double* hist) {
  if (st->iter == 0) {
    st->B2 = rr;
    if (rr == 0.0) { st->done = 1; st->status = kZeroRhs; return; }
    st->rmax = sqrt(rr);
    st->rho = rz;
    st->iter = 1;
    return;
  }
  const double resid = sqrt(rr / st->B2);
  record(st, hist, resid);
  st->refresh = 0;
  st->fold = 1;
  st->n_refine += 1;
  st->last_refresh = st->iter;
  if (resid < st->tol) { st->done = 1; st->status = kOk; return; }
  if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
  if (st->iter >= st->max_iter) { st->done = 1; st->status = kMaxIter; return; }
  st->rmax = sqrt(rr);
  st->rho = rz;
  if (Bicg) {
    if (rz == 0.0) { st->done = 1; st->status = kBreakdown; return; }
    st->beta = (st->rho / st->rho1) * (st->alpha / st->omega);
  } else {
    st->beta = st->rho / st->rho1;
  }
  st->iter += 1;
}

// Multi-rank FP32-refined CG: the scalar steps with the all-reduced sums in red[].
__global__ void shard_mixed_alpha_kernel(SolverState* st) {
  if (st->done) return;
  st->omega = st->red[0];
  st->alpha = st->rho / st->red[0];
  st->fold = 0;
}
__global__ void shard_mixed_inner_kernel(SolverState* st, double* hist) {
  if (st->done) return;
  fin_mixed_inner(st, st->red[0], st->red[1], hist);
}
template <bool Bicg>
__global__ void shard_mixed_refresh_kernel(SolverState* st, double* hist) {
  if (st->done || !(st->iter == 0 || st->refresh)) return;
  fin_mixed_refresh<Bicg>(st, st->red[0], st->red[1], hist);
}

// Refresh: r64 = b - A64 (x + y) with the FP64 matrix, r = fp32(r64),
// z = M^-1 r; dots <r64,r64> (the true residual) and <r,z>. Runs for the
// initial residual (iter == 0) and when the update kernel raised `refresh`;
// it sits in every iteration on a small grid, so the common case (nothing
// to do) costs one flag read per block.
// x + y (FP64 solution plus FP32 correction) as the multiplied vector.
struct XPlusY {
  const double* __restrict__ x;
  const float* __restrict__ y;
  __device__ __forceinline__ double operator()(long long i) const { return __ldg(x + i) + (double)__ldg(y + i); }
};

// BiCGSTAB mode (Bicg): the second dot is <r,rt> and the initial refresh
// also sets the shadow residual rt = r (z unused).
template <int B, int U, bool Bicg = false>
__global__ void __launch_bounds__(kThreads, SpmvMinBlocks<B>::value)
    mixed_refresh_kernel(SellView<double> A, const double* __restrict__ x, const float* __restrict__ y,
                         const double* __restrict__ b, float* __restrict__ r, float* __restrict__ z,
                         const float* __restrict__ alu, int prec, double* partials, unsigned int* ticket,
                         SolverState* st, double* hist, float* __restrict__ rt = nullptr) {
  if (st->done || !(st->iter == 0 || st->refresh)) return;
  const bool init = st->iter == 0;
  PlainAcc<2> v;
  const XPlusY xy{x, y};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < A.N; row += gridDim.x * blockDim.x) {
    // (A (x + y))[row] in FP64, blocks in CSR order, U slots in flight
    double ax[B];
    sell_row_f<B, U, double, double>(A, xy, row, ax);
    float t[B], w[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      const double rv = b[i] - ax[c];
      v.s[0] += rv * rv;
      t[c] = (float)rv;
      r[i] = t[c];
      w[c] = t[c];
    }
    if (Bicg) {
#pragma unroll
      for (int c = 0; c < B; c++) {
        const long long i = (long long)row * B + c;
        float rtv;
        if (init) { rt[i] = t[c]; rtv = t[c]; } else { rtv = rt[i]; }
        v.add(1, t[c], rtv);
      }
    } else {
      if (prec) diag_row<B, float>(alu, A.N, row, w);
#pragma unroll
      for (int c = 0; c < B; c++) {
        z[(long long)row * B + c] = w[c];
        v.add(1, t[c], w[c]);
      }
    }
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    if (st->sharded) {  // the finish after the all-reduce (shard_mixed_refresh_kernel)
      st->red[0] = tot[0];
      st->red[1] = tot[1];
      return;
    }
    fin_mixed_refresh<Bicg>(st, tot[0], tot[1], hist);
  });
}

// Final fold x += y after the loop (the solution is x + y).
__global__ void mixed_fold_kernel(long long n, double* __restrict__ x, float* __restrict__ y, const SolverState* st) {
  if (!st->fold) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += (double)y[i];
    y[i] = 0.0f;
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------


// Per-device stream-ordered pool for the solvers' work vectors, owned by the
// library. Its release threshold is unlimited: memory a solve frees stays
// mapped in the pool, and the next solve (of this struct or any other) takes
// it back without mapping pages again (the default pool returns freed memory
// to the driver at every synchronisation, and re-mapping a gigabyte of
// vectors cost milliseconds per solve). Null if it cannot be made (the
// stream's default pool is used then).
cudaMemPool_t work_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  static bool failed[64] = {};
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[d] && !failed[d]) {
    cudaMemPoolProps pr = {};
    pr.allocType = cudaMemAllocationTypePinned;
    pr.handleTypes = cudaMemHandleTypeNone;
    pr.location.type = cudaMemLocationTypeDevice;
    pr.location.id = d;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &pr) != cudaSuccess) {
      failed[d] = true;
      cudaGetLastError();
      return nullptr;
    }
    unsigned long long thr = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &thr);
    pools[d] = p;
  }
  return pools[d];
}

// Work vectors of one solve, from the work pool, freed (back to the pool)
// after the solve.
struct Vecs {
  Scratch& sc;
  cudaStream_t s;
  std::vector<void*> extra;
  ~Vecs() {
    for (void* p : extra) cudaFreeAsync(p, s);
  }
  template <class T>
  T* get(long long n) {
    const size_t bytes = (sizeof(T) * (size_t)(n > 0 ? n : 1) + 16 + 255) / 256 * 256;
    void* p = nullptr;
    cudaMemPool_t pool = work_pool();
    if ((pool ? cudaMallocFromPoolAsync(&p, bytes, pool, s) : cudaMallocAsync(&p, bytes, s)) != cudaSuccess)
      return nullptr;
    extra.push_back(p);
    return static_cast<T*>(p);
  }
};

// One solver as kernel launch sequences.
struct Plan {
  // enqueue one iteration; `special` adds the true-residual kernel (FP64);
  // ev (nullable) receives an event before and after every kernel slot
  std::function<void(cudaStream_t, cudaEvent_t*, bool special)> iteration;
  std::function<void(cudaStream_t)> finalize;  // mixed: final fold
  int kernels = 0;         // kernel slots of an iteration (FP64: the last is the special kernel)
  int launches = 0, launches_special = 0;  // kernels of an iteration, if not one per slot (multi-rank)
  bool always_all = false; // every slot launches every iteration (mixed)
  std::vector<int> kind;   // per slot: 0 SpMV, 1 other vector kernel, 2 precond-applying kernel
};

int largest_divisor_at_most(int v, int cap) {
  for (int d = cap; d > 1; d--)
    if (v % d == 0) return d;
  return 1;
}

}  // namespace

int solve_device(SellMatrix& m, Scratch& sc, const SolveParams& p, const double* d_b, double* d_x,
                 SolveResult& res, double* h_hist, cudaStream_t s) {
  const int N = m.N, nd = m.ndof;
  // Grids: a kernel's persistent grid, or one block per 256 rows when the
  // system is smaller than that, so a small system does not pay for entering
  // and reducing hundreds of idle blocks.
  const int gcap = (int)std::max<long long>(1, ((long long)N + kThreads - 1) / kThreads);
  auto pg = [gcap](auto k) { return std::min(pgrid(k), gcap); };
  const long long n = (long long)N * nd;
  const int prec = p.precond == 1 ? 1 : 0;
  if (prec && !m.have_alu) return kBadInput;
  if (p.method != 1 && p.method != 2 && p.method != 3 && p.method != 5) return kBadInput;
  if ((p.method == 2 || p.method == 3) && p.precision != 0) {
    fprintf(stderr, "** monolis_b200: GropCG and PipeCG run in FP64\n");
    return kBadInput;
  }
  if (p.shard && ((p.precision != 0 && p.method != 1 && p.method != 5) || p.np_rows < N)) {
    fprintf(stderr,
            "** monolis_b200: the multi-rank solve is FP64 (CG, GropCG, PipeCG, BiCGSTAB) or FP32-refined CG or "
            "BiCGSTAB\n");
    return kBadInput;
  }
  // vectors gathered by the SpMV hold the ghost rows too
  const long long n_ext = p.shard ? (long long)p.np_rows * nd : n;
  int rc = scratch_ensure(sc, (size_t)p.max_iter + 2);
  if (rc) return rc;
  if (p.precision == 1) {
    rc = sell_make_fp32(m, s);
    if (rc) return rc;
  }

  // true-residual interval: 200 for CG and BiCGSTAB, 50 for PipeCG (CG.f90:40,
  // BiCGSTAB.f90:41, PipeCG.f90:43)
  const int iter_rr = p.iter_rr > 0 ? p.iter_rr : (p.method == 3 ? 50 : 200);
  // Iterations per graph launch. FP64: the replacement iterations must fall
  // on the last iteration of a batch, so the batch divides iter_RR.
  int batch, period;
  if (p.precision == 1) {
    batch = p.batch > 0 ? p.batch : 16;
    period = 0;  // refreshes are decided on the device
  } else if (p.method == 2) {
    batch = p.batch > 0 ? p.batch : 25;
    period = 0;  // GropCG.f90 runs no true-residual replacement
  } else {
    period = iter_rr;
    batch = p.batch > 0 && iter_rr % p.batch == 0 ? p.batch : largest_divisor_at_most(iter_rr, 25);
  }

  SolverState h{};
  h.tol = p.tol;
  h.max_iter = p.max_iter;
  h.iter_rr = p.precision == 1 ? 0x7fffffff : iter_rr;  // mixed: refreshes replace the fixed schedule
  h.period = p.precision == 1 ? p.refresh_period : 0;
  // BiCGSTAB refreshes more often (its residual norm oscillates, so the
  // drop below the running maximum is measured against a higher peak): 0.2
  // took fewer iterations and less time than 0.01 .. 0.5 on 256^3
  // convection-diffusion at cell Peclet 0.5, 5 and 50
  h.delta = p.delta > 0 ? p.delta : (p.method == 5 ? 0.2 : 0.1);
  h.sharded = p.shard ? 1 : 0;
  MB_CUDA_OK(cudaMemcpyAsync(sc.st, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(cudaMemsetAsync(sc.ticket, 0, sizeof(unsigned int) * kTicketWords, s));
  if (p.init_x) MB_CUDA_OK(cudaMemsetAsync(d_x, 0, sizeof(double) * n_ext, s));

  Vecs vec{sc, s};
  const int gb = blocks_for(N);
  Plan plan;
  auto t0 = std::chrono::steady_clock::now();

  rc = dispatch_ndof(nd, [&](auto Bc) -> int {
   constexpr int B = decltype(Bc)::value;
   return dispatch_u(p.precision == 0 ? m.u64 : m.u32, [&](auto Uc) -> int {
    constexpr int U = eff_u(B, decltype(Uc)::value);
    SellView<double> A64 = view_of<double>(m);
    double* partials = sc.partials;
    unsigned int* ticket = sc.ticket;
    SolverState* st = sc.st;
    double* hist = sc.hist;
    const int gvec = (int)std::min<long long>(num_sms() * 8, std::max<long long>(1, (n + kThreads - 1) / kThreads));
    if (p.precision == 0) {
      const double* alu = m.d_alu64;
      double* x = d_x;
      const double* b = d_b;
      auto k_resid = resid_kernel<B, U, double, double>;
      const int g_resid = pg(k_resid);
      if (p.method == 1 && p.shard) {
        // multi-rank CG: halo updates before the products, all-reduced dots
        const ShardPlan* sp = p.shard;
        double *r = vec.get<double>(n), *z = vec.get<double>(n), *q = vec.get<double>(n),
               *pp = vec.get<double>(n_ext);
        if (!r || !z || !q || !pp) return kCudaError;
        if (cudaMemsetAsync(pp, 0, sizeof(double) * n_ext, s) != cudaSuccess) return kCudaError;
        auto k_spmv = cg_spmv_kernel<B, U, double, double, true>;
        auto k_upd = cg_update_kernel<B, double>;
        const int g_spmv = pg(k_spmv), g_upd = pg(k_upd);
        int rc2 = shard_halo(*sp, x, s);
        k_resid<<<g_resid, kThreads, 0, s>>>(A64, x, b, r, z, nullptr, alu, prec, 0, partials, ticket, st, hist);
        if (!rc2) rc2 = shard_allreduce(*sp, st->red, 2, s);
        shard_resid_kernel<<<1, 1, 0, s>>>(st, hist, 0);
        if (rc2) return rc2;
        const int hk = (sp->n_send > 0) + (sp->n_recv > 0);  // pack / unpack kernels of a halo update
        const int nb = sp->n_bnd > 0;                         // boundary-slice product
        const RowSet rs_int{sp->d_slices, sp->n_int}, rs_bnd{sp->d_slices + sp->n_int, sp->n_bnd};
        const int g_bnd = std::max(1, std::min(g_spmv, (int)(((long long)sp->n_bnd * kSlice + kThreads - 1) / kThreads)));
        plan.kernels = 5;
        plan.launches = 5 + hk + nb;
        plan.launches_special = 6 + 2 * hk + nb;
        plan.kind = {1, 0, 2, 1, 0};
        plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool special) {
          if (ev) cudaEventRecord(ev[0], ss);
          cg_p_kernel<double><<<gvec, kThreads, 0, ss>>>(n, pp, z, st);
          if (ev) cudaEventRecord(ev[1], ss);
          // interior rows while the halo update is in flight, then the boundary rows
          shard_halo_fork(*sp, pp, ss);
          k_spmv<<<g_spmv, kThreads, 0, ss>>>(A64, pp, q, partials, ticket, st, rs_int, 0);
          shard_halo_join(*sp, ss);
          if (nb) k_spmv<<<g_bnd, kThreads, 0, ss>>>(A64, pp, q, partials, ticket, st, rs_bnd, 1);
          shard_allreduce(*sp, st->red, 1, ss);
          shard_alpha_kernel<<<1, 1, 0, ss>>>(st);
          if (ev) cudaEventRecord(ev[2], ss);
          k_upd<<<g_upd, kThreads, 0, ss>>>(N, x, pp, r, q, z, alu, prec, partials, ticket, st, hist);
          if (ev) cudaEventRecord(ev[3], ss);
          if (!special) {
            shard_allreduce(*sp, st->red, 2, ss);
            shard_cg_kernel<<<1, 1, 0, ss>>>(st, hist);
          }
          if (ev) cudaEventRecord(ev[4], ss);
          if (special) {
            shard_halo(*sp, x, ss);
            k_resid<<<g_resid, kThreads, 0, ss>>>(A64, x, b, r, z, nullptr, alu, prec, 0, partials, ticket, st, hist);
            shard_allreduce(*sp, st->red, 2, ss);
            shard_resid_kernel<<<1, 1, 0, ss>>>(st, hist, 0);
          }
          if (ev) cudaEventRecord(ev[5], ss);
        };
      } else if (p.method == 2) {
        // GropCG: R, U, V, Q, P, S (GropCG.f90:58-63); V only on several ranks
        const ShardPlan* sp = p.shard;
        double *r = vec.get<double>(n), *u = vec.get<double>(n_ext), *q = vec.get<double>(n),
               *pp = vec.get<double>(n), *sv = vec.get<double>(n), *vv = sp ? vec.get<double>(n) : nullptr;
        if (!r || !u || !q || !pp || !sv || (sp && !vv)) return kCudaError;
        if (n_ext > n && cudaMemsetAsync(u, 0, sizeof(double) * n_ext, s) != cudaSuccess) return kCudaError;
        auto k_q = grop_q_kernel<B, double>;
        auto k_upd = grop_update_kernel<double>;
        auto k_mvps = grop_spmv_kernel<B, U, double, double>;
        auto k_mv = pipe_spmv_kernel<B, U, double, double>;
        const int g_q = pg(k_q), g_upd = pg(k_upd), g_mvps = pg(k_mvps), g_mv = pg(k_mv);
        // R = B - A X, U = M^-1 R, B2 and gamma = <R,U> (CG's initial step);
        // P = U, S = A P (GropCG.f90:67-86)
        int rc2 = sp ? shard_halo(*sp, x, s) : kOk;
        k_resid<<<g_resid, kThreads, 0, s>>>(A64, x, b, r, u, nullptr, alu, prec, 0, partials, ticket, st, hist);
        if (sp) {
          if (!rc2) rc2 = shard_allreduce(*sp, st->red, 2, s);
          shard_resid_kernel<<<1, 1, 0, s>>>(st, hist, 0);
          if (!rc2) rc2 = shard_halo(*sp, u, s);
        }
        if (cudaMemcpyAsync(pp, u, sizeof(double) * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return kCudaError;
        k_mv<<<g_mv, kThreads, 0, s>>>(A64, u, sv, st);
        if (rc2) return rc2;
        const int hk = sp ? (sp->n_send > 0) + (sp->n_recv > 0) : 0;
        plan.kernels = 3;
        plan.kind = {2, 1, 0};
        plan.launches = sp ? 6 + hk : 3;
        plan.launches_special = plan.launches;
        plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool) {
          if (ev) cudaEventRecord(ev[0], ss);
          k_q<<<g_q, kThreads, 0, ss>>>(N, pp, sv, q, alu, prec, partials, ticket, st);
          if (sp) {
            shard_allreduce(*sp, st->red, 1, ss);
            shard_grop_alpha_kernel<<<1, 1, 0, ss>>>(st);
          }
          if (ev) cudaEventRecord(ev[1], ss);
          k_upd<<<g_upd, kThreads, 0, ss>>>(n, x, r, u, pp, sv, q, partials, ticket, st, hist);
          if (ev) cudaEventRecord(ev[2], ss);
          if (sp) {
            // <R,U>, <R,R> all-reduced while V = A U runs (their sums do not feed the product)
            shard_halo(*sp, u, ss);
            shard_allreduce_fork(*sp, st->red, 2, ss);
            k_mv<<<g_mv, kThreads, 0, ss>>>(A64, u, vv, st);
            shard_halo_join(*sp, ss);
            shard_grop_kernel<<<1, 1, 0, ss>>>(st, hist);
            grop_ps_kernel<double><<<gvec, kThreads, 0, ss>>>(n, pp, sv, u, vv, st);
          } else {
            k_mvps<<<g_mvps, kThreads, 0, ss>>>(A64, u, pp, sv, st);
          }
          if (ev) cudaEventRecord(ev[3], ss);
        };
      } else if (p.method == 3 && p.shard) {
        // multi-rank PipeCG: the all-reduce of <R,U>, <V,U> runs on the side
        // stream while this rank multiplies L = A M (PipeCG.f90:88-95: the
        // sums do not feed the product)
        const ShardPlan* sp = p.shard;
        double *r = vec.get<double>(n), *u = vec.get<double>(n_ext), *vv = vec.get<double>(n),
               *q = vec.get<double>(n), *pp = vec.get<double>(n), *z = vec.get<double>(n), *l = vec.get<double>(n),
               *mm = vec.get<double>(n_ext), *sv = vec.get<double>(n);
        if (!r || !u || !vv || !q || !pp || !z || !l || !mm || !sv) return kCudaError;
        for (double* w : {q, pp, z, sv})
          if (cudaMemsetAsync(w, 0, sizeof(double) * n, s) != cudaSuccess) return kCudaError;
        for (double* w : {u, mm})
          if (cudaMemsetAsync(w, 0, sizeof(double) * n_ext, s) != cudaSuccess) return kCudaError;
        auto k_dots = pipe_dots_kernel<B, double>;
        auto k_mv = pipe_spmv_kernel<B, U, double, double>;
        auto k_upd = pipe_update_kernel<double>;
        const int g_dots = pg(k_dots), g_mv = pg(k_mv), g_upd = pg(k_upd);
        int rc2 = shard_halo(*sp, x, s);
        k_resid<<<g_resid, kThreads, 0, s>>>(A64, x, b, r, u, nullptr, alu, prec, 2, partials, ticket, st, hist);
        if (!rc2) rc2 = shard_allreduce(*sp, st->red, 2, s);
        shard_resid_kernel<<<1, 1, 0, s>>>(st, hist, 2);
        if (!rc2) rc2 = shard_halo(*sp, u, s);
        k_mv<<<g_mv, kThreads, 0, s>>>(A64, u, vv, st);
        if (rc2) return rc2;
        const int hk = (sp->n_send > 0) + (sp->n_recv > 0);
        plan.kernels = 5;
        plan.kind = {1, 0, 1, 0, 0};
        plan.launches = 5 + hk;
        plan.launches_special = 7 + 3 * hk;
        plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool special) {
          if (ev) cudaEventRecord(ev[0], ss);
          k_dots<<<g_dots, kThreads, 0, ss>>>(N, r, u, vv, mm, alu, prec, partials, ticket, st);
          if (ev) cudaEventRecord(ev[1], ss);
          shard_halo(*sp, mm, ss);
          shard_allreduce_fork(*sp, st->red, 2, ss);  // in flight during the product
          k_mv<<<g_mv, kThreads, 0, ss>>>(A64, mm, l, st);
          shard_halo_join(*sp, ss);
          shard_pipe_dots_kernel<<<1, 1, 0, ss>>>(st);
          if (ev) cudaEventRecord(ev[2], ss);
          k_upd<<<g_upd, kThreads, 0, ss>>>(n, x, r, u, vv, q, pp, z, l, mm, sv, partials, ticket, st, hist);
          if (!special) {
            shard_allreduce(*sp, st->red, 1, ss);
            shard_pipe_check_kernel<<<1, 1, 0, ss>>>(st, hist);
          }
          if (ev) cudaEventRecord(ev[3], ss);
          if (special) {
            shard_halo(*sp, x, ss);
            k_resid<<<g_resid, kThreads, 0, ss>>>(A64, x, b, r, u, nullptr, alu, prec, 2, partials, ticket, st,
                                                 hist);
            shard_allreduce(*sp, st->red, 2, ss);
            shard_resid_kernel<<<1, 1, 0, ss>>>(st, hist, 2);
          }
          if (ev) cudaEventRecord(ev[4], ss);
          if (special) {
            shard_halo(*sp, u, ss);
            k_mv<<<g_mv, kThreads, 0, ss>>>(A64, u, vv, st);
          }
          if (ev) cudaEventRecord(ev[5], ss);
        };
      } else if (p.method == 3) {
        // PipeCG: R, U, V, Q, P, Z, L, M, S (PipeCG.f90:51-59)
        double *r = vec.get<double>(n), *u = vec.get<double>(n), *vv = vec.get<double>(n), *q = vec.get<double>(n),
               *pp = vec.get<double>(n), *z = vec.get<double>(n), *l = vec.get<double>(n), *mm = vec.get<double>(n),
               *sv = vec.get<double>(n);
        if (!r || !u || !vv || !q || !pp || !z || !l || !mm || !sv) return kCudaError;
        for (double* w : {q, pp, z, sv})  // monolis_alloc_R_1d zero-fills
          if (cudaMemsetAsync(w, 0, sizeof(double) * n, s) != cudaSuccess) return kCudaError;
        auto k_dots = pipe_dots_kernel<B, double>;
        auto k_mv = pipe_spmv_kernel<B, U, double, double>;
        auto k_upd = pipe_update_kernel<double>;
        const int g_dots = pg(k_dots), g_mv = pg(k_mv), g_upd = pg(k_upd);
        // R = B - A X, U = M^-1 R, B2 (PipeCG.f90:67-83); V = A U
        k_resid<<<g_resid, kThreads, 0, s>>>(A64, x, b, r, u, nullptr, alu, prec, 2, partials, ticket, st, hist);
        k_mv<<<g_mv, kThreads, 0, s>>>(A64, u, vv, st);
        plan.kernels = 5;
        plan.kind = {1, 0, 1, 0, 0};
        plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool special) {
          if (ev) cudaEventRecord(ev[0], ss);
          k_dots<<<g_dots, kThreads, 0, ss>>>(N, r, u, vv, mm, alu, prec, partials, ticket, st);
          if (ev) cudaEventRecord(ev[1], ss);
          k_mv<<<g_mv, kThreads, 0, ss>>>(A64, mm, l, st);
          if (ev) cudaEventRecord(ev[2], ss);
          k_upd<<<g_upd, kThreads, 0, ss>>>(n, x, r, u, vv, q, pp, z, l, mm, sv, partials, ticket, st, hist);
          if (ev) cudaEventRecord(ev[3], ss);
          if (special)
            k_resid<<<g_resid, kThreads, 0, ss>>>(A64, x, b, r, u, nullptr, alu, prec, 2, partials, ticket, st, hist);
          if (ev) cudaEventRecord(ev[4], ss);
          if (special) k_mv<<<g_mv, kThreads, 0, ss>>>(A64, u, vv, st);
          if (ev) cudaEventRecord(ev[5], ss);
        };
        plan.launches = 3;
        plan.launches_special = 5;
      } else if (p.method == 1) {
        double *r = vec.get<double>(n), *z = vec.get<double>(n), *q = vec.get<double>(n), *pp = vec.get<double>(n);
        if (!r || !z || !q || !pp) return kCudaError;
        auto k_spmv = cg_spmv_kernel<B, U, double, double>;
        auto k_upd = cg_update_kernel<B, double>;
        const int g_spmv = pg(k_spmv), g_upd = pg(k_upd);
        k_resid<<<g_resid, kThreads, 0, s>>>(A64, x, b, r, z, nullptr, alu, prec, 0, partials, ticket, st, hist);
        plan.kernels = 4;
        plan.kind = {1, 0, 2, 0};
        plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool special) {
          if (ev) cudaEventRecord(ev[0], ss);
          cg_p_kernel<double><<<gvec, kThreads, 0, ss>>>(n, pp, z, st);
          if (ev) cudaEventRecord(ev[1], ss);
          k_spmv<<<g_spmv, kThreads, 0, ss>>>(A64, pp, q, partials, ticket, st, RowSet{nullptr, 0}, 0);
          if (ev) cudaEventRecord(ev[2], ss);
          k_upd<<<g_upd, kThreads, 0, ss>>>(N, x, pp, r, q, z, alu, prec, partials, ticket, st, hist);
          if (ev) cudaEventRecord(ev[3], ss);
          if (special) k_resid<<<g_resid, kThreads, 0, ss>>>(A64, x, b, r, z, nullptr, alu, prec, 0, partials, ticket,
                                                             st, hist);
          if (ev) cudaEventRecord(ev[4], ss);
        };
      } else if (p.shard) {
        // multi-rank BiCGSTAB: halo updates of PT and ST before the products,
        // all-reduced dots (alpha, omega, the residual norms)
        const ShardPlan* sp = p.shard;
        double *r = vec.get<double>(n), *rt = vec.get<double>(n), *pp = vec.get<double>(n),
               *pt = vec.get<double>(n_ext), *sv = vec.get<double>(n), *stv = vec.get<double>(n_ext),
               *t = vec.get<double>(n), *vv = vec.get<double>(n);
        if (!r || !rt || !pp || !pt || !sv || !stv || !t || !vv) return kCudaError;
        if (cudaMemsetAsync(pt, 0, sizeof(double) * n_ext, s) != cudaSuccess ||
            cudaMemsetAsync(stv, 0, sizeof(double) * n_ext, s) != cudaSuccess)
          return kCudaError;
        auto k_v = bicg_v_kernel<B, U, double, double, true>;
        auto k_t = bicg_t_kernel<B, U, double, double, true>;
        auto k_xr = bicg_xr_kernel<B, double>;
        const int g_v = pg(k_v), g_t = pg(k_t), g_xr = pg(k_xr);
        const int g_p = pg(bicg_p_kernel<B, double>), g_s = pg(bicg_s_kernel<B, double>);
        int rc2 = shard_halo(*sp, x, s);
        k_resid<<<g_resid, kThreads, 0, s>>>(A64, x, b, r, nullptr, rt, alu, prec, 1, partials, ticket, st, hist);
        if (!rc2) rc2 = shard_allreduce(*sp, st->red, 2, s);
        shard_resid_kernel<<<1, 1, 0, s>>>(st, hist, 1);
        if (rc2) return rc2;
        const int hk = (sp->n_send > 0) + (sp->n_recv > 0);
        const int nb = sp->n_bnd > 0;
        const RowSet rs_int{sp->d_slices, sp->n_int}, rs_bnd{sp->d_slices + sp->n_int, sp->n_bnd};
        const long long bnd_blocks = ((long long)sp->n_bnd * kSlice + kThreads - 1) / kThreads;
        const int gb_v = std::max(1, (int)std::min<long long>(g_v, bnd_blocks));
        const int gb_t = std::max(1, (int)std::min<long long>(g_t, bnd_blocks));
        plan.kernels = 6;
        plan.launches = 8 + 2 * hk + 2 * nb;
        plan.launches_special = 10 + 3 * hk + 2 * nb;
        plan.kind = {2, 0, 2, 0, 1, 0};
        plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool special) {
          if (ev) cudaEventRecord(ev[0], ss);
          bicg_p_kernel<B, double><<<g_p, kThreads, 0, ss>>>(N, pp, r, vv, pt, alu, prec, st);
          if (ev) cudaEventRecord(ev[1], ss);
          shard_halo_fork(*sp, pt, ss);
          k_v<<<g_v, kThreads, 0, ss>>>(A64, pt, vv, rt, partials, ticket, st, rs_int, 0);
          shard_halo_join(*sp, ss);
          if (nb) k_v<<<gb_v, kThreads, 0, ss>>>(A64, pt, vv, rt, partials, ticket, st, rs_bnd, 1);
          shard_allreduce(*sp, st->red, 1, ss);
          shard_bicg_alpha_kernel<<<1, 1, 0, ss>>>(st);
          if (ev) cudaEventRecord(ev[2], ss);
          bicg_s_kernel<B, double><<<g_s, kThreads, 0, ss>>>(N, sv, r, vv, stv, alu, prec, st);
          if (ev) cudaEventRecord(ev[3], ss);
          shard_halo_fork(*sp, stv, ss);
          k_t<<<g_t, kThreads, 0, ss>>>(A64, stv, t, sv, partials, ticket, st, rs_int, 0);
          shard_halo_join(*sp, ss);
          if (nb) k_t<<<gb_t, kThreads, 0, ss>>>(A64, stv, t, sv, partials, ticket, st, rs_bnd, 1);
          shard_allreduce(*sp, st->red, 2, ss);
          shard_bicg_omega_kernel<<<1, 1, 0, ss>>>(st);
          if (ev) cudaEventRecord(ev[4], ss);
          k_xr<<<g_xr, kThreads, 0, ss>>>(N, x, pt, stv, r, sv, t, rt, partials, ticket, st, hist, 0);
          if (!special) {
            shard_allreduce(*sp, st->red, 2, ss);
            shard_bicg_kernel<<<1, 1, 0, ss>>>(st, hist);
          }
          if (ev) cudaEventRecord(ev[5], ss);
          if (special) {
            shard_halo(*sp, x, ss);
            k_resid<<<g_resid, kThreads, 0, ss>>>(A64, x, b, r, nullptr, rt, alu, prec, 1, partials, ticket, st,
                                                 hist);
            shard_allreduce(*sp, st->red, 2, ss);
            shard_resid_kernel<<<1, 1, 0, ss>>>(st, hist, 1);
          }
          if (ev) cudaEventRecord(ev[6], ss);
        };
      } else {
        double *r = vec.get<double>(n), *rt = vec.get<double>(n), *pp = vec.get<double>(n),
               *pt = vec.get<double>(n), *sv = vec.get<double>(n), *stv = vec.get<double>(n),
               *t = vec.get<double>(n), *vv = vec.get<double>(n);
        if (!r || !rt || !pp || !pt || !sv || !stv || !t || !vv) return kCudaError;
        auto k_v = bicg_v_kernel<B, U, double, double>;
        auto k_t = bicg_t_kernel<B, U, double, double>;
        auto k_xr = bicg_xr_kernel<B, double>;
        const int g_v = pg(k_v), g_t = pg(k_t), g_xr = pg(k_xr);
        const int g_p = pg(bicg_p_kernel<B, double>), g_s = pg(bicg_s_kernel<B, double>);
        k_resid<<<g_resid, kThreads, 0, s>>>(A64, x, b, r, nullptr, rt, alu, prec, 1, partials, ticket, st, hist);
        plan.kernels = 6;
        plan.kind = {2, 0, 2, 0, 1, 0};
        plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool special) {
          if (ev) cudaEventRecord(ev[0], ss);
          bicg_p_kernel<B, double><<<g_p, kThreads, 0, ss>>>(N, pp, r, vv, pt, alu, prec, st);
          if (ev) cudaEventRecord(ev[1], ss);
          k_v<<<g_v, kThreads, 0, ss>>>(A64, pt, vv, rt, partials, ticket, st, RowSet{nullptr, 0}, 0);
          if (ev) cudaEventRecord(ev[2], ss);
          bicg_s_kernel<B, double><<<g_s, kThreads, 0, ss>>>(N, sv, r, vv, stv, alu, prec, st);
          if (ev) cudaEventRecord(ev[3], ss);
          k_t<<<g_t, kThreads, 0, ss>>>(A64, stv, t, sv, partials, ticket, st, RowSet{nullptr, 0}, 0);
          if (ev) cudaEventRecord(ev[4], ss);
          k_xr<<<g_xr, kThreads, 0, ss>>>(N, x, pt, stv, r, sv, t, rt, partials, ticket, st, hist, 0);
          if (ev) cudaEventRecord(ev[5], ss);
          if (special) k_resid<<<g_resid, kThreads, 0, ss>>>(A64, x, b, r, nullptr, rt, alu, prec, 1, partials, ticket,
                                                             st, hist);
          if (ev) cudaEventRecord(ev[6], ss);
        };
      }
    } else if (p.method == 5 && p.shard) {
      // multi-rank FP32-refined BiCGSTAB: FP32 halo updates of PT and ST
      // before the products, every dot product all-reduced, the refresh's
      // all-reduce in every iteration (the refresh is decided on the device,
      // from all-reduced sums, identically on every rank). The ghost entries
      // of y (y += alpha PT + omega ST after both halo updates) and of x (the
      // folds) follow the owners' arithmetic, so the FP64 refresh multiplies
      // x + y on the ghost rows without a halo update of its own.
      const ShardPlan* sp = p.shard;
      SellView2 A32 = view2_of(m);
      const float* alu32 = m.d_alu32;
      float *r = vec.get<float>(n), *rt = vec.get<float>(n), *pp = vec.get<float>(n),
            *pt = vec.get<float>(n_ext), *sv = vec.get<float>(n), *stv = vec.get<float>(n_ext),
            *t = vec.get<float>(n), *vv = vec.get<float>(n), *y = vec.get<float>(n_ext);
      if (!r || !rt || !pp || !pt || !sv || !stv || !t || !vv || !y) return kCudaError;
      double* x = d_x;
      const double* b = d_b;
      auto k_v = mbicg_v_kernel<B, U>;
      auto k_t = mbicg_t_kernel<B, U>;
      auto k_xr = bicg_xr_kernel<B, float, true>;
      auto k_ref = mixed_refresh_kernel<B, U, true>;
      const int g_v = pg(k_v), g_t = pg(k_t), g_xr = pg(k_xr), g_ref = pg(k_ref);
      const int g_p = pg(bicg_p_kernel<B, float>), g_s = pg(bicg_s_kernel<B, float>);
      if (cudaMemsetAsync(y, 0, sizeof(float) * n_ext, s) != cudaSuccess ||
          cudaMemsetAsync(pt, 0, sizeof(float) * n_ext, s) != cudaSuccess ||
          cudaMemsetAsync(stv, 0, sizeof(float) * n_ext, s) != cudaSuccess)
        return kCudaError;
      int rc2 = shard_halo(*sp, x, s);
      k_ref<<<g_ref, kThreads, 0, s>>>(A64, x, y, b, r, nullptr, alu32, prec, partials, ticket, st, hist, rt);
      if (!rc2) rc2 = shard_allreduce(*sp, st->red, 2, s);
      shard_mixed_refresh_kernel<true><<<1, 1, 0, s>>>(st, hist);
      if (rc2) return rc2;
      const int hk = (sp->n_send > 0) + (sp->n_recv > 0);  // pack / unpack kernels of a halo update
      const long long n_ghost = n_ext - n;
      plan.kernels = 6;
      plan.always_all = true;
      plan.launches = 10 + 2 * hk;
      plan.launches_special = plan.launches;
      plan.kind = {2, 0, 2, 0, 1, 0};
      plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool) {
        if (ev) cudaEventRecord(ev[0], ss);
        bicg_p_kernel<B, float><<<g_p, kThreads, 0, ss>>>(N, pp, r, vv, pt, alu32, prec, st, x, y, n_ext);
        if (ev) cudaEventRecord(ev[1], ss);
        shard_halo(*sp, pt, ss);
        k_v<<<g_v, kThreads, 0, ss>>>(A32, pt, vv, rt, partials, ticket, st);
        shard_allreduce(*sp, st->red, 1, ss);
        shard_mbicg_alpha_kernel<<<1, 1, 0, ss>>>(st);
        if (ev) cudaEventRecord(ev[2], ss);
        bicg_s_kernel<B, float><<<g_s, kThreads, 0, ss>>>(N, sv, r, vv, stv, alu32, prec, st);
        if (ev) cudaEventRecord(ev[3], ss);
        shard_halo(*sp, stv, ss);
        k_t<<<g_t, kThreads, 0, ss>>>(A32, stv, t, sv, partials, ticket, st);
        shard_allreduce(*sp, st->red, 2, ss);
        shard_bicg_omega_kernel<<<1, 1, 0, ss>>>(st);
        if (ev) cudaEventRecord(ev[4], ss);
        k_xr<<<g_xr, kThreads, 0, ss>>>(N, y, pt, stv, r, sv, t, rt, partials, ticket, st, hist, n_ghost);
        shard_allreduce(*sp, st->red, 2, ss);
        shard_mbicg_kernel<<<1, 1, 0, ss>>>(st, hist);
        if (ev) cudaEventRecord(ev[5], ss);
        k_ref<<<g_ref, kThreads, 0, ss>>>(A64, x, y, b, r, nullptr, alu32, prec, partials, ticket, st, hist, rt);
        shard_allreduce(*sp, st->red, 2, ss);
        shard_mixed_refresh_kernel<true><<<1, 1, 0, ss>>>(st, hist);
        if (ev) cudaEventRecord(ev[6], ss);
      };
      plan.finalize = [=](cudaStream_t ss) { mixed_fold_kernel<<<gvec, kThreads, 0, ss>>>(n_ext, x, y, st); };
    } else if (p.method == 5) {
      SellView2 A32 = view2_of(m);
      const float* alu32 = m.d_alu32;
      float *r = vec.get<float>(n), *rt = vec.get<float>(n), *pp = vec.get<float>(n), *pt = vec.get<float>(n),
            *sv = vec.get<float>(n), *stv = vec.get<float>(n), *t = vec.get<float>(n), *vv = vec.get<float>(n),
            *y = vec.get<float>(n);
      if (!r || !rt || !pp || !pt || !sv || !stv || !t || !vv || !y) return kCudaError;
      double* x = d_x;
      const double* b = d_b;
      auto k_v = mbicg_v_kernel<B, U>;
      auto k_t = mbicg_t_kernel<B, U>;
      auto k_xr = bicg_xr_kernel<B, float, true>;
      auto k_ref = mixed_refresh_kernel<B, U, true>;
      const int g_v = pg(k_v), g_t = pg(k_t), g_xr = pg(k_xr), g_ref = pg(k_ref);
      const int g_p = pg(bicg_p_kernel<B, float>), g_s = pg(bicg_s_kernel<B, float>);
      if (cudaMemsetAsync(y, 0, sizeof(float) * n, s) != cudaSuccess) return kCudaError;
      k_ref<<<g_ref, kThreads, 0, s>>>(A64, x, y, b, r, nullptr, alu32, prec, partials, ticket, st, hist, rt);
      plan.kernels = 6;
      plan.always_all = true;
      plan.kind = {2, 0, 2, 0, 1, 0};
      plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool) {
        if (ev) cudaEventRecord(ev[0], ss);
        bicg_p_kernel<B, float><<<g_p, kThreads, 0, ss>>>(N, pp, r, vv, pt, alu32, prec, st, x, y);
        if (ev) cudaEventRecord(ev[1], ss);
        k_v<<<g_v, kThreads, 0, ss>>>(A32, pt, vv, rt, partials, ticket, st);
        if (ev) cudaEventRecord(ev[2], ss);
        bicg_s_kernel<B, float><<<g_s, kThreads, 0, ss>>>(N, sv, r, vv, stv, alu32, prec, st);
        if (ev) cudaEventRecord(ev[3], ss);
        k_t<<<g_t, kThreads, 0, ss>>>(A32, stv, t, sv, partials, ticket, st);
        if (ev) cudaEventRecord(ev[4], ss);
        k_xr<<<g_xr, kThreads, 0, ss>>>(N, y, pt, stv, r, sv, t, rt, partials, ticket, st, hist, 0);
        if (ev) cudaEventRecord(ev[5], ss);
        k_ref<<<g_ref, kThreads, 0, ss>>>(A64, x, y, b, r, nullptr, alu32, prec, partials, ticket, st, hist, rt);
        if (ev) cudaEventRecord(ev[6], ss);
      };
      plan.finalize = [=](cudaStream_t ss) { mixed_fold_kernel<<<gvec, kThreads, 0, ss>>>(n, x, y, st); };
    } else if (p.shard) {
      // multi-rank FP32-refined CG: halo update of p (FP32) before the product,
      // every dot product all-reduced, the refresh's all-reduce in every
      // iteration (the refresh is decided on the device, from all-reduced
      // sums, identically on every rank). The ghost rows of y and x are
      // updated with the owners' arithmetic (y += alpha p after p's halo
      // update, the folds), so the FP64 refresh multiplies x + y on the
      // ghost rows without a halo update of its own.
      const ShardPlan* sp = p.shard;
      SellView2 A32 = view2_of(m);
      const float* alu32 = m.d_alu32;
      float *r = vec.get<float>(n), *z = vec.get<float>(n), *q = vec.get<float>(n), *pp = vec.get<float>(n_ext),
            *y = vec.get<float>(n_ext);
      if (!r || !z || !q || !pp || !y) return kCudaError;
      double* x = d_x;
      const double* b = d_b;
      const int NP = p.np_rows;
      auto k_spmv = cg_spmv2_kernel<B, U>;
      auto k_upd = mixed_update_kernel<B>;
      auto k_ref = mixed_refresh_kernel<B, U>;
      const int g_spmv = pg(k_spmv), g_upd = pg(k_upd), g_ref = pg(k_ref);
      if (cudaMemsetAsync(y, 0, sizeof(float) * n_ext, s) != cudaSuccess) return kCudaError;
      if (cudaMemsetAsync(pp, 0, sizeof(float) * n_ext, s) != cudaSuccess) return kCudaError;
      int rc2 = shard_halo(*sp, x, s);
      k_ref<<<g_ref, kThreads, 0, s>>>(A64, x, y, b, r, z, alu32, prec, partials, ticket, st, hist, nullptr);
      if (!rc2) rc2 = shard_allreduce(*sp, st->red, 2, s);
      shard_mixed_refresh_kernel<false><<<1, 1, 0, s>>>(st, hist);
      if (rc2) return rc2;
      const int hk = (sp->n_send > 0) + (sp->n_recv > 0);
      plan.kernels = 4;
      plan.always_all = true;
      plan.launches = 7 + hk;
      plan.launches_special = 7 + hk;
      plan.kind = {1, 0, 2, 0};
      plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool) {
        if (ev) cudaEventRecord(ev[0], ss);
        mixed_p_kernel<<<gvec, kThreads, 0, ss>>>(n, pp, z, x, y, st, n_ext);
        if (ev) cudaEventRecord(ev[1], ss);
        shard_halo(*sp, pp, ss);
        k_spmv<<<g_spmv, kThreads, 0, ss>>>(A32, pp, q, partials, ticket, st);
        shard_allreduce(*sp, st->red, 1, ss);
        shard_mixed_alpha_kernel<<<1, 1, 0, ss>>>(st);
        if (ev) cudaEventRecord(ev[2], ss);
        k_upd<<<g_upd, kThreads, 0, ss>>>(N, y, pp, r, q, z, alu32, prec, partials, ticket, st, hist, NP);
        shard_allreduce(*sp, st->red, 2, ss);
        shard_mixed_inner_kernel<<<1, 1, 0, ss>>>(st, hist);
        if (ev) cudaEventRecord(ev[3], ss);
        k_ref<<<g_ref, kThreads, 0, ss>>>(A64, x, y, b, r, z, alu32, prec, partials, ticket, st, hist, nullptr);
        shard_allreduce(*sp, st->red, 2, ss);
        shard_mixed_refresh_kernel<false><<<1, 1, 0, ss>>>(st, hist);
        if (ev) cudaEventRecord(ev[4], ss);
      };
      plan.finalize = [=](cudaStream_t ss) { mixed_fold_kernel<<<gvec, kThreads, 0, ss>>>(n_ext, x, y, st); };
    } else {
      SellView2 A32 = view2_of(m);
      const float* alu32 = m.d_alu32;
      float *r = vec.get<float>(n), *z = vec.get<float>(n), *q = vec.get<float>(n), *pp = vec.get<float>(n),
            *y = vec.get<float>(n);
      if (!r || !z || !q || !pp || !y) return kCudaError;
      double* x = d_x;
      const double* b = d_b;
      auto k_spmv = cg_spmv2_kernel<B, U>;
      auto k_upd = mixed_update_kernel<B>;
      auto k_ref = mixed_refresh_kernel<B, U>;
      const int g_spmv = pg(k_spmv), g_upd = pg(k_upd);
      const int g_ref = pg(k_ref);
      if (cudaMemsetAsync(y, 0, sizeof(float) * n, s) != cudaSuccess) return kCudaError;
      k_ref<<<g_ref, kThreads, 0, s>>>(A64, x, y, b, r, z, alu32, prec, partials, ticket, st, hist, nullptr);
      plan.kernels = 4;
      plan.always_all = true;
      plan.kind = {1, 0, 2, 0};
      plan.iteration = [=](cudaStream_t ss, cudaEvent_t* ev, bool) {
        if (ev) cudaEventRecord(ev[0], ss);
        mixed_p_kernel<<<gvec, kThreads, 0, ss>>>(n, pp, z, x, y, st);
        if (ev) cudaEventRecord(ev[1], ss);
        k_spmv<<<g_spmv, kThreads, 0, ss>>>(A32, pp, q, partials, ticket, st);
        if (ev) cudaEventRecord(ev[2], ss);
        k_upd<<<g_upd, kThreads, 0, ss>>>(N, y, pp, r, q, z, alu32, prec, partials, ticket, st, hist, 0);
        if (ev) cudaEventRecord(ev[3], ss);
        k_ref<<<g_ref, kThreads, 0, ss>>>(A64, x, y, b, r, z, alu32, prec, partials, ticket, st, hist, nullptr);
        if (ev) cudaEventRecord(ev[4], ss);
      };
      plan.finalize = [=](cudaStream_t ss) { mixed_fold_kernel<<<gvec, kThreads, 0, ss>>>(n, x, y, st); };
    }
    return kOk;
   });
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  long long launched_kernels = 1;
  auto kernels_of = [&](bool special) -> long long {
    if (plan.launches > 0) return special ? plan.launches_special : plan.launches;
    return plan.kernels - ((special || plan.always_all) ? 0 : 1);
  };

  auto finish = [&](SolverState fin) -> int {
    if (!fin.done) {
      fprintf(stderr, "** monolis_b200: solver loop ended without a verdict\n");
      fin.status = kTimeout;
    }
    if (fin.status == kZeroRhs) {
      fprintf(stderr, "** monolis error: norm of RHS vector B is 0.0\n");
      MB_CUDA_OK(cudaMemsetAsync(d_x, 0, sizeof(double) * n, s));
      MB_CUDA_OK(cudaStreamSynchronize(s));
      res.iter = 0;
      res.status = kOk;
      res.resid = 0.0;
      return kOk;
    }
    res.iter = fin.iter;
    res.status = fin.status;
    res.resid = fin.resid;
    res.n_refine = fin.n_refine;
    res.launches = launched_kernels;
    if (h_hist && fin.iter > 0)
      MB_CUDA_OK(cudaMemcpy(h_hist, sc.hist, sizeof(double) * ((size_t)fin.iter + 1), cudaMemcpyDeviceToHost));
    return kOk;
  };
  auto is_special = [&](long long it) { return period > 0 && it > 0 && it % period == 0; };
  auto read_state = [&](SolverState& out) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(sc.h_st, sc.st, sizeof(SolverState), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    out = sc.h_st[0];
    return e;
  };

  res.kernel_time.assign(plan.kernels, 0.0);
  SolverState cur{};
  cudaError_t err = read_state(cur);
  if (err != cudaSuccess) return report_cuda(err, "solver init", __FILE__, __LINE__);
  const long long iter_cap = (long long)p.max_iter + 4 * (long long)batch + 8;

  if (p.timers) {
    // Timing mode: no graph; events around every kernel, one iteration at a
    // time (the host waits for each iteration, so the loop itself is slower).
    std::vector<cudaEvent_t> tev(plan.kernels + 1);
    for (auto& e : tev) cudaEventCreate(&e);
    long long its = 0;
    while (err == cudaSuccess && !cur.done && its++ <= iter_cap) {
      const bool special = is_special(cur.iter);
      plan.iteration(s, tev.data(), special);
      launched_kernels += kernels_of(special);
      err = read_state(cur);
      if (err != cudaSuccess) break;
      for (int k = 0; k < plan.kernels; k++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, tev[k], tev[k + 1]);
        res.kernel_time[k] += ms * 1e-3;
      }
    }
    for (auto& e : tev) cudaEventDestroy(e);
    if (err != cudaSuccess) return report_cuda(err, "solver loop (timers)", __FILE__, __LINE__);
    for (int k = 0; k < plan.kernels; k++) res.t_kind[plan.kind[k]] += res.kernel_time[k];
  } else if (!cur.done && p.use_graph && !p.shard && cur.iter == 1 && (p.method != 3 || period <= 400)) {
    // One graph for the whole solve: a while node whose body is one batch of
    // iterations followed by loop_continue_kernel, which stops the loop on
    // the device once the solve has a verdict. The host launches it once and
    // waits: no host thread in the loop, so a late or descheduled host cannot
    // leave the GPU idle. With a true-residual interval (FP64), the last
    // iteration of every body carries the residual kernel: the batch divides
    // the interval, so every replacement iteration is the last of a body, and
    // in the other bodies the kernel returns at entry (its flag is raised by
    // the update kernel of a replacement iteration only). PipeCG's
    // replacement iteration also recomputes V = A U, which is not gated: its
    // body is the whole interval. After the verdict the rest of the last body
    // returns at kernel entry.
    const int body = p.method == 3 ? period : batch;
    const int cap = (int)std::min<long long>(iter_cap, 0x7fffffff);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaGraphCreate(&graph, 0);
    cudaGraphConditionalHandle handle{};
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t wnode = nullptr;
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = handle;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&wnode, graph, nullptr, 0, &cp);
    }
    if (e == cudaSuccess) {
      cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(s, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        for (int k = 0; k < body; k++) plan.iteration(s, nullptr, period > 0 && k == body - 1);
        loop_continue_kernel<<<1, 1, 0, s>>>(handle, sc.st, cap);
        cudaError_t e1 = cudaGetLastError();
        cudaError_t e2 = cudaStreamEndCapture(s, &bodyg);  // always ended: the stream stays usable
        e = e1 != cudaSuccess ? e1 : e2;
      }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return report_cuda(e, "solver loop (device-side while graph)", __FILE__, __LINE__);
    SolverState after{};
    err = read_state(after);
    if (err != cudaSuccess) return report_cuda(err, "solver loop state", __FILE__, __LINE__);
    launched_kernels += (long long)after.loops * ((long long)(body - (period > 0 ? 1 : 0)) * kernels_of(false) +
                                                 (period > 0 ? kernels_of(true) : 0) + 1);
  } else if (!cur.done) {
    // Host-driven loop (several ranks, a PipeCG interval above 400, or a
    // solve that does not start at the first iteration): two graphs of
    // `batch` iterations: plain, and with the true-residual kernel in the last
    // iteration (FP64 only).
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    const int ngraphs = period > 0 ? 2 : 1;
    if (p.use_graph) {
      for (int g = 0; g < ngraphs; g++) {
        cudaGraph_t graph = nullptr;
        MB_CUDA_OK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < batch; k++) plan.iteration(s, nullptr, g == 1 && k == batch - 1);
        MB_CUDA_OK(cudaStreamEndCapture(s, &graph));
        MB_CUDA_OK(cudaGraphInstantiate(&exec[g], graph, 0));
        cudaGraphDestroy(graph);
      }
    }
    // Several launches in flight: the host reads the state word of the oldest
    // while the others keep the GPU busy, so a late host thread (a busy core,
    // a driver query from another process) does not leave the device idle.
    // The depth is 3 to start with and, once the second launch has been timed,
    // enough launches to queue about 50 ms of work, at most kMaxInFlight. On
    // several ranks it stays 3: every rank must enqueue the same number of
    // launches (they hold collectives), and a timed depth could differ.
    // After the verdict the batches still queued return at kernel entry (a
    // few microseconds per kernel).
    constexpr int kMaxInFlight = 8;
    int depth = 3;
    cudaEvent_t ev[kMaxInFlight], t_ev[2];
    for (auto& e : ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    for (auto& e : t_ev) cudaEventCreate(&e);
    long long next = cur.iter;  // iteration the next enqueued batch starts with (batches start at 1 mod batch)
    int inflight = 0, slot = 0, launched = 0;
    bool depth_set = p.shard != nullptr;
    while (err == cudaSuccess) {
      if (launched == 1) cudaEventRecord(t_ev[0], s);
      const int special = is_special(next + batch - 1) ? 1 : 0;
      if (exec[special]) {
        err = cudaGraphLaunch(exec[special], s);
      } else {
        for (int k = 0; k < batch; k++) plan.iteration(s, nullptr, special && k == batch - 1);
        err = cudaGetLastError();
      }
      if (err != cudaSuccess) break;
      launched_kernels += (long long)(batch - 1) * kernels_of(false) + kernels_of(special);
      next += batch;
      if (++launched == 2) cudaEventRecord(t_ev[1], s);  // brackets the second launch
      cudaMemcpyAsync(&sc.h_st[slot], sc.st, sizeof(SolverState), cudaMemcpyDeviceToHost, s);
      cudaEventRecord(ev[slot], s);
      slot = (slot + 1) % kMaxInFlight;
      if (++inflight < depth) continue;
      const int oldest = (slot + kMaxInFlight - inflight) % kMaxInFlight;
      err = cudaEventSynchronize(ev[oldest]);
      if (err != cudaSuccess) break;
      inflight--;
      if (sc.h_st[oldest].done) break;
      if (!depth_set && launched >= 2 && cudaEventQuery(t_ev[1]) == cudaSuccess) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t_ev[0], t_ev[1]) == cudaSuccess && ms > 0.f)
          depth = std::max(3, std::min(kMaxInFlight, (int)std::ceil(50.0 / ms)));
        depth_set = true;
      }
      if (next > iter_cap) {
        fprintf(stderr, "** monolis_b200: iteration cap reached without a verdict\n");
        break;
      }
    }
    cudaError_t e2 = cudaStreamSynchronize(s);
    if (err == cudaSuccess) err = e2;
    for (auto& e : ev) cudaEventDestroy(e);
    for (auto& e : t_ev) cudaEventDestroy(e);
    for (auto& e : exec)
      if (e) cudaGraphExecDestroy(e);
    if (err != cudaSuccess) return report_cuda(err, "solver loop", __FILE__, __LINE__);
  }
  if (plan.finalize) {
    plan.finalize(s);
    launched_kernels += 1;
  }
  // several ranks: the ghost entries of the solution from their owners, as
  // the reference's solvers end (src/iterative/CG.f90:105,
  // BiCGSTAB.f90:174, GropCG.f90:121); every rank reaches this point
  if (p.shard) {
    rc = shard_halo(*p.shard, d_x, s);
    if (rc) return rc;
  }
  SolverState fin{};
  err = read_state(fin);
  if (err != cudaSuccess) return report_cuda(err, "solver final state", __FILE__, __LINE__);
  res.t_loop = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return finish(fin);
}

}  // namespace mb
