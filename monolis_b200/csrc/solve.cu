// solve.cu -- device-resident CG and BiCGSTAB (FP64, and FP32-inner with
// FP64 reliable-update refinement) built from fused kernels.
//
// Every scalar of the recurrences (rho, alpha, beta, omega, B2, the
// residual) lives in SolverState on the device. Each reduction is a one-pass
// grid reduction whose last block also evaluates the scalar update, so an
// iteration is a fixed sequence of kernels with no host round trip. The host
// captures `batch` iterations into one CUDA graph, launches it repeatedly
// and reads the done flag once per launch (two launches in flight); kernels
// return immediately once `done` is set.
//
// FP64 CG follows src/iterative/CG.f90:74-101 and BiCGSTAB follows
// src/iterative/BiCGSTAB.f90:87-170 operation by operation (same vector
// update expressions and roundings, true residual every 200 iterations,
// convergence relative to the initial residual); only the order in which the
// dot products are summed differs (tree instead of serial).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <functional>
#include <vector>

#include "spmv.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;
constexpr int kVecBlocks = 148 * 8;

inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

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

// ---------------------------------------------------------------------------
// Residual kernel: r = b - A x, then z = M^-1 r (CG) and the two dots.
// mode 0: CG (dots <r,r>, <r,z>); mode 1: BiCGSTAB (dots <r,r>, <r,rt>;
// at iter 0 also rt = r). gated: run only on iterations with iter % 200 == 0.
// ---------------------------------------------------------------------------
template <int B, int U, class V, class T>
__global__ void __launch_bounds__(kThreads)
    resid_kernel(SellView<V> A, const T* __restrict__ x, const T* __restrict__ b, T* __restrict__ r,
                 T* __restrict__ z, T* __restrict__ rt, const T* __restrict__ alu, int prec, int mode, int gated,
                 double* partials, unsigned int* ticket, SolverState* st, double* hist) {
  if (st->done) return;
  if (gated && !st->rr_flag) return;
  const bool init = st->iter == 0;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (row < A.N) {
    T y[B];
    sell_row<B, U, V, T>(A, x, row, y);
    T t[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      t[c] = sub_rn(b[i], y[c]);  // src/linalg/matvec.f90:902  R = 1.0*B + (-1.0)*R
      r[i] = t[c];
      v[0] += (double)t[c] * (double)t[c];
    }
    if (mode == 0) {
      T w[B];
#pragma unroll
      for (int c = 0; c < B; c++) w[c] = t[c];
      if (prec) diag_row<B, T>(alu, A.N, row, w);
#pragma unroll
      for (int c = 0; c < B; c++) {
        z[(long long)row * B + c] = w[c];
        v[1] += (double)t[c] * (double)w[c];
      }
    } else {
#pragma unroll
      for (int c = 0; c < B; c++) {
        const long long i = (long long)row * B + c;
        T rtv;
        if (init) { rt[i] = t[c]; rtv = t[c]; } else { rtv = rt[i]; }
        v[1] += (double)t[c] * (double)rtv;
      }
    }
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    st->rr_flag = 0;
    if (mode == 0) fin_cg(st, tot[0], tot[1], hist);
    else fin_bicg(st, tot[0], tot[1], hist);
  });
}

// ---------------------------------------------------------------------------
// CG kernels
// ---------------------------------------------------------------------------
// P = beta*P + 1.0*Z (src/iterative/CG.f90:78-83); P = Z on iteration 1.
template <class T>
__global__ void cg_p_kernel(long long n, T* __restrict__ p, const T* __restrict__ z, const SolverState* st) {
  if (st->done) return;
  const bool first = st->iter == 1;
  const T beta = (T)st->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = first ? z[i] : axpy_rn(beta, p[i], z[i]);
}

// Q = A P fused with omega = <P,Q>, alpha = rho/omega (CG.f90:85-87).
template <int B, int U, class V, class T>
__global__ void __launch_bounds__(kThreads)
    cg_spmv_kernel(SellView<V> A, const T* __restrict__ p, T* __restrict__ q, double* partials,
                   unsigned int* ticket, SolverState* st) {
  if (st->done) return;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (row < A.N) {
    T y[B];
    sell_row<B, U, V, T>(A, p, row, y);
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      q[i] = y[c];
      v[0] += (double)p[i] * (double)y[c];
    }
  }
  grid_reduce<1>(v, partials, ticket, [&](double* tot) {
    st->omega = tot[0];
    st->alpha = st->rho / tot[0];
  });
}

// X = alpha*P + X; R = -alpha*Q + R; Z = M^-1 R; <R,R>, <R,Z>
// (CG.f90:89-97 + the next iteration's precond apply and rho).
// On iterations with iter % 200 == 0 only X is updated here and the residual
// kernel recomputes R = B - A X.
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    cg_update_kernel(int N, T* __restrict__ x, const T* __restrict__ p, T* __restrict__ r,
                     const T* __restrict__ q, T* __restrict__ z, const T* __restrict__ alu, int prec,
                     double* partials, unsigned int* ticket, SolverState* st, double* hist) {
  if (st->done) return;
  const bool rr_iter = (st->iter % st->iter_rr) == 0;
  const T alpha = (T)st->alpha;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (row < N) {
    T t[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
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
      if (prec) diag_row<B, T>(alu, N, row, w);
#pragma unroll
      for (int c = 0; c < B; c++) {
        z[(long long)row * B + c] = w[c];
        v[0] += (double)t[c] * (double)t[c];
        v[1] += (double)t[c] * (double)w[c];
      }
    }
  }
  if (rr_iter) {
    // iteration counter is not advanced here: the residual kernel that
    // follows recomputes R = B - A X and finishes the iteration
    if (blockIdx.x == 0 && threadIdx.x == 0) st->rr_flag = 1;
    return;
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) { fin_cg(st, tot[0], tot[1], hist); });
}

// ---------------------------------------------------------------------------
// BiCGSTAB kernels (src/iterative/BiCGSTAB.f90:87-170)
// ---------------------------------------------------------------------------
// P = R + beta*(P - omega*V) (or P = R on iteration 1); PT = M^-1 P.
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    bicg_p_kernel(int N, T* __restrict__ p, const T* __restrict__ r, const T* __restrict__ vv,
                  T* __restrict__ pt, const T* __restrict__ alu, int prec, const SolverState* st) {
  if (st->done) return;
  const bool first = st->iter == 1;
  const T beta = (T)st->beta, omega = (T)st->omega;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= N) return;
  T w[B];
#pragma unroll
  for (int c = 0; c < B; c++) {
    const long long i = (long long)row * B + c;
    const T pv = first ? r[i] : add_rn(r[i], mul_rn(beta, sub_rn(p[i], mul_rn(omega, vv[i]))));
    p[i] = pv;
    w[c] = pv;
  }
  if (prec) diag_row<B, T>(alu, N, row, w);
#pragma unroll
  for (int c = 0; c < B; c++) pt[(long long)row * B + c] = w[c];
}

// V = A PT; c2 = <RT,V>; alpha = rho/c2 (BiCGSTAB.f90:113-123)
template <int B, int U, class V, class T>
__global__ void __launch_bounds__(kThreads)
    bicg_v_kernel(SellView<V> A, const T* __restrict__ pt, T* __restrict__ vv, const T* __restrict__ rt,
                  double* partials, unsigned int* ticket, SolverState* st) {
  if (st->done) return;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (row < A.N) {
    T y[B];
    sell_row<B, U, V, T>(A, pt, row, y);
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      vv[i] = y[c];
      v[0] += (double)rt[i] * (double)y[c];
    }
  }
  grid_reduce<1>(v, partials, ticket, [&](double* tot) {
    st->c2 = tot[0];
    if (tot[0] == 0.0) { st->done = 1; st->status = kBreakdown; return; }
    st->alpha = st->rho / tot[0];
  });
}

// S = -alpha*V + R; ST = M^-1 S (BiCGSTAB.f90:124-126)
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    bicg_s_kernel(int N, T* __restrict__ s, const T* __restrict__ r, const T* __restrict__ vv,
                  T* __restrict__ stv, const T* __restrict__ alu, int prec, const SolverState* st) {
  if (st->done) return;
  const T alpha = (T)st->alpha;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= N) return;
  T w[B];
#pragma unroll
  for (int c = 0; c < B; c++) {
    const long long i = (long long)row * B + c;
    const T sv = axpy_rn(-alpha, vv[i], r[i]);
    s[i] = sv;
    w[c] = sv;
  }
  if (prec) diag_row<B, T>(alu, N, row, w);
#pragma unroll
  for (int c = 0; c < B; c++) stv[(long long)row * B + c] = w[c];
}

// T = A ST; (T,S), (T,T); omega = (T,S)/(T,T) or 0 (BiCGSTAB.f90:128-146)
template <int B, int U, class V, class T>
__global__ void __launch_bounds__(kThreads)
    bicg_t_kernel(SellView<V> A, const T* __restrict__ stv, T* __restrict__ t, const T* __restrict__ s,
                  double* partials, unsigned int* ticket, SolverState* st) {
  if (st->done) return;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (row < A.N) {
    T y[B];
    sell_row<B, U, V, T>(A, stv, row, y);
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      t[i] = y[c];
      v[0] += (double)y[c] * (double)s[i];
      v[1] += (double)y[c] * (double)y[c];
    }
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    st->ts = tot[0];
    st->tt = tot[1];
    st->omega = tot[1] == 0.0 ? 0.0 : tot[0] / tot[1];
  });
}

// X = X + alpha*PT + omega*ST; R = -omega*T + S; <R,R>, <R,RT>
// (BiCGSTAB.f90:148-164). On iter % 200 == 0 only X is updated here.
template <int B, class T>
__global__ void __launch_bounds__(kThreads)
    bicg_xr_kernel(int N, T* __restrict__ x, const T* __restrict__ pt, const T* __restrict__ stv,
                   T* __restrict__ r, const T* __restrict__ s, const T* __restrict__ t, const T* __restrict__ rt,
                   double* partials, unsigned int* ticket, SolverState* st, double* hist) {
  if (st->done) return;
  const bool rr_iter = (st->iter % st->iter_rr) == 0;
  const T alpha = (T)st->alpha, omega = (T)st->omega;
  const long long n = (long long)N * B;
  double v[2] = {0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] = add_rn(add_rn(x[i], mul_rn(alpha, pt[i])), mul_rn(omega, stv[i]));
    if (!rr_iter) {
      const T rv = axpy_rn(-omega, t[i], s[i]);
      r[i] = rv;
      v[0] += (double)rv * (double)rv;
      v[1] += (double)rv * (double)rt[i];
    }
  }
  if (rr_iter) {
    if (blockIdx.x == 0 && threadIdx.x == 0) st->rr_flag = 1;
    return;
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) { fin_bicg(st, tot[0], tot[1], hist); });
}

// ---------------------------------------------------------------------------
// Mixed precision CG: FP32 matrix, vectors and arithmetic in the loop, FP64
// accumulation of every dot product and FP64 scalars; FP64 solution x and an
// FP64 true residual r = b - A x recomputed ("reliable update") whenever the
// iterated residual has dropped by `delta` since the last refresh, or looks
// converged. The Krylov direction p is kept across refreshes.
// ---------------------------------------------------------------------------
__device__ void fin_mixed_inner(SolverState* st, double rr, double rz, double* hist) {
  const double rn = sqrt(rr);
  const double resid = sqrt(rr / st->B2);
  record(st, hist, resid);
  if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
  if (rn > st->rmax) st->rmax = rn;
  if (rn < st->delta * st->rmax || resid < st->tol || st->iter >= st->max_iter) {
    st->refresh = 1;  // the refresh kernels finish this iteration
    st->rho1 = st->rho;
    st->rr = rz;      // kept in case the refresh is the last step
    return;
  }
  st->rho1 = st->rho;
  st->rho = rz;
  st->beta = st->rho / st->rho1;
  st->iter += 1;
}

// y += alpha*p; r -= alpha*q; z = M^-1 r; dots (FP32 vectors, FP64 sums)
template <int B>
__global__ void __launch_bounds__(kThreads)
    mixed_update_kernel(int N, float* __restrict__ y, const float* __restrict__ p, float* __restrict__ r,
                        const float* __restrict__ q, float* __restrict__ z, const float* __restrict__ alu, int prec,
                        double* partials, unsigned int* ticket, SolverState* st, double* hist) {
  if (st->done) return;
  const float alpha = (float)st->alpha;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (row < N) {
    float t[B], w[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      y[i] = fmaf(alpha, p[i], y[i]);
      t[c] = fmaf(-alpha, q[i], r[i]);
      r[i] = t[c];
      w[c] = t[c];
    }
    if (prec) diag_row<B, float>(alu, N, row, w);
#pragma unroll
    for (int c = 0; c < B; c++) {
      z[(long long)row * B + c] = w[c];
      v[0] += (double)t[c] * (double)t[c];
      v[1] += (double)t[c] * (double)w[c];
    }
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) { fin_mixed_inner(st, tot[0], tot[1], hist); });
}

// Refresh step: x += y (FP64), y = 0, r64 = b - A64 x, r = fp32(r64),
// z = M^-1 r; dots <r64,r64> (true residual) and <r,z>. Also the initial
// residual when iter == 0. Runs only when st->refresh or iter == 0.
template <int B, int U>
__global__ void __launch_bounds__(kThreads)
    mixed_resid_kernel(SellView<double> A, double* __restrict__ x, const double* __restrict__ b,
                       float* __restrict__ y, float* __restrict__ r, float* __restrict__ z,
                       const float* __restrict__ alu, int prec, double* partials, unsigned int* ticket,
                       SolverState* st, double* hist) {
  if (st->done) return;
  if (!(st->refresh || st->iter == 0)) return;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (row < A.N) {
    double ax[B];
    sell_row<B, U, double, double>(A, x, row, ax);
    float t[B], w[B];
#pragma unroll
    for (int c = 0; c < B; c++) {
      const long long i = (long long)row * B + c;
      const double rv = b[i] - ax[c];
      v[0] += rv * rv;
      t[c] = (float)rv;
      r[i] = t[c];
      w[c] = t[c];
      y[i] = 0.0f;
    }
    if (prec) diag_row<B, float>(alu, A.N, row, w);
#pragma unroll
    for (int c = 0; c < B; c++) {
      z[(long long)row * B + c] = w[c];
      v[1] += (double)t[c] * (double)w[c];
    }
  }
  grid_reduce<2>(v, partials, ticket, [&](double* tot) {
    const double rr = tot[0], rz = tot[1];
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
    st->n_refine += 1;
    if (resid < st->tol) { st->done = 1; st->status = kOk; return; }
    if (!isfinite(resid)) { st->done = 1; st->status = kNonFinite; return; }
    if (st->iter >= st->max_iter) { st->done = 1; st->status = kMaxIter; return; }
    st->rmax = sqrt(rr);
    st->rho = rz;
    st->beta = st->rho / st->rho1;
    st->iter += 1;
  });
}

// x += y before the refresh residual (separate pass: the residual kernel
// reads x at neighbouring rows).
__global__ void mixed_fold_kernel(long long n, double* __restrict__ x, const float* __restrict__ y,
                                  const SolverState* st) {
  if (st->done || !st->refresh) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] += (double)y[i];
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <class F>
int dispatch_ndof(int ndof, F&& f) {
  switch (ndof) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    default: return kBadInput;
  }
}

template <int B>
struct Unroll {
  static constexpr int value = B == 1 ? 4 : (B <= 3 ? 2 : 1);
};

struct Vecs {
  std::vector<void*> ptrs;
  cudaStream_t s;
  ~Vecs() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
  template <class T>
  T* get(long long n) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, sizeof(T) * (size_t)(n > 0 ? n : 1) + 16, s) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
};

}  // namespace

int solve_device(SellMatrix& m, Scratch& sc, const SolveParams& p, const double* d_b, double* d_x,
                 SolveResult& res, double* h_hist, cudaStream_t s) {
  const int N = m.N, nd = m.ndof;
  const long long n = (long long)N * nd;
  const int prec = p.precond == 1 ? 1 : 0;
  if (prec && !m.have_alu) return kBadInput;
  if (p.method != 1 && p.method != 5) return kBadInput;
  if (p.precision == 1 && p.method != 1) {
    fprintf(stderr, "** monolis_b200: mixed precision is implemented for CG\n");
    return kBadInput;
  }
  int rc = scratch_ensure(sc, (size_t)p.max_iter + 2);
  if (rc) return rc;
  if (p.precision == 1) {
    rc = sell_make_fp32(m, s);
    if (rc) return rc;
  }

  SolverState h{};
  h.tol = p.tol;
  h.max_iter = p.max_iter;
  h.iter_rr = p.iter_rr > 0 ? p.iter_rr : 200;
  h.delta = p.delta > 0 ? p.delta : 0.1;
  MB_CUDA_OK(cudaMemcpyAsync(sc.st, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(cudaMemsetAsync(sc.ticket, 0, sizeof(unsigned int) * 64, s));
  if (p.init_x) MB_CUDA_OK(cudaMemsetAsync(d_x, 0, sizeof(double) * n, s));

  Vecs vec{{}, s};
  const int gb = blocks_for(N);
  std::function<void(cudaStream_t)> iteration;
  int kernels_per_iter = 0;
  auto t0 = std::chrono::steady_clock::now();

  rc = dispatch_ndof(nd, [&](auto Bc) -> int {
    constexpr int B = decltype(Bc)::value;
    constexpr int U = Unroll<B>::value;
    SellView<double> A64 = view_of<double>(m);
    double* partials = sc.partials;
    unsigned int* ticket = sc.ticket;
    SolverState* st = sc.st;
    double* hist = sc.hist;
    if (p.precision == 0) {
      const double* alu = m.d_alu64;
      if (p.method == 1) {
        double *r = vec.get<double>(n), *z = vec.get<double>(n), *q = vec.get<double>(n), *pp = vec.get<double>(n);
        if (!r || !z || !q || !pp) return kCudaError;
        double* x = d_x;
        const double* b = d_b;
        resid_kernel<B, U, double, double><<<gb, kThreads, 0, s>>>(A64, x, b, r, z, nullptr, alu, prec, 0, 0,
                                                                   partials, ticket, st, hist);
        kernels_per_iter = 4;
        iteration = [=](cudaStream_t ss) {
          cg_p_kernel<double><<<kVecBlocks, kThreads, 0, ss>>>(n, pp, z, st);
          cg_spmv_kernel<B, U, double, double><<<gb, kThreads, 0, ss>>>(A64, pp, q, partials, ticket, st);
          cg_update_kernel<B, double><<<gb, kThreads, 0, ss>>>(N, x, pp, r, q, z, alu, prec, partials, ticket, st,
                                                               hist);
          resid_kernel<B, U, double, double><<<gb, kThreads, 0, ss>>>(A64, x, b, r, z, nullptr, alu, prec, 0, 1,
                                                                      partials, ticket, st, hist);
        };
      } else {
        double *r = vec.get<double>(n), *rt = vec.get<double>(n), *pp = vec.get<double>(n),
               *pt = vec.get<double>(n), *sv = vec.get<double>(n), *stv = vec.get<double>(n),
               *t = vec.get<double>(n), *vv = vec.get<double>(n);
        if (!r || !rt || !pp || !pt || !sv || !stv || !t || !vv) return kCudaError;
        double* x = d_x;
        const double* b = d_b;
        resid_kernel<B, U, double, double><<<gb, kThreads, 0, s>>>(A64, x, b, r, nullptr, rt, alu, prec, 1, 0,
                                                                   partials, ticket, st, hist);
        kernels_per_iter = 6;
        iteration = [=](cudaStream_t ss) {
          bicg_p_kernel<B, double><<<gb, kThreads, 0, ss>>>(N, pp, r, vv, pt, alu, prec, st);
          bicg_v_kernel<B, U, double, double><<<gb, kThreads, 0, ss>>>(A64, pt, vv, rt, partials, ticket, st);
          bicg_s_kernel<B, double><<<gb, kThreads, 0, ss>>>(N, sv, r, vv, stv, alu, prec, st);
          bicg_t_kernel<B, U, double, double><<<gb, kThreads, 0, ss>>>(A64, stv, t, sv, partials, ticket, st);
          bicg_xr_kernel<B, double><<<kVecBlocks, kThreads, 0, ss>>>(N, x, pt, stv, r, sv, t, rt, partials, ticket,
                                                                     st, hist);
          resid_kernel<B, U, double, double><<<gb, kThreads, 0, ss>>>(A64, x, b, r, nullptr, rt, alu, prec, 1, 1,
                                                                      partials, ticket, st, hist);
        };
      }
    } else {
      SellView<float> A32 = view_of<float>(m);
      const float* alu32 = m.d_alu32;
      float *r = vec.get<float>(n), *z = vec.get<float>(n), *q = vec.get<float>(n), *pp = vec.get<float>(n),
            *y = vec.get<float>(n);
      if (!r || !z || !q || !pp || !y) return kCudaError;
      double* x = d_x;
      const double* b = d_b;
      mixed_resid_kernel<B, U><<<gb, kThreads, 0, s>>>(A64, x, b, y, r, z, alu32, prec, partials, ticket, st, hist);
      kernels_per_iter = 5;
      iteration = [=](cudaStream_t ss) {
        cg_p_kernel<float><<<kVecBlocks, kThreads, 0, ss>>>(n, pp, z, st);
        cg_spmv_kernel<B, Unroll<B>::value + 1, float, float><<<gb, kThreads, 0, ss>>>(A32, pp, q, partials, ticket,
                                                                                    st);
        mixed_update_kernel<B><<<gb, kThreads, 0, ss>>>(N, y, pp, r, q, z, alu32, prec, partials, ticket, st, hist);
        mixed_fold_kernel<<<kVecBlocks, kThreads, 0, ss>>>(n, x, y, st);
        mixed_resid_kernel<B, U><<<gb, kThreads, 0, ss>>>(A64, x, b, y, r, z, alu32, prec, partials, ticket, st,
                                                          hist);
      };
    }
    return kOk;
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());

  // Batches of iterations, captured once into a graph.
  const int batch = p.batch > 0 ? p.batch : 16;
  cudaGraphExec_t exec = nullptr;
  if (p.use_graph) {
    cudaGraph_t g = nullptr;
    MB_CUDA_OK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < batch; k++) iteration(s);
    MB_CUDA_OK(cudaStreamEndCapture(s, &g));
    MB_CUDA_OK(cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
  }
  auto launch_batch = [&]() -> cudaError_t {
    if (exec) return cudaGraphLaunch(exec, s);
    for (int k = 0; k < batch; k++) iteration(s);
    return cudaGetLastError();
  };
  cudaEvent_t ev[2];
  cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
  const long long max_batches = (long long)p.max_iter / batch + 4;
  int cur = 0;
  long long launched = 0;
  bool finished = false;
  cudaError_t err = cudaSuccess;
  // prime: two batches in flight
  for (int k = 0; k < 2 && !finished; k++) {
    err = launch_batch();
    if (err != cudaSuccess) break;
    cudaMemcpyAsync(&sc.h_st[k], sc.st, sizeof(SolverState), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(ev[k], s);
    launched++;
  }
  while (err == cudaSuccess && !finished) {
    err = cudaEventSynchronize(ev[cur]);
    if (err != cudaSuccess) break;
    if (sc.h_st[cur].done || launched > max_batches) {
      finished = true;
      break;
    }
    err = launch_batch();
    if (err != cudaSuccess) break;
    cudaMemcpyAsync(&sc.h_st[cur], sc.st, sizeof(SolverState), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(ev[cur], s);
    launched++;
    cur ^= 1;
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (err == cudaSuccess) err = e2;
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (exec) cudaGraphExecDestroy(exec);
  if (err != cudaSuccess) return report_cuda(err, "solver loop", __FILE__, __LINE__);

  SolverState fin{};
  MB_CUDA_OK(cudaMemcpy(&fin, sc.st, sizeof(fin), cudaMemcpyDeviceToHost));
  res.t_loop = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
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
  res.launches = 1 + launched * batch * kernels_per_iter;
  res.iter = fin.iter;
  res.status = fin.status;
  res.resid = fin.resid;
  res.n_refine = fin.n_refine;
  if (h_hist && fin.iter > 0)
    MB_CUDA_OK(cudaMemcpy(h_hist, sc.hist, sizeof(double) * ((size_t)fin.iter + 1), cudaMemcpyDeviceToHost));
  return kOk;
}

}  // namespace mb
