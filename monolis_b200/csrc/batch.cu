// batch.cu -- many independent block-CSR systems solved by preconditioned CG
// in one persistent kernel.
//
// The systems are stacked into one block-diagonal matrix (each padded with
// identity rows to a multiple of 64 rows, so no slice of the device layout
// and no row pair of the FP32 layout spans two systems). A persistent kernel
// is launched in thread-block clusters of C CTAs; clusters take work items
// from a queue ordered by decreasing system size (longest first), so the
// largest systems start first and the small ones fill in behind them. A work
// item is either one system solved by the whole cluster -- its rows split
// between the C CTAs, dot products reduced through distributed shared memory
// and the phases of an iteration separated by the hardware cluster barrier
// -- or up to C small systems, one per CTA, reduced within the CTA. No block
// ever waits on a block outside its own cluster, and the cluster barrier is
// a hardware barrier (no spinning), so the kernel cannot deadlock on
// residency. Every system carries its own convergence state: a converged
// system stops, the others go on.
//
// Arithmetic: FP32 matrix values (paired sliced-ELL layout) and FP32 vectors
// inside the loop, FP64 accumulation of every dot product and FP64 scalars.
// With refinement the FP64 solution is x + y (y the FP32 correction) and a
// reliable update recomputes r = b - A (x + y) with the FP64 matrix whenever
// the iterated residual has dropped by `delta` since the last refresh or looks
// converged; convergence is then decided on that FP64 residual. Without
// refinement the iterated FP32 residual decides, and the true residual of the
// result is reported.
//
// Cluster size, CTA size and the size below which systems are solved one per
// CTA are chosen by timing the candidates on the batch itself
// (batch_autotune); the whole solve is one graph launch (queue reset + the
// persistent kernel).
#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "monolis_b200.h"
#include "spmv.cuh"

namespace cg = cooperative_groups;

namespace mb {
namespace {

constexpr int kBatchMaxThreads = 512;
constexpr int kBatchRowAlign = 64;
// The batched kernel is latency-bound (small systems, cluster barriers every
// phase), so it reads the 32-bit column ids: the 16-bit form's extra base load
// per slot cost more than its bytes save (C4: 0.165 s vs 0.144 s).
constexpr bool kBatchCols16 = false;

struct BatchSys {
  long long row0;  // first block row in the stacked matrix (multiple of 64)
  int nrows;       // block rows including padding (multiple of 64)
  int real_rows;
};

struct BatchItem {
  int first;  // position in the size order
  int count;  // systems in the item
  int split;  // 0: one system for the whole cluster; 1: one system per CTA
};

struct BatchArgs {
  SellView2 A32;
  SellView<double> A64;
  const float* alu32;
  int N, prec, refine, max_iter, nitems;
  double tol, delta;
  const BatchSys* sys;
  const int* order;
  const BatchItem* items;
  unsigned int* queue;
  const double* b;
  double* x;
  float *y, *r, *z, *p, *q;
  int *out_iter, *out_status, *out_nref;
  double* out_resid;
};

struct GroupShared {
  double red[32 * 2];
  double slot[2][2];  // this CTA's partial sums (double-buffered by parity)
  double bc[2];       // group sums, broadcast to the CTA
  int item;
};

// Sum of K doubles over the group (the cluster, or this CTA alone). All CTAs
// of a cluster add the partials in rank order, so they hold identical bits
// and take identical branches.
template <int K>
__device__ __forceinline__ void group_sum(double (&v)[K], GroupShared& sh, const cg::cluster_group& cl, int gsize,
                                          int& ph) {
  block_sum<K>(v, sh.red);
  if (gsize == 1) {
    if (threadIdx.x == 0)
#pragma unroll
      for (int k = 0; k < K; k++) sh.bc[k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = sh.bc[k];
    return;
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; k++) sh.slot[ph][k] = v[k];
  cl.sync();  // release/acquire at cluster scope: partials and all earlier global writes visible
  if (threadIdx.x == 0) {
    double t[K];
#pragma unroll
    for (int k = 0; k < K; k++) t[k] = 0.0;
    for (int rk = 0; rk < gsize; rk++) {
      const GroupShared* o = cl.map_shared_rank(&sh, rk);
#pragma unroll
      for (int k = 0; k < K; k++) t[k] += o->slot[ph][k];
    }
#pragma unroll
    for (int k = 0; k < K; k++) sh.bc[k] = t[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = sh.bc[k];
  ph ^= 1;
}

__device__ __forceinline__ void group_sync(const cg::cluster_group& cl, int gsize) {
  if (gsize > 1) cl.sync();
  else __syncthreads();
}

// x + y with coherent loads: both are written by the other CTAs of the
// cluster during this launch.
struct XPlusYCoherent {
  const double* x;
  const float* y;
  __device__ __forceinline__ double operator()(long long i) const { return __ldcg(x + i) + (double)__ldcg(y + i); }
};

// CG on system `si` by a group of gsize CTAs (this one has rank grank).
template <int B, int U>
__device__ __forceinline__ void solve_system(const BatchArgs a, int si, int gsize, int grank,
                                             const cg::cluster_group& cl, GroupShared& sh) {
  const BatchSys S = a.sys[si];
  // this CTA's rows: a multiple of 4 (a system has a multiple of 64), so the
  // vector phases can move whole 16-byte groups of R rows (RowGroup)
  const long long pair0 = S.row0 / 2, npairs = S.nrows / 2;
  const long long chunk = 2 * ((npairs / 2 + gsize - 1) / gsize);
  const long long plo = pair0 + min(npairs, chunk * grank);
  const long long phi = pair0 + min(npairs, chunk * (grank + 1));
  const long long rlo = 2 * plo, rhi = 2 * phi;  // this CTA's block rows
  const long long elo = rlo * B, ehi = rhi * B;  // and vector entries
  const int tid = threadIdx.x, nt = blockDim.x;
  int ph = 0;
  using RG = RowGroup<float, B>;
  constexpr int R = RG::R, E = RG::E;
  const long long g0 = rlo / R, g1 = rhi / R;
  const bool alu_vec = (a.N % R) == 0;
  // f(k-groups, first group) over this CTA's groups g0 + tid, g0 + tid + nt,
  // ..., Kc groups a step (each thread then has Kc 16-byte loads of every
  // operand in flight)
  auto for_groups = [&](auto Kc, auto&& f) {
    constexpr int K = decltype(Kc)::value;
    long long g = g0 + tid;
    if constexpr (K > 1)
      for (; g + (long long)(K - 1) * nt < g1; g += (long long)K * nt) f(Kc, g);
    for (; g < g1; g += nt) f(std::integral_constant<int, 1>{}, g);
  };
  // ndof 1: the vector phases move 16-byte groups of 4 rows, two groups a
  // step. Larger blocks keep one entry a thread a step: their groups (and
  // DIAG blocks) do not fit the register budget of 2 CTAs of 512 threads per
  // SM.
  constexpr int KP = 2;

  for (long long i = elo + tid; i < ehi; i += nt) {
    a.x[i] = 0.0;
    a.y[i] = 0.0f;
  }
  group_sync(cl, gsize);

  // r = b - A (x + y) in FP64 (stored FP32), z = M^-1 r, <r,r> and <r,z>
  auto refresh = [&](double (&v)[2]) {
    v[0] = v[1] = 0.0;
    for (long long row = rlo + tid; row < rhi; row += nt) {
      double ax[B];
      sell_row_f<B, U, double, double, kBatchCols16>(a.A64, XPlusYCoherent{a.x, a.y}, (int)row, ax);
      float t[B], w[B];
#pragma unroll
      for (int c = 0; c < B; c++) {
        const double rv = a.b[row * B + c] - ax[c];
        v[0] += rv * rv;
        t[c] = (float)rv;
        w[c] = t[c];
        a.r[row * B + c] = t[c];
      }
      if (a.prec) diag_row<B, float>(a.alu32, a.N, (int)row, w);
#pragma unroll
      for (int c = 0; c < B; c++) {
        a.z[row * B + c] = w[c];
        v[1] += (double)t[c] * (double)w[c];
      }
    }
    group_sum<2>(v, sh, cl, gsize, ph);
  };

  double v[2];
  refresh(v);
  const double B2 = v[0];
  int status = isfinite(B2) ? MONOLIS_B200_OK : MONOLIS_B200_NONFINITE, iter = 0, nref = 0;
  double resid = 0.0;  // B2 == 0: x = 0 solves the system (src/linalg/mat_converge.f90:40-48)
  if (B2 > 0.0 && isfinite(B2)) {
    double rmax = sqrt(v[0]), rho = v[1], rho1 = 0.0, beta = 0.0;
    bool fold = false;
    iter = 1;
    for (;;) {
      // P = Z + beta P (P = Z first); fold Y into X after a refresh
      const bool first = iter == 1;
      const float fb = (float)beta;
      if constexpr (B == 1) {
        for_groups(std::integral_constant<int, KP>{}, [&](auto Kc, long long g) {
          constexpr int KK = decltype(Kc)::value;
          float zv[KK][E], pv[KK][E];
#pragma unroll
          for (int k = 0; k < KK; k++) {
            const long long e0 = (g + (long long)k * nt) * E;
            vload<float, E>(a.z + e0, zv[k]);
            if (!first) vload<float, E>(a.p + e0, pv[k]);
          }
#pragma unroll
          for (int k = 0; k < KK; k++) {
#pragma unroll
            for (int e = 0; e < E; e++) pv[k][e] = first ? zv[k][e] : fmaf(fb, pv[k][e], zv[k][e]);
            vstore<float, E>(a.p + (g + (long long)k * nt) * E, pv[k]);
          }
          if (fold) {
#pragma unroll
            for (int k = 0; k < KK; k++) {
              const long long e0 = (g + (long long)k * nt) * E;
              double xv[E];
              float yv[E];
              vload<double, E>(a.x + e0, xv);
              vload<float, E>(a.y + e0, yv);
#pragma unroll
              for (int e = 0; e < E; e++) {
                xv[e] += (double)yv[e];
                yv[e] = 0.0f;
              }
              vstore<double, E>(a.x + e0, xv);
              vstore<float, E>(a.y + e0, yv);
            }
          }
        });
      } else {
        for (long long i = elo + tid; i < ehi; i += nt) {
          a.p[i] = first ? a.z[i] : fmaf(fb, a.p[i], a.z[i]);
          if (fold) {
            a.x[i] += (double)a.y[i];
            a.y[i] = 0.0f;
          }
        }
      }
      fold = false;
      group_sync(cl, gsize);
      // Q = A P (FP32), <P,Q>
      double w[1] = {0.0};
      if constexpr (B == 1) {
        // two row pairs a step, both pairs' loads in flight (sell_row2_two)
        auto xf = [&](long long i) { return ldx<true>(a.p + i); };
        for (long long t = plo + tid; t < phi; t += 2 * (long long)nt) {
          const long long tb = t + nt;
          const bool hb = tb < phi;
          float qa[2], qb[2];
          sell_row2_two<U, kBatchCols16>(a.A32, xf, (int)t, (int)(hb ? tb : t), hb, qa, qb);
          a.q[2 * t] = qa[0];
          a.q[2 * t + 1] = qa[1];
          w[0] += (double)a.p[2 * t] * (double)qa[0] + (double)a.p[2 * t + 1] * (double)qa[1];
          if (hb) {
            a.q[2 * tb] = qb[0];
            a.q[2 * tb + 1] = qb[1];
            w[0] += (double)a.p[2 * tb] * (double)qb[0] + (double)a.p[2 * tb + 1] * (double)qb[1];
          }
        }
      } else {
        for (long long t = plo + tid; t < phi; t += nt) {
          float q0[B], q1[B];
          sell_row2<B, U, true, kBatchCols16>(a.A32, a.p, (int)t, q0, q1);
#pragma unroll
          for (int c = 0; c < B; c++) {
            const long long i0 = 2 * t * B + c, i1 = (2 * t + 1) * B + c;
            a.q[i0] = q0[c];
            a.q[i1] = q1[c];
            w[0] += (double)a.p[i0] * (double)q0[c] + (double)a.p[i1] * (double)q1[c];
          }
        }
      }
      group_sum<1>(w, sh, cl, gsize, ph);
      if (w[0] == 0.0 || !isfinite(w[0])) {
        status = isfinite(w[0]) ? MONOLIS_B200_BREAKDOWN : MONOLIS_B200_NONFINITE;
        break;
      }
      const double alpha = rho / w[0];
      const float fa = (float)alpha;
      // Y += alpha P, R -= alpha Q, Z = M^-1 R, <R,R>, <R,Z>
      v[0] = v[1] = 0.0;
      if constexpr (B == 1) {
        for_groups(std::integral_constant<int, KP>{}, [&](auto Kc, long long g) {
          constexpr int KK = decltype(Kc)::value;
          float pv[KK][E], qv[KK][E], rv[KK][E], yv[KK][E];
#pragma unroll
          for (int k = 0; k < KK; k++) {
            const long long e0 = (g + (long long)k * nt) * E;
            vload<float, E>(a.p + e0, pv[k]);
            vload<float, E>(a.q + e0, qv[k]);
            vload<float, E>(a.r + e0, rv[k]);
            vload<float, E>(a.y + e0, yv[k]);
          }
#pragma unroll
          for (int k = 0; k < KK; k++) {
            const long long gk = g + (long long)k * nt, e0 = gk * E;
            float zz[E];
#pragma unroll
            for (int e = 0; e < E; e++) {
              yv[k][e] = fmaf(fa, pv[k][e], yv[k][e]);
              rv[k][e] = fmaf(-fa, qv[k][e], rv[k][e]);
              zz[e] = rv[k][e];
            }
            vstore<float, E>(a.y + e0, yv[k]);
            vstore<float, E>(a.r + e0, rv[k]);
            if (a.prec) diag_rows<B, float, R>(a.alu32, a.N, gk * R, alu_vec, zz);
            vstore<float, E>(a.z + e0, zz);
#pragma unroll
            for (int e = 0; e < E; e++) {
              v[0] += (double)rv[k][e] * (double)rv[k][e];
              v[1] += (double)rv[k][e] * (double)zz[e];
            }
          }
        });
      } else {
        for (long long row = rlo + tid; row < rhi; row += nt) {
          float t[B], zz[B];
#pragma unroll
          for (int c = 0; c < B; c++) {
            const long long i = row * B + c;
            a.y[i] = fmaf(fa, a.p[i], a.y[i]);
            t[c] = fmaf(-fa, a.q[i], a.r[i]);
            a.r[i] = t[c];
            zz[c] = t[c];
          }
          if (a.prec) diag_row<B, float>(a.alu32, a.N, (int)row, zz);
#pragma unroll
          for (int c = 0; c < B; c++) {
            a.z[row * B + c] = zz[c];
            v[0] += (double)t[c] * (double)t[c];
            v[1] += (double)t[c] * (double)zz[c];
          }
        }
      }
      group_sum<2>(v, sh, cl, gsize, ph);
      const double rn = sqrt(v[0]);
      resid = sqrt(v[0] / B2);
      if (!isfinite(resid)) {
        status = MONOLIS_B200_NONFINITE;
        break;
      }
      rmax = fmax(rmax, rn);
      const bool stop = resid < a.tol || iter >= a.max_iter;
      if (a.refine && (stop || rn < a.delta * rmax)) {
        refresh(v);  // every CTA has written its Y: the group_sum above synchronised
        nref++;
        fold = true;
        resid = sqrt(v[0] / B2);
        if (!isfinite(resid)) {
          status = MONOLIS_B200_NONFINITE;
          break;
        }
        if (resid < a.tol) break;
        if (iter >= a.max_iter) {
          status = MONOLIS_B200_MAXITER;
          break;
        }
        rmax = sqrt(v[0]);
      } else if (!a.refine && stop) {
        if (resid >= a.tol) status = MONOLIS_B200_MAXITER;
        refresh(v);  // true residual of x + y, reported
        resid = sqrt(v[0] / B2);
        fold = true;
        break;
      }
      rho1 = rho;
      rho = v[1];
      beta = rho / rho1;
      iter++;
    }
    if (fold) {  // every CTA has finished reading X and Y (the last group_sum)
      for (long long i = elo + tid; i < ehi; i += nt) {
        a.x[i] += (double)a.y[i];
        a.y[i] = 0.0f;
      }
    }
  }
  if (grank == 0 && tid == 0) {
    a.out_iter[si] = iter;
    a.out_status[si] = status;
    a.out_resid[si] = resid;
    a.out_nref[si] = nref;
  }
}

template <int B, int U>
__global__ void __launch_bounds__(kBatchMaxThreads, 2) batch_cg_kernel(const BatchArgs a) {
  __shared__ GroupShared sh;
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) sh.item = (int)atomicAdd(a.queue, 1u);
    cl.sync();
    const int item = *cl.map_shared_rank(&sh.item, 0);
    cl.sync();  // rank 0 rewrites sh.item only after every CTA has read it
    if (item >= a.nitems) return;
    const BatchItem it = a.items[item];
    // one call site (inlined): the whole cluster on one system, or one CTA per system
    const bool mine = !it.split || rank < it.count;
    if (mine)
      solve_system<B, U>(a, a.order[it.first + (it.split ? rank : 0)], it.split ? 1 : C, it.split ? 0 : rank, cl, sh);
  }
}

template <class P>
cudaError_t dalloc(P** p, size_t n) {
  return cudaMalloc((void**)p, n * sizeof(P) + 16);
}

}  // namespace

struct BatchConfig {
  int cluster = 0, threads = 0;
  long long split_rows = 0;
  int unroll = 0;  // SpMV slots in flight (0: the matrix's autotuned depth, at most 3)
};

struct BatchState {
  int ndof = 0;
  bool prepared = false;
  int prec = 1;
  // host CSR of the stacked matrix (0-based offsets, 1-based items)
  std::vector<int> index{0};
  std::vector<int> item;
  std::vector<double> val;
  std::vector<BatchSys> sys;
  long long nrows = 0;
  SellMatrix A;
  BatchSys* d_sys = nullptr;
  int* d_order = nullptr;
  BatchItem* d_items = nullptr;
  unsigned int* d_queue = nullptr;
  double *d_b = nullptr, *d_x = nullptr, *d_resid = nullptr;
  float *d_y = nullptr, *d_r = nullptr, *d_z = nullptr, *d_p = nullptr, *d_q = nullptr;
  int *d_iter = nullptr, *d_status = nullptr, *d_nref = nullptr;
  std::vector<int> order;  // systems by decreasing stored blocks
  BatchConfig cfg;
  int nitems = 0;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  double last_loop_s = 0.0;
};

namespace {

void free_state(BatchState* s) {
  if (s->exec) cudaGraphExecDestroy(s->exec);
  sell_free(s->A);
  cudaFree(s->d_sys);
  cudaFree(s->d_order);
  cudaFree(s->d_items);
  cudaFree(s->d_queue);
  cudaFree(s->d_b);
  cudaFree(s->d_x);
  cudaFree(s->d_resid);
  cudaFree(s->d_y);
  cudaFree(s->d_r);
  cudaFree(s->d_z);
  cudaFree(s->d_p);
  cudaFree(s->d_q);
  cudaFree(s->d_iter);
  cudaFree(s->d_status);
  cudaFree(s->d_nref);
}

// Work items for a configuration: systems in decreasing size; those with at
// least split_rows block rows each get the whole cluster, the rest go
// `cluster` at a time, one per CTA.
std::vector<BatchItem> make_items(const BatchState& s, const BatchConfig& c) {
  std::vector<BatchItem> items;
  const int n = (int)s.order.size();
  int i = 0;
  while (i < n) {
    if (c.cluster == 1 || s.sys[s.order[i]].nrows >= c.split_rows) {
      items.push_back({i, 1, c.cluster == 1 ? 1 : 0});
      i++;
    } else {
      const int k = std::min(c.cluster, n - i);
      items.push_back({i, k, 1});
      i += k;
    }
  }
  return items;
}

// The batch kernel runs at 2 CTAs of 512 threads per SM (64 registers a
// thread), so its rows take at most 3 slots in flight.
template <class F>
int dispatch_batch(int ndof, int u, F&& f) {
  return dispatch_ndof(ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    return dispatch_u(u > 3 ? 3 : u, [&](auto Uc) {
      constexpr int U = eff_u(B, decltype(Uc)::value > 3 ? 3 : decltype(Uc)::value);
      return f(batch_cg_kernel<B, U>);
    });
  });
}

// Record the solve (queue reset + persistent kernel) for configuration c.
int build_graph(BatchState* s, const BatchConfig& c, const BatchArgs& args0) {
  std::vector<BatchItem> items = make_items(*s, c);
  MB_CUDA_OK(cudaMemcpyAsync(s->d_items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice,
                             s->stream));
  BatchArgs args = args0;
  args.nitems = (int)items.size();
  s->nitems = args.nitems;
  if (s->exec) {
    cudaGraphExecDestroy(s->exec);
    s->exec = nullptr;
  }
  return dispatch_batch(s->ndof, c.unroll > 0 ? c.unroll : s->A.u32, [&](auto kernel) -> int {
    if (c.cluster > 8)
      MB_CUDA_OK(cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(c.threads);
    cfg.gridDim = dim3(c.cluster);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int max_clusters = 0;
    MB_CUDA_OK(cudaOccupancyMaxActiveClusters(&max_clusters, kernel, &cfg));
    if (max_clusters < 1) return kBadInput;
    // a resident grid: every cluster can run at once (more would only wait)
    const int nclusters = std::min(max_clusters, std::max(1, args.nitems));
    cfg.gridDim = dim3(nclusters * c.cluster);
    cudaGraph_t g;
    MB_CUDA_OK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(s->d_queue, 0, sizeof(unsigned int), s->stream);
    cudaLaunchKernelEx(&cfg, kernel, args);
    MB_CUDA_OK(cudaStreamEndCapture(s->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&s->exec, g, 0);
    cudaGraphDestroy(g);
    MB_CUDA_OK(e);
    return kOk;
  });
}

BatchArgs base_args(BatchState* s, double tol, int max_iter, int refine, double delta) {
  BatchArgs a{};
  a.A32 = view2_of(s->A);
  a.A64 = view_of<double>(s->A);
  a.alu32 = s->A.d_alu32;
  a.N = s->A.N;
  a.prec = s->prec;
  a.refine = refine;
  a.max_iter = max_iter;
  a.tol = tol;
  a.delta = delta > 0.0 ? delta : 0.1;
  a.sys = s->d_sys;
  a.order = s->d_order;
  a.items = s->d_items;
  a.queue = s->d_queue;
  a.b = s->d_b;
  a.x = s->d_x;
  a.y = s->d_y;
  a.r = s->d_r;
  a.z = s->d_z;
  a.p = s->d_p;
  a.q = s->d_q;
  a.out_iter = s->d_iter;
  a.out_status = s->d_status;
  a.out_nref = s->d_nref;
  a.out_resid = s->d_resid;
  return a;
}

int run_graph(BatchState* s, double* seconds) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s->stream);
  cudaError_t e = cudaGraphLaunch(s->exec, s->stream);
  cudaEventRecord(e1, s->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  MB_CUDA_OK(e);
  if (seconds) *seconds = ms * 1e-3;
  return kOk;
}

}  // namespace

int batch_add(BatchState* s, int N, int ndof, const int* index, const int* item, const double* val) {
  if (s->prepared || N <= 0 || ndof <= 0 || ndof > 6) return kBadInput;
  if (s->ndof && s->ndof != ndof) return kBadInput;
  s->ndof = ndof;
  const int B2 = ndof * ndof;
  const long long row0 = s->nrows;
  const int padded = (N + kBatchRowAlign - 1) / kBatchRowAlign * kBatchRowAlign;
  const long long nz = index[N];
  if ((long long)s->item.size() + nz + (padded - N) > 2147483647LL) return kBadInput;
  for (int i = 0; i < N; i++) {
    for (int k = index[i]; k < index[i + 1]; k++) {
      if (item[k] < 1 || item[k] > N) return kBadInput;
      s->item.push_back((int)(item[k] + row0));
    }
    s->index.push_back((int)s->item.size());
  }
  s->val.insert(s->val.end(), val, val + nz * B2);
  for (int i = N; i < padded; i++) {  // identity rows: x = b = 0 there
    s->item.push_back((int)(row0 + i + 1));
    s->index.push_back((int)s->item.size());
    for (int e = 0; e < B2; e++) s->val.push_back(e % (ndof + 1) == 0 ? 1.0 : 0.0);
  }
  s->sys.push_back({row0, padded, N});
  s->nrows += padded;
  return kOk;
}

int batch_prepare(BatchState* s, int precond, cudaStream_t stream) {
  if (s->sys.empty()) return kBadInput;
  if (s->nrows > 2147483647LL / 2) return kBadInput;
  s->stream = stream;
  s->prec = precond;
  const int N = (int)s->nrows, nd = s->ndof;
  int rc = sell_build(s->A, s->index.data(), s->item.data(), s->val.data(), N, nd, stream, nullptr);
  if (rc) return rc;
  rc = diag_setup(s->A, stream);
  if (rc) return rc;
  rc = sell_make_fp32(s->A, stream);
  if (rc) return rc;
  const int ns = (int)s->sys.size();
  s->order.resize(ns);
  std::iota(s->order.begin(), s->order.end(), 0);
  std::vector<long long> blocks(ns);
  for (int i = 0; i < ns; i++) blocks[i] = s->index[s->sys[i].row0 + s->sys[i].nrows] - s->index[s->sys[i].row0];
  std::stable_sort(s->order.begin(), s->order.end(), [&](int a, int b) { return blocks[a] > blocks[b]; });
  const size_t n = (size_t)N * nd;
  MB_CUDA_OK(dalloc(&s->d_sys, ns));
  MB_CUDA_OK(dalloc(&s->d_order, ns));
  MB_CUDA_OK(dalloc(&s->d_items, ns));
  MB_CUDA_OK(dalloc(&s->d_queue, 1));
  MB_CUDA_OK(dalloc(&s->d_b, n));
  MB_CUDA_OK(dalloc(&s->d_x, n));
  MB_CUDA_OK(dalloc(&s->d_y, n));
  MB_CUDA_OK(dalloc(&s->d_r, n));
  MB_CUDA_OK(dalloc(&s->d_z, n));
  MB_CUDA_OK(dalloc(&s->d_p, n));
  MB_CUDA_OK(dalloc(&s->d_q, n));
  MB_CUDA_OK(dalloc(&s->d_iter, ns));
  MB_CUDA_OK(dalloc(&s->d_status, ns));
  MB_CUDA_OK(dalloc(&s->d_nref, ns));
  MB_CUDA_OK(dalloc(&s->d_resid, ns));
  MB_CUDA_OK(cudaMemsetAsync(s->d_b, 0, n * sizeof(double), stream));
  MB_CUDA_OK(cudaMemsetAsync(s->d_x, 0, n * sizeof(double), stream));
  MB_CUDA_OK(cudaMemcpyAsync(s->d_sys, s->sys.data(), sizeof(BatchSys) * ns, cudaMemcpyHostToDevice, stream));
  MB_CUDA_OK(cudaMemcpyAsync(s->d_order, s->order.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, stream));
  MB_CUDA_OK(cudaStreamSynchronize(stream));
  // the host copy of the stacked CSR is no longer needed
  std::vector<int>().swap(s->item);
  std::vector<double>().swap(s->val);
  s->prepared = true;
  return kOk;
}

int batch_set_config(BatchState* s, int cluster, int threads, long long split_rows) {
  if (!s->prepared) return kBadInput;
  if (cluster < 1 || cluster > 16 || (cluster & (cluster - 1)) || threads < 64 || threads > kBatchMaxThreads ||
      threads % 32)
    return kBadInput;
  BatchConfig c{cluster, threads, split_rows, s->cfg.unroll};
  s->cfg = c;
  if (s->exec) {
    cudaGraphExecDestroy(s->exec);
    s->exec = nullptr;
  }
  return kOk;
}

int batch_solve_device(BatchState* s, double tol, int max_iter, int refine, double delta, double* seconds) {
  if (!s->prepared || s->cfg.cluster == 0) return kBadInput;
  int rc = build_graph(s, s->cfg, base_args(s, tol, max_iter, refine, delta));
  if (rc) return rc;
  rc = run_graph(s, seconds);
  if (seconds) s->last_loop_s = *seconds;
  return rc;
}

// Times each candidate configuration on the batch (right-hand side b = 1,
// `iters` iterations) and keeps the fastest; then, at that configuration,
// the SpMV unroll depth 1, 2 or 3.
int batch_autotune(BatchState* s, int iters, std::vector<std::pair<BatchConfig, double>>* log) {
  if (!s->prepared) return kBadInput;
  const size_t n = (size_t)s->nrows * s->ndof;
  std::vector<double> ones(n, 1.0);
  double* d_save = nullptr;
  MB_CUDA_OK(dalloc(&d_save, n));
  MB_CUDA_OK(cudaMemcpyAsync(d_save, s->d_b, n * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  MB_CUDA_OK(cudaMemcpyAsync(s->d_b, ones.data(), n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  long long max_rows = 0;
  for (auto& q : s->sys) max_rows = std::max<long long>(max_rows, q.nrows);
  std::vector<BatchConfig> cand;
  for (int c : {1, 2, 4, 8})
    for (int t : {256, 512})
      for (long long split : {0LL, 8192LL, 32768LL}) {
        if (c == 1 && split != 0) continue;
        if (split > max_rows) continue;
        cand.push_back({c, t, split});
      }
  double best = 1e30;
  BatchConfig bc{};
  int rc = kOk;
  for (const BatchConfig& c : cand) {
    s->cfg = c;
    double t0 = 0.0, t1 = 0.0;
    rc = batch_solve_device(s, 0.0, iters, 0, 0.0, &t0);  // warm
    if (!rc) rc = batch_solve_device(s, 0.0, iters, 0, 0.0, &t1);
    if (rc) break;
    if (log) log->push_back({c, t1});
    if (t1 < best) {
      best = t1;
      bc = c;
    }
  }
  for (int u = 1; u <= 3 && rc == kOk && bc.cluster > 0; u++) {
    BatchConfig c = bc;
    c.unroll = u;
    s->cfg = c;
    double t0 = 0.0, t1 = 0.0;
    rc = batch_solve_device(s, 0.0, iters, 0, 0.0, &t0);  // warm
    if (!rc) rc = batch_solve_device(s, 0.0, iters, 0, 0.0, &t1);
    if (rc) break;
    if (log) log->push_back({c, t1});
    if (t1 < best) {
      best = t1;
      bc = c;
    }
  }
  cudaMemcpyAsync(s->d_b, d_save, n * sizeof(double), cudaMemcpyDeviceToDevice, s->stream);
  cudaStreamSynchronize(s->stream);
  cudaFree(d_save);
  if (rc) return rc;
  s->cfg = bc;
  if (s->exec) {
    cudaGraphExecDestroy(s->exec);
    s->exec = nullptr;
  }
  return kOk;
}

}  // namespace mb

// ---------------------------------------------------------------------------
// C ABI (include/monolis_b200.h)
// ---------------------------------------------------------------------------
struct monolis_b200_batch {
  mb::BatchState s;
};

namespace {
cudaStream_t batch_stream() { return static_cast<cudaStream_t>(monolis_b200_stream()); }
}  // namespace

extern "C" {

int monolis_b200_batch_create(monolis_b200_batch** out) {
  if (!out) return MONOLIS_B200_BAD_INPUT;
  *out = new monolis_b200_batch();
  return MONOLIS_B200_OK;
}

void monolis_b200_batch_destroy(monolis_b200_batch* b) {
  if (!b) return;
  cudaStream_t st = batch_stream();
  if (st) cudaStreamSynchronize(st);
  mb::free_state(&b->s);
  delete b;
}

int monolis_b200_batch_add_system(monolis_b200_batch* b, MONOLIS* mat) {
  if (!b || !mat || !mat->mat.CSR.index || !mat->mat.CSR.item || !mat->mat.R.A) return MONOLIS_B200_BAD_INPUT;
  if (mat->mat.N != mat->mat.NP) return MONOLIS_B200_BAD_INPUT;
  return mb::batch_add(&b->s, mat->mat.N, mat->mat.NDOF, mat->mat.CSR.index, mat->mat.CSR.item, mat->mat.R.A);
}

int monolis_b200_batch_add_csr(monolis_b200_batch* b, int n, int ndof, const int* index, const int* item,
                               const double* val) {
  if (!b || !index || !item || !val || n <= 0) return MONOLIS_B200_BAD_INPUT;
  std::vector<int> it1(item, item + index[n]);
  for (int& v : it1) v += 1;
  return mb::batch_add(&b->s, n, ndof, index, it1.data(), val);
}

int monolis_b200_batch_prepare(monolis_b200_batch* b, int precond, int autotune) {
  if (!b || (precond != MONOLIS_PREC_NONE && precond != MONOLIS_PREC_DIAG)) return MONOLIS_B200_BAD_INPUT;
  cudaStream_t st = batch_stream();
  if (!st) return MONOLIS_B200_CUDA_ERROR;
  int rc = mb::batch_prepare(&b->s, precond == MONOLIS_PREC_DIAG ? 1 : 0, st);
  if (rc) return rc;
  if (autotune) return mb::batch_autotune(&b->s, 30, nullptr);
  return mb::batch_set_config(&b->s, 4, 256, 32768);
}

int monolis_b200_batch_set_config(monolis_b200_batch* b, int cluster, int threads, long long split_rows) {
  if (!b) return MONOLIS_B200_BAD_INPUT;
  return mb::batch_set_config(&b->s, cluster, threads, split_rows);
}

int monolis_b200_batch_get_config(monolis_b200_batch* b, int* cluster, int* threads, long long* split_rows) {
  if (!b || !b->s.prepared) return MONOLIS_B200_BAD_INPUT;
  if (cluster) *cluster = b->s.cfg.cluster;
  if (threads) *threads = b->s.cfg.threads;
  if (split_rows) *split_rows = b->s.cfg.split_rows;
  return MONOLIS_B200_OK;
}

int monolis_b200_batch_get_unroll(monolis_b200_batch* b, int* unroll) {
  if (!b || !b->s.prepared || !unroll) return MONOLIS_B200_BAD_INPUT;
  const int u = b->s.cfg.unroll > 0 ? b->s.cfg.unroll : b->s.A.u32;
  *unroll = u > 3 ? 3 : u;
  return MONOLIS_B200_OK;
}

int monolis_b200_batch_info(monolis_b200_batch* b, int* n_systems, long long* offsets) {
  if (!b) return MONOLIS_B200_BAD_INPUT;
  const auto& s = b->s;
  if (n_systems) *n_systems = (int)s.sys.size();
  if (offsets)
    for (size_t i = 0; i < s.sys.size(); i++) offsets[i] = s.sys[i].row0 * s.ndof;
  return MONOLIS_B200_OK;
}

int monolis_b200_batch_device_vectors(monolis_b200_batch* b, double** d_b, double** d_x) {
  if (!b || !b->s.prepared) return MONOLIS_B200_BAD_INPUT;
  if (d_b) *d_b = b->s.d_b;
  if (d_x) *d_x = b->s.d_x;
  return MONOLIS_B200_OK;
}

int monolis_b200_batch_device_solve_R(monolis_b200_batch* b, double tol, int max_iter, int refine, int* iter,
                                      double* resid, int* status) {
  if (!b || !b->s.prepared || max_iter < 1 || !(tol >= 0.0)) return MONOLIS_B200_BAD_INPUT;
  mb::BatchState& s = b->s;
  double t = 0.0;
  int rc = mb::batch_solve_device(&s, tol, max_iter, refine, 0.0, &t);
  if (rc) return rc;
  const size_t ns = s.sys.size();
  if (iter) MB_CUDA_OK(cudaMemcpyAsync(iter, s.d_iter, ns * sizeof(int), cudaMemcpyDeviceToHost, s.stream));
  if (resid) MB_CUDA_OK(cudaMemcpyAsync(resid, s.d_resid, ns * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
  if (status) MB_CUDA_OK(cudaMemcpyAsync(status, s.d_status, ns * sizeof(int), cudaMemcpyDeviceToHost, s.stream));
  MB_CUDA_OK(cudaStreamSynchronize(s.stream));
  return MONOLIS_B200_OK;
}

int monolis_b200_batch_solve_R(monolis_b200_batch* b, double** B, double** X, double tol, int max_iter, int refine,
                               int* iter, double* resid, int* status) {
  if (!b || !b->s.prepared || !B || !X) return MONOLIS_B200_BAD_INPUT;
  mb::BatchState& s = b->s;
  const int nd = s.ndof;
  for (size_t i = 0; i < s.sys.size(); i++) {
    const auto& q = s.sys[i];
    MB_CUDA_OK(cudaMemcpyAsync(s.d_b + q.row0 * nd, B[i], sizeof(double) * q.real_rows * nd, cudaMemcpyHostToDevice,
                               s.stream));
  }
  int rc = monolis_b200_batch_device_solve_R(b, tol, max_iter, refine, iter, resid, status);
  if (rc) return rc;
  for (size_t i = 0; i < s.sys.size(); i++) {
    const auto& q = s.sys[i];
    MB_CUDA_OK(cudaMemcpyAsync(X[i], s.d_x + q.row0 * nd, sizeof(double) * q.real_rows * nd, cudaMemcpyDeviceToHost,
                               s.stream));
  }
  MB_CUDA_OK(cudaStreamSynchronize(s.stream));
  return MONOLIS_B200_OK;
}

double monolis_b200_batch_last_seconds(monolis_b200_batch* b) { return b ? b->s.last_loop_s : 0.0; }

int monolis_b200_batch_autotune(monolis_b200_batch* b, int iters, int* n_candidates, int* clusters, int* threads,
                                long long* splits, double* seconds) {
  if (!b || !b->s.prepared || iters < 1) return MONOLIS_B200_BAD_INPUT;
  std::vector<std::pair<mb::BatchConfig, double>> log;
  int rc = mb::batch_autotune(&b->s, iters, &log);
  if (rc) return rc;
  const int cap = n_candidates ? *n_candidates : 0;
  for (int i = 0; i < (int)log.size() && i < cap; i++) {
    if (clusters) clusters[i] = log[i].first.cluster;
    if (threads) threads[i] = log[i].first.threads;
    if (splits) splits[i] = log[i].first.split_rows;
    if (seconds) seconds[i] = log[i].second;
  }
  if (n_candidates) *n_candidates = (int)log.size();
  return MONOLIS_B200_OK;
}

}  // extern "C"
