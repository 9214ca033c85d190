// dev.h -- host-visible device data structures and kernel launchers.
//
// Device layout of one block-CSR matrix (N block rows of ndof x ndof blocks):
// a sliced ELL ("SELL-32") copy built on the device from the uploaded CSR.
// Rows are grouped in slices of 32 consecutive rows (one warp); slice s owns
// 32 * w_s block slots, w_s = longest row in the slice. Slot k of the row at
// lane l of slice s is block b = slptr[s] + 32*k + l; its column id is col[b]
// and entry (r,c) of its value block is val[(slptr[s] + 32*k)*nd2 +
// (r*ndof + c)*32 + l]. A warp therefore reads every value and column id as a
// contiguous 128/256-byte line, one thread owns one block row and walks its
// blocks in CSR (ascending column) order, which is the reference's summation
// order. Padded slots (k >= row length) are never read: each thread stops at
// its own row length, taken from the CSR offsets.
//
// Column ids are also kept compressed: for slot k of slice s, cbase[slptr[s]/32
// + k] holds a base column c0 and col16[b] the 16-bit difference col[b] - c0 -
// l, which is zero wherever the 32 rows of a slice have the same stencil (a
// structured mesh) and small for any locally numbered mesh. A slice whose
// differences do not all fit in 16 bits keeps reading col[]; slc[s] is
// slptr[s] with bit 0 set for those slices. The compressed stream is 2 bytes
// per block plus 4 bytes per slot per warp instead of 4 bytes per block. A
// slice whose differences are all zero (every lane's block k at the same
// offset from its row, the interior of a structured mesh) has bit 1 set and
// reads only the bases: 4 bytes per slot per warp.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

namespace mb {

// Status codes written to Iarray[MONOLIS_PRM_I_IERR] (see monolis_b200.h).
enum Status : int {
  kOk = 0,
  kMaxIter = 1,
  kBreakdown = 2,
  kNonFinite = 3,
  kTimeout = 4,
  kBadInput = 5,
  kCudaError = 6,
  kZeroRhs = 7,  // internal: B2 == 0, x set to zero (reported as kOk)
};

struct SolverState {
  double rho, rho1, alpha, beta, omega, c2, B2, resid, tol;
  double rr, ts, tt;
  double rmax;   // mixed: largest iterated-residual norm since the last refresh
  double delta;  // mixed: refresh when the residual norm < delta * rmax
  int iter, max_iter, done, status;
  int iter_rr;   // true residual every iter_rr iterations (FP64 CG / BiCGSTAB)
  int rr_flag;   // true residual due in this iteration
  int period;    // mixed: refresh at the latest `period` iterations after the last (0: no limit)
  int last_refresh;
  int refresh;   // mixed: refresh due in this iteration
  int fold;      // mixed: y still to be folded into x
  int n_refine;  // mixed: refreshes done
  int sharded;   // multi-rank: reductions leave their local sums in red[] for the all-reduce
  int loops;     // device-side loop: bodies of iterations run (while-node graph)
  double red[4];
};

struct SellMatrix {
  int N = 0, ndof = 0, nslices = 0;
  long long nz = 0, padded = 0;
  int* d_rowptr = nullptr;        // CSR offsets (N+1)
  long long* d_slptr = nullptr;   // nslices+1, in blocks
  int* d_col = nullptr;           // padded block column ids, 0-based
  double* d_val64 = nullptr;
  float* d_val32 = nullptr;       // FP32 values in the paired layout below
  // FP32 copy in the paired layout: slices of 64 rows, lane l of a warp owns
  // rows 64s+2l and 64s+2l+1, so values and column ids are read as float2 /
  // int2 (8 bytes per lane, the byte rate of the FP64 layout).
  int nslices2 = 0;
  long long padded2 = 0;
  long long* d_slptr2 = nullptr;  // nslices2+1, in blocks
  int* d_col2 = nullptr;
  // compressed column ids (above) of both layouts; the paired layout has one
  // base per slot of 64 rows and a pair of differences per lane:
  // col = cbase2[slptr2[s]/64 + k] + 2l + h + col16p[slptr2[s] + 64k + 2l + h]
  long long* d_slc = nullptr;
  short* d_col16 = nullptr;
  int* d_cbase = nullptr;
  long long* d_slc2 = nullptr;
  short* d_col16p = nullptr;
  int* d_cbase2 = nullptr;
  long long wide64 = 0, wide32 = 0;  // slices that keep 32-bit column ids
  long long uniform64 = 0, uniform32 = 0;  // slices whose columns are the slot bases + lane (bit 1 of slc)
  double bytes64 = 0, bytes32 = 0;   // HBM bytes of one SpMV in each layout
  // unroll depth (slots in flight per thread) picked by the autotuner
  int u64 = 2, u32 = 2;
  // shape (N and ndof, NZ, padded slots) the depths were timed on: a rebuild
  // of the same shape keeps them (the depth only affects speed)
  long long tuned64[3] = {-1, -1, -1}, tuned32[3] = {-1, -1, -1};
  double* d_alu64 = nullptr;      // DIAG factors, entry-major: alu[e*N + row]
  float* d_alu32 = nullptr;
  // upload staging (kept between solves)
  int* d_item = nullptr;          // CSR items as uploaded (1-based)
  double* d_csrval = nullptr;
  size_t cap_rowptr = 0, cap_slptr = 0, cap_col = 0, cap_val64 = 0, cap_val32 = 0;
  size_t cap_alu64 = 0, cap_alu32 = 0, cap_item = 0, cap_csrval = 0, cap_slptr2 = 0, cap_col2 = 0;
  size_t cap_slc = 0, cap_col16 = 0, cap_cbase = 0, cap_slc2 = 0, cap_col16p = 0, cap_cbase2 = 0;
  bool have_val32 = false, have_alu = false, have_alu32 = false;
};

struct Scratch {
  double* partials = nullptr;     // (65536 + 256) * 4 doubles: block and group partial sums
  unsigned int* ticket = nullptr;
  SolverState* st = nullptr;
  SolverState* h_st = nullptr;    // pinned host mirror, one slot per launch in flight (8)
  double* hist = nullptr;         // residual history (max_iter + 1)
  size_t hist_cap = 0;
  size_t partials_cap = 0;
};

// ---- matrix build on the device ----
int sell_build(SellMatrix& m, const int* h_index, const int* h_item, const double* h_val,
               int N, int ndof, cudaStream_t s, double* t_h2d);
// Slices and FP64 values from the device CSR (d_rowptr, d_item, d_csrval).
int sell_layout(SellMatrix& m, cudaStream_t s);
// A^T from A's device CSR and the host CSC arrays of the pattern (offsets,
// 1-based rows, 1-based CSR positions; monolis_get_CSC_format).
int sell_build_transpose(SellMatrix& at, const SellMatrix& a, const int* h_csc_index, const int* h_csc_item,
                         const int* h_csc_perm, cudaStream_t s);
int sell_make_fp32(SellMatrix& m, cudaStream_t s);
// Times the SpMV unroll variants on the matrix and keeps the fastest (u64 / u32).
int sell_autotune(SellMatrix& m, bool fp32, cudaStream_t s);
int diag_setup(SellMatrix& m, cudaStream_t s);  // FP64 (+FP32 copy when have_val32)
void sell_free(SellMatrix& m);

// ---- kernels callable on their own ----
int spmv64(const SellMatrix& m, const double* x, double* y, cudaStream_t s);
int spmv32(const SellMatrix& m, const float* x, float* y, cudaStream_t s);
int dot64(long long n, const double* x, const double* y, double* out, Scratch& sc, cudaStream_t s);
int diag_apply64(const SellMatrix& m, const double* x, double* y, cudaStream_t s);

// ---- adjoint pieces (adjoint.cu) ----
// G (stored blocks x ndof^2, the layout of the matrix values) =
// scale * lambda_i x_j^T over the pattern of m.
int outer_product64(const SellMatrix& m, const double* lam, const double* x, double scale, double* G,
                    cudaStream_t s);
// grad[e] = scale * sum_ab lam_a K_e(a,b) x_b over each element's local dofs,
// lam_a taken as zero where fixed[dof] != 0 (fixed may be null).
int element_gradient64(int n_elem, int n_base, int ndof, const int* elem, const double* Ke, long long ke_stride,
                       const double* lam, const double* x, const int* fixed, double scale, double* grad,
                       cudaStream_t s);

// ---- solvers (device-resident loops) ----
// ---- row-partitioned (multi-rank) solve (shard.cu) ----
// Halo tables of one rank: for every neighbour, the local block rows it sends
// (send_item, 0-based) or receives into (recv_item, ghost rows), with offsets.
struct ShardTables {
  int rank = 0;  // this rank (a neighbour entry equal to it is a local copy)
  std::vector<int> send_pe, send_ptr, send_item, recv_pe, recv_ptr, recv_item;
};
struct ShardPlan {
  void* comm = nullptr;  // ncclComm_t
  int ndof = 0, rank = 0;
  std::vector<int> send_pe, recv_pe, send_ptr, recv_ptr;
  long long n_send = 0, n_recv = 0;
  int* d_send_item = nullptr;
  int* d_recv_item = nullptr;
  void* d_sendbuf = nullptr;
  void* d_recvbuf = nullptr;
  // 32-row slices of the device matrix: those whose rows read no ghost entry
  // (interior) first, then the others (boundary); the interior product runs
  // while the halo update is in flight on `side`
  int* d_slices = nullptr;
  int n_int = 0, n_bnd = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};
int shard_unique_id(void* out128);
int shard_comm_create(void** comm, const void* id128, int rank, int size);
void shard_comm_destroy(void* comm);
int shard_setup(ShardPlan& sp, const ShardTables& t, int ndof, const SellMatrix& A, cudaStream_t s);
void shard_free(ShardPlan& sp);
int shard_halo(const ShardPlan& sp, double* v, cudaStream_t s);
int shard_halo(const ShardPlan& sp, float* v, cudaStream_t s);  // FP32 vectors (refined solve)
// halo update of v on the side stream, ordered after the work already on s;
// shard_halo_join makes s wait for it
int shard_halo_fork(const ShardPlan& sp, double* v, cudaStream_t s);
int shard_halo_join(const ShardPlan& sp, cudaStream_t s);
// all-reduce of k doubles on the side stream, after the work already on s
// (shard_halo_join makes s wait for it); no other collective is issued until
// it has been joined
int shard_allreduce_fork(const ShardPlan& sp, double* d, int k, cudaStream_t s);
int shard_allreduce(const ShardPlan& sp, double* d, int k, cudaStream_t s);

struct SolveParams {
  int method;        // MONOLIS_ITER_CG / MONOLIS_ITER_BICGSTAB
  int precond;       // MONOLIS_PREC_NONE / MONOLIS_PREC_DIAG
  int max_iter;
  double tol;
  int init_x;        // zero x before solving
  int precision;     // 0 FP64, 1 FP32 inner + FP64 reliable refresh
  double delta;        // precision 1: refresh when ||r|| < delta * max ||r|| since the last one (0: 0.1 CG, 0.01 BiCGSTAB)
  int refresh_period;  // precision 1: refresh at the latest every n iterations (0: no limit)
  int iter_rr;       // true residual every iter_rr iterations (reference: 200)
  int batch;         // iterations per graph launch
  int use_graph;
  int timers;        // time every kernel with CUDA events (no graph)
  const ShardPlan* shard = nullptr;  // multi-rank solve (FP64 CG); x holds np_rows block rows (ghosts last)
  int np_rows = 0;
};
struct SolveResult {
  int iter = 0, status = 0, n_refine = 0;
  double resid = 0.0;
  double t_loop = 0.0;  // device loop seconds
  long long launches = 0;  // kernels launched by the solve
  std::vector<double> kernel_time;     // timers: seconds per kernel slot of an iteration
  double t_kind[3] = {0.0, 0.0, 0.0};  // timers: SpMV / other vector / precond kernels
};

int solve_device(SellMatrix& m, Scratch& sc, const SolveParams& p, const double* d_b, double* d_x,
                 SolveResult& res, double* h_hist, cudaStream_t s);

// ---- device assembly (assemble.cu): values of m's device CSR (d_csrval) ----
int device_add_elements(SellMatrix& m, int NP, int n_elem, int n_base, const int* d_elem, const double* d_val,
                        long long val_stride, const double* d_scale, cudaStream_t s);
// node/dof/val: host lists of n_bc conditions, applied as if in order; d_b device RHS
int device_dirichlet(SellMatrix& m, double* d_b, int n_bc, const int* node, const int* dof, const double* val,
                     cudaStream_t s);

// ---- many right-hand sides on one matrix (multi.cu) ----
struct MultiState;
MultiState* multi_new();
void multi_free(MultiState* ms);
// n_rhs systems A X_k = B_k with B_k at d_B + k*N*ndof (device); precision 1:
// FP32 loop with FP64 refresh, 0: FP64. build_id identifies the device
// matrix contents (the FP32 CSR copy is rebuilt when it changes).
// wait_limit: polls before a grid-barrier wait gives up (0: the default,
// seconds); delay_ns: testing, block 0 arrives that much later at the first
// barrier. A wait that gives up ends the solve with kTimeout.
int multi_solve(SellMatrix& m, MultiState& ms, long long build_id, int n_rhs, const double* d_B, double* d_X,
                int precision, int prec, double tol, int max_iter, double delta, unsigned long long wait_limit,
                unsigned int delay_ns, int* iter, double* resid, int* status, cudaStream_t s);

int scratch_ensure(Scratch& sc, size_t hist_len);
void scratch_free(Scratch& sc);

}  // namespace mb
