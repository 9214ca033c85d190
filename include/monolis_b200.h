/* monolis_b200.h -- entry points that libmonolis_b200.so adds to the monolis
 * C API (include/monolis.h). None of them has a counterpart in the reference
 * library unless its comment cites one; they expose what the reference keeps
 * internal (device residency, precision) and the added solver forms.
 *
 * All functions return 0 on success or a MONOLIS_B200_* status code; the
 * same code is written to mat->prm.Iarray[MONOLIS_PRM_I_IERR] by solves.
 */
#ifndef MONOLIS_B200_H
#define MONOLIS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#include <stdbool.h>
#include "monolis.h"

/* ---- status codes (Iarray[MONOLIS_PRM_I_IERR]; the reference leaves it at -1) ---- */
static const int MONOLIS_B200_OK         = 0;
static const int MONOLIS_B200_MAXITER    = 1; /* max_iter reached without convergence */
static const int MONOLIS_B200_BREAKDOWN  = 2; /* BiCGSTAB: rho or (RT,V) exactly zero */
static const int MONOLIS_B200_NONFINITE  = 3; /* residual became NaN/Inf */
static const int MONOLIS_B200_TIMEOUT    = 4; /* device loop gave no verdict */
static const int MONOLIS_B200_BAD_INPUT  = 5; /* unsupported method/precond/ndof or bad arrays */
static const int MONOLIS_B200_CUDA_ERROR = 6;

/* ---- added parameter slots (indices the reference leaves unused, >= 30) ---- */
static const int MONOLIS_B200_PRM_I_PRECISION      = 30; /* 0: FP64 (default), 1: FP32 inner + FP64 refinement */
static const int MONOLIS_B200_PRM_I_MATRIX_CACHE   = 31; /* 1: reuse the device matrix while MATRIX_VERSION is unchanged */
static const int MONOLIS_B200_PRM_I_MATRIX_VERSION = 32; /* bumped by every matrix-mutating call of this library */
static const int MONOLIS_B200_PRM_I_N_REFINE       = 33; /* out: FP64 residual refreshes of the mixed solver */
static const int MONOLIS_B200_PRM_I_BATCH          = 34; /* iterations per graph launch (0: 16) */
static const int MONOLIS_B200_PRM_I_CHECK          = 35; /* 1: validate CSR index/item before upload */
static const int MONOLIS_B200_PRM_I_LAUNCHES       = 36; /* out: kernels launched by the last solve */
static const int MONOLIS_B200_PRM_I_ITER_RR        = 37; /* true-residual interval of CG/BiCGSTAB/PipeCG (0: the
                                                            reference's 200, PipeCG 50; GropCG has none) */
static const int MONOLIS_B200_PRM_I_UNROLL_FP64    = 38; /* out: SpMV unroll depth picked by the autotuner (FP64) */
static const int MONOLIS_B200_PRM_I_UNROLL_FP32    = 39; /* out: same for the FP32 layout */
static const int MONOLIS_B200_PRM_I_KERNEL_TIMERS  = 40; /* 1: time every kernel with CUDA events (no graph; slower loop);
                                                            fills TIME_SPMV / DOTP / PREC and TIME_KERNEL+k */
static const int MONOLIS_B200_PRM_I_REFRESH_PERIOD = 41; /* mixed precision: FP64 residual refresh at the latest
                                                            n iterations after the previous one (0: no limit) */
static const int MONOLIS_B200_PRM_I_WIDE_SLICES_FP64 = 42; /* out: 32-row slices that keep 32-bit column ids (the
                                                              others store 16-bit differences to a base per slot) */
static const int MONOLIS_B200_PRM_I_WIDE_SLICES_FP32 = 43; /* out: same for the 64-row slices of the FP32 layout */
static const int MONOLIS_B200_PRM_I_WAIT_LIMIT     = 44; /* many right-hand sides: polls after which a grid-barrier
                                                            wait gives up and the solve returns MONOLIS_B200_TIMEOUT
                                                            (0: 4,194,304, seconds) */
static const int MONOLIS_B200_PRM_I_WAIT_DELAY_US  = 45; /* testing that bound: block 0 of the many-right-hand-side
                                                            kernel reaches its first barrier this many microseconds
                                                            late (0: off; at most 1,000,000) */
static const int MONOLIS_B200_PRM_I_UNIFORM_SLICES_FP64 = 46; /* out: 32-row slices whose block columns are the
                                                            per-slot base plus the lane (no column stream read) */
static const int MONOLIS_B200_PRM_I_UNIFORM_SLICES_FP32 = 47; /* out: same for the 64-row slices of the FP32 layout */

static const int MONOLIS_B200_PRM_R_REFRESH_DELTA  = 30; /* mixed precision: FP64 refresh when ||r|| has dropped
                                                            below delta * its largest value since the last one
                                                            (0: 0.1 for CG, 0.2 for BiCGSTAB) */
static const int MONOLIS_B200_PRM_R_TIME_H2D       = 31; /* out: seconds spent on host->device copies */
static const int MONOLIS_B200_PRM_R_TIME_D2H       = 32; /* out: seconds spent on device->host copies */
static const int MONOLIS_B200_PRM_R_TIME_LOOP      = 33; /* out: seconds in the device iteration loop */
static const int MONOLIS_B200_PRM_R_SPMV_BYTES_FP64 = 34; /* out: HBM bytes of one FP64 SpMV in the device layout:
                                                              values, column ids, row and slice offsets, x, y */
static const int MONOLIS_B200_PRM_R_SPMV_BYTES_FP32 = 35; /* out: same for the FP32 layout (0 before it is built) */
static const int MONOLIS_B200_PRM_R_TIME_KERNEL    = 40; /* out, timing mode: seconds per kernel slot k of an
                                                            iteration in Rarray[40 + k], k < 8 */

static const int MONOLIS_B200_PRECISION_FP64  = 0;
static const int MONOLIS_B200_PRECISION_MIXED = 1;

/* Precision of the Krylov loop. MIXED keeps values and vectors in FP32 inside
 * the loop, accumulates every dot product and the alpha/beta recurrences in
 * FP64, and refreshes an FP64 solution with an FP64 residual r = b - A x. */
int monolis_b200_set_precision(MONOLIS* mat, int precision);

/* Keep the device copy of the matrix between solves. Only calls of this
 * library that change the matrix invalidate it; a caller that writes
 * mat->mat.R.A directly must call monolis_b200_matrix_changed(). */
void monolis_b200_set_matrix_cache(MONOLIS* mat, bool enable);
void monolis_b200_matrix_changed(MONOLIS* mat);

/* ---- bulk host assembly ---- */

/* get_nonzero_pattern_by_simple_mesh_R with a flat element array
 * elem[e*n_base + a] (0-based); same resulting CSR as the int** form. */
int monolis_b200_get_nonzero_pattern_by_simple_mesh_flat_R(
  MONOLIS* mat, int n_node, int n_base, int n_dof, int n_elem, const int* elem);

/* Element-by-element monolis_add_matrix_to_sparse_matrix_R for n_elem
 * elements: element e adds scale[e] * val[e*val_stride + k] (row-major,
 * (n_base*ndof)^2 entries). scale may be NULL (1.0); val_stride 0 means all
 * elements share one matrix. Result is bit-identical to the calls made one
 * element at a time in order. */
int monolis_b200_add_elements_R(
  MONOLIS* mat, int n_elem, int n_base, const int* elem, const double* val,
  long long val_stride, const double* scale);

/* ---- device residency (device pointers; work is ordered on the library's
 * stream, monolis_b200_stream()) ---- */

/* Stream on which every device entry point of this library runs (cudaStream_t). */
void* monolis_b200_stream(void);

/* Upload the matrix, build the device layout and the DIAG factors (and the
 * FP32 copies when the precision parameter is MIXED). */
int monolis_b200_device_prepare(MONOLIS* mat);

/* Solve with b and x in device memory, using the prepared device matrix.
 * Synchronous; fills CUR_ITER, CUR_RESID, IERR and the timing slots. */
int monolis_b200_device_solve_R(MONOLIS* mat, const double* d_b, double* d_x);

/* The same with a MONOLIS_COM: when an NCCL communicator is attached to com
 * (monolis_b200_com_init_nccl), the row-partitioned multi-rank FP64 solve of
 * monolis_solve_R (halo updates through com's tables before each product,
 * dot products all-reduced; src/linalg/matvec.f90:144,
 * src/linalg/inner_product.f90:185) on device vectors of NP*NDOF entries,
 * ghost rows last; otherwise monolis_b200_device_solve_R. Every rank calls it
 * with the same parameters. Device-resident form of monolis_solve_R(mat, com,
 * b, x) (wrapper/solver/monolis_solver_c.h:17). */
int monolis_b200_device_solve_com_R(MONOLIS* mat, MONOLIS_COM* com, const double* d_b, double* d_x);

/* y = A x with device vectors (asynchronous on the library stream). */
int monolis_b200_device_matvec_R(MONOLIS* mat, const double* d_x, double* d_y);
int monolis_b200_device_matvec_R32(MONOLIS* mat, const float* d_x, float* d_y);

/* Layout facts of the prepared device matrix (block counts). */
int monolis_b200_device_info(MONOLIS* mat, long long* nz_blocks, long long* padded_blocks, int* n_slices);

/* ---- adjoint (transpose solve, sampled outer product, element gradients) ----
 * No counterpart in the reference library, which has no transpose product
 * or gradient. They let a caller differentiate a loss L(x) of the solution
 * of A(k) x = b with A = sum_e k_e K_e:
 *   1. monolis_solve_R                      x
 *   2. monolis_b200_solve_transpose_R       A^T lambda = dL/dx
 *   3. monolis_b200_element_gradient_R      dL/dk_e = -lambda_e^T K_e x_e
 * (or monolis_b200_sampled_outer_product_R for dL/dA over the pattern). */

/* A^T x = b with the struct's method, preconditioner, tolerance and
 * precision; same calling convention, parameters and outputs as
 * monolis_solve_R. A^T is built on the device from the struct's CSC arrays
 * (pattern + the CSC permutation of monolis_get_CSC_format) and cached with
 * the device matrix. One rank (N == NP). */
int monolis_b200_solve_transpose_R(MONOLIS* mat, MONOLIS_COM* com, double* b, double* x);
int monolis_b200_device_solve_transpose_R(MONOLIS* mat, const double* d_b, double* d_x);

/* y = A^T x (host vectors / device vectors). Row j of A^T sums the blocks of
 * column j of A in ascending row order. */
int monolis_b200_matvec_transpose_R(MONOLIS* mat, MONOLIS_COM* com, double* x, double* y);
int monolis_b200_device_matvec_transpose_R(MONOLIS* mat, const double* d_x, double* d_y);

/* G = scale * lambda x^T sampled on the sparsity pattern, in the layout of
 * mat->mat.R.A (NZ blocks of ndof^2 values, row-major in the block): entry
 * (r,c) of stored block (i,j) is scale * lambda[i*ndof+r] * x[j*ndof+c].
 * With scale = -1 and A lambda-adjoint as above, G = dL/dA. */
int monolis_b200_sampled_outer_product_R(MONOLIS* mat, const double* lambda, const double* x, double scale,
                                         double* G);
int monolis_b200_device_sampled_outer_product_R(MONOLIS* mat, const double* d_lambda, const double* d_x,
                                                double scale, double* d_G);

/* Per-element reduction of the sampled outer product:
 *   grad[e] = scale * sum_{a,b} lambda_a K_e(a,b) x_b
 * over the n_base*ndof local dofs of element e (elem[e*n_base + q], 0-based
 * nodes; local dof a = q*ndof + d, the order of the element matrices of
 * monolis_add_matrix_to_sparse_matrix_R). K_e is Ke + e*ke_stride (row-major,
 * (n_base*ndof)^2 values); ke_stride 0 shares one matrix. Rows of dofs with
 * fixed_dof[dof] != 0 are skipped (the Dirichlet rows that
 * monolis_set_Dirichlet_bc_R replaced do not depend on k); fixed_dof may be
 * NULL. With scale = -1 this is dL/dk_e. The host form checks the node ids;
 * the device form requires 0 <= elem < NP. */
int monolis_b200_element_gradient_R(MONOLIS* mat, int n_elem, int n_base, const int* elem, const double* Ke,
                                    long long ke_stride, const double* lambda, const double* x,
                                    const int* fixed_dof, double scale, double* grad);
int monolis_b200_device_element_gradient_R(MONOLIS* mat, int n_elem, int n_base, const int* d_elem,
                                           const double* d_Ke, long long ke_stride, const double* d_lambda,
                                           const double* d_x, const int* d_fixed_dof, double scale,
                                           double* d_grad);

/* ---- batched solver: many independent systems in one persistent kernel ----
 * No counterpart in the reference library (one system per monolis_solve_R).
 * Systems are added from assembled MONOLIS structs (or raw block CSR: 0-based
 * offsets and columns) and stacked on the device; each is solved by CG (+
 * DIAG) with its own convergence test, all of them in one persistent kernel
 * launched in thread-block clusters (one graph launch per solve). FP32 values
 * and vectors inside the loop, FP64 dot products and scalars; refine = 1 adds
 * FP64 reliable updates so that tol applies to the FP64 residual
 * ||b - A x|| / ||b|| (refine = 0: FP32 recursion, tol 1e-6 class). Cluster
 * size, CTA size and the system size below which systems are solved one per
 * CTA are picked by timing candidates on the batch (autotune = 1) or set. */
typedef struct monolis_b200_batch monolis_b200_batch;
int  monolis_b200_batch_create(monolis_b200_batch** batch);
void monolis_b200_batch_destroy(monolis_b200_batch* batch);
/* copies the matrix; systems are numbered in the order they are added; all
 * must have the same ndof */
int  monolis_b200_batch_add_system(monolis_b200_batch* batch, MONOLIS* mat);
int  monolis_b200_batch_add_csr(monolis_b200_batch* batch, int n, int ndof, const int* index, const int* item,
                                const double* val);
/* device layout, DIAG factors (precond MONOLIS_PREC_DIAG or NONE), tuning */
int  monolis_b200_batch_prepare(monolis_b200_batch* batch, int precond, int autotune);
int  monolis_b200_batch_set_config(monolis_b200_batch* batch, int cluster, int threads, long long split_rows);
int  monolis_b200_batch_get_config(monolis_b200_batch* batch, int* cluster, int* threads, long long* split_rows);
/* SpMV slots in flight per row of the batched kernel (1-3), picked by the autotuner */
int  monolis_b200_batch_get_unroll(monolis_b200_batch* batch, int* unroll);
/* re-times the candidates with `iters` iterations each and keeps the fastest;
 * on entry *n_candidates is the capacity of the output arrays, on return the
 * number of candidates timed */
int  monolis_b200_batch_autotune(monolis_b200_batch* batch, int iters, int* n_candidates, int* clusters,
                                 int* threads, long long* split_rows, double* seconds);
/* host b[i] / x[i] per system (x out); iter, resid (relative, FP64 true
 * residual), status per system (MONOLIS_B200_* codes) */
int  monolis_b200_batch_solve_R(monolis_b200_batch* batch, double** b, double** x, double tol, int max_iter,
                                int refine, int* iter, double* resid, int* status);
/* device-resident form: the stacked b and x (system i starts at offsets[i],
 * in dofs; rows between systems are padding and stay zero) */
int  monolis_b200_batch_info(monolis_b200_batch* batch, int* n_systems, long long* offsets);
int  monolis_b200_batch_device_vectors(monolis_b200_batch* batch, double** d_b, double** d_x);
int  monolis_b200_batch_device_solve_R(monolis_b200_batch* batch, double tol, int max_iter, int refine, int* iter,
                                       double* resid, int* status);
/* device seconds of the last batched solve (CUDA events around the graph launch) */
double monolis_b200_batch_last_seconds(monolis_b200_batch* batch);

/* ---- device assembly ----
 * No counterpart in the reference library (its assembly runs on the host).
 * These work on the library's device copy of the matrix (pattern from the
 * struct, values kept on the device) and give values bit-identical to the
 * host calls: monolis_add_matrix_to_sparse_matrix_R element by element in
 * order, then monolis_set_Dirichlet_bc_R condition by condition in order.
 * The host mat->mat.R.A is not written (read it back with
 * monolis_b200_device_get_values); solves and products of this library use
 * the device values until a host call changes the matrix.
 *   clear: device values = 0 (the pattern must exist);
 *   add_elements: d_elem[e*n_base + a] (0-based nodes, device), element e adds
 *     (d_scale ? d_scale[e] : 1) * d_val[e*val_stride + k] (row-major
 *     (n_base*ndof)^2, val_stride 0: one shared matrix), all device arrays;
 *   set_Dirichlet: n_bc conditions (host lists node_id, n_dof_bc, val, in
 *     call order), d_b the device right-hand side updated in place. */
int monolis_b200_device_clear_matrix(MONOLIS* mat);
int monolis_b200_device_add_elements_R(MONOLIS* mat, int n_elem, int n_base, const int* d_elem, const double* d_val,
                                       long long val_stride, const double* d_scale);
int monolis_b200_device_set_Dirichlet_bc_R(MONOLIS* mat, double* d_b, int n_bc, const int* node_id,
                                           const int* n_dof_bc, const double* val);
int monolis_b200_device_get_values(MONOLIS* mat, double* values);

/* The FP64 DIAG factors of the prepared device matrix (the precond parameter
 * DIAG when monolis_b200_device_prepare ran), written to alu (host, N*NDOF^2
 * doubles) in the reference's layout: block of row i at alu[i*NDOF^2], its
 * LU factors without pivoting, reciprocal pivots on the diagonal, a zero
 * pivot replaced by 1 (src/prec/diag/diag_33.f90:16-99, diag_nn.f90:16-86).
 * No counterpart in the reference's C API (its factors stay inside the
 * solver); for checking the device setup against a host one. */
int monolis_b200_device_get_diag(MONOLIS* mat, double* alu);

/* ---- many right-hand sides on one matrix ----
 * No counterpart in the reference library (one right-hand side per solve).
 * Solves A X_k = B_k for k < n_rhs with CG and the struct's preconditioner
 * (None or Diag), tolerance and max_iter; B_k and X_k are stored one after
 * another (B + k*N*ndof, like B(:,k)). Up to 32 right-hand sides share each
 * pass over the matrix (more are done 32 at a time), in one persistent
 * kernel; each converges on its own. PRECISION MIXED: FP32 loop with FP64
 * reliable updates (tol on the FP64 residual); FP64: the loop in double.
 * iter, resid (relative FP64 residual), status: per right-hand side. */
int monolis_b200_solve_multi_R(MONOLIS* mat, MONOLIS_COM* com, int n_rhs, double* B, double* X, int* iter,
                               double* resid, int* status);
int monolis_b200_device_solve_multi_R(MONOLIS* mat, int n_rhs, const double* d_B, double* d_X, int* iter,
                                      double* resid, int* status);

/* ---- multi-rank solve (one process per GPU, NCCL) ----
 * The reference runs one MPI rank per subdomain, each with the rows it owns
 * (mat->mat.N) followed by ghost rows (up to mat->mat.NP) and the halo tables
 * of MONOLIS_COM (recv/send neighbour ranks, offsets and 0-based local node
 * ids). Attaching an NCCL communicator to a MONOLIS_COM makes
 * monolis_solve_R(mat, com, b, x) solve the distributed system on the GPUs:
 * halo updates before every product, dot products summed over the ranks
 * (FP64 CG, GropCG, PipeCG or BiCGSTAB; b and x hold NP*ndof entries). Rank 0 creates the id, every rank
 * receives it (by any means, e.g. MPI or torch.distributed) and calls
 * monolis_b200_com_init_nccl with its current CUDA device set. NCCL is
 * loaded at run time (libnccl.so.2). No counterpart in the reference (which
 * uses MPI). */
int  monolis_b200_nccl_unique_id(void* id128);
int  monolis_b200_com_init_nccl(MONOLIS_COM* com, const void* id128, int rank, int size);
void monolis_b200_com_finalize_nccl(MONOLIS_COM* com);

/* ---- allocation-free inner product ----
 * No counterpart in the reference library.
 * *d_sum = sum_i d_x[i]*d_y[i] for device vectors of length n, enqueued on
 * `stream` (a cudaStream_t; NULL = legacy default stream), FP64 accumulation.
 * For callers that cannot call cudaMalloc when they need the result (an
 * application that reserved all device memory for its own pool, a loop that
 * must not take cudaMalloc's implicit synchronisation): this entry point
 * never allocates. Its reduction scratch is a fixed array in the library's
 * device image, held by every GPU that loads the library until the process
 * exits, which caps n at 16,777,216 elements; larger n is rejected with
 * MONOLIS_B200_BAD_INPUT and an error message. The first call on each device
 * looks up that array's address (make it before any stream capture); the
 * address is kept for the life of the process, so a cudaDeviceReset of a
 * device on which this entry point has been called makes later calls on it
 * invalid. All
 * calls share the one array: calls that overlap on the GPU (different
 * streams, or other host threads) race and must be serialised by the caller. */
int monolis_b200_inner_product_noalloc_R(long long n, const double* d_x, const double* d_y, double* d_sum,
                                         void* stream);

#ifdef __cplusplus
}
#endif

#endif
