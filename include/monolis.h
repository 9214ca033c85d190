/* monolis.h -- drop-in C interface of the monolis sparse iterative solver,
 * hot-path subset (real-valued block CSR, CG / BiCGSTAB, DIAG preconditioner).
 *
 * Struct layouts, constant values and function signatures are kept identical
 * to the reference C wrapper so that a user program compiled against the
 * reference headers links against libmonolis_b200.so unchanged. Each block
 * cites the reference declaration it replaces.
 *
 * Conventions (as in the reference C API):
 *  - node, dof and element indices passed by the caller are 0-based;
 *  - mat.CSR.index holds 0-based row offsets, mat.CSR.item holds 1-based
 *    column node ids (wrapper/matrix/monolis_spmat_nzpattern_util_c.c:36-38);
 *  - inside a stored block the values are row-major: entry (k,l) of block j
 *    is A[NDOF*NDOF*j + NDOF*k + l] (src/linalg/matvec.f90:783-826).
 */
#ifndef MONOLIS_H
#define MONOLIS_H

#ifdef __cplusplus
extern "C" {
#endif

#include <stdbool.h>
#include "monolis_utils.h"

/* ---- solver parameters: wrapper/define/monolis_def_solver_prm_c.h:12-146 ---- */

static const int MONOLIS_PRM_IARRAY_SIZE = 100;
static const int MONOLIS_PRM_RARRAY_SIZE = 100;

static const int MONOLIS_ITER_CG                  = 1;
static const int MONOLIS_ITER_GROPCG              = 2;
static const int MONOLIS_ITER_PIPECG              = 3;
static const int MONOLIS_ITER_PIPECR              = 4;
static const int MONOLIS_ITER_BICGSTAB            = 5;
static const int MONOLIS_ITER_PIPEBICGSTAB        = 6;
static const int MONOLIS_ITER_BICGSTAB_NOPREC     = 7;
static const int MONOLIS_ITER_PIPEBICGSTAB_NOPREC = 8;
static const int MONOLIS_ITER_BICGSTAB_N128       = 9;
static const int MONOLIS_ITER_SOR                 = 10;
static const int MONOLIS_ITER_BICGSAFE            = 11;
static const int MONOLIS_ITER_IDRS                = 12;
static const int MONOLIS_ITER_COCG                = 13;

static const int MONOLIS_PREC_NONE = 0;
static const int MONOLIS_PREC_DIAG = 1;
static const int MONOLIS_PREC_SOR  = 2;
static const int MONOLIS_PREC_LU   = 3;

static const int MONOLIS_PRM_I_METHOD                = 1;
static const int MONOLIS_PRM_I_PRECOND               = 2;
static const int MONOLIS_PRM_I_MAX_ITER              = 3;
static const int MONOLIS_PRM_I_CUR_ITER              = 4;
static const int MONOLIS_PRM_I_IERR                  = 5;
static const int MONOLIS_PRM_I_IS_INIT_X             = 10;
static const int MONOLIS_PRM_I_IS_SYM_MATRIX         = 11;
static const int MONOLIS_PRM_I_IS_DEBUG              = 12;
static const int MONOLIS_PRM_I_IS_MEASUREMENT        = 13;
static const int MONOLIS_PRM_I_IS_CHECK_DIAG         = 14;
static const int MONOLIS_PRM_I_IS_PREC_STORED        = 15;
static const int MONOLIS_PRM_I_IS_ERROR_ABORT        = 16;
static const int MONOLIS_PRM_I_SHOW_ITERLOG          = 20;
static const int MONOLIS_PRM_I_SHOW_TIME             = 21;
static const int MONOLIS_PRM_I_SHOW_SUMMARY          = 22;
static const int MONOLIS_PRM_I_SHOW_TIME_STATISTICS  = 23;
static const int MONOLIS_PRM_I_IDRS_DIM              = 24;
static const int MONOLIS_PRM_I_SPMV_FORMAT           = 25;

static const int MONOLIS_SPMV_ELL = 0;
static const int MONOLIS_SPMV_DIA = 1;

static const int MONOLIS_PRM_R_TOL        = 1;
static const int MONOLIS_PRM_R_CUR_RESID  = 2;
static const int MONOLIS_R_TIME_SOL       = 3;
static const int MONOLIS_R_TIME_PREP      = 4;
static const int MONOLIS_R_TIME_SPMV      = 5;
static const int MONOLIS_R_TIME_DOTP      = 6;
static const int MONOLIS_R_TIME_PREC      = 7;
static const int MONOLIS_R_TIME_COMM_DOTP = 8;
static const int MONOLIS_R_TIME_COMM_SPMV = 9;

/* wrapper/define/monolis_def_solver_prm_c.h:148-154 */
typedef struct {
  char   com_top_dir_name[1024];
  char   com_part_dir_name[1024];
  char   com_file_name[1024];
  int    Iarray[100];
  double Rarray[100];
} MONOLIS_PRM;

/* ---- matrix: wrapper/define/monolis_def_mat_c.h:8-57 ---- */

typedef struct {
  double* A;
  double* U;
  double* D;
  double* L;
  double* X;
  double* B;
} MONOLIS_MAT_VAL_R;

/* The complex twin is kept only for the struct layout; complex solves are
 * outside this library. */
typedef struct {
  void* A;
  void* U;
  void* D;
  void* L;
  void* X;
  void* B;
} MONOLIS_MAT_VAL_C;

typedef struct {
  int* indexU;
  int* indexL;
  int* itemU;
  int* itemL;
} MONOLIS_MAT_SEPARATED_CSR;

typedef struct {
  int* index;
  int* item;
} MONOLIS_MAT_CSR;

typedef struct {
  int* index;
  int* item;
  int* perm;
} MONOLIS_MAT_CSC;

typedef struct {
  int N;
  int NP;
  int NDOF;
  int* n_dof_list;
  int* n_dof_index;
  int* n_dof_index2;
  MONOLIS_MAT_VAL_R R;
  MONOLIS_MAT_VAL_C C;
  MONOLIS_MAT_SEPARATED_CSR SCSR;
  MONOLIS_MAT_CSR CSR;
  MONOLIS_MAT_CSC CSC;
} MONOLIS_MAT;

/* wrapper/define/monolis_def_struc_c.h:13-17 */
typedef struct {
  MONOLIS_PRM prm;
  MONOLIS_MAT mat;
  MONOLIS_MAT prec;
} MONOLIS;

/* ---- init / finalize: wrapper/define/monolis_def_struc_c.h:24-51,
 *      wrapper/define/monolis_def_mat_c.h:66-231,
 *      wrapper/define/monolis_def_solver_prm_c.h:161-171 ---- */
void monolis_global_initialize(void);
void monolis_global_finalize(void);
void monolis_initialize(MONOLIS* mat);
void monolis_finalize(MONOLIS* mat);
void monolis_prm_initialize(MONOLIS_PRM* prm);
void monolis_prm_finalize(MONOLIS_PRM* prm);
void monolis_mat_initialize(MONOLIS_MAT* mat);
void monolis_mat_finalize(MONOLIS_MAT* mat);
void monolis_get_vec_size(int N, int NP, int NDOF, int NZ,
                          int* n_dof_index, int* n_dof_index2,
                          int* N_size, int* NP_size, int* NZ_size);

/* ---- parameter setters / getters:
 *      wrapper/define/monolis_def_solver_prm_util_c.h:18-268 ---- */
void monolis_set_method(MONOLIS* mat, int param);
void monolis_set_precond(MONOLIS* mat, int param);
void monolis_set_spmv_format(MONOLIS* mat, int param);
void monolis_set_maxiter(MONOLIS* mat, int param);
void monolis_get_converge_iter(MONOLIS* mat, int* param);
void monolis_get_error_tag(MONOLIS* mat, int* param);
void monolis_set_init_x(MONOLIS* mat, bool param);
void monolis_set_sym_matrix(MONOLIS* mat, bool param);
void monolis_set_debug(MONOLIS* mat, bool param);
void monolis_set_performance_measurement(MONOLIS* mat, bool param);
void monolis_set_check_diag(MONOLIS* mat, bool param);
void monolis_set_prec_stored(MONOLIS* mat, bool param);
void monolis_set_error_abort(MONOLIS* mat, bool param);
void monolis_set_solver_IDRS_num_basis(MONOLIS* mat, int param);
void monolis_show_iterlog(MONOLIS* mat, bool param);
void monolis_show_timelog(MONOLIS* mat, bool param);
void monolis_show_summary(MONOLIS* mat, bool param);
void monolis_show_timelog_statistics(MONOLIS* mat, bool param);
void monolis_set_tolerance(MONOLIS* mat, double val);
void monolis_get_converge_residual(MONOLIS* mat, double* val);
void monolis_get_time_solver(MONOLIS* mat, double* val);
void monolis_get_time_preparing(MONOLIS* mat, double* val);
void monolis_get_time_spmv(MONOLIS* mat, double* val);
void monolis_get_time_inner_product(MONOLIS* mat, double* val);
void monolis_get_time_precondition(MONOLIS* mat, double* val);
void monolis_get_time_comm_inner_product(MONOLIS* mat, double* val);
void monolis_get_time_comm_spmv(MONOLIS* mat, double* val);

/* ---- nonzero pattern: wrapper/matrix/monolis_spmat_nzpattern_c.h:21,77;
 *      wrapper/matrix/monolis_spmat_nzpattern_util_c.h ---- */
void monolis_get_nonzero_pattern_by_simple_mesh_R(
  MONOLIS* mat, int n_node, int n_base, int n_dof, int n_elem, int** elem);
void monolis_get_nonzero_pattern_by_connectivity_R(
  MONOLIS* mat, int n_node, int n_dof, int n_elem, int* conn_index, int* conn_item);
void monolis_get_nonzero_pattern_by_nodal_graph_R(
  MONOLIS* mat, int n_node, int n_dof, int* index, int* item);
void monolis_get_CSC_format(int NC, int NR, int NZ, int* index, int* item,
                            int* indexR, int* itemR, int* permR);

/* ---- assembly: wrapper/matrix/monolis_spmat_handler_c.h:19-142 ---- */
void monolis_set_scalar_to_sparse_matrix_R(
  MONOLIS* mat, int i, int j, int submat_i, int submat_j, double val);
void monolis_add_scalar_to_sparse_matrix_R(
  MONOLIS* mat, int i, int j, int submat_i, int submat_j, double val);
void monolis_get_scalar_from_sparse_matrix_R(
  MONOLIS* mat, int i, int j, int submat_i, int submat_j, double* val, bool* is_find);
void monolis_add_matrix_to_sparse_matrix_R(
  MONOLIS* mat, int n_base, int* connectivity, double** val);
void monolis_add_matrix_to_sparse_matrix_offdiag_R(
  MONOLIS* mat, int n_base1, int n_base2, int* connectivity1, int* connectivity2, double** val);
void monolis_set_matrix_BCSR_R(
  MONOLIS* mat, int n, int np, int n_dof, int nz, double* A, int* index, int* item);
void monolis_set_Dirichlet_bc_R(
  MONOLIS* mat, double* b, int node_id, int n_dof_bc, double val);

/* ---- linear algebra: wrapper/linalg/monolis_matvec_c.h:19,
 *      wrapper/linalg/monolis_inner_product_c.h ---- */
void monolis_matvec_product_R(MONOLIS* mat, MONOLIS_COM* com, double* x, double* y);
void monolis_inner_product_R(MONOLIS* mat, MONOLIS_COM* com, int n_dof,
                             double* x, double* y, double* sum);

/* ---- solve: wrapper/solver/monolis_solver_c.h:17 ---- */
void monolis_solve_R(MONOLIS* mat, MONOLIS_COM* com, double* b, double* x);

#ifdef __cplusplus
}
#endif

#endif
