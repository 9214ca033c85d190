/* abi_layout.c -- prints the layout of the monolis C API's structs and the
 * values of its constants, one "name value" line each.
 *
 * Built two ways: against this library's include/monolis.h (the test), and,
 * by tests/golden/make_abi_layout.py, against the reference's own headers
 * (wrapper/define/monolis_def_struc_c.h and what it includes; -DABI_REFERENCE),
 * whose output is the committed fixture tests/golden/abi_layout_reference.txt.
 * A C program compiled against the reference headers can relink against this
 * library only if the two outputs are identical. MONOLIS_COM is defined by
 * the monolis_utils submodule, which the reference tree does not contain, so
 * it is not listed. */
#include <stddef.h>
#include <stdio.h>

#ifdef ABI_REFERENCE
#include "monolis_def_struc_c.h"
#else
#include "monolis.h"
#endif

#define SZ(T) printf("sizeof(" #T ") %zu\n", sizeof(T))
#define OFF(T, f) printf("offsetof(" #T "," #f ") %zu\n", offsetof(T, f))
#define CST(c) printf(#c " %d\n", (int)(c))

int main(void) {
  SZ(MONOLIS);
  OFF(MONOLIS, prm);
  OFF(MONOLIS, mat);
  OFF(MONOLIS, prec);
  SZ(MONOLIS_PRM);
  OFF(MONOLIS_PRM, com_top_dir_name);
  OFF(MONOLIS_PRM, com_part_dir_name);
  OFF(MONOLIS_PRM, com_file_name);
  OFF(MONOLIS_PRM, Iarray);
  OFF(MONOLIS_PRM, Rarray);
  SZ(MONOLIS_MAT);
  OFF(MONOLIS_MAT, N);
  OFF(MONOLIS_MAT, NP);
  OFF(MONOLIS_MAT, NDOF);
  OFF(MONOLIS_MAT, n_dof_list);
  OFF(MONOLIS_MAT, n_dof_index);
  OFF(MONOLIS_MAT, n_dof_index2);
  OFF(MONOLIS_MAT, R);
  OFF(MONOLIS_MAT, C);
  OFF(MONOLIS_MAT, SCSR);
  OFF(MONOLIS_MAT, CSR);
  OFF(MONOLIS_MAT, CSC);
  SZ(MONOLIS_MAT_VAL_R);
  OFF(MONOLIS_MAT_VAL_R, A);
  OFF(MONOLIS_MAT_VAL_R, U);
  OFF(MONOLIS_MAT_VAL_R, D);
  OFF(MONOLIS_MAT_VAL_R, L);
  OFF(MONOLIS_MAT_VAL_R, X);
  OFF(MONOLIS_MAT_VAL_R, B);
  SZ(MONOLIS_MAT_VAL_C);
  SZ(MONOLIS_MAT_SEPARATED_CSR);
  OFF(MONOLIS_MAT_SEPARATED_CSR, indexU);
  OFF(MONOLIS_MAT_SEPARATED_CSR, indexL);
  OFF(MONOLIS_MAT_SEPARATED_CSR, itemU);
  OFF(MONOLIS_MAT_SEPARATED_CSR, itemL);
  SZ(MONOLIS_MAT_CSR);
  OFF(MONOLIS_MAT_CSR, index);
  OFF(MONOLIS_MAT_CSR, item);
  SZ(MONOLIS_MAT_CSC);
  OFF(MONOLIS_MAT_CSC, index);
  OFF(MONOLIS_MAT_CSC, item);
  OFF(MONOLIS_MAT_CSC, perm);
  CST(MONOLIS_PRM_IARRAY_SIZE);
  CST(MONOLIS_PRM_RARRAY_SIZE);
  CST(MONOLIS_ITER_CG);
  CST(MONOLIS_ITER_GROPCG);
  CST(MONOLIS_ITER_PIPECG);
  CST(MONOLIS_ITER_PIPECR);
  CST(MONOLIS_ITER_BICGSTAB);
  CST(MONOLIS_ITER_PIPEBICGSTAB);
  CST(MONOLIS_ITER_BICGSTAB_NOPREC);
  CST(MONOLIS_ITER_PIPEBICGSTAB_NOPREC);
  CST(MONOLIS_ITER_BICGSTAB_N128);
  CST(MONOLIS_ITER_SOR);
  CST(MONOLIS_ITER_BICGSAFE);
  CST(MONOLIS_ITER_IDRS);
  CST(MONOLIS_ITER_COCG);
  CST(MONOLIS_PREC_NONE);
  CST(MONOLIS_PREC_DIAG);
  CST(MONOLIS_PREC_SOR);
  CST(MONOLIS_PREC_LU);
  CST(MONOLIS_PRM_I_METHOD);
  CST(MONOLIS_PRM_I_PRECOND);
  CST(MONOLIS_PRM_I_MAX_ITER);
  CST(MONOLIS_PRM_I_CUR_ITER);
  CST(MONOLIS_PRM_I_IERR);
  CST(MONOLIS_PRM_I_IS_INIT_X);
  CST(MONOLIS_PRM_I_IS_SYM_MATRIX);
  CST(MONOLIS_PRM_I_IS_DEBUG);
  CST(MONOLIS_PRM_I_IS_MEASUREMENT);
  CST(MONOLIS_PRM_I_IS_CHECK_DIAG);
  CST(MONOLIS_PRM_I_IS_PREC_STORED);
  CST(MONOLIS_PRM_I_IS_ERROR_ABORT);
  CST(MONOLIS_PRM_I_SHOW_ITERLOG);
  CST(MONOLIS_PRM_I_SHOW_TIME);
  CST(MONOLIS_PRM_I_SHOW_SUMMARY);
  CST(MONOLIS_PRM_I_SHOW_TIME_STATISTICS);
  CST(MONOLIS_PRM_I_IDRS_DIM);
  CST(MONOLIS_PRM_I_SPMV_FORMAT);
  CST(MONOLIS_SPMV_ELL);
  CST(MONOLIS_SPMV_DIA);
  CST(MONOLIS_PRM_R_TOL);
  CST(MONOLIS_PRM_R_CUR_RESID);
  CST(MONOLIS_R_TIME_SOL);
  CST(MONOLIS_R_TIME_PREP);
  CST(MONOLIS_R_TIME_SPMV);
  CST(MONOLIS_R_TIME_DOTP);
  CST(MONOLIS_R_TIME_PREC);
  CST(MONOLIS_R_TIME_COMM_DOTP);
  CST(MONOLIS_R_TIME_COMM_SPMV);
  return 0;
}
