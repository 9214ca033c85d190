/* solver_c.c -- a C program written against the monolis C API
 * (include/monolis.h), linked against either library (the product or the
 * CPU oracle) by tests/test_c_boundary.py.
 *
 * For ndof 1, 2 and 3: a 10-node chain whose blocks come from a fixed
 * linear congruential generator (diagonal blocks strongly dominant and
 * symmetric, each off-diagonal block the transpose of its mirror), b = A*1
 * by monolis_matvec_product_R, then monolis_solve_R with CG + DIAG and
 * BiCGSTAB + DIAG at tolerance 1e-10 must give x = 1 -- the check of the
 * reference's own C solver test (wrapper_test/solver/monolis_solver_c_test.c)
 * and its Fortran chain tests (src_test/iterative/CG_test.f90). The program
 * also reads the CSR arrays and counters the library wrote into the structs
 * (N, NDOF, CSR.index, CSR.item, Iarray, Rarray), so it fails if the struct
 * layout it was compiled with is not the library's. Prints one line per
 * case and exits non-zero on any failure. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "monolis.h"

static unsigned long long g_state = 0x9e3779b97f4a7c15ULL;

static double next_uniform(void) {
  g_state = g_state * 6364136223846793005ULL + 1442695040888963407ULL;
  return (double)(g_state >> 11) / 9007199254740992.0;
}

static int run_case(int n_dof, int method) {
  enum { n_node = 10, n_elem = 9 };
  int conn[n_elem][2];
  int* elem[n_elem];
  int fails = 0;
  for (int e = 0; e < n_elem; e++) {
    conn[e][0] = e;
    conn[e][1] = e + 1;
    elem[e] = conn[e];
  }
  MONOLIS mat;
  MONOLIS_COM com;
  monolis_initialize(&mat);
  monolis_com_initialize_by_self(&com);
  monolis_get_nonzero_pattern_by_simple_mesh_R(&mat, n_node, 2, n_dof, n_elem, elem);
  for (int i = 0; i < n_node; i++)
    for (int a = 0; a < n_dof; a++)
      for (int c = a; c < n_dof; c++) {
        const double v = a == c ? 6.0 + next_uniform() : 0.5 * next_uniform();
        monolis_add_scalar_to_sparse_matrix_R(&mat, i, i, a, c, v);
        if (c != a) monolis_add_scalar_to_sparse_matrix_R(&mat, i, i, c, a, v);
      }
  for (int e = 0; e < n_elem; e++)
    for (int a = 0; a < n_dof; a++)
      for (int c = 0; c < n_dof; c++) {
        const double v = next_uniform() - 0.5;
        monolis_add_scalar_to_sparse_matrix_R(&mat, conn[e][0], conn[e][1], a, c, v);
        monolis_add_scalar_to_sparse_matrix_R(&mat, conn[e][1], conn[e][0], c, a, v);
      }
  /* the pattern the library wrote into the struct: self + neighbours per
   * row, 0-based offsets, 1-based ascending items */
  if (mat.mat.N != n_node || mat.mat.NP != n_node || mat.mat.NDOF != n_dof) fails++;
  if (mat.mat.CSR.index[0] != 0 || mat.mat.CSR.index[n_node] != 3 * n_node - 2) fails++;
  if (mat.mat.CSR.item[0] != 1 || mat.mat.CSR.item[1] != 2 || mat.mat.CSR.item[2] != 1) fails++;
  double ones[30], b[30], x[30];
  const int n = n_node * n_dof;
  for (int i = 0; i < n; i++) {
    ones[i] = 1.0;
    x[i] = 0.0;
  }
  monolis_matvec_product_R(&mat, &com, ones, b);
  monolis_set_method(&mat, method);
  monolis_set_precond(&mat, MONOLIS_PREC_DIAG);
  monolis_set_tolerance(&mat, 1.0e-10);
  monolis_set_maxiter(&mat, 1000);
  monolis_show_summary(&mat, false);
  monolis_show_timelog(&mat, false);
  monolis_show_iterlog(&mat, false);
  monolis_solve_R(&mat, &com, b, x);
  int iter = -1;
  double resid = -1.0;
  monolis_get_converge_iter(&mat, &iter);
  monolis_get_converge_residual(&mat, &resid);
  double err = 0.0;
  for (int i = 0; i < n; i++) err = fmax(err, fabs(x[i] - 1.0));
  if (!(err < 1.0e-8)) fails++;
  if (iter < 1 || iter != mat.prm.Iarray[MONOLIS_PRM_I_CUR_ITER]) fails++;
  if (!(resid < 1.0e-10) || resid != mat.prm.Rarray[MONOLIS_PRM_R_CUR_RESID]) fails++;
  if (mat.prm.Iarray[MONOLIS_PRM_I_METHOD] != method || mat.prm.Rarray[MONOLIS_PRM_R_TOL] != 1.0e-10) fails++;
  printf("ndof %d %s: iter %d resid %.3e max|x-1| %.3e %s\n", n_dof, method == MONOLIS_ITER_CG ? "CG" : "BiCGSTAB",
         iter, resid, err, fails ? "FAIL" : "ok");
  monolis_finalize(&mat);
  monolis_com_finalize(&com);
  return fails;
}

int main(void) {
  int fails = 0;
  monolis_global_initialize();
  for (int n_dof = 1; n_dof <= 3; n_dof++) {
    fails += run_case(n_dof, MONOLIS_ITER_CG);
    fails += run_case(n_dof, MONOLIS_ITER_BICGSTAB);
  }
  monolis_global_finalize();
  printf("%s\n", fails ? "FAILED" : "all ok");
  return fails ? 1 : 0;
}
