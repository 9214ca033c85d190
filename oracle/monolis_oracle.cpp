// monolis_oracle.cpp -- CPU ORACLE (test infrastructure, not the product).
//
// A plain C++ restatement of the reference monolis hot path: nonzero pattern,
// assembly, Dirichlet condition, block-CSR SpMV, inner product, AXPBY, DIAG
// (block-Jacobi) preconditioner, convergence check, CG and BiCGSTAB, in the
// reference's own operation order. It exports the same C API as the product
// library (include/monolis.h) so one test driver can run against either.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline and
// reference arm load this library, and only as the checker / baseline. The
// product (monolis_b200/) never links or calls it.
//
// Parity pinning: the reference is Fortran and cannot be compiled in this
// image (no Fortran compiler, empty monolis_utils / gedatsu submodules). The
// restatement is pinned against the reference's own known-answer tests,
// restated in tests/test_oracle_kat.py (src_test/linalg/matvec_test.f90,
// src_test/linalg/mat_converge_test.f90, src_test/iterative/CG_test.f90,
// src_test/iterative/BiCGSTAB_test.f90, wrapper_test/solver/
// monolis_solver_c_test.c, src_test/input.f/mtx.dat + main.f90). Those pin
// semantics (x = 1, residual below tolerance, residual definition); iteration
// counts are pinned only by this restatement itself.
//
// Floating point: built with -O2 -ffp-contract=off so that a*b + c is two
// roundings, as gfortran -O2 emits for the reference on x86-64 (no FMA in the
// baseline ISA). Reductions run serially left to right when one thread is
// used (the reference default build has no -fopenmp, Makefile:5); with more
// threads the OpenMP reductions mirror the reference's !$omp directives.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "monolis.h"

namespace {

// iter_RR of src/iterative/CG.f90:40 and BiCGSTAB.f90:41 (200) and of
// src/iterative/PipeCG.f90:43 (50); settable through oracle_set_iter_rr() so
// tests can cross several replacements.
int g_iter_rr = 200;
int g_iter_rr_pipe = 50;

double now_sec() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Optional wall-clock log of a solve (CPU baseline timing): entry 0 at the
// start of monolis_solve_R, entry i at the end of iteration i (its
// convergence check). Set by oracle_set_iter_clock; the arithmetic is not
// touched.
double* g_iter_clock = nullptr;
int g_iter_clock_cap = 0;

template <class T>
T* alloc_zero(long long n) {
  if (n <= 0) n = 1;
  return static_cast<T*>(calloc(static_cast<size_t>(n), sizeof(T)));
}

template <class T>
void free_ptr(T** p) {
  if (*p) free(*p);
  *p = nullptr;
}

[[noreturn]] void error_stop(const char* msg) {
  fprintf(stderr, "** monolis error: %s\n", msg);
  fflush(stderr);
  exit(1);
}

// ---------------------------------------------------------------------------
// Nonzero pattern.
// gedatsu's mesh -> nodal graph (absent submodule) restated from its contract:
// node j is a neighbour of node i iff they share an element, i != j.
// ---------------------------------------------------------------------------
void nodal_graph_from_mesh(int n_node, int n_base, int n_elem, const int* elem,
                           std::vector<int>& index, std::vector<int>& item) {
  std::vector<std::vector<int>> nb(n_node);
  for (int e = 0; e < n_elem; ++e) {
    for (int a = 0; a < n_base; ++a) {
      int i = elem[(long long)e * n_base + a];
      for (int b = 0; b < n_base; ++b) {
        int j = elem[(long long)e * n_base + b];
        if (i != j) nb[i].push_back(j);
      }
    }
  }
  index.assign(n_node + 1, 0);
  item.clear();
  for (int i = 0; i < n_node; ++i) {
    std::sort(nb[i].begin(), nb[i].end());
    nb[i].erase(std::unique(nb[i].begin(), nb[i].end()), nb[i].end());
    index[i + 1] = index[i] + (int)nb[i].size();
    item.insert(item.end(), nb[i].begin(), nb[i].end());
  }
}

// wrapper/matrix/monolis_spmat_nzpattern_util_c.c:9-65
void pattern_by_nodal_graph_main(MONOLIS_MAT* mat, int n_node, int n_dof,
                                 const int* index, const int* item) {
  mat->N = n_node;
  mat->NP = n_node;
  mat->NDOF = n_dof;
  mat->CSR.index = alloc_zero<int>(n_node + 1);
  for (int i = 1; i < n_node + 1; i++) mat->CSR.index[i] = index[i] + i;
  int nz = mat->CSR.index[n_node];
  mat->CSR.item = alloc_zero<int>(nz);
  for (int i = 0; i < n_node; i++) {
    int jS = mat->CSR.index[i];
    int jE = mat->CSR.index[i + 1];
    mat->CSR.item[jS] = i + 1;
    for (int j = jS + 1; j < jE; j++) mat->CSR.item[j] = item[j - i - 1] + 1;
    std::sort(mat->CSR.item + jS, mat->CSR.item + jE);
  }
  mat->CSC.index = alloc_zero<int>(n_node + 1);
  mat->CSC.item = alloc_zero<int>(nz);
  mat->CSC.perm = alloc_zero<int>(nz);
  monolis_get_CSC_format(n_node, n_node, nz, mat->CSR.index, mat->CSR.item,
                         mat->CSC.index, mat->CSC.item, mat->CSC.perm);
}

// wrapper/matrix/monolis_spmat_nzpattern_util_c.c:139-168
void set_n_dof_index(MONOLIS_MAT* mat, const int* n_dof_list) {
  int np = mat->NP;
  int nz = mat->CSR.index[np];
  mat->n_dof_list = alloc_zero<int>(np);
  mat->n_dof_index = alloc_zero<int>(np + 1);
  mat->n_dof_index2 = alloc_zero<int>(nz + 1);
  for (int i = 0; i < np; ++i) mat->n_dof_list[i] = n_dof_list[i];
  for (int i = 0; i < np; ++i) mat->n_dof_index[i + 1] = mat->n_dof_index[i] + n_dof_list[i];
  for (int i = 0; i < np; ++i) {
    for (int j = mat->CSR.index[i]; j < mat->CSR.index[i + 1]; ++j) {
      int in = mat->CSR.item[j] - 1;
      mat->n_dof_index2[j + 1] = mat->n_dof_index2[j] + n_dof_list[i] * n_dof_list[in];
    }
  }
}

// wrapper/matrix/monolis_spmat_nzpattern_util_c.c:67-83
void alloc_mat_val(MONOLIS_MAT* mat) {
  int n = mat->N, nd = mat->NDOF;
  int nz = mat->CSR.index[n];
  mat->R.A = alloc_zero<double>((long long)nd * nd * nz);
  mat->R.X = alloc_zero<double>((long long)nd * n);
  mat->R.B = alloc_zero<double>((long long)nd * n);
}

void finish_pattern(MONOLIS* m, int n_node, int n_dof, const int* index, const int* item) {
  pattern_by_nodal_graph_main(&m->mat, n_node, n_dof, index, item);
  std::vector<int> list(n_node, n_dof);
  set_n_dof_index(&m->mat, list.data());
  alloc_mat_val(&m->mat);
}

// monolis_bsearch_I over item(jS:jE) (1-based values), 0-based positions.
int bsearch_item(const int* item, int jS, int jE, int key) {
  int lo = jS, hi = jE - 1;
  while (lo <= hi) {
    int mid = (lo + hi) / 2;
    if (item[mid] == key) return mid;
    if (item[mid] < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// src/matrix/spmat_handler_util.f90:306-348 (0-based i, j, sub indices).
double* scalar_slot(MONOLIS* m, int i, int j, int sub_i, int sub_j) {
  MONOLIS_MAT* a = &m->mat;
  int nd_i = a->n_dof_index[i + 1] - a->n_dof_index[i];
  int nd_j = a->n_dof_index[j + 1] - a->n_dof_index[j];
  if (sub_i >= nd_i || sub_j >= nd_j) error_stop("submatrix access out of range");
  int p = bsearch_item(a->CSR.item, a->CSR.index[i], a->CSR.index[i + 1], j + 1);
  if (p < 0) return nullptr;
  return &a->R.A[(long long)a->n_dof_index2[p] + (long long)nd_j * sub_i + sub_j];
}

// src/matrix/spmat_handler_util.f90:398-497: sort the element's node lists,
// reorder the dense element matrix, then merge-search each sorted row.
void add_matrix_main(MONOLIS* m, int n1, int n2, const int* e1, const int* e2,
                     const double* val /* n_rows x n_cols row-major */) {
  MONOLIS_MAT* a = &m->mat;
  const int* ndi = a->n_dof_index;
  std::vector<int> p1(n1), p2(n2);
  for (int i = 0; i < n1; ++i) p1[i] = i;
  for (int i = 0; i < n2; ++i) p2[i] = i;
  std::stable_sort(p1.begin(), p1.end(), [&](int x, int y) { return e1[x] < e1[y]; });
  std::stable_sort(p2.begin(), p2.end(), [&](int x, int y) { return e2[x] < e2[y]; });
  std::vector<int> idx1(n1 + 1, 0), idx2(n2 + 1, 0);
  for (int i = 0; i < n1; ++i) idx1[i + 1] = idx1[i] + ndi[e1[i] + 1] - ndi[e1[i]];
  for (int i = 0; i < n2; ++i) idx2[i + 1] = idx2[i] + ndi[e2[i] + 1] - ndi[e2[i]];
  int ncol = idx2[n2];
  for (int s1 = 0; s1 < n1; ++s1) {
    int r = e1[p1[s1]];
    int jS = a->CSR.index[r], jE = a->CSR.index[r + 1];
    int nr = ndi[r + 1] - ndi[r];
    for (int s2 = 0; s2 < n2; ++s2) {
      int c = e2[p2[s2]];
      int found = -1;
      for (int j = jS; j < jE; ++j) {
        if (a->CSR.item[j] == c + 1) { found = j; break; }
      }
      if (found < 0) error_stop("matrix assemble: entry not in the nonzero pattern");
      int kn = ndi[c + 1] - ndi[c];
      for (int k1 = 0; k1 < nr; ++k1)
        for (int k2 = 0; k2 < kn; ++k2) {
          long long im = (long long)a->n_dof_index2[found] + (long long)kn * k1 + k2;
          a->R.A[im] = a->R.A[im] + val[(long long)(idx1[p1[s1]] + k1) * ncol + idx2[p2[s2]] + k2];
        }
      jS = found;
    }
  }
}

// ---------------------------------------------------------------------------
// Linear algebra (src/linalg/*.f90)
// ---------------------------------------------------------------------------
void matvec(const MONOLIS_MAT* a, int N, const double* X, double* Y) {
  const int nd = a->NDOF, nd2 = nd * nd;
  const int* index = a->CSR.index;
  const int* item = a->CSR.item;
  const double* A = a->R.A;
  if (nd == 1) {  // src/linalg/matvec.f90:707-741
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
      double y = 0.0;
      for (int j = index[i]; j < index[i + 1]; j++) y = y + A[j] * X[item[j] - 1];
      Y[i] = y;
    }
  } else if (nd == 3) {  // src/linalg/matvec.f90:783-826
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
      double y1 = 0.0, y2 = 0.0, y3 = 0.0;
      for (int j = index[i]; j < index[i + 1]; j++) {
        long long in = item[j] - 1;
        double x1 = X[3 * in], x2 = X[3 * in + 1], x3 = X[3 * in + 2];
        const double* b = A + 9LL * j;
        y1 = y1 + b[0] * x1 + b[1] * x2 + b[2] * x3;
        y2 = y2 + b[3] * x1 + b[4] * x2 + b[5] * x3;
        y3 = y3 + b[6] * x1 + b[7] * x2 + b[8] * x3;
      }
      Y[3LL * i] = y1; Y[3LL * i + 1] = y2; Y[3LL * i + 2] = y3;
    }
  } else {  // src/linalg/matvec.f90:355-402
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
      double yt[16] = {0}, xt[16];
      for (int j = index[i]; j < index[i + 1]; j++) {
        long long in = item[j] - 1;
        for (int k = 0; k < nd; k++) xt[k] = X[nd * in + k];
        for (int k = 0; k < nd; k++)
          for (int l = 0; l < nd; l++) yt[k] = yt[k] + A[(long long)nd2 * j + nd * k + l] * xt[l];
      }
      for (int k = 0; k < nd; k++) Y[(long long)nd * i + k] = yt[k];
    }
  }
}

// Error-free addition (Knuth's TwoSum): s + e == a + b exactly.
inline void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
inline void dd_add(double& hi, double& lo, double p) {
  double s, e;
  two_sum(hi, p, s, e);
  e = e + lo;
  hi = s + e;
  lo = e - (hi - s);
}
inline void dd_merge(double& hi, double& lo, double h2, double l2) {
  double s, e;
  two_sum(hi, h2, s, e);
  e = e + (lo + l2);
  hi = s + e;
  lo = e - (hi - s);
}

// Sum of the rounded products X(i)*Y(i) in double-double, the arithmetic of
// the reference's pseudo-quadruple inner product
// (src/linalg/inner_product.f90:219-258: each product rounded to double,
// added to a two-double sum, the sum converted back to double). Each thread
// sums a contiguous chunk, every addition a double-double addition
// renormalised after each step (Dekker 1971), and the chunks are combined in
// thread order the same way; the result is within a small multiple of
// n eps^2 sum|x_i y_i| of the exact sum of the rounded products, so it does
// not depend on the thread count (nor on any other grouping) except in the
// rare case of an exact sum that close to a rounding boundary. The
// monolis_utils routine the reference calls for the two-double addition
// (monolis_add_R_N128) is not in the reference tree; this is the standard
// TwoSum-based addition.
double dot_n128(long long m, const double* X, const double* Y) {
#ifdef _OPENMP
  const int nt = omp_get_max_threads();
#else
  const int nt = 1;
#endif
  std::vector<double> H(nt, 0.0), L(nt, 0.0);
  int used = 1;
#pragma omp parallel
  {
#ifdef _OPENMP
    const int t = omp_get_thread_num(), T = omp_get_num_threads();
#else
    const int t = 0, T = 1;
#endif
    if (t == 0) used = T;
    const long long i0 = m * t / T, i1 = m * (t + 1) / T;
    double hi = 0.0, lo = 0.0;
    for (long long i = i0; i < i1; i++) dd_add(hi, lo, X[i] * Y[i]);
    H[t] = hi;
    L[t] = lo;
  }
  double hi = 0.0, lo = 0.0;
  for (int t = 0; t < used; t++) dd_merge(hi, lo, H[t], L[t]);
  return hi + lo;
}

// Dot products of the solvers and of monolis_inner_product_R: 0 = the
// reference's inner product (below); 1 = every dot product in double-double
// (dot_n128), the arithmetic the product library's FP64 kernels use.
int g_dot_mode = 0;

// src/linalg/inner_product.f90:148-190 (allreduce is the identity on one rank)
double dot(long long m, const double* X, const double* Y) {
  if (g_dot_mode == 1) return dot_n128(m, X, Y);
  double sum = 0.0;
#pragma omp parallel for reduction(+ : sum) schedule(static)
  for (long long i = 0; i < m; i++) sum = sum + X[i] * Y[i];
  return sum;
}

// src/linalg/inner_product.f90:262-331: products sorted by |x_i y_i|, summed.
double sorted_dot(long long m, const double* X, const double* Y) {
  std::vector<double> xy(m);
  for (long long i = 0; i < m; i++) xy[i] = X[i] * Y[i];
  std::stable_sort(xy.begin(), xy.end(), [](double a, double b) { return std::fabs(a) < std::fabs(b); });
  double s = 0.0;
  for (long long i = 0; i < m; i++) s = s + xy[i];
  return s;
}

// src/linalg/vec_util.f90:132-162  Z = alpha*X + beta*Y
void axpby(long long m, double alpha, const double* X, double beta, const double* Y, double* Z) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < m; i++) Z[i] = alpha * X[i] + beta * Y[i];
}

void vcopy(long long m, const double* X, double* Y) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < m; i++) Y[i] = X[i];
}

// ---------------------------------------------------------------------------
// DIAG preconditioner: src/prec/diag/diag_33.f90:16-139, diag_nn.f90:16-231
// ---------------------------------------------------------------------------
void diag_setup(const MONOLIS_MAT* a, std::vector<double>& ALU) {
  const int N = a->N, nd = a->NDOF, nd2 = nd * nd;
  ALU.assign((size_t)nd2 * N, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    double LU[256], T[16];
    bool found = false;
    for (int j = a->CSR.index[i]; j < a->CSR.index[i + 1]; j++) {
      if (a->CSR.item[j] - 1 == i) {
        for (int k = 0; k < nd2; k++) LU[k] = a->R.A[(long long)nd2 * j + k];
        found = true;
      }
    }
    if (!found) continue;  // row without a diagonal block keeps zeros
    for (int k = 0; k < nd; k++) {
      if (LU[k * nd + k] == 0.0) LU[k * nd + k] = 1.0;
      LU[k * nd + k] = 1.0 / LU[k * nd + k];
      for (int l = k + 1; l < nd; l++) {
        LU[l * nd + k] = LU[l * nd + k] * LU[k * nd + k];
        for (int j = k + 1; j < nd; j++) T[j] = LU[l * nd + j] - LU[l * nd + k] * LU[k * nd + j];
        for (int j = k + 1; j < nd; j++) LU[l * nd + j] = T[j];
      }
    }
    for (int k = 0; k < nd2; k++) ALU[(size_t)nd2 * i + k] = LU[k];
  }
}

void diag_apply(const MONOLIS_MAT* a, const std::vector<double>& ALU, const double* X, double* Y) {
  const int N = a->N, nd = a->NDOF, nd2 = nd * nd;
  if (nd == 3) {  // diag_33.f90:121-135
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
      const double* L = ALU.data() + 9LL * i;
      double x1 = X[3LL * i], x2 = X[3LL * i + 1], x3 = X[3LL * i + 2];
      x2 = x2 - L[3] * x1;
      x3 = x3 - L[6] * x1 - L[7] * x2;
      x3 = L[8] * x3;
      x2 = L[4] * (x2 - L[5] * x3);
      x1 = L[0] * (x1 - L[2] * x3 - L[1] * x2);
      Y[3LL * i] = x1; Y[3LL * i + 1] = x2; Y[3LL * i + 2] = x3;
    }
  } else {  // diag_nn.f90:185-231
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
      const double* L = ALU.data() + (size_t)nd2 * i;
      double T[16];
      for (int j = 0; j < nd; j++) T[j] = X[(long long)nd * i + j];
      for (int j = 1; j < nd; j++)
        for (int k = 0; k < j; k++) T[j] = T[j] - L[nd * j + k] * T[k];
      for (int j = nd - 1; j >= 0; j--) {
        for (int k = nd - 1; k > j; k--) T[j] = T[j] - L[nd * j + k] * T[k];
        T[j] = L[(nd + 1) * j] * T[j];
      }
      for (int k = 0; k < nd; k++) Y[(long long)nd * i + k] = T[k];
    }
  }
}

struct Prec {
  int kind = 0;
  std::vector<double> ALU;
};

// src/prec/precond.f90:147-231
void precond_apply(const MONOLIS_MAT* a, const Prec& pc, long long nndof, const double* X, double* Y) {
  if (pc.kind == 1) diag_apply(a, pc.ALU, X, Y);
  else vcopy(nndof, X, Y);
}

struct Timers {
  double spmv = 0, dotp = 0, prec = 0;
};

void residual(const MONOLIS_MAT* a, const double* X, const double* B, double* R, long long nndof, Timers& t) {
  double t1 = now_sec();
  matvec(a, a->N, X, R);
  t.spmv += now_sec() - t1;
  axpby(nndof, 1.0, B, -1.0, R, R);  // src/linalg/matvec.f90:877-903
}

// src/linalg/mat_converge.f90:90-141; returns true when converged.
bool check_converge(MONOLIS_PRM* prm, long long nndof, const double* R, double B2, int iter,
                    Timers& t, int* status) {
  double t1 = now_sec();
  double R2 = dot(nndof, R, R);
  t.dotp += now_sec() - t1;
  double resid = std::sqrt(R2 / B2);
  if (g_iter_clock && iter < g_iter_clock_cap) g_iter_clock[iter] = now_sec();
  prm->Iarray[MONOLIS_PRM_I_CUR_ITER] = iter;
  prm->Rarray[MONOLIS_PRM_R_CUR_RESID] = resid;
  if (prm->Iarray[MONOLIS_PRM_I_SHOW_ITERLOG] == MONOLIS_I_TRUE) printf("%7d%16.6E\n", iter, resid);
  if (resid < prm->Rarray[MONOLIS_PRM_R_TOL]) return true;
  if (!std::isfinite(resid)) *status = 3;
  if (iter == prm->Iarray[MONOLIS_PRM_I_MAX_ITER]) {
    *status = 1;
    if (prm->Iarray[MONOLIS_PRM_I_IS_MEASUREMENT] == MONOLIS_I_FALSE &&
        prm->Iarray[MONOLIS_PRM_I_IS_ERROR_ABORT] == MONOLIS_I_TRUE)
      error_stop("reached the maximum number of iterations");
  }
  return false;
}

// src/iterative/CG.f90:18-119
int solver_CG(MONOLIS_PRM* prm, MONOLIS_MAT* a, const Prec& pc, Timers& t) {
  double* X = a->R.X;
  const double* B = a->R.B;
  const int iter_RR = g_iter_rr;
  long long nndof = (long long)a->N * a->NDOF;
  if (prm->Iarray[MONOLIS_PRM_I_IS_INIT_X] == MONOLIS_I_TRUE)
    for (long long i = 0; i < (long long)a->NP * a->NDOF; i++) X[i] = 0.0;
  std::vector<double> R(nndof), Z(nndof), Q(nndof), P(nndof);
  residual(a, X, B, R.data(), nndof, t);
  double B2 = dot(nndof, R.data(), R.data());
  if (B2 == 0.0) {  // src/linalg/mat_converge.f90:40-48
    fprintf(stderr, "** monolis error: norm of RHS vector B is 0.0\n");
    for (long long i = 0; i < (long long)a->NP * a->NDOF; i++) X[i] = 0.0;
    return 0;
  }
  double rho = 0, rho1 = 0, alpha, beta, omega;
  int status = 0;
  for (int iter = 1; iter <= prm->Iarray[MONOLIS_PRM_I_MAX_ITER]; iter++) {
    double t1 = now_sec();
    precond_apply(a, pc, nndof, R.data(), Z.data());
    t.prec += now_sec() - t1;
    t1 = now_sec();
    rho = dot(nndof, R.data(), Z.data());
    t.dotp += now_sec() - t1;
    if (1 < iter) {
      beta = rho / rho1;
      axpby(nndof, beta, P.data(), 1.0, Z.data(), P.data());
    } else {
      vcopy(nndof, Z.data(), P.data());
    }
    t1 = now_sec();
    matvec(a, a->N, P.data(), Q.data());
    t.spmv += now_sec() - t1;
    t1 = now_sec();
    omega = dot(nndof, P.data(), Q.data());
    t.dotp += now_sec() - t1;
    alpha = rho / omega;
    axpby(nndof, alpha, P.data(), 1.0, X, X);
    if (iter % iter_RR == 0) residual(a, X, B, R.data(), nndof, t);
    else axpby(nndof, -alpha, Q.data(), 1.0, R.data(), R.data());
    if (check_converge(prm, nndof, R.data(), B2, iter, t, &status)) return 0;
    if (status == 3) return 3;
    rho1 = rho;
  }
  return status ? status : 1;
}

// src/iterative/BiCGSTAB.f90:18-192; with n128, src/iterative/
// BiCGSTAB_N128.f90:18-153, which takes rho = <R,RT> and c2 = <RT,V> in
// double-double (:73, :90) and everything else as BiCGSTAB.f90 (its
// (T,S), (T,T) pass through a double-double all-reduce, the identity at
// one rank, :104-108).
int solver_BiCGSTAB(MONOLIS_PRM* prm, MONOLIS_MAT* a, const Prec& pc, Timers& t, bool n128 = false) {
  double* X = a->R.X;
  const double* B = a->R.B;
  const int iter_RR = g_iter_rr;
  long long nndof = (long long)a->N * a->NDOF;
  if (prm->Iarray[MONOLIS_PRM_I_IS_INIT_X] == MONOLIS_I_TRUE)
    for (long long i = 0; i < (long long)a->NP * a->NDOF; i++) X[i] = 0.0;
  std::vector<double> R(nndof), RT(nndof), P(nndof), PT(nndof), S(nndof), ST(nndof), T(nndof), V(nndof);
  residual(a, X, B, R.data(), nndof, t);
  double B2 = dot(nndof, R.data(), R.data());
  if (B2 == 0.0) {
    fprintf(stderr, "** monolis error: norm of RHS vector B is 0.0\n");
    for (long long i = 0; i < (long long)a->NP * a->NDOF; i++) X[i] = 0.0;
    return 0;
  }
  vcopy(nndof, R.data(), RT.data());
  double alpha = 0, beta, rho, rho1 = 0, c2, omega = 0.0;
  int status = 0;
  for (int iter = 1; iter <= prm->Iarray[MONOLIS_PRM_I_MAX_ITER]; iter++) {
    double t1 = now_sec();
    rho = n128 ? dot_n128(nndof, R.data(), RT.data()) : dot(nndof, R.data(), RT.data());
    if (std::fabs(rho) == 0.0) rho = sorted_dot(nndof, R.data(), RT.data());
    t.dotp += now_sec() - t1;
    if (1 < iter) {
      beta = (rho / rho1) * (alpha / omega);
#pragma omp parallel for schedule(static)
      for (long long i = 0; i < nndof; i++) P[i] = R[i] + beta * (P[i] - omega * V[i]);
    } else {
      vcopy(nndof, R.data(), P.data());
    }
    t1 = now_sec();
    precond_apply(a, pc, nndof, P.data(), PT.data());
    t.prec += now_sec() - t1;
    t1 = now_sec();
    matvec(a, a->N, PT.data(), V.data());
    t.spmv += now_sec() - t1;
    t1 = now_sec();
    c2 = n128 ? dot_n128(nndof, RT.data(), V.data()) : dot(nndof, RT.data(), V.data());
    if (std::fabs(c2) == 0.0) c2 = sorted_dot(nndof, RT.data(), V.data());
    t.dotp += now_sec() - t1;
    alpha = rho / c2;
    axpby(nndof, -alpha, V.data(), 1.0, R.data(), S.data());
    t1 = now_sec();
    precond_apply(a, pc, nndof, S.data(), ST.data());
    t.prec += now_sec() - t1;
    t1 = now_sec();
    matvec(a, a->N, ST.data(), T.data());
    t.spmv += now_sec() - t1;
    t1 = now_sec();
    double cg1 = dot(nndof, T.data(), S.data());
    double cg2 = dot(nndof, T.data(), T.data());
    if (std::fabs(cg2) == 0.0) cg2 = sorted_dot(nndof, T.data(), T.data());
    t.dotp += now_sec() - t1;
    omega = (std::fabs(cg2) == 0.0) ? 0.0 : cg1 / cg2;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nndof; i++) X[i] = X[i] + alpha * PT[i] + omega * ST[i];
    if (iter % iter_RR == 0) residual(a, X, B, R.data(), nndof, t);
    else axpby(nndof, -omega, T.data(), 1.0, S.data(), R.data());
    if (check_converge(prm, nndof, R.data(), B2, iter, t, &status)) return 0;
    if (status == 3) return 3;
    rho1 = rho;
  }
  return status ? status : 1;
}

// src/iterative/PipeCG.f90:18-160 (pipelined CG: one reduction phase per
// iteration whose sums are independent of the product that follows)
int solver_PipeCG(MONOLIS_PRM* prm, MONOLIS_MAT* a, const Prec& pc, Timers& t) {
  double* X = a->R.X;
  const double* B = a->R.B;
  const int iter_RR = g_iter_rr_pipe;
  long long nndof = (long long)a->N * a->NDOF;
  if (prm->Iarray[MONOLIS_PRM_I_IS_INIT_X] == MONOLIS_I_TRUE)
    for (long long i = 0; i < (long long)a->NP * a->NDOF; i++) X[i] = 0.0;
  std::vector<double> R(nndof), U(nndof), V(nndof), Q(nndof), P(nndof), Z(nndof), L(nndof), M(nndof), S(nndof);
  residual(a, X, B, R.data(), nndof, t);
  double B2 = dot(nndof, R.data(), R.data());
  if (B2 == 0.0) {  // src/linalg/mat_converge.f90:40-48
    fprintf(stderr, "** monolis error: norm of RHS vector B is 0.0\n");
    for (long long i = 0; i < (long long)a->NP * a->NDOF; i++) X[i] = 0.0;
    return 0;
  }
  double t1 = now_sec();
  precond_apply(a, pc, nndof, R.data(), U.data());
  t.prec += now_sec() - t1;
  t1 = now_sec();
  matvec(a, a->N, U.data(), V.data());
  t.spmv += now_sec() - t1;
  double gamma = 1.0, alpha = 1.0, beta, delta;
  int status = 0;
  for (int iter = 1; iter <= prm->Iarray[MONOLIS_PRM_I_MAX_ITER]; iter++) {
    t1 = now_sec();
    const double cg1 = dot(nndof, R.data(), U.data());  // PipeCG.f90:88-91 (<R,R> there is not used)
    const double cg2 = dot(nndof, V.data(), U.data());
    t.dotp += now_sec() - t1;
    t1 = now_sec();
    precond_apply(a, pc, nndof, V.data(), M.data());
    t.prec += now_sec() - t1;
    t1 = now_sec();
    matvec(a, a->N, M.data(), L.data());
    t.spmv += now_sec() - t1;
    const double gamma1 = 1.0 / gamma;
    const double alpha1 = 1.0 / alpha;
    gamma = cg1;
    delta = cg2;
    if (1 < iter) {
      beta = gamma * gamma1;
      alpha = gamma / (delta - beta * gamma * alpha1);
    } else {
      alpha = gamma / delta;
      beta = 0.0;
    }
    axpby(nndof, beta, Z.data(), 1.0, L.data(), Z.data());
    axpby(nndof, beta, Q.data(), 1.0, M.data(), Q.data());
    axpby(nndof, beta, S.data(), 1.0, V.data(), S.data());
    axpby(nndof, beta, P.data(), 1.0, U.data(), P.data());
    if (iter % iter_RR == 0) {
      axpby(nndof, alpha, P.data(), 1.0, X, X);
      residual(a, X, B, R.data(), nndof, t);
      t1 = now_sec();
      precond_apply(a, pc, nndof, R.data(), U.data());
      t.prec += now_sec() - t1;
      t1 = now_sec();
      matvec(a, a->N, U.data(), V.data());
      t.spmv += now_sec() - t1;
    } else {
      axpby(nndof, -alpha, S.data(), 1.0, R.data(), R.data());
      axpby(nndof, -alpha, Q.data(), 1.0, U.data(), U.data());
      axpby(nndof, -alpha, Z.data(), 1.0, V.data(), V.data());
      axpby(nndof, alpha, P.data(), 1.0, X, X);
    }
    if (check_converge(prm, nndof, R.data(), B2, iter, t, &status)) return 0;
    if (status == 3) return 3;
  }
  return status ? status : 1;
}

// src/iterative/GropCG.f90:18-139 (Gropp's CG: <R,U> and <R,R> of an
// iteration are independent of the product V = A U that follows; the
// reference runs no true-residual replacement here)
int solver_GropCG(MONOLIS_PRM* prm, MONOLIS_MAT* a, const Prec& pc, Timers& t) {
  double* X = a->R.X;
  const double* B = a->R.B;
  long long nndof = (long long)a->N * a->NDOF;
  if (prm->Iarray[MONOLIS_PRM_I_IS_INIT_X] == MONOLIS_I_TRUE)
    for (long long i = 0; i < (long long)a->NP * a->NDOF; i++) X[i] = 0.0;
  std::vector<double> R(nndof), U(nndof), V(nndof), Q(nndof), P(nndof), S(nndof);
  residual(a, X, B, R.data(), nndof, t);
  double B2 = dot(nndof, R.data(), R.data());
  if (B2 == 0.0) {  // src/linalg/mat_converge.f90:40-48
    fprintf(stderr, "** monolis error: norm of RHS vector B is 0.0\n");
    for (long long i = 0; i < (long long)a->NP * a->NDOF; i++) X[i] = 0.0;
    return 0;
  }
  double t1 = now_sec();
  precond_apply(a, pc, nndof, R.data(), U.data());
  t.prec += now_sec() - t1;
  vcopy(nndof, U.data(), P.data());
  t1 = now_sec();
  matvec(a, a->N, P.data(), S.data());
  t.spmv += now_sec() - t1;
  t1 = now_sec();
  double gamma = dot(nndof, R.data(), U.data());
  t.dotp += now_sec() - t1;
  int status = 0;
  for (int iter = 1; iter <= prm->Iarray[MONOLIS_PRM_I_MAX_ITER]; iter++) {
    t1 = now_sec();
    const double delta = dot(nndof, P.data(), S.data());
    t.dotp += now_sec() - t1;
    t1 = now_sec();
    precond_apply(a, pc, nndof, S.data(), Q.data());
    t.prec += now_sec() - t1;
    const double alpha = gamma / delta;
    axpby(nndof, alpha, P.data(), 1.0, X, X);
    axpby(nndof, -alpha, S.data(), 1.0, R.data(), R.data());
    axpby(nndof, -alpha, Q.data(), 1.0, U.data(), U.data());
    t1 = now_sec();
    const double gamma1 = dot(nndof, R.data(), U.data());
    t.dotp += now_sec() - t1;
    t1 = now_sec();
    matvec(a, a->N, U.data(), V.data());
    t.spmv += now_sec() - t1;
    const double beta = gamma1 / gamma;
    gamma = gamma1;
    axpby(nndof, beta, P.data(), 1.0, U.data(), P.data());
    axpby(nndof, beta, S.data(), 1.0, V.data(), S.data());
    if (check_converge(prm, nndof, R.data(), B2, iter, t, &status)) return 0;
    if (status == 3) return 3;
  }
  return status ? status : 1;
}

const char* str_iter(int m) {
  static const char* names[] = {"CG", "GropCG", "PipeCG", "PipeCR", "BiCGSTAB", "PipeBiCGSTAB",
                                "BiCGSTAB_noprec", "PipeBiCGSTAB_noprec", "BiCGSTAB_N128", "SOR",
                                "BiCGSAFE", "IDR(s)", "COCG"};
  return (m >= 1 && m <= 13) ? names[m - 1] : "?";
}
const char* str_prec(int p) {
  static const char* names[] = {"None", "Diag", "SOR", "LU", "MUMPS", "MUMPSL"};
  return (p >= 0 && p <= 5) ? names[p] : "?";
}

// src/solver/solver.f90:77-185 + src/define/def_solver_prm.f90:237-355
void solve_main(MONOLIS_PRM* prm, MONOLIS_MAT* a) {
  double t_start = now_sec();
  int* I = prm->Iarray;
  double* Rr = prm->Rarray;
  for (int k = MONOLIS_R_TIME_SOL; k <= MONOLIS_R_TIME_COMM_SPMV; k++) Rr[k] = 0.0;
  Timers t;
  Prec pc;
  double t1 = now_sec();
  if (I[MONOLIS_PRM_I_PRECOND] == MONOLIS_PREC_DIAG) {
    pc.kind = 1;
    diag_setup(a, pc.ALU);
  } else if (I[MONOLIS_PRM_I_PRECOND] != MONOLIS_PREC_NONE) {
    error_stop("The preconditioner is not implemented in this library");
  }
  Rr[MONOLIS_R_TIME_PREP] += now_sec() - t1;
  if (I[MONOLIS_PRM_I_SHOW_SUMMARY] == MONOLIS_I_TRUE)
    printf("** MONOLIS solver: %s, prec: %s\n", str_iter(I[MONOLIS_PRM_I_METHOD]),
           str_prec(I[MONOLIS_PRM_I_PRECOND]));
  int status;
  if (I[MONOLIS_PRM_I_METHOD] == MONOLIS_ITER_CG) status = solver_CG(prm, a, pc, t);
  else if (I[MONOLIS_PRM_I_METHOD] == MONOLIS_ITER_BICGSTAB) status = solver_BiCGSTAB(prm, a, pc, t);
  else if (I[MONOLIS_PRM_I_METHOD] == MONOLIS_ITER_BICGSTAB_N128) status = solver_BiCGSTAB(prm, a, pc, t, true);
  else if (I[MONOLIS_PRM_I_METHOD] == MONOLIS_ITER_PIPECG) status = solver_PipeCG(prm, a, pc, t);
  else if (I[MONOLIS_PRM_I_METHOD] == MONOLIS_ITER_GROPCG) status = solver_GropCG(prm, a, pc, t);
  else error_stop("please select a linear solver for real numbers");
  I[MONOLIS_PRM_I_IERR] = status;
  Rr[MONOLIS_R_TIME_SPMV] = t.spmv;
  Rr[MONOLIS_R_TIME_DOTP] = t.dotp;
  Rr[MONOLIS_R_TIME_PREC] = t.prec;
  Rr[MONOLIS_R_TIME_SOL] = now_sec() - t_start;
  if (I[MONOLIS_PRM_I_SHOW_SUMMARY] == MONOLIS_I_TRUE) {
    printf("** MONOLIS converge iter:%10d\n", I[MONOLIS_PRM_I_CUR_ITER]);
    printf("** MONOLIS rel. residual:%10.3E\n", Rr[MONOLIS_PRM_R_CUR_RESID]);
  }
  if (I[MONOLIS_PRM_I_SHOW_SUMMARY] == MONOLIS_I_TRUE || I[MONOLIS_PRM_I_SHOW_TIME] == MONOLIS_I_TRUE)
    printf("** MONOLIS solution time:%10.3E\n", Rr[MONOLIS_R_TIME_SOL]);
  if (I[MONOLIS_PRM_I_SHOW_TIME] == MONOLIS_I_TRUE) {
    printf(" - solution/prepost time:%10.3E\n", Rr[MONOLIS_R_TIME_PREP]);
    printf(" - solution/SpMV    time:%10.3E\n", Rr[MONOLIS_R_TIME_SPMV]);
    printf(" - solution/inner p time:%10.3E\n", Rr[MONOLIS_R_TIME_DOTP]);
    printf(" - solution/precond time:%10.3E\n", Rr[MONOLIS_R_TIME_PREC]);
    printf(" - (comm time/inner p)  :%10.3E\n", Rr[MONOLIS_R_TIME_COMM_DOTP]);
    printf(" - (comm time/spmv)     :%10.3E\n", Rr[MONOLIS_R_TIME_COMM_SPMV]);
  }
  fflush(stdout);
}

}  // namespace

extern "C" {

// ---- monolis_utils subset ----
void monolis_com_initialize_by_self(MONOLIS_COM* com) {
  memset(com, 0, sizeof(*com));
  com->comm_size = 1;
  com->n_internal_vertex = 0;
  com->recv_index = alloc_zero<int>(1);
  com->send_index = alloc_zero<int>(1);
}
void monolis_com_finalize(MONOLIS_COM* com) {
  free_ptr(&com->recv_neib_pe); free_ptr(&com->recv_index); free_ptr(&com->recv_item);
  free_ptr(&com->send_neib_pe); free_ptr(&com->send_index); free_ptr(&com->send_item);
  memset(com, 0, sizeof(*com));
}

// ---- init / finalize: wrapper/define/*.c ----
void monolis_global_initialize(void) {}
void monolis_global_finalize(void) {}

void monolis_prm_initialize(MONOLIS_PRM* prm) {
  strcpy(prm->com_top_dir_name, ".");
  strcpy(prm->com_part_dir_name, "parted.0");
  strcpy(prm->com_file_name, "node.dat");
  for (int i = 0; i < MONOLIS_PRM_IARRAY_SIZE; ++i) prm->Iarray[i] = 0;
  for (int i = 0; i < MONOLIS_PRM_RARRAY_SIZE; ++i) prm->Rarray[i] = 0.0;
  prm->Iarray[MONOLIS_PRM_I_METHOD] = 1;
  prm->Iarray[MONOLIS_PRM_I_PRECOND] = 1;
  prm->Iarray[MONOLIS_PRM_I_MAX_ITER] = 1000;
  prm->Iarray[MONOLIS_PRM_I_CUR_ITER] = 0;
  prm->Iarray[MONOLIS_PRM_I_IERR] = -1;
  prm->Iarray[MONOLIS_PRM_I_IS_INIT_X] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_IS_ERROR_ABORT] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_SHOW_ITERLOG] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_SHOW_TIME] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_SHOW_SUMMARY] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_IDRS_DIM] = 4;
  prm->Rarray[MONOLIS_PRM_R_TOL] = 1.0e-8;
}
void monolis_prm_finalize(MONOLIS_PRM* prm) {
  for (int i = 0; i < MONOLIS_PRM_IARRAY_SIZE; ++i) prm->Iarray[i] = 0;
  for (int i = 0; i < MONOLIS_PRM_RARRAY_SIZE; ++i) prm->Rarray[i] = 0.0;
}
void monolis_mat_initialize(MONOLIS_MAT* mat) { memset(mat, 0, sizeof(*mat)); }
void monolis_mat_finalize(MONOLIS_MAT* mat) {
  free_ptr(&mat->n_dof_list); free_ptr(&mat->n_dof_index); free_ptr(&mat->n_dof_index2);
  free_ptr(&mat->R.A); free_ptr(&mat->R.U); free_ptr(&mat->R.D); free_ptr(&mat->R.L);
  free_ptr(&mat->R.X); free_ptr(&mat->R.B);
  free_ptr(&mat->SCSR.indexU); free_ptr(&mat->SCSR.indexL); free_ptr(&mat->SCSR.itemU);
  free_ptr(&mat->SCSR.itemL);
  free_ptr(&mat->CSR.index); free_ptr(&mat->CSR.item);
  free_ptr(&mat->CSC.index); free_ptr(&mat->CSC.item); free_ptr(&mat->CSC.perm);
  memset(mat, 0, sizeof(*mat));
}
void monolis_initialize(MONOLIS* m) {
  monolis_prm_initialize(&m->prm);
  monolis_mat_initialize(&m->mat);
  monolis_mat_initialize(&m->prec);
}
void monolis_finalize(MONOLIS* m) {
  monolis_prm_finalize(&m->prm);
  monolis_mat_finalize(&m->mat);
  monolis_mat_finalize(&m->prec);
}
void monolis_get_vec_size(int N, int NP, int NDOF, int NZ, int* n_dof_index, int* n_dof_index2,
                          int* N_size, int* NP_size, int* NZ_size) {
  if (NDOF == -1) {
    *N_size = n_dof_index[N]; *NP_size = n_dof_index[NP]; *NZ_size = n_dof_index2[NZ];
  } else {
    *N_size = N * NDOF; *NP_size = NP * NDOF; *NZ_size = NZ * NDOF * NDOF;
  }
}

// ---- parameters: wrapper/define/monolis_def_solver_prm_util_c.c ----
void monolis_set_method(MONOLIS* m, int p) { m->prm.Iarray[MONOLIS_PRM_I_METHOD] = p; }
void monolis_set_precond(MONOLIS* m, int p) { m->prm.Iarray[MONOLIS_PRM_I_PRECOND] = p; }
void monolis_set_spmv_format(MONOLIS* m, int p) { m->prm.Iarray[MONOLIS_PRM_I_SPMV_FORMAT] = p; }
void monolis_set_maxiter(MONOLIS* m, int p) { m->prm.Iarray[MONOLIS_PRM_I_MAX_ITER] = p; }
void monolis_get_converge_iter(MONOLIS* m, int* p) { *p = m->prm.Iarray[MONOLIS_PRM_I_CUR_ITER]; }
void monolis_get_error_tag(MONOLIS* m, int* p) { *p = m->prm.Iarray[MONOLIS_PRM_I_IERR]; }
void monolis_set_init_x(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_IS_INIT_X] = (int)p; }
void monolis_set_sym_matrix(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_IS_SYM_MATRIX] = p; }
void monolis_set_debug(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_IS_DEBUG] = p; }
void monolis_set_performance_measurement(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_IS_MEASUREMENT] = p; }
void monolis_set_check_diag(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_IS_CHECK_DIAG] = p; }
void monolis_set_prec_stored(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_IS_PREC_STORED] = p; }
void monolis_set_error_abort(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_IS_ERROR_ABORT] = p; }
void monolis_set_solver_IDRS_num_basis(MONOLIS* m, int p) { m->prm.Iarray[MONOLIS_PRM_I_IDRS_DIM] = p; }
void monolis_show_iterlog(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_SHOW_ITERLOG] = p; }
void monolis_show_timelog(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_SHOW_TIME] = p; }
void monolis_show_summary(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_SHOW_SUMMARY] = p; }
void monolis_show_timelog_statistics(MONOLIS* m, bool p) { m->prm.Iarray[MONOLIS_PRM_I_SHOW_TIME_STATISTICS] = p; }
void monolis_set_tolerance(MONOLIS* m, double v) { m->prm.Rarray[MONOLIS_PRM_R_TOL] = v; }
void monolis_get_converge_residual(MONOLIS* m, double* v) { *v = m->prm.Rarray[MONOLIS_PRM_R_CUR_RESID]; }
void monolis_get_time_solver(MONOLIS* m, double* v) { *v = m->prm.Rarray[MONOLIS_R_TIME_SOL]; }
void monolis_get_time_preparing(MONOLIS* m, double* v) { *v = m->prm.Rarray[MONOLIS_R_TIME_PREP]; }
void monolis_get_time_spmv(MONOLIS* m, double* v) { *v = m->prm.Rarray[MONOLIS_R_TIME_SPMV]; }
void monolis_get_time_inner_product(MONOLIS* m, double* v) { *v = m->prm.Rarray[MONOLIS_R_TIME_DOTP]; }
void monolis_get_time_precondition(MONOLIS* m, double* v) { *v = m->prm.Rarray[MONOLIS_R_TIME_PREC]; }
void monolis_get_time_comm_inner_product(MONOLIS* m, double* v) { *v = m->prm.Rarray[MONOLIS_R_TIME_COMM_DOTP]; }
void monolis_get_time_comm_spmv(MONOLIS* m, double* v) { *v = m->prm.Rarray[MONOLIS_R_TIME_COMM_SPMV]; }

// ---- nonzero pattern ----
// src/matrix/spmat_nzpattern_util.f90:162-218 (C: 0-based offsets, 1-based items)
void monolis_get_CSC_format(int NC, int NR, int NZ, int* index, int* item, int* indexR, int* itemR,
                            int* permR) {
  (void)NZ;
  std::vector<int> temp(NR + 1, 0);
  for (int i = 0; i < NC; i++)
    for (int j = index[i]; j < index[i + 1]; j++) temp[item[j] - 1]++;
  indexR[0] = 0;
  for (int i = 0; i < NR; i++) indexR[i + 1] = indexR[i] + temp[i];
  std::fill(temp.begin(), temp.end(), 0);
  for (int i = 0; i < NC; i++)
    for (int j = index[i]; j < index[i + 1]; j++) {
      int in = item[j] - 1;
      int p = indexR[in] + temp[in]++;
      itemR[p] = i + 1;
      permR[p] = j + 1;
    }
}

void monolis_get_nonzero_pattern_by_nodal_graph_R(MONOLIS* m, int n_node, int n_dof, int* index, int* item) {
  finish_pattern(m, n_node, n_dof, index, item);
}

void monolis_get_nonzero_pattern_by_simple_mesh_R(MONOLIS* m, int n_node, int n_base, int n_dof, int n_elem,
                                                  int** elem) {
  std::vector<int> flat((size_t)n_elem * n_base);
  for (int e = 0; e < n_elem; e++)
    for (int a = 0; a < n_base; a++) flat[(size_t)e * n_base + a] = elem[e][a];
  std::vector<int> index, item;
  nodal_graph_from_mesh(n_node, n_base, n_elem, flat.data(), index, item);
  finish_pattern(m, n_node, n_dof, index.data(), item.data());
}

void monolis_get_nonzero_pattern_by_connectivity_R(MONOLIS* m, int n_node, int n_dof, int n_elem,
                                                   int* conn_index, int* conn_item) {
  std::vector<std::vector<int>> nb(n_node);
  for (int e = 0; e < n_elem; e++)
    for (int a = conn_index[e]; a < conn_index[e + 1]; a++)
      for (int b = conn_index[e]; b < conn_index[e + 1]; b++)
        if (conn_item[a] != conn_item[b]) nb[conn_item[a]].push_back(conn_item[b]);
  std::vector<int> index(n_node + 1, 0), item;
  for (int i = 0; i < n_node; i++) {
    std::sort(nb[i].begin(), nb[i].end());
    nb[i].erase(std::unique(nb[i].begin(), nb[i].end()), nb[i].end());
    index[i + 1] = index[i] + (int)nb[i].size();
    item.insert(item.end(), nb[i].begin(), nb[i].end());
  }
  finish_pattern(m, n_node, n_dof, index.data(), item.data());
}

// ---- assembly ----
void monolis_set_scalar_to_sparse_matrix_R(MONOLIS* m, int i, int j, int si, int sj, double val) {
  double* p = scalar_slot(m, i, j, si, sj);
  if (!p) error_stop("matrix assemble: entry not in the nonzero pattern");
  *p = val;
}
void monolis_add_scalar_to_sparse_matrix_R(MONOLIS* m, int i, int j, int si, int sj, double val) {
  double* p = scalar_slot(m, i, j, si, sj);
  if (!p) error_stop("matrix assemble: entry not in the nonzero pattern");
  *p = *p + val;
}
void monolis_get_scalar_from_sparse_matrix_R(MONOLIS* m, int i, int j, int si, int sj, double* val,
                                             bool* is_find) {
  double* p = scalar_slot(m, i, j, si, sj);
  *is_find = p != nullptr;
  *val = p ? *p : 0.0;
}
void monolis_add_matrix_to_sparse_matrix_R(MONOLIS* m, int n_base, int* conn, double** val) {
  int nzm = 0;
  for (int i = 0; i < n_base; i++) nzm += m->mat.n_dof_index[conn[i] + 1] - m->mat.n_dof_index[conn[i]];
  std::vector<double> v((size_t)nzm * nzm);
  for (int i = 0; i < nzm; i++)
    for (int j = 0; j < nzm; j++) v[(size_t)i * nzm + j] = val[i][j];
  add_matrix_main(m, n_base, n_base, conn, conn, v.data());
}
void monolis_add_matrix_to_sparse_matrix_offdiag_R(MONOLIS* m, int n1, int n2, int* c1, int* c2,
                                                   double** val) {
  int r = 0, c = 0;
  for (int i = 0; i < n1; i++) r += m->mat.n_dof_index[c1[i] + 1] - m->mat.n_dof_index[c1[i]];
  for (int i = 0; i < n2; i++) c += m->mat.n_dof_index[c2[i] + 1] - m->mat.n_dof_index[c2[i]];
  std::vector<double> v((size_t)r * c);
  for (int i = 0; i < r; i++)
    for (int j = 0; j < c; j++) v[(size_t)i * c + j] = val[i][j];
  add_matrix_main(m, n1, n2, c1, c2, v.data());
}
// wrapper/matrix/monolis_spmat_handler_c.c:205-248 (allocations assigned, dof index set)
void monolis_set_matrix_BCSR_R(MONOLIS* m, int n, int np, int n_dof, int nz, double* A, int* index, int* item) {
  MONOLIS_MAT* a = &m->mat;
  a->N = n; a->NP = np; a->NDOF = n_dof;
  a->CSR.index = alloc_zero<int>(np + 1);
  a->CSR.item = alloc_zero<int>(nz);
  a->R.A = alloc_zero<double>((long long)n_dof * n_dof * nz);
  a->R.X = alloc_zero<double>((long long)n_dof * np);
  a->R.B = alloc_zero<double>((long long)n_dof * np);
  for (int i = 0; i < np + 1; i++) a->CSR.index[i] = index[i];
  for (int i = 0; i < nz; i++) a->CSR.item[i] = item[i] + 1;
  for (long long i = 0; i < (long long)n_dof * n_dof * nz; i++) a->R.A[i] = A[i];
  a->CSC.index = alloc_zero<int>(np + 1);
  a->CSC.item = alloc_zero<int>(nz);
  a->CSC.perm = alloc_zero<int>(nz);
  monolis_get_CSC_format(n, np, nz, a->CSR.index, a->CSR.item, a->CSC.index, a->CSC.item, a->CSC.perm);
  std::vector<int> list(np, n_dof);
  set_n_dof_index(a, list.data());
}
// src/matrix/spmat_handler_util.f90:604-677 (C: 0-based node_id and n_dof_bc)
void monolis_set_Dirichlet_bc_R(MONOLIS* m, double* B, int node_id, int ndof_bc, double val) {
  MONOLIS_MAT* a = &m->mat;
  const int* ndi = a->n_dof_index;
  const int* nd2 = a->n_dof_index2;
  int ndof1 = ndi[node_id + 1] - ndi[node_id];
  if (ndof_bc >= ndof1) error_stop("submatrix access out of range");
  for (int j = a->CSC.index[node_id]; j < a->CSC.index[node_id + 1]; j++) {
    int jn = a->CSC.item[j] - 1;
    int kn = a->CSC.perm[j] - 1;
    int ndof2 = ndi[jn + 1] - ndi[jn];
    for (int k = 0; k < ndof2; k++) {
      long long mm = (long long)nd2[kn] + (long long)ndof1 * k + ndof_bc;
      long long n = (long long)ndi[jn] + k;
      B[n] = B[n] - val * a->R.A[mm];
      a->R.A[mm] = 0.0;
    }
  }
  bool is_add = false;
  for (int j = a->CSR.index[node_id]; j < a->CSR.index[node_id + 1]; j++) {
    int jn = a->CSR.item[j] - 1;
    int ndof2 = ndi[jn + 1] - ndi[jn];
    for (int k = 0; k < ndof2; k++) a->R.A[(long long)nd2[j] + (long long)ndof2 * ndof_bc + k] = 0.0;
    if (jn == node_id) {
      a->R.A[(long long)nd2[j] + (long long)(ndof2 + 1) * ndof_bc] = 1.0;
      is_add = true;
    }
  }
  if (!is_add) error_stop("set Dirichlet: diagonal block not found");
  B[ndi[node_id] + ndof_bc] = val;
}

// ---- linear algebra API ----
void monolis_matvec_product_R(MONOLIS* m, MONOLIS_COM* com, double* x, double* y) {
  (void)com;
  matvec(&m->mat, m->mat.N, x, y);
}
void monolis_inner_product_R(MONOLIS* m, MONOLIS_COM* com, int n_dof, double* x, double* y, double* sum) {
  (void)com;
  *sum = dot((long long)m->mat.N * n_dof, x, y);
}

// src/solver/solver.f90:29-49: copy B and X in, solve, copy X out.
void monolis_solve_R(MONOLIS* m, MONOLIS_COM* com, double* b, double* x) {
  (void)com;
  if (g_iter_clock && g_iter_clock_cap > 0) g_iter_clock[0] = now_sec();
  MONOLIS_MAT* a = &m->mat;
  long long npndof = (long long)a->NP * a->NDOF;
  for (long long i = 0; i < npndof; i++) a->R.B[i] = b[i];
  for (long long i = 0; i < npndof; i++) a->R.X[i] = x[i];
  solve_main(&m->prm, a);
  for (long long i = 0; i < npndof; i++) x[i] = a->R.X[i];
}

// ---- oracle-only helpers (tests and the CPU baseline) ----

// Sets the OpenMP thread count; 1 reproduces the reference's serial build.
void oracle_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n < 1 ? 1 : n);
#else
  (void)n;
#endif
}
// Wall-clock log of the following solves (see g_iter_clock); buf = NULL
// switches it off.
void oracle_set_iter_clock(double* buf, int cap) {
  g_iter_clock = buf;
  g_iter_clock_cap = buf ? cap : 0;
}
void oracle_set_iter_rr(int n) {
  g_iter_rr = n > 0 ? n : 200;
  g_iter_rr_pipe = n > 0 ? n : 50;
}

int oracle_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Flat-array twin of get_nonzero_pattern_by_simple_mesh_R (elem[e*n_base+a]).
void oracle_pattern_by_simple_mesh_flat(MONOLIS* m, int n_node, int n_base, int n_dof, int n_elem,
                                        const int* elem) {
  std::vector<int> index, item;
  nodal_graph_from_mesh(n_node, n_base, n_elem, elem, index, item);
  finish_pattern(m, n_node, n_dof, index.data(), item.data());
}

// Element-by-element add_matrix_to_sparse_matrix_R calls: element e adds
// scale[e] * val[e*val_stride + :] (scale may be NULL = 1, val_stride 0 = shared).
void oracle_add_elements(MONOLIS* m, int n_elem, int n_base, const int* elem, const double* val,
                         long long val_stride, const double* scale) {
  int nd = m->mat.NDOF;
  int nzm = n_base * nd;
  std::vector<double> v((size_t)nzm * nzm);
  for (int e = 0; e < n_elem; e++) {
    const double* src = val + (long long)e * val_stride;
    if (scale) for (size_t k = 0; k < v.size(); k++) v[k] = scale[e] * src[k];
    else for (size_t k = 0; k < v.size(); k++) v[k] = src[k];
    add_matrix_main(m, n_base, n_base, elem + (long long)e * n_base, elem + (long long)e * n_base, v.data());
  }
}

// DIAG setup / apply exposed for element-wise checks.
void oracle_diag_setup(MONOLIS* m, double* ALU) {
  std::vector<double> v;
  diag_setup(&m->mat, v);
  memcpy(ALU, v.data(), v.size() * sizeof(double));
}
void oracle_diag_apply(MONOLIS* m, const double* ALU, const double* x, double* y) {
  long long n = (long long)m->mat.N * m->mat.NDOF * m->mat.NDOF;
  std::vector<double> v(ALU, ALU + n);
  diag_apply(&m->mat, v, x, y);
}
double oracle_dot(long long n, const double* x, const double* y) { return dot(n, x, y); }
double oracle_dot_n128(long long n, const double* x, const double* y) { return dot_n128(n, x, y); }
// 0: the reference's inner product in every solver and in monolis_inner_product_R;
// 1: double-double (dot_n128) everywhere.
void oracle_set_dot_mode(int mode) { g_dot_mode = mode == 1 ? 1 : 0; }
int oracle_get_dot_mode(void) { return g_dot_mode; }
double oracle_sorted_dot(long long n, const double* x, const double* y) { return sorted_dot(n, x, y); }

// check_converge restated for the known-answer test of mat_converge_test.f90.
int oracle_check_converge(MONOLIS* m, long long nndof, const double* R, double B2, int iter) {
  Timers t;
  int status = 0;
  return check_converge(&m->prm, nndof, R, B2, iter, t, &status) ? 1 : 0;
}

}  // extern "C"
