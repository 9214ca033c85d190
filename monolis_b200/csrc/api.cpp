// api.cpp -- the monolis C API (include/monolis.h + include/monolis_b200.h)
// on top of the B200 device solver.
//
// Host side: parameter arrays, nonzero pattern, assembly and Dirichlet
// conditions run on the host exactly as the reference defines them (CSR
// index 0-based, item 1-based, rows sorted ascending, blocks row-major), so
// the arrays in the MONOLIS struct are bit-identical to the reference's.
// The matrix arrays are allocated in pinned host memory when a GPU is
// present, so solves upload them at full PCIe bandwidth.
// Device side: every solve / matvec / inner product runs on the GPU
// (solve.cu, sell.cu); there is no CPU fallback.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include <cuda_runtime.h>

#include "dev.h"
#include "monolis.h"
#include "monolis_b200.h"

namespace {

// Return MONOLIS_B200_CUDA_ERROR from an entry point when a CUDA call fails.
#define MB_API_CUDA(call)                                   \
  do {                                                      \
    if ((call) != cudaSuccess) return MONOLIS_B200_CUDA_ERROR; \
  } while (0)

double now_sec() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

[[noreturn]] void error_stop(const char* msg) {
  fprintf(stderr, "** monolis error: %s\n", msg);
  fflush(stderr);
  exit(1);
}

// ---------------------------------------------------------------------------
// Host allocations: pinned when CUDA can provide it, zero-filled.
// ---------------------------------------------------------------------------
std::mutex g_alloc_mu;
std::unordered_map<void*, bool>& alloc_kind() {
  static std::unordered_map<void*, bool> m;
  return m;
}

int g_pinned_ok = -1;  // -1 unknown, 0 no device, 1 yes

void* host_alloc(size_t bytes) {
  if (bytes == 0) bytes = 16;
  void* p = nullptr;
  bool pinned = false;
  if (g_pinned_ok != 0) {
    if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) == cudaSuccess) {
      pinned = true;
      g_pinned_ok = 1;
    } else {
      cudaGetLastError();
      p = nullptr;
      if (g_pinned_ok == -1) g_pinned_ok = 0;
    }
  }
  if (!p) p = malloc(bytes);
  if (!p) error_stop("host allocation failed");
  memset(p, 0, bytes);
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  alloc_kind()[p] = pinned;
  return p;
}

template <class T>
T* halloc(long long n) {
  return static_cast<T*>(host_alloc(sizeof(T) * (size_t)(n > 0 ? n : 1)));
}

template <class T>
void hfree(T** pp) {
  void* p = *pp;
  *pp = nullptr;
  if (!p) return;
  bool pinned = false, known = false;
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    auto it = alloc_kind().find(p);
    if (it != alloc_kind().end()) {
      known = true;
      pinned = it->second;
      alloc_kind().erase(it);
    }
  }
  if (!known) return;  // not ours: the caller owns it
  if (pinned) cudaFreeHost(p);
  else free(p);
}

void bump_version(MONOLIS* m) { m->prm.Iarray[MONOLIS_B200_PRM_I_MATRIX_VERSION] += 1; }

// ---------------------------------------------------------------------------
// Nonzero pattern: row i = sorted {i} U {nodes sharing an element with i};
// items 1-based (wrapper/matrix/monolis_spmat_nzpattern_util_c.c:9-65).
// ---------------------------------------------------------------------------
void build_csr_from_rows(MONOLIS* m, int n_node, int n_dof, std::vector<int>& rowlen,
                         const std::function<void(int, std::vector<int>&)>& row_of) {
  MONOLIS_MAT* a = &m->mat;
  a->N = a->NP = n_node;
  a->NDOF = n_dof;
  a->CSR.index = halloc<int>(n_node + 1);
  for (int i = 0; i < n_node; i++) a->CSR.index[i + 1] = a->CSR.index[i] + rowlen[i];
  const long long nz = a->CSR.index[n_node];
  a->CSR.item = halloc<int>(nz);
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < n_node; i++) {
      row_of(i, buf);
      int* dst = a->CSR.item + a->CSR.index[i];
      for (size_t k = 0; k < buf.size(); k++) dst[k] = buf[k] + 1;
    }
  }
  a->CSC.index = halloc<int>(n_node + 1);
  a->CSC.item = halloc<int>(nz);
  a->CSC.perm = halloc<int>(nz);
  monolis_get_CSC_format(n_node, n_node, (int)nz, a->CSR.index, a->CSR.item, a->CSC.index, a->CSC.item,
                         a->CSC.perm);
  a->n_dof_list = halloc<int>(n_node);
  a->n_dof_index = halloc<int>(n_node + 1);
  a->n_dof_index2 = halloc<int>(nz + 1);
  for (int i = 0; i < n_node; i++) a->n_dof_list[i] = n_dof;
  for (int i = 0; i < n_node; i++) a->n_dof_index[i + 1] = a->n_dof_index[i] + n_dof;
  for (long long j = 0; j < nz; j++) a->n_dof_index2[j + 1] = a->n_dof_index2[j] + n_dof * n_dof;
  a->R.A = halloc<double>((long long)n_dof * n_dof * nz);
  a->R.X = halloc<double>((long long)n_dof * n_node);
  a->R.B = halloc<double>((long long)n_dof * n_node);
  bump_version(m);
}

// Mesh -> rows: node-to-element incidence, then per node the sorted union of
// its elements' nodes (self included).
void pattern_from_mesh(MONOLIS* m, int n_node, int n_base, int n_dof, int n_elem, const int* elem) {
  std::vector<int> ne(n_node + 1, 0);
  for (long long k = 0; k < (long long)n_elem * n_base; k++) ne[elem[k] + 1]++;
  for (int i = 0; i < n_node; i++) ne[i + 1] += ne[i];
  std::vector<int> el(ne[n_node]);
  {
    std::vector<int> fill(ne.begin(), ne.end() - 1);
    for (int e = 0; e < n_elem; e++)
      for (int a = 0; a < n_base; a++) el[fill[elem[(long long)e * n_base + a]]++] = e;
  }
  auto row_of = [&](int i, std::vector<int>& buf) {
    buf.clear();
    buf.push_back(i);
    for (int k = ne[i]; k < ne[i + 1]; k++) {
      const int* en = elem + (long long)el[k] * n_base;
      for (int a = 0; a < n_base; a++) buf.push_back(en[a]);
    }
    std::sort(buf.begin(), buf.end());
    buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
  };
  std::vector<int> rowlen(n_node);
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < n_node; i++) {
      row_of(i, buf);
      rowlen[i] = (int)buf.size();
    }
  }
  build_csr_from_rows(m, n_node, n_dof, rowlen, row_of);
}

// Slot of block (row i, column node j) or -1 (binary search, rows sorted).
inline long long find_block(const MONOLIS_MAT* a, int i, int j) {
  const int* it = a->CSR.item;
  int lo = a->CSR.index[i], hi = a->CSR.index[i + 1] - 1;
  const int key = j + 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    if (it[mid] == key) return mid;
    if (it[mid] < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

double* scalar_slot(MONOLIS* m, int i, int j, int si, int sj) {
  MONOLIS_MAT* a = &m->mat;
  if (i < 0 || i >= a->NP || j < 0 || j >= a->NP) error_stop("node id out of range");
  const int nd_i = a->n_dof_index[i + 1] - a->n_dof_index[i];
  const int nd_j = a->n_dof_index[j + 1] - a->n_dof_index[j];
  if (si < 0 || sj < 0 || si >= nd_i || sj >= nd_j) error_stop("submatrix access out of range");
  long long p = find_block(a, i, j);
  if (p < 0) return nullptr;
  return &a->R.A[(long long)a->n_dof_index2[p] + (long long)nd_j * si + sj];
}

// One element: rows r of e1, columns c of e2, dense val (n1*nd x n2*nd),
// added block by block (src/matrix/spmat_handler_util.f90:398-497).
void add_element(MONOLIS_MAT* a, int n1, int n2, const int* e1, const int* e2, const double* val, double scale,
                 bool scaled, int row_lo, int row_hi) {
  const int* ndi = a->n_dof_index;
  int off1 = 0;
  int ncol = 0;
  for (int q = 0; q < n2; q++) ncol += ndi[e2[q] + 1] - ndi[e2[q]];
  for (int pidx = 0; pidx < n1; pidx++) {
    const int r = e1[pidx];
    const int nr = ndi[r + 1] - ndi[r];
    if (r >= row_lo && r < row_hi) {
      int off2 = 0;
      for (int q = 0; q < n2; q++) {
        const int c = e2[q];
        const int kn = ndi[c + 1] - ndi[c];
        const long long slot = find_block(a, r, c);
        if (slot < 0) error_stop("matrix assemble: entry not in the nonzero pattern");
        double* dst = a->R.A + a->n_dof_index2[slot];
        for (int k1 = 0; k1 < nr; k1++)
          for (int k2 = 0; k2 < kn; k2++) {
            const double v = val[(long long)(off1 + k1) * ncol + off2 + k2];
            dst[kn * k1 + k2] = dst[kn * k1 + k2] + (scaled ? scale * v : v);
          }
        off2 += kn;
      }
    }
    off1 += nr;
  }
}

// ---------------------------------------------------------------------------
// NCCL communicators attached to MONOLIS_COM tables (multi-rank solve).
// ---------------------------------------------------------------------------
std::unordered_map<const MONOLIS_COM*, void*>& nccl_comms() {
  static std::unordered_map<const MONOLIS_COM*, void*> m;
  return m;
}

// ---------------------------------------------------------------------------
// Device context: one stream, one per-MONOLIS device state.
// ---------------------------------------------------------------------------
struct DevState {
  mb::SellMatrix A;
  mb::SellMatrix AT;  // A^T, built on demand from A's device CSR and the CSC arrays
  long long build_id = 0, at_build_id = -1;
  mb::MultiState* multi = nullptr;  // many-right-hand-side solver buffers
  mb::ShardPlan shard;              // multi-rank solve: halo buffers and tables
  bool device_values = false;       // the device values were assembled on the device (not uploaded)
  mb::Scratch sc;
  double* d_b = nullptr;
  double* d_x = nullptr;
  double* d_y = nullptr;
  size_t cap_vec = 0;
  // cache key
  const int* key_index = nullptr;
  const int* key_item = nullptr;
  const double* key_val = nullptr;
  int key_N = -1, key_ndof = -1, key_version = -1, key_prec = -1;
  bool prepared = false;
};

struct Ctx {
  bool init = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::unordered_map<const MONOLIS*, DevState*> states;
};

Ctx& ctx() {
  static Ctx c;
  return c;
}
std::mutex g_ctx_mu;

int ctx_init() {
  Ctx& c = ctx();
  if (c.init) return mb::kOk;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    fprintf(stderr, "** monolis_b200: no CUDA device available (%s); this library has no CPU path\n",
            cudaGetErrorString(e));
    return mb::kCudaError;
  }
  cudaGetDevice(&c.device);
  if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) return mb::kCudaError;
  c.init = true;
  return mb::kOk;
}

DevState* state_of(const MONOLIS* m) {
  Ctx& c = ctx();
  auto it = c.states.find(m);
  if (it != c.states.end()) return it->second;
  DevState* s = new DevState();
  c.states[m] = s;
  return s;
}

void state_release(const MONOLIS* m) {
  Ctx& c = ctx();
  auto it = c.states.find(m);
  if (it == c.states.end()) return;
  DevState* s = it->second;
  if (c.init) {
    cudaStreamSynchronize(c.stream);
    mb::sell_free(s->A);
    mb::sell_free(s->AT);
    mb::multi_free(s->multi);
    mb::shard_free(s->shard);
    mb::scratch_free(s->sc);
    cudaFree(s->d_b);
    cudaFree(s->d_x);
    cudaFree(s->d_y);
  }
  delete s;
  c.states.erase(it);
}

int ensure_vec(DevState* s, size_t n) {
  if (s->cap_vec >= n && s->d_b) return mb::kOk;
  cudaFree(s->d_b);
  cudaFree(s->d_x);
  cudaFree(s->d_y);
  s->d_b = s->d_x = s->d_y = nullptr;
  s->cap_vec = 0;
  if (cudaMalloc((void**)&s->d_b, n * sizeof(double) + 16) != cudaSuccess) return mb::kCudaError;
  if (cudaMalloc((void**)&s->d_x, n * sizeof(double) + 16) != cudaSuccess) return mb::kCudaError;
  if (cudaMalloc((void**)&s->d_y, n * sizeof(double) + 16) != cudaSuccess) return mb::kCudaError;
  s->cap_vec = n;
  return mb::kOk;
}

// CSR sanity (check mode): monotone offsets, items within [1, NP].
int check_csr(const MONOLIS_MAT* a) {
  if (!a->CSR.index || !a->CSR.item || !a->R.A) return mb::kBadInput;
  if (a->CSR.index[0] != 0) return mb::kBadInput;
  for (int i = 0; i < a->N; i++)
    if (a->CSR.index[i + 1] < a->CSR.index[i]) return mb::kBadInput;
  const long long nz = a->CSR.index[a->N];
  for (long long j = 0; j < nz; j++)
    if (a->CSR.item[j] < 1 || a->CSR.item[j] > a->NP) return mb::kBadInput;
  return mb::kOk;
}

// Upload (or reuse) the device matrix of m; DIAG factors; FP32 copies if asked.
int prepare(MONOLIS* m, DevState* s, bool need_diag, bool need_fp32, double* t_h2d) {
  MONOLIS_MAT* a = &m->mat;
  const int* I = m->prm.Iarray;
  if (a->NDOF < 1 || a->NDOF > 6 || a->N <= 0) {
    fprintf(stderr, "** monolis_b200: unsupported matrix (N=%d, NDOF=%d)\n", a->N, a->NDOF);
    return mb::kBadInput;
  }
  if (I[MONOLIS_B200_PRM_I_CHECK] == 1) {
    int rc = check_csr(a);
    if (rc) {
      fprintf(stderr, "** monolis_b200: CSR arrays failed validation\n");
      return rc;
    }
  }
  // device-assembled values stay until the host changes the matrix
  const bool keep = I[MONOLIS_B200_PRM_I_MATRIX_CACHE] == 1 || s->device_values;
  const bool cached = keep && s->prepared && s->key_index == a->CSR.index &&
                      s->key_item == a->CSR.item && s->key_val == a->R.A && s->key_N == a->N &&
                      s->key_ndof == a->NDOF && s->key_version == I[MONOLIS_B200_PRM_I_MATRIX_VERSION];
  cudaStream_t st = ctx().stream;
  if (t_h2d) *t_h2d = 0.0;
  if (!cached) {
    s->prepared = false;
    s->device_values = false;
    int rc = mb::sell_build(s->A, a->CSR.index, a->CSR.item, a->R.A, a->N, a->NDOF, st, t_h2d);
    if (rc) return rc;
    s->key_index = a->CSR.index;
    s->key_item = a->CSR.item;
    s->key_val = a->R.A;
    s->key_N = a->N;
    s->key_ndof = a->NDOF;
    s->key_version = I[MONOLIS_B200_PRM_I_MATRIX_VERSION];
    s->prepared = true;
    s->build_id++;
  }
  if (need_diag && !s->A.have_alu) {
    int rc = mb::diag_setup(s->A, st);
    if (rc) return rc;
  }
  if (need_fp32 && !s->A.have_val32) {
    int rc = mb::sell_make_fp32(s->A, st);
    if (rc) return rc;
  }
  m->prm.Iarray[MONOLIS_B200_PRM_I_UNROLL_FP64] = s->A.u64;
  m->prm.Iarray[MONOLIS_B200_PRM_I_UNROLL_FP32] = s->A.have_val32 ? s->A.u32 : 0;
  m->prm.Iarray[MONOLIS_B200_PRM_I_WIDE_SLICES_FP64] = (int)s->A.wide64;
  m->prm.Iarray[MONOLIS_B200_PRM_I_WIDE_SLICES_FP32] = s->A.have_val32 ? (int)s->A.wide32 : 0;
  m->prm.Iarray[MONOLIS_B200_PRM_I_UNIFORM_SLICES_FP64] = (int)s->A.uniform64;
  m->prm.Iarray[MONOLIS_B200_PRM_I_UNIFORM_SLICES_FP32] = s->A.have_val32 ? (int)s->A.uniform32 : 0;
  m->prm.Rarray[MONOLIS_B200_PRM_R_SPMV_BYTES_FP64] = s->A.bytes64;
  m->prm.Rarray[MONOLIS_B200_PRM_R_SPMV_BYTES_FP32] = s->A.have_val32 ? s->A.bytes32 : 0.0;
  return mb::kOk;
}

// A^T of the prepared matrix (rebuilt whenever A was), with its DIAG factors
// and FP32 copies as asked.
int prepare_transpose(MONOLIS* m, DevState* s, bool need_diag, bool need_fp32) {
  MONOLIS_MAT* a = &m->mat;
  if (a->N != a->NP) {
    fprintf(stderr, "** monolis_b200: transpose needs N == NP (one rank)\n");
    return mb::kBadInput;
  }
  cudaStream_t st = ctx().stream;
  if (s->at_build_id != s->build_id) {
    const int* ci = a->CSC.index;
    const int* cit = a->CSC.item;
    const int* cp = a->CSC.perm;
    std::vector<int> bi, bit, bp;
    if (!ci || !cit || !cp) {
      const int nz = a->CSR.index[a->N];
      bi.resize((size_t)a->N + 1);
      bit.resize((size_t)nz);
      bp.resize((size_t)nz);
      monolis_get_CSC_format(a->N, a->NP, nz, a->CSR.index, a->CSR.item, bi.data(), bit.data(), bp.data());
      ci = bi.data();
      cit = bit.data();
      cp = bp.data();
    }
    int rc = mb::sell_build_transpose(s->AT, s->A, ci, cit, cp, st);
    if (rc) return rc;
    s->at_build_id = s->build_id;
  }
  if (need_diag && !s->AT.have_alu) {
    int rc = mb::diag_setup(s->AT, st);
    if (rc) return rc;
  }
  if (need_fp32 && !s->AT.have_val32) {
    int rc = mb::sell_make_fp32(s->AT, st);
    if (rc) return rc;
  }
  return mb::kOk;
}

const char* str_iter(int mth) {
  static const char* names[] = {"CG", "GropCG", "PipeCG", "PipeCR", "BiCGSTAB", "PipeBiCGSTAB",
                                "BiCGSTAB_noprec", "PipeBiCGSTAB_noprec", "BiCGSTAB_N128", "SOR",
                                "BiCGSAFE", "IDR(s)", "COCG"};
  return (mth >= 1 && mth <= 13) ? names[mth - 1] : "?";
}
const char* str_prec(int p) {
  static const char* names[] = {"None", "Diag", "SOR", "LU", "MUMPS", "MUMPSL"};
  return (p >= 0 && p <= 5) ? names[p] : "?";
}

// Solve with device b/x already resident; prints and fills prm like
// src/solver/solver.f90:77-185 + src/define/def_solver_prm.f90:255-355.
int solve_resident(MONOLIS* m, DevState* s, mb::SellMatrix& A, const double* d_b, double* d_x, double t_start,
                   double t_prep, double t_h2d, const mb::ShardPlan* shard = nullptr) {
  int* I = m->prm.Iarray;
  double* R = m->prm.Rarray;
  mb::SolveParams p{};
  // BiCGSTAB_N128 (src/iterative/BiCGSTAB_N128.f90) is BiCGSTAB with
  // double-double dot products; the device FP64 BiCGSTAB sums every dot
  // product in double-double already
  p.method = I[MONOLIS_PRM_I_METHOD] == MONOLIS_ITER_BICGSTAB_N128 ? MONOLIS_ITER_BICGSTAB : I[MONOLIS_PRM_I_METHOD];
  p.precond = I[MONOLIS_PRM_I_PRECOND];
  p.max_iter = I[MONOLIS_PRM_I_MAX_ITER];
  p.tol = R[MONOLIS_PRM_R_TOL];
  p.init_x = I[MONOLIS_PRM_I_IS_INIT_X] == MONOLIS_I_TRUE;
  p.precision = I[MONOLIS_B200_PRM_I_PRECISION];
  p.delta = R[MONOLIS_B200_PRM_R_REFRESH_DELTA];
  p.refresh_period = I[MONOLIS_B200_PRM_I_REFRESH_PERIOD];
  p.batch = I[MONOLIS_B200_PRM_I_BATCH];
  p.iter_rr = I[MONOLIS_B200_PRM_I_ITER_RR];
  p.timers = I[MONOLIS_B200_PRM_I_KERNEL_TIMERS] == 1;
  p.use_graph = 1;
  p.shard = shard;
  p.np_rows = m->mat.NP;
  if (I[MONOLIS_PRM_I_SHOW_SUMMARY] == MONOLIS_I_TRUE)
    printf("** MONOLIS solver: %s, prec: %s\n", str_iter(p.method), str_prec(p.precond));
  const bool log = I[MONOLIS_PRM_I_SHOW_ITERLOG] == MONOLIS_I_TRUE;
  std::vector<double> hist;
  if (log) hist.assign((size_t)std::max(p.max_iter, 0) + 2, 0.0);
  mb::SolveResult res;
  int rc = mb::solve_device(A, s->sc, p, d_b, d_x, res, log ? hist.data() : nullptr, ctx().stream);
  if (rc) {
    I[MONOLIS_PRM_I_IERR] = rc;
    return rc;
  }
  if (log)
    for (int it = 1; it <= res.iter; it++) printf("%7d%16.6E\n", it, hist[it]);
  if (res.iter > 0) {
    I[MONOLIS_PRM_I_CUR_ITER] = res.iter;
    R[MONOLIS_PRM_R_CUR_RESID] = res.resid;
  }
  I[MONOLIS_PRM_I_IERR] = res.status;
  I[MONOLIS_B200_PRM_I_N_REFINE] = res.n_refine;
  I[MONOLIS_B200_PRM_I_LAUNCHES] = (int)std::min<long long>(res.launches, 2147483647LL);
  R[MONOLIS_R_TIME_PREP] = t_prep;
  R[MONOLIS_B200_PRM_R_TIME_H2D] = t_h2d;
  R[MONOLIS_B200_PRM_R_TIME_LOOP] = res.t_loop;
  // fused kernels: SpMV time = SpMV kernels (with their fused dots), precond
  // time = update kernels that apply M^-1 (with their AXPYs and dots), inner
  // product time = the remaining vector kernels; filled in timing mode only
  R[MONOLIS_R_TIME_SPMV] = res.t_kind[0];
  R[MONOLIS_R_TIME_DOTP] = res.t_kind[1];
  R[MONOLIS_R_TIME_PREC] = res.t_kind[2];
  for (int k = 0; k < 8; k++)
    R[MONOLIS_B200_PRM_R_TIME_KERNEL + k] = k < (int)res.kernel_time.size() ? res.kernel_time[k] : 0.0;
  R[MONOLIS_R_TIME_COMM_DOTP] = R[MONOLIS_R_TIME_COMM_SPMV] = 0.0;
  R[MONOLIS_R_TIME_SOL] = now_sec() - t_start;
  return mb::kOk;
}

void print_summary(MONOLIS* m) {
  const int* I = m->prm.Iarray;
  const double* R = m->prm.Rarray;
  if (I[MONOLIS_PRM_I_SHOW_SUMMARY] == MONOLIS_I_TRUE) {
    printf("** MONOLIS converge iter:%10d\n", I[MONOLIS_PRM_I_CUR_ITER]);
    printf("** MONOLIS rel. residual:%10.3E\n", R[MONOLIS_PRM_R_CUR_RESID]);
  }
  if (I[MONOLIS_PRM_I_SHOW_SUMMARY] == MONOLIS_I_TRUE || I[MONOLIS_PRM_I_SHOW_TIME] == MONOLIS_I_TRUE)
    printf("** MONOLIS solution time:%10.3E\n", R[MONOLIS_R_TIME_SOL]);
  if (I[MONOLIS_PRM_I_SHOW_TIME] == MONOLIS_I_TRUE) {
    printf(" - solution/prepost time:%10.3E\n", R[MONOLIS_R_TIME_PREP]);
    printf(" - solution/SpMV    time:%10.3E\n", R[MONOLIS_R_TIME_SPMV]);
    printf(" - solution/inner p time:%10.3E\n", R[MONOLIS_R_TIME_DOTP]);
    printf(" - solution/precond time:%10.3E\n", R[MONOLIS_R_TIME_PREC]);
    printf(" - (comm time/inner p)  :%10.3E\n", R[MONOLIS_R_TIME_COMM_DOTP]);
    printf(" - (comm time/spmv)     :%10.3E\n", R[MONOLIS_R_TIME_COMM_SPMV]);
  }
  fflush(stdout);
}

bool method_supported(const MONOLIS* m) {
  const int mth = m->prm.Iarray[MONOLIS_PRM_I_METHOD];
  const int pc = m->prm.Iarray[MONOLIS_PRM_I_PRECOND];
  if (mth != MONOLIS_ITER_CG && mth != MONOLIS_ITER_BICGSTAB && mth != MONOLIS_ITER_PIPECG &&
      mth != MONOLIS_ITER_GROPCG && mth != MONOLIS_ITER_BICGSTAB_N128) {
    fprintf(stderr,
            "** monolis_b200: solver %s is not provided by this library (CG, GropCG, PipeCG, BiCGSTAB, "
            "BiCGSTAB_N128)\n",
            str_iter(mth));
    return false;
  }
  if ((mth == MONOLIS_ITER_PIPECG || mth == MONOLIS_ITER_GROPCG || mth == MONOLIS_ITER_BICGSTAB_N128) &&
      m->prm.Iarray[MONOLIS_B200_PRM_I_PRECISION] != 0) {
    fprintf(stderr, "** monolis_b200: %s runs in FP64 (MONOLIS_B200_PRECISION_FP64)\n", str_iter(mth));
    return false;
  }
  if (pc != MONOLIS_PREC_NONE && pc != MONOLIS_PREC_DIAG) {
    fprintf(stderr, "** monolis_b200: preconditioner %s is not provided by this library (None, Diag)\n",
            str_prec(pc));
    return false;
  }
  return true;
}

}  // namespace

extern "C" {

// ---- monolis_utils subset ----
void monolis_com_initialize_by_self(MONOLIS_COM* com) {
  memset(com, 0, sizeof(*com));
  com->comm_size = 1;
  com->recv_index = halloc<int>(1);
  com->send_index = halloc<int>(1);
}
void monolis_com_finalize(MONOLIS_COM* com) {
  hfree(&com->recv_neib_pe); hfree(&com->recv_index); hfree(&com->recv_item);
  hfree(&com->send_neib_pe); hfree(&com->send_index); hfree(&com->send_item);
  memset(com, 0, sizeof(*com));
}

// ---- init / finalize (wrapper/define/monolis_def_struc_c.c, monolis_def_mat_c.c,
//      monolis_def_solver_prm_c.c) ----
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
  prm->Iarray[MONOLIS_PRM_I_IS_SYM_MATRIX] = MONOLIS_I_FALSE;
  prm->Iarray[MONOLIS_PRM_I_IS_DEBUG] = MONOLIS_I_FALSE;
  prm->Iarray[MONOLIS_PRM_I_IS_MEASUREMENT] = MONOLIS_I_FALSE;
  prm->Iarray[MONOLIS_PRM_I_IS_CHECK_DIAG] = MONOLIS_I_FALSE;
  prm->Iarray[MONOLIS_PRM_I_IS_PREC_STORED] = MONOLIS_I_FALSE;
  prm->Iarray[MONOLIS_PRM_I_IS_ERROR_ABORT] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_SHOW_ITERLOG] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_SHOW_TIME] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_SHOW_SUMMARY] = MONOLIS_I_TRUE;
  prm->Iarray[MONOLIS_PRM_I_SHOW_TIME_STATISTICS] = MONOLIS_I_FALSE;
  prm->Iarray[MONOLIS_PRM_I_IDRS_DIM] = 4;
  prm->Rarray[MONOLIS_PRM_R_TOL] = 1.0e-8;
}
void monolis_prm_finalize(MONOLIS_PRM* prm) {
  for (int i = 0; i < MONOLIS_PRM_IARRAY_SIZE; ++i) prm->Iarray[i] = 0;
  for (int i = 0; i < MONOLIS_PRM_RARRAY_SIZE; ++i) prm->Rarray[i] = 0.0;
}
void monolis_mat_initialize(MONOLIS_MAT* mat) { memset(mat, 0, sizeof(*mat)); }
void monolis_mat_finalize(MONOLIS_MAT* mat) {
  hfree(&mat->n_dof_list); hfree(&mat->n_dof_index); hfree(&mat->n_dof_index2);
  hfree(&mat->R.A); hfree(&mat->R.U); hfree(&mat->R.D); hfree(&mat->R.L); hfree(&mat->R.X); hfree(&mat->R.B);
  hfree(&mat->SCSR.indexU); hfree(&mat->SCSR.indexL); hfree(&mat->SCSR.itemU); hfree(&mat->SCSR.itemL);
  hfree(&mat->CSR.index); hfree(&mat->CSR.item);
  hfree(&mat->CSC.index); hfree(&mat->CSC.item); hfree(&mat->CSC.perm);
  memset(mat, 0, sizeof(*mat));
}
void monolis_initialize(MONOLIS* m) {
  monolis_prm_initialize(&m->prm);
  monolis_mat_initialize(&m->mat);
  monolis_mat_initialize(&m->prec);
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  state_release(m);
}
void monolis_finalize(MONOLIS* m) {
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    state_release(m);
  }
  monolis_prm_finalize(&m->prm);
  monolis_mat_finalize(&m->mat);
  monolis_mat_finalize(&m->prec);
}
void monolis_get_vec_size(int N, int NP, int NDOF, int NZ, int* n_dof_index, int* n_dof_index2, int* N_size,
                          int* NP_size, int* NZ_size) {
  if (NDOF == -1) {
    *N_size = n_dof_index[N]; *NP_size = n_dof_index[NP]; *NZ_size = n_dof_index2[NZ];
  } else {
    *N_size = N * NDOF; *NP_size = NP * NDOF; *NZ_size = NZ * NDOF * NDOF;
  }
}

// ---- parameters (wrapper/define/monolis_def_solver_prm_util_c.c) ----
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
// src/matrix/spmat_nzpattern_util.f90:162-218: column counts, offsets, then
// rows visited in ascending order (so each column's rows come out sorted).
void monolis_get_CSC_format(int NC, int NR, int NZ, int* index, int* item, int* indexR, int* itemR, int* permR) {
  (void)NZ;
  std::vector<int> cnt(NR + 1, 0);
  for (int i = 0; i < NC; i++)
    for (int j = index[i]; j < index[i + 1]; j++) cnt[item[j] - 1]++;
  indexR[0] = 0;
  for (int i = 0; i < NR; i++) indexR[i + 1] = indexR[i] + cnt[i];
  std::fill(cnt.begin(), cnt.end(), 0);
  for (int i = 0; i < NC; i++)
    for (int j = index[i]; j < index[i + 1]; j++) {
      const int c = item[j] - 1;
      const int p = indexR[c] + cnt[c]++;
      itemR[p] = i + 1;
      permR[p] = j + 1;
    }
}

void monolis_get_nonzero_pattern_by_simple_mesh_R(MONOLIS* m, int n_node, int n_base, int n_dof, int n_elem,
                                                  int** elem) {
  std::vector<int> flat((size_t)n_elem * n_base);
  for (int e = 0; e < n_elem; e++)
    for (int a = 0; a < n_base; a++) flat[(size_t)e * n_base + a] = elem[e][a];
  pattern_from_mesh(m, n_node, n_base, n_dof, n_elem, flat.data());
}

int monolis_b200_get_nonzero_pattern_by_simple_mesh_flat_R(MONOLIS* m, int n_node, int n_base, int n_dof,
                                                          int n_elem, const int* elem) {
  for (long long k = 0; k < (long long)n_elem * n_base; k++)
    if (elem[k] < 0 || elem[k] >= n_node) return MONOLIS_B200_BAD_INPUT;
  pattern_from_mesh(m, n_node, n_base, n_dof, n_elem, elem);
  return MONOLIS_B200_OK;
}

void monolis_get_nonzero_pattern_by_connectivity_R(MONOLIS* m, int n_node, int n_dof, int n_elem, int* conn_index,
                                                   int* conn_item) {
  // element e spans conn_item[conn_index[e] .. conn_index[e+1]); expand to
  // fixed-width rows padded with the element's first node
  int wmax = 0;
  for (int e = 0; e < n_elem; e++) wmax = std::max(wmax, conn_index[e + 1] - conn_index[e]);
  std::vector<int> flat((size_t)n_elem * std::max(wmax, 1));
  for (int e = 0; e < n_elem; e++)
    for (int a = 0; a < wmax; a++) {
      const int k = conn_index[e] + a;
      flat[(size_t)e * wmax + a] = k < conn_index[e + 1] ? conn_item[k] : conn_item[conn_index[e]];
    }
  pattern_from_mesh(m, n_node, wmax, n_dof, n_elem, flat.data());
}

void monolis_get_nonzero_pattern_by_nodal_graph_R(MONOLIS* m, int n_node, int n_dof, int* index, int* item) {
  std::vector<int> rowlen(n_node);
  for (int i = 0; i < n_node; i++) rowlen[i] = index[i + 1] - index[i] + 1;
  auto row_of = [&](int i, std::vector<int>& buf) {
    buf.clear();
    buf.push_back(i);
    for (int k = index[i]; k < index[i + 1]; k++) buf.push_back(item[k]);
    std::sort(buf.begin(), buf.end());
  };
  build_csr_from_rows(m, n_node, n_dof, rowlen, row_of);
}

// ---- assembly (wrapper/matrix/monolis_spmat_handler_c.c) ----
void monolis_set_scalar_to_sparse_matrix_R(MONOLIS* m, int i, int j, int si, int sj, double val) {
  double* p = scalar_slot(m, i, j, si, sj);
  if (!p) error_stop("matrix assemble: entry not in the nonzero pattern");
  *p = val;
  bump_version(m);
}
void monolis_add_scalar_to_sparse_matrix_R(MONOLIS* m, int i, int j, int si, int sj, double val) {
  double* p = scalar_slot(m, i, j, si, sj);
  if (!p) error_stop("matrix assemble: entry not in the nonzero pattern");
  *p = *p + val;
  bump_version(m);
}
void monolis_get_scalar_from_sparse_matrix_R(MONOLIS* m, int i, int j, int si, int sj, double* val, bool* is_find) {
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
  add_element(&m->mat, n_base, n_base, conn, conn, v.data(), 1.0, false, 0, m->mat.NP);
  bump_version(m);
}
void monolis_add_matrix_to_sparse_matrix_offdiag_R(MONOLIS* m, int n1, int n2, int* c1, int* c2, double** val) {
  int r = 0, c = 0;
  for (int i = 0; i < n1; i++) r += m->mat.n_dof_index[c1[i] + 1] - m->mat.n_dof_index[c1[i]];
  for (int i = 0; i < n2; i++) c += m->mat.n_dof_index[c2[i] + 1] - m->mat.n_dof_index[c2[i]];
  std::vector<double> v((size_t)r * c);
  for (int i = 0; i < r; i++)
    for (int j = 0; j < c; j++) v[(size_t)i * c + j] = val[i][j];
  add_element(&m->mat, n1, n2, c1, c2, v.data(), 1.0, false, 0, m->mat.NP);
  bump_version(m);
}

// Rows are split between threads; each thread walks all elements in order and
// adds only the blocks of its own rows, so every entry receives its
// contributions in element order (bit-identical to the serial loop).
int monolis_b200_add_elements_R(MONOLIS* m, int n_elem, int n_base, const int* elem, const double* val,
                                long long val_stride, const double* scale) {
  MONOLIS_MAT* a = &m->mat;
  if (!a->CSR.index || !a->R.A) return MONOLIS_B200_BAD_INPUT;
  for (long long k = 0; k < (long long)n_elem * n_base; k++)
    if (elem[k] < 0 || elem[k] >= a->NP) return MONOLIS_B200_BAD_INPUT;
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  const int NP = a->NP;
#pragma omp parallel num_threads(nthreads)
  {
    int tid = 0, nt = 1;
#ifdef _OPENMP
    tid = omp_get_thread_num();
    nt = omp_get_num_threads();
#endif
    const int lo = (int)((long long)NP * tid / nt), hi = (int)((long long)NP * (tid + 1) / nt);
    for (int e = 0; e < n_elem; e++) {
      const int* en = elem + (long long)e * n_base;
      bool mine = false;
      for (int q = 0; q < n_base; q++) mine |= (en[q] >= lo && en[q] < hi);
      if (!mine) continue;
      add_element(a, n_base, n_base, en, en, val + (long long)e * val_stride, scale ? scale[e] : 1.0,
                  scale != nullptr, lo, hi);
    }
  }
  bump_version(m);
  return MONOLIS_B200_OK;
}

void monolis_set_matrix_BCSR_R(MONOLIS* m, int n, int np, int n_dof, int nz, double* A, int* index, int* item) {
  MONOLIS_MAT* a = &m->mat;
  a->N = n; a->NP = np; a->NDOF = n_dof;
  a->CSR.index = halloc<int>(np + 1);
  a->CSR.item = halloc<int>(nz);
  a->R.A = halloc<double>((long long)n_dof * n_dof * nz);
  a->R.X = halloc<double>((long long)n_dof * np);
  a->R.B = halloc<double>((long long)n_dof * np);
  for (int i = 0; i < np + 1; i++) a->CSR.index[i] = index[i];
  for (int i = 0; i < nz; i++) a->CSR.item[i] = item[i] + 1;
  memcpy(a->R.A, A, sizeof(double) * (size_t)n_dof * n_dof * nz);
  a->CSC.index = halloc<int>(np + 1);
  a->CSC.item = halloc<int>(nz);
  a->CSC.perm = halloc<int>(nz);
  monolis_get_CSC_format(n, np, nz, a->CSR.index, a->CSR.item, a->CSC.index, a->CSC.item, a->CSC.perm);
  a->n_dof_list = halloc<int>(np);
  a->n_dof_index = halloc<int>(np + 1);
  a->n_dof_index2 = halloc<int>(nz + 1);
  for (int i = 0; i < np; i++) a->n_dof_list[i] = n_dof;
  for (int i = 0; i < np; i++) a->n_dof_index[i + 1] = a->n_dof_index[i] + n_dof;
  for (int j = 0; j < nz; j++) a->n_dof_index2[j + 1] = a->n_dof_index2[j] + n_dof * n_dof;
  bump_version(m);
}

// src/matrix/spmat_handler_util.f90:604-677 with 0-based node_id / n_dof_bc:
// column node_id*ndof+bc is moved to the RHS and zeroed (through the CSC
// permutation), the row is zeroed, the diagonal set to 1, B = val.
void monolis_set_Dirichlet_bc_R(MONOLIS* m, double* B, int node_id, int ndof_bc, double val) {
  MONOLIS_MAT* a = &m->mat;
  const int* ndi = a->n_dof_index;
  const int* nd2 = a->n_dof_index2;
  if (node_id < 0 || node_id >= a->NP) error_stop("set Dirichlet: node id out of range");
  const int ndof1 = ndi[node_id + 1] - ndi[node_id];
  if (ndof_bc < 0 || ndof_bc >= ndof1) error_stop("submatrix access out of range");
  for (int j = a->CSC.index[node_id]; j < a->CSC.index[node_id + 1]; j++) {
    const int jn = a->CSC.item[j] - 1;
    const int kn = a->CSC.perm[j] - 1;
    const int ndof2 = ndi[jn + 1] - ndi[jn];
    for (int k = 0; k < ndof2; k++) {
      const long long mm = (long long)nd2[kn] + (long long)ndof1 * k + ndof_bc;
      const long long n = (long long)ndi[jn] + k;
      B[n] = B[n] - val * a->R.A[mm];
      a->R.A[mm] = 0.0;
    }
  }
  bool is_add = false;
  for (int j = a->CSR.index[node_id]; j < a->CSR.index[node_id + 1]; j++) {
    const int jn = a->CSR.item[j] - 1;
    const int ndof2 = ndi[jn + 1] - ndi[jn];
    for (int k = 0; k < ndof2; k++) a->R.A[(long long)nd2[j] + (long long)ndof2 * ndof_bc + k] = 0.0;
    if (jn == node_id) {
      a->R.A[(long long)nd2[j] + (long long)(ndof2 + 1) * ndof_bc] = 1.0;
      is_add = true;
    }
  }
  if (!is_add) error_stop("set Dirichlet: diagonal block not found");
  B[ndi[node_id] + ndof_bc] = val;
  bump_version(m);
}

// ---- linear algebra on the device ----
void monolis_matvec_product_R(MONOLIS* m, MONOLIS_COM* com, double* x, double* y) {
  if (com && com->comm_size > 1) error_stop("monolis_b200: one rank per solve in this library");
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) error_stop("monolis_matvec_product_R: no CUDA device");
  DevState* s = state_of(m);
  if (prepare(m, s, false, false, nullptr)) error_stop("monolis_matvec_product_R: device upload failed");
  const size_t n = (size_t)m->mat.N * m->mat.NDOF;
  if (ensure_vec(s, n)) error_stop("monolis_matvec_product_R: device allocation failed");
  cudaStream_t st = ctx().stream;
  cudaMemcpyAsync(s->d_x, x, n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (mb::spmv64(s->A, s->d_x, s->d_y, st)) error_stop("monolis_matvec_product_R: kernel failed");
  cudaMemcpyAsync(y, s->d_y, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) error_stop("monolis_matvec_product_R: CUDA error");
}

void monolis_inner_product_R(MONOLIS* m, MONOLIS_COM* com, int n_dof, double* x, double* y, double* sum) {
  if (com && com->comm_size > 1) error_stop("monolis_b200: one rank per solve in this library");
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) error_stop("monolis_inner_product_R: no CUDA device");
  DevState* s = state_of(m);
  const size_t n = (size_t)m->mat.N * n_dof;
  if (ensure_vec(s, n)) error_stop("monolis_inner_product_R: device allocation failed");
  cudaStream_t st = ctx().stream;
  cudaMemcpyAsync(s->d_x, x, n * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->d_y, y, n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (mb::dot64((long long)n, s->d_x, s->d_y, s->d_b, s->sc, st)) error_stop("monolis_inner_product_R: kernel failed");
  cudaMemcpyAsync(sum, s->d_b, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) error_stop("monolis_inner_product_R: CUDA error");
}

}  // extern "C"

// The NCCL communicator attached to com (monolis_b200_com_init_nccl), or null.
static void* nccl_comm_of(MONOLIS_COM* com) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  auto it = com ? nccl_comms().find(com) : nccl_comms().end();
  return it != nccl_comms().end() ? it->second : nullptr;
}

// Methods and precisions of the multi-rank solve.
static bool sharded_supported(const MONOLIS* m) {
  const int* I = m->prm.Iarray;
  const int mth = I[MONOLIS_PRM_I_METHOD];
  // BiCGSTAB_N128 runs as BiCGSTAB (its dot products are double-double on
  // every rank; the ranks' partial sums are rounded before the all-reduce)
  const bool bicg = mth == MONOLIS_ITER_BICGSTAB || mth == MONOLIS_ITER_BICGSTAB_N128;
  if ((mth != MONOLIS_ITER_CG && !bicg && mth != MONOLIS_ITER_PIPECG && mth != MONOLIS_ITER_GROPCG) ||
      (I[MONOLIS_B200_PRM_I_PRECISION] != 0 && mth != MONOLIS_ITER_CG && !bicg)) {
    fprintf(stderr,
            "** monolis_b200: the multi-rank solve is FP64 (CG, GropCG, PipeCG, BiCGSTAB, BiCGSTAB_N128) or "
            "FP32-refined CG or BiCGSTAB\n");
    return false;
  }
  return true;
}

// Halo plan of the rank-local system from the MONOLIS_COM tables
// (src/linalg/matvec.f90:144 updates the ghost entries through them);
// caller holds g_ctx_mu and has prepared s->A.
static int attach_shard(MONOLIS* m, DevState* s, MONOLIS_COM* com, void* ncomm) {
  mb::ShardTables t;
  t.rank = com->my_rank;
  t.send_pe.assign(com->send_neib_pe, com->send_neib_pe + com->send_n_neib);
  t.send_ptr.assign(com->send_index, com->send_index + com->send_n_neib + 1);
  t.send_item.assign(com->send_item, com->send_item + (com->send_n_neib ? com->send_index[com->send_n_neib] : 0));
  t.recv_pe.assign(com->recv_neib_pe, com->recv_neib_pe + com->recv_n_neib);
  t.recv_ptr.assign(com->recv_index, com->recv_index + com->recv_n_neib + 1);
  t.recv_item.assign(com->recv_item, com->recv_item + (com->recv_n_neib ? com->recv_index[com->recv_n_neib] : 0));
  int rc = mb::shard_setup(s->shard, t, m->mat.NDOF, s->A, ctx().stream);
  s->shard.comm = ncomm;
  return rc;
}

// src/solver/solver.f90:29-49 + wrapper/solver/monolis_solver_c.c:8-60, for A
// or (transpose) A^T.
static int solve_host(MONOLIS* m, MONOLIS_COM* com, double* b, double* x, bool transpose) {
  const double t_start = now_sec();
  int* I = m->prm.Iarray;
  // multi-rank: an NCCL communicator attached with monolis_b200_com_init_nccl
  void* ncomm = nccl_comm_of(com);
  if (com && com->comm_size > 1 && !ncomm) {
    fprintf(stderr, "** monolis_b200: comm_size=%d needs an NCCL communicator (monolis_b200_com_init_nccl)\n",
            com->comm_size);
    I[MONOLIS_PRM_I_IERR] = MONOLIS_B200_BAD_INPUT;
    return MONOLIS_B200_BAD_INPUT;
  }
  const bool sharded = ncomm != nullptr;
  if (sharded && (transpose || !sharded_supported(m))) {
    I[MONOLIS_PRM_I_IERR] = MONOLIS_B200_BAD_INPUT;
    return MONOLIS_B200_BAD_INPUT;
  }
  if (!method_supported(m)) {
    I[MONOLIS_PRM_I_IERR] = MONOLIS_B200_BAD_INPUT;
    return MONOLIS_B200_BAD_INPUT;
  }
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) {
    I[MONOLIS_PRM_I_IERR] = MONOLIS_B200_CUDA_ERROR;
    return MONOLIS_B200_CUDA_ERROR;
  }
  DevState* s = state_of(m);
  const bool mixed = I[MONOLIS_B200_PRM_I_PRECISION] == 1;
  double t_h2d = 0.0;
  const bool diag = I[MONOLIS_PRM_I_PRECOND] == MONOLIS_PREC_DIAG;
  int rc = prepare(m, s, diag && !transpose, mixed && !transpose, &t_h2d);
  if (!rc && transpose) rc = prepare_transpose(m, s, diag, mixed);
  // multi-rank: x and b hold the ghost rows too (NP)
  const size_t n = (size_t)(sharded ? m->mat.NP : m->mat.N) * m->mat.NDOF;
  if (!rc) rc = ensure_vec(s, n);
  if (!rc && sharded) rc = attach_shard(m, s, com, ncomm);
  if (rc) {
    I[MONOLIS_PRM_I_IERR] = rc;
    return rc;
  }
  cudaStream_t st = ctx().stream;
  // B and X are copied into the struct's own arrays first, as the reference
  // does (src/define/def_mat.f90:579-635), then uploaded.
  if (m->mat.R.B && m->mat.R.B != b) memcpy(m->mat.R.B, b, n * sizeof(double));
  if (m->mat.R.X && m->mat.R.X != x) memcpy(m->mat.R.X, x, n * sizeof(double));
  const double t1 = now_sec();
  cudaMemcpyAsync(s->d_b, b, n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (I[MONOLIS_PRM_I_IS_INIT_X] != MONOLIS_I_TRUE)
    cudaMemcpyAsync(s->d_x, x, n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    I[MONOLIS_PRM_I_IERR] = MONOLIS_B200_CUDA_ERROR;
    return MONOLIS_B200_CUDA_ERROR;
  }
  t_h2d += now_sec() - t1;
  const double t_prep = now_sec() - t_start;
  rc = solve_resident(m, s, transpose ? s->AT : s->A, s->d_b, s->d_x, t_start, t_prep, t_h2d,
                      sharded ? &s->shard : nullptr);
  if (rc) return rc;
  const double t2 = now_sec();
  cudaMemcpyAsync(x, s->d_x, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (m->mat.R.X && m->mat.R.X != x) memcpy(m->mat.R.X, x, n * sizeof(double));
  m->prm.Rarray[MONOLIS_B200_PRM_R_TIME_D2H] = now_sec() - t2;
  m->prm.Rarray[MONOLIS_R_TIME_SOL] = now_sec() - t_start;
  print_summary(m);
  if (I[MONOLIS_PRM_I_IERR] == MONOLIS_B200_MAXITER && I[MONOLIS_PRM_I_IS_MEASUREMENT] == MONOLIS_I_FALSE &&
      I[MONOLIS_PRM_I_IS_ERROR_ABORT] == MONOLIS_I_TRUE)
    error_stop("reached the maximum number of iterations");  // src/linalg/mat_converge.f90:134-140
  return I[MONOLIS_PRM_I_IERR];
}

extern "C" {

void monolis_solve_R(MONOLIS* m, MONOLIS_COM* com, double* b, double* x) { solve_host(m, com, b, x, false); }

int monolis_b200_solve_transpose_R(MONOLIS* m, MONOLIS_COM* com, double* b, double* x) {
  return solve_host(m, com, b, x, true);
}


// ---- multi-rank communicator ----
int monolis_b200_nccl_unique_id(void* id128) {
  if (!id128) return MONOLIS_B200_BAD_INPUT;
  return mb::shard_unique_id(id128);
}

int monolis_b200_com_init_nccl(MONOLIS_COM* com, const void* id128, int rank, int size) {
  if (!com || !id128 || size < 1 || rank < 0 || rank >= size) return MONOLIS_B200_BAD_INPUT;
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  void* c = nullptr;
  int rc = mb::shard_comm_create(&c, id128, rank, size);
  if (rc) return rc;
  auto& reg = nccl_comms();
  auto it = reg.find(com);
  if (it != reg.end()) mb::shard_comm_destroy(it->second);
  reg[com] = c;
  com->my_rank = rank;
  com->comm_size = size;
  return MONOLIS_B200_OK;
}

void monolis_b200_com_finalize_nccl(MONOLIS_COM* com) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  auto& reg = nccl_comms();
  auto it = reg.find(com);
  if (it == reg.end()) return;
  if (ctx().init) cudaStreamSynchronize(ctx().stream);
  mb::shard_comm_destroy(it->second);
  reg.erase(it);
}

// ---- monolis_b200 extensions ----
int monolis_b200_set_precision(MONOLIS* m, int precision) {
  if (precision != 0 && precision != 1) return MONOLIS_B200_BAD_INPUT;
  m->prm.Iarray[MONOLIS_B200_PRM_I_PRECISION] = precision;
  return MONOLIS_B200_OK;
}
void monolis_b200_set_matrix_cache(MONOLIS* m, bool enable) {
  m->prm.Iarray[MONOLIS_B200_PRM_I_MATRIX_CACHE] = enable ? 1 : 0;
}
void monolis_b200_matrix_changed(MONOLIS* m) { bump_version(m); }

void* monolis_b200_stream(void) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return nullptr;
  return (void*)ctx().stream;
}

int monolis_b200_device_prepare(MONOLIS* m) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  const int* I = m->prm.Iarray;
  int rc = prepare(m, s, I[MONOLIS_PRM_I_PRECOND] == MONOLIS_PREC_DIAG, I[MONOLIS_B200_PRM_I_PRECISION] == 1,
                   &m->prm.Rarray[MONOLIS_B200_PRM_R_TIME_H2D]);
  if (rc) return rc;
  // keep the device copy for the device entry points
  s->key_version = I[MONOLIS_B200_PRM_I_MATRIX_VERSION];
  if (cudaStreamSynchronize(ctx().stream) != cudaSuccess) return MONOLIS_B200_CUDA_ERROR;
  return MONOLIS_B200_OK;
}

int monolis_b200_device_solve_R(MONOLIS* m, const double* d_b, double* d_x) {
  const double t_start = now_sec();
  if (!method_supported(m)) return MONOLIS_B200_BAD_INPUT;
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared) return MONOLIS_B200_BAD_INPUT;
  const int* I = m->prm.Iarray;
  if (I[MONOLIS_PRM_I_PRECOND] == MONOLIS_PREC_DIAG && !s->A.have_alu) {
    int rc = mb::diag_setup(s->A, ctx().stream);
    if (rc) return rc;
  }
  int rc = solve_resident(m, s, s->A, d_b, d_x, t_start, 0.0, 0.0);
  if (rc) return rc;
  print_summary(m);
  return m->prm.Iarray[MONOLIS_PRM_I_IERR];
}

int monolis_b200_device_solve_com_R(MONOLIS* m, MONOLIS_COM* com, const double* d_b, double* d_x) {
  const double t_start = now_sec();
  void* ncomm = nccl_comm_of(com);
  if (!ncomm) return monolis_b200_device_solve_R(m, d_b, d_x);
  if (!method_supported(m) || !sharded_supported(m)) return MONOLIS_B200_BAD_INPUT;
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared) return MONOLIS_B200_BAD_INPUT;
  const int* I = m->prm.Iarray;
  if (I[MONOLIS_PRM_I_PRECOND] == MONOLIS_PREC_DIAG && !s->A.have_alu) {
    int rc = mb::diag_setup(s->A, ctx().stream);
    if (rc) return rc;
  }
  int rc = attach_shard(m, s, com, ncomm);
  if (rc) return rc;
  rc = solve_resident(m, s, s->A, d_b, d_x, t_start, 0.0, 0.0, &s->shard);
  if (rc) return rc;
  print_summary(m);
  return m->prm.Iarray[MONOLIS_PRM_I_IERR];
}

int monolis_b200_device_solve_transpose_R(MONOLIS* m, const double* d_b, double* d_x) {
  const double t_start = now_sec();
  if (!method_supported(m)) return MONOLIS_B200_BAD_INPUT;
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared) return MONOLIS_B200_BAD_INPUT;
  const int* I = m->prm.Iarray;
  int rc = prepare_transpose(m, s, I[MONOLIS_PRM_I_PRECOND] == MONOLIS_PREC_DIAG,
                             I[MONOLIS_B200_PRM_I_PRECISION] == 1);
  if (rc) return rc;
  rc = solve_resident(m, s, s->AT, d_b, d_x, t_start, 0.0, 0.0);
  if (rc) return rc;
  print_summary(m);
  return m->prm.Iarray[MONOLIS_PRM_I_IERR];
}

int monolis_b200_device_solve_multi_R(MONOLIS* m, int n_rhs, const double* d_B, double* d_X, int* iter,
                                      double* resid, int* status) {
  int* I = m->prm.Iarray;
  const int mth = I[MONOLIS_PRM_I_METHOD], pc = I[MONOLIS_PRM_I_PRECOND];
  if (mth != MONOLIS_ITER_CG || (pc != MONOLIS_PREC_NONE && pc != MONOLIS_PREC_DIAG) || n_rhs < 1) {
    fprintf(stderr, "** monolis_b200: the many-right-hand-side solver runs CG with None or Diag\n");
    return MONOLIS_B200_BAD_INPUT;
  }
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  const bool mixed = I[MONOLIS_B200_PRM_I_PRECISION] == 1;
  int rc = prepare(m, s, pc == MONOLIS_PREC_DIAG, mixed, nullptr);
  if (rc) return rc;
  if (!s->multi) s->multi = mb::multi_new();
  const double t0 = now_sec();
  rc = mb::multi_solve(s->A, *s->multi, s->build_id, n_rhs, d_B, d_X, mixed ? 1 : 0, pc == MONOLIS_PREC_DIAG ? 1 : 0,
                       m->prm.Rarray[MONOLIS_PRM_R_TOL], I[MONOLIS_PRM_I_MAX_ITER],
                       m->prm.Rarray[MONOLIS_B200_PRM_R_REFRESH_DELTA],
                       (unsigned long long)std::max(I[MONOLIS_B200_PRM_I_WAIT_LIMIT], 0),
                       (unsigned int)std::min(std::max(I[MONOLIS_B200_PRM_I_WAIT_DELAY_US], 0), 1000000) * 1000u,
                       iter, resid, status, ctx().stream);
  m->prm.Rarray[MONOLIS_B200_PRM_R_TIME_LOOP] = now_sec() - t0;
  I[MONOLIS_PRM_I_IERR] = rc;
  return rc;
}

int monolis_b200_solve_multi_R(MONOLIS* m, MONOLIS_COM* com, int n_rhs, double* B, double* X, int* iter,
                               double* resid, int* status) {
  if ((com && com->comm_size > 1) || n_rhs < 1 || !B || !X) return MONOLIS_B200_BAD_INPUT;
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  }
  const size_t n = (size_t)m->mat.N * m->mat.NDOF * n_rhs;
  cudaStream_t st = ctx().stream;
  double *d_B = nullptr, *d_X = nullptr;
  MB_API_CUDA(cudaMalloc((void**)&d_B, n * sizeof(double)));
  if (cudaMalloc((void**)&d_X, n * sizeof(double)) != cudaSuccess) {
    cudaFree(d_B);
    return MONOLIS_B200_CUDA_ERROR;
  }
  int rc = MONOLIS_B200_OK;
  if (cudaMemcpyAsync(d_B, B, n * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
    rc = MONOLIS_B200_CUDA_ERROR;
  if (!rc) rc = monolis_b200_device_solve_multi_R(m, n_rhs, d_B, d_X, iter, resid, status);
  if (!rc && cudaMemcpyAsync(X, d_X, n * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    rc = MONOLIS_B200_CUDA_ERROR;
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = MONOLIS_B200_CUDA_ERROR;
  cudaFree(d_B);
  cudaFree(d_X);
  return rc;
}

// ---- device assembly ----
namespace {
// Device values changed: rebuild the SELL values (FP32 copy, DIAG factors and
// the transpose follow on demand).
int after_device_assembly(MONOLIS* m, DevState* s) {
  int rc = mb::sell_layout(s->A, ctx().stream);
  if (rc) return rc;
  s->device_values = true;
  s->build_id++;
  s->key_version = m->prm.Iarray[MONOLIS_B200_PRM_I_MATRIX_VERSION];
  return MONOLIS_B200_OK;
}
}  // namespace

int monolis_b200_device_clear_matrix(MONOLIS* m) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  int rc = prepare(m, s, false, false, nullptr);
  if (rc) return rc;
  const size_t nv = (size_t)s->A.nz * m->mat.NDOF * m->mat.NDOF;
  MB_API_CUDA(cudaMemsetAsync(s->A.d_csrval, 0, nv * sizeof(double), ctx().stream));
  return after_device_assembly(m, s);
}

int monolis_b200_device_add_elements_R(MONOLIS* m, int n_elem, int n_base, const int* d_elem, const double* d_val,
                                       long long val_stride, const double* d_scale) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  int rc = prepare(m, s, false, false, nullptr);
  if (rc) return rc;
  rc = mb::device_add_elements(s->A, m->mat.NP, n_elem, n_base, d_elem, d_val, val_stride, d_scale, ctx().stream);
  if (rc) return rc;
  return after_device_assembly(m, s);
}

int monolis_b200_device_set_Dirichlet_bc_R(MONOLIS* m, double* d_b, int n_bc, const int* node_id, const int* n_dof_bc,
                                           const double* val) {
  if (n_bc < 0 || (n_bc > 0 && (!node_id || !n_dof_bc || !val))) return MONOLIS_B200_BAD_INPUT;
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  int rc = prepare(m, s, false, false, nullptr);
  if (rc) return rc;
  rc = mb::device_dirichlet(s->A, d_b, n_bc, node_id, n_dof_bc, val, ctx().stream);
  if (rc) return rc;
  return after_device_assembly(m, s);
}

int monolis_b200_device_get_values(MONOLIS* m, double* values) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared) return MONOLIS_B200_BAD_INPUT;
  const size_t nv = (size_t)s->A.nz * s->A.ndof * s->A.ndof;
  MB_API_CUDA(cudaMemcpyAsync(values, s->A.d_csrval, nv * sizeof(double), cudaMemcpyDeviceToHost, ctx().stream));
  MB_API_CUDA(cudaStreamSynchronize(ctx().stream));
  return MONOLIS_B200_OK;
}

int monolis_b200_device_get_diag(MONOLIS* m, double* alu) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared || !s->A.have_alu || !alu) return MONOLIS_B200_BAD_INPUT;
  const int N = s->A.N, nd2 = s->A.ndof * s->A.ndof;
  std::vector<double> dev((size_t)nd2 * N);
  MB_API_CUDA(cudaMemcpyAsync(dev.data(), s->A.d_alu64, dev.size() * sizeof(double), cudaMemcpyDeviceToHost,
                              ctx().stream));
  MB_API_CUDA(cudaStreamSynchronize(ctx().stream));
  // device storage is entry-major (alu[e*N + row]); the reference's is
  // block by block (ALU(nd2*(row-1) + e))
  for (int row = 0; row < N; row++)
    for (int e = 0; e < nd2; e++) alu[(size_t)row * nd2 + e] = dev[(size_t)e * N + row];
  return MONOLIS_B200_OK;
}

int monolis_b200_device_matvec_transpose_R(MONOLIS* m, const double* d_x, double* d_y) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared) return MONOLIS_B200_BAD_INPUT;
  int rc = prepare_transpose(m, s, false, false);
  if (rc) return rc;
  return mb::spmv64(s->AT, d_x, d_y, ctx().stream);
}

int monolis_b200_matvec_transpose_R(MONOLIS* m, MONOLIS_COM* com, double* x, double* y) {
  if (com && com->comm_size > 1) return MONOLIS_B200_BAD_INPUT;
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  int rc = prepare(m, s, false, false, nullptr);
  if (!rc) rc = prepare_transpose(m, s, false, false);
  const size_t n = (size_t)m->mat.N * m->mat.NDOF;
  if (!rc) rc = ensure_vec(s, n);
  if (rc) return rc;
  cudaStream_t st = ctx().stream;
  MB_API_CUDA(cudaMemcpyAsync(s->d_x, x, n * sizeof(double), cudaMemcpyHostToDevice, st));
  rc = mb::spmv64(s->AT, s->d_x, s->d_y, st);
  if (rc) return rc;
  MB_API_CUDA(cudaMemcpyAsync(y, s->d_y, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  MB_API_CUDA(cudaStreamSynchronize(st));
  return MONOLIS_B200_OK;
}

int monolis_b200_device_sampled_outer_product_R(MONOLIS* m, const double* d_lambda, const double* d_x, double scale,
                                                double* d_G) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared) return MONOLIS_B200_BAD_INPUT;
  return mb::outer_product64(s->A, d_lambda, d_x, scale, d_G, ctx().stream);
}

int monolis_b200_sampled_outer_product_R(MONOLIS* m, const double* lambda, const double* x, double scale,
                                         double* G) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  int rc = prepare(m, s, false, false, nullptr);
  const size_t n = (size_t)m->mat.N * m->mat.NDOF;
  if (!rc) rc = ensure_vec(s, n);
  if (rc) return rc;
  cudaStream_t st = ctx().stream;
  const size_t ng = (size_t)s->A.nz * m->mat.NDOF * m->mat.NDOF;
  double* d_G = nullptr;
  MB_API_CUDA(cudaMallocAsync((void**)&d_G, ng * sizeof(double) + 16, st));
  MB_API_CUDA(cudaMemcpyAsync(s->d_x, x, n * sizeof(double), cudaMemcpyHostToDevice, st));
  MB_API_CUDA(cudaMemcpyAsync(s->d_y, lambda, n * sizeof(double), cudaMemcpyHostToDevice, st));
  rc = mb::outer_product64(s->A, s->d_y, s->d_x, scale, d_G, st);
  if (!rc && cudaMemcpyAsync(G, d_G, ng * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    rc = MONOLIS_B200_CUDA_ERROR;
  cudaFreeAsync(d_G, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = MONOLIS_B200_CUDA_ERROR;
  return rc;
}

int monolis_b200_device_element_gradient_R(MONOLIS* m, int n_elem, int n_base, const int* d_elem, const double* d_Ke,
                                           long long ke_stride, const double* d_lambda, const double* d_x,
                                           const int* d_fixed_dof, double scale, double* d_grad) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  return mb::element_gradient64(n_elem, n_base, m->mat.NDOF, d_elem, d_Ke, ke_stride, d_lambda, d_x, d_fixed_dof,
                                scale, d_grad, ctx().stream);
}

int monolis_b200_element_gradient_R(MONOLIS* m, int n_elem, int n_base, const int* elem, const double* Ke,
                                    long long ke_stride, const double* lambda, const double* x,
                                    const int* fixed_dof, double scale, double* grad) {
  const MONOLIS_MAT* a = &m->mat;
  if (n_elem < 0 || n_base <= 0 || ke_stride < 0 || a->NDOF <= 0) return MONOLIS_B200_BAD_INPUT;
  for (long long k = 0; k < (long long)n_elem * n_base; k++)
    if (elem[k] < 0 || elem[k] >= a->NP) return MONOLIS_B200_BAD_INPUT;
  if (n_elem == 0) return MONOLIS_B200_OK;
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  cudaStream_t st = ctx().stream;
  const long long nl = (long long)n_base * a->NDOF;
  const size_t n = (size_t)a->NP * a->NDOF;
  const size_t nk = ke_stride == 0 ? (size_t)(nl * nl) : (size_t)(ke_stride * (n_elem - 1) + nl * nl);
  const size_t ne = (size_t)n_elem * n_base;
  // one device buffer: elem | fixed | Ke | lambda | x | grad, 16-byte aligned parts
  auto al = [](size_t b) { return (b + 15) / 16 * 16; };
  const size_t o_fix = al(ne * sizeof(int)), o_ke = o_fix + al(fixed_dof ? n * sizeof(int) : 0);
  const size_t o_l = o_ke + al(nk * sizeof(double)), o_x = o_l + al(n * sizeof(double));
  const size_t o_g = o_x + al(n * sizeof(double)), total = o_g + al((size_t)n_elem * sizeof(double));
  char* buf = nullptr;
  MB_API_CUDA(cudaMallocAsync((void**)&buf, total, st));
  int rc = MONOLIS_B200_OK;
  auto up = [&](size_t off, const void* src, size_t bytes) {
    if (!rc && bytes && cudaMemcpyAsync(buf + off, src, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
      rc = MONOLIS_B200_CUDA_ERROR;
  };
  up(0, elem, ne * sizeof(int));
  if (fixed_dof) up(o_fix, fixed_dof, n * sizeof(int));
  up(o_ke, Ke, nk * sizeof(double));
  up(o_l, lambda, n * sizeof(double));
  up(o_x, x, n * sizeof(double));
  if (!rc)
    rc = mb::element_gradient64(n_elem, n_base, a->NDOF, (const int*)buf, (const double*)(buf + o_ke), ke_stride,
                                (const double*)(buf + o_l), (const double*)(buf + o_x),
                                fixed_dof ? (const int*)(buf + o_fix) : nullptr, scale, (double*)(buf + o_g), st);
  if (!rc && cudaMemcpyAsync(grad, buf + o_g, (size_t)n_elem * sizeof(double), cudaMemcpyDeviceToHost, st) !=
                 cudaSuccess)
    rc = MONOLIS_B200_CUDA_ERROR;
  cudaFreeAsync(buf, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = MONOLIS_B200_CUDA_ERROR;
  return rc;
}

int monolis_b200_device_matvec_R(MONOLIS* m, const double* d_x, double* d_y) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared) return MONOLIS_B200_BAD_INPUT;
  return mb::spmv64(s->A, d_x, d_y, ctx().stream);
}

int monolis_b200_device_matvec_R32(MONOLIS* m, const float* d_x, float* d_y) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (ctx_init()) return MONOLIS_B200_CUDA_ERROR;
  DevState* s = state_of(m);
  if (!s->prepared) return MONOLIS_B200_BAD_INPUT;
  if (!s->A.have_val32) {
    int rc = mb::sell_make_fp32(s->A, ctx().stream);
    if (rc) return rc;
  }
  return mb::spmv32(s->A, d_x, d_y, ctx().stream);
}

int monolis_b200_device_info(MONOLIS* m, long long* nz_blocks, long long* padded_blocks, int* n_slices) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  auto it = ctx().states.find(m);
  if (it == ctx().states.end() || !it->second->prepared) return MONOLIS_B200_BAD_INPUT;
  if (nz_blocks) *nz_blocks = it->second->A.nz;
  if (padded_blocks) *padded_blocks = it->second->A.padded;
  if (n_slices) *n_slices = it->second->A.nslices;
  return MONOLIS_B200_OK;
}

}  // extern "C"
