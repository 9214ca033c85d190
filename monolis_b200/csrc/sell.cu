// sell.cu -- device matrix build (CSR upload -> sliced ELL), DIAG factor
// setup, and the standalone SpMV / inner product / DIAG apply kernels.
#include <cstdio>
#include <cstring>
#include <vector>

#include "spmv.cuh"

namespace mb {

int report_cuda(cudaError_t e, const char* what, const char* file, int line) {
  fprintf(stderr, "** monolis_b200 CUDA error: %s (%s) at %s:%d\n", cudaGetErrorString(e), what, file, line);
  return kCudaError;
}

namespace {

template <class P>
cudaError_t grow(P** p, size_t& cap, size_t need) {
  if (*p && cap >= need) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void**)p, need * sizeof(P) + 16);
  if (e == cudaSuccess) cap = need;
  return e;
}

__global__ void slice_width_kernel(const int* __restrict__ rowptr, int N, int nslices, long long* __restrict__ width) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  int w = 0;
  for (int l = 0; l < kSlice; l++) {
    int r = s * kSlice + l;
    if (r < N) w = max(w, rowptr[r + 1] - rowptr[r]);
  }
  width[s] = (long long)w * kSlice;
}

// One warp per slice: lane l copies row (32s + l) into the slot-major layout.
template <int B>
__global__ void sell_fill_kernel(const int* __restrict__ rowptr, const int* __restrict__ item,
                                 const double* __restrict__ csrval, const long long* __restrict__ slptr,
                                 int N, int nslices, int* __restrict__ col, double* __restrict__ val) {
  constexpr int B2 = B * B;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nslices) return;
  const int row = warp * kSlice + lane;
  const long long base = slptr[warp];
  const int w = (int)((slptr[warp + 1] - base) / kSlice);
  const int len = row < N ? rowptr[row + 1] - rowptr[row] : 0;
  const long long j0 = row < N ? rowptr[row] : 0;
  for (int k = 0; k < w; k++) {
    const long long slot = base + (long long)k * kSlice;
    if (k < len) {
      col[slot + lane] = item[j0 + k] - 1;
#pragma unroll
      for (int e = 0; e < B2; e++) val[(slot * B2) + (long long)e * kSlice + lane] = csrval[(j0 + k) * B2 + e];
    } else {
      col[slot + lane] = row < N ? row : 0;
#pragma unroll
      for (int e = 0; e < B2; e++) val[(slot * B2) + (long long)e * kSlice + lane] = 0.0;
    }
  }
}

__global__ void to_fp32_kernel(const double* __restrict__ a, float* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// Extract the diagonal block of each row and factor it in place without
// pivoting (src/prec/diag/diag_nn.f90:54-78 and diag_33.f90:40-95): a zero
// pivot is replaced by 1, the diagonal holds reciprocal pivots, L below, U
// above. One thread per block row; output is entry-major.
template <int B>
__global__ void diag_setup_kernel(const int* __restrict__ rowptr, const int* __restrict__ item,
                                  const double* __restrict__ csrval, int N, double* __restrict__ alu) {
  constexpr int B2 = B * B;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double LU[B2];
#pragma unroll
  for (int e = 0; e < B2; e++) LU[e] = 0.0;
  bool found = false;
  for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
    if (item[j] - 1 == i) {
#pragma unroll
      for (int e = 0; e < B2; e++) LU[e] = csrval[(long long)j * B2 + e];
      found = true;
    }
  }
  if (found) {
#pragma unroll
    for (int k = 0; k < B; k++) {
      if (LU[k * B + k] == 0.0) LU[k * B + k] = 1.0;
      LU[k * B + k] = 1.0 / LU[k * B + k];
#pragma unroll
      for (int l = k + 1; l < B; l++) {
        LU[l * B + k] = __dmul_rn(LU[l * B + k], LU[k * B + k]);
        double T[B];
#pragma unroll
        for (int j = k + 1; j < B; j++) T[j] = __dsub_rn(LU[l * B + j], __dmul_rn(LU[l * B + k], LU[k * B + j]));
#pragma unroll
        for (int j = k + 1; j < B; j++) LU[l * B + j] = T[j];
      }
    }
  }
#pragma unroll
  for (int e = 0; e < B2; e++) alu[(long long)e * N + i] = LU[e];
}

template <int B, int U, class V, class T>
__global__ void __launch_bounds__(256) spmv_kernel(SellView<V> A, const T* __restrict__ x, T* __restrict__ y) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= A.N) return;
  T acc[B];
  sell_row<B, U, V, T>(A, x, row, acc);
#pragma unroll
  for (int r = 0; r < B; r++) y[(long long)row * B + r] = acc[r];
}

template <class T>
__global__ void dot_kernel(long long n, const T* __restrict__ x, const T* __restrict__ y, double* partials,
                           unsigned int* ticket, double* out) {
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[0] += (double)x[i] * (double)y[i];
  grid_reduce<1>(v, partials, ticket, [&](double* tot) { *out = tot[0]; });
}

template <int B>
__global__ void diag_apply_kernel(const double* __restrict__ alu, int N, const double* __restrict__ x,
                                  double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double t[B];
#pragma unroll
  for (int b = 0; b < B; b++) t[b] = x[(long long)i * B + b];
  diag_row<B, double>(alu, N, i, t);
#pragma unroll
  for (int b = 0; b < B; b++) y[(long long)i * B + b] = t[b];
}

template <class F>
int dispatch_ndof(int ndof, F&& f) {
  switch (ndof) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    default:
      fprintf(stderr, "** monolis_b200: NDOF=%d is not supported on the device (1..6)\n", ndof);
      return kBadInput;
  }
}

}  // namespace

int sell_build(SellMatrix& m, const int* h_index, const int* h_item, const double* h_val, int N, int ndof,
               cudaStream_t s, double* t_h2d) {
  if (N <= 0 || ndof <= 0) return kBadInput;
  const long long nz = h_index[N];
  const int B2 = ndof * ndof;
  const int nslices = (N + kSlice - 1) / kSlice;
  m.N = N;
  m.ndof = ndof;
  m.nz = nz;
  m.nslices = nslices;
  m.have_val32 = m.have_alu = m.have_alu32 = false;
  MB_CUDA_OK(grow(&m.d_rowptr, m.cap_rowptr, (size_t)N + 1));
  MB_CUDA_OK(grow(&m.d_slptr, m.cap_slptr, (size_t)nslices + 1));
  MB_CUDA_OK(grow(&m.d_item, m.cap_item, (size_t)nz));
  MB_CUDA_OK(grow(&m.d_csrval, m.cap_csrval, (size_t)nz * B2));

  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  MB_CUDA_OK(cudaMemcpyAsync(m.d_rowptr, h_index, sizeof(int) * (N + 1), cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(cudaMemcpyAsync(m.d_item, h_item, sizeof(int) * nz, cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(cudaMemcpyAsync(m.d_csrval, h_val, sizeof(double) * nz * B2, cudaMemcpyHostToDevice, s));
  cudaEventRecord(e1, s);

  // slice widths -> prefix on the host (nslices = N/32 values) -> slice pointers
  long long* d_w = nullptr;
  MB_CUDA_OK(cudaMallocAsync((void**)&d_w, sizeof(long long) * nslices, s));
  slice_width_kernel<<<(nslices + 255) / 256, 256, 0, s>>>(m.d_rowptr, N, nslices, d_w);
  std::vector<long long> w(nslices), ptr(nslices + 1);
  MB_CUDA_OK(cudaMemcpyAsync(w.data(), d_w, sizeof(long long) * nslices, cudaMemcpyDeviceToHost, s));
  MB_CUDA_OK(cudaStreamSynchronize(s));
  cudaFreeAsync(d_w, s);
  if (t_h2d) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    *t_h2d = ms * 1e-3;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ptr[0] = 0;
  for (int i = 0; i < nslices; i++) ptr[i + 1] = ptr[i] + w[i];
  m.padded = ptr[nslices];
  MB_CUDA_OK(cudaMemcpyAsync(m.d_slptr, ptr.data(), sizeof(long long) * (nslices + 1), cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(grow(&m.d_col, m.cap_col, (size_t)m.padded));
  MB_CUDA_OK(grow(&m.d_val64, m.cap_val64, (size_t)m.padded * B2));
  const int threads = 256;
  const int blocks = (int)(((long long)nslices * 32 + threads - 1) / threads);
  int rc = dispatch_ndof(ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    sell_fill_kernel<B><<<blocks, threads, 0, s>>>(m.d_rowptr, m.d_item, m.d_csrval, m.d_slptr, N, nslices, m.d_col,
                                                   m.d_val64);
    return kOk;
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

int sell_make_fp32(SellMatrix& m, cudaStream_t s) {
  if (m.have_val32) return kOk;
  const long long n = m.padded * m.ndof * m.ndof;
  MB_CUDA_OK(grow(&m.d_val32, m.cap_val32, (size_t)n));
  to_fp32_kernel<<<148 * 8, 256, 0, s>>>(m.d_val64, m.d_val32, n);
  MB_CUDA_OK(cudaGetLastError());
  m.have_val32 = true;
  if (m.have_alu) {
    const long long na = (long long)m.N * m.ndof * m.ndof;
    MB_CUDA_OK(grow(&m.d_alu32, m.cap_alu32, (size_t)na));
    to_fp32_kernel<<<148 * 8, 256, 0, s>>>(m.d_alu64, m.d_alu32, na);
    MB_CUDA_OK(cudaGetLastError());
    m.have_alu32 = true;
  }
  return kOk;
}

int diag_setup(SellMatrix& m, cudaStream_t s) {
  const long long na = (long long)m.N * m.ndof * m.ndof;
  MB_CUDA_OK(grow(&m.d_alu64, m.cap_alu64, (size_t)na));
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    diag_setup_kernel<B><<<(m.N + 255) / 256, 256, 0, s>>>(m.d_rowptr, m.d_item, m.d_csrval, m.N, m.d_alu64);
    return kOk;
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  m.have_alu = true;
  m.have_alu32 = false;
  if (m.have_val32) {
    MB_CUDA_OK(grow(&m.d_alu32, m.cap_alu32, (size_t)na));
    to_fp32_kernel<<<148 * 8, 256, 0, s>>>(m.d_alu64, m.d_alu32, na);
    MB_CUDA_OK(cudaGetLastError());
    m.have_alu32 = true;
  }
  return kOk;
}

void sell_free(SellMatrix& m) {
  cudaFree(m.d_rowptr);
  cudaFree(m.d_slptr);
  cudaFree(m.d_col);
  cudaFree(m.d_val64);
  cudaFree(m.d_val32);
  cudaFree(m.d_alu64);
  cudaFree(m.d_alu32);
  cudaFree(m.d_item);
  cudaFree(m.d_csrval);
  m = SellMatrix();
}

int spmv64(const SellMatrix& m, const double* x, double* y, cudaStream_t s) {
  SellView<double> A = view_of<double>(m);
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    constexpr int U = B == 1 ? 4 : (B <= 3 ? 2 : 1);
    spmv_kernel<B, U, double, double><<<(m.N + 255) / 256, 256, 0, s>>>(A, x, y);
    return kOk;
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

int spmv32(const SellMatrix& m, const float* x, float* y, cudaStream_t s) {
  if (!m.have_val32) return kBadInput;
  SellView<float> A = view_of<float>(m);
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    constexpr int U = B == 1 ? 4 : (B <= 3 ? 2 : 1);
    spmv_kernel<B, U, float, float><<<(m.N + 255) / 256, 256, 0, s>>>(A, x, y);
    return kOk;
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

int scratch_ensure(Scratch& sc, size_t hist_len) {
  const size_t need = 65536 * 4;
  if (sc.partials_cap < need) {
    if (sc.partials) cudaFree(sc.partials);
    MB_CUDA_OK(cudaMalloc((void**)&sc.partials, need * sizeof(double)));
    sc.partials_cap = need;
  }
  if (!sc.ticket) {
    MB_CUDA_OK(cudaMalloc((void**)&sc.ticket, 64 * sizeof(unsigned int)));
    MB_CUDA_OK(cudaMemset(sc.ticket, 0, 64 * sizeof(unsigned int)));
  }
  if (!sc.st) MB_CUDA_OK(cudaMalloc((void**)&sc.st, sizeof(SolverState)));
  if (!sc.h_st) MB_CUDA_OK(cudaMallocHost((void**)&sc.h_st, 4 * sizeof(SolverState)));
  if (sc.hist_cap < hist_len) {
    if (sc.hist) cudaFree(sc.hist);
    MB_CUDA_OK(cudaMalloc((void**)&sc.hist, hist_len * sizeof(double)));
    sc.hist_cap = hist_len;
  }
  return kOk;
}

void scratch_free(Scratch& sc) {
  cudaFree(sc.partials);
  cudaFree(sc.ticket);
  cudaFree(sc.st);
  cudaFreeHost(sc.h_st);
  cudaFree(sc.hist);
  sc = Scratch();
}

int dot64(long long n, const double* x, const double* y, double* out, Scratch& sc, cudaStream_t s) {
  int rc = scratch_ensure(sc, 1);
  if (rc) return rc;
  dot_kernel<double><<<148 * 4, 256, 0, s>>>(n, x, y, sc.partials, sc.ticket, out);
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

int diag_apply64(const SellMatrix& m, const double* x, double* y, cudaStream_t s) {
  if (!m.have_alu) return kBadInput;
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    diag_apply_kernel<B><<<(m.N + 255) / 256, 256, 0, s>>>(m.d_alu64, m.N, x, y);
    return kOk;
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

}  // namespace mb
