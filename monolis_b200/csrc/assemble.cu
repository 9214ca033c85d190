// assemble.cu -- assembly of the block-CSR values on the device: element
// matrices (monolis_add_matrix_to_sparse_matrix_R for many elements) and
// Dirichlet conditions (monolis_set_Dirichlet_bc_R for a list of them),
// bit-identical to the host calls made in order.
//
// Elements: one thread per block row walks the elements incident to its row in
// ascending element order (a node -> element incidence list built on the
// device and sorted per node), and within an element the (a, b) pairs in the
// order of src/matrix/spmat_handler_util.f90:398-497, adding
// scale * K_e(a,b) to the blocks of its own row. Every entry therefore
// receives its contributions in element order, as with the serial loop, and
// no two threads write the same block.
//
// Dirichlet (src/matrix/spmat_handler_util.f90:604-677) applied to a list of
// (node, dof, value) in order has a closed form that this file evaluates in
// parallel:
//   * a dof never fixed: b[n] -= v_c * A[n][c] for every fixed column c of its
//     row, in the order of each column's first occurrence in the list, with
//     the value of that first occurrence (a repeated column finds its entries
//     already zero);
//   * every entry in a fixed row or a fixed column becomes 0, the diagonal
//     entry of a fixed dof 1;
//   * b of a fixed dof is the value of its last occurrence.
// (Contributions to a dof's b made before its own condition is processed are
// overwritten by it; after its row is zeroed the column moves add v * 0.)
#include <algorithm>
#include <cstdio>
#include <vector>

#include "spmv.cuh"

namespace mb {
namespace {

__global__ void check_elements_kernel(const int* __restrict__ elem, long long n, int NP, int* __restrict__ bad) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (elem[i] < 0 || elem[i] >= NP) atomicOr(bad, 1);
}

// incidence counts: element e counted once per distinct node
__global__ void incidence_count_kernel(const int* __restrict__ elem, int n_elem, int n_base, int* __restrict__ cnt) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_elem;
       e += (long long)gridDim.x * blockDim.x) {
    const int* en = elem + e * n_base;
    for (int a = 0; a < n_base; a++) {
      bool dup = false;
      for (int q = 0; q < a; q++) dup |= en[q] == en[a];
      if (!dup) atomicAdd(cnt + en[a], 1);
    }
  }
}

__global__ void incidence_fill_kernel(const int* __restrict__ elem, int n_elem, int n_base,
                                      const int* __restrict__ ptr, int* __restrict__ fill, int* __restrict__ list) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_elem;
       e += (long long)gridDim.x * blockDim.x) {
    const int* en = elem + e * n_base;
    for (int a = 0; a < n_base; a++) {
      bool dup = false;
      for (int q = 0; q < a; q++) dup |= en[q] == en[a];
      if (!dup) list[ptr[en[a]] + atomicAdd(fill + en[a], 1)] = (int)e;
    }
  }
}

// the atomics above fill each node's list in arbitrary order: sort it
__global__ void incidence_sort_kernel(const int* __restrict__ ptr, int N, int* __restrict__ list) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int lo = ptr[i], hi = ptr[i + 1];
    for (int p = lo + 1; p < hi; p++) {
      const int v = list[p];
      int q = p - 1;
      while (q >= lo && list[q] > v) {
        list[q + 1] = list[q];
        q--;
      }
      list[q + 1] = v;
    }
  }
}

__device__ __forceinline__ int find_slot(const int* __restrict__ rowptr, const int* __restrict__ item, int i, int j) {
  int lo = rowptr[i], hi = rowptr[i + 1] - 1;
  const int key = j + 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = item[mid];
    if (v == key) return mid;
    if (v < key) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

template <int B>
__global__ void add_elements_kernel(const int* __restrict__ rowptr, const int* __restrict__ item, int N,
                                    const int* __restrict__ iptr, const int* __restrict__ ilist,
                                    const int* __restrict__ elem, int n_base, const double* __restrict__ val,
                                    long long val_stride, const double* __restrict__ scale,
                                    double* __restrict__ A, int* __restrict__ bad) {
  constexpr int B2 = B * B;
  const int ncol = n_base * B;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    for (int q = iptr[i]; q < iptr[i + 1]; q++) {
      const long long e = ilist[q];
      const int* en = elem + e * n_base;
      const double* Ke = val + e * val_stride;
      const double s = scale ? scale[e] : 1.0;
      for (int a = 0; a < n_base; a++) {
        if (en[a] != i) continue;
        for (int b = 0; b < n_base; b++) {
          const int k = find_slot(rowptr, item, i, en[b]);
          if (k < 0) {
            atomicOr(bad, 2);
            continue;
          }
          double* dst = A + (long long)k * B2;
#pragma unroll
          for (int k1 = 0; k1 < B; k1++)
#pragma unroll
            for (int k2 = 0; k2 < B; k2++) {
              const double v = Ke[(long long)(a * B + k1) * ncol + b * B + k2];
              dst[k1 * B + k2] = __dadd_rn(dst[k1 * B + k2], scale ? __dmul_rn(s, v) : v);
            }
        }
      }
    }
  }
}

// b[n] -= v_first(c) * A[n][c] over the fixed columns c of row i, in the
// order of their first occurrence, for the never-fixed dofs n of the row.
template <int B>
__global__ void dirichlet_rhs_kernel(const int* __restrict__ rowptr, const int* __restrict__ item, int N,
                                     const double* __restrict__ A, const int* __restrict__ ord,
                                     const double* __restrict__ vfirst, double* __restrict__ b) {
  constexpr int B2 = B * B;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int lo = rowptr[i], hi = rowptr[i + 1];
    int prev = -1;
    for (;;) {
      // the fixed column of this row with the smallest first occurrence after prev
      int best = 0x7fffffff, bk = -1, bc = 0;
      for (int k = lo; k < hi; k++) {
        const long long j = item[k] - 1;
#pragma unroll
        for (int c = 0; c < B; c++) {
          const int o = ord[j * B + c];
          if (o > prev && o < best) {
            best = o;
            bk = k;
            bc = c;
          }
        }
      }
      if (bk < 0) break;
      const long long jc = (long long)(item[bk] - 1) * B + bc;
      const double v = vfirst[jc];
#pragma unroll
      for (int r = 0; r < B; r++) {
        const long long n = (long long)i * B + r;
        if (ord[n] >= 0) continue;
        b[n] = __dsub_rn(b[n], __dmul_rn(v, A[(long long)bk * B2 + r * B + bc]));
      }
      prev = best;
    }
  }
}

// zero fixed rows and columns, unit diagonal of fixed dofs, b = last value
template <int B>
__global__ void dirichlet_matrix_kernel(const int* __restrict__ rowptr, const int* __restrict__ item, int N,
                                        double* __restrict__ A, const int* __restrict__ ord,
                                        const double* __restrict__ vlast, double* __restrict__ b,
                                        int* __restrict__ bad) {
  constexpr int B2 = B * B;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    bool diag_found[B];
#pragma unroll
    for (int r = 0; r < B; r++) diag_found[r] = false;
    for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
      const long long j = item[k] - 1;
#pragma unroll
      for (int r = 0; r < B; r++) {
        const bool fr = ord[(long long)i * B + r] >= 0;
#pragma unroll
        for (int c = 0; c < B; c++) {
          const bool fc = ord[j * B + c] >= 0;
          if (fr || fc) {
            const bool unit = fr && j == i && c == r;
            A[(long long)k * B2 + r * B + c] = unit ? 1.0 : 0.0;
            if (unit) diag_found[r] = true;
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < B; r++) {
      const long long n = (long long)i * B + r;
      if (ord[n] >= 0) {
        b[n] = vlast[n];
        if (!diag_found[r]) atomicOr(bad, 4);
      }
    }
  }
}

template <class P>
cudaError_t dalloc_async(P** p, size_t n, cudaStream_t s) {
  return cudaMallocAsync((void**)p, n * sizeof(P) + 16, s);
}

}  // namespace

int device_add_elements(SellMatrix& m, int NP, int n_elem, int n_base, const int* d_elem, const double* d_val,
                        long long val_stride, const double* d_scale, cudaStream_t s) {
  if (n_elem < 0 || n_base <= 0 || val_stride < 0 || !m.d_csrval) return kBadInput;
  if (n_elem == 0) return kOk;
  const int N = m.N;
  const long long ne = (long long)n_elem * n_base;
  int *d_bad = nullptr, *d_cnt = nullptr, *d_ptr = nullptr, *d_fill = nullptr, *d_list = nullptr;
  MB_CUDA_OK(dalloc_async(&d_bad, 1, s));
  MB_CUDA_OK(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
  check_elements_kernel<<<148 * 8, 256, 0, s>>>(d_elem, ne, NP, d_bad);
  int bad = 0;
  MB_CUDA_OK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  MB_CUDA_OK(cudaStreamSynchronize(s));
  if (bad || NP != N) {
    cudaFreeAsync(d_bad, s);
    return kBadInput;
  }
  // node -> elements, ascending per node
  MB_CUDA_OK(dalloc_async(&d_cnt, (size_t)N, s));
  MB_CUDA_OK(dalloc_async(&d_fill, (size_t)N, s));
  MB_CUDA_OK(dalloc_async(&d_ptr, (size_t)N + 1, s));
  MB_CUDA_OK(dalloc_async(&d_list, (size_t)ne, s));
  MB_CUDA_OK(cudaMemsetAsync(d_cnt, 0, sizeof(int) * N, s));
  MB_CUDA_OK(cudaMemsetAsync(d_fill, 0, sizeof(int) * N, s));
  incidence_count_kernel<<<148 * 8, 256, 0, s>>>(d_elem, n_elem, n_base, d_cnt);
  std::vector<int> cnt(N), ptr(N + 1);
  MB_CUDA_OK(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * N, cudaMemcpyDeviceToHost, s));
  MB_CUDA_OK(cudaStreamSynchronize(s));
  ptr[0] = 0;
  for (int i = 0; i < N; i++) ptr[i + 1] = ptr[i] + cnt[i];
  MB_CUDA_OK(cudaMemcpyAsync(d_ptr, ptr.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice, s));
  incidence_fill_kernel<<<148 * 8, 256, 0, s>>>(d_elem, n_elem, n_base, d_ptr, d_fill, d_list);
  incidence_sort_kernel<<<(N + 255) / 256, 256, 0, s>>>(d_ptr, N, d_list);
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    add_elements_kernel<B><<<(N + 127) / 128, 128, 0, s>>>(m.d_rowptr, m.d_item, N, d_ptr, d_list, d_elem, n_base,
                                                           d_val, val_stride, d_scale, m.d_csrval, d_bad);
    return kOk;
  });
  MB_CUDA_OK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  cudaFreeAsync(d_cnt, s);
  cudaFreeAsync(d_fill, s);
  cudaFreeAsync(d_ptr, s);
  cudaFreeAsync(d_list, s);
  cudaFreeAsync(d_bad, s);
  MB_CUDA_OK(cudaStreamSynchronize(s));
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  if (bad) {
    fprintf(stderr, "** monolis_b200: device assembly: an element entry is not in the nonzero pattern\n");
    return kBadInput;
  }
  return kOk;
}

int device_dirichlet(SellMatrix& m, double* d_b, int n_bc, const int* node, const int* dof, const double* val,
                     cudaStream_t s) {
  const int N = m.N, nd = m.ndof;
  const long long n = (long long)N * nd;
  std::vector<int> ord(n, -1);
  std::vector<double> vfirst(n, 0.0), vlast(n, 0.0);
  for (int q = 0; q < n_bc; q++) {
    if (node[q] < 0 || node[q] >= N || dof[q] < 0 || dof[q] >= nd) return kBadInput;
    const long long d = (long long)node[q] * nd + dof[q];
    if (ord[d] < 0) {
      ord[d] = q;
      vfirst[d] = val[q];
    }
    vlast[d] = val[q];
  }
  int* d_ord = nullptr;
  double *d_vf = nullptr, *d_vl = nullptr;
  int* d_bad = nullptr;
  MB_CUDA_OK(dalloc_async(&d_ord, (size_t)n, s));
  MB_CUDA_OK(dalloc_async(&d_vf, (size_t)n, s));
  MB_CUDA_OK(dalloc_async(&d_vl, (size_t)n, s));
  MB_CUDA_OK(dalloc_async(&d_bad, 1, s));
  MB_CUDA_OK(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
  MB_CUDA_OK(cudaMemcpyAsync(d_ord, ord.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(cudaMemcpyAsync(d_vf, vfirst.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(cudaMemcpyAsync(d_vl, vlast.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  int rc = dispatch_ndof(nd, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    const int grid = (N + 127) / 128;
    dirichlet_rhs_kernel<B><<<grid, 128, 0, s>>>(m.d_rowptr, m.d_item, N, m.d_csrval, d_ord, d_vf, d_b);
    dirichlet_matrix_kernel<B><<<grid, 128, 0, s>>>(m.d_rowptr, m.d_item, N, m.d_csrval, d_ord, d_vl, d_b, d_bad);
    return kOk;
  });
  int bad = 0;
  MB_CUDA_OK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  cudaFreeAsync(d_ord, s);
  cudaFreeAsync(d_vf, s);
  cudaFreeAsync(d_vl, s);
  cudaFreeAsync(d_bad, s);
  MB_CUDA_OK(cudaStreamSynchronize(s));
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  if (bad) {
    fprintf(stderr, "** monolis_b200: set Dirichlet: diagonal block not found\n");
    return kBadInput;
  }
  return kOk;
}

}  // namespace mb
