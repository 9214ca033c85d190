// adjoint.cu -- the pieces of a discrete adjoint around the block-CSR solve:
// the transposed matrix on the device (for A^T lambda = dL/dx), the sampled
// outer product -lambda_i x_j^T over the sparsity pattern (dL/dA in the
// layout of the matrix values), and its reduction to per-element coefficient
// gradients dL/dk_e = -sum_ab lambda_a K_e(a,b) x_b for A = sum_e k_e K_e.
//
// The transpose follows the reference's CSC arrays
// (src/matrix/spmat_nzpattern_util.f90:162-218): row j of A^T lists the rows
// i of column j in ascending order, so A^T's SpMV sums each row in that
// order and its CSR is exactly the BCSR of the explicit transpose.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "spmv.cuh"

namespace mb {
namespace {

template <class P>
cudaError_t grow_buf(P** p, size_t& cap, size_t need) {
  if (*p && cap >= need) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void**)p, need * sizeof(P) + 16);
  if (e == cudaSuccess) cap = need;
  return e;
}

// A^T's CSR values: block k of A^T is block perm[k]-1 of A, transposed.
template <int B>
__global__ void transpose_values_kernel(const int* __restrict__ perm, long long nz, const double* __restrict__ val,
                                        double* __restrict__ valt) {
  constexpr int B2 = B * B;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nz * B2;
       e += (long long)gridDim.x * blockDim.x) {
    const long long k = e / B2;
    const int rc = (int)(e - k * B2);
    const int r = rc / B, c = rc - (rc / B) * B;
    valt[e] = val[(long long)(perm[k] - 1) * B2 + c * B + r];
  }
}

// G[k](r,c) = scale * lambda[i*B+r] * x[j*B+c] for stored block k = (i, j).
// One warp per block row; lanes walk the row's ndof^2 * len contiguous
// outputs, so the stores are coalesced.
template <int B>
__global__ void outer_product_kernel(const int* __restrict__ rowptr, const int* __restrict__ item, int N,
                                     const double* __restrict__ lam, const double* __restrict__ x, double scale,
                                     double* __restrict__ G) {
  constexpr int B2 = B * B;
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; row < N; row += warps) {
    double l[B];
#pragma unroll
    for (int r = 0; r < B; r++) l[r] = __dmul_rn(scale, lam[row * B + r]);
    const long long k0 = rowptr[row];
    const long long len = (long long)(rowptr[row + 1] - k0) * B2;
    for (long long e = lane; e < len; e += 32) {
      const long long k = k0 + e / B2;
      const int rc = (int)(e % B2);
      const int r = rc / B, c = rc % B;
      const long long j = item[k] - 1;
      double lr = l[0];
#pragma unroll
      for (int q = 1; q < B; q++)
        if (r == q) lr = l[q];
      G[k0 * B2 + e] = __dmul_rn(lr, x[j * B + c]);
    }
  }
}

// grad[e] = scale * sum_a lam_a * (sum_b K(a,b) x_b) over the element's
// NL = n_base * ndof local dofs (node-major, dof-minor like the element
// matrices of monolis_add_matrix_to_sparse_matrix_R); lam_a counts as zero
// where fixed[dof] != 0 (Dirichlet rows do not depend on the coefficients).
// K is shared by all elements (ke_stride == 0, staged in shared memory) or
// per element at Ke + e*ke_stride.
template <int NL>
__global__ void __launch_bounds__(128) element_gradient_kernel(int n_elem, int n_base, int ndof,
                                                               const int* __restrict__ elem,
                                                               const double* __restrict__ Ke, long long ke_stride,
                                                               const double* __restrict__ lam,
                                                               const double* __restrict__ x,
                                                               const int* __restrict__ fixed, double scale,
                                                               double* __restrict__ grad) {
  __shared__ double Ks[NL * NL];
  if (ke_stride == 0) {
    for (int i = threadIdx.x; i < NL * NL; i += blockDim.x) Ks[i] = Ke[i];
    __syncthreads();
  }
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_elem;
       e += (long long)gridDim.x * blockDim.x) {
    double xe[NL], le[NL];
#pragma unroll
    for (int a = 0; a < NL; a++) {
      const int node = elem[e * n_base + a / ndof];
      const long long d = (long long)node * ndof + (a % ndof);
      xe[a] = x[d];
      le[a] = (fixed && fixed[d]) ? 0.0 : lam[d];
    }
    const double* K = ke_stride == 0 ? Ks : Ke + e * ke_stride;
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < NL; a++) {
      double t = 0.0;
#pragma unroll
      for (int b = 0; b < NL; b++) t = fma(K[a * NL + b], xe[b], t);
      acc = fma(le[a], t, acc);
    }
    grad[e] = scale * acc;
  }
}

// Any other element size: the same sum with the element's values read from
// global memory (L1-resident) instead of registers.
__global__ void element_gradient_generic_kernel(int n_elem, int n_base, int ndof, const int* __restrict__ elem,
                                                const double* __restrict__ Ke, long long ke_stride,
                                                const double* __restrict__ lam, const double* __restrict__ x,
                                                const int* __restrict__ fixed, double scale,
                                                double* __restrict__ grad) {
  const int NL = n_base * ndof;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_elem;
       e += (long long)gridDim.x * blockDim.x) {
    const double* K = Ke + e * ke_stride;
    const int* en = elem + e * n_base;
    double acc = 0.0;
    for (int a = 0; a < NL; a++) {
      const long long da = (long long)en[a / ndof] * ndof + a % ndof;
      if (fixed && fixed[da]) continue;
      double t = 0.0;
      for (int b = 0; b < NL; b++) t = fma(K[(long long)a * NL + b], x[(long long)en[b / ndof] * ndof + b % ndof], t);
      acc = fma(lam[da], t, acc);
    }
    grad[e] = scale * acc;
  }
}

}  // namespace

int sell_build_transpose(SellMatrix& at, const SellMatrix& a, const int* h_csc_index, const int* h_csc_item,
                         const int* h_csc_perm, cudaStream_t s) {
  if (!a.d_csrval || a.N <= 0) return kBadInput;
  const long long nz = a.nz;
  const int B2 = a.ndof * a.ndof;
  at.N = a.N;
  at.ndof = a.ndof;
  at.nz = nz;
  MB_CUDA_OK(grow_buf(&at.d_rowptr, at.cap_rowptr, (size_t)a.N + 1));
  MB_CUDA_OK(grow_buf(&at.d_item, at.cap_item, (size_t)nz));
  MB_CUDA_OK(grow_buf(&at.d_csrval, at.cap_csrval, (size_t)nz * B2));
  int* d_perm = nullptr;
  MB_CUDA_OK(cudaMallocAsync((void**)&d_perm, sizeof(int) * (nz + 1), s));
  MB_CUDA_OK(cudaMemcpyAsync(at.d_rowptr, h_csc_index, sizeof(int) * (a.N + 1), cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(cudaMemcpyAsync(at.d_item, h_csc_item, sizeof(int) * nz, cudaMemcpyHostToDevice, s));
  MB_CUDA_OK(cudaMemcpyAsync(d_perm, h_csc_perm, sizeof(int) * nz, cudaMemcpyHostToDevice, s));
  int rc = dispatch_ndof(a.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    transpose_values_kernel<B><<<148 * 16, 256, 0, s>>>(d_perm, nz, a.d_csrval, at.d_csrval);
    return kOk;
  });
  cudaFreeAsync(d_perm, s);
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  return sell_layout(at, s);
}

int outer_product64(const SellMatrix& m, const double* lam, const double* x, double scale, double* G,
                    cudaStream_t s) {
  if (!m.d_rowptr || !m.d_item) return kBadInput;
  const long long warps_needed = m.N;
  const int blocks = (int)std::min<long long>((warps_needed + 7) / 8, 148LL * 64);
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    outer_product_kernel<B><<<blocks, 256, 0, s>>>(m.d_rowptr, m.d_item, m.N, lam, x, scale, G);
    return kOk;
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

int element_gradient64(int n_elem, int n_base, int ndof, const int* elem, const double* Ke, long long ke_stride,
                       const double* lam, const double* x, const int* fixed, double scale, double* grad,
                       cudaStream_t s) {
  if (n_elem < 0 || n_base <= 0 || ndof <= 0 || ke_stride < 0) return kBadInput;
  if (n_elem == 0) return kOk;
  const int NL = n_base * ndof;
  const int threads = 128;
  const int blocks = (int)std::min<long long>(((long long)n_elem + threads - 1) / threads, 148LL * 32);
  auto launch = [&](auto NLc) {
    constexpr int L = decltype(NLc)::value;
    element_gradient_kernel<L><<<blocks, threads, 0, s>>>(n_elem, n_base, ndof, elem, Ke, ke_stride, lam, x, fixed,
                                                          scale, grad);
  };
  switch (NL) {
    case 4: launch(std::integral_constant<int, 4>{}); break;
    case 8: launch(std::integral_constant<int, 8>{}); break;
    case 12: launch(std::integral_constant<int, 12>{}); break;
    case 24: launch(std::integral_constant<int, 24>{}); break;
    default:
      element_gradient_generic_kernel<<<blocks, threads, 0, s>>>(n_elem, n_base, ndof, elem, Ke, ke_stride, lam, x,
                                                                 fixed, scale, grad);
  }
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

}  // namespace mb
