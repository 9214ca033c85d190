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

// Slots of slice s (h rows): h times the longest row of the slice.
__global__ void slice_width_kernel(const int* __restrict__ rowptr, int N, int nslices, int h,
                                   long long* __restrict__ width) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  int w = 0;
  for (int l = 0; l < h; l++) {
    int r = s * h + l;
    if (r < N) w = max(w, rowptr[r + 1] - rowptr[r]);
  }
  width[s] = (long long)w * h;
}

// Paired FP32 layout: one warp per slice of 64 rows, lane l writes rows
// 64s+2l and 64s+2l+1 at adjacent positions of every slot line.
template <int B>
__global__ void sell2_fill_kernel(const int* __restrict__ rowptr, const int* __restrict__ item,
                                  const double* __restrict__ csrval, const long long* __restrict__ slptr2, int N,
                                  int nslices, int* __restrict__ col, float* __restrict__ val) {
  constexpr int B2 = B * B;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nslices) return;
  const long long base = slptr2[warp];
  const int w = (int)((slptr2[warp + 1] - base) / 64);
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int row = warp * 64 + 2 * lane + j;
    const int len = row < N ? rowptr[row + 1] - rowptr[row] : 0;
    const long long j0 = row < N ? rowptr[row] : 0;
    for (int k = 0; k < w; k++) {
      const long long slot = base + (long long)k * 64;
      const long long pos = 2 * lane + j;
      if (k < len) {
        col[slot + pos] = item[j0 + k] - 1;
#pragma unroll
        for (int e = 0; e < B2; e++) val[slot * B2 + (long long)e * 64 + pos] = (float)csrval[(j0 + k) * B2 + e];
      } else {
        col[slot + pos] = row < N ? row : 0;
#pragma unroll
        for (int e = 0; e < B2; e++) val[slot * B2 + (long long)e * 64 + pos] = 0.0f;
      }
    }
  }
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

// Compressed column ids of one layout, P rows per lane (P = 1: 32-row slices;
// P = 2: the paired 64-row slices). One warp per slice. For slot position k,
// with e = col - P*l - h over the real blocks of the slot, the base is the
// midpoint c0 = min e + (max e - min e)/2 and every slot stores e - c0 in 16
// bits, so a slot fits when its blocks span less than 65535 columns (beyond
// the lane offset). On a structured mesh the rows at the two ends of a grid
// line put neighbours one stencil position apart into the same slot; the
// midpoint keeps those within range. A padded slot gets the difference of the
// column clamp(c0 + P*l + h, 0, N-1), a valid column within 64 of c0 + P*l + h,
// because the paired layout gathers at padded slots (their values are zero).
// If any real slot of the slice does not fit, the slice is marked wide (bit 0
// of slc) and keeps reading col[]. If every slot of the slice, padded ones
// included, has difference 0 -- every lane's block k sits at the same offset
// from its row, as in the interior of a structured mesh -- the slice is
// marked uniform (bit 1 of slc): its columns are the bases plus the lane
// position, and the difference stream is not read at all.
// stats: [0] wide slices, [1] real blocks in wide slices, [2] slot positions
// of compressed slices (uniform ones included), [3] real blocks in uniform
// slices, [4] uniform slices.
template <int P>
__global__ void col_compact_kernel(const int* __restrict__ rowptr, const long long* __restrict__ slptr, int N,
                                   int nslices, const int* __restrict__ col, short* __restrict__ col16,
                                   int* __restrict__ cbase, long long* __restrict__ slc,
                                   unsigned long long* __restrict__ stats) {
  constexpr int H = 32 * P;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nslices) return;  // whole warps (blockDim is a multiple of 32)
  const long long base = slptr[warp];
  const int w = (int)((slptr[warp + 1] - base) / H);
  int len[P];
#pragma unroll
  for (int h = 0; h < P; h++) {
    const long long row = warp * H + P * lane + h;
    len[h] = row < N ? rowptr[row + 1] - rowptr[row] : 0;
  }
  bool fit = true, uni = true;
  unsigned long long nreal = 0;
  for (int k = 0; k < w; k++) {
    const long long slot = base + (long long)k * H;
    int c[P];
    int emin = 0x7fffffff, emax = -0x7fffffff - 1;
#pragma unroll
    for (int h = 0; h < P; h++) {
      c[h] = col[slot + P * lane + h];
      if (k < len[h]) {
        const int e = c[h] - P * lane - h;  // >= -63, < N
        emin = min(emin, e);
        emax = max(emax, e);
      }
    }
    // some row of the slice is at least w long, so some lane has a real slot k
    emin = __reduce_min_sync(0xffffffffu, emin);
    emax = __reduce_max_sync(0xffffffffu, emax);
    const long long c0 = (long long)emin + (((long long)emax - emin) >> 1);
#pragma unroll
    for (int h = 0; h < P; h++) {
      const long long pos = (long long)P * lane + h;
      long long d;
      if (k < len[h]) {
        d = (long long)c[h] - c0 - pos;
        nreal++;
      } else {
        const long long tgt = c0 + pos < 0 ? 0 : (c0 + pos > N - 1 ? N - 1 : c0 + pos);
        d = tgt - c0 - pos;
      }
      fit = fit && d >= -32768 && d <= 32767;
      uni = uni && d == 0;
      col16[slot + pos] = (short)d;
    }
    if (lane == 0) cbase[base / H + k] = (int)c0;
  }
  fit = __all_sync(0xffffffffu, fit);
  uni = __all_sync(0xffffffffu, uni);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nreal += __shfl_xor_sync(0xffffffffu, nreal, o);
  if (lane == 0) {
    slc[warp] = base | (fit ? 0 : 1) | (uni ? 2 : 0);
    if (!fit) {
      atomicAdd(&stats[0], 1ULL);
      atomicAdd(&stats[1], nreal);
    } else {
      atomicAdd(&stats[2], (unsigned long long)w);
      if (uni) {
        atomicAdd(&stats[3], nreal);
        atomicAdd(&stats[4], 1ULL);
      }
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

// Grid-stride loops: launched with one thread per row (pair) for a plain
// product, or with a persistent grid when the unroll depth is tuned for the
// solver kernels, which all run persistent grids.
template <int B, int U, class V, class T>
__global__ void __launch_bounds__(256, SpmvMinBlocks<B>::value) spmv_kernel(SellView<V> A, const T* __restrict__ x, T* __restrict__ y) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < A.N; row += gridDim.x * blockDim.x) {
    T acc[B];
    sell_row<B, U, V, T>(A, x, row, acc);
#pragma unroll
    for (int r = 0; r < B; r++) y[(long long)row * B + r] = acc[r];
  }
}

template <int B, int U>
__global__ void __launch_bounds__(256, SpmvMinBlocks2<B>::value) spmv2_kernel(SellView2 A, const float* __restrict__ x, float* __restrict__ y) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; 2 * t < A.N; t += gridDim.x * blockDim.x) {
    float y0[B], y1[B];
    sell_row2<B, U>(A, x, t, y0, y1);
#pragma unroll
    for (int r = 0; r < B; r++) y[(long long)2 * t * B + r] = y0[r];
    if (2 * t + 1 < A.N) {
#pragma unroll
      for (int r = 0; r < B; r++) y[(long long)(2 * t + 1) * B + r] = y1[r];
    }
  }
}

// Resident blocks of 256 threads per SM x SMs.
template <class K>
int persistent_blocks(K kernel) {
  int b = 0, d = 0, sms = 0;
  cudaGetDevice(&d);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 256, 0) != cudaSuccess || b < 1) b = 1;
  return b * (sms > 0 ? sms : 148);
}

template <class T>
__global__ void dot_kernel(long long n, const T* __restrict__ x, const T* __restrict__ y, double* partials,
                           unsigned int* ticket, double* out) {
  DotAcc<1, T> v;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v.add(0, x[i], y[i]);
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


// Compressed column ids for one layout (P rows per lane); returns the column
// bytes one SpMV streams: 2 per block and 4 per slot position in compressed
// slices, 4 per slot position only in uniform slices, 4 per block in wide
// slices.
template <int P>
int compact_columns(const SellMatrix& m, const long long* d_slptr, int nslices, long long padded,
                    const int* d_col, short** col16, size_t& cap16, int** cbase, size_t& capb, long long** slc,
                    size_t& capslc, long long& wide, long long& uniform, double& col_bytes, cudaStream_t s) {
  MB_CUDA_OK(grow(col16, cap16, (size_t)padded + 2));
  MB_CUDA_OK(grow(cbase, capb, (size_t)(padded / (32 * P)) + 1));
  MB_CUDA_OK(grow(slc, capslc, (size_t)nslices + 1));
  unsigned long long* d_stats = nullptr;
  MB_CUDA_OK(cudaMallocAsync((void**)&d_stats, 5 * sizeof(unsigned long long), s));
  MB_CUDA_OK(cudaMemsetAsync(d_stats, 0, 5 * sizeof(unsigned long long), s));
  if (nslices > 0) {
    const long long threads = (long long)nslices * 32;
    col_compact_kernel<P><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(m.d_rowptr, d_slptr, m.N, nslices, d_col,
                                                                          *col16, *cbase, *slc, d_stats);
  }
  unsigned long long st[5] = {0, 0, 0, 0, 0};
  MB_CUDA_OK(cudaGetLastError());
  MB_CUDA_OK(cudaMemcpyAsync(st, d_stats, sizeof(st), cudaMemcpyDeviceToHost, s));
  MB_CUDA_OK(cudaStreamSynchronize(s));
  cudaFreeAsync(d_stats, s);
  wide = (long long)st[0];
  uniform = (long long)st[4];
  col_bytes = 2.0 * (double)(m.nz - (long long)st[1] - (long long)st[3]) + 4.0 * (double)st[1] + 4.0 * (double)st[2];
  return kOk;
}

}  // namespace

int sell_build(SellMatrix& m, const int* h_index, const int* h_item, const double* h_val, int N, int ndof,
               cudaStream_t s, double* t_h2d) {
  if (N <= 0 || ndof <= 0) return kBadInput;
  const long long nz = h_index[N];
  const int B2 = ndof * ndof;
  m.N = N;
  m.ndof = ndof;
  m.nz = nz;
  MB_CUDA_OK(grow(&m.d_rowptr, m.cap_rowptr, (size_t)N + 1));
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
  int rc = sell_layout(m, s);
  if (t_h2d) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);  // sell_layout has synchronized the stream
    *t_h2d = ms * 1e-3;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int sell_layout(SellMatrix& m, cudaStream_t s) {
  const int N = m.N, ndof = m.ndof;
  const int B2 = ndof * ndof;
  const int nslices = (N + kSlice - 1) / kSlice;
  m.nslices = nslices;
  m.have_val32 = m.have_alu = m.have_alu32 = false;
  MB_CUDA_OK(grow(&m.d_slptr, m.cap_slptr, (size_t)nslices + 1));
  // slice widths -> prefix on the host (nslices = N/32 values) -> slice pointers
  long long* d_w = nullptr;
  MB_CUDA_OK(cudaMallocAsync((void**)&d_w, sizeof(long long) * nslices, s));
  slice_width_kernel<<<(nslices + 255) / 256, 256, 0, s>>>(m.d_rowptr, N, nslices, kSlice, d_w);
  std::vector<long long> w(nslices), ptr(nslices + 1);
  MB_CUDA_OK(cudaMemcpyAsync(w.data(), d_w, sizeof(long long) * nslices, cudaMemcpyDeviceToHost, s));
  MB_CUDA_OK(cudaStreamSynchronize(s));
  cudaFreeAsync(d_w, s);
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
  double col_bytes = 0;
  rc = compact_columns<1>(m, m.d_slptr, nslices, m.padded, m.d_col, &m.d_col16, m.cap_col16, &m.d_cbase, m.cap_cbase,
                          &m.d_slc, m.cap_slc, m.wide64, m.uniform64, col_bytes, s);
  if (rc) return rc;
  // values, column ids, row offsets, slice offsets, x once and y
  m.bytes64 = (double)m.nz * B2 * 8 + col_bytes + 4.0 * (N + 1) + 8.0 * nslices + 2.0 * N * ndof * 8;
  return sell_autotune(m, false, s);
}

int sell_make_fp32(SellMatrix& m, cudaStream_t s) {
  if (m.have_val32) return kOk;
  const int N = m.N, B2 = m.ndof * m.ndof;
  const int ns = (N + 63) / 64;
  long long* d_w = nullptr;
  MB_CUDA_OK(cudaMallocAsync((void**)&d_w, sizeof(long long) * ns, s));
  slice_width_kernel<<<(ns + 255) / 256, 256, 0, s>>>(m.d_rowptr, N, ns, 64, d_w);
  std::vector<long long> w(ns), ptr(ns + 1);
  MB_CUDA_OK(cudaMemcpyAsync(w.data(), d_w, sizeof(long long) * ns, cudaMemcpyDeviceToHost, s));
  MB_CUDA_OK(cudaStreamSynchronize(s));
  cudaFreeAsync(d_w, s);
  ptr[0] = 0;
  for (int i = 0; i < ns; i++) ptr[i + 1] = ptr[i] + w[i];
  m.nslices2 = ns;
  m.padded2 = ptr[ns];
  MB_CUDA_OK(grow(&m.d_slptr2, m.cap_slptr2, (size_t)ns + 1));
  MB_CUDA_OK(grow(&m.d_col2, m.cap_col2, (size_t)m.padded2));
  MB_CUDA_OK(grow(&m.d_val32, m.cap_val32, (size_t)m.padded2 * B2));
  MB_CUDA_OK(cudaMemcpyAsync(m.d_slptr2, ptr.data(), sizeof(long long) * (ns + 1), cudaMemcpyHostToDevice, s));
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    sell2_fill_kernel<B><<<(ns * 32 + 255) / 256, 256, 0, s>>>(m.d_rowptr, m.d_item, m.d_csrval, m.d_slptr2, N, ns,
                                                              m.d_col2, m.d_val32);
    return kOk;
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  double col_bytes = 0;
  rc = compact_columns<2>(m, m.d_slptr2, ns, m.padded2, m.d_col2, &m.d_col16p, m.cap_col16p, &m.d_cbase2,
                          m.cap_cbase2, &m.d_slc2, m.cap_slc2, m.wide32, m.uniform32, col_bytes, s);
  if (rc) return rc;
  m.bytes32 = (double)m.nz * B2 * 4 + col_bytes + 4.0 * (N + 1) + 8.0 * ns + 2.0 * N * m.ndof * 4;
  m.have_val32 = true;
  if (m.have_alu) {
    const long long na = (long long)m.N * m.ndof * m.ndof;
    MB_CUDA_OK(grow(&m.d_alu32, m.cap_alu32, (size_t)na));
    to_fp32_kernel<<<148 * 8, 256, 0, s>>>(m.d_alu64, m.d_alu32, na);
    MB_CUDA_OK(cudaGetLastError());
    m.have_alu32 = true;
  }
  return sell_autotune(m, true, s);
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
  cudaFree(m.d_slptr2);
  cudaFree(m.d_col2);
  cudaFree(m.d_slc);
  cudaFree(m.d_col16);
  cudaFree(m.d_cbase);
  cudaFree(m.d_slc2);
  cudaFree(m.d_col16p);
  cudaFree(m.d_cbase2);
  m = SellMatrix();
}


int spmv64_u(const SellMatrix& m, int u, const double* x, double* y, cudaStream_t s, bool persistent = false) {
  SellView<double> A = view_of<double>(m);
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    return dispatch_u(u, [&](auto Uc) {
      constexpr int U = eff_u(B, decltype(Uc)::value);
      auto k = spmv_kernel<B, U, double, double>;
      k<<<persistent ? persistent_blocks(k) : (m.N + 255) / 256, 256, 0, s>>>(A, x, y);
      return (int)kOk;
    });
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

int spmv32_u(const SellMatrix& m, int u, const float* x, float* y, cudaStream_t s, bool persistent = false) {
  if (!m.have_val32) return kBadInput;
  SellView2 A = view2_of(m);
  const int threads = (m.N + 1) / 2;
  int rc = dispatch_ndof(m.ndof, [&](auto Bc) {
    constexpr int B = decltype(Bc)::value;
    return dispatch_u(u, [&](auto Uc) {
      constexpr int U = eff_u(B, decltype(Uc)::value);
      auto k = spmv2_kernel<B, U>;
      k<<<persistent ? persistent_blocks(k) : (threads + 255) / 256, 256, 0, s>>>(A, x, y);
      return (int)kOk;
    });
  });
  if (rc) return rc;
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

int spmv64(const SellMatrix& m, const double* x, double* y, cudaStream_t s) { return spmv64_u(m, m.u64, x, y, s); }
int spmv32(const SellMatrix& m, const float* x, float* y, cudaStream_t s) { return spmv32_u(m, m.u32, x, y, s); }

// Unroll depth per matrix (1, 2, 3 slots in flight; also 4 and 8 for 1x1
// blocks): each variant is launched 3 times on zero vectors (the kernels have
// no data-dependent control flow) and the fastest kept. The launches use the
// persistent grid of the solver kernels: a one-thread-per-row grid streams
// the matrix at the HBM rate for every depth and would not tell them apart.
int sell_autotune(SellMatrix& m, bool fp32, cudaStream_t s) {
  if (m.ndof >= 4) {
    m.u64 = m.u32 = 1;
    return kOk;
  }
  // a matrix rebuilt with the same shape (every solve when the device copy
  // is not cached) keeps the depth timed for it
  long long* key = fp32 ? m.tuned32 : m.tuned64;
  const long long shape[3] = {(long long)m.N * 8 + m.ndof, m.nz, fp32 ? m.padded2 : m.padded};
  if (key[0] == shape[0] && key[1] == shape[1] && key[2] == shape[2]) return kOk;
  const size_t n = (size_t)m.N * m.ndof;
  const size_t bytes = n * (fp32 ? sizeof(float) : sizeof(double));
  void *x = nullptr, *y = nullptr;
  MB_CUDA_OK(cudaMallocAsync(&x, bytes + 16, s));
  MB_CUDA_OK(cudaMallocAsync(&y, bytes + 16, s));
  MB_CUDA_OK(cudaMemsetAsync(x, 0, bytes, s));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int best_u = 2;
  int rc = kOk;
  static const int cand1[] = {1, 2, 3, 4, 8}, cand23[] = {1, 2, 3};
  const int* cand = m.ndof == 1 ? cand1 : cand23;
  const int ncand = m.ndof == 1 ? 5 : 3;
  for (int ci = 0; ci < ncand && rc == kOk; ci++) {
    const int u = cand[ci];
    auto run = [&]() {
      return fp32 ? spmv32_u(m, u, (const float*)x, (float*)y, s, true)
                  : spmv64_u(m, u, (const double*)x, (double*)y, s, true);
    };
    rc = run();  // warm
    if (rc) break;
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; r++) run();
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = kCudaError;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) {
      best = ms;
      best_u = u;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(x, s);
  cudaFreeAsync(y, s);
  if (rc) return rc;
  if (fp32) m.u32 = best_u;
  else m.u64 = best_u;
  for (int i = 0; i < 3; i++) key[i] = shape[i];
  return kOk;
}

int scratch_ensure(Scratch& sc, size_t hist_len) {
  // up to 65536 blocks of 4 doubles, or of 2 double-double sums
  const size_t need = (65536 + 256) * 4;
  if (sc.partials_cap < need) {
    if (sc.partials) cudaFree(sc.partials);
    MB_CUDA_OK(cudaMalloc((void**)&sc.partials, need * sizeof(double)));
    sc.partials_cap = need;
  }
  if (!sc.ticket) {
    MB_CUDA_OK(cudaMalloc((void**)&sc.ticket, kTicketWords * sizeof(unsigned int)));
    MB_CUDA_OK(cudaMemset(sc.ticket, 0, kTicketWords * sizeof(unsigned int)));
  }
  if (!sc.st) MB_CUDA_OK(cudaMalloc((void**)&sc.st, sizeof(SolverState)));
  if (!sc.h_st) MB_CUDA_OK(cudaMallocHost((void**)&sc.h_st, 8 * sizeof(SolverState)));  // launches in flight
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
  MB_CUDA_OK(cudaMemsetAsync(sc.ticket, 0, sizeof(unsigned int) * kTicketWords, s));
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
