// shard.cu -- the row-partitioned (multi-rank) solve: one process per GPU,
// each holding the rows it owns plus ghost columns, the layout of the
// reference's MPI runs (MONOLIS_COM tables: src/linalg/matvec.f90:144 updates
// the ghost entries of the multiplied vector, src/linalg/inner_product.f90:185
// sums the dot products over the ranks).
//
// Here the halo update is a pack kernel, NCCL send/receive pairs with every
// neighbour inside one NCCL group (a neighbour entry naming this rank itself
// is a device copy), and an unpack kernel; a dot product is the
// device-resident local sum followed by an NCCL all-reduce and a one-thread
// kernel that applies the scalar update with the global sums. Before the
// products of the iteration the halo update runs on a side stream while the
// solver stream multiplies the interior slices (rows that read no ghost
// entry); the boundary slices follow once the update has landed. Everything
// is enqueued on the solver stream or forked from it with events, so it is
// captured in the solver's CUDA graphs like the rest of the iteration. Every rank evaluates the scalar
// recurrences from the same all-reduced bits, so all ranks stop at the same
// iteration and issue the same sequence of collectives.
//
// NCCL is loaded at run time (dlopen "libnccl.so.2") when a communicator is
// first created, so single-rank use needs no NCCL; a process that has already
// loaded NCCL (e.g. through PyTorch) reuses that library.
#include <dlfcn.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <nccl.h>

#include "spmv.cuh"

namespace mb {
namespace {

struct NcclApi {
  bool loaded = false;
  void* handle = nullptr;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t) =
      nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      fprintf(stderr, "** monolis_b200: libnccl.so.2 not found (%s)\n", dlerror());
      return;
    }
    api.handle = h;
    bool ok = true;
    auto get = [&](auto& fn, const char* name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
      ok &= fn != nullptr;
    };
    get(api.GetUniqueId, "ncclGetUniqueId");
    get(api.CommInitRank, "ncclCommInitRank");
    get(api.CommDestroy, "ncclCommDestroy");
    get(api.AllReduce, "ncclAllReduce");
    get(api.Send, "ncclSend");
    get(api.Recv, "ncclRecv");
    get(api.GroupStart, "ncclGroupStart");
    get(api.GroupEnd, "ncclGroupEnd");
    get(api.GetErrorString, "ncclGetErrorString");
    api.loaded = ok;
    if (!ok) fprintf(stderr, "** monolis_b200: libnccl.so.2 lacks a required symbol\n");
  });
  return api;
}

int nccl_check(ncclResult_t r, const char* what) {
  if (r == ncclSuccess) return kOk;
  fprintf(stderr, "** monolis_b200: %s failed: %s\n", what, nccl().GetErrorString ? nccl().GetErrorString(r) : "?");
  return kCudaError;
}

template <class T>
__global__ void pack_kernel(const T* __restrict__ v, const int* __restrict__ item, long long n, int nd,
                            T* __restrict__ buf) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * nd; i += (long long)gridDim.x * blockDim.x) {
    const long long q = i / nd;
    buf[i] = v[(long long)item[q] * nd + (i - q * nd)];
  }
}

template <class T>
__global__ void unpack_kernel(T* __restrict__ v, const int* __restrict__ item, long long n, int nd,
                              const T* __restrict__ buf) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * nd; i += (long long)gridDim.x * blockDim.x) {
    const long long q = i / nd;
    v[(long long)item[q] * nd + (i - q * nd)] = buf[i];
  }
}

// Flag per 32-row slice: 1 when one of its rows reads a ghost entry
// (block column >= N, the ghost rows following the owned ones).
__global__ void boundary_slices_kernel(const int* __restrict__ rowptr, const int* __restrict__ item, int N,
                                       int nslices, int* __restrict__ flag) {
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long sl = gt >> 5;
  if (sl >= nslices) return;  // whole warps (blockDim is a multiple of 32)
  const long long row = gt;   // slice sl, lane gt & 31
  bool ghost = false;
  if (row < N)
    for (int j = rowptr[row]; j < rowptr[row + 1]; j++) ghost = ghost || (item[j] - 1 >= N);
  const unsigned any = __ballot_sync(0xffffffffu, ghost);
  if ((gt & 31) == 0) flag[sl] = any != 0;
}

}  // namespace

int shard_unique_id(void* out128) {
  NcclApi& a = nccl();
  if (!a.loaded) return kCudaError;
  ncclUniqueId id;
  int rc = nccl_check(a.GetUniqueId(&id), "ncclGetUniqueId");
  if (rc) return rc;
  memcpy(out128, &id, sizeof(id));
  return kOk;
}

int shard_comm_create(void** comm, const void* id128, int rank, int size) {
  NcclApi& a = nccl();
  if (!a.loaded) return kCudaError;
  ncclUniqueId id;
  memcpy(&id, id128, sizeof(id));
  ncclComm_t c = nullptr;
  int rc = nccl_check(a.CommInitRank(&c, size, id, rank), "ncclCommInitRank");
  if (rc) return rc;
  *comm = c;
  return kOk;
}

void shard_comm_destroy(void* comm) {
  if (comm && nccl().loaded) nccl().CommDestroy(static_cast<ncclComm_t>(comm));
}

int shard_setup(ShardPlan& sp, const ShardTables& t, int ndof, const SellMatrix& A, cudaStream_t s) {
  sp.ndof = ndof;
  sp.rank = t.rank;
  sp.send_pe = t.send_pe;
  sp.recv_pe = t.recv_pe;
  sp.send_ptr = t.send_ptr;
  sp.recv_ptr = t.recv_ptr;
  const size_t ns = t.send_ptr.empty() ? 0 : (size_t)t.send_ptr.back();
  const size_t nr = t.recv_ptr.empty() ? 0 : (size_t)t.recv_ptr.back();
  sp.n_send = (long long)ns;
  sp.n_recv = (long long)nr;
  auto up_int = [&](int** dst, const std::vector<int>& src) -> int {
    cudaFree(*dst);
    *dst = nullptr;
    MB_CUDA_OK(cudaMalloc((void**)dst, sizeof(int) * (src.size() + 1)));
    if (!src.empty()) MB_CUDA_OK(cudaMemcpy(*dst, src.data(), sizeof(int) * src.size(), cudaMemcpyHostToDevice));
    return kOk;
  };
  int rc = up_int(&sp.d_send_item, t.send_item);
  if (!rc) rc = up_int(&sp.d_recv_item, t.recv_item);
  if (rc) return rc;
  cudaFree(sp.d_sendbuf);
  cudaFree(sp.d_recvbuf);
  sp.d_sendbuf = sp.d_recvbuf = nullptr;
  MB_CUDA_OK(cudaMalloc(&sp.d_sendbuf, sizeof(double) * (ns * ndof + 2)));
  MB_CUDA_OK(cudaMalloc(&sp.d_recvbuf, sizeof(double) * (nr * ndof + 2)));
  // a neighbour entry naming this rank exchanges with itself: the matching
  // send and receive lists must have the same length
  for (size_t q = 0; q < t.send_pe.size(); q++) {
    if (t.send_pe[q] != t.rank) continue;
    bool ok = false;
    for (size_t r = 0; r < t.recv_pe.size(); r++)
      if (t.recv_pe[r] == t.rank)
        ok = t.recv_ptr[r + 1] - t.recv_ptr[r] == t.send_ptr[q + 1] - t.send_ptr[q];
    if (!ok) {
      fprintf(stderr, "** monolis_b200: halo tables: the self-exchange lists differ in length\n");
      return kBadInput;
    }
  }
  // interior / boundary slices of the device matrix
  const int nsl = A.nslices;
  std::vector<int> flag(nsl > 0 ? nsl : 1, 0);
  int* d_flag = nullptr;
  MB_CUDA_OK(cudaMalloc((void**)&d_flag, sizeof(int) * (nsl + 1)));
  if (nsl > 0) {
    const long long threads = (long long)nsl * 32;
    boundary_slices_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(A.d_rowptr, A.d_item, A.N, nsl, d_flag);
    MB_CUDA_OK(cudaGetLastError());
    MB_CUDA_OK(cudaMemcpyAsync(flag.data(), d_flag, sizeof(int) * nsl, cudaMemcpyDeviceToHost, s));
  }
  MB_CUDA_OK(cudaStreamSynchronize(s));
  cudaFree(d_flag);
  std::vector<int> order;
  order.reserve(nsl);
  for (int i = 0; i < nsl; i++)
    if (!flag[i]) order.push_back(i);
  sp.n_int = (int)order.size();
  for (int i = 0; i < nsl; i++)
    if (flag[i]) order.push_back(i);
  sp.n_bnd = nsl - sp.n_int;
  rc = up_int(&sp.d_slices, order);
  if (rc) return rc;
  if (!sp.side) MB_CUDA_OK(cudaStreamCreateWithFlags(&sp.side, cudaStreamNonBlocking));
  if (!sp.ev_fork) MB_CUDA_OK(cudaEventCreateWithFlags(&sp.ev_fork, cudaEventDisableTiming));
  if (!sp.ev_join) MB_CUDA_OK(cudaEventCreateWithFlags(&sp.ev_join, cudaEventDisableTiming));
  return kOk;
}

void shard_free(ShardPlan& sp) {
  cudaFree(sp.d_send_item);
  cudaFree(sp.d_recv_item);
  cudaFree(sp.d_sendbuf);
  cudaFree(sp.d_recvbuf);
  cudaFree(sp.d_slices);
  if (sp.side) cudaStreamDestroy(sp.side);
  if (sp.ev_fork) cudaEventDestroy(sp.ev_fork);
  if (sp.ev_join) cudaEventDestroy(sp.ev_join);
  sp = ShardPlan();
}

namespace {
template <class T>
constexpr ncclDataType_t nccl_type();
template <>
constexpr ncclDataType_t nccl_type<double>() { return ncclDouble; }
template <>
constexpr ncclDataType_t nccl_type<float>() { return ncclFloat; }

// Ghost entries of v (block rows of ndof) from their owners. The staging
// buffers hold ndof doubles per listed row, so FP32 vectors fit as well.
template <class T>
int halo_update(const ShardPlan& sp, T* v, cudaStream_t s) {
  NcclApi& a = nccl();
  const int nd = sp.ndof;
  T* sb = static_cast<T*>(sp.d_sendbuf);
  T* rb = static_cast<T*>(sp.d_recvbuf);
  if (sp.n_send > 0) pack_kernel<T><<<148 * 2, 256, 0, s>>>(v, sp.d_send_item, sp.n_send, nd, sb);
  // the list this rank sends to itself lands directly in its receive buffer
  for (size_t q = 0; q < sp.send_pe.size(); q++) {
    if (sp.send_pe[q] != sp.rank) continue;
    for (size_t r = 0; r < sp.recv_pe.size(); r++) {
      if (sp.recv_pe[r] != sp.rank) continue;
      const size_t cnt = (size_t)(sp.send_ptr[q + 1] - sp.send_ptr[q]) * nd;
      if (cnt)
        MB_CUDA_OK(cudaMemcpyAsync(rb + (size_t)sp.recv_ptr[r] * nd, sb + (size_t)sp.send_ptr[q] * nd,
                                   cnt * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
  }
  bool remote = false;
  for (int pe : sp.send_pe) remote = remote || pe != sp.rank;
  for (int pe : sp.recv_pe) remote = remote || pe != sp.rank;
  if (remote) {
    int rc = nccl_check(a.GroupStart(), "ncclGroupStart");
    for (size_t q = 0; !rc && q < sp.send_pe.size(); q++) {
      if (sp.send_pe[q] == sp.rank) continue;
      const size_t off = (size_t)sp.send_ptr[q] * nd, cnt = (size_t)(sp.send_ptr[q + 1] - sp.send_ptr[q]) * nd;
      rc = nccl_check(a.Send(sb + off, cnt, nccl_type<T>(), sp.send_pe[q], static_cast<ncclComm_t>(sp.comm), s),
                      "ncclSend");
    }
    for (size_t q = 0; !rc && q < sp.recv_pe.size(); q++) {
      if (sp.recv_pe[q] == sp.rank) continue;
      const size_t off = (size_t)sp.recv_ptr[q] * nd, cnt = (size_t)(sp.recv_ptr[q + 1] - sp.recv_ptr[q]) * nd;
      rc = nccl_check(a.Recv(rb + off, cnt, nccl_type<T>(), sp.recv_pe[q], static_cast<ncclComm_t>(sp.comm), s),
                      "ncclRecv");
    }
    const int rc2 = nccl_check(a.GroupEnd(), "ncclGroupEnd");
    if (rc || rc2) return rc ? rc : rc2;
  }
  if (sp.n_recv > 0) unpack_kernel<T><<<148 * 2, 256, 0, s>>>(v, sp.d_recv_item, sp.n_recv, nd, rb);
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}
}  // namespace

int shard_halo(const ShardPlan& sp, double* v, cudaStream_t s) { return halo_update<double>(sp, v, s); }
int shard_halo(const ShardPlan& sp, float* v, cudaStream_t s) { return halo_update<float>(sp, v, s); }

int shard_halo_fork(const ShardPlan& sp, double* v, cudaStream_t s) {
  MB_CUDA_OK(cudaEventRecord(sp.ev_fork, s));
  MB_CUDA_OK(cudaStreamWaitEvent(sp.side, sp.ev_fork, 0));
  const int rc = shard_halo(sp, v, sp.side);
  MB_CUDA_OK(cudaEventRecord(sp.ev_join, sp.side));
  return rc;
}

int shard_allreduce_fork(const ShardPlan& sp, double* d, int k, cudaStream_t s) {
  MB_CUDA_OK(cudaEventRecord(sp.ev_fork, s));
  MB_CUDA_OK(cudaStreamWaitEvent(sp.side, sp.ev_fork, 0));
  const int rc = shard_allreduce(sp, d, k, sp.side);
  MB_CUDA_OK(cudaEventRecord(sp.ev_join, sp.side));
  return rc;
}

int shard_halo_join(const ShardPlan& sp, cudaStream_t s) {
  MB_CUDA_OK(cudaStreamWaitEvent(s, sp.ev_join, 0));
  return kOk;
}

// In-place sum of k doubles over the ranks.
int shard_allreduce(const ShardPlan& sp, double* d, int k, cudaStream_t s) {
  return nccl_check(nccl().AllReduce(d, d, (size_t)k, ncclDouble, ncclSum, static_cast<ncclComm_t>(sp.comm), s),
                    "ncclAllReduce");
}

}  // namespace mb
