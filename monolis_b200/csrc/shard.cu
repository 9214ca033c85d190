// shard.cu -- the row-partitioned (multi-rank) solve: one process per GPU,
// each holding the rows it owns plus ghost columns, the layout of the
// reference's MPI runs (MONOLIS_COM tables: src/linalg/matvec.f90:144 updates
// the ghost entries of the multiplied vector, src/linalg/inner_product.f90:185
// sums the dot products over the ranks).
//
// Here the halo update is a pack kernel, NCCL send/receive pairs with every
// neighbour inside one NCCL group, and an unpack kernel; a dot product is the
// device-resident local sum followed by an NCCL all-reduce and a one-thread
// kernel that applies the scalar update with the global sums. Everything is
// enqueued on the solver stream, so it is captured in the solver's CUDA
// graphs like the rest of the iteration. Every rank evaluates the scalar
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

int shard_setup(ShardPlan& sp, const ShardTables& t, int ndof) {
  sp.ndof = ndof;
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
  return kOk;
}

void shard_free(ShardPlan& sp) {
  cudaFree(sp.d_send_item);
  cudaFree(sp.d_recv_item);
  cudaFree(sp.d_sendbuf);
  cudaFree(sp.d_recvbuf);
  sp = ShardPlan();
}

// Ghost entries of v (FP64, block rows of ndof) from their owners.
int shard_halo(const ShardPlan& sp, double* v, cudaStream_t s) {
  NcclApi& a = nccl();
  const int nd = sp.ndof;
  double* sb = static_cast<double*>(sp.d_sendbuf);
  double* rb = static_cast<double*>(sp.d_recvbuf);
  if (sp.n_send > 0) pack_kernel<double><<<148 * 2, 256, 0, s>>>(v, sp.d_send_item, sp.n_send, nd, sb);
  if (sp.n_send > 0 || sp.n_recv > 0) {
    int rc = nccl_check(a.GroupStart(), "ncclGroupStart");
    for (size_t q = 0; !rc && q < sp.send_pe.size(); q++) {
      const size_t off = (size_t)sp.send_ptr[q] * nd, cnt = (size_t)(sp.send_ptr[q + 1] - sp.send_ptr[q]) * nd;
      rc = nccl_check(a.Send(sb + off, cnt, ncclDouble, sp.send_pe[q], static_cast<ncclComm_t>(sp.comm), s),
                      "ncclSend");
    }
    for (size_t q = 0; !rc && q < sp.recv_pe.size(); q++) {
      const size_t off = (size_t)sp.recv_ptr[q] * nd, cnt = (size_t)(sp.recv_ptr[q + 1] - sp.recv_ptr[q]) * nd;
      rc = nccl_check(a.Recv(rb + off, cnt, ncclDouble, sp.recv_pe[q], static_cast<ncclComm_t>(sp.comm), s),
                      "ncclRecv");
    }
    const int rc2 = nccl_check(a.GroupEnd(), "ncclGroupEnd");
    if (rc || rc2) return rc ? rc : rc2;
  }
  if (sp.n_recv > 0) unpack_kernel<double><<<148 * 2, 256, 0, s>>>(v, sp.d_recv_item, sp.n_recv, nd, rb);
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}

// In-place sum of k doubles over the ranks.
int shard_allreduce(const ShardPlan& sp, double* d, int k, cudaStream_t s) {
  return nccl_check(nccl().AllReduce(d, d, (size_t)k, ncclDouble, ncclSum, static_cast<ncclComm_t>(sp.comm), s),
                    "ncclAllReduce");
}

}  // namespace mb
