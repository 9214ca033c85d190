// noalloc.cu -- inner product of two device vectors that allocates no memory.
//
// Who needs it: callers that cannot call cudaMalloc at the moment they need a
// dot product -- for example a host application that reserves all of the
// GPU's memory for its own pool at start-up (so any further cudaMalloc would
// fail), or a latency-critical loop that must not pay cudaMalloc's implicit
// device synchronisation. The regular device entry points of this library
// allocate their reduction scratch on first use; this one never does.
//
// How: the per-block partial sums and the arrival ticket of the one-pass
// grid reduction live in a file-scope device array of fixed size, created
// when the library is loaded and held by every GPU that loads it until the
// process exits. Host code cannot use the array's name as a device address,
// so on the first call on each device (with that device current) the
// address is fetched once with cudaGetSymbolAddress and cached; that first
// call should therefore come before any stream capture.
#include <cstdio>
#include <mutex>

#include "common.cuh"

namespace mb {
namespace {

// Capacity: one partial sum per block (plus one per group of blocks), blocks of 256 threads each reducing
// 4 elements per thread -> at most kNoAllocBlocks * 1024 elements.
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocPerThread = 4;
constexpr int kNoAllocBlocks = 16384;
constexpr long long kNoAllocMaxN = (long long)kNoAllocBlocks * kNoAllocThreads * kNoAllocPerThread;

struct NoAllocScratch {
  double partials[kNoAllocBlocks + kNoAllocBlocks / kReduceGroup];  // block and group partial sums
  unsigned int ticket[1 + kNoAllocBlocks / kReduceGroup];           // arrival tickets
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_mu;
NoAllocScratch* g_addr[kMaxDevices] = {nullptr};

__global__ void dot_noalloc_kernel(long long n, const double* __restrict__ x, const double* __restrict__ y,
                                   NoAllocScratch* sc, double* out) {
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[0] += x[i] * y[i];
  grid_reduce<1>(v, sc->partials, sc->ticket, [&](double* tot) { *out = tot[0]; });
}

}  // namespace
}  // namespace mb

extern "C" int monolis_b200_inner_product_noalloc_R(long long n, const double* d_x, const double* d_y, double* d_sum,
                                                    void* stream) {
  using namespace mb;
  if (n < 0 || n > kNoAllocMaxN) {
    fprintf(stderr,
            "** monolis_b200_inner_product_noalloc_R: n = %lld exceeds the fixed scratch capacity "
            "(at most %lld elements)\n",
            n, kNoAllocMaxN);
    return kBadInput;
  }
  if (!d_sum || (n > 0 && (!d_x || !d_y))) return kBadInput;
  int dev = 0;
  MB_CUDA_OK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return kBadInput;
  NoAllocScratch* sc = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      // once per device, with that device current
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return report_cuda(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
      g_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    sc = g_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the arrival tickets must start at zero (a previous call leaves them at
  // zero; clearing them again costs nothing and recovers from an aborted call)
  MB_CUDA_OK(cudaMemsetAsync(sc->ticket, 0, sizeof(sc->ticket), s));
  long long blocks = (n + (long long)kNoAllocThreads * kNoAllocPerThread - 1) / ((long long)kNoAllocThreads * kNoAllocPerThread);
  if (blocks < 1) blocks = 1;
  dot_noalloc_kernel<<<(int)blocks, kNoAllocThreads, 0, s>>>(n, d_x, d_y, sc, d_sum);
  MB_CUDA_OK(cudaGetLastError());
  return kOk;
}
