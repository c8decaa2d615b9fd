// hpcg_b200_dot_noalloc: the dot product x'y for callers that cannot allocate
// device memory.
//
// Who needs it. Some callers have handed all of a GPU's memory to their own
// allocator, or run a phase in which a device allocation is not allowed:
//  - a solver sized to fill HBM (HPCG asks for at least a quarter of memory;
//    a 512^3 problem plus its hierarchy takes ~70 GB) whose host reserved the
//    rest for other work;
//  - frameworks whose caching allocator owns the memory pool;
//  - timed inner loops, where a cudaMalloc or cudaFree would also synchronise
//    the whole device.
// hpcg_b200_dot allocates: its per-device context (reduction partials,
// staging for host vectors) is created with cudaMalloc on first use. This entry
// point takes device vectors and writes the result to device memory, and its
// only scratch is a fixed array that is part of the library image itself.
//
// Scratch. g_noalloc_partials below holds one partial sum per block of
// kChunk entries. It is a file-scope __device__ array, so every GPU that loads
// this library holds its 512 KiB from load until process exit, whether or not
// the entry point is called. That fixes the largest vector length at
// kChunk * kMaxPartials = 2^28 entries; longer vectors are rejected.
//
// Set-up. Host code cannot take the address of a __device__ array directly:
// the name only stands for it on the host. The first call on each device (with
// that device current) looks the address up with cudaGetSymbolAddress and
// keeps it; make that first call before any stream capture on the device. The
// kept address belongs to the device's context as it was then: after a
// cudaDeviceReset on that device, do not call this entry point again in the
// same process.
//
// Sharing. All calls on a device share the one array and it keeps the last
// call's contents. Nothing in it has to start at zero: each call's first
// kernel writes every partial its second kernel reads. Calls that overlap on
// the GPU (on different streams, or from different host threads) race on the
// array and may return wrong sums; serialise them.
#include <cstdio>
#include <mutex>

#include "common.cuh"

namespace hb {
void set_error_text(const char* msg);
}

namespace {

constexpr int kNaThreads = 256;
constexpr int kChunk = 4096;               // entries summed by one block
constexpr int kMaxPartials = 65536;        // capacity of the scratch array (512 KiB)
constexpr long long kMaxN = (long long)kChunk * kMaxPartials;  // 2^28 entries

static __device__ __align__(256) double g_noalloc_partials[kMaxPartials];

void* g_partials[64] = {nullptr};  // device address of g_noalloc_partials, per device
std::mutex g_partials_mu;

// Block sum with a fixed shuffle tree (valid in thread 0).
__device__ __forceinline__ double na_block_sum(double v) {
  __shared__ double warp_part[kNaThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_part[w] = v;
  __syncthreads();
  double s = 0.0;
  if (w == 0) {
    s = lane < kNaThreads / 32 ? warp_part[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;
}

// Block b sums x[i] * y[i] over its chunk [b * kChunk, (b+1) * kChunk) with a
// fixed thread order and shuffle tree, so the result depends only on n.
__global__ void __launch_bounds__(kNaThreads) k_na_partials(int n, const double* __restrict__ x,
                                                             const double* __restrict__ y,
                                                             double* __restrict__ partials) {
  const long long begin = (long long)blockIdx.x * kChunk;
  const long long end = begin + kChunk < n ? begin + kChunk : n;
  double acc = 0.0;
  for (long long i = begin + threadIdx.x; i < end; i += blockDim.x) acc += x[i] * y[i];
  const double s = na_block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kNaThreads) k_na_final(const double* __restrict__ partials, int np,
                                                          double* __restrict__ result) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
  const double s = na_block_sum(acc);
  if (threadIdx.x == 0) *result = s;
}

int scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    hb::set_error("cudaGetDevice", e);
    return hb::status_of(e);
  }
  if (dev < 0 || dev >= 64) {
    hb::set_error_text("hpcg_b200_dot_noalloc: device ordinals of 64 and above are not supported");
    return HPCG_B200_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_partials_mu);
  if (!g_partials[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) {
      hb::set_error("cudaGetSymbolAddress(g_noalloc_partials)", e);
      return hb::status_of(e);
    }
    g_partials[dev] = p;
  }
  *out = static_cast<double*>(g_partials[dev]);
  return HPCG_B200_OK;
}

}  // namespace

extern "C" int hpcg_b200_dot_noalloc(int n, const double* x, const double* y, double* result, void* stream) {
  if (n < 0 || (long long)n > kMaxN) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "hpcg_b200_dot_noalloc: n = %d outside [0, %lld] (fixed scratch of %d partials)",
                  n, kMaxN, kMaxPartials);
    hb::set_error_text(msg);
    return HPCG_B200_ERR_ARG;
  }
  if (!x || !y || !result) {
    hb::set_error_text("hpcg_b200_dot_noalloc: x, y and result must be device memory of the current GPU");
    return HPCG_B200_ERR_ARG;
  }
  int cur = 0;
  const cudaError_t ge = cudaGetDevice(&cur);
  if (ge != cudaSuccess) {
    hb::set_error("cudaGetDevice", ge);
    return hb::status_of(ge);
  }
  // device memory of the current GPU only: host memory, and another GPU's
  // memory (which locate_ptr refuses with its own message), are not accepted
  const void* args[3] = {x, y, result};
  for (const void* a : args) {
    bool on_device = false;
    const int st = hb::locate_ptr(a, cur, &on_device, "hpcg_b200_dot_noalloc");
    if (st != HPCG_B200_OK) return st;
    if (!on_device) {
      hb::set_error_text("hpcg_b200_dot_noalloc: x, y and result must be device memory of the current GPU");
      return HPCG_B200_ERR_ARG;
    }
  }
  double* partials = nullptr;
  const int s = scratch_address(&partials);
  if (s != HPCG_B200_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int np = (int)((n + (long long)kChunk - 1) / kChunk);
  if (np > 0) k_na_partials<<<np, kNaThreads, 0, st>>>(n, x, y, partials);
  k_na_final<<<1, kNaThreads, 0, st>>>(partials, np, result);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    hb::set_error("hpcg_b200_dot_noalloc launch", e);
    return hb::status_of(e);
  }
  return HPCG_B200_OK;
}
