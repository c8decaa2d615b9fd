// Per-device context, device allocation accounting and error reporting.
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "bulk.cuh"
#include "common.cuh"

namespace hb {

namespace {
thread_local char g_last_error[512] = "";
Context* g_ctx[64] = {nullptr};
std::mutex g_ctx_mu;
size_t g_budget = 0;        // 0 = unlimited
size_t g_allocated = 0;
bool g_budget_read = false;

size_t budget() {
  if (!g_budget_read) {
    g_budget_read = true;
    const char* s = std::getenv("HPCG_B200_DEVICE_BUDGET");
    if (s && *s) g_budget = (size_t)std::strtoull(s, nullptr, 10);
  }
  return g_budget;
}
}  // namespace

void set_error(const char* what, cudaError_t e) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
}

void set_error_text(const char* msg) { std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg); }

int status_of(cudaError_t e) {
  return e == cudaErrorMemoryAllocation ? HPCG_B200_ERR_NOMEM : HPCG_B200_ERR_CUDA;
}

int dev_alloc(void** ptr, size_t bytes, size_t* counter) {
  *ptr = nullptr;
  if (bytes == 0) return HPCG_B200_OK;
  const size_t lim = budget();
  if (lim && g_allocated + bytes > lim) {
    std::snprintf(g_last_error, sizeof(g_last_error), "device budget of %zu bytes exceeded (%zu requested)",
                  lim, g_allocated + bytes);
    return HPCG_B200_ERR_NOMEM;
  }
  HB_CK(cudaMalloc(ptr, bytes));
  g_allocated += bytes;
  if (counter) *counter += bytes;
  return HPCG_B200_OK;
}

// The budget counter is released by the owner of the allocations (free_problem).
void dev_free(void* ptr) {
  if (ptr) cudaFree(ptr);
}

void release_accounted(size_t bytes) { g_allocated = bytes > g_allocated ? 0 : g_allocated - bytes; }

int locate_ptr(const void* ptr, int device, bool* on_device, const char* what) {
  *on_device = false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();  // plain pageable host memory on older runtimes
    return HPCG_B200_OK;
  }
  if (a.type == cudaMemoryTypeManaged) {
    *on_device = true;
    return HPCG_B200_OK;
  }
  if (a.type != cudaMemoryTypeDevice) return HPCG_B200_OK;  // pinned or registered host memory
  if (a.device != device) {
    std::snprintf(g_last_error, sizeof(g_last_error),
                  "%s: a pointer to device memory of GPU %d was passed to a call on GPU %d", what, a.device, device);
    return HPCG_B200_ERR_ARG;
  }
  *on_device = true;
  return HPCG_B200_OK;
}

Context* context_for(int device) {
  if (device < 0 || device >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(g_ctx_mu);
  if (g_ctx[device]) return g_ctx[device];
  Context* c = new Context;
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  // a blocking stream: ordered with work on the legacy default stream (where
  // callers such as torch write the device vectors they pass in)
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault);
  if (e == cudaSuccess) e = cudaMalloc(&c->partials, sizeof(double) * kRedBlocksMax);
  if (e == cudaSuccess) e = cudaMalloc(&c->scal, sizeof(Scalars));
  if (e == cudaSuccess) e = cudaMemset(c->scal, 0, sizeof(Scalars));
  if (e == cudaSuccess) e = cudaMallocHost(&c->scal_host, sizeof(Scalars));
  if (e == cudaSuccess) e = cudaHostAlloc(&c->fault, sizeof(unsigned), cudaHostAllocMapped);
  if (e == cudaSuccess) *c->fault = 0;
  if (e != cudaSuccess) {
    set_error("context set-up", e);
    if (c->stream) cudaStreamDestroy(c->stream);
    cudaFree(c->partials);
    cudaFree(c->scal);
    delete c;
    return nullptr;
  }
  g_ctx[device] = c;
  return c;
}

Context* current_context() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("cudaGetDevice", e);
    return nullptr;
  }
  return context_for(dev);
}

int ensure_stage(Context* c, size_t n) {
  if (n <= c->stage_cap) return HPCG_B200_OK;
  for (int i = 0; i < 3; ++i) {
    cudaFree(c->stage[i]);
    c->stage[i] = nullptr;
  }
  c->stage_cap = 0;
  for (int i = 0; i < 3; ++i) HB_CK(cudaMalloc(&c->stage[i], n * sizeof(double)));
  c->stage_cap = n;
  return HPCG_B200_OK;
}

// ---- host memory <-> device through pinned chunks ----------------------------
// A copy from or to pageable host memory runs through the driver's own bounce
// buffers at a fraction of the link's speed. Large ones go through the
// context's two pinned chunks instead, double-buffered: host threads copy
// chunk i between the caller's memory and one pinned chunk while the copy
// engine moves the neighbouring chunk through the other. Pinned host memory,
// and copies of under kPinMin entries, go directly.
namespace {
constexpr size_t kPinChunk = (size_t)1 << 23;  // doubles per chunk (64 MB)
constexpr size_t kPinMin = (size_t)1 << 20;

bool pageable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

int ensure_pin(Context* c) {
  if (c->pin[0]) return HPCG_B200_OK;
  for (int i = 0; i < 2; ++i) {
    HB_CK(cudaMallocHost(&c->pin[i], kPinChunk * sizeof(double)));
    HB_CK(cudaEventCreateWithFlags(&c->pin_ev[i], cudaEventDisableTiming));
    HB_CK(cudaEventRecord(c->pin_ev[i], c->stream));
  }
  return HPCG_B200_OK;
}

void host_copy(double* dst, const double* src, size_t n) {
  host_parallel((int64_t)n, [&](int64_t lo, int64_t hi) {
    std::memcpy(dst + lo, src + lo, sizeof(double) * (size_t)(hi - lo));
  });
}
}  // namespace

int host_to_device(Context* c, double* dst, const double* src, size_t n) {
  if (n < kPinMin || !pageable(src)) {
    HB_CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    return HPCG_B200_OK;
  }
  HB_TRY(ensure_pin(c));
  for (size_t off = 0, i = 0; off < n; off += kPinChunk, ++i) {
    const size_t len = std::min(kPinChunk, n - off);
    const int b = (int)(i & 1);
    HB_CK(cudaEventSynchronize(c->pin_ev[b]));  // the copy engine is done with this chunk's last use
    host_copy(c->pin[b], src + off, len);
    HB_CK(cudaMemcpyAsync(dst + off, c->pin[b], sizeof(double) * len, cudaMemcpyHostToDevice, c->stream));
    HB_CK(cudaEventRecord(c->pin_ev[b], c->stream));
  }
  return HPCG_B200_OK;
}

int device_to_host(Context* c, double* dst, const double* src, size_t n) {
  if (n < kPinMin || !pageable(dst)) {
    HB_CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    HB_CK(cudaStreamSynchronize(c->stream));
    return HPCG_B200_OK;
  }
  HB_TRY(ensure_pin(c));
  const size_t chunks = (n + kPinChunk - 1) / kPinChunk;
  auto issue = [&](size_t i) -> int {
    const size_t off = i * kPinChunk, len = std::min(kPinChunk, n - off);
    HB_CK(cudaMemcpyAsync(c->pin[i & 1], src + off, sizeof(double) * len, cudaMemcpyDeviceToHost, c->stream));
    HB_CK(cudaEventRecord(c->pin_ev[i & 1], c->stream));
    return HPCG_B200_OK;
  };
  HB_TRY(issue(0));
  for (size_t i = 0; i < chunks; ++i) {
    if (i + 1 < chunks) HB_TRY(issue(i + 1));  // the other chunk is free: its host copy finished below
    HB_CK(cudaEventSynchronize(c->pin_ev[i & 1]));
    const size_t off = i * kPinChunk;
    host_copy(dst + off, c->pin[i & 1], std::min(kPinChunk, n - off));
  }
  return HPCG_B200_OK;
}

// cuTensorMapEncodeTiled, looked up once through the runtime (no link to the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
    else
      cudaGetLastError();
  }
  return fn;
}

// 2-D map of one slot-major array: x = row (pitch entries, the row stride), y =
// slot (27); box kBulkRows x 27.
static bool encode_slot_major(CUtensorMap* m, CUtensorMapDataType type, size_t esize, const void* base, int64_t pitch) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)pitch, (cuuint64_t)kSlots};
  const cuuint64_t strides[1] = {(cuuint64_t)pitch * esize};
  const cuuint32_t box[2] = {(cuuint32_t)kBulkRows, (cuuint32_t)kSlots};
  const cuuint32_t elem[2] = {1, 1};
  return fn(m, type, 2, const_cast<void*>(base), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The level's FP64 tensor maps (built on first use, rebuilt if the arrays moved);
// nullptr if they cannot be encoded.
const BulkMaps* bulk_maps(const Level& L) {
  if (!L.maps) L.maps = new BulkMaps();
  BulkMaps* m = L.maps;
  if (m->val_ptr != L.val || m->col_ptr != L.col) {
    m->ok = encode_slot_major(&m->val, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, sizeof(double), L.val, L.pitch) &&
            encode_slot_major(&m->col, CU_TENSOR_MAP_DATA_TYPE_INT32, sizeof(int), L.col, L.pitch);
    m->val_ptr = L.val;
    m->col_ptr = L.col;
  }
  return m->ok ? m : nullptr;
}

int stream_sync(Context* c) {
  HB_CK(cudaStreamSynchronize(c->stream));
  volatile unsigned* f = c->fault;
  if (f && *f) {
    const unsigned code = *f;
    *f = 0;
    set_error_text(code == 5   ? "a device-side wait gave up (bounded wait at the batched iteration's grid barrier)"
                   : code == 6 ? "a device-side wait gave up (bounded wait of a wavefront sweep on its dependencies)"
                               : "a device-side wait gave up (bounded mbarrier wait of the bulk-copy pipeline)");
    return HPCG_B200_ERR_TIMEOUT;
  }
  return HPCG_B200_OK;
}

namespace {
int take_event(Context* c, cudaEvent_t* e) {
  if (!c->ev_pool.empty()) {
    *e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return HPCG_B200_OK;
  }
  HB_CK(cudaEventCreate(e));
  return HPCG_B200_OK;
}
}  // namespace

int prof_begin(Context* c, int kind, cudaEvent_t* start) {
  *start = nullptr;
  if (!c->prof || kind < 0 || kind >= kProfKinds) return HPCG_B200_OK;
  HB_TRY(take_event(c, start));
  HB_CK(cudaEventRecord(*start, c->stream));
  return HPCG_B200_OK;
}

int prof_end(Context* c, int kind, cudaEvent_t start, int64_t rows) {
  if (!start) return HPCG_B200_OK;
  cudaEvent_t stop;
  HB_TRY(take_event(c, &stop));
  HB_CK(cudaEventRecord(stop, c->stream));
  c->ev_open[kind].push_back(std::make_pair(start, stop));
  c->prof_rows[kind] += rows;
  return HPCG_B200_OK;
}

int prof_flush(Context* c) {
  bool any = false;
  for (int k = 0; k < kProfKinds; ++k) any = any || !c->ev_open[k].empty();
  if (!any) return HPCG_B200_OK;
  HB_CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < kProfKinds; ++k) {
    for (auto& pr : c->ev_open[k]) {
      float ms = 0.f;
      HB_CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
      c->prof_ms[k] += ms;
      c->prof_launches[k] += 1;
      c->ev_pool.push_back(pr.first);
      c->ev_pool.push_back(pr.second);
    }
    c->ev_open[k].clear();
  }
  return HPCG_B200_OK;
}

}  // namespace hb

using namespace hb;

extern "C" {

const char* hpcg_b200_last_error(void) { return hb::g_last_error; }

void* hpcg_b200_stream(int device) {
  Context* c = context_for(device);
  return c ? (void*)c->stream : nullptr;
}

int hpcg_b200_profile(int device, int enable) {
  Context* c = context_for(device);
  if (!c) return HPCG_B200_ERR_CUDA;
  HB_TRY(prof_flush(c));
  c->prof = enable != 0;
  for (int k = 0; k < kProfKinds; ++k) {
    c->prof_ms[k] = 0;
    c->prof_launches[k] = 0;
    c->prof_rows[k] = 0;
  }
  return HPCG_B200_OK;
}

int hpcg_b200_profile_read(int device, int kind, double* total_ms, int64_t* launches, int64_t* rows) {
  Context* c = context_for(device);
  if (!c) return HPCG_B200_ERR_CUDA;
  if (kind < 0 || kind >= kProfKinds) return HPCG_B200_ERR_ARG;
  HB_TRY(prof_flush(c));
  if (total_ms) *total_ms = c->prof_ms[kind];
  if (launches) *launches = c->prof_launches[kind];
  if (rows) *rows = c->prof_rows[kind];
  return HPCG_B200_OK;
}

}  // extern "C"
