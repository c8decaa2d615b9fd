// Internal definitions shared by the translation units of libhpcg_b200.so.
//
// Device layout of one grid level (all in HBM, allocated once at set-up):
//   - rows are renumbered into 8 colour blocks by the parity of (ix, iy, iz); the
//     blocks are stored in sweep order, natural order inside a block;
//   - the matrix is a 27-slot ELL stored slot-major: val[k*pitch + q], col[k*pitch + q]
//     for slot k = (sz+1)*9 + (sy+1)*3 + (sx+1), the stencil direction, so slot 13 is
//     the diagonal and the slot order is the reference's entry order
//     (GenerateProblem_ref.cpp:152-172); a direction that leaves the grid holds
//     val = 0 and col = n + next, the index of a permanently zero vector entry;
//   - a rank of a run over several GPUs also references `next` external columns,
//     the halo values of its neighbours, stored at [n, n + next) of every vector
//     the matrix multiplies (refreshed by the halo exchange);
//   - every colour-order vector has `pitch` >= n+next+1 entries, entry n+next always 0.
#pragma once

#include <cuda.h>  // CUtensorMap (encoded through the runtime's driver entry point)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <utility>
#include <vector>

#include "hpcg_b200.h"

namespace hb {

constexpr int kSlots = 27;
constexpr int kDiagSlot = 13;
constexpr int kColours = 8;
constexpr int kMaxLevels = 4;
constexpr uint64_t kMagic = 0x48504347b2000001ull;  // "HPCG" + version

// Rows per block of the FP32 V-cycle's matrix copy (see mat_index): one tile of
// the bulk-copy Gauss-Seidel phases, so that a tile's values and columns are
// two runs of memory (two copies).
constexpr int kRowBlock32 = 128;

// Position of slot k of row q in a level's matrix arrays (values and columns).
// The FP64 arrays are slot-major: 27 runs of `pitch` entries, so a warp's 32
// rows read one coalesced run of a slot. The FP32 copy of the V-cycle (values
// and its own columns) is stored in blocks of kRowBlock32 rows, each block
// holding its 27 slots one after another: a warp still reads one coalesced run,
// and an FP32 phase streams one run of memory per array instead of 27 far
// apart. Measured at 512^3: the FP32 phases 17% faster than slot-major (as fast
// with 128-row as with 1024-row blocks), while the same blocking made the FP64
// phases 20% slower.
// B: rows per block, 0 for slot-major (the default for FP64; the batched path's
// FP32 copy and the multi-system path's FP64 copy choose their own).
template <typename T, int B = (sizeof(T) == 4 ? kRowBlock32 : 0)>
__host__ __device__ __forceinline__ int64_t mat_index(int k, int64_t q, int64_t pitch) {
  if constexpr (B > 0)
    return ((q / B) * kSlots + k) * B + (q % B);
  else
    return (int64_t)k * pitch + q;
}

// Entries of a matrix array of a level with `pitch` in blocks of `rows` rows.
inline int64_t blocked_entries(int64_t pitch, int rows) { return (pitch + rows - 1) / rows * rows * kSlots; }

// Parity colours in sweep order. The injected (f2c) points, parity colour 0
// (all coordinates even), are swept last in the forward sweep: swept first they
// would overwrite the prolonged coarse correction before any other row reads
// it, and swept last in the backward sweep (i.e. first in the forward sweep) they
// would hold a zero residual, so restriction would pass nothing down.
constexpr int kSweepDefault[kColours] = {7, 6, 3, 5, 4, 1, 2, 0};

// The parity bit pattern a stencil direction flips: bit0 for sx = +-1, bit1 for sy, bit2 for sz.
__host__ __device__ constexpr int slot_flip(int k) {
  const int sx = k % 3 - 1, sy = (k / 3) % 3 - 1, sz = k / 9 - 1;
  return (sx != 0 ? 1 : 0) | (sy != 0 ? 2 : 0) | (sz != 0 ? 4 : 0);
}

// Geometry of the colour ordering of one (nx, ny, nz) grid.
struct ColourGrid {
  int nx, ny, nz;
  int sweep[kColours];   // parity colour at sweep position s
  int pos[kColours];     // sweep position of parity colour c
  int start[kColours + 1];  // first colour-order row of sweep position s

  // points with ix parity b: ix = b, b+2, ... < nx
  __host__ __device__ static int half(int n, int b) { return (n - b + 1) / 2; }

  __host__ void init(int nx_, int ny_, int nz_, const int* sweep_order) {
    nx = nx_; ny = ny_; nz = nz_;
    for (int s = 0; s < kColours; ++s) { sweep[s] = sweep_order[s]; pos[sweep_order[s]] = s; }
    start[0] = 0;
    for (int s = 0; s < kColours; ++s) {
      const int c = sweep[s];
      start[s + 1] = start[s] + half(nx, c & 1) * half(ny, (c >> 1) & 1) * half(nz, (c >> 2) & 1);
    }
  }

  // natural row of (ix, iy, iz) -> colour-order row
  __host__ __device__ int old2new(int ix, int iy, int iz) const {
    const int c = (ix & 1) | ((iy & 1) << 1) | ((iz & 1) << 2);
    const int hx = half(nx, c & 1), hy = half(ny, (c >> 1) & 1);
    return start[pos[c]] + ((iz >> 1) * hy + (iy >> 1)) * hx + (ix >> 1);
  }

  // colour-order row -> (ix, iy, iz)
  __host__ __device__ void coords(int q, int& ix, int& iy, int& iz) const {
    int s = 0;
    while (s + 1 < kColours && q >= start[s + 1]) ++s;
    const int c = sweep[s];
    const int hx = half(nx, c & 1), hy = half(ny, (c >> 1) & 1);
    const int m = q - start[s];
    ix = 2 * (m % hx) + (c & 1);
    iy = 2 * ((m / hx) % hy) + ((c >> 1) & 1);
    iz = 2 * (m / (hx * hy)) + ((c >> 2) & 1);
  }
};

// Slots read by a first-sweep colour phase: neighbours of colours swept
// earlier in this sweep. All others (and the diagonal) multiply x = 0.
inline uint32_t first_mask(const ColourGrid& g, int s) {
  const int c = g.sweep[s];
  uint32_t m = 0;
  for (int k = 0; k < kSlots; ++k) {
    if (k == kDiagSlot) continue;
    if (g.pos[c ^ slot_flip(k)] < s) m |= 1u << k;
  }
  return m;
}

// The same mask for the default sweep order, at compile time (the mask depends
// only on the sweep order and the colour parities, not on the grid).
constexpr uint32_t first_mask_default(int s) {
  int pos[kColours] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < kColours; ++i) pos[kSweepDefault[i]] = i;
  const int c = kSweepDefault[s];
  uint32_t m = 0;
  for (int k = 0; k < kSlots; ++k) {
    if (k == kDiagSlot) continue;
    if (pos[c ^ slot_flip(k)] < s) m |= 1u << k;
  }
  return m;
}

// Halo exchange plan of one level of one rank (the data SetupHalo_ref.cpp:121-172
// builds): neighbours in ascending rank order; neighbour i's externals are
// entries [n + off[i], n + off[i+1]) and the rows sent to it are
// send_rows[off[i] .. off[i+1]) (the stencil is symmetric, so a rank sends a
// neighbour as many entries as it receives from it). Both lists are in
// ascending global row order, so they pair up across ranks.
struct HaloPlan {
  int nnb = 0;
  int nbr[26];                 // neighbour ranks, ascending
  int dir[26];                 // their directions (dz+1)*9 + (dy+1)*3 + (dx+1)
  int off[27];                 // entry offsets per neighbour, off[nnb] = total
  int ext_off[27];             // by direction: offset of that neighbour's externals, -1 if none
  int total = 0;
  int* send_rows = nullptr;    // device [total], colour-order rows
  double* send_buf = nullptr;  // device [total]
};

// Position of one rank in the reference's process grid (GenerateGeometry.cpp:89-91).
struct RankGeom {
  int size = 1, rank = 0;
  int npx = 1, npy = 1, npz = 1;
  int ipx = 0, ipy = 0, ipz = 0;
};

// Tensor maps of a level's FP64 matrix arrays for the bulk-copy Gauss-Seidel
// phases: 2-D (x = row over the pitch, y = slot), box kBulkRows x 27.
struct BulkMaps {
  CUtensorMap val;
  CUtensorMap col;
  const void* val_ptr = nullptr;  // the arrays they describe
  const void* col_ptr = nullptr;
  bool ok = false;                // encoded (false: the encoder is unavailable)
};

// The shape of one wavefront sweep of a level (wave.cuh).
struct WaveGeom {
  int H;         // z pairs
  int P;         // phases of the sweep (8 forward, 7 backward)
  int lag;       // z pairs between consecutive phases
  int tpu;       // tiles per unit: (nx/2)(ny/2) / kBulkRows
  int per;       // rows per unit: (nx/2)(ny/2)
  int dot_from;  // phases j >= dot_from add r'x to the partials (P: none)
  int self_dep;  // >= 0: every unit waits for this virtual unit (the bounded-wait check); -1 normally
  int start[kColours];  // first row of phase j's colour block
};

struct Level {
  ColourGrid g;
  int n = 0;                 // rows
  int next = 0;              // external columns (halo), 0 on a single rank
  HaloPlan* halo = nullptr;  // exchange plan (ranks with neighbours only)
  int64_t pitch = 0;         // slot stride (>= n+next+1, multiple of 256)
  double* val = nullptr;     // [27][pitch]
  int* col = nullptr;        // [27][pitch]
  float* val32 = nullptr;    // FP32 copy for the mixed-precision V-cycle (built on first use), blocked
  int* col32 = nullptr;      // its columns in the same blocked layout (mat_index<float>)
  int* new2old = nullptr;    // [n] colour row -> natural row
  int* old2new = nullptr;    // [n]
  int* f2c = nullptr;        // [n of next level] coarse colour row -> fine colour row
  int* tf = nullptr;         // transfer pairs (fine row, coarse row) sorted by fine row:
  int* tq = nullptr;         //   tf[t] = f2c[tq[t]], tf increasing
  int tf_run = -1;           // f0 if tf[t] = f0 + t for every t (one run of fine rows), else -1
  double* r = nullptr;       // coarse right-hand side (levels > 0), [pitch]
  double* x = nullptr;       // coarse solution (levels > 0), [pitch]
  float* r32 = nullptr;      // FP32 V-cycle vectors, [pitch]
  float* x32 = nullptr;
  // kernel configuration of this level's row kernels, chosen by the autotuner
  int gs_sched = 1;          // kernel configuration of the Gauss-Seidel phases (FP64)
  int gs_sched32 = 1;        // kernel configuration of the Gauss-Seidel phases (FP32 V-cycle)
  int gs_first32 = 1;        // ... of its first-sweep phases
  int gs_first = 1;          // kernel configuration of the first-sweep phases (FP64)
  // the first-sweep configuration per sweep position, tuned position by
  // position (a phase reads 0 to 26 slots by its position); -1: gs_first /
  // gs_first32 at every position
  int gs_first_at[kColours] = {-1, -1, -1, -1, -1, -1, -1, -1};
  int gs_first32_at[kColours] = {-1, -1, -1, -1, -1, -1, -1, -1};
  int mv_sched = 1;          // kernel configuration of SpMV / restriction
  int mv_order = 0;          // SpMV row order: 0 storage, 1 natural, 2 slab (see k_spmv)
  bool tuned = false;
  // level-scheduled natural order (built on first use)
  int* wave_rows = nullptr;  // colour-order rows sorted by ix + 2 iy + 4 iz
  int nwaves = 0;
  int* wave_start = nullptr; // host array [nwaves+1]
  mutable BulkMaps* maps = nullptr;  // host; built on the first bulk-copy phase
  // the columns packed for the bulk-copy kernels (one record per 128-row tile:
  // 27 bases and offsets of `pack` bytes), nullptr (pack 0) if they do not pack
  unsigned char* colp = nullptr;
  int pack = 0;
  // wavefront sweeps (wave.cuh): the geometry of the forward and the backward
  // sweep, tiles per unit (0: not set up yet, -1: the level does not cut into
  // whole-tile units), the per-unit counters of finished tiles (device); wf:
  // the sweeps that do not start from x = 0 run as one launch each
  // (HPCG_B200_WAVE or the level's configuration string; off by default)
  WaveGeom wf_geom[2] = {};
  int wf_tpu = 0;
  unsigned* wf_done = nullptr;
  int wf = 0;
};

struct Context;
struct MultiState;
struct Comm;

}  // namespace hb

struct hpcg_b200_problem {
  uint64_t magic;
  int device;
  hb::Context* ctx;
  int nlev;
  hb::Level lev[hb::kMaxLevels];
  int symgs_mode;
  // level-0 vectors, colour order, [pitch] each
  double *b, *x, *r, *z, *p, *Ap, *zprev;
  hb::MultiState* multi;  // work vectors of the multi-system path (created on first use)
  cudaGraphExec_t cg_graph[2];  // instantiated CG loop, [unpreconditioned, preconditioned]
  bool cg_graph_failed;         // capture was refused once: stay with stream launches
  cudaGraphExec_t coarse_graph[2];  // the V-cycle below level 0 as one graph, [FP64, FP32]
  bool coarse_graph_failed;         // its capture was refused once: stream launches
  hb::RankGeom* geom;  // position in a run over several ranks (nullptr: one rank)
  size_t bytes;  // device bytes held
  // hpcg_b200_cg's host right-hand side as last sent (a host copy of n entries)
  // and whether b still holds it (every other load into b clears the flag)
  double* b_kept_host;
  bool b_kept;
  int host_reuse;  // hpcg_b200_cg may skip sending an unchanged b and a zero x (hpcg_b200_set_host_reuse)
};

namespace hb {

// ---- error plumbing ------------------------------------------------------
void set_error(const char* what, cudaError_t e);
int status_of(cudaError_t e);

#define HB_CK(call)                                   \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) {                          \
      ::hb::set_error(#call, e_);                     \
      return ::hb::status_of(e_);                     \
    }                                                 \
  } while (0)

#define HB_TRY(call)                 \
  do {                               \
    int s_ = (call);                 \
    if (s_ != HPCG_B200_OK) return s_; \
  } while (0)

// ---- per-device context ------------------------------------------------------
constexpr int kRedBlocksMax = 16384;  // reduction partial slots
// Partial slots per colour position of the Gauss-Seidel phases that also reduce
// r'z (kColours * kDotStride <= kRedBlocksMax); a phase's grid is capped to it.
constexpr int kDotStride = 2048;

struct Scalars {
  double rtz, oldrtz, alpha, beta, pAp, normr2, rzprev, tmp;
  // loop state of the graph-launched CG (CG.cpp:100's condition on the device)
  double normr0, tol;
  int iter;      // iterations completed
  int max_iter;
};

// Scalar updates that close a reduction (k_finalize and its rank-order twin).
enum FinOp : int {
  kFinStore = 0,     // *out = sum
  kFinNormr = 1,     // s->normr2 = sum
  kFinRtzFirst = 2,  // s->rtz = sum
  kFinRtz = 3,       // oldrtz = rtz; rtz = sum; beta = rtz / oldrtz   (CG.cpp:112-114)
  kFinPap = 4,       // pAp = sum; alpha = rtz / pAp                    (CG.cpp:119-120)
  kFinFlex = 5,      // oldrtz = rtz; rtz = sum; beta = (rtz - sum2) / oldrtz (flexible PR)
  kFinMax = 6,       // *out = max of partials
  kFinNormr0 = 7,    // normr2 = sum; normr0 = sqrt(sum)           (CG.cpp:89-96)
  kFinRtzIter = 8,   // iteration 1: rtz = sum; later: as kFinRtz  (CG.cpp:107-115)
};

// Kernel classes timed by the optional launch profiler.
enum ProfKind : int {
  kProfGsFull = 0,   // Gauss-Seidel colour phase on level 0, all 27 slots
  kProfGsFirst = 1,  // first forward sweep on level 0 (x = 0, masked slots)
  kProfSpmv = 2,     // CG SpMV + p'Ap on level 0
  kProfRestrict = 3, // residual + restriction, level 0 -> 1
  kProfGs32Full = 4,   // FP32 V-cycle: Gauss-Seidel colour phase on level 0, all 27 slots
  kProfGs32First = 5,  // FP32 V-cycle: first forward sweep on level 0
  kProfGsSweep = 6,    // a whole Gauss-Seidel sweep on level 0 in one launch (wave.cuh)
  kProfKinds = 7,
};

struct Context {
  int device = -1;
  int sms = 0;
  cudaStream_t stream = nullptr;
  double* partials = nullptr;      // [kRedBlocksMax]
  Scalars* scal = nullptr;         // device scalars
  Scalars* scal_host = nullptr;    // pinned mirror
  double* stage[3] = {nullptr, nullptr, nullptr};  // natural-order staging
  size_t stage_cap = 0;            // entries per staging buffer
  // pinned chunks for copies from and to pageable host memory (host_to_device,
  // device_to_host), allocated on first use; pin_ev[i]: the last copy that
  // used pin[i]
  double* pin[2] = {nullptr, nullptr};
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  // launch profiler: CUDA events around selected launches on `stream`
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;                   // free events
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_open[kProfKinds];
  double prof_ms[kProfKinds] = {};
  long prof_launches[kProfKinds] = {};
  int64_t prof_rows[kProfKinds] = {};                 // rows processed by the timed launches
  // fault word of the kernels with bounded waits (pinned, mapped): nonzero once a
  // wait gave up; read and cleared by stream_sync
  unsigned* fault = nullptr;
};

// Event pair around one launch of `kind` (no-op unless profiling); prof_end after the launch.
int prof_begin(Context* c, int kind, cudaEvent_t* start);
int prof_end(Context* c, int kind, cudaEvent_t start, int64_t rows);
// Folds finished event pairs into the totals (synchronises the stream).
int prof_flush(Context* c);

// Context of `device` (created on first use); nullptr on failure (error recorded).
Context* context_for(int device);
// Context of the current device.
Context* current_context();
// Grows the staging buffers to at least n entries.
int ensure_stage(Context* c, size_t n);
// n doubles from host memory to device memory, queued on c's stream; returns
// once src has been read (the copy itself may still be in flight).
int host_to_device(Context* c, double* dst, const double* src, size_t n);
// n doubles from device memory (after the work queued on c's stream) to host
// memory; dst is complete on return.
int device_to_host(Context* c, double* dst, const double* src, size_t n);
// Synchronises c's stream; HPCG_B200_ERR_TIMEOUT if a kernel's bounded wait gave
// up since the last call (the fault word is cleared).
int stream_sync(Context* c);
// The level's FP64 tensor maps for the bulk-copy kernels (built on first use,
// rebuilt if the arrays moved); nullptr if they cannot be encoded.
const BulkMaps* bulk_maps(const Level& L);

// Device allocation accounted against the optional budget HPCG_B200_DEVICE_BUDGET (bytes).
int dev_alloc(void** ptr, size_t bytes, size_t* counter);
void dev_free(void* ptr);

// Where a vector argument of a call on GPU `device` lives: *on_device = false
// for host memory (pageable or pinned: moved through copies), true for device
// memory of `device` or managed memory (used in place). Device memory of
// another GPU is refused with HPCG_B200_ERR_ARG (the error text names `what`
// and both GPUs): a kernel on `device` would fault on it.
int locate_ptr(const void* ptr, int device, bool* on_device, const char* what);

// body(begin, end) over [0, n) on up to 16 host threads (one below 1 Mi entries)
template <typename F>
inline void host_parallel(int64_t n, F&& body) {
  unsigned t = std::thread::hardware_concurrency();
  t = t == 0 ? 1 : std::min(t, 16u);
  if (n < (1 << 20) || t == 1) {
    body((int64_t)0, n);
    return;
  }
  std::vector<std::thread> pool;
  const int64_t chunk = (n + t - 1) / t;
  for (unsigned i = 1; i < t; ++i) {
    const int64_t b = (int64_t)i * chunk, e = std::min<int64_t>(n, b + chunk);
    if (b < e) pool.emplace_back([&body, b, e] { body(b, e); });
  }
  body((int64_t)0, std::min<int64_t>(n, chunk));
  for (auto& th : pool) th.join();
}

// Raises a kernel's dynamic shared-memory limit to `smem` on `device` (the
// current device) once: `done` is the kernel's own set of devices already
// raised. The bit is set with fetch_or after the call, so two host threads
// driving different devices cannot lose each other's bit, and a thread that
// sees the bit also sees the raised limit.
template <typename Kern>
inline void bulk_attr(Kern k, int smem, int device, std::atomic<uint64_t>* done) {
  const uint64_t bit = 1ull << device;
  if (done->load(std::memory_order_acquire) & bit) return;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  done->fetch_or(bit, std::memory_order_release);
}

// problem handle validity
inline bool valid(const hpcg_b200_problem* p) { return p != nullptr && p->magic == kMagic; }

// Grid size for grid-stride kernels: a whole number of waves over the SMs.
inline int grid_for(const Context* c, int64_t work, int threads, int per_sm) {
  int64_t blocks = (work + threads - 1) / threads;
  const int64_t cap = (int64_t)c->sms * per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

// Releases the multi-system work vectors of p (multi.cu).
void free_multi(hpcg_b200_problem* p);

// Builds the sorted transfer pairs (tf, tq) of level l from its device f2c.
int build_transfer(hpcg_b200_problem* p, int l);

constexpr uint32_t kAllSlots = (1u << kSlots) - 1;

// Resident blocks per SM of a kernel (at least 1).
template <typename K>
int resident(K kernel) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 256, 0) != cudaSuccess || b < 1) {
    cudaGetLastError();
    b = 1;
  }
  return b;
}

// Grid of a grid-stride row kernel: every SM filled once with resident blocks.
template <typename K>
int grid_of(Context* c, K kernel, int64_t rows) {
  return grid_for(c, rows, 256, resident(kernel));
}

// Index of the zero entry padded slots point at.
inline int sink_of(const Level& L) { return L.n + L.next; }

// true for a rank of a run over several ranks: the single-rank entry points
// refuse it (its halo would never be exchanged)
inline bool is_rank(const hpcg_b200_problem* p) { return p->geom != nullptr && p->geom->size > 1; }

// natural <-> colour order vector movement (solver.cu)
int load_vector(hpcg_b200_problem* p, int level, const double* src_natural, double* dst_colour);
int store_vector(hpcg_b200_problem* p, int level, const double* src_colour, double* dst_natural);

}  // namespace hb
