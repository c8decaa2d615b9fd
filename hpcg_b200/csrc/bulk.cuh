// The bulk-copy pipeline shared by the Gauss-Seidel, SpMV and multi-system
// kernels: TMA and mbarrier helpers, pipeline shapes and the producer/consumer
// skeleton. Device functions and templates only, so that every translation
// unit with kernels may include it.
#pragma once

#include "common.cuh"
#include "reduce.cuh"

namespace hb {

// ---- bulk-copy pipeline ------------------------------------------------------
// A persistent block per SM walks tiles of kBulkRows rows (of a Gauss-Seidel
// phase, of the SpMV, of a multi-system phase). A
// producer warp streams each tile's matrix (all 27 slots' values and columns)
// into shared-memory stages with two asynchronous copies by the SM's copy unit:
// no thread holds the stream in registers, and the stream does not wait on the
// row arithmetic. A stage's "full" mbarrier completes when all its bytes have
// landed (transaction count). Groups of kBulkRows x `lanes` consumer threads
// take the block's tiles in turn (tile i to group i mod G), `lanes` threads per
// row: they gather x from global memory through the columns on chip, write the
// row and arrive on the stage's "empty" mbarrier, after which the producer
// refills it.
// Each group owns a ring of stages (the group's k-th tile uses stage k mod
// ring of its own), so a stage's fills are consumed in order by one
// group and no wait on a barrier can start more than one phase early (an
// mbarrier parity wait cannot tell phase n from phase n - 2). The kernels that
// use it keep the slot order of their register-pipelined twins: the same bits.
// A first sweep copies all slots too (it reads about half), so the autotuner
// usually keeps another configuration for it.
// Every wait gives up after kBulkWaitNs of global time: the thread then sets
// the context's fault word (host-mapped; stream_sync turns it into
// HPCG_B200_ERR_TIMEOUT) and stops; before its block exits the producer waits,
// bounded again, for the copies it issued.
// Tiles start on multiples of their rows (kBulkRows, or 2 kBulkRows for the
// FP32 phases' two-block tiles; r0 rounded down); rows outside [r0, r1) are
// copied and not computed. The last tile ends at r1 rounded up to its rows,
// at most 256, which is within the pitch (a multiple of 256 above n).
constexpr int kBulkRows = 128;                             // rows per block (tile) = threads per consumer group
constexpr unsigned long long kBulkWaitNs = 1000000000ull;  // 1 s per wait
// How a tile reaches shared memory. FP32 (blocked copy with kRowBlock32 ==
// kBulkRows): a tile is one block of the layout, its values one run of memory
// and its columns another, two bulk copies. FP64 (slot-major): one 2-D tensor
// copy per array (box kBulkRows rows x 27 slots of a map with the pitch as row
// stride). Either way two requests per tile: the SM's copy unit takes a roughly
// fixed time per request, so 2 x 27 per-slot copies of 0.5-1 KB capped the
// phases near 4 TB/s.
template <typename T>
__host__ __device__ constexpr bool bulk_whole_tile() {
  return sizeof(T) == 4 && kRowBlock32 == kBulkRows;
}
template <typename T>
__host__ __device__ constexpr bool bulk_tensor_tile() {
  return sizeof(T) == 8;
}
// Packed columns: a level's column indices as one record per kBulkRows-row
// tile of its storage (tile j: rows kBulkRows j ..): kSlots 32-bit bases and a
// word that holds the record's form w (the rest then starts on 16 bytes), then
//  - w = 1, 2: kSlots x kBulkRows offsets of w bytes, slot-major. Slot k of row
//    t is column base[k] + offset, or the level's zero sink where the offset is
//    pack_sink(w). w = 1 where every tile's columns of each slot (sink aside)
//    span at most pack_max_span(1) = 254, else 2 where they span at most 65534;
//  - w = 3 (diagonal): kSlots x 4 words of sink bits. Slot k of row t is column
//    base[k] + t, or the sink where bit t of the slot's 128 bits is set: for
//    tiles whose every slot's columns, sink aside, are one diagonal (column -
//    row the same for every row). In the colour order of a 27-point stencil
//    whose colour blocks fill whole tiles every tile is so;
// tried in the order 3, 1, 2; a level that fits none keeps only its 32-bit
// columns. 4.25 (w = 3), 27.9 (w = 1) or 54.9 (w = 2) bytes a row instead of
// 108; one bulk copy per tile, as the blocked FP32 columns.
constexpr int kPackBaseWords = 28;
constexpr int kPackDiag = 3;  // the diagonal form's code
__host__ __device__ constexpr int pack_rec(int w) {
  return kPackBaseWords * 4 + (w == kPackDiag ? kSlots * (kBulkRows / 32) * 4 : kSlots * kBulkRows * w);
}
__host__ __device__ constexpr unsigned pack_sink(int w) { return w == 1 ? 0xFFu : 0xFFFFu; }
__host__ __device__ constexpr int pack_max_span(int w) { return w == 1 ? 0xFE : 0xFFFE; }
static_assert(pack_rec(1) % 16 == 0 && pack_rec(2) % 16 == 0 && pack_rec(kPackDiag) % 16 == 0,
              "a record is one bulk copy");

// Shape of a pipeline: G consumer groups of kBulkRows x LANES threads, each
// with a ring of RING stages of one tile. A stage holds the tile's values and
// its columns: 32-bit (PW = 0), or the packed record of form PW (1, 2: offsets
// of PW bytes; 3: diagonal), or, with PW = -1, a record whose form each tile
// states (the batched kernel, whose tiles come from several levels): staged
// for the largest one, each fill expecting its own record's bytes. Stages are rounded up to
// 128 bytes (tensor copies land on 128-byte boundaries): FP64 stages are 41.5
// KB with 32-bit columns (33.9 / 30.5 / 28.3 KB with 16-bit offsets, 8-bit
// offsets, the diagonal form) and FP32 one-block stages 27 KB (20.4 / 17 /
// 14.4 KB); all stages of a block share at most 227 KB of shared memory (one
// block per SM).
// TB: kBulkRows-row blocks per tile (1, or 2 for whole-tile copies: the
// blocks of a tile are consecutive in the blocked layout and in the packed
// records, so a tile of TB blocks is still one copy of values and one of
// columns, with TB times the bytes per request). A consumer group then has
// kBulkRows x LANES x TB threads; thread t works on block t / (kBulkRows x
// LANES) of the tile.
template <typename T, int G, int RING, int LANES = 1, int PW = 0, int TB = 1>
struct BulkShape {
  static constexpr int groups = G;
  static constexpr int ring = RING;
  static constexpr int lanes = LANES;
  static constexpr int pack = PW;
  static constexpr bool packed = PW != 0;
  static constexpr int blocks = TB;
  static constexpr int tile_rows = kBulkRows * TB;
  static constexpr int block_threads = kBulkRows * LANES;
  static constexpr int group_threads = block_threads * TB;
  static constexpr int stages = groups * ring;
  static constexpr int threads = 32 + groups * group_threads;  // producer warp + consumers
  static constexpr int block_value_bytes = kSlots * kBulkRows * (int)sizeof(T);
  static constexpr int block_col_bytes =
      PW == 0 ? kSlots * kBulkRows * (int)sizeof(int) : pack_rec(PW < 0 ? 2 : PW);
  static constexpr int value_bytes = block_value_bytes * TB;
  static constexpr int col_bytes = block_col_bytes * TB;
  static_assert(TB == 1 || (TB == 2 && bulk_whole_tile<T>() && PW >= 0 && LANES == 1),
                "tiles of two blocks: whole-tile copies, one record form, one thread per row");
  static constexpr int tx_bytes = value_bytes + col_bytes;  // bytes landing in a stage per fill (PW >= 0)
  static constexpr int stage_bytes = (tx_bytes + 127) / 128 * 128;
  // stages + per stage two barriers and the tile's first row + slack to align
  // the stages to 128 bytes (tensor copies)
  static constexpr int smem = stages * stage_bytes + 3 * stages * (int)sizeof(uint64_t) + 128;
  static_assert(smem <= 227 * 1024, "shared memory of one block");
  static_assert(threads <= 1024, "threads of one block");
  static_assert(PW >= -1 && PW <= kPackDiag, "column form");
};
// The shapes in use: rings of two stages (measured at 512^3: two groups of two
// stages beat four groups of one for the Gauss-Seidel phases by 8% and tied for
// the SpMV), with as many consumer groups as asked for and as fit in 227 KB.
// A phase's consumers wait on their gathers of x, and one block per SM leaves
// few warps to cover that latency: with 8-bit offsets (31 KB FP64 stages,
// 17 KB FP32 ones) measured at 512^3, three FP64 groups instead of two took a
// phase from 0.93 to 0.80 ms and four FP32 groups instead of three from 11.4
// to 10.0 ms per iteration (five: 10.2). With the diagonal form (28 KB FP64
// stages), same box and run, a third SpMV group took the SpMV from 6.14 to
// 5.52 ms and the restriction from 0.80 to 0.73 ms, while a fourth FP64 phase
// group changed nothing. The FP32 phases take tiles of two blocks (256 rows,
// 28.8 KB a stage) in two groups: their consumers release a stage early, so
// the copy side bounds them, and two-block tiles halve its requests per byte.
// Measured at 512^3 (FP32 level-0 phases of one V-cycle): 8.52-8.56 ms against
// 9.08-9.14 ms for one-block tiles in four groups; three two-block groups
// 9.43, two with rings of three 8.68, one with a ring of four 11.93. A shape
// whose stages do not fit (32-bit columns) gets fewer groups.
#ifndef HB_GS64_GROUPS
#define HB_GS64_GROUPS 3
#endif
#ifndef HB_GS32_GROUPS
#define HB_GS32_GROUPS 2
#endif
#ifndef HB_SPMV32_GROUPS
#define HB_SPMV32_GROUPS 4
#endif
#ifndef HB_SPMV_GROUPS
#define HB_SPMV_GROUPS 3
#endif
#ifndef HB_BULK_RING
#define HB_BULK_RING 2
#endif
#ifndef HB_GS32_RING
#define HB_GS32_RING HB_BULK_RING
#endif
#ifndef HB_GS32_TILE
#define HB_GS32_TILE 2
#endif
// Whether the Gauss-Seidel phases, the SpMV and the restriction hand a stage
// back once the row's values and columns are in registers (bulk_tiles_src's
// EARLY), per value type. Measured at 512^3 on one box: the FP32 phases went
// from 10.01 to 9.09 ms per iteration; the FP64 phases (15.68 -> 15.85 ms),
// the SpMV (5.60 -> 5.59 ms) and the FP64 restriction (0.73 -> 0.76 ms) did
// not gain, their 27 values taking registers the gathers need (128 per thread).
#ifndef HB_EARLY32
#define HB_EARLY32 1
#endif
#ifndef HB_EARLY64
#define HB_EARLY64 0
#endif
template <typename T>
__host__ __device__ constexpr bool bulk_early() {
  return sizeof(T) == 4 ? HB_EARLY32 != 0 : HB_EARLY64 != 0;
}
#ifndef HB_SPMV_GATHER_FIRST
#define HB_SPMV_GATHER_FIRST 0
#endif
// The FP64 SpMV: three groups of one stage whose consumers hand the stage
// back once the row is in registers (85 KB of shared memory, the rest of the
// SM's 256 KB left to L1 for the gathers); the restriction keeps rings of two
// without early release.
#ifndef HB_SPMV_RING
#define HB_SPMV_RING 1
#endif
#ifndef HB_SPMV_EARLY64
#define HB_SPMV_EARLY64 1
#endif
#ifndef HB_RESTRICT_RING
#define HB_RESTRICT_RING 2
#endif
#ifndef HB_RESTRICT_EARLY64
#define HB_RESTRICT_EARLY64 0
#endif
#ifndef HB_FIRST_EARLY64
#define HB_FIRST_EARLY64 0
#endif
template <typename T, int PW, int TB = 1>
__host__ __device__ constexpr int fit_groups(int want, int ring) {
  while (want > 1 && (BulkShape<T, 1, 2, 1, PW, TB>::stage_bytes * ring * want + 24 * ring * want + 128 > 227 * 1024 ||
                      32 + want * kBulkRows * TB > 1024))
    --want;
  return want;
}
template <typename T>
__host__ __device__ constexpr int gs_ring() {
  return sizeof(T) == 8 ? HB_BULK_RING : HB_GS32_RING;
}
// blocks per tile of the Gauss-Seidel phases: FP32 with one record form (the
// batched kernel's per-tile forms keep one block)
template <typename T, int PW>
__host__ __device__ constexpr int gs_blocks() {
  return sizeof(T) == 4 && PW >= 0 ? HB_GS32_TILE : 1;
}
template <typename T, int PW = 0>
using GsShape = BulkShape<T,
                          fit_groups<T, PW, gs_blocks<T, PW>()>(sizeof(T) == 8 ? HB_GS64_GROUPS : HB_GS32_GROUPS,
                                                                gs_ring<T>()),
                          gs_ring<T>(), 1, PW, gs_blocks<T, PW>()>;
template <typename T, int PW = 0>
using SpmvShape = BulkShape<T, fit_groups<T, PW>(sizeof(T) == 8 ? HB_SPMV_GROUPS : HB_SPMV32_GROUPS, sizeof(T) == 8 ? HB_SPMV_RING : HB_BULK_RING),
                            sizeof(T) == 8 ? HB_SPMV_RING : HB_BULK_RING, 1, PW>;
template <typename T>
__host__ __device__ constexpr bool spmv_early() {
  return sizeof(T) == 4 ? HB_EARLY32 != 0 : HB_SPMV_EARLY64 != 0;
}
template <typename T>
__host__ __device__ constexpr bool restrict_early() {
  return sizeof(T) == 4 ? HB_EARLY32 != 0 : HB_RESTRICT_EARLY64 != 0;
}
// the Gauss-Seidel phases: FIRST (x entering zero, masked slots) separately
template <typename T, bool FIRST>
__host__ __device__ constexpr bool gs_early() {
  return bulk_early<T>() || (FIRST && sizeof(T) == 8 && HB_FIRST_EARLY64 != 0);
}
template <typename T, int PW = 0>
using RestrictShape =
    BulkShape<T, fit_groups<T, PW>(sizeof(T) == 8 ? HB_SPMV_GROUPS : HB_SPMV32_GROUPS, sizeof(T) == 8 ? HB_RESTRICT_RING : HB_BULK_RING),
              sizeof(T) == 8 ? HB_RESTRICT_RING : HB_BULK_RING, 1, PW>;

// Column of slot k of row t of a tile in a stage (sc: the stage's column area)
// for the column form PW of BulkShape.
template <int PW>
__device__ __forceinline__ int stage_col(const int* sc, int k, int t, int sink) {
  if constexpr (PW == 0) {
    return sc[k * kBulkRows + t];
  } else if constexpr (PW == 1) {
    const unsigned o = reinterpret_cast<const unsigned char*>(sc + kPackBaseWords)[k * kBulkRows + t];
    return o == pack_sink(1) ? sink : sc[k] + (int)o;
  } else if constexpr (PW == 2) {
    const unsigned o = reinterpret_cast<const unsigned short*>(sc + kPackBaseWords)[k * kBulkRows + t];
    return o == pack_sink(2) ? sink : sc[k] + (int)o;
  } else if constexpr (PW == kPackDiag) {
    // the warp's 32 rows share one word of sink bits (a broadcast load)
    const unsigned bits = reinterpret_cast<const unsigned*>(sc + kPackBaseWords)[k * (kBulkRows / 32) + (t >> 5)];
    return (bits >> (t & 31)) & 1u ? sink : sc[k] + t;
  } else {
    const int w = sc[kSlots];
    return w == 1 ? stage_col<1>(sc, k, t, sink) : w == 2 ? stage_col<2>(sc, k, t, sink)
                                                           : stage_col<kPackDiag>(sc, k, t, sink);
  }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// makes the initialised barriers visible to the other threads and to the bulk-copy unit
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// true once the barrier's phase of the given parity has completed; false after limit_ns
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          unsigned long long limit_ns = kBulkWaitNs) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_test(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
// global -> shared bulk copy completing on `bar`, streamed with an evict-first L2 policy
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}
// global -> shared 2-D tensor tile (box of the map at column x, row y) completing on `bar`
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar,
                                            uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}
__device__ __forceinline__ uint64_t evict_first_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while the kernel before it on the stream finishes;
// griddep_wait() returns once that kernel has completed and its writes are
// visible (at once for a kernel launched without the attribute), and
// griddep_launch_dependents() lets the next such kernel start.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ void record_fault(unsigned* fault, unsigned code) {
  *(volatile unsigned*)fault = code;
  __threadfence_system();
}

// Where a tile comes from: its first row and, when the tile is one block of
// the layout (whole-tile copies), the addresses of its value and column blocks;
// with packed columns, the address of its record and (read only when the
// shape's offset width is per tile, PW = -1) the record's bytes.
template <typename T>
struct TileSrc {
  int64_t q0;
  const T* vals;
  const int* cols;
  const unsigned char* rec;
  int rec_bytes;
};

// The producer/consumer pipeline of the bulk-copy kernels, run by the whole
// block. The block's tiles are blockIdx.x, + gridDim.x, ... below ntiles, less
// those for which skip(tile) holds (every thread of the block must get the same
// answer); the i-th tile kept goes to consumer group i mod G. src(tile) gives
// the tile's TileSrc; the tensor maps (FP64 tiles only) are kernel parameters.
// Each consumer thread calls row(tile, q0, sv, sc, t) for
// every tile of its group, t its index in the group (row t / LANES of the tile,
// lane t % LANES), with the tile's values sv[k * kBulkRows + row] and columns
// on chip: sc[k * kBulkRows + row], or the packed record at sc
// (stage_col<Shape::pack> reads any of them). The tile's first row q0 comes
// from the producer through the stage (it computed src(tile) for the copies),
// so the consumers' loads wait on no index arithmetic of their own.
// EARLY: row(tile, q0, sv, sc, t, release) takes what it needs of the stage
// into registers and calls release() (exactly once, on every path) to hand
// the stage back to the producer before it gathers and computes, so a stage
// is held for its shared-memory reads only and the ring keeps more fills in
// flight; otherwise the stage is released after row() returns.
template <typename T, typename Shape, bool EARLY = false, typename Src, typename Skip, typename RowFn>
__device__ __forceinline__ void bulk_tiles_src(int ntiles, Src src, Skip skip, RowFn row, unsigned* fault,
                                               const CUtensorMap* tm_val, const CUtensorMap* tm_col) {
  constexpr int G = Shape::groups;
  constexpr int RING = Shape::ring;
  constexpr int S = Shape::stages;
  constexpr int SB = Shape::stage_bytes;
  constexpr int VB = Shape::value_bytes;  // value bytes of a stage (columns follow)
  static_assert(bulk_whole_tile<T>() || bulk_tensor_tile<T>(), "a tile must arrive in two copies");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * SB);
  uint64_t* empty = full + S;
  int64_t* first = reinterpret_cast<int64_t*>(empty + S);  // q0 of the tile in each stage
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], Shape::group_threads);
    }
    mbar_init_fence();
  }
  __syncthreads();
  // Under a programmatic dependent launch the producer streams the first tiles
  // while the previous kernel finishes: it reads only the matrix, and every
  // kernel that writes a matrix array is followed by a stream synchronisation.
  // (The batched kernel's skip predicate reads convergence flags; it is
  // launched without the attribute, so the wait is already over.) The
  // consumers read and write the vectors: they wait for that kernel first.
  if (threadIdx.x == 0) griddep_launch_dependents();
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    // the producer warp: lane 0 waits for a free stage and posts the byte
    // count, then lanes 0 and 1 issue the tile's two copies
    const int lane = threadIdx.x;
    const uint64_t policy = evict_first_policy();
    int last[S];  // last fill issued into each stage (-1: none)
#pragma unroll
    for (int s = 0; s < S; ++s) last[s] = -1;
    int i = 0;  // tiles kept so far: tile i goes to group i % G, as its (i / G)-th
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      if (skip(tile)) continue;
      const int kg = i / G;
      const int s = (i % G) * RING + kg % RING, use = kg / RING;
      const TileSrc<T> ts = src(tile);
      const int rec_bytes = Shape::pack < 0 ? ts.rec_bytes : Shape::col_bytes;
      int ok = 1;
      if (lane == 0) {
        if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1)) {
          record_fault(fault, 1);
          ok = 0;
        } else {
          first[s] = ts.q0;  // released to the consumers by the arrival below
          mbar_expect_tx(&full[s], Shape::value_bytes + rec_bytes);
        }
      }
      if (!__shfl_sync(0xffffffffu, ok, 0)) break;
      T* sv = reinterpret_cast<T*>(smem + s * SB);
      int* sc = reinterpret_cast<int*>(smem + s * SB + VB);
      if constexpr (bulk_whole_tile<T>()) {
        // the tile is one block of the layout: all slots' values in one run, all columns in another
        if (lane == 0) bulk_g2s(sv, ts.vals, VB, &full[s], policy);
      } else {
        // rows q0 .. q0 + kBulkRows of all 27 slots, [slot][row] in shared memory
        if (lane == 0) tma_load_2d(sv, tm_val, (int)ts.q0, 0, &full[s], policy);
      }
      if constexpr (Shape::packed) {
        if (lane == 1) bulk_g2s(sc, ts.rec, rec_bytes, &full[s], policy);
      } else if constexpr (bulk_whole_tile<T>()) {
        if (lane == 1) bulk_g2s(sc, ts.cols, Shape::col_bytes, &full[s], policy);
      } else {
        if (lane == 1) tma_load_2d(sc, tm_col, (int)ts.q0, 0, &full[s], policy);
      }
#pragma unroll
      for (int u = 0; u < S; ++u)
        if (u == s) last[u] = use;
      ++i;
    }
    // no copy may still be landing when the block exits: the last fill of
    // every stage has completed (consumed or not)
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < S; ++s)
        if (last[s] >= 0 && !mbar_wait(&full[s], last[s] & 1)) record_fault(fault, 2);
    }
    __syncwarp();
  } else {
    griddep_wait();
    const int g = (warp - 1) / (Shape::group_threads / 32);   // consumer group
    const int t = (threadIdx.x - 32) % Shape::group_threads;  // index in the group
    int i = 0;                                                // tiles kept so far
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      if (skip(tile)) continue;
      if (i % G == g) {
        const int kg = i / G;
        const int s = g * RING + kg % RING, use = kg / RING;
        if (!mbar_wait(&full[s], use & 1)) {
          record_fault(fault, 3);
          break;
        }
        // the thread's block of the tile: its first row, values and columns
        const int h = t / Shape::block_threads;
        const int64_t q0 = first[s] + (int64_t)h * kBulkRows;
        const T* sv = reinterpret_cast<const T*>(smem + s * SB + h * Shape::block_value_bytes);
        const int* sc = reinterpret_cast<const int*>(smem + s * SB + VB + h * Shape::block_col_bytes);
        const int tb = t - h * Shape::block_threads;
        if constexpr (EARLY) {
          row(tile, q0, sv, sc, tb, [&] { mbar_arrive(&empty[s]); });
        } else {
          row(tile, q0, sv, sc, tb);
          mbar_arrive(&empty[s]);
        }
      }
      ++i;
    }
  }
}

// The common case: one matrix (val, col or the packed records colp, pitch),
// tile `tile` starting at row first_row(tile) (a multiple of kBulkRows with
// packed columns or whole-tile copies), no tile skipped; row(q0, sv, sc, t).
// EARLY: row(q0, sv, sc, t, release), as bulk_tiles_src's.
template <typename T, typename Shape, bool EARLY = false, typename FirstRow, typename RowFn>
__device__ __forceinline__ void bulk_tiles(const T* __restrict__ val, const int* __restrict__ col, int64_t pitch,
                                           int ntiles, FirstRow first_row, RowFn row, unsigned* fault,
                                           const CUtensorMap& tm_val, const CUtensorMap& tm_col,
                                           const unsigned char* colp = nullptr) {
  bulk_tiles_src<T, Shape, EARLY>(
      ntiles,
      [&](int tile) {
        const int64_t q0 = first_row(tile);
        static_assert(Shape::pack >= 0, "one offset width per level");
        return TileSrc<T>{q0, val + mat_index<T>(0, q0, pitch), col + mat_index<T>(0, q0, pitch),
                          Shape::packed ? colp + (q0 / kBulkRows) * pack_rec(Shape::pack) : nullptr,
                          Shape::col_bytes};
      },
      [](int) { return false; },
      [&](int, int64_t q0, const T* sv, const int* sc, int t, auto&&... release) { row(q0, sv, sc, t, release...); },
      fault, &tm_val, &tm_col);
}

}  // namespace hb
