// Device kernels of the PCG path. The library is compiled with -fmad=false, so
// every a*b+c below rounds twice exactly as the reference's C++ does when built
// without contraction; the per-row summation order is the reference's entry
// order (slot order). Results of the row kernels are therefore bitwise those of
// the reference routines on the same ordering; only the dot-product reductions
// differ (fixed-shape tree instead of a serial loop, deterministic run to run).
#pragma once

#include "bulk.cuh"
#include "common.cuh"
#include "reduce.cuh"
#include "rows.cuh"

namespace hb {

// ---------------------------------------------------------------------------
// Gauss-Seidel colour phase: rows [r0, r1) of one colour, updated in parallel
// (no two rows of a colour are neighbours). Row update as
// ComputeSYMGS_ref.cpp:72-80: sum = r_i - sum_j a_ij x_j (diagonal included),
// sum += x_i a_ii, x_i = sum / a_ii.
// FIRST: the sweep starts from x = 0 (ComputeMG_ref.cpp:42); slots not in `mask`
// (neighbours not yet swept, and the diagonal) multiply a zero and are skipped,
// which leaves every sum bitwise unchanged.
// ---------------------------------------------------------------------------
// Kernel configurations the autotuner chooses from. Every configuration
// computes the same bits; they differ in how the loads are issued:
//  - schedule: kPlain issues loads as the compiler schedules the slot loop;
//    kStaged issues all masked value/column loads first (27 independent loads in
//    flight per thread), then the 27 gathers of x, then the sum, and reads the
//    matrix with evict-first hints (__ldcs) so that the stream of values and
//    columns, read once per phase, does not push the vector out of L2;
//  - rows per thread (R): with R > 1 a thread updates R adjacent rows of a
//    colour with vector loads (double2, float2/float4, int2/int4), so each load
//    instruction moves R times the bytes and more bytes are in flight per thread
//    (the FP32 matrix stream otherwise moves only 4 bytes a load); R > 1 needs
//    the row range to start on a multiple of R (checked on the host);
//  - the minimum resident 256-thread blocks per SM, which caps registers per
//    thread (4 -> 64, 2 -> 128, 1 -> 255).

//  - interleaved rows (Gauss-Seidel phases only, configurations 7 and 8): a
//    thread updates R rows 32 apart, so every load of a warp is one coalesced
//    run (no vector loads, no strided gathers) and each thread still has R
//    independent rows' loads in flight.
//  - tiled (configuration 9, Gauss-Seidel phases only): see k_gs_tile.
//  - bulk-copy pipeline (Gauss-Seidel configuration 10, SpMV configuration 7):
//    see bulk_tiles, k_gs_bulk and k_spmv_bulk.
constexpr int kConfigs = 8;     // configurations of the SpMV and the restriction
constexpr int kBulkMvCfg = 7;   // the SpMV through the bulk-copy pipeline (k_spmv_bulk)
constexpr int kGsConfigs = 11;  // configurations of the Gauss-Seidel phases
constexpr int kTileCfg = 9;     // the tiled configuration
constexpr int kBulkCfg = 10;    // the bulk-copy pipeline
// configurations without a row-alignment requirement that run their own kernels
__host__ __device__ constexpr bool cfg_tiled(int cfg) { return cfg >= kTileCfg; }
__host__ __device__ constexpr int cfg_sched(int cfg) { return cfg == 2 || cfg == 3 ? kStaged : kPlain; }
__host__ __device__ constexpr int cfg_minb(int cfg) {
  return cfg == 0 || cfg == 4 ? 4 : cfg == 2 ? 1 : 2;
}
__host__ __device__ constexpr int cfg_rows(int cfg) {
  return cfg == 4 || cfg == 5 || cfg == 7 ? 2 : cfg == 6 || cfg == 8 ? 4 : 1;
}
__host__ __device__ constexpr bool cfg_interleaved(int cfg) { return cfg == 7 || cfg == 8; }

// Gauss-Seidel colour phase: rows [r0, r1) of one colour, updated in parallel
// (no two rows of a colour are neighbours).
// CMASK >= 0: the slot mask is that compile-time constant (the first sweep's
// masks of the default sweep order), so unused slots drop out of the code;
// CMASK < 0: the runtime `mask`.
// DOT: the phase also writes block partials of sum_i rhs_i * x_i over its rows
// (the new x) to dot[blockIdx.x]: run on the phases that write each colour's
// final value, they give the CG's r'z without another pass over r and z.
template <typename T, typename TR, bool FIRST, int CFG, int64_t CMASK = -1, int SCHED = cfg_sched(CFG),
          int R = cfg_rows(CFG), bool DOT = false>
__global__ void __launch_bounds__(kThreads, cfg_minb(CFG)) k_gs_phase(const T* __restrict__ val,
                                                                      const int* __restrict__ col, int64_t pitch,
                                                                      const TR* __restrict__ rhs, T* x, int r0,
                                                                      int r1, uint32_t mask_arg,
                                                                      double* __restrict__ dot) {
  const uint32_t mask = CMASK >= 0 ? (uint32_t)CMASK : mask_arg;
  double acc = 0.0;
  if (cfg_interleaved(CFG)) {
    // tiles of blockDim.x * R rows; warp w takes 32 * R of them, lane l rows l + 32 r
    const int64_t tile = (int64_t)blockDim.x * R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t b0 = r0 + (int64_t)blockIdx.x * tile; b0 < r1; b0 += (int64_t)gridDim.x * tile) {
      const int64_t q0 = b0 + (int64_t)warp * 32 * R + lane;
      T sum[R], xd[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        sum[r] = q0 + 32 * r < r1 ? (T)rhs[q0 + 32 * r] : (T)0;
        xd[r] = (T)0;
      }
#pragma unroll
      for (int k = 0; k < kSlots; ++k) {
        if (mask & (1u << k)) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int64_t q = q0 + 32 * r;
            if (q < r1) {
              const T a = val[mat_index<T>(k, q, pitch)];
              const T xv = __ldg(x + col[mat_index<T>(k, q, pitch)]);
              sum[r] -= a * xv;
              if (k == kDiagSlot) xd[r] = xv;
            }
          }
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int64_t q = q0 + 32 * r;
        if (q < r1) {
          const T d = val[mat_index<T>(kDiagSlot, q, pitch)];
          if (!FIRST) sum[r] += xd[r] * d;
          const T out = sum[r] / d;
          x[q] = out;
          if (DOT) acc += (double)rhs[q] * (double)out;
        }
      }
    }
    if (DOT) {
      const double s = block_sum(acc);
      if (threadIdx.x == 0) dot[blockIdx.x] = s;
    }
    return;
  }
  if (R == 1) {
    const int stride = gridDim.x * blockDim.x;
    for (int q = r0 + blockIdx.x * blockDim.x + threadIdx.x; q < r1; q += stride) {
      const T out = gs_row<T, TR, FIRST, SCHED>(val, col, pitch, rhs, x, q, mask);
      if (DOT) acc += (double)rhs[q] * (double)out;
    }
    if (DOT) {
      const double s = block_sum(acc);
      if (threadIdx.x == 0) dot[blockIdx.x] = s;
    }
    return;
  }
  const int64_t stride = (int64_t)gridDim.x * blockDim.x * R;
  for (int64_t q0 = r0 + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * R; q0 < r1; q0 += stride) {
    if (q0 + R > r1) {
      for (int q = (int)q0; q < r1; ++q) {
        const T out = gs_row<T, TR, FIRST, kPlain>(val, col, pitch, rhs, x, q, mask);
        if (DOT) acc += (double)rhs[q] * (double)out;
      }
      continue;
    }
    TR rv[R];
    load_vec<TR, R>(rhs + q0, rv);
    T sum[R], xd[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      sum[r] = (T)rv[r];
      xd[r] = (T)0;
    }
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      if (mask & (1u << k)) {
        T a[R];
        int c[R];
        load_vec<T, R>(val + mat_index<T>(k, q0, pitch), a);
        load_vec<int, R>(col + mat_index<T>(k, q0, pitch), c);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const T xv = __ldg(x + c[r]);
          sum[r] -= a[r] * xv;
          if (k == kDiagSlot) xd[r] = xv;
        }
      }
    }
    T d[R], out[R];
    load_vec<T, R>(val + mat_index<T>(kDiagSlot, q0, pitch), d);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!FIRST) sum[r] += xd[r] * d[r];
      out[r] = sum[r] / d[r];
      if (DOT) acc += (double)rv[r] * (double)out[r];
    }
    store_vec<T, R>(x + q0, out);
  }
  if (DOT) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) dot[blockIdx.x] = s;
  }
}

// ---- tiled Gauss-Seidel phase (configuration 9) -----------------------------
// One thread per row; a block walks tiles of TILE rows. The values and columns
// of the next STAGES-1 tiles stream into shared memory with asynchronous 16-byte
// copies (cp.async) while the current tile computes, so the matrix loads are
// never waited on by the row arithmetic, and each thread issues its 27 gathers
// of x back to back from columns already on chip. STAGES x 27 slots x TILE rows
// x (value + column) bytes of dynamic shared memory. Tiles start on a 4-row
// boundary (16 bytes for both float and double); rows of a tile outside
// [r0, r1) are copied (in bounds) or skipped (at and beyond r1 rounded up to 4,
// which never exceeds the pitch) and never computed. The arithmetic is
// gs_row's, in slot order: the same bits.
// Measured at 512^3 it runs level 0 at half the speed of the plain
// configurations (two blocks per SM leave too few threads to cover the gathers'
// latency; three or four stages, one block per SM, ran three times slower), so
// the autotuner picks it only on some coarse levels.

// tile rows and pipeline stages of the tiled configuration
template <typename T>
__host__ __device__ constexpr int gs_tile_rows(int) {
  return sizeof(T) == 8 ? 128 : 256;
}
__host__ __device__ constexpr int gs_tile_stages(int) { return 2; }

template <typename T>
__host__ __device__ constexpr int gs_tile_smem(int cfg) {
  return gs_tile_stages(cfg) * kSlots * gs_tile_rows<T>(cfg) * (int)(sizeof(T) + sizeof(int));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// returns once at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename T, typename TR, bool FIRST, int CFG, int64_t CMASK = -1, bool DOT = false>
__global__ void __launch_bounds__(gs_tile_rows<T>(CFG)) k_gs_tile(const T* __restrict__ val,
                                                                  const int* __restrict__ col, int64_t pitch,
                                                                  const TR* __restrict__ rhs, T* x, int r0, int r1,
                                                                  uint32_t mask_arg, double* __restrict__ dot) {
  constexpr int TILE = gs_tile_rows<T>(CFG);
  constexpr int STAGES = gs_tile_stages(CFG);
  constexpr int VCH = TILE * (int)sizeof(T) / 16;  // 16-byte chunks of one slot's values in a tile
  constexpr int CCH = TILE * 4 / 16;               // ... of its columns
  extern __shared__ __align__(16) unsigned char smem[];
  T* sval = reinterpret_cast<T*>(smem);                                            // [STAGES][27][TILE]
  int* scol = reinterpret_cast<int*>(smem + STAGES * kSlots * TILE * sizeof(T));  // [STAGES][27][TILE]
  const uint32_t mask = CMASK >= 0 ? (uint32_t)CMASK : mask_arg;
  const int a0 = r0 & ~3;
  const int lim = (r1 + 3) & ~3;
  const int ntiles = (r1 - a0 + TILE - 1) / TILE;
  // all (slot, chunk) pairs of a tile spread over the block's threads; the first
  // sweep copies only its masked slots' values and columns and the diagonal value
  auto issue = [&](int tile, int buf) {
    const int b0 = a0 + tile * TILE;
    for (int i = threadIdx.x; i < kSlots * VCH; i += TILE) {
      const int k = i / VCH, ch = i - k * VCH;
      const int row = b0 + ch * (16 / (int)sizeof(T));
      if (((mask >> k) & 1u || (FIRST && k == kDiagSlot)) && row < lim)
        cp_async16(sval + (buf * kSlots + k) * TILE + ch * (16 / sizeof(T)), val + mat_index<T>(k, row, pitch));
    }
    for (int i = threadIdx.x; i < kSlots * CCH; i += TILE) {
      const int k = i / CCH, ch = i - k * CCH;
      const int row = b0 + ch * 4;
      if ((mask >> k) & 1u && row < lim) cp_async16(scol + (buf * kSlots + k) * TILE + ch * 4, col + mat_index<T>(k, row, pitch));
    }
  };
  double acc = 0.0;
  // prologue: the first STAGES-1 tiles of this block, one commit group each
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    const int t = blockIdx.x + s * gridDim.x;
    if (t < ntiles) issue(t, s);
    cp_async_commit();
  }
  int tile = blockIdx.x;
  for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
    const int next = tile + (STAGES - 1) * gridDim.x;
    if (next < ntiles) issue(next, (it + STAGES - 1) % STAGES);
    cp_async_commit();
    cp_async_wait<STAGES - 1>();  // this thread's copies of the current tile have landed
    __syncthreads();              // and every other thread's
    const int buf = it % STAGES;
    const int q = a0 + tile * TILE + threadIdx.x;
    if (q >= r0 && q < r1) {
      T sum = (T)rhs[q];
      T xd = (T)0;
#pragma unroll
      for (int k = 0; k < kSlots; ++k) {
        if (mask & (1u << k)) {
          const T a = sval[(buf * kSlots + k) * TILE + threadIdx.x];
          const T xv = __ldg(x + scol[(buf * kSlots + k) * TILE + threadIdx.x]);
          sum -= a * xv;
          if (k == kDiagSlot) xd = xv;
        }
      }
      const T d = sval[(buf * kSlots + kDiagSlot) * TILE + threadIdx.x];
      if (!FIRST) sum += xd * d;
      const T out = sum / d;
      x[q] = out;
      if (DOT) acc += (double)rhs[q] * (double)out;
    }
    __syncthreads();  // the buffer is refilled by the next iteration's copies
  }
  if (DOT) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) dot[blockIdx.x] = s;
  }
}

// Check of the bounded wait itself: thread 0 waits on a barrier that nothing
// arrives on; after limit_ns it records fault code 4 and the kernel returns.
__global__ void k_wait_selftest(unsigned long long limit_ns, unsigned* fault) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0, limit_ns)) record_fault(fault, 4);
}

// Gauss-Seidel colour phase over rows [r0, r1) through the pipeline
// (configuration 10); PW: the level's column form (0: 32-bit columns; 1, 2:
// the packed record colp with offsets of PW bytes, sink its zero column).
template <typename T, typename TR, bool FIRST, int64_t CMASK = -1, bool DOT = false, int PW = 0>
__global__ void __launch_bounds__(GsShape<T, PW>::threads, 1)
    k_gs_bulk(const T* __restrict__ val, const int* __restrict__ col, int64_t pitch, const TR* __restrict__ rhs,
              T* x, int r0, int r1, uint32_t mask_arg, double* __restrict__ dot, unsigned* fault,
              const __grid_constant__ CUtensorMap tm_val, const __grid_constant__ CUtensorMap tm_col,
              const unsigned char* __restrict__ colp, int sink) {
  constexpr int TROWS = GsShape<T, PW>::tile_rows;  // 128, or 256 for FP32 tiles of two blocks
  const uint32_t mask = CMASK >= 0 ? (uint32_t)CMASK : mask_arg;
  const int a0 = r0 & ~(TROWS - 1);
  const int ntiles = (r1 - a0 + TROWS - 1) / TROWS;
  double acc = 0.0;
  bulk_tiles<T, GsShape<T, PW>, gs_early<T, FIRST>()>(
      val, col, pitch, ntiles, [&](int tile) { return a0 + (int64_t)tile * TROWS; },
      [&](int64_t q0, const T* sv, const int* sc, int t, auto&&... release) {
        const int64_t q = q0 + t;
        if constexpr (sizeof...(release) > 0) {
          // the row's values and columns into registers, the stage back to the producer
          T a[kSlots];
          int c[kSlots];
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            if (mask & (1u << k)) {
              a[k] = sv[k * kBulkRows + t];
              c[k] = stage_col<PW>(sc, k, t, sink);
            }
          }
          const T d = sv[kDiagSlot * kBulkRows + t];
          (release(), ...);
          if (q < r0 || q >= r1) return;
          T sum = (T)rhs[q];
          T xd = (T)0;
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            if (mask & (1u << k)) {
              const T xv = __ldg(x + c[k]);
              sum -= a[k] * xv;
              if (k == kDiagSlot) xd = xv;
            }
          }
          if (!FIRST) sum += xd * d;
          const T out = sum / d;
          x[q] = out;
          if (DOT) acc += (double)rhs[q] * (double)out;
        } else {
          if (q < r0 || q >= r1) return;
          T sum = (T)rhs[q];
          T xd = (T)0;
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            if (mask & (1u << k)) {
              const T a = sv[k * kBulkRows + t];
              const T xv = __ldg(x + stage_col<PW>(sc, k, t, sink));
              sum -= a * xv;
              if (k == kDiagSlot) xd = xv;
            }
          }
          const T d = sv[kDiagSlot * kBulkRows + t];
          if (!FIRST) sum += xd * d;
          const T out = sum / d;
          x[q] = out;
          if (DOT) acc += (double)rhs[q] * (double)out;
        }
      },
      fault, tm_val, tm_col, colp);
  if (DOT) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) dot[blockIdx.x] = s;
  }
}

// The FP64 Gauss-Seidel phase's copy pipeline (GsShape, the level's column
// form PW) over every tile of a level's matrix, each stage handed straight back
// by its consumers: the rate at which the phases' tiles stream when no
// consumer holds a stage (hpcg_b200_stream_probe). Reads the matrix only.
template <int PW>
__global__ void __launch_bounds__(GsShape<double, PW>::threads, 1)
    k_stream_probe(const double* __restrict__ val, const int* __restrict__ col, int64_t pitch, int ntiles,
                   unsigned* fault, const __grid_constant__ CUtensorMap tm_val,
                   const __grid_constant__ CUtensorMap tm_col, const unsigned char* __restrict__ colp) {
  bulk_tiles<double, GsShape<double, PW>, true>(
      val, col, pitch, ntiles, [](int tile) { return (int64_t)tile * kBulkRows; },
      [](int64_t, const double*, const int*, int, auto&& release) { release(); }, fault, tm_val, tm_col, colp);
}

// The FP32 V-cycle's matrix: values rounded to FP32 and the columns, moved from
// the slot-major FP64 arrays into the blocked layout of mat_index<float>.
__global__ void k_block32(const double* __restrict__ val, const int* __restrict__ col, int64_t pitch,
                          float* __restrict__ val32, int* __restrict__ col32) {
  const int64_t total = (int64_t)kSlots * pitch;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const int k = (int)(i / pitch);
    const int64_t q = i - (int64_t)k * pitch;
    const int64_t d = mat_index<float>(k, q, pitch);
    val32[d] = (float)val[i];
    col32[d] = col[i];
  }
}

// Natural-order (level-scheduled) Gauss-Seidel: the rows of one wavefront
// ix + 2 iy + 4 iz = const, which only read rows of other wavefronts.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_gs_rows(const T* __restrict__ val, const int* __restrict__ col,
                                                      int64_t pitch, const T* __restrict__ rhs, T* x,
                                                      const int* __restrict__ rows, int count) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride) {
    const int q = rows[t];
    T sum = rhs[q];
    T xd = (T)0;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const T a = val[mat_index<T>(k, q, pitch)];
      const T xv = x[col[mat_index<T>(k, q, pitch)]];
      sum -= a * xv;
      if (k == kDiagSlot) xd = xv;
    }
    const T d = val[mat_index<T>(kDiagSlot, q, pitch)];
    sum += xd * d;
    x[q] = sum / d;
  }
}

// Storage row of the t-th row in slab order: z pair after z pair, inside a z
// pair colour after colour (each one run of storage). Needs even grid
// dimensions. Rows are below 2^31, so the divisions are 32-bit ones.
__device__ __forceinline__ int64_t slab_row(const ColourGrid& g, int64_t t) {
  const unsigned per = (unsigned)(g.nx >> 1) * (unsigned)(g.ny >> 1);  // rows of one colour in one z pair
  const unsigned u = (unsigned)t;
  const unsigned h = u / (kColours * per);
  const unsigned rem = u - h * kColours * per;
  const unsigned s = rem / per;
  return g.start[s] + (int64_t)h * per + (rem - s * per);
}

// y = A x (ComputeSPMV_ref.cpp:61-70); DOT: also partials of x'y
// (the p'Ap of CG.cpp:119, fused).
// ORDER 0: rows in storage order (colour block after colour block). Each colour
// block then gathers the other seven colours' x across the whole grid again.
// ORDER 1: natural grid order (row q = old2new of the thread's natural index):
// the gathered x stay in a window of a few planes held in L2, but each warp
// reads two short runs of every slot.
// ORDER 2: slab order: the rows of one z pair in all eight colours, then the
// next z pair; inside a colour a slab is one contiguous run of storage, so the
// matrix streams in long runs and the x window still fits in L2 (needs even
// grid dimensions: every colour then holds (nx/2)(ny/2) rows per z pair).
template <typename T, bool DOT, int CFG, int ORDER, int SCHED = cfg_sched(CFG), int R = ORDER == 1 ? 1 : cfg_rows(CFG)>
__global__ void __launch_bounds__(kThreads, cfg_minb(CFG)) k_spmv(ColourGrid g, const T* __restrict__ val,
                                                                  const int* __restrict__ col, int64_t pitch,
                                                                  const T* __restrict__ x, T* __restrict__ y, int n,
                                                                  double* __restrict__ partials) {
  double acc = 0.0;
  if (R == 1) {
    const int stride = gridDim.x * blockDim.x;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
      int q = t;
      if (ORDER == 1) {
        const int ix = t % g.nx, iy = (t / g.nx) % g.ny, iz = t / (g.nx * g.ny);
        q = g.old2new(ix, iy, iz);
      } else if (ORDER == 2) {
        q = (int)slab_row(g, t);
      }
      T sum = (T)0;
      T xq = (T)0;
      if (SCHED == kStaged) {
        T a[kSlots];
        int cl[kSlots];
#pragma unroll
        for (int k = 0; k < kSlots; ++k) {
          a[k] = __ldcs(val + mat_index<T>(k, q, pitch));
          cl[k] = __ldcs(col + mat_index<T>(k, q, pitch));
        }
        T xv[kSlots];
#pragma unroll
        for (int k = 0; k < kSlots; ++k) xv[k] = __ldg(x + cl[k]);
#pragma unroll
        for (int k = 0; k < kSlots; ++k) sum += a[k] * xv[k];
        xq = xv[kDiagSlot];
      } else {
#pragma unroll
        for (int k = 0; k < kSlots; ++k) {
          const T xv = __ldg(x + col[mat_index<T>(k, q, pitch)]);
          sum += val[mat_index<T>(k, q, pitch)] * xv;
          if (k == kDiagSlot) xq = xv;
        }
      }
      y[q] = sum;
      if (DOT) acc += (double)xq * (double)sum;
    }
  } else {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * R;
    for (int64_t t0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * R; t0 < n; t0 += stride) {
      int64_t q0 = t0;
      // R rows of one run: per is a multiple of R (checked on the host)
      if (ORDER == 2) q0 = slab_row(g, t0);
      const int cnt = t0 + R <= n ? R : (int)(n - t0);
      if (cnt < R) {
        for (int q = (int)q0; q < n; ++q) {
          T sum = (T)0, xq = (T)0;
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            const T xv = __ldg(x + col[mat_index<T>(k, q, pitch)]);
            sum += val[mat_index<T>(k, q, pitch)] * xv;
            if (k == kDiagSlot) xq = xv;
          }
          y[q] = sum;
          if (DOT) acc += (double)xq * (double)sum;
        }
        continue;
      }
      T sum[R], xq[R];
#pragma unroll
      for (int r = 0; r < R; ++r) sum[r] = xq[r] = (T)0;
#pragma unroll
      for (int k = 0; k < kSlots; ++k) {
        T a[R];
        int c[R];
        load_vec<T, R>(val + mat_index<T>(k, q0, pitch), a);
        load_vec<int, R>(col + mat_index<T>(k, q0, pitch), c);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const T xv = __ldg(x + c[r]);
          sum[r] += a[r] * xv;
          if (k == kDiagSlot) xq[r] = xv;
        }
      }
      store_vec<T, R>(y + q0, sum);
      if (DOT) {
#pragma unroll
        for (int r = 0; r < R; ++r) acc += (double)xq[r] * (double)sum[r];
      }
    }
  }
  if (DOT) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
  }
}

// y = A x (and, DOT, the p'Ap partials) through the bulk-copy pipeline (SpMV
// configuration 7): the same sums as k_spmv, slot order from zero. ORDER 0:
// tiles in storage order; ORDER 2: slab order (tiles of one z pair in all eight
// colours, then the next z pair), which needs slab runs that split into whole
// tiles and colour blocks that start on an even row (checked on the host).
// Partials: one per block.
template <typename T, bool DOT, int ORDER, int PW = 0>
__global__ void __launch_bounds__(SpmvShape<T, PW>::threads, 1)
    k_spmv_bulk(ColourGrid g, const T* __restrict__ val, const int* __restrict__ col, int64_t pitch,
                const T* __restrict__ x, T* __restrict__ y, int n, double* __restrict__ partials, unsigned* fault,
                const __grid_constant__ CUtensorMap tm_val, const __grid_constant__ CUtensorMap tm_col,
                const unsigned char* __restrict__ colp, int sink) {
  static_assert(ORDER == 0 || ORDER == 2, "storage or slab order");
  const int ntiles = (n + kBulkRows - 1) / kBulkRows;
  double acc = 0.0;
  bulk_tiles<T, SpmvShape<T, PW>, spmv_early<T>()>(
      val, col, pitch, ntiles,
      [&](int tile) {
        return ORDER == 2 ? slab_row(g, (int64_t)tile * kBulkRows) : (int64_t)tile * kBulkRows;
      },
      [&](int64_t q0, const T* sv, const int* sc, int t, auto&&... release) {
        const int64_t q = q0 + t;
        if constexpr (sizeof...(release) > 0) {
          // the row's values and columns into registers, the stage back to the producer
          T a[kSlots];
          int c[kSlots];
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            a[k] = sv[k * kBulkRows + t];
            c[k] = stage_col<PW>(sc, k, t, sink);
          }
          (release(), ...);
          if (q >= n) return;
          T sum = (T)0;
          T xq = (T)0;
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            const T xv = __ldg(x + c[k]);
            sum += a[k] * xv;
            if (k == kDiagSlot) xq = xv;
          }
          y[q] = sum;
          if (DOT) acc += (double)xq * (double)sum;
          return;
        }
        if (q >= n) return;
        T sum = (T)0;
        T xq = (T)0;
#if HB_SPMV_GATHER_FIRST
        // all 27 gathers issued before the first product (the same sum)
        T xv[kSlots];
#pragma unroll
        for (int k = 0; k < kSlots; ++k) xv[k] = __ldg(x + stage_col<PW>(sc, k, t, sink));
#pragma unroll
        for (int k = 0; k < kSlots; ++k) sum += sv[k * kBulkRows + t] * xv[k];
        xq = xv[kDiagSlot];
#else
#pragma unroll
        for (int k = 0; k < kSlots; ++k) {
          const T xv = __ldg(x + stage_col<PW>(sc, k, t, sink));
          sum += sv[k * kBulkRows + t] * xv;
          if (k == kDiagSlot) xq = xv;
        }
#endif
        y[q] = sum;
        if (DOT) acc += (double)xq * (double)sum;
      },
      fault, tm_val, tm_col, colp);
  if (DOT) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
  }
}

// Restriction fused with the residual it needs (ComputeMG_ref.cpp:49-51):
// rc[q] = rf[f] - (A xf)[f] for each transfer pair (f, q) of f2c; the residual
// is formed only at the injected rows (ComputeRestriction_ref.cpp:51 reads no
// others). The pairs are sorted by fine row, so the matrix rows are streamed in
// storage order and only the coarse writes scatter.
template <typename T, int CFG, int SCHED = cfg_sched(CFG)>
__global__ void __launch_bounds__(kThreads, cfg_minb(CFG)) k_restrict(const T* __restrict__ val, const int* __restrict__ col,
                                                                      int64_t pitch, const T* __restrict__ rf,
                                                                      const T* __restrict__ xf,
                                                                      const int* __restrict__ tf,
                                                                      const int* __restrict__ tq, T* __restrict__ rc,
                                                                      int nc) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nc; t += stride) {
    const int f = tf[t];
    T sum = (T)0;
    if (SCHED == kStaged) {
      T a[kSlots];
      int cl[kSlots];
#pragma unroll
      for (int k = 0; k < kSlots; ++k) {
        a[k] = __ldcs(val + mat_index<T>(k, f, pitch));
        cl[k] = __ldcs(col + mat_index<T>(k, f, pitch));
      }
      T xv[kSlots];
#pragma unroll
      for (int k = 0; k < kSlots; ++k) xv[k] = __ldg(xf + cl[k]);
#pragma unroll
      for (int k = 0; k < kSlots; ++k) sum += a[k] * xv[k];
    } else {
#pragma unroll
      for (int k = 0; k < kSlots; ++k) sum += val[mat_index<T>(k, f, pitch)] * __ldg(xf + col[mat_index<T>(k, f, pitch)]);
    }
    rc[tq[t]] = rf[f] - sum;
  }
}

// The restriction through the bulk-copy pipeline (with SpMV configuration 7),
// when the injected rows are one run f0 .. f0 + nc of fine rows (tf[t] = f0 + t,
// checked on the host): the run is tiled like a phase. Same sums as k_restrict.
template <typename T, int PW = 0>
__global__ void __launch_bounds__(RestrictShape<T, PW>::threads, 1)
    k_restrict_bulk(const T* __restrict__ val, const int* __restrict__ col, int64_t pitch, const T* __restrict__ rf,
                    const T* __restrict__ xf, const int* __restrict__ tq, T* __restrict__ rc, int f0, int nc,
                    unsigned* fault, const __grid_constant__ CUtensorMap tm_val,
                    const __grid_constant__ CUtensorMap tm_col, const unsigned char* __restrict__ colp, int sink) {
  const int r1 = f0 + nc;
  const int a0 = f0 & ~(kBulkRows - 1);
  const int ntiles = (r1 - a0 + kBulkRows - 1) / kBulkRows;
  bulk_tiles<T, RestrictShape<T, PW>, restrict_early<T>()>(
      val, col, pitch, ntiles, [&](int tile) { return a0 + (int64_t)tile * kBulkRows; },
      [&](int64_t q0, const T* sv, const int* sc, int t, auto&&... release) {
        const int64_t f = q0 + t;
        if constexpr (sizeof...(release) > 0) {
          // the row's values and columns into registers, the stage back to the producer
          T a[kSlots];
          int c[kSlots];
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            a[k] = sv[k * kBulkRows + t];
            c[k] = stage_col<PW>(sc, k, t, sink);
          }
          (release(), ...);
          if (f < f0 || f >= r1) return;
          T sum = (T)0;
#pragma unroll
          for (int k = 0; k < kSlots; ++k) sum += a[k] * __ldg(xf + c[k]);
          rc[tq[f - f0]] = rf[f] - sum;
          return;
        }
        if (f < f0 || f >= r1) return;
        T sum = (T)0;
#pragma unroll
        for (int k = 0; k < kSlots; ++k) sum += sv[k * kBulkRows + t] * __ldg(xf + stage_col<PW>(sc, k, t, sink));
        rc[tq[f - f0]] = rf[f] - sum;
      },
      fault, tm_val, tm_col, colp);
}

// ComputeProlongation_ref.cpp:49 over the same sorted pairs
template <typename T>
__global__ void __launch_bounds__(kThreads) k_prolong(const int* __restrict__ tf, const int* __restrict__ tq,
                                                      const T* __restrict__ xc, T* __restrict__ xf, int nc) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nc; t += stride) xf[tf[t]] += xc[tq[t]];
}

// ---- vectors ----------------------------------------------------------------

// dst[i] = src[idx[i]]
template <typename T>
__global__ void __launch_bounds__(kThreads) k_gather(T* __restrict__ dst, const T* __restrict__ src,
                                                     const int* __restrict__ idx, int n) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[idx[i]];
}

// w = alpha x + beta y (ComputeWAXPBY_ref.cpp:52-67; its alpha == 1 and
// beta == 1 branches give the same bits, multiplication by 1.0 being exact).
// NORM: partials of w'w.
template <bool NORM>
__global__ void __launch_bounds__(kThreads) k_waxpby(int n, double alpha, const double* x, double beta,
                                                     const double* y, double* w,
                                                     double* __restrict__ partials) {
  const int stride = gridDim.x * blockDim.x;
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double v = alpha * x[i] + beta * y[i];
    w[i] = v;
    if (NORM) acc += v * v;
  }
  if (NORM) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
  }
}

// partials of x'y (ComputeDotProduct_ref.cpp:54-64); TWO: also of x'y2 into
// partials[gridDim.x + block] (the r'z_prev of flexible CG, sharing the read of x).
template <bool TWO>
__global__ void __launch_bounds__(kThreads) k_dot(int n, const double* __restrict__ x, const double* __restrict__ y,
                                                  const double* __restrict__ y2, double* __restrict__ partials) {
  const int stride = gridDim.x * blockDim.x;
  double acc = 0.0, acc2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double xi = x[i];
    acc += xi * y[i];
    if (TWO) acc2 += xi * y2[i];
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  if (TWO) {
    const double s2 = block_sum(acc2);
    if (threadIdx.x == 0) partials[gridDim.x + blockIdx.x] = s2;
  }
}

// Flexible-CG step of the mixed form: z = widen(x32) together with the partials
// of r'z (and of r'zprev for TWO) in k_dot<TWO>'s layout and order, so the
// conversion pass and the copy of z into zprev go away (z and zprev are two
// buffers whose roles alternate).
template <bool TWO>
__global__ void __launch_bounds__(kThreads) k_widen_dot(int n, const float* __restrict__ x32,
                                                        const double* __restrict__ r, double* __restrict__ z,
                                                        const double* __restrict__ zprev,
                                                        double* __restrict__ partials) {
  const int stride = gridDim.x * blockDim.x;
  double acc = 0.0, acc2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double zi = (double)x32[i];
    z[i] = zi;
    const double ri = r[i];
    acc += ri * zi;
    if (TWO) acc2 += ri * zprev[i];
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  if (TWO) {
    const double s2 = block_sum(acc2);
    if (threadIdx.x == 0) partials[gridDim.x + blockIdx.x] = s2;
  }
}

// partial maxima of |v1 - v2| (ComputeResidual.cpp:70-75)
__global__ void __launch_bounds__(kThreads) k_maxdiff(int n, const double* __restrict__ a,
                                                      const double* __restrict__ b, double* __restrict__ partials) {
  const int stride = gridDim.x * blockDim.x;
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double d = fabs(a[i] - b[i]);
    if (d > m) m = d;
  }
  const double s = block_max(m);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// ---- CG scalar bookkeeping on the device -----------------------------------


// The scalar update of `op` given the reduced value(s) (thread 0 only).
__device__ __forceinline__ void apply_fin(int op, double sum, double sum2, Scalars* s, double* out) {
  switch (op) {
    case kFinStore: *out = sum; break;
    case kFinNormr: s->normr2 = sum; break;
    case kFinRtzFirst: s->rtz = sum; break;
    case kFinRtz: s->oldrtz = s->rtz; s->rtz = sum; s->beta = sum / s->oldrtz; break;
    case kFinPap: s->pAp = sum; s->alpha = s->rtz / sum; break;
    case kFinFlex: s->oldrtz = s->rtz; s->rtz = sum; s->rzprev = sum2; s->beta = (sum - sum2) / s->oldrtz; break;
    case kFinMax: *out = sum; break;
    case kFinNormr0: s->normr2 = sum; s->normr0 = sqrt(sum); break;
    case kFinRtzIter:
      if (s->iter == 0) {
        s->rtz = sum;
      } else {
        s->oldrtz = s->rtz;
        s->rtz = sum;
        s->beta = sum / s->oldrtz;
      }
      break;
    default: break;
  }
}

// One block: fixed-order reduction of nparts partials (and of the second set
// at partials[nparts..] for kFinFlex), then the scalar update of `op`.
__global__ void __launch_bounds__(kThreads) k_finalize(const double* __restrict__ partials, int nparts, int op,
                                                       Scalars* s, double* out) {
  double acc = 0.0, acc2 = 0.0;
  if (op == kFinMax) {
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc = fmax(acc, partials[i]);
    const double m = block_max(acc);
    if (threadIdx.x == 0) *out = m;
    return;
  }
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += partials[i];
  if (op == kFinFlex)
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc2 += partials[nparts + i];
  const double sum = block_sum(acc);
  const double sum2 = op == kFinFlex ? block_sum(acc2) : 0.0;
  if (threadIdx.x != 0) return;
  apply_fin(op, sum, sum2, s, out);
}

// The ranks' values of one reduction, combined in rank order (a sum, or the
// maximum for kFinMax), then the scalar update of `op`: the allreduce of
// ComputeDotProduct_ref.cpp:70 / ComputeResidual.cpp:82 as one left fold.
__global__ void k_finalize_ranks(const double* __restrict__ vals, int nvals, int op, Scalars* s, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double acc = vals[0];
  for (int i = 1; i < nvals; ++i) acc = op == kFinMax ? fmax(acc, vals[i]) : acc + vals[i];
  apply_fin(op, acc, 0.0, s, out);
}

// p = z + beta p (CG.cpp:115 as WAXPBY(1, z, beta, p)) with the previous
// iteration's x update folded in: x = x + alpha p (CG.cpp:121, alpha still the
// previous iteration's) reads the p that this kernel reads anyway, so the r
// update that follows the SpMV need not read p. The same operations on the
// same values as x = x + alpha p after the SpMV and p = z + beta p here.
// first (iteration 1): p = z (CG.cpp:109), x untouched.
__device__ __forceinline__ void update_px(int n, const double* __restrict__ z, double* p, double* x,
                                          const Scalars* __restrict__ s, bool first) {
  const double beta = s->beta, alpha = s->alpha;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (first) {
      p[i] = z[i];
    } else {
      const double pi = p[i];
      x[i] = x[i] + alpha * pi;
      p[i] = z[i] + beta * pi;
    }
  }
}
__global__ void __launch_bounds__(kThreads) k_update_px(int n, const double* __restrict__ z, double* p, double* x,
                                                        const Scalars* __restrict__ s) {
  update_px(n, z, p, x, s, false);
}
// iteration-aware form for the graph's loop body (s->iter: iterations completed)
__global__ void __launch_bounds__(kThreads) k_update_px_iter(int n, const double* __restrict__ z, double* p,
                                                             double* x, const Scalars* __restrict__ s) {
  update_px(n, z, p, x, s, s->iter == 0);
}

// r = r + (-alpha) Ap (CG.cpp:122) and partials of r'r (CG.cpp:123); x waits
// for the next k_update_px (or k_update_x after the loop). r32 (the mixed
// form): also r narrowed to FP32 for the next V-cycle.
__global__ void __launch_bounds__(kThreads) k_update_r(int n, double* r, const double* __restrict__ Ap,
                                                       const Scalars* __restrict__ s, double* __restrict__ partials,
                                                       float* __restrict__ r32 = nullptr) {
  const double malpha = -s->alpha;
  const int stride = gridDim.x * blockDim.x;
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double ri = r[i] + malpha * Ap[i];
    r[i] = ri;
    if (r32) r32[i] = (float)ri;
    acc += ri * ri;
  }
  const double sum = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = sum;
}

// The last iteration's x = x + alpha p (CG.cpp:121), after the loop; with
// iter_gate, only if the graph's loop completed an iteration (s->iter > 0).
__global__ void __launch_bounds__(kThreads) k_update_x(int n, double* x, const double* __restrict__ p,
                                                       const Scalars* __restrict__ s, int iter_gate) {
  if (iter_gate && s->iter == 0) return;
  const double alpha = s->alpha;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = x[i] + alpha * p[i];
}

// The loop condition of CG.cpp:100, k <= max_iter && normr/normr0 > tolerance,
// evaluated on the device for the graph's while node. advance = 0 before the
// loop (no iteration done yet), 1 at the end of each iteration.
__global__ void k_cg_condition(Scalars* s, cudaGraphConditionalHandle h, int advance) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  s->iter = advance ? s->iter + 1 : 0;
  const bool go = s->iter + 1 <= s->max_iter && sqrt(s->normr2) / s->normr0 > s->tol;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

__global__ void k_cg_setup(Scalars* s, int max_iter, double tol) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s->max_iter = max_iter;
    s->tol = tol;
    s->iter = 0;
  }
}

// Implicit adjoint, value part: with lambda solving A' lambda = dL/dx (A is
// symmetric), dL/da_ij = -lambda_i x_j for every stored slot. One thread per
// natural row i writes its 27 slots out[i*27 + k] (0 for a direction that leaves
// the grid), the layout hpcg_b200_set_values takes; lambda and x are in colour
// order.
__global__ void __launch_bounds__(kThreads) k_adjoint_values(ColourGrid g, const int* __restrict__ col,
                                                             int64_t pitch, int n, const double* __restrict__ lam,
                                                             const double* __restrict__ x,
                                                             double* __restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int ix = i % g.nx, iy = (i / g.nx) % g.ny, iz = i / (g.nx * g.ny);
    const int q = g.old2new(ix, iy, iz);
    const double l = lam[q];
    double* o = out + (int64_t)i * kSlots;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const int c = col[mat_index<double>(k, q, pitch)];
      o[k] = c == n ? 0.0 : -(l * x[c]);
    }
  }
}

// precision conversion for the FP32 V-cycle
template <typename TO, typename TI>
__global__ void __launch_bounds__(kThreads) k_convert(TO* __restrict__ dst, const TI* __restrict__ src, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = (TO)src[i];
}

}  // namespace hb
