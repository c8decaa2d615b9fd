// One Gauss-Seidel sweep (all its colour phases) in one launch, as a wavefront
// over z pairs, so that x crosses DRAM about once per sweep instead of once per
// phase.
//
// A phase-by-phase sweep reads, in every phase, the other seven colours' x
// around each row from DRAM (L2 holds no x between phases: each phase streams
// its matrix through it), 56 of the 292.25 bytes a row moves on the diagonal
// column form. Here the work is cut into units: the rows of one phase (sweep
// position) in one z pair, (nx/2)(ny/2) rows of whole 128-row tiles. Unit
// (j, h), phase j of the sweep in z pair h, reads x of z pairs h-1 .. h+1 and
// needs phase j-1 finished there; by induction that makes every earlier phase
// finished on every row it reads, and no later phase writes a row it reads
// before it has finished (phase j+1 at h' waits for phase j at h'-1 .. h'+1).
// So each row computes exactly the bits of the phase-by-phase sweep.
//
// The units go in the order of t = h + lag * j (phase j runs lag z pairs behind
// phase j-1), and their tiles one after another; tile i goes to block i mod
// grid, each block's in order, so every tile waits only on tiles before it and,
// with every block resident (a cooperative launch), the sweep always advances.
// The x of the z pairs between the leading and the trailing phase (about
// 8 * lag + 3 z pairs) stays in L2 while the matrix streams past it
// (evict-first), so x is read once and written once per sweep.
//
// The pipeline is the bulk-copy one (bulk.cuh) with two additions on the
// producer lane:
//   - before a tile's stage is released to the consumers it waits until the
//     tile's unit's dependencies have finished (the per-unit counters of
//     finished tiles, polled with relaxed loads, then one fence), on the full
//     barrier's second arrival, so the matrix copies are in flight meanwhile;
//   - when the consumers have released a stage it counts the tile as finished:
//     a fence at GPU scope (cumulative: it publishes the consumers' x writes,
//     which the empty barrier ordered before it), then one atomic add on the
//     unit's counter. It serves these while it waits for anything, so its own
//     finished tiles never hold up the tiles it waits for.
// Every wait is bounded (limit_ns of global time, kBulkWaitNs in the solver):
// one that gives up records fault code 6 (dependency) or 1-3 (pipeline) and
// the kernel winds down; the host's stream synchronisation returns
// HPCG_B200_ERR_TIMEOUT.
#pragma once

#include "bulk.cuh"

namespace hb {

// One unit of a wavefront sweep: its first row and the units it waits for
// (indices in the launch's unit order, -1: none); dot: its rows add r'x.
struct WaveUnit {
  int row0;
  int dep[3];
  int dot;
  int pad[3];
};

__device__ __forceinline__ unsigned ld_relaxed_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Gauss-Seidel sweep of `nunits` units of `tpu` tiles each (configuration 10's
// phase arithmetic, all 27 slots, x entering nonzero); done: one zeroed counter
// per unit; dot (or nullptr): block partials of r'x of the rows of units with
// dot set, at dot[blockIdx.x].
template <typename T, int PW>
__global__ void __launch_bounds__(GsShape<T, PW>::threads, 1)
    k_gs_wave(const T* __restrict__ val, const int* __restrict__ col, int64_t pitch, const T* __restrict__ rhs,
              T* x, const WaveUnit* __restrict__ units, int nunits, int tpu, unsigned* done,
              double* __restrict__ dot, unsigned* fault, const __grid_constant__ CUtensorMap tm_val,
              const __grid_constant__ CUtensorMap tm_col, const unsigned char* __restrict__ colp, int sink,
              unsigned long long limit_ns) {
  using Shape = GsShape<T, PW>;
  static_assert(bulk_tensor_tile<T>(), "FP64 tiles by tensor copy");
  constexpr int G = Shape::groups;
  constexpr int RING = Shape::ring;
  constexpr int S = Shape::stages;
  constexpr int SB = Shape::stage_bytes;
  constexpr int VB = Shape::value_bytes;
  constexpr int64_t kDotBit = 1ll << 62;  // marks a tile whose rows add r'x
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * SB);
  uint64_t* empty = full + S;
  int64_t* first = reinterpret_cast<int64_t*>(empty + S);  // q0 (| kDotBit) of the tile in each stage
  __shared__ int issued_end;  // the producer's count of released tiles once it stops (INT_MAX before)
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 2);  // the copies' arrival and the dependencies' arrival
      mbar_init(&empty[s], Shape::group_threads);
    }
    mbar_init_fence();
    issued_end = 0x7fffffff;
  }
  __syncthreads();
  const int ntiles = nunits * tpu;
  const int warp = threadIdx.x >> 5;
  double acc = 0.0;
  if (warp == 0) {
    if (threadIdx.x == 0) {
      const uint64_t policy = evict_first_policy();
      int fill_unit[S], fill_use[S];
      bool pending[S];  // consumed-but-not-counted state of each stage's last fill
#pragma unroll
      for (int s = 0; s < S; ++s) {
        fill_unit[s] = -1;
        fill_use[s] = -1;
        pending[s] = false;
      }
      // counts every stage whose last fill the consumers have released
      auto service = [&]() {
        bool any = false;
#pragma unroll
        for (int s = 0; s < S; ++s)
          if (pending[s] && mbar_test(&empty[s], fill_use[s] & 1)) any = true;
        if (!any) return;
        __threadfence();
#pragma unroll
        for (int s = 0; s < S; ++s)
          if (pending[s] && mbar_test(&empty[s], fill_use[s] & 1)) {
            pending[s] = false;
            atomicAdd(done + fill_unit[s], 1u);
          }
      };
      bool ok = true;
      int checked = -1;  // the last unit whose dependencies were seen finished
      int i = 0;         // tiles released so far
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int u = tile / tpu;
        const int kg = i / G;
        const int s = (i % G) * RING + kg % RING, use = kg / RING;
        if (use > 0) {  // the stage's previous tile must be consumed (and is counted here)
          const unsigned long long t0 = global_ns();
          while (!mbar_test(&empty[s], (use - 1) & 1)) {
            service();
            if (global_ns() - t0 > limit_ns) {
              record_fault(fault, 1);
              ok = false;
              break;
            }
          }
          if (!ok) break;
          service();
        }
        const WaveUnit wu = units[u];
        const int64_t q0 = (int64_t)wu.row0 + (int64_t)(tile - u * tpu) * kBulkRows;
        first[s] = q0 | (wu.dot ? kDotBit : 0);
#pragma unroll
        for (int v = 0; v < S; ++v)  // constant indices keep the stage state in registers
          if (v == s) {
            fill_unit[v] = u;
            fill_use[v] = use;
            pending[v] = true;
          }
        T* sv = reinterpret_cast<T*>(smem + s * SB);
        int* sc = reinterpret_cast<int*>(smem + s * SB + VB);
        mbar_expect_tx(&full[s], Shape::tx_bytes);
        tma_load_2d(sv, &tm_val, (int)q0, 0, &full[s], policy);
        if constexpr (Shape::packed)
          bulk_g2s(sc, colp + (q0 / kBulkRows) * pack_rec(PW), Shape::col_bytes, &full[s], policy);
        else
          tma_load_2d(sc, &tm_col, (int)q0, 0, &full[s], policy);
        if (u != checked) {
          const unsigned long long t0 = global_ns();
          for (int d = 0; d < 3 && ok; ++d) {
            const int du = wu.dep[d];
            if (du < 0) continue;
            while (ld_relaxed_gpu(done + du) < (unsigned)tpu) {
              service();
              if (global_ns() - t0 > limit_ns) {
                record_fault(fault, 6);
                ok = false;
                break;
              }
            }
          }
          if (ok) {
            __threadfence();  // with the loads that saw the counters: the dependencies' x writes are visible
            checked = u;
          }
        }
        // the stage goes to its consumers (after a dependency wait gave up too:
        // the launch's results are void then, but the stage's copies must land
        // and be consumed before the block may exit)
        mbar_arrive(&full[s]);
        ++i;
        if (!ok) break;
      }
      *(volatile int*)&issued_end = i;  // the consumers stop there
      // count the tiles still in flight once their consumers release them
      const unsigned long long t0 = global_ns();
      for (;;) {
        service();
        bool left = false;
#pragma unroll
        for (int s = 0; s < S; ++s) left = left || pending[s];
        if (!left) break;
        if (global_ns() - t0 > limit_ns) {
          record_fault(fault, 2);
          break;
        }
      }
    }
  } else {
    const int g = (warp - 1) / (Shape::group_threads / 32);
    const int t = (threadIdx.x - 32) % Shape::group_threads;
    int i = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
      if (i % G != g) continue;
      const int kg = i / G;
      const int s = g * RING + kg % RING, use = kg / RING;
      bool got = true;
      const unsigned long long t0 = global_ns();
      while (!mbar_test(&full[s], use & 1)) {
        if (i >= *(volatile int*)&issued_end) {  // the producer stopped before this tile
          got = false;
          break;
        }
        if (global_ns() - t0 > limit_ns) {
          record_fault(fault, 3);
          got = false;
          break;
        }
      }
      if (!got) break;
      const int64_t f = first[s];
      const int64_t q = (f & ~kDotBit) + t;
      const T* sv = reinterpret_cast<const T*>(smem + s * SB);
      const int* sc = reinterpret_cast<const int*>(smem + s * SB + VB);
      T sum = rhs[q];
      T xd = (T)0;
#pragma unroll
      for (int k = 0; k < kSlots; ++k) {
        const T a = sv[k * kBulkRows + t];
        const T xv = x[stage_col<PW>(sc, k, t, sink)];  // coherent load: other blocks write x in this launch
        sum -= a * xv;
        if (k == kDiagSlot) xd = xv;
      }
      const T d = sv[kDiagSlot * kBulkRows + t];
      sum += xd * d;
      const T out = sum / d;
      x[q] = out;
      if (f & kDotBit) acc += (double)rhs[q] * (double)out;
      mbar_arrive(&empty[s]);
    }
  }
  if (dot) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) dot[blockIdx.x] = s;
  }
}

}  // namespace hb
