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
// phase j-1): virtual unit v = t * P + j for t = 0 .. H + lag (P - 1) - 1,
// empty where h = t - lag j falls outside the grid. Their tiles follow one
// another; tile i goes to block i mod grid, each block's in order, so every
// tile waits only on tiles before it and, with every block resident (a
// cooperative launch), the sweep always advances. The x of the z pairs between
// the leading and the trailing phase (about lag * P + 3 z pairs) stays in L2
// while the matrix streams past it (evict-first), so x is read once and
// written once per sweep.
//
// The pipeline is the bulk-copy one (bulk.cuh) with a fourth role:
//   - the producer lane gives a tile's stage to its consumers only once the
//     tile's unit's dependencies have finished: per-unit counters of finished
//     tiles, read with relaxed loads (a tile ahead), then one fence. That is
//     the full barrier's second arrival, so the matrix copies are in flight
//     meanwhile;
//   - a counting lane (warp 1) takes each stage its consumers have released,
//     in the block's tile order, as a finished tile of its unit, and hands the
//     stage back to the producer (the `counted` barrier, on which the producer
//     refills). It adds the counts to the unit counters in batches: one fence
//     at GPU scope (cumulative: it publishes the consumers' x writes, which the
//     empty barrier ordered before it) and one atomic add, when the next tile
//     belongs to another unit and whenever it has to wait, so the block's own
//     finished tiles never hold up the tiles its producer waits for.
// Each role walks the block's tiles with the same division-free iterator.
// Every wait is bounded (limit_ns of global time, kBulkWaitNs in the solver;
// twice that for the waits that may sit behind a dependency wait): one that
// gives up records fault code 6 (dependency) or 1-3 (pipeline) and the kernel
// winds down; the host's stream synchronisation returns HPCG_B200_ERR_TIMEOUT.
#pragma once

#include "bulk.cuh"

namespace hb {

// virtual units of a sweep (WaveGeom, common.cuh): P per step of t, empty ones included
__host__ __device__ inline int wave_units(const WaveGeom& w) { return w.P * (w.H + w.lag * (w.P - 1)); }

__device__ __forceinline__ unsigned ld_relaxed_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
// non-blocking: whether the barrier's phase of this parity has completed
__device__ __forceinline__ bool mbar_probe(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// The block's walk over the virtual tiles blockIdx.x, + gridDim.x, ...: unit
// v = t * P + j (t the wavefront step, j the phase), tile k of the unit.
// The sweep's pipeline shape: consumer groups (HB_WAVE_GROUPS, as many as fit)
// of two-stage rings.
#ifndef HB_WAVE_GROUPS
#define HB_WAVE_GROUPS 3
#endif
template <typename T, int PW>
using WaveShape = BulkShape<T, fit_groups<T, PW>(HB_WAVE_GROUPS, HB_BULK_RING), HB_BULK_RING, 1, PW>;

struct WaveIter {
  int v, k, t, j;
  __device__ __forceinline__ void init(int tile, int tpu, int P) {
    v = tile / tpu;
    k = tile - v * tpu;
    t = v / P;
    j = v - t * P;
  }
  __device__ __forceinline__ void next(int tpu, int P) {
    k += gridDim.x;
    while (k >= tpu) {
      k -= tpu;
      ++v;
      if (++j == P) {
        j = 0;
        ++t;
      }
    }
  }
  __device__ __forceinline__ int h(int lag) const { return t - lag * j; }
  __device__ __forceinline__ bool valid(int lag, int H) const { return h(lag) >= 0 && h(lag) < H; }
};

// Gauss-Seidel sweep over the units of w (configuration 10's phase
// arithmetic, all 27 slots, x entering nonzero); done: one zeroed counter per
// virtual unit; dot (or nullptr): block partials of r'x of the rows of phases
// j >= w.dot_from, at dot[blockIdx.x]. Blocks of wave_threads<T, PW>() threads.
template <typename T, int PW>
__host__ __device__ constexpr int wave_threads() {
  return WaveShape<T, PW>::threads + 32;
}
template <typename T, int PW>
__global__ void __launch_bounds__(wave_threads<T, PW>(), 1)
    k_gs_wave(const T* __restrict__ val, const int* __restrict__ col, int64_t pitch, const T* __restrict__ rhs,
              T* x, const WaveGeom w, unsigned* done, double* __restrict__ dot, unsigned* fault,
              const __grid_constant__ CUtensorMap tm_val, const __grid_constant__ CUtensorMap tm_col,
              const unsigned char* __restrict__ colp, int sink, unsigned long long limit_ns) {
  using Shape = WaveShape<T, PW>;
  static_assert(bulk_tensor_tile<T>(), "FP64 tiles by tensor copy");
  constexpr int G = Shape::groups;
  constexpr int RING = Shape::ring;
  constexpr int S = Shape::stages;
  constexpr int SB = Shape::stage_bytes;
  constexpr int VB = Shape::value_bytes;
  constexpr int64_t kDotBit = 1ll << 62;  // marks a tile whose rows add r'x
  static_assert(S <= 16, "stage bookkeeping");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * SB);
  uint64_t* empty = full + S;
  int64_t* first = reinterpret_cast<int64_t*>(empty + S);  // q0 (| kDotBit) of the tile in each stage
  __shared__ uint64_t counted[S];  // the counting lane has taken the stage's tile: the producer may refill
  __shared__ int stage_unit[S];     // virtual unit of the tile in each stage
  __shared__ int issued_end;        // the producer's count of released tiles once it stops (INT_MAX before)
  __shared__ int start[kColours];   // w.start (indexed by phase)
  // the geometry in registers (the parameter struct would be copied to local memory)
  const int H = w.H, P = w.P, lag = w.lag, tpu = w.tpu, per = w.per, dot_from = w.dot_from;
  const int self_dep = w.self_dep;
#pragma unroll
  for (int q = 0; q < kColours; ++q)  // constant indices: the parameter stays in the constant bank
    if (threadIdx.x == q) start[q] = w.start[q];
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 2);  // the copies' arrival and the dependencies' arrival
      mbar_init(&empty[s], Shape::group_threads);
      mbar_init(&counted[s], 1);
    }
    mbar_init_fence();
    issued_end = 0x7fffffff;
  }
  __syncthreads();
  const int nunits = P * (H + lag * (P - 1));
  const int warp = threadIdx.x >> 5;
  double acc = 0.0;
  if (warp == 0) {
    if (threadIdx.x == 0) {
      // ---- producer
      const uint64_t policy = evict_first_policy();
      auto deps_of = [&](int j, int h, int (&dv)[3]) {
        dv[0] = dv[1] = dv[2] = -1;
        if (self_dep >= 0) {
          dv[0] = self_dep;
          return;
        }
        if (j == 0) return;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int hh = h - 1 + d;
          if (hh >= 0 && hh < H) dv[d] = (hh + lag * (j - 1)) * P + (j - 1);
        }
      };
      auto read_counts = [&](const int (&dv)[3], unsigned (&cnt)[3]) {
#pragma unroll
        for (int d = 0; d < 3; ++d) cnt[d] = dv[d] >= 0 ? ld_relaxed_gpu(done + dv[d]) : (unsigned)tpu;
      };
      auto all_done = [&](const unsigned (&cnt)[3]) {
        return cnt[0] >= (unsigned)tpu && cnt[1] >= (unsigned)tpu && cnt[2] >= (unsigned)tpu;
      };
      bool ok = true;
      int checked = -1;  // the last unit whose dependencies were seen finished
      int i = 0;         // tiles released so far
      int pre_v = -1, pre_dv[3] = {-1, -1, -1};  // the next unit's dependencies and their counters
      unsigned pre_cnt[3] = {0, 0, 0};
      WaveIter it;
      for (it.init(blockIdx.x, tpu, P); it.v < nunits; it.next(tpu, P)) {
        if (!it.valid(lag, H)) continue;
        const int v = it.v, j = it.j, h = it.h(lag);
        const int kg = i / G;
        const int s = (i % G) * RING + kg % RING, use = kg / RING;
        if (use > 0 && !mbar_wait(&counted[s], (use - 1) & 1, 2 * limit_ns)) {
          record_fault(fault, 1);
          ok = false;
          break;
        }
        const int64_t q0 = (int64_t)start[j] + (int64_t)h * per + (int64_t)it.k * kBulkRows;
        first[s] = q0 | (j >= dot_from ? kDotBit : 0);
        stage_unit[s] = v;
        T* sv = reinterpret_cast<T*>(smem + s * SB);
        int* sc = reinterpret_cast<int*>(smem + s * SB + VB);
        mbar_expect_tx(&full[s], Shape::tx_bytes);
        tma_load_2d(sv, &tm_val, (int)q0, 0, &full[s], policy);
        if constexpr (Shape::packed)
          bulk_g2s(sc, colp + (q0 / kBulkRows) * pack_rec(PW), Shape::col_bytes, &full[s], policy);
        else
          tma_load_2d(sc, &tm_col, (int)q0, 0, &full[s], policy);
        if (v != checked) {
          int dv[3];
          unsigned cnt[3];
          if (v == pre_v) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              dv[d] = pre_dv[d];
              cnt[d] = pre_cnt[d];
            }
          } else {
            deps_of(j, h, dv);
            read_counts(dv, cnt);
          }
          const unsigned long long t0 = global_ns();
          while (!all_done(cnt)) {
            if (global_ns() - t0 > limit_ns) {
              record_fault(fault, 6);
              ok = false;
              break;
            }
            read_counts(dv, cnt);
          }
          if (ok) {
            fence_acq_rel_gpu();  // with the loads that saw the counters: the dependencies' x writes are visible
            checked = v;
          }
          // read the next unit's dependency counters now (its first tile is
          // usually the block's next but few)
          int nt = v + 1, nj = j + 1, ntt = it.t;
          if (nj == P) {
            nj = 0;
            ++ntt;
          }
          for (int guard = 0; guard < P && nt < nunits; ++guard) {  // the next non-empty unit
            const int nh = ntt - lag * nj;
            if (nh >= 0 && nh < H) {
              pre_v = nt;
              deps_of(nj, nh, pre_dv);
              read_counts(pre_dv, pre_cnt);
              break;
            }
            ++nt;
            if (++nj == P) {
              nj = 0;
              ++ntt;
            }
          }
        }
        // the stage goes to its consumers (after a dependency wait gave up too:
        // the launch's results are void then, but the stage's copies must land
        // and be consumed before the block may exit)
        mbar_arrive(&full[s]);
        ++i;
        if (!ok) break;
      }
      *(volatile int*)&issued_end = i;  // the consumers and the counting lane stop there
    }
  } else if (warp == 1) {
    if (threadIdx.x == 32) {
      // ---- counting lane
      int pub_unit = -1;  // finished tiles not yet added to the counters: unit and count
      unsigned pub_cnt = 0;
      auto publish = [&]() {
        if (!pub_cnt) return;
        fence_acq_rel_gpu();
        atomicAdd(done + pub_unit, pub_cnt);
        pub_cnt = 0;
      };
      int i = 0;
      WaveIter it;
      for (it.init(blockIdx.x, tpu, P); it.v < nunits; it.next(tpu, P)) {
        if (!it.valid(lag, H)) continue;
        const int kg = i / G;
        const int s = (i % G) * RING + kg % RING, use = kg / RING;
        bool got = true;
        if (!mbar_probe(&empty[s], use & 1)) {
          publish();  // about to wait: nothing of this block's may stay unpublished
          const unsigned long long t0 = global_ns();
          while (!mbar_test(&empty[s], use & 1)) {
            if (i >= *(volatile int*)&issued_end) {  // the producer stopped before this tile
              got = false;
              break;
            }
            if (global_ns() - t0 > 2 * limit_ns) {
              record_fault(fault, 2);
              got = false;
              break;
            }
          }
        }
        if (!got) break;
        const int u = stage_unit[s];
        if (pub_cnt && pub_unit != u) publish();
        pub_unit = u;
        ++pub_cnt;
        mbar_arrive(&counted[s]);
        ++i;
      }
      publish();
    }
  } else {
    // ---- consumers
    const int g = (warp - 2) / (Shape::group_threads / 32);
    const int t = (threadIdx.x - 64) % Shape::group_threads;
    int i = 0;
    WaveIter it;
    for (it.init(blockIdx.x, tpu, P); it.v < nunits; it.next(tpu, P)) {
      if (!it.valid(lag, H)) continue;
      if (i % G != g) {
        ++i;
        continue;
      }
      const int kg = i / G;
      const int s = g * RING + kg % RING, use = kg / RING;
      bool got = true;
      const unsigned long long t0 = global_ns();
      while (!mbar_test(&full[s], use & 1)) {
        if (i >= *(volatile int*)&issued_end) {  // the producer stopped before this tile
          got = false;
          break;
        }
        if (global_ns() - t0 > 2 * limit_ns) {  // the producer may spend limit_ns on the tile's dependencies
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
      ++i;
    }
  }
  if (dot) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) dot[blockIdx.x] = s;
  }
}

}  // namespace hb
