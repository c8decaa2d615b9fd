// Batched solves: many independent HPCG problems of different sizes advanced
// together by flexible CG in FP64 around the FP32 V-cycle (the mixed form of
// hpcg_b200_cg_mixed, per problem).
//
// Every step of an iteration is ONE kernel launch for the whole batch: the
// launch walks a work list of row tiles that spans all problems (a colour phase
// of every problem's level, a restriction, a vector update...), so a batch of
// small problems costs the launches of one. The iteration loop itself is one
// CUDA graph launch: a conditional while node repeats the iteration while any
// problem is still above its tolerance and the iteration limit is not reached;
// problems that have converged skip their tiles. No kernel waits on another.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bulk.cuh"
#include "reduce.cuh"
#include "rows.cuh"

namespace hb {

int prepare_f32(hpcg_b200_problem* p);
int free_problem(hpcg_b200_problem* p);
void release_accounted(size_t bytes);

namespace {

constexpr int kTile = kThreads;  // rows per tile: one thread per row
constexpr int kBlocksPerSm = 8;
constexpr uint64_t kBatchMagic = 0x48504347b2000b01ull;

// one problem's share of a Gauss-Seidel colour phase (FP32 V-cycle)
struct BGs {
  const float* val;
  const int* col;
  int64_t pitch;
  const float* rhs;
  float* x;
  int r0, r1;
  uint32_t mask;
  int first;
  int prob;
  const unsigned char* colp;  // the level's packed columns (bulk-copy phases)
  int pack;                   // their offset width in bytes
  int sink;                   // the level's zero sink column
};
// residual + restriction, and prolongation, of one problem's level
struct BRes {
  const float* val;
  const int* col;
  int64_t pitch;
  const float* rf;
  const float* xf;
  const int* tf;
  const int* tq;
  float* rc;
  int nc;
  int prob;
};
// the level-0 (outer, FP64) vectors of one problem
struct BVec {
  const double* val;
  const int* col;
  int64_t pitch;
  int n;
  double *b, *x, *r, *z, *zprev, *p, *Ap;
  float *r32, *x32;
};
struct BTile {
  int item;   // index into the step's item array (or the problem for vector tiles)
  int start;  // first row of the tile
};
// per-problem CG scalars
struct BScal {
  double rtz, oldrtz, alpha, beta, pAp, normr2, normr0, rzprev;
  int active, niters;
};
struct BCtl {
  int iter;  // iterations completed
  int max_iter;
  double tol;
};

// ---- kernels -----------------------------------------------------------------

__device__ __forceinline__ void b_gs(const BGs* __restrict__ items, const BTile* __restrict__ tiles,
                                                   int ntiles, const BScal* __restrict__ sc) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    const BGs it = items[tl.item];
    if (!sc[it.prob].active) continue;
    const int q = tl.start + threadIdx.x;
    if (q >= it.r1) continue;
    if (it.first)
      gs_row<float, float, true, kPlain, 0>(it.val, it.col, it.pitch, it.rhs, it.x, q, it.mask);
    else
      gs_row<float, float, false, kPlain, 0>(it.val, it.col, it.pitch, it.rhs, it.x, q, it.mask);
  }
}
__global__ void __launch_bounds__(kThreads) k_b_gs(const BGs* __restrict__ items, const BTile* __restrict__ tiles,
                                                   int ntiles, const BScal* __restrict__ sc) { b_gs(items, tiles, ntiles, sc); }

// The batched colour phase through the bulk-copy pipeline (bulk.cuh): every
// tile is one 128-row block of its problem's blocked FP32 values (val32 of the
// single-problem path) and one record of its packed columns, so it arrives by
// two copies; the tiles of problems that have converged are skipped on both
// sides. Same arithmetic as k_b_gs. The problems' levels may pack their
// columns with different offset widths: each tile's record states its own.
// Four consumer groups of one-block tiles.
#ifndef HB_BATCH_GROUPS
#define HB_BATCH_GROUPS 4
#endif
using BatchShape = BulkShape<float, fit_groups<float, -1>(HB_BATCH_GROUPS, HB_BULK_RING), HB_BULK_RING, 1, -1>;
__global__ void __launch_bounds__(BatchShape::threads, 1)
    k_b_gs_bulk(const BGs* __restrict__ items, const BTile* __restrict__ tiles, int ntiles,
                const BScal* __restrict__ sc, unsigned* fault) {
  bulk_tiles_src<float, BatchShape>(
      ntiles,
      [&](int t) {
        const BTile tl = tiles[t];
        const BGs& it = items[tl.item];
        return TileSrc<float>{tl.start, it.val + mat_index<float>(0, tl.start, it.pitch),
                              it.col + mat_index<float>(0, tl.start, it.pitch),
                              it.colp + (tl.start / kBulkRows) * pack_rec(it.pack), pack_rec(it.pack)};
      },
      [&](int t) { return !sc[items[tiles[t].item].prob].active; },
      [&](int t, int64_t q0, const float* sv, const int* scol, int row) {
        const BGs& it = items[tiles[t].item];
        const int64_t q = q0 + row;
        if (q < it.r0 || q >= it.r1) return;
        const uint32_t mask = it.mask;
        float sum = it.rhs[q];
        float xd = 0.0f;
        if (mask == kAllSlots) {  // full-slot phases: the 27 gathers without a test each
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            const float a = sv[k * kBulkRows + row];
            const float xv = __ldg(it.x + stage_col<-1>(scol, k, row, it.sink));
            sum -= a * xv;
            if (k == kDiagSlot) xd = xv;
          }
        } else {
#pragma unroll
          for (int k = 0; k < kSlots; ++k) {
            if (mask & (1u << k)) {
              const float a = sv[k * kBulkRows + row];
              const float xv = __ldg(it.x + stage_col<-1>(scol, k, row, it.sink));
              sum -= a * xv;
              if (k == kDiagSlot) xd = xv;
            }
          }
        }
        const float d = sv[kDiagSlot * kBulkRows + row];
        if (!it.first) sum += xd * d;
        it.x[q] = sum / d;
      },
      fault, nullptr, nullptr);
}

// rc = (rf - A xf) at the injected rows (ComputeMG_ref.cpp:49-51, sorted pairs)
__device__ __forceinline__ void b_restrict(const BRes* __restrict__ items,
                                                         const BTile* __restrict__ tiles, int ntiles,
                                                         const BScal* __restrict__ sc) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    const BRes it = items[tl.item];
    if (!sc[it.prob].active) continue;
    const int u = tl.start + threadIdx.x;
    if (u >= it.nc) continue;
    const int f = it.tf[u];
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < kSlots; ++k)
      sum += it.val[mat_index<float, 0>(k, f, it.pitch)] * __ldg(it.xf + it.col[mat_index<float, 0>(k, f, it.pitch)]);
    it.rc[it.tq[u]] = it.rf[f] - sum;
  }
}
__global__ void __launch_bounds__(kThreads) k_b_restrict(const BRes* __restrict__ items,
                                                         const BTile* __restrict__ tiles, int ntiles,
                                                         const BScal* __restrict__ sc) { b_restrict(items, tiles, ntiles, sc); }

// xf[f] += xc[q] (ComputeProlongation_ref.cpp:49); prolongation items carry xc in
// rf and the fine solution in rc
__device__ __forceinline__ void b_prolong(const BRes* __restrict__ items,
                                                        const BTile* __restrict__ tiles, int ntiles,
                                                        const BScal* __restrict__ sc) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    const BRes it = items[tl.item];
    if (!sc[it.prob].active) continue;
    const int u = tl.start + threadIdx.x;
    if (u >= it.nc) continue;
    it.rc[it.tf[u]] += it.rf[it.tq[u]];
  }
}
__global__ void __launch_bounds__(kThreads) k_b_prolong(const BRes* __restrict__ items,
                                                        const BTile* __restrict__ tiles, int ntiles,
                                                        const BScal* __restrict__ sc) { b_prolong(items, tiles, ntiles, sc); }

// y = A x (FP64 outer SpMV, CG.cpp:118); DOT: partial of x'y per tile
template <bool DOT>
__device__ __forceinline__ void b_spmv(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                     int ntiles, int use_p, const BScal* __restrict__ sc,
                                                     double* __restrict__ partials) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    const BVec it = v[tl.item];
    double acc = 0.0;
    const bool act = sc == nullptr || sc[tl.item].active;
    const int q = tl.start + threadIdx.x;
    if (act && q < it.n) {
      const double* x = use_p ? it.p : it.x;
      double sum = 0.0, xq = 0.0;
#pragma unroll
      for (int k = 0; k < kSlots; ++k) {
        const double xv = __ldg(x + it.col[k * it.pitch + q]);
        sum += it.val[k * it.pitch + q] * xv;
        if (k == kDiagSlot) xq = xv;
      }
      it.Ap[q] = sum;
      if (DOT) acc = xq * sum;
    }
    if (DOT) {
      const double s = block_sum(acc);
      if (threadIdx.x == 0) partials[t] = s;
    }
  }
}
template <bool DOT>
__global__ void __launch_bounds__(kThreads) k_b_spmv(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                     int ntiles, int use_p, const BScal* __restrict__ sc,
                                                     double* __restrict__ partials) { b_spmv<DOT>(v, tiles, ntiles, use_p, sc, partials); }

// r = 1.0 b + (-1.0) Ap (CG.cpp:88) and partial of r'r
__device__ __forceinline__ void b_resid(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                      int ntiles, double* __restrict__ partials) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    const BVec it = v[tl.item];
    const int q = tl.start + threadIdx.x;
    double acc = 0.0;
    if (q < it.n) {
      const double r = 1.0 * it.b[q] + -1.0 * it.Ap[q];
      it.r[q] = r;
      acc = r * r;
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) partials[t] = s;
  }
}
__global__ void __launch_bounds__(kThreads) k_b_resid(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                      int ntiles, double* __restrict__ partials) { b_resid(v, tiles, ntiles, partials); }

// r32 = (float) r: the FP32 V-cycle's right-hand side
__device__ __forceinline__ void b_to32(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                     int ntiles, const BScal* __restrict__ sc) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    if (!sc[tl.item].active) continue;
    const BVec it = v[tl.item];
    const int q = tl.start + threadIdx.x;
    if (q < it.n) it.r32[q] = (float)it.r[q];
  }
}
__global__ void __launch_bounds__(kThreads) k_b_to32(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                     int ntiles, const BScal* __restrict__ sc) { b_to32(v, tiles, ntiles, sc); }

// z = (double) x32; partials of r'z and r'zprev (flexible beta)
__device__ __forceinline__ void b_to64_dots(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                          int ntiles, const BScal* __restrict__ sc,
                                                          double* __restrict__ partials) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    const BVec it = v[tl.item];
    const int q = tl.start + threadIdx.x;
    double a1 = 0.0, a2 = 0.0;
    if (sc[tl.item].active && q < it.n) {
      const double z = (double)it.x32[q];
      it.z[q] = z;
      const double r = it.r[q];
      a1 = r * z;
      a2 = r * it.zprev[q];
    }
    const double s1 = block_sum(a1);
    const double s2 = block_sum(a2);
    if (threadIdx.x == 0) {
      partials[t] = s1;
      partials[ntiles + t] = s2;
    }
  }
}
__global__ void __launch_bounds__(kThreads) k_b_to64_dots(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                          int ntiles, const BScal* __restrict__ sc,
                                                          double* __restrict__ partials) { b_to64_dots(v, tiles, ntiles, sc, partials); }

// iteration 1: p = z; later: p = z + beta p; then zprev = z
__device__ __forceinline__ void b_update_p(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                         int ntiles, const BScal* __restrict__ sc,
                                                         const BCtl* __restrict__ ctl) {
  const bool first = ctl->iter == 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    if (!sc[tl.item].active) continue;
    const BVec it = v[tl.item];
    const double beta = sc[tl.item].beta;
    const int q = tl.start + threadIdx.x;
    if (q < it.n) {
      const double z = it.z[q];
      it.p[q] = first ? z : z + beta * it.p[q];
      it.zprev[q] = z;
    }
  }
}
__global__ void __launch_bounds__(kThreads) k_b_update_p(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                         int ntiles, const BScal* __restrict__ sc,
                                                         const BCtl* __restrict__ ctl) { b_update_p(v, tiles, ntiles, sc, ctl); }

// x += alpha p, r += (-alpha) Ap (CG.cpp:121-122); partial of r'r
__device__ __forceinline__ void b_update_xr(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                          int ntiles, const BScal* __restrict__ sc,
                                                          double* __restrict__ partials) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BTile tl = tiles[t];
    const BVec it = v[tl.item];
    const int q = tl.start + threadIdx.x;
    double acc = 0.0;
    if (q < it.n) {
      double r = it.r[q];
      if (sc[tl.item].active) {
        const double alpha = sc[tl.item].alpha;
        it.x[q] = it.x[q] + alpha * it.p[q];
        r = r + -alpha * it.Ap[q];
        it.r[q] = r;
      }
      acc = r * r;
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) partials[t] = s;
  }
}
__global__ void __launch_bounds__(kThreads) k_b_update_xr(const BVec* __restrict__ v, const BTile* __restrict__ tiles,
                                                          int ntiles, const BScal* __restrict__ sc,
                                                          double* __restrict__ partials) { b_update_xr(v, tiles, ntiles, sc, partials); }

enum BFin : int { kBNorm0 = 0, kBRtz = 1, kBPap = 2, kBNormr = 3 };

// Problem p's fixed-order sum over its tiles, then its scalar step; block b
// takes problems b, b + gridDim.x, ...
__device__ __forceinline__ void b_finalize(BScal* sc, const double* __restrict__ partials, int ntiles,
                                           const int* __restrict__ range, int op, const BCtl* __restrict__ ctl,
                                           int m) {
  for (int p = blockIdx.x; p < m; p += gridDim.x) {
    const int t0 = range[p], t1 = range[p + 1];
    double a1 = 0.0, a2 = 0.0;
    for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
      a1 += partials[t];
      if (op == kBRtz) a2 += partials[ntiles + t];
    }
    const double s1 = block_sum(a1);
    const double s2 = op == kBRtz ? block_sum(a2) : 0.0;
    if (threadIdx.x != 0) continue;
    BScal& s = sc[p];
    switch (op) {
      case kBNorm0:
        s.normr2 = s1;
        s.normr0 = sqrt(s1);
        s.active = s.normr0 / s.normr0 > ctl->tol ? 1 : 0;
        s.niters = 0;
        break;
      case kBRtz:
        if (!s.active) break;
        if (ctl->iter == 0) {
          s.rtz = s1;
        } else {
          s.oldrtz = s.rtz;
          s.rtz = s1;
          s.rzprev = s2;
          s.beta = (s1 - s2) / s.oldrtz;  // Polak-Ribiere
        }
        break;
      case kBPap:
        if (!s.active) break;
        s.pAp = s1;
        s.alpha = s.rtz / s1;
        break;
      case kBNormr:
        s.normr2 = s1;
        if (s.active) {
          s.niters = ctl->iter + 1;
          s.active = sqrt(s1) / s.normr0 > ctl->tol ? 1 : 0;
        }
        break;
      default: break;
    }
  }
}

// One block per problem.
__global__ void __launch_bounds__(kThreads) k_b_finalize(BScal* sc, const double* __restrict__ partials,
                                                         int ntiles, const int* __restrict__ range, int op,
                                                         const BCtl* __restrict__ ctl, int m) {
  b_finalize(sc, partials, ntiles, range, op, ctl, m);
}

// ---- the whole iteration in one launch ------------------------------------------
// A cooperative launch (every block resident at once) walks the iteration's
// steps, the same work lists as the launches above, in the same order, with a
// grid barrier wherever a step reads what the step before wrote. So each
// problem computes the same bits as with one launch per step on the register
// kernels.
//
// The barrier: every block's thread 0 reads the generation word, arrives on
// the counter, and the last to arrive zeroes the counter and advances the
// generation; the others wait for the generation to move. The two words sit on
// separate 128-byte lines, so the waiting blocks' polls do not queue behind the
// arrivals. Each wait gives up after kBatchWaitNs of global time: it records
// fault code 5 in the context's fault word and the block leaves the kernel. A block that left stops arriving,
// so every other block's next wait runs out too and the launch ends; the
// loop's condition kernel reads the fault word and ends the loop, and the
// host's stream synchronisation returns HPCG_B200_ERR_TIMEOUT.
constexpr unsigned long long kBatchWaitNs = 1000000000ull;  // 1 s per wait

// The barrier's state (device memory): arrivals, and the generation on a line
// of its own.
struct BBar {
  unsigned count;
  unsigned pad0[31];
  unsigned gen;
  unsigned pad1[31];
};

// A load of the generation word from L2 without acquire semantics: an acquire
// at GPU scope also discards the SM's L1 contents, and a block polling on an
// SM where other blocks still work would take their cached lines away with
// every poll. The waiter orders itself once, with the fence after the loop.
__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// true once every one of the `expected` blocks has arrived; false if the wait
// gave up (the caller leaves the kernel)
__device__ __forceinline__ bool grid_barrier(BBar* bar, unsigned expected, unsigned* fault,
                                             unsigned long long limit_ns = kBatchWaitNs) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    const unsigned g = ld_relaxed_u32(&bar->gen);  // cannot move before this block arrives
    __threadfence();  // this block's writes are visible before its arrival
    if (atomicAdd(&bar->count, 1u) + 1u == expected) {
      bar->count = 0;  // nobody touches the counter until the generation moves
      __threadfence();
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&bar->gen), "r"(g + 1u) : "memory");
    } else {
      const unsigned long long t0 = global_ns();
      unsigned pause = 32;  // polls back off to one per ~0.5 us: fewer loads on the line while steps run
      while (ld_relaxed_u32(&bar->gen) == g) {
        if (global_ns() - t0 > limit_ns) {
          record_fault(fault, 5);
          ok = 0;
          break;
        }
        __nanosleep(pause);
        pause = pause < 512 ? pause * 2 : 512;
      }
    }
    __threadfence();  // with the load that saw the new generation: the other blocks' writes are visible
  }
  __syncthreads();
  return ok != 0;
}

// A step of the V-cycle on the device: 0 colour phase, 1 restriction, 2 prolongation.
struct DStep {
  int kind, tile_off, ntiles;
};

struct BIter {
  const DStep* steps;
  int nsteps;
  const BGs* gs_items;
  const BRes* res_items;
  const BTile* tiles;
  const BVec* vec;
  const BTile* vtiles;
  int nvt;
  const int* vrange;
  double* partials;
  BScal* sc;
  const BCtl* ctl;
  int m;
  BBar* bar;
  unsigned* fault;
  int vcycle_only;  // 1: the V-cycle's steps alone (timing at creation)
};

// One flexible-CG iteration of every active problem (the launches of
// iteration() below, in one launch).
__global__ void __launch_bounds__(kThreads) k_b_iteration(BIter a) {
  const unsigned nb = gridDim.x;
  if (*(volatile unsigned*)a.fault) return;  // an earlier launch gave up: do nothing
  if (!a.vcycle_only) {
    b_to32(a.vec, a.vtiles, a.nvt, a.sc);
    if (!grid_barrier(a.bar, nb, a.fault)) return;
  }
  for (int i = 0; i < a.nsteps; ++i) {
    const DStep st = a.steps[i];
    if (st.kind == 0)
      b_gs(a.gs_items, a.tiles + st.tile_off, st.ntiles, a.sc);
    else if (st.kind == 1)
      b_restrict(a.res_items, a.tiles + st.tile_off, st.ntiles, a.sc);
    else
      b_prolong(a.res_items, a.tiles + st.tile_off, st.ntiles, a.sc);
    if (!grid_barrier(a.bar, nb, a.fault)) return;
  }
  if (a.vcycle_only) return;
  b_to64_dots(a.vec, a.vtiles, a.nvt, a.sc, a.partials);
  if (!grid_barrier(a.bar, nb, a.fault)) return;
  b_finalize(a.sc, a.partials, a.nvt, a.vrange, kBRtz, a.ctl, a.m);
  if (!grid_barrier(a.bar, nb, a.fault)) return;
  b_update_p(a.vec, a.vtiles, a.nvt, a.sc, a.ctl);
  if (!grid_barrier(a.bar, nb, a.fault)) return;
  b_spmv<true>(a.vec, a.vtiles, a.nvt, 1, a.sc, a.partials);
  if (!grid_barrier(a.bar, nb, a.fault)) return;
  b_finalize(a.sc, a.partials, a.nvt, a.vrange, kBPap, a.ctl, a.m);
  if (!grid_barrier(a.bar, nb, a.fault)) return;
  b_update_xr(a.vec, a.vtiles, a.nvt, a.sc, a.partials);
  if (!grid_barrier(a.bar, nb, a.fault)) return;
  b_finalize(a.sc, a.partials, a.nvt, a.vrange, kBNormr, a.ctl, a.m);
}

// Check of the barrier's bounded wait: every block waits for one more arrival
// than the grid holds, so every wait runs out; records fault code 5 and returns.
__global__ void __launch_bounds__(kThreads) k_b_barrier_selftest(BBar* bar, unsigned long long limit_ns,
                                                                 unsigned* fault) {
  grid_barrier(bar, gridDim.x + 1, fault, limit_ns);
}

__global__ void k_b_setup(BCtl* ctl, int max_iter, double tol) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->iter = 0;
    ctl->max_iter = max_iter;
    ctl->tol = tol;
  }
}

// while (iter < max_iter && any problem active), and no bounded wait gave up;
// also zeroes the one-launch iteration's barrier counter
__global__ void k_b_condition(BCtl* ctl, const BScal* __restrict__ sc, int m, cudaGraphConditionalHandle h,
                              int advance, BBar* bar, const unsigned* fault) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (advance) ctl->iter += 1;
  bool any = false;
  for (int p = 0; p < m; ++p) any = any || sc[p].active;
  bar->count = 0;
  const bool gave_up = *(volatile const unsigned*)fault != 0;
  cudaGraphSetConditional(h, any && !gave_up && ctl->iter < ctl->max_iter ? 1u : 0u);
}

// ---- host ---------------------------------------------------------------------

struct Step {
  int kind;      // 0 = GS phase, 1 = restriction, 2 = prolongation
  int item_off;  // first item of the step (tiles index the whole item array)
  int tile_off;  // first tile of the step
  int ntiles;
  int btile_off = 0;  // GS phases: the step's 128-row tiles for k_b_gs_bulk
  int bntiles = 0;
};

}  // namespace
}  // namespace hb

struct hpcg_b200_batch {
  uint64_t magic;
  int device;
  hb::Context* ctx;
  int m;
  std::vector<hpcg_b200_problem*> probs;
  // work lists (device) and the V-cycle's step sequence
  hb::BGs* gs_items;
  hb::BRes* res_items;
  hb::BTile* tiles;
  hb::BGs* gs_bitems;  // the GS items on the blocked FP32 copies (bulk-copy phases)
  hb::BTile* btiles;   // their 128-row tiles
  bool bulk;           // GS phases on k_b_gs_bulk (chosen by timing at creation)
  bool persist;        // the whole iteration as one cooperative launch (k_b_iteration), chosen likewise
  int persist_grid;    // its blocks: as many as the SMs hold at once
  hb::DStep* dsteps;   // the V-cycle's steps for k_b_iteration
  hb::BBar* bar;       // its grid barrier
  bool packed;         // every level of every problem has packed columns (k_b_gs_bulk reads them)
  std::vector<hb::Step> steps;
  hb::BVec* vec;
  hb::BTile* vtiles;  // row tiles of every problem's level 0
  int nvt;
  int* vrange;        // [m+1] tile range of each problem
  double* partials;   // [2 * nvt]
  hb::BScal* sc;
  hb::BScal* sc_host;
  hb::BCtl* ctl;
  // slot-major FP32 values of every problem's levels, [problem * kMaxLevels + level]:
  // the batched kernels walk tiles of 256 rows, for which the single-problem
  // path's blocked FP32 layout was measured slower
  std::vector<float*> val32;
  size_t bytes;
  cudaGraphExec_t graph;
};

namespace hb {
namespace {

bool valid_batch(const hpcg_b200_batch* b) { return b && b->magic == kBatchMagic; }

int alloc_copy(hpcg_b200_batch* B, void** dst, const void* src, size_t bytes) {
  HB_TRY(dev_alloc(dst, bytes, &B->bytes));
  HB_CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  return HPCG_B200_OK;
}

// FP32 copy of FP64 values, element for element (round to nearest).
__global__ void k_narrow(float* __restrict__ dst, const double* __restrict__ src, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = (float)src[i];
}

void tiles_of(std::vector<BTile>& tiles, int item, int r0, int r1) {
  for (int s = r0; s < r1; s += kTile) tiles.push_back({item, s});
}

// 128-row tiles of the bulk-copy phase: blocks of the blocked FP32 copy that
// hold rows of [r0, r1)
void bulk_tiles_of(std::vector<BTile>& tiles, int item, int r0, int r1) {
  for (int s = r0 & ~(kBulkRows - 1); s < r1; s += kBulkRows) tiles.push_back({item, s});
}

// The V-cycle of every problem as one step sequence (ComputeMG_ref.cpp:39-63
// with the colour sweeps of the single-problem path): level l pre-smooth
// (forward from x = 0, backward without the last colour), restriction,
// recursion, prolongation, post-smooth; the coarsest level one symmetric sweep.
void build_vcycle(hpcg_b200_batch* B, int l, std::vector<BGs>& gs, std::vector<BRes>& res,
                  std::vector<BTile>& tiles, std::vector<BGs>& gsb, std::vector<BTile>& btiles) {
  auto phase = [&](int s, bool first) {
    Step st{0, (int)gs.size(), (int)tiles.size(), 0};
    st.btile_off = (int)btiles.size();
    for (int p = 0; p < B->m; ++p) {
      const Level& L = B->probs[p]->lev[l];
      const int item = (int)gs.size();
      BGs it;
      it.val = B->val32[p * kMaxLevels + l];
      it.col = L.col;
      it.pitch = L.pitch;
      it.rhs = L.r32;
      it.x = L.x32;
      it.r0 = L.g.start[s];
      it.r1 = L.g.start[s + 1];
      it.mask = first ? first_mask(L.g, s) : kAllSlots;
      it.first = first ? 1 : 0;
      it.prob = p;
      it.colp = nullptr;
      it.pack = 0;
      it.sink = 0;
      gs.push_back(it);
      tiles_of(tiles, item, it.r0, it.r1);
      BGs bit = it;  // the same phase on the blocked copies (item index = gs index)
      bit.val = L.val32;
      bit.col = L.col32;
      bit.colp = L.colp;
      bit.pack = L.pack;
      bit.sink = sink_of(L);
      if (!L.colp) B->packed = false;  // the bulk-copy phases need packed columns
      gsb.push_back(bit);
      bulk_tiles_of(btiles, item, it.r0, it.r1);
    }
    st.ntiles = (int)tiles.size() - st.tile_off;
    st.bntiles = (int)btiles.size() - st.btile_off;
    B->steps.push_back(st);
  };
  auto sweep = [&](bool first) {
    for (int s = 0; s < kColours; ++s) phase(s, first);
    for (int s = kColours - 2; s >= 0; --s) phase(s, false);
  };
  auto transfer = [&](int kind) {
    Step st{kind, (int)res.size(), (int)tiles.size(), 0};
    for (int p = 0; p < B->m; ++p) {
      const Level& L = B->probs[p]->lev[l];
      const Level& C = B->probs[p]->lev[l + 1];
      const int item = (int)res.size();
      BRes it;
      it.val = B->val32[p * kMaxLevels + l];
      it.col = L.col;
      it.pitch = L.pitch;
      it.tf = L.tf;
      it.tq = L.tq;
      it.nc = C.n;
      it.prob = p;
      if (kind == 1) {  // rc = rf - A xf
        it.rf = L.r32;
        it.xf = L.x32;
        it.rc = C.r32;
      } else {  // xf += xc: xc travels in rf, the fine solution in rc
        it.rf = C.x32;
        it.xf = nullptr;
        it.rc = L.x32;
      }
      res.push_back(it);
      tiles_of(tiles, item, 0, it.nc);
    }
    st.ntiles = (int)tiles.size() - st.tile_off;
    B->steps.push_back(st);
  };
  sweep(true);
  if (l + 1 < 4) {
    transfer(1);
    build_vcycle(B, l + 1, gs, res, tiles, gsb, btiles);
    transfer(2);
    sweep(false);
  }
}

int grid_tiles(Context* c, int ntiles) {
  int g = c->sms * kBlocksPerSm;
  return ntiles < g ? (ntiles < 1 ? 1 : ntiles) : g;
}

int launch_step(hpcg_b200_batch* B, const Step& s) {
  Context* c = B->ctx;
  const int g = grid_tiles(c, s.ntiles);
  // tiles hold indices into the whole item array, so the items go in unshifted
  if (s.kind == 0 && B->bulk) {
    using Sh = BatchShape;
    static std::atomic<uint64_t> attr_set{0};  // devices on which the shared-memory size is enabled
    bulk_attr(k_b_gs_bulk, Sh::smem, c->device, &attr_set);
    const int gb = s.bntiles < c->sms ? (s.bntiles < 1 ? 1 : s.bntiles) : c->sms;
    k_b_gs_bulk<<<gb, Sh::threads, Sh::smem, c->stream>>>(B->gs_bitems, B->btiles + s.btile_off, s.bntiles, B->sc,
                                                          c->fault);
  } else if (s.kind == 0)
    k_b_gs<<<g, kThreads, 0, c->stream>>>(B->gs_items, B->tiles + s.tile_off, s.ntiles, B->sc);
  else if (s.kind == 1)
    k_b_restrict<<<g, kThreads, 0, c->stream>>>(B->res_items, B->tiles + s.tile_off, s.ntiles, B->sc);
  else
    k_b_prolong<<<g, kThreads, 0, c->stream>>>(B->res_items, B->tiles + s.tile_off, s.ntiles, B->sc);
  HB_CK(cudaGetLastError());
  return HPCG_B200_OK;
}

int finalize_b(hpcg_b200_batch* B, int op) {
  k_b_finalize<<<B->m, kThreads, 0, B->ctx->stream>>>(B->sc, B->partials, B->nvt, B->vrange, op, B->ctl, B->m);
  HB_CK(cudaGetLastError());
  return HPCG_B200_OK;
}

// one flexible-CG iteration of every active problem
int iteration(hpcg_b200_batch* B) {
  Context* c = B->ctx;
  const int gv = grid_tiles(c, B->nvt);
  k_b_to32<<<gv, kThreads, 0, c->stream>>>(B->vec, B->vtiles, B->nvt, B->sc);
  HB_CK(cudaGetLastError());
  for (const Step& s : B->steps) HB_TRY(launch_step(B, s));
  k_b_to64_dots<<<gv, kThreads, 0, c->stream>>>(B->vec, B->vtiles, B->nvt, B->sc, B->partials);
  HB_CK(cudaGetLastError());
  HB_TRY(finalize_b(B, kBRtz));
  k_b_update_p<<<gv, kThreads, 0, c->stream>>>(B->vec, B->vtiles, B->nvt, B->sc, B->ctl);
  k_b_spmv<true><<<gv, kThreads, 0, c->stream>>>(B->vec, B->vtiles, B->nvt, 1, B->sc, B->partials);
  HB_CK(cudaGetLastError());
  HB_TRY(finalize_b(B, kBPap));
  k_b_update_xr<<<gv, kThreads, 0, c->stream>>>(B->vec, B->vtiles, B->nvt, B->sc, B->partials);
  HB_CK(cudaGetLastError());
  return finalize_b(B, kBNormr);
}

// k_b_iteration as a cooperative launch (vcycle_only: the V-cycle's steps alone)
int launch_iteration(hpcg_b200_batch* B, bool vcycle_only) {
  Context* c = B->ctx;
  if (B->persist_grid < 1) return HPCG_B200_ERR_UNSUPPORTED;
  BIter a;
  a.steps = B->dsteps;
  a.nsteps = (int)B->steps.size();
  a.gs_items = B->gs_items;
  a.res_items = B->res_items;
  a.tiles = B->tiles;
  a.vec = B->vec;
  a.vtiles = B->vtiles;
  a.nvt = B->nvt;
  a.vrange = B->vrange;
  a.partials = B->partials;
  a.sc = B->sc;
  a.ctl = B->ctl;
  a.m = B->m;
  a.bar = B->bar;
  a.fault = c->fault;
  a.vcycle_only = vcycle_only ? 1 : 0;
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(B->persist_grid);
  cfg.blockDim = dim3(kThreads);
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  HB_CK(cudaMemsetAsync(B->bar, 0, sizeof(BBar), c->stream));  // the barrier counts from zero each launch
  HB_CK(cudaLaunchKernelEx(&cfg, k_b_iteration, a));
  return HPCG_B200_OK;
}

int end_capture_b(cudaStream_t st, int status) {
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  if (status == HPCG_B200_OK && e != cudaSuccess) {
    set_error("cudaStreamEndCapture", e);
    return status_of(e);
  }
  return status;
}

int build_graph(hpcg_b200_batch* B) {
  Context* c = B->ctx;
  cudaGraph_t g = nullptr;
  HB_CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault);
  int st = HPCG_B200_OK;
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(c->stream, g, nullptr, nullptr, 0,
                                                            cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    k_b_condition<<<1, 32, 0, c->stream>>>(B->ctl, B->sc, B->m, h, 0, B->bar, c->fault);
    e = cudaGetLastError();
    st = end_capture_b(c->stream, e == cudaSuccess ? HPCG_B200_OK : status_of(e));
  }
  size_t num = 0;
  cudaGraphNode_t init = nullptr;
  if (e == cudaSuccess && st == HPCG_B200_OK) e = cudaGraphGetNodes(g, nullptr, &num);
  if (e == cudaSuccess && st == HPCG_B200_OK && num == 1) e = cudaGraphGetNodes(g, &init, &num);
  alignas(cudaGraphNodeParams) unsigned char buf[sizeof(cudaGraphNodeParams)];
  std::memset(buf, 0, sizeof(buf));
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(buf);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t loop = nullptr;
  if (e == cudaSuccess && st == HPCG_B200_OK) e = cudaGraphAddNode(&loop, g, &init, 1, &cp);
  if (e == cudaSuccess && st == HPCG_B200_OK)
    e = cudaStreamBeginCaptureToGraph(c->stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess || st != HPCG_B200_OK) {
    cudaGraphDestroy(g);
    if (e != cudaSuccess) set_error("batch graph", e);
    return st != HPCG_B200_OK ? st : status_of(e);
  }
  st = B->persist ? launch_iteration(B, false) : iteration(B);
  if (st == HPCG_B200_OK) {
    k_b_condition<<<1, 32, 0, c->stream>>>(B->ctl, B->sc, B->m, h, 1, B->bar, c->fault);
    if (cudaGetLastError() != cudaSuccess) st = HPCG_B200_ERR_CUDA;
  }
  st = end_capture_b(c->stream, st);
  if (st == HPCG_B200_OK) {
    e = cudaGraphInstantiate(&B->graph, g, 0);
    if (e != cudaSuccess) {
      set_error("cudaGraphInstantiate (batch)", e);
      st = status_of(e);
    }
  }
  cudaGraphDestroy(g);
  return st;
}

// The form of an iteration: one launch per step with the colour phases on the
// register kernel (k_b_gs) or on the bulk-copy kernel (k_b_gs_bulk, every
// level packed), or the whole iteration as one cooperative launch
// (k_b_iteration, register phases). The fastest V-cycle (all problems active,
// three rounds each way, round-robin), or HPCG_B200_BATCH_PERSIST (1: one
// launch) / HPCG_B200_BATCH_BULK (one launch per step; 1: bulk-copy phases).
// Every V-cycle starts its sweeps from the right-hand side alone, so the work
// vectors it leaves behind are rewritten by the next solve.
int choose_form(hpcg_b200_batch* B) {
  const char* fp = std::getenv("HPCG_B200_BATCH_PERSIST");
  const char* fb = std::getenv("HPCG_B200_BATCH_BULK");
  if (fp && *fp) {
    B->persist = std::atoi(fp) != 0 && B->persist_grid > 0;
    B->bulk = !B->persist && B->packed && fb && *fb && std::atoi(fb) != 0;
    return HPCG_B200_OK;
  }
  if (fb && *fb) {
    B->persist = false;
    B->bulk = B->packed && std::atoi(fb) != 0;
    return HPCG_B200_OK;
  }
  Context* c = B->ctx;
  std::vector<BScal> on(B->m);
  for (BScal& x : on) {
    std::memset(&x, 0, sizeof(x));
    x.active = 1;
  }
  HB_CK(cudaMemcpy(B->sc, on.data(), sizeof(BScal) * B->m, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  HB_CK(cudaEventCreate(&e0));
  HB_CK(cudaEventCreate(&e1));
  float best[3] = {1e30f, 1e30f, 1e30f};
  const bool can[3] = {true, B->packed, B->persist_grid > 0};
  int st = HPCG_B200_OK;
  for (int rep = 0; rep < 3 && st == HPCG_B200_OK; ++rep) {
    for (int f = 0; f < 3 && st == HPCG_B200_OK; ++f) {
      if (!can[f]) continue;
      B->bulk = f == 1;
      if (cudaEventRecord(e0, c->stream) != cudaSuccess) st = HPCG_B200_ERR_CUDA;
      if (f == 2) {
        if (st == HPCG_B200_OK) st = launch_iteration(B, true);
      } else {
        for (const Step& s : B->steps)
          if (st == HPCG_B200_OK) st = launch_step(B, s);
      }
      if (st == HPCG_B200_OK && cudaEventRecord(e1, c->stream) != cudaSuccess) st = HPCG_B200_ERR_CUDA;
      if (st == HPCG_B200_OK) st = stream_sync(c);
      float ms = 0.f;
      if (st == HPCG_B200_OK && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) st = HPCG_B200_ERR_CUDA;
      if (st == HPCG_B200_OK && ms < best[f]) best[f] = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HB_TRY(st);
  int f = 0;
  for (int i = 1; i < 3; ++i)
    if (best[i] < best[f]) f = i;
  B->bulk = f == 1;
  B->persist = f == 2;
  HB_CK(cudaMemset(B->sc, 0, sizeof(BScal) * B->m));
  return HPCG_B200_OK;
}

void destroy(hpcg_b200_batch* B) {
  if (!B) return;
  cudaSetDevice(B->device);
  if (B->ctx) cudaStreamSynchronize(B->ctx->stream);
  if (B->graph) cudaGraphExecDestroy(B->graph);
  void* v[] = {B->gs_items, B->res_items, B->tiles, B->gs_bitems, B->btiles, B->vec, B->vtiles, B->vrange,
               B->partials, B->sc, B->ctl, B->dsteps, B->bar};
  for (void* q : v) cudaFree(q);
  for (float* q : B->val32) cudaFree(q);
  if (B->sc_host) cudaFreeHost(B->sc_host);
  release_accounted(B->bytes);
  for (hpcg_b200_problem* p : B->probs) free_problem(p);
  B->magic = 0;
  delete B;
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

int hpcg_b200_batch_create(int count, const int* nx, const int* ny, const int* nz, int device,
                           hpcg_b200_batch** out) {
  if (!out || count < 1 || !nx || !ny || !nz) return HPCG_B200_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < count; ++i)  // every level even: all 8 colours present on every level
    if (nx[i] % 16 || ny[i] % 16 || nz[i] % 16 || nx[i] < 16 || ny[i] < 16 || nz[i] < 16)
      return HPCG_B200_ERR_UNSUPPORTED;
  Context* c = context_for(device);
  if (!c) return HPCG_B200_ERR_CUDA;
  HB_CK(cudaSetDevice(device));
  hpcg_b200_batch* B = new hpcg_b200_batch;
  B->magic = kBatchMagic;
  B->device = device;
  B->ctx = c;
  B->m = count;
  B->gs_items = nullptr; B->res_items = nullptr; B->tiles = nullptr; B->vec = nullptr; B->vtiles = nullptr;
  B->gs_bitems = nullptr; B->btiles = nullptr; B->bulk = false; B->packed = true;
  B->persist = false; B->persist_grid = 0; B->dsteps = nullptr; B->bar = nullptr;
  B->vrange = nullptr; B->partials = nullptr; B->sc = nullptr; B->sc_host = nullptr; B->ctl = nullptr;
  B->bytes = 0;
  B->graph = nullptr;
  B->nvt = 0;
  int st = HPCG_B200_OK;
  for (int i = 0; i < count && st == HPCG_B200_OK; ++i) {
    hpcg_b200_problem* p = nullptr;
    st = hpcg_b200_generate(nx[i], ny[i], nz[i], 4, device, &p);
    if (st == HPCG_B200_OK) {
      B->probs.push_back(p);
      st = prepare_f32(p);
    }
    for (int l = 0; l < kMaxLevels && st == HPCG_B200_OK; ++l) {
      float* v = nullptr;
      if (l < p->nlev) {
        const Level& L = p->lev[l];
        const int64_t cnt = (int64_t)kSlots * L.pitch;
        st = dev_alloc((void**)&v, sizeof(float) * cnt, &B->bytes);
        if (st == HPCG_B200_OK) {
          k_narrow<<<grid_for(c, cnt, kThreads, 8), kThreads, 0, c->stream>>>(v, L.val, cnt);
          if (cudaGetLastError() != cudaSuccess) st = HPCG_B200_ERR_CUDA;
        }
      }
      B->val32.push_back(v);
    }
  }
  if (st == HPCG_B200_OK) {
    std::vector<BGs> gs, gsb;
    std::vector<BRes> res;
    std::vector<BTile> tiles, btiles;
    build_vcycle(B, 0, gs, res, tiles, gsb, btiles);
    std::vector<BVec> vec(count);
    std::vector<BTile> vt;
    std::vector<int> range(count + 1, 0);
    for (int p = 0; p < count; ++p) {
      hpcg_b200_problem* P = B->probs[p];
      const Level& L = P->lev[0];
      vec[p] = BVec{L.val, L.col, L.pitch, L.n, P->b, P->x, P->r, P->z, P->zprev, P->p, P->Ap, L.r32, L.x32};
      range[p] = (int)vt.size();
      tiles_of(vt, p, 0, L.n);
    }
    range[count] = (int)vt.size();
    B->nvt = (int)vt.size();
    st = alloc_copy(B, (void**)&B->gs_items, gs.data(), sizeof(BGs) * gs.size());
    if (!st && !res.empty()) st = alloc_copy(B, (void**)&B->res_items, res.data(), sizeof(BRes) * res.size());
    if (!st) st = alloc_copy(B, (void**)&B->tiles, tiles.data(), sizeof(BTile) * tiles.size());
    if (!st) st = alloc_copy(B, (void**)&B->gs_bitems, gsb.data(), sizeof(BGs) * gsb.size());
    if (!st) st = alloc_copy(B, (void**)&B->btiles, btiles.data(), sizeof(BTile) * btiles.size());
    if (!st) st = alloc_copy(B, (void**)&B->vec, vec.data(), sizeof(BVec) * vec.size());
    if (!st) st = alloc_copy(B, (void**)&B->vtiles, vt.data(), sizeof(BTile) * vt.size());
    if (!st) st = alloc_copy(B, (void**)&B->vrange, range.data(), sizeof(int) * range.size());
    if (!st) st = dev_alloc((void**)&B->partials, sizeof(double) * 2 * B->nvt, &B->bytes);
    if (!st) st = dev_alloc((void**)&B->sc, sizeof(BScal) * count, &B->bytes);
    if (!st) st = dev_alloc((void**)&B->ctl, sizeof(BCtl), &B->bytes);
    if (!st) {
      std::vector<DStep> ds;
      for (const Step& x : B->steps) ds.push_back(DStep{x.kind, x.tile_off, x.ntiles});
      st = alloc_copy(B, (void**)&B->dsteps, ds.data(), sizeof(DStep) * ds.size());
    }
    if (!st) st = dev_alloc((void**)&B->bar, sizeof(BBar), &B->bytes);
    if (!st && cudaMemset(B->bar, 0, sizeof(BBar)) != cudaSuccess) st = HPCG_B200_ERR_CUDA;
    if (!st) {
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_b_iteration, kThreads, 0) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 0;
      }
      // measurement knob HPCG_B200_BATCH_PERSIST_BLOCKS: resident blocks per SM
      const char* pb = std::getenv("HPCG_B200_BATCH_PERSIST_BLOCKS");
      const int want = pb && *pb ? std::atoi(pb) : kBlocksPerSm;
      B->persist_grid = c->sms * std::max(0, std::min({per_sm, kBlocksPerSm, want}));
    }
    if (!st && cudaMallocHost(&B->sc_host, sizeof(BScal) * count) != cudaSuccess) st = HPCG_B200_ERR_NOMEM;
    if (!st && cudaMemset(B->sc, 0, sizeof(BScal) * count) != cudaSuccess) st = HPCG_B200_ERR_CUDA;
    if (!st) st = choose_form(B);
  }
  if (st != HPCG_B200_OK) {
    destroy(B);
    return st;
  }
  *out = B;
  return HPCG_B200_OK;
}

int hpcg_b200_batch_problem(hpcg_b200_batch* B, int i, hpcg_b200_problem** out) {
  if (!valid_batch(B)) return HPCG_B200_ERR_HANDLE;
  if (!out || i < 0 || i >= B->m) return HPCG_B200_ERR_ARG;
  *out = B->probs[i];
  return HPCG_B200_OK;
}

int hpcg_b200_batch_cg_mixed(hpcg_b200_batch* B, const double* const* b, double* const* x, int max_iter,
                             double tolerance, int* niters, double* normr, double* normr0) {
  if (!valid_batch(B)) return HPCG_B200_ERR_HANDLE;
  if (!b || !x || !niters || !normr || !normr0 || max_iter < 0) return HPCG_B200_ERR_ARG;
  for (int p = 0; p < B->m; ++p)
    if (!b[p] || !x[p]) return HPCG_B200_ERR_ARG;
  HB_CK(cudaSetDevice(B->device));
  Context* c = B->ctx;
  for (int p = 0; p < B->m; ++p) {
    HB_TRY(load_vector(B->probs[p], 0, b[p], B->probs[p]->b));
    HB_TRY(load_vector(B->probs[p], 0, x[p], B->probs[p]->x));
  }
  // preamble: Ap = A x; r = b - Ap; normr0 (CG.cpp:86-96), every problem
  const int gv = grid_tiles(c, B->nvt);
  k_b_setup<<<1, 32, 0, c->stream>>>(B->ctl, max_iter, tolerance);
  k_b_spmv<false><<<gv, kThreads, 0, c->stream>>>(B->vec, B->vtiles, B->nvt, 0, nullptr, nullptr);
  k_b_resid<<<gv, kThreads, 0, c->stream>>>(B->vec, B->vtiles, B->nvt, B->partials);
  HB_CK(cudaGetLastError());
  HB_TRY(finalize_b(B, kBNorm0));
  if (!B->graph) {
    int gs = build_graph(B);
    if (gs != HPCG_B200_OK && B->persist) {  // a cooperative launch refused inside a capture
      cudaGetLastError();
      B->persist = false;
      gs = build_graph(B);
    }
    HB_TRY(gs);
  }
  HB_CK(cudaGraphLaunch(B->graph, c->stream));
  HB_CK(cudaMemcpyAsync(B->sc_host, B->sc, sizeof(BScal) * B->m, cudaMemcpyDeviceToHost, c->stream));
  HB_TRY(stream_sync(c));
  for (int p = 0; p < B->m; ++p) {
    niters[p] = B->sc_host[p].niters;
    normr[p] = std::sqrt(B->sc_host[p].normr2);
    normr0[p] = B->sc_host[p].normr0;
    HB_TRY(store_vector(B->probs[p], 0, B->probs[p]->x, x[p]));
  }
  return HPCG_B200_OK;
}

int hpcg_b200_batch_form(const hpcg_b200_batch* B, int* form) {
  if (!valid_batch(B)) return HPCG_B200_ERR_HANDLE;
  if (!form) return HPCG_B200_ERR_ARG;
  *form = B->persist ? 2 : B->bulk ? 1 : 0;
  return HPCG_B200_OK;
}

int hpcg_b200_grid_wait_selftest(int device, double seconds) {
  if (!(seconds > 0.0 && seconds <= 2.0)) return HPCG_B200_ERR_ARG;
  Context* c = context_for(device);
  if (!c) return HPCG_B200_ERR_CUDA;
  HB_CK(cudaSetDevice(device));
  BBar* bar = nullptr;
  HB_CK(cudaMalloc(&bar, sizeof(BBar)));
  cudaError_t e = cudaMemsetAsync(bar, 0, sizeof(BBar), c->stream);
  if (e == cudaSuccess) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(c->sms);
    cfg.blockDim = dim3(kThreads);
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_b_barrier_selftest, bar, (unsigned long long)(seconds * 1e9), c->fault);
  }
  if (e != cudaSuccess) {
    set_error("grid wait self-test", e);
    cudaStreamSynchronize(c->stream);
    cudaFree(bar);
    return status_of(e);
  }
  const int st = stream_sync(c);
  cudaFree(bar);
  return st;
}

int hpcg_b200_batch_free(hpcg_b200_batch* B) {
  if (!valid_batch(B)) return HPCG_B200_ERR_HANDLE;
  destroy(B);
  return HPCG_B200_OK;
}

}  // extern "C"
