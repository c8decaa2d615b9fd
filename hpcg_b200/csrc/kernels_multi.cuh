// Kernels of the multi-right-hand-side path: K independent systems with the
// same matrix, solved in lockstep so that each matrix row is read once for all
// K. Vectors interleave the K right-hand sides: entry (row q, system j) lives
// at q*K + j, so the K values a slot gathers are one contiguous, 16-byte
// aligned run (K = 2, 4 or 8 doubles). For every system the arithmetic is the
// single-system sequence of kernels.cuh, in the same order, so each system's
// V-cycle is bitwise the one hpcg_b200_mg computes.
#pragma once

#include "bulk.cuh"
#include "reduce.cuh"

namespace hb {

constexpr int kMaxRhs = 8;

// Per-system CG scalars on the device.
struct MScalars {
  double rtz[kMaxRhs], oldrtz[kMaxRhs], alpha[kMaxRhs], beta[kMaxRhs], pAp[kMaxRhs], normr2[kMaxRhs],
      normr0[kMaxRhs];
  int active[kMaxRhs];  // still iterating (normr/normr0 > tolerance)
  int niters[kMaxRhs];  // iterations done while active
};

template <int K>
__device__ __forceinline__ void load_k(const double* __restrict__ p, double (&v)[K]) {
  static_assert(K % 2 == 0, "K doubles must fill whole 16-byte loads");
#pragma unroll
  for (int c = 0; c < K / 2; ++c) {
    const uint4 u = __ldg(reinterpret_cast<const uint4*>(p) + c);
    memcpy(&v[2 * c], &u, 16);
  }
}

template <int K>
__device__ __forceinline__ void store_k(double* __restrict__ p, const double (&v)[K]) {
#pragma unroll
  for (int c = 0; c < K / 2; ++c) {
    uint4 u;
    memcpy(&u, &v[2 * c], 16);
    reinterpret_cast<uint4*>(p)[c] = u;
  }
}

// Gauss-Seidel colour phase for K systems (ComputeSYMGS_ref.cpp:72-80 per system).
// LANES threads share a row, each with S = K/LANES of its systems: every lane
// re-reads the row's values and columns (one transaction for the lanes of a
// row) and gathers S-entry runs of x. More lanes, fewer registers per thread
// and more rows' loads in flight per SM.
template <int K, int LANES, bool FIRST>
__global__ void __launch_bounds__(kThreads) k_gs_phase_m(const double* __restrict__ val, const int* __restrict__ col,
                                                         int64_t pitch, const double* __restrict__ rhs, double* x,
                                                         int r0, int r1, uint32_t mask) {
  constexpr int S = K / LANES;
  const int64_t work = (int64_t)(r1 - r0) * LANES;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < work; t += stride) {
    const int q = r0 + (int)(t / LANES);
    const int off = (int)(t % LANES) * S;
    double sum[S], xd[S];
    load_k<S>(rhs + (int64_t)q * K + off, sum);
#pragma unroll
    for (int j = 0; j < S; ++j) xd[j] = 0.0;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      if (mask & (1u << k)) {
        const double a = val[k * pitch + q];
        double xv[S];
        load_k<S>(x + (int64_t)col[k * pitch + q] * K + off, xv);
#pragma unroll
        for (int j = 0; j < S; ++j) {
          sum[j] -= a * xv[j];
          if (k == kDiagSlot) xd[j] = xv[j];
        }
      }
    }
    const double d = val[kDiagSlot * pitch + q];
    double out[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
      if (!FIRST) sum[j] += xd[j] * d;
      out[j] = sum[j] / d;
    }
    store_k<S>(x + (int64_t)q * K + off, out);
  }
}

// y = A x for K systems; DOT: partials of x_j'y_j at partials[j*gridDim.x + block].
// LANES as in k_gs_phase_m.
template <int K, int LANES, bool DOT>
__global__ void __launch_bounds__(kThreads) k_spmv_m(const double* __restrict__ val, const int* __restrict__ col,
                                                     int64_t pitch, const double* __restrict__ x,
                                                     double* __restrict__ y, int n, double* __restrict__ partials) {
  constexpr int S = K / LANES;
  const int64_t work = (int64_t)n * LANES;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int off = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) % LANES) * S;  // stride % LANES == 0
  double acc[S];
#pragma unroll
  for (int j = 0; j < S; ++j) acc[j] = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < work; t += stride) {
    const int q = (int)(t / LANES);
    double sum[S], xq[S];
#pragma unroll
    for (int j = 0; j < S; ++j) sum[j] = xq[j] = 0.0;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const double a = val[k * pitch + q];
      double xv[S];
      load_k<S>(x + (int64_t)col[k * pitch + q] * K + off, xv);
#pragma unroll
      for (int j = 0; j < S; ++j) {
        sum[j] += a * xv[j];
        if (k == kDiagSlot) xq[j] = xv[j];
      }
    }
    store_k<S>(y + (int64_t)q * K + off, sum);
    if (DOT) {
#pragma unroll
      for (int j = 0; j < S; ++j) acc[j] += xq[j] * sum[j];
    }
  }
  if (DOT) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const double s = block_sum(off == (j / S) * S ? acc[j % S] : 0.0);
      if (threadIdx.x == 0) partials[j * gridDim.x + blockIdx.x] = s;
    }
  }
}

// Pipeline shapes of the multi-system kernels: LANES threads per row, at most
// 1024 threads a block (four lanes: one group with a ring of four stages). The
// columns arrive packed (the level's packed record per tile, offsets of PW bytes).
template <int LANES, int PW>
using MultiShape = BulkShape<double, LANES == 4 ? 1 : 2, LANES == 4 ? 4 : 2, LANES, PW>;

// k_gs_phase_m through the bulk-copy pipeline (bulk.cuh): the tile's values
// arrive on chip by a tensor copy and its packed columns (colp, sink) by a bulk
// copy; the lanes of a row gather their S-entry runs of x as in k_gs_phase_m,
// in the same order: the same bits. The full-slot phases (FIRST false) take all
// 27 slots.
template <int K, int LANES, bool FIRST, int PW>
__global__ void __launch_bounds__(MultiShape<LANES, PW>::threads, 1)
    k_gs_phase_m_bulk(const double* __restrict__ val, const int* __restrict__ col, int64_t pitch,
                      const double* __restrict__ rhs, double* x, int r0, int r1, uint32_t mask_arg, unsigned* fault,
                      const __grid_constant__ CUtensorMap tm_val, const __grid_constant__ CUtensorMap tm_col,
                      const unsigned char* __restrict__ colp, int sink) {
  constexpr int S = K / LANES;
  const uint32_t mask = FIRST ? mask_arg : kAllSlots;
  const int a0 = r0 & ~(kBulkRows - 1);
  const int ntiles = (r1 - a0 + kBulkRows - 1) / kBulkRows;
  bulk_tiles<double, MultiShape<LANES, PW>>(
      val, col, pitch, ntiles, [&](int tile) { return a0 + (int64_t)tile * kBulkRows; },
      [&](int64_t q0, const double* sv, const int* sc, int t) {
        const int row = t / LANES;
        const int off = (t % LANES) * S;
        const int64_t q = q0 + row;
        if (q < r0 || q >= r1) return;
        double sum[S], xd[S];
        load_k<S>(rhs + q * K + off, sum);
#pragma unroll
        for (int j = 0; j < S; ++j) xd[j] = 0.0;
#pragma unroll
        for (int k = 0; k < kSlots; ++k) {
          if (mask & (1u << k)) {
            const double a = sv[k * kBulkRows + row];
            double xv[S];
            load_k<S>(x + (int64_t)stage_col<PW>(sc, k, row, sink) * K + off, xv);
#pragma unroll
            for (int j = 0; j < S; ++j) {
              sum[j] -= a * xv[j];
              if (k == kDiagSlot) xd[j] = xv[j];
            }
          }
        }
        const double d = sv[kDiagSlot * kBulkRows + row];
        double out[S];
#pragma unroll
        for (int j = 0; j < S; ++j) {
          if (!FIRST) sum[j] += xd[j] * d;
          out[j] = sum[j] / d;
        }
        store_k<S>(x + q * K + off, out);
      },
      fault, tm_val, tm_col, colp);
}

// k_spmv_m through the bulk-copy pipeline (packed columns), rows in storage
// order; DOT: partials of x_j'y_j at partials[j*gridDim.x + block].
template <int K, int LANES, bool DOT, int PW>
__global__ void __launch_bounds__(MultiShape<LANES, PW>::threads, 1)
    k_spmv_m_bulk(const double* __restrict__ val, const int* __restrict__ col, int64_t pitch,
                  const double* __restrict__ x, double* __restrict__ y, int n, double* __restrict__ partials,
                  unsigned* fault, const __grid_constant__ CUtensorMap tm_val,
                  const __grid_constant__ CUtensorMap tm_col, const unsigned char* __restrict__ colp, int sink) {
  constexpr int S = K / LANES;
  const int off = (int)(threadIdx.x % LANES) * S;  // the producer warp (32 threads) keeps the lanes aligned
  double acc[S];
#pragma unroll
  for (int j = 0; j < S; ++j) acc[j] = 0.0;
  const int ntiles = (n + kBulkRows - 1) / kBulkRows;
  bulk_tiles<double, MultiShape<LANES, PW>>(
      val, col, pitch, ntiles, [&](int tile) { return (int64_t)tile * kBulkRows; },
      [&](int64_t q0, const double* sv, const int* sc, int t) {
        const int row = t / LANES;
        const int64_t q = q0 + row;
        if (q >= n) return;
        double sum[S], xq[S];
#pragma unroll
        for (int j = 0; j < S; ++j) sum[j] = xq[j] = 0.0;
#pragma unroll
        for (int k = 0; k < kSlots; ++k) {
          const double a = sv[k * kBulkRows + row];
          double xv[S];
          load_k<S>(x + (int64_t)stage_col<PW>(sc, k, row, sink) * K + off, xv);
#pragma unroll
          for (int j = 0; j < S; ++j) {
            sum[j] += a * xv[j];
            if (k == kDiagSlot) xq[j] = xv[j];
          }
        }
        store_k<S>(y + q * K + off, sum);
        if (DOT) {
#pragma unroll
          for (int j = 0; j < S; ++j) acc[j] += xq[j] * sum[j];
        }
      },
      fault, tm_val, tm_col, colp);
  if (DOT) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const double s = block_sum(off == (j / S) * S ? acc[j % S] : 0.0);
      if (threadIdx.x == 0) partials[j * gridDim.x + blockIdx.x] = s;
    }
  }
}

// rc = (rf - A xf) at the injected rows (sorted transfer pairs), K systems; LANES as in k_gs_phase_m.
template <int K, int LANES>
__global__ void __launch_bounds__(kThreads) k_restrict_m(const double* __restrict__ val, const int* __restrict__ col,
                                                         int64_t pitch, const double* __restrict__ rf,
                                                         const double* __restrict__ xf, const int* __restrict__ tf,
                                                         const int* __restrict__ tq, double* __restrict__ rc, int nc) {
  constexpr int S = K / LANES;
  const int64_t work = (int64_t)nc * LANES;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += stride) {
    const int t = (int)(w / LANES);
    const int off = (int)(w % LANES) * S;
    const int f = tf[t];
    double sum[S];
#pragma unroll
    for (int j = 0; j < S; ++j) sum[j] = 0.0;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const double a = val[k * pitch + f];
      double xv[S];
      load_k<S>(xf + (int64_t)col[k * pitch + f] * K + off, xv);
#pragma unroll
      for (int j = 0; j < S; ++j) sum[j] += a * xv[j];
    }
    double r[S], out[S];
    load_k<S>(rf + (int64_t)f * K + off, r);
#pragma unroll
    for (int j = 0; j < S; ++j) out[j] = r[j] - sum[j];
    store_k<S>(rc + (int64_t)tq[t] * K + off, out);
  }
}

template <int K>
__global__ void __launch_bounds__(kThreads) k_prolong_m(const int* __restrict__ tf, const int* __restrict__ tq,
                                                        const double* __restrict__ xc, double* __restrict__ xf,
                                                        int nc) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nc; t += stride) {
    double a[K], c[K];
    load_k<K>(xf + (int64_t)tf[t] * K, a);
    load_k<K>(xc + (int64_t)tq[t] * K, c);
#pragma unroll
    for (int j = 0; j < K; ++j) a[j] += c[j];
    store_k<K>(xf + (int64_t)tf[t] * K, a);
  }
}

// natural, system-major src[j*n + i] (j < nrhs) -> interleaved colour order; systems
// j >= nrhs are zero
template <int K>
__global__ void __launch_bounds__(kThreads) k_gather_in_m(double* __restrict__ dst, const double* __restrict__ src,
                                                          const int* __restrict__ new2old, int n, int nrhs) {
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    const int64_t i = new2old[q];
    double v[K];
#pragma unroll
    for (int j = 0; j < K; ++j) v[j] = j < nrhs ? src[(int64_t)j * n + i] : 0.0;
    store_k<K>(dst + (int64_t)q * K, v);
  }
}

template <int K>
__global__ void __launch_bounds__(kThreads) k_scatter_out_m(double* __restrict__ dst, const double* __restrict__ src,
                                                            const int* __restrict__ old2new, int n, int nrhs) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double v[K];
    load_k<K>(src + (int64_t)old2new[i] * K, v);
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (j < nrhs) dst[(int64_t)j * n + i] = v[j];
  }
}

// r = 1.0 b + (-1.0) Ap (CG.cpp:88) and partials of r_j'r_j
template <int K>
__global__ void __launch_bounds__(kThreads) k_resid_m(const double* __restrict__ b, const double* __restrict__ Ap,
                                                      double* __restrict__ r, int n, double* __restrict__ partials) {
  const int stride = gridDim.x * blockDim.x;
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; ++j) acc[j] = 0.0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    double bv[K], av[K], rv[K];
    load_k<K>(b + (int64_t)q * K, bv);
    load_k<K>(Ap + (int64_t)q * K, av);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      rv[j] = 1.0 * bv[j] + -1.0 * av[j];
      acc[j] += rv[j] * rv[j];
    }
    store_k<K>(r + (int64_t)q * K, rv);
  }
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const double s = block_sum(acc[j]);
    if (threadIdx.x == 0) partials[j * gridDim.x + blockIdx.x] = s;
  }
}

// partials of x_j'y_j
template <int K>
__global__ void __launch_bounds__(kThreads) k_dot_m(const double* __restrict__ x, const double* __restrict__ y, int n,
                                                    double* __restrict__ partials) {
  const int stride = gridDim.x * blockDim.x;
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; ++j) acc[j] = 0.0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    double a[K], b[K];
    load_k<K>(x + (int64_t)q * K, a);
    load_k<K>(y + (int64_t)q * K, b);
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] += a[j] * b[j];
  }
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const double s = block_sum(acc[j]);
    if (threadIdx.x == 0) partials[j * gridDim.x + blockIdx.x] = s;
  }
}

// p = z + beta_j p (CG.cpp:115)
template <int K>
__global__ void __launch_bounds__(kThreads) k_update_p_m(const double* __restrict__ z, double* __restrict__ p, int n,
                                                         const MScalars* __restrict__ s) {
  double beta[K];
#pragma unroll
  for (int j = 0; j < K; ++j) beta[j] = s->beta[j];
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    double zv[K], pv[K];
    load_k<K>(z + (int64_t)q * K, zv);
    load_k<K>(p + (int64_t)q * K, pv);
#pragma unroll
    for (int j = 0; j < K; ++j) pv[j] = zv[j] + beta[j] * pv[j];
    store_k<K>(p + (int64_t)q * K, pv);
  }
}

// x += alpha_j p, r += (-alpha_j) Ap for the systems still iterating (CG.cpp:121-122);
// partials of r_j'r_j
template <int K>
__global__ void __launch_bounds__(kThreads) k_update_xr_m(double* __restrict__ x, const double* __restrict__ p,
                                                          double* __restrict__ r, const double* __restrict__ Ap,
                                                          int n, const MScalars* __restrict__ s,
                                                          double* __restrict__ partials) {
  double alpha[K], malpha[K];
  bool act[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    alpha[j] = s->alpha[j];
    malpha[j] = -s->alpha[j];
    act[j] = s->active[j] != 0;
  }
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; ++j) acc[j] = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    double xv[K], pv[K], rv[K], av[K];
    load_k<K>(x + (int64_t)q * K, xv);
    load_k<K>(p + (int64_t)q * K, pv);
    load_k<K>(r + (int64_t)q * K, rv);
    load_k<K>(Ap + (int64_t)q * K, av);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (act[j]) {
        xv[j] = xv[j] + alpha[j] * pv[j];
        rv[j] = rv[j] + malpha[j] * av[j];
      }
      acc[j] += rv[j] * rv[j];
    }
    store_k<K>(x + (int64_t)q * K, xv);
    store_k<K>(r + (int64_t)q * K, rv);
  }
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const double sum = block_sum(acc[j]);
    if (threadIdx.x == 0) partials[j * gridDim.x + blockIdx.x] = sum;
  }
}

enum MFinOp : int { kMNorm0 = 0, kMRtzFirst = 1, kMRtz = 2, kMPap = 3, kMNormr = 4 };

// One block: fixed-order reduction of the K partial sets, then the scalar step of
// `op` for every system (the single-system rules of CG.cpp:96-124, per system).
template <int K>
__global__ void __launch_bounds__(kThreads) k_finalize_m(const double* __restrict__ partials, int nparts, int op,
                                                         MScalars* s, int iter, double tol) {
  double sum[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += partials[j * nparts + i];
    sum[j] = block_sum(acc);
  }
  if (threadIdx.x != 0) return;
  for (int j = 0; j < K; ++j) {
    switch (op) {
      case kMNorm0: {
        s->normr2[j] = sum[j];
        const double nr = sqrt(sum[j]);
        s->normr0[j] = nr;
        s->active[j] = (nr / nr > tol) ? 1 : 0;
        s->niters[j] = 0;
        break;
      }
      case kMRtzFirst: s->rtz[j] = sum[j]; break;
      case kMRtz:
        s->oldrtz[j] = s->rtz[j];
        s->rtz[j] = sum[j];
        s->beta[j] = sum[j] / s->oldrtz[j];
        break;
      case kMPap:
        s->pAp[j] = sum[j];
        s->alpha[j] = s->active[j] ? s->rtz[j] / sum[j] : 0.0;
        break;
      case kMNormr:
        s->normr2[j] = sum[j];
        if (s->active[j]) {
          s->niters[j] = iter;
          s->active[j] = sqrt(sum[j]) / s->normr0[j] > tol ? 1 : 0;
        }
        break;
      default: break;
    }
  }
}

}  // namespace hb
