// Multi-right-hand-side solves: hpcg_b200_cg_multi and hpcg_b200_mg_multi.
// K systems with the same matrix advance in lockstep through the kernels of
// kernels_multi.cuh; each matrix row is read once per sweep for all K.
#include <cmath>
#include <cstdlib>
#include <vector>

#include "kernels_multi.cuh"

namespace hb {

void release_accounted(size_t bytes);

// Work vectors of the multi-system path, interleaved [row][K], per level.
struct MultiState {
  int K = 0;
  int lanes = 1;  // threads per row of the matrix kernels (K/lanes systems each), tuned on creation
  double *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr;
  double* lr[kMaxLevels] = {nullptr};  // coarse right-hand sides (levels > 0)
  double* lx[kMaxLevels] = {nullptr};  // coarse solutions (levels > 0)
  double* stage = nullptr;             // natural, system-major staging (nrhs * n)
  size_t stage_cap = 0;
  double* partials = nullptr;          // [K][kParts]
  MScalars* s = nullptr;
  MScalars* s_host = nullptr;
  size_t bytes = 0;
};

namespace {

constexpr int kParts = 1024;  // reduction blocks of the vector kernels (fixed: deterministic)

void free_state(MultiState* m) {
  if (!m) return;
  void* v[] = {m->b, m->x, m->r, m->z, m->p, m->Ap, m->stage, m->partials, m->s};
  for (void* q : v) cudaFree(q);
  for (int l = 0; l < kMaxLevels; ++l) {
    cudaFree(m->lr[l]);
    cudaFree(m->lx[l]);
  }
  if (m->s_host) cudaFreeHost(m->s_host);
  release_accounted(m->bytes);
  delete m;
}

int alloc_z(MultiState* m, double** p, size_t count, cudaStream_t st) {
  HB_TRY(dev_alloc((void**)p, sizeof(double) * count, &m->bytes));
  HB_CK(cudaMemsetAsync(*p, 0, sizeof(double) * count, st));
  return HPCG_B200_OK;
}

template <int K, int LANES>
int mg_m(hpcg_b200_problem* P, MultiState* m, int l, const double* r, double* x);

// The matrix work of one CG iteration with LANES threads per row: a V-cycle and
// the SpMV with its p'Ap partials.
template <int K, int LANES>
int time_iteration(hpcg_b200_problem* P, MultiState* m, cudaEvent_t e0, cudaEvent_t e1, float* best) {
  Context* c = P->ctx;
  const Level& L = P->lev[0];
  HB_CK(cudaEventRecord(e0, c->stream));
  HB_TRY((mg_m<K, LANES>(P, m, 0, m->r, m->z)));
  k_spmv_m<K, LANES, true><<<kParts, kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, m->p, m->Ap, L.n, m->partials);
  HB_CK(cudaGetLastError());
  HB_CK(cudaEventRecord(e1, c->stream));
  HB_CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  HB_CK(cudaEventElapsedTime(&ms, e0, e1));
  if (ms < *best) *best = ms;
  return HPCG_B200_OK;
}

// Threads per row of the matrix kernels: the fastest V-cycle + SpMV (round-robin
// repetitions), or HPCG_B200_MULTI_LANES. Same V-cycle bits either way.
int tune_lanes(hpcg_b200_problem* P, MultiState* m) {
  const int K = m->K;
  const char* force = std::getenv("HPCG_B200_MULTI_LANES");
  if (force && *force) {
    const int f = std::atoi(force);
    m->lanes = f >= 4 && K >= 8 ? 4 : f >= 2 && K >= 4 ? 2 : 1;
    return HPCG_B200_OK;
  }
  Context* c = P->ctx;
  cudaEvent_t e0, e1;
  HB_CK(cudaEventCreate(&e0));
  HB_CK(cudaEventCreate(&e1));
  float t_[3] = {1e30f, 1e30f, 1e30f};  // lanes 1, 2, 4
  int st = HPCG_B200_OK;
  for (int rep = 0; rep < 3 && st == HPCG_B200_OK; ++rep) {
    if (K == 2) st = time_iteration<2, 1>(P, m, e0, e1, &t_[0]);
    if (K == 4) {
      st = time_iteration<4, 1>(P, m, e0, e1, &t_[0]);
      if (!st) st = time_iteration<4, 2>(P, m, e0, e1, &t_[1]);
    }
    if (K == 8) {
      st = time_iteration<8, 1>(P, m, e0, e1, &t_[0]);
      if (!st) st = time_iteration<8, 2>(P, m, e0, e1, &t_[1]);
      if (!st) st = time_iteration<8, 4>(P, m, e0, e1, &t_[2]);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HB_TRY(st);
  int best = 0;
  for (int i = 1; i < 3; ++i)
    if (t_[i] < t_[best]) best = i;
  m->lanes = 1 << best;
  // the timed work wrote z, Ap and the coarse vectors: every solve loads its own
  // b and x and every V-cycle starts from zero, but leave the state as created
  HB_CK(cudaMemsetAsync(m->z, 0, sizeof(double) * (size_t)P->lev[0].pitch * K, c->stream));
  HB_CK(cudaMemsetAsync(m->Ap, 0, sizeof(double) * (size_t)P->lev[0].pitch * K, c->stream));
  for (int l = 1; l < P->nlev; ++l) {
    HB_CK(cudaMemsetAsync(m->lr[l], 0, sizeof(double) * (size_t)P->lev[l].pitch * K, c->stream));
    HB_CK(cudaMemsetAsync(m->lx[l], 0, sizeof(double) * (size_t)P->lev[l].pitch * K, c->stream));
  }
  return HPCG_B200_OK;
}

// The state for K systems (re-created when K changes). Vectors are zeroed, so
// the zero row n of every level (padded stencil slots) reads 0 for all K.
int ensure_state(hpcg_b200_problem* P, int K, MultiState** out) {
  MultiState*& m = P->multi;
  if (m && m->K == K) {
    *out = m;
    return HPCG_B200_OK;
  }
  free_state(m);
  m = new MultiState;
  m->K = K;
  cudaStream_t st = P->ctx->stream;
  const Level& L0 = P->lev[0];
  double** v0[] = {&m->b, &m->x, &m->r, &m->z, &m->p, &m->Ap};
  for (double** v : v0) HB_TRY(alloc_z(m, v, (size_t)L0.pitch * K, st));
  for (int l = 1; l < P->nlev; ++l) {
    HB_TRY(alloc_z(m, &m->lr[l], (size_t)P->lev[l].pitch * K, st));
    HB_TRY(alloc_z(m, &m->lx[l], (size_t)P->lev[l].pitch * K, st));
  }
  HB_TRY(alloc_z(m, &m->partials, (size_t)kMaxRhs * kParts, st));
  HB_TRY(dev_alloc((void**)&m->s, sizeof(MScalars), &m->bytes));
  HB_CK(cudaMemsetAsync(m->s, 0, sizeof(MScalars), st));
  HB_CK(cudaMallocHost(&m->s_host, sizeof(MScalars)));
  HB_TRY(tune_lanes(P, m));
  *out = m;
  return HPCG_B200_OK;
}

template <int K, int LANES>
void launch_phase_m(Context* c, const Level& L, const double* rhs, double* x, int r0, int r1, bool first,
                    uint32_t mask) {
  const int64_t work = (int64_t)(r1 - r0) * LANES;
  if (first) {
    auto k = k_gs_phase_m<K, LANES, true>;
    k<<<grid_of(c, k, work), kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, rhs, x, r0, r1, mask);
  } else {
    auto k = k_gs_phase_m<K, LANES, false>;
    k<<<grid_of(c, k, work), kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, rhs, x, r0, r1, mask);
  }
}

template <int K, int LANES>
int gs_colour_m(Context* c, const Level& L, const double* rhs, double* x, bool first) {
  int last = -1;
  for (int s = 0; s < kColours; ++s) {
    const int r0 = L.g.start[s], r1 = L.g.start[s + 1];
    if (r1 <= r0) continue;
    last = s;
    launch_phase_m<K, LANES>(c, L, rhs, x, r0, r1, first, first ? first_mask(L.g, s) : kAllSlots);
  }
  // backward sweep, without repeating the last colour (as the single-system path)
  for (int s = last - 1; s >= 0; --s) {
    const int r0 = L.g.start[s], r1 = L.g.start[s + 1];
    if (r1 <= r0) continue;
    launch_phase_m<K, LANES>(c, L, rhs, x, r0, r1, false, kAllSlots);
  }
  HB_CK(cudaGetLastError());
  return HPCG_B200_OK;
}

// ComputeMG_ref.cpp:39-63 for K systems on level l (colour order, interleaved).
template <int K, int LANES>
int mg_m(hpcg_b200_problem* P, MultiState* m, int l, const double* r, double* x) {
  const Level& L = P->lev[l];
  Context* c = P->ctx;
  HB_TRY((gs_colour_m<K, LANES>(c, L, r, x, true)));
  if (l + 1 < P->nlev) {
    const Level& C = P->lev[l + 1];
    auto kr = k_restrict_m<K, LANES>;
    kr<<<grid_of(c, kr, (int64_t)C.n * LANES), kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, r, x, L.tf, L.tq,
                                                                          m->lr[l + 1], C.n);
    HB_CK(cudaGetLastError());
    HB_TRY((mg_m<K, LANES>(P, m, l + 1, m->lr[l + 1], m->lx[l + 1])));
    auto kp = k_prolong_m<K>;
    kp<<<grid_of(c, kp, C.n), kThreads, 0, c->stream>>>(L.tf, L.tq, m->lx[l + 1], x, C.n);
    HB_CK(cudaGetLastError());
    HB_TRY((gs_colour_m<K, LANES>(c, L, r, x, false)));
  }
  return HPCG_B200_OK;
}

// system-major natural src (host or device) -> interleaved colour-order dst
template <int K>
int load_m(hpcg_b200_problem* P, MultiState* m, int nrhs, const double* src, double* dst) {
  const Level& L = P->lev[0];
  Context* c = P->ctx;
  const double* s = src;
  if (!is_device_ptr(src)) {
    const size_t need = (size_t)nrhs * L.n;
    if (m->stage_cap < need) {
      cudaFree(m->stage);
      m->stage = nullptr;
      m->stage_cap = 0;
      HB_CK(cudaMalloc(&m->stage, sizeof(double) * need));
      m->stage_cap = need;
    }
    HB_CK(cudaMemcpyAsync(m->stage, src, sizeof(double) * need, cudaMemcpyHostToDevice, c->stream));
    s = m->stage;
  }
  auto k = k_gather_in_m<K>;
  k<<<grid_of(c, k, L.n), kThreads, 0, c->stream>>>(dst, s, L.new2old, L.n, nrhs);
  HB_CK(cudaGetLastError());
  return HPCG_B200_OK;
}

template <int K>
int store_m(hpcg_b200_problem* P, MultiState* m, int nrhs, const double* src, double* dst) {
  const Level& L = P->lev[0];
  Context* c = P->ctx;
  const bool dev = is_device_ptr(dst);
  double* d = dst;
  const size_t need = (size_t)nrhs * L.n;
  if (!dev) {
    if (m->stage_cap < need) {
      cudaFree(m->stage);
      m->stage = nullptr;
      m->stage_cap = 0;
      HB_CK(cudaMalloc(&m->stage, sizeof(double) * need));
      m->stage_cap = need;
    }
    d = m->stage;
  }
  auto k = k_scatter_out_m<K>;
  k<<<grid_of(c, k, L.n), kThreads, 0, c->stream>>>(d, src, L.old2new, L.n, nrhs);
  HB_CK(cudaGetLastError());
  if (!dev) HB_CK(cudaMemcpyAsync(dst, d, sizeof(double) * need, cudaMemcpyDeviceToHost, c->stream));
  HB_CK(cudaStreamSynchronize(c->stream));
  return HPCG_B200_OK;
}

template <int K>
int finalize_m(Context* c, MultiState* m, int op, int iter, double tol) {
  k_finalize_m<K><<<1, kThreads, 0, c->stream>>>(m->partials, kParts, op, m->s, iter, tol);
  HB_CK(cudaGetLastError());
  return HPCG_B200_OK;
}

// CG.cpp:59-143 for K systems in lockstep; a system stops updating once its
// scaled residual is at or below the tolerance; the loop ends when none is left
// or after max_iter iterations.
template <int K, int LANES>
int cg_m(hpcg_b200_problem* P, MultiState* m, int max_iter, double tol, int* any_iters) {
  const Level& L = P->lev[0];
  Context* c = P->ctx;
  const int n = L.n;
  auto ks = k_spmv_m<K, LANES, false>;
  ks<<<grid_of(c, ks, (int64_t)n * LANES), kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, m->x, m->Ap, n, nullptr);
  k_resid_m<K><<<kParts, kThreads, 0, c->stream>>>(m->b, m->Ap, m->r, n, m->partials);
  HB_CK(cudaGetLastError());
  HB_TRY(finalize_m<K>(c, m, kMNorm0, 0, tol));
  HB_CK(cudaMemcpyAsync(m->s_host, m->s, sizeof(MScalars), cudaMemcpyDeviceToHost, c->stream));
  HB_CK(cudaStreamSynchronize(c->stream));
  int k = 1;
  for (; k <= max_iter; ++k) {
    bool any = false;
    for (int j = 0; j < K; ++j) any = any || m->s_host->active[j];
    if (!any) break;
    HB_TRY((mg_m<K, LANES>(P, m, 0, m->r, m->z)));
    k_dot_m<K><<<kParts, kThreads, 0, c->stream>>>(m->r, m->z, n, m->partials);
    HB_CK(cudaGetLastError());
    if (k == 1) {
      HB_TRY(finalize_m<K>(c, m, kMRtzFirst, k, tol));
      HB_CK(cudaMemcpyAsync(m->p, m->z, sizeof(double) * (size_t)n * K, cudaMemcpyDeviceToDevice, c->stream));
    } else {
      HB_TRY(finalize_m<K>(c, m, kMRtz, k, tol));
      k_update_p_m<K><<<kParts, kThreads, 0, c->stream>>>(m->z, m->p, n, m->s);
      HB_CK(cudaGetLastError());
    }
    k_spmv_m<K, LANES, true><<<kParts, kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, m->p, m->Ap, n, m->partials);
    HB_CK(cudaGetLastError());
    HB_TRY(finalize_m<K>(c, m, kMPap, k, tol));
    k_update_xr_m<K><<<kParts, kThreads, 0, c->stream>>>(m->x, m->p, m->r, m->Ap, n, m->s, m->partials);
    HB_CK(cudaGetLastError());
    HB_TRY(finalize_m<K>(c, m, kMNormr, k, tol));
    HB_CK(cudaMemcpyAsync(m->s_host, m->s, sizeof(MScalars), cudaMemcpyDeviceToHost, c->stream));
    HB_CK(cudaStreamSynchronize(c->stream));
  }
  *any_iters = k - 1;
  return HPCG_B200_OK;
}

template <int K>
int run_cg_multi(hpcg_b200_problem* P, int nrhs, const double* b, double* x, int max_iter, double tol, int* niters,
                 double* normr, double* normr0) {
  MultiState* m = nullptr;
  HB_TRY(ensure_state(P, K, &m));
  HB_TRY(load_m<K>(P, m, nrhs, b, m->b));
  HB_TRY(load_m<K>(P, m, nrhs, x, m->x));
  int done = 0;
  if (m->lanes == 4) {
    if constexpr (K >= 8) HB_TRY((cg_m<K, 4>(P, m, max_iter, tol, &done)));
  } else if (m->lanes == 2) {
    if constexpr (K >= 4) HB_TRY((cg_m<K, 2>(P, m, max_iter, tol, &done)));
  } else {
    HB_TRY((cg_m<K, 1>(P, m, max_iter, tol, &done)));
  }
  HB_TRY(store_m<K>(P, m, nrhs, m->x, x));
  for (int j = 0; j < nrhs; ++j) {
    niters[j] = m->s_host->niters[j];
    normr[j] = std::sqrt(m->s_host->normr2[j]);
    normr0[j] = m->s_host->normr0[j];
  }
  return HPCG_B200_OK;
}

template <int K>
int run_mg_multi(hpcg_b200_problem* P, int nrhs, const double* r, double* x) {
  MultiState* m = nullptr;
  HB_TRY(ensure_state(P, K, &m));
  HB_TRY(load_m<K>(P, m, nrhs, r, m->r));
  if (m->lanes == 4) {
    if constexpr (K >= 8) HB_TRY((mg_m<K, 4>(P, m, 0, m->r, m->z)));
  } else if (m->lanes == 2) {
    if constexpr (K >= 4) HB_TRY((mg_m<K, 2>(P, m, 0, m->r, m->z)));
  } else {
    HB_TRY((mg_m<K, 1>(P, m, 0, m->r, m->z)));
  }
  return store_m<K>(P, m, nrhs, m->z, x);
}

struct Setter {
  int prev = -1;
  explicit Setter(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~Setter() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

void free_multi(hpcg_b200_problem* p) {
  free_state(p->multi);
  p->multi = nullptr;
}

}  // namespace hb

using namespace hb;

extern "C" {

int hpcg_b200_cg_multi(hpcg_b200_problem* p, int nrhs, const double* b, double* x, int max_iter, double tolerance,
                       int* niters, double* normr, double* normr0) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (is_rank(p)) return HPCG_B200_ERR_UNSUPPORTED;  // a rank: use the hpcg_b200_shard_* routines
  if (nrhs < 1 || nrhs > kMaxRhs || !b || !x || !niters || !normr || !normr0 || max_iter < 0)
    return HPCG_B200_ERR_ARG;
  Setter dev(p->device);
  if (nrhs <= 2) return run_cg_multi<2>(p, nrhs, b, x, max_iter, tolerance, niters, normr, normr0);
  if (nrhs <= 4) return run_cg_multi<4>(p, nrhs, b, x, max_iter, tolerance, niters, normr, normr0);
  return run_cg_multi<8>(p, nrhs, b, x, max_iter, tolerance, niters, normr, normr0);
}

int hpcg_b200_mg_multi(hpcg_b200_problem* p, int nrhs, const double* r, double* x) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (is_rank(p)) return HPCG_B200_ERR_UNSUPPORTED;  // a rank: use the hpcg_b200_shard_* routines
  if (nrhs < 1 || nrhs > kMaxRhs || !r || !x) return HPCG_B200_ERR_ARG;
  Setter dev(p->device);
  if (nrhs <= 2) return run_mg_multi<2>(p, nrhs, r, x);
  if (nrhs <= 4) return run_mg_multi<4>(p, nrhs, r, x);
  return run_mg_multi<8>(p, nrhs, r, x);
}

}  // extern "C"
