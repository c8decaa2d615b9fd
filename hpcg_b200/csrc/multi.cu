// Multi-right-hand-side solves: hpcg_b200_cg_multi and hpcg_b200_mg_multi.
// K systems with the same matrix advance in lockstep through the kernels of
// kernels_multi.cuh; each matrix row is read once per sweep for all K.
#include <cmath>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "kernels_multi.cuh"

namespace hb {

void release_accounted(size_t bytes);

// Work vectors of the multi-system path, interleaved [row][K], per level.
struct MultiState {
  int K = 0;
  int lanes = 1;  // threads per row of the matrix kernels (K/lanes systems each), tuned on creation
  int bulk = 0;   // 0: register-pipelined kernels; 1: bulk-copy full phases and SpMV; 2: first sweep too
  double *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr;
  double* lr[kMaxLevels] = {nullptr};  // coarse right-hand sides (levels > 0)
  double* lx[kMaxLevels] = {nullptr};  // coarse solutions (levels > 0)
  double* stage = nullptr;             // natural, system-major staging (nrhs * n)
  size_t stage_cap = 0;
  double* partials = nullptr;          // [K][kParts]
  MScalars* s = nullptr;
  MScalars* s_host = nullptr;
  size_t bytes = 0;
  // the V-cycle below level 0 as one captured graph (see coarse_m)
  cudaGraphExec_t coarse = nullptr;
  int coarse_key = -1;         // lanes * 4 + bulk of the captured kernels
  bool coarse_failed = false;  // a capture was refused: stream launches from then on
  bool tuning = false;         // while the forms are being timed, no graph
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
  if (m->coarse) cudaGraphExecDestroy(m->coarse);
  release_accounted(m->bytes);
  delete m;
}

int alloc_z(MultiState* m, double** p, size_t count, cudaStream_t st) {
  HB_TRY(dev_alloc((void**)p, sizeof(double) * count, &m->bytes));
  HB_CK(cudaMemsetAsync(*p, 0, sizeof(double) * count, st));
  return HPCG_B200_OK;
}

template <int K, int LANES, int BULK>
int mg_m(hpcg_b200_problem* P, MultiState* m, int l, const double* r, double* x);
template <int K, int LANES, int BULK, bool DOT>
int spmv_m(Context* c, const Level& L, const double* x, double* y, double* partials);

template <int V>
using IC = std::integral_constant<int, V>;

// Calls f(IC<LANES>, IC<BULK>) for the state's configuration.
template <int K, typename F>
int dispatch_m(const MultiState* m, F&& f) {
  if (m->lanes == 4) {
    if constexpr (K >= 8) {
      if (m->bulk == 1) return f(IC<4>{}, IC<1>{});
      if (m->bulk == 2) return f(IC<4>{}, IC<2>{});
      return f(IC<4>{}, IC<0>{});
    }
  } else if (m->lanes == 2) {
    if constexpr (K >= 4) {
      if (m->bulk == 1) return f(IC<2>{}, IC<1>{});
      if (m->bulk == 2) return f(IC<2>{}, IC<2>{});
      return f(IC<2>{}, IC<0>{});
    }
  }
  if (m->bulk == 1) return f(IC<1>{}, IC<1>{});
  if (m->bulk == 2) return f(IC<1>{}, IC<2>{});
  return f(IC<1>{}, IC<0>{});
}

// The matrix work of one CG iteration in one configuration: a V-cycle and the
// SpMV with its p'Ap partials.
template <int K, int LANES, int BULK>
int time_iteration(hpcg_b200_problem* P, MultiState* m, cudaEvent_t e0, cudaEvent_t e1, float* best) {
  Context* c = P->ctx;
  const Level& L = P->lev[0];
  HB_CK(cudaEventRecord(e0, c->stream));
  HB_TRY((mg_m<K, LANES, BULK>(P, m, 0, m->r, m->z)));
  const int g = spmv_m<K, LANES, BULK, true>(c, L, m->p, m->Ap, m->partials);
  if (g < 0) return -g;
  HB_CK(cudaEventRecord(e1, c->stream));
  HB_CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  HB_CK(cudaEventElapsedTime(&ms, e0, e1));
  if (ms < *best) *best = ms;
  return HPCG_B200_OK;
}

// Threads per row and kernel form of the matrix kernels: the fastest V-cycle +
// SpMV (round-robin repetitions over lanes 1, 2, 4 x register-pipelined, bulk
// full phases, bulk everywhere), or HPCG_B200_MULTI_LANES / HPCG_B200_MULTI_BULK.
// Same V-cycle bits either way.
template <int K>
int tune_lanes(hpcg_b200_problem* P, MultiState* m) {
  const char* force = std::getenv("HPCG_B200_MULTI_LANES");
  const char* force_bulk = std::getenv("HPCG_B200_MULTI_BULK");
  const bool have_maps = bulk_maps(P->lev[0]) != nullptr;
  if ((force && *force) || (force_bulk && *force_bulk)) {
    const int f = force && *force ? std::atoi(force) : 1;
    m->lanes = f >= 4 && K >= 8 ? 4 : f >= 2 && K >= 4 ? 2 : 1;
    const int b = force_bulk && *force_bulk ? std::atoi(force_bulk) : 0;
    m->bulk = have_maps ? (b < 0 ? 0 : b > 2 ? 2 : b) : 0;
    return HPCG_B200_OK;
  }
  Context* c = P->ctx;
  cudaEvent_t e0, e1;
  HB_CK(cudaEventCreate(&e0));
  HB_CK(cudaEventCreate(&e1));
  m->tuning = true;
  float t_[3][3];  // [lanes 1, 2, 4][bulk 0, 1, 2]
  for (auto& row : t_)
    for (float& v : row) v = 1e30f;
  const int nbulk = have_maps ? 3 : 1;
  int st = HPCG_B200_OK;
  for (int rep = 0; rep < 3 && st == HPCG_B200_OK; ++rep) {
    for (int li = 0; li < 3 && st == HPCG_B200_OK; ++li) {
      const int lanes = 1 << li;
      if ((lanes == 2 && K < 4) || (lanes == 4 && K < 8)) continue;
      for (int b = 0; b < nbulk && st == HPCG_B200_OK; ++b) {
        MultiState probe;
        probe.lanes = lanes;
        probe.bulk = b;
        float* slot = &t_[li][b];
        st = dispatch_m<K>(&probe, [&](auto l, auto bk) {
          return time_iteration<K, decltype(l)::value, decltype(bk)::value>(P, m, e0, e1, slot);
        });
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  m->tuning = false;
  HB_TRY(st);
  int bl = 0, bb = 0;
  for (int li = 0; li < 3; ++li)
    for (int b = 0; b < 3; ++b)
      if (t_[li][b] < t_[bl][bb]) {
        bl = li;
        bb = b;
      }
  m->lanes = 1 << bl;
  m->bulk = bb;
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
template <int K>
int ensure_state(hpcg_b200_problem* P, MultiState** out) {
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
  HB_TRY(tune_lanes<K>(P, m));
  *out = m;
  return HPCG_B200_OK;
}

// The multi-system phase on the bulk-copy pipeline, packed columns of PW bytes.
template <int K, int LANES, int PW>
void launch_phase_m_bulk(Context* c, const Level& L, const BulkMaps* bm, const double* rhs, double* x, int r0,
                         int r1, bool first, uint32_t mask) {
  using Sh = MultiShape<LANES, PW>;
  const int64_t tiles = ((int64_t)r1 - (r0 & ~(kBulkRows - 1)) + kBulkRows - 1) / kBulkRows;
  const int g = (int)std::min<int64_t>(tiles, (int64_t)c->sms);
  static std::atomic<uint64_t> done[2] = {{0}, {0}};
  if (first) {
    auto k = k_gs_phase_m_bulk<K, LANES, true, PW>;
    bulk_attr(k, Sh::smem, c->device, &done[0]);
    k<<<g, Sh::threads, Sh::smem, c->stream>>>(L.val, L.col, L.pitch, rhs, x, r0, r1, mask, c->fault, bm->val,
                                                bm->col, L.colp, sink_of(L));
  } else {
    auto k = k_gs_phase_m_bulk<K, LANES, false, PW>;
    bulk_attr(k, Sh::smem, c->device, &done[1]);
    k<<<g, Sh::threads, Sh::smem, c->stream>>>(L.val, L.col, L.pitch, rhs, x, r0, r1, mask, c->fault, bm->val,
                                                bm->col, L.colp, sink_of(L));
  }
}

template <int K, int LANES, int BULK>
void launch_phase_m(Context* c, const Level& L, const double* rhs, double* x, int r0, int r1, bool first,
                    uint32_t mask) {
  // the bulk-copy kernels read the packed columns: a level without them runs
  // the register-pipelined kernels
  const BulkMaps* bm = L.colp && (BULK == 2 || (BULK == 1 && !first)) ? bulk_maps(L) : nullptr;
  if (bm) {
    if (L.pack == kPackDiag)
      launch_phase_m_bulk<K, LANES, kPackDiag>(c, L, bm, rhs, x, r0, r1, first, mask);
    else if (L.pack == 1)
      launch_phase_m_bulk<K, LANES, 1>(c, L, bm, rhs, x, r0, r1, first, mask);
    else
      launch_phase_m_bulk<K, LANES, 2>(c, L, bm, rhs, x, r0, r1, first, mask);
    return;
  }
  const int64_t work = (int64_t)(r1 - r0) * LANES;
  if (first) {
    auto k = k_gs_phase_m<K, LANES, true>;
    k<<<grid_of(c, k, work), kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, rhs, x, r0, r1, mask);
  } else {
    auto k = k_gs_phase_m<K, LANES, false>;
    k<<<grid_of(c, k, work), kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, rhs, x, r0, r1, mask);
  }
}

// The multi-system SpMV on the bulk-copy pipeline, packed columns of PW bytes;
// returns the grid.
template <int K, int LANES, bool DOT, int PW>
int spmv_m_bulk(Context* c, const Level& L, const BulkMaps* bm, const double* x, double* y, double* partials) {
  using Sh = MultiShape<LANES, PW>;
  auto k = k_spmv_m_bulk<K, LANES, DOT, PW>;
  static std::atomic<uint64_t> done{0};
  bulk_attr(k, Sh::smem, c->device, &done);
  const int64_t tiles = ((int64_t)L.n + kBulkRows - 1) / kBulkRows;
  const int g = (int)std::min<int64_t>(tiles, (int64_t)c->sms);
  k<<<g, Sh::threads, Sh::smem, c->stream>>>(L.val, L.col, L.pitch, x, y, L.n, partials, c->fault, bm->val, bm->col,
                                              L.colp, sink_of(L));
  return g;
}

// y = A x for K systems; returns the number of blocks (DOT: partial sets written)
// or a negative status.
template <int K, int LANES, int BULK, bool DOT>
int spmv_m(Context* c, const Level& L, const double* x, double* y, double* partials) {
  const BulkMaps* bm = BULK && L.colp ? bulk_maps(L) : nullptr;
  if (bm) {
    const int g = L.pack == kPackDiag ? spmv_m_bulk<K, LANES, DOT, kPackDiag>(c, L, bm, x, y, partials)
                  : L.pack == 1       ? spmv_m_bulk<K, LANES, DOT, 1>(c, L, bm, x, y, partials)
                                      : spmv_m_bulk<K, LANES, DOT, 2>(c, L, bm, x, y, partials);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error("k_spmv_m_bulk", e);
      return -status_of(e);
    }
    return g;
  }
  auto k = k_spmv_m<K, LANES, DOT>;
  const int g = DOT ? kParts : grid_of(c, k, (int64_t)L.n * LANES);
  k<<<g, kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, x, y, L.n, partials);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("k_spmv_m", e);
    return -status_of(e);
  }
  return g;
}

template <int K, int LANES, int BULK>
int gs_colour_m(Context* c, const Level& L, const double* rhs, double* x, bool first) {
  int last = -1;
  for (int s = 0; s < kColours; ++s) {
    const int r0 = L.g.start[s], r1 = L.g.start[s + 1];
    if (r1 <= r0) continue;
    last = s;
    launch_phase_m<K, LANES, BULK>(c, L, rhs, x, r0, r1, first, first ? first_mask(L.g, s) : kAllSlots);
  }
  // backward sweep, without repeating the last colour (as the single-system path)
  for (int s = last - 1; s >= 0; --s) {
    const int r0 = L.g.start[s], r1 = L.g.start[s + 1];
    if (r1 <= r0) continue;
    launch_phase_m<K, LANES, BULK>(c, L, rhs, x, r0, r1, false, kAllSlots);
  }
  HB_CK(cudaGetLastError());
  return HPCG_B200_OK;
}

template <int K, int LANES, int BULK>
int coarse_m(hpcg_b200_problem* P, MultiState* m);

// ComputeMG_ref.cpp:39-63 for K systems on level l (colour order, interleaved).
template <int K, int LANES, int BULK>
int mg_m(hpcg_b200_problem* P, MultiState* m, int l, const double* r, double* x) {
  const Level& L = P->lev[l];
  Context* c = P->ctx;
  HB_TRY((gs_colour_m<K, LANES, BULK>(c, L, r, x, true)));
  if (l + 1 < P->nlev) {
    const Level& C = P->lev[l + 1];
    auto kr = k_restrict_m<K, LANES>;
    kr<<<grid_of(c, kr, (int64_t)C.n * LANES), kThreads, 0, c->stream>>>(L.val, L.col, L.pitch, r, x, L.tf, L.tq,
                                                                          m->lr[l + 1], C.n);
    HB_CK(cudaGetLastError());
    if (l == 0) {
      HB_TRY((coarse_m<K, LANES, BULK>(P, m)));
    } else {
      HB_TRY((mg_m<K, LANES, BULK>(P, m, l + 1, m->lr[l + 1], m->lx[l + 1])));
    }
    auto kp = k_prolong_m<K>;
    kp<<<grid_of(c, kp, C.n), kThreads, 0, c->stream>>>(L.tf, L.tq, m->lx[l + 1], x, C.n);
    HB_CK(cudaGetLastError());
    HB_TRY((gs_colour_m<K, LANES, BULK>(c, L, r, x, false)));
  }
  return HPCG_B200_OK;
}

// The levels below 0 of a K-system V-cycle as one captured CUDA graph (its
// small coarse kernels cost one launch), recaptured when the lanes or the
// kernel form change; launched directly while the forms are being timed, inside
// another capture, or with HPCG_B200_GRAPH=0. The same kernels either way.
template <int K, int LANES, int BULK>
int coarse_m(hpcg_b200_problem* P, MultiState* m) {
  Context* c = P->ctx;
  auto direct = [&]() -> int { return mg_m<K, LANES, BULK>(P, m, 1, m->lr[1], m->lx[1]); };
  const char* ge = std::getenv("HPCG_B200_GRAPH");
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HB_CK(cudaStreamIsCapturing(c->stream, &cs));
  if (m->tuning || m->coarse_failed || (ge && ge[0] == '0') || cs != cudaStreamCaptureStatusNone) return direct();
  const int key = LANES * 4 + BULK;
  if (!m->coarse || m->coarse_key != key) {
    if (m->coarse) cudaGraphExecDestroy(m->coarse);
    m->coarse = nullptr;
    HB_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int st = direct();
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (st == HPCG_B200_OK && e == cudaSuccess) e = cudaGraphInstantiate(&m->coarse, g, 0);
    if (g) cudaGraphDestroy(g);
    if (st != HPCG_B200_OK || e != cudaSuccess) {
      cudaGetLastError();
      m->coarse = nullptr;
      m->coarse_failed = true;
      return direct();
    }
    m->coarse_key = key;
  }
  HB_CK(cudaGraphLaunch(m->coarse, c->stream));
  return HPCG_B200_OK;
}

// system-major natural src (host or device) -> interleaved colour-order dst
template <int K>
int load_m(hpcg_b200_problem* P, MultiState* m, int nrhs, const double* src, double* dst) {
  const Level& L = P->lev[0];
  Context* c = P->ctx;
  const double* s = src;
  bool dev = false;
  HB_TRY(locate_ptr(src, P->device, &dev, "input vectors"));
  if (!dev) {
    const size_t need = (size_t)nrhs * L.n;
    if (m->stage_cap < need) {
      cudaFree(m->stage);
      m->stage = nullptr;
      m->stage_cap = 0;
      HB_CK(cudaMalloc(&m->stage, sizeof(double) * need));
      m->stage_cap = need;
    }
    HB_TRY(host_to_device(c, m->stage, src, need));
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
  bool dev = false;
  HB_TRY(locate_ptr(dst, P->device, &dev, "output vectors"));
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
  if (!dev) HB_TRY(device_to_host(c, dst, d, need));
  return stream_sync(c);
}

template <int K>
int finalize_m(Context* c, MultiState* m, int op, int iter, double tol, int nparts = kParts) {
  k_finalize_m<K><<<1, kThreads, 0, c->stream>>>(m->partials, nparts, op, m->s, iter, tol);
  HB_CK(cudaGetLastError());
  return HPCG_B200_OK;
}

// CG.cpp:59-143 for K systems in lockstep; a system stops updating once its
// scaled residual is at or below the tolerance; the loop ends when none is left
// or after max_iter iterations.
template <int K, int LANES, int BULK>
int cg_m(hpcg_b200_problem* P, MultiState* m, int max_iter, double tol, int* any_iters) {
  const Level& L = P->lev[0];
  Context* c = P->ctx;
  const int n = L.n;
  int g = spmv_m<K, LANES, BULK, false>(c, L, m->x, m->Ap, nullptr);
  if (g < 0) return -g;
  k_resid_m<K><<<kParts, kThreads, 0, c->stream>>>(m->b, m->Ap, m->r, n, m->partials);
  HB_CK(cudaGetLastError());
  HB_TRY(finalize_m<K>(c, m, kMNorm0, 0, tol));
  HB_CK(cudaMemcpyAsync(m->s_host, m->s, sizeof(MScalars), cudaMemcpyDeviceToHost, c->stream));
  HB_TRY(stream_sync(c));
  int k = 1;
  for (; k <= max_iter; ++k) {
    bool any = false;
    for (int j = 0; j < K; ++j) any = any || m->s_host->active[j];
    if (!any) break;
    HB_TRY((mg_m<K, LANES, BULK>(P, m, 0, m->r, m->z)));
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
    g = spmv_m<K, LANES, BULK, true>(c, L, m->p, m->Ap, m->partials);
    if (g < 0) return -g;
    HB_TRY(finalize_m<K>(c, m, kMPap, k, tol, g));
    k_update_xr_m<K><<<kParts, kThreads, 0, c->stream>>>(m->x, m->p, m->r, m->Ap, n, m->s, m->partials);
    HB_CK(cudaGetLastError());
    HB_TRY(finalize_m<K>(c, m, kMNormr, k, tol));
    HB_CK(cudaMemcpyAsync(m->s_host, m->s, sizeof(MScalars), cudaMemcpyDeviceToHost, c->stream));
    HB_TRY(stream_sync(c));
  }
  *any_iters = k - 1;
  return HPCG_B200_OK;
}

template <int K>
int run_cg_multi(hpcg_b200_problem* P, int nrhs, const double* b, double* x, int max_iter, double tol, int* niters,
                 double* normr, double* normr0) {
  MultiState* m = nullptr;
  HB_TRY(ensure_state<K>(P, &m));
  HB_TRY(load_m<K>(P, m, nrhs, b, m->b));
  HB_TRY(load_m<K>(P, m, nrhs, x, m->x));
  int done = 0;
  HB_TRY(dispatch_m<K>(m, [&](auto l, auto bk) {
    return cg_m<K, decltype(l)::value, decltype(bk)::value>(P, m, max_iter, tol, &done);
  }));
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
  HB_TRY(ensure_state<K>(P, &m));
  HB_TRY(load_m<K>(P, m, nrhs, r, m->r));
  HB_TRY(dispatch_m<K>(m, [&](auto l, auto bk) {
    return mg_m<K, decltype(l)::value, decltype(bk)::value>(P, m, 0, m->r, m->z);
  }));
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
