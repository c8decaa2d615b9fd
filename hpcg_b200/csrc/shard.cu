// The run over several ranks, one per GPU: the reference's MPI decomposition
// (each rank a block of the global grid, a halo exchange before every SpMV and
// every symmetric Gauss-Seidel step, an allreduce per dot product) on B200.
//
// Communicators:
//   - NCCL: one rank per process (one process per GPU); the halo moves with
//     grouped ncclSend/ncclRecv straight into the external entries of the
//     receiving vector, the reductions with ncclAllReduce. libnccl is opened at
//     run time, so single-rank users need none.
//   - local: every rank in this process, on one GPU and one stream; the halo
//     moves with device-to-device copies and the reductions are folded in rank
//     order on the device. It runs the multi-rank algorithm where only one GPU
//     is available and is the checked twin of the NCCL path (same drivers, same
//     kernels; only the two transport calls differ).
//
// No kernel here waits on another rank: every dependency between ranks is a
// stream-ordered copy or a NCCL call.
#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <cmath>
#include <mutex>
#include <string>
#include <tuple>

#include "shard.cuh"

namespace hb {

void set_error_text(const char* text);

namespace {

constexpr uint64_t kCommMagic = 0x48504347c0330001ull;

// ---- NCCL, opened at run time --------------------------------------------------

struct NcclApi {
  bool ok = false;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    // a process that already loaded NCCL (e.g. through torch) gets that copy
    void* so = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!so) so = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!so) return;
    bool ok = true;
    auto sym = [&](const char* name) {
      void* f = dlsym(so, name);
      if (!f) ok = false;
      return f;
    };
    api.GetUniqueId = (decltype(api.GetUniqueId))sym("ncclGetUniqueId");
    api.CommInitRank = (decltype(api.CommInitRank))sym("ncclCommInitRank");
    api.CommDestroy = (decltype(api.CommDestroy))sym("ncclCommDestroy");
    api.Send = (decltype(api.Send))sym("ncclSend");
    api.Recv = (decltype(api.Recv))sym("ncclRecv");
    api.AllReduce = (decltype(api.AllReduce))sym("ncclAllReduce");
    api.GroupStart = (decltype(api.GroupStart))sym("ncclGroupStart");
    api.GroupEnd = (decltype(api.GroupEnd))sym("ncclGroupEnd");
    api.GetErrorString = (decltype(api.GetErrorString))sym("ncclGetErrorString");
    api.ok = ok;
  });
  return api;
}

int nccl_status(ncclResult_t r, const char* what) {
  if (r == ncclSuccess) return HPCG_B200_OK;
  std::string m = std::string(what) + ": " + (nccl().GetErrorString ? nccl().GetErrorString(r) : "NCCL error");
  set_error_text(m.c_str());
  return HPCG_B200_ERR_CUDA;
}

#define HB_NCCL(call, what)                      \
  do {                                           \
    int s_ = nccl_status((call), what);          \
    if (s_ != HPCG_B200_OK) return s_;           \
  } while (0)

// CUDA-event timing of the parts of a CG call into the reference's times[]
// slots (CG.cpp:132-139): 1 dot products, 2 vector updates, 3 SpMV (with its
// halo exchange, as ComputeSPMV_ref.cpp:53 does it), 4 the allreduce step of
// the dot products (inside their slot-1 time, as ComputeDotProduct_ref.cpp:69-72
// measures it), 5 the preconditioner. Pairs may nest; off when `c` is null.
struct PartTimer {
  Context* c = nullptr;
  std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> parts;
  // starts a part of `slot`; *id identifies it for stop()
  int start(int slot, int* id) {
    *id = -1;
    if (!c) return HPCG_B200_OK;
    cudaEvent_t e;
    HB_CK(cudaEventCreate(&e));
    parts.emplace_back(slot, e, nullptr);
    *id = (int)parts.size() - 1;
    HB_CK(cudaEventRecord(e, c->stream));
    return HPCG_B200_OK;
  }
  int stop(int id) {
    if (!c || id < 0) return HPCG_B200_OK;
    cudaEvent_t e;
    HB_CK(cudaEventCreate(&e));
    std::get<2>(parts[id]) = e;
    HB_CK(cudaEventRecord(e, c->stream));
    return HPCG_B200_OK;
  }
  // adds the parts' durations to times[slot] (synchronises the stream)
  int add_to(double* times) {
    if (!c) return HPCG_B200_OK;
    HB_CK(cudaStreamSynchronize(c->stream));
    for (auto& p : parts) {
      float ms = 0.f;
      if (std::get<2>(p)) HB_CK(cudaEventElapsedTime(&ms, std::get<1>(p), std::get<2>(p)));
      times[std::get<0>(p)] += ms * 1e-3;
    }
    release();
    return HPCG_B200_OK;
  }
  void release() {
    for (auto& p : parts) {
      cudaEventDestroy(std::get<1>(p));
      if (std::get<2>(p)) cudaEventDestroy(std::get<2>(p));
    }
    parts.clear();
  }
  ~PartTimer() { release(); }
};

}  // namespace

struct Comm {
  uint64_t magic = kCommMagic;
  bool use_nccl = false;
  int size = 1;                             // ranks in the run
  std::vector<hpcg_b200_problem*> ranks;    // the ranks this process drives (local: all, by rank)
  Context* ctx = nullptr;                   // their device's context
  double* red = nullptr;                    // device: per-rank values of one reduction [size] (+1 for NCCL)
  ncclComm_t nc = nullptr;
  // local: for rank i, level l, neighbour j: offset of rank i's entries in the neighbour's send buffer
  std::vector<std::vector<int> > src_off[kMaxLevels];
  PartTimer* timer = nullptr;               // set while a CG call times its parts
};

namespace {

bool valid_comm(const Comm* c) { return c != nullptr && c->magic == kCommMagic; }

// x[i] (colour order, with externals) of each driven rank at level l: refreshes
// the externals from the neighbours (ExchangeHalo.cpp:33-109).
int exchange(Comm* C, int l, double* const* x) {
  Context* c = C->ctx;
  const int nl = (int)C->ranks.size();
  for (int i = 0; i < nl; ++i) {
    const Level& L = C->ranks[i]->lev[l];
    if (L.halo) HB_TRY(pack_halo(c, *L.halo, x[i]));
  }
  if (C->use_nccl) {
    const Level& L = C->ranks[0]->lev[l];
    if (!L.halo || L.halo->nnb == 0) return HPCG_B200_OK;
    const HaloPlan& h = *L.halo;
    NcclApi& api = nccl();
    HB_NCCL(api.GroupStart(), "ncclGroupStart");
    for (int j = 0; j < h.nnb; ++j) {
      const size_t cnt = (size_t)(h.off[j + 1] - h.off[j]);
      HB_NCCL(api.Send(h.send_buf + h.off[j], cnt, ncclFloat64, h.nbr[j], C->nc, c->stream), "ncclSend");
      HB_NCCL(api.Recv(x[0] + L.n + h.off[j], cnt, ncclFloat64, h.nbr[j], C->nc, c->stream), "ncclRecv");
    }
    HB_NCCL(api.GroupEnd(), "ncclGroupEnd");
    return HPCG_B200_OK;
  }
  for (int i = 0; i < nl; ++i) {
    const Level& L = C->ranks[i]->lev[l];
    if (!L.halo) continue;
    const HaloPlan& h = *L.halo;
    for (int j = 0; j < h.nnb; ++j) {
      const HaloPlan& hn = *C->ranks[h.nbr[j]]->lev[l].halo;
      const size_t bytes = sizeof(double) * (size_t)(h.off[j + 1] - h.off[j]);
      HB_CK(cudaMemcpyAsync(x[i] + L.n + h.off[j], hn.send_buf + C->src_off[l][i][j], bytes,
                            cudaMemcpyDeviceToDevice, c->stream));
    }
  }
  return HPCG_B200_OK;
}

// The per-rank values red[i] of the driven ranks (already written) combined
// over the whole run, then the scalar update `op` (ComputeDotProduct_ref.cpp:70).
int reduce(Comm* C, int op, double* out = nullptr) {
  Context* c = C->ctx;
  int id = -1;
  if (C->timer) HB_TRY(C->timer->start(4, &id));  // the allreduce step (times[4])
  if (C->use_nccl) {
    HB_NCCL(nccl().AllReduce(C->red, C->red + 1, 1, ncclFloat64, op == kFinMax ? ncclMax : ncclSum, C->nc, c->stream),
            "ncclAllReduce");
    HB_TRY(launch_finalize_ranks(c, C->red + 1, 1, op, out));
  } else {
    HB_TRY(launch_finalize_ranks(c, C->red, C->size, op, out));
  }
  if (C->timer) HB_TRY(C->timer->stop(id));
  return HPCG_B200_OK;
}

// Block partials of one rank's reduction (in c->partials) -> red[i].
int store_partial(Comm* C, int i, int nparts, bool max = false) {
  if (nparts < 0) return -nparts;
  return launch_finalize(C->ctx, nparts, max ? kFinMax : kFinStore, C->red + i);
}

int read_scal(Context* c) {
  HB_CK(cudaMemcpyAsync(c->scal_host, c->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, c->stream));
  HB_TRY(stream_sync(c));
  return HPCG_B200_OK;
}

// ComputeMG_ref.cpp:39-63 on every driven rank, colour-order vectors of level l.
// rtz (level 0): each rank's post-smoother also leaves its r'z in red[i], as the
// single-rank CG takes it from the smoother.
int mg_ranks(Comm* C, int l, double* const* r, double* const* x, bool rtz = false) {
  Context* c = C->ctx;
  const int nl = (int)C->ranks.size();
  std::vector<double*> xc(nl), rc(nl);
  for (int i = 0; i < nl; ++i) {
    const Level& L = C->ranks[i]->lev[l];
    // ZeroVector(x) zeroes the externals too; the exchange inside the first
    // SYMGS would bring the neighbours' zeros
    if (L.next) HB_CK(cudaMemsetAsync(x[i] + L.n, 0, sizeof(double) * L.next, c->stream));
    HB_TRY(symgs_step(C->ranks[i], l, r[i], x[i], true));
  }
  hpcg_b200_problem* P0 = C->ranks[0];
  if (l + 1 >= P0->nlev) return HPCG_B200_OK;
  HB_TRY(exchange(C, l, x));  // ComputeSPMV_ref.cpp:53
  for (int i = 0; i < nl; ++i) {
    hpcg_b200_problem* P = C->ranks[i];
    rc[i] = P->lev[l + 1].r;
    xc[i] = P->lev[l + 1].x;
    HB_TRY(restrict_level(P, l, r[i], x[i], rc[i]));
  }
  HB_TRY(mg_ranks(C, l + 1, rc.data(), xc.data()));
  for (int i = 0; i < nl; ++i) HB_TRY(prolong_level(C->ranks[i], l, xc[i], x[i]));
  HB_TRY(exchange(C, l, x));  // ComputeSYMGS_ref.cpp:59
  for (int i = 0; i < nl; ++i) {
    if (rtz) {
      HB_CK(cudaMemsetAsync(c->partials, 0, sizeof(double) * kColours * kDotStride, c->stream));
      HB_TRY(symgs_step(C->ranks[i], l, r[i], x[i], false, c->partials));
      HB_TRY(store_partial(C, i, kColours * kDotStride));
    } else {
      HB_TRY(symgs_step(C->ranks[i], l, r[i], x[i], false));
    }
  }
  return HPCG_B200_OK;
}

int tune_all(Comm* C) {
  for (hpcg_b200_problem* P : C->ranks) HB_TRY(autotune_problem(P));
  return HPCG_B200_OK;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// CG.cpp:59-143 (CG_ref.cpp:58-144) over every rank of the run, the driven
// ranks' colour-order vectors resident: b -> x. times (may be null) receives
// the parts' device times in slots 1-5 as CG.cpp:132-139 files them.
int cg_ranks(Comm* C, int max_iter, double tol, bool prec, int* niters, double* normr_out, double* normr0_out,
             double* times) {
  Context* c = C->ctx;
  const int nl = (int)C->ranks.size();
  std::vector<double*> xs(nl), ps(nl), rs(nl), zs(nl);
  for (int i = 0; i < nl; ++i) {
    xs[i] = C->ranks[i]->x;
    ps[i] = C->ranks[i]->p;
    rs[i] = C->ranks[i]->r;
    zs[i] = C->ranks[i]->z;
  }
  PartTimer timer;
  if (times) timer.c = c;
  C->timer = times ? &timer : nullptr;
  struct Detach {  // the timer lives on this frame only
    Comm* C;
    ~Detach() { C->timer = nullptr; }
  } detach{C};
  int part = -1;
  // p = x; Ap = A p; r = b - Ap; normr = sqrt(r'r)   (CG.cpp:86-90)
  HB_TRY(exchange(C, 0, xs.data()));
  for (int i = 0; i < nl; ++i) {
    hpcg_b200_problem* P = C->ranks[i];
    HB_TRY(spmv_level(P, 0, P->x, P->Ap, false));
    HB_TRY(store_partial(C, i, launch_residual(c, P->lev[0].n, P->b, P->Ap, P->r)));
  }
  HB_TRY(reduce(C, kFinNormr));
  HB_TRY(read_scal(c));
  double normr = std::sqrt(c->scal_host->normr2);
  const double normr0 = normr;
  *niters = 0;
  const bool fused = prec && rtz_from_smoother(C->ranks[0]);
  for (int k = 1; k <= max_iter && normr / normr0 > tol; ++k) {
    HB_TRY(timer.start(5, &part));  // preconditioner (:101-106)
    if (prec) {
      HB_TRY(mg_ranks(C, 0, rs.data(), zs.data(), fused));  // CG.cpp:103
    } else {
      for (int i = 0; i < nl; ++i)
        HB_CK(cudaMemcpyAsync(zs[i], rs[i], sizeof(double) * C->ranks[i]->lev[0].n, cudaMemcpyDeviceToDevice,
                              c->stream));
    }
    HB_TRY(timer.stop(part));
    HB_TRY(timer.start(1, &part));  // rtz = r'z (:110 / :113)
    if (!fused) {
      for (int i = 0; i < nl; ++i)
        HB_TRY(store_partial(C, i, launch_dot(c, C->ranks[i]->lev[0].n, rs[i], zs[i])));
    }
    HB_TRY(reduce(C, k == 1 ? kFinRtzFirst : kFinRtz));
    HB_TRY(timer.stop(part));
    HB_TRY(timer.start(2, &part));  // p = z or p = z + beta p (:109 / :115), with x of iteration k - 1
    for (int i = 0; i < nl; ++i) {
      const int n = C->ranks[i]->lev[0].n;
      if (k == 1) {
        HB_CK(cudaMemcpyAsync(ps[i], zs[i], sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));  // :109
      } else {
        HB_TRY(launch_update_px(c, n, zs[i], ps[i], xs[i]));  // :115, and :121 of k - 1
      }
    }
    HB_TRY(timer.stop(part));
    HB_TRY(timer.start(3, &part));  // Ap = A p with its halo exchange (:118)
    HB_TRY(exchange(C, 0, ps.data()));  // ComputeSPMV_ref.cpp:53
    for (int i = 0; i < nl; ++i) {
      hpcg_b200_problem* P = C->ranks[i];
      const int parts = spmv_level(P, 0, P->p, P->Ap, true);  // Ap = A p, p'Ap partials (:118-119)
      HB_TRY(store_partial(C, i, parts));
    }
    HB_TRY(timer.stop(part));
    HB_TRY(timer.start(1, &part));  // pAp (:119)
    HB_TRY(reduce(C, kFinPap));  // alpha = rtz / pAp (:120)
    HB_TRY(timer.stop(part));
    HB_TRY(timer.start(2, &part));  // r update (:122-123), r'r partials with it; x waits for the next p update
    for (int i = 0; i < nl; ++i) {
      hpcg_b200_problem* P = C->ranks[i];
      HB_TRY(store_partial(C, i, launch_update_r(c, P->lev[0].n, P->r, P->Ap)));  // :122-123
    }
    HB_TRY(timer.stop(part));
    HB_TRY(timer.start(1, &part));  // normr = sqrt(r'r) (:124)
    HB_TRY(reduce(C, kFinNormr));
    HB_TRY(timer.stop(part));
    HB_TRY(read_scal(c));
    normr = std::sqrt(c->scal_host->normr2);
    *niters = k;
  }
  if (*niters > 0) {  // the last iteration's x update (:121)
    HB_TRY(timer.start(2, &part));
    for (int i = 0; i < nl; ++i) HB_TRY(launch_update_x(c, C->ranks[i]->lev[0].n, xs[i], ps[i]));
    HB_TRY(timer.stop(part));
  }
  *normr_out = normr;
  *normr0_out = normr0;
  if (times) HB_TRY(timer.add_to(times));
  return HPCG_B200_OK;
}

// A natural-order input vector (host or device) of driven rank i into the
// colour-order device vector dst (externals untouched).
int load(Comm* C, int i, int l, const double* src, double* dst) { return load_vector(C->ranks[i], l, src, dst); }

int check_vectors(const Comm* C, const void* const* v) {
  if (!v) return HPCG_B200_ERR_ARG;
  for (size_t i = 0; i < C->ranks.size(); ++i)
    if (!v[i]) return HPCG_B200_ERR_ARG;
  return HPCG_B200_OK;
}

struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int d) {
    cudaGetDevice(&prev);
    cudaSetDevice(d);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int comm_common(Comm* C) {
  Context* c = C->ctx;
  return dev_alloc((void**)&C->red, sizeof(double) * (size_t)(C->size + 1), nullptr) ||
                 cudaMemsetAsync(C->red, 0, sizeof(double) * (size_t)(C->size + 1), c->stream) != cudaSuccess
             ? HPCG_B200_ERR_NOMEM
             : HPCG_B200_OK;
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

int hpcg_b200_comm_unique_id(void* id) {
  if (!id) return HPCG_B200_ERR_ARG;
  NcclApi& api = nccl();
  if (!api.ok) {
    set_error_text("libnccl.so.2 could not be opened");
    return HPCG_B200_ERR_UNSUPPORTED;
  }
  ncclUniqueId u;
  HB_NCCL(api.GetUniqueId(&u), "ncclGetUniqueId");
  std::memcpy(id, &u, sizeof(u));
  return HPCG_B200_OK;
}

int hpcg_b200_comm_nccl(const void* id, int nranks, int rank, hpcg_b200_problem* p, hpcg_b200_comm** out) {
  if (!out) return HPCG_B200_ERR_ARG;
  *out = nullptr;
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (!id || nranks < 1) return HPCG_B200_ERR_ARG;
  const RankGeom g = p->geom ? *p->geom : RankGeom();
  if (g.size != nranks || g.rank != rank) return HPCG_B200_ERR_ARG;
  NcclApi& api = nccl();
  if (!api.ok) {
    set_error_text("libnccl.so.2 could not be opened");
    return HPCG_B200_ERR_UNSUPPORTED;
  }
  DeviceScope dev(p->device);
  Comm* C = new Comm;
  C->use_nccl = true;
  C->size = nranks;
  C->ranks.push_back(p);
  C->ctx = p->ctx;
  ncclUniqueId u;
  std::memcpy(&u, id, sizeof(u));
  int st = nccl_status(api.CommInitRank(&C->nc, nranks, u, rank), "ncclCommInitRank");
  if (st == HPCG_B200_OK) st = comm_common(C);
  if (st != HPCG_B200_OK) {
    if (C->nc) api.CommDestroy(C->nc);
    dev_free(C->red);
    delete C;
    return st;
  }
  *out = reinterpret_cast<hpcg_b200_comm*>(C);
  return HPCG_B200_OK;
}

int hpcg_b200_comm_local(int nranks, hpcg_b200_problem* const* ranks, hpcg_b200_comm** out) {
  if (!out) return HPCG_B200_ERR_ARG;
  *out = nullptr;
  if (!ranks || nranks < 1) return HPCG_B200_ERR_ARG;
  for (int i = 0; i < nranks; ++i) {
    if (!valid(ranks[i])) return HPCG_B200_ERR_HANDLE;
    const RankGeom g = ranks[i]->geom ? *ranks[i]->geom : RankGeom();
    if (g.size != nranks || g.rank != i || ranks[i]->device != ranks[0]->device ||
        ranks[i]->nlev != ranks[0]->nlev)
      return HPCG_B200_ERR_ARG;
  }
  DeviceScope dev(ranks[0]->device);
  Comm* C = new Comm;
  C->size = nranks;
  C->ranks.assign(ranks, ranks + nranks);
  C->ctx = ranks[0]->ctx;
  for (int l = 0; l < ranks[0]->nlev; ++l) {
    C->src_off[l].resize(nranks);
    for (int i = 0; i < nranks; ++i) {
      const HaloPlan* h = ranks[i]->lev[l].halo;
      if (!h) continue;
      for (int j = 0; j < h->nnb; ++j) {
        const HaloPlan* hn = ranks[h->nbr[j]]->lev[l].halo;
        int m = 0;
        while (hn && m < hn->nnb && hn->nbr[m] != i) ++m;
        if (!hn || m == hn->nnb || hn->off[m + 1] - hn->off[m] != h->off[j + 1] - h->off[j]) {
          delete C;
          return HPCG_B200_ERR_ARG;  // the ranks are not one decomposition
        }
        C->src_off[l][i].push_back(hn->off[m]);
      }
    }
  }
  const int st = comm_common(C);
  if (st != HPCG_B200_OK) {
    delete C;
    return st;
  }
  *out = reinterpret_cast<hpcg_b200_comm*>(C);
  return HPCG_B200_OK;
}

int hpcg_b200_comm_free(hpcg_b200_comm* comm) {
  Comm* C = reinterpret_cast<Comm*>(comm);
  if (!valid_comm(C)) return HPCG_B200_ERR_HANDLE;
  DeviceScope dev(C->ranks[0]->device);
  cudaStreamSynchronize(C->ctx->stream);
  if (C->nc) nccl().CommDestroy(C->nc);
  dev_free(C->red);
  C->magic = 0;
  delete C;
  return HPCG_B200_OK;
}

int hpcg_b200_shard_spmv(hpcg_b200_comm* comm, const double* const* x, double* const* y) {
  Comm* C = reinterpret_cast<Comm*>(comm);
  if (!valid_comm(C)) return HPCG_B200_ERR_HANDLE;
  HB_TRY(check_vectors(C, (const void* const*)x));
  HB_TRY(check_vectors(C, (const void* const*)y));
  DeviceScope dev(C->ranks[0]->device);
  HB_TRY(tune_all(C));
  const int nl = (int)C->ranks.size();
  std::vector<double*> ps(nl);
  for (int i = 0; i < nl; ++i) {
    ps[i] = C->ranks[i]->p;
    HB_TRY(load(C, i, 0, x[i], ps[i]));
  }
  HB_TRY(exchange(C, 0, ps.data()));
  for (int i = 0; i < nl; ++i) HB_TRY(spmv_level(C->ranks[i], 0, ps[i], C->ranks[i]->Ap, false));
  for (int i = 0; i < nl; ++i) HB_TRY(store_vector(C->ranks[i], 0, C->ranks[i]->Ap, y[i]));
  return HPCG_B200_OK;
}

int hpcg_b200_shard_symgs(hpcg_b200_comm* comm, const double* const* r, double* const* x) {
  Comm* C = reinterpret_cast<Comm*>(comm);
  if (!valid_comm(C)) return HPCG_B200_ERR_HANDLE;
  HB_TRY(check_vectors(C, (const void* const*)r));
  HB_TRY(check_vectors(C, (const void* const*)x));
  DeviceScope dev(C->ranks[0]->device);
  HB_TRY(tune_all(C));
  const int nl = (int)C->ranks.size();
  std::vector<double*> xs(nl);
  for (int i = 0; i < nl; ++i) {
    xs[i] = C->ranks[i]->x;
    HB_TRY(load(C, i, 0, r[i], C->ranks[i]->r));
    HB_TRY(load(C, i, 0, x[i], xs[i]));
  }
  HB_TRY(exchange(C, 0, xs.data()));  // ComputeSYMGS_ref.cpp:59
  for (int i = 0; i < nl; ++i) HB_TRY(symgs_step(C->ranks[i], 0, C->ranks[i]->r, xs[i], false));
  for (int i = 0; i < nl; ++i) HB_TRY(store_vector(C->ranks[i], 0, xs[i], x[i]));
  return HPCG_B200_OK;
}

int hpcg_b200_shard_mg(hpcg_b200_comm* comm, const double* const* r, double* const* x) {
  Comm* C = reinterpret_cast<Comm*>(comm);
  if (!valid_comm(C)) return HPCG_B200_ERR_HANDLE;
  HB_TRY(check_vectors(C, (const void* const*)r));
  HB_TRY(check_vectors(C, (const void* const*)x));
  DeviceScope dev(C->ranks[0]->device);
  HB_TRY(tune_all(C));
  const int nl = (int)C->ranks.size();
  std::vector<double*> rs(nl), zs(nl);
  for (int i = 0; i < nl; ++i) {
    rs[i] = C->ranks[i]->r;
    zs[i] = C->ranks[i]->z;
    HB_TRY(load(C, i, 0, r[i], rs[i]));
  }
  HB_TRY(mg_ranks(C, 0, rs.data(), zs.data()));
  for (int i = 0; i < nl; ++i) HB_TRY(store_vector(C->ranks[i], 0, zs[i], x[i]));
  return HPCG_B200_OK;
}

int hpcg_b200_shard_dot(hpcg_b200_comm* comm, const double* const* x, const double* const* y, double* result) {
  Comm* C = reinterpret_cast<Comm*>(comm);
  if (!valid_comm(C)) return HPCG_B200_ERR_HANDLE;
  HB_TRY(check_vectors(C, (const void* const*)x));
  HB_TRY(check_vectors(C, (const void* const*)y));
  if (!result) return HPCG_B200_ERR_ARG;
  DeviceScope dev(C->ranks[0]->device);
  Context* c = C->ctx;
  const int nl = (int)C->ranks.size();
  for (int i = 0; i < nl; ++i) {
    hpcg_b200_problem* P = C->ranks[i];
    const int n = P->lev[0].n;
    // natural order in place (device) or staged (host): the sum runs in the caller's order
    const double* xd = x[i];
    const double* yd = y[i];
    bool xdev = false, ydev = false;
    HB_TRY(locate_ptr(xd, P->device, &xdev, "input vector"));
    HB_TRY(locate_ptr(yd, P->device, &ydev, "input vector"));
    if (!xdev || !ydev) {
      HB_TRY(ensure_stage(c, (size_t)n));
      if (!xdev) {
        HB_TRY(host_to_device(c, c->stage[0], xd, (size_t)n));
        xd = c->stage[0];
      }
      if (!ydev) {
        HB_TRY(host_to_device(c, c->stage[1], yd, (size_t)n));
        yd = c->stage[1];
      }
    }
    HB_TRY(store_partial(C, i, launch_dot(c, n, xd, yd)));
  }
  double* out = C->use_nccl ? C->red + 1 : C->red + C->size;
  HB_TRY(reduce(C, kFinStore, out));
  HB_CK(cudaMemcpyAsync(result, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HB_TRY(stream_sync(c));
  return HPCG_B200_OK;
}

int hpcg_b200_shard_cg(hpcg_b200_comm* comm, const double* const* b, double* const* x, int max_iter,
                       double tolerance, int do_preconditioning, int* niters, double* normr, double* normr0,
                       double* times) {
  Comm* C = reinterpret_cast<Comm*>(comm);
  if (!valid_comm(C)) return HPCG_B200_ERR_HANDLE;
  HB_TRY(check_vectors(C, (const void* const*)b));
  HB_TRY(check_vectors(C, (const void* const*)x));
  if (!niters || !normr || !normr0 || max_iter < 0) return HPCG_B200_ERR_ARG;
  DeviceScope dev(C->ranks[0]->device);
  HB_TRY(tune_all(C));
  const double t0 = now_s();
  for (int i = 0; i < (int)C->ranks.size(); ++i) {
    HB_TRY(load(C, i, 0, b[i], C->ranks[i]->b));
    HB_TRY(load(C, i, 0, x[i], C->ranks[i]->x));
  }
  HB_TRY(cg_ranks(C, max_iter, tolerance, do_preconditioning != 0, niters, normr, normr0, times));
  for (int i = 0; i < (int)C->ranks.size(); ++i) HB_TRY(store_vector(C->ranks[i], 0, C->ranks[i]->x, x[i]));
  if (times) times[0] += now_s() - t0;
  return HPCG_B200_OK;
}

}  // extern "C"
