// Problem set-up: the device hierarchy built from the reference's host
// structures (OptimizeProblem) or generated on the device, plus release,
// accounting and inspection.
#include <algorithm>
#include <climits>
#include <atomic>
#include <functional>
#include <thread>
#include <type_traits>
#include <vector>

#include "bulk.cuh"
#include "common.cuh"
#include "shard.cuh"

namespace hb {

void release_accounted(size_t bytes);

namespace {

int64_t pitch_for(int n) { return ((int64_t)n + 1 + 255) / 256 * 256; }

template <typename T>
int alloc_n(hpcg_b200_problem* p, T** ptr, int64_t count) {
  return dev_alloc((void**)ptr, sizeof(T) * (size_t)count, &p->bytes);
}

// Releases the captured coarse V-cycle (0: FP64, 1: FP32); the next stream-run
// V-cycle captures it again.
void drop_coarse_graph(hpcg_b200_problem* p, int which) {
  if (p->coarse_graph[which]) cudaGraphExecDestroy(p->coarse_graph[which]);
  p->coarse_graph[which] = nullptr;
}

hpcg_b200_problem* new_problem(int device, Context* c) {
  hpcg_b200_problem* p = new hpcg_b200_problem;
  std::memset(p, 0, sizeof(*p));
  p->magic = kMagic;
  p->device = device;
  p->ctx = c;
  p->symgs_mode = HPCG_B200_SYMGS_COLOUR;
  const char* reuse = std::getenv("HPCG_B200_HOST_REUSE");
  p->host_reuse = reuse && reuse[0] == '0' ? 0 : 1;
  for (int l = 0; l < kMaxLevels; ++l) p->lev[l] = Level();
  return p;
}

// Vectors of every level, zeroed so that entry n (the zero sink of padded slots) is 0.
int alloc_vectors(hpcg_b200_problem* p) {
  Level& L0 = p->lev[0];
  double** v0[] = {&p->b, &p->x, &p->r, &p->z, &p->p, &p->Ap, &p->zprev};
  for (double** v : v0) {
    HB_TRY(alloc_n(p, v, L0.pitch));
    HB_CK(cudaMemsetAsync(*v, 0, sizeof(double) * L0.pitch, p->ctx->stream));
  }
  for (int l = 1; l < p->nlev; ++l) {
    Level& L = p->lev[l];
    HB_TRY(alloc_n(p, &L.r, L.pitch));
    HB_TRY(alloc_n(p, &L.x, L.pitch));
    HB_CK(cudaMemsetAsync(L.r, 0, sizeof(double) * L.pitch, p->ctx->stream));
    HB_CK(cudaMemsetAsync(L.x, 0, sizeof(double) * L.pitch, p->ctx->stream));
  }
  return HPCG_B200_OK;
}

void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)>& body) {
  unsigned t = std::thread::hardware_concurrency();
  if (t == 0) t = 1;
  if (t > 32) t = 32;
  if (n < 65536 || t == 1) {
    body(0, n);
    return;
  }
  std::vector<std::thread> pool;
  const int64_t chunk = (n + t - 1) / t;
  for (unsigned i = 0; i < t; ++i) {
    const int64_t b = i * chunk, e = std::min<int64_t>(n, b + chunk);
    if (b < e) pool.emplace_back(body, b, e);
  }
  for (auto& th : pool) th.join();
}

// ---- device generator (GenerateProblem_ref.cpp:131-183 in colour order) -----

// Where this level's block sits in the global grid (one rank: the whole grid).
struct GenGeom {
  int gnx, gny, gnz;  // global grid of the level
  int gx0, gy0, gz0;  // first global coordinate of this rank's block
  int ext_off[27];    // by direction (dz+1)*9+(dy+1)*3+(dx+1): first external column of that neighbour, -1 none
  int sink;           // the zero column of padded slots
};

// Rows, values and columns of one level. A direction inside the global grid but
// outside this rank's block is a nonzero of the reference's matrix too
// (GenerateProblem_ref.cpp:152-162 tests the global bounds); its column is the
// neighbour's external entry, numbered as the halo plan orders them.
__global__ void k_generate(ColourGrid g, int n, int64_t pitch, GenGeom G, double* __restrict__ val,
                           int* __restrict__ col, int* __restrict__ new2old, int* __restrict__ old2new,
                           double* __restrict__ b) {
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    int ix, iy, iz;
    g.coords(q, ix, iy, iz);
    const int i = (iz * g.ny + iy) * g.nx + ix;
    new2old[q] = i;
    old2new[i] = q;
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const int jx = ix + k % 3 - 1, jy = iy + (k / 3) % 3 - 1, jz = iz + k / 9 - 1;
      const bool local = jx >= 0 && jx < g.nx && jy >= 0 && jy < g.ny && jz >= 0 && jz < g.nz;
      const int gx = G.gx0 + jx, gy = G.gy0 + jy, gz = G.gz0 + jz;
      bool in = gx >= 0 && gx < G.gnx && gy >= 0 && gy < G.gny && gz >= 0 && gz < G.gnz;
      int c = G.sink;
      if (local) {
        c = g.old2new(jx, jy, jz);
      } else if (in) {
        const int ex = jx < 0 ? -1 : jx >= g.nx ? 1 : 0;
        const int ey = jy < 0 ? -1 : jy >= g.ny ? 1 : 0;
        const int ez = jz < 0 ? -1 : jz >= g.nz ? 1 : 0;
        const int off = G.ext_off[(ez + 1) * 9 + (ey + 1) * 3 + (ex + 1)];
        if (off >= 0) {
          const int lx = ex == 0 ? jx : 0, wx = ex == 0 ? g.nx : 1;
          const int ly = ey == 0 ? jy : 0, wy = ey == 0 ? g.ny : 1;
          const int lz = ez == 0 ? jz : 0;
          c = n + off + (lz * wy + ly) * wx + lx;
        } else {
          in = false;  // no such neighbour: cannot happen for a block of the process grid
        }
      }
      col[k * pitch + q] = c;
      val[k * pitch + q] = in ? (k == kDiagSlot ? 26.0 : -1.0) : 0.0;
      cnt += in ? 1 : 0;
    }
    if (b) b[q] = 26.0 - (double)(cnt - 1);
  }
}

// f2c (GenerateCoarseProblem.cpp:71-82) between two colour orders
__global__ void k_generate_f2c(ColourGrid gf, ColourGrid gc, int nc, int* __restrict__ f2c) {
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nc; q += stride) {
    int ix, iy, iz;
    gc.coords(q, ix, iy, iz);
    f2c[q] = gf.old2new(2 * ix, 2 * iy, 2 * iz);
  }
}

// scatter of natural-order diagonal values into slot 13
__global__ void k_set_diag(const double* __restrict__ d, const int* __restrict__ old2new, double* __restrict__ val13,
                           int n) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) val13[old2new[i]] = d[i];
}

// natural-order direction-slot values [n][27] into the colour-order slot-major layout
__global__ void k_set_values(const double* __restrict__ v, const int* __restrict__ new2old, double* __restrict__ val,
                             int64_t pitch, int n) {
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    const int64_t i = new2old[q];
    for (int k = 0; k < kSlots; ++k) val[k * pitch + q] = v[i * kSlots + k];
  }
}

int check_dims(int nx, int ny, int nz, int nlevels) {
  if (nx < 1 || ny < 1 || nz < 1 || nlevels < 1 || nlevels > kMaxLevels) return HPCG_B200_ERR_ARG;
  if ((int64_t)nx * ny * nz >= (int64_t)1 << 31) return HPCG_B200_ERR_UNSUPPORTED;
  for (int l = 1; l < nlevels; ++l) {  // GenerateCoarseProblem.cpp:50
    const int f = 1 << (l - 1);
    if ((nx / f) % 2 || (ny / f) % 2 || (nz / f) % 2) return HPCG_B200_ERR_UNSUPPORTED;
  }
  return HPCG_B200_OK;
}

}  // namespace

// The pairs (f2c[q], q) ordered by fine row: counting by fine row, since f2c is
// injective into [0, n).
int build_transfer(hpcg_b200_problem* p, int l) {
  Level& L = p->lev[l];
  if (!L.f2c || l + 1 >= p->nlev) return HPCG_B200_OK;
  const int nc = p->lev[l + 1].n;
  std::vector<int> f(nc);
  HB_CK(cudaMemcpy(f.data(), L.f2c, sizeof(int) * nc, cudaMemcpyDeviceToHost));
  std::vector<int> inv(L.n, -1);
  for (int q = 0; q < nc; ++q) {
    if (f[q] < 0 || f[q] >= L.n || inv[f[q]] >= 0) return HPCG_B200_ERR_ARG;
    inv[f[q]] = q;
  }
  std::vector<int> tf(nc), tq(nc);
  int t = 0;
  for (int i = 0; i < L.n; ++i)
    if (inv[i] >= 0) { tf[t] = i; tq[t] = inv[i]; ++t; }
  HB_TRY(alloc_n(p, &L.tf, nc));
  HB_TRY(alloc_n(p, &L.tq, nc));
  HB_CK(cudaMemcpy(L.tf, tf.data(), sizeof(int) * nc, cudaMemcpyHostToDevice));
  HB_CK(cudaMemcpy(L.tq, tq.data(), sizeof(int) * nc, cudaMemcpyHostToDevice));
  // the injected rows as one run of storage (the colour-0 block of the parity
  // colouring): the bulk-copy restriction tiles it like a phase
  bool run = nc > 0;
  for (int u = 0; u < nc && run; ++u) run = tf[u] == tf[0] + u;
  L.tf_run = run ? tf[0] : -1;
  return HPCG_B200_OK;
}

// The packed columns of a level with offsets of W bytes (records of
// pack_rec(W) bytes, one per kBulkRows-row tile of the storage): block b builds
// tiles b, b + gridDim.x, ..., thread t row t of the tile. Rows at or beyond n
// are stored as the sink (they are never computed). Sets *bad if the columns
// of a slot of a tile span more than pack_max_span(W).
template <int W>
__global__ void __launch_bounds__(kBulkRows) k_pack_cols(const int* __restrict__ col, int64_t pitch, int n,
                                                         int sink, int64_t ntiles, unsigned char* __restrict__ colp,
                                                         int* bad) {
  using Off = typename std::conditional<W == 1, unsigned char, unsigned short>::type;
  constexpr int NW = kBulkRows / 32;
  __shared__ int wlo[NW], whi[NW];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t q = tile * kBulkRows + t;
    int* base = reinterpret_cast<int*>(colp + tile * pack_rec(W));
    Off* off = reinterpret_cast<Off*>(base + kPackBaseWords);
    if (t == 0) base[kSlots] = W;  // the record states its offset width
    for (int k = 0; k < kSlots; ++k) {
      const int c = q < n ? col[mat_index<double>(k, q, pitch)] : sink;
      const bool real = c != sink;
      int lo = real ? c : INT_MAX, hi = real ? c : INT_MIN;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      }
      if (lane == 0) {
        wlo[w] = lo;
        whi[w] = hi;
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < NW; ++i) {
        lo = min(lo, wlo[i]);
        hi = max(hi, whi[i]);
      }
      __syncthreads();
      const int b = lo == INT_MAX ? 0 : lo;
      if (t == 0) {
        base[k] = b;
        if (lo != INT_MAX && (int64_t)hi - lo > pack_max_span(W)) *bad = 1;
      }
      off[k * kBulkRows + t] = real ? (Off)(c - b) : (Off)pack_sink(W);
    }
  }
}

// The packed columns of a level in the diagonal form (records of
// pack_rec(kPackDiag) bytes): slot k's base is column - row of the tile's
// columns that are not the sink, and its sink bits mark the rest. Rows at or
// beyond n are stored as the sink. Sets *bad if a slot's columns of a tile are
// not one diagonal (column - row differs between two of its rows).
__global__ void __launch_bounds__(kBulkRows) k_pack_cols_diag(const int* __restrict__ col, int64_t pitch, int n,
                                                              int sink, int64_t ntiles,
                                                              unsigned char* __restrict__ colp, int* bad) {
  constexpr int NW = kBulkRows / 32;
  __shared__ int wlo[NW], whi[NW];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t q = tile * kBulkRows + t;
    int* base = reinterpret_cast<int*>(colp + tile * pack_rec(kPackDiag));
    unsigned* bits = reinterpret_cast<unsigned*>(base + kPackBaseWords);
    if (t == 0) base[kSlots] = kPackDiag;  // the record states its form
    for (int k = 0; k < kSlots; ++k) {
      const int c = q < n ? col[mat_index<double>(k, q, pitch)] : sink;
      const bool real = c != sink;
      const int d = c - t;  // the diagonal this row's column lies on
      int lo = real ? d : INT_MAX, hi = real ? d : INT_MIN;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      }
      const unsigned sinks = __ballot_sync(0xffffffffu, !real);
      if (lane == 0) {
        wlo[w] = lo;
        whi[w] = hi;
        bits[k * NW + w] = sinks;
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < NW; ++i) {
        lo = min(lo, wlo[i]);
        hi = max(hi, whi[i]);
      }
      __syncthreads();
      if (t == 0) {
        base[k] = lo == INT_MAX ? 0 : lo;
        if (lo != INT_MAX && lo != hi) *bad = 1;
      }
    }
  }
}

// Packs level l's columns with W-byte offsets into a new allocation; on return
// L.colp / L.pack describe it, or are left empty if a tile does not pack.
template <int W>
void launch_pack(Context* c, const Level& L, int64_t ntiles, unsigned char* colp, int* bad) {
  const int g = (int)std::min<int64_t>(ntiles, (int64_t)c->sms * 16);
  if constexpr (W == kPackDiag)
    k_pack_cols_diag<<<g, kBulkRows, 0, c->stream>>>(L.col, L.pitch, L.n, sink_of(L), ntiles, colp, bad);
  else
    k_pack_cols<W><<<g, kBulkRows, 0, c->stream>>>(L.col, L.pitch, L.n, sink_of(L), ntiles, colp, bad);
}

template <int W>
int try_pack(hpcg_b200_problem* p, int l) {
  Level& L = p->lev[l];
  Context* c = p->ctx;
  const int64_t ntiles = L.pitch / kBulkRows;
  const size_t bytes = (size_t)ntiles * pack_rec(W);
  unsigned char* colp = nullptr;
  HB_TRY(dev_alloc((void**)&colp, bytes, &p->bytes));
  int* bad = nullptr;
  cudaError_t err = cudaMalloc(&bad, sizeof(int));
  int h = 0;
  if (err == cudaSuccess) err = cudaMemsetAsync(bad, 0, sizeof(int), c->stream);
  if (err == cudaSuccess) {
    launch_pack<W>(c, L, ntiles, colp, bad);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(c->stream);
  cudaFree(bad);
  if (err != cudaSuccess || h) {  // failed, or a tile does not pack: give the memory back
    dev_free(colp);
    p->bytes -= bytes;
    release_accounted(bytes);
    if (err != cudaSuccess) {
      set_error("pack columns", err);
      return status_of(err);
    }
    return HPCG_B200_OK;
  }
  L.colp = colp;
  L.pack = W;
  return HPCG_B200_OK;
}

// The packed columns of level l for the bulk-copy kernels: the diagonal form
// where every tile's slots are diagonals, else 8-bit offsets where every
// tile's spans allow, else 16-bit ones; the level keeps only its 32-bit
// columns if a tile does not pack any of these ways.
// HPCG_B200_PACKED at creation (for comparisons): "0" leaves every level
// unpacked, "8" starts at the 8-bit offsets, "16" takes 16-bit ones only.
int build_packed(hpcg_b200_problem* p, int l) {
  Level& L = p->lev[l];
  const char* e = std::getenv("HPCG_B200_PACKED");
  if ((e && e[0] == '0') || L.n <= 0) return HPCG_B200_OK;
  const bool only16 = e && std::strcmp(e, "16") == 0;
  const bool from8 = e && std::strcmp(e, "8") == 0;
  if (!only16 && !from8) HB_TRY(try_pack<kPackDiag>(p, l));
  if (!L.colp && !only16) HB_TRY(try_pack<1>(p, l));
  if (!L.colp) HB_TRY(try_pack<2>(p, l));
  return HPCG_B200_OK;
}

int free_problem(hpcg_b200_problem* p) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  cudaSetDevice(p->device);
  if (p->ctx) cudaStreamSynchronize(p->ctx->stream);
  for (int l = 0; l < kMaxLevels; ++l) {
    Level& L = p->lev[l];
    void* ptrs[] = {L.val, L.col, L.val32, L.col32, L.new2old, L.old2new, L.f2c, L.tf, L.tq, L.r, L.x, L.r32, L.x32,
                    L.wave_rows, L.colp, L.wf_done};
    for (void* q : ptrs) dev_free(q);
    delete[] L.wave_start;
    delete L.maps;
  }
  void* vs[] = {p->b, p->x, p->r, p->z, p->p, p->Ap, p->zprev};
  for (void* q : vs) dev_free(q);
  delete[] p->b_kept_host;
  free_multi(p);
  free_plans(p);
  for (int i = 0; i < 2; ++i) {
    if (p->cg_graph[i]) cudaGraphExecDestroy(p->cg_graph[i]);
    if (p->coarse_graph[i]) cudaGraphExecDestroy(p->coarse_graph[i]);
  }
  release_accounted(p->bytes);
  p->magic = 0;
  delete p;
  return HPCG_B200_OK;
}

// Device generation of the hierarchy of one rank (geom == nullptr: the whole grid
// on one rank), GenerateProblem_ref.cpp:131-183, GenerateCoarseProblem.cpp:71-104
// and, for a rank with neighbours, the halo plan of SetupHalo_ref.cpp:69-176.
int generate_impl(int nx, int ny, int nz, int nlevels, int device, const RankGeom* geom, hpcg_b200_problem** out) {
  if (!out) return HPCG_B200_ERR_ARG;
  *out = nullptr;
  HB_TRY(check_dims(nx, ny, nz, nlevels));
  Context* c = context_for(device);
  if (!c) return HPCG_B200_ERR_CUDA;
  HB_CK(cudaSetDevice(device));
  hpcg_b200_problem* p = new_problem(device, c);
  p->nlev = nlevels;
  if (geom) p->geom = new RankGeom(*geom);
  const RankGeom G = geom ? *geom : RankGeom();
  std::vector<std::vector<int> > sends(nlevels);
  for (int l = 0; l < nlevels; ++l) {
    Level& L = p->lev[l];
    L.g.init(nx >> l, ny >> l, nz >> l, kSweepDefault);
    L.n = (nx >> l) * (ny >> l) * (nz >> l);
    if (G.size > 1) {
      L.halo = new HaloPlan;
      plan_level(G, nx >> l, ny >> l, nz >> l, *L.halo, sends[l]);
      L.next = L.halo->total;
    }
    L.pitch = pitch_for(L.n + L.next);
  }
  int status = HPCG_B200_OK;
  for (int l = 0; l < nlevels && status == HPCG_B200_OK; ++l) {
    Level& L = p->lev[l];
    status = alloc_n(p, &L.val, kSlots * L.pitch);
    if (!status) status = alloc_n(p, &L.col, kSlots * L.pitch);
    if (!status) status = alloc_n(p, &L.new2old, L.n);
    if (!status) status = alloc_n(p, &L.old2new, L.n);
    if (!status && l + 1 < nlevels) status = alloc_n(p, &L.f2c, p->lev[l + 1].n);
  }
  if (status == HPCG_B200_OK) status = alloc_vectors(p);
  for (int l = 0; l < nlevels && status == HPCG_B200_OK; ++l) {
    Level& L = p->lev[l];
    // padding columns of the tail [n, pitch) are never read; zero them anyway
    cudaError_t e = cudaMemsetAsync(L.val, 0, sizeof(double) * kSlots * L.pitch, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(L.col, 0, sizeof(int) * kSlots * L.pitch, c->stream);
    if (e != cudaSuccess) { set_error("generate memset", e); status = status_of(e); break; }
    const int lx = nx >> l, ly = ny >> l, lz = nz >> l;
    GenGeom gg;
    gg.gnx = G.npx * lx; gg.gny = G.npy * ly; gg.gnz = G.npz * lz;
    gg.gx0 = G.ipx * lx; gg.gy0 = G.ipy * ly; gg.gz0 = G.ipz * lz;
    for (int d = 0; d < 27; ++d) gg.ext_off[d] = L.halo ? L.halo->ext_off[d] : -1;
    gg.sink = sink_of(L);
    k_generate<<<grid_for(c, L.n, 256, 8), 256, 0, c->stream>>>(L.g, L.n, L.pitch, gg, L.val, L.col, L.new2old,
                                                                  L.old2new, l == 0 ? p->b : nullptr);
    if (l + 1 < nlevels) {
      const Level& C = p->lev[l + 1];
      k_generate_f2c<<<grid_for(c, C.n, 256, 8), 256, 0, c->stream>>>(L.g, C.g, C.n, L.f2c);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { set_error("generate", e); status = status_of(e); }
  }
  for (int l = 0; l + 1 < nlevels && status == HPCG_B200_OK; ++l) status = build_transfer(p, l);
  for (int l = 0; l < nlevels && status == HPCG_B200_OK; ++l) status = upload_plan(p, l, sends[l]);
  for (int l = 0; l < nlevels && status == HPCG_B200_OK; ++l) status = build_packed(p, l);
  if (status != HPCG_B200_OK) {
    free_problem(p);
    return status;
  }
  *out = p;
  return HPCG_B200_OK;
}

}  // namespace hb

using namespace hb;

extern "C" {

int hpcg_b200_optimize(const hpcg_b200_level_desc* desc, int nlevels, int device, hpcg_b200_problem** out) {
  if (!desc || !out || nlevels < 1 || nlevels > kMaxLevels) return HPCG_B200_ERR_ARG;
  *out = nullptr;
  for (int l = 0; l < nlevels; ++l) {
    const hpcg_b200_level_desc& d = desc[l];
    if (!d.nonzeros_in_row || !d.mtx_ind_l || !d.matrix_values) return HPCG_B200_ERR_ARG;
    if ((int64_t)d.nx * d.ny * d.nz != d.nrow || d.ncol != d.nrow || d.nrow < 1) return HPCG_B200_ERR_ARG;
    if (l + 1 < nlevels) {
      if (!d.f2c) return HPCG_B200_ERR_ARG;
      const hpcg_b200_level_desc& c = desc[l + 1];
      if (c.nx * 2 != d.nx || c.ny * 2 != d.ny || c.nz * 2 != d.nz) return HPCG_B200_ERR_UNSUPPORTED;
    }
  }
  Context* c = context_for(device);
  if (!c) return HPCG_B200_ERR_CUDA;
  HB_CK(cudaSetDevice(device));
  hpcg_b200_problem* p = new_problem(device, c);
  p->nlev = nlevels;
  std::vector<ColourGrid> grids(nlevels);
  for (int l = 0; l < nlevels; ++l) {
    grids[l].init(desc[l].nx, desc[l].ny, desc[l].nz, kSweepDefault);
    p->lev[l].g = grids[l];
    p->lev[l].n = desc[l].nrow;
    p->lev[l].pitch = pitch_for(desc[l].nrow);
  }
  int status = HPCG_B200_OK;
  for (int l = 0; l < nlevels && status == HPCG_B200_OK; ++l) {
    const hpcg_b200_level_desc& d = desc[l];
    Level& L = p->lev[l];
    const ColourGrid& g = grids[l];
    const int n = L.n;
    const int64_t pitch = L.pitch;
    std::vector<double> val((size_t)kSlots * pitch, 0.0);
    std::vector<int> col((size_t)kSlots * pitch, n);
    std::vector<int> n2o(n), o2n(n);
    std::atomic<int> bad(0);
    parallel_for(n, [&](int64_t b, int64_t e) {
      for (int64_t i = b; i < e; ++i) {
        const int ix = (int)(i % d.nx), iy = (int)((i / d.nx) % d.ny), iz = (int)(i / ((int64_t)d.nx * d.ny));
        const int q = g.old2new(ix, iy, iz);
        n2o[q] = (int)i;
        o2n[i] = q;
        const int cnt = d.nonzeros_in_row[i];
        if (cnt < 1 || cnt > kSlots) { bad = 1; continue; }
        uint32_t seen = 0;
        for (int j = 0; j < cnt; ++j) {
          const int cj = d.mtx_ind_l[i][j];
          if (cj < 0 || cj >= n) { bad = 1; break; }
          const int dx = cj % d.nx - ix, dy = (cj / d.nx) % d.ny - iy, dz = cj / (d.nx * d.ny) - iz;
          if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) { bad = 1; break; }
          const int k = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
          if (seen & (1u << k)) { bad = 1; break; }
          seen |= 1u << k;
          val[(size_t)k * pitch + q] = d.matrix_values[i][j];
          col[(size_t)k * pitch + q] = g.old2new(ix + dx, iy + dy, iz + dz);
        }
        if (!(seen & (1u << kDiagSlot))) bad = 1;
      }
    });
    if (bad) { status = HPCG_B200_ERR_UNSUPPORTED; break; }
    status = alloc_n(p, &L.val, kSlots * pitch);
    if (!status) status = alloc_n(p, &L.col, kSlots * pitch);
    if (!status) status = alloc_n(p, &L.new2old, n);
    if (!status) status = alloc_n(p, &L.old2new, n);
    if (status) break;
    cudaError_t e = cudaMemcpy(L.val, val.data(), sizeof(double) * val.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(L.col, col.data(), sizeof(int) * col.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(L.new2old, n2o.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(L.old2new, o2n.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { set_error("optimize upload", e); status = status_of(e); break; }
    if (l + 1 < nlevels) {
      const int nc = desc[l + 1].nrow;
      const ColourGrid& gc = grids[l + 1];
      std::vector<int> f(nc);
      for (int qc = 0; qc < nc && !bad; ++qc) {
        int cx, cy, cz;
        gc.coords(qc, cx, cy, cz);
        const int natc = (cz * desc[l + 1].ny + cy) * desc[l + 1].nx + cx;
        const int ff = d.f2c[natc];
        if (ff < 0 || ff >= n) { bad = 1; break; }
        f[qc] = o2n[ff];
      }
      if (bad) { status = HPCG_B200_ERR_ARG; break; }
      status = alloc_n(p, &L.f2c, nc);
      if (status) break;
      e = cudaMemcpy(L.f2c, f.data(), sizeof(int) * nc, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) { set_error("optimize f2c upload", e); status = status_of(e); break; }
    }
  }
  if (status == HPCG_B200_OK) status = alloc_vectors(p);
  for (int l = 0; l + 1 < nlevels && status == HPCG_B200_OK; ++l) status = build_transfer(p, l);
  for (int l = 0; l < nlevels && status == HPCG_B200_OK; ++l) status = build_packed(p, l);
  if (status == HPCG_B200_OK) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { set_error("optimize sync", e); status = status_of(e); }
  }
  if (status != HPCG_B200_OK) {
    free_problem(p);
    return status;
  }
  *out = p;
  return HPCG_B200_OK;
}

int hpcg_b200_generate(int nx, int ny, int nz, int nlevels, int device, hpcg_b200_problem** out) {
  return generate_impl(nx, ny, nz, nlevels, device, nullptr, out);
}

int hpcg_b200_generate_rank(int nx, int ny, int nz, int npx, int npy, int npz, int rank, int nlevels, int device,
                            hpcg_b200_problem** out) {
  if (!out) return HPCG_B200_ERR_ARG;
  *out = nullptr;
  RankGeom g;
  if (!make_geom(npx, npy, npz, rank, g)) return HPCG_B200_ERR_ARG;
  if ((int64_t)npx * nx >= (1 << 30) || (int64_t)npy * ny >= (1 << 30) || (int64_t)npz * nz >= (1 << 30))
    return HPCG_B200_ERR_UNSUPPORTED;
  return generate_impl(nx, ny, nz, nlevels, device, &g, out);
}

int hpcg_b200_process_grid(int nranks, int* npx, int* npy, int* npz) {
  if (nranks < 1 || !npx || !npy || !npz) return HPCG_B200_ERR_ARG;
  optimal_shape(nranks, *npx, *npy, *npz);
  return HPCG_B200_OK;
}

int hpcg_b200_halo_plan(int nx, int ny, int nz, int npx, int npy, int npz, int rank, int* nneighbors,
                        int* neighbors, int* counts, int* send_rows, long long* ext_global) {
  RankGeom g;
  if (!make_geom(npx, npy, npz, rank, g) || nx < 1 || ny < 1 || nz < 1 || !nneighbors) return HPCG_B200_ERR_ARG;
  HaloPlan h;
  std::vector<int> send;
  plan_level(g, nx, ny, nz, h, send);
  *nneighbors = h.nnb;
  for (int i = 0; i < h.nnb; ++i) {
    if (neighbors) neighbors[i] = h.nbr[i];
    if (counts) counts[i] = h.off[i + 1] - h.off[i];
  }
  if (send_rows) std::copy(send.begin(), send.end(), send_rows);
  if (ext_global) {
    std::vector<long long> ext;
    plan_externals(g, nx, ny, nz, h, ext);
    std::copy(ext.begin(), ext.end(), ext_global);
  }
  return HPCG_B200_OK;
}

int hpcg_b200_rank_info(const hpcg_b200_problem* p, int level, int* info) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (!info || level < 0 || level >= p->nlev) return HPCG_B200_ERR_ARG;
  const RankGeom g = p->geom ? *p->geom : RankGeom();
  const Level& L = p->lev[level];
  const int v[10] = {g.rank, g.size, g.npx, g.npy, g.npz, g.ipx, g.ipy, g.ipz, L.halo ? L.halo->nnb : 0, L.next};
  std::copy(v, v + 10, info);
  return HPCG_B200_OK;
}

int hpcg_b200_free(hpcg_b200_problem* p) { return free_problem(p); }

int hpcg_b200_colour_permutation(int nx, int ny, int nz, int* new2old, int* colour_start) {
  if (nx < 1 || ny < 1 || nz < 1 || (int64_t)nx * ny * nz >= ((int64_t)1 << 31)) return HPCG_B200_ERR_ARG;
  ColourGrid g;
  g.init(nx, ny, nz, kSweepDefault);
  if (colour_start)
    for (int s = 0; s <= kColours; ++s) colour_start[s] = g.start[s];
  if (new2old)
    for (int iz = 0; iz < nz; ++iz)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) new2old[g.old2new(ix, iy, iz)] = (iz * ny + iy) * nx + ix;
  return HPCG_B200_OK;
}

double hpcg_b200_memory_use(const hpcg_b200_problem* p) { return valid(p) ? (double)p->bytes : 0.0; }

int hpcg_b200_get_rhs(hpcg_b200_problem* p, double* b) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (!b) return HPCG_B200_ERR_ARG;
  HB_CK(cudaSetDevice(p->device));
  return store_vector(p, 0, p->b, b);
}

int hpcg_b200_set_diagonal(hpcg_b200_problem* p, const double* diagonal) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (!diagonal) return HPCG_B200_ERR_ARG;
  HB_CK(cudaSetDevice(p->device));
  Level& L = p->lev[0];
  Context* c = p->ctx;
  const double* src = diagonal;
  bool dev = false;
  HB_TRY(locate_ptr(diagonal, p->device, &dev, "hpcg_b200_set_diagonal"));
  if (!dev) {
    HB_TRY(ensure_stage(c, L.n));
    HB_TRY(host_to_device(c, c->stage[1], diagonal, (size_t)L.n));
    src = c->stage[1];
  }
  k_set_diag<<<grid_for(c, L.n, 256, 8), 256, 0, c->stream>>>(src, L.old2new, L.val + kDiagSlot * L.pitch, L.n);
  HB_CK(cudaGetLastError());
  if (L.val32) {  // the FP32 copy is rebuilt on next use
    dev_free(L.val32);
    L.val32 = nullptr;
    dev_free(L.col32);
    L.col32 = nullptr;
    drop_coarse_graph(p, 1);  // it holds the old copy's addresses
  }
  HB_CK(cudaStreamSynchronize(c->stream));
  return HPCG_B200_OK;
}

int hpcg_b200_set_values(hpcg_b200_problem* p, int level, const double* values27) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (!values27 || level < 0 || level >= p->nlev) return HPCG_B200_ERR_ARG;
  HB_CK(cudaSetDevice(p->device));
  Level& L = p->lev[level];
  Context* c = p->ctx;
  double* tmp = nullptr;
  const double* src = values27;
  bool dev = false;
  HB_TRY(locate_ptr(values27, p->device, &dev, "hpcg_b200_set_values"));
  if (!dev) {
    HB_CK(cudaMalloc(&tmp, sizeof(double) * (size_t)kSlots * L.n));
    cudaError_t e = cudaMemcpy(tmp, values27, sizeof(double) * (size_t)kSlots * L.n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(tmp);
      set_error("set_values upload", e);
      return status_of(e);
    }
    src = tmp;
  }
  k_set_values<<<grid_for(c, L.n, 256, 8), 256, 0, c->stream>>>(src, L.new2old, L.val, L.pitch, L.n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) {
    set_error("set_values", e);
    return status_of(e);
  }
  if (L.val32) {
    dev_free(L.val32);
    L.val32 = nullptr;
    dev_free(L.col32);
    L.col32 = nullptr;
    drop_coarse_graph(p, 1);  // it holds the old copy's addresses
  }
  return HPCG_B200_OK;
}

int hpcg_b200_set_host_reuse(hpcg_b200_problem* p, int enable) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  p->host_reuse = enable != 0;
  p->b_kept = false;
  return HPCG_B200_OK;
}

int hpcg_b200_set_symgs_mode(hpcg_b200_problem* p, int mode) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (mode != HPCG_B200_SYMGS_COLOUR && mode != HPCG_B200_SYMGS_NATURAL) return HPCG_B200_ERR_ARG;
  if (mode != p->symgs_mode) {
    // a captured CG loop holds the previous mode's kernels
    cudaSetDevice(p->device);
    for (int i = 0; i < 2; ++i) {
      if (p->cg_graph[i]) cudaGraphExecDestroy(p->cg_graph[i]);
      p->cg_graph[i] = nullptr;
      drop_coarse_graph(p, i);
    }
  }
  p->symgs_mode = mode;
  return HPCG_B200_OK;
}

int hpcg_b200_level_info(const hpcg_b200_problem* p, int level, int* nrow, int64_t* pitch, int* colour_start) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (level < 0 || level >= p->nlev) return HPCG_B200_ERR_ARG;
  const Level& L = p->lev[level];
  if (nrow) *nrow = L.n;
  if (pitch) *pitch = L.pitch;
  if (colour_start)
    for (int s = 0; s <= kColours; ++s) colour_start[s] = L.g.start[s];
  return HPCG_B200_OK;
}

int hpcg_b200_level_packed(const hpcg_b200_problem* p, int level, int64_t* bytes) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (!bytes || level < 0 || level >= p->nlev) return HPCG_B200_ERR_ARG;
  const Level& L = p->lev[level];
  *bytes = L.colp ? L.pitch / kBulkRows * pack_rec(L.pack) : 0;
  return HPCG_B200_OK;
}

int hpcg_b200_export_level(const hpcg_b200_problem* p, int level, int* new2old, int* cols, double* vals, int* f2c) {
  if (!valid(p)) return HPCG_B200_ERR_HANDLE;
  if (level < 0 || level >= p->nlev) return HPCG_B200_ERR_ARG;
  HB_CK(cudaSetDevice(p->device));
  const Level& L = p->lev[level];
  HB_CK(cudaStreamSynchronize(p->ctx->stream));
  if (new2old) HB_CK(cudaMemcpy(new2old, L.new2old, sizeof(int) * L.n, cudaMemcpyDeviceToHost));
  if (cols) HB_CK(cudaMemcpy(cols, L.col, sizeof(int) * kSlots * L.pitch, cudaMemcpyDeviceToHost));
  if (vals) HB_CK(cudaMemcpy(vals, L.val, sizeof(double) * kSlots * L.pitch, cudaMemcpyDeviceToHost));
  if (f2c && L.f2c) HB_CK(cudaMemcpy(f2c, L.f2c, sizeof(int) * p->lev[level + 1].n, cudaMemcpyDeviceToHost));
  return HPCG_B200_OK;
}

}  // extern "C"
