// The process grid and the halo exchange plan of a run over several ranks.
//
// Each rank owns an nx*ny*nz block of the global grid (GenerateGeometry.cpp),
// and its matrix references the points of its neighbours that touch its block:
// faces, edges and corners of up to 26 neighbours. The reference's SetupHalo_ref
// (SetupHalo_ref.cpp:69-176) finds them by scanning every nonzero's global
// column; here they follow from the geometry directly, in the same order
// (neighbours by ascending rank, each neighbour's points by ascending global
// row), so the rows a rank sends and the externals its neighbour receives pair
// up entry for entry.
#include <algorithm>
#include <cmath>
#include <map>

#include "shard.cuh"

namespace hb {

namespace {

// Prime factors of n with multiplicities, ascending; {1: 1} for n = 1
// (ComputePrimeFactors, ComputeOptimalShapeXYZ.cpp:47-70).
std::map<int, int> prime_factors(int n) {
  std::map<int, int> f;
  while (n > 1 && n % 2 == 0) {
    ++f[2];
    n /= 2;
  }
  const int lim = (int)std::sqrt((double)n) + 1;
  for (int d = 3; d <= lim; d += 2)
    while (n % d == 0) {
      ++f[d];
      n /= d;
    }
  if (n > 1 || f.empty()) ++f[n];
  return f;
}

int ipow(int b, int e) {
  int v = 1;
  while (e-- > 0) v *= b;
  return v;
}

// Exponent vectors counted in mixed radix, digit 0 fastest (MixedBaseCounter.cpp).
bool next_vector(std::vector<int>& v, const std::vector<int>& max) {
  for (size_t i = 0; i < v.size(); ++i) {
    if (++v[i] <= max[i]) return true;
    v[i] = 0;
  }
  return false;  // wrapped to zero
}

int product(const std::vector<int>& primes, const std::vector<int>& e) {
  int x = 1;
  for (size_t i = 0; i < e.size(); ++i) x *= ipow(primes[i], e[i]);
  return x;
}

__global__ void k_pack(int total, const int* __restrict__ rows, const double* __restrict__ x, double* __restrict__ buf) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) buf[i] = x[rows[i]];
}

}  // namespace

// ComputeOptimalShapeXYZ.cpp:80-157 (the default build, without
// HPCG_CUBIC_RADICAL_SEARCH): the special cases by the prime signature of
// `size`, otherwise the split of the prime factors into three products with the
// least surface area, first found wins.
void optimal_shape(int size, int& x, int& y, int& z) {
  const std::map<int, int> f = prime_factors(size);
  std::vector<int> primes, counts;
  for (const auto& kv : f) {
    primes.push_back(kv.first);
    counts.push_back(kv.second);
  }
  if (primes.size() == 1) {
    const int p = primes[0], e = counts[0];
    z = ipow(p, e / 3);
    y = ipow(p, e / 3 + (e % 3 >= 2 ? 1 : 0));
    x = ipow(p, e / 3 + (e % 3 >= 1 ? 1 : 0));
    return;
  }
  x = primes[0];
  y = primes[1];
  if (primes.size() == 2 && counts[0] == 1 && counts[1] == 1) {
    z = 1;
    return;
  }
  if (primes.size() == 2 && counts[0] + counts[1] == 3) {
    z = counts[0] == 2 ? primes[0] : primes[1];
    return;
  }
  if (primes.size() == 3 && counts[0] == 1 && counts[1] == 1 && counts[2] == 1) {
    z = primes[2];
    return;
  }
  double best = 2.0 * size + 1.0;
  std::vector<int> c1(primes.size(), 0);
  while (next_vector(c1, counts)) {
    std::vector<int> rest(primes.size()), c2(primes.size(), 0);
    for (size_t i = 0; i < primes.size(); ++i) rest[i] = counts[i] - c1[i];
    while (next_vector(c2, rest)) {
      const int t1 = product(primes, c1), t2 = product(primes, c2);
      const int t3 = size / t1 / t2;
      const double area = t1 * (double)t2 + t2 * (double)t3 + t1 * (double)t3;
      if (area < best) {
        best = area;
        x = t1;
        y = t2;
        z = t3;
      }
    }
  }
}

bool make_geom(int npx, int npy, int npz, int rank, RankGeom& g) {
  if (npx < 1 || npy < 1 || npz < 1) return false;
  const int64_t size = (int64_t)npx * npy * npz;
  if (size > (1 << 20) || rank < 0 || rank >= size) return false;
  g.size = (int)size;
  g.rank = rank;
  g.npx = npx;
  g.npy = npy;
  g.npz = npz;
  g.ipz = rank / (npx * npy);  // GenerateGeometry.cpp:89-91
  g.ipy = (rank - g.ipz * npx * npy) / npx;
  g.ipx = rank % npx;
  return true;
}

void plan_level(const RankGeom& G, int nx, int ny, int nz, HaloPlan& h, std::vector<int>& send) {
  struct Nb {
    int rank, dx, dy, dz;
  };
  std::vector<Nb> nbs;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        if (!dx && !dy && !dz) continue;
        const int px = G.ipx + dx, py = G.ipy + dy, pz = G.ipz + dz;
        if (px < 0 || px >= G.npx || py < 0 || py >= G.npy || pz < 0 || pz >= G.npz) continue;
        nbs.push_back(Nb{(pz * G.npy + py) * G.npx + px, dx, dy, dz});
      }
  std::sort(nbs.begin(), nbs.end(), [](const Nb& a, const Nb& b) { return a.rank < b.rank; });
  h.nnb = (int)nbs.size();
  for (int d = 0; d < 27; ++d) h.ext_off[d] = -1;
  send.clear();
  int off = 0;
  for (int i = 0; i < h.nnb; ++i) {
    const Nb& b = nbs[i];
    h.nbr[i] = b.rank;
    h.dir[i] = (b.dz + 1) * 9 + (b.dy + 1) * 3 + (b.dx + 1);
    h.off[i] = off;
    h.ext_off[h.dir[i]] = off;
    // this rank's points next to the neighbour: its last layer towards +1, first towards -1
    const int x0 = b.dx > 0 ? nx - 1 : 0, x1 = b.dx < 0 ? 1 : nx;
    const int y0 = b.dy > 0 ? ny - 1 : 0, y1 = b.dy < 0 ? 1 : ny;
    const int z0 = b.dz > 0 ? nz - 1 : 0, z1 = b.dz < 0 ? 1 : nz;
    for (int z = z0; z < z1; ++z)
      for (int y = y0; y < y1; ++y)
        for (int x = x0; x < x1; ++x) send.push_back((z * ny + y) * nx + x);
    off = (int)send.size();
  }
  h.off[h.nnb] = off;
  h.total = off;
}

void plan_externals(const RankGeom& G, int nx, int ny, int nz, const HaloPlan& h, std::vector<long long>& ext) {
  const long long gnx = (long long)G.npx * nx, gny = (long long)G.npy * ny;
  const long long gx0 = (long long)G.ipx * nx, gy0 = (long long)G.ipy * ny, gz0 = (long long)G.ipz * nz;
  ext.clear();
  for (int i = 0; i < h.nnb; ++i) {
    const int d = h.dir[i];
    const int dx = d % 3 - 1, dy = (d / 3) % 3 - 1, dz = d / 9 - 1;
    // the neighbour's points next to this rank: the layer just outside this block
    const long long xa = dx < 0 ? gx0 - 1 : dx > 0 ? gx0 + nx : gx0, xb = dx == 0 ? gx0 + nx : xa + 1;
    const long long ya = dy < 0 ? gy0 - 1 : dy > 0 ? gy0 + ny : gy0, yb = dy == 0 ? gy0 + ny : ya + 1;
    const long long za = dz < 0 ? gz0 - 1 : dz > 0 ? gz0 + nz : gz0, zb = dz == 0 ? gz0 + nz : za + 1;
    for (long long z = za; z < zb; ++z)
      for (long long y = ya; y < yb; ++y)
        for (long long x = xa; x < xb; ++x) ext.push_back((z * gny + y) * gnx + x);
  }
}

int upload_plan(hpcg_b200_problem* p, int l, const std::vector<int>& send_natural) {
  Level& L = p->lev[l];
  if (!L.halo || L.halo->total == 0) return HPCG_B200_OK;
  HaloPlan& h = *L.halo;
  std::vector<int> rows(h.total);
  const int nx = L.g.nx, ny = L.g.ny;
  for (int i = 0; i < h.total; ++i) {
    const int nat = send_natural[i];
    rows[i] = L.g.old2new(nat % nx, (nat / nx) % ny, nat / (nx * ny));
  }
  HB_TRY(dev_alloc((void**)&h.send_rows, sizeof(int) * (size_t)h.total, &p->bytes));
  HB_TRY(dev_alloc((void**)&h.send_buf, sizeof(double) * (size_t)h.total, &p->bytes));
  HB_CK(cudaMemcpy(h.send_rows, rows.data(), sizeof(int) * (size_t)h.total, cudaMemcpyHostToDevice));
  return HPCG_B200_OK;
}

void free_plans(hpcg_b200_problem* p) {
  for (int l = 0; l < kMaxLevels; ++l) {
    HaloPlan* h = p->lev[l].halo;
    if (!h) continue;
    dev_free(h->send_rows);
    dev_free(h->send_buf);
    delete h;
    p->lev[l].halo = nullptr;
  }
  delete p->geom;
  p->geom = nullptr;
}

int pack_halo(Context* c, const HaloPlan& h, const double* x) {
  if (h.total == 0) return HPCG_B200_OK;
  k_pack<<<grid_for(c, h.total, 256, 4), 256, 0, c->stream>>>(h.total, h.send_rows, x, h.send_buf);
  HB_CK(cudaGetLastError());
  return HPCG_B200_OK;
}

}  // namespace hb
