// C entry points over the HPCG 3.1 reference routines run as several MPI ranks.
// The reference's MPI branch (HPCG_NO_MPI undefined: SetupHalo_ref.cpp:69-176,
// ExchangeHalo.cpp:33-109, ComputeDotProduct_ref.cpp:66-73) is compiled from its
// own sources against oracle/mpi_shim, a thread-based stand-in for the MPI calls
// it makes, into oracle/_ref/libhpcg_ref_mpi.so by oracle/Makefile. Every rank is
// a thread; every entry point below runs the reference routine on all ranks at
// once, as mpirun would.
//
// TEST INFRASTRUCTURE ONLY: the tests use it as the parity pin of the sharded
// (one rank per GPU) path. Nothing in the product links it.
//
// Each rank's problem is set up as src/main.cpp:121-163 does: GenerateGeometry
// with the given process grid, GenerateProblem, SetupHalo, 3x
// GenerateCoarseProblem, InitializeSparseCGData.
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <vector>

#include "mpi.h"

#include "CGData.hpp"
#include "CG_ref.hpp"
#include "ComputeDotProduct_ref.hpp"
#include "ComputeMG_ref.hpp"
#include "ComputeOptimalShapeXYZ.hpp"
#include "ComputeSPMV_ref.hpp"
#include "ComputeSYMGS_ref.hpp"
#include "GenerateCoarseProblem.hpp"
#include "GenerateGeometry.hpp"
#include "GenerateProblem.hpp"
#include "Geometry.hpp"
#include "SetupHalo.hpp"
#include "SparseMatrix.hpp"
#include "Vector.hpp"

std::ofstream HPCG_fout;  // the reference's log stream (init.cpp), unused here

namespace {

const int kLevels = 4;  // main.cpp:139

struct Rank {
  SparseMatrix A;
  Vector b, x, xexact;
  CGData data;
};

struct World {
  int npx, npy, npz, nx, ny, nz;
  std::vector<Rank*> ranks;
};

SparseMatrix* level(Rank* p, int lev) {
  SparseMatrix* m = &p->A;
  for (int i = 0; i < lev && m; ++i) m = m->Ac;
  return m;
}

Vector wrap(const double* v, int n) {
  Vector w;
  w.localLength = n;
  w.values = const_cast<double*>(v);
  w.optimizationData = 0;
  return w;
}

template <typename F>
void on_all_ranks(int nranks, F f) {
  shim_run(
      nranks, [](int rank, void* arg) { (*static_cast<F*>(arg))(rank); }, &f);
}

}  // namespace

extern "C" {

void* refmpi_create(int npx, int npy, int npz, int nx, int ny, int nz) {
  World* w = new World{npx, npy, npz, nx, ny, nz, std::vector<Rank*>(npx * npy * npz, nullptr)};
  const int size = npx * npy * npz;
  on_all_ranks(size, [w, size](int rank) {
    Rank* p = new Rank;
    Geometry* geom = new Geometry;
    GenerateGeometry(size, rank, 1, 0, 0, 0, w->nx, w->ny, w->nz, w->npx, w->npy, w->npz, geom);
    InitializeSparseMatrix(p->A, geom);
    GenerateProblem(p->A, &p->b, &p->x, &p->xexact);
    SetupHalo(p->A);
    SparseMatrix* cur = &p->A;
    for (int l = 1; l < kLevels; ++l) {
      GenerateCoarseProblem(*cur);
      cur = cur->Ac;
    }
    InitializeSparseCGData(p->A, p->data);
    w->ranks[rank] = p;
  });
  return w;
}

// The reference's default process grid (ComputeOptimalShapeXYZ.cpp), as
// GenerateGeometry.cpp:52-53 calls it with npx = npy = npz = 0.
void refmpi_optimal_shape(int size, int* npx, int* npy, int* npz) {
  int x = 0, y = 0, z = 0;
  ComputeOptimalShapeXYZ(size, x, y, z);
  *npx = x;
  *npy = y;
  *npz = z;
}

void refmpi_destroy(void* h) {
  World* w = static_cast<World*>(h);
  for (Rank* p : w->ranks) {
    DeleteMatrix(p->A);
    DeleteCGData(p->data);
    DeleteVector(p->x);
    DeleteVector(p->b);
    DeleteVector(p->xexact);
    delete p;
  }
  delete w;
}

// nrow, ncol (rows + externals), neighbours, total entries sent.
void refmpi_level_sizes(void* h, int rank, int lev, int* sizes4) {
  const SparseMatrix* A = level(static_cast<World*>(h)->ranks[rank], lev);
  sizes4[0] = A->localNumberOfRows;
  sizes4[1] = A->localNumberOfColumns;
  sizes4[2] = A->numberOfSendNeighbors;
  sizes4[3] = A->totalToBeSent;
}

// One level of one rank in the oracle's layout (27 slots per row, entry order
// kept, empty slots point at the row itself with value 0); the halo plan as
// SetupHalo_ref.cpp:121-140 stores it: neighbours in ascending rank order, the
// receive and send lengths per neighbour, the local rows sent (elementsToSend),
// and the global index of every external column nrow..ncol-1.
void refmpi_export_level(void* h, int rank, int lev, int* nnz, int* cols, double* vals, int* f2c, int* neighbors,
                         int* recv_len, int* send_len, int* send_rows, long long* ext_global, long long* l2g) {
  const SparseMatrix* A = level(static_cast<World*>(h)->ranks[rank], lev);
  const int n = A->localNumberOfRows;
  for (int i = 0; i < n; ++i) {
    const int k = A->nonzerosInRow[i];
    if (nnz) nnz[i] = k;
    for (int j = 0; j < 27; ++j) {
      if (cols) cols[(long long)i * 27 + j] = j < k ? A->mtxIndL[i][j] : i;
      if (vals) vals[(long long)i * 27 + j] = j < k ? A->matrixValues[i][j] : 0.0;
    }
    if (l2g) l2g[i] = A->localToGlobalMap[i];
  }
  if (f2c && A->mgData) std::memcpy(f2c, A->mgData->f2cOperator, sizeof(int) * A->Ac->localNumberOfRows);
#ifndef HPCG_NO_MPI
  for (int i = 0; i < A->numberOfSendNeighbors; ++i) {
    if (neighbors) neighbors[i] = A->neighbors[i];
    if (recv_len) recv_len[i] = A->receiveLength[i];
    if (send_len) send_len[i] = A->sendLength[i];
  }
  if (send_rows) std::memcpy(send_rows, A->elementsToSend, sizeof(int) * A->totalToBeSent);
  if (ext_global) {
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < A->nonzerosInRow[i]; ++j) {
        const int c = A->mtxIndL[i][j];
        if (c >= n) ext_global[c - n] = A->mtxIndG[i][j];
      }
  }
#endif
}

void refmpi_get_b(void* h, int rank, double* b) {
  Rank* p = static_cast<World*>(h)->ranks[rank];
  std::memcpy(b, p->b.values, sizeof(double) * p->A.localNumberOfRows);
}

void refmpi_set_b(void* h, int rank, const double* b) {
  Rank* p = static_cast<World*>(h)->ranks[rank];
  std::memcpy(p->b.values, b, sizeof(double) * p->A.localNumberOfRows);
}

// The routines on every rank at once. Vectors per rank: x has ncol entries (its
// externals are overwritten by the halo exchange), r and y have nrow.
int refmpi_spmv(void* h, int lev, double* const* x, double* const* y) {
  World* w = static_cast<World*>(h);
  std::vector<int> err(w->ranks.size(), 0);
  on_all_ranks((int)w->ranks.size(), [&](int r) {
    SparseMatrix* A = level(w->ranks[r], lev);
    Vector xv = wrap(x[r], A->localNumberOfColumns), yv = wrap(y[r], A->localNumberOfRows);
    err[r] = ComputeSPMV_ref(*A, xv, yv);
  });
  int e = 0;
  for (int v : err) e |= v;
  return e;
}

int refmpi_symgs(void* h, int lev, double* const* r, double* const* x) {
  World* w = static_cast<World*>(h);
  std::vector<int> err(w->ranks.size(), 0);
  on_all_ranks((int)w->ranks.size(), [&](int k) {
    SparseMatrix* A = level(w->ranks[k], lev);
    Vector rv = wrap(r[k], A->localNumberOfRows), xv = wrap(x[k], A->localNumberOfColumns);
    err[k] = ComputeSYMGS_ref(*A, rv, xv);
  });
  int e = 0;
  for (int v : err) e |= v;
  return e;
}

int refmpi_mg(void* h, int lev, double* const* r, double* const* x) {
  World* w = static_cast<World*>(h);
  std::vector<int> err(w->ranks.size(), 0);
  on_all_ranks((int)w->ranks.size(), [&](int k) {
    SparseMatrix* A = level(w->ranks[k], lev);
    Vector rv = wrap(r[k], A->localNumberOfRows), xv = wrap(x[k], A->localNumberOfColumns);
    err[k] = ComputeMG_ref(*A, rv, xv);
  });
  int e = 0;
  for (int v : err) e |= v;
  return e;
}

// ComputeDotProduct_ref with its MPI_Allreduce: the same value on every rank.
double refmpi_dot(void* h, double* const* x, double* const* y) {
  World* w = static_cast<World*>(h);
  std::vector<double> res(w->ranks.size(), 0.0);
  on_all_ranks((int)w->ranks.size(), [&](int k) {
    const int n = w->ranks[k]->A.localNumberOfRows;
    Vector xv = wrap(x[k], n), yv = wrap(y[k], n);
    double t = 0.0;
    ComputeDotProduct_ref(n, xv, x[k] == y[k] ? xv : yv, res[k], t);
  });
  return res[0];
}

// CG_ref on every rank with the rank's own b; x[k] has ncol entries, in/out.
int refmpi_cg(void* h, double* const* x, int max_iter, double tol, int do_prec, int* niters, double* normr,
              double* normr0) {
  World* w = static_cast<World*>(h);
  std::vector<int> err(w->ranks.size(), 0), it(w->ranks.size(), 0);
  std::vector<double> nr(w->ranks.size(), 0.0), nr0(w->ranks.size(), 0.0);
  on_all_ranks((int)w->ranks.size(), [&](int k) {
    Rank* p = w->ranks[k];
    Vector xv = wrap(x[k], p->A.localNumberOfColumns);
    std::vector<double> times(10, 0.0);
    err[k] = CG_ref(p->A, p->data, p->b, xv, max_iter, tol, it[k], nr[k], nr0[k], &times[0], do_prec != 0);
  });
  *niters = it[0];
  *normr = nr[0];
  *normr0 = nr0[0];
  int e = 0;
  for (int v : err) e |= v;
  return e;
}

// Renumbers the local rows of every level of one rank: new row q of level l is
// old row new2old[l][q]. Local columns, diagonal pointers, f2c operators, the
// local-to-global map, the rows sent and b/x/xexact follow; external columns
// (>= nrow) keep their numbers, so the halo plan is unchanged.
void refmpi_permute(void* h, int rank, const int* const* new2old) {
  Rank* p = static_cast<World*>(h)->ranks[rank];
  std::vector<std::vector<int> > old2new(kLevels);
  for (int l = 0; l < kLevels; ++l) {
    const SparseMatrix* A = level(p, l);
    old2new[l].resize(A->localNumberOfRows);
    for (int q = 0; q < A->localNumberOfRows; ++q) old2new[l][new2old[l][q]] = q;
  }
  for (int l = 0; l < kLevels; ++l) {
    SparseMatrix* A = level(p, l);
    const int n = A->localNumberOfRows;
    std::vector<char> nz(n);
    std::vector<double*> vals(n), diag(n);
    std::vector<int*> ind(n);
    std::vector<global_int_t*> indg(n);
    std::vector<global_int_t> l2g(n);
    for (int q = 0; q < n; ++q) {
      const int o = new2old[l][q];
      nz[q] = A->nonzerosInRow[o];
      vals[q] = A->matrixValues[o];
      diag[q] = A->matrixDiagonal[o];
      ind[q] = A->mtxIndL[o];
      indg[q] = A->mtxIndG[o];
      l2g[q] = A->localToGlobalMap[o];
    }
    for (int q = 0; q < n; ++q) {
      A->nonzerosInRow[q] = nz[q];
      A->matrixValues[q] = vals[q];
      A->matrixDiagonal[q] = diag[q];
      A->mtxIndL[q] = ind[q];
      A->mtxIndG[q] = indg[q];
      A->localToGlobalMap[q] = l2g[q];
      for (int j = 0; j < nz[q]; ++j)
        if (ind[q][j] < n) ind[q][j] = old2new[l][ind[q][j]];
    }
#ifndef HPCG_NO_MPI
    for (int i = 0; i < A->totalToBeSent; ++i) A->elementsToSend[i] = old2new[l][A->elementsToSend[i]];
#endif
    if (A->mgData) {
      const int nc = A->Ac->localNumberOfRows;
      std::vector<int> f(nc);
      for (int q = 0; q < nc; ++q) f[q] = old2new[l][A->mgData->f2cOperator[new2old[l + 1][q]]];
      std::memcpy(A->mgData->f2cOperator, &f[0], sizeof(int) * nc);
    }
  }
  const int n0 = p->A.localNumberOfRows;
  std::vector<double> tmp(n0);
  Vector* vs[3] = {&p->b, &p->x, &p->xexact};
  for (int v = 0; v < 3; ++v) {
    for (int q = 0; q < n0; ++q) tmp[q] = vs[v]->values[new2old[0][q]];
    std::memcpy(vs[v]->values, &tmp[0], sizeof(double) * n0);
  }
}

}  // extern "C"
