// C entry points over the HPCG 3.1 reference routines, compiled together with
// the reference's own sources (every src/*.cpp except main.cpp) into
// oracle/_ref/libhpcg_ref.so by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY: the tests use it to pin the C oracle against the
// reference itself and to produce golden vectors. Nothing in the product links it.
//
// The problem is set up exactly as src/main.cpp:121-163 does for one process:
// GenerateGeometry, GenerateProblem, SetupHalo, 3x GenerateCoarseProblem,
// InitializeSparseCGData.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "CG.hpp"
#include "CGData.hpp"
#include "CG_ref.hpp"
#include "ComputeDotProduct_ref.hpp"
#include "ComputeMG_ref.hpp"
#include "ComputeResidual.hpp"
#include "ComputeSPMV_ref.hpp"
#include "ComputeSYMGS_ref.hpp"
#include "ComputeWAXPBY_ref.hpp"
#include "GenerateCoarseProblem.hpp"
#include "GenerateGeometry.hpp"
#include "GenerateProblem.hpp"
#include "Geometry.hpp"
#include "SetupHalo.hpp"
#include "SparseMatrix.hpp"
#include "TestCG.hpp"
#include "TestSymmetry.hpp"
#include "Vector.hpp"
#include "hpcg.hpp"

namespace {

const int kLevels = 4;  // main.cpp:139

struct RefProblem {
  SparseMatrix A;
  Vector b, x, xexact;
  CGData data;
};

SparseMatrix* level(RefProblem* p, int lev) {
  SparseMatrix* m = &p->A;
  for (int i = 0; i < lev && m; ++i) m = m->Ac;
  return m;
}

// A Vector header over caller memory (no allocation, never deleted).
Vector wrap(const double* v, int n) {
  Vector w;
  w.localLength = n;
  w.values = const_cast<double*>(v);
  w.optimizationData = 0;
  return w;
}

}  // namespace

extern "C" {

void* ref_create(int nx, int ny, int nz) {
  RefProblem* p = new RefProblem;
  Geometry* geom = new Geometry;
  GenerateGeometry(1, 0, 1, 0, 0, 0, nx, ny, nz, 1, 1, 1, geom);
  InitializeSparseMatrix(p->A, geom);
  GenerateProblem(p->A, &p->b, &p->x, &p->xexact);
  SetupHalo(p->A);
  SparseMatrix* cur = &p->A;
  for (int l = 1; l < kLevels; ++l) {
    GenerateCoarseProblem(*cur);
    cur = cur->Ac;
  }
  InitializeSparseCGData(p->A, p->data);
  return p;
}

void ref_destroy(void* h) {
  RefProblem* p = static_cast<RefProblem*>(h);
  DeleteMatrix(p->A);
  DeleteCGData(p->data);
  DeleteVector(p->x);
  DeleteVector(p->b);
  DeleteVector(p->xexact);
  delete p;
}

int ref_levels(void*) { return kLevels; }

int ref_level_rows(void* h, int lev) { return level(static_cast<RefProblem*>(h), lev)->localNumberOfRows; }

long long ref_level_nnz(void* h, int lev) {
  return level(static_cast<RefProblem*>(h), lev)->totalNumberOfNonzeros;
}

// Copies one level out in the oracle's layout (27 slots per row, entry order kept).
void ref_export_level(void* h, int lev, int* nnz, int* cols, double* vals, int* diag, int* f2c) {
  const SparseMatrix* A = level(static_cast<RefProblem*>(h), lev);
  for (int i = 0; i < A->localNumberOfRows; ++i) {
    const int k = A->nonzerosInRow[i];
    nnz[i] = k;
    diag[i] = static_cast<int>(A->matrixDiagonal[i] - A->matrixValues[i]);
    for (int j = 0; j < 27; ++j) {
      cols[(long long)i * 27 + j] = j < k ? A->mtxIndL[i][j] : i;
      vals[(long long)i * 27 + j] = j < k ? A->matrixValues[i][j] : 0.0;
    }
  }
  if (f2c && A->mgData)
    std::memcpy(f2c, A->mgData->f2cOperator, sizeof(int) * A->Ac->localNumberOfRows);
}

void ref_get_vectors(void* h, double* b, double* x, double* xexact) {
  RefProblem* p = static_cast<RefProblem*>(h);
  const size_t n = p->A.localNumberOfRows;
  if (b) std::memcpy(b, p->b.values, n * sizeof(double));
  if (x) std::memcpy(x, p->x.values, n * sizeof(double));
  if (xexact) std::memcpy(xexact, p->xexact.values, n * sizeof(double));
}

void ref_set_b(void* h, const double* b) {
  RefProblem* p = static_cast<RefProblem*>(h);
  std::memcpy(p->b.values, b, sizeof(double) * p->A.localNumberOfRows);
}

// Overwrites the matrix values of one level (same sparsity); values laid out as in ref_export_level.
void ref_set_values(void* h, int lev, const double* vals) {
  SparseMatrix* A = level(static_cast<RefProblem*>(h), lev);
  for (int i = 0; i < A->localNumberOfRows; ++i)
    for (int j = 0; j < A->nonzerosInRow[i]; ++j) A->matrixValues[i][j] = vals[(long long)i * 27 + j];
}

int ref_spmv(void* h, int lev, const double* x, double* y) {
  SparseMatrix* A = level(static_cast<RefProblem*>(h), lev);
  Vector xv = wrap(x, A->localNumberOfColumns), yv = wrap(y, A->localNumberOfRows);
  return ComputeSPMV_ref(*A, xv, yv);
}

int ref_symgs(void* h, int lev, const double* r, double* x) {
  SparseMatrix* A = level(static_cast<RefProblem*>(h), lev);
  Vector rv = wrap(r, A->localNumberOfRows), xv = wrap(x, A->localNumberOfColumns);
  return ComputeSYMGS_ref(*A, rv, xv);
}

int ref_mg(void* h, int lev, const double* r, double* x) {
  SparseMatrix* A = level(static_cast<RefProblem*>(h), lev);
  Vector rv = wrap(r, A->localNumberOfRows), xv = wrap(x, A->localNumberOfColumns);
  return ComputeMG_ref(*A, rv, xv);
}

double ref_dot(int n, const double* x, const double* y) {
  Vector xv = wrap(x, n), yv = wrap(y, n);
  double res = 0.0, t = 0.0;
  ComputeDotProduct_ref(n, xv, x == y ? xv : yv, res, t);
  return res;
}

void ref_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w) {
  Vector xv = wrap(x, n), yv = wrap(y, n), wv = wrap(w, n);
  ComputeWAXPBY_ref(n, alpha, xv, beta, yv, wv);
}

double ref_residual(int n, const double* v1, const double* v2) {
  Vector a = wrap(v1, n), b = wrap(v2, n);
  double res = 0.0;
  ComputeResidual(n, a, b, res);
  return res;
}

// CG_ref on the problem's own b; x is in/out (length nrow).
int ref_cg(void* h, double* x, int max_iter, double tol, int do_prec, int* niters, double* normr,
           double* normr0) {
  RefProblem* p = static_cast<RefProblem*>(h);
  Vector xv = wrap(x, p->A.localNumberOfColumns);
  std::vector<double> times(10, 0.0);
  *niters = 0;
  return CG_ref(p->A, p->data, p->b, xv, max_iter, tol, *niters, *normr, *normr0, &times[0], do_prec != 0);
}

// Renumbers every level: new row q of level l is old row new2old[l][q]. Column
// indices, diagonal pointers, f2c operators and the local-to-global map follow,
// so the permuted hierarchy is the same operator in the new order.
void ref_permute(void* h, const int* const* new2old) {
  RefProblem* p = static_cast<RefProblem*>(h);
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
    std::vector<global_int_t> l2g(n);
    for (int q = 0; q < n; ++q) {
      const int o = new2old[l][q];
      nz[q] = A->nonzerosInRow[o];
      vals[q] = A->matrixValues[o];
      diag[q] = A->matrixDiagonal[o];
      ind[q] = A->mtxIndL[o];
      l2g[q] = A->localToGlobalMap[o];
    }
    for (int q = 0; q < n; ++q) {
      A->nonzerosInRow[q] = nz[q];
      A->matrixValues[q] = vals[q];
      A->matrixDiagonal[q] = diag[q];
      A->mtxIndL[q] = ind[q];
      A->localToGlobalMap[q] = l2g[q];
      for (int j = 0; j < nz[q]; ++j) ind[q][j] = old2new[l][ind[q][j]];
    }
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

// TestCG.cpp:52-123 through the reference's CG (src/CG.cpp) and its stubs.
void ref_test_cg(void* h, int* count_pass, int* count_fail, int* niters_no_prec, int* niters_prec) {
  RefProblem* p = static_cast<RefProblem*>(h);
  TestCGData d;
  d.count_pass = d.count_fail = 0;
  TestCG(p->A, p->data, p->b, p->x, d);
  *count_pass = d.count_pass;
  *count_fail = d.count_fail;
  *niters_no_prec = d.niters_max_no_prec;
  *niters_prec = d.niters_max_prec;
}

// TestSymmetry.cpp:60-138 (uses rand(); call srand first for a fixed stream).
void ref_test_symmetry(void* h, unsigned seed, double* depsym_spmv, double* depsym_mg, int* count_fail) {
  RefProblem* p = static_cast<RefProblem*>(h);
  std::srand(seed);
  TestSymmetryData d;
  TestSymmetry(p->A, p->b, p->xexact, d);
  *depsym_spmv = d.depsym_spmv;
  *depsym_mg = d.depsym_mg;
  *count_fail = d.count_fail;
}

}  // extern "C"
