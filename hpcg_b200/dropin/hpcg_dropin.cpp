// Drop-in replacement for the optimisable translation units of HPCG 3.1:
//   src/CG.cpp, src/ComputeSPMV.cpp, src/ComputeSYMGS.cpp, src/ComputeMG.cpp,
//   src/ComputeDotProduct.cpp, src/ComputeWAXPBY.cpp, src/ComputeResidual.cpp,
//   src/OptimizeProblem.cpp.
// Build the reference without those eight files, add this one, and link
// libhpcg_b200.so: the reference's main, V&V tests and report then run on the
// B200 through the C ABI of include/hpcg_b200.h. The signatures are the
// reference's (src/CG.hpp:22-24, ComputeSPMV.hpp:20, ComputeSYMGS.hpp:20,
// ComputeMG.hpp:20, ComputeDotProduct.hpp:18-19, ComputeWAXPBY.hpp:18-19,
// ComputeResidual.hpp:18, OptimizeProblem.hpp:22-28).
//
// Host/device coherence. The reference keeps working on the host arrays
// around these calls: main zeroes x before every CG (src/main.cpp:282, :335)
// and TestCG rewrites the fine diagonal in place (src/TestCG.cpp:79, :114). So
// every call takes its vectors from the host arrays, and the calls that use
// the fine matrix first compare its diagonal with the copy last sent to the
// device and resend it if the host changed it. CG's b and x go through
// hpcg_b200_cg, which sends b only when it changed since its last call and
// zeroes an all-zero x on the device instead of sending it.
//
// MPI builds (HPCG_NO_MPI undefined) with more than one rank: each rank's block
// and halo plan are generated on its GPU (hpcg_b200_generate_rank, the same
// matrix GenerateProblem_ref + SetupHalo_ref built on the host), the ranks are
// joined by a NCCL communicator whose id rank 0 broadcasts with MPI_Bcast, and
// SPMV/SYMGS/MG/CG run as hpcg_b200_shard_* calls; dot products and the residual
// keep the reference's local-result-plus-MPI_Allreduce structure.
#ifndef HPCG_NO_MPI
#include <mpi.h>
#endif
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <vector>

#include "CG.hpp"
#include "CGData.hpp"
#include "ComputeDotProduct.hpp"
#include "ComputeMG.hpp"
#include "ComputeResidual.hpp"
#include "ComputeSPMV.hpp"
#include "ComputeSYMGS.hpp"
#include "ComputeWAXPBY.hpp"
#include "OptimizeProblem.hpp"
#include "SparseMatrix.hpp"
#include "Vector.hpp"
#include "hpcg.hpp"
#include "hpcg_b200.h"
#include "mytimer.hpp"

namespace {

// State the drop-in keeps per optimised matrix, reached through A.optimizationData.
struct DropinState {
  hpcg_b200_problem* problem;
  hpcg_b200_comm* comm;           // ranks of an MPI run (NULL on one rank)
  std::vector<double> diag_sent;  // fine diagonal as last sent to the device
};

DropinState* state_of(const SparseMatrix& A) { return static_cast<DropinState*>(A.optimizationData); }

int device_index() {
  const char* s = std::getenv("HPCG_B200_DEVICE");
  return s ? std::atoi(s) : 0;
}

void log_error(const char* where, int status) {
  HPCG_fout << where << " failed with status " << status << ": " << hpcg_b200_last_error() << std::endl;
}

// Resends the fine diagonal if the host copy changed since the last call.
int sync_diagonal(const SparseMatrix& A, DropinState* st) {
  const local_int_t n = A.localNumberOfRows;
  bool changed = false;
  for (local_int_t i = 0; i < n; ++i) {
    const double d = *A.matrixDiagonal[i];
    if (d != st->diag_sent[i] || std::signbit(d) != std::signbit(st->diag_sent[i])) {
      changed = true;
      break;
    }
  }
  if (!changed) return 0;
  for (local_int_t i = 0; i < n; ++i) st->diag_sent[i] = *A.matrixDiagonal[i];
  return hpcg_b200_set_diagonal(st->problem, &st->diag_sent[0]);
}

}  // namespace

#ifndef HPCG_NO_MPI
// One rank of an MPI run: the rank's hierarchy generated on its GPU, and the
// NCCL communicator of all ranks.
int optimize_rank(SparseMatrix& A, DropinState* st) {
  const Geometry& g = *A.geom;
  if (g.npartz != 1) return HPCG_B200_ERR_UNSUPPORTED;  // equal local blocks only
  int nlevels = 0;
  for (const SparseMatrix* m = &A; m; m = m->Ac) ++nlevels;
  int device = device_index();
  if (!std::getenv("HPCG_B200_DEVICE")) {  // one rank per GPU: the launcher's node-local rank
    const char* local = std::getenv("OMPI_COMM_WORLD_LOCAL_RANK");
    if (!local) local = std::getenv("MPI_LOCALRANKID");
    if (!local) local = std::getenv("SLURM_LOCALID");
    device = local ? std::atoi(local) : 0;
  }
  int s = hpcg_b200_generate_rank(g.nx, g.ny, g.nz, g.npx, g.npy, g.npz, g.rank, nlevels, device, &st->problem);
  if (s) return s;
  unsigned char id[HPCG_B200_COMM_ID_BYTES];
  std::memset(id, 0, sizeof(id));
  if (g.rank == 0) s = hpcg_b200_comm_unique_id(id);
  MPI_Bcast(&s, 1, MPI_INT, 0, MPI_COMM_WORLD);
  if (s) return s;
  MPI_Bcast(id, (int)sizeof(id), MPI_CHAR, 0, MPI_COMM_WORLD);
  return hpcg_b200_comm_nccl(id, g.size, g.rank, st->problem, &st->comm);
}
#endif

int OptimizeProblem(SparseMatrix& A, CGData& data, Vector& b, Vector& x, Vector& xexact) {
  (void)data; (void)b; (void)x; (void)xexact;
#ifndef HPCG_NO_MPI
  if (A.geom->size > 1) {
    DropinState* st = new DropinState;
    st->problem = 0;
    st->comm = 0;
    const int status = optimize_rank(A, st);
    if (status) {
      log_error("OptimizeProblem", status);
      if (st->problem) hpcg_b200_free(st->problem);
      delete st;
      return status;
    }
    st->diag_sent.resize(A.localNumberOfRows);
    for (local_int_t i = 0; i < A.localNumberOfRows; ++i) st->diag_sent[i] = *A.matrixDiagonal[i];
    A.optimizationData = st;
    return 0;
  }
#endif
  std::vector<hpcg_b200_level_desc> levels;
  for (const SparseMatrix* m = &A; m; m = m->Ac) {
    hpcg_b200_level_desc d;
    d.nx = m->geom->nx;
    d.ny = m->geom->ny;
    d.nz = m->geom->nz;
    d.nrow = m->localNumberOfRows;
    d.ncol = m->localNumberOfColumns;
    d.nonzeros_in_row = m->nonzerosInRow;
    d.mtx_ind_l = m->mtxIndL;
    d.matrix_values = m->matrixValues;
    d.f2c = m->mgData ? m->mgData->f2cOperator : 0;
    levels.push_back(d);
  }
  DropinState* st = new DropinState;
  st->comm = 0;
  const int status = hpcg_b200_optimize(&levels[0], (int)levels.size(), device_index(), &st->problem);
  if (status) {
    log_error("OptimizeProblem", status);
    delete st;
    return status;
  }
  st->diag_sent.resize(A.localNumberOfRows);
  for (local_int_t i = 0; i < A.localNumberOfRows; ++i) st->diag_sent[i] = *A.matrixDiagonal[i];
  A.optimizationData = st;
  return 0;
}

double OptimizeProblemMemoryUse(const SparseMatrix& A) {
  const DropinState* st = state_of(A);
  return st ? hpcg_b200_memory_use(st->problem) : 0.0;
}

int ComputeSPMV(const SparseMatrix& A, Vector& x, Vector& y) {
  DropinState* st = state_of(A);
  if (!st) return HPCG_B200_ERR_HANDLE;
  int s = sync_diagonal(A, st);
  if (!s) s = st->comm ? hpcg_b200_shard_spmv(st->comm, &x.values, &y.values)
                       : hpcg_b200_spmv(st->problem, x.values, y.values);
  if (s) log_error("ComputeSPMV", s);
  return s;
}

int ComputeSYMGS(const SparseMatrix& A, const Vector& r, Vector& x) {
  DropinState* st = state_of(A);
  if (!st) return HPCG_B200_ERR_HANDLE;
  int s = sync_diagonal(A, st);
  if (!s) s = st->comm ? hpcg_b200_shard_symgs(st->comm, &r.values, &x.values)
                       : hpcg_b200_symgs(st->problem, r.values, x.values);
  if (s) log_error("ComputeSYMGS", s);
  return s;
}

int ComputeMG(const SparseMatrix& A, const Vector& r, Vector& x) {
  DropinState* st = state_of(A);
  if (!st) return HPCG_B200_ERR_HANDLE;
  int s = sync_diagonal(A, st);
  if (!s) s = st->comm ? hpcg_b200_shard_mg(st->comm, &r.values, &x.values)
                       : hpcg_b200_mg(st->problem, r.values, x.values);
  if (s) log_error("ComputeMG", s);
  return s;
}

int ComputeDotProduct(const local_int_t n, const Vector& x, const Vector& y, double& result,
                      double& time_allreduce, bool& isOptimized) {
  (void)isOptimized;  // left true: this is the optimised version
  double local = 0.0;
  const int s = hpcg_b200_dot(n, x.values, y.values, &local);
  if (s) log_error("ComputeDotProduct", s);
#ifndef HPCG_NO_MPI
  const double t0 = MPI_Wtime();  // ComputeDotProduct_ref.cpp:66-73
  double global = 0.0;
  MPI_Allreduce(&local, &global, 1, MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD);
  result = global;
  time_allreduce += MPI_Wtime() - t0;
#else
  time_allreduce += 0.0;  // one process: no allreduce
  result = local;
#endif
  return s;
}

int ComputeWAXPBY(const local_int_t n, const double alpha, const Vector& x, const double beta, const Vector& y,
                  Vector& w, bool& isOptimized) {
  (void)isOptimized;
  const int s = hpcg_b200_waxpby(n, alpha, x.values, beta, y.values, w.values);
  if (s) log_error("ComputeWAXPBY", s);
  return s;
}

int ComputeResidual(const local_int_t n, const Vector& v1, const Vector& v2, double& residual) {
  double local = 0.0;
  const int s = hpcg_b200_residual(n, v1.values, v2.values, &local);
  if (s) log_error("ComputeResidual", s);
#ifndef HPCG_NO_MPI
  MPI_Allreduce(&local, &residual, 1, MPI_DOUBLE, MPI_MAX, MPI_COMM_WORLD);  // ComputeResidual.cpp:79-83
#else
  residual = local;
#endif
  return s;
}

int CG(const SparseMatrix& A, CGData& data, const Vector& b, Vector& x, const int max_iter,
       const double tolerance, int& niters, double& normr, double& normr0, double* times,
       bool doPreconditioning) {
  (void)data;  // the iteration vectors live on the device
  // times[0] covers the whole call, as src/CG.cpp:63 and :140 measure it (the
  // vectors' way to and from the device included); the library files the
  // parts' device times into times[1..5]
  const double t_begin = mytimer();
  DropinState* st = state_of(A);
  if (!st) return HPCG_B200_ERR_HANDLE;
  if (!doPreconditioning && A.geom->rank == 0)
    HPCG_fout << "WARNING: PERFORMING UNPRECONDITIONED ITERATIONS" << std::endl;  // as src/CG.cpp:75
  double parts[6] = {0, 0, 0, 0, 0, 0};
  int s = sync_diagonal(A, st);
  if (!s && st->comm)
    s = hpcg_b200_shard_cg(st->comm, &b.values, &x.values, max_iter, tolerance, doPreconditioning ? 1 : 0,
                           &niters, &normr, &normr0, times ? parts : 0);
  else if (!s)
    s = hpcg_b200_cg(st->problem, b.values, x.values, max_iter, tolerance, doPreconditioning ? 1 : 0, &niters,
                     &normr, &normr0, times ? parts : 0);
  if (s) log_error("CG", s);
  if (times) {
    for (int i = 1; i < 6; ++i) times[i] += parts[i];
    times[0] += mytimer() - t_begin;
  }
  return s;
}
