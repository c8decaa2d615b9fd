// Times the reference's own CPU implementation of the PCG path: CG_ref over the
// problem that src/main.cpp:121-163 sets up, built from the reference's sources
// with the reference's OpenMP flags (setup/Make.GCC_OMP:121) by oracle/Makefile.
//
// Usage: hpcg_ref_timer NX NY NZ ITERS REPS [WARMUP]
// Runs WARMUP untimed calls, then REPS timed calls of CG_ref(ITERS iterations,
// tolerance 0). Prints one JSON line: per-call seconds and the HPCG model flop
// count of one call (ReportResults.cpp:81-97 with one set of ITERS iterations).
//
// TEST/BASELINE INFRASTRUCTURE ONLY: used as the CPU baseline, never shipped.
#include <cstdio>
#include <cstdlib>
#include <vector>
#ifndef HPCG_NO_OPENMP
#include <omp.h>
#endif

#include "CGData.hpp"
#include "CG_ref.hpp"
#include "GenerateCoarseProblem.hpp"
#include "GenerateGeometry.hpp"
#include "GenerateProblem.hpp"
#include "SetupHalo.hpp"
#include "SparseMatrix.hpp"
#include "Vector.hpp"
#include "hpcg.hpp"
#include "mytimer.hpp"

int main(int argc, char** argv) {
  if (argc != 6 && argc != 7) {
    std::fprintf(stderr, "usage: %s NX NY NZ ITERS REPS [WARMUP]\n", argv[0]);
    return 2;
  }
  const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), nz = std::atoi(argv[3]);
  const int iters = std::atoi(argv[4]), reps = std::atoi(argv[5]);
  const int warmup = argc == 7 ? std::atoi(argv[6]) : 0;
  int threads = 1;
#ifndef HPCG_NO_OPENMP
  threads = omp_get_max_threads();
#endif
  Geometry* geom = new Geometry;
  GenerateGeometry(1, 0, threads, 0, 0, 0, nx, ny, nz, 1, 1, 1, geom);
  SparseMatrix A;
  InitializeSparseMatrix(A, geom);
  Vector b, x, xexact;
  double t_setup = mytimer();
  GenerateProblem(A, &b, &x, &xexact);
  SetupHalo(A);
  SparseMatrix* cur = &A;
  for (int l = 1; l < 4; ++l) {
    GenerateCoarseProblem(*cur);
    cur = cur->Ac;
  }
  t_setup = mytimer() - t_setup;
  CGData data;
  InitializeSparseCGData(A, data);

  double flops = 0.0;
  {
    const double it = iters, nrow = (double)A.totalNumberOfRows, nnz = (double)A.totalNumberOfNonzeros;
    flops += (3.0 * it + 1.0) * 2.0 * nrow * 2.0;  // ddot + waxpby
    flops += (it + 1.0) * 2.0 * nnz;                // spmv
    const SparseMatrix* Af = &A;
    for (int l = 1; l < 4; ++l) {
      flops += it * 10.0 * (double)Af->totalNumberOfNonzeros;  // pre + residual + post
      Af = Af->Ac;
    }
    flops += it * 4.0 * (double)Af->totalNumberOfNonzeros;  // coarsest SYMGS
  }

  std::vector<double> times(10, 0.0);
  std::vector<double> per_call;
  int niters = 0;
  double normr = 0.0, normr0 = 0.0;
  for (int r = 0; r < warmup + reps; ++r) {
    ZeroVector(x);
    const double t0 = mytimer();
    CG_ref(A, data, b, x, iters, 0.0, niters, normr, normr0, &times[0], true);
    if (r >= warmup) per_call.push_back(mytimer() - t0);
  }
  double best = per_call.empty() ? 0.0 : per_call[0], sum = 0.0;
  for (size_t i = 0; i < per_call.size(); ++i) {
    sum += per_call[i];
    if (per_call[i] < best) best = per_call[i];
  }
  std::printf(
      "{\"nx\": %d, \"ny\": %d, \"nz\": %d, \"iters\": %d, \"reps\": %d, \"threads\": %d, "
      "\"setup_s\": %.6f, \"mean_s\": %.6f, \"best_s\": %.6f, \"flops_per_call\": %.6e, "
      "\"normr_over_normr0\": %.6e, \"niters\": %d}\n",
      nx, ny, nz, iters, reps, threads, t_setup, per_call.empty() ? 0.0 : sum / per_call.size(), best, flops,
      normr0 > 0 ? normr / normr0 : 0.0, niters);
  DeleteMatrix(A);
  DeleteCGData(data);
  DeleteVector(x);
  DeleteVector(b);
  DeleteVector(xexact);
  return 0;
}
