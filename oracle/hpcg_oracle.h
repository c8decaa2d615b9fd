/*
 * CPU oracle for the HPCG 3.1 preconditioned-CG path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product library links or calls this
 * code; only the test-suite, the smoke check and the CPU-baseline leg of the
 * benchmark load it, and only to compare results against.
 *
 * It restates, in plain C99 with strict IEEE-754 double arithmetic (built with
 * -ffp-contract=off, no fast-math), the reference routines of HPCG 3.1:
 *   problem generation   src/GenerateProblem_ref.cpp:131-183
 *   coarse f2c operator  src/GenerateCoarseProblem.cpp:71-82
 *   SpMV                 src/ComputeSPMV_ref.cpp:61-70
 *   symmetric GS         src/ComputeSYMGS_ref.cpp:67-100
 *   V-cycle              src/ComputeMG_ref.cpp:39-63
 *   restriction          src/ComputeRestriction_ref.cpp:51
 *   prolongation         src/ComputeProlongation_ref.cpp:49
 *   dot product          src/ComputeDotProduct_ref.cpp:54-64
 *   WAXPBY               src/ComputeWAXPBY_ref.cpp:52-67
 *   inf-norm residual    src/ComputeResidual.cpp:70-75
 *   PCG                  src/CG_ref.cpp:58-144
 * plus the changed forms the GPU library adds (an FP32 V-cycle inside a
 * flexible FP64 PCG, and the implicit adjoint of the solve), each restated on
 * top of the same reference routines.
 *
 * The matrix of one level is stored row-major with up to 27 entries per row, in
 * the reference's entry order (lexicographic in (sz, sy, sx), so lower entries
 * precede the diagonal): cols[i*27 + j], vals[i*27 + j] for j < nnz[i], and
 * diag[i] is the slot of the diagonal inside row i.
 *
 * Parity pin: this restatement is checked against the reference itself, built
 * from its own sources into oracle/_ref/ (see oracle/Makefile), and against the
 * committed golden vectors in tests/golden/.
 */
#ifndef HPCG_ORACLE_H
#define HPCG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORA_SLOTS 27

typedef struct ora_level {
  int nx, ny, nz;       /* grid of this level */
  int n;                /* rows (= columns, single process) */
  const int* nnz;       /* entries per row */
  const int* cols;      /* n*27, column of entry j of row i at i*27+j */
  const double* vals;   /* n*27 */
  const int* diag;      /* slot of the diagonal entry in each row */
  const int* f2c;       /* fine row injected into coarse row q (length n of the next level), NULL on the coarsest */
} ora_level;

/* GenerateProblem_ref.cpp:131-183 for one process (gix0 = giy0 = giz0 = 0).
 * b, x, xexact may be NULL. Returns the number of nonzeros. */
int64_t ora_generate(int nx, int ny, int nz, int* nnz, int* cols, double* vals, int* diag,
                     double* b, double* x, double* xexact);

/* GenerateCoarseProblem.cpp:71-82: f2c[coarse row] = fine row at (2ix, 2iy, 2iz). */
void ora_f2c(int nxf, int nyf, int nzf, int* f2c);

/* ComputeSPMV_ref.cpp:61-70 */
void ora_spmv(const ora_level* A, const double* x, double* y);
/* ComputeSYMGS_ref.cpp:67-100 (forward then backward sweep, in place on x) */
void ora_symgs(const ora_level* A, const double* r, double* x);
/* forward sweep only / backward sweep only (the two halves of the above) */
void ora_gs_forward(const ora_level* A, const double* r, double* x);
void ora_gs_backward(const ora_level* A, const double* r, double* x);
/* ComputeSYMGS_ref.cpp:67-100 with the backward update of the last `skip` rows
 * left out. The library sweeps colour blocks in row order and does not repeat
 * the last block at the turn of the sweep (its other-colour inputs are
 * unchanged); with the reference's subtract-then-add-back diagonal term the
 * repeat would differ from the forward value only by rounding. skip = 0 is
 * ComputeSYMGS_ref itself. */
void ora_symgs_skip(const ora_level* A, const double* r, double* x, int skip);
/* ComputeMG_ref.cpp:39-63 with ora_symgs_skip(skip[l]) on level l. */
int ora_mg_skip(const ora_level* levels, int nlev, int lev, const double* r, double* x, const int* skip);
/* CG_ref.cpp:58-144 with that V-cycle (skip may be NULL: the reference's). */
int ora_cg_skip(const ora_level* levels, int nlev, const double* b, double* x, int max_iter, double tolerance,
                int do_prec, int* niters, double* normr, double* normr0, double* hist, const int* skip);

/* ComputeRestriction_ref.cpp:51 */
void ora_restriction(int nc, const int* f2c, const double* rf, const double* Axf, double* rc);
/* ComputeProlongation_ref.cpp:49 */
void ora_prolongation(int nc, const int* f2c, const double* xc, double* xf);
/* ComputeMG_ref.cpp:39-63 applied at level `lev` of `levels` (nlev levels in all). */
int ora_mg(const ora_level* levels, int nlev, int lev, const double* r, double* x);
/* ComputeDotProduct_ref.cpp:54-64 (serial left-to-right sum) */
double ora_dot(int n, const double* x, const double* y);
/* ComputeWAXPBY_ref.cpp:52-67 */
void ora_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w);
/* ComputeResidual.cpp:70-75 (max |v1 - v2|) */
double ora_residual(int n, const double* v1, const double* v2);

/* CG_ref.cpp:58-144. hist (optional, length max_iter+1) receives normr after
 * the preamble (hist[0]) and after every iteration k (hist[k]). */
int ora_cg(const ora_level* levels, int nlev, const double* b, double* x, int max_iter, double tolerance,
           int do_prec, int* niters, double* normr, double* normr0, double* hist);

/* Reorders a level: new row p is old row new2old[p]; columns are relabelled with
 * old2new; the entry order inside each row is kept. f2c of the permuted level is
 * written separately with ora_permute_f2c. Output arrays have the input's sizes. */
void ora_permute_level(int n, const int* new2old, const int* old2new, const int* nnz, const int* cols,
                       const double* vals, const int* diag, int* pnnz, int* pcols, double* pvals, int* pdiag);
/* pf2c[q] = fine_old2new[f2c[coarse_new2old[q]]] */
void ora_permute_f2c(int nc, const int* f2c, const int* coarse_new2old, const int* fine_old2new, int* pf2c);

/* ---- FP32 V-cycle form: the same V-cycle with every value, vector and
 *      operation in binary32 (ComputeMG_ref.cpp:39-63 on float data). ---- */
typedef struct ora_level_f32 {
  int n;
  const int* nnz;
  const int* cols;
  const float* vals;
  const int* diag;
  const int* f2c;
} ora_level_f32;
int ora_mg_f32(const ora_level_f32* levels, int nlev, int lev, const float* r, float* x);
/* The same with the last `skip[lev]` rows of each level's forward sweep not repeated
 * at the start of its backward sweep (the B200 colour order's last colour). */
int ora_mg_f32_skip(const ora_level_f32* levels, int nlev, int lev, const float* r, float* x, const int* skip);

/* Flexible PCG (Polak-Ribiere beta = r'(z - z_prev)/oldrtz) in FP64 with the
 * FP32 V-cycle as preconditioner: r is converted to float, the V-cycle runs in
 * float, z is widened back. The outer SpMV, dots, alpha/beta and x, r updates
 * are FP64 on the FP64 matrix `levels[0]`. Stops at normr/normr0 <= tolerance. */
int ora_cg_mixed(const ora_level* levels, const ora_level_f32* levels32, int nlev, const double* b,
                 double* x, int max_iter, double tolerance, int* niters, double* normr, double* normr0,
                 double* hist);
/* The same around the FP32 V-cycle of ora_mg_f32_skip (skip: per-level rows not
 * repeated at the turn of each sweep, NULL for the reference's sweep). */
int ora_cg_mixed_skip(const ora_level* levels, const ora_level_f32* levels32, int nlev, const double* b,
                      double* x, int max_iter, double tolerance, int* niters, double* normr, double* normr0,
                      double* hist, const int* skip);

#ifdef __cplusplus
}
#endif
#endif
