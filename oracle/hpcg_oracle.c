/*
 * CPU oracle for the HPCG 3.1 PCG path -- TEST INFRASTRUCTURE ONLY (see
 * hpcg_oracle.h). Strict IEEE double arithmetic: build with -ffp-contract=off
 * and without -ffast-math so every expression rounds exactly as written.
 */
#include "hpcg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* GenerateProblem_ref.cpp:131-183: the 27-point stencil over the (nx, ny, nz)
 * box, entries visited in (sz, sy, sx) order, 26 on the diagonal and -1 off it;
 * b_i = 26 - (nnz_i - 1) (:178), x = 0 (:179), xexact = 1 (:180). */
int64_t ora_generate(int nx, int ny, int nz, int* nnz, int* cols, double* vals, int* diag, double* b,
                     double* x, double* xexact) {
  int64_t total = 0;
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        const int row = (iz * ny + iy) * nx + ix;
        int k = 0;
        for (int sz = -1; sz <= 1; ++sz) {
          if (iz + sz < 0 || iz + sz >= nz) continue;
          for (int sy = -1; sy <= 1; ++sy) {
            if (iy + sy < 0 || iy + sy >= ny) continue;
            for (int sx = -1; sx <= 1; ++sx) {
              if (ix + sx < 0 || ix + sx >= nx) continue;
              const int col = row + (sz * ny + sy) * nx + sx;
              cols[(int64_t)row * ORA_SLOTS + k] = col;
              if (col == row) {
                vals[(int64_t)row * ORA_SLOTS + k] = 26.0;
                diag[row] = k;
              } else {
                vals[(int64_t)row * ORA_SLOTS + k] = -1.0;
              }
              ++k;
            }
          }
        }
        for (int j = k; j < ORA_SLOTS; ++j) {  /* unused tail: keep it defined */
          cols[(int64_t)row * ORA_SLOTS + j] = row;
          vals[(int64_t)row * ORA_SLOTS + j] = 0.0;
        }
        nnz[row] = k;
        total += k;
        if (b) b[row] = 26.0 - (double)(k - 1);
        if (x) x[row] = 0.0;
        if (xexact) xexact[row] = 1.0;
      }
  return total;
}

/* GenerateCoarseProblem.cpp:71-82 */
void ora_f2c(int nxf, int nyf, int nzf, int* f2c) {
  const int nxc = nxf / 2, nyc = nyf / 2, nzc = nzf / 2;
  for (int izc = 0; izc < nzc; ++izc)
    for (int iyc = 0; iyc < nyc; ++iyc)
      for (int ixc = 0; ixc < nxc; ++ixc)
        f2c[(izc * nyc + iyc) * nxc + ixc] = ((2 * izc) * nyf + 2 * iyc) * nxf + 2 * ixc;
}

/* ComputeSPMV_ref.cpp:61-70: left-to-right sum over the row's entries. */
void ora_spmv(const ora_level* A, const double* x, double* y) {
  for (int i = 0; i < A->n; ++i) {
    const int* c = A->cols + (int64_t)i * ORA_SLOTS;
    const double* v = A->vals + (int64_t)i * ORA_SLOTS;
    double s = 0.0;
    for (int j = 0; j < A->nnz[i]; ++j) s += v[j] * x[c[j]];
    y[i] = s;
  }
}

/* One Gauss-Seidel row update as ComputeSYMGS_ref.cpp:72-80 writes it: the
 * diagonal term is subtracted with the others and added back afterwards. */
static inline double gs_row(const ora_level* A, int i, const double* r, const double* x) {
  const int* c = A->cols + (int64_t)i * ORA_SLOTS;
  const double* v = A->vals + (int64_t)i * ORA_SLOTS;
  const double d = v[A->diag[i]];
  double s = r[i];
  for (int j = 0; j < A->nnz[i]; ++j) s -= v[j] * x[c[j]];
  s += x[i] * d;
  return s / d;
}

void ora_gs_forward(const ora_level* A, const double* r, double* x) {
  for (int i = 0; i < A->n; ++i) x[i] = gs_row(A, i, r, x);  /* ComputeSYMGS_ref.cpp:67-82 */
}

void ora_gs_backward(const ora_level* A, const double* r, double* x) {
  for (int i = A->n - 1; i >= 0; --i) x[i] = gs_row(A, i, r, x);  /* ComputeSYMGS_ref.cpp:86-100 */
}

void ora_symgs(const ora_level* A, const double* r, double* x) {
  ora_gs_forward(A, r, x);
  ora_gs_backward(A, r, x);
}

void ora_symgs_skip(const ora_level* A, const double* r, double* x, int skip) {
  ora_gs_forward(A, r, x);
  for (int i = A->n - 1 - skip; i >= 0; --i) x[i] = gs_row(A, i, r, x);
}

void ora_restriction(int nc, const int* f2c, const double* rf, const double* Axf, double* rc) {
  for (int i = 0; i < nc; ++i) rc[i] = rf[f2c[i]] - Axf[f2c[i]];
}

void ora_prolongation(int nc, const int* f2c, const double* xc, double* xf) {
  for (int i = 0; i < nc; ++i) xf[f2c[i]] += xc[i];
}

/* ComputeMG_ref.cpp:39-63: x = 0; one pre-smoothing SYMGS; Axf = A x;
 * restrict; recurse on the coarse level; prolong; one post-smoothing SYMGS.
 * The coarsest level does a single SYMGS. */
int ora_mg(const ora_level* L, int nlev, int lev, const double* r, double* x) {
  return ora_mg_skip(L, nlev, lev, r, x, NULL);
}

int ora_mg_skip(const ora_level* L, int nlev, int lev, const double* r, double* x, const int* skip) {
  const ora_level* A = &L[lev];
  const int sk = skip ? skip[lev] : 0;
  memset(x, 0, sizeof(double) * (size_t)A->n);
  if (lev + 1 < nlev) {
    const int nc = L[lev + 1].n;
    double* Axf = (double*)malloc(sizeof(double) * (size_t)A->n);
    double* rc = (double*)malloc(sizeof(double) * (size_t)nc);
    double* xc = (double*)malloc(sizeof(double) * (size_t)nc);
    if (!Axf || !rc || !xc) { free(Axf); free(rc); free(xc); return 1; }
    ora_symgs_skip(A, r, x, sk);
    ora_spmv(A, x, Axf);
    ora_restriction(nc, A->f2c, r, Axf, rc);
    int err = ora_mg_skip(L, nlev, lev + 1, rc, xc, skip);
    if (!err) {
      ora_prolongation(nc, A->f2c, xc, x);
      ora_symgs_skip(A, r, x, sk);
    }
    free(Axf); free(rc); free(xc);
    return err;
  }
  ora_symgs_skip(A, r, x, sk);
  return 0;
}

double ora_dot(int n, const double* x, const double* y) {
  double s = 0.0;
  if (x == y) {
    for (int i = 0; i < n; ++i) s += x[i] * x[i];
  } else {
    for (int i = 0; i < n; ++i) s += x[i] * y[i];
  }
  return s;
}

/* ComputeWAXPBY_ref.cpp:52-67 including its alpha == 1 and beta == 1 branches. */
void ora_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w) {
  if (alpha == 1.0) {
    for (int i = 0; i < n; ++i) w[i] = x[i] + beta * y[i];
  } else if (beta == 1.0) {
    for (int i = 0; i < n; ++i) w[i] = alpha * x[i] + y[i];
  } else {
    for (int i = 0; i < n; ++i) w[i] = alpha * x[i] + beta * y[i];
  }
}

double ora_residual(int n, const double* v1, const double* v2) {
  double m = 0.0;
  for (int i = 0; i < n; ++i) {
    const double d = fabs(v1[i] - v2[i]);
    if (d > m) m = d;
  }
  return m;
}

/* CG_ref.cpp:58-144 */
int ora_cg(const ora_level* L, int nlev, const double* b, double* x, int max_iter, double tolerance,
           int do_prec, int* niters, double* normr_out, double* normr0_out, double* hist) {
  return ora_cg_skip(L, nlev, b, x, max_iter, tolerance, do_prec, niters, normr_out, normr0_out, hist, NULL);
}

int ora_cg_skip(const ora_level* L, int nlev, const double* b, double* x, int max_iter, double tolerance,
                int do_prec, int* niters, double* normr_out, double* normr0_out, double* hist, const int* skip) {
  const ora_level* A = &L[0];
  const int n = A->n;
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* z = (double*)malloc(sizeof(double) * (size_t)n);
  double* p = (double*)malloc(sizeof(double) * (size_t)n);
  double* Ap = (double*)malloc(sizeof(double) * (size_t)n);
  if (!r || !z || !p || !Ap) { free(r); free(z); free(p); free(Ap); return 1; }
  double rtz = 0.0, oldrtz = 0.0, alpha = 0.0, beta = 0.0, pAp = 0.0;
  memcpy(p, x, sizeof(double) * (size_t)n);               /* :87 */
  ora_spmv(A, p, Ap);                                      /* :88 */
  ora_waxpby(n, 1.0, b, -1.0, Ap, r);                      /* :89 */
  double normr = sqrt(ora_dot(n, r, r));                   /* :90-91 */
  const double normr0 = normr;
  if (hist) hist[0] = normr;
  *niters = 0;
  int err = 0;
  for (int k = 1; k <= max_iter && normr / normr0 > tolerance; ++k) {
    if (do_prec) {
      err = ora_mg_skip(L, nlev, 0, r, z, skip);           /* :104 */
      if (err) break;
    } else {
      ora_waxpby(n, 1.0, r, 0.0, r, z);                    /* :106 */
    }
    if (k == 1) {
      memcpy(p, z, sizeof(double) * (size_t)n);            /* :110 */
      rtz = ora_dot(n, r, z);                              /* :111 */
    } else {
      oldrtz = rtz;
      rtz = ora_dot(n, r, z);                              /* :114 */
      beta = rtz / oldrtz;
      ora_waxpby(n, 1.0, z, beta, p, p);                   /* :116 */
    }
    ora_spmv(A, p, Ap);                                    /* :119 */
    pAp = ora_dot(n, p, Ap);                               /* :120 */
    alpha = rtz / pAp;
    ora_waxpby(n, 1.0, x, alpha, p, x);                    /* :122 */
    ora_waxpby(n, 1.0, r, -alpha, Ap, r);                  /* :123 */
    normr = sqrt(ora_dot(n, r, r));                        /* :124-125 */
    if (hist) hist[k] = normr;
    *niters = k;
  }
  *normr_out = normr;
  *normr0_out = normr0;
  free(r); free(z); free(p); free(Ap);
  return err;
}

void ora_permute_level(int n, const int* new2old, const int* old2new, const int* nnz, const int* cols,
                       const double* vals, const int* diag, int* pnnz, int* pcols, double* pvals, int* pdiag) {
  for (int p = 0; p < n; ++p) {
    const int o = new2old[p];
    pnnz[p] = nnz[o];
    pdiag[p] = diag[o];
    for (int j = 0; j < ORA_SLOTS; ++j) {
      pcols[(int64_t)p * ORA_SLOTS + j] = old2new[cols[(int64_t)o * ORA_SLOTS + j]];
      pvals[(int64_t)p * ORA_SLOTS + j] = vals[(int64_t)o * ORA_SLOTS + j];
    }
  }
}

void ora_permute_f2c(int nc, const int* f2c, const int* coarse_new2old, const int* fine_old2new, int* pf2c) {
  for (int q = 0; q < nc; ++q) pf2c[q] = fine_old2new[f2c[coarse_new2old[q]]];
}

/* ---------------------------------------------------------------------------
 * FP32 V-cycle: ComputeMG_ref.cpp:39-63 and ComputeSYMGS_ref.cpp:67-100 with
 * float values, float vectors and float accumulation.
 * ------------------------------------------------------------------------- */
static inline float gs_row_f32(const ora_level_f32* A, int i, const float* r, const float* x) {
  const int* c = A->cols + (int64_t)i * ORA_SLOTS;
  const float* v = A->vals + (int64_t)i * ORA_SLOTS;
  const float d = v[A->diag[i]];
  float s = r[i];
  for (int j = 0; j < A->nnz[i]; ++j) s -= v[j] * x[c[j]];
  s += x[i] * d;
  return s / d;
}

/* skip: rows at the end of the forward sweep not repeated at the start of the
 * backward one (0: ComputeSYMGS_ref.cpp:67-100 exactly); see ora_symgs_skip. */
static void symgs_f32(const ora_level_f32* A, const float* r, float* x, int skip) {
  for (int i = 0; i < A->n; ++i) x[i] = gs_row_f32(A, i, r, x);
  for (int i = A->n - 1 - skip; i >= 0; --i) x[i] = gs_row_f32(A, i, r, x);
}

int ora_mg_f32(const ora_level_f32* L, int nlev, int lev, const float* r, float* x) {
  return ora_mg_f32_skip(L, nlev, lev, r, x, NULL);
}

int ora_mg_f32_skip(const ora_level_f32* L, int nlev, int lev, const float* r, float* x, const int* skip) {
  const ora_level_f32* A = &L[lev];
  const int sk = skip ? skip[lev] : 0;
  memset(x, 0, sizeof(float) * (size_t)A->n);
  if (lev + 1 < nlev) {
    const int nc = L[lev + 1].n;
    float* Axf = (float*)malloc(sizeof(float) * (size_t)A->n);
    float* rc = (float*)malloc(sizeof(float) * (size_t)nc);
    float* xc = (float*)malloc(sizeof(float) * (size_t)nc);
    if (!Axf || !rc || !xc) { free(Axf); free(rc); free(xc); return 1; }
    symgs_f32(A, r, x, sk);
    for (int i = 0; i < A->n; ++i) {
      const int* c = A->cols + (int64_t)i * ORA_SLOTS;
      const float* v = A->vals + (int64_t)i * ORA_SLOTS;
      float s = 0.0f;
      for (int j = 0; j < A->nnz[i]; ++j) s += v[j] * x[c[j]];
      Axf[i] = s;
    }
    for (int q = 0; q < nc; ++q) rc[q] = r[A->f2c[q]] - Axf[A->f2c[q]];
    int err = ora_mg_f32_skip(L, nlev, lev + 1, rc, xc, skip);
    if (!err) {
      for (int q = 0; q < nc; ++q) x[A->f2c[q]] += xc[q];
      symgs_f32(A, r, x, sk);
    }
    free(Axf); free(rc); free(xc);
    return err;
  }
  symgs_f32(A, r, x, sk);
  return 0;
}

int ora_cg_mixed(const ora_level* L, const ora_level_f32* L32, int nlev, const double* b, double* x,
                 int max_iter, double tolerance, int* niters, double* normr_out, double* normr0_out,
                 double* hist) {
  return ora_cg_mixed_skip(L, L32, nlev, b, x, max_iter, tolerance, niters, normr_out, normr0_out, hist, NULL);
}

int ora_cg_mixed_skip(const ora_level* L, const ora_level_f32* L32, int nlev, const double* b, double* x,
                      int max_iter, double tolerance, int* niters, double* normr_out, double* normr0_out,
                      double* hist, const int* skip) {
  const ora_level* A = &L[0];
  const int n = A->n;
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* z = (double*)malloc(sizeof(double) * (size_t)n);
  double* zprev = (double*)malloc(sizeof(double) * (size_t)n);
  double* p = (double*)malloc(sizeof(double) * (size_t)n);
  double* Ap = (double*)malloc(sizeof(double) * (size_t)n);
  float* r32 = (float*)malloc(sizeof(float) * (size_t)n);
  float* z32 = (float*)malloc(sizeof(float) * (size_t)n);
  int err = 0;
  if (!r || !z || !zprev || !p || !Ap || !r32 || !z32) { err = 1; goto done; }
  double rtz = 0.0, oldrtz = 0.0;
  ora_spmv(A, x, Ap);
  ora_waxpby(n, 1.0, b, -1.0, Ap, r);
  double normr = sqrt(ora_dot(n, r, r));
  const double normr0 = normr;
  if (hist) hist[0] = normr;
  *niters = 0;
  for (int k = 1; k <= max_iter && normr / normr0 > tolerance; ++k) {
    for (int i = 0; i < n; ++i) r32[i] = (float)r[i];
    err = ora_mg_f32_skip(L32, nlev, 0, r32, z32, skip);
    if (err) break;
    for (int i = 0; i < n; ++i) z[i] = (double)z32[i];
    if (k == 1) {
      memcpy(p, z, sizeof(double) * (size_t)n);
      rtz = ora_dot(n, r, z);
    } else {
      oldrtz = rtz;
      rtz = ora_dot(n, r, z);
      const double rzprev = ora_dot(n, r, zprev);
      const double beta = (rtz - rzprev) / oldrtz;  /* Polak-Ribiere: r_k'(z_k - z_{k-1}) / r_{k-1}'z_{k-1} */
      ora_waxpby(n, 1.0, z, beta, p, p);
    }
    memcpy(zprev, z, sizeof(double) * (size_t)n);
    ora_spmv(A, p, Ap);
    const double pAp = ora_dot(n, p, Ap);
    const double alpha = rtz / pAp;
    ora_waxpby(n, 1.0, x, alpha, p, x);
    ora_waxpby(n, 1.0, r, -alpha, Ap, r);
    normr = sqrt(ora_dot(n, r, r));
    if (hist) hist[k] = normr;
    *niters = k;
  }
  *normr_out = normr;
  *normr0_out = normr0;
done:
  free(r); free(z); free(zprev); free(p); free(Ap); free(r32); free(z32);
  return err;
}
