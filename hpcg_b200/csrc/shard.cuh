// Internal declarations of the multi-rank path (one rank per GPU): the process
// grid, the halo exchange plan, the communicators and the solver pieces the
// sharded drivers share with the single-rank ones.
#pragma once

#include "common.cuh"

namespace hb {

// ---- process grid and halo plan (halo.cu; host only) ------------------------

// The reference's default factoring of `size` ranks into npx*npy*npz
// (ComputeOptimalShapeXYZ.cpp:80-157).
void optimal_shape(int size, int& npx, int& npy, int& npz);

// Fills g for rank `rank` of an npx*npy*npz grid; false on bad arguments.
bool make_geom(int npx, int npy, int npz, int rank, RankGeom& g);

// Host part of the plan of one level with local grid nx*ny*nz: neighbours,
// offsets, and the rows to send in LOCAL NATURAL order (send_natural[total]).
void plan_level(const RankGeom& G, int nx, int ny, int nz, HaloPlan& h, std::vector<int>& send_natural);

// Global index of every external column n..n+total-1 of that plan (ascending
// per neighbour, as SetupHalo_ref.cpp:127-129 numbers them).
void plan_externals(const RankGeom& G, int nx, int ny, int nz, const HaloPlan& h, std::vector<long long>& ext);

// Uploads the colour-order send rows of level l and allocates its send buffer.
int upload_plan(hpcg_b200_problem* p, int l, const std::vector<int>& send_natural);

// Releases the device arrays and the plan of every level.
void free_plans(hpcg_b200_problem* p);

// send_buf[i] = x[send_rows[i]] for every entry of the plan (ExchangeHalo.cpp:77).
int pack_halo(Context* c, const HaloPlan& h, const double* x);

// ---- solver pieces shared with the sharded drivers (solver.cu) --------------

int autotune_problem(hpcg_b200_problem* p);
// SpMV of level l (dot: fused partials of x'y into c->partials); returns the
// number of partials written.
int spmv_level(hpcg_b200_problem* p, int l, const double* x, double* y, bool dot);
// rc = (rf - A xf) at the injected rows (ComputeMG_ref.cpp:49 + ComputeRestriction_ref.cpp:51)
int restrict_level(hpcg_b200_problem* p, int l, const double* rf, const double* xf, double* rc);
// xf += xc at the injected rows (ComputeProlongation_ref.cpp:49)
int prolong_level(hpcg_b200_problem* p, int l, const double* xc, double* xf);
// one symmetric Gauss-Seidel step of level l, in the problem's mode; dot (colour
// mode, x entering nonzero): r'x block partials of the final writes at
// dot[0 .. kColours * kDotStride), which the caller zeroes first
int symgs_step(hpcg_b200_problem* p, int l, const double* rhs, double* x, bool x_is_zero, double* dot = nullptr);
// true when the CG takes r'z from the post-smoother (colour mode, two or more levels)
bool rtz_from_smoother(const hpcg_b200_problem* p);
// grid of the reductions over n rows (number of partials)
int reduction_blocks(const Context* c, int64_t n);

// vector kernels of the CG loop; those that reduce return the number of partials
// written to c->partials (or a negative status)
int launch_residual(Context* c, int n, const double* b, const double* Ap, double* r);  // r = b - Ap, r'r
int launch_dot(Context* c, int n, const double* x, const double* y);                   // x'y
// x = x + alpha p with the previous iteration's alpha, then p = z + beta p
int launch_update_px(Context* c, int n, const double* z, double* p, double* x);
int launch_update_r(Context* c, int n, double* r, const double* Ap);  // r = r - alpha Ap, r'r
int launch_update_x(Context* c, int n, double* x, const double* p);   // x = x + alpha p (after the loop)
// k_finalize over c->partials / k_finalize_ranks over per-rank values
int launch_finalize(Context* c, int nparts, int op, double* out);
int launch_finalize_ranks(Context* c, const double* vals, int nvals, int op, double* out);

}  // namespace hb
