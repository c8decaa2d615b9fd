/*
 * hpcg_b200 -- C ABI of the B200 (sm_100a) implementation of the HPCG 3.1
 * preconditioned-CG path.
 *
 * Every entry point replaces one optimisable routine of the reference and is
 * called from the drop-in translation unit hpcg_b200/dropin/hpcg_dropin.cpp,
 * which keeps the reference's C++ signatures. Conventions:
 *
 *  - Every function returns an int status: 0 (HPCG_B200_OK) on success, a
 *    positive HPCG_B200_ERR_* code otherwise, like the reference's routines
 *    (callers such as src/main.cpp:190 only log non-zero codes). Nothing aborts.
 *  - Vectors are passed as plain double pointers in the reference's natural row
 *    order (row = (iz*ny + iy)*nx + ix). A pointer may be host memory (pageable or
 *    pinned) or device memory of the problem's GPU; the library detects which.
 *    Device memory of any other GPU is refused with HPCG_B200_ERR_ARG before
 *    anything is launched.
 *    Host results are complete when the call returns (calls synchronise, since the
 *    reference times them with a host clock, src/mytimer.cpp).
 *  - Internally the matrix is device-resident in an 8-colour order; vectors are
 *    permuted on the way in and out.
 */
#ifndef HPCG_B200_H
#define HPCG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPCG_B200_OK 0
#define HPCG_B200_ERR_CUDA 1        /* a CUDA runtime call failed */
#define HPCG_B200_ERR_ARG 2         /* null pointer, bad size or mismatched lengths */
#define HPCG_B200_ERR_UNSUPPORTED 3 /* matrix is not a 27-point stencil over its grid, or grid not coarsenable */
#define HPCG_B200_ERR_NOMEM 4       /* device memory exhausted (or the configured budget exceeded) */
#define HPCG_B200_ERR_HANDLE 5      /* null or corrupted problem handle */
#define HPCG_B200_ERR_TIMEOUT 6     /* a bounded device-side wait gave up */

/* Gauss-Seidel orderings */
#define HPCG_B200_SYMGS_COLOUR 0    /* 8-colour sweep (the performance path) */
#define HPCG_B200_SYMGS_NATURAL 1   /* level-scheduled natural order: ComputeSYMGS_ref's operator exactly */

typedef struct hpcg_b200_problem hpcg_b200_problem; /* opaque; the drop-in keeps it in A.optimizationData */

/*
 * One level of the multigrid hierarchy, as the reference's structures hold it
 * (src/SparseMatrix.hpp:39-76, src/MGData.hpp:28-40, src/Geometry.hpp:50-74).
 */
typedef struct hpcg_b200_level_desc {
  int nx, ny, nz;                         /* Geometry::nx/ny/nz of this level */
  int nrow;                               /* SparseMatrix::localNumberOfRows */
  int ncol;                               /* SparseMatrix::localNumberOfColumns (== nrow, one process) */
  const char* nonzeros_in_row;            /* SparseMatrix::nonzerosInRow */
  const int* const* mtx_ind_l;            /* SparseMatrix::mtxIndL */
  const double* const* matrix_values;     /* SparseMatrix::matrixValues */
  const int* f2c;                         /* MGData::f2cOperator (NULL on the coarsest level) */
} hpcg_b200_level_desc;

/* ---- setup ------------------------------------------------------------- */

/* Replaces OptimizeProblem (src/OptimizeProblem.cpp:37). Builds the device
 * hierarchy from the reference's host structures: `levels[0]` is the fine
 * matrix A, levels[l+1] is levels[l]'s A.Ac. Checks that every row holds only
 * 27-point-stencil neighbours of its grid point. */
int hpcg_b200_optimize(const hpcg_b200_level_desc* levels, int nlevels, int device, hpcg_b200_problem** out);

/* Builds the same hierarchy directly on the device, as GenerateProblem_ref
 * (src/GenerateProblem_ref.cpp:131-183) and GenerateCoarseProblem
 * (src/GenerateCoarseProblem.cpp:71-104) would for one process, without host
 * arrays: the route for grids whose host structures would not fit (512^3 has
 * 3.6e9 nonzeros, beyond the reference's int local_int_t). The reference's
 * right-hand side (b_i = 27 - nnz_i, :178) is kept on the device; read it with
 * hpcg_b200_get_rhs. */
int hpcg_b200_generate(int nx, int ny, int nz, int nlevels, int device, hpcg_b200_problem** out);

/* Copies the problem's right-hand side (natural order) to b (host or device). */
int hpcg_b200_get_rhs(hpcg_b200_problem* p, double* b);

/* Releases everything a problem holds (the reference's DeleteMatrix never frees
 * optimizationData, src/SparseMatrix.hpp:151-183, so the drop-in calls this). */
int hpcg_b200_free(hpcg_b200_problem* p);

/* Replaces OptimizeProblemMemoryUse (src/OptimizeProblem.cpp:103): bytes of device
 * memory the problem retains. Returns 0.0 for a null handle. */
double hpcg_b200_memory_use(const hpcg_b200_problem* p);

/* Re-reads the fine-level diagonal after the host changed it through
 * ReplaceMatrixDiagonal (src/SparseMatrix.hpp:139; TestCG.cpp:79 and :114 do).
 * `diagonal` holds one value per row in natural order. */
int hpcg_b200_set_diagonal(hpcg_b200_problem* p, const double* diagonal);

/* Overwrites every value of one level, keeping its sparsity. values27 holds 27
 * values per row, rows in natural order, value k of a row belonging to the
 * stencil direction k = (sz+1)*9 + (sy+1)*3 + (sx+1) (the reference's entry
 * order, GenerateProblem_ref.cpp:152-172, with directions that leave the grid
 * present and ignored). */
int hpcg_b200_set_values(hpcg_b200_problem* p, int level, const double* values27);

/* Whether hpcg_b200_cg may skip moving its host inputs when it can tell they
 * are unchanged (default on; HPCG_B200_HOST_REUSE=0 at creation turns it off):
 * a host b equal bit for bit to the b it sent last is not sent again (compared
 * on host threads against a copy the problem keeps), and an all-zero host x is
 * zeroed on the device instead of sent. The reference's timed loop
 * (src/main.cpp:334-340) passes the same b and a zeroed x to every set. No
 * reference counterpart. */
int hpcg_b200_set_host_reuse(hpcg_b200_problem* p, int enable);

/* Selects the SYMGS ordering used by hpcg_b200_symgs / _mg / _cg. */
int hpcg_b200_set_symgs_mode(hpcg_b200_problem* p, int mode);

/* ---- kernels (all vectors natural order, host or device memory) --------- */

/* y = A x on level 0. Replaces ComputeSPMV (src/ComputeSPMV.cpp:40; ComputeSPMV_ref.cpp:47-72). */
int hpcg_b200_spmv(hpcg_b200_problem* p, const double* x, double* y);

/* One symmetric Gauss-Seidel step on x with right-hand side r. Replaces
 * ComputeSYMGS (src/ComputeSYMGS.cpp:50; ComputeSYMGS_ref.cpp:54-103). */
int hpcg_b200_symgs(hpcg_b200_problem* p, const double* r, double* x);

/* x = V-cycle(r). Replaces ComputeMG (src/ComputeMG.cpp:33; ComputeMG_ref.cpp:39-63). */
int hpcg_b200_mg(hpcg_b200_problem* p, const double* r, double* x);

/* result = x'y over n entries. Replaces ComputeDotProduct
 * (src/ComputeDotProduct.cpp:41; ComputeDotProduct_ref.cpp:46-80). Deterministic. */
int hpcg_b200_dot(int n, const double* x, const double* y, double* result);

/* w = alpha x + beta y. Replaces ComputeWAXPBY (src/ComputeWAXPBY.cpp:42; ComputeWAXPBY_ref.cpp:42-70). */
int hpcg_b200_waxpby(int n, double alpha, const double* x, double beta, const double* y, double* w);

/* residual = max_i |v1_i - v2_i|. Replaces ComputeResidual (src/ComputeResidual.cpp:49-89). */
int hpcg_b200_residual(int n, const double* v1, const double* v2, double* residual);

/* Preconditioned CG. Replaces CG (src/CG.cpp:59-143): same arguments and
 * stopping rule (k <= max_iter && normr/normr0 > tolerance). times (may be
 * NULL) accumulates like the reference's times[0..5]. */
int hpcg_b200_cg(hpcg_b200_problem* p, const double* b, double* x, int max_iter, double tolerance,
                 int do_preconditioning, int* niters, double* normr, double* normr0, double* times);

/* ---- changed form 1: FP32 V-cycle inside FP64 flexible PCG --------------- */

/* As hpcg_b200_cg, but the V-cycle (values, vectors, smoother, transfers) runs
 * in FP32 and beta is the flexible Polak-Ribiere form; the SpMV, dots, alpha,
 * beta and x/r updates stay FP64. No reference counterpart (changed form). */
int hpcg_b200_cg_mixed(hpcg_b200_problem* p, const double* b, double* x, int max_iter, double tolerance,
                       int* niters, double* normr, double* normr0);

/* The FP32 V-cycle alone, as hpcg_b200_cg_mixed applies it:
 * x = widen(MG32(narrow(r))), natural order, host or device vectors. */
int hpcg_b200_mg_f32(hpcg_b200_problem* p, const double* r, double* x);

/* ---- changed form 2: several right-hand sides at once ---------------------- */

/* Preconditioned CG (CG.cpp:59-143 semantics) for nrhs <= 8 systems with the
 * problem's matrix, advanced in lockstep so that every matrix row is read once
 * per sweep for all of them. b and x hold the systems one after another:
 * b[j*n + i], natural order, n = rows (host or device memory); x is the initial
 * guess on entry and the solution on exit. System j stops updating once
 * normr_j / normr0_j <= tolerance; niters, normr and normr0 receive one value per
 * system. No reference counterpart (changed form). */
int hpcg_b200_cg_multi(hpcg_b200_problem* p, int nrhs, const double* b, double* x, int max_iter, double tolerance,
                       int* niters, double* normr, double* normr0);

/* x_j = V-cycle(r_j) for nrhs <= 8 systems, layout as hpcg_b200_cg_multi. Each
 * x_j is bitwise what hpcg_b200_mg gives for r_j. */
int hpcg_b200_mg_multi(hpcg_b200_problem* p, int nrhs, const double* r, double* x);

/* Many independent problems of different sizes solved together (flexible FP64
 * CG around the FP32 V-cycle, as hpcg_b200_cg_mixed for each). Every step of an
 * iteration walks a work list of row tiles spanning all the problems, either
 * as one kernel launch per step or all steps in one cooperative launch
 * (hpcg_b200_batch_form), and the iteration loop is one CUDA graph launch (a
 * conditional while node runs while any problem is above its tolerance);
 * converged problems skip their tiles. Every grid dimension must be a
 * multiple of 16. No reference counterpart (changed form). */
typedef struct hpcg_b200_batch hpcg_b200_batch;

/* Generates problem i on the device as hpcg_b200_generate(nx[i], ny[i], nz[i], 4). */
int hpcg_b200_batch_create(int count, const int* nx, const int* ny, const int* nz, int device,
                           hpcg_b200_batch** out);
/* The problem handle of batch member i (owned by the batch: do not free it). */
int hpcg_b200_batch_problem(hpcg_b200_batch* batch, int i, hpcg_b200_problem** out);
/* b[i], x[i]: natural-order vectors of problem i (host or device); x[i] is the
 * initial guess and receives the solution. Per problem: iterations done while
 * above `tolerance`, final and initial residual norms. */
int hpcg_b200_batch_cg_mixed(hpcg_b200_batch* batch, const double* const* b, double* const* x, int max_iter,
                             double tolerance, int* niters, double* normr, double* normr0);
int hpcg_b200_batch_free(hpcg_b200_batch* batch);
/* How the batch runs an iteration, chosen by timing at creation (or by
 * HPCG_B200_BATCH_PERSIST / HPCG_B200_BATCH_BULK): 0 one launch per step with
 * the colour phases on the register kernel, 1 the same on the bulk-copy
 * kernel, 2 the whole iteration as one cooperative launch whose steps are
 * separated by grid barriers with bounded waits (a wait that gives up ends the
 * solve with HPCG_B200_ERR_TIMEOUT). */
int hpcg_b200_batch_form(const hpcg_b200_batch* batch, int* form);

/* Check of the bounded wait of the batched iteration's grid barrier: a
 * cooperative launch of one block per SM in which every block waits for one
 * arrival more than the grid holds, so every wait gives up after `seconds`
 * (0 < seconds <= 2) and records the fault. Returns HPCG_B200_ERR_TIMEOUT (the
 * expected outcome) with the device context still usable. No reference
 * counterpart: test support for the wait path. */
int hpcg_b200_grid_wait_selftest(int device, double seconds);

/* ---- changed form 3: implicit adjoint of the solve ------------------------ */

/* Gradients of a loss L(x) through the solve A x = b, given the converged
 * forward solution x and g = dL/dx (both natural order). Solves A lambda = g
 * with the same preconditioned CG and hierarchy (A is symmetric, so A' = A),
 * from lambda = 0 to `tolerance`, then writes dL/db = lambda into grad_b and
 * dL/da = -lambda_i x_j into grad_values27, in the layout of
 * hpcg_b200_set_values (natural rows, 27 direction slots, 0 outside the grid).
 * Keeps no iterate history. No reference counterpart (changed form). */
int hpcg_b200_adjoint(hpcg_b200_problem* p, const double* x, const double* g, int max_iter, double tolerance,
                      double* grad_b, double* grad_values27, int* niters);

/* ---- dot product without device allocation -------------------------------- */

/* result[0] = x'y over n entries, for callers that cannot allocate device
 * memory (their allocator owns the GPU's memory, or allocation is not allowed
 * where they call from). No counterpart in the reference: it is an extra entry
 * point beside hpcg_b200_dot, which allocates its per-device work buffers on
 * first use. x, y and result must be device memory of the current GPU; the two
 * kernels are queued on `stream` (a cudaStream_t; NULL = the legacy default
 * stream) and the call returns without waiting. Its only scratch is a fixed
 * 512 KiB array inside the library (present on every GPU that loads it), so
 * n is limited to HPCG_B200_DOT_NOALLOC_MAX_N; larger n returns
 * HPCG_B200_ERR_ARG, as do host memory and another GPU's memory. The first
 * call on each device looks the array's address up and keeps it (make it
 * before any stream capture; after a cudaDeviceReset of that device the kept
 * address is stale, so do not call again in that process). Calls that overlap
 * on the GPU share the array and race: serialise them. */
#define HPCG_B200_DOT_NOALLOC_MAX_N 268435456
int hpcg_b200_dot_noalloc(int n, const double* x, const double* y, double* result, void* stream);

/* ---- several ranks, one per GPU ----------------------------------------------
 *
 * The reference's MPI decomposition: npx*npy*npz ranks, each owning an
 * nx*ny*nz block of the (npx*nx) x (npy*ny) x (npz*nz) grid, rank r at
 * (r % npx, (r / npx) % npy, r / (npx*npy)) (src/GenerateGeometry.cpp:89-91).
 * Each rank's matrix has the rows of its block and, as external columns, the
 * neighbours' points next to it (src/SetupHalo_ref.cpp:69-176). Every SpMV and
 * every symmetric Gauss-Seidel step starts with a halo exchange
 * (src/ComputeSPMV_ref.cpp:53, src/ComputeSYMGS_ref.cpp:59, src/ExchangeHalo.cpp),
 * every dot product ends with an allreduce (src/ComputeDotProduct_ref.cpp:70).
 * The single-rank entry points above refuse a rank of a run over several ranks
 * (HPCG_B200_ERR_UNSUPPORTED); the hpcg_b200_shard_* routines drive it. */

/* The reference's default process grid for nranks (src/ComputeOptimalShapeXYZ.cpp). */
int hpcg_b200_process_grid(int nranks, int* npx, int* npy, int* npz);

/* Generates rank `rank`'s block and hierarchy on `device`, with the halo plan of
 * every level (the reference's GenerateProblem + SetupHalo + GenerateCoarseProblem
 * run by that rank). nx, ny, nz are the LOCAL block sides. */
int hpcg_b200_generate_rank(int nx, int ny, int nz, int npx, int npy, int npz, int rank, int nlevels, int device,
                            hpcg_b200_problem** out);

/* The halo plan of one rank's level with local sides nx, ny, nz, computed on
 * the host (no GPU): neighbour ranks in ascending order, the entries exchanged
 * with each (sent = received), the local natural rows sent in that order
 * (elementsToSend), and the global row of every external column in local column
 * order (SetupHalo_ref.cpp:121-140). Arrays may be NULL; neighbors/counts hold
 * up to 26, the two lists the sum of counts. */
int hpcg_b200_halo_plan(int nx, int ny, int nz, int npx, int npy, int npz, int rank, int* nneighbors,
                        int* neighbors, int* counts, int* send_rows, long long* ext_global);

/* 10 ints for one level: rank, nranks, npx, npy, npz, ipx, ipy, ipz,
 * neighbours, external columns. */
int hpcg_b200_rank_info(const hpcg_b200_problem* p, int level, int* info);

/* Communicators. NCCL: one rank per process; every rank passes the same
 * 128-byte id, made once by hpcg_b200_comm_unique_id and broadcast by the
 * caller (MPI_Bcast, torch.distributed, ...); libnccl.so.2 is opened at run
 * time. Local: all nranks ranks of the run in this process, on one GPU, in rank
 * order (halo by device copies, reductions folded in rank order). */
typedef struct hpcg_b200_comm hpcg_b200_comm;
#define HPCG_B200_COMM_ID_BYTES 128
int hpcg_b200_comm_unique_id(void* id);
int hpcg_b200_comm_nccl(const void* id, int nranks, int rank, hpcg_b200_problem* p, hpcg_b200_comm** out);
int hpcg_b200_comm_local(int nranks, hpcg_b200_problem* const* ranks, hpcg_b200_comm** out);
int hpcg_b200_comm_free(hpcg_b200_comm* comm);

/* The routines over every rank of the run. Each takes one vector per rank this
 * process drives (one for a NCCL communicator, nranks for a local one), in the
 * rank's local natural row order, host or device memory; x of symgs is in/out.
 * Every process of a NCCL run calls the same routine with the same arguments. */
int hpcg_b200_shard_spmv(hpcg_b200_comm* comm, const double* const* x, double* const* y);
int hpcg_b200_shard_symgs(hpcg_b200_comm* comm, const double* const* r, double* const* x);
int hpcg_b200_shard_mg(hpcg_b200_comm* comm, const double* const* r, double* const* x);
int hpcg_b200_shard_dot(hpcg_b200_comm* comm, const double* const* x, const double* const* y, double* result);
int hpcg_b200_shard_cg(hpcg_b200_comm* comm, const double* const* b, double* const* x, int max_iter,
                       double tolerance, int do_preconditioning, int* niters, double* normr, double* normr0,
                       double* times);

/* ---- inspection (tests) -------------------------------------------------- */

/* Rows, padded pitch and colour-block boundaries (9 ints) of one level. */
int hpcg_b200_level_info(const hpcg_b200_problem* p, int level, int* nrow, int64_t* pitch, int* colour_start);

/* Bytes of one level's packed column index, 0 if the level keeps only its
 * 32-bit columns (a 128-row tile whose columns of one slot span more than 65534,
 * or HPCG_B200_PACKED=0 at creation). One 7024-byte record per 128-row tile of
 * the storage: 27 32-bit bases, a word of padding and 27 x 128 16-bit offsets
 * (0xFFFF: the zero sink); the bulk-copy kernels read it instead of the 32-bit
 * columns, with the same column for every entry. */
int hpcg_b200_level_packed(const hpcg_b200_problem* p, int level, int64_t* bytes);

/* Copies one level's device layout to host: new2old[nrow] (colour row -> natural
 * row), cols[27*pitch] and vals[27*pitch] (slot-major, colour order), f2c[nrow of
 * next level] (colour order, NULL allowed). */
int hpcg_b200_export_level(const hpcg_b200_problem* p, int level, int* new2old, int* cols, double* vals,
                           int* f2c);

/* The autotuner's choices for one level (7 ints): kernel configuration of the
 * Gauss-Seidel phases, of the first-sweep phases, of the FP32 phases, of the
 * SpMV/restriction, the SpMV row order (0 storage, 1 natural, 2 slab), whether
 * the level has been tuned yet (tuning happens on first use), and the
 * configuration of the FP32 first-sweep phases. */
int hpcg_b200_level_config(const hpcg_b200_problem* p, int level, int* config);

/* The configuration of the first forward sweep's phase at each of the 8 sweep
 * positions of one level (a phase reads 0 to 26 slots by its position, so the
 * tuner chooses per position): fp64 for the FP64 V-cycle, fp32 for the FP32
 * one (8 ints each, either may be NULL). */
int hpcg_b200_level_first_config(const hpcg_b200_problem* p, int level, int* fp64, int* fp32);

/* Whether the level runs each FP64 Gauss-Seidel sweep that starts from a
 * nonzero x (all but the pre-smoother's first) as one wavefront launch: a
 * cooperative kernel in which phase j of the sweep follows phase j - 1 two z
 * pairs behind, so the neighbours' x stays in L2 across the phases; the same
 * bits as the phases launched one by one. Off unless HPCG_B200_WAVE=1 (every
 * level that allows it) or HPCG_B200_WAVE=tune (the autotuner times both)
 * asks for it, or the level's configuration string sets it; a level allows it
 * where its sides are even and each colour of a z pair fills whole 128-row
 * tiles. *on receives 0 or 1. */
int hpcg_b200_level_wavefront(const hpcg_b200_problem* p, int level, int* on);

/* Check of the wavefront sweep's bounded dependency wait: launches the sweep
 * kernel on level 0 with one unit that waits for itself, so every block's wait
 * runs out after limit_seconds (0 < limit <= 10); the blocks then release
 * what they hold and leave. Returns HPCG_B200_ERR_TIMEOUT with the wavefront
 * message in hpcg_b200_last_error when the wait gave up and the context is
 * still usable, HPCG_B200_ERR_UNSUPPORTED where level 0 has no wavefront
 * tables. Writes only the problem's scratch vector Ap. */
int hpcg_b200_wave_wait_selftest(hpcg_b200_problem* p, double limit_seconds);

/* Measurement aid, with no counterpart in the reference: one launch of the
 * FP64 Gauss-Seidel phases' copy pipeline (the same stages, tensor copies and
 * column records) over every 128-row tile of the level's matrix, with
 * consumers that hand each stage straight back. *ms: its device time; *bytes:
 * the bytes it streamed (values and column index of every tile). Their ratio is
 * the rate at which the phases' tiles can stream when nothing holds a stage,
 * the ceiling of the copy side of the pipeline on this level's data. Reads
 * the matrix only. HPCG_B200_ERR_UNSUPPORTED where the level has no tensor
 * maps. */
int hpcg_b200_stream_probe(hpcg_b200_problem* p, int level, float* ms, double* bytes);

/* Check of the device-side bounded wait used by the bulk-copy Gauss-Seidel
 * phases (configuration 10): one thread waits `seconds` (0 < seconds <= 2) on
 * an mbarrier that nothing completes, gives up, records the fault and returns.
 * Returns HPCG_B200_ERR_TIMEOUT (the expected outcome) with the device context
 * still usable. No reference counterpart: test support for the wait path. */
int hpcg_b200_wait_selftest(int device, double seconds);

/* The row order the library uses for an (nx, ny, nz) grid, computed on the host
 * (no GPU needed): new2old[q] = natural row of colour-order row q, and
 * colour_start[s]..colour_start[s+1] the rows of the s-th colour swept (9 ints).
 * The colours are the parity classes of (ix, iy, iz), an 8-colouring of the
 * 27-point stencil (the greedy colouring of src/OptimizeProblem.cpp:50-96 finds
 * the same classes); the class of the injected points (all coordinates even,
 * src/GenerateCoarseProblem.cpp:71-82) is swept last. */
int hpcg_b200_colour_permutation(int nx, int ny, int nz, int* new2old, int* colour_start);

/* ---- measurement ---------------------------------------------------------- */

/* The CUDA stream (a cudaStream_t) the library launches on for `device`. All
 * work of an entry point is ordered on it; callers may record events on it. */
void* hpcg_b200_stream(int device);

/* Launch profiler: with enable != 0, CUDA events are recorded around each launch
 * of the timed kernel classes; enabling resets the totals. Kinds:
 * 0 Gauss-Seidel colour phase on level 0 (all slots), 1 first forward sweep on
 * level 0, 2 CG SpMV on level 0, 3 residual+restriction from level 0, 4 and 5
 * the same two phase kinds of the FP32 V-cycle, 6 a whole sweep on level 0 in
 * one wavefront launch (rows: the rows it updates). */
#define HPCG_B200_PROF_GS_FULL 0
#define HPCG_B200_PROF_GS_FIRST 1
#define HPCG_B200_PROF_SPMV 2
#define HPCG_B200_PROF_RESTRICT 3
#define HPCG_B200_PROF_GS32_FULL 4   /* FP32 V-cycle (hpcg_b200_cg_mixed): colour phase on level 0 */
#define HPCG_B200_PROF_GS32_FIRST 5  /* FP32 V-cycle: first forward sweep on level 0 */
#define HPCG_B200_PROF_GS_SWEEP 6    /* one-launch wavefront sweep on level 0 (forward or backward) */
int hpcg_b200_profile(int device, int enable);
int hpcg_b200_profile_read(int device, int kind, double* total_ms, int64_t* launches, int64_t* rows);

/* The CUDA error string of the last failing call on this thread ("" if none). */
const char* hpcg_b200_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* HPCG_B200_H */
