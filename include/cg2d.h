/*
 * cg2d.h -- C ABI of the B200 CG2D free-surface solver (libcg2d.so).
 *
 * The solver is the preconditioned conjugate-gradient iteration of mitgcm_jax's CG2D
 * (mitgcm_jax/core/cg2d.py:205-269, itself a port of MITgcm cg2d.F) on the 13-tile LLC
 * exch2 grid. Arrays cross this boundary in the reference layout: float64, row-major
 * [batch][tile][j][i] with OLx = OLy halo points on every side (mitgcm_jax/layout.py:16-54),
 * so a caller hands over exactly the arrays it would hand to cg2d_fortran. All pointers
 * passed to the solve entry points are DEVICE pointers unless stated otherwise; every call
 * is stream-ordered on the given stream and returns before the GPU work completes.
 *
 * Reference interface each entry point replaces:
 *   cg2d_topology_create   Exchanger(ExchangeMaps) for kind "T" (mitgcm_jax/parallel/exchange.py:146-183):
 *                          the exch2 halo map becomes per-tile-edge neighbour tables read by the stencil.
 *   cg2d_solve_f64         cg2d_fortran(ex, ops, cg2d_b, cg2d_x, ...) (mitgcm_jax/core/cg2d.py:205-269),
 *                          batched; cg2d_solve (cg2d.py:351-375) is this call plus the Python-side mask.
 *   cg2d_solve_groups      the same solver for several uniform batches in one persistent launch
 *                          (mixed LLC90/LLC270 batches, forward + adjoint right-hand sides sharing
 *                          one operator).
 *   cg2d_apply_operator    _matvec (cg2d.py:292-298): (A / cg2dNorm) v on the interior, 0 on halos.
 *   cg2d_edge_products     transpose of _matvec with respect to the coefficients, i.e. the
 *                          coefficient cotangents of _cg2d_implicit_jvp (cg2d.py:318-348).
 *   cg2d_exchange_scalar   Exchanger.exch_xy (exchange.py:136-142,182-183) for kind "T".
 */
#ifndef CG2D_B200_H
#define CG2D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* cg2d_stream_t; /* == cudaStream_t */

typedef enum {
  CG2D_OK = 0,
  CG2D_NOT_CONVERGED = 1,     /* per-solve diag status only: numIters == max_iters (cg2d.py:238-241) */
  CG2D_NAN = 2,               /* per-solve diag status only: the final residual is NaN */
  CG2D_BARRIER_TIMEOUT = 3,   /* a grid-wide wait exceeded params.timeout_s; results are invalid */
  CG2D_BAD_ARG = 4,
  CG2D_CUDA_ERROR = 5,
  CG2D_WORKSPACE_TOO_SMALL = 6,
  CG2D_UNSUPPORTED = 7,
  CG2D_INTERNAL_ERROR = 8     /* a device-side consistency check failed (e.g. a halo target outside its vector);
                                 results are invalid */
} cg2d_status_t;

typedef enum { CG2D_PREC_F64 = 0, CG2D_PREC_MIXED = 1 } cg2d_precision_t;

typedef enum {
  /* per row: lane partials over i = lane + 32k, then an xor butterfly over the 32 lanes;
     rows of a block of rows_per_block added in order; blocks of a tile in order; tiles in
     order from 0 (global_sum.py:20-26). Same result for every launch geometry. */
  CG2D_SUM_ROWBLOCK = 0,
  /* "fortran" order of cg2d.py:141-161: s = 0; DO j; DO i; s = s + a(i,j), then the tiles in
     order from 0. Bitwise equal to the reference's sum_order="fortran"; slow (one thread per tile). */
  CG2D_SUM_FORTRAN = 1
} cg2d_sum_order_t;

/* Launch / numerics options (fields of Cg2dParams that are not per-solve live in the group). */
typedef struct {
  int precision;       /* cg2d_precision_t */
  int sum_order;       /* cg2d_sum_order_t */
  int rows_per_block;  /* ROWBLOCK block height in rows (multiple of 8; default 8). A mixed-precision single-group
                          launch whose 15-row chunks fit in shared memory (tiles up to about 130 points wide) runs on
                          the 16-warp build and uses blocks of 15 rows instead */
  int replace_every;   /* MIXED: FP64 true-residual replacement period in iterations (default 25) */
  double replace_above;/* MIXED: replace only while the residual is above replace_above * tolerance (default 100) */
  int grid_ctas;       /* 0 = as many as can be co-resident (capped by the work units) */
  int ctas_per_sm;     /* 0 = occupancy maximum. FP64 has two kernel builds: for 1 CTA per SM and for 2 (fewer
                          registers a thread). 2 takes the second; 0 takes it when every group has one right-hand
                          side and there are at least 8 work units per SM, otherwise the first. Results-neutral */
  double timeout_s;    /* bound on every grid-wide wait (default 10 s) */
  int test_missing_arrivals; /* testing only (default 0): the first grid-wide wait expects this many
                                arrivals more than there are CTAs, so it runs out after timeout_s and
                                every solve reports CG2D_BARRIER_TIMEOUT (exercises the bounded wait) */
  int profile;         /* 1: record per-CTA phase times in the workspace (cg2d_workspace_profile) */
  int unit_deal;       /* how the work units (instance, tile, row block) are dealt to the CTAs:
                          0 = round-robin (default), 1 = contiguous runs. Like grid_ctas and ctas_per_sm it moves
                          work between CTAs only: every sum is formed in the same fixed order, so results are the
                          same bit for bit whatever the schedule (the autotuner's search space) */
  int stages;          /* depth of the copy pipeline of a CTA: 0 = the default (3 on the 16-warp mixed build, else
                          2), or 2..4 stage buffers, capped at what fits on the 16-warp build; deeper pipelines need
                          more shared memory per CTA (fewer CTAs per SM). Also results-neutral */
} cg2d_params_t;

/* Per-solve diagnostics: the diag dict of cg2d_fortran (cg2d.py:267-268) plus a status. */
typedef struct {
  double firstResidual;
  double lastResidual;
  double sumRHS;
  double rhsMax;
  int32_t numIters;
  int32_t status;        /* cg2d_status_t */
  int32_t replacements;  /* MIXED: true-residual recomputations done */
  int32_t reserved;
} cg2d_diag_t;

typedef struct cg2d_topology cg2d_topology_t;

/* Build the device neighbour tables of one LLC layout from the exch2 scalar ("T") halo map in
 * the reference's ExchangeMaps format (exchange.py:73-93): for every padded point p of
 * [nTiles][sNy+2*OLy][sNx+2*OLx], comp[p] == 1 means out[p] = a[src[p]], comp[p] == 0 means the
 * point keeps its value. src/comp are HOST arrays of length nTiles*(sNy+2OLy)*(sNx+2OLx).
 * Every point the 5-point stencil reads (first halo row/column, corners excluded) must take its
 * value from an interior point or be unwritten (comp 0); anything else is CG2D_BAD_ARG.
 * Allocates device memory (the tables and a copy of the full map for the x_fortran halos). */
cg2d_status_t cg2d_topology_create(int sNx, int sNy, int OLx, int OLy, int nTiles,
                                   const int32_t* src, const int8_t* comp,
                                   cg2d_topology_t** out);
cg2d_status_t cg2d_topology_destroy(cg2d_topology_t* topo);

/* One uniform batch of `count` instances on one topology. Array arguments are device pointers
 * to [count][nTiles][ny][nx] float64 (ny = sNy + 2 OLy, nx = sNx + 2 OLx). Each instance has
 * nrhs (1 or 2) right-hand sides that share its operator and preconditioner (e.g. a forward
 * solve and an adjoint solve); slot k of every instance uses b[k], x0[k], x_out[k], ...
 * x_out: interior = solution, halos = 0 (cg2d_solve's x, cg2d.py:351-356).
 * x_fortran (nullable): the array exactly as cg2d_fortran returns it -- interior = solution,
 * halos = exchanged normalised first guess, unwritten halo points = the first guess
 * (cg2d.py:208-210, 227-228). diag: device array of `count` cg2d_diag_t per slot. */
typedef struct {
  const cg2d_topology_t* topo;
  int count;
  int nrhs;
  const double* aW2d; const double* aS2d; const double* aC2d;
  const double* pW; const double* pS; const double* pC;
  double cg2dNorm;                 /* used when cg2dNorm_per_instance is NULL */
  const double* cg2dNorm_per_instance; /* device [count], nullable */
  const double* b[2];
  const double* x0[2];
  double* x_out[2];
  double* x_fortran[2];
  cg2d_diag_t* diag[2];
  double tolerance[2];             /* cg2dTolerance (normalised residual, cg2d.py:219,241) */
  int max_iters[2];                /* cg2dMaxIters */
} cg2d_group_t;

#define CG2D_MAX_GROUPS 4
#define CG2D_MAX_SOLVES 256        /* instances x nrhs over all groups of one call */

void cg2d_default_params(cg2d_params_t* p);

/* Bytes of device workspace a cg2d_solve_groups call with these groups needs. */
size_t cg2d_workspace_size(const cg2d_group_t* groups, int ngroups, const cg2d_params_t* params);

/* Solve every right-hand side of every group in ONE persistent cooperative launch.
 * The workspace (device, >= cg2d_workspace_size bytes, 256-byte aligned) is scratch; it is not
 * read before being written. Returns CG2D_OK when the work was enqueued; per-solve outcomes
 * (convergence, NaN, barrier timeout) are in each solve's diag.status. */
cg2d_status_t cg2d_solve_groups(const cg2d_group_t* groups, int ngroups, const cg2d_params_t* params,
                                void* workspace, size_t workspace_bytes, cg2d_stream_t stream);

/* cg2d_fortran on a uniform batch, one right-hand side per instance (cg2d.py:205). */
cg2d_status_t cg2d_solve_f64(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                             const double* aW2d, const double* aS2d, const double* aC2d,
                             const double* pW, const double* pS, const double* pC,
                             const double* cg2d_b, const double* cg2d_x,
                             double tolerance, int max_iters,
                             double* x_out, double* x_fortran, cg2d_diag_t* diag,
                             const cg2d_params_t* params,
                             void* workspace, size_t workspace_bytes, cg2d_stream_t stream);

/* cg2d_solve_f64 in mixed precision (FP32 vectors and matvec, FP64 dot products, solution and residual
 * replacement; the params' precision field is ignored). Same arguments; the workspace is sized by
 * cg2d_workspace_size with precision CG2D_PREC_MIXED. */
cg2d_status_t cg2d_solve_mixed(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                               const double* aW2d, const double* aS2d, const double* aC2d,
                               const double* pW, const double* pS, const double* pC,
                               const double* cg2d_b, const double* cg2d_x,
                               double tolerance, int max_iters,
                               double* x_out, double* x_fortran, cg2d_diag_t* diag,
                               const cg2d_params_t* params,
                               void* workspace, size_t workspace_bytes, cg2d_stream_t stream);

/* The adjoint of cg2d_solve (_cg2d_implicit_jvp, cg2d.py:318-348, transposed) for J = <x_bar, x>:
 * lam = A^-1 x_bar by a tight CG from a zero first guess (adj_tolerance, adj_max_iters; the reference's
 * tight_transpose, cg2d.py:333-344), which is the cotangent of cg2d_b; with coeff_grad = 1 also the coefficient
 * cotangents gW, gS, gC as edge products of lam and the forward solution x (cg2d_edge_products); with
 * coeff_grad = 0 the operator is passive (the reference's ECCO mode, stop_coeff_grad, cg2d.py:370-371) and gW, gS,
 * gC (nullable) are zeroed. x: the forward solution (interior; its halos are ignored). diag: the tight solve's.
 * The workspace is cg2d_adjoint_ecco_workspace_size bytes (the solver's, plus the zero first guess). */
size_t cg2d_adjoint_ecco_workspace_size(const cg2d_topology_t* topo, int batch, int adj_max_iters,
                                        const cg2d_params_t* params);
cg2d_status_t cg2d_adjoint_ecco(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                                const double* cg2dNorm_per_instance,
                                const double* aW2d, const double* aS2d, const double* aC2d,
                                const double* pW, const double* pS, const double* pC,
                                const double* x, const double* x_bar, double adj_tolerance, int adj_max_iters,
                                int coeff_grad, double* lam, double* gW, double* gS, double* gC,
                                cg2d_diag_t* diag, const cg2d_params_t* params,
                                void* workspace, size_t workspace_bytes, cg2d_stream_t stream);

/* Exact-mode adjoint: the cotangents of x_out = cg2d_solve_f64(...) (its interior) with respect to cg2d_b and to
 * the six coefficient arrays, for J = <x_bar, x_out>, by reverse mode through the CG iterations that the forward
 * took (each instance's numIters, read from fwd_diag, the diag of the forward solve). The "exact mode" of the
 * solver; the reference has no counterpart (its JAX code cannot reverse a while_loop; it differentiates implicitly, which is
 * cg2d_edge_products after an adjoint solve). The forward must be an FP64 ROWBLOCK solve with rows_per_block rows
 * per block; the recording forward inside reproduces it bit for bit (x_check, nullable, receives its x_out).
 * Memory: r and the previous search direction every checkpoint_every iterations (0 = one segment), and one
 * segment's r, z, s, q; segments are recomputed from their checkpoint with the recorded alpha and beta.
 * Outputs (device, [batch][T][ny][nx], written in full): b_bar (interior), gW/gS/gC and gpW/gpS/gpC on the
 * faces and points edge_products writes. x0 is treated as constant (cg2d.py:372). Synchronises the stream once
 * to read the forward's iteration counts (each must be <= max_iters, which sizes the workspace). */
size_t cg2d_adjoint_exact_workspace_size(const cg2d_topology_t* topo, int batch, int max_iters,
                                         int checkpoint_every);
cg2d_status_t cg2d_adjoint_exact(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                                 const double* cg2dNorm_per_instance,
                                 const double* aW2d, const double* aS2d, const double* aC2d,
                                 const double* pW, const double* pS, const double* pC,
                                 const double* cg2d_b, const double* cg2d_x, const cg2d_diag_t* fwd_diag,
                                 const double* x_bar, int max_iters, int rows_per_block, int checkpoint_every,
                                 double* b_bar, double* gW, double* gS, double* gC,
                                 double* gpW, double* gpS, double* gpC, double* x_check,
                                 void* workspace, size_t workspace_bytes, cg2d_stream_t stream);

/* The FP64 ROWBLOCK solve and the exact-mode adjoint in one call: the forward solve (x_out, diag, as
 * cg2d_solve_f64) stores the checkpoints and keeps its sums, and the reverse sweep (as cg2d_adjoint_exact,
 * outputs b_bar, gW/gS/gC, gpW/gpS/gpC) starts from them, with no second forward pass. The gradients equal
 * cg2d_adjoint_exact's on the same inputs bit for bit. Synchronises the stream once (the iteration counts).
 * Workspace: cg2d_solve_exact_workspace_size bytes, 256-byte aligned. */
size_t cg2d_solve_exact_workspace_size(const cg2d_topology_t* topo, int batch, int max_iters, int rows_per_block,
                                       int checkpoint_every);
cg2d_status_t cg2d_solve_exact(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                               const double* cg2dNorm_per_instance,
                               const double* aW2d, const double* aS2d, const double* aC2d,
                               const double* pW, const double* pS, const double* pC,
                               const double* cg2d_b, const double* cg2d_x, double tolerance, int max_iters,
                               const double* x_bar, int rows_per_block, int checkpoint_every,
                               double* x_out, cg2d_diag_t* diag, double* b_bar, double* gW, double* gS, double* gC,
                               double* gpW, double* gpS, double* gpC,
                               void* workspace, size_t workspace_bytes, cg2d_stream_t stream);

/* cg2d_solve_f64 without a caller workspace and without any allocation (no counterpart in the reference, whose
 * JAX arrays are allocated by XLA). For callers that cannot allocate device memory where they solve: a step
 * inside a framework that owns the whole device pool and hands a custom call only its operands, or code that
 * must not let a cudaMalloc synchronise the device. The workspace is a fixed array of
 * CG2D_NOALLOC_SCRATCH_BYTES in the library's device memory (enough for two LLC90 solves in FP64). A solve needing
 * more returns CG2D_WORKSPACE_TOO_SMALL. The array is reserved on a device when the library's device code is
 * loaded there; under CUDA's lazy module loading (the default) that happens in the FIRST call of this entry point
 * on the device, which also looks up the array's device address (with that device current). So make the first
 * call at start-up: before a framework reserves its memory pool (or it may fail with CG2D_CUDA_ERROR, out of
 * memory) and before any stream capture. Later calls reserve nothing; the device holds the array until the
 * process exits. The address is looked up again in a new context (after cudaDeviceReset). params->profile must
 * be 0 (CG2D_BAD_ARG otherwise: the profile would land in the hidden array); other invalid arguments give the
 * status cg2d_solve_f64 gives. The topology is created beforehand (cg2d_topology_create allocates); inputs and
 * outputs are the caller's, as for cg2d_solve_f64. All calls on a device share the array: calls that overlap on
 * the GPU (other streams, other threads) race and give wrong results; serialise them. */
#define CG2D_NOALLOC_SCRATCH_BYTES (32u << 20)
cg2d_status_t cg2d_solve_f64_noalloc(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                                     const double* aW2d, const double* aS2d, const double* aC2d,
                                     const double* pW, const double* pS, const double* pC,
                                     const double* cg2d_b, const double* cg2d_x,
                                     double tolerance, int max_iters,
                                     double* x_out, double* x_fortran, cg2d_diag_t* diag,
                                     const cg2d_params_t* params, cg2d_stream_t stream);

/* ---- The steps either side of the solve in SOLVE_FOR_PRESSURE, batched. 3-D fields are [batch][T][Nr][ny][nx],
 * per-instance 2-D fields [batch][T][ny][nx], grid fields [T][ny][nx] shared by the batch (all float64, device,
 * the reference layout). Results are bit for bit those of the reference's functions. The vertical factors
 * deepFacC, rhoFacC, deepFac2F of the reference are all 1 (free_surface.py:121-125) and are not taken. */

/* The FreeSurfParams fields these steps read (mitgcm_jax/core/free_surface.py). */
typedef struct {
  double deltaTMom, deltaTFreeSurf, freeSurfFac, implicSurfPress, implicDiv2DFlow, mass2rUnit;
  int useRealFreshWaterFlux;
  int Nr;
} cg2d_freesurf_t;

/* update_cg2d (mitgcm_jax/core/solve_for_pressure.py:29-65): aW2d, aS2d from the level sums of the r* face areas
 * (hFacW, hFacS after UPDATE_R_STAR, halos filled), scaled by cg2dNorm (per instance when cg2dNorm_per_instance
 * is non-null), aC2d exchanged, and pW, pS, pC rewritten on i, j = 1..sNx+1, 1..sNy+1 (in place: the other points
 * keep their values). Grid fields: drF [Nr], dyG, dxG, recip_dxC, recip_dyC, rA, recip_Bo. */
cg2d_status_t cg2d_update_operator(const cg2d_topology_t* topo, int batch, const cg2d_freesurf_t* fs,
                                   double cg2dNorm, const double* cg2dNorm_per_instance, double cg2dpcOffDFac,
                                   const double* hFacW, const double* hFacS, const double* drF,
                                   const double* dyG, const double* dxG, const double* recip_dxC,
                                   const double* recip_dyC, const double* rA, const double* recip_Bo,
                                   double* aW2d, double* aS2d, double* aC2d, double* pW, double* pS, double* pC,
                                   cg2d_stream_t stream);

/* cg2d_rhs (solve_for_pressure.py:68-106): cg2d_b on the interior (0 on halos) from the fresh-water flux EmPmR
 * (when fs->useRealFreshWaterFlux), the divergence of the g-hat transports (gU, gV, hFacW, hFacS; levels Nr..1) and
 * the exactConserv etaH term; cg2d_x = Bo_surf etaN on the full array. Grid fields: drF [Nr], dyG, dxG, rA,
 * maskInC, Bo_surf. */
cg2d_status_t cg2d_pressure_rhs(const cg2d_topology_t* topo, int batch, const cg2d_freesurf_t* fs,
                                const double* gU, const double* gV, const double* hFacW, const double* hFacS,
                                const double* EmPmR, const double* etaN, const double* etaH, const double* drF,
                                const double* dyG, const double* dxG, const double* rA, const double* maskInC,
                                const double* Bo_surf, double* cg2d_b, double* cg2d_x, cg2d_stream_t stream);

/* ini_cg2d_norm (mitgcm_jax/core/cg2d.py:108-134, ini_cg2d.F:90-135), once at set-up: per instance cg2dNorm =
 * 1 / max over the interior faces of |aW|, |aS| of the un-normalised operator, aW = the sum over k = 1..Nr in order
 * of implicSurfPress implicDiv2DFlow dyG drF(k) hFacW(k) recip_dxC (aS likewise with dxG, hFacS, recip_dyC), 1 where
 * the maximum is 0. hFacW, hFacS: the initial face fractions [batch][T][Nr][ny][nx]; grid fields drF [Nr] and dyG,
 * dxG, recip_dxC, recip_dyC [T][ny][nx]; cg2dNorm: device [batch], written. Bit for bit the reference's value. */
cg2d_status_t cg2d_ini_norm(const cg2d_topology_t* topo, int batch, int Nr, double implicSurfPress,
                            double implicDiv2DFlow, const double* hFacW, const double* hFacS, const double* drF,
                            const double* dyG, const double* dxG, const double* recip_dxC, const double* recip_dyC,
                            double* cg2dNorm, cg2d_stream_t stream);

/* After the solve (solve_for_pressure.py:116-121): etaN = recip_Bo x, x the solution on the interior and, on halo
 * points, its exchanged value, or the first guess cg2d_x where the exchange writes nothing. recip_Bo is a grid
 * field [T][ny][nx]. */
cg2d_status_t cg2d_pressure_post(const cg2d_topology_t* topo, int batch, const double* x, const double* cg2d_x,
                                 const double* recip_Bo, double* etaN, cg2d_stream_t stream);

/* Host-side error word of the last solve that used this workspace (synchronises the stream). */
cg2d_status_t cg2d_workspace_status(const void* workspace, cg2d_stream_t stream);

/* out = (A / cg2dNorm) v on the interior and 0 on halo points, with v's cross-tile neighbours
 * gathered through the exchange (v's own halos are ignored, unwritten halo points read 0):
 * _matvec of cg2d.py:292-298. Arrays [batch][T][ny][nx]. */
cg2d_status_t cg2d_apply_operator(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                                  const double* aW2d, const double* aS2d, const double* aC2d,
                                  const double* v, double* out, cg2d_stream_t stream);

/* Coefficient cotangents of J for the implicit derivative dx = A^-1 (db - dA x)
 * (cg2d.py:331, 346-347): with lam = A^-1 xbar (an adjoint solve) and c = lam / cg2dNorm,
 *   gW[j][i] = -(c(j,i) x(j,i-1) + c(j,i-1) x(j,i))  for interior rows, columns 1..sNx+1,
 *   gS[j][i] = -(c(j,i) x(j-1,i) + c(j-1,i) x(j,i))  for interior columns, rows 1..sNy+1,
 *   gC[j][i] = -c(j,i) x(j,i)                        on the interior,
 * where x's cross-tile neighbours come through the exchange (unwritten halo points read 0);
 * every other point of gW/gS/gC is set to 0. lam and x: [batch][T][ny][nx], halos ignored. */
cg2d_status_t cg2d_edge_products(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                                 const double* cg2dNorm_per_instance,
                                 const double* lam, const double* x,
                                 double* gW, double* gS, double* gC, cg2d_stream_t stream);

/* Exchanger.exch_xy for kind "T" (exchange.py:136-142): out[p] = comp[p] ? a[src[p]] : a[p]
 * over the full halo map given to cg2d_topology_create. a and out: [batch][T][ny][nx]; out may
 * not alias a. */
cg2d_status_t cg2d_exchange_scalar(const cg2d_topology_t* topo, int batch, const double* a, double* out,
                                   cg2d_stream_t stream);

/* Phase times of the last solve that used this workspace with params->profile = 1 (synchronises the
 * stream). out (host, >= 1 + 12 * cap values): out[0] = number of CTAs G, then for CTA c at
 * out[1 + 12c .. 12c + 12] the nanoseconds of
 *   thread 0:        [0] grid-wide waits, [1] waits for bulk-copied chunk data, [3] compute, [4] end-of-pass
 *                    reductions, [5] direct passes, [6] the rest, [7] total, [8] wait at the end of a pass for
 *                    the copy warp's last row sums, [9] reducer waits for unit counts (within [4]),
 *                    [10] control code between passes;
 *   the copy warp:   [2] busy issuing copies and folding row sums, [11] waiting for the compute warps.
 * Returns CG2D_BAD_ARG when the groups/params do not describe that workspace's layout. */
cg2d_status_t cg2d_workspace_profile(const void* workspace, const cg2d_group_t* groups, int ngroups,
                                     const cg2d_params_t* params, uint64_t* out, int cap, cg2d_stream_t stream);

/* Human-readable name of a status code (static string). */
const char* cg2d_status_string(cg2d_status_t s);

#ifdef __cplusplus
}
#endif

#endif /* CG2D_B200_H */
