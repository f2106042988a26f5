// Internal device-side declarations shared by the CG2D kernels and the C ABI host code.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cg2d.h"

namespace cg2d {

// Compute warps per CTA (a chunk has at most as many rows, one warp per row; the next warp issues the bulk copies
// and folds the row sums): kWarps in the FP64 and FORTRAN-order builds (two CTAs of 9 warps per SM), kMixedWarps in
// the mixed-precision ROWBLOCK build for tiles whose 15-row chunks fit (one CTA of 16 warps per SM, 128 registers a
// thread: the register file splits evenly over the SM's four schedulers). KParams::nw holds the launch's count.
constexpr int kWarps = 8;
constexpr int kThreads = (kWarps + 1) * 32;
constexpr int kMixedWarps = 15;
constexpr int kMixedThreads = (kMixedWarps + 1) * 32;
constexpr int kMaxWarps = kMixedWarps;
constexpr int kMaxStages = 4;              // stage buffers of the copy pipeline (cg2d_params_t.stages)
constexpr int kMaxUnitsPerCta = 512;       // work units one CTA owns in a launch (its unit table)
constexpr int kMaxGroups = CG2D_MAX_GROUPS;
constexpr int kMaxSolves = CG2D_MAX_SOLVES; // right-hand sides per launch (one thread owns each)
constexpr int kMaxOps = 256;               // operators (instances) per launch
constexpr int kMaxTiles = 256;
constexpr int kMaxNi = 1024;               // tile width limit
constexpr int kSmemLimit = 227 * 1024;     // dynamic shared memory per CTA on sm_100

// pass kinds of the persistent kernel
enum Pass : int { P_MAX = 0, P_INIT = 1, P_Z = 2, P_S = 3, P_X = 4, P_R = 5, P_NPASS = 6 };
// per-solve action inside a pass
enum Act : int { A_NONE = 0, A_ACTIVE = 1, A_FIN = 2 };
// per-solve scalar history: one slot per (kind, iteration), each written at most once
enum Hist : int { H_RRX = 0, H_ETAX = 1, H_SQ = 2, H_RRR = 3, H_ETAZ = 4, H_SUM = 5, H_NKIND = 6 };
// per-solve vectors, each [T][nj+2][P]: every tile row with its west and east neighbour cell, plus the south
// and north neighbour rows (the tile's halo ring); see vec_pitch
enum VecId : int { V_X = 0, V_R0 = 1, V_R1 = 2, V_S0 = 3, V_S1 = 4, V_Z = 5, V_Q = 6, V_NVEC = 7 };

// Row pitch (elements) of every per-solve vector: the tile row plus its two neighbour cells, rounded up to 4
// elements so that rows start 16-byte aligned for the bulk copies in FP32 and FP64 alike. One pitch for all
// vectors lets one table of push targets serve every vector. Point (t, j, i), -1 <= j, i <= n, is element
// (t (nj + 2) + j + 1) P + i + 1.
__host__ __device__ inline int vec_pitch(int ni) { return (ni + 2 + 3) & ~3; }
// Row pitch of the packed coefficient rows: columns i = 0 .. ni (the east face of the last point included).
__host__ __device__ inline int coef_pitch(int ni) { return (ni + 1 + 3) & ~3; }

// tables of one tile layout (device)
struct TopoDev {
  const int* nbr;           // [4][T*len]: W (len nj), E (nj), S (ni), N (ni); compact source index or -1
  // push targets: vector elements (halo-ring cells of other tiles) that take the value of a tile-edge point,
  // -1 = none. WE [T][nj][4] (west-edge point of row j: 2 targets, east-edge point: 2 targets), then
  // S [T][nip][2] and N [T][nip][2] by column. A point on two edges uses the W/E entry.
  const int* tg;
  const int* map_src;       // full padded "T" map (src), for x_fortran halos and cg2d_exchange_scalar
  const int8_t* map_comp;
  int ni, nj, OLx, OLy, npx, npy, T;
  int nip;                  // column pitch of the S/N target lists (even: 16-byte aligned per tile)
  int P;                    // vec_pitch(ni)
};

struct GroupDev {
  TopoDev tp;
  int count, nrhs;
  int nblk, units;          // work units (row blocks) per tile / per instance
  int unit_base, op_base, rhs_base;
  long long pad_elems;      // T*npy*npx
  int ldc;                  // coef_pitch(ni)
  const double* a64[6];     // aW2d, aS2d, aC2d, pW, pS, pC: [count][pad_elems]
  // packed coefficients [count][2 (A, M)][T][nj+1][3][ldc], FP32 in MIXED, FP64 otherwise: the rows a
  // chunk needs are one contiguous block. A: aW2d, aS2d, aC2d; M: pW, pS, pC; row j, column i = point (j, i).
  void* cpk;
  double norm;
  const double* norm_arr;   // nullable [count]
  const double* b[2];
  const double* x0[2];
  double* x_out[2];
  double* x_fortran[2];
  cg2d_diag_t* diag[2];
  double tol[2];
  int max_iters[2];
  char* vec;                // [count][nrhs] vector blocks, or [count] blocks of pairs (pair)
  long long vec_stride;     // bytes per vector block
  long long vec_off[V_NVEC];
  // MIXED with two right-hand sides: both solves of an instance interleaved point by point (float2 vectors, x as
  // double2), so that one load or store moves a point of both; element e of slot s's vector is scalar 2 e + s
  int pair;
};

// Shared-memory image of one chunk for a pipelined pass (offsets in bytes from the stage buffer).
struct StageLay {
  int packed;                   // coefficients: 1 packed block (S, X, Z) or 3 FP64 arrays (R)
  unsigned coef, coef_stride;   // R: the 3 arrays, (ch+1) padded rows each
  int csize;
  int nvec;                     // stencil vectors per solve
  unsigned vec[2][2];           // rows jc-1 .. jc+nr of each vector, pitch P
  int vsize[2];
  unsigned xo[2];               // P_S: own rows of x (double, pitch P)
  unsigned twe, ts, tn;         // push targets of the chunk's edge points
  unsigned total;
};

__host__ __device__ inline unsigned al128(unsigned x) { return (x + 127u) & ~127u; }
__host__ __device__ inline unsigned al16(unsigned x) { return (x + 15u) & ~15u; }

// pair: the group's two right-hand sides interleaved (GroupDev::pair): each staged vector holds both (vec[1][v] is
// slot 1's first scalar inside vec[0][v]'s rows; element e of slot s at scalar 2 e of vec[s][v])
__host__ __device__ inline StageLay stage_layout(int pt, int mixed, int ch, int nrhs, int ni, int npx, int pair = 0) {
  StageLay L;
  const int P = vec_pitch(ni), ldc = coef_pitch(ni);
  unsigned o = 0;
  L.packed = pt != P_R;
  L.coef = o;
  if (L.packed) {
    L.csize = mixed ? 4 : 8;
    L.coef_stride = al128((unsigned)((ch + 1) * 3 * ldc * L.csize));
    o += L.coef_stride;
  } else {
    L.csize = 8;
    L.coef_stride = al128((unsigned)((ch + 1) * npx * 8));
    o += 3 * L.coef_stride;
  }
  L.nvec = (pt == P_Z) ? 1 : 2;
  const int vs = mixed ? 4 : 8;
  for (int v = 0; v < 2; ++v) L.vsize[v] = (pt == P_R && v == 0) ? 8 : vs;
  if (pair) {
    for (int v = 0; v < 2; ++v) {
      L.vec[0][v] = L.vec[1][v] = 0;
      if (v < L.nvec) {
        L.vec[0][v] = o;
        L.vec[1][v] = o + (unsigned)L.vsize[v];
        o += al128((unsigned)((ch + 2) * P * 2 * L.vsize[v]));
      }
    }
    L.xo[0] = L.xo[1] = 0;
    if (pt == P_S) { L.xo[0] = o; L.xo[1] = o + 8u; o += al128((unsigned)(ch * P * 16)); }
  } else {
    for (int s = 0; s < 2; ++s)
      for (int v = 0; v < 2; ++v) {
        L.vec[s][v] = 0;
        if (s < nrhs && v < L.nvec) { L.vec[s][v] = o; o += al128((unsigned)((ch + 2) * P * L.vsize[v])); }
      }
    for (int s = 0; s < 2; ++s) {
      L.xo[s] = 0;
      if (pt == P_S && s < nrhs) { L.xo[s] = o; o += al128((unsigned)(ch * P * 8)); }
    }
  }
  L.twe = o; o += al128((unsigned)(ch * 16));
  L.ts = o; o += al128(al16((unsigned)(ni * 8)));
  L.tn = o; o += al128(al16((unsigned)(ni * 8)));
  L.total = al128(o);
  return L;
}

struct KParams {
  GroupDev g[kMaxGroups];
  int ngroups, total_units, total_rhs, total_ops;
  int mixed, serial, rows_per_block, replace_every;
  double replace_above;
  int max_ni;
  int fp64_cps;             // FP64: the kernel built for 1 or 2 CTAs per SM (96 registers a thread at 2)
  int ch;                   // rows per chunk (<= nw)
  int nw;                   // compute warps per CTA (kWarps or kMixedWarps); warp nw is the copy warp
  int nstage[P_NPASS];      // pipeline depth of each pass kind (1 or 2)
  unsigned stage_bytes;     // bytes of one stage buffer
  double* hist;             // [total_rhs][H_NKIND][hist_len]
  int hist_len;
  double* part;             // [total_rhs][2][part_units]
  int part_units;
  unsigned long long* rmax; // [total_rhs] max|b*cg2dNorm| as ordered bits
  // [0] grid-wide wait arrivals, [1] error word, [2] where a time limit ran out, [3] pass << 16 | CTA
  unsigned* gs;
  unsigned long long timeout_ns;
  int unit_deal;            // 0: units dealt round-robin to the CTAs; 1: contiguous runs (cg2d_params_t)
  int test_missing;         // extra arrivals the first grid-wide wait expects (testing the time limit)
  unsigned long long* prof; // nullable: [1 + grid * kProfSlots] phase times (ns) per CTA
  // FP64, one group of one right-hand side: checkpoints for the exact-mode adjoint (nullable). At every iteration
  // k with (k + 1) % ck_every == 0 pass X_k stores r_{k+1} into ck_r + ((k + 1) / ck_every) ck_stride and pass S_k
  // stores s_k into ck_s + ((k + 1) / ck_every) ck_stride, in the reference layout [count][T][ny][nx] (interior)
  double* ck_r;
  double* ck_s;
  long long ck_stride;
  int ck_every;
  StageLay lay[kMaxGroups][P_NPASS];  // shared-memory image of a chunk, per group and pipelined pass
};

constexpr int kMaxCtas = 148 * 8;
// phase times of a CTA: thread 0's timeline (grid-wide waits, waits for stage data, compute, end-of-pass
// reductions, direct passes, the rest, total; within those: the wait for the producer's last row sums at the end
// of a pass, a reducer's wait for the unit counts, the control code between passes) and the producer warp's
// (busy issuing and folding row sums; waiting for the compute warps)
enum ProfPhase : int { PR_BAR = 0, PR_MBAR = 1, PR_ISSUE = 2, PR_COMP = 3, PR_FIN = 4, PR_DIRECT = 5, PR_OTHER = 6,
                       PR_TOTAL = 7, PR_DRAIN = 8, PR_RWAIT = 9, PR_CTRL = 10, PR_PWAIT = 11, kProfSlots = 12 };

// exact-mode adjoint (cg2d_adjoint.cu)
struct ExactArgs {
  int batch, max_iters, checkpoint, rows_per_block;
  int max_iters_cap;           // the max_iters the workspace was sized for (checkpoint slots are carved from it)
  // recorded: the forward solve stored the checkpoints (cg2d_solve_exact) and its sums are in hist
  // ([batch][H_NKIND][hist_len], one group of one right-hand side); no recording forward runs
  int recorded;
  const double* hist;
  int hist_len;
  double norm;
  const double* norm_arr;
  const double *aW, *aS, *aC, *pW, *pS, *pC, *b, *x0, *xbar;
  const cg2d_diag_t* fwd_diag;
  double *b_bar, *gW, *gS, *gC, *gpW, *gpS, *gpC, *x_check;
};
size_t exact_adjoint_workspace(const TopoDev& tp, int batch, int max_iters, int checkpoint);
// where the checkpoint blocks of an exact-adjoint workspace lie: r_c at ck_r0 + c stride, s_{c-1} at
// ck_s0 + c stride (elements), c = 0 .. max_iters / checkpoint
void exact_checkpoints(const TopoDev& tp, int batch, int max_iters, int checkpoint, void* ws, double** ck_r0,
                       double** ck_s0, long long* stride);
cudaError_t exact_adjoint(const TopoDev& tp, const ExactArgs& args, void* workspace, cudaStream_t stream);

// launchers (cg2d_solver.cu)
size_t fixed_smem_bytes(int max_ni, int serial);
cudaError_t launch_solver(const KParams& kp, int grid, size_t smem, cudaStream_t stream);
cudaError_t solver_occupancy(const KParams& kp, size_t smem, int* blocks_per_sm);
cudaError_t launch_pack_coef(const GroupDev& g, int mixed, cudaStream_t stream);
cudaError_t launch_apply_operator(const TopoDev& tp, int batch, double norm, const double* aW, const double* aS,
                                  const double* aC, const double* v, double* out, cudaStream_t stream);
cudaError_t launch_edge_products(const TopoDev& tp, int batch, double norm, const double* norm_arr,
                                 const double* lam, const double* x, double* gW, double* gS, double* gC,
                                 cudaStream_t stream);
cudaError_t launch_exchange(const TopoDev& tp, int batch, const double* a, double* out, cudaStream_t stream);

// ---- the steps either side of the solve (cg2d_pressure.cu)
struct UpdateArgs {
  int batch, Nr;
  const double *hFacW, *hFacS;                                  // [batch][T][Nr][ny][nx]
  const double *drF, *dyG, *dxG, *recip_dxC, *recip_dyC, *rA, *recip_Bo;   // shared grid fields
  double norm;                                                  // cg2dNorm when norm_arr is null
  const double* norm_arr;                                       // [batch] or null
  double offd, implicSurfPress, implicDiv2DFlow, freeSurfFac, deltaTMom, deltaTFreeSurf;
  double *aW2d, *aS2d, *aC2d, *pW, *pS, *pC;                    // [batch][T][ny][nx]
};
struct RhsIn {
  int batch, Nr, useRealFreshWaterFlux;
  const double *gU, *gV, *hFacW, *hFacS;                        // [batch][T][Nr][ny][nx]
  const double *EmPmR, *etaN, *etaH;                            // [batch][T][ny][nx]
  const double *drF, *dyG, *dxG, *rA, *maskInC, *Bo_surf;       // shared grid fields
  double freeSurfFac, mass2rUnit, implicDiv2DFlow, deltaTMom, deltaTFreeSurf;
  double *cg2d_b, *cg2d_x;
};
cudaError_t pressure_update(const TopoDev& tp, const UpdateArgs& U, cudaStream_t st);
cudaError_t pressure_rhs(const TopoDev& tp, const RhsIn& R, cudaStream_t st);
cudaError_t pressure_post(const TopoDev& tp, int batch, const double* x, const double* cg2d_x,
                          const double* recip_Bo, double* etaN, cudaStream_t st);
cudaError_t pressure_ini_norm(const TopoDev& tp, int batch, int Nr, double implicSurfPress, double implicDiv2DFlow,
                              const double* hFacW, const double* hFacS, const double* drF, const double* dyG,
                              const double* dxG, const double* recip_dxC, const double* recip_dyC, double* norm,
                              cudaStream_t st);

}  // namespace cg2d
