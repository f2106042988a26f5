// Internal device-side declarations shared by the CG2D kernels and the C ABI host code.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cg2d.h"

namespace cg2d {

constexpr int kWarps = 8;                  // rows per chunk = warps per CTA (one warp per row)
constexpr int kThreads = kWarps * 32;
constexpr int kMaxGroups = CG2D_MAX_GROUPS;
constexpr int kMaxSolves = CG2D_MAX_SOLVES; // right-hand sides per launch (one thread owns each)
constexpr int kMaxOps = 256;               // operators (instances) per launch
constexpr int kMaxTiles = 256;
constexpr int kMaxNi = 1024;               // tile width limit (shared-memory staging rows)

// pass kinds of the persistent kernel
enum Pass : int { P_MAX = 0, P_INIT = 1, P_Z = 2, P_S = 3, P_X = 4 };
// per-solve action inside a pass
enum Act : int { A_NONE = 0, A_ACTIVE = 1, A_FIN = 2, A_REPLACE = 3 };
// per-solve scalar history: one slot per (kind, iteration), each written at most once
enum Hist : int { H_RRX = 0, H_ETAX = 1, H_SQ = 2, H_RRR = 3, H_ETAZ = 4, H_SUM = 5, H_NKIND = 6 };

// neighbour tables of one tile layout (device)
struct TopoDev {
  const int* nbr;           // [4][T*len]: W (len nj), E (nj), S (ni), N (ni); compact source index or -1
  const int* map_src;       // full padded "T" map (src), for x_fortran halos and cg2d_exchange_scalar
  const int8_t* map_comp;
  int ni, nj, OLx, OLy, npx, npy, T;
};

struct GroupDev {
  TopoDev tp;
  int count, nrhs;
  int nblk, units;          // work units (row blocks) per tile / per instance
  int unit_base, op_base, rhs_base;
  long long pad_elems;      // T*npy*npx
  long long cmp_elems;      // T*nj*ni
  const double* a64[6];     // aW2d, aS2d, aC2d, pW, pS, pC: [count][pad_elems]
  float* c32;               // MIXED: [count][6][pad_elems] float copies of a64
  double norm;
  const double* norm_arr;   // nullable [count]
  const double* b[2];
  const double* x0[2];
  double* x_out[2];
  double* x_fortran[2];
  cg2d_diag_t* diag[2];
  double tol[2];
  int max_iters[2];
  char* vec;                // [count][nrhs] vector blocks (x, r0, r1, s0, s1, z, q)
  long long vec_stride;     // bytes per vector block
  long long vec_off[7];     // byte offsets of x, r0, r1, s0, s1, z, q inside a block
};

struct KParams {
  GroupDev g[kMaxGroups];
  int ngroups, total_units, total_rhs, total_ops;
  int mixed, serial, rows_per_block, replace_every;
  double replace_above;
  int max_ni;
  double* hist;             // [total_rhs][H_NKIND][hist_len]
  int hist_len;
  double* part;             // [total_rhs][2][part_units]
  int part_units;
  unsigned* cnt;            // [total_ops] monotonic per-operator unit counters
  unsigned long long* rmax; // [total_rhs] max|b*cg2dNorm| as ordered bits
  unsigned* gs;             // [0] grid barrier arrivals, [1] error word
  unsigned long long timeout_ns;
  int test_missing;         // extra arrivals the first grid-wide wait expects (testing the time limit)
};

size_t smem_bytes(int max_ni, int serial);

// launchers (cg2d_solver.cu)
cudaError_t launch_solver(const KParams& kp, int grid, size_t smem, cudaStream_t stream);
cudaError_t solver_occupancy(int mixed, size_t smem, int* blocks_per_sm);
cudaError_t launch_pack32(const GroupDev& g, cudaStream_t stream);
cudaError_t launch_apply_operator(const TopoDev& tp, int batch, double norm, const double* aW, const double* aS,
                                  const double* aC, const double* v, double* out, cudaStream_t stream);
cudaError_t launch_edge_products(const TopoDev& tp, int batch, double norm, const double* norm_arr,
                                 const double* lam, const double* x, double* gW, double* gS, double* gC,
                                 cudaStream_t stream);
cudaError_t launch_exchange(const TopoDev& tp, int batch, const double* a, double* out, cudaStream_t stream);

}  // namespace cg2d
