// Exact-mode adjoint of the FP64 CG2D iteration: reverse mode through the iterations of cg2d_fortran
// (mitgcm_jax/core/cg2d.py:205-269) as they were taken, with the iteration count of the forward solve.
//
// The reference has no such adjoint: its JAX code cannot reverse a while_loop and differentiates implicitly
// (cg2d.py:307-348). This one differentiates the map b, A, M -> x_K of K literal CG iterations:
//   forward, iteration k:  z = M r;  eta = <z, r>;  beta = eta / eta_prev;  s = z + beta s_prev;  q = A s;
//                          sigma = <s, q>;  alpha = eta / sigma;  x += alpha s;  r -= alpha q
//   reverse, iteration k (given rbar = rbar_{k+1}, sbar = beta_{k+1} sbar_{k+1}, the eta cotangent carried from
//   iteration k+1, and xbar, which is constant):
//     abar = <xbar, s> - <rbar, q>;  sigbar = -abar alpha / sigma;  etabar = carry + abar / sigma
//     qbar = sigbar s - alpha rbar;  sbar += alpha xbar + sigbar q;  sbar += A qbar;  Abar += qbar (x) s
//     bbar = <sbar, s_prev>;  etabar += bbar / eta_prev;  carry = -bbar eta / eta_prev^2
//     zbar = sbar + etabar r;  rbar += etabar z;  sbar = beta sbar;  rbar += M zbar;  Mbar += zbar (x) r
// and at the start r_0 = b_n - A x_0: bbar_n = rbar_0, Abar -= rbar_0 (x) x_0. A and M are symmetric operators,
// so their transposes are themselves; (x) is the transpose of the stencil in its coefficients (edge products,
// as for the implicit derivative). The normalisation by rhsNorm cancels (x_K is homogeneous of degree 1 in
// (b, x_0)), so it enters only as the scale of b and x.
//
// Memory: the recording forward keeps r and s_prev every `checkpoint` iterations; the reverse sweep takes the
// segments from the last, recomputes each one's r, z, s, q from its checkpoint with the stored alpha and beta
// (bit for bit the recorded values), then reverses through it. The recording forward performs the same
// floating-point operations in the same order as cg2d_solve_f64 (ROWBLOCK sums), so it reproduces its iterates
// exactly.

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "cg2d_internal.cuh"

namespace cg2d {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// apply_operator / apply_preconditioner addition orders (cg2d.py:181-198)
__device__ __forceinline__ double opA(double aw, double ae, double as, double an, double ac, double vw, double ve,
                                     double vs, double vn, double vc) {
  double t = mul(aw, vw);
  t = add(t, mul(ae, ve));
  t = add(t, mul(as, vs));
  t = add(t, mul(an, vn));
  return add(t, mul(ac, vc));
}
__device__ __forceinline__ double opM(double pc, double pw, double pe, double ps, double pn, double vc, double vw,
                                     double ve, double vs, double vn) {
  double t = mul(pc, vc);
  t = add(t, mul(pw, vw));
  t = add(t, mul(pe, ve));
  t = add(t, mul(ps, vs));
  return add(t, mul(pn, vn));
}

__device__ __forceinline__ long long padded(const TopoDev& tp, int t, int j, int i) {
  return ((long long)t * tp.npy + j + tp.OLy) * tp.npx + i + tp.OLx;
}
__device__ __forceinline__ long long cmp_pad(const TopoDev& tp, int c) {
  const int per = tp.nj * tp.ni;
  const int t = c / per, rem = c - t * per, j = rem / tp.ni;
  return padded(tp, t, j, rem - j * tp.ni);
}
// source of the value at (t, j, i), -1 <= i <= ni, -1 <= j <= nj (not a corner): its padded index in the same
// instance, or -1 for an unwritten halo point
__device__ __forceinline__ long long source(const TopoDev& tp, int t, int j, int i) {
  if (i >= 0 && i < tp.ni && j >= 0 && j < tp.nj) return padded(tp, t, j, i);
  int src;
  if (i < 0) src = tp.nbr[t * tp.nj + j];
  else if (i >= tp.ni) src = tp.nbr[tp.T * tp.nj + t * tp.nj + j];
  else if (j < 0) src = tp.nbr[2 * tp.T * tp.nj + t * tp.ni + i];
  else src = tp.nbr[2 * tp.T * tp.nj + tp.T * tp.ni + t * tp.ni + i];
  return src >= 0 ? cmp_pad(tp, src) : -1;
}
// a CG vector at (t, j, i) as the exchange gives it: unwritten halo points read 0
__device__ __forceinline__ double nbv(const TopoDev& tp, const double* v, int t, int j, int i) {
  const long long s = source(tp, t, j, i);
  return s >= 0 ? v[s] : 0.0;
}
// the normalised first guess at (t, j, i): interior points scaled, unwritten halo points keep cg2d_x
// (cg2d.py:227-228)
__device__ __forceinline__ double nbx0(const TopoDev& tp, const double* x0, double rn, int t, int j, int i) {
  const long long s = source(tp, t, j, i);
  return s >= 0 ? mul(x0[s], rn) : x0[padded(tp, t, j, i)];
}

struct Geo {
  TopoDev tp;
  int batch;
  long long pe;     // padded elements per instance
  long long pts;    // interior points per instance
  const int* nbp;   // tp.nbr with padded offsets in the instance instead of compact indices (-1: unwritten)
};

// nbp from tp.nbr: the same [W: T nj][E: T nj][S: T ni][N: T ni] layout, each entry the padded offset of the
// source point (cmp_pad) or -1
__global__ void k_nbp(TopoDev tp, int* nbp) {
  const int n = 2 * tp.T * (tp.nj + tp.ni);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int src = tp.nbr[e];
    nbp[e] = src >= 0 ? (int)cmp_pad(tp, src) : -1;
  }
}
// Point kernels run one thread per interior point: threadIdx.x = i, one tile row per threadIdx.y,
// blockIdx.x = group of rows (row = t nj + j), blockIdx.y = instance. Face kernels use the same shape over
// i = 0..ni and rows j = 0..nj of each tile.
#define POINT(G, in, t, j, i, p)                                                         \
  const int i = threadIdx.x, in = blockIdx.y;                                            \
  const int row_ = blockIdx.x * blockDim.y + threadIdx.y;                                \
  if (i >= (G).tp.ni || row_ >= (G).tp.T * (G).tp.nj) return;                            \
  const int t = row_ / (G).tp.nj, j = row_ - t * (G).tp.nj;                              \
  const long long p = (long long)in * (G).pe + padded((G).tp, t, j, i)
__device__ __forceinline__ bool live(const int* K, int in, int k) { return k < K[in]; }

// r = b_n - A x0_n and x = x0_n on the interior, b_n = b cg2dNorm rhsNorm (cg2d.py:221-232)
__global__ void k_init(Geo G, const double* aW, const double* aS, const double* aC, const double* b, const double* x0,
                       const double* norm, const double* rn, double* r, double* x) {
  POINT(G, in, t, j, i, p);
  const TopoDev& tp = G.tp;
  const double* x0i = x0 + (long long)in * G.pe;
  const double rni = rn[in];
  const double vc = nbx0(tp, x0i, rni, t, j, i);
  const double ax = opA(aW[p], aW[p + 1], aS[p], aS[p + tp.npx], aC[p], nbx0(tp, x0i, rni, t, j, i - 1),
                        nbx0(tp, x0i, rni, t, j, i + 1), nbx0(tp, x0i, rni, t, j - 1, i),
                        nbx0(tp, x0i, rni, t, j + 1, i), vc);
  r[p] = sub(mul(mul(b[p], norm[in]), rni), ax);
  x[p] = vc;
}

// row sums of up to two products a0 b0, a1 b1 of live instances: rs[(in 2 + q)][t nj + j], one warp per row,
// lane partials over i = lane + 32 m in order, then an xor butterfly (the solver's ROWBLOCK row sums)
__global__ void k_rowdot(Geo G, const double* a0, const double* b0, const double* a1, const double* b1, double* rs,
                         const int* K, int k) {
  const int lane = threadIdx.x & 31;
  const int rows = G.tp.T * G.tp.nj;
  const int in = blockIdx.y;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= rows || !live(K, in, k)) return;
  const int t = row / G.tp.nj, j = row - t * G.tp.nj;
  const long long p0 = (long long)in * G.pe + padded(G.tp, t, j, 0);
  double s0 = 0.0, s1 = 0.0;
  for (int i = lane; i < G.tp.ni; i += 32) {
    s0 = add(s0, mul(a0[p0 + i], b0[p0 + i]));
    if (a1) s1 = add(s1, mul(a1[p0 + i], b1[p0 + i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 = add(s0, __shfl_xor_sync(0xffffffffu, s0, o));
    s1 = add(s1, __shfl_xor_sync(0xffffffffu, s1, o));
  }
  if (lane == 0) {
    rs[((long long)in * 2 + 0) * rows + row] = s0;
    if (a1) rs[((long long)in * 2 + 1) * rows + row] = s1;
  }
}

// The sum of an instance's row sums in ROWBLOCK order (rows of a block of R in order, blocks of a tile in order,
// tiles in order from 0), by the whole thread block: the block sums in parallel, then the tile sums, then the
// total -- the same additions in the same order as one thread summing row by row. sh holds T (ceil(nj / R) + 1)
// doubles. The result is valid in thread 0.
__device__ double fold(const Geo& G, int R, const double* rs, double* sh) {
  const int T = G.tp.T, nj = G.tp.nj, nb = (nj + R - 1) / R;
  for (int u = threadIdx.x; u < T * nb; u += blockDim.x) {
    const int t = u / nb, j0 = (u - t * nb) * R, j1 = min(nj, j0 + R);
    double v = 0.0;
    for (int j = j0; j < j1; ++j) v = add(v, rs[t * nj + j]);
    sh[u] = v;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < T; t += blockDim.x) {
    double ts = 0.0;
    for (int b = 0; b < nb; ++b) ts = add(ts, sh[t * nb + b]);
    sh[T * nb + t] = ts;
  }
  __syncthreads();
  double total = 0.0;
  if (threadIdx.x == 0)
    for (int t = 0; t < T; ++t) total = add(total, sh[T * nb + t]);
  __syncthreads();   // sh may be reused by a second fold
  return total;
}

// The folds of rs0 and rs1 side by side, by the whole thread block: the same additions in the same order as two
// calls of fold, with both sets of block sums and tile sums formed at once and the two totals by two warps. sh holds
// 2 T (ceil(nj / R) + 1) doubles. Both totals are valid in thread 0.
__device__ void fold2(const Geo& G, int R, const double* rs0, const double* rs1, double* sh, double& f0, double& f1) {
  const int T = G.tp.T, nj = G.tp.nj, nb = (nj + R - 1) / R, per = T * (nb + 1);
  for (int u = threadIdx.x; u < 2 * T * nb; u += blockDim.x) {
    const int q = u >= T * nb, w = u - q * T * nb;
    const int t = w / nb, j0 = (w - t * nb) * R, j1 = min(nj, j0 + R);
    const double* rs = q ? rs1 : rs0;
    double v = 0.0;
    for (int j = j0; j < j1; ++j) v = add(v, rs[t * nj + j]);
    sh[q * per + w] = v;
  }
  __syncthreads();
  for (int u = threadIdx.x; u < 2 * T; u += blockDim.x) {
    const int q = u >= T, t = u - q * T;
    double ts = 0.0;
    for (int b = 0; b < nb; ++b) ts = add(ts, sh[q * per + t * nb + b]);
    sh[q * per + T * nb + t] = ts;
  }
  __syncthreads();
  const int q = threadIdx.x == 0 ? 0 : (threadIdx.x == 32 ? 1 : -1);
  double total = 0.0;
  if (q >= 0)
    for (int t = 0; t < T; ++t) total = add(total, sh[q * per + T * nb + t]);
  __syncthreads();
  if (q == 1) sh[0] = total;
  __syncthreads();
  f0 = total;
  f1 = sh[0];
}

// per-instance scalar steps, one thread block per instance (blockIdx.x), thread 0 updating the scalars;
// S = scalar arrays [kind][Kmax][batch]
struct Scal {
  double *eta, *beta, *sig, *alpha;   // [Kmax][batch] (recorded)
  double *carry, *etabar, *sigbar;    // [batch] (reverse)
};
__global__ void k_fwd_eta(Geo G, int R, const double* rs, Scal S, const int* K, int k) {
  extern __shared__ double sh[];
  const int in = blockIdx.x;
  if (!live(K, in, k)) return;
  const int rows = G.tp.T * G.tp.nj;
  const double eta = fold(G, R, rs + (long long)in * 2 * rows, sh);              // cg2d.py:246
  if (threadIdx.x != 0) return;
  const double eta_prev = k > 0 ? S.eta[(long long)(k - 1) * G.batch + in] : 1.0;
  S.eta[(long long)k * G.batch + in] = eta;
  S.beta[(long long)k * G.batch + in] = __ddiv_rn(eta, eta_prev);             // cg2d.py:247
}
__global__ void k_fwd_sigma(Geo G, int R, const double* rs, Scal S, const int* K, int k) {
  extern __shared__ double sh[];
  const int in = blockIdx.x;
  if (!live(K, in, k)) return;
  const int rows = G.tp.T * G.tp.nj;
  const double sig = fold(G, R, rs + (long long)in * 2 * rows, sh);              // cg2d.py:252
  if (threadIdx.x != 0) return;
  S.sig[(long long)k * G.batch + in] = sig;
  S.alpha[(long long)k * G.batch + in] = __ddiv_rn(S.eta[(long long)k * G.batch + in], sig);   // cg2d.py:253
}
// reverse: abar = <xbar, s> - <rbar, q>
__global__ void k_rev_alpha(Geo G, int R, const double* rs, Scal S, const int* K, int k) {
  extern __shared__ double sh[];
  const int in = blockIdx.x;
  if (!live(K, in, k)) return;
  const int rows = G.tp.T * G.tp.nj;
  double f0, f1;
  fold2(G, R, rs + (long long)in * 2 * rows, rs + ((long long)in * 2 + 1) * rows, sh, f0, f1);
  if (threadIdx.x != 0) return;
  const double abar = f0 - f1;
  const long long o = (long long)k * G.batch + in;
  S.sigbar[in] = -abar * S.alpha[o] / S.sig[o];
  S.etabar[in] = S.carry[in] + abar / S.sig[o];
}
// reverse: bbar = <sbar, s_prev>
__global__ void k_rev_beta(Geo G, int R, const double* rs, Scal S, const int* K, int k) {
  extern __shared__ double sh[];
  const int in = blockIdx.x;
  if (!live(K, in, k)) return;
  if (k == 0) {   // eta_{-1} = 1 is a constant, s_{-1} = 0
    if (threadIdx.x == 0) S.carry[in] = 0.0;
    return;
  }
  const int rows = G.tp.T * G.tp.nj;
  const double bbar = fold(G, R, rs + (long long)in * 2 * rows, sh);
  if (threadIdx.x != 0) return;
  const double eta = S.eta[(long long)k * G.batch + in], etap = S.eta[(long long)(k - 1) * G.batch + in];
  S.etabar[in] += bbar / etap;
  S.carry[in] = -bbar * eta / (etap * etap);
}

// ---- fused iteration kernels: one thread per interior point (POINT layout), the whole block returning together
// when its instance (blockIdx.y) takes no part, so that the row sums may synchronise the block

#define POINT_IN(G)                                                                       \
  const TopoDev& tp = (G).tp;                                                             \
  const int i = threadIdx.x, in = blockIdx.y;                                             \
  const int row = blockIdx.x * blockDim.y + threadIdx.y;                                  \
  const bool inb = i < tp.ni && row < tp.T * tp.nj;                                       \
  const int t = inb ? row / tp.nj : 0, j = inb ? row - t * tp.nj : 0;                     \
  const long long base = (long long)in * (G).pe;                                          \
  const int off = ((t * tp.npy + j + tp.OLy) * tp.npx) + i + tp.OLx;                      \
  const long long p = base + off;                                                         \
  int ow = -1, oe = -1, os = -1, on = -1;                                                 \
  if (inb) neighbours(G, t, j, i, off, ow, oe, os, on)

// padded offsets (in the instance) of the west, east, south and north neighbours of interior point (t, j, i) at
// offset off, as the exchange supplies them: the next point in the tile, or across a tile edge the source the
// exch2 map names (-1: unwritten, reads 0)
__device__ __forceinline__ void neighbours(const Geo& G, int t, int j, int i, int off, int& ow, int& oe, int& os,
                                           int& on) {
  const TopoDev& tp = G.tp;
  const int T = tp.T, nj = tp.nj, ni = tp.ni;
  ow = i > 0 ? off - 1 : G.nbp[t * nj + j];
  oe = i < ni - 1 ? off + 1 : G.nbp[T * nj + t * nj + j];
  os = j > 0 ? off - tp.npx : G.nbp[2 * T * nj + t * ni + i];
  on = j < nj - 1 ? off + tp.npx : G.nbp[2 * T * nj + T * ni + t * ni + i];
}

// Iteration kernels march over rows: thread (x, y) of a block takes point i = x of the rows
// row0 + h blockDim.y + y, h = 0 .. kRows - 1, row0 = blockIdx.x blockDim.y kRows, so that the instance check, the
// iteration's scalars and the block's row-sum tail are paid once per kRows rows.
constexpr int kRows = 4;

// one row of the march: the point (t, j, i) and its neighbours' padded offsets in the instance
#define ROW_POINT(G, row)                                                                 \
  const bool inb = i < tp.ni && (row) < tp.T * tp.nj;                                     \
  const int t = inb ? (row) / tp.nj : 0, j = inb ? (row) - t * tp.nj : 0;                 \
  const int off = ((t * tp.npy + j + tp.OLy) * tp.npx) + i + tp.OLx;                      \
  const long long p = base + off;                                                         \
  int ow = -1, oe = -1, os = -1, on = -1;                                                 \
  if (inb) neighbours(G, t, j, i, off, ow, oe, os, on)

// The row products of march step h (q: which product) go through shared memory, [2][kRows][blockDim.y][blockDim.x]
// doubles; points outside the tile store 0
__device__ __forceinline__ void put_prod(int q, int h, double v) {
  extern __shared__ double shp[];
  shp[((q * kRows + h) * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x] = v;
}
// Row sums of the block's rows, in k_rowdot's order: lane partials over i = lane + 32 m in order, then the xor
// butterfly; the first warp of thread row y sums the rows it marched over. Every thread of the block calls it.
__device__ void row_sums(const Geo& G, int in, int row0, int nq, double* rs) {
  extern __shared__ double shp[];
  __syncthreads();
  const int bx = blockDim.x, by = blockDim.y, x = threadIdx.x, y = threadIdx.y;
  const int rows = G.tp.T * G.tp.nj;
  if (x >= 32) return;
  for (int h = 0; h < kRows; ++h) {
    const int row = row0 + h * by + y;
    if (row >= rows) break;
    for (int q = 0; q < nq; ++q) {
      const double* sp_ = shp + ((q * kRows + h) * by + y) * bx;
      double v = 0.0;
      for (int ii = x; ii < G.tp.ni; ii += 32) v = add(v, sp_[ii]);
      for (int o = 16; o > 0; o >>= 1) v = add(v, __shfl_xor_sync(0xffffffffu, v, o));
      if (x == 0) rs[((long long)in * 2 + q) * rows + row] = v;
    }
  }
}

#define MARCH_BEGIN                                                                       \
  const TopoDev& tp = G.tp;                                                               \
  const int i = threadIdx.x, in = blockIdx.y;                                             \
  const long long base = (long long)in * G.pe;                                            \
  const int row0 = blockIdx.x * blockDim.y * kRows;                                       \
  for (int h = 0; h < kRows; ++h) {                                                       \
    const int row = row0 + h * blockDim.y + threadIdx.y;                                  \
    ROW_POINT(G, row);

// Iteration k, first half, with the updates of iteration k-1 (upd, k >= 1):
//   r_k = r_{k-1} - alpha_{k-1} q_{k-1}  (cg2d.py:255; written to rout when non-null),
//   x += alpha_{k-1} s_{k-1}              (cg2d.py:254; when x is non-null),
//   z_k = M r_k (cg2d.py:245), the row sums of z_k r_k (cg2d.py:246; when rs is non-null),
//   checkpoints of r_k and s_{k-1} (when ckr / cks are non-null).
// Without upd, r_k is rp itself. r_k at a neighbour is formed from that neighbour's r_{k-1} and q_{k-1}: the
// value its owner computes, as the exchange of r gives it (cg2d.py:260). The updates of iteration k-1 run for
// instances that took it (k - 1 < K), the rest for instances that take iteration k.
__global__ void k_fa(Geo G, const double* __restrict__ pW, const double* __restrict__ pS,
                     const double* __restrict__ pC, const double* __restrict__ rp, const double* __restrict__ qp,
                     const double* __restrict__ sp, double* __restrict__ x, double* __restrict__ rout,
                     double* __restrict__ z, double* __restrict__ ckr, double* __restrict__ cks,
                     double* __restrict__ rs, Scal S, const int* __restrict__ K, int k, int upd) {
  const int Kin = K[blockIdx.y];
  const bool zl = k < Kin, ul = upd && k - 1 < Kin;
  if (!zl && !ul) return;
  const double a = ul ? S.alpha[(long long)(k - 1) * G.batch + blockIdx.y] : 0.0;
  MARCH_BEGIN
    auto R = [&](int o) -> double {
      if (o < 0) return 0.0;
      return upd ? sub(rp[base + o], mul(a, qp[base + o])) : rp[base + o];
    };
    double prod = 0.0;
    if (inb) {
      const double rc = R(off);
      if (ul && rout) rout[p] = rc;
      if (ul && x) x[p] = add(x[p], mul(a, sp[p]));
      if (zl) {
        if (ckr) ckr[p] = rc;
        if (cks) cks[p] = sp[p];
        const double zc = opM(pC[p], pW[p], pW[p + 1], pS[p], pS[p + tp.npx], rc, R(ow), R(oe), R(os), R(on));
        z[p] = zc;
        prod = mul(zc, rc);
      }
    }
    if (rs && zl) put_prod(0, h, prod);
  }
  if (rs && zl) row_sums(G, in, row0, 1, rs);
}

// Iteration k, second half: s_k = z_k + beta_k s_{k-1} (cg2d.py:249), q_k = A s_k (cg2d.py:251), the row sums of
// s_k q_k (cg2d.py:252; when rs is non-null). s_k at a neighbour is formed from that neighbour's z_k and s_{k-1}.
__global__ void k_fb(Geo G, const double* __restrict__ aW, const double* __restrict__ aS,
                     const double* __restrict__ aC, const double* __restrict__ z, const double* __restrict__ sp,
                     double* __restrict__ s, double* __restrict__ q, double* __restrict__ rs, Scal S,
                     const int* __restrict__ K, int k) {
  if (k >= K[blockIdx.y]) return;
  const double beta = S.beta[(long long)k * G.batch + blockIdx.y];
  MARCH_BEGIN
    auto Sv = [&](int o) -> double { return o < 0 ? 0.0 : add(z[base + o], mul(beta, sp[base + o])); };
    double prod = 0.0;
    if (inb) {
      const double sc = Sv(off);
      const double qc = opA(aW[p], aW[p + 1], aS[p], aS[p + tp.npx], aC[p], Sv(ow), Sv(oe), Sv(os), Sv(on), sc);
      s[p] = sc;
      q[p] = qc;
      prod = mul(sc, qc);
    }
    if (rs) put_prod(0, h, prod);
  }
  if (rs) row_sums(G, in, row0, 1, rs);
}

// Reverse of iteration k, first half. With qbar = sigbar s_k - alpha_k rbar (formed at each stencil point):
//   sbar = bs sbar + alpha_k xbar + sigbar q_k + A qbar, bs = beta_{k+1} (the scaling of sbar left from the
//   reverse of iteration k+1; none when k + 1 = K), and the row sums of sbar s_{k-1}. qbar is stored (qb) for the
//   segment's edge products (k_seg_edges).
__global__ void k_rq(Geo G, const double* __restrict__ aW, const double* __restrict__ aS,
                     const double* __restrict__ aC, const double* __restrict__ s, const double* __restrict__ q,
                     const double* __restrict__ xbar, const double* __restrict__ rbar, double* __restrict__ sbar,
                     const double* __restrict__ sp, double* __restrict__ qb, double* __restrict__ rs, Scal S,
                     const int* __restrict__ K, int k) {
  const int Kin = K[blockIdx.y];
  if (k >= Kin) return;
  const long long o_ = (long long)k * G.batch + blockIdx.y;
  const double a = S.alpha[o_], sg = S.sigbar[blockIdx.y];
  const bool scale = k + 1 < Kin;
  const double bs = scale ? S.beta[o_ + G.batch] : 0.0;
  MARCH_BEGIN
    auto SV = [&](int o) -> double { return o < 0 ? 0.0 : s[base + o]; };
    auto RB = [&](int o) -> double { return o < 0 ? 0.0 : rbar[base + o]; };
    double prod = 0.0;
    if (inb) {
      const double sc = SV(off), sw = SV(ow), se = SV(oe), ss = SV(os), sn = SV(on);
      auto QB = [&](double sv, double rv) -> double { return sub(mul(sg, sv), mul(a, rv)); };
      const double qc = QB(sc, RB(off)), qw = QB(sw, RB(ow)), qe = QB(se, RB(oe)), qs = QB(ss, RB(os)),
                   qn = QB(sn, RB(on));
      double sb = scale ? mul(bs, sbar[p]) : sbar[p];
      sb = add(add(sb, mul(a, xbar[p])), mul(sg, q[p]));
      sb = add(sb, opA(aW[p], aW[p + 1], aS[p], aS[p + tp.npx], aC[p], qw, qe, qs, qn, qc));
      sbar[p] = sb;
      qb[p] = qc;
      prod = mul(sb, sp[p]);
    }
    put_prod(0, h, prod);
  }
  row_sums(G, in, row0, 1, rs);
}

// Reverse of iteration k, second half. With zbar = sbar + etabar r_k (formed at each stencil point):
//   rbar += etabar z_k + M zbar, zbar stored (zb) for the segment's edge products; and, when s1 / q1 (s_{k-1},
//   q_{k-1}) are given, the row sums
//   of xbar s_{k-1} and rbar q_{k-1} for the reverse of iteration k-1. Those row sums are also formed for the
//   instances whose last iteration is k-1 (K = k): their reverse starts there, with rbar still 0.
__global__ void k_rz(Geo G, const double* __restrict__ pW, const double* __restrict__ pS,
                     const double* __restrict__ pC, const double* __restrict__ r, const double* __restrict__ z,
                     const double* __restrict__ sbar, double* __restrict__ rbar, double* __restrict__ zb,
                     const double* __restrict__ xbar, const double* __restrict__ s1, const double* __restrict__ q1,
                     double* __restrict__ rs, Scal S, const int* __restrict__ K, int k) {
  const int Kin = K[blockIdx.y];
  const bool live = k < Kin, next = s1 != nullptr && k - 1 < Kin;
  if (!live && !next) return;
  const double e = live ? S.etabar[blockIdx.y] : 0.0;
  MARCH_BEGIN
    auto RV = [&](int o) -> double { return o < 0 ? 0.0 : r[base + o]; };
    auto SB = [&](int o) -> double { return o < 0 ? 0.0 : sbar[base + o]; };
    double p0 = 0.0, p1 = 0.0;
    if (inb) {
      double rb = rbar[p];
      if (live) {
        const double rc = RV(off), rw = RV(ow), re = RV(oe), rs_ = RV(os), rn_ = RV(on);
        auto ZB = [&](double sv, double rv) -> double { return add(sv, mul(e, rv)); };
        const double zc = ZB(SB(off), rc), zw = ZB(SB(ow), rw), ze = ZB(SB(oe), re), zs = ZB(SB(os), rs_),
                     zn = ZB(SB(on), rn_);
        rb = add(rb, mul(e, z[p]));
        rb = add(rb, opM(pC[p], pW[p], pW[p + 1], pS[p], pS[p + tp.npx], zc, zw, ze, zs, zn));
        rbar[p] = rb;
        zb[p] = zc;
      }
      if (next) {
        p0 = mul(xbar[p], s1[p]);
        p1 = mul(rb, q1[p]);
      }
    }
    if (next) {
      put_prod(0, h, p0);
      put_prod(1, h, p1);
    }
  }
  if (next) row_sums(G, in, row0, 2, rs);
}

// The edge products of one segment (iterations c0 .. c0 + len - 1) for one operator, added to its coefficient
// cotangents once per point: gA += qbar_k (x) s_k (M false) or gM += zbar_k (x) r_k (M true) for k from the last
// iteration down, the same terms in the same order as adding them one iteration at a time: the west and south faces
// of the point, its diagonal entry, and the east / north halo face when the point is the last of its row / column
// (the faces edge_products_kernel writes). The cotangent u_m (qbar_m or zbar_m) is at u0 + m vstr; the stencil
// input (s_m or r_m) at v0 + m sstr for s, and for r at v0 (m = 0, the checkpoint) and v1 + m sstr (m >= 1).
// The two operators run as two launches, so that each thread holds one set of accumulators (more CTAs per SM).
template <bool M>
__global__ void k_seg_edges(Geo G, int c0, int len, const double* __restrict__ u0, long long vstr,
                            const double* __restrict__ v0, const double* __restrict__ v1, long long sstr,
                            double* __restrict__ gW, double* __restrict__ gS, double* __restrict__ gC,
                            const int* __restrict__ K) {
  const int Kin = K[blockIdx.y];
  if (c0 >= Kin) return;
  POINT_IN(G);
  if (!inb) return;
  const bool ie = i == tp.ni - 1, jn = j == tp.nj - 1;
  const long long pe_ = p + 1, pn_ = p + tp.npx;
  double aw = gW[p], as = gS[p], ac = gC[p], ae = ie ? gW[pe_] : 0.0, an = jn ? gS[pn_] : 0.0;
  // iterations c0 + m < K only: m runs from min(len, K - c0) - 1 down, with no test inside, so that the loads of
  // the next iterations are issued ahead of the additions (which stay in order)
#pragma unroll 2
  for (int m = min(len, Kin - c0) - 1; m >= 0; --m) {
    const double* u = u0 + m * vstr + base;
    const double* v = (M ? (m == 0 ? v0 : v1 + m * sstr) : v0 + m * sstr) + base;
    auto V = [&](int o) -> double { return o < 0 ? 0.0 : v[o]; };
    const double uc = u[off], vc = v[off];
    aw = aw + add(mul(uc, V(ow)), i >= 1 ? mul(u[off - 1], vc) : 0.0);
    as = as + add(mul(uc, V(os)), j >= 1 ? mul(u[off - tp.npx], vc) : 0.0);
    ac = ac + mul(uc, vc);
    if (ie) ae = ae + mul(uc, V(oe));
    if (jn) an = an + mul(uc, V(on));
  }
  gW[p] = aw; gS[p] = as; gC[p] = ac;
  if (ie) gW[pe_] = ae;
  if (jn) gS[pn_] = an;
}

// coefficient cotangents of a stencil application out = C v: gW/gS/gC += sign (u (x) v) on the faces and points
// of live instances, u the cotangent of out (interior), v the stencil input as the stencil read it (X0: the
// first-guess rule); the same faces as edge_products_kernel. One thread per (j, i), 0 <= j <= nj, 0 <= i <= ni.
template <bool X0>
__global__ void k_edges(Geo G, const double* u, const double* v, const double* rn, double sign, double* gW,
                        double* gS, double* gC, const int* K, int k) {
  const TopoDev& tp = G.tp;
  const int i = threadIdx.x, in = blockIdx.y;
  const int row = blockIdx.x * blockDim.y + threadIdx.y;
  if (i > tp.ni || row >= tp.T * (tp.nj + 1)) return;
  if (K && !live(K, in, k)) return;
  const int t = row / (tp.nj + 1), j = row - t * (tp.nj + 1);
  const long long idx = (long long)in * G.pe + padded(tp, t, j, i);
  const double* ui = u + (long long)in * G.pe;
  const double* vi = v + (long long)in * G.pe;
  auto V = [&](int jj, int ii) -> double {
    return X0 ? nbx0(tp, vi, rn[in], t, jj, ii) : nbv(tp, vi, t, jj, ii);
  };
  auto U = [&](int jj, int ii) -> double { return ui[padded(tp, t, jj, ii)]; };
  const bool jin = j < tp.nj, iin = i < tp.ni;
  if (jin) {   // face between (j, i-1) and (j, i)
    double a = 0.0;
    if (i < tp.ni) a += U(j, i) * V(j, i - 1);
    if (i >= 1) a += U(j, i - 1) * V(j, i);
    gW[idx] += sign * a;
  }
  if (iin) {   // face between (j-1, i) and (j, i)
    double a = 0.0;
    if (j < tp.nj) a += U(j, i) * V(j - 1, i);
    if (j >= 1) a += U(j - 1, i) * V(j, i);
    gS[idx] += sign * a;
  }
  if (jin && iin) gC[idx] += sign * U(j, i) * V(j, i);
}

// xbar_K = xbar_out / rhsNorm on the interior;  bbar = rbar_0 cg2dNorm rhsNorm on the interior
__global__ void k_scale(Geo G, const double* in_, const double* norm, const double* rn, double* out, int mode) {
  POINT(G, in, t, j, i, p);
  out[p] = mode == 0 ? in_[p] / rn[in] : in_[p] * norm[in] * rn[in];
}
// x_out of the recording forward: x / rhsNorm on the interior (cg2d.py:266)
__global__ void k_xout(Geo G, const double* x, const double* rn, double* out) {
  POINT(G, in, t, j, i, p);
  out[p] = __ddiv_rn(x[p], rn[in]);
}
// alpha, beta, eta, sigma of every iteration from a forward solve's sum history (one group of one right-hand side:
// solve index = instance): eta_0 = z.r of the first Z pass, eta_k (k >= 1) = z.r of pass X_{k-1}, sigma_k = s.q
// of pass S_k; beta_k = eta_k / eta_{k-1} (eta_{-1} = 1) and alpha_k = eta_k / sigma_k with the solver's divisions
// One thread block per instance (blockIdx.x), its threads over the iterations: every k is independent, since
// eta_{k-1} is read from the history rather than carried.
__global__ void k_hist_scalars(Geo G, const double* hist, int hist_len, Scal S, const int* K) {
  const int in = blockIdx.x;
  const double* h = hist + (size_t)in * H_NKIND * hist_len;
  auto eta_of = [&](int k) { return k == 0 ? h[(size_t)H_ETAZ * hist_len] : h[(size_t)H_ETAX * hist_len + k]; };
  for (int k = threadIdx.x; k < K[in]; k += blockDim.x) {
    const double eta = eta_of(k), eta_prev = k > 0 ? eta_of(k - 1) : 1.0;
    const double sig = h[(size_t)H_SQ * hist_len + k];
    const long long o = (long long)k * G.batch + in;
    S.eta[o] = eta;
    S.beta[o] = __ddiv_rn(eta, eta_prev);
    S.sig[o] = sig;
    S.alpha[o] = __ddiv_rn(eta, sig);
  }
}

// per-instance rhsNorm from the forward's rhsMax (cg2d.py:225) and cg2dNorm, iteration counts
__global__ void k_setup(int batch, const cg2d_diag_t* diag, double norm, const double* norm_arr, double* rn,
                        double* nrm, int* K) {
  const int in = blockIdx.x * blockDim.x + threadIdx.x;
  if (in >= batch) return;
  const double m = diag[in].rhsMax;
  rn[in] = (m != 0.0) ? __ddiv_rn(1.0, m) : 1.0;
  nrm[in] = norm_arr ? norm_arr[in] : norm;
  K[in] = diag[in].numIters;
}


}  // namespace

size_t exact_adjoint_workspace(const TopoDev& tp, int batch, int max_iters, int checkpoint) {
  const size_t pe = (size_t)tp.T * tp.npy * tp.npx, vec = pe * batch * sizeof(double);
  const int C = checkpoint > 0 ? checkpoint : std::max(1, max_iters);
  const int nseg = (max_iters + C - 1) / C;
  const size_t rows = (size_t)tp.T * tp.nj;
  size_t b = 0;
  b += vec * 5;                                   // r, s, z, q, x of the recording forward
  b += vec * 2 * (size_t)(std::max(1, nseg) + 1); // checkpoints r_c, s_{c-1}; one slot more for a forward that
                                                  // records at its last iteration
  b += vec * 6 * (size_t)C;                       // a segment's r, z, s, q, qbar, zbar
  b += vec * 3;                                   // xbar, rbar, sbar
  b += sizeof(double) * batch * 2 * rows;         // row sums
  b += sizeof(double) * ((size_t)4 * std::max(1, max_iters) * batch + 5 * batch);   // scalars, rn, norm
  b += sizeof(int) * batch;
  b += sizeof(int) * 2 * (size_t)tp.T * (tp.nj + tp.ni);   // padded-offset neighbour table
  b += 256 * (size_t)(35 + 2 * std::max(1, nseg) + 6 * C);   // each buffer starts 256-byte aligned
  return b;
}

void exact_checkpoints(const TopoDev& tp, int batch, int max_iters, int checkpoint, void* ws, double** ck_r0,
                       double** ck_s0, long long* stride) {
  const size_t vecn = (size_t)tp.T * tp.npy * tp.npx * batch;
  const size_t vstride = (vecn * sizeof(double) + 255) & ~size_t(255);
  const int C = checkpoint > 0 ? checkpoint : std::max(1, max_iters);
  const int nck = std::max(1, (max_iters + C - 1) / C) + 1;
  char* base = static_cast<char*>(ws) + 5 * vstride;   // after r, s, z, q, x (exact_adjoint's carve)
  *ck_r0 = reinterpret_cast<double*>(base);
  *ck_s0 = reinterpret_cast<double*>(base + nck * vstride);
  *stride = (long long)(vstride / sizeof(double));
}

cudaError_t exact_adjoint(const TopoDev& tp, const ExactArgs& A, void* ws, cudaStream_t st) {
  Geo G;
  G.tp = tp;
  G.batch = A.batch;
  G.pe = (long long)tp.T * tp.npy * tp.npx;
  G.pts = (long long)tp.T * tp.nj * tp.ni;
  const int Kmax = A.max_iters;
  if (A.recorded && (A.x_check || !A.hist)) return cudaErrorInvalidValue;
  const int C = A.checkpoint > 0 ? A.checkpoint : std::max(1, A.recorded ? std::max(A.max_iters_cap, Kmax) : Kmax);
  const int nseg = (Kmax + C - 1) / C;
  const size_t vecn = (size_t)G.pe * A.batch;
  const int rows = tp.T * tp.nj;
  char* w = static_cast<char*>(ws);
  auto take = [&](size_t bytes) { char* p = w; w += (bytes + 255) & ~size_t(255); return p; };
  auto vec = [&]() { return reinterpret_cast<double*>(take(vecn * sizeof(double))); };
  double *r = vec(), *s = vec(), *z = vec(), *q = vec(), *x = vec();
  // checkpoint blocks: r_c and s_{c-1} for c = 0 .. cap / C, carved from the capacity (a recording forward stores
  // into them before the iteration counts are known); exact_checkpoints gives the same addresses
  const int cap = std::max(A.max_iters_cap, Kmax);
  const int nck = std::max(1, (cap + C - 1) / C) + 1;
  const size_t vstride = (vecn * sizeof(double) + 255) & ~size_t(255);
  char* ckr0 = take(vstride * nck);
  char* cks0 = take(vstride * nck);
  std::vector<double*> ck_r(nck), ck_s(nck);
  for (int c = 0; c < nck; ++c) {
    ck_r[c] = reinterpret_cast<double*>(ckr0 + c * vstride);
    ck_s[c] = reinterpret_cast<double*>(cks0 + c * vstride);
  }
  std::vector<double*> sg_r(C), sg_z(C), sg_s(C), sg_q(C);
  for (int c = 0; c < C; ++c) { sg_r[c] = vec(); sg_z[c] = vec(); sg_s[c] = vec(); sg_q[c] = vec(); }
  // qbar_m, zbar_m of the segment being reversed (edge products added once per segment)
  double* qb0 = reinterpret_cast<double*>(take(vstride * C));
  double* zb0 = reinterpret_cast<double*>(take(vstride * C));
  const long long vstr = (long long)(vstride / sizeof(double)), sstr = 4 * vstr;
  double *xbar = vec(), *rbar = vec(), *sbar = vec();
  double* rs = reinterpret_cast<double*>(take(sizeof(double) * A.batch * 2 * rows));
  Scal S;
  const size_t kb = (size_t)std::max(1, Kmax) * A.batch * sizeof(double);
  S.eta = reinterpret_cast<double*>(take(kb));
  S.beta = reinterpret_cast<double*>(take(kb));
  S.sig = reinterpret_cast<double*>(take(kb));
  S.alpha = reinterpret_cast<double*>(take(kb));
  S.carry = reinterpret_cast<double*>(take(sizeof(double) * A.batch));
  S.etabar = reinterpret_cast<double*>(take(sizeof(double) * A.batch));
  S.sigbar = reinterpret_cast<double*>(take(sizeof(double) * A.batch));
  double* rn = reinterpret_cast<double*>(take(sizeof(double) * A.batch));
  double* nrm = reinterpret_cast<double*>(take(sizeof(double) * A.batch));
  int* K = reinterpret_cast<int*>(take(sizeof(int) * A.batch));
  int* nbp = reinterpret_cast<int*>(take(sizeof(int) * 2 * (size_t)tp.T * (tp.nj + tp.ni)));
  G.nbp = nbp;

  // point kernels: a row of ni threads (rounded up to whole warps) per threadIdx.y; face kernels the same over
  // ni + 1 faces and nj + 1 face rows; row sums one warp per row; scalar steps one block per instance
  const int bxp = 32 * ((tp.ni + 31) / 32), bxe = 32 * ((tp.ni + 1 + 31) / 32);
  if (bxe > 1024 || A.batch > 65535) return cudaErrorInvalidValue;
  const dim3 bp(bxp, std::max(1, 384 / bxp)), be(bxe, std::max(1, 384 / bxe));
  const dim3 gp((rows + bp.y - 1) / bp.y, A.batch), ge((tp.T * (tp.nj + 1) + be.y - 1) / be.y, A.batch);
  const dim3 gm((rows + bp.y * kRows - 1) / (bp.y * kRows), A.batch);   // the marching iteration kernels
  const dim3 gw((rows + 7) / 8, A.batch);
  const int gi = (A.batch + 127) / 128, nbk = (tp.nj + A.rows_per_block - 1) / A.rows_per_block;
  const size_t fold_sh = sizeof(double) * (size_t)tp.T * (nbk + 1);
  const size_t row_sh = sizeof(double) * 2 * kRows * bp.x * bp.y;   // row_sums: two products per point
  if (fold_sh > 24 * 1024) return cudaErrorInvalidValue;   // (k_rev_alpha takes two side by side)
  const size_t vb = vecn * sizeof(double);
  cudaError_t e;
#define CK(x)                              \
  do {                                     \
    if ((e = (x)) != cudaSuccess) return e; \
  } while (0)
#define LK()                                  \
  do {                                        \
    if ((e = cudaGetLastError()) != cudaSuccess) return e; \
  } while (0)
  CK(cudaMemsetAsync(s, 0, vb, st));          // s_{-1} = 0
  for (double* g : {A.gW, A.gS, A.gC, A.gpW, A.gpS, A.gpC, A.b_bar}) CK(cudaMemsetAsync(g, 0, vb, st));
  for (double* v : {xbar, rbar, sbar}) CK(cudaMemsetAsync(v, 0, vb, st));
  CK(cudaMemsetAsync(S.carry, 0, sizeof(double) * A.batch, st));
  k_setup<<<gi, 128, 0, st>>>(A.batch, A.fwd_diag, A.norm, A.norm_arr, rn, nrm, K);
  LK();
  k_nbp<<<(2 * tp.T * (tp.nj + tp.ni) + 255) / 256, 256, 0, st>>>(tp, nbp);
  LK();
  if (A.recorded) {
    // the forward solve stored r_c and s_{c-1} for c >= 1 and kept its sums: r_0 and s_{-1} = 0 here, alpha and
    // beta rebuilt from the sums with the solver's own divisions
    CK(cudaMemsetAsync(ck_s[0], 0, vb, st));
    k_init<<<gp, bp, 0, st>>>(G, A.aW, A.aS, A.aC, A.b, A.x0, nrm, rn, ck_r[0], x);
    LK();
    k_hist_scalars<<<A.batch, 256, 0, st>>>(G, A.hist, A.hist_len, S, K);
    LK();
  } else {
    k_init<<<gp, bp, 0, st>>>(G, A.aW, A.aS, A.aC, A.b, A.x0, nrm, rn, r, x);
    LK();
  }

  // ---- recording forward: scalars of every iteration, checkpoints of r_k and s_{k-1} every C iterations. r and s
  // alternate between two buffers (a stencil reads its neighbours' old values while every point writes its new
  // one); the second ones borrow the first segment buffers, which the reverse sweep fills later.
  double *rcur = r, *rnext = sg_r[0];
  double *sprev = s, *snew = sg_s[0];
  for (int k = 0; k <= Kmax && !A.recorded; ++k) {
    const bool ck = k < Kmax && k % C == 0;
    if (k == Kmax && !A.x_check) break;   // the last updates only move x
    k_fa<<<gm, bp, row_sh, st>>>(G, A.pW, A.pS, A.pC, rcur, q, sprev, A.x_check ? x : nullptr, rnext, z,
                                 ck ? ck_r[k / C] : nullptr, ck ? ck_s[k / C] : nullptr, k < Kmax ? rs : nullptr,
                                 S, K, k, k > 0);
    LK();
    if (k > 0) std::swap(rcur, rnext);
    if (k == Kmax) break;
    k_fwd_eta<<<A.batch, 256, fold_sh, st>>>(G, A.rows_per_block, rs, S, K, k);
    LK();
    k_fb<<<gm, bp, row_sh, st>>>(G, A.aW, A.aS, A.aC, z, sprev, snew, q, rs, S, K, k);
    LK();
    k_fwd_sigma<<<A.batch, 256, fold_sh, st>>>(G, A.rows_per_block, rs, S, K, k);
    LK();
    std::swap(sprev, snew);
  }
  if (A.x_check) {
    k_xout<<<gp, bp, 0, st>>>(G, x, rn, A.x_check);
    LK();
  }

  // ---- reverse sweep, segment by segment from the last
  k_scale<<<gp, bp, 0, st>>>(G, A.xbar, nrm, rn, xbar, 0);
  LK();
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int c0 = seg * C, c1 = std::min(Kmax, c0 + C), len = c1 - c0;
    auto rr = [&](int m) -> double* { return m == 0 ? ck_r[seg] : sg_r[m]; };
    auto sp = [&](int m) -> double* { return m == 0 ? ck_s[seg] : sg_s[m - 1]; };
    // recompute the segment's r, z, s, q with the recorded alpha and beta (the recording forward's operations)
    for (int m = 0; m < len; ++m) {
      const int k = c0 + m;
      k_fa<<<gm, bp, row_sh, st>>>(G, A.pW, A.pS, A.pC, m == 0 ? ck_r[seg] : rr(m - 1), m == 0 ? nullptr : sg_q[m - 1],
                                   nullptr, nullptr, m == 0 ? nullptr : sg_r[m], sg_z[m], nullptr, nullptr, nullptr,
                                   S, K, k, m > 0);
      LK();
      k_fb<<<gm, bp, row_sh, st>>>(G, A.aW, A.aS, A.aC, sg_z[m], sp(m), sg_s[m], sg_q[m], nullptr, S, K, k);
      LK();
    }
    // the row sums of alphabar for the segment's last iteration (inside a segment k_rz forms them)
    k_rowdot<<<gw, 256, 0, st>>>(G, xbar, sg_s[len - 1], rbar, sg_q[len - 1], rs, K, c1 - 1);
    LK();
    for (int m = len - 1; m >= 0; --m) {
      const int k = c0 + m;
      k_rev_alpha<<<A.batch, 256, 2 * fold_sh, st>>>(G, A.rows_per_block, rs, S, K, k);
      LK();
      k_rq<<<gm, bp, row_sh, st>>>(G, A.aW, A.aS, A.aC, sg_s[m], sg_q[m], xbar, rbar, sbar, sp(m), qb0 + m * vstr,
                                   rs, S, K, k);
      LK();
      k_rev_beta<<<A.batch, 256, fold_sh, st>>>(G, A.rows_per_block, rs, S, K, k);
      LK();
      k_rz<<<gm, bp, row_sh, st>>>(G, A.pW, A.pS, A.pC, rr(m), sg_z[m], sbar, rbar, zb0 + m * vstr, xbar,
                                   m > 0 ? sg_s[m - 1] : nullptr, m > 0 ? sg_q[m - 1] : nullptr, rs, S, K, k);
      LK();
    }
    k_seg_edges<false><<<gp, bp, 0, st>>>(G, c0, len, qb0, vstr, sg_s[0], nullptr, sstr, A.gW, A.gS, A.gC, K);
    LK();
    k_seg_edges<true><<<gp, bp, 0, st>>>(G, c0, len, zb0, vstr, ck_r[seg], sg_r[0], sstr, A.gpW, A.gpS, A.gpC, K);
    LK();
  }
  // r_0 = b_n - A x0_n: the cotangents of b and, through x0_n, of A
  k_scale<<<gp, bp, 0, st>>>(G, rbar, nrm, rn, A.b_bar, 1);
  LK();
  k_edges<true><<<ge, be, 0, st>>>(G, rbar, A.x0, rn, -1.0, A.gW, A.gS, A.gC, nullptr, 0);
  LK();
#undef CK
#undef LK
  return cudaSuccess;
}

}  // namespace cg2d
