// Persistent cooperative CG2D solver for sm_100a.
//
// One launch runs every right-hand side of every instance to convergence. The iteration is the
// preconditioned CG of mitgcm_jax/core/cg2d.py:205-269 (cg2d.F), with the same floating-point
// operations in the same order (products and sums rounded separately, no FMA contraction), so the
// only freedom left is the order of the global sums, which is fixed by cg2d_sum_order_t and is
// independent of the launch geometry.
//
// Data movement per iteration k (per solve), two grid-wide waits:
//   pass S_k : s_k = z_k + beta_k s_{k-1};  q_k = A s_k;  x_k = x_{k-1} + alpha_{k-1} s_{k-1};  sum s_k.q_k
//   pass X_k : r_{k+1} = r_k - alpha_k q_k;  z_{k+1} = M r_{k+1};  sums r.r and z.r
// The stencils need values at the four neighbours of a point; they are recomputed while staging a
// chunk of rows into shared memory (the neighbour's s or r is formed from its z/s or r/q exactly as
// its owner forms it), so no exchange step and no extra wait is needed. Cross-tile neighbours
// (the exch2 halo of cg2d.py:228,235,250,260) are gathered through per-tile-edge tables.
// The x update is deferred by one pass (it needs s_{k-1}, which pass S_k reads anyway); the
// arithmetic is the reference's x_i = x + alpha * s_i (cg2d.py:254).
//
// MIXED precision keeps r, s, z, q and the operator copies in FP32 (FP32 stencils), x and all dot
// products in FP64, and replaces r by the FP64 true residual b - A x every replace_every iterations
// while the residual is above replace_above * tolerance (near the FP64 rounding floor of b - A x a
// replacement would only add noise); the stop rule is the reference's, on the carried residual.

#include <cuda_runtime.h>
#include <cstdint>

#include "cg2d_internal.cuh"

namespace cg2d {

// ------------------------------------------------------------------------------------------------
// arithmetic without contraction (the reference rounds every product and every sum)

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }

// apply_operator (cg2d.py:181-188): aW(i)x(i-1) + aW(i+1)x(i+1) + aS(j)x(j-1) + aS(j+1)x(j+1) + aC x
template <class T>
__device__ __forceinline__ T op_A(T aw, T ae, T as, T an, T ac, T vw, T ve, T vs, T vn, T vc) {
  T t = mul(aw, vw);
  t = add(t, mul(ae, ve));
  t = add(t, mul(as, vs));
  t = add(t, mul(an, vn));
  t = add(t, mul(ac, vc));
  return t;
}

// apply_preconditioner (cg2d.py:191-198): pC r + pW(i)r(i-1) + pW(i+1)r(i+1) + pS(j)r(j-1) + pS(j+1)r(j+1)
template <class T>
__device__ __forceinline__ T op_M(T pc, T pw, T pe, T ps, T pn, T vc, T vw, T ve, T vs, T vn) {
  T t = mul(pc, vc);
  t = add(t, mul(pw, vw));
  t = add(t, mul(pe, ve));
  t = add(t, mul(ps, vs));
  t = add(t, mul(pn, vn));
  return t;
}

template <bool MIXED> struct Prec;
template <> struct Prec<false> { using V = double; using C = double; };
template <> struct Prec<true> { using V = float; using C = float; };

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ void stcg(double* p, double v) { __stcg(p, v); }
__device__ __forceinline__ void stcg(float* p, float v) { __stcg(p, v); }

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ------------------------------------------------------------------------------------------------
// shared memory carve

struct Smem {
  int* act;          // [kMaxSolves] action of each solve in the current pass
  double* c1;        // [kMaxSolves] pass coefficient (beta in S, alpha in X)
  double* c2;        // [kMaxSolves] alpha_{k-1} for the deferred x update
  double* rnorm;     // [kMaxSolves] rhsNorm
  double* norm;      // [kMaxSolves] cg2dNorm
  int* has_alpha;    // [kMaxSolves]
  int* opp;          // [kMaxOps] operator takes part in the pass
  double* rowsum;    // [2 slots][2 kinds][kWarps]
  double* tsum;      // [kMaxTiles]
  int* misc;         // [4]: barrier ok flag, last-arriver flag
  double* stage;     // [2 slots][kWarps + 2][max_ni + 2]
  double* prod;      // FORTRAN order: [2 slots][2 kinds][kWarps][max_ni]
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

size_t smem_bytes(int max_ni, int serial) {
  size_t s = 0;
  s += align16(sizeof(int) * kMaxSolves);
  s += 4 * align16(sizeof(double) * kMaxSolves);
  s += align16(sizeof(int) * kMaxSolves);
  s += align16(sizeof(int) * kMaxOps);
  s += align16(sizeof(double) * 2 * 2 * kWarps);
  s += align16(sizeof(double) * kMaxTiles);
  s += align16(sizeof(int) * 4);
  s += align16(sizeof(double) * 2 * (kWarps + 2) * (size_t)(max_ni + 2));
  if (serial) s += align16(sizeof(double) * 2 * 2 * kWarps * (size_t)max_ni);
  return s;
}

__device__ inline Smem carve(unsigned char* base, int max_ni, int serial) {
  Smem m;
  size_t o = 0;
  m.act = reinterpret_cast<int*>(base + o); o += align16(sizeof(int) * kMaxSolves);
  m.c1 = reinterpret_cast<double*>(base + o); o += align16(sizeof(double) * kMaxSolves);
  m.c2 = reinterpret_cast<double*>(base + o); o += align16(sizeof(double) * kMaxSolves);
  m.rnorm = reinterpret_cast<double*>(base + o); o += align16(sizeof(double) * kMaxSolves);
  m.norm = reinterpret_cast<double*>(base + o); o += align16(sizeof(double) * kMaxSolves);
  m.has_alpha = reinterpret_cast<int*>(base + o); o += align16(sizeof(int) * kMaxSolves);
  m.opp = reinterpret_cast<int*>(base + o); o += align16(sizeof(int) * kMaxOps);
  m.rowsum = reinterpret_cast<double*>(base + o); o += align16(sizeof(double) * 2 * 2 * kWarps);
  m.tsum = reinterpret_cast<double*>(base + o); o += align16(sizeof(double) * kMaxTiles);
  m.misc = reinterpret_cast<int*>(base + o); o += align16(sizeof(int) * 4);
  m.stage = reinterpret_cast<double*>(base + o); o += align16(sizeof(double) * 2 * (kWarps + 2) * (size_t)(max_ni + 2));
  m.prod = serial ? reinterpret_cast<double*>(base + o) : nullptr;
  return m;
}

// ------------------------------------------------------------------------------------------------
// grid-wide wait with a time limit: every CTA arrives once; the wait ends when all have arrived,
// when another CTA has flagged an error, or after timeout_ns (then this CTA flags the error).

__device__ bool grid_barrier(const KParams& kp, unsigned& target, int* flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    target += gridDim.x;
    __threadfence();
    atomicAdd(&kp.gs[0], 1u);
    const unsigned long long t0 = globaltimer();
    int ok = 1;
    for (unsigned spins = 0;; ++spins) {
      const unsigned v = ld_acquire(&kp.gs[0]);
      if ((int)(v - target) >= 0) break;
      if (ld_relaxed(&kp.gs[1]) != 0u) { ok = 0; break; }
      if ((spins & 63u) == 63u && globaltimer() - t0 > kp.timeout_ns) {
        atomicCAS(&kp.gs[1], 0u, (unsigned)CG2D_BARRIER_TIMEOUT);
        ok = 0;
        break;
      }
    }
    __threadfence();
    *flag = ok;
  }
  __syncthreads();
  const int ok = *flag;
  return ok != 0;
}

// ------------------------------------------------------------------------------------------------
// helpers on one instance / solve

__device__ __forceinline__ double* hist_ptr(const KParams& kp, int rid, int kind, int idx) {
  return kp.hist + ((size_t)rid * H_NKIND + kind) * (size_t)kp.hist_len + idx;
}

template <class V>
__device__ __forceinline__ V* vec_ptr(const GroupDev& g, int inst, int slot, int which) {
  return reinterpret_cast<V*>(g.vec + (long long)(inst * g.nrhs + slot) * g.vec_stride + g.vec_off[which]);
}
enum VecId { V_X = 0, V_R0 = 1, V_R1 = 2, V_S0 = 3, V_S1 = 4, V_Z = 5, V_Q = 6 };

// does a solve with action `a` stage a neighbour field in pass `pt`?
__device__ __forceinline__ bool stages(int pt, int a) {
  if (a == A_NONE || a == A_FIN) return false;
  return pt == P_INIT || pt == P_Z || pt == P_S || pt == P_X;
}
// number of sums a solve contributes in pass `pt`
__device__ __forceinline__ int nsums(int pt, int a) {
  if (a == A_NONE || a == A_FIN) return 0;
  switch (pt) {
    case P_INIT: return 2;                     // r.r, sum(b)
    case P_Z: return 1;                        // z.r
    case P_S: return 1;                        // s.q
    case P_X: return a == A_REPLACE ? 1 : 2;   // r.r (, z.r)
    default: return 0;
  }
}
__device__ __forceinline__ int hist_kind(int pt, int a, int kind) {
  switch (pt) {
    case P_INIT: return kind == 0 ? H_RRR : H_SUM;
    case P_Z: return H_ETAZ;
    case P_S: return H_SQ;
    case P_X: return a == A_REPLACE ? H_RRR : (kind == 0 ? H_RRX : H_ETAX);
    default: return 0;
  }
}

// compact index -> padded index of the same point
__device__ __forceinline__ long long cmp_to_pad(const TopoDev& tp, int c) {
  const int per = tp.nj * tp.ni;
  const int t = c / per;
  const int rem = c - t * per;
  const int j = rem / tp.ni;
  const int i = rem - j * tp.ni;
  return ((long long)t * tp.npy + (j + tp.OLy)) * tp.npx + (i + tp.OLx);
}

// ------------------------------------------------------------------------------------------------
// one work unit: rows [j0, j1) of tile t of one instance, in chunks of kWarps rows

template <bool MIXED>
__device__ void process_unit(const KParams& kp, const GroupDev& g, int inst, int lu, int pt, int k, int hidx,
                             const Smem& sm) {
  using V = typename Prec<MIXED>::V;
  using C = typename Prec<MIXED>::C;
  const TopoDev& tp = g.tp;
  const int ni = tp.ni, nj = tp.nj, npx = tp.npx;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t = lu / g.nblk, blk = lu - (lu / g.nblk) * g.nblk;
  const int R = kp.serial ? nj : kp.rows_per_block;
  const int j0 = blk * R, j1 = min(nj, j0 + R);
  const int op = g.op_base + inst;
  const long long pe = g.pad_elems;
  const int W = ni + 2;                                    // staged row width (cols -1..ni)
  const int SW = (kWarps + 2) * (kp.max_ni + 2);           // staged slot size

  int rid[2], act[2];
  double c1[2], c2[2], rnorm[2], norm[2];
  int has_alpha[2];
  for (int s = 0; s < 2; ++s) {
    rid[s] = g.rhs_base + inst * g.nrhs + s;
    act[s] = (s < g.nrhs) ? sm.act[rid[s]] : A_NONE;
    c1[s] = (s < g.nrhs) ? sm.c1[rid[s]] : 0.0;
    c2[s] = (s < g.nrhs) ? sm.c2[rid[s]] : 0.0;
    rnorm[s] = (s < g.nrhs) ? sm.rnorm[rid[s]] : 1.0;
    norm[s] = (s < g.nrhs) ? sm.norm[rid[s]] : 1.0;
    has_alpha[s] = (s < g.nrhs) ? sm.has_alpha[rid[s]] : 0;
  }

  // coefficients of this instance: FP64 (caller) and the type the CG stencils use
  const double* aW = g.a64[0] + inst * pe;
  const double* aS = g.a64[1] + inst * pe;
  const double* aC = g.a64[2] + inst * pe;
  const double* pW = g.a64[3] + inst * pe;
  const double* pS = g.a64[4] + inst * pe;
  const double* pC = g.a64[5] + inst * pe;
  const C *cW, *cS, *cC, *qW, *qS, *qC;
  if constexpr (MIXED) {
    const float* base = g.c32 + (long long)inst * 6 * pe;
    cW = base; cS = base + pe; cC = base + 2 * pe; qW = base + 3 * pe; qS = base + 4 * pe; qC = base + 5 * pe;
  } else {
    cW = aW; cS = aS; cC = aC; qW = pW; qS = pS; qC = pC;
  }

  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};   // thread 0: unit partial sums
  unsigned long long vmax[2] = {0ull, 0ull};       // P_MAX: max |b cg2dNorm| as ordered bits (NaN wins)

  for (int jc = j0; jc < j1; jc += kWarps) {
    const int nr = min(kWarps, j1 - jc);

    // ---- stage the neighbour field of every staging solve: rows jc-1 .. jc+nr, cols -1 .. ni
    bool any_stage = false;
    for (int s = 0; s < g.nrhs; ++s) any_stage |= stages(pt, act[s]);
    if (any_stage) {
      const int total = (nr + 2) * W;
      for (int idx = tid; idx < total; idx += kThreads) {
        const int rr = idx / W;
        const int cc = idx - rr * W;
        const int j = jc + rr - 1, i = cc - 1;
        const bool own = (rr >= 1 && rr <= nr);
        const bool iin = (i >= 0 && i < ni);
        if (!own && !iin) continue;           // corner cells: the 5-point stencil never reads them
        int src;
        long long hp = -1;                    // padded position of this halo cell in its own tile
        if (iin && j >= 0 && j < nj) {
          src = (t * nj + j) * ni + i;
        } else {
          if (i < 0) src = tp.nbr[0 * tp.T * nj + t * nj + j];
          else if (i >= ni) src = tp.nbr[1 * tp.T * nj + t * nj + j];
          else if (j < 0) src = tp.nbr[2 * tp.T * nj + t * ni + i];
          else src = tp.nbr[2 * tp.T * nj + tp.T * ni + t * ni + i];
          hp = ((long long)t * tp.npy + (j + tp.OLy)) * npx + (i + tp.OLx);
        }
        for (int s = 0; s < g.nrhs; ++s) {
          if (!stages(pt, act[s])) continue;
          double v = 0.0;
          if (pt == P_INIT) {
            const double* x0 = g.x0[s] + inst * pe;
            // cg2d.py:227-228: interior scaled by rhsNorm, exchanged; unwritten halo points keep cg2d_x
            v = (src >= 0) ? mul(__ldg(x0 + cmp_to_pad(tp, src)), rnorm[s]) : __ldg(x0 + hp);
          } else if (pt == P_Z) {
            const V* r = vec_ptr<V>(g, inst, s, (hidx & 1) ? V_R1 : V_R0);
            v = (src >= 0) ? (double)ldcg(r + src) : 0.0;
          } else if (pt == P_S) {
            // s_k(nbr) = z_k(nbr) + beta_k s_{k-1}(nbr)   (cg2d.py:249; halo points never written hold 0)
            const V* z = vec_ptr<V>(g, inst, s, V_Z);
            const V* so = vec_ptr<V>(g, inst, s, ((k + 1) & 1) ? V_S1 : V_S0);
            if (src >= 0) v = (double)(V)add((double)ldcg(z + src), mul(c1[s], (double)ldcg(so + src)));
          } else {  // P_X
            if (act[s] == A_REPLACE) {
              // x_{k+1}(nbr) = x_k(nbr) + alpha_k s_k(nbr); unwritten halo points keep cg2d_x
              const double* x = vec_ptr<double>(g, inst, s, V_X);
              const V* sk = vec_ptr<V>(g, inst, s, (k & 1) ? V_S1 : V_S0);
              v = (src >= 0) ? add(ldcg(x + src), mul(c1[s], (double)ldcg(sk + src)))
                             : __ldg(g.x0[s] + inst * pe + hp);
            } else {
              // r_{k+1}(nbr) = r_k(nbr) - alpha_k q_k(nbr)   (cg2d.py:255)
              const V* ro = vec_ptr<V>(g, inst, s, (k & 1) ? V_R1 : V_R0);
              const V* q = vec_ptr<V>(g, inst, s, V_Q);
              if (src >= 0) v = (double)(V)sub((double)ldcg(ro + src), mul(c1[s], (double)ldcg(q + src)));
            }
          }
          sm.stage[s * SW + rr * W + cc] = v;
        }
      }
      __syncthreads();
    }

    // ---- compute: warp w owns row jc + w, lane owns i = lane + 32m
    double lp[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    if (warp < nr) {
      const int j = jc + warp;
      const long long prow = ((long long)t * tp.npy + (j + tp.OLy)) * npx + tp.OLx;   // padded (j, 0)
      const int crow = (t * nj + j) * ni;                                               // compact (j, 0)
      for (int i = lane; i < ni; i += 32) {
        const long long po = prow + i;
        const int pc = crow + i;
        const int sc = (warp + 1) * W + (i + 1);   // staged centre
        for (int s = 0; s < g.nrhs; ++s) {
          const int a = act[s];
          if (a == A_NONE) continue;
          const double* st = sm.stage + s * SW;
          double p0 = 0.0, p1 = 0.0;
          if (pt == P_MAX) {
            const double bv = __ldg(g.b[s] + inst * pe + po);
            const unsigned long long m = (unsigned long long)__double_as_longlong(fabs(mul(bv, norm[s])));  // cg2d.py:222-223
            vmax[s] = m > vmax[s] ? m : vmax[s];
          } else if (pt == P_INIT) {
            const double vc = st[sc], vw = st[sc - 1], ve = st[sc + 1], vs = st[sc - W], vn = st[sc + W];
            stcg(vec_ptr<double>(g, inst, s, V_X) + pc, vc);
            const double bn = mul(mul(__ldg(g.b[s] + inst * pe + po), norm[s]), rnorm[s]);   // cg2d.py:221,226
            const double ax = op_A<double>(__ldg(aW + po), __ldg(aW + po + 1), __ldg(aS + po), __ldg(aS + po + npx),
                                           __ldg(aC + po), vw, ve, vs, vn, vc);
            const V r0 = (V)sub(bn, ax);                                                   // cg2d.py:232
            stcg(vec_ptr<V>(g, inst, s, V_R0) + pc, r0);
            stcg(vec_ptr<V>(g, inst, s, V_S1) + pc, (V)0);                                 // s = 0 (cg2d.py:231)
            p0 = mul((double)r0, (double)r0);
            p1 = bn;
          } else if (pt == P_Z) {
            const C vc = (C)st[sc], vw = (C)st[sc - 1], ve = (C)st[sc + 1], vs = (C)st[sc - W], vn = (C)st[sc + W];
            const V z = (V)op_M<C>(__ldg(qC + po), __ldg(qW + po), __ldg(qW + po + 1), __ldg(qS + po),
                                   __ldg(qS + po + npx), vc, vw, ve, vs, vn);
            stcg(vec_ptr<V>(g, inst, s, V_Z) + pc, z);
            p0 = mul((double)z, (double)vc);                     // cg2d.py:246
          } else if (pt == P_S) {
            const V* so = vec_ptr<V>(g, inst, s, ((k + 1) & 1) ? V_S1 : V_S0);
            double* x = vec_ptr<double>(g, inst, s, V_X);
            if (a == A_FIN) {
              double xv = ldcg(x + pc);
              if (has_alpha[s]) xv = add(xv, mul(c2[s], (double)ldcg(so + pc)));   // cg2d.py:254
              const double xf = __ddiv_rn(xv, rnorm[s]);                          // cg2d.py:266
              g.x_out[s][inst * pe + po] = xf;
              if (g.x_fortran[s]) g.x_fortran[s][inst * pe + po] = xf;
            } else {
              const C vc = (C)st[sc], vw = (C)st[sc - 1], ve = (C)st[sc + 1], vs = (C)st[sc - W], vn = (C)st[sc + W];
              stcg(vec_ptr<V>(g, inst, s, (k & 1) ? V_S1 : V_S0) + pc, (V)vc);
              const V q = (V)op_A<C>(__ldg(cW + po), __ldg(cW + po + 1), __ldg(cS + po), __ldg(cS + po + npx),
                                     __ldg(cC + po), vw, ve, vs, vn, vc);                 // cg2d.py:251
              stcg(vec_ptr<V>(g, inst, s, V_Q) + pc, q);
              if (has_alpha[s]) {
                const double xv = ldcg(x + pc);
                stcg(x + pc, add(xv, mul(c2[s], (double)ldcg(so + pc))));
              }
              p0 = mul((double)vc, (double)q);                                             // cg2d.py:252
            }
          } else {  // P_X
            V* rn = vec_ptr<V>(g, inst, s, ((k + 1) & 1) ? V_R1 : V_R0);
            if (a == A_REPLACE) {
              const double vc = st[sc], vw = st[sc - 1], ve = st[sc + 1], vs = st[sc - W], vn = st[sc + W];
              const double bn = mul(mul(__ldg(g.b[s] + inst * pe + po), norm[s]), rnorm[s]);
              const double ax = op_A<double>(__ldg(aW + po), __ldg(aW + po + 1), __ldg(aS + po),
                                             __ldg(aS + po + npx), __ldg(aC + po), vw, ve, vs, vn, vc);
              const V r = (V)sub(bn, ax);
              stcg(rn + pc, r);
              p0 = mul((double)r, (double)r);
            } else {
              const C vc = (C)st[sc], vw = (C)st[sc - 1], ve = (C)st[sc + 1], vs = (C)st[sc - W], vn = (C)st[sc + W];
              stcg(rn + pc, (V)vc);
              const V z = (V)op_M<C>(__ldg(qC + po), __ldg(qW + po), __ldg(qW + po + 1), __ldg(qS + po),
                                     __ldg(qS + po + npx), vc, vw, ve, vs, vn);            // cg2d.py:245
              stcg(vec_ptr<V>(g, inst, s, V_Z) + pc, z);
              p0 = mul((double)vc, (double)vc);                                            // cg2d.py:256
              p1 = mul((double)z, (double)vc);                                             // cg2d.py:246
            }
          }
          if (kp.serial) {
            double* pr = sm.prod + ((s * 2 + 0) * kWarps + warp) * kp.max_ni;
            pr[i] = p0;
            pr[kWarps * kp.max_ni + i] = p1;
          } else {
            lp[s][0] = add(lp[s][0], p0);
            lp[s][1] = add(lp[s][1], p1);
          }
        }
      }
      if (pt == P_MAX) {
        for (int s = 0; s < g.nrhs; ++s) {
          unsigned long long m = vmax[s];
          for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long y = __shfl_xor_sync(0xffffffffu, m, o);
            m = y > m ? y : m;
          }
          vmax[s] = m;
        }
      } else if (!kp.serial) {
        // row sum: xor butterfly over the lanes (every lane ends with the same value)
        for (int s = 0; s < g.nrhs; ++s)
          for (int q = 0; q < 2; ++q) {
            double v = lp[s][q];
            for (int o = 16; o > 0; o >>= 1) v = add(v, __shfl_xor_sync(0xffffffffu, v, o));
            if (lane == 0) sm.rowsum[(s * 2 + q) * kWarps + warp] = v;
          }
      }
    }
    if (pt == P_MAX) {
      if (warp < nr && lane == 0) {
        for (int s = 0; s < g.nrhs; ++s)
          if (act[s] != A_NONE)
            atomicMax(&kp.rmax[rid[s]], vmax[s]);
      }
      __syncthreads();
      continue;
    }
    __syncthreads();
    if (tid == 0) {
      for (int s = 0; s < g.nrhs; ++s) {
        const int ns = nsums(pt, act[s]);
        for (int q = 0; q < ns; ++q) {
          double a = acc[s][q];
          if (kp.serial) {
            const double* pr = sm.prod + ((s * 2 + q) * kWarps) * kp.max_ni;
            for (int w = 0; w < nr; ++w)
              for (int i = 0; i < ni; ++i) a = add(a, pr[w * kp.max_ni + i]);   // s = s + a(i,j), j outer
          } else {
            for (int w = 0; w < nr; ++w) a = add(a, sm.rowsum[(s * 2 + q) * kWarps + w]);
          }
          acc[s][q] = a;
        }
      }
    }
  }

  if (pt == P_MAX) return;

  // ---- unit partials, then the last unit of the instance forms the instance's sums in fixed order
  int any_sum = 0;
  for (int s = 0; s < g.nrhs; ++s) any_sum |= nsums(pt, act[s]);
  if (!any_sum) return;
  if (tid == 0) {
    for (int s = 0; s < g.nrhs; ++s) {
      const int ns = nsums(pt, act[s]);
      for (int q = 0; q < ns; ++q) stcg(kp.part + ((size_t)rid[s] * 2 + q) * kp.part_units + lu, acc[s][q]);
    }
    __threadfence();
    const unsigned old = atomicAdd(&kp.cnt[op], 1u);
    sm.misc[1] = ((old + 1u) % (unsigned)g.units) == 0u;
  }
  __syncthreads();
  if (sm.misc[1] && warp == 0) {
    __threadfence();
    for (int s = 0; s < g.nrhs; ++s) {
      const int ns = nsums(pt, act[s]);
      for (int q = 0; q < ns; ++q) {
        const double* P = kp.part + ((size_t)rid[s] * 2 + q) * kp.part_units;
        for (int tt = lane; tt < tp.T; tt += 32) {       // tile partial: blocks in order from 0
          double a = 0.0;
          for (int b = 0; b < g.nblk; ++b) a = add(a, ldcg(P + tt * g.nblk + b));
          sm.tsum[tt] = a;
        }
        __syncwarp();
        if (lane == 0) {                                  // GLOBAL_SUM_TILE: tiles in order from 0
          double a = 0.0;
          for (int tt = 0; tt < tp.T; ++tt) a = add(a, sm.tsum[tt]);
          stcg(hist_ptr(kp, rid[s], hist_kind(pt, act[s], q), hidx), a);
        }
        __syncwarp();
      }
    }
  }
}

template <bool MIXED>
__device__ void run_pass(const KParams& kp, int pt, int k, int hidx, const Smem& sm) {
  for (int u = blockIdx.x; u < kp.total_units; u += gridDim.x) {
    int gi = 0;
    while (gi + 1 < kp.ngroups && u >= kp.g[gi + 1].unit_base) ++gi;
    const GroupDev& g = kp.g[gi];
    const int rel = u - g.unit_base;
    const int inst = rel / g.units;
    const int lu = rel - inst * g.units;
    if (!sm.opp[g.op_base + inst]) continue;
    process_unit<MIXED>(kp, g, inst, lu, pt, k, hidx, sm);
  }
}

// which group / instance / slot a global solve index belongs to
__device__ __forceinline__ void locate(const KParams& kp, int r, int& gi, int& inst, int& slot) {
  gi = 0;
  while (gi + 1 < kp.ngroups && r >= kp.g[gi + 1].rhs_base) ++gi;
  const int rel = r - kp.g[gi].rhs_base;
  inst = rel / kp.g[gi].nrhs;
  slot = rel - inst * kp.g[gi].nrhs;
}

// publish the actions of this pass: act[] for every solve and opp[] for every operator
__device__ void set_actions(const KParams& kp, const Smem& sm, int my_act, double my_c1, double my_c2) {
  const int tid = threadIdx.x;
  if (tid < kp.total_ops) sm.opp[tid] = 0;
  __syncthreads();
  if (tid < kp.total_rhs) {
    sm.act[tid] = my_act;
    sm.c1[tid] = my_c1;
    sm.c2[tid] = my_c2;
    if (my_act != A_NONE) {
      int gi, inst, slot;
      locate(kp, tid, gi, inst, slot);
      sm.opp[kp.g[gi].op_base + inst] = 1;
    }
  }
  __syncthreads();
}

template <bool MIXED>
__global__ void __launch_bounds__(kThreads, 2) cg2d_persistent(const __grid_constant__ KParams kp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Smem sm = carve(smem_raw, kp.max_ni, kp.serial);
  const int tid = threadIdx.x;
  unsigned target = (unsigned)kp.test_missing;

  // state of solve `tid` (identical in every CTA: computed from the same write-once sums)
  const bool own = tid < kp.total_rhs;
  int gi = 0, inst = 0, slot = 0;
  double tol2 = 0.0, rep2 = 0.0, rhsNorm = 1.0, rhsMax = 0.0, eta = 0.0, eta_prev = 1.0, alpha = 0.0, rr = 0.0;
  int maxit = 0, k_done = -1, nrep = 0, has_alpha = 0;
  if (own) {
    locate(kp, tid, gi, inst, slot);
    const GroupDev& g = kp.g[gi];
    tol2 = g.tol[slot] * g.tol[slot];                      // cg2d.py:219
    rep2 = (kp.replace_above * g.tol[slot]) * (kp.replace_above * g.tol[slot]);
    maxit = g.max_iters[slot];
    sm.norm[tid] = g.norm_arr ? g.norm_arr[inst] : g.norm;
    sm.rnorm[tid] = 1.0;
    sm.has_alpha[tid] = 0;
  }
  int k = 0;
  bool ok = true;

  // ---- rhsMax = max |b cg2dNorm| (cg2d.py:221-225)
  set_actions(kp, sm, own ? A_ACTIVE : A_NONE, 0.0, 0.0);
  run_pass<MIXED>(kp, P_MAX, 0, 0, sm);
  ok = grid_barrier(kp, target, sm.misc);
  if (!ok) goto epilogue;
  if (own) {
    rhsMax = __longlong_as_double((long long)__ldcg(&kp.rmax[tid]));
    rhsNorm = (rhsMax != 0.0) ? __ddiv_rn(1.0, rhsMax) : 1.0;
    sm.rnorm[tid] = rhsNorm;
  }
  // ---- x = x0 rhsNorm, r = b - A x, s = 0, err^2, sumRHS (cg2d.py:226-236)
  set_actions(kp, sm, own ? A_ACTIVE : A_NONE, 0.0, 0.0);
  run_pass<MIXED>(kp, P_INIT, 0, 0, sm);
  ok = grid_barrier(kp, target, sm.misc);
  if (!ok) goto epilogue;
  if (own) rr = __ldcg(hist_ptr(kp, tid, H_RRR, 0));
  // ---- z = M r and eta for the first iteration
  set_actions(kp, sm, own ? A_ACTIVE : A_NONE, 0.0, 0.0);
  run_pass<MIXED>(kp, P_Z, 0, 0, sm);
  ok = grid_barrier(kp, target, sm.misc);
  if (!ok) goto epilogue;
  if (own) eta = __ldcg(hist_ptr(kp, tid, H_ETAZ, 0));

  for (k = 0;; ++k) {
    // stop rule before every iteration (cg2d.py:238-241)
    int a = A_NONE;
    double beta = 0.0;
    if (own && k_done < 0) {
      if (!(k < maxit) || rr < tol2) {
        k_done = k;
        a = A_FIN;
      } else {
        a = A_ACTIVE;
        beta = __ddiv_rn(eta, eta_prev);                   // cg2d.py:247
        eta_prev = eta;                                     // cg2d.py:248
      }
    }
    if (own) sm.has_alpha[tid] = has_alpha;
    set_actions(kp, sm, a, beta, alpha);
    const int any_active = __syncthreads_or(a == A_ACTIVE);
    const int any_fin = __syncthreads_or(a == A_FIN);
    if (!any_active && !any_fin) break;
    run_pass<MIXED>(kp, P_S, k, k, sm);
    ok = grid_barrier(kp, target, sm.misc);
    if (!ok) goto epilogue;
    if (!any_active) break;
    if (a == A_ACTIVE) {
      const double sq = __ldcg(hist_ptr(kp, tid, H_SQ, k));
      alpha = __ddiv_rn(eta, sq);                           // cg2d.py:252-253
      has_alpha = 1;
    }
    // ---- r, z, err^2, next eta
    int ax = A_NONE;
    if (a == A_ACTIVE)
      ax = (kp.mixed && kp.replace_every > 0 && ((k + 1) % kp.replace_every) == 0 && rr > rep2) ? A_REPLACE
                                                                                                : A_ACTIVE;
    set_actions(kp, sm, ax, alpha, 0.0);
    run_pass<MIXED>(kp, P_X, k, k + 1, sm);
    ok = grid_barrier(kp, target, sm.misc);
    if (!ok) goto epilogue;
    if (ax == A_ACTIVE) {
      rr = __ldcg(hist_ptr(kp, tid, H_RRX, k + 1));
      eta = __ldcg(hist_ptr(kp, tid, H_ETAX, k + 1));
    } else if (ax == A_REPLACE) {
      rr = __ldcg(hist_ptr(kp, tid, H_RRR, k + 1));
      ++nrep;
    }
    if (kp.mixed) {
      // z = M r and eta from a replaced residual
      const int az = (ax == A_REPLACE) ? A_ACTIVE : A_NONE;
      if (__syncthreads_or(az != A_NONE)) {
        set_actions(kp, sm, az, 0.0, 0.0);
        run_pass<MIXED>(kp, P_Z, k, k + 1, sm);
        ok = grid_barrier(kp, target, sm.misc);
        if (!ok) goto epilogue;
        if (az == A_ACTIVE) eta = __ldcg(hist_ptr(kp, tid, H_ETAZ, k + 1));
      }
    }
  }

epilogue:
  // ---- halo points of the outputs: x_out 0; x_fortran = exchanged normalised first guess, unwritten
  //      points keep cg2d_x (cg2d.py:208-210, 227-228)
  {
    const long long gstride = (long long)gridDim.x * kThreads;
    for (int gg = 0; gg < kp.ngroups; ++gg) {
      const GroupDev& g = kp.g[gg];
      const TopoDev& tp = g.tp;
      const long long per = g.pad_elems;
      const long long tot = per * g.count * g.nrhs;
      for (long long idx = (long long)blockIdx.x * kThreads + tid; idx < tot; idx += gstride) {
        const long long ins_slot = idx / per;
        const long long p = idx - ins_slot * per;
        const int in = (int)(ins_slot / g.nrhs);
        const int s = (int)(ins_slot - (long long)in * g.nrhs);
        const int plane = tp.npy * tp.npx;
        const int pt_ = (int)(p % plane);
        const int jj = pt_ / tp.npx, ii = pt_ - (pt_ / tp.npx) * tp.npx;
        const bool interior = jj >= tp.OLy && jj < tp.OLy + tp.nj && ii >= tp.OLx && ii < tp.OLx + tp.ni;
        if (interior) continue;
        const long long off = (long long)in * per + p;
        g.x_out[s][off] = 0.0;
        if (g.x_fortran[s]) {
          const double* x0 = g.x0[s] + (long long)in * per;
          double v = __ldg(x0 + p);
          if (tp.map_comp[p] == 1) {
            const int sp = tp.map_src[p];
            const int spl = sp % plane;
            const int sj = spl / tp.npx, si = spl - (spl / tp.npx) * tp.npx;
            const bool sin = sj >= tp.OLy && sj < tp.OLy + tp.nj && si >= tp.OLx && si < tp.OLx + tp.ni;
            const double rn = sm.rnorm[g.rhs_base + in * g.nrhs + s];
            v = sin ? mul(__ldg(x0 + sp), rn) : __ldg(x0 + sp);
          }
          g.x_fortran[s][off] = v;
        }
      }
    }
  }
  if (blockIdx.x == 0 && own) {
    const GroupDev& g = kp.g[gi];
    cg2d_diag_t d;
    d.firstResidual = sqrt(__ldcg(hist_ptr(kp, tid, H_RRR, 0)));
    d.lastResidual = sqrt(rr);
    d.sumRHS = __ldcg(hist_ptr(kp, tid, H_SUM, 0));
    d.rhsMax = rhsMax;
    d.numIters = k_done >= 0 ? k_done : k;
    d.replacements = nrep;
    d.reserved = 0;
    if (!ok || __ldcg(&kp.gs[1]) != 0u) d.status = CG2D_BARRIER_TIMEOUT;
    else if (rr != rr) d.status = CG2D_NAN;
    else if (!(rr < tol2)) d.status = CG2D_NOT_CONVERGED;
    else d.status = CG2D_OK;
    if (!ok) { d.firstResidual = d.lastResidual = d.sumRHS = __longlong_as_double(0x7ff8000000000000LL); }
    g.diag[slot][inst] = d;
  }
}

// ------------------------------------------------------------------------------------------------
// MIXED: FP32 copies of the six coefficient arrays, [inst][6][pad_elems]

__global__ void pack32_kernel(GroupDev g) {
  const long long pe = g.pad_elems;
  const long long tot = pe * 6 * g.count;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long in = idx / (6 * pe);
    const long long rem = idx - in * 6 * pe;
    const int which = (int)(rem / pe);
    const long long p = rem - (long long)which * pe;
    g.c32[idx] = __double2float_rn(g.a64[which][in * pe + p]);
  }
}

// ------------------------------------------------------------------------------------------------
// _matvec (cg2d.py:292-298): out = (A / cg2dNorm) v on the interior, 0 on halos

__device__ __forceinline__ double gathered(const TopoDev& tp, const double* v, int t, int j, int i) {
  // v's value at (t, j, i) after exch_xy(where(inner, v, 0)): in-tile points read v, cross-tile
  // neighbours read their source, unwritten halo points read 0
  int src;
  if (i >= 0 && i < tp.ni && j >= 0 && j < tp.nj) return v[((long long)t * tp.npy + j + tp.OLy) * tp.npx + i + tp.OLx];
  if (i < 0) src = tp.nbr[0 * tp.T * tp.nj + t * tp.nj + j];
  else if (i >= tp.ni) src = tp.nbr[1 * tp.T * tp.nj + t * tp.nj + j];
  else if (j < 0) src = tp.nbr[2 * tp.T * tp.nj + t * tp.ni + i];
  else src = tp.nbr[2 * tp.T * tp.nj + tp.T * tp.ni + t * tp.ni + i];
  return src >= 0 ? v[cmp_to_pad(tp, src)] : 0.0;
}

__global__ void apply_operator_kernel(TopoDev tp, int batch, double norm, const double* aW, const double* aS,
                                      const double* aC, const double* v, double* out) {
  const long long pe = (long long)tp.T * tp.npy * tp.npx;
  const long long tot = pe * batch;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long in = idx / pe;
    const long long p = idx - in * pe;
    const int plane = tp.npy * tp.npx;
    const int t = (int)(p / plane);
    const int rem = (int)(p - (long long)t * plane);
    const int j = rem / tp.npx - tp.OLy, i = rem - (rem / tp.npx) * tp.npx - tp.OLx;
    double r = 0.0;
    if (j >= 0 && j < tp.nj && i >= 0 && i < tp.ni) {
      const double* vi = v + in * pe;
      const long long po = in * pe + p;
      const double ax = op_A<double>(aW[po], aW[po + 1], aS[po], aS[po + tp.npx], aC[po],
                                     gathered(tp, vi, t, j, i - 1), gathered(tp, vi, t, j, i + 1),
                                     gathered(tp, vi, t, j - 1, i), gathered(tp, vi, t, j + 1, i), vi[p]);
      r = __ddiv_rn(ax, norm);
    }
    out[idx] = r;
  }
}

// coefficient cotangents of the implicit derivative (transpose of _matvec in the coefficients)
__global__ void edge_products_kernel(TopoDev tp, int batch, double norm, const double* norm_arr, const double* lam,
                                     const double* x, double* gW, double* gS, double* gC) {
  const long long pe = (long long)tp.T * tp.npy * tp.npx;
  const long long tot = pe * batch;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long in = idx / pe;
    const long long p = idx - in * pe;
    const int plane = tp.npy * tp.npx;
    const int t = (int)(p / plane);
    const int rem = (int)(p - (long long)t * plane);
    const int j = rem / tp.npx - tp.OLy, i = rem - (rem / tp.npx) * tp.npx - tp.OLx;
    const double nrm = norm_arr ? norm_arr[in] : norm;
    const double* li = lam + in * pe;
    const double* xi = x + in * pe;
    const bool jin = j >= 0 && j < tp.nj, iin = i >= 0 && i < tp.ni;
    double w = 0.0, s = 0.0, c = 0.0;
    // interior lam / cg2dNorm at (t, jj, ii) (0 off the interior)
    auto cl = [&](int jj, int ii) -> double {
      return __ddiv_rn(li[((long long)t * tp.npy + jj + tp.OLy) * tp.npx + ii + tp.OLx], nrm);
    };
    if (jin && i >= 0 && i <= tp.ni) {      // gW: the face between (j, i-1) and (j, i)
      double a = 0.0;
      if (i < tp.ni) a = add(a, mul(cl(j, i), gathered(tp, xi, t, j, i - 1)));
      if (i >= 1) a = add(a, mul(cl(j, i - 1), gathered(tp, xi, t, j, i)));
      w = -a;
    }
    if (iin && j >= 0 && j <= tp.nj) {      // gS: the face between (j-1, i) and (j, i)
      double a = 0.0;
      if (j < tp.nj) a = add(a, mul(cl(j, i), gathered(tp, xi, t, j - 1, i)));
      if (j >= 1) a = add(a, mul(cl(j - 1, i), gathered(tp, xi, t, j, i)));
      s = -a;
    }
    if (jin && iin) c = -mul(cl(j, i), xi[p]);
    gW[idx] = w;
    gS[idx] = s;
    gC[idx] = c;
  }
}

__global__ void exchange_kernel(TopoDev tp, int batch, const double* a, double* out) {
  const long long pe = (long long)tp.T * tp.npy * tp.npx;
  const long long tot = pe * batch;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long in = idx / pe;
    const long long p = idx - in * pe;
    out[idx] = tp.map_comp[p] == 1 ? a[in * pe + tp.map_src[p]] : a[idx];
  }
}

// ------------------------------------------------------------------------------------------------
// launchers

static int grid_for(long long work) {
  long long b = (work + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

cudaError_t solver_occupancy(int mixed, size_t smem, int* blocks_per_sm) {
  const void* fn = mixed ? (const void*)cg2d_persistent<true> : (const void*)cg2d_persistent<false>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, kThreads, smem);
}

cudaError_t launch_solver(const KParams& kp, int grid, size_t smem, cudaStream_t stream) {
  const void* fn = kp.mixed ? (const void*)cg2d_persistent<true> : (const void*)cg2d_persistent<false>;
  void* args[] = {const_cast<KParams*>(&kp)};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, smem, stream);
}

cudaError_t launch_pack32(const GroupDev& g, cudaStream_t stream) {
  pack32_kernel<<<grid_for(g.pad_elems * 6 * g.count), 256, 0, stream>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_apply_operator(const TopoDev& tp, int batch, double norm, const double* aW, const double* aS,
                                  const double* aC, const double* v, double* out, cudaStream_t stream) {
  const long long tot = (long long)tp.T * tp.npy * tp.npx * batch;
  apply_operator_kernel<<<grid_for(tot), 256, 0, stream>>>(tp, batch, norm, aW, aS, aC, v, out);
  return cudaGetLastError();
}

cudaError_t launch_edge_products(const TopoDev& tp, int batch, double norm, const double* norm_arr,
                                 const double* lam, const double* x, double* gW, double* gS, double* gC,
                                 cudaStream_t stream) {
  const long long tot = (long long)tp.T * tp.npy * tp.npx * batch;
  edge_products_kernel<<<grid_for(tot), 256, 0, stream>>>(tp, batch, norm, norm_arr, lam, x, gW, gS, gC);
  return cudaGetLastError();
}

cudaError_t launch_exchange(const TopoDev& tp, int batch, const double* a, double* out, cudaStream_t stream) {
  const long long tot = (long long)tp.T * tp.npy * tp.npx * batch;
  exchange_kernel<<<grid_for(tot), 256, 0, stream>>>(tp, batch, a, out);
  return cudaGetLastError();
}

}  // namespace cg2d
