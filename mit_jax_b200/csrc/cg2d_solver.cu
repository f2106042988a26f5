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
// Work is cut into chunks of up to 8 rows of one tile. For every chunk the lanes of warp 0 issue
// bulk asynchronous copies (cp.async.bulk, completion counted on an mbarrier) into shared memory:
// one for the packed coefficient rows, one per vector (rows j-1 .. j+8 with their neighbour cells)
// and the push targets of the chunk's edge points; the next chunk's copies are in flight while the
// current one is computed (two stage buffers). Values at the four neighbours of a point are formed
// in shared memory exactly as their owner forms them (a neighbour's s_k from its z_k and s_{k-1},
// its r_{k+1} from r_k and q_k), so no exchange step and no extra wait is needed. Every vector tile
// is stored with its halo ring (one cell on each side); cross-tile neighbours -- the exch2 halo of
// cg2d.py:228,235,250,260 -- are pushed by the owner of each tile-edge point into the rings of the
// tiles that read it whenever it writes the value, so the stencil needs no edge cases. The x update
// is deferred by one pass (it needs s_{k-1}, which pass S_k reads anyway); its arithmetic is the
// reference's x + alpha * s (cg2d.py:254).
//
// MIXED precision keeps r, s, z, q and the operator copies in FP32 (FP32 stencils), x and all dot
// products in FP64, and replaces r by the FP64 true residual b - A x every replace_every iterations
// while the residual is above replace_above * tolerance (near the FP64 rounding floor of b - A x a
// replacement would only add noise); the stop rule is the reference's, on the carried residual.

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "cg2d_internal.cuh"

namespace cg2d {

// ------------------------------------------------------------------------------------------------
// arithmetic without contraction (the reference rounds every product and every sum)

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

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
// where a time limit ran out: gs[2] = 1 grid-wide wait, 2 bulk-copy wait, 3 unit-count wait; gs[3] = pass << 16 | CTA
__device__ __forceinline__ void note_timeout(unsigned* gs, unsigned where, unsigned pass) {
  if (atomicCAS(&gs[1], 0u, (unsigned)CG2D_BARRIER_TIMEOUT) == 0u) {
    gs[2] = where;
    gs[3] = (pass << 16) | (blockIdx.x & 0xffffu);
  }
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// phase timers (thread 0, profiling only)
#define PROF_T0(kp) (((kp).prof && threadIdx.x == 0) ? globaltimer() : 0ull)
#define PROF_ADD(kp, sm, ph, t0)                                               \
  do {                                                                         \
    if ((kp).prof && threadIdx.x == 0) (sm).pacc()[ph] += globaltimer() - (t0); \
  } while (0)

// ---- bulk asynchronous copies and mbarriers

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// global -> shared bulk copy (no multicast), completion counted in bytes on `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// orders this thread's generic-proxy accesses against async-proxy (bulk copy) accesses
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// the same, letting the thread sleep up to hint_ns while the phase is incomplete (it wakes when the phase
// completes), so that waiting warps leave the issue slots to the computing ones
__device__ __forceinline__ bool mbar_try_wait_sleep(unsigned long long* bar, unsigned parity, unsigned hint_ns) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// bounded wait for an mbarrier phase
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  for (unsigned it = 1;; ++it) {
    if (mbar_try_wait_sleep(bar, parity, 20000u)) return true;
    if ((it & 15u) == 0u && globaltimer() - t0 > limit_ns) return false;
  }
}

// ------------------------------------------------------------------------------------------------
// shared memory carve

// the dynamic shared memory of the persistent kernel; pointers derived from this symbol are known to the
// compiler to address shared memory (shared loads, no aliasing with global stores)
extern __shared__ __align__(128) unsigned char smem_raw[];

// CG scalars of one solve between passes (one entry per solve; the thread of the same index owns it)
struct SolveState {
  double eta, eta_prev, alpha, rr;
  int k_done, nrep;
};
static_assert(sizeof(SolveState) == 40, "SolveState layout");

// Fixed part of the shared-memory layout: compile-time offsets, so that no registers hold its addresses.
__host__ __device__ constexpr size_t a16(size_t x) { return (x + 15) & ~size_t(15); }
namespace smo {
constexpr size_t act = 0;                                                    // int [kMaxSolves] action of each solve
constexpr size_t c1 = act + a16(sizeof(int) * kMaxSolves);                  // double [kMaxSolves] beta (S) / alpha (X, R)
constexpr size_t c2 = c1 + a16(sizeof(double) * kMaxSolves);                // double [kMaxSolves] alpha_{k-1} (x update)
constexpr size_t rnorm = c2 + a16(sizeof(double) * kMaxSolves);             // double [kMaxSolves] rhsNorm
constexpr size_t norm = rnorm + a16(sizeof(double) * kMaxSolves);           // double [kMaxSolves] cg2dNorm
constexpr size_t has_alpha = norm + a16(sizeof(double) * kMaxSolves);       // int [kMaxSolves]
constexpr size_t opp = has_alpha + a16(sizeof(int) * kMaxSolves);           // int [kMaxOps] operator in the pass
constexpr size_t rowsum = opp + a16(sizeof(int) * kMaxOps);                 // double [kMaxStages][4][kWarps]
constexpr size_t misc = rowsum + a16(sizeof(double) * kMaxStages * 4 * kWarps);   // int [4]
constexpr size_t full = misc + a16(sizeof(int) * 4);                        // mbarrier [kMaxStages]
constexpr size_t empty = full + a16(8 * kMaxStages);                        // mbarrier [kMaxStages]
constexpr size_t pacc = empty + a16(8 * kMaxStages);                        // u64 [kProfSlots]
constexpr size_t uacc = pacc + a16(8 * kProfSlots);                         // double [4]
constexpr size_t utab = uacc + a16(sizeof(double) * 4);                     // int2 [kMaxUnitsPerCta]
constexpr size_t pend = utab + a16(sizeof(int2) * kMaxUnitsPerCta);         // int4 [kMaxStages]
constexpr size_t state = pend + a16(sizeof(int4) * kMaxStages);             // SolveState [kMaxSolves + 1]
constexpr size_t end = state + a16(40 * (kMaxSolves + 1));                   // then prod (FORTRAN order)
}  // namespace smo

// Views of the shared memory. Fixed arrays:
//   act, c1, c2, rnorm, norm, has_alpha   per solve: action in the pass, pass coefficients, rhsNorm, cg2dNorm,
//                                          whether alpha_{k-1} exists
//   opp                                    per operator: takes part in the pass
//   rowsum                                 row sums of the chunk in each stage [stage][4 sums][kWarps]
//   misc                                   [0] grid-wide wait ok, [3] units in utab
//   full, empty                            stage mbarriers: copies landed / compute warps done with the stage
//   pacc, uacc                             phase times (profiling); the current unit's partial sums
//   utab, pend                             this CTA's work units; the chunk in each stage awaiting its row sums
//   state                                  CG scalars of each solve (SolveState), one spare entry
// then prod (FORTRAN order: [2 slots][2 kinds][kWarps][max_ni]) and the stage buffers at `stage` (kMaxStages x
// stage_bytes, 128-aligned; also the direct-pass staging area and the tile-sum buffers of the pass sums).
struct Smem {
  unsigned stage;
  template <class T>
  __device__ __forceinline__ static T* at(size_t off) { return reinterpret_cast<T*>(smem_raw + off); }
  __device__ __forceinline__ int* act() const { return at<int>(smo::act); }
  __device__ __forceinline__ double* c1() const { return at<double>(smo::c1); }
  __device__ __forceinline__ double* c2() const { return at<double>(smo::c2); }
  __device__ __forceinline__ double* rnorm() const { return at<double>(smo::rnorm); }
  __device__ __forceinline__ double* norm() const { return at<double>(smo::norm); }
  __device__ __forceinline__ int* has_alpha() const { return at<int>(smo::has_alpha); }
  __device__ __forceinline__ int* opp() const { return at<int>(smo::opp); }
  __device__ __forceinline__ double* rowsum() const { return at<double>(smo::rowsum); }
  __device__ __forceinline__ int* misc() const { return at<int>(smo::misc); }
  __device__ __forceinline__ unsigned long long* full() const { return at<unsigned long long>(smo::full); }
  __device__ __forceinline__ unsigned long long* empty() const { return at<unsigned long long>(smo::empty); }
  __device__ __forceinline__ unsigned long long* pacc() const { return at<unsigned long long>(smo::pacc); }
  __device__ __forceinline__ double* uacc() const { return at<double>(smo::uacc); }
  __device__ __forceinline__ int2* utab() const { return at<int2>(smo::utab); }
  __device__ __forceinline__ int4* pend() const { return at<int4>(smo::pend); }
  __device__ __forceinline__ SolveState* state() const { return at<SolveState>(smo::state); }
  __device__ __forceinline__ double* prod() const { return at<double>(smo::end); }
};

static size_t prod_bytes(int max_ni, int serial) {
  return serial ? a16(sizeof(double) * 2 * 2 * kWarps * (size_t)max_ni) : 0;
}
size_t fixed_smem_bytes(int max_ni, int serial) { return (smo::end + prod_bytes(max_ni, serial) + 127) & ~size_t(127); }

__device__ inline Smem carve(int max_ni, int serial) {
  Smem m;
  const size_t pb = serial ? a16(sizeof(double) * 2 * 2 * kWarps * (size_t)max_ni) : 0;
  m.stage = (unsigned)((smo::end + pb + 127) & ~size_t(127));
  return m;
}

// ------------------------------------------------------------------------------------------------
// grid-wide wait: every CTA arrives once (after this CTA's stores, release); the wait ends when all have
// arrived (acquire), when another CTA has flagged an error, or after timeout_ns (then this CTA flags the error).

__device__ __forceinline__ unsigned atom_add_release(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.release.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// `target` counts the arrivals this CTA waits for (uniform in the grid)
__device__ bool grid_wait(const KParams& kp, unsigned& target, int pt, const Smem& sm) {
  const unsigned long long tb = PROF_T0(kp);
  fence_proxy_async();        // this thread's stores before the next pass's bulk copies
  __syncthreads();
  target += gridDim.x;
  if (threadIdx.x == 0) {
    atom_add_release(&kp.gs[0], 1u);
    const unsigned long long t0 = globaltimer();
    int ok = 1;
    for (unsigned spins = 0;; ++spins) {
      if ((int)(ld_acquire(&kp.gs[0]) - target) >= 0) break;
      if (spins > 8) __nanosleep(32);
      if ((spins & 63u) == 63u) {
        if (ld_relaxed(&kp.gs[1]) != 0u) { ok = 0; break; }
        if (globaltimer() - t0 > kp.timeout_ns) {
          note_timeout(kp.gs, 1u, (unsigned)pt);
          ok = 0;
          break;
        }
      }
    }
    fence_proxy_async();
    sm.misc()[0] = ok;
    if (kp.prof) sm.pacc()[PR_BAR] += globaltimer() - tb;
  }
  __syncthreads();
  return sm.misc()[0] != 0;
}

__device__ __forceinline__ double* hist_ptr(const KParams& kp, int rid, int kind, int idx);
__device__ __forceinline__ int nsums(int pt, int a);
__device__ __forceinline__ int hist_kind(int pt, int kind);
__device__ __forceinline__ void locate(const KParams& kp, int r, int& gi, int& inst, int& slot);

// The sums of pass pt from the unit partials, in fixed order: blocks of a tile in order, then tiles in order
// from 0 (GLOBAL_SUM_TILE, global_sum.py:20-26). Sum (solve r, kind q) is formed by warp r * 2 + q of the grid
// (modulo its warps): lane l adds the blocks of tiles l, l + 32, ..., lane 0 the tile sums.
__device__ void form_sums(const KParams& kp, int pt, int hidx, const Smem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* tbuf = reinterpret_cast<double*>(smem_raw + sm.stage) + warp * kMaxTiles;   // free between passes
  const int nw = (int)gridDim.x * kAllWarps;
  for (int s = (int)blockIdx.x * kAllWarps + warp; s < 2 * kp.total_rhs; s += nw) {
    const int r = s >> 1, q = s & 1;
    if (q >= nsums(pt, sm.act()[r])) continue;
    int gi, inst, slot;
    locate(kp, r, gi, inst, slot);
    const GroupDev& g = kp.g[gi];
    const double* p = kp.part + ((size_t)r * 2 + q) * kp.part_units;
    for (int t = lane; t < g.tp.T; t += 32) {
      const double* pt_ = p + t * g.nblk;
      double a = 0.0;
#pragma unroll 8
      for (int b = 0; b < g.nblk; ++b) a = add(a, __ldcg(pt_ + b));
      tbuf[t] = a;
    }
    __syncwarp();
    if (lane == 0) {
      double total = 0.0;
      for (int t = 0; t < g.tp.T; ++t) total = add(total, tbuf[t]);
      stcg(hist_ptr(kp, r, hist_kind(pt, q), hidx), total);
    }
    __syncwarp();
  }
}

// end of a pass: wait for every CTA's unit partials, form the sums, wait until every sum is written
__device__ bool grid_sync(const KParams& kp, unsigned& target, int pt, int hidx, const Smem& sm) {
  if (!grid_wait(kp, target, pt, sm)) return false;
  if (pt == P_MAX) return true;
  const unsigned long long tf = PROF_T0(kp);
  form_sums(kp, pt, hidx, sm);
  PROF_ADD(kp, sm, PR_FIN, tf);
  return grid_wait(kp, target, pt, sm);
}

// ------------------------------------------------------------------------------------------------
// helpers on one instance / solve

__device__ __forceinline__ double* hist_ptr(const KParams& kp, int rid, int kind, int idx) {
  return kp.hist + ((size_t)rid * H_NKIND + kind) * (size_t)kp.hist_len + idx;
}

// a solve's vector (ringed tiles, [T][nj+2][P])
template <class T>
__device__ __forceinline__ T* vec_ptr(const GroupDev& g, int inst, int slot, int which) {
  return reinterpret_cast<T*>(g.vec + (long long)(inst * g.nrhs + slot) * g.vec_stride + g.vec_off[which]);
}
// element of point (t, j, i) in a ringed vector; -1 <= j <= nj, -1 <= i <= ni
__device__ __forceinline__ long long vidx(const TopoDev& tp, int t, int j, int i) {
  return ((long long)t * (tp.nj + 2) + j + 1) * tp.P + i + 1;
}

// one push store: target a (-1 = none) must lie inside the vector (lim elements); anything else is an internal
// inconsistency, recorded in the error word instead of stored
template <class T>
__device__ __forceinline__ void push_one(T* vec, int a, T v, unsigned lim, unsigned* gs) {
  if ((unsigned)a < lim) stcg(vec + a, v);
  else if (a != -1) atomicCAS(&gs[1], 0u, (unsigned)CG2D_INTERNAL_ERROR);
}

// store the value of point (t, j, i) into the ring cells of the tiles that read it across an edge
template <class T>
__device__ __forceinline__ void push(const TopoDev& tp, T* vec, int t, int j, int i, T v, unsigned* gs) {
  const int* e;
  if (i == 0) e = tp.tg + ((size_t)t * tp.nj + j) * 4;
  else if (i == tp.ni - 1) e = tp.tg + ((size_t)t * tp.nj + j) * 4 + 2;
  else if (j == 0) e = tp.tg + (size_t)tp.T * tp.nj * 4 + ((size_t)t * tp.nip + i) * 2;
  else if (j == tp.nj - 1) e = tp.tg + (size_t)tp.T * tp.nj * 4 + ((size_t)(tp.T + t) * tp.nip + i) * 2;
  else return;
  const unsigned lim = (unsigned)tp.T * (unsigned)(tp.nj + 2) * (unsigned)tp.P;
  push_one(vec, __ldg(e), v, lim, gs);
  push_one(vec, __ldg(e + 1), v, lim, gs);
}

// the same with the chunk's target lists staged in shared memory (row w of the chunk = tile row j)
struct PushTab {
  const int4* twe;
  const int2 *ts, *tn;
  int ni, nj;
  unsigned lim;   // elements of a vector
  unsigned* gs;
};
template <class T>
__device__ __forceinline__ void push_s(const PushTab& pt, T* vec, int j, int w, int i, T v) {
  int a, b;
  if (i == 0) { const int4 e = pt.twe[w]; a = e.x; b = e.y; }
  else if (i == pt.ni - 1) { const int4 e = pt.twe[w]; a = e.z; b = e.w; }
  else if (j == 0) { const int2 e = pt.ts[i]; a = e.x; b = e.y; }
  else if (j == pt.nj - 1) { const int2 e = pt.tn[i]; a = e.x; b = e.y; }
  else return;
  push_one(vec, a, v, pt.lim, pt.gs);
  push_one(vec, b, v, pt.lim, pt.gs);
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

// number of sums a solve contributes in pass `pt`, and where each goes
__device__ __forceinline__ int nsums(int pt, int a) {
  if (a != A_ACTIVE) return 0;
  switch (pt) {
    case P_INIT: return 2;   // r.r, sum(b)
    case P_Z: return 1;      // z.r
    case P_S: return 1;      // s.q
    case P_X: return 2;      // r.r, z.r
    case P_R: return 1;      // r.r
    default: return 0;
  }
}
__device__ __forceinline__ int hist_kind(int pt, int kind) {
  switch (pt) {
    case P_INIT: return kind == 0 ? H_RRR : H_SUM;
    case P_Z: return H_ETAZ;
    case P_S: return H_SQ;
    case P_X: return kind == 0 ? H_RRX : H_ETAX;
    case P_R: return H_RRR;
    default: return 0;
  }
}

// the solve slots of an instance and their scalars, read from shared memory by solve index
struct Slots {
  const Smem* sm;
  int rid0, nrhs;
  __device__ __forceinline__ int rid(int s) const { return rid0 + s; }
  __device__ __forceinline__ int act(int s) const { return s < nrhs ? sm->act()[rid0 + s] : (int)A_NONE; }
  __device__ __forceinline__ double c1(int s) const { return sm->c1()[rid0 + s]; }
  __device__ __forceinline__ double c2(int s) const { return sm->c2()[rid0 + s]; }
  __device__ __forceinline__ double rnorm(int s) const { return sm->rnorm()[rid0 + s]; }
  __device__ __forceinline__ double norm(int s) const { return sm->norm()[rid0 + s]; }
  __device__ __forceinline__ int has_alpha(int s) const { return sm->has_alpha()[rid0 + s]; }
};
__device__ __forceinline__ Slots slots_of(const GroupDev& g, int inst, const Smem& sm) {
  Slots q;
  q.sm = &sm;
  q.rid0 = g.rhs_base + inst * g.nrhs;
  q.nrhs = g.nrhs;
  return q;
}

// ------------------------------------------------------------------------------------------------
// row sums of one chunk into the unit partials, and the unit partials into the instance sums

// warp w holds per-lane partials lp of row w: xor butterfly (every lane ends with the same value)
struct Lanes {
  double v[4];   // (slot 0, kind 0), (0, 1), (1, 0), (1, 1): always indexed with constants
};
__device__ __forceinline__ double butterfly(double v) {
  for (int o = 16; o > 0; o >>= 1) v = add(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// (two: the pass forms two sums per solve; otherwise the second kind is not read and not reduced)
__device__ __forceinline__ void row_sums(const GroupDev& g, const Lanes& lp, const Smem& sm, int st, bool two) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double r0 = butterfly(lp.v[0]), r1 = two ? butterfly(lp.v[1]) : 0.0;
  double r2 = 0.0, r3 = 0.0;
  if (g.nrhs > 1) {
    r2 = butterfly(lp.v[2]);
    if (two) r3 = butterfly(lp.v[3]);
  }
  if (lane == 0) {
    double* rs = sm.rowsum() + st * 4 * kWarps;
    rs[0 * kWarps + warp] = r0;
    rs[1 * kWarps + warp] = r1;
    rs[2 * kWarps + warp] = r2;
    rs[3 * kWarps + warp] = r3;
  }
}

// one warp: add the chunk's rows (row sums of stage st) into the unit's partial sums, lane l < 4 owning sum
// (slot l >> 1, kind l & 1); `first` starts the unit from 0 (ROWBLOCK: row sums in row order; FORTRAN: every
// product in j, i order). Ends with the warp converged, so its lane 0 may read the partials.
__device__ __forceinline__ void accumulate_chunk(const KParams& kp, const GroupDev& g, int ns0, int ns1, int nr,
                                                 int st, bool first, const Smem& sm) {
  const int lane = threadIdx.x & 31;
  const int s = lane >> 1, q = lane & 1;
  if (lane < 4 && q < (s == 0 ? ns0 : ns1)) {
    double a = first ? 0.0 : sm.uacc()[lane];
    if (kp.serial) {
      const double* pr = sm.prod() + (lane * kWarps) * kp.max_ni;
      for (int w = 0; w < nr; ++w)
        for (int i = 0; i < g.tp.ni; ++i) a = add(a, pr[w * kp.max_ni + i]);   // s = s + a(i,j), j outer
    } else {
      const double* rs = sm.rowsum() + (st * 4 + lane) * kWarps;
      double v[kWarps];
#pragma unroll
      for (int w = 0; w < kWarps; ++w) v[w] = rs[w];
#pragma unroll
      for (int w = 0; w < kWarps; ++w)
        if (w < nr) a = add(a, v[w]);
    }
    sm.uacc()[lane] = a;
  }
  __syncwarp();
}

// lane 0 of the accumulating warp writes the unit's partials (the grid-wide wait at the end of the pass makes them
// visible to the warps that form the sums)
__device__ __forceinline__ void finish_unit(const KParams& kp, const GroupDev& g, int inst, int lu, int ns0, int ns1,
                                            const Smem& sm) {
  if ((threadIdx.x & 31) != 0 || ns0 + ns1 == 0) return;
  const int rid0 = g.rhs_base + inst * g.nrhs;
  if (ns0 > 0) stcg(kp.part + ((size_t)rid0 * 2 + 0) * kp.part_units + lu, sm.uacc()[0]);
  if (ns0 > 1) stcg(kp.part + ((size_t)rid0 * 2 + 1) * kp.part_units + lu, sm.uacc()[1]);
  if (ns1 > 0) stcg(kp.part + ((size_t)(rid0 + 1) * 2 + 0) * kp.part_units + lu, sm.uacc()[2]);
  if (ns1 > 1) stcg(kp.part + ((size_t)(rid0 + 1) * 2 + 1) * kp.part_units + lu, sm.uacc()[3]);
}

// ------------------------------------------------------------------------------------------------
// the two passes that run once per solve (rhsMax; x, r, s initialisation): direct loads, neighbours
// through the gather tables

template <bool MIXED>
__device__ void process_unit_direct(const KParams& kp, const GroupDev& g, int inst, int lu, int pt, const Smem& sm) {
  using V = typename Prec<MIXED>::V;
  const TopoDev& tp = g.tp;
  const int ni = tp.ni, nj = tp.nj, npx = tp.npx;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t = lu / g.nblk, blk = lu - (lu / g.nblk) * g.nblk;
  const int R = kp.serial ? nj : kp.rows_per_block;
  const int j0 = blk * R, j1 = min(nj, j0 + R);
  const long long pe = g.pad_elems;
  const int W = ni + 2;
  const int SW = (kWarps + 2) * (kp.max_ni + 2);
  double* stage = reinterpret_cast<double*>(smem_raw + sm.stage);
  const Slots si = slots_of(g, inst, sm);
  const int ns0 = nsums(pt, si.act(0));
  const int ns1 = g.nrhs > 1 ? nsums(pt, si.act(1)) : 0;
  const double* aW = g.a64[0] + inst * pe;
  const double* aS = g.a64[1] + inst * pe;
  const double* aC = g.a64[2] + inst * pe;

  unsigned long long vmax0 = 0ull, vmax1 = 0ull;

  if (pt == P_MAX) {
    // ring cells of r, s, z and q read 0 unless a neighbour pushes a value into them (the exchange leaves
    // unwritten halo points as they are, and the reference's r, s, z, q start with zero halos): zero the
    // west and east cells of the unit's rows, and the south / north rows at the tile's edges. Pushes come
    // after the next grid-wide wait.
    const int P = tp.P;
    const int nrow = j1 - j0;
    const int n_we = 2 * nrow, n_s = (j0 == 0) ? P : 0, n_n = (j1 == nj) ? P : 0;
    const int per = n_we + n_s + n_n;
    for (int idx = tid; idx < per * g.nrhs * (V_NVEC - 1); idx += kThreads) {
      const int sv = idx / per, e = idx - (idx / per) * per;
      const int s = sv / (V_NVEC - 1), v = 1 + sv - (sv / (V_NVEC - 1)) * (V_NVEC - 1);
      V* vb = vec_ptr<V>(g, inst, s, v);
      long long o;
      if (e < n_we) o = vidx(tp, t, j0 + (e >> 1), (e & 1) ? ni : -1);
      else if (e < n_we + n_s) o = ((long long)t * (nj + 2)) * P + (e - n_we);
      else o = ((long long)t * (nj + 2) + nj + 1) * P + (e - n_we - n_s);
      vb[o] = (V)0;
    }
  }

  for (int jc = j0; jc < j1; jc += kWarps) {
    const int nr = min(kWarps, j1 - jc);
    if (pt == P_INIT) {
      // x0 scaled by rhsNorm at the chunk's rows and neighbours (cg2d.py:227-228): interior points are
      // scaled, unwritten halo points keep cg2d_x
      const int total = (nr + 2) * W;
      for (int idx = tid; idx < total; idx += kThreads) {
        const int rr = idx / W, cc = idx - (idx / W) * W;
        const int j = jc + rr - 1, i = cc - 1;
        const bool own = (rr >= 1 && rr <= nr), iin = (i >= 0 && i < ni);
        if (!own && !iin) continue;
        int src;
        long long hp = -1;
        if (iin && j >= 0 && j < nj) {
          src = (t * nj + j) * ni + i;
        } else {
          if (i < 0) src = tp.nbr[t * nj + j];
          else if (i >= ni) src = tp.nbr[tp.T * nj + t * nj + j];
          else if (j < 0) src = tp.nbr[2 * tp.T * nj + t * ni + i];
          else src = tp.nbr[2 * tp.T * nj + tp.T * ni + t * ni + i];
          hp = ((long long)t * tp.npy + (j + tp.OLy)) * npx + (i + tp.OLx);
        }
        for (int s = 0; s < g.nrhs; ++s) {
          if (si.act(s) != A_ACTIVE) continue;
          const double* x0 = g.x0[s] + inst * pe;
          stage[s * SW + rr * W + cc] =
              (src >= 0) ? mul(__ldg(x0 + cmp_to_pad(tp, src)), si.rnorm(s)) : __ldg(x0 + hp);
        }
      }
      __syncthreads();
    }
    Lanes lp = {{0.0, 0.0, 0.0, 0.0}};
    if (warp < nr) {
      const int j = jc + warp;
      const long long prow = ((long long)t * tp.npy + (j + tp.OLy)) * npx + tp.OLx;
      for (int i = lane; i < ni; i += 32) {
        const long long po = prow + i;
        for (int s = 0; s < g.nrhs; ++s) {
          if (si.act(s) != A_ACTIVE) continue;
          double p0 = 0.0, p1 = 0.0;
          if (pt == P_MAX) {
            const double bv = __ldg(g.b[s] + inst * pe + po);
            const unsigned long long m =
                (unsigned long long)__double_as_longlong(fabs(mul(bv, si.norm(s))));   // cg2d.py:222-223
            if (s == 0) vmax0 = m > vmax0 ? m : vmax0;
            else vmax1 = m > vmax1 ? m : vmax1;
          } else {
            const double* st = stage + s * SW;
            const int sc = (warp + 1) * W + (i + 1);
            const double vc = st[sc], vw = st[sc - 1], ve = st[sc + 1], vs = st[sc - W], vn = st[sc + W];
            const long long vo = vidx(tp, t, j, i);
            stcg(vec_ptr<double>(g, inst, s, V_X) + vo, vc);
            const double bn = mul(mul(__ldg(g.b[s] + inst * pe + po), si.norm(s)), si.rnorm(s));   // cg2d.py:221,226
            const double ax = op_A<double>(__ldg(aW + po), __ldg(aW + po + 1), __ldg(aS + po), __ldg(aS + po + npx),
                                           __ldg(aC + po), vw, ve, vs, vn, vc);
            const V r0 = (V)sub(bn, ax);                                                   // cg2d.py:232
            V* rv = vec_ptr<V>(g, inst, s, V_R0);
            stcg(rv + vo, r0);
            push(tp, rv, t, j, i, r0, kp.gs);
            stcg(vec_ptr<V>(g, inst, s, V_S1) + vo, (V)0);                               // s = 0 (cg2d.py:231)
            p0 = mul((double)r0, (double)r0);
            p1 = bn;
          }
          if (kp.serial && pt != P_MAX) {
            double* pr = sm.prod() + ((s * 2 + 0) * kWarps + warp) * kp.max_ni;
            pr[i] = p0;
            pr[kWarps * kp.max_ni + i] = p1;
          } else if (s == 0) {
            lp.v[0] = add(lp.v[0], p0);
            lp.v[1] = add(lp.v[1], p1);
          } else {
            lp.v[2] = add(lp.v[2], p0);
            lp.v[3] = add(lp.v[3], p1);
          }
        }
      }
      if (pt == P_MAX) {
        for (int o = 16; o > 0; o >>= 1) {
          const unsigned long long y0 = __shfl_xor_sync(0xffffffffu, vmax0, o);
          const unsigned long long y1 = __shfl_xor_sync(0xffffffffu, vmax1, o);
          vmax0 = y0 > vmax0 ? y0 : vmax0;
          vmax1 = y1 > vmax1 ? y1 : vmax1;
        }
      } else if (!kp.serial) {
        row_sums(g, lp, sm, 0, true);
      }
    }
    if (pt == P_MAX) {
      if (warp < nr && lane == 0)
        for (int s = 0; s < g.nrhs; ++s)
          if (si.act(s) == A_ACTIVE) atomicMax(&kp.rmax[si.rid(s)], s == 0 ? vmax0 : vmax1);
      __syncthreads();
      continue;
    }
    __syncthreads();
    if (tid < 32) accumulate_chunk(kp, g, ns0, ns1, nr, 0, jc == j0, sm);
  }
  if (pt == P_MAX) return;
  if (tid < 32) finish_unit(kp, g, inst, lu, ns0, ns1, sm);
  __syncthreads();   // the unit accumulators are reused by the next unit
}

template <bool MIXED>
__device__ bool run_pass_direct(const KParams& kp, int pt, const Smem& sm) {
  const unsigned long long t0 = PROF_T0(kp);
  for (int u = blockIdx.x; u < kp.total_units; u += gridDim.x) {
    int gi = 0;
    while (gi + 1 < kp.ngroups && u >= kp.g[gi + 1].unit_base) ++gi;
    const GroupDev& g = kp.g[gi];
    const int rel = u - g.unit_base;
    const int inst = rel / g.units;
    if (!sm.opp()[g.op_base + inst]) continue;
    process_unit_direct<MIXED>(kp, g, inst, rel - inst * g.units, pt, sm);
  }
  PROF_ADD(kp, sm, PR_DIRECT, t0);
  return true;
}

// x ring cells at the start: the exchanged normalised first guess; unwritten points keep cg2d_x
// (cg2d.py:227-228). Later values are pushed by the owners as x is updated.
__device__ void init_x_ring(const KParams& kp, const Smem& sm) {
  const long long gstride = (long long)gridDim.x * kThreads;
  for (int gg = 0; gg < kp.ngroups; ++gg) {
    const GroupDev& g = kp.g[gg];
    const TopoDev& tp = g.tp;
    const int T = tp.T, nj = tp.nj, ni = tp.ni;
    const long long per = (long long)T * (2 * nj + 2 * ni);   // W, E [T][nj], S, N [T][ni]
    const long long tot = per * g.count * g.nrhs;
    for (long long idx = (long long)blockIdx.x * kThreads + threadIdx.x; idx < tot; idx += gstride) {
      const long long ins_slot = idx / per;
      const int h = (int)(idx - ins_slot * per);
      const int inst = (int)(ins_slot / g.nrhs), s = (int)(ins_slot - (long long)inst * g.nrhs);
      int t, j, i, src;
      if (h < 2 * T * nj) {
        const int side = h / (T * nj);
        const int r = h - side * T * nj;
        t = r / nj; j = r - t * nj;
        i = side == 0 ? -1 : ni;
        src = tp.nbr[side * T * nj + r];
      } else {
        const int h2 = h - 2 * T * nj;
        const int side = h2 / (T * ni);
        const int r = h2 - side * T * ni;
        t = r / ni; i = r - t * ni;
        j = side == 0 ? -1 : nj;
        src = tp.nbr[2 * T * nj + side * T * ni + r];
      }
      const double* x0 = g.x0[s] + inst * g.pad_elems;
      const double rn = sm.rnorm()[g.rhs_base + inst * g.nrhs + s];
      const double v = (src >= 0) ? mul(__ldg(x0 + cmp_to_pad(tp, src)), rn)
                                  : __ldg(x0 + ((long long)t * tp.npy + (j + tp.OLy)) * tp.npx + (i + tp.OLx));
      vec_ptr<double>(g, inst, s, V_X)[vidx(tp, t, j, i)] = v;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// pipelined passes: chunks of this CTA in order, bulk copies into two stage buffers

// this CTA's work units (dealt by build_unit_table), packed once at the start of the launch
//   x = gi | inst << 2 | lu << 10,   y = t | j0 << 8 | j1 << 19
struct Unit {
  int gi, inst, lu, t, j0, j1;
};
__device__ __forceinline__ Unit unit_at(const Smem& sm, int ui) {
  const int2 e = sm.utab()[ui];
  Unit u;
  u.gi = e.x & 3; u.inst = (e.x >> 2) & 255; u.lu = (unsigned)e.x >> 10;
  u.t = e.y & 255; u.j0 = (e.y >> 8) & 2047; u.j1 = (unsigned)e.y >> 19;
  return u;
}
__device__ void build_unit_table(const KParams& kp, const Smem& sm) {
  // Units are taken in this order: every group's full row blocks (instance, tile, block), then the shorter last
  // blocks of the tiles. They are dealt to the CTAs round-robin (unit_deal 0: every CTA gets the same number of
  // rows to within one unit) or as contiguous runs of that order (unit_deal 1: neighbouring blocks of a tile on
  // one CTA; the runs differ in length by at most one unit).
  const int R = kp.rows_per_block;
  int nfull = 0;
  for (int gi = 0; gi < kp.ngroups; ++gi) {
    const GroupDev& g = kp.g[gi];
    nfull += g.count * g.tp.T * (kp.serial ? 1 : g.tp.nj / R);
  }
  const int lo = (int)((long long)blockIdx.x * kp.total_units / gridDim.x);
  const int hi = (int)((long long)(blockIdx.x + 1) * kp.total_units / gridDim.x);
  const int n = kp.unit_deal ? hi - lo : (kp.total_units - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  for (int q = threadIdx.x; q < n; q += kThreads) {
    int o = kp.unit_deal ? lo + q : (int)blockIdx.x + q * (int)gridDim.x;
    const bool full = o < nfull;
    if (!full) o -= nfull;
    int gi = 0, inst = 0, t = 0, blk = 0;
    for (gi = 0; gi < kp.ngroups; ++gi) {
      const GroupDev& g = kp.g[gi];
      const int nf = kp.serial ? 1 : g.tp.nj / R;                                        // full blocks per tile
      const int per = full ? g.tp.T * nf : ((!kp.serial && g.tp.nj % R) ? g.tp.T : 0);   // units per instance
      if (o < g.count * per) {
        inst = o / per;
        const int r2 = o - inst * per;
        if (full) { t = r2 / nf; blk = r2 - t * nf; }
        else { t = r2; blk = nf; }
        break;
      }
      o -= g.count * per;
    }
    const GroupDev& g = kp.g[gi];
    const int lu = t * g.nblk + blk;
    const int Rg = kp.serial ? g.tp.nj : R;
    const int j0 = blk * Rg, j1 = min(g.tp.nj, j0 + Rg);
    sm.utab()[q] = make_int2(gi | (inst << 2) | (lu << 10), t | (j0 << 8) | (j1 << 19));
  }
  if (threadIdx.x == 0) sm.misc()[3] = n > 0 ? n : 0;
}

// position in this CTA's chunk sequence of a pass: unit ui of the table, first row jc; units of operators that
// take no part in the pass are skipped
struct Cursor {
  int ui, jc;
};
__device__ __forceinline__ bool cursor_unit(const KParams& kp, const Smem& sm, Cursor& c) {
  const int n = sm.misc()[3];
  for (++c.ui; c.ui < n; ++c.ui) {
    const Unit u = unit_at(sm, c.ui);
    if (sm.opp()[kp.g[u.gi].op_base + u.inst]) {
      c.jc = u.j0;
      return true;
    }
  }
  return false;
}
__device__ __forceinline__ bool cursor_first(const KParams& kp, const Smem& sm, Cursor& c) {
  c.ui = -1;
  c.jc = 0;
  return cursor_unit(kp, sm, c);
}
__device__ __forceinline__ bool cursor_next(const KParams& kp, const Smem& sm, Cursor& c) {
  const Unit u = unit_at(sm, c.ui);
  if (c.jc + kp.ch < u.j1) {
    c.jc += kp.ch;
    return true;
  }
  return cursor_unit(kp, sm, c);
}

struct Chunk {
  int gi, inst, lu, t, j0u, j1u, jc, nr;
};

// The group and stage layout of a chunk. ONE: the launch has one group, so both are read at addresses fixed at
// compile time (the parameter loads fold into the instructions that use them instead of loads by index).
template <bool ONE>
__device__ __forceinline__ const GroupDev& group_of(const KParams& kp, int gi) { return kp.g[ONE ? 0 : gi]; }
template <bool ONE>
__device__ __forceinline__ const StageLay& stage_lay(const KParams& kp, int gi, int pt) {
  if (!ONE) return kp.lay[gi][pt];
  switch (pt) {
    case P_S: return kp.lay[0][P_S];
    case P_X: return kp.lay[0][P_X];
    case P_Z: return kp.lay[0][P_Z];
    default: return kp.lay[0][P_R];
  }
}
__device__ __forceinline__ Chunk chunk_at(const KParams& kp, const Smem& sm, int ui, int jc) {
  const Unit u = unit_at(sm, ui);
  Chunk c;
  c.gi = u.gi; c.inst = u.inst; c.lu = u.lu; c.t = u.t; c.j0u = u.j0; c.j1u = u.j1;
  c.jc = jc;
  c.nr = min(kp.ch, u.j1 - jc);
  return c;
}

// the vector a pass stages as stencil input v (0, 1) of a solve
__device__ __forceinline__ int pass_vector(int pt, int k, int hidx, int v) {
  if (pt == P_S) return v == 0 ? V_Z : (((k + 1) & 1) ? V_S1 : V_S0);
  if (pt == P_X) return v == 0 ? ((k & 1) ? V_R1 : V_R0) : V_Q;
  if (pt == P_R) return v == 0 ? V_X : ((k & 1) ? V_S1 : V_S0);
  return (hidx & 1) ? V_R1 : V_R0;
}

// warp 0: bulk copies of chunk c into the stage buffer sb, completion on bar. Each lane owns one fixed copy
// (a lane whose copy is not needed moves 0 bytes): lane 0 the packed coefficient rows (pass R: lanes 0-2
// the three FP64 operator arrays), 3 the west/east push targets of the chunk's rows, 4 and 5 the south /
// north push targets (first / last chunk of a tile), 6 + 2 s + v vector v of slot s (rows jc-1 .. jc+nr,
// ring cells included), 10 + s the own rows of x (pass S).
__device__ void issue_chunk(const KParams& kp, const Chunk& c, int pt, int k, int hidx, const Smem& sm, int st) {
  const GroupDev& g = kp.g[c.gi];
  const TopoDev& tp = g.tp;
  const int lane = threadIdx.x & 31;
  const StageLay& L = kp.lay[c.gi][pt];
  unsigned char* sb = smem_raw + sm.stage + st * kp.stage_bytes;
  unsigned long long* bar = &sm.full()[st];
  const int rid0 = g.rhs_base + c.inst * g.nrhs;
  const bool act0 = sm.act()[rid0] == A_ACTIVE;
  const bool act1 = g.nrhs > 1 && sm.act()[rid0 + 1] == A_ACTIVE;
  const bool any = act0 || act1;
  const int T = tp.T, nj = tp.nj, ni = tp.ni, P = tp.P;
  const bool bottom = c.jc == 0, top = c.jc + c.nr == nj;
  void* dst = nullptr;
  const void* src = nullptr;
  unsigned bytes = 0;
  if (lane < 3) {
    if (any && L.packed && lane == 0) {
      const int op = (pt == P_X || pt == P_Z) ? 1 : 0;   // M = (pW, pS, pC) or A = (aW2d, aS2d, aC2d)
      const long long row = ((long long)(c.inst * 2 + op) * T + c.t) * (nj + 1) + c.jc;
      src = static_cast<const char*>(g.cpk) + row * 3 * g.ldc * L.csize;
      dst = sb + L.coef;
      bytes = (unsigned)((c.nr + 1) * 3 * g.ldc * L.csize);
    } else if (any && !L.packed) {
      src = g.a64[lane] + (long long)c.inst * g.pad_elems + ((long long)c.t * tp.npy + c.jc + tp.OLy) * tp.npx;
      dst = sb + L.coef + lane * L.coef_stride;
      bytes = (unsigned)((c.nr + 1) * tp.npx * 8);
    }
  } else if (lane < 6) {
    if (any) {
      if (lane == 3) {
        src = tp.tg + ((long long)c.t * nj + c.jc) * 4;
        dst = sb + L.twe;
        bytes = (unsigned)(c.nr * 16);
      } else if ((lane == 4 && bottom) || (lane == 5 && top)) {
        src = tp.tg + (long long)T * nj * 4 + ((long long)((lane - 4) * T + c.t) * tp.nip) * 2;
        dst = sb + (lane == 4 ? L.ts : L.tn);
        bytes = al16((unsigned)(ni * 8));
      }
    }
  } else if (lane < 10) {
    const int s = (lane - 6) >> 1, v = (lane - 6) & 1;
    if (s < g.nrhs && (s == 0 ? act0 : act1) && v < L.nvec) {
      const int sz = L.vsize[v];
      src = vec_ptr<const char>(g, c.inst, s, pass_vector(pt, k, hidx, v)) +
            ((long long)c.t * (nj + 2) + c.jc) * P * sz;
      dst = sb + L.vec[s][v];
      bytes = (unsigned)((c.nr + 2) * P * sz);
    }
  } else if (lane < 12) {
    const int s = lane - 10;
    if (pt == P_S && s < g.nrhs && (s == 0 ? act0 : act1) && sm.has_alpha()[rid0 + s]) {
      src = vec_ptr<const char>(g, c.inst, s, V_X) + ((long long)c.t * (nj + 2) + c.jc + 1) * P * 8;
      dst = sb + L.xo[s];
      bytes = (unsigned)(c.nr * P * 8);
    }
  }
  const unsigned total = __reduce_add_sync(0xffffffffu, bytes);
  if (lane == 0) mbar_arrive_expect_tx(bar, total);
  __syncwarp();
  if (bytes) bulk_g2s(dst, src, bytes, bar);
}

// compute one chunk from its stage buffer: warp w owns row jc + w, lane owns i = lane + 32m, m = 0, 1, ...
// (MAXM > 0: exactly MAXM column steps, unrolled; 0: any width). The right-hand sides of the instance active in
// the pass are processed in the same step, sharing the coefficient loads. In shared memory point (w, i) of a
// vector is element (w + 1) P + i + 1 (its neighbours at -1, +1, -P, +P) and of the packed coefficients element
// w 3 ldc + i (columns: W/pW, +ldc S/pS, +2 ldc C/pC; east face +1, north face +3 ldc). A point pushes its new
// values to the rings of the tiles that read it when it lies on the tile's edge (every point of the first and
// last row, the first and last point of the others).
//
// Each lane addresses its rows through base pointers set once per chunk (the point's row and the rows above and
// below, in shared memory; the output rows in global memory), so that a column step m is an immediate offset.
// MIXED fuses the FP32 stencils and vector updates (fmaf: a multiply-add rounded once) and the FP64 solution
// update; the dot products are FP32 products, exact in FP64, accumulated with FP64 fused multiply-adds, which is
// the same arithmetic as a rounded product and a rounded sum. FP64 rounds every product and every sum as the
// reference does. SERIAL (the FORTRAN sum order) writes every product into the product rows instead of the lane
// partials.

template <bool MIXED> struct Ar;
template <> struct Ar<false> {   // FP64: rounded product, rounded sum (no contraction)
  __device__ static __forceinline__ double madd(double a, double b, double c) { return add(mul(a, b), c); }
  __device__ static __forceinline__ double dot(double a, double b, double c) { return add(c, mul(a, b)); }
};
template <> struct Ar<true> {    // MIXED: FP32 stencils and updates fused; FP64 solution update and dots fused
  __device__ static __forceinline__ float madd(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  __device__ static __forceinline__ double madd(double a, double b, double c) { return __fma_rn(a, b, c); }
  __device__ static __forceinline__ double dot(double a, double b, double c) { return __fma_rn(a, b, c); }
};

// apply_operator / apply_preconditioner with the arithmetic of Ar (same terms in the same order as op_A / op_M)
template <bool MIXED, class T>
__device__ __forceinline__ T stencil5(T c0, T c1, T c2, T c3, T c4, T v0, T v1, T v2, T v3, T v4) {
  using A = Ar<MIXED>;
  T t = mul(c0, v0);
  t = A::madd(c1, v1, t);
  t = A::madd(c2, v2, t);
  t = A::madd(c3, v3, t);
  return A::madd(c4, v4, t);
}

// one right-hand side's rows in a pipelined pass, set once per chunk: the two staged stencil inputs (point row
// and the rows above and below, shared memory), the global output rows, the pass coefficient and the product rows
// (SERIAL)
template <class V>
struct RowSet {
  const V *a_c, *a_s, *a_n;      // stencil input 0 (z in S, r in X / Z), rows w, w - 1, w + 1, column of this lane
  const V *b_c, *b_s, *b_n;      // stencil input 1 (s_{k-1} in S, q_k in X)
  const double* xo;              // S: staged x_{k-1}, row w, column of this lane
  V *o1, *o2;                    // S: s_k, q_k; X: r_{k+1}, z_{k+1}; Z: z (o2); rows of this lane's column
  double* ox;                    // S: x_k
  double* ck;                    // FP64: the exact-mode checkpoint row of this lane's column, or null
  double* pr;                    // SERIAL: product rows (kind 0, kind 1 at + kWarps max_ni) of this lane's column
  V coef;                        // beta_k (S), alpha_k (X)
  double alpha_prev;             // S: alpha_{k-1}
  bool upd;                      // S: alpha_{k-1} exists (x update due)
  V *vs1, *vs2;                  // bases of the output vectors (for the ring pushes)
  double* vsx;
};

template <bool MIXED, int MAXM, bool ONE, bool SERIAL>
__device__ Lanes compute_chunk(const KParams& kp, const Chunk& c, int pt, int k, const Slots& si, int st,
                               const Smem& sm) {
  Lanes lp = {{0.0, 0.0, 0.0, 0.0}};
  using V = typename Prec<MIXED>::V;
  using C = typename Prec<MIXED>::C;
  using A = Ar<MIXED>;
  const GroupDev& g = group_of<ONE>(kp, c.gi);
  const TopoDev& tp = g.tp;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= c.nr) return lp;
  const StageLay& L = stage_lay<ONE>(kp, c.gi, pt);
  const unsigned char* sb = smem_raw + sm.stage + st * kp.stage_bytes;
  const int ni = tp.ni, nj = tp.nj, t = c.t, w = warp, j = c.jc + w;
  const int P = tp.P, CL = g.ldc, CR = 3 * g.ldc;
  const long long grow = ((long long)t * (nj + 2) + j + 1) * P + 1;   // element of (t, j, 0)
  const long long pe = g.pad_elems;
  const long long prow = (long long)c.inst * pe + ((long long)t * tp.npy + j + tp.OLy) * tp.npx + tp.OLx;
  const bool er = (j == 0) | (j == nj - 1);
  PushTab ptab;
  ptab.twe = reinterpret_cast<const int4*>(sb + L.twe);
  ptab.ts = reinterpret_cast<const int2*>(sb + L.ts);
  ptab.tn = reinterpret_cast<const int2*>(sb + L.tn);
  ptab.ni = ni;
  ptab.nj = nj;
  ptab.lim = (unsigned)tp.T * (unsigned)(nj + 2) * (unsigned)P;
  ptab.gs = kp.gs;
  const int act0 = si.act(0), act1 = si.act(1);

  // pass S after convergence: the pending x update, un-normalised (cg2d.py:254, 266)
  if (pt == P_S && (act0 == A_FIN || act1 == A_FIN)) {
    for (int s = 0; s < g.nrhs; ++s) {
      if ((s == 0 ? act0 : act1) != A_FIN) continue;
      const V* so = vec_ptr<V>(g, c.inst, s, ((k + 1) & 1) ? V_S1 : V_S0);
      const double* x = vec_ptr<double>(g, c.inst, s, V_X);
      for (int i = lane; i < ni; i += 32) {
        double xv = ldcg(x + grow + i);
        if (si.has_alpha(s)) xv = A::madd(si.c2(s), (double)ldcg(so + grow + i), xv);
        const double xf = __ddiv_rn(xv, si.rnorm(s));
        g.x_out[s][prow + i] = xf;
        if (g.x_fortran[s]) g.x_fortran[s][prow + i] = xf;
      }
    }
  }
  const bool on0 = act0 == A_ACTIVE, on1 = act1 == A_ACTIVE;
  if (!on0 && !on1) return lp;

  // coefficient rows of this lane's column: W (and the east face at +1), S, N (the south face of row w + 1), C
  const C* cw = reinterpret_cast<const C*>(sb + L.coef) + w * CR + lane;
  const C* cs = cw + CL;
  const C* cn = cs + CR;
  const C* cc = cw + 2 * CL;
  const int off_c = (w + 1) * P + 1 + lane;   // this lane's column of row w in a staged vector

  auto rows = [&](int s) {
    RowSet<V> q;
    const V* a = reinterpret_cast<const V*>(sb + L.vec[s][0]) + off_c;
    const V* b = reinterpret_cast<const V*>(sb + L.vec[s][1]) + off_c;
    q.a_c = a; q.a_s = a - P; q.a_n = a + P;
    q.b_c = b; q.b_s = b - P; q.b_n = b + P;
    q.xo = reinterpret_cast<const double*>(sb + L.xo[s]) + w * P + 1 + lane;
    q.pr = SERIAL ? sm.prod() + ((s * 2) * kWarps + w) * kp.max_ni + lane : nullptr;
    q.ck = nullptr;
    q.ox = nullptr;
    q.vsx = nullptr;
    q.alpha_prev = 0.0;
    q.upd = false;
    if (pt == P_S) {
      q.vs1 = vec_ptr<V>(g, c.inst, s, (k & 1) ? V_S1 : V_S0);
      q.vs2 = vec_ptr<V>(g, c.inst, s, V_Q);
      q.vsx = vec_ptr<double>(g, c.inst, s, V_X);
      q.ox = q.vsx + grow + lane;
      q.coef = (V)si.c1(s);
      q.alpha_prev = si.c2(s);
      q.upd = si.has_alpha(s) != 0;
      if (!MIXED && kp.ck_s && ((k + 1) % kp.ck_every) == 0)
        q.ck = kp.ck_s + ((k + 1) / kp.ck_every) * kp.ck_stride + prow + lane;
    } else {
      q.vs1 = vec_ptr<V>(g, c.inst, s, ((k + 1) & 1) ? V_R1 : V_R0);
      q.vs2 = vec_ptr<V>(g, c.inst, s, V_Z);
      q.coef = (V)si.c1(s);
      if (!MIXED && pt == P_X && kp.ck_r && ((k + 1) % kp.ck_every) == 0)
        q.ck = kp.ck_r + ((k + 1) / kp.ck_every) * kp.ck_stride + prow + lane;
    }
    q.o1 = q.vs1 + grow + lane;
    q.o2 = q.vs2 + grow + lane;
    return q;
  };

  // NS right-hand sides q[0..NS-1]; sums into acc[s][kind]
  auto run = [&](auto ns_tag, const RowSet<V>* q, double (&acc)[2][2]) {
    constexpr int NS = decltype(ns_tag)::value;
    auto col = [&](int m) {
      const int i = lane + 32 * m;
      const int o = 32 * m;
      const bool edge = er | (i == 0) | (i == ni - 1);
      if (pt == P_S) {
        // s_k = z_k + beta_k s_{k-1} (cg2d.py:249) at the point and its neighbours; q_k = A s_k (cg2d.py:251);
        // x_k = x_{k-1} + alpha_{k-1} s_{k-1} (cg2d.py:254); s_k.q_k (cg2d.py:252)
        const C aw = cw[o], ae = cw[o + 1], as = cs[o], an = cn[o], ac = cc[o];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const RowSet<V>& r = q[s];
          const V be = r.coef;
          const V sp = r.b_c[o];
          const V vc = A::madd(be, sp, r.a_c[o]);
          const V vw = A::madd(be, r.b_c[o - 1], r.a_c[o - 1]);
          const V ve = A::madd(be, r.b_c[o + 1], r.a_c[o + 1]);
          const V vs = A::madd(be, r.b_s[o], r.a_s[o]);
          const V vn = A::madd(be, r.b_n[o], r.a_n[o]);
          const V qv = stencil5<MIXED, C>(aw, ae, as, an, ac, vw, ve, vs, vn, vc);
          stcg(r.o1 + o, vc);
          stcg(r.o2 + o, qv);
          if constexpr (!MIXED) {
            if (r.ck) r.ck[o] = (double)vc;                                      // checkpoint s_k
          }
          double xn = 0.0;
          if (r.upd) {
            xn = A::madd(r.alpha_prev, (double)sp, r.xo[o]);
            stcg(r.ox + o, xn);
          }
          if (edge) {
            push_s(ptab, r.vs1, j, w, i, vc);
            push_s(ptab, r.vs2, j, w, i, qv);
            if (MIXED && r.upd) push_s(ptab, r.vsx, j, w, i, xn);   // x's neighbours: replacement pass only
          }
          if constexpr (SERIAL) r.pr[o] = mul((double)vc, (double)qv);
          else acc[s][0] = A::dot((double)vc, (double)qv, acc[s][0]);
        }
      } else {
        // X: r_{k+1} = r_k - alpha_k q_k (cg2d.py:255) at the point and its neighbours; z_{k+1} = M r_{k+1}
        //    (cg2d.py:245); r.r and z.r (cg2d.py:256, 246).  Z: z = M r and z.r
        const C pw = cw[o], pe_ = cw[o + 1], ps = cs[o], pn = cn[o], pc = cc[o];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const RowSet<V>& r = q[s];
          V vc, vw, ve, vs, vn;
          if (pt == P_X) {
            const V na = -r.coef;
            vc = A::madd(na, r.b_c[o], r.a_c[o]);
            vw = A::madd(na, r.b_c[o - 1], r.a_c[o - 1]);
            ve = A::madd(na, r.b_c[o + 1], r.a_c[o + 1]);
            vs = A::madd(na, r.b_s[o], r.a_s[o]);
            vn = A::madd(na, r.b_n[o], r.a_n[o]);
          } else {
            vc = r.a_c[o]; vw = r.a_c[o - 1]; ve = r.a_c[o + 1]; vs = r.a_s[o]; vn = r.a_n[o];
          }
          const V z = stencil5<MIXED, C>(pc, pw, pe_, ps, pn, vc, vw, ve, vs, vn);
          if (pt == P_X) stcg(r.o1 + o, vc);
          if constexpr (!MIXED) {
            if (r.ck) r.ck[o] = (double)vc;                                      // checkpoint r_{k+1}
          }
          stcg(r.o2 + o, z);
          if (edge) {
            if (pt == P_X) push_s(ptab, r.vs1, j, w, i, vc);
            push_s(ptab, r.vs2, j, w, i, z);
          }
          if constexpr (SERIAL) {
            if (pt == P_X) {
              r.pr[o] = mul((double)vc, (double)vc);
              r.pr[o + kWarps * kp.max_ni] = mul((double)z, (double)vc);
            } else {
              r.pr[o] = mul((double)z, (double)vc);
            }
          } else if (pt == P_X) {
            acc[s][0] = A::dot((double)vc, (double)vc, acc[s][0]);
            acc[s][1] = A::dot((double)z, (double)vc, acc[s][1]);
          } else {
            acc[s][0] = A::dot((double)z, (double)vc, acc[s][0]);
          }
        }
      }
    };
    if constexpr (MAXM > 0) {
#pragma unroll
      for (int m = 0; m < MAXM; ++m)
        if (lane + 32 * m < ni) col(m);
    } else {
      for (int m = 0; lane + 32 * m < ni; ++m) col(m);
    }
  };

  if (pt == P_R) {
    // the FP64 true residual b - A x_{k+1}, x_{k+1} = x_k + alpha_k s_k formed on the fly (cg2d.py:232, 254)
    const double* aw = reinterpret_cast<const double*>(sb + L.coef);
    const double* as = reinterpret_cast<const double*>(sb + L.coef + L.coef_stride);
    const double* ac = reinterpret_cast<const double*>(sb + L.coef + 2 * L.coef_stride);
    const int NP = tp.npx, col0 = tp.OLx;
    for (int s = 0; s < g.nrhs; ++s) {
      if (!(s == 0 ? on0 : on1)) continue;
      const double* xr = reinterpret_cast<const double*>(sb + L.vec[s][0]);
      const V* sk = reinterpret_cast<const V*>(sb + L.vec[s][1]);
      const double alpha = si.c1(s);
      V* r_out = vec_ptr<V>(g, c.inst, s, ((k + 1) & 1) ? V_R1 : V_R0);
      double* pr = SERIAL ? sm.prod() + ((s * 2) * kWarps + w) * kp.max_ni : nullptr;
      auto x1 = [&](double xx, V ss) -> double { return A::madd(alpha, (double)ss, xx); };
      for (int i = lane; i < ni; i += 32) {
        const int rc = (w + 1) * P + i + 1;
        const double vc = x1(xr[rc], sk[rc]);
        const double vw = x1(xr[rc - 1], sk[rc - 1]);
        const double ve = x1(xr[rc + 1], sk[rc + 1]);
        const double vs = x1(xr[rc - P], sk[rc - P]);
        const double vn = x1(xr[rc + P], sk[rc + P]);
        const int cr = w * NP + col0 + i;
        const double bn = mul(mul(__ldg(g.b[s] + prow + i), si.norm(s)), si.rnorm(s));
        const V r = (V)sub(bn, op_A<double>(aw[cr], aw[cr + 1], as[cr], as[cr + NP], ac[cr], vw, ve, vs, vn, vc));
        stcg(r_out + grow + i, r);
        if (er | (i == 0) | (i == ni - 1)) push_s(ptab, r_out, j, w, i, r);
        if constexpr (SERIAL) pr[i] = mul((double)r, (double)r);
        else if (s == 0) lp.v[0] = A::dot((double)r, (double)r, lp.v[0]);
        else lp.v[2] = A::dot((double)r, (double)r, lp.v[2]);
      }
    }
    return lp;
  }

  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  if (on0 && on1) {
    const RowSet<V> q[2] = {rows(0), rows(1)};
    run(std::integral_constant<int, 2>{}, q, acc);
    lp.v[0] = acc[0][0]; lp.v[1] = acc[0][1]; lp.v[2] = acc[1][0]; lp.v[3] = acc[1][1];
  } else {
    const int s = on0 ? 0 : 1;
    const RowSet<V> q[1] = {rows(s)};
    run(std::integral_constant<int, 1>{}, q, acc);
    if (s == 0) { lp.v[0] = acc[0][0]; lp.v[1] = acc[0][1]; }
    else { lp.v[2] = acc[0][0]; lp.v[3] = acc[0][1]; }
  }
  return lp;
}

// Copy pipeline of a pass. The producer warp walks this CTA's chunks, issues each chunk's bulk copies into the
// next stage buffer (full barrier) and, before it reuses a stage, waits until the compute warps are done with it
// (empty barrier) and folds that chunk's row sums into its unit's partial sums, in chunk order. The compute
// warps walk the same chunks: wait for the stage, compute, write their row sums, release the stage. Each thread
// keeps the parity bits of its role: the next wait on each stage's full (compute warps) and empty barrier
// (producer), the parity of each stage's latest copy and the stages whose chunk awaits its row sums (producer).
struct Pipe {
  unsigned fph, eph, cph, pend;
};

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// producer: wait until the compute warps release stage st, then add its chunk's rows to the unit partials
__device__ bool release_stage(const KParams& kp, int pt, const Smem& sm, int st, Pipe& pp,
                              unsigned long long& t_wait) {
  const unsigned long long t0 = kp.prof ? globaltimer() : 0ull;
  const bool ok = mbar_wait(&sm.empty()[st], (pp.eph >> st) & 1u, kp.timeout_ns);
  pp.eph ^= 1u << st;
  if (kp.prof) t_wait += globaltimer() - t0;
  if (!__all_sync(0xffffffffu, ok)) return false;
  pp.pend &= ~(1u << st);
  const int4 e = sm.pend()[st];
  const Chunk c = chunk_at(kp, sm, e.x, e.y);
  const GroupDev& g = kp.g[c.gi];
  const Slots si = slots_of(g, c.inst, sm);
  const int ns0 = nsums(pt, si.act(0));
  const int ns1 = g.nrhs > 1 ? nsums(pt, si.act(1)) : 0;
  accumulate_chunk(kp, g, ns0, ns1, c.nr, st, c.jc == c.j0u, sm);
  if (c.jc + c.nr >= c.j1u) finish_unit(kp, g, c.inst, c.lu, ns0, ns1, sm);
  return true;
}

__device__ bool produce_pass(const KParams& kp, int pt, int k, int hidx, const Smem& sm, Pipe& pp) {
  const int lane = threadIdx.x & 31;
  const int ns = kp.nstage[pt];
  const unsigned long long t_start = kp.prof ? globaltimer() : 0ull;
  unsigned long long t_wait = 0ull;
  int st = 0;
  bool ok = true;
  Cursor cur;
  bool have = cursor_first(kp, sm, cur);
  while (have) {
    if ((pp.pend >> st) & 1u) {
      if (!release_stage(kp, pt, sm, st, pp, t_wait)) { ok = false; break; }
    }
    const Chunk c = chunk_at(kp, sm, cur.ui, cur.jc);
    issue_chunk(kp, c, pt, k, hidx, sm, st);
    pp.cph ^= 1u << st;
    if (lane == 0) sm.pend()[st] = make_int4(cur.ui, cur.jc, 0, 0);
    __syncwarp();
    pp.pend |= 1u << st;
    st = (st + 1 == ns) ? 0 : st + 1;
    have = cursor_next(kp, sm, cur);
  }
  // the last chunks, oldest first
  for (int q = 0; q < ns && ok; ++q) {
    if ((pp.pend >> st) & 1u) ok = release_stage(kp, pt, sm, st, pp, t_wait);
    st = (st + 1 == ns) ? 0 : st + 1;
  }
  if (!ok) {
    if (lane == 0) note_timeout(kp.gs, 2u, (unsigned)pt);
    // a bounded wait for copies still in flight into this CTA's shared memory
    for (int s2 = 0; s2 < kMaxStages; ++s2)
      if ((pp.pend >> s2) & 1u) mbar_wait(&sm.full()[s2], ((pp.cph >> s2) & 1u) ^ 1u, kp.timeout_ns);
    pp.pend = 0u;
  }
  if (kp.prof && lane == 0) {
    sm.pacc()[PR_ISSUE] += (globaltimer() - t_start) - t_wait;
    sm.pacc()[PR_PWAIT] += t_wait;
  }
  return ok;
}

template <bool MIXED, int MAXM, bool ONE, bool SERIAL>
__device__ bool consume_pass(const KParams& kp, int pt, int k, const Smem& sm, Pipe& pp) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ns = kp.nstage[pt];
  int st = 0;
  Cursor cur;
  bool have = cursor_first(kp, sm, cur);
  while (have) {
    unsigned long long t0 = PROF_T0(kp);
    const bool ok = mbar_wait(&sm.full()[st], (pp.fph >> st) & 1u, kp.timeout_ns);
    pp.fph ^= 1u << st;
    PROF_ADD(kp, sm, PR_MBAR, t0);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) note_timeout(kp.gs, 2u, (unsigned)pt);
      return false;
    }
    t0 = PROF_T0(kp);
    const Chunk c = chunk_at(kp, sm, cur.ui, cur.jc);
    const GroupDev& g = group_of<ONE>(kp, c.gi);
    const Slots si = slots_of(g, c.inst, sm);
    const Lanes lp = compute_chunk<MIXED, MAXM, ONE, SERIAL>(kp, c, pt, k, si, st, sm);
    if (!SERIAL && warp < c.nr) row_sums(g, lp, sm, st, pt == P_X);
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty()[st]);
    PROF_ADD(kp, sm, PR_COMP, t0);
    st = (st + 1 == ns) ? 0 : st + 1;
    have = cursor_next(kp, sm, cur);
  }
  return true;
}

template <bool MIXED, int MAXM, bool ONE, bool SERIAL>
__device__ bool run_pass_pipe(const KParams& kp, int pt, int k, int hidx, const Smem& sm, Pipe& pp) {
  bool ok;
  if ((threadIdx.x >> 5) == kProducer) ok = produce_pass(kp, pt, k, hidx, sm, pp);
  else ok = consume_pass<MIXED, MAXM, ONE, SERIAL>(kp, pt, k, sm, pp);
  const unsigned long long td = PROF_T0(kp);
  const int bad = __syncthreads_or(!ok);
  PROF_ADD(kp, sm, PR_DRAIN, td);
  return !bad;
}

// ------------------------------------------------------------------------------------------------

// which group / instance / slot a global solve index belongs to
__device__ __forceinline__ void locate(const KParams& kp, int r, int& gi, int& inst, int& slot) {
  gi = 0;
  while (gi + 1 < kp.ngroups && r >= kp.g[gi + 1].rhs_base) ++gi;
  const int rel = r - kp.g[gi].rhs_base;
  inst = rel / kp.g[gi].nrhs;
  slot = rel - inst * kp.g[gi].nrhs;
}

// tolerance and iteration limit of solve r
__device__ __forceinline__ double solve_tol(const KParams& kp, int r) {
  int gi, inst, slot;
  locate(kp, r, gi, inst, slot);
  return kp.g[gi].tol[slot];
}
__device__ __forceinline__ int solve_max_iters(const KParams& kp, int r) {
  int gi, inst, slot;
  locate(kp, r, gi, inst, slot);
  return kp.g[gi].max_iters[slot];
}

// publish the actions of this pass: act[] for every solve and opp[] for every operator
__device__ void set_actions(const KParams& kp, const Smem& sm, int my_act, double my_c1, double my_c2) {
  const int tid = threadIdx.x;
  const unsigned long long t0 = PROF_T0(kp);
  if (tid < kp.total_ops) sm.opp()[tid] = 0;
  __syncthreads();
  if (tid < kp.total_rhs) {
    sm.act()[tid] = my_act;
    sm.c1()[tid] = my_c1;
    sm.c2()[tid] = my_c2;
    if (my_act != A_NONE) {
      int gi, inst, slot;
      locate(kp, tid, gi, inst, slot);
      sm.opp()[kp.g[gi].op_base + inst] = 1;
    }
  }
  __syncthreads();
  PROF_ADD(kp, sm, PR_CTRL, t0);
}

template <bool MIXED, int MAXM, bool ONE, int CPS, bool SERIAL>
__global__ void __launch_bounds__(kThreads, CPS) cg2d_persistent(const __grid_constant__ KParams kp) {
  const Smem sm = carve(kp.max_ni, kp.serial);
  const int tid = threadIdx.x;
  unsigned target = (unsigned)kp.test_missing;
  Pipe pp = {0u, 0u, 0u, 0u};
  const unsigned long long t_start = PROF_T0(kp);
  if (tid < kProfSlots) sm.pacc()[tid] = 0ull;
  if (tid == 0) {
    for (int s = 0; s < kMaxStages; ++s) {
      mbar_init(&sm.full()[s], 1);          // the producer's arrive (with the copies' byte count)
      mbar_init(&sm.empty()[s], kWarps);    // one arrive per compute warp
    }
    fence_mbar_init();
  }
  build_unit_table(kp, sm);
  __syncthreads();

  // state of solve `tid` (identical in every CTA: computed from the same write-once sums), kept in shared
  // memory so that it holds no registers while the passes run
  const bool own = tid < kp.total_rhs;
  SolveState* S = sm.state() + (own ? tid : kMaxSolves);
  if (own) {
    int gi, inst, slot;
    locate(kp, tid, gi, inst, slot);
    const GroupDev& g = kp.g[gi];
    sm.norm()[tid] = g.norm_arr ? g.norm_arr[inst] : g.norm;
    sm.rnorm()[tid] = 1.0;
    sm.has_alpha()[tid] = 0;
    S->eta = 0.0;
    S->eta_prev = 1.0;
    S->alpha = 0.0;
    S->rr = 0.0;
    S->k_done = -1;
    S->nrep = 0;
  }
  int k = 0;
  bool ok = true;

  // ---- rhsMax = max |b cg2dNorm| (cg2d.py:221-225)
  set_actions(kp, sm, own ? A_ACTIVE : A_NONE, 0.0, 0.0);
  ok = run_pass_direct<MIXED>(kp, P_MAX, sm);
  ok = grid_sync(kp, target, P_MAX, 0, sm) && ok;
  if (!ok) goto epilogue;
  if (own) {
    const double rhsMax = __longlong_as_double((long long)__ldcg(&kp.rmax[tid]));
    sm.rnorm()[tid] = (rhsMax != 0.0) ? __ddiv_rn(1.0, rhsMax) : 1.0;
  }
  // ---- x = x0 rhsNorm, r = b - A x, s = 0, err^2, sumRHS (cg2d.py:226-236)
  set_actions(kp, sm, own ? A_ACTIVE : A_NONE, 0.0, 0.0);
  init_x_ring(kp, sm);
  ok = run_pass_direct<MIXED>(kp, P_INIT, sm);
  ok = grid_sync(kp, target, P_INIT, 0, sm) && ok;
  if (!ok) goto epilogue;
  if (own) S->rr = __ldcg(hist_ptr(kp, tid, H_RRR, 0));
  // ---- z = M r and eta for the first iteration
  set_actions(kp, sm, own ? A_ACTIVE : A_NONE, 0.0, 0.0);
  ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL>(kp, P_Z, 0, 0, sm, pp);
  ok = grid_sync(kp, target, P_Z, 0, sm) && ok;
  if (!ok) goto epilogue;
  if (own) S->eta = __ldcg(hist_ptr(kp, tid, H_ETAZ, 0));

  for (k = 0;; ++k) {
    // stop rule before every iteration (cg2d.py:238-241)
    int a = A_NONE;
    double beta = 0.0;
    if (own && S->k_done < 0) {
      const double tol = solve_tol(kp, tid);
      if (!(k < solve_max_iters(kp, tid)) || S->rr < tol * tol) {       // cg2d.py:219, 241
        S->k_done = k;
        a = A_FIN;
      } else {
        a = A_ACTIVE;
        beta = __ddiv_rn(S->eta, S->eta_prev);                           // cg2d.py:247
        S->eta_prev = S->eta;                                             // cg2d.py:248
      }
    }
    set_actions(kp, sm, a, beta, own ? S->alpha : 0.0);
    const int any_active = __syncthreads_or(a == A_ACTIVE);
    const int any_fin = __syncthreads_or(a == A_FIN);
    if (!any_active && !any_fin) break;
    ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL>(kp, P_S, k, k, sm, pp);
    ok = grid_sync(kp, target, P_S, k, sm) && ok;
    if (!ok) goto epilogue;
    if (!any_active) break;
    if (a == A_ACTIVE) {
      const double sq = __ldcg(hist_ptr(kp, tid, H_SQ, k));
      S->alpha = __ddiv_rn(S->eta, sq);                                   // cg2d.py:252-253
      sm.has_alpha()[tid] = 1;                                            // read from the next pass on
    }
    // ---- r, z, err^2 and the next eta; or, every replace_every iterations (MIXED), the true residual
    int ax = A_NONE, ar = A_NONE;
    if (a == A_ACTIVE) {
      const double rep = kp.replace_above * solve_tol(kp, tid);
      if (kp.mixed && kp.replace_every > 0 && ((k + 1) % kp.replace_every) == 0 && S->rr > rep * rep) ar = A_ACTIVE;
      else ax = A_ACTIVE;
    }
    if (__syncthreads_or(ax != A_NONE)) {
      set_actions(kp, sm, ax, own ? S->alpha : 0.0, 0.0);
      ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL>(kp, P_X, k, k + 1, sm, pp);
      ok = grid_sync(kp, target, P_X, k + 1, sm) && ok;
      if (!ok) goto epilogue;
      if (ax == A_ACTIVE) {
        S->rr = __ldcg(hist_ptr(kp, tid, H_RRX, k + 1));
        S->eta = __ldcg(hist_ptr(kp, tid, H_ETAX, k + 1));
      }
    }
    if (__syncthreads_or(ar != A_NONE)) {
      set_actions(kp, sm, ar, own ? S->alpha : 0.0, 0.0);
      ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL>(kp, P_R, k, k + 1, sm, pp);
      ok = grid_sync(kp, target, P_R, k + 1, sm) && ok;
      if (!ok) goto epilogue;
      if (ar == A_ACTIVE) {
        S->rr = __ldcg(hist_ptr(kp, tid, H_RRR, k + 1));
        ++S->nrep;
      }
      set_actions(kp, sm, ar, 0.0, 0.0);
      ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL>(kp, P_Z, k, k + 1, sm, pp);
      ok = grid_sync(kp, target, P_Z, k + 1, sm) && ok;
      if (!ok) goto epilogue;
      if (ar == A_ACTIVE) S->eta = __ldcg(hist_ptr(kp, tid, H_ETAZ, k + 1));
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
            const int sj = spl / tp.npx, si_ = spl - (spl / tp.npx) * tp.npx;
            const bool sin = sj >= tp.OLy && sj < tp.OLy + tp.nj && si_ >= tp.OLx && si_ < tp.OLx + tp.ni;
            const double rn = sm.rnorm()[g.rhs_base + in * g.nrhs + s];
            v = sin ? mul(__ldg(x0 + sp), rn) : __ldg(x0 + sp);
          }
          g.x_fortran[s][off] = v;
        }
      }
    }
  }
  if (blockIdx.x == 0 && own) {
    int gi, inst, slot;
    locate(kp, tid, gi, inst, slot);
    const GroupDev& g = kp.g[gi];
    const double rr = S->rr, tol = solve_tol(kp, tid);
    cg2d_diag_t d;
    d.firstResidual = sqrt(__ldcg(hist_ptr(kp, tid, H_RRR, 0)));
    d.lastResidual = sqrt(rr);
    d.sumRHS = __ldcg(hist_ptr(kp, tid, H_SUM, 0));
    d.rhsMax = __longlong_as_double((long long)__ldcg(&kp.rmax[tid]));
    d.numIters = S->k_done >= 0 ? S->k_done : k;
    d.replacements = S->nrep;
    d.reserved = 0;
    const unsigned err = __ldcg(&kp.gs[1]);
    if (!ok || err != 0u) d.status = err != 0u ? (int)err : CG2D_BARRIER_TIMEOUT;
    else if (rr != rr) d.status = CG2D_NAN;
    else if (!(rr < tol * tol)) d.status = CG2D_NOT_CONVERGED;
    else d.status = CG2D_OK;
    if (!ok) { d.firstResidual = d.lastResidual = d.sumRHS = __longlong_as_double(0x7ff8000000000000LL); }
    g.diag[slot][inst] = d;
  }
  if (kp.prof) __syncthreads();   // the producer warp's copy-issue time
  if (kp.prof && tid == 0 && blockIdx.x < kMaxCtas) {
    unsigned long long* o = kp.prof + 1 + (size_t)blockIdx.x * kProfSlots;
    const unsigned long long tot = globaltimer() - t_start;
    unsigned long long acc = 0;   // thread 0's phases (the copy issue runs on the producer warp, beside them)
    for (int i = 0; i < kProfSlots; ++i) o[i] = sm.pacc()[i];
    for (int i : {PR_BAR, PR_MBAR, PR_COMP, PR_FIN, PR_DIRECT, PR_DRAIN, PR_CTRL}) acc += sm.pacc()[i];
    o[PR_OTHER] = tot > acc ? tot - acc : 0ull;
    o[PR_TOTAL] = tot;
    if (blockIdx.x == 0) kp.prof[0] = gridDim.x;
  }
}

// ------------------------------------------------------------------------------------------------
// packed coefficients: [inst][A, M][T][nj+1][3][ldc] in the solver's precision, rows j = 0 .. nj and
// columns i = 0 .. ni of (aW2d, aS2d, aC2d) and (pW, pS, pC); columns past ni are 0

template <class C>
__global__ void pack_coef_kernel(GroupDev g) {
  const TopoDev& tp = g.tp;
  const int ldc = g.ldc, rows = tp.nj + 1;
  const long long tot = (long long)g.count * 2 * tp.T * rows * 3 * ldc;
  C* out = static_cast<C*>(g.cpk);
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r = idx / ldc;
    const int i = (int)(idx - r * ldc);
    const int w = (int)(r % 3); r /= 3;
    const int j = (int)(r % rows); r /= rows;
    const int t = (int)(r % tp.T); r /= tp.T;
    const int op = (int)(r % 2);
    const long long in = r / 2;
    C v = (C)0;
    if (i <= tp.ni) {
      const double a = g.a64[op * 3 + w][in * g.pad_elems + ((long long)t * tp.npy + j + tp.OLy) * tp.npx + i + tp.OLx];
      if constexpr (sizeof(C) == 4) v = __double2float_rn(a);
      else v = a;
    }
    out[idx] = v;
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
    // interior lam / cg2dNorm at (t, jj, ii)
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

// the kernel instantiation for a launch: precision, the column steps per row (ceil(max_ni / 32), unrolled for
// tiles up to 96 and 288 points wide), whether the launch has a single group and, FP64, the CTAs per SM it is
// built for (MIXED: always 2)
template <bool ONE, int CPS>
static const void* solver_fn_of(int mixed, int max_ni) {
  if (mixed) {
    if (max_ni <= 96) return (const void*)cg2d_persistent<true, 3, ONE, 2, false>;
    if (max_ni <= 288) return (const void*)cg2d_persistent<true, 9, ONE, 2, false>;
    return (const void*)cg2d_persistent<true, 0, ONE, 2, false>;
  }
  if (max_ni <= 96) return (const void*)cg2d_persistent<false, 3, ONE, CPS, false>;
  if (max_ni <= 288) return (const void*)cg2d_persistent<false, 9, ONE, CPS, false>;
  return (const void*)cg2d_persistent<false, 0, ONE, CPS, false>;
}
static const void* solver_fn(const KParams& kp) {
  // the FORTRAN sum order (bitwise parity, not speed): one generic build per precision
  if (kp.serial) return kp.mixed ? (const void*)cg2d_persistent<true, 0, false, 2, true>
                                 : (const void*)cg2d_persistent<false, 0, false, 1, true>;
  const bool two = !kp.mixed && kp.fp64_cps == 2;
  if (kp.ngroups == 1) return two ? solver_fn_of<true, 2>(kp.mixed, kp.max_ni) : solver_fn_of<true, 1>(kp.mixed, kp.max_ni);
  return two ? solver_fn_of<false, 2>(kp.mixed, kp.max_ni) : solver_fn_of<false, 1>(kp.mixed, kp.max_ni);
}

cudaError_t solver_occupancy(const KParams& kp, size_t smem, int* blocks_per_sm) {
  const void* fn = solver_fn(kp);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, kThreads, smem);
}

cudaError_t launch_solver(const KParams& kp, int grid, size_t smem, cudaStream_t stream) {
  const void* fn = solver_fn(kp);
  void* args[] = {const_cast<KParams*>(&kp)};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, smem, stream);
}

cudaError_t launch_pack_coef(const GroupDev& g, int mixed, cudaStream_t stream) {
  const long long tot = (long long)g.count * 2 * g.tp.T * (g.tp.nj + 1) * 3 * g.ldc;
  if (mixed) pack_coef_kernel<float><<<grid_for(tot), 256, 0, stream>>>(g);
  else pack_coef_kernel<double><<<grid_for(tot), 256, 0, stream>>>(g);
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
