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
__device__ __forceinline__ void stcg(float2* p, float2 v) { __stcg(p, v); }
__device__ __forceinline__ void stcg(double2* p, double2 v) { __stcg(p, v); }

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
constexpr size_t rowsum = opp + a16(sizeof(int) * kMaxOps);                 // double [kMaxStages][4][kMaxWarps]
constexpr size_t misc = rowsum + a16(sizeof(double) * kMaxStages * 4 * kMaxWarps);   // int [4]
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
//   rowsum                                 row sums of the chunk in each stage [stage][4 sums][kMaxWarps]
//   misc                                   [0] grid-wide wait ok, [3] units in utab
//   full, empty                            stage mbarriers: copies landed / compute warps done with the stage
//   pacc, uacc                             phase times (profiling); the current unit's partial sums
//   utab, pend                             this CTA's work units; the chunk in each stage awaiting its row sums
//   state                                  CG scalars of each solve (SolveState), one spare entry
// then prod (FORTRAN order, kWarps compute warps: [2 slots][2 kinds][kWarps][max_ni]) and the stage buffers at `stage` (kMaxStages x
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
  const int wpc = (int)(blockDim.x >> 5);   // warps per CTA
  const int nw = (int)gridDim.x * wpc;
  for (int s = (int)blockIdx.x * wpc + warp; s < 2 * kp.total_rhs; s += nw) {
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

// a solve's vector (ringed tiles, [T][nj+2][P]): element e is at [e] or, paired (GroupDev::pair), at [2 e]
template <class T>
__device__ __forceinline__ T* vec_ptr(const GroupDev& g, int inst, int slot, int which) {
  if (g.pair)
    return reinterpret_cast<T*>(g.vec + (long long)inst * g.vec_stride + g.vec_off[which]) + slot;
  return reinterpret_cast<T*>(g.vec + (long long)(inst * g.nrhs + slot) * g.vec_stride + g.vec_off[which]);
}
// the element stride of a group's vectors (1, or 2 when both solves are interleaved)
__device__ __forceinline__ int vstride(const GroupDev& g) { return g.pair ? 2 : 1; }
// element of point (t, j, i) in a ringed vector; -1 <= j <= nj, -1 <= i <= ni
__device__ __forceinline__ long long vidx(const TopoDev& tp, int t, int j, int i) {
  return ((long long)t * (tp.nj + 2) + j + 1) * tp.P + i + 1;
}

// one push store: target a (-1 = none) must lie inside the vector (lim elements); anything else is an internal
// inconsistency, recorded in the error word instead of stored
// (es: the vector's element stride in T)
template <class T>
__device__ __forceinline__ void push_one(T* vec, int a, T v, unsigned lim, unsigned* gs, int es = 1) {
  if ((unsigned)a < lim) stcg(vec + (long long)a * es, v);
  else if (a != -1) atomicCAS(&gs[1], 0u, (unsigned)CG2D_INTERNAL_ERROR);
}

// store the value of point (t, j, i) into the ring cells of the tiles that read it across an edge
template <class T>
__device__ __forceinline__ void push(const TopoDev& tp, T* vec, int t, int j, int i, T v, unsigned* gs, int es = 1) {
  const int* e;
  if (i == 0) e = tp.tg + ((size_t)t * tp.nj + j) * 4;
  else if (i == tp.ni - 1) e = tp.tg + ((size_t)t * tp.nj + j) * 4 + 2;
  else if (j == 0) e = tp.tg + (size_t)tp.T * tp.nj * 4 + ((size_t)t * tp.nip + i) * 2;
  else if (j == tp.nj - 1) e = tp.tg + (size_t)tp.T * tp.nj * 4 + ((size_t)(tp.T + t) * tp.nip + i) * 2;
  else return;
  const unsigned lim = (unsigned)tp.T * (unsigned)(tp.nj + 2) * (unsigned)tp.P;
  push_one(vec, __ldg(e), v, lim, gs, es);
  push_one(vec, __ldg(e + 1), v, lim, gs, es);
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
__device__ __forceinline__ void push_s(const PushTab& pt, T* vec, int j, int w, int i, T v, int es = 1) {
  int a, b;
  if (i == 0) { const int4 e = pt.twe[w]; a = e.x; b = e.y; }
  else if (i == pt.ni - 1) { const int4 e = pt.twe[w]; a = e.z; b = e.w; }
  else if (j == 0) { const int2 e = pt.ts[i]; a = e.x; b = e.y; }
  else if (j == pt.nj - 1) { const int2 e = pt.tn[i]; a = e.x; b = e.y; }
  else return;
  push_one(vec, a, v, pt.lim, pt.gs, es);
  push_one(vec, b, v, pt.lim, pt.gs, es);
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
// The row sums of a warp's lane partials: for each sum, the xor butterfly over the 32 lanes (lane l adds the
// partner l ^ o's value for o = 16, 8, 4, 2, 1). With several sums the butterflies share their first levels: at
// level o a lane keeps half of its sums and hands the other half to its partner, which keeps those (the partner of a
// lane that keeps sum q keeps q too, so every addition is the one the sum's own butterfly makes: the results are
// the same bit for bit), so that two sums cost 5 exchanges instead of 10 and four 7 instead of 20 (each exchange of
// a double is two shuffles). Sum q of 2 ends in lanes 16q..16q+15, of 4 in lanes 8q..8q+7.
__device__ __forceinline__ double xchg(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ double butterfly(double v) {
  for (int o = 16; o > 0; o >>= 1) v = add(v, xchg(v, o));
  return v;
}
// two sums: the result of a in lanes 0..15, of b in lanes 16..31
__device__ __forceinline__ double butterfly2(double a, double b) {
  const bool lo = (threadIdx.x & 16) == 0;
  double v = add(lo ? a : b, xchg(lo ? b : a, 16));
  for (int o = 8; o > 0; o >>= 1) v = add(v, xchg(v, o));
  return v;
}
// four sums: the result of sum q in lanes 8q..8q+7
__device__ __forceinline__ double butterfly4(double a0, double a1, double a2, double a3) {
  const bool lo16 = (threadIdx.x & 16) == 0, lo8 = (threadIdx.x & 8) == 0;
  const double b0 = add(lo16 ? a0 : a2, xchg(lo16 ? a2 : a0, 16));
  const double b1 = add(lo16 ? a1 : a3, xchg(lo16 ? a3 : a1, 16));
  double v = add(lo8 ? b0 : b1, xchg(lo8 ? b1 : b0, 8));
  for (int o = 4; o > 0; o >>= 1) v = add(v, xchg(v, o));
  return v;
}
// (two: the pass forms two sums per solve; otherwise the second kind is not read and not reduced)
__device__ __forceinline__ void row_sums(const GroupDev& g, const Lanes& lp, const Smem& sm, int st, bool two) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* rs = sm.rowsum() + st * 4 * kMaxWarps + warp;
  if (g.nrhs > 1 && two) {          // (slot, kind) = (0, 0), (0, 1), (1, 0), (1, 1)
    const double v = butterfly4(lp.v[0], lp.v[1], lp.v[2], lp.v[3]);
    if ((lane & 7) == 0) rs[(lane >> 3) * kMaxWarps] = v;
  } else if (g.nrhs > 1) {          // (0, 0), (1, 0)
    const double v = butterfly2(lp.v[0], lp.v[2]);
    if ((lane & 15) == 0) rs[(lane >> 3) * kMaxWarps] = v;
  } else if (two) {                 // (0, 0), (0, 1)
    const double v = butterfly2(lp.v[0], lp.v[1]);
    if ((lane & 15) == 0) rs[(lane >> 4) * kMaxWarps] = v;
  } else {
    const double v = butterfly(lp.v[0]);
    if (lane == 0) rs[0] = v;
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
      const double* rs = sm.rowsum() + (st * 4 + lane) * kMaxWarps;
      double v[kMaxWarps];
#pragma unroll
      for (int w = 0; w < kMaxWarps; ++w) v[w] = w < nr ? rs[w] : 0.0;
#pragma unroll
      for (int w = 0; w < kMaxWarps; ++w)
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
  const int SW = (kp.nw + 2) * (kp.max_ni + 2);
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
    for (int idx = tid; idx < per * g.nrhs * (V_NVEC - 1); idx += (int)blockDim.x) {
      const int sv = idx / per, e = idx - (idx / per) * per;
      const int s = sv / (V_NVEC - 1), v = 1 + sv - (sv / (V_NVEC - 1)) * (V_NVEC - 1);
      V* vb = vec_ptr<V>(g, inst, s, v);
      long long o;
      if (e < n_we) o = vidx(tp, t, j0 + (e >> 1), (e & 1) ? ni : -1);
      else if (e < n_we + n_s) o = ((long long)t * (nj + 2)) * P + (e - n_we);
      else o = ((long long)t * (nj + 2) + nj + 1) * P + (e - n_we - n_s);
      vb[o * vstride(g)] = (V)0;
    }
  }

  for (int jc = j0; jc < j1; jc += kp.nw) {
    const int nr = min(kp.nw, j1 - jc);
    if (pt == P_INIT) {
      // x0 scaled by rhsNorm at the chunk's rows and neighbours (cg2d.py:227-228): interior points are
      // scaled, unwritten halo points keep cg2d_x
      const int total = (nr + 2) * W;
      for (int idx = tid; idx < total; idx += (int)blockDim.x) {
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
            const int es = vstride(g);
            const long long vo = vidx(tp, t, j, i) * es;
            stcg(vec_ptr<double>(g, inst, s, V_X) + vo, vc);
            const double bn = mul(mul(__ldg(g.b[s] + inst * pe + po), si.norm(s)), si.rnorm(s));   // cg2d.py:221,226
            const double ax = op_A<double>(__ldg(aW + po), __ldg(aW + po + 1), __ldg(aS + po), __ldg(aS + po + npx),
                                           __ldg(aC + po), vw, ve, vs, vn, vc);
            const V r0 = (V)sub(bn, ax);                                                   // cg2d.py:232
            V* rv = vec_ptr<V>(g, inst, s, V_R0);
            stcg(rv + vo, r0);
            push(tp, rv, t, j, i, r0, kp.gs, es);
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
  const long long gstride = (long long)gridDim.x * blockDim.x;
  for (int gg = 0; gg < kp.ngroups; ++gg) {
    const GroupDev& g = kp.g[gg];
    const TopoDev& tp = g.tp;
    const int T = tp.T, nj = tp.nj, ni = tp.ni;
    const long long per = (long long)T * (2 * nj + 2 * ni);   // W, E [T][nj], S, N [T][ni]
    const long long tot = per * g.count * g.nrhs;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot; idx += gstride) {
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
      vec_ptr<double>(g, inst, s, V_X)[vidx(tp, t, j, i) * vstride(g)] = v;
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
  for (int q = threadIdx.x; q < n; q += (int)blockDim.x) {
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
    // (paired: slot 0's lanes copy the rows of both solves)
    const int s = (lane - 6) >> 1, v = (lane - 6) & 1;
    const bool on = g.pair ? (s == 0 && any) : (s < g.nrhs && (s == 0 ? act0 : act1));
    if (on && v < L.nvec) {
      const int sz = L.vsize[v] * (g.pair ? 2 : 1);
      src = vec_ptr<const char>(g, c.inst, s, pass_vector(pt, k, hidx, v)) +
            ((long long)c.t * (nj + 2) + c.jc) * P * sz;
      dst = sb + L.vec[s][v];
      bytes = (unsigned)((c.nr + 2) * P * sz);
    }
  } else if (lane < 12) {
    const int s = lane - 10;
    const bool on = g.pair ? (s == 0 && any) : (s < g.nrhs && (s == 0 ? act0 : act1));
    if (pt == P_S && on) {   // every S pass (before alpha_{k-1}: x unchanged)
      const int sz = g.pair ? 16 : 8;
      src = vec_ptr<const char>(g, c.inst, s, V_X) + ((long long)c.t * (nj + 2) + c.jc + 1) * P * sz;
      dst = sb + L.xo[s];
      bytes = (unsigned)(c.nr * P * sz);
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

// ---- both right-hand sides of an instance at once (MIXED, GroupDev::pair): every vector element is a float2 of the
// two solves (x a double2), so one shared-memory load, one packed FP32 multiply-add (fma.rn.f32x2) and one store
// serve both. The arithmetic of each solve is that of compute_chunk's MIXED path, term for term.

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
// stencil5 (apply_operator / apply_preconditioner terms in the reference's order) on both solves
__device__ __forceinline__ float2 stencil5p(float c0, float c1, float c2, float c3, float c4, float2 v0, float2 v1,
                                           float2 v2, float2 v3, float2 v4) {
  float2 t = mul2(f2(c0), v0);
  t = fma2(f2(c1), v1, t);
  t = fma2(f2(c2), v2, t);
  t = fma2(f2(c3), v3, t);
  return fma2(f2(c4), v4, t);
}
__device__ __forceinline__ void stcg2(float2* p, float2 v) { stcg(p, v); }
__device__ __forceinline__ void stcg2(double2* p, double2 v) { stcg(p, v); }
template <class T>
__device__ __forceinline__ void push_pair(const PushTab& pt, T* vec, int j, int w, int i, T v) {
  push_s(pt, vec, j, w, i, v);   // an element of the pair vector is the pair itself
}

template <int MAXM, bool ONE>
__device__ Lanes compute_pair(const KParams& kp, const Chunk& c, int pt, int k, const Slots& si, int st,
                              const Smem& sm) {
  Lanes lp = {{0.0, 0.0, 0.0, 0.0}};
  const GroupDev& g = group_of<ONE>(kp, c.gi);
  const TopoDev& tp = g.tp;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const StageLay& L = stage_lay<ONE>(kp, c.gi, pt);
  const unsigned char* sb = smem_raw + sm.stage + st * kp.stage_bytes;
  const int ni = tp.ni, nj = tp.nj, t = c.t, w = warp, j = c.jc + w;
  const int P = tp.P, CL = g.ldc, CR = 3 * g.ldc;
  const long long grow = ((long long)t * (nj + 2) + j + 1) * P + 1 + lane;   // element of (t, j, lane)
  const bool er = (j == 0) | (j == nj - 1);
  PushTab ptab;
  ptab.twe = reinterpret_cast<const int4*>(sb + L.twe);
  ptab.ts = reinterpret_cast<const int2*>(sb + L.ts);
  ptab.tn = reinterpret_cast<const int2*>(sb + L.tn);
  ptab.ni = ni;
  ptab.nj = nj;
  ptab.lim = (unsigned)tp.T * (unsigned)(nj + 2) * (unsigned)P;
  ptab.gs = kp.gs;
  const float* cw = reinterpret_cast<const float*>(sb + L.coef) + w * CR + lane;
  const float* cs = cw + CL;
  const float* cn = cs + CR;
  const float* cc = cw + 2 * CL;
  const int off_c = (w + 1) * P + 1 + lane;
  // rows w, w - 1, w + 1 of the two staged vectors at this lane's column
  const float2* A = reinterpret_cast<const float2*>(sb + L.vec[0][0]) + off_c;   // z (S), r (X, Z)
  const float2* B = reinterpret_cast<const float2*>(sb + L.vec[0][1]) + off_c;   // s_{k-1} (S), q_k (X)
  const float2 *As = A - P, *An = A + P, *Bs = B - P, *Bn = B + P;
  const double2* XO = reinterpret_cast<const double2*>(sb + L.xo[0]) + w * P + 1 + lane;
  const float2 coef = make_float2((float)si.c1(0), (float)si.c1(1));   // beta_k (S), alpha_k (X)
  const double ap0 = si.c2(0), ap1 = si.c2(1);                          // S: alpha_{k-1}
  const bool up0 = si.has_alpha(0) != 0, up1 = si.has_alpha(1) != 0;
  float2 *o1, *o2;   // S: s_k, q_k; X: r_{k+1}, z_{k+1}; Z: z (o2)
  double2* ox = nullptr;
  if (pt == P_S) {
    o1 = reinterpret_cast<float2*>(vec_ptr<float>(g, c.inst, 0, (k & 1) ? V_S1 : V_S0));
    o2 = reinterpret_cast<float2*>(vec_ptr<float>(g, c.inst, 0, V_Q));
    ox = reinterpret_cast<double2*>(vec_ptr<double>(g, c.inst, 0, V_X));
  } else {
    o1 = reinterpret_cast<float2*>(vec_ptr<float>(g, c.inst, 0, ((k + 1) & 1) ? V_R1 : V_R0));
    o2 = reinterpret_cast<float2*>(vec_ptr<float>(g, c.inst, 0, V_Z));
  }
  // this lane's column of the row in the output vectors (the ring pushes take the vectors' bases)
  float2* const r1 = o1 + grow;
  float2* const r2 = o2 + grow;
  double2* const rx = pt == P_S ? ox + grow : nullptr;
  double a00 = 0.0, a01 = 0.0, a10 = 0.0, a11 = 0.0;   // sums (slot, kind)
  const bool whole = MAXM > 0 && ni > 32 * (MAXM - 1);

  // one column step: o the lane's column offset from m = 0; valid: the column lies in the row; push: a tile-edge
  // point (every point of the tile's first and last row, the row's first and last point)
  auto col = [&](auto pt_tag, int m, int o, bool valid, bool push) {
    constexpr int PT = decltype(pt_tag)::value;
    const int i = lane + 32 * m;
    if constexpr (PT == P_S) {
      // s_k = z_k + beta_k s_{k-1} (cg2d.py:249) at the point and its neighbours; q_k = A s_k (cg2d.py:251);
      // x_k = x_{k-1} + alpha_{k-1} s_{k-1} (cg2d.py:254); s_k.q_k (cg2d.py:252)
      const float2 sp = B[o];
      const float2 vc = fma2(coef, sp, A[o]);
      const float2 vw = fma2(coef, B[o - 1], A[o - 1]);
      const float2 ve = fma2(coef, B[o + 1], A[o + 1]);
      const float2 vs = fma2(coef, Bs[o], As[o]);
      const float2 vn = fma2(coef, Bn[o], An[o]);
      const float2 qv = stencil5p(cw[o], cw[o + 1], cs[o], cn[o], cc[o], vw, ve, vs, vn, vc);
      const double2 xo = XO[o];
      double2 xn;
      xn.x = up0 ? __fma_rn(ap0, (double)sp.x, xo.x) : xo.x;
      xn.y = up1 ? __fma_rn(ap1, (double)sp.y, xo.y) : xo.y;
      if (valid) {
        stcg2(r1 + o, vc);
        stcg2(r2 + o, qv);
        stcg2(rx + o, xn);
        a00 = __fma_rn((double)vc.x, (double)qv.x, a00);
        a10 = __fma_rn((double)vc.y, (double)qv.y, a10);
      }
      if (push) {
        push_pair(ptab, o1, j, w, i, vc);
        push_pair(ptab, o2, j, w, i, qv);
        push_pair(ptab, ox, j, w, i, xn);   // x's neighbours: read by the replacement pass only
      }
    } else {
      // X: r_{k+1} = r_k - alpha_k q_k (cg2d.py:255) at the point and its neighbours; z_{k+1} = M r_{k+1}
      //    (cg2d.py:245); r.r and z.r (cg2d.py:256, 246).  Z: z = M r and z.r
      float2 vc, vw, ve, vs, vn;
      if constexpr (PT == P_X) {
        const float2 na = make_float2(-coef.x, -coef.y);
        vc = fma2(na, B[o], A[o]);
        vw = fma2(na, B[o - 1], A[o - 1]);
        ve = fma2(na, B[o + 1], A[o + 1]);
        vs = fma2(na, Bs[o], As[o]);
        vn = fma2(na, Bn[o], An[o]);
      } else {
        vc = A[o]; vw = A[o - 1]; ve = A[o + 1]; vs = As[o]; vn = An[o];
      }
      const float2 z = stencil5p(cc[o], cw[o], cw[o + 1], cs[o], cn[o], vc, vw, ve, vs, vn);
      if (valid) {
        if constexpr (PT == P_X) stcg2(r1 + o, vc);
        stcg2(r2 + o, z);
        if constexpr (PT == P_X) {
          a00 = __fma_rn((double)vc.x, (double)vc.x, a00);
          a01 = __fma_rn((double)z.x, (double)vc.x, a01);
          a10 = __fma_rn((double)vc.y, (double)vc.y, a10);
          a11 = __fma_rn((double)z.y, (double)vc.y, a11);
        } else {
          a00 = __fma_rn((double)z.x, (double)vc.x, a00);
          a10 = __fma_rn((double)z.y, (double)vc.y, a10);
        }
      }
      if (push) {
        if constexpr (PT == P_X) push_pair(ptab, o1, j, w, i, vc);
        push_pair(ptab, o2, j, w, i, z);
      }
    }
  };
  // the row: whole steps with immediate offsets and no tests; the last (or every) step partial: a lane past the
  // row reads its last column again and stores and sums nothing
  auto row = [&](auto pt_tag, auto edge_tag, auto mf_tag) {
    constexpr bool EDGE = decltype(edge_tag)::value;
    constexpr int MF = decltype(mf_tag)::value;
    auto part = [&](int m) {
      const int i = lane + 32 * m;
      const bool valid = i < ni;
      col(pt_tag, m, min(i, ni - 1) - lane, valid, EDGE ? valid : ((i == 0) | (i == ni - 1)));
    };
    if constexpr (MF >= 0) {
#pragma unroll
      for (int m = 0; m < MF; ++m) {
        const int i = lane + 32 * m;
        col(pt_tag, m, 32 * m, true, EDGE || (i == 0) || (i == ni - 1));
      }
#pragma unroll
      for (int m = MF; m < (MAXM > 0 ? MAXM : 1); ++m)
        if (32 * m < ni) part(m);
    } else {
      for (int m = 0; 32 * m < ni; ++m) part(m);
    }
  };
  auto by_edge = [&](auto pt_tag) {
    using F = std::integral_constant<int, (MAXM > 0 ? MAXM - 1 : 0)>;
    using G = std::integral_constant<int, -1>;
    if (er) row(pt_tag, std::true_type{}, G{});
    else if (whole) row(pt_tag, std::false_type{}, F{});
    else row(pt_tag, std::false_type{}, G{});
  };
  if (pt == P_S) by_edge(std::integral_constant<int, P_S>{});
  else if (pt == P_X) by_edge(std::integral_constant<int, P_X>{});
  else by_edge(std::integral_constant<int, P_Z>{});
  lp.v[0] = a00; lp.v[1] = a01; lp.v[2] = a10; lp.v[3] = a11;
  return lp;
}

template <bool MIXED, int MAXM, bool ONE, bool SERIAL, bool WIDE>
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
      const int es = vstride(g);
      for (int i = lane; i < ni; i += 32) {
        double xv = ldcg(x + (grow + i) * es);
        if (si.has_alpha(s)) xv = A::madd(si.c2(s), (double)ldcg(so + (grow + i) * es), xv);
        const double xf = __ddiv_rn(xv, si.rnorm(s));
        g.x_out[s][prow + i] = xf;
        if (g.x_fortran[s]) g.x_fortran[s][prow + i] = xf;
      }
    }
  }
  const bool on0 = act0 == A_ACTIVE, on1 = act1 == A_ACTIVE;
  if (!on0 && !on1) return lp;
  if constexpr (MIXED && !SERIAL && ONE) {
    if (g.pair && pt != P_R) return compute_pair<MAXM, ONE>(kp, c, pt, k, si, st, sm);
  }

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

  // NS right-hand sides q[0..NS-1] in pass PT (S, X or Z); sums into acc[s][kind]. A separate loop body per pass
  // kind, right-hand-side count and edge mode, so that the column loop tests none of them:
  //   EDGE   the tile's first or last row: every point pushes its new values to the rings of the tiles that read it;
  //   else   only the row's first and last points push (one test per column step, not per right-hand side).
  // Column steps m < MF are whole (every lane's column lies in the row: offsets are immediates and nothing is
  // tested); the steps from MF on are partial: a lane past the row's end reads the row's last column again (in
  // bounds) and stores and sums nothing. MF < 0: every step is partial (any width).
  auto run = [&](auto ns_tag, auto pt_tag, auto edge_tag, auto mf_tag, const RowSet<V>* q, double (&acc)[2][2]) {
    constexpr int NS = decltype(ns_tag)::value;
    constexpr int PT = decltype(pt_tag)::value;
    constexpr bool EDGE = decltype(edge_tag)::value;
    constexpr int MF = decltype(mf_tag)::value;
    auto col = [&](int m, int o, bool valid) {
      const int i = lane + 32 * m;
      const bool push = EDGE ? valid : ((i == 0) | (i == ni - 1));
      V v1[NS], v2[NS];      // S: s_k, q_k; X: r_{k+1}, z_{k+1}; Z: z (v2)
      double xn[NS];         // S: x_k
      if constexpr (PT == P_S) {
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
          // the x update is due once alpha_{k-1} exists; before it x is stored back unchanged
          const double xo = r.xo[o];
          const double x1 = r.upd ? A::madd(r.alpha_prev, (double)sp, xo) : xo;
          if (valid) {
            stcg(r.o1 + o, vc);
            stcg(r.o2 + o, qv);
            stcg(r.ox + o, x1);
            if constexpr (!MIXED) {
              if (r.ck) r.ck[o] = (double)vc;                                    // checkpoint s_k
            }
            if constexpr (SERIAL) r.pr[o] = mul((double)vc, (double)qv);
            else acc[s][0] = A::dot((double)vc, (double)qv, acc[s][0]);
          }
          v1[s] = vc;
          v2[s] = qv;
          xn[s] = x1;
        }
      } else {
        // X: r_{k+1} = r_k - alpha_k q_k (cg2d.py:255) at the point and its neighbours; z_{k+1} = M r_{k+1}
        //    (cg2d.py:245); r.r and z.r (cg2d.py:256, 246).  Z: z = M r and z.r
        const C pw = cw[o], pe_ = cw[o + 1], ps = cs[o], pn = cn[o], pc = cc[o];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const RowSet<V>& r = q[s];
          V vc, vw, ve, vs, vn;
          if constexpr (PT == P_X) {
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
          if (valid) {
            if constexpr (PT == P_X) stcg(r.o1 + o, vc);
            if constexpr (!MIXED) {
              if (r.ck) r.ck[o] = (double)vc;                                    // checkpoint r_{k+1}
            }
            stcg(r.o2 + o, z);
            if constexpr (SERIAL) {
              if constexpr (PT == P_X) {
                r.pr[o] = mul((double)vc, (double)vc);
                r.pr[o + kWarps * kp.max_ni] = mul((double)z, (double)vc);
              } else {
                r.pr[o] = mul((double)z, (double)vc);
              }
            } else if constexpr (PT == P_X) {
              acc[s][0] = A::dot((double)vc, (double)vc, acc[s][0]);
              acc[s][1] = A::dot((double)z, (double)vc, acc[s][1]);
            } else {
              acc[s][0] = A::dot((double)z, (double)vc, acc[s][0]);
            }
          }
          v1[s] = vc;
          v2[s] = z;
          xn[s] = 0.0;
        }
      }
      // ring pushes of the tile-edge points
      if (push) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const RowSet<V>& r = q[s];
          if constexpr (PT != P_Z) push_s(ptab, r.vs1, j, w, i, v1[s]);
          push_s(ptab, r.vs2, j, w, i, v2[s]);
          if constexpr (MIXED && PT == P_S) push_s(ptab, r.vsx, j, w, i, xn[s]);   // read by the R pass only
        }
      }
    };
    // a partial step: lanes past the row read its last column (offset relative to the lane's column at m = 0)
    auto part = [&](int m) {
      const int i = lane + 32 * m;
      col(m, min(i, ni - 1) - lane, i < ni);
    };
    if constexpr (MF >= 0) {
#pragma unroll
      for (int m = 0; m < MF; ++m) col(m, 32 * m, true);
#pragma unroll
      for (int m = MF; m < (MAXM > 0 ? MAXM : 1); ++m)
        if (32 * m < ni) part(m);
    } else {
      for (int m = 0; 32 * m < ni; ++m) part(m);
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
      const int es = vstride(g);   // paired: element e of this solve at scalar 2 e (staged and in the workspace)
      double* pr = SERIAL ? sm.prod() + ((s * 2) * kWarps + w) * kp.max_ni : nullptr;
      auto x1 = [&](double xx, V ss) -> double { return A::madd(alpha, (double)ss, xx); };
      for (int i = lane; i < ni; i += 32) {
        const int rc = (w + 1) * P + i + 1;
        auto X1 = [&](int e) -> double { return x1(xr[e * es], sk[e * es]); };
        const double vc = X1(rc);
        const double vw = X1(rc - 1);
        const double ve = X1(rc + 1);
        const double vs = X1(rc - P);
        const double vn = X1(rc + P);
        const int cr = w * NP + col0 + i;
        const double bn = mul(mul(__ldg(g.b[s] + prow + i), si.norm(s)), si.rnorm(s));
        const V r = (V)sub(bn, op_A<double>(aw[cr], aw[cr + 1], as[cr], as[cr + NP], ac[cr], vw, ve, vs, vn, vc));
        stcg(r_out + (grow + i) * es, r);
        if (er | (i == 0) | (i == ni - 1)) push_s(ptab, r_out, j, w, i, r, es);
        if constexpr (SERIAL) pr[i] = mul((double)r, (double)r);
        else if (s == 0) lp.v[0] = A::dot((double)r, (double)r, lp.v[0]);
        else lp.v[2] = A::dot((double)r, (double)r, lp.v[2]);
      }
    }
    return lp;
  }

  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  // whole column steps: all but the last when the row is longer than MAXM - 1 steps (then every lane's column of
  // those steps lies in the row), none otherwise (a group narrower than the build's width, or any width). WIDE
  // builds compile the unrolled whole-step loop; the FP64 build for two CTAs per SM does not (its 96 registers a
  // thread would spill it), and takes the step loop for every row.
  const bool whole = WIDE && MAXM > 0 && ni > 32 * (MAXM - 1);
  auto pass_e = [&](auto ns_tag, auto pt_tag, const RowSet<V>* q) {
    using F = std::integral_constant<int, (MAXM > 0 ? MAXM - 1 : 0)>;
    using G = std::integral_constant<int, -1>;
    if (er) {
      run(ns_tag, pt_tag, std::true_type{}, G{}, q, acc);
    } else if constexpr (WIDE) {
      if (whole) run(ns_tag, pt_tag, std::false_type{}, F{}, q, acc);
      else run(ns_tag, pt_tag, std::false_type{}, G{}, q, acc);
    } else {
      run(ns_tag, pt_tag, std::false_type{}, G{}, q, acc);
    }
  };
  auto pass = [&](auto ns_tag, const RowSet<V>* q) {
    if (pt == P_S) pass_e(ns_tag, std::integral_constant<int, P_S>{}, q);
    else if (pt == P_X) pass_e(ns_tag, std::integral_constant<int, P_X>{}, q);
    else pass_e(ns_tag, std::integral_constant<int, P_Z>{}, q);
  };
  if (on0 && on1) {
    const RowSet<V> q[2] = {rows(0), rows(1)};
    pass(std::integral_constant<int, 2>{}, q);
    lp.v[0] = acc[0][0]; lp.v[1] = acc[0][1]; lp.v[2] = acc[1][0]; lp.v[3] = acc[1][1];
  } else {
    const int s = on0 ? 0 : 1;
    const RowSet<V> q[1] = {rows(s)};
    pass(std::integral_constant<int, 1>{}, q);
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

template <bool MIXED, int MAXM, bool ONE, bool SERIAL, bool WIDE>
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
    const Lanes lp = compute_chunk<MIXED, MAXM, ONE, SERIAL, WIDE>(kp, c, pt, k, si, st, sm);
    if (!SERIAL && warp < c.nr) row_sums(g, lp, sm, st, pt == P_X);
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty()[st]);
    PROF_ADD(kp, sm, PR_COMP, t0);
    st = (st + 1 == ns) ? 0 : st + 1;
    have = cursor_next(kp, sm, cur);
  }
  return true;
}

template <bool MIXED, int MAXM, bool ONE, bool SERIAL, bool WIDE>
__device__ bool run_pass_pipe(const KParams& kp, int pt, int k, int hidx, const Smem& sm, Pipe& pp) {
  bool ok;
  if ((int)(threadIdx.x >> 5) == kp.nw) ok = produce_pass(kp, pt, k, hidx, sm, pp);
  else ok = consume_pass<MIXED, MAXM, ONE, SERIAL, WIDE>(kp, pt, k, sm, pp);
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

template <bool MIXED, int MAXM, bool ONE, int CPS, bool SERIAL, int NT>
__global__ void __launch_bounds__(NT, CPS) cg2d_persistent(const __grid_constant__ KParams kp) {
  const Smem sm = carve(kp.max_ni, kp.serial);
  const int tid = threadIdx.x;
  unsigned target = (unsigned)kp.test_missing;
  Pipe pp = {0u, 0u, 0u, 0u};
  const unsigned long long t_start = PROF_T0(kp);
  if (tid < kProfSlots) sm.pacc()[tid] = 0ull;
  if (tid == 0) {
    for (int s = 0; s < kMaxStages; ++s) {
      mbar_init(&sm.full()[s], 1);          // the producer's arrive (with the copies' byte count)
      mbar_init(&sm.empty()[s], kp.nw);     // one arrive per compute warp
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
  ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL, (MIXED || CPS == 1)>(kp, P_Z, 0, 0, sm, pp);
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
    ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL, (MIXED || CPS == 1)>(kp, P_S, k, k, sm, pp);
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
      ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL, (MIXED || CPS == 1)>(kp, P_X, k, k + 1, sm, pp);
      ok = grid_sync(kp, target, P_X, k + 1, sm) && ok;
      if (!ok) goto epilogue;
      if (ax == A_ACTIVE) {
        S->rr = __ldcg(hist_ptr(kp, tid, H_RRX, k + 1));
        S->eta = __ldcg(hist_ptr(kp, tid, H_ETAX, k + 1));
      }
    }
    if (__syncthreads_or(ar != A_NONE)) {
      set_actions(kp, sm, ar, own ? S->alpha : 0.0, 0.0);
      ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL, (MIXED || CPS == 1)>(kp, P_R, k, k + 1, sm, pp);
      ok = grid_sync(kp, target, P_R, k + 1, sm) && ok;
      if (!ok) goto epilogue;
      if (ar == A_ACTIVE) {
        S->rr = __ldcg(hist_ptr(kp, tid, H_RRR, k + 1));
        ++S->nrep;
      }
      set_actions(kp, sm, ar, 0.0, 0.0);
      ok = run_pass_pipe<MIXED, MAXM, ONE, SERIAL, (MIXED || CPS == 1)>(kp, P_Z, k, k + 1, sm, pp);
      ok = grid_sync(kp, target, P_Z, k + 1, sm) && ok;
      if (!ok) goto epilogue;
      if (ar == A_ACTIVE) S->eta = __ldcg(hist_ptr(kp, tid, H_ETAZ, k + 1));
    }
  }

epilogue:
  // ---- halo points of the outputs: x_out 0; x_fortran = exchanged normalised first guess, unwritten
  //      points keep cg2d_x (cg2d.py:208-210, 227-228)
  {
    const long long gstride = (long long)gridDim.x * blockDim.x;
    for (int gg = 0; gg < kp.ngroups; ++gg) {
      const GroupDev& g = kp.g[gg];
      const TopoDev& tp = g.tp;
      const long long per = g.pad_elems;
      const long long tot = per * g.count * g.nrhs;
      for (long long idx = (long long)blockIdx.x * blockDim.x + tid; idx < tot; idx += gstride) {
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
// built for; mixed precision has the 16-warp build (15 compute warps, one CTA per SM) for single-group launches whose
// 15-row chunks fit, and the 9-warp build (two CTAs per SM) otherwise
template <bool ONE, int CPS>
static const void* solver_fn_of(int mixed, int nw, int max_ni) {
  if (mixed) {
    if (ONE && nw == kMixedWarps) {
      if (max_ni <= 96) return (const void*)cg2d_persistent<true, 3, true, 1, false, kMixedThreads>;
      return (const void*)cg2d_persistent<true, 0, true, 1, false, kMixedThreads>;
    }
    if (max_ni <= 96) return (const void*)cg2d_persistent<true, 3, ONE, 2, false, kThreads>;
    if (max_ni <= 288) return (const void*)cg2d_persistent<true, 9, ONE, 2, false, kThreads>;
    return (const void*)cg2d_persistent<true, 0, ONE, 2, false, kThreads>;
  }
  if (max_ni <= 96) return (const void*)cg2d_persistent<false, 3, ONE, CPS, false, kThreads>;
  if (max_ni <= 288) return (const void*)cg2d_persistent<false, 9, ONE, CPS, false, kThreads>;
  return (const void*)cg2d_persistent<false, 0, ONE, CPS, false, kThreads>;
}
static const void* solver_fn(const KParams& kp) {
  // the FORTRAN sum order (bitwise parity, not speed): one generic build per precision
  if (kp.serial) return kp.mixed ? (const void*)cg2d_persistent<true, 0, false, 2, true, kThreads>
                                 : (const void*)cg2d_persistent<false, 0, false, 1, true, kThreads>;
  const bool two = !kp.mixed && kp.fp64_cps == 2;
  if (kp.ngroups == 1)
    return two ? solver_fn_of<true, 2>(kp.mixed, kp.nw, kp.max_ni) : solver_fn_of<true, 1>(kp.mixed, kp.nw, kp.max_ni);
  return two ? solver_fn_of<false, 2>(kp.mixed, kp.nw, kp.max_ni) : solver_fn_of<false, 1>(kp.mixed, kp.nw, kp.max_ni);
}

int solver_threads(const KParams& kp) { return (kp.nw + 1) * 32; }

cudaError_t solver_occupancy(const KParams& kp, size_t smem, int* blocks_per_sm) {
  const void* fn = solver_fn(kp);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, solver_threads(kp), smem);
}

cudaError_t launch_solver(const KParams& kp, int grid, size_t smem, cudaStream_t stream) {
  const void* fn = solver_fn(kp);
  void* args[] = {const_cast<KParams*>(&kp)};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(solver_threads(kp)), args, smem, stream);
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
