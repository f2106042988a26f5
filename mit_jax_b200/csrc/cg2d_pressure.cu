// The steps either side of the CG2D solve in SOLVE_FOR_PRESSURE, on a batch of instances:
//   update_cg2d  (mitgcm_jax/core/solve_for_pressure.py:29-65): the operator aW2d, aS2d, aC2d from the level sums of
//                the face areas, its diagonal exchanged, and the preconditioner pW, pS, pC;
//   cg2d_rhs     (solve_for_pressure.py:68-106): the right-hand side (fresh-water flux, the divergence of the g-hat
//                transports summed from level Nr up to 1, the exactConserv etaH term) and the first guess;
//   post-solve   (solve_for_pressure.py:116-121): the exchange of the solution and etaN = recip_Bo x;
// and, once at set-up, ini_cg2d_norm (mitgcm_jax/core/cg2d.py:108-134): cg2dNorm from the initial face fractions.
// Every operation is the reference's, in its order, without contraction (__dmul_rn / __dadd_rn / __ddiv_rn), so
// results are bit for bit those of the reference. The vertical factors deepFacC, rhoFacC, deepFac2F are all 1 in
// the reference (free_surface.py:121-125); the products with them are exact and are left out.
//
// Layout: 3-D fields [batch][T][Nr][ny][nx], 2-D per-instance fields [batch][T][ny][nx], grid fields [T][ny][nx]
// shared by the batch (padded, the reference layout). One thread per padded point of an instance (blockIdx.y);
// the level loops stream Nr planes with coalesced rows. All are HBM-bound.

#include <cuda_runtime.h>

#include <cmath>

#include "cg2d_internal.cuh"

namespace cg2d {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

struct Pt {
  int t, j, i;   // tile; interior coordinates (Fortran index - 1): -OLy <= j < nj + OLy, -OLx <= i < ni + OLx
};
__device__ __forceinline__ Pt decode(const TopoDev& tp, int q) {
  const int plane = tp.npy * tp.npx;
  Pt p;
  p.t = q / plane;
  const int rem = q - p.t * plane;
  const int jp = rem / tp.npx;
  p.j = jp - tp.OLy;
  p.i = rem - jp * tp.npx - tp.OLx;
  return p;
}
__device__ __forceinline__ bool interior(const TopoDev& tp, const Pt& p) {
  return p.j >= 0 && p.j < tp.nj && p.i >= 0 && p.i < tp.ni;
}

#define FOR_Q(tp)                                                                          \
  const int pe_ = (tp).T * (tp).npy * (tp).npx;                                            \
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < pe_; q += gridDim.x * blockDim.x)

// Asynchronous 8-byte copies global -> shared (cp.async), counted per thread in commit groups: the level loops
// below stream their per-level fields a few levels ahead of use through shared memory, each thread copying and
// later reading only its own slots (so the copies need no block barrier).
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// aW2d, aS2d on j, i = 1..sNy+1, 1..sNx+1 (0 elsewhere): sum over k = 1..Nr in order of
// ((dyG drF(k)) hFacW(k)) recip_dxC, then times cg2dNorm, implicSurfPress, implicDiv2DFlow (:41-47). One thread per
// padded point (blockIdx.x blocks of kUfThreads cover an instance, blockIdx.y = instance); hFacW and hFacS stream
// kUfStages levels ahead of the ordered sums.
constexpr int kUfThreads = 256, kUfStages = 8;
constexpr size_t kUfSmem = sizeof(double) * kUfStages * 2 * kUfThreads;
__global__ void __launch_bounds__(kUfThreads) k_update_faces(TopoDev tp, int Nr, const double* hFacW,
                                                             const double* hFacS, const double* drF, const double* dyG,
                                                             const double* dxG, const double* rdxC, const double* rdyC,
                                                             double norm, const double* norm_arr, double isp,
                                                             double idf, double* aW2d, double* aS2d) {
  extern __shared__ double stage[];   // [kUfStages][2][kUfThreads]: hFacW, hFacS
  const int in = blockIdx.y;
  const int plane = tp.npy * tp.npx;
  const int q = blockIdx.x * kUfThreads + threadIdx.x;
  if (q >= tp.T * plane) return;
  const long long o2 = (long long)in * tp.T * plane;
  const Pt p = decode(tp, q);
  const bool face = p.j >= 0 && p.j <= tp.nj && p.i >= 0 && p.i <= tp.ni;
  double w = 0.0, s = 0.0;
  if (face) {
    const long long b3 = ((long long)in * tp.T + p.t) * Nr * plane + (q - p.t * plane);
    const double* hw = hFacW + b3;
    const double* hs = hFacS + b3;
    auto slot = [&](int k, int f) { return stage + ((k % kUfStages) * 2 + f) * kUfThreads + threadIdx.x; };
    auto issue = [&](int k) {   // level k into its stage (one commit group, maybe empty)
      if (k < Nr) {
        cp_async8(slot(k, 0), hw + (long long)k * plane);
        cp_async8(slot(k, 1), hs + (long long)k * plane);
      }
      cp_async_commit();
    };
    for (int k = 0; k < kUfStages; ++k) issue(k);
    const double dy = dyG[q], dx = dxG[q], rx = rdxC[q], ry = rdyC[q];
    for (int k = 0; k < Nr; ++k) {
      cp_async_wait<kUfStages - 1>();   // level k's group (the oldest pending) has landed
      const double d = __ldg(drF + k);
      const double hwk = *slot(k, 0), hsk = *slot(k, 1);
      issue(k + kUfStages);             // into the stage just read
      w = add(w, mul(mul(mul(dy, d), hwk), rx));
      s = add(s, mul(mul(mul(dx, d), hsk), ry));
    }
    const double nrm = norm_arr ? norm_arr[in] : norm;
    w = mul(mul(mul(w, nrm), isp), idf);
    s = mul(mul(mul(s, nrm), isp), idf);
  }
  aW2d[o2 + q] = w;
  aS2d[o2 + q] = s;
}

struct DiagArgs {
  const double *aW2d, *aS2d, *recip_Bo, *rA;
  double fn;      // freeSurfFac cg2dNorm (per instance when norm_arr is given)
  const double* norm_arr;
  double fsf, dTm, dTfs;
};

// aC2d at padded point q of instance in, as the exchange leaves it (:49-53): at an interior point
// -(aW2d + aW2d(i+1) + aS2d + aS2d(j+1) + freeSurfFac cg2dNorm recip_Bo rA / deltaTMom / deltaTFreeSurf); at a halo
// point the value at its exch2 source, or 0 where the map writes nothing
__device__ double aC_at(const TopoDev& tp, const DiagArgs& A, int in, int q) {
  Pt p = decode(tp, q);
  if (!interior(tp, p)) {
    if (tp.map_comp[q] != 1) return 0.0;
    q = tp.map_src[q];
    p = decode(tp, q);
    if (!interior(tp, p)) return 0.0;
  }
  const long long o = (long long)in * tp.T * tp.npy * tp.npx;
  const double f = A.norm_arr ? mul(A.fsf, A.norm_arr[in]) : A.fn;
  const double sum = add(add(add(A.aW2d[o + q], A.aW2d[o + q + 1]), A.aS2d[o + q]), A.aS2d[o + q + tp.npx]);
  const double ex = dvd(dvd(mul(mul(f, A.recip_Bo[q]), A.rA[q]), A.dTm), A.dTfs);
  return -add(sum, ex);
}

// aC2d on every padded point; pW, pS, pC on j, i = 1..sNy+1, 1..sNx+1 (:55-65): pC = 1/a (1 where a = 0),
// pW = -aW2d / (cg2dpcOffDFac (a + aC2d(i-1)))^2 (0 where the sum is 0), pS likewise with aC2d(j-1)
__global__ void k_update_diag(TopoDev tp, DiagArgs A, double offd, double* aC2d, double* pW, double* pS,
                              double* pC) {
  const int in = blockIdx.y;
  const long long o = (long long)in * tp.T * tp.npy * tp.npx;
  FOR_Q(tp) {
    const Pt p = decode(tp, q);
    const double a = aC_at(tp, A, in, q);
    aC2d[o + q] = a;
    if (p.j >= 0 && p.j <= tp.nj && p.i >= 0 && p.i <= tp.ni) {
      pC[o + q] = a == 0.0 ? 1.0 : dvd(1.0, a);
      const double tw = add(a, aC_at(tp, A, in, q - 1));
      const double ts = add(a, aC_at(tp, A, in, q - tp.npx));
      const double cw = mul(offd, tw), cs = mul(offd, ts);
      pW[o + q] = tw == 0.0 ? 0.0 : dvd(-A.aW2d[o + q], mul(cw, cw));
      pS[o + q] = ts == 0.0 ? 0.0 : dvd(-A.aS2d[o + q], mul(cs, cs));
    }
  }
}

struct RhsArgs {
  const double *gU, *gV, *hFacW, *hFacS, *EmPmR, *etaN, *etaH;   // per instance
  const double *drF, *dyG, *dxG, *rA, *maskInC, *Bo_surf;         // shared
  double tmpFac, fsf, dTm, dTfs;
  double rdTm;   // RN(1 / deltaTMom) for div_fixed, or 0 (deltaTMom outside [2^-64, 2^64]: plain divisions)
  int fresh_water, Nr;
};

// a / b correctly rounded (the IEEE quotient, bit for bit) for a divisor b fixed over the launch, given y = RN(1/b):
// q = RN(a y) is within an ulp of a / b, the remainder r = a - q b is exact by FMA, and RN(q + r y) is RN(a / b)
// when y is within half an ulp of 1 / b (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34 (1990) 111-119; J.-M. Muller et al., Handbook of Floating-Point
// Arithmetic, the division section). Intermediates stay normal for 2^-900 <= |a| <= 2^900 and 2^-64 <= |b| <= 2^64;
// zero returns the exact signed zero a y, anything else (tiny, huge, inf, NaN, y = 0) takes the division itself.
// One multiply and two FMAs in place of a division: the level loop of k_rhs does two per face and level.
__device__ __forceinline__ double div_fixed(double a, double b, double y) {
  if (a == 0.0) return mul(a, y);
  const double m = fabs(a);
  if (!(m >= 0x1p-900 && m <= 0x1p900) || y == 0.0) return dvd(a, b);
  const double q = mul(a, y);
  return __fma_rn(__fma_rn(-q, b, a), y, q);
}

// cg2d_x = Bo_surf etaN everywhere (:76); cg2d_b = 0 on halos (the interior is k_rhs's)
__global__ void k_rhs_fill(TopoDev tp, const double* Bo_surf, const double* etaN, double* cg2d_b, double* cg2d_x) {
  const int in = blockIdx.y;
  const long long o = (long long)in * tp.T * tp.npy * tp.npx;
  FOR_Q(tp) {
    cg2d_x[o + q] = mul(Bo_surf[q], etaN[o + q]);
    if (!interior(tp, decode(tp, q))) cg2d_b[o + q] = 0.0;
  }
}

// cg2d_b on the interior (:77-106): the fresh-water term, then for k = Nr..1 in order (:95-101)
//   b = (b + pu(i+1)) - pu(i),  b = (b + pv(j+1)) - pv(j),
// pu(i) = ((dyG(i) drF(k)) hFacW(i, k)) gU(i, k) / deltaTMom the transport through the west face of point i (:90, :92),
// pv(j) likewise through the south face; then the etaH term (:103-105). A face is shared by the two points on either
// side: each thread forms the terms of its own west and south faces once per level, and takes its east and north
// face's terms from the threads that own those faces (the next lane by shuffle, the next row through shared memory).
// A block of 32 lanes x kRhsRows rows owns 31 columns x (kRhsRows - 1) rows of points; its last lane and last row
// only form faces (the east / north faces of the block's points; the next block owns their points). The terms are
// the same floating-point operations on the same operands whichever thread forms them, so the sums are the
// reference's bit for bit, with about 2.2 divisions per point and level instead of 4, each by deltaTMom and so
// formed by div_fixed.
constexpr int kRhsRows = 8;
constexpr int kRhsCols = 31, kRhsOwnRows = kRhsRows - 1;   // points a block owns
// The four face fields of a level stream through shared memory kRhsStages levels ahead of their use: each thread
// copies its own four values with asynchronous 8-byte copies (cp.async, one commit group per level) and reads back
// only what it copied, so the copies need no block barrier; the level chain itself (ordered sums, one barrier per
// level) then never waits on a load issued less than kRhsStages levels earlier.
constexpr int kRhsStages = 5;
constexpr size_t kRhsSmem = sizeof(double) * kRhsStages * 4 * kRhsRows * 32;

__global__ void __launch_bounds__(32 * kRhsRows, 4) k_rhs(TopoDev tp, RhsArgs A, double* cg2d_b) {
  __shared__ double pvs[2][2][kRhsRows][32];   // [pair buffer][level of the pair][row][lane]
  extern __shared__ double stage[];   // [kRhsStages][4][kRhsRows][32]: hFacW, gU, hFacS, gV
  const int in = blockIdx.z;
  const int nrb = (tp.nj + kRhsOwnRows - 1) / kRhsOwnRows;   // row blocks per tile
  const int t = blockIdx.y / nrb, jb = blockIdx.y - t * nrb;
  const int lane = threadIdx.x, y = threadIdx.y;
  const int i = blockIdx.x * kRhsCols + lane, j = jb * kRhsOwnRows + y;
  const bool face = i <= tp.ni && j <= tp.nj;             // forms the terms of its west / south face
  const bool own = lane < kRhsCols && y < kRhsOwnRows && i < tp.ni && j < tp.nj;   // sums cg2d_b
  const int plane = tp.npy * tp.npx;
  const int q = t * plane + (j + tp.OLy) * tp.npx + i + tp.OLx;   // padded point (in bounds when face)
  const long long o = (long long)in * tp.T * plane;
  const long long b3 = ((long long)in * tp.T + t) * A.Nr * plane + (q - t * plane);
  const double dTm = A.dTm, rdTm = A.rdTm;
  const double dyc = face ? A.dyG[q] : 0.0, dxc = face ? A.dxG[q] : 0.0;
  double b = 0.0;
  if (own && A.fresh_water) b = mul(dvd(mul(mul(A.tmpFac, A.rA[q]), A.EmPmR[o + q]), A.dTm), A.maskInC[q]);
  // this thread's slot of field f in stage s
  auto slot = [&](int s, int f) { return stage + ((s * 4 + f) * kRhsRows + y) * 32 + lane; };
  auto issue = [&](int k) {   // level k's four values into stage k % kRhsStages (one commit group, maybe empty)
    if (face && k >= 0) {
      const long long c = b3 + (long long)k * plane;
      const int s = k % kRhsStages;
      cp_async8(slot(s, 0), A.hFacW + c);
      cp_async8(slot(s, 1), A.gU + c);
      cp_async8(slot(s, 2), A.hFacS + c);
      cp_async8(slot(s, 3), A.gV + c);
    }
    cp_async_commit();
  };
  for (int s = 0; s < kRhsStages; ++s) issue(A.Nr - 1 - s);
  // level k's two face terms from its stage (waiting for its copies), then its stage refilled with level k - stages
  auto terms = [&](int k, double& pu, double& pv) {
    cp_async_wait<kRhsStages - 1>();   // level k's group (the oldest pending) has landed
    pu = 0.0;
    pv = 0.0;
    if (face) {
      const double d = __ldg(A.drF + k);
      const int s = k % kRhsStages;
      const double hw0 = *slot(s, 0), u0 = *slot(s, 1), hs0 = *slot(s, 2), v0 = *slot(s, 3);
      pu = div_fixed(mul(mul(mul(dyc, d), hw0), u0), dTm, rdTm);                             // :90, :92
      pv = div_fixed(mul(mul(mul(dxc, d), hs0), v0), dTm, rdTm);                             // :91, :93
    }
    issue(k - kRhsStages);   // into the stage just read (this thread's own slots, read above)
  };
  // two levels per block barrier: their south-face terms through shared memory (double-buffered by pair), their
  // west-face terms by shuffle, then the sums of both in order
  for (int k = A.Nr - 1, pair = 0; k >= 0; k -= 2, ++pair) {                  // :95-101, k = Nr..1
    double pua, pva, pub = 0.0, pvb = 0.0;
    terms(k, pua, pva);
    const bool two = k >= 1;
    if (two) terms(k - 1, pub, pvb);
    const int buf = pair & 1;
    pvs[buf][0][y][lane] = pva;
    pvs[buf][1][y][lane] = pvb;
    const double pua1 = __shfl_down_sync(0xffffffffu, pua, 1);
    const double pub1 = __shfl_down_sync(0xffffffffu, pub, 1);
    __syncthreads();
    if (own) {
      b = sub(add(b, pua1), pua);                                                             // :97, level k
      b = sub(add(b, pvs[buf][0][y + 1][lane]), pva);                                         // :98
      if (two) {
        b = sub(add(b, pub1), pub);                                                           // level k - 1
        b = sub(add(b, pvs[buf][1][y + 1][lane]), pvb);
      }
    }
  }
  if (own) {
    b = sub(b, mul(dvd(dvd(mul(A.fsf, A.rA[q]), A.dTm), A.dTfs), A.etaH[o + q]));            // :103-105
    cg2d_b[o + q] = b;
  }
}

// etaN = recip_Bo x with x the solution on the interior and, on halos, its exchanged value, or the first guess
// where the map writes nothing (:116-121)
__global__ void k_post(TopoDev tp, const double* x, const double* cg2d_x, const double* recip_Bo, double* etaN) {
  const int in = blockIdx.y;
  const long long o = (long long)in * tp.T * tp.npy * tp.npx;
  FOR_Q(tp) {
    const Pt p = decode(tp, q);
    double v;
    if (interior(tp, p)) {
      v = x[o + q];
    } else if (tp.map_comp[q] == 1) {
      const int s = tp.map_src[q];
      v = interior(tp, decode(tp, s)) ? x[o + s] : cg2d_x[o + s];
    } else {
      v = cg2d_x[o + q];
    }
    etaN[o + q] = mul(recip_Bo[q], v);
  }
}

// ini_cg2d_norm (mitgcm_jax/core/cg2d.py:108-134, ini_cg2d.F:90-135), first kernel: per instance, the maximum over
// the interior faces of |aW| and |aS|, aW = sum over k = 1..Nr in order of ((fac ((dyG drF(k)) hFacW(k))) recip_dxC),
// fac = implicSurfPress implicDiv2DFlow, aS likewise with dxG, hFacS, recip_dyC. The maximum is order-free; it is
// taken on the IEEE bits of the magnitudes (non-negative doubles order as their bits do) in bits[in], zeroed first.
__global__ void k_ini_norm_max(TopoDev tp, int Nr, const double* hFacW, const double* hFacS, const double* drF,
                               const double* dyG, const double* dxG, const double* rdxC, const double* rdyC,
                               double fac, unsigned long long* bits) {
  const int in = blockIdx.y;
  const int plane = tp.npy * tp.npx;
  unsigned long long m = 0ull;
  FOR_Q(tp) {
    const Pt p = decode(tp, q);
    if (interior(tp, p)) {
      const long long b3 = ((long long)in * tp.T + p.t) * Nr * plane + (q - p.t * plane);
      const double* __restrict__ hw = hFacW + b3;
      const double* __restrict__ hs = hFacS + b3;
      const double dy = dyG[q], dx = dxG[q], rx = rdxC[q], ry = rdyC[q];
      double w = 0.0, s = 0.0;
#pragma unroll 5
      for (int k = 0; k < Nr; ++k) {
        const double d = __ldg(drF + k);
        const double hwk = __ldg(hw + (long long)k * plane), hsk = __ldg(hs + (long long)k * plane);
        w = add(w, mul(mul(fac, mul(mul(dy, d), hwk)), rx));
        s = add(s, mul(mul(fac, mul(mul(dx, d), hsk)), ry));
      }
      const unsigned long long bw = (unsigned long long)__double_as_longlong(fabs(w));
      const unsigned long long bs = (unsigned long long)__double_as_longlong(fabs(s));
      m = bw > m ? bw : m;
      m = bs > m ? bs : m;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, m, o);
    m = y > m ? y : m;
  }
  if ((threadIdx.x & 31) == 0 && m != 0ull) atomicMax(bits + in, m);
}

// second kernel: cg2dNorm = 1 / myNorm, 1 where myNorm is 0 (cg2d.py:131-134), in place over the bits
__global__ void k_ini_norm_fin(int batch, unsigned long long* bits) {
  const int in = blockIdx.x * blockDim.x + threadIdx.x;
  if (in >= batch) return;
  const double my = __longlong_as_double((long long)bits[in]);
  reinterpret_cast<double*>(bits)[in] = my != 0.0 ? dvd(1.0, my) : 1.0;
}

dim3 grid_of(const TopoDev& tp, int batch) {
  const int pe = tp.T * tp.npy * tp.npx;
  return dim3((unsigned)((pe + 255) / 256), (unsigned)batch);
}

}  // namespace

cudaError_t pressure_update(const TopoDev& tp, const UpdateArgs& U, cudaStream_t st) {
  if (U.batch < 1 || U.batch > 65535 || U.Nr < 1) return cudaErrorInvalidValue;
  const dim3 g = grid_of(tp, U.batch);
  cudaError_t e = cudaFuncSetAttribute(k_update_faces, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUfSmem);
  if (e != cudaSuccess) return e;
  const dim3 gf((unsigned)((tp.T * tp.npy * tp.npx + kUfThreads - 1) / kUfThreads), (unsigned)U.batch);
  k_update_faces<<<gf, kUfThreads, kUfSmem, st>>>(tp, U.Nr, U.hFacW, U.hFacS, U.drF, U.dyG, U.dxG, U.recip_dxC,
                                                  U.recip_dyC, U.norm, U.norm_arr, U.implicSurfPress,
                                                  U.implicDiv2DFlow, U.aW2d, U.aS2d);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  DiagArgs D;
  D.aW2d = U.aW2d;
  D.aS2d = U.aS2d;
  D.recip_Bo = U.recip_Bo;
  D.rA = U.rA;
  D.fsf = U.freeSurfFac;
  D.norm_arr = U.norm_arr;
  D.fn = U.norm_arr ? 0.0 : U.freeSurfFac * U.norm;   // the scalar product the reference forms once (:51)
  D.dTm = U.deltaTMom;
  D.dTfs = U.deltaTFreeSurf;
  k_update_diag<<<g, 256, 0, st>>>(tp, D, U.offd, U.aC2d, U.pW, U.pS, U.pC);
  return cudaGetLastError();
}

cudaError_t pressure_rhs(const TopoDev& tp, const RhsIn& R, cudaStream_t st) {
  if (R.batch < 1 || R.batch > 65535 || R.Nr < 1) return cudaErrorInvalidValue;
  RhsArgs A;
  A.gU = R.gU; A.gV = R.gV; A.hFacW = R.hFacW; A.hFacS = R.hFacS;
  A.EmPmR = R.EmPmR; A.etaN = R.etaN; A.etaH = R.etaH;
  A.drF = R.drF; A.dyG = R.dyG; A.dxG = R.dxG; A.rA = R.rA; A.maskInC = R.maskInC; A.Bo_surf = R.Bo_surf;
  A.tmpFac = R.freeSurfFac * R.mass2rUnit * R.implicDiv2DFlow;     // :79, formed once as the reference does
  A.fsf = R.freeSurfFac;
  A.dTm = R.deltaTMom;
  {
    const double m = std::fabs(R.deltaTMom);
    A.rdTm = (m >= 0x1p-64 && m <= 0x1p64) ? 1.0 / R.deltaTMom : 0.0;   // host IEEE division: RN(1 / deltaTMom)
  }
  A.dTfs = R.deltaTFreeSurf;
  A.fresh_water = R.useRealFreshWaterFlux;
  A.Nr = R.Nr;
  k_rhs_fill<<<grid_of(tp, R.batch), 256, 0, st>>>(tp, R.Bo_surf, R.etaN, R.cg2d_b, R.cg2d_x);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int nrb = (tp.nj + kRhsOwnRows - 1) / kRhsOwnRows;
  const dim3 grid((unsigned)((tp.ni + kRhsCols - 1) / kRhsCols), (unsigned)(tp.T * nrb), (unsigned)R.batch);
  e = cudaFuncSetAttribute(k_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRhsSmem);
  if (e != cudaSuccess) return e;
  k_rhs<<<grid, dim3(32, kRhsRows), kRhsSmem, st>>>(tp, A, R.cg2d_b);
  return cudaGetLastError();
}

cudaError_t pressure_ini_norm(const TopoDev& tp, int batch, int Nr, double implicSurfPress, double implicDiv2DFlow,
                              const double* hFacW, const double* hFacS, const double* drF, const double* dyG,
                              const double* dxG, const double* recip_dxC, const double* recip_dyC, double* norm,
                              cudaStream_t st) {
  if (batch < 1 || batch > 65535 || Nr < 1) return cudaErrorInvalidValue;
  unsigned long long* bits = reinterpret_cast<unsigned long long*>(norm);
  cudaError_t e = cudaMemsetAsync(bits, 0, sizeof(double) * (size_t)batch, st);
  if (e != cudaSuccess) return e;
  // fac = implicSurfPress * implicDiv2DFlow, formed once as the reference does (cg2d.py:124)
  k_ini_norm_max<<<grid_of(tp, batch), 256, 0, st>>>(tp, Nr, hFacW, hFacS, drF, dyG, dxG, recip_dxC, recip_dyC,
                                                     implicSurfPress * implicDiv2DFlow, bits);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_ini_norm_fin<<<(batch + 127) / 128, 128, 0, st>>>(batch, bits);
  return cudaGetLastError();
}

cudaError_t pressure_post(const TopoDev& tp, int batch, const double* x, const double* cg2d_x,
                          const double* recip_Bo, double* etaN, cudaStream_t st) {
  if (batch < 1 || batch > 65535) return cudaErrorInvalidValue;
  k_post<<<grid_of(tp, batch), 256, 0, st>>>(tp, x, cg2d_x, recip_Bo, etaN);
  return cudaGetLastError();
}

}  // namespace cg2d
