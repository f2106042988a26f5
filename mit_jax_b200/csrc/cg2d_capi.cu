// C ABI of libcg2d.so: topology tables, workspace layout, argument checks and launches.
// Declarations and the reference interfaces they replace: include/cg2d.h.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "cg2d_internal.cuh"

struct cg2d_topology {
  int sNx, sNy, OLx, OLy, nTiles;
  int nip;           // column pitch of the S/N push-target lists (even)
  int* d_nbr;        // [4][...] W, E (T*sNy each), S, N (T*sNx each)
  int* d_tg;         // push targets (ring cells of the vectors, -1 = none): WE [T][sNy][4], S, N [T][nip][2]
  int* d_src;        // full padded map
  int8_t* d_comp;
  int device;
};

namespace {

using namespace cg2d;

constexpr size_t kAlign = 256;
inline size_t al(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

TopoDev topo_dev(const cg2d_topology* tp) {
  TopoDev d;
  d.nbr = tp->d_nbr;
  d.tg = tp->d_tg;
  d.nip = tp->nip;
  d.P = vec_pitch(tp->sNx);
  d.map_src = tp->d_src;
  d.map_comp = tp->d_comp;
  d.ni = tp->sNx;
  d.nj = tp->sNy;
  d.OLx = tp->OLx;
  d.OLy = tp->OLy;
  d.npx = tp->sNx + 2 * tp->OLx;
  d.npy = tp->sNy + 2 * tp->OLy;
  d.T = tp->nTiles;
  return d;
}

struct WsLayout {
  size_t gs, rmax, prof, zero_end, hist, part, total;
  size_t vec[kMaxGroups], cpk[kMaxGroups];
  long long vec_stride[kMaxGroups];
  long long vec_off[kMaxGroups][V_NVEC];
  int hist_len, part_units, total_rhs, total_ops, total_units, max_ni;
  int nblk[kMaxGroups], units[kMaxGroups];
  int ch, nw, rpb, nstage[P_NPASS];   // chunk rows, compute warps, ROWBLOCK block rows
  unsigned stage_bytes;
  size_t smem;
};

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

cg2d_status_t check_params(const cg2d_params_t* p) {
  if (!p) return CG2D_BAD_ARG;
  if (p->precision != CG2D_PREC_F64 && p->precision != CG2D_PREC_MIXED) return CG2D_BAD_ARG;
  if (p->sum_order != CG2D_SUM_ROWBLOCK && p->sum_order != CG2D_SUM_FORTRAN) return CG2D_BAD_ARG;
  if (p->rows_per_block < 8 || p->rows_per_block % 8 != 0) return CG2D_BAD_ARG;
  if (p->replace_every < 0 || !(p->replace_above >= 0.0)) return CG2D_BAD_ARG;
  if (p->grid_ctas < 0 || p->ctas_per_sm < 0) return CG2D_BAD_ARG;
  if (!(p->timeout_s > 0.0) || p->timeout_s > 3600.0) return CG2D_BAD_ARG;
  if (p->test_missing_arrivals < 0 || p->test_missing_arrivals > 1024) return CG2D_BAD_ARG;
  if (p->unit_deal != 0 && p->unit_deal != 1) return CG2D_BAD_ARG;
  if (p->stages != 0 && (p->stages < 2 || p->stages > kMaxStages)) return CG2D_BAD_ARG;
  return CG2D_OK;
}

// mixed precision with two right-hand sides in the ROWBLOCK order keeps both solves of an instance interleaved
// (GroupDev::pair) in single-group launches (the builds for several groups leave the paired path out: its
// registers would make them spill)
inline int paired(int mixed, int serial, int nrhs, int ngroups) {
  return mixed && !serial && nrhs == 2 && ngroups == 1 ? 1 : 0;
}

// chunk height and stage buffers for nw compute warps: the largest chunk (nw rows; with 8 warps 8, else 4 rows)
// whose `ns` stage buffers fit
cg2d_status_t size_stages(const cg2d_group_t* gr, int ng, int mixed, int serial, int ns, int nw, WsLayout* L) {
  const size_t fixed = fixed_smem_bytes(L->max_ni, serial);
  const int chs[2] = {nw, nw == kWarps ? 4 : 0};
  for (int ch : chs) {
    if (ch == 0) break;
    unsigned hot = 0, rep = 0;
    for (int g = 0; g < ng; ++g) {
      const cg2d_topology* tp = gr[g].topo;
      const int npx = tp->sNx + 2 * tp->OLx;
      const int pair = paired(mixed, serial, gr[g].nrhs, ng);
      for (int pt : {P_S, P_X, P_Z}) {
        const StageLay S = stage_layout(pt, mixed, ch, gr[g].nrhs, tp->sNx, npx, pair);
        if (S.total > hot) hot = S.total;
      }
      if (mixed) {
        const StageLay S = stage_layout(P_R, mixed, ch, gr[g].nrhs, tp->sNx, npx, pair);
        if (S.total > rep) rep = S.total;
      }
    }
    // the direct-load passes stage (nw + 2) rows of (max_ni + 2) doubles per solve slot in the same area
    const unsigned direct = (unsigned)(2 * (nw + 2) * (L->max_ni + 2) * sizeof(double));
    // the sums of a pass are formed with a tile-sum buffer per warp in the same area
    const unsigned sums = (unsigned)((nw + 1) * kMaxTiles * sizeof(double));
    // the stage area (ns buffers) also holds a replacement pass's single stage, the direct passes' staging and the
    // tile-sum buffers
    unsigned sb = hot;
    if (ns * sb < sums) sb = (sums + ns - 1) / ns;
    if (ns * sb < rep) sb = (rep + ns - 1) / ns;
    if (ns * sb < direct) sb = (direct + ns - 1) / ns;
    sb = al128(sb);
    const size_t smem = fixed + (size_t)ns * sb;
    if (smem <= (size_t)kSmemLimit) {
      L->ch = ch;
      L->nw = nw;
      L->stage_bytes = sb;
      L->smem = smem;
      // FORTRAN order keeps every element product of a chunk in one buffer: one stage
      for (int i = 0; i < P_NPASS; ++i) L->nstage[i] = serial ? 1 : ns;
      L->nstage[P_R] = (!serial && rep <= sb) ? ns : 1;
      return CG2D_OK;
    }
  }
  return CG2D_UNSUPPORTED;
}

cg2d_status_t compute_layout(const cg2d_group_t* gr, int ng, const cg2d_params_t* p, WsLayout* L) {
  if (!gr || ng < 1 || ng > kMaxGroups) return CG2D_BAD_ARG;
  std::memset(L, 0, sizeof(*L));
  const bool mixed = p->precision == CG2D_PREC_MIXED;
  const bool serial = p->sum_order == CG2D_SUM_FORTRAN;
  const size_t vsz = mixed ? sizeof(float) : sizeof(double);
  int max_iters = 0;
  for (int g = 0; g < ng; ++g) {
    const cg2d_group_t& G = gr[g];
    if (!G.topo || G.count < 1 || G.nrhs < 1 || G.nrhs > 2) return CG2D_BAD_ARG;
    const cg2d_topology* tp = G.topo;
    if (tp->nTiles > kMaxTiles || tp->sNx > kMaxNi || tp->sNy > kMaxNi) return CG2D_UNSUPPORTED;
    // bulk copies move whole padded coefficient rows: 16-byte multiples
    if (((tp->sNx + 2 * tp->OLx) * 8) % 16 != 0) return CG2D_UNSUPPORTED;
    if (tp->sNx > L->max_ni) L->max_ni = tp->sNx;
  }
  // Mixed precision in the ROWBLOCK order runs a single group on the 16-warp build when two stages of its 15-row
  // chunks fit: blocks (work units) of kMixedWarps rows, one chunk each, with the deepest pipeline up to the one
  // asked for that fits (so that the pipeline depth, a schedule option, never changes the sum order). Otherwise 8
  // compute warps and rows_per_block rows.
  // (default depth: 3 stages on the 16-warp build, where one CTA per SM leaves the room, 2 elsewhere)
  const int ns = p->stages ? p->stages : 2;
  cg2d_status_t st = CG2D_UNSUPPORTED;
  if (mixed && !serial && ng == 1) {
    for (int n = p->stages ? p->stages : 3; n >= 2 && st != CG2D_OK; --n)
      st = size_stages(gr, ng, mixed, serial, n, kMixedWarps, L);
    if (st == CG2D_OK) L->rpb = kMixedWarps;
  }
  if (st != CG2D_OK) {
    st = size_stages(gr, ng, mixed, serial, ns, kWarps, L);
    if (st != CG2D_OK) return st;
    L->rpb = p->rows_per_block;
  }
  for (int g = 0; g < ng; ++g) {
    const cg2d_group_t& G = gr[g];
    const cg2d_topology* tp = G.topo;
    for (int s = 0; s < G.nrhs; ++s) {
      if (G.max_iters[s] < 0 || !(G.tolerance[s] >= 0.0)) return CG2D_BAD_ARG;
      if (G.max_iters[s] > max_iters) max_iters = G.max_iters[s];
    }
    L->nblk[g] = serial ? 1 : (tp->sNy + L->rpb - 1) / L->rpb;
    L->units[g] = L->nblk[g] * tp->nTiles;
    if (L->units[g] > L->part_units) L->part_units = L->units[g];
    L->total_rhs += G.count * G.nrhs;
    L->total_ops += G.count;
    const long long tu = (long long)L->total_units + (long long)G.count * L->units[g];
    if (tu > (1ll << 30)) return CG2D_UNSUPPORTED;
    L->total_units = (int)tu;
  }
  if (L->total_rhs > kMaxSolves || L->total_ops > kMaxOps) return CG2D_UNSUPPORTED;
  L->hist_len = max_iters + 2;
  size_t o = 0;
  L->gs = o; o += al(8 * sizeof(unsigned));
  L->rmax = o; o += al(sizeof(unsigned long long) * L->total_rhs);
  L->prof = o;
  if (p->profile) o += al(sizeof(unsigned long long) * (1 + (size_t)kMaxCtas * kProfSlots));
  L->zero_end = o;
  L->hist = o; o += al(sizeof(double) * (size_t)L->total_rhs * H_NKIND * L->hist_len);
  L->part = o; o += al(sizeof(double) * (size_t)L->total_rhs * 2 * L->part_units);
  for (int g = 0; g < ng; ++g) {
    const cg2d_topology* tp = gr[g].topo;
    // ringed vector tiles [T][sNy+2][P]; paired: one block per instance with both solves in every element
    const long long elems = (long long)tp->nTiles * (tp->sNy + 2) * vec_pitch(tp->sNx);
    const int pair = paired(mixed, serial, gr[g].nrhs, ng), per = pair ? 2 : 1;
    long long off = 0;
    L->vec_off[g][V_X] = off; off += (long long)al(sizeof(double) * per * elems);
    for (int v = 1; v < V_NVEC; ++v) { L->vec_off[g][v] = off; off += (long long)al(vsz * per * elems); }
    L->vec_stride[g] = off;
    L->vec[g] = o; o += al((size_t)off * gr[g].count * (pair ? 1 : gr[g].nrhs));
    // packed coefficients [count][2][T][sNy+1][3][ldc] (the solver's precision)
    L->cpk[g] = o;
    o += al(vsz * 2 * (size_t)tp->nTiles * (tp->sNy + 1) * 3 * coef_pitch(tp->sNx) * gr[g].count);
  }
  L->total = o;
  return CG2D_OK;
}

}  // namespace

extern "C" {

void cg2d_default_params(cg2d_params_t* p) {
  if (!p) return;
  p->precision = CG2D_PREC_F64;
  p->sum_order = CG2D_SUM_ROWBLOCK;
  p->rows_per_block = 8;
  p->replace_every = 25;
  p->replace_above = 100.0;
  p->grid_ctas = 0;
  p->ctas_per_sm = 0;
  p->timeout_s = 10.0;
  p->test_missing_arrivals = 0;
  p->profile = 0;
  p->unit_deal = 0;
  p->stages = 0;
}

const char* cg2d_status_string(cg2d_status_t s) {
  switch (s) {
    case CG2D_OK: return "ok";
    case CG2D_NOT_CONVERGED: return "not converged (numIters == max_iters)";
    case CG2D_NAN: return "final residual is NaN";
    case CG2D_BARRIER_TIMEOUT: return "grid-wide wait timed out; results invalid";
    case CG2D_BAD_ARG: return "bad argument";
    case CG2D_CUDA_ERROR: return "CUDA error";
    case CG2D_WORKSPACE_TOO_SMALL: return "workspace too small";
    case CG2D_UNSUPPORTED: return "unsupported size";
    case CG2D_INTERNAL_ERROR: return "device-side consistency check failed; results invalid";
  }
  return "unknown status";
}

cg2d_status_t cg2d_topology_create(int sNx, int sNy, int OLx, int OLy, int nTiles, const int32_t* src,
                                   const int8_t* comp, cg2d_topology_t** out) {
  if (!out || !src || !comp) return CG2D_BAD_ARG;
  *out = nullptr;
  if (sNx < 1 || sNy < 1 || OLx < 1 || OLy < 1 || nTiles < 1) return CG2D_BAD_ARG;
  if (nTiles > kMaxTiles || sNx > kMaxNi) return CG2D_UNSUPPORTED;
  const int npx = sNx + 2 * OLx, npy = sNy + 2 * OLy;
  const long long npad = (long long)nTiles * npy * npx;
  if (npad > (1ll << 31) - 1) return CG2D_UNSUPPORTED;
  for (long long p = 0; p < npad; ++p) {
    if (comp[p] != 0 && comp[p] != 1) return CG2D_BAD_ARG;     // scalar map: no component swap
    if (comp[p] == 1 && (src[p] < 0 || src[p] >= npad)) return CG2D_BAD_ARG;
  }
  auto pad = [&](int t, int jj, int ii) { return ((long long)t * npy + jj) * npx + ii; };
  auto to_cmp = [&](long long s, int* c) -> bool {
    const int t = (int)(s / ((long long)npy * npx));
    const long long rem = s - (long long)t * npy * npx;
    const int jj = (int)(rem / npx), ii = (int)(rem - (long long)jj * npx);
    if (jj < OLy || jj >= OLy + sNy || ii < OLx || ii >= OLx + sNx) return false;
    *c = (t * sNy + (jj - OLy)) * sNx + (ii - OLx);
    return true;
  };
  std::vector<int> nbr((size_t)nTiles * (2 * sNy + 2 * sNx), -1);
  int* W = nbr.data();
  int* E = W + (size_t)nTiles * sNy;
  int* S = E + (size_t)nTiles * sNy;
  int* N = S + (size_t)nTiles * sNx;
  for (int t = 0; t < nTiles; ++t) {
    for (int j = 0; j < sNy; ++j) {
      const long long pw = pad(t, j + OLy, OLx - 1), pe = pad(t, j + OLy, OLx + sNx);
      if (comp[pw] == 1 && !to_cmp(src[pw], &W[t * sNy + j])) return CG2D_BAD_ARG;
      if (comp[pe] == 1 && !to_cmp(src[pe], &E[t * sNy + j])) return CG2D_BAD_ARG;
    }
    for (int i = 0; i < sNx; ++i) {
      const long long ps = pad(t, OLy - 1, i + OLx), pn = pad(t, OLy + sNy, i + OLx);
      if (comp[ps] == 1 && !to_cmp(src[ps], &S[t * sNx + i])) return CG2D_BAD_ARG;
      if (comp[pn] == 1 && !to_cmp(src[pn], &N[t * sNx + i])) return CG2D_BAD_ARG;
    }
  }
  // push targets: every ring cell (side, tile, position) of the vectors that has a source is filled by that
  // point's owner whenever it writes the value. A source must lie on its own tile's edge, with at most two
  // target cells per edge point. A target is the cell's element in a ringed vector [T][sNy+2][P].
  const int P = vec_pitch(sNx);
  const int nip = round_up(sNx, 2);
  if ((long long)nTiles * (sNy + 2) * P > (1ll << 31) - 1) return CG2D_UNSUPPORTED;
  auto cell = [&](int t, int j, int i) { return (int)(((long long)t * (sNy + 2) + j + 1) * P + i + 1); };
  // lists by the source point's position: i == 0 -> WE row j (first pair), i == sNx-1 -> WE row j (second
  // pair), otherwise j == 0 -> S column i, j == sNy-1 -> N column i
  const size_t n_we = (size_t)nTiles * sNy * 4;
  std::vector<int> tg(n_we + (size_t)nTiles * nip * 4, -1);
  auto add_target = [&](int c, int target) -> bool {
    const int t = c / (sNy * sNx), rem = c - t * sNy * sNx, j = rem / sNx, i = rem - j * sNx;
    int* q;
    if (i == 0) q = &tg[((size_t)t * sNy + j) * 4];
    else if (i == sNx - 1) q = &tg[((size_t)t * sNy + j) * 4 + 2];
    else if (j == 0) q = &tg[n_we + ((size_t)t * nip + i) * 2];
    else if (j == sNy - 1) q = &tg[n_we + ((size_t)(nTiles + t) * nip + i) * 2];
    else return false;
    if (q[0] < 0) q[0] = target;
    else if (q[1] < 0) q[1] = target;
    else return false;
    return true;
  };
  for (int t = 0; t < nTiles; ++t) {
    for (int k = 0; k < sNy; ++k) {
      if (W[t * sNy + k] >= 0 && !add_target(W[t * sNy + k], cell(t, k, -1))) return CG2D_BAD_ARG;
      if (E[t * sNy + k] >= 0 && !add_target(E[t * sNy + k], cell(t, k, sNx))) return CG2D_BAD_ARG;
    }
    for (int k = 0; k < sNx; ++k) {
      if (S[t * sNx + k] >= 0 && !add_target(S[t * sNx + k], cell(t, -1, k))) return CG2D_BAD_ARG;
      if (N[t * sNx + k] >= 0 && !add_target(N[t * sNx + k], cell(t, sNy, k))) return CG2D_BAD_ARG;
    }
  }
  cg2d_topology* tp = new cg2d_topology();
  tp->sNx = sNx; tp->sNy = sNy; tp->OLx = OLx; tp->OLy = OLy; tp->nTiles = nTiles;
  tp->nip = nip;
  tp->d_nbr = nullptr; tp->d_tg = nullptr; tp->d_src = nullptr; tp->d_comp = nullptr;
  cudaGetDevice(&tp->device);
  bool ok = cudaMalloc(&tp->d_nbr, nbr.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&tp->d_tg, tg.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&tp->d_src, (size_t)npad * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&tp->d_comp, (size_t)npad) == cudaSuccess &&
            cudaMemcpy(tp->d_nbr, nbr.data(), nbr.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(tp->d_tg, tg.data(), tg.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(tp->d_src, src, (size_t)npad * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(tp->d_comp, comp, (size_t)npad, cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    cudaFree(tp->d_nbr); cudaFree(tp->d_tg); cudaFree(tp->d_src); cudaFree(tp->d_comp);
    delete tp;
    cudaGetLastError();
    return CG2D_CUDA_ERROR;
  }
  *out = tp;
  return CG2D_OK;
}

cg2d_status_t cg2d_topology_destroy(cg2d_topology_t* tp) {
  if (!tp) return CG2D_BAD_ARG;
  cudaFree(tp->d_nbr);
  cudaFree(tp->d_tg);
  cudaFree(tp->d_src);
  cudaFree(tp->d_comp);
  delete tp;
  return CG2D_OK;
}

size_t cg2d_workspace_size(const cg2d_group_t* groups, int ngroups, const cg2d_params_t* params) {
  cg2d_params_t def;
  if (!params) { cg2d_default_params(&def); params = &def; }
  if (check_params(params) != CG2D_OK) return 0;
  WsLayout L;
  if (compute_layout(groups, ngroups, params, &L) != CG2D_OK) return 0;
  return L.total;
}

// checkpoint recording for the exact-mode adjoint (see KParams::ck_r), and where the launch keeps its sums
struct CkRec {
  double* ck_r;
  double* ck_s;
  long long stride;
  int every;
  const double** hist;   // out: the launch's sum history [total_rhs][H_NKIND][hist_len]
  int* hist_len;
};

static cg2d_status_t solve_groups_impl(const cg2d_group_t* groups, int ngroups, const cg2d_params_t* params,
                                       void* workspace, size_t workspace_bytes, cg2d_stream_t stream_,
                                       const CkRec* ck) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  cg2d_params_t def;
  if (!params) { cg2d_default_params(&def); params = &def; }
  cg2d_status_t st = check_params(params);
  if (st != CG2D_OK) return st;
  WsLayout L;
  st = compute_layout(groups, ngroups, params, &L);
  if (st != CG2D_OK) return st;
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) % kAlign) != 0) return CG2D_BAD_ARG;
  if (workspace_bytes < L.total) return CG2D_WORKSPACE_TOO_SMALL;
  for (int g = 0; g < ngroups; ++g) {
    const cg2d_group_t& G = groups[g];
    if (!G.aW2d || !G.aS2d || !G.aC2d || !G.pW || !G.pS || !G.pC) return CG2D_BAD_ARG;
    for (const double* a : {G.aW2d, G.aS2d, G.aC2d, G.pW, G.pS, G.pC})
      if (reinterpret_cast<uintptr_t>(a) % 16 != 0) return CG2D_BAD_ARG;   // bulk-copy sources
    for (int s = 0; s < G.nrhs; ++s)
      if (!G.b[s] || !G.x0[s] || !G.x_out[s] || !G.diag[s]) return CG2D_BAD_ARG;
  }
  char* ws = static_cast<char*>(workspace);
  KParams kp;
  std::memset(&kp, 0, sizeof(kp));
  kp.ngroups = ngroups;
  kp.total_units = L.total_units;
  kp.total_rhs = L.total_rhs;
  kp.total_ops = L.total_ops;
  kp.mixed = params->precision == CG2D_PREC_MIXED;
  kp.serial = params->sum_order == CG2D_SUM_FORTRAN;
  kp.rows_per_block = L.rpb;
  kp.nw = L.nw;
  kp.replace_every = params->replace_every;
  kp.replace_above = params->replace_above;
  kp.max_ni = L.max_ni;
  kp.ch = L.ch;
  for (int i = 0; i < P_NPASS; ++i) kp.nstage[i] = L.nstage[i];
  kp.stage_bytes = L.stage_bytes;
  kp.hist = reinterpret_cast<double*>(ws + L.hist);
  kp.hist_len = L.hist_len;
  kp.part = reinterpret_cast<double*>(ws + L.part);
  kp.part_units = L.part_units;
  kp.rmax = reinterpret_cast<unsigned long long*>(ws + L.rmax);
  kp.gs = reinterpret_cast<unsigned*>(ws + L.gs);
  kp.timeout_ns = (unsigned long long)(params->timeout_s * 1e9);
  kp.test_missing = params->test_missing_arrivals;
  kp.unit_deal = params->unit_deal;
  kp.prof = params->profile ? reinterpret_cast<unsigned long long*>(ws + L.prof) : nullptr;
  if (ck) {
    if (ngroups != 1 || groups[0].nrhs != 1 || params->precision != CG2D_PREC_F64 || ck->every < 1)
      return CG2D_BAD_ARG;
    kp.ck_r = ck->ck_r;
    kp.ck_s = ck->ck_s;
    kp.ck_stride = ck->stride;
    kp.ck_every = ck->every;
    if (ck->hist) *ck->hist = kp.hist;
    if (ck->hist_len) *ck->hist_len = kp.hist_len;
  }
  for (int g = 0; g < ngroups; ++g) {
    const cg2d_topology* tp = groups[g].topo;
    for (int pt = 0; pt < P_NPASS; ++pt)
      kp.lay[g][pt] = stage_layout(pt, kp.mixed, L.ch, groups[g].nrhs, tp->sNx, tp->sNx + 2 * tp->OLx,
                                   paired(kp.mixed, kp.serial, groups[g].nrhs, ngroups));
  }
  int unit_base = 0, op_base = 0, rhs_base = 0;
  for (int g = 0; g < ngroups; ++g) {
    const cg2d_group_t& G = groups[g];
    GroupDev& d = kp.g[g];
    d.tp = topo_dev(G.topo);
    d.count = G.count;
    d.nrhs = G.nrhs;
    d.nblk = L.nblk[g];
    d.units = L.units[g];
    d.unit_base = unit_base;
    d.op_base = op_base;
    d.rhs_base = rhs_base;
    d.pad_elems = (long long)d.tp.T * d.tp.npy * d.tp.npx;
    d.ldc = coef_pitch(d.tp.ni);
    d.a64[0] = G.aW2d; d.a64[1] = G.aS2d; d.a64[2] = G.aC2d;
    d.a64[3] = G.pW; d.a64[4] = G.pS; d.a64[5] = G.pC;
    d.cpk = ws + L.cpk[g];
    d.norm = G.cg2dNorm;
    d.norm_arr = G.cg2dNorm_per_instance;
    for (int s = 0; s < 2; ++s) {
      const bool on = s < G.nrhs;
      d.b[s] = on ? G.b[s] : nullptr;
      d.x0[s] = on ? G.x0[s] : nullptr;
      d.x_out[s] = on ? G.x_out[s] : nullptr;
      d.x_fortran[s] = on ? G.x_fortran[s] : nullptr;
      d.diag[s] = on ? G.diag[s] : nullptr;
      d.tol[s] = on ? G.tolerance[s] : 0.0;
      d.max_iters[s] = on ? G.max_iters[s] : 0;
    }
    d.vec = ws + L.vec[g];
    d.vec_stride = L.vec_stride[g];
    d.pair = paired(kp.mixed, kp.serial, G.nrhs, ngroups);
    for (int v = 0; v < V_NVEC; ++v) d.vec_off[v] = L.vec_off[g][v];
    unit_base += G.count * d.units;
    op_base += G.count;
    rhs_base += G.count * G.nrhs;
  }

  const size_t smem = L.smem;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // FP64 has a kernel built for 1 CTA per SM (no register limit below the SM's) and one for 2 (96 registers a
  // thread). ctas_per_sm 2 takes the second; 0 takes it when every group has one right-hand side and there are at
  // least 8 units per SM, where its doubled warps pay for the spills (exact-mode forward solves); otherwise the first.
  kp.fp64_cps = 1;
  if (!kp.mixed) {
    bool one_rhs = true;
    for (int g = 0; g < ngroups; ++g) one_rhs = one_rhs && groups[g].nrhs == 1;
    if (params->ctas_per_sm == 2 || (params->ctas_per_sm == 0 && one_rhs && kp.total_units >= 8 * nsm))
      kp.fp64_cps = 2;
  }
  int bps = 0;
  if (solver_occupancy(kp, smem, &bps) != cudaSuccess || bps < 1) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  if (params->ctas_per_sm > 0 && params->ctas_per_sm < bps) bps = params->ctas_per_sm;
  long long grid = (long long)bps * nsm;
  if (params->grid_ctas > 0 && params->grid_ctas < grid) grid = params->grid_ctas;
  if (grid > kp.total_units) grid = kp.total_units;
  if (grid > kMaxCtas) grid = kMaxCtas;
  if (grid < 1) grid = 1;
  if ((kp.total_units + grid - 1) / grid > kMaxUnitsPerCta) return CG2D_UNSUPPORTED;   // unit table of a CTA
  if (cudaMemsetAsync(ws, 0, L.zero_end, stream) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  for (int g = 0; g < ngroups; ++g)
    if (launch_pack_coef(kp.g[g], kp.mixed, stream) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }

  if (launch_solver(kp, (int)grid, smem, stream) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

cg2d_status_t cg2d_solve_groups(const cg2d_group_t* groups, int ngroups, const cg2d_params_t* params,
                                void* workspace, size_t workspace_bytes, cg2d_stream_t stream) {
  return solve_groups_impl(groups, ngroups, params, workspace, workspace_bytes, stream, nullptr);
}

cg2d_status_t cg2d_solve_f64(const cg2d_topology_t* topo, int batch, double cg2dNorm, const double* aW2d,
                             const double* aS2d, const double* aC2d, const double* pW, const double* pS,
                             const double* pC, const double* cg2d_b, const double* cg2d_x, double tolerance,
                             int max_iters, double* x_out, double* x_fortran, cg2d_diag_t* diag,
                             const cg2d_params_t* params, void* workspace, size_t workspace_bytes,
                             cg2d_stream_t stream) {
  cg2d_group_t g;
  std::memset(&g, 0, sizeof(g));
  g.topo = topo;
  g.count = batch;
  g.nrhs = 1;
  g.aW2d = aW2d; g.aS2d = aS2d; g.aC2d = aC2d; g.pW = pW; g.pS = pS; g.pC = pC;
  g.cg2dNorm = cg2dNorm;
  g.b[0] = cg2d_b;
  g.x0[0] = cg2d_x;
  g.x_out[0] = x_out;
  g.x_fortran[0] = x_fortran;
  g.diag[0] = diag;
  g.tolerance[0] = tolerance;
  g.max_iters[0] = max_iters;
  return cg2d_solve_groups(&g, 1, params, workspace, workspace_bytes, stream);
}

cg2d_status_t cg2d_solve_mixed(const cg2d_topology_t* topo, int batch, double cg2dNorm, const double* aW2d,
                               const double* aS2d, const double* aC2d, const double* pW, const double* pS,
                               const double* pC, const double* cg2d_b, const double* cg2d_x, double tolerance,
                               int max_iters, double* x_out, double* x_fortran, cg2d_diag_t* diag,
                               const cg2d_params_t* params, void* workspace, size_t workspace_bytes,
                               cg2d_stream_t stream) {
  cg2d_params_t p;
  if (params) p = *params; else cg2d_default_params(&p);
  p.precision = CG2D_PREC_MIXED;
  return cg2d_solve_f64(topo, batch, cg2dNorm, aW2d, aS2d, aC2d, pW, pS, pC, cg2d_b, cg2d_x, tolerance, max_iters,
                        x_out, x_fortran, diag, &p, workspace, workspace_bytes, stream);
}

namespace {
// one uniform group of `batch` single right-hand-side solves (the pointers are filled by the caller)
cg2d_group_t one_group(const cg2d_topology_t* topo, int batch, double tol, int max_iters) {
  cg2d_group_t g;
  std::memset(&g, 0, sizeof(g));
  g.topo = topo;
  g.count = batch;
  g.nrhs = 1;
  g.tolerance[0] = tol;
  g.max_iters[0] = max_iters;
  return g;
}
size_t round256(size_t n) { return (n + 255) & ~size_t(255); }
}  // namespace

size_t cg2d_adjoint_ecco_workspace_size(const cg2d_topology_t* topo, int batch, int adj_max_iters,
                                        const cg2d_params_t* params) {
  if (!topo || batch < 1 || adj_max_iters < 0) return 0;
  cg2d_group_t g = one_group(topo, batch, 0.0, adj_max_iters);
  const size_t solver = cg2d_workspace_size(&g, 1, params);
  if (solver == 0) return 0;
  const TopoDev tp = topo_dev(topo);
  return round256(solver) + sizeof(double) * (size_t)batch * tp.T * tp.npy * tp.npx;
}

cg2d_status_t cg2d_adjoint_ecco(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                                const double* cg2dNorm_per_instance, const double* aW2d, const double* aS2d,
                                const double* aC2d, const double* pW, const double* pS, const double* pC,
                                const double* x, const double* x_bar, double adj_tolerance, int adj_max_iters,
                                int coeff_grad, double* lam, double* gW, double* gS, double* gC, cg2d_diag_t* diag,
                                const cg2d_params_t* params, void* workspace, size_t workspace_bytes,
                                cg2d_stream_t stream) {
  if (!topo || batch < 1 || !x_bar || !lam || !diag || !workspace || (coeff_grad && (!x || !gW || !gS || !gC)) ||
      coeff_grad < 0 || coeff_grad > 1)
    return CG2D_BAD_ARG;
  const size_t need = cg2d_adjoint_ecco_workspace_size(topo, batch, adj_max_iters, params);
  if (need == 0) return CG2D_BAD_ARG;
  if (workspace_bytes < need) return CG2D_WORKSPACE_TOO_SMALL;
  cg2d_group_t g = one_group(topo, batch, adj_tolerance, adj_max_iters);
  const size_t solver = round256(cg2d_workspace_size(&g, 1, params));
  const TopoDev tp = topo_dev(topo);
  const size_t vb = sizeof(double) * (size_t)batch * tp.T * tp.npy * tp.npx;
  double* zero = reinterpret_cast<double*>(static_cast<char*>(workspace) + solver);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(zero, 0, vb, st) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  g.aW2d = aW2d; g.aS2d = aS2d; g.aC2d = aC2d; g.pW = pW; g.pS = pS; g.pC = pC;
  g.cg2dNorm = cg2dNorm;
  g.cg2dNorm_per_instance = cg2dNorm_per_instance;
  g.b[0] = x_bar;
  g.x0[0] = zero;
  g.x_out[0] = lam;
  g.diag[0] = diag;
  cg2d_status_t s = cg2d_solve_groups(&g, 1, params, workspace, solver, stream);
  if (s != CG2D_OK) return s;
  if (coeff_grad) return cg2d_edge_products(topo, batch, cg2dNorm, cg2dNorm_per_instance, lam, x, gW, gS, gC, stream);
  for (double* gg : {gW, gS, gC})
    if (gg && cudaMemsetAsync(gg, 0, vb, st) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

size_t cg2d_adjoint_exact_workspace_size(const cg2d_topology_t* topo, int batch, int max_iters,
                                         int checkpoint_every) {
  if (!topo || batch < 1 || max_iters < 0 || checkpoint_every < 0) return 0;
  return exact_adjoint_workspace(topo_dev(topo), batch, max_iters, checkpoint_every);
}

cg2d_status_t cg2d_adjoint_exact(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                                 const double* cg2dNorm_per_instance, const double* aW2d, const double* aS2d,
                                 const double* aC2d, const double* pW, const double* pS, const double* pC,
                                 const double* cg2d_b, const double* cg2d_x, const cg2d_diag_t* fwd_diag,
                                 const double* x_bar, int max_iters, int rows_per_block, int checkpoint_every,
                                 double* b_bar, double* gW, double* gS, double* gC, double* gpW, double* gpS,
                                 double* gpC, double* x_check, void* workspace, size_t workspace_bytes,
                                 cg2d_stream_t stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  if (!topo || batch < 1 || max_iters < 0 || checkpoint_every < 0 || rows_per_block < 1) return CG2D_BAD_ARG;
  for (const void* p : {(const void*)aW2d, (const void*)aS2d, (const void*)aC2d, (const void*)pW, (const void*)pS,
                        (const void*)pC, (const void*)cg2d_b, (const void*)cg2d_x, (const void*)fwd_diag,
                        (const void*)x_bar, (const void*)b_bar, (const void*)gW, (const void*)gS, (const void*)gC,
                        (const void*)gpW, (const void*)gpS, (const void*)gpC})
    if (!p) return CG2D_BAD_ARG;
  const size_t need = exact_adjoint_workspace(topo_dev(topo), batch, max_iters, checkpoint_every);
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) % kAlign) != 0) return CG2D_BAD_ARG;
  if (workspace_bytes < need) return CG2D_WORKSPACE_TOO_SMALL;
  // the forward's iteration counts bound the reverse sweep: read them once
  std::vector<cg2d_diag_t> d((size_t)batch);
  if (cudaMemcpyAsync(d.data(), fwd_diag, sizeof(cg2d_diag_t) * batch, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  int kmax = 0;
  for (const cg2d_diag_t& r : d) {
    if (r.numIters < 0 || r.numIters > max_iters) return CG2D_BAD_ARG;
    kmax = r.numIters > kmax ? r.numIters : kmax;
  }
  ExactArgs a{};
  a.batch = batch;
  a.max_iters = kmax;
  a.max_iters_cap = max_iters;
  a.checkpoint = checkpoint_every;
  a.rows_per_block = rows_per_block;
  a.norm = cg2dNorm;
  a.norm_arr = cg2dNorm_per_instance;
  a.aW = aW2d; a.aS = aS2d; a.aC = aC2d; a.pW = pW; a.pS = pS; a.pC = pC;
  a.b = cg2d_b; a.x0 = cg2d_x; a.xbar = x_bar; a.fwd_diag = fwd_diag;
  a.b_bar = b_bar; a.gW = gW; a.gS = gS; a.gC = gC; a.gpW = gpW; a.gpS = gpS; a.gpC = gpC; a.x_check = x_check;
  if (exact_adjoint(topo_dev(topo), a, workspace, stream) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

namespace {
cg2d_params_t exact_params(int rows_per_block) {
  cg2d_params_t p;
  cg2d_default_params(&p);
  p.precision = CG2D_PREC_F64;
  p.sum_order = CG2D_SUM_ROWBLOCK;
  p.rows_per_block = rows_per_block;
  return p;
}
}  // namespace

size_t cg2d_solve_exact_workspace_size(const cg2d_topology_t* topo, int batch, int max_iters, int rows_per_block,
                                       int checkpoint_every) {
  if (!topo || batch < 1 || max_iters < 0 || checkpoint_every < 0) return 0;
  const cg2d_params_t p = exact_params(rows_per_block);
  cg2d_group_t g = one_group(topo, batch, 0.0, max_iters);
  const size_t solver = cg2d_workspace_size(&g, 1, &p);
  if (solver == 0) return 0;
  return round256(exact_adjoint_workspace(topo_dev(topo), batch, max_iters, checkpoint_every)) + solver;
}

cg2d_status_t cg2d_solve_exact(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                               const double* cg2dNorm_per_instance, const double* aW2d, const double* aS2d,
                               const double* aC2d, const double* pW, const double* pS, const double* pC,
                               const double* cg2d_b, const double* cg2d_x, double tolerance, int max_iters,
                               const double* x_bar, int rows_per_block, int checkpoint_every, double* x_out,
                               cg2d_diag_t* diag, double* b_bar, double* gW, double* gS, double* gC, double* gpW,
                               double* gpS, double* gpC, void* workspace, size_t workspace_bytes,
                               cg2d_stream_t stream_) {
  if (!topo || batch < 1 || max_iters < 0 || checkpoint_every < 0 || rows_per_block < 8 || !x_bar || !x_out ||
      !diag || !b_bar || !gW || !gS || !gC || !gpW || !gpS || !gpC || !workspace)
    return CG2D_BAD_ARG;
  const size_t need = cg2d_solve_exact_workspace_size(topo, batch, max_iters, rows_per_block, checkpoint_every);
  if (need == 0) return CG2D_BAD_ARG;
  if (workspace_bytes < need) return CG2D_WORKSPACE_TOO_SMALL;
  if ((reinterpret_cast<uintptr_t>(workspace) % kAlign) != 0) return CG2D_BAD_ARG;
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  const TopoDev tp = topo_dev(topo);
  // workspace: the adjoint's (its checkpoint blocks receive the forward's r_c, s_{c-1}), then the solver's
  char* adj = static_cast<char*>(workspace);
  const size_t adj_bytes = round256(exact_adjoint_workspace(tp, batch, max_iters, checkpoint_every));
  CkRec ck;
  exact_checkpoints(tp, batch, max_iters, checkpoint_every, adj, &ck.ck_r, &ck.ck_s, &ck.stride);
  ck.every = checkpoint_every > 0 ? checkpoint_every : (max_iters > 0 ? max_iters : 1);
  const double* hist = nullptr;
  int hist_len = 0;
  ck.hist = &hist;
  ck.hist_len = &hist_len;
  const cg2d_params_t p = exact_params(rows_per_block);
  cg2d_group_t g = one_group(topo, batch, tolerance, max_iters);
  g.aW2d = aW2d; g.aS2d = aS2d; g.aC2d = aC2d; g.pW = pW; g.pS = pS; g.pC = pC;
  g.cg2dNorm = cg2dNorm;
  g.cg2dNorm_per_instance = cg2dNorm_per_instance;
  g.b[0] = cg2d_b;
  g.x0[0] = cg2d_x;
  g.x_out[0] = x_out;
  g.diag[0] = diag;
  cg2d_status_t s = solve_groups_impl(&g, 1, &p, adj + adj_bytes, workspace_bytes - adj_bytes, stream_, &ck);
  if (s != CG2D_OK) return s;
  std::vector<cg2d_diag_t> d((size_t)batch);
  if (cudaMemcpyAsync(d.data(), diag, sizeof(cg2d_diag_t) * batch, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  int kmax = 0;
  for (const cg2d_diag_t& r : d) {
    if (r.status == CG2D_BARRIER_TIMEOUT || r.status == CG2D_INTERNAL_ERROR) return (cg2d_status_t)r.status;
    kmax = r.numIters > kmax ? r.numIters : kmax;
  }
  ExactArgs a{};
  a.batch = batch;
  a.max_iters = kmax;
  a.max_iters_cap = max_iters;
  a.checkpoint = checkpoint_every;
  a.rows_per_block = rows_per_block;
  a.recorded = 1;
  a.hist = hist;
  a.hist_len = hist_len;
  a.norm = cg2dNorm;
  a.norm_arr = cg2dNorm_per_instance;
  a.aW = aW2d; a.aS = aS2d; a.aC = aC2d; a.pW = pW; a.pS = pS; a.pC = pC;
  a.b = cg2d_b; a.x0 = cg2d_x; a.xbar = x_bar; a.fwd_diag = diag;
  a.b_bar = b_bar; a.gW = gW; a.gS = gS; a.gC = gC; a.gpW = gpW; a.gpS = gpS; a.gpC = gpC; a.x_check = nullptr;
  if (exact_adjoint(tp, a, adj, stream) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

cg2d_status_t cg2d_workspace_status(const void* workspace, cg2d_stream_t stream) {
  if (!workspace) return CG2D_BAD_ARG;
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  unsigned w[2] = {0, 0};
  if (cudaMemcpy(w, workspace, sizeof(w), cudaMemcpyDeviceToHost) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return w[1] ? (cg2d_status_t)w[1] : CG2D_OK;
}

cg2d_status_t cg2d_workspace_profile(const void* workspace, const cg2d_group_t* groups, int ngroups,
                                     const cg2d_params_t* params, uint64_t* out, int cap, cg2d_stream_t stream) {
  if (!workspace || !out || cap < 1 || !params || !params->profile) return CG2D_BAD_ARG;
  WsLayout L;
  if (check_params(params) != CG2D_OK || compute_layout(groups, ngroups, params, &L) != CG2D_OK) return CG2D_BAD_ARG;
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  const size_t n = 1 + (size_t)(cap < kMaxCtas ? cap : kMaxCtas) * kProfSlots;
  if (cudaMemcpy(out, static_cast<const char*>(workspace) + L.prof, n * sizeof(uint64_t), cudaMemcpyDeviceToHost) !=
      cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

cg2d_status_t cg2d_apply_operator(const cg2d_topology_t* topo, int batch, double cg2dNorm, const double* aW2d,
                                  const double* aS2d, const double* aC2d, const double* v, double* out,
                                  cg2d_stream_t stream) {
  if (!topo || batch < 1 || !aW2d || !aS2d || !aC2d || !v || !out || v == out) return CG2D_BAD_ARG;
  if (launch_apply_operator(topo_dev(topo), batch, cg2dNorm, aW2d, aS2d, aC2d, v, out,
                            reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

cg2d_status_t cg2d_edge_products(const cg2d_topology_t* topo, int batch, double cg2dNorm,
                                 const double* cg2dNorm_per_instance, const double* lam, const double* x,
                                 double* gW, double* gS, double* gC, cg2d_stream_t stream) {
  if (!topo || batch < 1 || !lam || !x || !gW || !gS || !gC) return CG2D_BAD_ARG;
  if (launch_edge_products(topo_dev(topo), batch, cg2dNorm, cg2dNorm_per_instance, lam, x, gW, gS, gC,
                           reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

cg2d_status_t cg2d_exchange_scalar(const cg2d_topology_t* topo, int batch, const double* a, double* out,
                                   cg2d_stream_t stream) {
  if (!topo || batch < 1 || !a || !out || a == out) return CG2D_BAD_ARG;
  if (launch_exchange(topo_dev(topo), batch, a, out, reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

cg2d_status_t cg2d_update_operator(const cg2d_topology_t* topo, int batch, const cg2d_freesurf_t* fs,
                                   double cg2dNorm, const double* cg2dNorm_per_instance, double cg2dpcOffDFac,
                                   const double* hFacW, const double* hFacS, const double* drF,
                                   const double* dyG, const double* dxG, const double* recip_dxC,
                                   const double* recip_dyC, const double* rA, const double* recip_Bo,
                                   double* aW2d, double* aS2d, double* aC2d, double* pW, double* pS, double* pC,
                                   cg2d_stream_t stream) {
  if (!topo || !fs || batch < 1 || batch > 65535 || fs->Nr < 1) return CG2D_BAD_ARG;
  for (const void* q : {(const void*)hFacW, (const void*)hFacS, (const void*)drF, (const void*)dyG,
                        (const void*)dxG, (const void*)recip_dxC, (const void*)recip_dyC, (const void*)rA,
                        (const void*)recip_Bo, (const void*)aW2d, (const void*)aS2d, (const void*)aC2d,
                        (const void*)pW, (const void*)pS, (const void*)pC})
    if (!q) return CG2D_BAD_ARG;
  UpdateArgs U;
  U.batch = batch;
  U.Nr = fs->Nr;
  U.hFacW = hFacW; U.hFacS = hFacS; U.drF = drF; U.dyG = dyG; U.dxG = dxG;
  U.recip_dxC = recip_dxC; U.recip_dyC = recip_dyC; U.rA = rA; U.recip_Bo = recip_Bo;
  U.norm = cg2dNorm;
  U.norm_arr = cg2dNorm_per_instance;
  U.offd = cg2dpcOffDFac;
  U.implicSurfPress = fs->implicSurfPress;
  U.implicDiv2DFlow = fs->implicDiv2DFlow;
  U.freeSurfFac = fs->freeSurfFac;
  U.deltaTMom = fs->deltaTMom;
  U.deltaTFreeSurf = fs->deltaTFreeSurf;
  U.aW2d = aW2d; U.aS2d = aS2d; U.aC2d = aC2d; U.pW = pW; U.pS = pS; U.pC = pC;
  if (pressure_update(topo_dev(topo), U, reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

cg2d_status_t cg2d_pressure_rhs(const cg2d_topology_t* topo, int batch, const cg2d_freesurf_t* fs,
                                const double* gU, const double* gV, const double* hFacW, const double* hFacS,
                                const double* EmPmR, const double* etaN, const double* etaH, const double* drF,
                                const double* dyG, const double* dxG, const double* rA, const double* maskInC,
                                const double* Bo_surf, double* cg2d_b, double* cg2d_x, cg2d_stream_t stream) {
  if (!topo || !fs || batch < 1 || batch > 65535 || fs->Nr < 1) return CG2D_BAD_ARG;
  for (const void* q : {(const void*)gU, (const void*)gV, (const void*)hFacW, (const void*)hFacS,
                        (const void*)etaN, (const void*)etaH, (const void*)drF, (const void*)dyG, (const void*)dxG,
                        (const void*)rA, (const void*)Bo_surf, (const void*)cg2d_b, (const void*)cg2d_x})
    if (!q) return CG2D_BAD_ARG;
  if (fs->useRealFreshWaterFlux && (!EmPmR || !maskInC)) return CG2D_BAD_ARG;
  RhsIn R;
  R.batch = batch;
  R.Nr = fs->Nr;
  R.useRealFreshWaterFlux = fs->useRealFreshWaterFlux ? 1 : 0;
  R.gU = gU; R.gV = gV; R.hFacW = hFacW; R.hFacS = hFacS; R.EmPmR = EmPmR; R.etaN = etaN; R.etaH = etaH;
  R.drF = drF; R.dyG = dyG; R.dxG = dxG; R.rA = rA; R.maskInC = maskInC; R.Bo_surf = Bo_surf;
  R.freeSurfFac = fs->freeSurfFac;
  R.mass2rUnit = fs->mass2rUnit;
  R.implicDiv2DFlow = fs->implicDiv2DFlow;
  R.deltaTMom = fs->deltaTMom;
  R.deltaTFreeSurf = fs->deltaTFreeSurf;
  R.cg2d_b = cg2d_b;
  R.cg2d_x = cg2d_x;
  if (pressure_rhs(topo_dev(topo), R, reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

cg2d_status_t cg2d_ini_norm(const cg2d_topology_t* topo, int batch, int Nr, double implicSurfPress,
                             double implicDiv2DFlow, const double* hFacW, const double* hFacS, const double* drF,
                             const double* dyG, const double* dxG, const double* recip_dxC, const double* recip_dyC,
                             double* cg2dNorm, cg2d_stream_t stream) {
  if (!topo || batch < 1 || batch > 65535 || Nr < 1) return CG2D_BAD_ARG;
  for (const void* q : {(const void*)hFacW, (const void*)hFacS, (const void*)drF, (const void*)dyG, (const void*)dxG,
                        (const void*)recip_dxC, (const void*)recip_dyC, (const void*)cg2dNorm})
    if (!q) return CG2D_BAD_ARG;
  if (pressure_ini_norm(topo_dev(topo), batch, Nr, implicSurfPress, implicDiv2DFlow, hFacW, hFacS, drF, dyG, dxG,
                        recip_dxC, recip_dyC, cg2dNorm, reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) {
    cudaGetLastError();
    return CG2D_CUDA_ERROR;
  }
  return CG2D_OK;
}

cg2d_status_t cg2d_pressure_post(const cg2d_topology_t* topo, int batch, const double* x, const double* cg2d_x,
                                 const double* recip_Bo, double* etaN, cg2d_stream_t stream) {
  if (!topo || batch < 1 || batch > 65535 || !x || !cg2d_x || !recip_Bo || !etaN || etaN == x || etaN == cg2d_x)
    return CG2D_BAD_ARG;
  if (pressure_post(topo_dev(topo), batch, x, cg2d_x, recip_Bo, etaN, reinterpret_cast<cudaStream_t>(stream)) !=
      cudaSuccess) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  return CG2D_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Solve without any allocation. Some callers cannot allocate device memory at the point where they solve: a
// solver step running inside a framework that owns the whole device pool (an XLA custom call handed only its
// operands, a model step under a memory-capped allocator), or code where a cudaMalloc would synchronise the
// device and stall its other streams. They use this entry point, whose workspace is a fixed array in the
// library's device memory. The array is reserved on a device when the module holding it is loaded there: with
// CUDA's lazy module loading (the default) that is the first call of this entry point on the device, which may
// fail with an out-of-memory error if a framework has taken the whole pool by then, so make that first call at
// start-up. From then on the device holds CG2D_NOALLOC_SCRATCH_BYTES for it until the process exits, and calls
// reserve nothing more; all calls on a device share it.
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[CG2D_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch, looked up with the device current and kept per device together with the
// unique ID of the context it was looked up in (cuCtxGetId, reached through the runtime's driver entry points so
// that the library needs no link to libcuda). A context created after a cudaDeviceReset has a new ID, so the
// address is looked up again there instead of reusing one from the destroyed context. The first lookup in a
// context loads the library's device module under lazy loading, which reserves the array.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {};
unsigned long long g_noalloc_ctx[kMaxDevices] = {};

using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);

// ID of the current context, 0 when there is none or the driver does not report IDs (then every call looks the
// address up again, which allocates nothing once the module is loaded)
unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

cg2d_status_t noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  unsigned long long id = current_ctx_id();
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (id != 0 && g_noalloc_ptr[dev] && g_noalloc_ctx[dev] == id) {
    *out = g_noalloc_ptr[dev];
    return CG2D_OK;
  }
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) { cudaGetLastError(); return CG2D_CUDA_ERROR; }
  if (id == 0) id = current_ctx_id();   // the lookup made the device's primary context current
  g_noalloc_ptr[dev] = p;
  g_noalloc_ctx[dev] = id;
  *out = p;
  return CG2D_OK;
}

}  // namespace

extern "C" {

cg2d_status_t cg2d_solve_f64_noalloc(const cg2d_topology_t* topo, int batch, double cg2dNorm, const double* aW2d,
                                     const double* aS2d, const double* aC2d, const double* pW, const double* pS,
                                     const double* pC, const double* cg2d_b, const double* cg2d_x,
                                     double tolerance, int max_iters, double* x_out, double* x_fortran,
                                     cg2d_diag_t* diag, const cg2d_params_t* params, cg2d_stream_t stream) {
  cg2d_group_t g;
  std::memset(&g, 0, sizeof(g));
  g.topo = topo;
  g.count = batch;
  g.nrhs = 1;
  g.aW2d = aW2d; g.aS2d = aS2d; g.aC2d = aC2d; g.pW = pW; g.pS = pS; g.pC = pC;
  g.cg2dNorm = cg2dNorm;
  g.b[0] = cg2d_b;
  g.x0[0] = cg2d_x;
  g.x_out[0] = x_out;
  g.x_fortran[0] = x_fortran;
  g.diag[0] = diag;
  g.tolerance[0] = tolerance;
  g.max_iters[0] = max_iters;
  // the workspace this solve needs must fit the fixed array
  // phase profiles would be written into the hidden array, where no caller can read them back
  if (params && params->profile) return CG2D_BAD_ARG;
  const size_t need = cg2d_workspace_size(&g, 1, params);
  // arguments the solver rejects: the same status as cg2d_solve_f64 (the checks run before the workspace is used)
  if (need == 0) return cg2d_solve_groups(&g, 1, params, nullptr, 0, stream);
  if (need > (size_t)CG2D_NOALLOC_SCRATCH_BYTES) return CG2D_WORKSPACE_TOO_SMALL;
  void* ws = nullptr;
  const cg2d_status_t st = noalloc_scratch(&ws);
  if (st != CG2D_OK) return st;
  // the solve zeroes the part of the workspace that must start at zero (the grid-wait counter, the error word,
  // the rhsMax words) and writes everything else before reading it, so the previous call's contents do no harm
  return cg2d_solve_groups(&g, 1, params, ws, (size_t)CG2D_NOALLOC_SCRATCH_BYTES, stream);
}

}  // extern "C"
