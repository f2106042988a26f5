// XLA FFI handlers over the C ABI of libcg2d.so: the jax.ffi custom calls behind mit_jax_b200.jax_ffi.
//
// Built only where jaxlib's FFI headers exist (jax.ffi.include_dir()); it needs no CUDA compiler:
//   g++ -std=c++17 -O2 -shared -fPIC -I<jax.ffi.include_dir()> -I<cuda>/include -I<repo>/include \
//       cg2d_ffi.cc -L<package dir> -lcg2d -Wl,-rpath,'$ORIGIN' -o libcg2d_ffi.so
//
// Handlers (every buffer is float64 in the reference layout [batch][T][ny][nx] unless stated; the batch is the
// buffer's element count over T ny nx, so a leading vmap dimension is a batch):
//   cg2d_b200_solve    cg2d_fortran (mitgcm_jax/core/cg2d.py:205-269), the literal CG forward of
//                      _cg2d_implicit (cg2d.py:307-315): args aW2d aS2d aC2d pW pS pC cg2d_b cg2d_x cg2dNorm[batch];
//                      results x (interior solution, 0 on halos), x_fortran (cg2d_fortran's array), diag u8[batch][48]
//                      (cg2d_diag_t); attrs topo (cg2d_topology_t* as int64), tolerance, max_iters, precision
//                      (0 FP64, 1 mixed), sum_order (0 ROWBLOCK, 1 FORTRAN).
//   cg2d_b200_adjoint  the transpose of the implicit derivative (_cg2d_implicit_jvp, cg2d.py:318-348): args aW2d
//                      aS2d aC2d pW pS pC x x_bar cg2dNorm[batch]; results lam (= the cotangent of cg2d_b), gW, gS, gC (the
//                      coefficient cotangents, 0 when coeff_grad is 0: the reference's stop_coeff_grad), diag; attrs
//                      topo, adj_tolerance, adj_max_iters, coeff_grad.
// The workspace comes from XLA's scratch allocator; a failed allocation or a status other than CG2D_OK is an FFI
// error. Per-solve outcomes (convergence, NaN) are in diag, as in the reference, where non-convergence is not an
// error.

#include <cuda_runtime_api.h>

#include <cstdint>
#include <optional>
#include <string>

#include "cg2d.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

constexpr size_t kAlign = 256;

ffi::Error status_error(cg2d_status_t st, const char* where) {
  if (st == CG2D_OK) return ffi::Error::Success();
  const ffi::ErrorCode code = (st == CG2D_BAD_ARG || st == CG2D_UNSUPPORTED) ? ffi::ErrorCode::kInvalidArgument
                              : st == CG2D_WORKSPACE_TOO_SMALL              ? ffi::ErrorCode::kResourceExhausted
                                                                            : ffi::ErrorCode::kInternal;
  return ffi::Error(code, std::string(where) + ": " + cg2d_status_string(st));
}

// instances in a buffer of [batch][T][ny][nx]; 0 when the size is not a whole number of instances
int64_t batch_of(size_t elements, int64_t per) { return (per > 0 && elements % per == 0) ? (int64_t)(elements / per) : 0; }

// scratch of `bytes`, 256-byte aligned
std::optional<void*> workspace(ffi::ScratchAllocator& scratch, size_t bytes) {
  auto p = scratch.Allocate(bytes + kAlign, kAlign);
  if (!p.has_value()) return std::nullopt;
  const uintptr_t a = (reinterpret_cast<uintptr_t>(*p) + kAlign - 1) & ~uintptr_t(kAlign - 1);
  return reinterpret_cast<void*>(a);
}

ffi::Error SolveImpl(cudaStream_t stream, ffi::ScratchAllocator scratch, ffi::Buffer<ffi::F64> aW,
                     ffi::Buffer<ffi::F64> aS, ffi::Buffer<ffi::F64> aC, ffi::Buffer<ffi::F64> pW,
                     ffi::Buffer<ffi::F64> pS, ffi::Buffer<ffi::F64> pC, ffi::Buffer<ffi::F64> b,
                     ffi::Buffer<ffi::F64> x0, ffi::Buffer<ffi::F64> norm, ffi::ResultBuffer<ffi::F64> x,
                     ffi::ResultBuffer<ffi::F64> x_fortran, ffi::ResultBuffer<ffi::U8> diag, int64_t topo,
                     double tolerance, int32_t max_iters, int32_t precision, int32_t sum_order, int64_t per_instance) {
  const int64_t batch = batch_of(b.element_count(), per_instance);
  if (batch < 1 || batch > 65535) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "cg2d_b200_solve: batch");
  if (diag->size_bytes() != (size_t)batch * sizeof(cg2d_diag_t))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "cg2d_b200_solve: diag size");
  // cg2dNorm per instance, on the device (the caller broadcasts one value to the batch)
  if (norm.element_count() != (size_t)batch)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "cg2d_b200_solve: cg2dNorm size");
  cg2d_params_t p;
  cg2d_default_params(&p);
  p.precision = precision;
  p.sum_order = sum_order;
  cg2d_group_t g = {};
  g.topo = reinterpret_cast<const cg2d_topology_t*>(topo);
  g.count = (int)batch;
  g.nrhs = 1;
  g.aW2d = aW.typed_data(); g.aS2d = aS.typed_data(); g.aC2d = aC.typed_data();
  g.pW = pW.typed_data(); g.pS = pS.typed_data(); g.pC = pC.typed_data();
  g.cg2dNorm = 0.0;
  g.cg2dNorm_per_instance = norm.typed_data();
  g.b[0] = b.typed_data();
  g.x0[0] = x0.typed_data();
  g.x_out[0] = x->typed_data();
  g.x_fortran[0] = x_fortran->typed_data();
  g.diag[0] = reinterpret_cast<cg2d_diag_t*>(diag->typed_data());
  g.tolerance[0] = tolerance;
  g.max_iters[0] = max_iters;
  const size_t bytes = cg2d_workspace_size(&g, 1, &p);
  if (bytes == 0) return status_error(cg2d_solve_groups(&g, 1, &p, nullptr, 0, stream), "cg2d_b200_solve");
  auto ws = workspace(scratch, bytes);
  if (!ws) return ffi::Error(ffi::ErrorCode::kResourceExhausted, "cg2d_b200_solve: workspace");
  return status_error(cg2d_solve_groups(&g, 1, &p, *ws, bytes, stream), "cg2d_b200_solve");
}

ffi::Error AdjointImpl(cudaStream_t stream, ffi::ScratchAllocator scratch, ffi::Buffer<ffi::F64> aW,
                       ffi::Buffer<ffi::F64> aS, ffi::Buffer<ffi::F64> aC, ffi::Buffer<ffi::F64> pW,
                       ffi::Buffer<ffi::F64> pS, ffi::Buffer<ffi::F64> pC, ffi::Buffer<ffi::F64> xs,
                       ffi::Buffer<ffi::F64> xbar, ffi::Buffer<ffi::F64> norm, ffi::ResultBuffer<ffi::F64> lam,
                       ffi::ResultBuffer<ffi::F64> gW, ffi::ResultBuffer<ffi::F64> gS, ffi::ResultBuffer<ffi::F64> gC,
                       ffi::ResultBuffer<ffi::U8> diag, int64_t topo, double adj_tolerance, int32_t adj_max_iters,
                       int32_t coeff_grad, int64_t per_instance) {
  const int64_t batch = batch_of(xbar.element_count(), per_instance);
  if (batch < 1 || batch > 65535) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "cg2d_b200_adjoint: batch");
  if (diag->size_bytes() != (size_t)batch * sizeof(cg2d_diag_t))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "cg2d_b200_adjoint: diag size");
  if (norm.element_count() != (size_t)batch)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "cg2d_b200_adjoint: cg2dNorm size");
  cg2d_params_t p;
  cg2d_default_params(&p);
  const cg2d_topology_t* tp = reinterpret_cast<const cg2d_topology_t*>(topo);
  const size_t bytes = cg2d_adjoint_ecco_workspace_size(tp, (int)batch, adj_max_iters, &p);
  if (bytes == 0) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "cg2d_b200_adjoint: arguments");
  auto ws = workspace(scratch, bytes);
  if (!ws) return ffi::Error(ffi::ErrorCode::kResourceExhausted, "cg2d_b200_adjoint: workspace");
  return status_error(
      cg2d_adjoint_ecco(tp, (int)batch, 0.0, norm.typed_data(), aW.typed_data(), aS.typed_data(), aC.typed_data(),
                        pW.typed_data(), pS.typed_data(), pC.typed_data(), xs.typed_data(), xbar.typed_data(),
                        adj_tolerance, adj_max_iters, coeff_grad, lam->typed_data(), gW->typed_data(),
                        gS->typed_data(), gC->typed_data(), reinterpret_cast<cg2d_diag_t*>(diag->typed_data()), &p,
                        *ws, bytes, stream),
      "cg2d_b200_adjoint");
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(cg2d_b200_solve, SolveImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Ctx<ffi::ScratchAllocator>()
                                  .Arg<ffi::Buffer<ffi::F64>>()   // aW2d
                                  .Arg<ffi::Buffer<ffi::F64>>()   // aS2d
                                  .Arg<ffi::Buffer<ffi::F64>>()   // aC2d
                                  .Arg<ffi::Buffer<ffi::F64>>()   // pW
                                  .Arg<ffi::Buffer<ffi::F64>>()   // pS
                                  .Arg<ffi::Buffer<ffi::F64>>()   // pC
                                  .Arg<ffi::Buffer<ffi::F64>>()   // cg2d_b
                                  .Arg<ffi::Buffer<ffi::F64>>()   // cg2d_x
                                  .Arg<ffi::Buffer<ffi::F64>>()   // cg2dNorm [batch]
                                  .Ret<ffi::Buffer<ffi::F64>>()   // x
                                  .Ret<ffi::Buffer<ffi::F64>>()   // x_fortran
                                  .Ret<ffi::Buffer<ffi::U8>>()    // diag
                                  .Attr<int64_t>("topo")
                                  .Attr<double>("tolerance")
                                  .Attr<int32_t>("max_iters")
                                  .Attr<int32_t>("precision")
                                  .Attr<int32_t>("sum_order")
                                  .Attr<int64_t>("per_instance"));

XLA_FFI_DEFINE_HANDLER_SYMBOL(cg2d_b200_adjoint, AdjointImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Ctx<ffi::ScratchAllocator>()
                                  .Arg<ffi::Buffer<ffi::F64>>()   // aW2d
                                  .Arg<ffi::Buffer<ffi::F64>>()   // aS2d
                                  .Arg<ffi::Buffer<ffi::F64>>()   // aC2d
                                  .Arg<ffi::Buffer<ffi::F64>>()   // pW
                                  .Arg<ffi::Buffer<ffi::F64>>()   // pS
                                  .Arg<ffi::Buffer<ffi::F64>>()   // pC
                                  .Arg<ffi::Buffer<ffi::F64>>()   // x (forward solution)
                                  .Arg<ffi::Buffer<ffi::F64>>()   // x_bar
                                  .Arg<ffi::Buffer<ffi::F64>>()   // cg2dNorm [batch]
                                  .Ret<ffi::Buffer<ffi::F64>>()   // lam
                                  .Ret<ffi::Buffer<ffi::F64>>()   // gW
                                  .Ret<ffi::Buffer<ffi::F64>>()   // gS
                                  .Ret<ffi::Buffer<ffi::F64>>()   // gC
                                  .Ret<ffi::Buffer<ffi::U8>>()    // diag
                                  .Attr<int64_t>("topo")
                                  .Attr<double>("adj_tolerance")
                                  .Attr<int32_t>("adj_max_iters")
                                  .Attr<int32_t>("coeff_grad")
                                  .Attr<int64_t>("per_instance"));
