// XLA FFI handlers over the SISL C ABI (include/sisl_b200.h): the jax.ffi
// binding of the reference's SISL calls.
//
// The reference (suetes/regional3d/steppers.py) is pure JAX; a maintainer
// who switches it to this library registers these handlers with
// jax.ffi.register_ffi_target(..., platform="CUDA") and calls them through
// jax.ffi.ffi_call (suetes_b200/jax_binding.py does both).  Each handler
// forwards XLA's device buffers and CUDA stream to one C-ABI entry point:
//
//   sisl_step           SISLStepper3D.step            steppers.py:720-1073
//   sisl_step_taped     the step keeping its two solves (jax.checkpoint
//                       residuals, steppers.py:792-850)
//   sisl_step_vjp       the step's VJP (custom_vjp backward rule)
//   sisl_gmres_solve    SemiImplicitSolver3D.solve    steppers.py:401-496
//   sisl_gmres_solve_t  its custom_linear_solve transpose, steppers.py:473-485
//   sisl_tricubic       tensor_product_interp_3d      operators.py:146-209
//   sisl_tricubic_vjp   its VJP w.r.t. the field
//
// The coefficient set (SislCore) is created once per (grid, dt, alpha,
// precision) on the Python side with sisl_core_create and passed as the
// 64-bit attribute "core"; an optional SislRelaxation is passed the same way
// ("relax", 0 for none).  Scratch memory is an extra output buffer of
// sisl_workspace_bytes() bytes that XLA allocates ("workspace", the last
// result), so nothing here allocates.  Buffers are x-fastest (the caller
// requests the column-major layout (0, 1, 2) for every 3-D operand).
//
// Build (needs jaxlib's FFI headers, absent from this repository's build
// image): make -C suetes_b200/csrc ffi  -- skipped when xla/ffi/api/ffi.h is
// not found under jax.ffi.include_dir().
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "sisl_b200.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

constexpr int kStateFields = 12;  // SislState: 7 prognostic + 5 history fields
constexpr int kSolveFields = 10;  // two solves x (u, v, w, pi_p, eta_dot)

ffi::Error status_error(int rc, const char* what) {
  if (rc >= 0) return ffi::Error::Success();  // SISL_NOT_CONVERGED keeps its outputs, as the reference does
  return ffi::Error(ffi::ErrorCode::kInternal, std::string(what) + ": " + sisl_status_string(rc));
}

// The 12 state fields of SislState in its member order, from `n` consecutive
// buffers starting at `first`.
template <typename Get>
SislState state_from(Get get, int first, double is_first_step) {
  void* p[kStateFields];
  for (int q = 0; q < kStateFields; ++q) p[q] = get(first + q);
  SislState s;
  s.u = p[0];
  s.v = p[1];
  s.w = p[2];
  s.eta_dot = p[3];
  s.pi_p = p[4];
  s.th_p = p[5];
  s.rho = p[6];
  s.u_prev = p[7];
  s.v_prev = p[8];
  s.w_prev = p[9];
  s.eta_dot_prev = p[10];
  s.tend_th_prev = p[11];
  s.is_first_step = is_first_step;
  return s;
}

ffi::Error StepImpl(cudaStream_t stream, uint64_t core, uint64_t relax, double is_first_step, int64_t taped,
                    ffi::RemainingArgs args, ffi::RemainingRets rets) {
  const int nsolve = taped ? kSolveFields : 0;
  if (args.size() != kStateFields || rets.size() != (size_t)(kStateFields + nsolve + 1))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "sisl_step: 12 state inputs, 12 (+10) outputs + workspace");
  auto in_ptr = [&](int q) { return args.get<ffi::AnyBuffer>(q).value().untyped_data(); };
  auto out_ptr = [&](int q) { return (*rets.get<ffi::AnyBuffer>(q).value()).untyped_data(); };
  SislState in = state_from(in_ptr, 0, is_first_step);
  SislState out = state_from(out_ptr, 0, 0.0);
  auto ws = *rets.get<ffi::AnyBuffer>(kStateFields + nsolve).value();
  void* solves[kSolveFields];
  for (int q = 0; q < nsolve; ++q) solves[q] = out_ptr(kStateFields + q);
  const SislRelaxation* rl = reinterpret_cast<const SislRelaxation*>(relax);
  SislCore* c = reinterpret_cast<SislCore*>(core);
  int rc = taped ? sisl_step_taped(c, &in, &out, rl, solves, ws.untyped_data(), ws.size_bytes(), stream, nullptr)
                 : sisl_step(c, &in, &out, rl, ws.untyped_data(), ws.size_bytes(), stream, nullptr);
  return status_error(rc, "sisl_step");
}

// inputs: state (12), solves (10), out_bar (12); outputs: in_bar (12), workspace
ffi::Error StepVjpImpl(cudaStream_t stream, uint64_t core, uint64_t relax, double is_first_step,
                       ffi::RemainingArgs args, ffi::RemainingRets rets) {
  if (args.size() != 2 * kStateFields + kSolveFields || rets.size() != kStateFields + 1)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "sisl_step_vjp: 34 inputs, 12 outputs + workspace");
  auto in_ptr = [&](int q) { return args.get<ffi::AnyBuffer>(q).value().untyped_data(); };
  auto out_ptr = [&](int q) { return (*rets.get<ffi::AnyBuffer>(q).value()).untyped_data(); };
  SislState in = state_from(in_ptr, 0, is_first_step);
  void* solves[kSolveFields];
  for (int q = 0; q < kSolveFields; ++q) solves[q] = in_ptr(kStateFields + q);
  SislState out_bar = state_from(in_ptr, kStateFields + kSolveFields, 0.0);
  SislState in_bar = state_from(out_ptr, 0, 0.0);
  auto ws = *rets.get<ffi::AnyBuffer>(kStateFields).value();
  int rc = sisl_step_vjp(reinterpret_cast<SislCore*>(core), &in, solves,
                         reinterpret_cast<const SislRelaxation*>(relax), &out_bar, &in_bar, ws.untyped_data(),
                         ws.size_bytes(), stream, nullptr);
  return status_error(rc, "sisl_step_vjp");
}

// inputs: rhs (5: u, v, w, pi_p, eta_dot); outputs: x (5), workspace.
// transpose = 1: the cotangent of the rhs from the cotangent of x.
ffi::Error SolveImpl(cudaStream_t stream, uint64_t core, int64_t transpose, ffi::RemainingArgs args,
                     ffi::RemainingRets rets) {
  if (args.size() != 5 || rets.size() != 6)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "sisl_gmres_solve: 5 inputs, 5 outputs + workspace");
  const void* b[5];
  void* x[5];
  for (int q = 0; q < 5; ++q) {
    b[q] = args.get<ffi::AnyBuffer>(q).value().untyped_data();
    x[q] = (*rets.get<ffi::AnyBuffer>(q).value()).untyped_data();
  }
  auto ws = *rets.get<ffi::AnyBuffer>(5).value();
  SislCore* c = reinterpret_cast<SislCore*>(core);
  int rc = transpose ? sisl_gmres_solve_transpose(c, b, nullptr, x, ws.untyped_data(), ws.size_bytes(), stream,
                                                  nullptr)
                     : sisl_gmres_solve(c, b, nullptr, x, ws.untyped_data(), ws.size_bytes(), stream, nullptr);
  return status_error(rc, "sisl_gmres_solve");
}

int dtype_code(ffi::DataType t) { return t == ffi::DataType::F64 ? SISL_F64 : SISL_F32; }

bool shape3(const ffi::AnyBuffer& b, int32_t out[3]) {
  auto dims = b.dimensions();
  if (dims.size() != 3) return false;
  for (int q = 0; q < 3; ++q) out[q] = (int32_t)dims[q];
  return true;
}

// inputs: field, cx, cy, cz (coordinate arrays of the output's shape); output: values
ffi::Error TricubicImpl(cudaStream_t stream, int64_t use_limiter, ffi::AnyBuffer field, ffi::AnyBuffer cx,
                        ffi::AnyBuffer cy, ffi::AnyBuffer cz, ffi::Result<ffi::AnyBuffer> out) {
  int32_t src[3], dst[3];
  if (!shape3(field, src) || !shape3(cx, dst))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "sisl_tricubic: 3-D field and coordinates");
  const void* coords[3] = {cx.untyped_data(), cy.untyped_data(), cz.untyped_data()};
  int rc = sisl_tricubic(dtype_code(field.element_type()), src, field.untyped_data(), dst, coords,
                         out->untyped_data(), (int)use_limiter, stream);
  return status_error(rc, "sisl_tricubic");
}

// inputs: field, cx, cy, cz, cot; output: grad (zeroed here, then accumulated)
ffi::Error TricubicVjpImpl(cudaStream_t stream, int64_t use_limiter, ffi::AnyBuffer field, ffi::AnyBuffer cx,
                           ffi::AnyBuffer cy, ffi::AnyBuffer cz, ffi::AnyBuffer cot,
                           ffi::Result<ffi::AnyBuffer> grad) {
  int32_t src[3], dst[3];
  if (!shape3(field, src) || !shape3(cx, dst))
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "sisl_tricubic_vjp: 3-D field and coordinates");
  if (cudaMemsetAsync(grad->untyped_data(), 0, grad->size_bytes(), stream) != cudaSuccess)
    return ffi::Error(ffi::ErrorCode::kInternal, "sisl_tricubic_vjp: clearing the gradient");
  const void* coords[3] = {cx.untyped_data(), cy.untyped_data(), cz.untyped_data()};
  int rc = sisl_tricubic_vjp(dtype_code(field.element_type()), src, field.untyped_data(), dst, coords,
                             cot.untyped_data(), grad->untyped_data(), (int)use_limiter, 1.0, stream);
  return status_error(rc, "sisl_tricubic_vjp");
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(SislStep, StepImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<uint64_t>("core")
                                  .Attr<uint64_t>("relax")
                                  .Attr<double>("is_first_step")
                                  .Attr<int64_t>("taped")
                                  .RemainingArgs()
                                  .RemainingRets());

XLA_FFI_DEFINE_HANDLER_SYMBOL(SislStepVjp, StepVjpImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<uint64_t>("core")
                                  .Attr<uint64_t>("relax")
                                  .Attr<double>("is_first_step")
                                  .RemainingArgs()
                                  .RemainingRets());

XLA_FFI_DEFINE_HANDLER_SYMBOL(SislGmresSolve, SolveImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<uint64_t>("core")
                                  .Attr<int64_t>("transpose")
                                  .RemainingArgs()
                                  .RemainingRets());

XLA_FFI_DEFINE_HANDLER_SYMBOL(SislTricubic, TricubicImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("use_limiter")
                                  .Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(SislTricubicVjp, TricubicVjpImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("use_limiter")
                                  .Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>());
