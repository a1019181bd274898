// XLA FFI handlers: the C ABI's residual, J.v and Newton block as jax.ffi custom calls, so
// that a JAX program (the reference's own driver, src/jaxrans/solvers/driver.py:87-105,
// which fuses block_iters Newton steps into one jitted device call) can hand the hot path
// to this library on XLA's stream.  The reference has no FFI; these targets stand in for
// make_residual(...).residual (src/jaxrans/numerics/residual.py:273-334), the jvp of
// jax.linearize(jacobian_source.residual, U) (src/jaxrans/solvers/implicit.py:104-116) and
// the driver's block of Newton steps.
//
// Built only where JAX's FFI headers are present (jaxrans_b200.build.build_ffi); the
// library (libjaxrans_b200.so) is linked in.  The plan (jr_plan_create) stays owned by the
// caller and is passed as an int64 attribute; XLA owns every buffer.  Each handler first
// points the plan at XLA's stream for the call (jr_plan_set_stream, a no-op when it is
// already that stream), so the work orders with XLA's own kernels and nothing synchronises.
#include <cmath>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "jaxrans_b200.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error failed(const char* what) {
  return ffi::Error(ffi::ErrorCode::kInternal, std::string(what) + ": " + jr_last_error());
}

ffi::Error bad(const std::string& what) { return ffi::Error(ffi::ErrorCode::kInvalidArgument, what); }

// The plan behind an attribute, set to run on `stream`; checks that a field buffer of
// `count` doubles is the plan's whole state (nvar x every case's canvas).
ffi::Error bind_plan(int64_t handle, cudaStream_t stream, size_t count, jr_plan** out) {
  jr_plan* plan = reinterpret_cast<jr_plan*>(handle);
  if (plan == nullptr) return bad("the plan attribute is null");
  int64_t n_canvas = 0;
  if (jr_plan_sizes(plan, &n_canvas, nullptr) != JR_OK) return failed("jr_plan_sizes");
  if (n_canvas <= 0 || count % (size_t)n_canvas != 0 || (count / n_canvas != 4 && count / n_canvas != 5))
    return bad("a field buffer must hold nvar x " + std::to_string(n_canvas) + " doubles (nvar 4 or 5)");
  if (jr_plan_set_stream(plan, stream) != JR_OK) return failed("jr_plan_set_stream");
  *out = plan;
  return ffi::Error::Success();
}

ffi::Error Residual(cudaStream_t stream, int64_t plan_handle, int32_t first_order, ffi::Buffer<ffi::F64> U,
                    ffi::ResultBuffer<ffi::F64> R) {
  if (U.element_count() != R->element_count()) return bad("U and R differ in size");
  jr_plan* plan = nullptr;
  ffi::Error e = bind_plan(plan_handle, stream, U.element_count(), &plan);
  if (e.failure()) return e;
  if (jr_residual(plan, U.typed_data(), R->typed_data(), first_order) != JR_OK) return failed("jr_residual");
  return ffi::Error::Success();
}

ffi::Error Jvp(cudaStream_t stream, int64_t plan_handle, ffi::Buffer<ffi::F64> U, ffi::Buffer<ffi::F64> v,
               ffi::ResultBuffer<ffi::F64> Jv) {
  if (U.element_count() != v.element_count() || U.element_count() != Jv->element_count())
    return bad("U, v and Jv differ in size");
  jr_plan* plan = nullptr;
  ffi::Error e = bind_plan(plan_handle, stream, U.element_count(), &plan);
  if (e.failure()) return e;
  if (jr_jvp(plan, U.typed_data(), v.typed_data(), Jv->typed_data()) != JR_OK) return failed("jr_jvp");
  return ffi::Error::Success();
}

// n_steps Newton steps from U_in: restart != 0 starts every case at (U_in, cfl, |R| = inf);
// otherwise the plan's CFL and |R| carry on from its last block and only U is replaced.
// U_out receives the state after the steps, history the |R| of every case before each
// step (n_steps x cases, step-major).
ffi::Error NewtonBlock(cudaStream_t stream, int64_t plan_handle, int32_t n_steps, int32_t restart, double cfl,
                       ffi::Buffer<ffi::F64> U_in, ffi::ResultBuffer<ffi::F64> U_out,
                       ffi::ResultBuffer<ffi::F64> history) {
  if (U_in.element_count() != U_out->element_count()) return bad("U_in and U_out differ in size");
  jr_plan* plan = nullptr;
  ffi::Error e = bind_plan(plan_handle, stream, U_in.element_count(), &plan);
  if (e.failure()) return e;
  if (n_steps < 1 || history->element_count() != (size_t)n_steps * (size_t)jr_plan_cases(plan))
    return bad("history must hold n_steps x cases doubles, n_steps >= 1");
  const size_t bytes = U_in.element_count() * sizeof(double);
  if (restart != 0) {
    if (jr_state_set_device(plan, U_in.typed_data(), cfl, INFINITY) != JR_OK) return failed("jr_state_set_device");
  } else if (cudaMemcpyAsync(jr_state_device(plan), U_in.typed_data(), bytes, cudaMemcpyDeviceToDevice, stream) !=
             cudaSuccess) {
    return bad("the state copy failed");
  }
  if (jr_newton_steps_async(plan, n_steps, history->typed_data()) != JR_OK) return failed("jr_newton_steps_async");
  if (cudaMemcpyAsync(U_out->typed_data(), jr_state_device(plan), bytes, cudaMemcpyDeviceToDevice, stream) !=
      cudaSuccess)
    return bad("the state copy failed");
  return ffi::Error::Success();
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(JrResidual, Residual,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("plan")
                                  .Attr<int32_t>("first_order")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(JrJvp, Jvp,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("plan")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(JrNewtonBlock, NewtonBlock,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("plan")
                                  .Attr<int32_t>("n_steps")
                                  .Attr<int32_t>("restart")
                                  .Attr<double>("cfl")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>());
