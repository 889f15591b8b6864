// FP32 instantiations of the residual / JVP tile kernel (stencil_impl.cuh):
// the linearised residual of the mixed-precision Newton-Krylov solver.  This
// translation unit is compiled with approximate FP32 division and square root
// and flush-to-zero (see aero2d_b200/build.py); in the mixed mode the FP32
// product only defines the Krylov operator, while the FP64 residual on the
// right-hand side fixes the converged solution, so FP32 operations a couple of
// ulp off round-to-nearest are immaterial to the result.
#include <cuda_bf16.h>

#include "stencil_impl.cuh"

namespace a2d {

template void launch_stencil<float, false, double>(const Batch&, const StencilArgs<double>&, cudaStream_t, int);
template void launch_stencil<float, true, double>(const Batch&, const StencilArgs<double>&, cudaStream_t, int);
template void launch_stencil<float, true, float>(const Batch&, const StencilArgs<float>&, cudaStream_t, int);
template void launch_stencil<float, true, __nv_bfloat16>(const Batch&, const StencilArgs<__nv_bfloat16>&,
                                                         cudaStream_t, int);


template <typename VT>
static void caps_of() {
  stencil_cap<float, true, VT, kTI, kTJ>();
  stencil_cap<float, true, VT, 32, 16>();
  stencil_cap<float, true, VT, 64, 4>();
  stencil_cap<float, true, VT, 16, 16>();
}

void stencil_init_fp32() {
  stencil_cap<float, false, double, kTI, kTJ>();
  caps_of<double>();
  caps_of<float>();
  caps_of<__nv_bfloat16>();
}

}  // namespace a2d
