// Argument blocks and launchers of the GMRES / Newton-update kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "batch.cuh"

namespace a2d {

struct CtlParams {
  double cfl0 = 10.0;
  double cfl_max = 300.0;
  double tol = 1e-8;
  int retire = 1;
};

template <typename TB>
struct CombineArgs {
  const double* x0 = nullptr;
  const TB* V = nullptr;
  size_t vstride = 0;
  const double* y = nullptr;
  const double* scale = nullptr;  // [q][case] scale of raw basis vector q
  const CaseCtl* ctl = nullptr;
  double* out = nullptr;
  uint32_t need = 0;
};

template <typename TB> void launch_combine(const Batch& b, const CombineArgs<TB>& a, cudaStream_t s);
void launch_lstsq(const Batch& b, const uint32_t* live, CaseCtl* ctl, double* H, double* y, cudaStream_t s);
void launch_gm_setup(const Batch& b, const double* part, int pstride, CaseCtl* ctl, double gtol,
                     cudaStream_t s);
void launch_norms2(const Batch& b, const double* x, const double* y, double* part, int pstride,
                   uint32_t need, cudaStream_t s);
void launch_norm1(const Batch& b, const double* x, double* part, uint32_t need, cudaStream_t s);
void launch_update_rel(const Batch& b, const double* U, const double* dU, double* tpart, uint32_t need,
                       cudaStream_t s);
void launch_update_check(const Batch& b, const double* U, const double* dU, double* tpart, CaseCtl* ctl,
                         double max_update, uint32_t need, cudaStream_t s);
void launch_controller(const Batch& b, const double* tpart, CaseCtl* ctl, uint32_t* live, double* hist_rn,
                       int hist_cap, const CtlParams& p, cudaStream_t s);
void launch_commit(const Batch& b, double* U, const double* dU, const CaseCtl* ctl, cudaStream_t s);
void launch_mark_stepped(const Batch& b, const uint32_t* live, CaseCtl* ctl, cudaStream_t s);

}  // namespace a2d
