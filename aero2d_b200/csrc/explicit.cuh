// Launchers of the explicit RK4 + residual-smoothing kernels.
#pragma once
#include <cuda_runtime.h>

#include "batch.cuh"

namespace a2d {

// fp32: the explicit iteration's FP32 form (compute in FP32, values kept in the FP64 arrays)
void launch_local_dt(const Batch& b, const double* U, double* dt, double cfl, bool fp32, cudaStream_t s);
// one case's local time steps from primitives in the reference layout W[4][ni][nc] -> dt[ni][nc]
void launch_local_dt_prim(const GridDev& g, const double* W, double* dt, double cfl, cudaStream_t s);
// R (in) -> tmp (out, smoothed along i then j)
void launch_irs(const Batch& b, double* R, double* tmp, double e, int max_ni, int max_nc, bool fp32,
                cudaStream_t s);
void launch_rk_stage(const Batch& b, const double* U0, const double* R, const double* dt, double* U, double a,
                     bool fp32, cudaStream_t s);
void launch_rk_res(const Batch& b, const double* U0, const double* U, const double* dt, double* tpart,
                   cudaStream_t s);
void launch_rk_finish(const Batch& b, const double* tpart, const double* coef, double* res, double* circ,
                      cudaStream_t s);

// FAS multigrid transfers between a batch and its coarse batch (same cases, ni/2 x nc/2)
void launch_add_forcing(const Batch& b, double* R, const double* P, cudaStream_t s);
void launch_fas_restrict(const Batch& fine, const Batch& coarse, const double* Uf, double* Uc, double* Uc0,
                         cudaStream_t s);
void launch_fas_forcing(const Batch& fine, const Batch& coarse, const double* Rf, double* Pc, cudaStream_t s);
void launch_fas_prolong(const Batch& fine, const Batch& coarse, double* Uf, const double* Uc, const double* Uc0,
                        cudaStream_t s);

}  // namespace a2d
