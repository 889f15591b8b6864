// Argument blocks and launchers of the Gram-Schmidt kernels (gs.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "batch.cuh"

namespace a2d {

constexpr int kHStride = kMaxRestart + 2;   // per-case stride of coefficient arrays
constexpr int kGsSlice = 32;                // basis vectors one pass handles (more: chained slices)

template <typename TB>
struct GsArgs {
  const double* w = nullptr;      // vector being orthogonalised
  const TB* V = nullptr;          // raw basis, vector q at V + q * vstride
  size_t vstride = 0;
  int nq = 0;                     // basis vectors taken
  int q0 = 0;                     // first vector of the slice (set by the launchers)
  int with_norm = 0;              // pass 1: also w . w
  int norm_slot = 0;              // partial slot of w . w (set by the launchers)
  double* part = nullptr;         // per-chunk partials [chunk][pstride]
  int pstride = 0;
  const double* h1 = nullptr;     // [case][kHStride] coefficients of pass 1
  const double* h2 = nullptr;     // [case][kHStride] coefficients of pass 2
  const double* scale = nullptr;  // [q][case] scale of raw basis vector q
  int both = 0;                   // subtraction uses h1 + h2
  TB* Vout = nullptr;             // pass 3 / start: raw basis vector written
  double* wout = nullptr;         // subtraction result kept in FP64 (chained path)
  double* tmp = nullptr;          // scratch vector of the chained path (more than 32 vectors)
  double* part_norm = nullptr;    // per-chunk squared norm of the result
  uint32_t* err = nullptr;        // set to 1 when a bulk-copy wait runs out of time
  uint32_t need = 0;
  // Folded per-case reduction (one slice, nq <= 32): when fold_part is set, every CTA
  // reduces its case's chunk partials fold_part[chunk][q] itself (the order of
  // k_gs_reduce) into this pass's coefficients, h_q = scale_q * sum, while its first
  // bulk copies are in flight; the case's first chunk also stores h in fold_h (and, with
  // fold_wn0, the norm of w from the partials' slot nq).  project: the coefficients are
  // h1; sub (both): h1 from h1 plus the folded h2.
  const double* fold_part = nullptr;
  double* fold_h = nullptr;
  double* fold_wn0 = nullptr;
};

struct GsReduceArgs {
  const double* part = nullptr;
  int pstride = 0;
  int nq = 0;
  const double* scale = nullptr;  // [q][case]
  double* h = nullptr;            // [case][kHStride]
  double* wn0 = nullptr;          // if set: sqrt of slot nq (norm of w before orthogonalisation)
  uint32_t need = 0;
};

struct GsCloseArgs {
  const double* part_norm = nullptr;
  const double* wn0 = nullptr;
  const double* h1 = nullptr;
  const double* h2 = nullptr;
  double* H = nullptr;            // [case][kMaxRestart][kMaxRestart+1], column k = step k
  double* scale = nullptr;        // [q][case]; k = -1 writes row 0
  CaseCtl* ctl = nullptr;
  uint32_t* live = nullptr;
  int k = -1;
  uint32_t need = 0;
};

template <typename TB> void launch_gs_dots(const Batch& b, const GsArgs<TB>& a, cudaStream_t s);
void launch_gs_reduce(const Batch& b, const GsReduceArgs& a, cudaStream_t s);
template <typename TB> void launch_gs_project(const Batch& b, const GsArgs<TB>& a, cudaStream_t s);
template <typename TB> void launch_gs_finish(const Batch& b, const GsArgs<TB>& a, cudaStream_t s);
template <typename TB> void launch_gs_start(const Batch& b, const GsArgs<TB>& a, cudaStream_t s);
void launch_gs_close(const Batch& b, const GsCloseArgs& a, cudaStream_t s);
// raises the dynamic shared-memory limit of the streaming passes (host, once per device)
cudaError_t gs_init();

}  // namespace a2d
