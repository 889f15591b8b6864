// Launcher declarations and argument blocks of the Euler-path kernels.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "batch.cuh"

namespace a2d {

// Storage type of the sweep factors (G, C, P, Q) for a Jacobian type: the
// mixed-precision path keeps them in FP16 (they are products with the pivot
// inverse, so their entries are O(1)); the pivot inverses stay in the Jacobian
// type.  The factors only steer GMRES: the Newton residual stays FP64.
template <typename TJ> struct FactorStore { using type = TJ; };
template <> struct FactorStore<float> { using type = __half; };

__device__ __forceinline__ double to_f64(float v) { return v; }
__device__ __forceinline__ double to_f64(double v) { return v; }
__device__ __forceinline__ double to_f64(__half v) { return (double)__half2float(v); }

template <typename T> __device__ __forceinline__ T from_f64(double v) { return T(v); }
// saturating: an entry beyond the FP16 range is stored as +-65504, never as inf
template <> __device__ __forceinline__ __half from_f64<__half>(double v) {
  const float f = (float)v;
  return __float2half_rn(fminf(fmaxf(f, -65504.0f), 65504.0f));
}

// 1 when a factor entry lies outside the storage type's finite range, i.e. the
// FP16 store above saturates it (or it is not finite); never for FP32/FP64 storage
template <typename TF> __device__ __forceinline__ unsigned out_of_range(double) { return 0u; }
template <> __device__ __forceinline__ unsigned out_of_range<__half>(double v) {
  return (fabs(v) <= 65504.0) ? 0u : 1u;
}

template <typename VT>
struct StencilArgs {
  const double* U = nullptr;       // conserved state (FP64), packed cell vectors
  const VT* V = nullptr;           // tangent direction (linearised mode)
  const double* vscale = nullptr;  // per-case factor applied to V (a raw Krylov vector's 1/norm)
  const double* circ_in = nullptr; // per-case circulation; nullptr: Gamma(U) from the wall rows
  const double* diag = nullptr;    // per-cell vol / dtau (linearised mode; nullptr: J v alone)
  const double* bvec = nullptr;    // linearised mode: out = b - (diag v + J v) when set
  double* out = nullptr;
  double sign = 1.0;               // residual mode: out = sign * R
  double* circ_out = nullptr;      // residual mode: per-case circulation used
  double* tile_part = nullptr;     // residual mode: per-tile sum of (R_rho / vol)^2
  double lim_k = 0.02;
  int order = 2;
  int vortex = 1;
  uint32_t need = 0;               // status bits a case needs to be processed
};

struct JacArgs {
  const double* U = nullptr;
  const double* circ = nullptr;    // per-case circulation (held fixed in the far-field block)
  void* JIL = nullptr;             // i-face blocks dF/dU_left  [rows nc]
  void* JIR = nullptr;             // i-face blocks dF/dU_right [rows nc]
  void* JJL = nullptr;             // j-face blocks dF/dU_low   [rows nc+1] (row nc: far field)
  void* JJR = nullptr;             // j-face blocks dF/dU_high  [rows nc+1] (row 0: wall)
  int vortex = 1;
  uint32_t need = 0;
};

struct FactorArgs {
  const double* U = nullptr;
  const CaseCtl* ctl = nullptr;    // per-case pseudo-time CFL
  const void* JIL = nullptr;
  const void* JIR = nullptr;
  const void* JJL = nullptr;
  const void* JJR = nullptr;
  void* INV = nullptr;             // inverse of the block-Thomas pivots [rows nc]
  void* CF = nullptr;              // upper factors c_j                 [rows nc]
  void* PQG = nullptr;             // per row: P = inv_j JIL(i) (coupling to line i-1),
                                   // Q = inv_j JIR(i+1) (to line i+1), G = -inv_j A_j  [rows nc]
  double* diag = nullptr;          // per-cell vol / dtau
  double cfl_base = 2.5;           // EulerSolver.cfl, which local_dt multiplies and step() divides out
  unsigned long long* sat = nullptr; // counts factor entries saturated by the FP16 store
  uint32_t need = 0;
};

// One line-Jacobi sweep x = M_line^-1 (r - off(xprev)), with the factors of
// k_factor.  The first sweep (no previous iterate) computes e0 = inv r and may
// keep it for the later sweeps, whose right-hand side is e0 + P xprev[i-1] -
// Q xprev[i+1].  All vectors are cell vectors [4][nc][ni]; r and the result of
// the last sweep are FP64, the intermediate ones (e0, xprev, x of the other
// sweeps) hold entries of the sweep's vector type (FP32 in the mixed path,
// packed at the start of the buffer).
struct SweepArgs {
  const double* r = nullptr;       // first sweep: right-hand side
  double* e0 = nullptr;            // first sweep: inv r written when set; later sweeps: read
  const double* xprev = nullptr;   // later sweeps: previous iterate (must not alias x)
  double* x = nullptr;             // result (the first sweep may write it over r)
  double* dtmp = nullptr;          // last sweep: scratch for the forward values d_j
  const void* INV = nullptr;
  const void* PQG = nullptr;       // P, Q, G blocks interleaved per row (fbidx3)
  const void* CF = nullptr;
  uint32_t* err = nullptr;         // set to 1 when a copy wait runs out of time
  uint32_t need = 0;
};

void launch_metrics(int ni, int nc, const double* x, const double* y, double* md, float* mf,
                    cudaStream_t s);

// shape: the tile shape of b's tile list (kTile*; only the FP32 linearised
// stencil has shapes other than kTile32x8)
template <typename T, bool LIN, typename VT>
void launch_stencil(const Batch& b, const StencilArgs<VT>& a, cudaStream_t s, int shape = kTile32x8);
// resident-CTA queries of the persistent stencil launches (host, before any capture)
void stencil_init_fp64();
void stencil_init_fp32();

void launch_forces(const Batch& b, const double* U, double* coef, double* cp, const long long* cp_off,
                   const CaseCtl* ctl, double* hist_cl, int hist_cap, cudaStream_t s);

template <typename T>
void launch_face_jac(const Batch& b, const JacArgs& a, cudaStream_t s);

template <typename TJ, typename TF>
void launch_factor(const Batch& b, const FactorArgs& a, cudaStream_t s);

// kernel variants of the line-Jacobi sweep, a plan's tuning knob, by warps per
// half line group: one, a lane solving all four block rows of its line
// (sweep.cu); two, two lanes per line with two block rows each (sweep_pairs.cu);
// four, a warp per block row (sweep_rows.cu)
enum : int { kSweepLanes = 0, kSweepRows = 1, kSweepPairs = 2, kSweepHalves = 3, kNumSweepVariants = 4 };

// one line-Jacobi sweep; FIRST: the sweep without i-coupling; last: x is the
// FP64 result (else an intermediate vector).  Every variant computes the same
// arithmetic in the same order
template <typename TI, bool FIRST>
void launch_sweep(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s, int variant = kSweepLanes);
template <typename TI, bool FIRST>
void launch_sweep_rows(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s);
template <typename TI, bool FIRST>
void launch_sweep_pairs(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s);
template <bool FIRST>   // mixed precision only
void launch_sweep_halves(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s);

// raises the dynamic shared-memory limit of the sweep kernels (host, once per device)
cudaError_t sweep_init();
cudaError_t sweep_rows_init();
cudaError_t sweep_pairs_init();
cudaError_t sweep_halves_init();

}  // namespace a2d
