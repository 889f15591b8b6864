// Host runtime of the Euler path: batch plans, workspace layout, the
// pseudo-transient Newton step as a sequence of kernels (replayed as one CUDA
// graph), the explicit RK iteration, and the extern "C" entry points declared
// in include/aero2d_b200.h.
//
// A plan owns no device memory: every device array lives in the caller's
// workspace, carved at bind time.  The Newton loop's per-case bookkeeping
// (rollback, freeze, SER CFL, convergence test, aero2d/implicit.py:216-244)
// runs on the device, so the host synchronises once per step only to learn
// whether any case is still live.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "aero2d_b200.h"
#include "batch.cuh"
#include "explicit.cuh"
#include "kernels.cuh"

#include <nvtx3/nvToolsExt.h>
#include "gs.cuh"
#include "krylov.cuh"
#include "physics.cuh"

namespace a2d {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define A2D_CK(call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(A2D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
  } while (0)

struct Carve {
  size_t off = 0;
  size_t take(size_t bytes) {
    off = (off + 255) & ~size_t(255);
    const size_t o = off;
    off += bytes;
    return o;
  }
};

static size_t metrics_total_bytes(int ni, int nc) {
  return metrics_float_offset(ni, nc) + metrics_floats(ni, nc) * 4;
}

// Krylov basis storage of the mixed path: BF16 (the basis is the raw,
// unnormalised Arnoldi vectors with FP64 scales; Gram-Schmidt, the Hessenberg
// matrix and the update are FP64)
using Basis16 = __nv_bfloat16;

enum VecSlot { kU = 0, kR, kVin, kJV, kDU, kB, kX0, kT, kRr, kZ, kW, kPA, kPB, kU0, kPE, kPD, kNumVec };

}  // namespace a2d

using namespace a2d;

struct a2d_plan {
  a2d_params p{};
  int ncases = 0;
  int m = 0;               // GMRES restart
  int max_ni = 0, max_nc = 0;
  std::vector<CaseDev> cases;
  std::vector<Tile> tiles;
  std::vector<Tile> jtiles;    // tiles of the FP32 linearised stencil, in the shape jvp_tile
  // tuning knobs (a2d_plan_set_tuning); the defaults are the fastest measured on a B200 on
  // the batch shapes timed (64, 4 x 16 and 8 cases of 256 x 64); FP64 plans start with the
  // lanes sweep
  int jvp_tile = kTile32x16;
  int sweep_variant = kSweepHalves;
  int max_jtiles = 0;          // the most tiles any JVP tile shape needs (workspace room)
  std::vector<Chunk> chunks;
  std::vector<Group> groups;
  std::vector<long long> cp_off;
  long long C = 0, rows_nc = 0, rows_nc1 = 0, total_ni = 0;
  size_t tj = 8, tb = 8;   // bytes of face-Jacobian and basis storage entries
  size_t tf = 8;           // bytes of the sweep factor entries (G, C, P, Q)
  // workspace layout (offsets)
  size_t o_cases = 0, o_tiles = 0, o_chunks = 0, o_groups = 0, o_cpoff = 0, o_live = 0, o_ctl = 0;
  size_t o_vec[kNumVec] = {};
  size_t o_diag = 0, o_dt = 0, o_JIL = 0, o_JIR = 0, o_JJL = 0, o_JJR = 0, o_INV = 0, o_CF = 0, o_PQG = 0, o_V = 0;
  size_t o_H = 0, o_h1 = 0, o_h2 = 0, o_scale = 0, o_y = 0, o_wn0 = 0, o_circ = 0, o_circ_rk = 0;
  size_t o_tpart = 0, o_cpart = 0, o_cpart2 = 0, o_cpartn = 0, o_coef = 0, o_cp = 0, o_hrn = 0, o_hcl = 0,
         o_cnt = 0, o_idx = 0;
  size_t o_sat = 0;        // saturated FP16 factor entries since bind (a2d_factor_saturations)
  size_t o_jtiles = 0;
  Batch jbatch{};          // the batch with the JVP's tile list
  int pstride = 0;
  size_t bytes = 0;
  char* ws = nullptr;
  Batch batch{};
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  int* host_count = nullptr;
  int steps_taken = 0;
  int kernels_per_step = 0;
  a2d_plan* coarse = nullptr;   // FAS multigrid: the same cases on grids of every other node

  template <typename X> X* at(size_t off) const { return reinterpret_cast<X*>(ws + off); }
  double* vec(int s) const { return at<double>(o_vec[s]); }
  CaseCtl* ctl() const { return at<CaseCtl>(o_ctl); }
  uint32_t* live() const { return at<uint32_t>(o_live); }
};

namespace a2d {

// ---------------------------------------------------------------------------
// plan construction
// ---------------------------------------------------------------------------
// tiles of every case in the given shape, case after case
static std::vector<Tile> tile_list(const a2d_plan* P, int shape) {
  const int TI = tile_w(shape), TJ = tile_h(shape);
  std::vector<Tile> out;
  for (int k = 0; k < P->ncases; ++k) {
    const int ni = P->cases[k].g.ni, nc = P->cases[k].g.nc;
    for (int j0 = 0; j0 < nc; j0 += TJ)
      for (int i0 = 0; i0 < ni; i0 += TI)
        out.push_back(Tile{k, i0, j0, std::min(TI, ni - i0), std::min(TJ, nc - j0)});
  }
  return out;
}

static void build_tables(a2d_plan* P, const int* ni, const int* nc, const void* const* metrics,
                         const double* winf) {
  long long cell = 0, rnc = 0, rnc1 = 0, cpo = 0;
  for (int k = 0; k < P->ncases; ++k) {
    CaseDev c{};
    c.g = grid_view(metrics[k], ni[k], nc[k]);
    for (int q = 0; q < 4; ++q) c.winf[q] = winf[4 * k + q];
    c.cell_off = cell;
    c.rows_nc = rnc;
    c.rows_nc1 = rnc1;
    const int ngr = (ni[k] + kLanes - 1) / kLanes;
    c.tile0 = (int)P->tiles.size();
    for (int j0 = 0; j0 < nc[k]; j0 += kTJ)
      for (int i0 = 0; i0 < ni[k]; i0 += kTI)
        P->tiles.push_back(Tile{k, i0, j0, std::min(kTI, ni[k] - i0), std::min(kTJ, nc[k] - j0)});
    c.ntiles = (int)P->tiles.size() - c.tile0;
    const long long n4 = 4LL * ni[k] * nc[k];
    c.chunk0 = (int)P->chunks.size();
    for (long long b0 = 0; b0 < n4; b0 += kChunk)
      P->chunks.push_back(Chunk{k, (int)b0, (int)std::min<long long>(kChunk, n4 - b0)});
    c.nchunks = (int)P->chunks.size() - c.chunk0;
    c.group0 = (int)P->groups.size();
    for (int g = 0; g < ngr; ++g)
      P->groups.push_back(Group{k, g, g * kLanes, std::min(kLanes, ni[k] - g * kLanes)});
    c.ngroups = ngr;
    P->cases.push_back(c);
    P->cp_off.push_back(cpo);
    cell += (long long)ni[k] * nc[k];
    rnc += (long long)ngr * nc[k];
    rnc1 += (long long)ngr * (nc[k] + 1);
    cpo += ni[k];
    P->max_ni = std::max(P->max_ni, ni[k]);
    P->max_nc = std::max(P->max_nc, nc[k]);
  }
  P->C = cell;
  P->rows_nc = rnc;
  P->rows_nc1 = rnc1;
  P->total_ni = cpo;
  for (int sh = 0; sh < kNumTileShapes; ++sh) P->max_jtiles = std::max(P->max_jtiles, (int)tile_list(P, sh).size());
  P->jtiles = tile_list(P, P->jvp_tile);
}

static void layout(a2d_plan* P) {
  Carve cv;
  const int B = P->ncases;
  const size_t C = (size_t)P->C;
  P->o_cases = cv.take(sizeof(CaseDev) * B);
  P->o_tiles = cv.take(sizeof(Tile) * P->tiles.size());
  P->o_chunks = cv.take(sizeof(Chunk) * P->chunks.size());
  P->o_groups = cv.take(sizeof(Group) * P->groups.size());
  P->o_cpoff = cv.take(sizeof(long long) * B);
  P->o_live = cv.take(sizeof(uint32_t) * B);
  P->o_ctl = cv.take(sizeof(CaseCtl) * B);
  for (int s = 0; s < kNumVec; ++s) P->o_vec[s] = cv.take(8 * 4 * C);
  P->o_diag = cv.take(8 * C);
  P->o_dt = cv.take(8 * C);
  const size_t lb = (size_t)16 * kLanes;
  P->o_JIL = cv.take(P->tj * lb * P->rows_nc);
  P->o_JIR = cv.take(P->tj * lb * P->rows_nc);
  P->o_JJL = cv.take(P->tj * lb * P->rows_nc1);
  P->o_JJR = cv.take(P->tj * lb * P->rows_nc1);
  P->o_INV = cv.take(P->tj * lb * P->rows_nc);
  P->o_CF = cv.take(P->tf * lb * P->rows_nc);
  P->o_PQG = cv.take(3 * P->tf * lb * P->rows_nc);
  P->o_V = cv.take(P->tb * 4 * C * (size_t)(P->m + 1));
  P->o_H = cv.take(8 * (size_t)B * kMaxRestart * (kMaxRestart + 1));
  P->o_h1 = cv.take(8 * (size_t)B * kHStride);
  P->o_h2 = cv.take(8 * (size_t)B * kHStride);
  P->o_scale = cv.take(8 * (size_t)B * (P->m + 1));
  P->o_y = cv.take(8 * (size_t)B * kMaxRestart);
  P->o_wn0 = cv.take(8 * (size_t)B);
  P->o_circ = cv.take(8 * (size_t)B);
  P->o_circ_rk = cv.take(8 * (size_t)B);
  P->o_tpart = cv.take(8 * kTilePartStride * P->tiles.size());
  P->pstride = P->m + 2;
  P->o_cpart = cv.take(8 * (size_t)P->pstride * P->chunks.size());
  P->o_cpart2 = cv.take(8 * (size_t)P->pstride * P->chunks.size());   // pass-2 partials of the folded path
  P->o_cpartn = cv.take(8 * P->chunks.size());
  P->o_coef = cv.take(8 * 3 * (size_t)B);
  P->o_cp = cv.take(8 * (size_t)P->total_ni);
  P->o_hrn = cv.take(8 * (size_t)B * P->p.max_iter);
  P->o_hcl = cv.take(8 * (size_t)B * P->p.max_iter);
  P->o_cnt = cv.take(8);   // [0] live-case count, [1] sweep copy-wait failure flag
  P->o_idx = cv.take(sizeof(int) * (size_t)B);   // case index lists of a2d_case_restart / _retire
  P->o_sat = cv.take(sizeof(unsigned long long));
  P->o_jtiles = cv.take(sizeof(Tile) * (size_t)P->max_jtiles);
  P->bytes = cv.off + 256;
}

// ---------------------------------------------------------------------------
// kernels of this file: init, counting, layout conversion, point flux
// ---------------------------------------------------------------------------
__global__ void k_init_state(Batch b, double* U) {
  const Tile t = b.tiles[blockIdx.x];
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  const double rho = cs.winf[0], u = cs.winf[1], v = cs.winf[2], p = cs.winf[3];
  const double Uc[4] = {rho, rho * u, rho * v, p / kGm1 + 0.5 * rho * (u * u + v * v)};
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
#pragma unroll
    for (int k = 0; k < 4; ++k) U[4 * cs.cell_off + vidx(g, k, j, i)] = Uc[k];
  }
}

__global__ void k_reset(int ncases, CaseCtl* ctl, uint32_t* live, double cfl0) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncases) return;
  CaseCtl c{};
  c.cfl = cfl0;
  c.rn = NAN;
  c.lastrn = NAN;
  c.r0 = 1.0;
  c.omega = 1.0;
  ctl[k] = c;
  live[k] = kLiveNewton;
}

// restarts the listed cases (one block each) with the freestream now in their
// table entry: U := freestream and Newton state as k_reset; with keep, U stays
// (the previous point's solution) and so does r0, the residual reference of
// the sweep's first (cold) point, so that the tolerance keeps its absolute
// level and the SER CFL starts from the converged state's small residual
__global__ void k_restart_cases(Batch b, const int* idx, int keep, double* U, CaseCtl* ctl, uint32_t* live,
                                double cfl0) {
  const int k = idx[blockIdx.x];
  const CaseDev cs = b.cases[k];
  if (!keep) {
    const double rho = cs.winf[0], u = cs.winf[1], v = cs.winf[2], p = cs.winf[3];
    const double Uc[4] = {rho, rho * u, rho * v, p / kGm1 + 0.5 * rho * (u * u + v * v)};
    const long long n = (long long)cs.g.ni * cs.g.nc;
    double* Uk = U + 4 * cs.cell_off;
    for (long long c = threadIdx.x; c < n; c += blockDim.x) {
#pragma unroll
      for (int q = 0; q < 4; ++q) Uk[q * n + c] = Uc[q];
    }
  }
  if (threadIdx.x == 0) {
    const double r0 = ctl[k].r0;
    const bool carry = keep && ctl[k].nsteps > 0 && isfinite(r0) && r0 > 0.0;
    CaseCtl c{};
    c.cfl = cfl0;
    c.rn = NAN;
    c.lastrn = NAN;
    c.r0 = carry ? r0 : 1.0;
    c.keep_r0 = carry ? 1 : 0;
    c.omega = 1.0;
    ctl[k] = c;
    live[k] = kLiveNewton;
  }
}

__global__ void k_retire_cases(const int* idx, int n, uint32_t* live) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) live[idx[q]] = 0;
}

__global__ void k_count(int ncases, const CaseCtl* ctl, const uint32_t* live, int retire, int* out) {
  __shared__ int s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  for (int k = threadIdx.x; k < ncases; k += blockDim.x) {
    const int busy = retire ? ((live[k] & kLiveNewton) ? 1 : 0) : (ctl[k].done ? 0 : 1);
    if (busy) atomicAdd(&s, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) *out = s;
}

// reference layout [4][ni][nc] <-> internal [4][nc][ni] of one case
__global__ void k_to_internal(int ni, int nc, const double* __restrict__ src, double* __restrict__ dst) {
  const size_t n = 4 * (size_t)ni * nc;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(t / ((size_t)ni * nc));
    const size_t r = t % ((size_t)ni * nc);
    const int i = (int)(r / nc), j = (int)(r % nc);
    dst[((size_t)k * nc + j) * ni + i] = src[t];
  }
}
__global__ void k_to_reference(int ni, int nc, const double* __restrict__ src, double* __restrict__ dst) {
  const size_t n = 4 * (size_t)ni * nc;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(t / ((size_t)ni * nc));
    const size_t r = t % ((size_t)ni * nc);
    const int i = (int)(r / nc), j = (int)(r % nc);
    dst[t] = src[((size_t)k * nc + j) * ni + i];
  }
}

// primitives of one case's cell vector, internal [4][nc][ni] -> reference [4][ni][nc]
__global__ void k_to_reference_prim(int ni, int nc, const double* __restrict__ src, double* __restrict__ dst) {
  const size_t N = (size_t)ni * nc;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N; q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q / nc), j = (int)(q % nc);
    State4<double> u;
#pragma unroll
    for (int k = 0; k < 4; ++k) u.c[k] = src[((size_t)k * nc + j) * ni + i];
    const State4<double> w = cons_to_prim<double, double>(u);
#pragma unroll
    for (int k = 0; k < 4; ++k) dst[k * N + q] = w.c[k];
  }
}

__global__ void k_point_flux(int n, const double* WL, const double* WR, const double* S, double* F) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  State4<double> L, R;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    L.c[k] = WL[(size_t)k * n + q];
    R.c[k] = WR[(size_t)k * n + q];
  }
  const State4<double> f = hllc<double, double>(L, R, S[q], S[(size_t)n + q]);
#pragma unroll
  for (int k = 0; k < 4; ++k) F[(size_t)k * n + q] = f.c[k];
}

}  // namespace a2d

// ---------------------------------------------------------------------------
// orchestration
// ---------------------------------------------------------------------------
namespace a2d {

// NVTX range for profilers (no cost without one attached): the stages of a Newton
// step when it runs without a graph, and the C ABI's solver entry points
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

static SweepArgs sweep_args(const a2d_plan* P, uint32_t need) {
  SweepArgs a;
  a.INV = P->at<void>(P->o_INV);
  a.PQG = P->at<void>(P->o_PQG);
  a.dtmp = P->vec(kPD);
  a.CF = P->at<void>(P->o_CF);
  a.err = P->at<uint32_t>(P->o_cnt) + 1;
  a.need = need;
  return a;
}

static FactorArgs factor_args(const a2d_plan* P, uint32_t need) {
  FactorArgs fa;
  fa.U = P->vec(kU);
  fa.ctl = P->ctl();
  fa.JIL = P->at<void>(P->o_JIL);
  fa.JIR = P->at<void>(P->o_JIR);
  fa.JJL = P->at<void>(P->o_JJL);
  fa.JJR = P->at<void>(P->o_JJR);
  fa.INV = P->at<void>(P->o_INV);
  fa.CF = P->at<void>(P->o_CF);
  fa.PQG = P->at<void>(P->o_PQG);
  fa.diag = P->at<double>(P->o_diag);
  fa.cfl_base = P->p.cfl;
  fa.sat = P->at<unsigned long long>(P->o_sat);
  fa.need = need;
  return fa;
}

// x = M^-1 r: jacobi_sweeps line-Jacobi sweeps (aero2d/implicit.py:150-157);
// rin may be dst
template <typename TJ>
static void precond(a2d_plan* P, const Batch& B, const double* rin, double* dst, uint32_t need, cudaStream_t s) {
  SweepArgs a = sweep_args(P, need);
  const int sweeps = std::max(1, P->p.jacobi_sweeps);
  double* bufs[2] = {P->vec(kPA), P->vec(kPB)};
  a.r = rin;
  a.e0 = sweeps > 1 ? P->vec(kPE) : nullptr;
  a.x = sweeps > 1 ? bufs[0] : dst;
  launch_sweep<TJ, true>(B, a, sweeps == 1, s, P->sweep_variant);
  for (int sw = 1; sw < sweeps; ++sw) {
    const bool last = sw == sweeps - 1;
    a.xprev = a.x;
    a.x = last ? dst : bufs[sw & 1];
    launch_sweep<TJ, false>(B, a, last, s, P->sweep_variant);
  }
}

template <typename TJ>
static void precond_setup(a2d_plan* P, const Batch& B, uint32_t need, cudaStream_t s) {
  JacArgs ja;
  ja.U = P->vec(kU);
  ja.circ = P->at<double>(P->o_circ);
  ja.JIL = P->at<void>(P->o_JIL);
  ja.JIR = P->at<void>(P->o_JIR);
  ja.JJL = P->at<void>(P->o_JJL);
  ja.JJR = P->at<void>(P->o_JJR);
  ja.vortex = P->p.vortex_correction;
  ja.need = need;
  launch_face_jac<TJ>(B, ja, s);
  launch_factor<TJ, typename FactorStore<TJ>::type>(B, factor_args(P, need), s);
}

static StencilArgs<double> residual_args(a2d_plan* P) {
  StencilArgs<double> a;
  a.U = P->vec(kU);
  a.lim_k = P->p.lim_k;
  a.order = P->p.order;
  a.vortex = P->p.vortex_correction;
  return a;
}

// the linearised stencil (J v): in FP32 on the plan's JVP tile list and shape,
// in FP64 on the standard tiles
template <typename TV, typename VT>
static void launch_jvp(const a2d_plan* P, const StencilArgs<VT>& a, cudaStream_t s) {
  if constexpr (sizeof(TV) == 4) {
    Batch jb = P->jbatch;
    jb.live = P->batch.live;
    launch_stencil<TV, true, VT>(jb, a, s, P->jvp_tile);
  } else {
    launch_stencil<TV, true, VT>(P->batch, a, s);
  }
}

template <typename TV, typename TJ, typename TB>
static void newton_step_launches(a2d_plan* P, cudaStream_t s) {
  const Batch& B = P->batch;
  const uint32_t NW = kLiveNewton, KR = kLiveNewton | kLiveKrylov;
  double* U = P->vec(kU);
  double* b = P->vec(kB);
  double* x0 = P->vec(kX0);
  double* t = P->vec(kT);
  double* r = P->vec(kRr);
  double* z = P->vec(kZ);
  double* w = P->vec(kW);
  double* dU = P->vec(kDU);
  double* diag = P->at<double>(P->o_diag);
  double* tpart = P->at<double>(P->o_tpart);
  double* cpart = P->at<double>(P->o_cpart);
  double* cpartn = P->at<double>(P->o_cpartn);
  TB* V = P->at<TB>(P->o_V);
  const size_t vs = 4 * (size_t)P->C;
  CaseCtl* ctl = P->ctl();
  uint32_t* live = P->live();

  nvtxRangePushA("newton: residual and line preconditioner");
  launch_mark_stepped(B, live, ctl, s);
  // Newton right-hand side b = -R(U) in FP64, circulation from U, residual-norm partials
  StencilArgs<double> ra = residual_args(P);
  ra.out = b;
  ra.sign = -1.0;
  ra.circ_out = P->at<double>(P->o_circ);
  ra.tile_part = tpart;
  ra.need = NW;
  launch_stencil<double, false, double>(B, ra, s);
  // line preconditioner at U
  precond_setup<TJ>(P, B, NW, s);
  nvtxRangePop();
  nvtxRangePushA("newton: GMRES start");
  // x0 = M b; ptol from ||b||, ||M b||
  precond<TJ>(P, B, b, x0, NW, s);
  launch_norms2(B, b, x0, cpart, P->pstride, NW, s);
  launch_gm_setup(B, cpart, P->pstride, ctl, P->p.gmres_tol, s);
  // t = b - A x0, A v = diag v + J v
  StencilArgs<double> ta = residual_args(P);
  ta.V = x0;
  ta.diag = diag;
  ta.bvec = b;
  ta.out = t;
  ta.need = NW;
  launch_jvp<TV, double>(P, ta, s);
  // r = M t, v0 = r / ||r||
  precond<TJ>(P, B, t, r, NW, s);
  double* h1 = P->at<double>(P->o_h1);
  double* h2 = P->at<double>(P->o_h2);
  double* wn0 = P->at<double>(P->o_wn0);
  double* scale = P->at<double>(P->o_scale);
  GsArgs<TB> g0;
  g0.w = r;
  g0.Vout = V;
  g0.part_norm = cpartn;
  g0.need = NW;
  launch_gs_start<TB>(B, g0, s);
  GsCloseArgs c0;
  c0.part_norm = cpartn;
  c0.scale = scale;
  c0.ctl = ctl;
  c0.live = live;
  c0.k = -1;
  c0.need = NW;
  launch_gs_close(B, c0, s);
  nvtxRangePop();
  nvtxRangePushA("newton: Arnoldi");
  for (int k = 0; k < P->m; ++k) {
    StencilArgs<TB> za;
    za.U = U;
    za.V = V + (size_t)k * vs;
    za.vscale = scale + (size_t)k * P->ncases;
    za.diag = diag;
    za.out = z;
    za.lim_k = P->p.lim_k;
    za.order = P->p.order;
    za.vortex = P->p.vortex_correction;
    za.need = KR;
    launch_jvp<TV, TB>(P, za, s);
    precond<TJ>(P, B, z, w, KR, s);
    // classical Gram-Schmidt run twice, three passes over the basis
    GsArgs<TB> g;
    g.err = P->at<uint32_t>(P->o_cnt) + 1;
    g.w = w;
    g.V = V;
    g.vstride = vs;
    g.nq = k + 1;
    g.part = cpart;
    g.pstride = P->pstride;
    g.h1 = h1;
    g.h2 = h2;
    g.scale = scale;
    g.Vout = V + (size_t)(k + 1) * vs;
    g.part_norm = cpartn;
    g.tmp = t;
    g.need = KR;
    g.with_norm = 1;
    launch_gs_dots<TB>(B, g, s);
    if (k + 1 <= kGsSlice) {
      // one slice: the per-case reductions run inside the next pass (no reduce launches);
      // pass 2 writes its partials to a second buffer while it reads pass 1's
      GsArgs<TB> gp = g;
      gp.fold_part = cpart;
      gp.fold_h = h1;
      gp.fold_wn0 = wn0;
      gp.part = P->at<double>(P->o_cpart2);
      launch_gs_project<TB>(B, gp, s);
      GsArgs<TB> gf = g;
      gf.fold_part = P->at<double>(P->o_cpart2);
      gf.fold_h = h2;
      launch_gs_finish<TB>(B, gf, s);
    } else {
      GsReduceArgs rd;
      rd.part = cpart;
      rd.pstride = P->pstride;
      rd.nq = k + 1;
      rd.scale = scale;
      rd.h = h1;
      rd.wn0 = wn0;
      rd.need = KR;
      launch_gs_reduce(B, rd, s);
      launch_gs_project<TB>(B, g, s);
      rd.h = h2;
      rd.wn0 = nullptr;
      launch_gs_reduce(B, rd, s);
      launch_gs_finish<TB>(B, g, s);
    }
    GsCloseArgs ck;
    ck.part_norm = cpartn;
    ck.wn0 = wn0;
    ck.h1 = h1;
    ck.h2 = h2;
    ck.H = P->at<double>(P->o_H);
    ck.scale = scale;
    ck.ctl = ctl;
    ck.live = live;
    ck.k = k;
    ck.need = KR;
    launch_gs_close(B, ck, s);
  }
  nvtxRangePop();
  nvtxRangePushA("newton: least squares and update");
  launch_lstsq(B, live, ctl, P->at<double>(P->o_H), P->at<double>(P->o_y), s);
  CombineArgs<TB> ca;
  ca.x0 = x0;
  ca.V = V;
  ca.vstride = vs;
  ca.y = P->at<double>(P->o_y);
  ca.scale = scale;
  ca.ctl = ctl;
  ca.out = dU;
  ca.need = NW;
  launch_combine<TB>(B, ca, s);
  // positivity step limit, finiteness, per-case controller, commit, forces
  launch_update_rel(B, U, dU, tpart, NW, s);
  launch_update_check(B, U, dU, tpart, ctl, P->p.max_update, NW, s);
  CtlParams cp;
  cp.cfl0 = P->p.cfl0;
  cp.cfl_max = P->p.cfl_max;
  cp.tol = P->p.tol;
  cp.retire = P->p.retire;
  launch_controller(B, tpart, ctl, live, P->at<double>(P->o_hrn), P->p.max_iter, cp, s);
  launch_commit(B, U, dU, ctl, s);
  launch_forces(B, U, P->at<double>(P->o_coef), P->at<double>(P->o_cp), P->at<long long>(P->o_cpoff), ctl,
                P->at<double>(P->o_hcl), P->p.max_iter, s);
  nvtxRangePop();
}

static void newton_dispatch(a2d_plan* P, cudaStream_t s) {
  if (P->p.precision == A2D_MIXED) newton_step_launches<float, float, Basis16>(P, s);
  else newton_step_launches<double, double, double>(P, s);
}

static int newton_step(a2d_plan* P, cudaStream_t s) {
  if (!P->p.use_graph) {
    newton_dispatch(P, s);
    A2D_CK(cudaGetLastError());
    return A2D_OK;
  }
  if (P->graph == nullptr) {
    cudaStream_t cap;
    A2D_CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t g;
    A2D_CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    newton_dispatch(P, cap);
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (e != cudaSuccess) return fail(A2D_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    size_t nn = 0;
    if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
      std::vector<cudaGraphNode_t> nodes(nn);
      if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess) {
        int nk = 0;
        for (size_t q = 0; q < nn; ++q) {
          cudaGraphNodeType ty;
          if (cudaGraphNodeGetType(nodes[q], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++nk;
        }
        P->kernels_per_step = nk;
      }
    }
    e = cudaGraphInstantiate(&P->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(A2D_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  A2D_CK(cudaGraphLaunch(P->graph, s));
  return A2D_OK;
}

}  // namespace a2d

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
#define A2D_BOUND(P)                                                     \
  do {                                                                   \
    if ((P) == nullptr) return fail(A2D_ERR_ARG, "null plan");           \
    if ((P)->ws == nullptr) return fail(A2D_ERR_STATE, "plan not bound"); \
  } while (0)

extern "C" {

int a2d_version(void) { return 100; }

const char* a2d_last_error(void) { return g_last_error.c_str(); }

void a2d_default_params(a2d_params* p) {
  if (p == nullptr) return;
  p->gmres_restart = 50;
  p->jacobi_sweeps = 4;
  p->gmres_tol = 0.01;
  p->cfl0 = 10.0;
  p->cfl_max = 300.0;
  p->max_update = 0.2;
  p->tol = 1e-8;
  p->cfl = 2.5;
  p->irs_eps = 0.6;
  p->lim_k = 0.02;
  p->order = 2;
  p->vortex_correction = 1;
  p->precision = A2D_FP64;
  p->retire = 1;
  p->max_iter = 200;
  p->use_graph = 1;
}

int a2d_metrics_bytes(int ni, int nj, size_t* bytes) {
  if (bytes == nullptr || ni < 4 || nj < 3) return fail(A2D_ERR_ARG, "metrics: need ni >= 4, nj >= 3");
  *bytes = metrics_total_bytes(ni, nj - 1);
  return A2D_OK;
}

int a2d_metrics_build(int ni, int nj, const double* x, const double* y, void* metrics, void* stream) {
  if (x == nullptr || y == nullptr || metrics == nullptr || ni < 4 || nj < 3)
    return fail(A2D_ERR_ARG, "metrics: bad arguments");
  const int nc = nj - 1;
  double* md = static_cast<double*>(metrics);
  float* mf = reinterpret_cast<float*>(static_cast<char*>(metrics) + metrics_float_offset(ni, nc));
  launch_metrics(ni, nc, x, y, md, mf, static_cast<cudaStream_t>(stream));
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_plan_create(int ncases, const int* ni, const int* nc, const void* const* metrics, const double* winf,
                    const a2d_params* params, a2d_plan** out) {
  if (out == nullptr || ncases <= 0 || ni == nullptr || nc == nullptr || metrics == nullptr || winf == nullptr)
    return fail(A2D_ERR_ARG, "plan_create: bad arguments");
  a2d_params p;
  a2d_default_params(&p);
  if (params != nullptr) p = *params;
  if (p.gmres_restart < 1 || p.gmres_restart > kMaxRestart)
    return fail(A2D_ERR_ARG, "gmres_restart must be in [1, 64]");
  if (p.jacobi_sweeps < 1) return fail(A2D_ERR_ARG, "jacobi_sweeps must be >= 1");
  if (p.order != 1 && p.order != 2) return fail(A2D_ERR_ARG, "order must be 1 or 2");
  if (p.precision != A2D_FP64 && p.precision != A2D_MIXED) return fail(A2D_ERR_ARG, "unknown precision");
  if (p.max_iter < 1) return fail(A2D_ERR_ARG, "max_iter must be >= 1");
  for (int k = 0; k < ncases; ++k) {
    if (ni[k] < 4 || nc[k] < 2 || metrics[k] == nullptr)
      return fail(A2D_ERR_ARG, "case " + std::to_string(k) + ": need ni >= 4, nc >= 2 and metrics");
  }
  a2d_plan* P = new a2d_plan();
  P->p = p;
  if (p.precision != A2D_MIXED) P->sweep_variant = kSweepLanes;   // rows runs mixed plans only
  P->ncases = ncases;
  P->m = p.gmres_restart;
  P->tj = p.precision == A2D_MIXED ? 4 : 8;
  P->tf = p.precision == A2D_MIXED ? 2 : 8;
  P->tb = p.precision == A2D_MIXED ? sizeof(Basis16) : 8;
  build_tables(P, ni, nc, metrics, winf);
  layout(P);
  *out = P;
  return A2D_OK;
}

int a2d_plan_workspace_bytes(const a2d_plan* P, size_t* bytes) {
  if (P == nullptr || bytes == nullptr) return fail(A2D_ERR_ARG, "null argument");
  *bytes = P->bytes;
  return A2D_OK;
}

int a2d_plan_ncases(const a2d_plan* P) { return P ? P->ncases : 0; }

int a2d_plan_set_tuning(a2d_plan* P, int jvp_tile, int sweep_variant, void* stream) {
  if (P == nullptr) return fail(A2D_ERR_ARG, "null plan");
  if (jvp_tile < 0 || jvp_tile >= kNumTileShapes) return fail(A2D_ERR_ARG, "set_tuning: unknown JVP tile shape");
  if (sweep_variant < 0 || sweep_variant >= kNumSweepVariants)
    return fail(A2D_ERR_ARG, "set_tuning: unknown sweep variant");
  if ((sweep_variant == kSweepRows || sweep_variant == kSweepHalves) && P->p.precision != A2D_MIXED)
    return fail(A2D_ERR_ARG, "set_tuning: the rows and halves sweeps run mixed-precision plans only");
  if (jvp_tile != P->jvp_tile) {
    P->jvp_tile = jvp_tile;
    P->jtiles = tile_list(P, jvp_tile);
    if (P->ws != nullptr) {
      cudaStream_t s = static_cast<cudaStream_t>(stream);
      A2D_CK(cudaMemcpyAsync(P->ws + P->o_jtiles, P->jtiles.data(), sizeof(Tile) * P->jtiles.size(),
                             cudaMemcpyHostToDevice, s));
      A2D_CK(cudaStreamSynchronize(s));
      P->jbatch.ntiles = (int)P->jtiles.size();
    }
  }
  P->sweep_variant = sweep_variant;
  if (P->graph != nullptr) {   // the captured step holds the old launch configuration
    cudaGraphExecDestroy(P->graph);
    P->graph = nullptr;
  }
  return A2D_OK;
}

int a2d_plan_get_tuning(const a2d_plan* P, int* jvp_tile, int* sweep_variant) {
  if (P == nullptr) return fail(A2D_ERR_ARG, "null plan");
  if (jvp_tile != nullptr) *jvp_tile = P->jvp_tile;
  if (sweep_variant != nullptr) *sweep_variant = P->sweep_variant;
  return A2D_OK;
}

int a2d_plan_bind(a2d_plan* P, void* workspace, size_t bytes, void* stream) {
  if (P == nullptr || workspace == nullptr) return fail(A2D_ERR_ARG, "bind: null argument");
  if (bytes < P->bytes) return fail(A2D_ERR_ARG, "bind: workspace too small");
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return fail(A2D_ERR_ARG, "bind: workspace not 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (P->graph != nullptr) {
    cudaGraphExecDestroy(P->graph);
    P->graph = nullptr;
  }
  P->ws = static_cast<char*>(workspace);
  A2D_CK(cudaMemcpyAsync(P->ws + P->o_cases, P->cases.data(), sizeof(CaseDev) * P->ncases,
                         cudaMemcpyHostToDevice, s));
  A2D_CK(cudaMemcpyAsync(P->ws + P->o_tiles, P->tiles.data(), sizeof(Tile) * P->tiles.size(),
                         cudaMemcpyHostToDevice, s));
  A2D_CK(cudaMemcpyAsync(P->ws + P->o_chunks, P->chunks.data(), sizeof(Chunk) * P->chunks.size(),
                         cudaMemcpyHostToDevice, s));
  A2D_CK(cudaMemcpyAsync(P->ws + P->o_groups, P->groups.data(), sizeof(Group) * P->groups.size(),
                         cudaMemcpyHostToDevice, s));
  A2D_CK(cudaMemcpyAsync(P->ws + P->o_cpoff, P->cp_off.data(), sizeof(long long) * P->ncases,
                         cudaMemcpyHostToDevice, s));
  A2D_CK(cudaMemsetAsync(P->ws + P->o_vec[0], 0, P->o_diag - P->o_vec[0], s));
  Batch& B = P->batch;
  B.cases = P->at<CaseDev>(P->o_cases);
  B.tiles = P->at<Tile>(P->o_tiles);
  B.chunks = P->at<Chunk>(P->o_chunks);
  B.groups = P->at<Group>(P->o_groups);
  B.live = P->live();
  B.ncases = P->ncases;
  B.ntiles = (int)P->tiles.size();
  B.nchunks = (int)P->chunks.size();
  B.ngroups = (int)P->groups.size();
  A2D_CK(cudaMemcpyAsync(P->ws + P->o_jtiles, P->jtiles.data(), sizeof(Tile) * P->jtiles.size(),
                         cudaMemcpyHostToDevice, s));
  P->jbatch = B;
  P->jbatch.tiles = P->at<Tile>(P->o_jtiles);
  P->jbatch.ntiles = (int)P->jtiles.size();
  if (P->host_count == nullptr) A2D_CK(cudaMallocHost(&P->host_count, 2 * sizeof(int)));
  A2D_CK(cudaMemsetAsync(P->ws + P->o_cnt, 0, 8, s));
  A2D_CK(cudaMemsetAsync(P->ws + P->o_sat, 0, sizeof(unsigned long long), s));
  A2D_CK(sweep_init());
  A2D_CK(gs_init());
  stencil_init_fp64();
  stencil_init_fp32();
  k_reset<<<(P->ncases + 63) / 64, 64, 0, s>>>(P->ncases, P->ctl(), P->live(), P->p.cfl0);
  A2D_CK(cudaMemsetAsync(P->ws + P->o_circ_rk, 0, 8 * (size_t)P->ncases, s));
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_plan_destroy(a2d_plan* P) {
  if (P == nullptr) return A2D_OK;
  if (P->graph != nullptr) cudaGraphExecDestroy(P->graph);
  if (P->host_count != nullptr) cudaFreeHost(P->host_count);
  delete P;
  return A2D_OK;
}

static int check_case(const a2d_plan* P, int slot, int k) {
  if (slot < 0 || slot > A2D_VEC_DU) return fail(A2D_ERR_ARG, "unknown vector slot");
  if (k < 0 || k >= P->ncases) return fail(A2D_ERR_ARG, "case index out of range");
  return A2D_OK;
}

int a2d_vec_set(a2d_plan* P, int slot, int k, const double* src, void* stream) {
  A2D_BOUND(P);
  if (int e = check_case(P, slot, k)) return e;
  if (src == nullptr) return fail(A2D_ERR_ARG, "null source");
  const CaseDev& c = P->cases[k];
  k_to_internal<<<256, 256, 0, static_cast<cudaStream_t>(stream)>>>(c.g.ni, c.g.nc, src,
                                                                     P->vec(slot) + 4 * c.cell_off);
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_vec_get(const a2d_plan* P, int slot, int k, double* dst, void* stream) {
  A2D_BOUND(P);
  if (int e = check_case(P, slot, k)) return e;
  if (dst == nullptr) return fail(A2D_ERR_ARG, "null destination");
  const CaseDev& c = P->cases[k];
  k_to_reference<<<256, 256, 0, static_cast<cudaStream_t>(stream)>>>(c.g.ni, c.g.nc,
                                                                      P->vec(slot) + 4 * c.cell_off, dst);
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_vec_get_prim(const a2d_plan* P, int slot, int k, double* dst, void* stream) {
  A2D_BOUND(P);
  if (int e = check_case(P, slot, k)) return e;
  if (dst == nullptr) return fail(A2D_ERR_ARG, "null destination");
  const CaseDev& c = P->cases[k];
  k_to_reference_prim<<<256, 256, 0, static_cast<cudaStream_t>(stream)>>>(c.g.ni, c.g.nc,
                                                                           P->vec(slot) + 4 * c.cell_off, dst);
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_local_dt(const a2d_plan* P, int k, const double* W, double* dt, void* stream) {
  A2D_BOUND(P);
  if (k < 0 || k >= P->ncases) return fail(A2D_ERR_ARG, "local_dt: case index out of range");
  if (W == nullptr || dt == nullptr) return fail(A2D_ERR_ARG, "local_dt: null pointer");
  launch_local_dt_prim(P->cases[k].g, W, dt, P->p.cfl, static_cast<cudaStream_t>(stream));
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_init_freestream(a2d_plan* P, void* stream) {
  A2D_BOUND(P);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_init_state<<<P->batch.ntiles, 256, 0, s>>>(P->batch, P->vec(kU));
  k_reset<<<(P->ncases + 63) / 64, 64, 0, s>>>(P->ncases, P->ctl(), P->live(), P->p.cfl0);
  A2D_CK(cudaGetLastError());
  P->steps_taken = 0;
  return A2D_OK;
}

int a2d_reset(a2d_plan* P, void* stream) {
  A2D_BOUND(P);
  k_reset<<<(P->ncases + 63) / 64, 64, 0, static_cast<cudaStream_t>(stream)>>>(P->ncases, P->ctl(), P->live(),
                                                                                P->p.cfl0);
  A2D_CK(cudaGetLastError());
  P->steps_taken = 0;
  return A2D_OK;
}

int a2d_case_restart(a2d_plan* P, int n, const int* cases, const double* winf, int keep_state, void* stream) {
  A2D_BOUND(P);
  if (n < 0 || n > P->ncases || (n > 0 && (cases == nullptr || winf == nullptr)))
    return fail(A2D_ERR_ARG, "case_restart: bad arguments");
  if (n == 0) return A2D_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int q = 0; q < n; ++q) {
    const int k = cases[q];
    if (k < 0 || k >= P->ncases) return fail(A2D_ERR_ARG, "case_restart: case index out of range");
    for (int c = 0; c < 4; ++c) P->cases[k].winf[c] = winf[4 * q + c];
  }
  // the per-case table and the index list; pageable sources are staged before the call returns
  A2D_CK(cudaMemcpyAsync(P->ws + P->o_cases, P->cases.data(), sizeof(CaseDev) * P->ncases,
                         cudaMemcpyHostToDevice, s));
  A2D_CK(cudaMemcpyAsync(P->at<int>(P->o_idx), cases, sizeof(int) * n, cudaMemcpyHostToDevice, s));
  k_restart_cases<<<n, 256, 0, s>>>(P->batch, P->at<int>(P->o_idx), keep_state, P->vec(kU), P->ctl(), P->live(),
                                    P->p.cfl0);
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_case_forces(a2d_plan* P, double* coef, double* cp, void* stream) {
  A2D_BOUND(P);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Batch B = P->batch;
  B.live = nullptr;
  launch_forces(B, P->vec(kU), P->at<double>(P->o_coef), P->at<double>(P->o_cp), P->at<long long>(P->o_cpoff),
                nullptr, nullptr, 0, s);
  if (coef != nullptr)
    A2D_CK(cudaMemcpyAsync(coef, P->at<double>(P->o_coef), 8 * 3 * (size_t)P->ncases, cudaMemcpyDeviceToHost, s));
  if (cp != nullptr)
    A2D_CK(cudaMemcpyAsync(cp, P->at<double>(P->o_cp), 8 * (size_t)P->total_ni, cudaMemcpyDeviceToHost, s));
  A2D_CK(cudaStreamSynchronize(s));
  return A2D_OK;
}

int a2d_case_set_grid(a2d_plan* P, int n, const int* cases, const void* const* metrics, void* stream) {
  A2D_BOUND(P);
  if (n < 0 || n > P->ncases || (n > 0 && (cases == nullptr || metrics == nullptr)))
    return fail(A2D_ERR_ARG, "case_set_grid: bad arguments");
  if (n == 0) return A2D_OK;
  for (int q = 0; q < n; ++q) {
    const int k = cases[q];
    if (k < 0 || k >= P->ncases) return fail(A2D_ERR_ARG, "case_set_grid: case index out of range");
    if (metrics[q] == nullptr) return fail(A2D_ERR_ARG, "case_set_grid: null metrics");
  }
  for (int q = 0; q < n; ++q) {
    CaseDev& c = P->cases[cases[q]];
    c.g = grid_view(metrics[q], c.g.ni, c.g.nc);
  }
  A2D_CK(cudaMemcpyAsync(P->ws + P->o_cases, P->cases.data(), sizeof(CaseDev) * P->ncases, cudaMemcpyHostToDevice,
                         static_cast<cudaStream_t>(stream)));
  return A2D_OK;
}

int a2d_case_retire(a2d_plan* P, int n, const int* cases, void* stream) {
  A2D_BOUND(P);
  if (n < 0 || n > P->ncases || (n > 0 && cases == nullptr)) return fail(A2D_ERR_ARG, "case_retire: bad arguments");
  if (n == 0) return A2D_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int q = 0; q < n; ++q)
    if (cases[q] < 0 || cases[q] >= P->ncases) return fail(A2D_ERR_ARG, "case_retire: case index out of range");
  A2D_CK(cudaMemcpyAsync(P->at<int>(P->o_idx), cases, sizeof(int) * n, cudaMemcpyHostToDevice, s));
  k_retire_cases<<<(n + 63) / 64, 64, 0, s>>>(P->at<int>(P->o_idx), n, P->live());
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_residual(a2d_plan* P, const double* circ, void* stream) {
  A2D_BOUND(P);
  StencilArgs<double> a = residual_args(P);
  a.circ_in = circ;
  a.out = P->vec(kR);
  a.sign = 1.0;
  a.circ_out = P->at<double>(P->o_circ);
  a.tile_part = P->at<double>(P->o_tpart);
  Batch B = P->batch;
  B.live = nullptr;
  launch_stencil<double, false, double>(B, a, static_cast<cudaStream_t>(stream));
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_jvp(a2d_plan* P, void* stream) {
  A2D_BOUND(P);
  StencilArgs<double> a = residual_args(P);
  a.V = P->vec(kVin);
  a.out = P->vec(kJV);
  Batch B = P->batch;
  B.live = nullptr;
  if (P->p.precision == A2D_MIXED) {
    Batch jb = P->jbatch;
    jb.live = nullptr;
    launch_stencil<float, true, double>(jb, a, static_cast<cudaStream_t>(stream), P->jvp_tile);
  } else {
    launch_stencil<double, true, double>(B, a, static_cast<cudaStream_t>(stream));
  }
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_forces(a2d_plan* P, double* coef, double* cp, void* stream) {
  A2D_BOUND(P);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Batch B = P->batch;
  B.live = nullptr;
  launch_forces(B, P->vec(kU), P->at<double>(P->o_coef), P->at<double>(P->o_cp), P->at<long long>(P->o_cpoff),
                nullptr, nullptr, 0, s);
  if (coef != nullptr)
    A2D_CK(cudaMemcpyAsync(coef, P->at<double>(P->o_coef), 8 * 3 * (size_t)P->ncases, cudaMemcpyDeviceToDevice, s));
  if (cp != nullptr)
    A2D_CK(cudaMemcpyAsync(cp, P->at<double>(P->o_cp), 8 * (size_t)P->total_ni, cudaMemcpyDeviceToDevice, s));
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_set_cfl(a2d_plan* P, const double* cfl, void* stream) {
  A2D_BOUND(P);
  if (cfl == nullptr) return fail(A2D_ERR_ARG, "null cfl");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int k = 0; k < P->ncases; ++k)
    A2D_CK(cudaMemcpyAsync(&P->ctl()[k].cfl, &cfl[k], sizeof(double), cudaMemcpyHostToDevice, s));
  A2D_CK(cudaStreamSynchronize(s));
  return A2D_OK;
}

int a2d_precond_setup(a2d_plan* P, void* stream) {
  A2D_BOUND(P);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // circulation of U for the far-field block (as the Newton step forms it)
  StencilArgs<double> a = residual_args(P);
  a.out = P->vec(kB);
  a.sign = -1.0;
  a.circ_out = P->at<double>(P->o_circ);
  a.tile_part = P->at<double>(P->o_tpart);
  Batch B = P->batch;
  B.live = nullptr;
  launch_stencil<double, false, double>(B, a, s);
  if (P->p.precision == A2D_MIXED) precond_setup<float>(P, B, 0, s);
  else precond_setup<double>(P, B, 0, s);
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_precond_apply(a2d_plan* P, void* stream) {
  A2D_BOUND(P);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Batch B = P->batch;
  B.live = nullptr;
  if (P->p.precision == A2D_MIXED) precond<float>(P, B, P->vec(kVin), P->vec(kJV), 0, s);
  else precond<double>(P, B, P->vec(kVin), P->vec(kJV), 0, s);
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_newton_step(a2d_plan* P, void* stream) {
  A2D_BOUND(P);
  Range range("a2d_newton_step");
  const int e = newton_step(P, static_cast<cudaStream_t>(stream));
  if (e == A2D_OK) P->steps_taken += 1;
  return e;
}

int a2d_newton_run(a2d_plan* P, int max_steps, int* steps, void* stream) {
  A2D_BOUND(P);
  Range range("a2d_newton_run");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int done = 0;
  int* dcount = P->at<int>(P->o_cnt);
  for (int it = 0; it < max_steps; ++it) {
    if (P->steps_taken >= P->p.max_iter) break;
    if (int e = newton_step(P, s)) return e;
    P->steps_taken += 1;
    ++done;
    k_count<<<1, 256, 0, s>>>(P->ncases, P->ctl(), P->live(), P->p.retire, dcount);
    A2D_CK(cudaMemcpyAsync(P->host_count, dcount, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    A2D_CK(cudaStreamSynchronize(s));
    if (P->host_count[1] != 0) return fail(A2D_ERR_CUDA, "line sweep: a bulk-copy wait ran out of time");
    if (*P->host_count == 0) break;
  }
  if (steps != nullptr) *steps = done;
  return A2D_OK;
}

int a2d_factor_saturations(a2d_plan* P, unsigned long long* count, int reset, void* stream) {
  A2D_BOUND(P);
  if (count == nullptr) return fail(A2D_ERR_ARG, "null output");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  A2D_CK(cudaMemcpyAsync(count, P->ws + P->o_sat, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  if (reset) A2D_CK(cudaMemsetAsync(P->ws + P->o_sat, 0, sizeof(unsigned long long), s));
  A2D_CK(cudaStreamSynchronize(s));
  return A2D_OK;
}

int a2d_live_count(a2d_plan* P, int* n, void* stream) {
  A2D_BOUND(P);
  if (n == nullptr) return fail(A2D_ERR_ARG, "null output");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* dcount = P->at<int>(P->o_cnt);
  k_count<<<1, 256, 0, s>>>(P->ncases, P->ctl(), P->live(), P->p.retire, dcount);
  A2D_CK(cudaMemcpyAsync(P->host_count, dcount, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  A2D_CK(cudaStreamSynchronize(s));
  if (P->host_count[1] != 0) return fail(A2D_ERR_CUDA, "line sweep: a bulk-copy wait ran out of time");
  *n = *P->host_count;
  return A2D_OK;
}

int a2d_plan_stats(const a2d_plan* P, int* kernels_per_step, int* steps_taken, size_t* table_bytes) {
  if (P == nullptr) return fail(A2D_ERR_ARG, "null plan");
  if (kernels_per_step) *kernels_per_step = P->kernels_per_step;
  if (steps_taken) *steps_taken = P->steps_taken;
  if (table_bytes)
    *table_bytes = sizeof(CaseDev) * P->ncases + sizeof(Tile) * P->tiles.size() + sizeof(Chunk) * P->chunks.size() +
                   sizeof(Group) * P->groups.size() + sizeof(long long) * P->ncases;
  return A2D_OK;
}

int a2d_time_kernel(a2d_plan* P, int which, int reps, float* ms, void* stream) {
  A2D_BOUND(P);
  if (ms == nullptr || reps < 1) return fail(A2D_ERR_ARG, "time_kernel: bad arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Batch B = P->batch;
  B.live = nullptr;
  const bool mixed = P->p.precision == A2D_MIXED;
  const size_t vs = 4 * (size_t)P->C;
  const int half = std::max(1, P->m / 2);
  auto launch_once = [&]() {
    switch (which) {
      case A2D_K_JVP: {
        if (mixed) {
          StencilArgs<Basis16> a;
          a.U = P->vec(kU);
          a.V = P->at<Basis16>(P->o_V);
          a.diag = P->at<double>(P->o_diag);
          a.out = P->vec(kZ);
          a.lim_k = P->p.lim_k;
          a.order = P->p.order;
          a.vortex = P->p.vortex_correction;
          Batch jb = P->jbatch;
          jb.live = nullptr;
          launch_stencil<float, true, Basis16>(jb, a, s, P->jvp_tile);
        } else {
          StencilArgs<double> a = residual_args(P);
          a.V = P->at<double>(P->o_V);
          a.diag = P->at<double>(P->o_diag);
          a.out = P->vec(kZ);
          launch_stencil<double, true, double>(B, a, s);
        }
        break;
      }
      case A2D_K_SWEEP: {
        SweepArgs a = sweep_args(P, 0);
        a.e0 = P->vec(kPE);
        a.xprev = P->vec(kPB);
        a.x = P->vec(kPA);
        if (mixed) launch_sweep<float, false>(B, a, false, s, P->sweep_variant);
        else launch_sweep<double, false>(B, a, false, s, P->sweep_variant);
        break;
      }
      case A2D_K_SWEEP_FIRST: {
        SweepArgs a = sweep_args(P, 0);
        a.r = P->vec(kZ);
        a.e0 = P->vec(kPE);
        a.x = P->vec(kPA);
        if (mixed) launch_sweep<float, true>(B, a, false, s, P->sweep_variant);
        else launch_sweep<double, true>(B, a, false, s, P->sweep_variant);
        break;
      }
      case A2D_K_DOTS:
      case A2D_K_UPDATE:
      case A2D_K_PROJECT: {
        // Gram-Schmidt passes with restart/2 basis vectors; the output vector is a
        // scratch slot past the ones read
        auto run = [&](auto* Vb) {
          using TB = std::remove_pointer_t<decltype(Vb)>;
          GsArgs<TB> g;
          g.err = P->at<uint32_t>(P->o_cnt) + 1;
          g.w = P->vec(kW);
          g.V = Vb;
          g.vstride = vs;
          g.nq = half;
          g.with_norm = 1;
          g.part = P->at<double>(P->o_cpart);
          g.pstride = P->pstride;
          g.h1 = P->at<double>(P->o_h1);
          g.h2 = P->at<double>(P->o_h2);
          g.scale = P->at<double>(P->o_scale);
          g.Vout = Vb + (size_t)P->m * vs;
          g.part_norm = P->at<double>(P->o_cpartn);
          g.tmp = P->vec(kPB);
          if (which == A2D_K_DOTS) launch_gs_dots<TB>(B, g, s);
          else if (which == A2D_K_PROJECT) launch_gs_project<TB>(B, g, s);
          else launch_gs_finish<TB>(B, g, s);
        };
        if (mixed) run(P->at<Basis16>(P->o_V));
        else run(P->at<double>(P->o_V));
        break;
      }
      case A2D_K_RESIDUAL: {
        StencilArgs<double> a = residual_args(P);
        a.out = P->vec(kPA);
        a.sign = -1.0;
        a.circ_out = P->at<double>(P->o_circ);
        a.tile_part = P->at<double>(P->o_tpart);
        launch_stencil<double, false, double>(B, a, s);
        break;
      }
      case A2D_K_FACEJAC:
      case A2D_K_FACTOR: {
        JacArgs ja;
        ja.U = P->vec(kU);
        ja.circ = P->at<double>(P->o_circ);
        ja.JIL = P->at<void>(P->o_JIL);
        ja.JIR = P->at<void>(P->o_JIR);
        ja.JJL = P->at<void>(P->o_JJL);
        ja.JJR = P->at<void>(P->o_JJR);
        ja.vortex = P->p.vortex_correction;
        if (which == A2D_K_FACEJAC) {
          if (mixed) launch_face_jac<float>(B, ja, s);
          else launch_face_jac<double>(B, ja, s);
        } else {
          const FactorArgs fa = factor_args(P, 0);
          if (mixed) launch_factor<float, __half>(B, fa, s);
          else launch_factor<double, double>(B, fa, s);
        }
        break;
      }
      default:
        break;
    }
  };
  if (which < 0 || which > A2D_K_PROJECT) return fail(A2D_ERR_ARG, "time_kernel: unknown kernel");
  cudaEvent_t e0, e1;
  A2D_CK(cudaEventCreate(&e0));
  A2D_CK(cudaEventCreate(&e1));
  launch_once();   // warm-up launch
  A2D_CK(cudaEventRecord(e0, s));
  for (int q = 0; q < reps; ++q) launch_once();
  A2D_CK(cudaEventRecord(e1, s));
  A2D_CK(cudaEventSynchronize(e1));
  float t = 0.f;
  A2D_CK(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  A2D_CK(cudaGetLastError());
  *ms = t / reps;
  return A2D_OK;
}

int a2d_case_status(const a2d_plan* P, int* nsteps, int* done, int* frozen, double* lastrn, double* r0,
                    void* stream) {
  A2D_BOUND(P);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<CaseCtl> h(P->ncases);
  A2D_CK(cudaMemcpyAsync(h.data(), P->ctl(), sizeof(CaseCtl) * P->ncases, cudaMemcpyDeviceToHost, s));
  A2D_CK(cudaStreamSynchronize(s));
  for (int k = 0; k < P->ncases; ++k) {
    if (nsteps) nsteps[k] = h[k].nsteps;
    if (done) done[k] = h[k].done;
    if (frozen) frozen[k] = h[k].frozen;
    if (lastrn) lastrn[k] = h[k].lastrn;
    if (r0) r0[k] = h[k].r0;
  }
  return A2D_OK;
}

int a2d_case_scalars(const a2d_plan* P, double* out, void* stream) {
  A2D_BOUND(P);
  if (out == nullptr) return fail(A2D_ERR_ARG, "null output");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<CaseCtl> h(P->ncases);
  std::vector<double> circ(P->ncases);
  A2D_CK(cudaMemcpyAsync(h.data(), P->ctl(), sizeof(CaseCtl) * P->ncases, cudaMemcpyDeviceToHost, s));
  A2D_CK(cudaMemcpyAsync(circ.data(), P->at<double>(P->o_circ), 8 * (size_t)P->ncases, cudaMemcpyDeviceToHost, s));
  A2D_CK(cudaStreamSynchronize(s));
  for (int k = 0; k < P->ncases; ++k) {
    double* o = out + 8 * (size_t)k;
    o[0] = h[k].rn;
    o[1] = h[k].omega;
    o[2] = h[k].cfl;
    o[3] = h[k].r0;
    o[4] = circ[k];
    o[5] = h[k].beta;
    o[6] = (double)h[k].k_used;
    o[7] = (double)h[k].commit;
  }
  return A2D_OK;
}

int a2d_history(const a2d_plan* P, int steps, double* rn, double* cl, void* stream) {
  A2D_BOUND(P);
  if (steps < 0 || steps > P->p.max_iter) return fail(A2D_ERR_ARG, "history: steps out of range");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t n = (size_t)steps * P->ncases * 8;
  if (rn != nullptr && n) A2D_CK(cudaMemcpyAsync(rn, P->at<double>(P->o_hrn), n, cudaMemcpyDeviceToHost, s));
  if (cl != nullptr && n) A2D_CK(cudaMemcpyAsync(cl, P->at<double>(P->o_hcl), n, cudaMemcpyDeviceToHost, s));
  A2D_CK(cudaStreamSynchronize(s));
  return A2D_OK;
}

int a2d_set_circulation(a2d_plan* P, const double* circ, void* stream) {
  A2D_BOUND(P);
  if (circ == nullptr) return fail(A2D_ERR_ARG, "null circulation");
  A2D_CK(cudaMemcpyAsync(P->at<double>(P->o_circ_rk), circ, 8 * (size_t)P->ncases, cudaMemcpyHostToDevice,
                         static_cast<cudaStream_t>(stream)));
  return A2D_OK;
}

int a2d_smooth(a2d_plan* P, void* stream) {
  A2D_BOUND(P);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Batch B = P->batch;
  B.live = nullptr;
  launch_irs(B, P->vec(kR), P->vec(kPA), P->p.irs_eps, P->max_ni, P->max_nc, P->p.precision == A2D_MIXED, s);
  if (P->p.irs_eps > 0)
    A2D_CK(cudaMemcpyAsync(P->vec(kR), P->vec(kPA), 8 * 4 * (size_t)P->C, cudaMemcpyDeviceToDevice, s));
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_plan_set_coarse(a2d_plan* P, a2d_plan* coarse) {
  if (P == nullptr) return fail(A2D_ERR_ARG, "null plan");
  if (coarse != nullptr) {
    if (coarse == P || coarse->ncases != P->ncases) return fail(A2D_ERR_ARG, "set_coarse: not the same cases");
    for (int k = 0; k < P->ncases; ++k) {
      const GridDev& f = P->cases[k].g;
      const GridDev& c = coarse->cases[k].g;
      if (f.ni % 2 || f.nc % 2 || c.ni * 2 != f.ni || c.nc * 2 != f.nc)
        return fail(A2D_ERR_ARG, "set_coarse: the coarse grids must have ni/2 x nc/2 cells (even ni, nc)");
    }
    for (const a2d_plan* q = coarse; q != nullptr; q = q->coarse)
      if (q == P) return fail(A2D_ERR_ARG, "set_coarse: the levels would form a cycle");
  }
  P->coarse = coarse;
  return A2D_OK;
}

}  // extern "C"

namespace a2d {

// one 4-stage RK iteration of plan P (aero2d/euler.py:334-346): residual at the
// circulation circ (per case), plus the FAS forcing when given, smoothed, stage update
static cudaError_t rk_iter(a2d_plan* P, const double* circ, const double* forcing, cudaStream_t s) {
  Batch B = P->batch;
  B.live = nullptr;
  double* U = P->vec(kU);
  double* U0 = P->vec(kU0);
  double* R = P->vec(kR);
  double* Rs = P->vec(kPA);
  double* dt = P->at<double>(P->o_dt);
  const double alphas[4] = {0.25, 1.0 / 3.0, 0.5, 1.0};
  // dtype=float32: residual, local time steps, smoothing and stage update in FP32
  // (the reference casts its whole explicit iteration to the solver dtype,
  // aero2d/euler.py:222-234); the state keeps FP32-rounded values in FP64 storage
  const bool fp32 = P->p.precision == A2D_MIXED;
  if (cudaError_t e = cudaMemcpyAsync(U0, U, 8 * 4 * (size_t)P->C, cudaMemcpyDeviceToDevice, s)) return e;
  launch_local_dt(B, U, dt, P->p.cfl, fp32, s);
  for (int st = 0; st < 4; ++st) {
    StencilArgs<double> a = residual_args(P);
    a.circ_in = circ;
    a.out = R;
    a.sign = 1.0;
    if (fp32) launch_stencil<float, false, double>(B, a, s);
    else launch_stencil<double, false, double>(B, a, s);
    if (forcing != nullptr) launch_add_forcing(B, R, forcing, s);
    const double* Ruse = R;
    if (P->p.irs_eps > 0) {
      launch_irs(B, R, Rs, P->p.irs_eps, P->max_ni, P->max_nc, fp32, s);
      Ruse = Rs;
    }
    launch_rk_stage(B, U0, Ruse, dt, U, alphas[st], fp32, s);
  }
  return cudaGetLastError();
}

// one FAS V-cycle from plan P down (aero2d/euler.py:368-381); at the top level
// the pseudo-time residual of the first iteration goes to the tile partials
static cudaError_t fas_cycle(a2d_plan* P, const double* circ, const double* forcing, bool top, cudaStream_t s) {
  Batch B = P->batch;
  B.live = nullptr;
  if (cudaError_t e = rk_iter(P, circ, forcing, s)) return e;
  if (top) launch_rk_res(B, P->vec(kU0), P->vec(kU), P->at<double>(P->o_dt), P->at<double>(P->o_tpart), s);
  a2d_plan* Cp = P->coarse;
  if (Cp == nullptr) return cudaGetLastError();
  Batch CB = Cp->batch;
  CB.live = nullptr;
  // fine residual (plus this level's forcing) at the smoothed state
  StencilArgs<double> a = residual_args(P);
  a.circ_in = circ;
  a.out = P->vec(kR);
  a.sign = 1.0;
  if (P->p.precision == A2D_MIXED) launch_stencil<float, false, double>(B, a, s);
  else launch_stencil<double, false, double>(B, a, s);
  if (forcing != nullptr) launch_add_forcing(B, P->vec(kR), forcing, s);
  // coarse start state Uc0 (kept in the coarse plan's JV slot) and forcing (its V slot)
  double* Uc = Cp->vec(kU);
  double* Uc0 = Cp->vec(kJV);
  double* Pc = Cp->vec(kVin);
  launch_fas_restrict(B, CB, P->vec(kU), Uc, Uc0, s);
  StencilArgs<double> ca = residual_args(Cp);
  ca.circ_in = circ;
  ca.out = Pc;
  ca.sign = 1.0;
  if (Cp->p.precision == A2D_MIXED) launch_stencil<float, false, double>(CB, ca, s);
  else launch_stencil<double, false, double>(CB, ca, s);
  launch_fas_forcing(B, CB, P->vec(kR), Pc, s);
  if (cudaError_t e = fas_cycle(Cp, circ, Pc, false, s)) return e;
  launch_fas_prolong(B, CB, P->vec(kU), Uc, Uc0, s);
  return rk_iter(P, circ, forcing, s);
}

}  // namespace a2d

extern "C" {

int a2d_rk_iterate(a2d_plan* P, int n, double* res, void* stream) {
  A2D_BOUND(P);
  Range range("a2d_rk_iterate");
  if (n < 0) return fail(A2D_ERR_ARG, "negative iteration count");
  for (const a2d_plan* q = P->coarse; q != nullptr; q = q->coarse)
    if (q->ws == nullptr) return fail(A2D_ERR_STATE, "rk_iterate: a coarse level is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Batch B = P->batch;
  B.live = nullptr;
  double* circ = P->at<double>(P->o_circ_rk);
  double* tpart = P->at<double>(P->o_tpart);
  for (int it = 0; it < n; ++it) {
    A2D_CK(fas_cycle(P, circ, nullptr, true, s));
    launch_forces(B, P->vec(kU), P->at<double>(P->o_coef), P->at<double>(P->o_cp), P->at<long long>(P->o_cpoff), nullptr,
                  nullptr, 0, s);
    launch_rk_finish(B, tpart, P->at<double>(P->o_coef), (it == n - 1) ? res : nullptr, circ, s);
  }
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

int a2d_hllc_flux(int n, const double* WL, const double* WR, const double* S, double* F, void* stream) {
  if (n < 0 || (n > 0 && (WL == nullptr || WR == nullptr || S == nullptr || F == nullptr)))
    return fail(A2D_ERR_ARG, "hllc_flux: bad arguments");
  if (n == 0) return A2D_OK;
  k_point_flux<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(n, WL, WR, S, F);
  A2D_CK(cudaGetLastError());
  return A2D_OK;
}

}  // extern "C"
