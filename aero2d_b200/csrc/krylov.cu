// GMRES and Newton-update kernels of the pseudo-transient Newton-Krylov solver
// (aero2d/implicit.py:169-253 and the jax.scipy.sparse.linalg.gmres cycle it
// calls with restart=m, maxiter=1, solve_method="batched").
//
// Every reduction is per case and runs in a fixed order: each CTA writes the
// partial sum of its chunk (or tile), and every consumer sums the partials of
// its case in chunk order.  A case's results therefore do not depend on which
// other cases share the batch.  Gram-Schmidt arithmetic, Hessenberg least
// squares, norms and the state update are FP64; the Krylov basis is stored as
// TB (FP64, or FP32 in the mixed-precision mode).
#include <cfloat>
#include <cuda_bf16.h>

#include "batch.cuh"
#include "krylov.cuh"
#include "physics.cuh"

namespace a2d {

template <typename T, int NV>
__device__ __forceinline__ void block_sum_k(T (&v)[NV], T* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) scratch[warp * NV + q] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    T s = T(0);
    for (int w = 0; w < nw; ++w) s += scratch[w * NV + q];
    v[q] = s;
  }
  __syncthreads();
}

// NaN-propagating maximum (jnp.max semantics)
__device__ __forceinline__ double nmax(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  return a > b ? a : b;
}

__device__ __forceinline__ void block_max(double& v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double s = scratch[0];
  for (int w = 1; w < nw; ++w) s = nmax(s, scratch[w]);
  v = s;
  __syncthreads();
}

constexpr int kVB = 256;                 // threads per vector block
constexpr int kPer = kChunk / kVB;       // entries per thread

// ---------------------------------------------------------------------------
// Hessenberg least squares min || beta e1 - H y || by Givens rotations (H
// column k = Arnoldi step k).  One warp per case copies the case's columns
// into shared memory; its first lane then rotates and back-substitutes there
// (a sequential chain of dependent updates: in shared memory each costs a few
// tens of cycles instead of a global-memory round trip).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32) k_lstsq(int ncases, const uint32_t* live, CaseCtl* ctl, const double* Hall,
                                              double* yall) {
  const int cs = blockIdx.x;
  if (!(live[cs] & kLiveNewton)) return;
  const int k = ctl[cs].k_used;
  if (k == 0) return;
  constexpr int L = kMaxRestart + 1;
  __shared__ double Hc[kMaxRestart * L];   // column j at Hc[j * L + q]; rotated in place
  __shared__ double g[L], cr[L], sr[L];
  const double* Hg = Hall + (size_t)cs * kMaxRestart * L;
  for (int e = threadIdx.x; e < k * L; e += blockDim.x) Hc[e] = Hg[e];
  __syncthreads();
  if (threadIdx.x != 0) return;
  double* y = yall + (size_t)cs * kMaxRestart;
  for (int q = 0; q <= k; ++q) g[q] = 0.0;
  g[0] = ctl[cs].beta;
  for (int j = 0; j < k; ++j) {
    double* col = Hc + (size_t)j * L;
    for (int q = 0; q < j; ++q) {
      const double t = cr[q] * col[q] + sr[q] * col[q + 1];
      col[q + 1] = -sr[q] * col[q] + cr[q] * col[q + 1];
      col[q] = t;
    }
    const double a = col[j], c = col[j + 1];
    const double d = hypot(a, c);
    double cc = 1.0, ss = 0.0;
    if (d != 0.0) {
      cc = a / d;
      ss = c / d;
    }
    cr[j] = cc;
    sr[j] = ss;
    col[j] = cc * a + ss * c;
    col[j + 1] = 0.0;
    const double gj = g[j], gj1 = g[j + 1];
    g[j] = cc * gj + ss * gj1;
    g[j + 1] = -ss * gj + cc * gj1;
  }
  for (int i = k - 1; i >= 0; --i) {
    double s = g[i];
    for (int j = i + 1; j < k; ++j) s -= Hc[(size_t)j * L + i] * y[j];
    const double rii = Hc[(size_t)i * L + i];
    y[i] = rii != 0.0 ? s / rii : 0.0;
  }
}

// dU = x0 + V y
// one basis entry in FP64
__device__ __forceinline__ double basis_f64(double v) { return v; }
__device__ __forceinline__ double basis_f64(float v) { return v; }
__device__ __forceinline__ double basis_f64(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename TB>
__global__ void __launch_bounds__(kVB) k_combine(Batch b, CombineArgs<TB> a) {
  const Chunk ch = b.chunks[blockIdx.x];
  if (!case_live(b, ch.cs, a.need)) return;
  const CaseDev cs = b.cases[ch.cs];
  const size_t base = 4 * cs.cell_off + ch.begin;
  const int k = a.ctl[ch.cs].k_used;
  const double* y = a.y + (size_t)ch.cs * kMaxRestart;
  __shared__ double ys[kMaxRestart];
  // raw basis vectors carry their normalisation in scale[q][case]
  for (int q = threadIdx.x; q < k; q += blockDim.x) ys[q] = y[q] * a.scale[(size_t)q * b.ncases + ch.cs];
  __syncthreads();
#pragma unroll
  for (int s = 0; s < kPer; ++s) {
    const int e = threadIdx.x + s * kVB;
    if (e < ch.len) {
      double acc = 0.0;
      for (int q = 0; q < k; ++q) acc += basis_f64(a.V[(size_t)q * a.vstride + base + e]) * ys[q];
      a.out[base + e] = a.x0[base + e] + acc;
    }
  }
}

// per-case norms of b and x0 -> ptol (jax gmres: ptol = ||M b|| * min(1, tol ||b|| / ||b||))
__global__ void k_gm_setup(Batch b, const double* part, int pstride, CaseCtl* ctl, double gtol) {
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= b.ncases) return;
  if (!case_live(b, cs, kLiveNewton)) return;
  const CaseDev c = b.cases[cs];
  double sb = 0.0, sx = 0.0;
  for (int q = 0; q < c.nchunks; ++q) {
    sb += part[(size_t)(c.chunk0 + q) * pstride + 0];
    sx += part[(size_t)(c.chunk0 + q) * pstride + 1];
  }
  const double bn = sqrt(sb), xn = sqrt(sx);
  ctl[cs].bnorm = bn;
  ctl[cs].x0norm = xn;
  const double atol = fmax(gtol * bn, 0.0);
  ctl[cs].ptol = bn > 0.0 ? xn * fmin(1.0, atol / bn) : 0.0;
}

// two squared norms per chunk (||b||^2, ||x0||^2)
__global__ void __launch_bounds__(kVB) k_norms2(Batch b, const double* x, const double* y, double* part,
                                                int pstride, uint32_t need) {
  const Chunk ch = b.chunks[blockIdx.x];
  if (!case_live(b, ch.cs, need)) return;
  const CaseDev cs = b.cases[ch.cs];
  const size_t base = 4 * cs.cell_off + ch.begin;
  __shared__ double scratch[64];
  double acc[2] = {0.0, 0.0};
  for (int e = threadIdx.x; e < ch.len; e += blockDim.x) {
    const double u = x[base + e], v = y[base + e];
    acc[0] += u * u;
    acc[1] += v * v;
  }
  block_sum_k<double, 2>(acc, scratch);
  if (threadIdx.x == 0) {
    part[(size_t)blockIdx.x * pstride + 0] = acc[0];
    part[(size_t)blockIdx.x * pstride + 1] = acc[1];
  }
}

// squared norm per chunk
__global__ void __launch_bounds__(kVB) k_norm1(Batch b, const double* x, double* part, uint32_t need) {
  const Chunk ch = b.chunks[blockIdx.x];
  if (!case_live(b, ch.cs, need)) return;
  const CaseDev cs = b.cases[ch.cs];
  const size_t base = 4 * cs.cell_off + ch.begin;
  __shared__ double scratch[32];
  double acc[1] = {0.0};
  for (int e = threadIdx.x; e < ch.len; e += blockDim.x) acc[0] += x[base + e] * x[base + e];
  block_sum_k<double, 1>(acc, scratch);
  if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

// ---------------------------------------------------------------------------
// Newton update (aero2d/implicit.py:186-192) and the per-case host-loop logic
// of aero2d/implicit.py:216-244, both on the device
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_update_rel(Batch b, const double* U, const double* dU,
                                                    double* tpart, uint32_t need) {
  const Tile t = b.tiles[blockIdx.x];
  if (!case_live(b, t.cs, need)) return;
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  const size_t base = 4 * cs.cell_off;
  double m = 0.0;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
    State4<double> u, un;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t q = base + vidx(g, k, j, i);
      u.c[k] = U[q];
      un.c[k] = U[q] + dU[q];
    }
    const State4<double> W = cons_to_prim<double, double>(u);
    const State4<double> Wn = cons_to_prim<double, double>(un);
    m = nmax(m, fabs(Wn.c[0] - W.c[0]) / W.c[0]);
    m = nmax(m, fabs(Wn.c[3] - W.c[3]) / W.c[3]);
  }
  __shared__ double scratch[32];
  block_max(m, scratch);
  if (threadIdx.x == 0) tpart[(size_t)blockIdx.x * kTilePartStride + 1] = m;
}

__global__ void __launch_bounds__(256) k_update_check(Batch b, const double* U, const double* dU,
                                                      double* tpart, CaseCtl* ctl, double max_update,
                                                      uint32_t need) {
  const Tile t = b.tiles[blockIdx.x];
  if (!case_live(b, t.cs, need)) return;
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  double rel = 0.0;
  for (int q = 0; q < cs.ntiles; ++q) {
    const double v = tpart[(size_t)(cs.tile0 + q) * kTilePartStride + 1];
    rel = q == 0 ? v : nmax(rel, v);
  }
  double omega = max_update / (rel + 1e-30);
  omega = (omega != omega) ? omega : (omega < 1.0 ? omega : 1.0);
  const size_t base = 4 * cs.cell_off;
  double bad = 0.0;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t q = base + vidx(g, k, j, i);
      const double un = U[q] + omega * dU[q];
      if (!isfinite(un)) bad = 1.0;
    }
  }
  double v[1] = {bad};
  __shared__ double scratch[32];
  block_sum_k<double, 1>(v, scratch);
  if (threadIdx.x == 0) {
    tpart[(size_t)blockIdx.x * kTilePartStride + 2] = v[0];
    if (blockIdx.x == cs.tile0) ctl[t.cs].omega = omega;
  }
}

__global__ void k_controller(Batch b, const double* tpart, CaseCtl* ctl, uint32_t* live, double* hist_rn,
                             int hist_cap, CtlParams p) {
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= b.ncases) return;
  if (!(live[cs] & kLiveNewton)) return;
  const CaseDev c = b.cases[cs];
  CaseCtl& s = ctl[cs];
  double sr = 0.0, nbad = 0.0;
  for (int q = 0; q < c.ntiles; ++q) {
    sr += tpart[(size_t)(c.tile0 + q) * kTilePartStride + 0];
    nbad += tpart[(size_t)(c.tile0 + q) * kTilePartStride + 2];
  }
  const double N = (double)c.g.ni * (double)c.g.nc;
  const double rn = sqrt(sr / N);
  const bool finite = isfinite(rn) && nbad == 0.0;
  const bool bad = !finite || s.frozen;
  if (!finite) s.fails += 1;
  if (s.fails >= 5) s.frozen = 1;
  s.commit = bad ? 0 : 1;
  const double rnr = finite ? rn : NAN;
  if (s.nsteps == 0 && !s.keep_r0) s.r0 = isfinite(rnr) ? fmax(rnr, 1e-30) : 1.0;
  const double den = isfinite(rnr) ? fmax(rnr, 1e-30) : s.r0;
  const double ser = p.cfl0 * (s.r0 / den);
  double cfl = fmin(fmax(ser, p.cfl0), p.cfl_max);
  if (s.omega < 1.0) cfl = fmax(cfl * 0.5, 1.0);
  if (!finite) cfl = 1.0;
  s.cfl = cfl;
  s.rn = rnr;
  if (finite) s.lastrn = rnr;
  if (s.nsteps < hist_cap) hist_rn[(size_t)s.nsteps * b.ncases + cs] = rnr;
  const bool done = (rnr / s.r0 < p.tol) || s.frozen;
  s.done = done ? 1 : 0;
  s.nsteps += 1;
  if (done && p.retire) live[cs] &= ~kLiveNewton;
}

__global__ void __launch_bounds__(256) k_commit(Batch b, double* U, const double* dU, const CaseCtl* ctl,
                                                uint32_t need_mask_unused) {
  const Tile t = b.tiles[blockIdx.x];
  const CaseCtl& s = ctl[t.cs];
  if (!s.commit || !s.stepped) return;
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  const size_t base = 4 * cs.cell_off;
  const double omega = s.omega;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t q = base + vidx(g, k, j, i);
      U[q] = U[q] + omega * dU[q];
    }
  }
}

// marks which cases take this step (before the controller may retire them)
__global__ void k_mark_stepped(int ncases, const uint32_t* live, CaseCtl* ctl) {
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= ncases) return;
  ctl[cs].stepped = (live[cs] & kLiveNewton) ? 1 : 0;
  ctl[cs].commit = 0;
}

// ---------------------------------------------------------------------------
// launchers
template <typename TB>
void launch_combine(const Batch& b, const CombineArgs<TB>& a, cudaStream_t s) {
  if (b.nchunks) k_combine<TB><<<b.nchunks, kVB, 0, s>>>(b, a);
}
void launch_lstsq(const Batch& b, const uint32_t* live, CaseCtl* ctl, double* H, double* y, cudaStream_t s) {
  k_lstsq<<<b.ncases, 32, 0, s>>>(b.ncases, live, ctl, H, y);
}
void launch_gm_setup(const Batch& b, const double* part, int pstride, CaseCtl* ctl, double gtol,
                     cudaStream_t s) {
  k_gm_setup<<<(b.ncases + 63) / 64, 64, 0, s>>>(b, part, pstride, ctl, gtol);
}
void launch_norms2(const Batch& b, const double* x, const double* y, double* part, int pstride,
                   uint32_t need, cudaStream_t s) {
  if (b.nchunks) k_norms2<<<b.nchunks, kVB, 0, s>>>(b, x, y, part, pstride, need);
}
void launch_norm1(const Batch& b, const double* x, double* part, uint32_t need, cudaStream_t s) {
  if (b.nchunks) k_norm1<<<b.nchunks, kVB, 0, s>>>(b, x, part, need);
}
void launch_update_rel(const Batch& b, const double* U, const double* dU, double* tpart, uint32_t need,
                       cudaStream_t s) {
  if (b.ntiles) k_update_rel<<<b.ntiles, 256, 0, s>>>(b, U, dU, tpart, need);
}
void launch_update_check(const Batch& b, const double* U, const double* dU, double* tpart, CaseCtl* ctl,
                         double max_update, uint32_t need, cudaStream_t s) {
  if (b.ntiles) k_update_check<<<b.ntiles, 256, 0, s>>>(b, U, dU, tpart, ctl, max_update, need);
}
void launch_controller(const Batch& b, const double* tpart, CaseCtl* ctl, uint32_t* live, double* hist_rn,
                       int hist_cap, const CtlParams& p, cudaStream_t s) {
  k_controller<<<(b.ncases + 63) / 64, 64, 0, s>>>(b, tpart, ctl, live, hist_rn, hist_cap, p);
}
void launch_commit(const Batch& b, double* U, const double* dU, const CaseCtl* ctl, cudaStream_t s) {
  if (b.ntiles) k_commit<<<b.ntiles, 256, 0, s>>>(b, U, dU, ctl, 0);
}
void launch_mark_stepped(const Batch& b, const uint32_t* live, CaseCtl* ctl, cudaStream_t s) {
  k_mark_stepped<<<(b.ncases + 63) / 64, 64, 0, s>>>(b.ncases, live, ctl);
}

template void launch_combine<double>(const Batch&, const CombineArgs<double>&, cudaStream_t);
template void launch_combine<float>(const Batch&, const CombineArgs<float>&, cudaStream_t);
template void launch_combine<__nv_bfloat16>(const Batch&, const CombineArgs<__nv_bfloat16>&, cudaStream_t);

}  // namespace a2d
