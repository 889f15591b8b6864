// The residual / JVP tile kernel and its helpers, shared by the translation
// units that instantiate it: stencil.cu (FP64, IEEE-exact arithmetic) and
// stencil_fp32.cu (the FP32 linearisation of the mixed-precision solver, built
// with approximate FP32 division and square root).  See stencil.cu for the
// description of the kernel.
#pragma once
#include <type_traits>

#include "batch.cuh"
#include "kernels.cuh"
#include "physics.cuh"

namespace a2d {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
template <typename T> struct Tangent { using type = T; };

template <typename S, typename T>
__device__ __forceinline__ void set_val(S& s, T v);
template <> __device__ __forceinline__ void set_val<double, double>(double& s, double v) { s = v; }
template <> __device__ __forceinline__ void set_val<float, float>(float& s, float v) { s = v; }

template <typename T, typename VT>
__device__ __forceinline__ State4<T> load_cons(const double* U, const GridDev& g, int j, int i) {
  State4<T> r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.c[k] = T(U[vidx(g, k, j, i)]);
  return r;
}

template <typename T, typename VT>
__device__ __forceinline__ State4<Dual<T, 1>> load_cons_dual(const double* U, const VT* V,
                                                             const GridDev& g, int j, int i) {
  State4<Dual<T, 1>> r;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const size_t q = vidx(g, k, j, i);
    r.c[k].v = T(U[q]);
    r.c[k].d[0] = T(V[q]);
  }
  return r;
}

// Fixed-order block reduction of NV values (all threads receive the result).
// Deterministic for a given blockDim, which is what makes a case's results
// independent of the other cases in the batch.
template <typename T, int NV>
__device__ __forceinline__ void block_sum(T (&v)[NV], T* scratch /* >= 32*NV */) {
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

// Circulation Gamma = 1/2 Cl M of one case from its wall rows, and with a
// tangent V its derivative (aero2d/implicit.py:160-164, euler.py:315-331).
// Called by all threads of the block.
template <typename T, bool LIN, typename VT>
__device__ void block_circulation(const CaseDev& cs, const double* U, const VT* V, T* scratch,
                                  T& circ, T& dcirc) {
  const GridDev& g = cs.g;
  Metric<T> m{g};
  const T uinf = T(cs.winf[1]), vinf = T(cs.winf[2]), pinf = T(cs.winf[3]);
  const T q = T(0.5) * (uinf * uinf + vinf * vinf);
  T acc[4] = {T(0), T(0), T(0), T(0)};
  for (int i = threadIdx.x; i < g.ni; i += blockDim.x) {
    if constexpr (LIN) {
      const State4<Dual<T, 1>> W0 = cons_to_prim<Dual<T, 1>, T>(load_cons_dual<T, VT>(U, V, g, 0, i));
      const State4<Dual<T, 1>> W1 = cons_to_prim<Dual<T, 1>, T>(load_cons_dual<T, VT>(U, V, g, 1, i));
      const Dual<T, 1> pw = T(1.5) * W0.c[3] - T(0.5) * W1.c[3];
      const Dual<T, 1> cp = (pw - pinf) / q;
      const T s0 = m.sj(0, 0, i), s1 = m.sj(1, 0, i);
      acc[0] += cp.v * s0;
      acc[1] += cp.v * s1;
      acc[2] += cp.d[0] * s0;
      acc[3] += cp.d[0] * s1;
    } else {
      const State4<T> W0 = cons_to_prim<T, T>(load_cons<T, VT>(U, g, 0, i));
      const State4<T> W1 = cons_to_prim<T, T>(load_cons<T, VT>(U, g, 1, i));
      const T pw = T(1.5) * W0.c[3] - T(0.5) * W1.c[3];
      const T cp = (pw - pinf) / q;
      acc[0] += cp * m.sj(0, 0, i);
      acc[1] += cp * m.sj(1, 0, i);
    }
  }
  block_sum<T, 4>(acc, scratch);
  const T mach = dsqrt(T(2) * q);
  const T ca = uinf / mach, sa = vinf / mach;
  const T fx = -acc[0], fy = -acc[1];
  const T cl = fy * ca - fx * sa;
  const T mach2 = dsqrt(uinf * uinf + vinf * vinf);
  circ = T(0.5) * cl * mach2;
  if (LIN) {
    const T dfx = -acc[2], dfy = -acc[3];
    const T dcl = dfy * ca - dfx * sa;
    dcirc = T(0.5) * dcl * mach2;
  } else {
    dcirc = T(0);
  }
}

// ---------------------------------------------------------------------------
// the fused residual / JVP tile kernel
// ---------------------------------------------------------------------------
template <typename T, bool LIN, typename VT, int TI, int TJ>
__device__ __forceinline__ void stencil_tile(const Batch& b, const StencilArgs<VT>& a, int tile) {
  using S = typename std::conditional<LIN, Dual<T, 1>, T>::type;
  constexpr int WI = TI + 4, WJ = TJ + 4;
  __shared__ S sW[4][WJ][WI];
  __shared__ T sFi[4][TJ][TI + 1];
  __shared__ T sFj[4][TJ + 1][TI];
  __shared__ T sred[32 * 4];
  __shared__ T sGam[2];

  const Tile t = b.tiles[tile];
  if (!case_live(b, t.cs, a.need)) return;
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  Metric<T> m{g};
  const int ni = g.ni, nc = g.nc;
  const double* U = a.U + 4 * cs.cell_off;
  const VT* V = LIN ? a.V + 4 * cs.cell_off : nullptr;

  const T rinf = T(cs.winf[0]), uinf = T(cs.winf[1]), vinf = T(cs.winf[2]), pinf = T(cs.winf[3]);
  T eps[4];
  {
    const T mach = dsqrt(uinf * uinf + vinf * vinf);
    const T sc[4] = {rinf, mach, mach, pinf};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const T e = T(a.lim_k) * sc[k];
      eps[k] = e * e;
    }
  }

  // circulation for the far-field ghosts of this tile (fixed-order reduction)
  const bool touches_far = t.j0 + t.tj + 2 > nc;
  if (touches_far) {
    T gam = T(0), dgam = T(0);
    if (a.circ_in != nullptr && !LIN) {
      gam = T(a.circ_in[t.cs]);
    } else {
      block_circulation<T, LIN, VT>(cs, U, V, sred, gam, dgam);
    }
    if (!a.vortex) {
      gam = T(0);
      dgam = T(0);
    }
    if (threadIdx.x == 0) {
      sGam[0] = gam;
      sGam[1] = dgam;
      if (!LIN && a.circ_out != nullptr && t.i0 == 0) a.circ_out[t.cs] = (double)gam;
    }
  }
  __syncthreads();

  // stage primitive states with halo and ghosts
  const int wr = t.tj + 4, wc = t.ti + 4;
  for (int idx = threadIdx.x; idx < wr * wc; idx += blockDim.x) {
    const int r = idx / wc, c = idx % wc;
    const int gj = t.j0 + r - 2;
    int gi = t.i0 + c - 2;
    gi = gi < 0 ? gi + ni : (gi >= ni ? gi - ni : gi);
    State4<S> W;
    if (gj >= 0 && gj < nc) {
      if constexpr (LIN) W = cons_to_prim<S, T>(load_cons_dual<T, VT>(U, V, g, gj, gi));
      else W = cons_to_prim<S, T>(load_cons<T, VT>(U, g, gj, gi));
    } else if (gj < 0) {
      State4<S> Wi;
      if constexpr (LIN) Wi = cons_to_prim<S, T>(load_cons_dual<T, VT>(U, V, g, -1 - gj, gi));
      else Wi = cons_to_prim<S, T>(load_cons<T, VT>(U, g, -1 - gj, gi));
      W = wall_mirror<S, T>(Wi, m.sj(0, 0, gi), m.sj(1, 0, gi));
    } else {
      State4<S> Wi;
      if constexpr (LIN) Wi = cons_to_prim<S, T>(load_cons_dual<T, VT>(U, V, g, nc - 1, gi));
      else Wi = cons_to_prim<S, T>(load_cons<T, VT>(U, g, nc - 1, gi));
      S circ;
      if constexpr (LIN) {
        circ.v = sGam[0];
        circ.d[0] = sGam[1];
      } else {
        circ = sGam[0];
      }
      W = farfield_ghost<S, T>(Wi, m.sj(0, nc, gi), m.sj(1, nc, gi), rinf, uinf, vinf, pinf,
                               m.xf(gi), m.yf(gi), circ);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) sW[k][r][c] = W.c[k];
  }
  __syncthreads();

  // face fluxes: i-faces (tj rows x ti+1 faces), then j-faces (tj+1 faces x ti columns)
  const int nfi = t.tj * (t.ti + 1);
  const int nfj = (t.tj + 1) * t.ti;
  const bool second = a.order == 2;
  for (int f = threadIdx.x; f < nfi + nfj; f += blockDim.x) {
    State4<S> Wm, W0, Wp, Wpp;
    T sx, sy;
    if (f < nfi) {
      const int jl = f / (t.ti + 1), fl = f % (t.ti + 1);
      const int r = jl + 2;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        Wm.c[k] = sW[k][r][fl];
        W0.c[k] = sW[k][r][fl + 1];
        Wp.c[k] = sW[k][r][fl + 2];
        Wpp.c[k] = sW[k][r][fl + 3];
      }
      int fi = t.i0 + fl;
      if (fi >= ni) fi -= ni;
      sx = m.si(0, t.j0 + jl, fi);
      sy = m.si(1, t.j0 + jl, fi);
      State4<S> WL, WR;
      recon<S, T>(Wm, W0, Wp, Wpp, eps, second, WL, WR);
      const State4<S> F = hllc<S, T>(WL, WR, sx, sy);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if constexpr (LIN) sFi[k][jl][fl] = F.c[k].d[0];
        else sFi[k][jl][fl] = F.c[k];
      }
    } else {
      const int f2 = f - nfi;
      const int fl = f2 / t.ti, il = f2 % t.ti;
      const int c = il + 2;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        Wm.c[k] = sW[k][fl][c];
        W0.c[k] = sW[k][fl + 1][c];
        Wp.c[k] = sW[k][fl + 2][c];
        Wpp.c[k] = sW[k][fl + 3][c];
      }
      sx = m.sj(0, t.j0 + fl, t.i0 + il);
      sy = m.sj(1, t.j0 + fl, t.i0 + il);
      State4<S> WL, WR;
      recon<S, T>(Wm, W0, Wp, Wpp, eps, second, WL, WR);
      const State4<S> F = hllc<S, T>(WL, WR, sx, sy);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if constexpr (LIN) sFj[k][fl][il] = F.c[k].d[0];
        else sFj[k][fl][il] = F.c[k];
      }
    }
  }
  __syncthreads();

  // cell residuals and epilogue
  double part = 0.0;
  const size_t base = 4 * cs.cell_off;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int jl = c / t.ti, il = c % t.ti;
    const int gj = t.j0 + jl, gi = t.i0 + il;
    T R[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
      R[k] = (sFi[k][jl][il + 1] - sFi[k][jl][il]) + (sFj[k][jl + 1][il] - sFj[k][jl][il]);
    if constexpr (LIN) {
      const T dg = a.diag != nullptr ? T(a.diag[cs.cell_off + (size_t)gj * ni + gi]) : T(0);
      // the product is linear in V: a raw Krylov vector's scale applies to the result
      const T vs = a.vscale != nullptr ? T(a.vscale[t.cs]) : T(1);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const size_t q = vidx(g, k, gj, gi);
        T y = (a.diag != nullptr ? dg * T(V[q]) + R[k] : R[k]) * vs;
        if (a.bvec != nullptr) y = T(a.bvec[base + q]) - y;
        a.out[base + q] = (double)y;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) a.out[base + vidx(g, k, gj, gi)] = a.sign * (double)R[k];
      const double rv = (double)R[0] / g.vol[(size_t)gj * ni + gi];
      part += rv * rv;
    }
  }
  if constexpr (!LIN) {
    if (a.tile_part != nullptr) {
      double v[1] = {part};
      __shared__ double sredd[32];
      block_sum<double, 1>(v, sredd);
      if (threadIdx.x == 0) a.tile_part[(size_t)tile * kTilePartStride] = v[0];
    }
  }
}

// Persistent: the grid is at most the CTAs resident on the GPU, and each CTA
// walks the batch's tile list (every case's tiles, whatever their grid size)
// with a stride of the grid size.  TI x TJ is the tile shape of that list.
template <typename T, bool LIN, typename VT, int TI, int TJ>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 1) k_stencil(Batch b, StencilArgs<VT> a) {
  for (int tile = blockIdx.x; tile < b.ntiles; tile += gridDim.x) {
    if (tile != (int)blockIdx.x) __syncthreads();   // the previous tile is done with shared memory
    stencil_tile<T, LIN, VT, TI, TJ>(b, a, tile);
  }
}

// CTAs of a persistent stencil launch: the tiles, at most the CTAs of kernel f
// resident at once on the current device (its occupancy times the SMs)
inline int persistent_grid(const void* f, int threads, int items) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    sms = 148;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, threads, 0) != cudaSuccess || per_sm <= 0)
    per_sm = 1;
  const long long cap = (long long)sms * per_sm;
  return items < cap ? items : (int)cap;
}

// resident CTAs of one instantiation, queried once (stencil_init_fp64/_fp32 at
// plan bind, so that no query runs while a Newton step is being captured)
template <typename T, bool LIN, typename VT, int TI, int TJ>
int stencil_cap() {
  static int cap = 0;
  if (cap == 0) cap = persistent_grid(reinterpret_cast<const void*>(&k_stencil<T, LIN, VT, TI, TJ>), 256, 1 << 30);
  return cap;
}

template <typename T, bool LIN, typename VT, int TI, int TJ>
void launch_stencil_shape(const Batch& b, const StencilArgs<VT>& a, cudaStream_t s) {
  const int cap = stencil_cap<T, LIN, VT, TI, TJ>();
  k_stencil<T, LIN, VT, TI, TJ><<<b.ntiles < cap ? b.ntiles : cap, 256, 0, s>>>(b, a);
}

template <typename T, bool LIN, typename VT>
void launch_stencil(const Batch& b, const StencilArgs<VT>& a, cudaStream_t s, int shape) {
  if (b.ntiles == 0) return;
  if constexpr (LIN && sizeof(T) == 4) {
    switch (shape) {
      case kTile32x16: launch_stencil_shape<T, LIN, VT, 32, 16>(b, a, s); return;
      case kTile64x4: launch_stencil_shape<T, LIN, VT, 64, 4>(b, a, s); return;
      case kTile16x16: launch_stencil_shape<T, LIN, VT, 16, 16>(b, a, s); return;
      default: break;
    }
  }
  launch_stencil_shape<T, LIN, VT, kTI, kTJ>(b, a, s);
}

}  // namespace a2d
