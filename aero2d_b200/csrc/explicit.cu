// Explicit 4-stage Runge-Kutta pseudo-time stepping with local time steps and
// implicit residual smoothing, the fallback solver of aero2d/euler.py:289-346.
//
// Smoothing along i (periodic, constant coefficients -e, 1+2e, -e) is the
// exact solution of the circulant system, which the reference obtains by FFT
// (euler.py:302-303).  Here it is applied through the system's periodic Green's
// function g_m = G0 (l^m + l^(n-m)) / (1 - l^n), l the root in (0,1) of
// e l^2 - (1+2e) l + e = 0 and G0 = 1 / (e (1/l - l)); terms with l^|m| below
// 1e-18 of the diagonal are dropped, so results equal the FFT's to rounding.
// Smoothing along j is a Thomas solve of (-e, 1+2e, -e) with end diagonals 1+e.
#include <algorithm>

#include "batch.cuh"
#include "explicit.cuh"
#include "physics.cuh"

namespace a2d {

// local time step of cell (j, i) from its primitives W = (rho, u, v, p):
// dt = cfl vol / (lambda_i + lambda_j), face vectors averaged to the cell
// centre, in the operation order of euler.py:289-296; T is the compute type
// (FP32 reads the grid's FP32 metric copies)
template <typename T>
__device__ __forceinline__ T local_dt_cell(const GridDev& g, const State4<T>& W, int j, int i, T cfl) {
  const Metric<T> m{g};
  const int ip = (i + 1 == g.ni) ? 0 : i + 1;
  const T cc = sqrt(T(kGamma) * W.c[3] / W.c[0]);
  const T s0 = T(0.5) * (m.si(0, j, i) + m.si(0, j, ip));
  const T s1 = T(0.5) * (m.si(1, j, i) + m.si(1, j, ip));
  const T t0 = T(0.5) * (m.sj(0, j + 1, i) + m.sj(0, j, i));
  const T t1 = T(0.5) * (m.sj(1, j + 1, i) + m.sj(1, j, i));
  const T li = fabs(W.c[1] * s0 + W.c[2] * s1) + cc * sqrt(s0 * s0 + s1 * s1);
  const T lj = fabs(W.c[1] * t0 + W.c[2] * t1) + cc * sqrt(t0 * t0 + t1 * t1);
  return cfl * m.vol(j, i) / (li + lj);
}

// local time steps of every case from its conserved state (the RK iteration)
template <typename T>
__global__ void __launch_bounds__(256) k_local_dt(Batch b, const double* __restrict__ U, double* __restrict__ dt,
                                                  double cfl) {
  const Tile t = b.tiles[blockIdx.x];
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  const double* Uc = U + 4 * cs.cell_off;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
    State4<T> u;
#pragma unroll
    for (int k = 0; k < 4; ++k) u.c[k] = T(Uc[vidx(g, k, j, i)]);
    dt[cs.cell_off + (size_t)j * g.ni + i] = (double)local_dt_cell<T>(g, cons_to_prim<T, T>(u), j, i, T(cfl));
  }
}

// local time steps of one case from primitives given in the reference layout
// W[4][ni][nc], written as dt[ni][nc] (EulerSolver.local_dt, euler.py:289-296)
__global__ void __launch_bounds__(256) k_local_dt_prim(GridDev g, const double* __restrict__ W,
                                                       double* __restrict__ dt, double cfl) {
  const size_t N = (size_t)g.ni * g.nc;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N; q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q / g.nc), j = (int)(q % g.nc);
    State4<double> w;
#pragma unroll
    for (int k = 0; k < 4; ++k) w.c[k] = W[k * N + q];
    dt[q] = local_dt_cell<double>(g, w, j, i, cfl);
  }
}

// periodic smoothing along i: one block per (case, component, row j); T is the
// compute type (values stay in FP64 arrays, rounded to T when T is FP32)
template <typename T>
__global__ void __launch_bounds__(256) k_irs_i(Batch b, const double* __restrict__ R, double* __restrict__ out,
                                               double e_) {
  const int row = blockIdx.x;   // rows enumerated as (case, k, j) via the row table below
  const int cs_id = blockIdx.y;
  const CaseDev cs = b.cases[cs_id];
  const GridDev& g = cs.g;
  const int ni = g.ni, nc = g.nc;
  if (row >= 4 * nc) return;
  const int k = row / nc, j = row % nc;
  extern __shared__ __align__(8) unsigned char irs_sm[];
  T* r = reinterpret_cast<T*>(irs_sm);   // ni
  T* gm = r + ni;                         // up to ni/2 + 1
  const double* src = R + 4 * cs.cell_off + vidx(g, k, j, 0);
  for (int i = threadIdx.x; i < ni; i += blockDim.x) r[i] = T(src[i]);
  // the Green's function in FP64, then rounded to T (its terms below 1e-18 of
  // the diagonal dropped: the FFT's solution to rounding)
  const double e = e_;
  const double lam = ((1.0 + 2.0 * e) - sqrt(1.0 + 4.0 * e)) / (2.0 * e);
  const double G0 = 1.0 / (e * (1.0 / lam - lam));
  int M = (int)ceil(log(1e-18) / log(lam));
  if (M > ni / 2) M = ni / 2;
  const double ln = pow(lam, (double)ni);
  for (int m = threadIdx.x; m <= M; m += blockDim.x)
    gm[m] = T(G0 * (pow(lam, (double)m) + pow(lam, (double)(ni - m))) / (1.0 - ln));
  __syncthreads();
  double* dst = out + 4 * cs.cell_off + vidx(g, k, j, 0);
  const bool full = (2 * M + 1 >= ni);
  for (int i = threadIdx.x; i < ni; i += blockDim.x) {
    T s = gm[0] * r[i];
    if (full) {
      for (int d = 1; d < ni; ++d) {
        const int m = d <= ni / 2 ? d : ni - d;
        int q = i - d;
        if (q < 0) q += ni;
        s += gm[m] * r[q];
      }
    } else {
      for (int m = 1; m <= M; ++m) {
        int qm = i - m, qp = i + m;
        if (qm < 0) qm += ni;
        if (qp >= ni) qp -= ni;
        s += gm[m] * (r[qm] + r[qp]);
      }
    }
    dst[i] = (double)s;
  }
}

// smoothing along j: Thomas solve per (case, component, line i); thread per line.
// The elimination coefficients depend on j only and are formed once per block.
template <typename T>
__global__ void __launch_bounds__(128) k_irs_j(Batch b, double* __restrict__ R, double e_) {
  const int cs_id = blockIdx.y;
  const CaseDev cs = b.cases[cs_id];
  const GridDev& g = cs.g;
  const int ni = g.ni, nc = g.nc;
  extern __shared__ __align__(8) unsigned char irs_sm[];
  T* cpj = reinterpret_cast<T*>(irs_sm);   // nc
  const T e = T(e_);
  if (threadIdx.x == 0) {
    T cp = T(0);
    for (int j = 0; j < nc; ++j) {
      const T dj = (j == 0 || j == nc - 1) ? T(1) + e : T(1) + T(2) * e;
      const T lj = (j == 0) ? T(0) : -e;
      const T uj = (j == nc - 1) ? T(0) : -e;
      cp = uj / (dj - lj * cp);
      cpj[j] = cp;
    }
  }
  __syncthreads();
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= 4 * ni) return;
  const int k = line / ni, i = line % ni;
  double* x = R + 4 * cs.cell_off;
  T dprev = T(0);
  for (int j = 0; j < nc; ++j) {
    const T dj = (j == 0 || j == nc - 1) ? T(1) + e : T(1) + T(2) * e;
    const T lj = (j == 0) ? T(0) : -e;
    const T den = dj - lj * (j == 0 ? T(0) : cpj[j - 1]);
    const T v = (T(x[vidx(g, k, j, i)]) - lj * dprev) / den;
    x[vidx(g, k, j, i)] = (double)v;
    dprev = v;
  }
  T xn = T(0);
  for (int j = nc - 1; j >= 0; --j) {
    const T v = T(x[vidx(g, k, j, i)]) - cpj[j] * xn;
    x[vidx(g, k, j, i)] = (double)v;
    xn = v;
  }
}

// U = U0 - a (dt / vol) R   (euler.py:344), in the compute type T (with FP32
// the state is rounded to FP32 at every stage, as the reference's float32 run keeps it)
template <typename T>
__global__ void __launch_bounds__(256) k_rk_stage(Batch b, const double* __restrict__ U0,
                                                  const double* __restrict__ R, const double* __restrict__ dt,
                                                  double* __restrict__ U, double a) {
  const Tile t = b.tiles[blockIdx.x];
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  const Metric<T> m{g};
  const size_t base = 4 * cs.cell_off;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
    const size_t cell = (size_t)j * g.ni + i;
    const T f = T(a) * (T(dt[cs.cell_off + cell]) / m.vol(j, i));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t q = base + vidx(g, k, j, i);
      U[q] = (double)(T(U0[q]) - f * T(R[q]));
    }
  }
}

// per-tile sum of ((U_rho - U0_rho) / dt)^2
__global__ void __launch_bounds__(256) k_rk_res(Batch b, const double* __restrict__ U0,
                                                const double* __restrict__ U, const double* __restrict__ dt,
                                                double* __restrict__ tpart) {
  const Tile t = b.tiles[blockIdx.x];
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  const size_t base = 4 * cs.cell_off;
  double s = 0.0;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
    const size_t q = base + vidx(g, 0, j, i);
    const double r = (U[q] - U0[q]) / dt[cs.cell_off + (size_t)j * g.ni + i];
    s += r * r;
  }
  __shared__ double sc[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) sc[w] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) tot += sc[q];
    tpart[(size_t)blockIdx.x * kTilePartStride + 3] = tot;
  }
}

// res = sqrt(mean(...)) per case; circ = 1/2 Cl M from the forces   (euler.py:345, :401-403)
__global__ void k_rk_finish(Batch b, const double* tpart, const double* coef, double* res, double* circ) {
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= b.ncases) return;
  const CaseDev c = b.cases[cs];
  double s = 0.0;
  for (int q = 0; q < c.ntiles; ++q) s += tpart[(size_t)(c.tile0 + q) * kTilePartStride + 3];
  const double N = (double)c.g.ni * (double)c.g.nc;
  if (res != nullptr) res[cs] = sqrt(s / N);
  const double mach = sqrt(c.winf[1] * c.winf[1] + c.winf[2] * c.winf[2]);
  circ[cs] = 0.5 * coef[3 * cs] * mach;
}

// ---------------------------------------------------------------------------
// FAS multigrid transfers (aero2d/euler.py:349-381) between a fine batch and
// the coarse batch of the same cases on grids of every other node (ni/2 x nc/2
// cells).  Every sum and product is rounded separately, in the reference's
// order, as the NumPy/JAX expressions evaluate them.
// ---------------------------------------------------------------------------
// R += P over the cells of every case (the forcing term of a coarse level)
__global__ void __launch_bounds__(256) k_add_forcing(Batch b, double* __restrict__ R, const double* __restrict__ P) {
  const Tile t = b.tiles[blockIdx.x];
  const CaseDev cs = b.cases[t.cs];
  const size_t base = 4 * cs.cell_off;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t q = base + vidx(cs.g, k, j, i);
      R[q] = __dadd_rn(R[q], P[q]);
    }
  }
}

// sum4(a) = a(2i, 2j) + a(2i+1, 2j) + a(2i, 2j+1) + a(2i+1, 2j+1), left to right
__device__ __forceinline__ double sum4(double a00, double a10, double a01, double a11) {
  return __dadd_rn(__dadd_rn(__dadd_rn(a00, a10), a01), a11);
}

// one thread per coarse cell (tiles of the coarse batch): Uc = Uc0 = sum4(U vol) / sum4(vol);
// with R != nullptr also Pc = sum4(R (+ P)) - Rc, where Rc is read from Pc (the coarse
// residual at Uc0) and P (nullable) is the fine level's own forcing
__global__ void __launch_bounds__(256) k_fas_restrict(Batch fb, Batch cb, const double* __restrict__ Uf,
                                                     double* __restrict__ Uc, double* __restrict__ Uc0) {
  const Tile t = cb.tiles[blockIdx.x];
  const CaseDev cc = cb.cases[t.cs];
  const CaseDev cf = fb.cases[t.cs];
  const GridDev& gf = cf.g;
  const size_t bf = 4 * cf.cell_off, bc = 4 * cc.cell_off;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int jc = t.j0 + c / t.ti, ic = t.i0 + c % t.ti;
    const int i0 = 2 * ic, j0 = 2 * jc;
    const double v00 = gf.vol[(size_t)j0 * gf.ni + i0], v10 = gf.vol[(size_t)j0 * gf.ni + i0 + 1];
    const double v01 = gf.vol[(size_t)(j0 + 1) * gf.ni + i0], v11 = gf.vol[(size_t)(j0 + 1) * gf.ni + i0 + 1];
    const double vs = sum4(v00, v10, v01, v11);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double* u = Uf + bf;
      const double a = sum4(__dmul_rn(u[vidx(gf, k, j0, i0)], v00), __dmul_rn(u[vidx(gf, k, j0, i0 + 1)], v10),
                            __dmul_rn(u[vidx(gf, k, j0 + 1, i0)], v01),
                            __dmul_rn(u[vidx(gf, k, j0 + 1, i0 + 1)], v11));
      const size_t q = bc + vidx(cc.g, k, jc, ic);
      const double r = __ddiv_rn(a, vs);
      Uc[q] = r;
      Uc0[q] = r;
    }
  }
}

// Pc := sum4(Rf) - Pc (Pc holds the coarse residual at Uc0 on entry); Rf already includes
// the fine level's forcing
__global__ void __launch_bounds__(256) k_fas_forcing(Batch fb, Batch cb, const double* __restrict__ Rf,
                                                    double* __restrict__ Pc) {
  const Tile t = cb.tiles[blockIdx.x];
  const CaseDev cc = cb.cases[t.cs];
  const CaseDev cf = fb.cases[t.cs];
  const GridDev& gf = cf.g;
  const double* r = Rf + 4 * cf.cell_off;
  const size_t bc = 4 * cc.cell_off;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int jc = t.j0 + c / t.ti, ic = t.i0 + c % t.ti;
    const int i0 = 2 * ic, j0 = 2 * jc;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double a = sum4(r[vidx(gf, k, j0, i0)], r[vidx(gf, k, j0, i0 + 1)], r[vidx(gf, k, j0 + 1, i0)],
                            r[vidx(gf, k, j0 + 1, i0 + 1)]);
      const size_t q = bc + vidx(cc.g, k, jc, ic);
      Pc[q] = __dsub_rn(a, Pc[q]);
    }
  }
}

// Uf += prolong(Uc - Uc0): in i 3/4 d(ic) + 1/4 d(ic -+ 1) (periodic), then in j
// 3/4 a(jc) + 1/4 a(jc -+ 1) held at the ends (aero2d/euler.py:354-366); one thread
// per fine cell
__global__ void __launch_bounds__(256) k_fas_prolong(Batch fb, Batch cb, double* __restrict__ Uf,
                                                    const double* __restrict__ Uc,
                                                    const double* __restrict__ Uc0) {
  const Tile t = fb.tiles[blockIdx.x];
  const CaseDev cf = fb.cases[t.cs];
  const CaseDev cc = cb.cases[t.cs];
  const GridDev& gc = cc.g;
  const size_t bf = 4 * cf.cell_off, bc = 4 * cc.cell_off;
  for (int c = threadIdx.x; c < t.ti * t.tj; c += blockDim.x) {
    const int j = t.j0 + c / t.ti, i = t.i0 + c % t.ti;
    const int ic = i >> 1, jc = j >> 1;
    const int icn = (i & 1) ? (ic + 1 == gc.ni ? 0 : ic + 1) : (ic == 0 ? gc.ni - 1 : ic - 1);
    const int jcn = (j & 1) ? (jc + 1 == gc.nc ? jc : jc + 1) : (jc == 0 ? 0 : jc - 1);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      auto d = [&](int jj, int ii) {
        const size_t q = bc + vidx(gc, k, jj, ii);
        return __dsub_rn(Uc[q], Uc0[q]);
      };
      const double a0 = __dadd_rn(__dmul_rn(0.75, d(jc, ic)), __dmul_rn(0.25, d(jc, icn)));
      const double a1 = __dadd_rn(__dmul_rn(0.75, d(jcn, ic)), __dmul_rn(0.25, d(jcn, icn)));
      const double v = __dadd_rn(__dmul_rn(0.75, a0), __dmul_rn(0.25, a1));
      const size_t q = bf + vidx(cf.g, k, j, i);
      Uf[q] = __dadd_rn(Uf[q], v);
    }
  }
}

void launch_local_dt(const Batch& b, const double* U, double* dt, double cfl, bool fp32, cudaStream_t s) {
  if (b.ntiles == 0) return;
  if (fp32) k_local_dt<float><<<b.ntiles, 256, 0, s>>>(b, U, dt, cfl);
  else k_local_dt<double><<<b.ntiles, 256, 0, s>>>(b, U, dt, cfl);
}
void launch_local_dt_prim(const GridDev& g, const double* W, double* dt, double cfl, cudaStream_t s) {
  const size_t N = (size_t)g.ni * g.nc;
  const int blocks = (int)std::min<size_t>((N + 255) / 256, 148 * 8);
  if (N) k_local_dt_prim<<<blocks, 256, 0, s>>>(g, W, dt, cfl);
}
void launch_irs(const Batch& b, double* R, double* tmp, double e, int max_ni, int max_nc, bool fp32,
                cudaStream_t s) {
  if (e <= 0.0 || b.ncases == 0) return;
  dim3 gi(4 * max_nc, b.ncases);
  const size_t sm = (size_t)(max_ni + max_ni / 2 + 2) * sizeof(double);
  dim3 gj((4 * max_ni + 127) / 128, b.ncases);
  if (fp32) {
    k_irs_i<float><<<gi, 256, sm, s>>>(b, R, tmp, e);
    k_irs_j<float><<<gj, 128, (size_t)max_nc * sizeof(double), s>>>(b, tmp, e);
  } else {
    k_irs_i<double><<<gi, 256, sm, s>>>(b, R, tmp, e);
    k_irs_j<double><<<gj, 128, (size_t)max_nc * sizeof(double), s>>>(b, tmp, e);
  }
}
void launch_rk_stage(const Batch& b, const double* U0, const double* R, const double* dt, double* U, double a,
                     bool fp32, cudaStream_t s) {
  if (b.ntiles == 0) return;
  if (fp32) k_rk_stage<float><<<b.ntiles, 256, 0, s>>>(b, U0, R, dt, U, a);
  else k_rk_stage<double><<<b.ntiles, 256, 0, s>>>(b, U0, R, dt, U, a);
}
void launch_rk_res(const Batch& b, const double* U0, const double* U, const double* dt, double* tpart,
                   cudaStream_t s) {
  if (b.ntiles) k_rk_res<<<b.ntiles, 256, 0, s>>>(b, U0, U, dt, tpart);
}
void launch_rk_finish(const Batch& b, const double* tpart, const double* coef, double* res, double* circ,
                      cudaStream_t s) {
  k_rk_finish<<<(b.ncases + 63) / 64, 64, 0, s>>>(b, tpart, coef, res, circ);
}

void launch_add_forcing(const Batch& b, double* R, const double* P, cudaStream_t s) {
  if (b.ntiles) k_add_forcing<<<b.ntiles, 256, 0, s>>>(b, R, P);
}
void launch_fas_restrict(const Batch& fine, const Batch& coarse, const double* Uf, double* Uc, double* Uc0,
                         cudaStream_t s) {
  if (coarse.ntiles) k_fas_restrict<<<coarse.ntiles, 256, 0, s>>>(fine, coarse, Uf, Uc, Uc0);
}
void launch_fas_forcing(const Batch& fine, const Batch& coarse, const double* Rf, double* Pc, cudaStream_t s) {
  if (coarse.ntiles) k_fas_forcing<<<coarse.ntiles, 256, 0, s>>>(fine, coarse, Rf, Pc);
}
void launch_fas_prolong(const Batch& fine, const Batch& coarse, double* Uf, const double* Uc, const double* Uc0,
                        cudaStream_t s) {
  if (fine.ntiles) k_fas_prolong<<<fine.ntiles, 256, 0, s>>>(fine, coarse, Uf, Uc, Uc0);
}

}  // namespace a2d
