// Block-tridiagonal line preconditioner of the Newton-Krylov solver.
//
//  k_face_jac   4x4 Jacobian blocks dF/dU_left, dF/dU_right of the first-order
//               HLLC flux on every i- and j-face, plus the wall and far-field
//               closures (aero2d/implicit.py:32-64), by forward-mode dual
//               numbers; one thread per cell, 32 lines x 8 rows per CTA.
//  k_factor     assembles D = sum of face blocks + vol/dtau I and runs the
//               block-Thomas forward elimination along each wall-normal line
//               in FP64: den_j = D_j - A_j c_{j-1}, inv_j = den_j^-1,
//               c_j = inv_j C_j (aero2d/implicit.py:81-128), and stores inv_j,
//               c_j and G_j = -inv_j A_j.  One thread per line, 32 lines (one
//               warp) per line group.
//  k_rhs        first half of a line-Jacobi sweep (aero2d/implicit.py:150-157):
//               moves the i-coupling of the previous sweep to the right-hand
//               side and applies inv_j, e_j = inv_j (r_j - off_j); fully
//               parallel over cells.
//  k_lines      second half: the sequential recurrences d_j = e_j + G_j d_{j-1}
//               and x_j = d_j - c_j x_{j+1} along each line
//               (aero2d/implicit.py:130-148), which equal the reference's
//               d_j = inv_j (r_j - A_j d_{j-1}) in exact arithmetic.  Only 20
//               words per step remain on the sequential path, loaded 4 steps
//               ahead.
//
// The blocks are stored lane-blocked ([group][row][entry][lane]) so that at
// every step of the sequential j recurrence a warp reads each matrix entry of
// its 32 lines as one coalesced 256 B (FP64) or 128 B (FP32) transaction.
#include "batch.cuh"
#include "kernels.cuh"
#include "physics.cuh"

namespace a2d {

template <typename T>
__device__ __forceinline__ State4<T> load_state(const double* U, const GridDev& g, int j, int i) {
  State4<T> r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.c[k] = T(U[vidx(g, k, j, i)]);
  return r;
}

// Jacobian d f / d u (f: conserved state -> flux, 4x4 [out][in]) by one dual pass
template <typename T, class F>
__device__ __forceinline__ void jac4(const State4<T>& u, F f, T J[16]) {
  using D = Dual<T, 4>;
  State4<D> ud;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    ud.c[k].v = u.c[k];
#pragma unroll
    for (int q = 0; q < 4; ++q) ud.c[k].d[q] = (q == k) ? T(1) : T(0);
  }
  const State4<D> r = f(ud);
#pragma unroll
  for (int o = 0; o < 4; ++o)
#pragma unroll
    for (int q = 0; q < 4; ++q) J[o * 4 + q] = r.c[o].d[q];
}

template <typename T>
__device__ __forceinline__ State4<Dual<T, 4>> const_dual(const State4<T>& u) {
  State4<Dual<T, 4>> r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.c[k] = make_const<T, 4>(u.c[k]);
  return r;
}

// dF/dUL, dF/dUR of the first-order flux hllc(prim(UL), prim(UR), S)
template <typename T>
__device__ __forceinline__ void face_jac(const State4<T>& UL, const State4<T>& UR, T sx, T sy, T AL[16],
                                         T AR[16]) {
  using D = Dual<T, 4>;
  const State4<D> WRc = cons_to_prim<D, T>(const_dual(UR));
  jac4<T>(UL, [&](const State4<D>& u) { return hllc<D, T>(cons_to_prim<D, T>(u), WRc, sx, sy); }, AL);
  const State4<D> WLc = cons_to_prim<D, T>(const_dual(UL));
  jac4<T>(UR, [&](const State4<D>& u) { return hllc<D, T>(WLc, cons_to_prim<D, T>(u), sx, sy); }, AR);
}

template <typename TS, typename T>
__device__ __forceinline__ void store_block(TS* base, long long row0, int rows, int g, int j, int lane,
                                            const T A[16]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) base[lbidx(row0, rows, g, j, e, lane)] = TS(A[e]);
}

template <typename T>
__global__ void __launch_bounds__(256) k_face_jac(Batch b, JacArgs a) {
  const Tile t = b.tiles[blockIdx.x];
  if (!case_live(b, t.cs, a.need)) return;
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  Metric<T> m{g};
  const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;
  if (lane >= t.ti || row >= t.tj) return;
  const int ni = g.ni, nc = g.nc;
  const int i = t.i0 + lane, j = t.j0 + row, grp = t.i0 / kLanes;
  const double* U = a.U + 4 * cs.cell_off;
  T* JIL = static_cast<T*>(a.JIL);
  T* JIR = static_cast<T*>(a.JIR);
  T* JJL = static_cast<T*>(a.JJL);
  T* JJR = static_cast<T*>(a.JJR);
  const State4<T> Uc = load_state<T>(U, g, j, i);
  T AL[16], AR[16];
  {  // i-face between cells i-1 and i
    const int im = i == 0 ? ni - 1 : i - 1;
    face_jac<T>(load_state<T>(U, g, j, im), Uc, m.si(0, j, i), m.si(1, j, i), AL, AR);
    store_block(JIL, cs.rows_nc, nc, grp, j, lane, AL);
    store_block(JIR, cs.rows_nc, nc, grp, j, lane, AR);
  }
  if (j == 0) {  // wall face: mirrored ghost on its low side
    const T sx = m.sj(0, 0, i), sy = m.sj(1, 0, i);
    using D = Dual<T, 4>;
    jac4<T>(Uc,
            [&](const State4<D>& u) {
              const State4<D> w = cons_to_prim<D, T>(u);
              return hllc<D, T>(wall_mirror<D, T>(w, sx, sy), w, sx, sy);
            },
            AR);
#pragma unroll
    for (int e = 0; e < 16; ++e) AL[e] = T(0);
    store_block(JJL, cs.rows_nc1, nc + 1, grp, 0, lane, AL);
    store_block(JJR, cs.rows_nc1, nc + 1, grp, 0, lane, AR);
  } else {  // interior j-face between cells j-1 and j
    face_jac<T>(load_state<T>(U, g, j - 1, i), Uc, m.sj(0, j, i), m.sj(1, j, i), AL, AR);
    store_block(JJL, cs.rows_nc1, nc + 1, grp, j, lane, AL);
    store_block(JJR, cs.rows_nc1, nc + 1, grp, j, lane, AR);
  }
  if (j == nc - 1) {  // far-field face, circulation held fixed (implicit.py:54-59)
    const T sx = m.sj(0, nc, i), sy = m.sj(1, nc, i);
    const T rinf = T(cs.winf[0]), uinf = T(cs.winf[1]), vinf = T(cs.winf[2]), pinf = T(cs.winf[3]);
    const T circ = a.vortex ? T(a.circ[t.cs]) : T(0);
    const T xf = m.xf(i), yf = m.yf(i);
    using D = Dual<T, 4>;
    const D cd = make_const<T, 4>(circ);
    jac4<T>(Uc,
            [&](const State4<D>& u) {
              const State4<D> w = cons_to_prim<D, T>(u);
              const State4<D> wb = farfield_ghost<D, T>(w, sx, sy, rinf, uinf, vinf, pinf, xf, yf, cd);
              return hllc<D, T>(w, wb, sx, sy);
            },
            AL);
#pragma unroll
    for (int e = 0; e < 16; ++e) AR[e] = T(0);
    store_block(JJL, cs.rows_nc1, nc + 1, grp, nc, lane, AL);
    store_block(JJR, cs.rows_nc1, nc + 1, grp, nc, lane, AR);
  }
}

// ---------------------------------------------------------------------------
// 4x4 FP64 inverse by Gauss-Jordan elimination with partial pivoting
// ---------------------------------------------------------------------------
__device__ __forceinline__ void inv4(const double A[16], double X[16]) {
  double a[4][8];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      a[r][c] = A[r * 4 + c];
      a[r][c + 4] = (r == c) ? 1.0 : 0.0;
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int p = c;
    double best = fabs(a[c][c]);
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      const double v = fabs(a[r][c]);
      if (v > best) {
        best = v;
        p = r;
      }
    }
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      if (p == r) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const double tmp = a[c][k];
          a[c][k] = a[r][k];
          a[r][k] = tmp;
        }
      }
    }
    const double ip = 1.0 / a[c][c];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[c][k] *= ip;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (r != c) {
        const double f = a[r][c];
#pragma unroll
        for (int k = 0; k < 8; ++k) a[r][k] -= f * a[c][k];
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) X[r * 4 + c] = a[r][c + 4];
}

template <typename TJ>
__device__ __forceinline__ void load_block(const TJ* base, long long row0, int rows, int g, int j, int lane,
                                           double A[16]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) A[e] = (double)base[lbidx(row0, rows, g, j, e, lane)];
}

template <typename TJ, typename TF>
__global__ void __launch_bounds__(128) k_factor(Batch b, FactorArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gid = blockIdx.x * 4 + warp;
  if (gid >= b.ngroups) return;
  const Group grp = b.groups[gid];
  if (!case_live(b, grp.cs, a.need)) return;
  if (lane >= grp.n) return;
  const CaseDev cs = b.cases[grp.cs];
  const GridDev& g = cs.g;
  const int ni = g.ni, nc = g.nc;
  const int i = grp.i0 + lane;
  const int ip = (i + 1 == ni) ? 0 : i + 1;
  const int gp = ip / kLanes, lp = ip % kLanes;
  const TJ* JIL = static_cast<const TJ*>(a.JIL);
  const TJ* JIR = static_cast<const TJ*>(a.JIR);
  const TJ* JJL = static_cast<const TJ*>(a.JJL);
  const TJ* JJR = static_cast<const TJ*>(a.JJR);
  TF* INV = static_cast<TF*>(a.INV);
  TF* CF = static_cast<TF*>(a.CF);
  TF* G = static_cast<TF*>(a.G);
  const double* U = a.U + 4 * cs.cell_off;
  const double cfl = a.ctl[grp.cs].cfl;
  double cprev[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) cprev[e] = 0.0;
  for (int j = 0; j < nc; ++j) {
    double D[16], T1[16];
    load_block(JIL, cs.rows_nc, nc, gp, j, lp, D);
    load_block(JIR, cs.rows_nc, nc, grp.g, j, lane, T1);
#pragma unroll
    for (int e = 0; e < 16; ++e) D[e] = D[e] - T1[e];
    if (j < nc - 1) {
      load_block(JJL, cs.rows_nc1, nc + 1, grp.g, j + 1, lane, T1);
#pragma unroll
      for (int e = 0; e < 16; ++e) D[e] = D[e] + T1[e];
    }
    load_block(JJR, cs.rows_nc1, nc + 1, grp.g, j, lane, T1);
#pragma unroll
    for (int e = 0; e < 16; ++e) D[e] = D[e] - T1[e];
    if (j == nc - 1) {
      load_block(JJL, cs.rows_nc1, nc + 1, grp.g, nc, lane, T1);
#pragma unroll
      for (int e = 0; e < 16; ++e) D[e] = D[e] + T1[e];
    }
    // local pseudo-time step (aero2d/euler.py:289-296, aero2d/implicit.py:173-177)
    {
      const State4<double> W = cons_to_prim<double, double>(load_state<double>(U, g, j, i));
      const double c = sqrt(kGamma * W.c[3] / W.c[0]);
      const size_t N = (size_t)ni * nc;
      const double* Si = g.Si;
      const double* Sj = g.Sj;
      const double s0 = 0.5 * (Si[(size_t)j * ni + i] + Si[(size_t)j * ni + ip]);
      const double s1 = 0.5 * (Si[N + (size_t)j * ni + i] + Si[N + (size_t)j * ni + ip]);
      const size_t NJ = (size_t)(nc + 1) * ni;
      const double t0 = 0.5 * (Sj[(size_t)(j + 1) * ni + i] + Sj[(size_t)j * ni + i]);
      const double t1 = 0.5 * (Sj[NJ + (size_t)(j + 1) * ni + i] + Sj[NJ + (size_t)j * ni + i]);
      const double li = fabs(W.c[1] * s0 + W.c[2] * s1) + c * sqrt(s0 * s0 + s1 * s1);
      const double lj = fabs(W.c[1] * t0 + W.c[2] * t1) + c * sqrt(t0 * t0 + t1 * t1);
      const double vol = g.vol[(size_t)j * ni + i];
      const double dt = a.cfl_base * vol / (li + lj);
      const double dtl = dt / a.cfl_base * cfl;
      const double dinv = 1.0 / dtl;
      const double dg = vol * dinv;
      a.diag[cs.cell_off + (size_t)j * ni + i] = dg;
      D[0] += dg;
      D[5] += dg;
      D[10] += dg;
      D[15] += dg;
    }
    // pivot block den = D - A c_prev with A = -JJL(j); inv = den^-1
    double A[16];
    load_block(JJL, cs.rows_nc1, nc + 1, grp.g, j, lane, A);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double s = A[r * 4 + 0] * cprev[0 * 4 + c];
#pragma unroll
        for (int k = 1; k < 4; ++k) s += A[r * 4 + k] * cprev[k * 4 + c];
        D[r * 4 + c] = D[r * 4 + c] + s;
      }
    double inv[16];
    inv4(D, inv);
    // G = inv * JJL(j) = -inv A: the forward recurrence becomes d_j = inv r_j + G d_{j-1}
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double s = inv[r * 4 + 0] * A[0 * 4 + c];
#pragma unroll
        for (int k = 1; k < 4; ++k) s += inv[r * 4 + k] * A[k * 4 + c];
        D[r * 4 + c] = s;
      }
    load_block(JJR, cs.rows_nc1, nc + 1, grp.g, j + 1, lane, T1);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double s = inv[r * 4 + 0] * T1[0 * 4 + c];
#pragma unroll
        for (int k = 1; k < 4; ++k) s += inv[r * 4 + k] * T1[k * 4 + c];
        cprev[r * 4 + c] = s;
      }
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const size_t q = lbidx(cs.rows_nc, nc, grp.g, j, e, lane);
      INV[q] = TF(inv[e]);
      CF[q] = TF(cprev[e]);
      G[q] = TF(D[e]);
    }
  }
}

// ---------------------------------------------------------------------------
// right-hand side of one line-Jacobi sweep, fully parallel over cells:
//   e = inv_j (r - off),  off = Bim x[i-1] + Bip x[i+1] = -(JIL x[i-1]) + JIR(i+1) x[i+1]
// (off = 0 on the first sweep).  One thread per cell, 32 x 8 cells per CTA.
// ---------------------------------------------------------------------------
template <typename TJ, typename TF>
__global__ void __launch_bounds__(256) k_rhs(Batch b, RhsArgs a) {
  const Tile t = b.tiles[blockIdx.x];
  if (!case_live(b, t.cs, a.need)) return;
  const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;
  if (lane >= t.ti || row >= t.tj) return;
  const CaseDev cs = b.cases[t.cs];
  const GridDev& g = cs.g;
  const int ni = g.ni, nc = g.nc;
  const int i = t.i0 + lane, j = t.j0 + row, grp = t.i0 / kLanes;
  const size_t base = 4 * cs.cell_off;
  double rhs[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) rhs[k] = a.r[base + vidx(g, k, j, i)];
  if (a.xprev != nullptr) {
    const int ip = (i + 1 == ni) ? 0 : i + 1;
    const int im = (i == 0) ? ni - 1 : i - 1;
    const double* xp = a.xprev + base;
    double xm4[4], xp4[4], AL[16], AR[16];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      xm4[k] = xp[vidx(g, k, j, im)];
      xp4[k] = xp[vidx(g, k, j, ip)];
    }
    load_block(static_cast<const TJ*>(a.JIL), cs.rows_nc, nc, grp, j, lane, AL);
    load_block(static_cast<const TJ*>(a.JIR), cs.rows_nc, nc, ip / kLanes, j, ip % kLanes, AR);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double s1 = AL[q * 4 + 0] * xm4[0];
      double s2 = AR[q * 4 + 0] * xp4[0];
#pragma unroll
      for (int k = 1; k < 4; ++k) {
        s1 += AL[q * 4 + k] * xm4[k];
        s2 += AR[q * 4 + k] * xp4[k];
      }
      rhs[q] = rhs[q] - (-s1 + s2);
    }
  }
  double IV[16];
  load_block(static_cast<const TF*>(a.INV), cs.rows_nc, nc, grp, j, lane, IV);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double s = IV[q * 4 + 0] * rhs[0];
#pragma unroll
    for (int k = 1; k < 4; ++k) s += IV[q * 4 + k] * rhs[k];
    a.out[base + vidx(g, q, j, i)] = s;
  }
}

// ---------------------------------------------------------------------------
// the sequential part of the block-Thomas solve, in place on x:
//   forward   d_j = e_j + G_j d_{j-1}
//   backward  x_j = d_j - C_j x_{j+1}
// Four threads per line, one per row of the 4x4 blocks; the quad exchanges
// the previous step's 4-vector by shuffles.  Each thread keeps the operands of
// its row for the next kAhead steps in registers (one FP64 vector entry and
// four block entries per step), so a step waits on 1/kAhead of the memory
// latency, and a 32-line group fills four warps.
// ---------------------------------------------------------------------------
constexpr int kAhead = 8;

template <typename TF>
struct RowStep {
  double v;
  TF m[4];
};

template <typename TF>
__device__ __forceinline__ void load_row(RowStep<TF>& s, const double* x, const TF* M, const CaseDev& cs,
                                         const GridDev& g, int grp, int lane, int i, int q, int j) {
  if (j < 0 || j >= g.nc) return;
  s.v = x[vidx(g, q, j, i)];
#pragma unroll
  for (int c = 0; c < 4; ++c) s.m[c] = M[lbidx(cs.rows_nc, g.nc, grp, j, q * 4 + c, lane)];
}

// the 4 components of the quad's current vector, from the quad's lanes
__device__ __forceinline__ void quad_gather(double mine, int base, double out[4]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) out[c] = __shfl_sync(0xffffffffu, mine, base | c);
}

// one CTA of 128 threads per 32-line group: warp w holds lines 8w..8w+7,
// lane 4l+q is row q of line l
template <typename TF>
__global__ void __launch_bounds__(128) k_lines(Batch b, LinesArgs a) {
  const int gid = blockIdx.x;
  if (gid >= b.ngroups) return;
  const Group grp = b.groups[gid];
  if (!case_live(b, grp.cs, a.need)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int l = warp * 8 + (lane >> 2);       // line within the group
  const int q = lane & 3;                      // row of the 4x4 blocks owned
  const int base = lane & ~3;                  // first lane of the quad
  const bool owner = l < grp.n;                // quads past the group's last line only shuffle
  const int ll = owner ? l : grp.n - 1;        // their loads stay on a valid line
  const CaseDev cs = b.cases[grp.cs];
  const GridDev& g = cs.g;
  const int nc = g.nc;
  const int i = grp.i0 + ll;
  double* x = a.x + 4 * cs.cell_off;
  const TF* G = static_cast<const TF*>(a.G);
  const TF* CF = static_cast<const TF*>(a.CF);
  RowStep<TF> buf[kAhead];
  // forward: d_j = e_j + G_j d_{j-1}
  double d = 0.0;
#pragma unroll
  for (int u = 0; u < kAhead; ++u) load_row(buf[u], x, G, cs, g, grp.g, ll, i, q, u);
  for (int j0 = 0; j0 < nc; j0 += kAhead) {
#pragma unroll
    for (int u = 0; u < kAhead; ++u) {
      const int j = j0 + u;
      if (j < nc) {
        double dp[4];
        quad_gather(d, base, dp);
        double acc = buf[u].v;
#pragma unroll
        for (int c = 0; c < 4; ++c) acc += (double)buf[u].m[c] * dp[c];
        d = acc;
        if (owner) x[vidx(g, q, j, i)] = acc;
        load_row(buf[u], x, G, cs, g, grp.g, ll, i, q, j + kAhead);
      }
    }
  }
  // backward: x_j = d_j - C_j x_{j+1}
  double xn = 0.0;
  const int top = nc - 1;
#pragma unroll
  for (int u = 0; u < kAhead; ++u) load_row(buf[u], x, CF, cs, g, grp.g, ll, i, q, top - u);
  for (int j0 = top; j0 >= 0; j0 -= kAhead) {
#pragma unroll
    for (int u = 0; u < kAhead; ++u) {
      const int j = j0 - u;
      if (j >= 0) {
        double xp[4];
        quad_gather(xn, base, xp);
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) acc += (double)buf[u].m[c] * xp[c];
        xn = buf[u].v - acc;
        if (owner) x[vidx(g, q, j, i)] = xn;
        load_row(buf[u], x, CF, cs, g, grp.g, ll, i, q, j - kAhead);
      }
    }
  }
}

template <typename T>
void launch_face_jac(const Batch& b, const JacArgs& a, cudaStream_t s) {
  if (b.ntiles == 0) return;
  k_face_jac<T><<<b.ntiles, 256, 0, s>>>(b, a);
}
template <typename TJ, typename TF>
void launch_factor(const Batch& b, const FactorArgs& a, cudaStream_t s) {
  if (b.ngroups == 0) return;
  k_factor<TJ, TF><<<(b.ngroups + 3) / 4, 128, 0, s>>>(b, a);
}
template <typename TJ, typename TF>
void launch_rhs(const Batch& b, const RhsArgs& a, cudaStream_t s) {
  if (b.ntiles == 0) return;
  k_rhs<TJ, TF><<<b.ntiles, 256, 0, s>>>(b, a);
}
template <typename TF>
void launch_lines(const Batch& b, const LinesArgs& a, cudaStream_t s) {
  if (b.ngroups == 0) return;
  k_lines<TF><<<b.ngroups, 128, 0, s>>>(b, a);
}

template void launch_face_jac<double>(const Batch&, const JacArgs&, cudaStream_t);
template void launch_face_jac<float>(const Batch&, const JacArgs&, cudaStream_t);
template void launch_factor<double, double>(const Batch&, const FactorArgs&, cudaStream_t);
template void launch_factor<float, float>(const Batch&, const FactorArgs&, cudaStream_t);
template void launch_rhs<double, double>(const Batch&, const RhsArgs&, cudaStream_t);
template void launch_rhs<float, float>(const Batch&, const RhsArgs&, cudaStream_t);
template void launch_lines<double>(const Batch&, const LinesArgs&, cudaStream_t);
template void launch_lines<float>(const Batch&, const LinesArgs&, cudaStream_t);

}  // namespace a2d
