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
//               c_j, G_j = -inv_j A_j and the premultiplied i-couplings
//               P_j = inv_j JIL(i), Q_j = inv_j JIR(i+1) of the sweeps.  One
//               thread per line, 32 lines (one warp) per line group.
// The sweeps themselves are in sweep.cu.
//
// The blocks are stored lane-blocked ([group][row][entry][lane]): the blocks
// of one line group at one row j are one contiguous run, which the sweep
// kernel streams with bulk copies.
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

// block m of the interleaved P, Q, G rows = A B (4x4, FP64), stored in TF (fbidx3)
template <typename TF>
__device__ __forceinline__ void mul4_store(const double A[16], const double B[16], TF* out, long long row0,
                                           int rows, int g, int j, int m, int lane, unsigned& nsat) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double s = A[r * 4 + 0] * B[0 * 4 + c];
#pragma unroll
      for (int k = 1; k < 4; ++k) s += A[r * 4 + k] * B[k * 4 + c];
      nsat += out_of_range<TF>(s);
      out[fbidx3(row0, rows, g, j, m, r, c, lane)] = from_f64<TF>(s);
    }
}

// Two warps per 32-line group (a lane per line): the even warp eliminates from
// the wall, the odd warp from the far field, in parallel; they meet at the twist
// row through shared memory (one named barrier of the pair), which the wall warp
// finishes.  The arithmetic of every row is the same as one thread running both
// eliminations after each other.
template <typename TJ, typename TF>
__global__ void __launch_bounds__(128) k_factor(Batch b, FactorArgs a) {
  __shared__ double cfar[2][16][kLanes];   // per group of the CTA: c'_{k+1} of each line
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pair = warp >> 1;              // group slot of the CTA
  const int half = warp & 1;               // 0: from the wall, 1: from the far field
  const int gid = blockIdx.x * 2 + pair;
  if (gid >= b.ngroups) return;            // both warps of the pair leave together
  const Group grp = b.groups[gid];
  if (!case_live(b, grp.cs, a.need)) return;
  const bool own = lane < grp.n;           // lanes past the group's last line only meet the barrier
  const CaseDev cs = b.cases[grp.cs];
  const GridDev& g = cs.g;
  const int ni = g.ni, nc = g.nc;
  const int i = grp.i0 + (own ? lane : grp.n - 1);
  const int ip = (i + 1 == ni) ? 0 : i + 1;
  const int gp = ip / kLanes, lp = ip % kLanes;
  const TJ* JIL = static_cast<const TJ*>(a.JIL);
  const TJ* JIR = static_cast<const TJ*>(a.JIR);
  const TJ* JJL = static_cast<const TJ*>(a.JJL);
  const TJ* JJR = static_cast<const TJ*>(a.JJR);
  TJ* INV = static_cast<TJ*>(a.INV);
  TF* CF = static_cast<TF*>(a.CF);
  TF* PQG = static_cast<TF*>(a.PQG);
  const double* U = a.U + 4 * cs.cell_off;
  const double cfl = a.ctl[grp.cs].cfl;
  const int k = nc / 2;   // twist row: the elimination from the wall and the one from the far field meet here
  unsigned nsat = 0;      // factor entries this line stores saturated (FP16 storage)
  // D_j: the diagonal block of row j (face blocks + vol/dtau I); writes diag
  auto assemble = [&](int j, double D[16]) {
    double T1[16];
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
  };
  // C = sgn A B (4x4)
  auto mul = [](const double A[16], const double B[16], double C[16], double sgn) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double s = A[r * 4 + 0] * B[0 * 4 + c];
#pragma unroll
        for (int q = 1; q < 4; ++q) s += A[r * 4 + q] * B[q * 4 + c];
        C[r * 4 + c] = sgn * s;
      }
  };
  // D += sgn A B
  auto mul_add = [](const double A[16], const double B[16], double D[16], double sgn) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double s = A[r * 4 + 0] * B[0 * 4 + c];
#pragma unroll
        for (int q = 1; q < 4; ++q) s += A[r * 4 + q] * B[q * 4 + c];
        D[r * 4 + c] = D[r * 4 + c] + sgn * s;
      }
  };
  // row j's sweep factors: inv, G (the forward-recurrence coupling), C (the
  // back-substitution coupling), and the i-couplings P = inv JIL(i), Q = inv JIR(i+1)
  auto store_row = [&](int j, const double inv[16], const double Gm[16], const double Cm[16]) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const size_t q = fbidx(cs.rows_nc, nc, grp.g, j, e >> 2, e & 3, lane);
      INV[q] = TJ(inv[e]);
      nsat += out_of_range<TF>(Cm[e]) + out_of_range<TF>(Gm[e]);
      CF[q] = from_f64<TF>(Cm[e]);
      PQG[fbidx3(cs.rows_nc, nc, grp.g, j, 2, e >> 2, e & 3, lane)] = from_f64<TF>(Gm[e]);
    }
    double T1[16];
    load_block(JIL, cs.rows_nc, nc, grp.g, j, lane, T1);
    mul4_store(inv, T1, PQG, cs.rows_nc, nc, grp.g, j, 0, lane, nsat);
    load_block(JIR, cs.rows_nc, nc, gp, j, lp, T1);
    mul4_store(inv, T1, PQG, cs.rows_nc, nc, grp.g, j, 1, lane, nsat);
  };
  // The line system is L_j x_{j-1} + D_j x_j + U_j x_{j+1} = r_j with L_j = -JJL(j),
  // U_j = JJR(j+1) (aero2d/implicit.py:81-128).
  // From the wall, rows 0 .. k-1: den_j = D_j - L_j c_{j-1}, c_j = den_j^-1 U_j,
  // G_j = -den_j^-1 L_j; later d_j = inv_j r_j + G_j d_{j-1}, x_j = d_j - c_j x_{j+1}.
  double cprev[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) cprev[e] = 0.0;
  if (half == 0 && own) {
    for (int j = 0; j < k; ++j) {
      double D[16], A[16], inv[16], Gm[16], T1[16];
      assemble(j, D);
      load_block(JJL, cs.rows_nc1, nc + 1, grp.g, j, lane, A);
      mul_add(A, cprev, D, 1.0);
      inv4(D, inv);
      mul(inv, A, Gm, 1.0);
      load_block(JJR, cs.rows_nc1, nc + 1, grp.g, j + 1, lane, T1);
      mul(inv, T1, cprev, 1.0);
      store_row(j, inv, Gm, cprev);
    }
  }
  // From the far field, rows nc-1 .. k+1: den'_j = D_j - U_j c'_{j+1},
  // c'_j = den'_j^-1 L_j, G'_j = -den'_j^-1 U_j; later d'_j = inv'_j r_j + G'_j d'_{j+1},
  // x_j = d'_j - c'_j x_{j-1}.
  double cnext[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) cnext[e] = 0.0;
  if (half == 1) {
    if (own) {
      for (int j = nc - 1; j > k; --j) {
        double D[16], A[16], Um[16], inv[16], Gm[16];
        assemble(j, D);
        load_block(JJR, cs.rows_nc1, nc + 1, grp.g, j + 1, lane, Um);
        mul_add(Um, cnext, D, -1.0);
        inv4(D, inv);
        mul(inv, Um, Gm, -1.0);
        load_block(JJL, cs.rows_nc1, nc + 1, grp.g, j, lane, A);
        mul(inv, A, cnext, -1.0);
        store_row(j, inv, Gm, cnext);
      }
    }
#pragma unroll
    for (int e = 0; e < 16; ++e) cfar[pair][e][lane] = cnext[e];
  }
  asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory");   // the pair's two warps
  if (half == 1 || !own) {
    if (nsat != 0 && a.sat != nullptr) atomicAdd(a.sat, (unsigned long long)nsat);
    return;
  }
#pragma unroll
  for (int e = 0; e < 16; ++e) cnext[e] = cfar[pair][e][lane];
  // Row k: den_k = D_k - L_k c_{k-1} - U_k c'_{k+1};
  // x_k = inv_k r_k + G_k d_{k-1} + H_k d'_{k+1}, G_k = -inv_k L_k, H_k = -inv_k U_k
  // (H is kept in the C slot of row k, which has no back substitution).
  {
    double D[16], A[16], Um[16], inv[16], Gm[16], Hm[16];
    assemble(k, D);
    load_block(JJL, cs.rows_nc1, nc + 1, grp.g, k, lane, A);
    load_block(JJR, cs.rows_nc1, nc + 1, grp.g, k + 1, lane, Um);
    mul_add(A, cprev, D, 1.0);
    mul_add(Um, cnext, D, -1.0);
    inv4(D, inv);
    mul(inv, A, Gm, 1.0);
    mul(inv, Um, Hm, -1.0);
    store_row(k, inv, Gm, Hm);
  }
  if (nsat != 0 && a.sat != nullptr) atomicAdd(a.sat, (unsigned long long)nsat);
}

template <typename T>
void launch_face_jac(const Batch& b, const JacArgs& a, cudaStream_t s) {
  if (b.ntiles == 0) return;
  k_face_jac<T><<<b.ntiles, 256, 0, s>>>(b, a);
}
template <typename TJ, typename TF>
void launch_factor(const Batch& b, const FactorArgs& a, cudaStream_t s) {
  if (b.ngroups == 0) return;
  k_factor<TJ, TF><<<(b.ngroups + 1) / 2, 128, 0, s>>>(b, a);
}

template void launch_face_jac<double>(const Batch&, const JacArgs&, cudaStream_t);
template void launch_face_jac<float>(const Batch&, const JacArgs&, cudaStream_t);
template void launch_factor<double, double>(const Batch&, const FactorArgs&, cudaStream_t);
template void launch_factor<float, __half>(const Batch&, const FactorArgs&, cudaStream_t);

}  // namespace a2d
