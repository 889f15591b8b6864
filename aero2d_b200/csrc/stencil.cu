// Fused finite-volume residual of the 2-D Euler equations on the O-grid and its
// forward linearisation (the Jacobian-vector product of the Newton-Krylov
// solver), plus the grid metrics, the wall forces and the circulation.
//
// One CTA owns a 32 (i) x 8 (j) tile of cells of one case.  It stages the
// primitive state of the tile and a 2-cell halo in shared memory (wall and
// far-field ghosts are formed while staging), computes every i- and j-face
// flux of the tile once (MUSCL + smooth van Albada + positivity clamp + HLLC),
// and writes R = (F_i[i+1] - F_i[i]) + (F_j[j+1] - F_j[j]) per cell.  The
// linearised variant runs the same code on dual numbers; its far-field ghost
// carries the derivative of the circulation, which every far-field tile
// reduces itself from the wall rows in a fixed order.
//
// Reference: aero2d/euler.py:44-60 (metrics), :259-287 (residual),
// :315-331 (forces), aero2d/implicit.py:160-181 (circulation and JVP).
#include <type_traits>

#include "batch.cuh"
#include "kernels.cuh"
#include "physics.cuh"
#include "stencil_impl.cuh"

namespace a2d {

// ---------------------------------------------------------------------------
// metrics from node coordinates (reference layout x[i][j], nj = nc + 1)
// ---------------------------------------------------------------------------
__global__ void k_metrics(int ni, int nc, const double* __restrict__ x, const double* __restrict__ y,
                          double* __restrict__ md, float* __restrict__ mf) {
  const int nj = nc + 1;
  const size_t N = (size_t)ni * nc;
  double* vol = md;
  double* Si = vol + N;
  double* Sj = Si + 2 * N;
  double* xf = Sj + 2 * (N + ni);
  double* yf = xf + ni;
  double* xw = yf + ni;
  double* yw = xw + ni;
  float* vol_f = mf;
  float* Si_f = vol_f + N;
  float* Sj_f = Si_f + 2 * N;
  float* xf_f = Sj_f + 2 * (N + ni);
  float* yf_f = xf_f + ni;
  const size_t total = (size_t)ni * nj;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(t / ni), i = (int)(t % ni);
    const int i1 = (i + 1 == ni) ? 0 : i + 1;
    const double x00 = x[(size_t)i * nj + j], y00 = y[(size_t)i * nj + j];
    const double x10 = x[(size_t)i1 * nj + j], y10 = y[(size_t)i1 * nj + j];
    // j-faces: edge (i,j)->(i+1,j), normal (dy, -dx)
    const double sjx = __dsub_rn(y10, y00), sjy = -__dsub_rn(x10, x00);
    Sj[(size_t)j * ni + i] = sjx;
    Sj[(N + ni) + (size_t)j * ni + i] = sjy;
    Sj_f[(size_t)j * ni + i] = (float)sjx;
    Sj_f[(N + ni) + (size_t)j * ni + i] = (float)sjy;
    if (j == 0) {
      xw[i] = 0.5 * __dadd_rn(x00, x10);
      yw[i] = 0.5 * __dadd_rn(y00, y10);
    }
    if (j == nc) {
      xf[i] = 0.5 * __dadd_rn(x00, x10);
      yf[i] = 0.5 * __dadd_rn(y00, y10);
      xf_f[i] = (float)xf[i];
      yf_f[i] = (float)yf[i];
    }
    if (j < nc) {
      const double x01 = x[(size_t)i * nj + j + 1], y01 = y[(size_t)i * nj + j + 1];
      const double x11 = x[(size_t)i1 * nj + j + 1], y11 = y[(size_t)i1 * nj + j + 1];
      // i-faces: edge (i,j)->(i,j+1), normal (-dy, dx)
      const double six = -__dsub_rn(y01, y00), siy = __dsub_rn(x01, x00);
      Si[(size_t)j * ni + i] = six;
      Si[N + (size_t)j * ni + i] = siy;
      Si_f[(size_t)j * ni + i] = (float)six;
      Si_f[N + (size_t)j * ni + i] = (float)siy;
      // area from the diagonals (aero2d/grid.py:24-31), no fused multiply-add
      const double d1x = __dsub_rn(x11, x00), d1y = __dsub_rn(y11, y00);
      const double d2x = __dsub_rn(x01, x10), d2y = __dsub_rn(y01, y10);
      const double a = -0.5 * __dsub_rn(__dmul_rn(d1x, d2y), __dmul_rn(d1y, d2x));
      vol[(size_t)j * ni + i] = a;
      vol_f[(size_t)j * ni + i] = (float)a;
    }
  }
}


// ---------------------------------------------------------------------------
// wall forces: Cl, Cd, Cm and the wall pressure coefficient (euler.py:315-331)
// one block per case
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_forces(Batch b, const double* __restrict__ U,
                                                double* __restrict__ coef /* [ncases][3] */,
                                                double* __restrict__ cp_out, const long long* cp_off,
                                                const CaseCtl* ctl, double* hist_cl, int hist_cap) {
  const int cs_id = blockIdx.x;
  if (!case_live(b, cs_id, 0)) return;
  const CaseDev cs = b.cases[cs_id];
  const GridDev& g = cs.g;
  const double* Uc = U + 4 * cs.cell_off;
  const double uinf = cs.winf[1], vinf = cs.winf[2], pinf = cs.winf[3];
  const double q = 0.5 * (uinf * uinf + vinf * vinf);
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < g.ni; i += blockDim.x) {
    const State4<double> W0 = cons_to_prim<double, double>(load_cons<double, double>(Uc, g, 0, i));
    const State4<double> W1 = cons_to_prim<double, double>(load_cons<double, double>(Uc, g, 1, i));
    const double pw = 1.5 * W0.c[3] - 0.5 * W1.c[3];
    const double cp = (pw - pinf) / q;
    const double s0 = g.Sj[i], s1 = g.Sj[(size_t)(g.nc + 1) * g.ni + i];
    acc[0] += cp * s0;
    acc[1] += cp * s1;
    acc[2] += cp * ((g.xw[i] - 0.25) * s1 - g.yw[i] * s0);
    if (cp_out != nullptr) cp_out[cp_off[cs_id] + i] = cp;
  }
  __shared__ double scratch[32 * 3];
  block_sum<double, 3>(acc, scratch);
  if (threadIdx.x == 0) {
    const double fx = -acc[0], fy = -acc[1];
    const double mach = sqrt(2 * q);
    const double ca = uinf / mach, sa = vinf / mach;
    coef[3 * cs_id + 0] = fy * ca - fx * sa;
    coef[3 * cs_id + 1] = fx * ca + fy * sa;
    coef[3 * cs_id + 2] = acc[2];
    if (ctl != nullptr && ctl[cs_id].stepped) {
      const int it = ctl[cs_id].nsteps - 1;
      if (it >= 0 && it < hist_cap) hist_cl[(size_t)it * b.ncases + cs_id] = fy * ca - fx * sa;
    }
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
void launch_metrics(int ni, int nc, const double* x, const double* y, double* md, float* mf,
                    cudaStream_t s) {
  const size_t total = (size_t)ni * (nc + 1);
  const int blocks = (int)((total + 255) / 256);
  k_metrics<<<blocks, 256, 0, s>>>(ni, nc, x, y, md, mf);
}

template void launch_stencil<double, false, double>(const Batch&, const StencilArgs<double>&, cudaStream_t, int);
template void launch_stencil<double, true, double>(const Batch&, const StencilArgs<double>&, cudaStream_t, int);

void stencil_init_fp64() {
  stencil_cap<double, false, double, kTI, kTJ>();
  stencil_cap<double, true, double, kTI, kTJ>();
}

void launch_forces(const Batch& b, const double* U, double* coef, double* cp, const long long* cp_off,
                   const CaseCtl* ctl, double* hist_cl, int hist_cap, cudaStream_t s) {
  if (b.ncases == 0) return;
  k_forces<<<b.ncases, 256, 0, s>>>(b, U, coef, cp, cp_off, ctl, hist_cl, hist_cap);
}

}  // namespace a2d
