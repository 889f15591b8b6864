// O-grid generation on the device (a2d_grid_spacing, a2d_grid_build in
// include/aero2d_b200.h): the hyperbolic marching of aero2d/grid.py:50-81 for
// many airfoils at once, one CTA per grid, one thread per circumferential node.
//
// The layers are sequential in j and every smoothing pass couples each node to
// its two neighbours along the layer, so a CTA keeps the current layer and the
// smoothed field in shared memory (ping-pong buffers: one barrier per pass) and
// writes each finished layer once.  Every operation is the reference's, in its
// order and with IEEE rounding at each step (no contraction into FMAs), so
// layers 0 .. nj-2 are bitwise the host generator's; the spacings come from the
// host (a2d_grid_spacing) for the same reason.  The outer layer is snapped to a
// circle with CUDA's atan2/cos/sin, whose last bits may differ from the host
// library's; its mean radius is summed in NumPy's pairwise order, so only
// those functions' rounding separates it from the host grid.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "aero2d_b200.h"

namespace a2d {

int fail(int code, const std::string& msg);

namespace {

constexpr int kMaxRing = 1024;

// a + eps * (a[i-1] + a[i+1] - 2 a), the reference's expression order (aero2d/grid.py:44-47)
__device__ __forceinline__ double smooth1(double am, double a, double ap, double eps) {
  const double t = __dsub_rn(__dadd_rn(am, ap), __dmul_rn(2.0, a));
  return __dadd_rn(a, __dmul_rn(eps, t));
}

// `passes` smoothing passes of the 2-vector field (vx, vy) of node i; buf is
// [2][2][ni] ping-pong storage in shared memory; returns the smoothed value
__device__ void smooth_ring(double& vx, double& vy, double eps, int passes, int i, int im, int ip, int ni,
                            double* buf, bool on) {
  int b = 0;
  if (on) {
    buf[i] = vx;
    buf[ni + i] = vy;
  }
  __syncthreads();
  for (int p = 0; p < passes; ++p) {
    const double* src = buf + b * 2 * ni;
    double* dst = buf + (b ^ 1) * 2 * ni;
    if (on) {
      vx = smooth1(src[im], src[i], src[ip], eps);
      vy = smooth1(src[ni + im], src[ni + i], src[ni + ip], eps);
      dst[i] = vx;
      dst[ni + i] = vy;
    }
    b ^= 1;
    __syncthreads();
  }
}

// NumPy's pairwise summation of a contiguous float64 array (blocks of 8
// partial sums up to 128 entries, halves at multiples of 8 above): the order of
// np.mean in aero2d/grid.py:75, so the mean radius is the host's to the bit
__device__ double pairwise_sum(const double* a, int n) {
  // explicit stack instead of recursion: (offset, length, state) frames
  struct Frame {
    int lo, n, stage;
    double left;
  };
  Frame st[16];
  int top = 0;
  st[0] = {0, n, 0, 0.0};
  double ret = 0.0;
  while (true) {
    Frame& f = st[top];
    if (f.n <= 128 && f.stage == 0) {
      double res;
      if (f.n < 8) {
        res = -0.0;
        for (int q = 0; q < f.n; ++q) res = __dadd_rn(res, a[f.lo + q]);
      } else {
        double r[8];
        for (int k = 0; k < 8; ++k) r[k] = a[f.lo + k];
        int q = 8;
        for (; q < f.n - (f.n % 8); q += 8)
          for (int k = 0; k < 8; ++k) r[k] = __dadd_rn(r[k], a[f.lo + q + k]);
        res = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                        __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
        for (; q < f.n; ++q) res = __dadd_rn(res, a[f.lo + q]);
      }
      ret = res;
      if (top == 0) return ret;
      --top;
      continue;
    }
    int n2 = f.n / 2;
    n2 -= n2 % 8;
    if (f.stage == 0) {           // left half first
      f.stage = 1;
      st[++top] = {f.lo, n2, 0, 0.0};
    } else if (f.stage == 1) {    // left done: keep it, then the right half
      f.left = ret;
      f.stage = 2;
      st[++top] = {f.lo + n2, f.n - n2, 0, 0.0};
    } else {                      // both done
      ret = __dadd_rn(f.left, ret);
      if (top == 0) return ret;
      --top;
    }
  }
}

// one grid per CTA; ring [n][ni][2], spacing [n][nj-1], x/y [n][ni][nj], min_area [n]
__global__ void __launch_bounds__(kMaxRing) k_ogrid(int ni, int nj, const double* __restrict__ ring,
                                                    const double* __restrict__ spacing, int normal_smoothing,
                                                    double* __restrict__ x, double* __restrict__ y,
                                                    double* __restrict__ min_area) {
  extern __shared__ double sm[];
  double* cur = sm;             // [2][ni] current layer
  double* buf = sm + 2 * ni;    // [2][2][ni] smoothing ping-pong
  const int g = blockIdx.x;
  const int i = threadIdx.x;
  const bool on = i < ni;
  const int im = on ? (i == 0 ? ni - 1 : i - 1) : 0;
  const int ip = on ? (i == ni - 1 ? 0 : i + 1) : 0;
  const double* rg = ring + 2 * (size_t)ni * g;
  const double* sp = spacing + (size_t)(nj - 1) * g;
  double* xg = x + (size_t)ni * nj * g;
  double* yg = y + (size_t)ni * nj * g;

  double cx = 0.0, cy = 0.0;
  if (on) {
    cx = rg[2 * i];
    cy = rg[2 * i + 1];
    cur[i] = cx;
    cur[ni + i] = cy;
    xg[(size_t)i * nj] = cx;
    yg[(size_t)i * nj] = cy;
  }
  __syncthreads();
  for (int j = 1; j < nj; ++j) {
    // unit tangent from the neighbours, normal = (t_y, -t_x) (aero2d/grid.py:58-60)
    double nx = 0.0, ny = 0.0;
    if (on) {
      const double tx = __dsub_rn(cur[ip], cur[im]);
      const double ty = __dsub_rn(cur[ni + ip], cur[ni + im]);
      const double len = __dsqrt_rn(__dadd_rn(__dmul_rn(tx, tx), __dmul_rn(ty, ty)));
      nx = __ddiv_rn(ty, len);
      ny = -__ddiv_rn(tx, len);
    }
    smooth_ring(nx, ny, 0.25, j > 1 ? normal_smoothing : 2, i, im, ip, ni, buf, on);
    if (on) {
      const double len = __dsqrt_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)));
      nx = __ddiv_rn(nx, len);
      ny = __ddiv_rn(ny, len);
    }
    // step out by this layer's spacing, then smooth along the layer (:62-64)
    const double frac = __ddiv_rn((double)j, (double)(nj - 1));
    const double s = sp[j - 1];
    double px = 0.0, py = 0.0;
    if (on) {
      px = __dadd_rn(cx, __dmul_rn(s, nx));
      py = __dadd_rn(cy, __dmul_rn(s, ny));
    }
    const double eps = __dadd_rn(0.1, __dmul_rn(0.3, frac));
    const int passes = 2 + (int)__dmul_rn(8.0, frac);
    smooth_ring(px, py, eps, passes, i, im, ip, ni, buf, on);
    cx = px;
    cy = py;
    if (on) {
      cur[i] = cx;
      cur[ni + i] = cy;
      if (j < nj - 1) {
        xg[(size_t)i * nj + j] = cx;
        yg[(size_t)i * nj + j] = cy;
      }
    }
    __syncthreads();
  }
  // outer layer on a circle of the mean radius about (0.5, 0) (:65-69)
  double rx = 0.0, ry = 0.0;
  if (on) {
    rx = __dsub_rn(cx, 0.5);
    ry = __dsub_rn(cy, 0.0);
    buf[i] = __dsqrt_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)));
  }
  __syncthreads();
  __shared__ double rmean;
  if (i == 0) rmean = __ddiv_rn(pairwise_sum(buf, ni), (double)ni);
  __syncthreads();
  if (on) {
    const double ang = atan2(ry, rx);
    cx = __dadd_rn(0.5, __dmul_rn(rmean, cos(ang)));
    cy = __dadd_rn(0.0, __dmul_rn(rmean, sin(ang)));
    xg[(size_t)i * nj + nj - 1] = cx;
    yg[(size_t)i * nj + nj - 1] = cy;
  }
  __syncthreads();
  // smallest cell area from the two diagonals (aero2d/grid.py:24-31, :78-80)
  double amin = INFINITY;
  if (on) {
    const double* x0 = xg + (size_t)i * nj;
    const double* y0 = yg + (size_t)i * nj;
    const double* x1 = xg + (size_t)ip * nj;
    const double* y1 = yg + (size_t)ip * nj;
    for (int j = 0; j < nj - 1; ++j) {
      const double d1x = x1[j + 1] - x0[j], d1y = y1[j + 1] - y0[j];
      const double d2x = x0[j + 1] - x1[j], d2y = y0[j + 1] - y1[j];
      amin = fmin(amin, -0.5 * (d1x * d2y - d1y * d2x));
    }
  }
  for (int o = 16; o > 0; o >>= 1) amin = fmin(amin, __shfl_xor_sync(0xffffffffu, amin, o));
  __shared__ double wmin[kMaxRing / 32];
  if ((i & 31) == 0) wmin[i >> 5] = amin;
  __syncthreads();
  if (i == 0) {
    double m = INFINITY;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmin(m, wmin[w]);
    min_area[g] = m;
  }
}

}  // namespace
}  // namespace a2d

using namespace a2d;

extern "C" {

int a2d_grid_spacing(int nj, double ds0, double radius, double* spacing) {
  if (nj < 2 || !(ds0 > 0.0) || !(radius > ds0) || spacing == nullptr)
    return fail(A2D_ERR_ARG, "grid_spacing: bad arguments");
  // growth ratio by 200 bisection steps on [1 + 1e-9, 2] (aero2d/grid.py:34-41)
  const int n = nj - 1;
  double lo = 1.0 + 1e-9, hi = 2.0;
  for (int it = 0; it < 200; ++it) {
    const double r = 0.5 * (lo + hi);
    const double total = ds0 * (std::pow(r, (double)n) - 1.0) / (r - 1.0);
    if (total < radius) lo = r;
    else hi = r;
  }
  const double r = 0.5 * (lo + hi);
  for (int k = 0; k < n; ++k) spacing[k] = ds0 * std::pow(r, (double)k);
  return A2D_OK;
}

int a2d_grid_build(int n, int ni, int nj, const double* ring, const double* spacing, int normal_smoothing,
                   double* x, double* y, double* min_area, void* stream) {
  if (n < 0 || ni < 3 || ni > kMaxRing || nj < 2 || normal_smoothing < 0 || normal_smoothing > 1000)
    return fail(A2D_ERR_ARG, "grid_build: bad sizes (3 <= ni <= 1024, nj >= 2)");
  if (n == 0) return A2D_OK;
  if (ring == nullptr || spacing == nullptr || x == nullptr || y == nullptr || min_area == nullptr)
    return fail(A2D_ERR_ARG, "grid_build: null pointer");
  const int threads = (ni + 31) / 32 * 32;
  const size_t smem = sizeof(double) * 6 * (size_t)ni;
  cudaFuncSetAttribute(k_ogrid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(double) * 6 * kMaxRing));
  k_ogrid<<<n, threads, smem, static_cast<cudaStream_t>(stream)>>>(ni, nj, ring, spacing, normal_smoothing, x,
                                                                   y, min_area);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(A2D_ERR_CUDA, std::string("grid_build: ") + cudaGetErrorString(e));
  return A2D_OK;
}

}  // extern "C"
