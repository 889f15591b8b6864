// Device-side description of a batch of Euler cases and its work
// decomposition.  A batch is a list of cases; each case has its own O-grid
// (several cases may point at the same grid metrics) and its own freestream.
// Uniform batches (one shared grid) and ragged batches (mixed grid sizes) use
// the same tables, so every kernel runs both from one launch.
//
// Memory layout in HBM (per case, cases packed one after another):
//   cell vectors     [4][nc][ni]   component, wall-normal j, circumferential i
//                                  (i fastest: a warp reads 32 neighbouring
//                                  j-lines of one row in one 256 B transaction)
//   scalar per cell  [nc][ni]
//   line blocks      [group][row][16][32]  4x4 blocks of the j-lines, 32 lines
//                                  (one warp) per group, lane fastest, so the
//                                  line solver's loads are coalesced per entry
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace a2d {

constexpr int kTI = 32;        // stencil tile width  (i, circumferential cells)
constexpr int kTJ = 8;         // stencil tile height (j, wall-normal cells)

// tile shapes of the FP32 linearised stencil (the JVP), a plan's tuning knob;
// every other tile kernel uses kTI x kTJ
enum : int { kTile32x8 = 0, kTile32x16 = 1, kTile64x4 = 2, kTile16x16 = 3, kNumTileShapes = 4 };
__host__ __device__ constexpr int tile_w(int shape) {
  return shape == kTile64x4 ? 64 : (shape == kTile16x16 ? 16 : 32);
}
__host__ __device__ constexpr int tile_h(int shape) {
  return shape == kTile32x16 || shape == kTile16x16 ? 16 : (shape == kTile64x4 ? 4 : 8);
}
constexpr int kLanes = 32;     // j-lines per line group
constexpr int kChunk = 4096;   // vector entries per reduction chunk (16 per thread of a 256-thread CTA)
constexpr int kMaxRestart = 64;

// status word bits per case
enum : uint32_t {
  kLiveNewton = 1u,   // case takes part in the current Newton step
  kLiveKrylov = 2u,   // case's Arnoldi process is still running
};

struct GridDev {
  int ni, nc;
  const double* vol;   // [nc][ni]           cell areas
  const double* Si;    // [2][nc][ni]        face between cells i-1 and i, normal toward +i
  const double* Sj;    // [2][nc+1][ni]      face j (0 = wall), normal toward +j
  const double* xf;    // [ni]               far-field face midpoints
  const double* yf;
  const double* xw;    // [ni]               wall face midpoints
  const double* yw;
  const float* vol_f;  // FP32 copies (rounded from the FP64 values)
  const float* Si_f;
  const float* Sj_f;
  const float* xf_f;
  const float* yf_f;
};

struct CaseDev {
  GridDev g;
  double winf[4];        // freestream primitives (rho, u, v, p)
  long long cell_off;    // first cell of the case in packed per-cell arrays
  long long rows_nc;     // first 32-lane row of the case in line blocks with nc rows per line
  long long rows_nc1;    // same for line blocks with nc+1 rows per line
  int tile0, ntiles;     // stencil tiles
  int chunk0, nchunks;   // reduction chunks over the 4*ni*nc vector entries
  int group0, ngroups;   // line groups
  int pad;
};

struct Tile {
  int cs, i0, j0, ti, tj;
};
struct Chunk {
  int cs, begin, len;
};
struct Group {
  int cs, g, i0, n;      // case, group index within case, first line, lines in group
};

constexpr int kTilePartStride = 4;   // per-tile partials: rho-residual^2, max rel change, non-finite, spare

// per-case state of the pseudo-transient Newton loop, on the device
struct CaseCtl {
  double circ;     // circulation used by the last residual
  double cfl;      // pseudo-time CFL of the next step
  double r0;       // first residual norm (SER reference)
  double rn;       // residual norm of the last step (NaN if it failed)
  double lastrn;   // last finite residual norm
  double omega;    // step length of the last step
  double bnorm;    // ||b|| = ||R||
  double x0norm;   // ||M b||
  double ptol;     // GMRES skip threshold
  double beta;     // ||M (b - A x0)||
  double cl, cd, cm;
  int k_used;      // Arnoldi vectors built in the last step
  int fails;       // non-finite steps so far
  int frozen;      // 1 after 5 failed steps
  int done;        // reached the tolerance (or frozen)
  int commit;      // the last step was accepted
  int stepped;     // the case took the current step
  int nsteps;      // Newton steps taken
  int keep_r0;     // r0 was carried over from the previous point of a sweep
};

struct Batch {
  const CaseDev* cases;
  const Tile* tiles;
  const Chunk* chunks;
  const Group* groups;
  const uint32_t* live;  // per-case status word (nullptr: all live)
  int ncases, ntiles, nchunks, ngroups;
};

// Layout of a grid's metrics blob: FP64 vol, Si, Sj, xf, yf, xw, yw, then (from the
// next 256-byte boundary) FP32 copies of vol, Si, Sj, xf, yf.
__host__ __device__ inline size_t metrics_doubles(int ni, int nc) {
  return 5 * (size_t)ni * nc + 6 * (size_t)ni;
}
__host__ __device__ inline size_t metrics_floats(int ni, int nc) {
  return 5 * (size_t)ni * nc + 4 * (size_t)ni;
}
__host__ __device__ inline size_t metrics_float_offset(int ni, int nc) {
  return (metrics_doubles(ni, nc) * 8 + 255) & ~size_t(255);
}
__host__ __device__ inline GridDev grid_view(const void* blob, int ni, int nc) {
  GridDev g;
  g.ni = ni;
  g.nc = nc;
  const size_t N = (size_t)ni * nc;
  const double* d = static_cast<const double*>(blob);
  g.vol = d;
  g.Si = d + N;
  g.Sj = g.Si + 2 * N;
  g.xf = g.Sj + 2 * (N + ni);
  g.yf = g.xf + ni;
  g.xw = g.yf + ni;
  g.yw = g.xw + ni;
  const float* f = reinterpret_cast<const float*>(static_cast<const char*>(blob) + metrics_float_offset(ni, nc));
  g.vol_f = f;
  g.Si_f = f + N;
  g.Sj_f = g.Si_f + 2 * N;
  g.xf_f = g.Sj_f + 2 * (N + ni);
  g.yf_f = g.xf_f + ni;
  return g;
}

// metric accessors in the compute precision
template <typename T> struct Metric;
template <> struct Metric<double> {
  const GridDev& g;
  __device__ __forceinline__ double vol(int j, int i) const { return g.vol[(size_t)j * g.ni + i]; }
  __device__ __forceinline__ double si(int k, int j, int i) const {
    return g.Si[((size_t)k * g.nc + j) * g.ni + i];
  }
  __device__ __forceinline__ double sj(int k, int j, int i) const {
    return g.Sj[((size_t)k * (g.nc + 1) + j) * g.ni + i];
  }
  __device__ __forceinline__ double xf(int i) const { return g.xf[i]; }
  __device__ __forceinline__ double yf(int i) const { return g.yf[i]; }
};
template <> struct Metric<float> {
  const GridDev& g;
  __device__ __forceinline__ float vol(int j, int i) const { return g.vol_f[(size_t)j * g.ni + i]; }
  __device__ __forceinline__ float si(int k, int j, int i) const {
    return g.Si_f[((size_t)k * g.nc + j) * g.ni + i];
  }
  __device__ __forceinline__ float sj(int k, int j, int i) const {
    return g.Sj_f[((size_t)k * (g.nc + 1) + j) * g.ni + i];
  }
  __device__ __forceinline__ float xf(int i) const { return g.xf_f[i]; }
  __device__ __forceinline__ float yf(int i) const { return g.yf_f[i]; }
};

// index of (component k, row j, column i) in a case's cell vector
__device__ __forceinline__ size_t vidx(const GridDev& g, int k, int j, int i) {
  return ((size_t)k * g.nc + j) * g.ni + i;
}

// index of entry e of row j of line (group g, lane) in a line-block array
__device__ __forceinline__ size_t lbidx(long long row0, int rows_per_line, int g, int j, int e,
                                        int lane) {
  return (((size_t)(row0 + (long long)g * rows_per_line + j)) * 16 + e) * kLanes + lane;
}

// index of entry (r, c) of row j of line (group g, lane) in the factor arrays of
// the sweeps: the group's blocks of one row are one contiguous run, as in
// lbidx, ordered [block row r][lane][column c], so that a thread holding block
// row r of one line reads its four entries with one vector load
__device__ __forceinline__ size_t fbidx(long long row0, int rows_per_line, int g, int j, int r, int c,
                                        int lane) {
  return ((((size_t)(row0 + (long long)g * rows_per_line + j)) * 4 + r) * kLanes + lane) * 4 + c;
}

// the same for the factors P, Q, G of the forward sweep (m = 0, 1, 2), kept
// interleaved per row so that one copy brings all three blocks of a step
__device__ __forceinline__ size_t fbidx3(long long row0, int rows_per_line, int g, int j, int m, int r, int c,
                                         int lane) {
  return (((((size_t)(row0 + (long long)g * rows_per_line + j)) * 3 + m) * 4 + r) * kLanes + lane) * 4 + c;
}

__device__ __forceinline__ bool case_live(const Batch& b, int cs, uint32_t need) {
  return b.live == nullptr || (b.live[cs] & need) == need;
}

}  // namespace a2d
