// Residual and per-case residual norms of a batch of cases without any device
// allocation (a2d_residual_norms_static in include/aero2d_b200.h).
//
// Some callers cannot call cudaMalloc: a host application whose memory
// manager owns all device memory and does not let a plugin allocate, or a
// loop that must not allocate while it runs.  This entry point serves them: the
// caller passes the inputs and outputs, and the only other device memory it
// touches is g_scratch below, a file-scope array that every GPU loading the
// library holds until the process exits.  The scratch holds the batch's case
// and tile tables and the per-tile partial sums of the residual norm.
//
// Every call rebuilds the tables and overwrites every partial it reads, so
// nothing carries over between calls; calls whose kernels overlap on the GPU
// (on two streams at once) share the array and race.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "aero2d_b200.h"
#include "batch.cuh"
#include "kernels.cuh"

namespace a2d {

int fail(int code, const std::string& msg);

// the largest batch the entry point serves
constexpr int kStaticMaxCases = 64;
constexpr int kStaticMaxNi = 512;
constexpr int kStaticMaxNc = 128;
constexpr int kStaticTilesPerCase = ((kStaticMaxNi + kTI - 1) / kTI) * ((kStaticMaxNc + kTJ - 1) / kTJ);
constexpr int kStaticMaxTiles = kStaticMaxCases * kStaticTilesPerCase;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffCases = 0;
constexpr size_t kOffTiles = align256(kOffCases + sizeof(CaseDev) * kStaticMaxCases);
constexpr size_t kOffPart = align256(kOffTiles + sizeof(Tile) * kStaticMaxTiles);
constexpr size_t kStaticScratchBytes = align256(kOffPart + sizeof(double) * kTilePartStride * kStaticMaxTiles);

// about 0.86 MB per GPU
static __device__ __align__(256) unsigned char g_scratch[kStaticScratchBytes];

// case and tile tables of a uniform batch (every case on one grid), built on the device
__global__ void k_static_tables(unsigned char* scratch, const void* metrics, int ni, int nc, int ncases,
                                const double* winf) {
  CaseDev* cases = reinterpret_cast<CaseDev*>(scratch + kOffCases);
  Tile* tiles = reinterpret_cast<Tile*>(scratch + kOffTiles);
  const int nti = (ni + kTI - 1) / kTI, ntj = (nc + kTJ - 1) / kTJ;
  const int tpc = nti * ntj;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ncases) {
    CaseDev c{};
    c.g = grid_view(metrics, ni, nc);
    for (int q = 0; q < 4; ++q) c.winf[q] = winf[4 * t + q];
    c.cell_off = (long long)t * ni * nc;
    c.tile0 = t * tpc;
    c.ntiles = tpc;
    cases[t] = c;
  }
  if (t < ncases * tpc) {
    const int k = t / tpc, r = t % tpc;
    const int i0 = (r % nti) * kTI, j0 = (r / nti) * kTJ;
    tiles[t] = Tile{k, i0, j0, ni - i0 < kTI ? ni - i0 : kTI, nc - j0 < kTJ ? nc - j0 : kTJ};
  }
}

// rn = sqrt(mean((R_rho / vol)^2)) per case from its tile partials, in tile order
__global__ void k_static_norms(const unsigned char* scratch, int ncases, int cells, double* rnorm) {
  const CaseDev* cases = reinterpret_cast<const CaseDev*>(scratch + kOffCases);
  const double* part = reinterpret_cast<const double*>(scratch + kOffPart);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncases) return;
  const CaseDev c = cases[k];
  double s = 0.0;
  for (int q = 0; q < c.ntiles; ++q) s += part[(size_t)(c.tile0 + q) * kTilePartStride];
  rnorm[k] = sqrt(s / (double)cells);
}

// device address of g_scratch for the calling thread's current context.  The
// address is looked up (cudaGetSymbolAddress, with the device current) on the
// first call on a device and again whenever that device's current context has
// changed since (e.g. the primary context was destroyed by cudaDeviceReset and
// re-created), since a module's symbols get new addresses in a new context.
// The context is identified by cuCtxGetId, fetched through the runtime's driver
// entry-point query, so the library needs no link against libcuda.
using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);

static int current_context_id(unsigned long long* id) {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault) == cudaSuccess)
      get_current = reinterpret_cast<PfnCtxGetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault) == cudaSuccess)
      get_id = reinterpret_cast<PfnCtxGetId>(f);
  });
  *id = 0;
  if (get_current == nullptr || get_id == nullptr)
    return fail(A2D_ERR_CUDA, "residual_norms_static: the driver does not export cuCtxGetCurrent/cuCtxGetId");
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return fail(A2D_ERR_CUDA, "residual_norms_static: cuCtxGetCurrent failed");
  if (ctx == nullptr) return A2D_OK;   // no context yet: id 0, the lookup creates the primary context
  if (get_id(ctx, id) != CUDA_SUCCESS) return fail(A2D_ERR_CUDA, "residual_norms_static: cuCtxGetId failed");
  return A2D_OK;
}

static int scratch_address(unsigned char** out) {
  static std::mutex mu;
  static unsigned char* addr[128] = {};
  static unsigned long long ctx_of[128] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(A2D_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 128) return fail(A2D_ERR_ARG, "device ordinal out of range");
  unsigned long long ctx = 0;
  if (int rc = current_context_id(&ctx)) return rc;
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev] == nullptr || ctx == 0 || ctx != ctx_of[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess)
      return fail(A2D_ERR_CUDA, std::string("cudaGetSymbolAddress(g_scratch): ") + cudaGetErrorString(e));
    if (ctx == 0 && current_context_id(&ctx) != A2D_OK) return A2D_ERR_CUDA;
    addr[dev] = static_cast<unsigned char*>(p);
    ctx_of[dev] = ctx;
  }
  *out = addr[dev];
  return A2D_OK;
}

}  // namespace a2d

using namespace a2d;

extern "C" int a2d_residual_norms_static(const void* metrics, int ni, int nj, int ncases, const double* U,
                                         const double* winf, const double* circ, const a2d_params* params,
                                         double* R, double* rnorm, void* stream) {
  const int nc = nj - 1;
  if (metrics == nullptr || U == nullptr || winf == nullptr || R == nullptr || rnorm == nullptr)
    return fail(A2D_ERR_ARG, "residual_norms_static: null pointer");
  if (ncases < 1 || ncases > kStaticMaxCases)
    return fail(A2D_ERR_ARG, "residual_norms_static: ncases must be in [1, " + std::to_string(kStaticMaxCases) +
                                 "], got " + std::to_string(ncases));
  if (ni < 4 || ni > kStaticMaxNi || nc < 2 || nc > kStaticMaxNc)
    return fail(A2D_ERR_ARG, "residual_norms_static: grid of " + std::to_string(ni) + " x " + std::to_string(nc) +
                                 " cells exceeds the static scratch (ni in [4, " + std::to_string(kStaticMaxNi) +
                                 "], nc in [2, " + std::to_string(kStaticMaxNc) + "])");
  a2d_params p;
  a2d_default_params(&p);
  if (params != nullptr) p = *params;
  if (p.order != 1 && p.order != 2) return fail(A2D_ERR_ARG, "residual_norms_static: order must be 1 or 2");
  unsigned char* scratch = nullptr;
  if (int e = scratch_address(&scratch)) return e;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int tpc = ((ni + kTI - 1) / kTI) * ((nc + kTJ - 1) / kTJ);
  const int ntiles = ncases * tpc;
  k_static_tables<<<(ntiles + 255) / 256, 256, 0, s>>>(scratch, metrics, ni, nc, ncases, winf);
  Batch b{};
  b.cases = reinterpret_cast<const CaseDev*>(scratch + kOffCases);
  b.tiles = reinterpret_cast<const Tile*>(scratch + kOffTiles);
  b.live = nullptr;
  b.ncases = ncases;
  b.ntiles = ntiles;
  StencilArgs<double> a;
  a.U = U;
  a.circ_in = circ;
  a.out = R;
  a.sign = 1.0;
  a.tile_part = reinterpret_cast<double*>(scratch + kOffPart);
  a.lim_k = p.lim_k;
  a.order = p.order;
  a.vortex = p.vortex_correction;
  launch_stencil<double, false, double>(b, a, s);
  k_static_norms<<<(ncases + 63) / 64, 64, 0, s>>>(scratch, ncases, ni * nc, rnorm);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(A2D_ERR_CUDA, std::string("residual_norms_static: ") + cudaGetErrorString(e));
  return A2D_OK;
}
