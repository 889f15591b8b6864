// Arnoldi orthogonalisation of the GMRES cycle: classical Gram-Schmidt run
// twice (the scheme of aero2d/krylov.py:45-50), in three passes over the
// Krylov basis per Arnoldi step.
//
//   pass 1  k_gs_dots     raw projections V_raw[q] . w and w . w, per chunk
//   reduce  k_gs_reduce   per case, fixed chunk order: h1_q = s_q (V_raw[q] . w)
//   pass 2  k_gs_project  w' = w - sum_q V_raw[q] s_q h1_q and V_raw[q] . w' from one
//                         read of the basis (the sub-tile stays in shared memory
//                         between the subtraction and the projection)
//   reduce  k_gs_reduce   h2_q
//   pass 3  k_gs_sub      w'' = w - sum_q V_raw[q] s_q (h1_q + h2_q), written as the
//                         next raw basis vector, with its squared norm
//   close   k_gs_close    per case: h_{k+1,k} = ||w''||, the breakdown test against
//                         eps ||w|| (jax.scipy.sparse.linalg.gmres semantics), the
//                         Hessenberg column and s_{k+1} = 1 / ||w''||
//
// The three passes stream a 4096-entry chunk per CTA through shared memory by
// bulk copies (see "streaming passes" below); a thread keeps one partial sum
// per basis vector in registers (the count is a template tier NQ of 8, 16, 24
// or 32), so a chunk needs a single block reduction.  Bases of more than 32
// vectors are processed in slices of 32 by chained launches.  Basis vectors
// are stored unnormalised with their scale s_q, so no normalisation pass is
// needed; w' is never stored, since pass 3 subtracts h1 + h2 from the
// original w (equal to the two successive subtractions in exact arithmetic).
#include <cfloat>
#include <cuda_bf16.h>
#include <type_traits>

#include "batch.cuh"
#include "gs.cuh"
#include "tma.cuh"

namespace a2d {

constexpr int kGB = 256;                 // threads per block
constexpr int kGE = kChunk / kGB;        // entries per thread
static_assert(kGE * kGB == kChunk, "chunk must split evenly over the block");

// fixed-order reduction of NV values over the block; thread t < NV receives value t
template <int NV>
__device__ __forceinline__ double gs_reduce_to_thread(double (&v)[NV], double* scratch /* 8*NV */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) scratch[warp * NV + q] = v[q];
  }
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < NV) {
    for (int w = 0; w < kGB / 32; ++w) s += scratch[w * NV + threadIdx.x];
  }
  return s;
}

// fixed-order sum of a per-chunk partial over a case's chunks (every lane gets it)
__device__ __forceinline__ double warp_chunk_sum(const double* p, size_t stride, int nchunks) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int c = lane; c < nchunks; c += 32) s += p[(size_t)c * stride];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// s_q (h1_q [+ h2_q]) of the slice's vectors into shared memory
template <typename TB>
__device__ __forceinline__ void coef_to_smem(const GsArgs<TB>& a, int cs, int ncases, double* coef, bool both) {
  for (int q = threadIdx.x; q < a.nq; q += blockDim.x) {
    const int qq = a.q0 + q;
    double h = a.h1[(size_t)cs * kHStride + qq];
    if (both) h += a.h2[(size_t)cs * kHStride + qq];
    coef[q] = h * a.scale[(size_t)qq * ncases + cs];
  }
  __syncthreads();
}

// the same from the folded reduction: one warp per coefficient reduces the case's
// chunk partials in k_gs_reduce's order; the case's first chunk stores the result
template <typename TB>
__device__ __forceinline__ void coef_folded(const GsArgs<TB>& a, const CaseDev& cs, int cs_id, int ncases,
                                            bool first_chunk, double* coef, bool both) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nred = a.nq + (a.fold_wn0 != nullptr ? 1 : 0);
  for (int q = warp; q < nred; q += blockDim.x >> 5) {
    const double sum = warp_chunk_sum(a.fold_part + (size_t)cs.chunk0 * a.pstride + q, a.pstride, cs.nchunks);
    if (lane == 0) {
      if (q < a.nq) {
        const double sc = a.scale[(size_t)q * ncases + cs_id];
        const double h = sum * sc;
        if (first_chunk) a.fold_h[(size_t)cs_id * kHStride + q] = h;
        const double hh = both ? a.h1[(size_t)cs_id * kHStride + q] + h : h;
        coef[q] = hh * sc;
      } else if (first_chunk) {
        a.fold_wn0[cs_id] = sqrt(sum);
      }
    }
  }
  __syncthreads();
}

// vector loads and stores of N consecutive entries (chunks start on multiples of
// 4 entries and every case vector and basis vector on a 256-byte boundary)
__device__ __forceinline__ void ldv(const float* p, double (&v)[4]) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ldv(const double* p, double (&v)[4]) {
  const double2 t0 = *reinterpret_cast<const double2*>(p);
  const double2 t1 = *reinterpret_cast<const double2*>(p + 2);
  v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
}
__device__ __forceinline__ void ldv(const float* p, double (&v)[2]) {
  const float2 t = *reinterpret_cast<const float2*>(p);
  v[0] = t.x; v[1] = t.y;
}
__device__ __forceinline__ void ldv(const double* p, double (&v)[2]) {
  const double2 t = *reinterpret_cast<const double2*>(p);
  v[0] = t.x; v[1] = t.y;
}
__device__ __forceinline__ void stv(float* p, const double (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
__device__ __forceinline__ void stv(double* p, const double (&v)[4]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
}
// one basis entry in FP64, and back in its storage precision
__device__ __forceinline__ double entry_f64(double v) { return v; }
__device__ __forceinline__ double entry_f64(float v) { return v; }
__device__ __forceinline__ double entry_f64(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename TB> __device__ __forceinline__ TB to_basis(double x) { return TB(x); }
template <> __device__ __forceinline__ __nv_bfloat16 to_basis<__nv_bfloat16>(double x) {
  return __float2bfloat16_rn((float)x);
}

__device__ __forceinline__ void stv(__nv_bfloat16* p, const double (&v)[4]) {
  __nv_bfloat162 lo = __floats2bfloat162_rn((float)v[0], (float)v[1]);
  __nv_bfloat162 hi = __floats2bfloat162_rn((float)v[2], (float)v[3]);
  uint2 raw;
  raw.x = *reinterpret_cast<uint32_t*>(&lo);
  raw.y = *reinterpret_cast<uint32_t*>(&hi);
  *reinterpret_cast<uint2*>(p) = raw;
}

// ---------------------------------------------------------------------------
// streaming passes.  A CTA of kGT threads owns one chunk and walks it in
// sub-tiles of E entries; the E entries of w and of every basis vector of the
// slice for one sub-tile (one stage) arrive by bulk copies on one mbarrier,
// through a ring of as many stages as the shared-memory budget holds, issued
// by thread 0 as soon as a stage is free.  The BF16 basis takes a smaller budget
// than the others, so that more CTAs fit on an SM (measured at 64 cases: resident
// CTAs hide the bulk copies better than a deeper ring).  Thread t works on entries
// t*EPT .. t*EPT+EPT-1 of each sub-tile and keeps one partial sum per basis
// vector in registers (NQ >= nq of them, a template tier); the chunk ends with
// one fixed-order block reduction, so the result does not depend on which
// other cases share the batch.
// ---------------------------------------------------------------------------
constexpr int kGT = 256;
constexpr int kGsMaxStages = 8;
constexpr size_t kGsSmemBudget = 74 * 1024;     // three CTAs per SM
constexpr int kGsHeader = 128;                  // mbarriers and abort flags before the stages

template <typename TB> struct GsTile;
// 2 KB runs of every basis vector per stage (measured: larger runs beat deeper
// rings; three CTAs per SM beat one CTA with more stages)
template <> struct GsTile<float> { static constexpr int E = 512; };
template <> struct GsTile<double> { static constexpr int E = 256; };
template <> struct GsTile<__nv_bfloat16> { static constexpr int E = 1024; };

template <typename TB>
__host__ __device__ inline uint32_t gs_stage_bytes(int nq) {
  return (uint32_t)GsTile<TB>::E * (uint32_t)(nq * sizeof(TB) + 8);
}
static_assert(kGsSmemBudget >= (size_t)GsTile<float>::E * (32 * 4 + 8) &&
                  kGsSmemBudget >= (size_t)GsTile<double>::E * (32 * 8 + 8) &&
                  kGsSmemBudget >= (size_t)GsTile<__nv_bfloat16>::E * (32 * 2 + 8),
              "one stage of a 32-vector slice must fit the shared-memory budget");

// shared-memory budget of the ring: 40 KB for the BF16 basis (slices of up to 13
// vectors keep 2 stages or more, larger ones one stage and four or five CTAs per SM)
template <typename TB>
__host__ __device__ constexpr size_t gs_budget() {
  return std::is_same<TB, __nv_bfloat16>::value ? 40 * 1024 : kGsSmemBudget;
}

template <typename TB>
__host__ __device__ inline int gs_stages(int nq) {
  const int s = (int)(gs_budget<TB>() / gs_stage_bytes<TB>(nq));
  return s < 1 ? 1 : (s > kGsMaxStages ? kGsMaxStages : s);
}

// fixed-order reduction of NV values over the kGT threads; thread t < NV receives value t
template <int NV>
__device__ __forceinline__ double gs_block_reduce(double (&v)[NV], double* scratch /* (kGT/32)*NV */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
  __syncthreads();   // the scratch may alias the last stage, still read above
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) scratch[warp * NV + q] = v[q];
  }
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < NV) {
#pragma unroll
    for (int w = 0; w < kGT / 32; ++w) s += scratch[w * NV + threadIdx.x];
  }
  return s;
}

// EPT consecutive entries in their storage precision, from shared memory
template <typename TB, int EPT> struct VecOf;
template <> struct VecOf<float, 1> { using type = float; };
template <> struct VecOf<float, 2> { using type = float2; };
template <> struct VecOf<float, 4> { using type = float4; };
template <> struct VecOf<double, 1> { using type = double; };
template <> struct VecOf<double, 2> { using type = double2; };
struct alignas(16) Double4x { double2 lo, hi; };
template <> struct VecOf<double, 4> { using type = Double4x; };
template <> struct VecOf<__nv_bfloat16, 1> { using type = __nv_bfloat16; };
template <> struct VecOf<__nv_bfloat16, 2> { using type = __nv_bfloat162; };
struct alignas(8) Bf16x4 { __nv_bfloat162 lo, hi; };
template <> struct VecOf<__nv_bfloat16, 4> { using type = Bf16x4; };

template <typename TB, int EPT>
struct Entries {
  alignas(sizeof(typename VecOf<TB, EPT>::type)) TB v[EPT];
  __device__ __forceinline__ void load(const TB* p) {
    using V = typename VecOf<TB, EPT>::type;
    *reinterpret_cast<V*>(v) = *reinterpret_cast<const V*>(p);
  }
  __device__ __forceinline__ double operator[](int u) const { return entry_f64(v[u]); }
};

// the ring of one streaming pass over a chunk
template <typename TB>
struct GsRing {
  static constexpr int E = GsTile<TB>::E;
  static constexpr int EPT = E / kGT;
  unsigned char* stages;
  uint64_t* full;
  int* abort;
  int S, nq, len, nsub;
  uint32_t stage_bytes;
  const TB* V;        // first vector of the slice, at the chunk's first entry
  size_t vstride;
  const double* w;    // at the chunk's first entry
  uint64_t pol;       // L2 policy of the basis runs: evict first, so that w (re-read by the
                      // three passes of an Arnoldi step) stays in L2

  __device__ void init(unsigned char* smem, const GsArgs<TB>& a, const Chunk& ch, size_t base) {
    full = reinterpret_cast<uint64_t*>(smem);
    abort = reinterpret_cast<int*>(smem + 8 * kGsMaxStages);
    stages = smem + kGsHeader;
    nq = a.nq;
    S = gs_stages<TB>(nq);
    stage_bytes = gs_stage_bytes<TB>(nq);
    len = ch.len;
    nsub = (len + E - 1) / E;
    V = a.V + (size_t)a.q0 * a.vstride + base;
    vstride = a.vstride;
    w = a.w + base;
    pol = l2_evict_first();
    if (threadIdx.x == 0) {
      for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
      mbar_init_fence();
      abort[0] = abort[1] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int u = 0; u < S; ++u) issue(u);
  }
  // sub-tile u: entries u*E .. of the chunk (len is a multiple of 4 entries, so
  // every copy is a multiple of 16 bytes)
  __device__ void issue(int u) const {
    if (u >= nsub) return;
    const int e0 = u * E;
    const int n = min(E, len - e0);
    const int s = u % S;
    unsigned char* st = stages + (size_t)s * stage_bytes;
    mbar_arrive_expect(&full[s], (uint32_t)n * (uint32_t)(nq * sizeof(TB) + 8));
    for (int q = 0; q < nq; ++q)
      bulk_load_hint(st + (size_t)q * E * sizeof(TB), V + (size_t)q * vstride + e0, n * sizeof(TB), &full[s], pol);
    bulk_load(st + (size_t)nq * E * sizeof(TB), w + e0, n * 8, &full[s]);
  }
  __device__ const TB* vec(int u, int q) const {
    return reinterpret_cast<const TB*>(stages + (size_t)(u % S) * stage_bytes) + (size_t)q * E;
  }
  __device__ const double* wvec(int u) const {
    return reinterpret_cast<const double*>(stages + (size_t)(u % S) * stage_bytes + (size_t)nq * E * sizeof(TB));
  }
  __device__ void wait(int u) const {
    if (!mbar_wait(&full[u % S], (u / S) & 1)) abort[u & 1] = 1;
  }
  // after consuming sub-tile u: frees its stage; false once a wait has run out
  __device__ bool release(int u) const {
    __syncthreads();
    if (abort[u & 1]) return false;
    if (threadIdx.x == 0) issue(u + S);
    return true;
  }
  // error exit: record the failure and give the copies in flight a bounded time
  __device__ void drain(int u, uint32_t* err) const {
    if (threadIdx.x == 0) {
      if (err != nullptr) atomicExch(err, 1u);
      for (int v = u; v < u + S && v < nsub; ++v) (void)mbar_wait(&full[v % S], (v / S) & 1);
    }
    __syncthreads();
  }
};

// pass 1 (and the re-projection of the chained path) ---------------------------
template <typename TB, int NQ>
__global__ void __launch_bounds__(kGT) k_gs_dots(Batch b, GsArgs<TB> a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const Chunk ch = b.chunks[blockIdx.x];
  if (!case_live(b, ch.cs, a.need)) return;
  const CaseDev cs = b.cases[ch.cs];
  GsRing<TB> ring;
  ring.init(smem, a, ch, 4 * cs.cell_off + ch.begin);
  constexpr int EPT = GsRing<TB>::EPT;
  double acc[NQ + 1];
#pragma unroll
  for (int q = 0; q <= NQ; ++q) acc[q] = 0.0;
  const int nq = a.nq;
#pragma unroll 1
  for (int u = 0; u < ring.nsub; ++u) {
    ring.wait(u);
    const int e = threadIdx.x * EPT;
    if (e < ring.len - u * GsRing<TB>::E) {
      const double* ws = ring.wvec(u) + e;
      double w[EPT];
#pragma unroll
      for (int t = 0; t < EPT; ++t) w[t] = ws[t];
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        Entries<TB, EPT> v;
        v.load(ring.vec(u, q < nq ? q : nq - 1) + e);
        if (q < nq) {
#pragma unroll
          for (int t = 0; t < EPT; ++t) acc[q] += v[t] * w[t];
        }
      }
#pragma unroll
      for (int t = 0; t < EPT; ++t) acc[NQ] += w[t] * w[t];
    }
    if (!ring.release(u)) {
      ring.drain(u, a.err);
      return;
    }
  }
  const double r = gs_block_reduce<NQ + 1>(acc, reinterpret_cast<double*>(ring.stages));
  double* part = a.part + (size_t)blockIdx.x * a.pstride;
  if (threadIdx.x < nq) part[a.q0 + threadIdx.x] = r;
  if (a.with_norm && threadIdx.x == NQ) part[a.norm_slot] = r;
}

// pass 2, fused: w' = w - V (s h1), then V . w' --------------------------------
template <typename TB, int NQ>
__global__ void __launch_bounds__(kGT, (NQ == 24 && std::is_same<TB, __nv_bfloat16>::value) ? 3 : 0)
    k_gs_project(Batch b, GsArgs<TB> a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double coef[NQ];
  const Chunk ch = b.chunks[blockIdx.x];
  if (!case_live(b, ch.cs, a.need)) return;
  const CaseDev cs = b.cases[ch.cs];
  GsRing<TB> ring;
  ring.init(smem, a, ch, 4 * cs.cell_off + ch.begin);   // the first bulk copies go out first
  if (a.fold_part != nullptr) coef_folded(a, cs, ch.cs, b.ncases, ch.begin == 0, coef, false);
  else coef_to_smem(a, ch.cs, b.ncases, coef, false);
  constexpr int EPT = GsRing<TB>::EPT;
  double acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
  const int nq = a.nq;
#pragma unroll 1
  for (int u = 0; u < ring.nsub; ++u) {
    ring.wait(u);
    const int e = threadIdx.x * EPT;
    if (e < ring.len - u * GsRing<TB>::E) {
      const double* ws = ring.wvec(u) + e;
      double sub[EPT];
#pragma unroll
      for (int t = 0; t < EPT; ++t) sub[t] = 0.0;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        Entries<TB, EPT> v;
        v.load(ring.vec(u, q < nq ? q : nq - 1) + e);
        if (q < nq) {
#pragma unroll
          for (int t = 0; t < EPT; ++t) sub[t] += v[t] * coef[q];
        }
      }
      double wp[EPT];
#pragma unroll
      for (int t = 0; t < EPT; ++t) wp[t] = ws[t] - sub[t];
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        Entries<TB, EPT> v;
        v.load(ring.vec(u, q < nq ? q : nq - 1) + e);
        if (q < nq) {
#pragma unroll
          for (int t = 0; t < EPT; ++t) acc[q] += v[t] * wp[t];
        }
      }
    }
    if (!ring.release(u)) {
      ring.drain(u, a.err);
      return;
    }
  }
  const double r = gs_block_reduce<NQ>(acc, reinterpret_cast<double*>(ring.stages));
  if (threadIdx.x < nq) a.part[(size_t)blockIdx.x * a.pstride + threadIdx.x] = r;
}

// out = in - V (s h): pass 3, and the subtraction slices of the chained path ----
template <typename TB, int NQ>
__global__ void __launch_bounds__(kGT) k_gs_sub(Batch b, GsArgs<TB> a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double coef[NQ];
  const Chunk ch = b.chunks[blockIdx.x];
  if (!case_live(b, ch.cs, a.need)) return;
  const CaseDev cs = b.cases[ch.cs];
  const size_t base = 4 * cs.cell_off + ch.begin;
  GsRing<TB> ring;
  ring.init(smem, a, ch, base);   // the first bulk copies go out first
  if (a.fold_part != nullptr) coef_folded(a, cs, ch.cs, b.ncases, ch.begin == 0, coef, a.both != 0);
  else coef_to_smem(a, ch.cs, b.ncases, coef, a.both != 0);
  constexpr int EPT = GsRing<TB>::EPT;
  constexpr int E = GsRing<TB>::E;
  const int nq = a.nq;
  double nrm = 0.0;
#pragma unroll 1
  for (int u = 0; u < ring.nsub; ++u) {
    ring.wait(u);
    const int e = threadIdx.x * EPT;
    if (e < ring.len - u * E) {
      const double* ws = ring.wvec(u) + e;
      double sub[EPT];
#pragma unroll
      for (int t = 0; t < EPT; ++t) sub[t] = 0.0;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        Entries<TB, EPT> v;
        v.load(ring.vec(u, q < nq ? q : nq - 1) + e);
        if (q < nq) {
#pragma unroll
          for (int t = 0; t < EPT; ++t) sub[t] += v[t] * coef[q];
        }
      }
      const size_t g = base + (size_t)u * E + e;
#pragma unroll
      for (int t = 0; t < EPT; ++t) {
        const double x = ws[t] - sub[t];
        nrm += x * x;
        if (a.wout != nullptr) a.wout[g + t] = x;
        if (a.Vout != nullptr) a.Vout[g + t] = to_basis<TB>(x);
      }
    }
    if (!ring.release(u)) {
      ring.drain(u, a.err);
      return;
    }
  }
  if (a.part_norm != nullptr) {
    double v[1] = {nrm};
    const double r = gs_block_reduce<1>(v, reinterpret_cast<double*>(ring.stages));
    if (threadIdx.x == 0) a.part_norm[blockIdx.x] = r;
  }
}

// start vector: V_raw[0] = r and its squared norm ------------------------------
template <typename TB>
__global__ void __launch_bounds__(kGB) k_gs_start(Batch b, GsArgs<TB> a) {
  const Chunk ch = b.chunks[blockIdx.x];
  if (!case_live(b, ch.cs, a.need)) return;
  const CaseDev cs = b.cases[ch.cs];
  const size_t base = 4 * cs.cell_off + ch.begin;
  __shared__ double scratch[8];
  double nrm = 0.0;
#pragma unroll
  for (int s = 0; s < kGE / 4; ++s) {
    const int e = 4 * (threadIdx.x + s * kGB);
    if (e < ch.len) {
      double x[4];
      ldv(a.w + base + e, x);
      stv(a.Vout + base + e, x);
#pragma unroll
      for (int u = 0; u < 4; ++u) nrm += x[u] * x[u];
    }
  }
  double v[1] = {nrm};
  const double r = gs_reduce_to_thread<1>(v, scratch);
  if (threadIdx.x == 0) a.part_norm[blockIdx.x] = r;
}

// sum over a case's chunks of one partial, by one warp: lane c takes chunks
// c, c+32, ... in order, then a fixed butterfly; every lane gets the total
// per-case reduction of the chunk partials: one block per case, one warp per coefficient
__global__ void __launch_bounds__(256) k_gs_reduce(Batch b, GsReduceArgs a) {
  const int cs_id = blockIdx.x;
  if (!case_live(b, cs_id, a.need)) return;
  const CaseDev cs = b.cases[cs_id];
  const int nred = a.nq + (a.wn0 != nullptr ? 1 : 0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = warp; q < nred; q += blockDim.x >> 5) {
    const double s = warp_chunk_sum(a.part + (size_t)cs.chunk0 * a.pstride + q, a.pstride, cs.nchunks);
    if (lane == 0) {
      if (q < a.nq) a.h[(size_t)cs_id * kHStride + q] = s * a.scale[(size_t)q * b.ncases + cs_id];
      else a.wn0[cs_id] = sqrt(s);
    }
  }
}

// per-case close of an Arnoldi step (k >= 0) or of the start vector (k = -1),
// one warp per case ----
__global__ void __launch_bounds__(32) k_gs_close(Batch b, GsCloseArgs a) {
  const int cs_id = blockIdx.x;
  if ((a.live[cs_id] & a.need) != a.need) return;
  const CaseDev cs = b.cases[cs_id];
  const int lane = threadIdx.x;
  const double hn = sqrt(warp_chunk_sum(a.part_norm + cs.chunk0, 1, cs.nchunks));
  CaseCtl& c = a.ctl[cs_id];
  if (a.k < 0) {
    if (lane != 0) return;
    // _safe_normalize of the preconditioned residual: threshold eps
    const bool use = hn > DBL_EPSILON;
    const double beta = use ? hn : 0.0;
    a.scale[cs_id] = use ? 1.0 / hn : 0.0;
    c.beta = beta;
    c.k_used = 0;
    const bool run = beta > c.ptol && c.bnorm > 0.0;
    if (run) a.live[cs_id] |= kLiveKrylov;
    else a.live[cs_id] &= ~kLiveKrylov;
    return;
  }
  const int k = a.k;
  const bool use = hn > DBL_EPSILON * a.wn0[cs_id];
  double* H = a.H + (size_t)cs_id * kMaxRestart * (kMaxRestart + 1) + (size_t)k * (kMaxRestart + 1);
  const double* h1 = a.h1 + (size_t)cs_id * kHStride;
  const double* h2 = a.h2 + (size_t)cs_id * kHStride;
  for (int q = lane; q <= k; q += 32) H[q] = h1[q] + h2[q];
  if (lane == 0) {
    H[k + 1] = use ? hn : 0.0;
    a.scale[(size_t)(k + 1) * b.ncases + cs_id] = use ? 1.0 / hn : 0.0;
    c.k_used = k + 1;
    if (!use) a.live[cs_id] &= ~kLiveKrylov;
  }
}

// ---------------------------------------------------------------------------
// host side: tier dispatch and the chained path for more than 32 vectors
// ---------------------------------------------------------------------------
constexpr int kSlice = kGsSlice;

#define A2D_GS_DISPATCH(KERNEL)                                                              \
  template <typename TB>                                                                     \
  static void dispatch_##KERNEL(const Batch& b, const GsArgs<TB>& a, cudaStream_t s) {       \
    if (!b.nchunks) return;                                                                  \
    const size_t smem = kGsHeader + (size_t)gs_stages<TB>(a.nq) * gs_stage_bytes<TB>(a.nq);  \
    if (a.nq <= 8) KERNEL<TB, 8><<<b.nchunks, kGT, smem, s>>>(b, a);                          \
    else if (a.nq <= 16) KERNEL<TB, 16><<<b.nchunks, kGT, smem, s>>>(b, a);                   \
    else if (a.nq <= 24) KERNEL<TB, 24><<<b.nchunks, kGT, smem, s>>>(b, a);                   \
    else KERNEL<TB, 32><<<b.nchunks, kGT, smem, s>>>(b, a);                                   \
  }
A2D_GS_DISPATCH(k_gs_dots)
A2D_GS_DISPATCH(k_gs_project)
A2D_GS_DISPATCH(k_gs_sub)
#undef A2D_GS_DISPATCH

template <typename TB>
void launch_gs_dots(const Batch& b, const GsArgs<TB>& a0, cudaStream_t s) {
  GsArgs<TB> a = a0;
  a.norm_slot = a0.nq;
  for (int q0 = 0; q0 < a0.nq; q0 += kSlice) {
    a.q0 = q0;
    a.nq = a0.nq - q0 < kSlice ? a0.nq - q0 : kSlice;
    a.with_norm = a0.with_norm && q0 == 0;
    dispatch_k_gs_dots<TB>(b, a, s);
  }
}

template <typename TB>
void launch_gs_project(const Batch& b, const GsArgs<TB>& a0, cudaStream_t s) {
  if (a0.nq <= kSlice) {
    GsArgs<TB> a = a0;
    a.q0 = 0;
    dispatch_k_gs_project<TB>(b, a, s);
    return;
  }
  // chained: w' = w - V (s h1) into the scratch vector, then its projections
  GsArgs<TB> a = a0;
  a.both = 0;
  a.Vout = nullptr;
  a.part_norm = nullptr;
  for (int q0 = 0; q0 < a0.nq; q0 += kSlice) {
    a.q0 = q0;
    a.nq = a0.nq - q0 < kSlice ? a0.nq - q0 : kSlice;
    a.w = q0 == 0 ? a0.w : a0.tmp;
    a.wout = a0.tmp;
    dispatch_k_gs_sub<TB>(b, a, s);
  }
  GsArgs<TB> d = a0;
  d.w = a0.tmp;
  d.with_norm = 0;
  launch_gs_dots<TB>(b, d, s);
}

template <typename TB>
void launch_gs_finish(const Batch& b, const GsArgs<TB>& a0, cudaStream_t s) {
  GsArgs<TB> a = a0;
  a.both = 1;
  for (int q0 = 0; q0 < a0.nq; q0 += kSlice) {
    const bool last = q0 + kSlice >= a0.nq;
    a.q0 = q0;
    a.nq = a0.nq - q0 < kSlice ? a0.nq - q0 : kSlice;
    a.w = q0 == 0 ? a0.w : a0.tmp;
    a.wout = last ? nullptr : a0.tmp;
    a.Vout = last ? a0.Vout : nullptr;
    a.part_norm = last ? a0.part_norm : nullptr;
    dispatch_k_gs_sub<TB>(b, a, s);
  }
}

template <typename TB>
void launch_gs_start(const Batch& b, const GsArgs<TB>& a, cudaStream_t s) {
  if (b.nchunks) k_gs_start<TB><<<b.nchunks, kGB, 0, s>>>(b, a);
}
void launch_gs_reduce(const Batch& b, const GsReduceArgs& a, cudaStream_t s) {
  if (b.ncases) k_gs_reduce<<<b.ncases, 256, 0, s>>>(b, a);
}
void launch_gs_close(const Batch& b, const GsCloseArgs& a, cudaStream_t s) {
  if (b.ncases) k_gs_close<<<b.ncases, 32, 0, s>>>(b, a);
}

#define A2D_GS_INST(TB)                                                                 \
  template void launch_gs_dots<TB>(const Batch&, const GsArgs<TB>&, cudaStream_t);     \
  template void launch_gs_project<TB>(const Batch&, const GsArgs<TB>&, cudaStream_t);  \
  template void launch_gs_finish<TB>(const Batch&, const GsArgs<TB>&, cudaStream_t);   \
  template void launch_gs_start<TB>(const Batch&, const GsArgs<TB>&, cudaStream_t);
A2D_GS_INST(double)
A2D_GS_INST(float)
A2D_GS_INST(__nv_bfloat16)
#undef A2D_GS_INST

cudaError_t gs_init() {
  cudaError_t e = cudaSuccess;
  const int bytes = (int)(kGsHeader + kGsSmemBudget);
  auto set = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
#define A2D_GS_ATTR(TB, NQ)                                            \
  set(reinterpret_cast<const void*>(&k_gs_dots<TB, NQ>));              \
  set(reinterpret_cast<const void*>(&k_gs_project<TB, NQ>));           \
  set(reinterpret_cast<const void*>(&k_gs_sub<TB, NQ>));
  A2D_GS_ATTR(float, 8) A2D_GS_ATTR(float, 16) A2D_GS_ATTR(float, 24) A2D_GS_ATTR(float, 32)
  A2D_GS_ATTR(double, 8) A2D_GS_ATTR(double, 16) A2D_GS_ATTR(double, 24) A2D_GS_ATTR(double, 32)
  A2D_GS_ATTR(__nv_bfloat16, 8) A2D_GS_ATTR(__nv_bfloat16, 16) A2D_GS_ATTR(__nv_bfloat16, 24)
  A2D_GS_ATTR(__nv_bfloat16, 32)
#undef A2D_GS_ATTR
  return e;
}

}  // namespace a2d
