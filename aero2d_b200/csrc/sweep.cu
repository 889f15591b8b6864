// One line-Jacobi sweep of the block-tridiagonal line preconditioner
// (aero2d/implicit.py:130-157), right-hand side and both block-Thomas
// recurrences fused in one kernel:
//
//   e_j = inv_j r_j                                   (first sweep)
//   e_j = e0_j + P_j x'[i-1]_j - Q_j x'[i+1]_j         (later sweeps; x' = previous sweep)
//   d_j = e_j + G_j d_{j-1}                           j = 0 .. nc-1
//   x_j = d_j - C_j x_{j+1}                           j = nc-1 .. 0
//
// with P = inv JIL(i), Q = inv JIR(i+1), G = inv JJL and C the upper factors of
// k_factor.  In exact arithmetic e_j = inv_j (r_j - off_j), off_j = -JIL(i)
// x'[i-1] + JIR(i+1) x'[i+1], the reference's sweep.
//
// One CTA of 128 threads per 32-line group: lane l = line, warp q = row of the
// 4x4 blocks.  The blocks of every step are one contiguous run per factor
// (fbidx: [row q][line][column c], so a thread's four entries are one vector
// load and a warp reads 256 B in one go), streamed by the TMA engine through a
// ring of kStages stages, one mbarrier per stage, issued kStages steps ahead by
// thread 0; the vector entries of the forward steps come in the same ring by
// per-thread cp.async, stored [line][component] so that a thread reads the
// 4-vector of its line with one load.  The previous step's 4-vector passes
// between the four row warps through a two-slot exchange buffer, with one CTA
// barrier per step.  d_j goes to x (the last sweep, whose x is FP64: to a
// scratch vector) and comes back, register-prefetched, in the backward
// recurrence.  The factors P, Q, G of a step are interleaved (fbidx3), one copy.
//
// Arithmetic and intermediate vectors are in the sweep's compute type: FP64
// in the FP64 path; FP32 in the mixed path, whose factors are FP16 and pivot
// inverses FP32 (a preconditioner only steers GMRES; the Newton residual and
// the Krylov reductions stay FP64).
#include <type_traits>

#include "batch.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace a2d {

constexpr int kSweepThreads = 128;
constexpr int kBlockEntries = 16 * kLanes;   // one 4x4 block for the 32 lines of a group
constexpr int kBackAhead = 8;                // register prefetch depth of d in the backward pass

// TI: pivot inverses (the Jacobian type); TF: the other factors (FactorStore);
// TC: arithmetic and intermediate vectors
template <typename TI> struct SweepTypes;
template <> struct SweepTypes<float> {
  using TF = __half;
  using TC = float;
  static constexpr int kStages = 8;
};
template <> struct SweepTypes<double> {
  using TF = double;
  using TC = double;
  static constexpr int kStages = 3;
};

template <typename TI>
struct SweepSmem {
  using TF = typename SweepTypes<TI>::TF;
  using TC = typename SweepTypes<TI>::TC;
  static constexpr int kS = SweepTypes<TI>::kStages;
  static constexpr uint32_t kBytesI = kBlockEntries * sizeof(TI);
  static constexpr uint32_t kBytesF = kBlockEntries * sizeof(TF);
  static constexpr uint32_t kMatBytes = (kBytesI + kBytesF > 3 * kBytesF) ? kBytesI + kBytesF : 3 * kBytesF;
  // forward: r (FP64) or (e0, x'[i-1], x'[i+1]) in TC, each [line][component]
  static constexpr uint32_t kVecBytes =
      (3 * kLanes * 4 * sizeof(TC) > kLanes * 4 * sizeof(double)) ? 3 * kLanes * 4 * sizeof(TC)
                                                                   : kLanes * 4 * sizeof(double);
  alignas(128) unsigned char mat[kS][kMatBytes];   // forward: (INV, G) or (P, Q, G); backward: C
  alignas(16) unsigned char vec[kS][kVecBytes];
  alignas(16) TC xchg[2][kLanes][4];               // previous step's 4-vector of every line
  uint64_t full[kS];
  int abort[2];                                    // wait failures, by step parity
};

// the four entries of one block row of one line, converted to the compute type
__device__ __forceinline__ void load4(const __half* p, float (&v)[4]) {
  const uint2 raw = *reinterpret_cast<const uint2*>(p);
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void load4(const float* p, float (&v)[4]) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void load4(const double* p, float (&v)[4]) {
  const double2 t0 = *reinterpret_cast<const double2*>(p);
  const double2 t1 = *reinterpret_cast<const double2*>(p + 2);
  v[0] = (float)t0.x; v[1] = (float)t0.y; v[2] = (float)t1.x; v[3] = (float)t1.y;
}
__device__ __forceinline__ void load4(const double* p, double (&v)[4]) {
  const double2 t0 = *reinterpret_cast<const double2*>(p);
  const double2 t1 = *reinterpret_cast<const double2*>(p + 2);
  v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
}

// asynchronous copy of one vector entry
__device__ __forceinline__ void async_copy_entry(float* dst, const float* src) { async_copy4(dst, src); }
__device__ __forceinline__ void async_copy_entry(double* dst, const double* src) { async_copy8(dst, src); }

template <typename TI, bool FIRST, bool LAST>
__global__ void __launch_bounds__(kSweepThreads) k_sweep(Batch b, SweepArgs a) {
  using SM = SweepSmem<TI>;
  using TF = typename SM::TF;
  using TC = typename SM::TC;
  using TX = typename std::conditional<LAST, double, TC>::type;   // type of x (and of d kept in it)
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SM& sm = *reinterpret_cast<SM*>(smem_raw);
  constexpr int S = SM::kS;
  constexpr uint32_t kBytesI = SM::kBytesI, kBytesF = SM::kBytesF;
  static_assert(S >= 2, "the vector copies are waited for one step ahead");

  const Group grp = b.groups[blockIdx.x];
  if (!case_live(b, grp.cs, a.need)) return;
  const int tid = threadIdx.x;
  const int l = tid & 31;                     // line within the group
  const int q = tid >> 5;                     // row of the blocks owned by this warp
  const bool owner = l < grp.n;               // lanes past the group's last line only compute
  const int ll = owner ? l : grp.n - 1;       // and read a valid line
  const CaseDev cs = b.cases[grp.cs];
  const int ni = cs.g.ni, nc = cs.g.nc;
  const int i = grp.i0 + ll;
  const int im = (i == 0) ? ni - 1 : i - 1;
  const int ip = (i + 1 == ni) ? 0 : i + 1;
  const size_t vq = 4 * (size_t)cs.cell_off + (size_t)q * nc * ni;   // component q of the case's vectors
  const TI* INV = static_cast<const TI*>(a.INV);
  const TF* PQG = static_cast<const TF*>(a.PQG);
  const TF* CF = static_cast<const TF*>(a.CF);
  const TC* e0v = reinterpret_cast<const TC*>(a.e0);
  const TC* xpv = reinterpret_cast<const TC*>(a.xprev);
  TX* x = reinterpret_cast<TX*>(a.x) + vq;
  // d_j in the compute type: in x itself, or (last sweep, FP64 x) in the scratch
  TC* dv = reinterpret_cast<TC*>(LAST ? a.dtmp : a.x) + vq;
  const size_t blk0 = lbidx(cs.rows_nc, nc, grp.g, 0, 0, 0);   // step j block at blk0 + j * kBlockEntries
  const int eo = (q * kLanes + l) * 4;                           // this thread's entries in a block
  const int nsteps = 2 * nc;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(&sm.full[s], 1);
    mbar_init_fence();
    sm.abort[0] = sm.abort[1] = 0;
  }
  sm.xchg[1][l][q] = TC(0);   // d_{-1} = 0

  // vector slot k of stage s, [line][component]; the first sweep's r slot is FP64
  auto slot = [&](int s, int k) { return reinterpret_cast<TC*>(sm.vec[s]) + k * kLanes * 4; };
  auto rslot = [&](int s) { return reinterpret_cast<double*>(sm.vec[s]); };

  // step t < nc: forward row j = t; t >= nc: backward row j = 2 nc - 1 - t
  auto issue = [&](int t) {
    if (t < nsteps) {
      const int s = t % S;
      if (tid == 0) {
        unsigned char* m = sm.mat[s];
        if (t < nc) {
          const size_t o = blk0 + (size_t)t * kBlockEntries;
          if constexpr (FIRST) {
            mbar_arrive_expect(&sm.full[s], kBytesI + kBytesF);
            bulk_load(m, INV + o, kBytesI, &sm.full[s]);
            bulk_load(m + kBytesI, PQG + 3 * o + 2 * kBlockEntries, kBytesF, &sm.full[s]);
          } else {
            // P, Q, G of the step: one contiguous 3-block run
            mbar_arrive_expect(&sm.full[s], 3 * kBytesF);
            bulk_load(m, PQG + 3 * o, 3 * kBytesF, &sm.full[s]);
          }
        } else {
          const size_t o = blk0 + (size_t)(nsteps - 1 - t) * kBlockEntries;
          mbar_arrive_expect(&sm.full[s], kBytesF);
          bulk_load(m, CF + o, kBytesF, &sm.full[s]);
        }
      }
      if (t < nc) {
        const size_t row = vq + (size_t)t * ni;
        if constexpr (FIRST) {
          async_copy8(rslot(s) + l * 4 + q, a.r + row + i);
        } else {
          async_copy_entry(slot(s, 0) + l * 4 + q, e0v + row + i);
          async_copy_entry(slot(s, 1) + l * 4 + q, xpv + row + im);
          async_copy_entry(slot(s, 2) + l * 4 + q, xpv + row + ip);
        }
      }
    }
    async_commit();   // one group per step, empty ones included, keeps the group count regular
  };
  // waits for the blocks of step t; a wait that runs out marks the step's
  // parity slot, which every warp reads after the step's CTA barrier
  auto arrive = [&](int t) {
    if (!mbar_wait(&sm.full[t % S], (t / S) & 1)) sm.abort[t & 1] = 1;
  };

  __syncthreads();    // barriers initialised, exchange slot cleared
#pragma unroll 1
  for (int t = 0; t < S; ++t) issue(t);
  async_wait<S - 1>();
  __syncthreads();    // vector entries of step 0 visible to every warp

  int tstop = -1;     // step at which a wait ran out
  // ---- forward: d_j = e_j + G_j d_{j-1} ----
#pragma unroll 1
  for (int t = 0; t < nc; ++t) {
    const int s = t % S;
    arrive(t);
    const unsigned char* m = sm.mat[s];
    TC e;
    const TF* Gs;
    if constexpr (FIRST) {
      Gs = reinterpret_cast<const TF*>(m + kBytesI);
      TC iv[4], rv[4];
      load4(reinterpret_cast<const TI*>(m) + eo, iv);
      load4(rslot(s) + l * 4, rv);
      e = iv[0] * rv[0];
#pragma unroll
      for (int c = 1; c < 4; ++c) e += iv[c] * rv[c];
      if (a.e0 != nullptr && owner) reinterpret_cast<TC*>(a.e0)[vq + (size_t)t * ni + i] = e;
    } else {
      Gs = reinterpret_cast<const TF*>(m + 2 * kBytesF);
      TC pv[4], qv[4], xm[4], xp[4];
      load4(reinterpret_cast<const TF*>(m) + eo, pv);
      load4(reinterpret_cast<const TF*>(m + kBytesF) + eo, qv);
      load4(slot(s, 1) + l * 4, xm);
      load4(slot(s, 2) + l * 4, xp);
      TC s1 = pv[0] * xm[0];
      TC s2 = qv[0] * xp[0];
#pragma unroll
      for (int c = 1; c < 4; ++c) {
        s1 += pv[c] * xm[c];
        s2 += qv[c] * xp[c];
      }
      e = slot(s, 0)[l * 4 + q] + s1 - s2;
    }
    TC gv[4], dp[4];
    load4(Gs + eo, gv);
    load4(&sm.xchg[(t + 1) & 1][l][0], dp);
    TC d = e;
#pragma unroll
    for (int c = 0; c < 4; ++c) d += gv[c] * dp[c];
    sm.xchg[t & 1][l][q] = d;
    if (owner) dv[(size_t)t * ni + i] = d;
    async_wait<S - 2>();
    __syncthreads();
    if (sm.abort[t & 1]) {
      tstop = t;
      break;
    }
    issue(t + S);
  }
  // ---- backward: x_j = d_j - C_j x_{j+1} ----
  if (tstop < 0) {
    TC dbuf[kBackAhead];
#pragma unroll
    for (int u = 0; u < kBackAhead; ++u) {
      const int j = nc - 1 - u;
      dbuf[u] = (j >= 0) ? dv[(size_t)j * ni + i] : TC(0);
    }
#pragma unroll 1
    for (int b0 = 0; b0 < nc && tstop < 0; b0 += kBackAhead) {
#pragma unroll
      for (int u = 0; u < kBackAhead; ++u) {
        const int bk = b0 + u;
        if (bk < nc && tstop < 0) {
          const int t = nc + bk;
          const int j = nc - 1 - bk;
          const int s = t % S;
          arrive(t);
          TC acc = TC(0);
          if (bk > 0) {
            TC cv[4], xn[4];
            load4(reinterpret_cast<const TF*>(sm.mat[s]) + eo, cv);
            load4(&sm.xchg[(t + 1) & 1][l][0], xn);
            acc = cv[0] * xn[0];
#pragma unroll
            for (int c = 1; c < 4; ++c) acc += cv[c] * xn[c];
          }
          const TC xv = dbuf[u] - acc;
          sm.xchg[t & 1][l][q] = xv;
          if (owner) x[(size_t)j * ni + i] = TX(xv);
          const int jn = j - kBackAhead;
          if (jn >= 0) dbuf[u] = dv[(size_t)jn * ni + i];
          __syncthreads();
          if (sm.abort[t & 1]) tstop = t;
          else issue(t + S);
        }
      }
    }
  }
  if (tstop >= 0) {
    // a copy never completed: record it, and give the copies still in flight
    // (issued for steps tstop .. tstop+S-1) a bounded time to land before exit
    if (tid == 0) {
      if (a.err != nullptr) atomicExch(a.err, 1u);
#pragma unroll 1
      for (int u = tstop; u < tstop + S && u < nsteps; ++u) (void)mbar_wait(&sm.full[u % S], (u / S) & 1);
    }
    async_wait<0>();
    __syncthreads();
  }
}

template <typename TI, bool FIRST>
void launch_sweep(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s) {
  if (b.ngroups == 0) return;
  if (last) k_sweep<TI, FIRST, true><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
  else k_sweep<TI, FIRST, false><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
}

cudaError_t sweep_init() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f, size_t bytes) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  };
#define A2D_SWEEP_ATTR(TI, F, L) set(reinterpret_cast<const void*>(&k_sweep<TI, F, L>), sizeof(SweepSmem<TI>));
  A2D_SWEEP_ATTR(float, true, true) A2D_SWEEP_ATTR(float, true, false)
  A2D_SWEEP_ATTR(float, false, true) A2D_SWEEP_ATTR(float, false, false)
  A2D_SWEEP_ATTR(double, true, true) A2D_SWEEP_ATTR(double, true, false)
  A2D_SWEEP_ATTR(double, false, true) A2D_SWEEP_ATTR(double, false, false)
#undef A2D_SWEEP_ATTR
  return e;
}

template void launch_sweep<float, true>(const Batch&, const SweepArgs&, bool, cudaStream_t);
template void launch_sweep<float, false>(const Batch&, const SweepArgs&, bool, cudaStream_t);
template void launch_sweep<double, true>(const Batch&, const SweepArgs&, bool, cudaStream_t);
template void launch_sweep<double, false>(const Batch&, const SweepArgs&, bool, cudaStream_t);

}  // namespace a2d
