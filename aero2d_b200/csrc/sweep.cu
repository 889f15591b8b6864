// One line-Jacobi sweep of the block-tridiagonal line preconditioner
// (aero2d/implicit.py:130-157): right-hand side and a twisted block-Thomas
// solve of every wall-normal line, fused in one kernel.
//
//   e_j = inv_j r_j                                 (first sweep)
//   e_j = e0_j + P_j x'[i-1]_j - Q_j x'[i+1]_j       (later sweeps; x' = previous sweep)
//   from the wall       d_j  = e_j + G_j d_{j-1}      j = 0 .. k-1
//   from the far field  d'_j = e_j + G'_j d'_{j+1}    j = nc-1 .. k+1
//   twist row           x_k  = e_k + G_k d_{k-1} + H_k d'_{k+1}
//   back substitution   x_j = d_j - C_j x_{j+1} (j < k),  x_j = d'_j - C'_j x_{j-1} (j > k)
//
// with the factors of k_factor (inv_j the inverse of row j's pivot, P = inv
// JIL(i), Q = inv JIR(i+1)).  In exact arithmetic this is the reference's
// line solve of each sweep (e_j = inv_j (r_j - off_j), off_j = -JIL(i) x'[i-1]
// + JIR(i+1) x'[i+1]); eliminating from both ends halves the sequential depth
// of a line from 2 nc to about nc dependent steps.
//
// One CTA of 256 threads per 32-line group: warps 0-3 run the wall half,
// warps 4-7 the far-field half, in parallel; in each half lane l = line and
// warp q = row of the 4x4 blocks.  Each half streams its rows' blocks (one
// contiguous run per row: fbidx/fbidx3, a thread's block row is one vector
// load) by TMA bulk copies through its own ring of kStages stages with one
// mbarrier per stage, issued kStages steps ahead by the half's first thread;
// the vector entries of the forward steps come in the same ring by per-thread
// cp.async.  A line's 4-vector passes between the four row warps of a half
// through a two-slot exchange buffer with one named barrier per step; the two
// halves meet twice, around the twist row.  d_j goes to x (the last sweep,
// whose x is FP64: to a scratch vector) and comes back, register-prefetched,
// in the back substitution.
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

constexpr int kHalfThreads = 128;
constexpr int kSweepThreads = 2 * kHalfThreads;
constexpr int kBlockEntries = 16 * kLanes;   // one 4x4 block for the 32 lines of a group
constexpr int kBackAhead = 8;                // register prefetch depth of d in the back substitution

// TI: pivot inverses (the Jacobian type); TF: the other factors (FactorStore);
// TC: arithmetic and intermediate vectors
template <typename TI> struct SweepTypes;
template <> struct SweepTypes<float> {
  using TF = __half;
  using TC = float;
  static constexpr int kStages = 4;   // per half
};
template <> struct SweepTypes<double> {
  using TF = double;
  using TC = double;
  static constexpr int kStages = 2;
};

template <typename TI>
struct SweepSmem {
  using TF = typename SweepTypes<TI>::TF;
  using TC = typename SweepTypes<TI>::TC;
  static constexpr int kS = SweepTypes<TI>::kStages;
  static constexpr uint32_t kBytesI = kBlockEntries * sizeof(TI);
  static constexpr uint32_t kBytesF = kBlockEntries * sizeof(TF);
  // the twist step carries the most: (INV, G, H) or (P, Q, G, H)
  static constexpr uint32_t kMatBytes = (kBytesI + 2 * kBytesF > 4 * kBytesF) ? kBytesI + 2 * kBytesF : 4 * kBytesF;
  // forward: r (FP64) or (e0, x'[i-1], x'[i+1]) in TC, each [line][component]
  static constexpr uint32_t kVecBytes =
      (3 * kLanes * 4 * sizeof(TC) > kLanes * 4 * sizeof(double)) ? 3 * kLanes * 4 * sizeof(TC)
                                                                   : kLanes * 4 * sizeof(double);
  alignas(128) unsigned char mat[2][kS][kMatBytes];
  alignas(16) unsigned char vec[2][kS][kVecBytes];
  alignas(16) TC xchg[2][2][kLanes][4];   // per half: the previous step's 4-vector of every line
  alignas(16) TC xk[kLanes][4];           // the twist row's solution
  uint64_t full[2][kS];
  int abort[2][2];                        // per half: wait failures, by step parity
  int failed[2];                          // per half: stopped early
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

// barrier of the 128 threads of one half (ids 1, 2; id 0 is __syncthreads)
__device__ __forceinline__ void half_sync(int h) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + h), "r"(kHalfThreads) : "memory");
}

template <typename TI, bool FIRST, bool LAST>
__global__ void __launch_bounds__(kSweepThreads) k_sweep(Batch b, SweepArgs a) {
  using SM = SweepSmem<TI>;
  using TF = typename SM::TF;
  using TC = typename SM::TC;
  using TX = typename std::conditional<LAST, double, TC>::type;   // type of x
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SM& sm = *reinterpret_cast<SM*>(smem_raw);
  constexpr int S = SM::kS;
  constexpr uint32_t kBytesI = SM::kBytesI, kBytesF = SM::kBytesF;
  static_assert(S >= 2, "the vector copies are waited for one step ahead");

  const Group grp = b.groups[blockIdx.x];
  if (!case_live(b, grp.cs, a.need)) return;
  const int tid = threadIdx.x;
  const int h = tid / kHalfThreads;           // 0: from the wall, 1: from the far field
  const int ht = tid % kHalfThreads;          // thread within the half
  const int l = ht & 31;                      // line within the group
  const int q = ht >> 5;                      // row of the blocks owned by this warp
  const bool owner = l < grp.n;               // lanes past the group's last line only compute
  const int ll = owner ? l : grp.n - 1;       // and read a valid line
  const CaseDev cs = b.cases[grp.cs];
  const int ni = cs.g.ni, nc = cs.g.nc;
  const int k = nc / 2;                       // twist row (as in k_factor)
  const int nf = h == 0 ? k : nc - 1 - k;     // forward steps of this half
  // step t of a half: t < nf forward; wall half t == k twist; then back substitution
  const int nsteps = h == 0 ? 2 * k + 1 : 2 * nf;
  auto row_of = [&](int t) {
    if (h == 0) return t <= k ? t : 2 * k - t;
    return t < nf ? nc - 1 - t : k + 1 + (t - nf);
  };
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
  const size_t blk0 = lbidx(cs.rows_nc, nc, grp.g, 0, 0, 0);   // row j's block at blk0 + j * kBlockEntries
  const int eo = (q * kLanes + l) * 4;                           // this thread's entries in a block
  uint64_t* full = sm.full[h];

  if (ht == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
    mbar_init_fence();
    sm.abort[h][0] = sm.abort[h][1] = 0;
    sm.failed[h] = 0;
  }
  sm.xchg[h][0][l][q] = TC(0);
  sm.xchg[h][1][l][q] = TC(0);   // d_{-1} = d'_{nc} = 0

  // vector slot k of stage s, [line][component]; the first sweep's r slot is FP64
  auto slot = [&](int s, int kk) { return reinterpret_cast<TC*>(sm.vec[h][s]) + kk * kLanes * 4; };
  auto rslot = [&](int s) { return reinterpret_cast<double*>(sm.vec[h][s]); };

  auto issue = [&](int t) {
    if (t < nsteps) {
      const int s = t % S;
      const int j = row_of(t);
      const bool fwd = t < nf || (h == 0 && t == k);
      if (ht == 0) {
        unsigned char* m = sm.mat[h][s];
        const size_t o = blk0 + (size_t)j * kBlockEntries;
        if (fwd) {
          const bool twist = h == 0 && t == k;
          if constexpr (FIRST) {
            mbar_arrive_expect(&full[s], kBytesI + (twist ? 2 : 1) * kBytesF);
            bulk_load(m, INV + o, kBytesI, &full[s]);
            bulk_load(m + kBytesI, PQG + 3 * o + 2 * kBlockEntries, kBytesF, &full[s]);
            if (twist) bulk_load(m + kBytesI + kBytesF, CF + o, kBytesF, &full[s]);
          } else {
            mbar_arrive_expect(&full[s], (twist ? 4 : 3) * kBytesF);
            bulk_load(m, PQG + 3 * o, 3 * kBytesF, &full[s]);   // P, Q, G: one run
            if (twist) bulk_load(m + 3 * kBytesF, CF + o, kBytesF, &full[s]);
          }
        } else {
          mbar_arrive_expect(&full[s], kBytesF);
          bulk_load(m, CF + o, kBytesF, &full[s]);
        }
      }
      if (fwd) {
        const size_t row = vq + (size_t)j * ni;
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
  // waits for the blocks of step t; a wait that runs out marks the step's parity
  // slot, which every warp of the half reads after the step's barrier
  auto arrive = [&](int t) {
    if (!mbar_wait(&full[t % S], (t / S) & 1)) sm.abort[h][t & 1] = 1;
  };
  // e_j of step t (stage s) from the forward blocks
  auto rhs = [&](int s, int j) -> TC {
    const unsigned char* m = sm.mat[h][s];
    TC e;
    if constexpr (FIRST) {
      TC iv[4], rv[4];
      load4(reinterpret_cast<const TI*>(m) + eo, iv);
      load4(rslot(s) + l * 4, rv);
      e = iv[0] * rv[0];
#pragma unroll
      for (int c = 1; c < 4; ++c) e += iv[c] * rv[c];
      if (a.e0 != nullptr && owner) reinterpret_cast<TC*>(a.e0)[vq + (size_t)j * ni + i] = e;
    } else {
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
    return e;
  };
  constexpr uint32_t kOffG = FIRST ? kBytesI : 2 * kBytesF;   // G's block in a forward stage
  constexpr uint32_t kOffH = kOffG + kBytesF;                // H's block in the twist stage

  __syncthreads();    // barriers initialised, exchange slots cleared
#pragma unroll 1
  for (int t = 0; t < S; ++t) issue(t);
  async_wait<S - 1>();
  half_sync(h);       // vector entries of step 0 visible to every warp of the half

  int tstop = -1;     // step at which a wait ran out
  // ---- forward eliminations of both halves ----
#pragma unroll 1
  for (int t = 0; t < nf; ++t) {
    const int s = t % S;
    const int j = row_of(t);
    arrive(t);
    const TC e = rhs(s, j);
    TC gv[4], dp[4];
    load4(reinterpret_cast<const TF*>(sm.mat[h][s] + kOffG) + eo, gv);
    load4(&sm.xchg[h][(t + 1) & 1][l][0], dp);
    TC d = e;
#pragma unroll
    for (int c = 0; c < 4; ++c) d += gv[c] * dp[c];
    sm.xchg[h][t & 1][l][q] = d;
    if (owner) dv[(size_t)j * ni + i] = d;
    async_wait<S - 2>();
    half_sync(h);
    if (sm.abort[h][t & 1]) {
      tstop = t;
      break;
    }
    issue(t + S);
  }
  if (tstop >= 0 && ht == 0) sm.failed[h] = 1;
  __syncthreads();    // (A) both forward eliminations done
  const bool stop = sm.failed[0] || sm.failed[1];
  // ---- twist row k (wall half) ----
  if (!stop && h == 0) {
    const int t = k;
    const int s = t % S;
    arrive(t);
    const TC e = rhs(s, k);
    TC gv[4], hv[4], dm[4], dpl[4];
    load4(reinterpret_cast<const TF*>(sm.mat[h][s] + kOffG) + eo, gv);
    load4(reinterpret_cast<const TF*>(sm.mat[h][s] + kOffH) + eo, hv);
    load4(&sm.xchg[0][(k + 1) & 1][l][0], dm);                               // d_{k-1}
    if (nc - 1 - k > 0) load4(&sm.xchg[1][(nc - 1 - k + 1) & 1][l][0], dpl); // d'_{k+1}
    else dpl[0] = dpl[1] = dpl[2] = dpl[3] = TC(0);
    TC xv = e;
#pragma unroll
    for (int c = 0; c < 4; ++c) xv += gv[c] * dm[c];
#pragma unroll
    for (int c = 0; c < 4; ++c) xv += hv[c] * dpl[c];
    sm.xk[l][q] = xv;
    if (owner) x[(size_t)k * ni + i] = TX(xv);
    half_sync(h);
    if (sm.abort[h][t & 1]) sm.failed[h] = 1;
    else issue(t + S);
  }
  __syncthreads();    // (B) x_k visible to both halves
  // ---- back substitutions of both halves, outward from the twist row ----
  const int t0 = h == 0 ? k + 1 : nf;
  if (!(sm.failed[0] || sm.failed[1])) {
    TC dbuf[kBackAhead];
#pragma unroll
    for (int u = 0; u < kBackAhead; ++u) {
      const int t = t0 + u;
      dbuf[u] = t < nsteps ? dv[(size_t)row_of(t) * ni + i] : TC(0);
    }
#pragma unroll 1
    for (int b0 = t0; b0 < nsteps && tstop < 0; b0 += kBackAhead) {
#pragma unroll
      for (int u = 0; u < kBackAhead; ++u) {
        const int t = b0 + u;
        if (t < nsteps && tstop < 0) {
          const int j = row_of(t);
          const int s = t % S;
          arrive(t);
          TC cv[4], xn[4];
          load4(reinterpret_cast<const TF*>(sm.mat[h][s]) + eo, cv);
          load4(t == t0 ? &sm.xk[l][0] : &sm.xchg[h][(t + 1) & 1][l][0], xn);
          TC acc = cv[0] * xn[0];
#pragma unroll
          for (int c = 1; c < 4; ++c) acc += cv[c] * xn[c];
          const TC xv = dbuf[u] - acc;
          sm.xchg[h][t & 1][l][q] = xv;
          if (owner) x[(size_t)j * ni + i] = TX(xv);
          const int tn = t + kBackAhead;
          if (tn < nsteps) dbuf[u] = dv[(size_t)row_of(tn) * ni + i];
          half_sync(h);
          if (sm.abort[h][t & 1]) tstop = t;
          else issue(t + S);
        }
      }
    }
  } else if (tstop < 0) {
    // a half stopped: the copies this half issued beyond its last consumed
    // step (the twist row for the wall half) are still to be drained
    tstop = h == 0 ? k : nf;
  }
  if (tstop >= 0) {
    // a copy never completed: record it, and give the copies still in flight
    // (issued for steps tstop .. tstop+S-1) a bounded time to land before exit
    if (ht == 0) {
      if (a.err != nullptr) atomicExch(a.err, 1u);
#pragma unroll 1
      for (int u = tstop; u < tstop + S && u < nsteps; ++u) (void)mbar_wait(&full[u % S], (u / S) & 1);
    }
    async_wait<0>();
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
