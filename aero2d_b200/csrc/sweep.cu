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
// 4x4 blocks, so a warp reads one block entry of its 32 lines as 32
// consecutive words of shared memory.  The blocks of every step (lane-blocked,
// one contiguous run per block: 1 KB for the FP16 factors of the mixed path,
// 2 KB for its FP32 pivot inverses, 4 KB in FP64) are streamed by the
// TMA engine through a ring of kStages stages, one mbarrier per stage, issued
// kStages steps ahead by thread 0; the vector entries of the forward steps
// come in the same ring by per-thread 8-byte cp.async.  The previous step's
// 4-vector passes between the four row warps through a two-slot exchange
// buffer, with one CTA barrier per step.  d_j goes to x in HBM (mostly L2) and
// comes back, register-prefetched, in the backward recurrence.
#include "batch.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace a2d {

constexpr int kSweepThreads = 128;
constexpr int kBlockEntries = 16 * kLanes;   // one 4x4 block for the 32 lines of a group
constexpr int kBackAhead = 8;                // register prefetch depth of d in the backward pass

// stages of the ring per Jacobian type (FP32: FP16 factors, 6 KB a stage)
template <typename TI> struct SweepStages;
template <> struct SweepStages<float> { static constexpr int value = 8; };
template <> struct SweepStages<double> { static constexpr int value = 3; };

// TI: pivot inverses (the Jacobian type); TF: the other factors (FactorStore)
template <typename TI>
struct SweepSmem {
  using TF = typename FactorStore<TI>::type;
  static constexpr int kS = SweepStages<TI>::value;
  static constexpr uint32_t kBytesI = kBlockEntries * sizeof(TI);
  static constexpr uint32_t kBytesF = kBlockEntries * sizeof(TF);
  static constexpr uint32_t kMatBytes = (kBytesI + kBytesF > 3 * kBytesF) ? kBytesI + kBytesF : 3 * kBytesF;
  // forward: (INV, G) or (P, Q, G); backward: C
  alignas(128) unsigned char mat[kS][kMatBytes];
  double vec[kS][3][4][kLanes];          // forward: r or (e0, x'[i-1], x'[i+1]), [component][line]
  double xchg[2][4][kLanes];             // previous step's 4-vector of every line
  uint64_t full[kS];
  int abort[2];                          // wait failures, by step parity
};

template <typename TI, bool FIRST>
__global__ void __launch_bounds__(kSweepThreads) k_sweep(Batch b, SweepArgs a) {
  using SM = SweepSmem<TI>;
  using TF = typename SM::TF;
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
  const size_t vb = 4 * (size_t)cs.cell_off;
  const size_t row_q = (size_t)q * nc * ni;   // component q of the case's vectors
  const TI* INV = static_cast<const TI*>(a.INV);
  const TF* Pm = static_cast<const TF*>(a.P);
  const TF* Qm = static_cast<const TF*>(a.Q);
  const TF* Gm = static_cast<const TF*>(a.G);
  const TF* CF = static_cast<const TF*>(a.CF);
  const size_t blk0 = lbidx(cs.rows_nc, nc, grp.g, 0, 0, 0);   // step j block at blk0 + j * kBlockEntries
  const int nsteps = 2 * nc;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(&sm.full[s], 1);
    mbar_init_fence();
    sm.abort[0] = sm.abort[1] = 0;
  }
  sm.xchg[1][q][l] = 0.0;   // d_{-1} = 0

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
            bulk_load(m + kBytesI, Gm + o, kBytesF, &sm.full[s]);
          } else {
            mbar_arrive_expect(&sm.full[s], 3 * kBytesF);
            bulk_load(m, Pm + o, kBytesF, &sm.full[s]);
            bulk_load(m + kBytesF, Qm + o, kBytesF, &sm.full[s]);
            bulk_load(m + 2 * kBytesF, Gm + o, kBytesF, &sm.full[s]);
          }
        } else {
          const size_t o = blk0 + (size_t)(nsteps - 1 - t) * kBlockEntries;
          mbar_arrive_expect(&sm.full[s], kBytesF);
          bulk_load(m, CF + o, kBytesF, &sm.full[s]);
        }
      }
      if (t < nc) {
        const size_t row = vb + row_q + (size_t)t * ni;
        if (FIRST) {
          async_copy8(&sm.vec[s][0][q][l], a.r + row + i);
        } else {
          async_copy8(&sm.vec[s][0][q][l], a.e0 + row + i);
          async_copy8(&sm.vec[s][1][q][l], a.xprev + row + im);
          async_copy8(&sm.vec[s][2][q][l], a.xprev + row + ip);
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

  double* x = a.x + vb + row_q;
  int tstop = -1;     // step at which a wait ran out
  // ---- forward: d_j = e_j + G_j d_{j-1} ----
#pragma unroll 1
  for (int t = 0; t < nc; ++t) {
    const int s = t % S;
    arrive(t);
    const unsigned char* m = sm.mat[s];
    double e;
    const TF* Gs;
    if constexpr (FIRST) {
      const TI* M0 = reinterpret_cast<const TI*>(m);
      Gs = reinterpret_cast<const TF*>(m + kBytesI);
      double r[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) r[c] = sm.vec[s][0][c][l];
      e = to_f64(M0[(q * 4) * kLanes + l]) * r[0];
#pragma unroll
      for (int c = 1; c < 4; ++c) e += to_f64(M0[(q * 4 + c) * kLanes + l]) * r[c];
      if (a.e0 != nullptr && owner) a.e0[vb + row_q + (size_t)t * ni + i] = e;
    } else {
      const TF* M0 = reinterpret_cast<const TF*>(m);
      const TF* M1 = reinterpret_cast<const TF*>(m + kBytesF);
      Gs = reinterpret_cast<const TF*>(m + 2 * kBytesF);
      double s1 = to_f64(M0[(q * 4) * kLanes + l]) * sm.vec[s][1][0][l];
      double s2 = to_f64(M1[(q * 4) * kLanes + l]) * sm.vec[s][2][0][l];
#pragma unroll
      for (int c = 1; c < 4; ++c) {
        s1 += to_f64(M0[(q * 4 + c) * kLanes + l]) * sm.vec[s][1][c][l];
        s2 += to_f64(M1[(q * 4 + c) * kLanes + l]) * sm.vec[s][2][c][l];
      }
      e = sm.vec[s][0][q][l] + s1 - s2;
    }
    const double* dp = &sm.xchg[(t + 1) & 1][0][0];
    double d = e;
#pragma unroll
    for (int c = 0; c < 4; ++c) d += to_f64(Gs[(q * 4 + c) * kLanes + l]) * dp[c * kLanes + l];
    sm.xchg[t & 1][q][l] = d;
    if (owner) x[(size_t)t * ni + i] = d;
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
    double dbuf[kBackAhead];
#pragma unroll
    for (int u = 0; u < kBackAhead; ++u) {
      const int j = nc - 1 - u;
      dbuf[u] = (j >= 0) ? x[(size_t)j * ni + i] : 0.0;
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
          const TF* C = reinterpret_cast<const TF*>(sm.mat[s]);
          const double* xp = &sm.xchg[(t + 1) & 1][0][0];
          double acc = 0.0;
          if (bk > 0) {
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += to_f64(C[(q * 4 + c) * kLanes + l]) * xp[c * kLanes + l];
          }
          const double xn = dbuf[u] - acc;
          sm.xchg[t & 1][q][l] = xn;
          if (owner) x[(size_t)j * ni + i] = xn;
          const int jn = j - kBackAhead;
          if (jn >= 0) dbuf[u] = x[(size_t)jn * ni + i];
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
void launch_sweep(const Batch& b, const SweepArgs& a, cudaStream_t s) {
  if (b.ngroups == 0) return;
  k_sweep<TI, FIRST><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
}

cudaError_t sweep_init() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f, size_t bytes) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  };
  set(reinterpret_cast<const void*>(&k_sweep<float, true>), sizeof(SweepSmem<float>));
  set(reinterpret_cast<const void*>(&k_sweep<float, false>), sizeof(SweepSmem<float>));
  set(reinterpret_cast<const void*>(&k_sweep<double, true>), sizeof(SweepSmem<double>));
  set(reinterpret_cast<const void*>(&k_sweep<double, false>), sizeof(SweepSmem<double>));
  return e;
}

template void launch_sweep<float, true>(const Batch&, const SweepArgs&, cudaStream_t);
template void launch_sweep<float, false>(const Batch&, const SweepArgs&, cudaStream_t);
template void launch_sweep<double, true>(const Batch&, const SweepArgs&, cudaStream_t);
template void launch_sweep<double, false>(const Batch&, const SweepArgs&, cudaStream_t);

}  // namespace a2d
