// The cluster-pair variant of the row-warp line sweep (sweep_rows.cu has the row
// arithmetic this file repeats line for line; sweep.cu the mathematics): a
// cluster of two CTAs of five warps per 32-line group, CTA rank 0 running the
// wall half of the lines' twisted solve and rank 1 the far-field half, so a
// 64-case batch is 1024 CTAs, seven resident per SM, where the rows variant's
// 512 CTAs of nine warps sit four on some SMs and three on others and the launch
// lasts as long as the SMs holding four.  In each CTA warps 0-3 are the block rows
// q (lane = line) and warp 4 the producer streaming the half's factor blocks by
// bulk copies into a ring of full/empty mbarriers, as in the rows variant, except
// that the back substitution takes four steps per ring stage: its steps read one C
// block each (1 KB of a 4 KB stage), and the rows of four consecutive steps are
// consecutive, so one bulk copy brings a pack and the ring holds 16 back steps.  The
// halves meet twice, through distributed shared memory: the far-field CTA stores
// its last forward vector d'_{k+1} into the wall CTA's shared memory and arrives
// on an mbarrier there; the wall CTA solves the twist row and stores x_k into the
// far-field CTA the same way.  Every line's arithmetic is the rows variant's, in
// the same order, so the results are bitwise the same.  Mixed-precision plans
// only.  Every mbarrier wait is bounded; the CTAs of a cluster leave together
// (one cluster barrier that every thread still running reaches once), so neither
// exits while the other may write into its shared memory.  No cluster multicast.
#include <type_traits>

#include "batch.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace a2d {
namespace halves {

using TI = float;     // pivot inverses
using TF = __half;    // the other factors
using TC = float;     // arithmetic and intermediate vectors

constexpr int kConsumerThreads = 128;
constexpr int kProducerWarp = kConsumerThreads / 32;    // warp 4
constexpr int kSweepThreads = kConsumerThreads + 32;
constexpr int kBlockEntries = 16 * kLanes;              // one 4x4 block for the 32 lines of a group
constexpr int kBackAhead = 8;                           // register prefetch depth of d in the back substitution
constexpr int kStages = 4;                              // bulk-copy ring stages
constexpr int kAhead = 4;                               // steps between loading a vector entry and its use
constexpr int kPack = 4;                                // back-substitution steps per ring stage (their rows are contiguous)
static_assert(kBackAhead % kPack == 0, "a back prefetch block holds whole packs");

struct SweepSmem {
  static constexpr uint32_t kBytesI = kBlockEntries * sizeof(TI);
  static constexpr uint32_t kBytesF = kBlockEntries * sizeof(TF);
  // the twist step carries the most: (INV, G, H) or (P, Q, G, H)
  static constexpr uint32_t kMatBytes = (kBytesI + 2 * kBytesF > 4 * kBytesF) ? kBytesI + 2 * kBytesF : 4 * kBytesF;
  // forward: r (FP64) or (e0, x'[i-1], x'[i+1]) in TC, each [line][component]
  static constexpr uint32_t kVecBytes =
      (3 * kLanes * 4 * sizeof(TC) > kLanes * 4 * sizeof(double)) ? 3 * kLanes * 4 * sizeof(TC)
                                                                  : kLanes * 4 * sizeof(double);
  alignas(128) unsigned char mat[kStages][kMatBytes];
  alignas(16) unsigned char vec[2][kVecBytes];   // by step parity
  alignas(16) TC xchg[2][kLanes][4];             // the previous step's 4-vector of every line
  alignas(16) TC xk[kLanes][4];                  // the twist row's solution (rank 1: from rank 0)
  alignas(16) TC dfar[kLanes][4];                // rank 0: d'_{k+1} of the far-field half (from rank 1)
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t xbar;                                 // one arrival from the other CTA of the cluster
  int failed;
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

// barrier of the 128 consumer threads (id 1; the producer warp takes part in none),
// OR-reducing a per-thread flag
__device__ __forceinline__ bool consumers_sync_or(bool flag) {
  uint32_t r;
  asm volatile(
      "{\n"
      " .reg .pred pi, po;\n"
      " setp.ne.u32 pi, %1, 0;\n"
      " bar.red.or.pred po, 1, %2, pi;\n"
      " selp.u32 %0, 1, 0, po;\n"
      "}\n"
      : "=r"(r)
      : "r"((uint32_t)flag), "r"(kConsumerThreads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void consumers_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(kConsumerThreads) : "memory");
}

// ---- the cluster of two ----
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// every thread of the cluster that has not exited (whole warps)
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// the address of `p` (this CTA's shared memory) in the shared memory of CTA `rank`
__device__ __forceinline__ uint32_t peer_addr(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ void peer_store(uint32_t addr, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}
__device__ __forceinline__ void fence_cluster() {
  asm volatile("fence.acq_rel.cluster;" ::: "memory");
}
// one arrival on an mbarrier in the other CTA's shared memory, releasing this
// thread's (and, through the preceding barrier and fences, its CTA's) stores
__device__ __forceinline__ void peer_arrive(uint32_t bar_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_addr) : "memory");
}
// the local wait for that arrival, bounded like every other wait
__device__ __forceinline__ bool xbar_wait(uint64_t* bar) {
  auto try_once = [&]() {
    uint32_t ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar))
        : "memory");
    return ok != 0;
  };
  if (try_once()) return true;
  const unsigned long long t0 = global_ns();
  while (!try_once()) {
    if (global_ns() - t0 > kWaitLimitNs) return false;
  }
  return true;
}

template <bool FIRST, bool LAST>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kSweepThreads, 7) k_sweep(Batch b, SweepArgs a) {
  using SM = SweepSmem;
  using TX = typename std::conditional<LAST, double, TC>::type;   // type of x
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SM& sm = *reinterpret_cast<SM*>(smem_raw);
  constexpr int S = kStages;
  constexpr uint32_t kBytesI = SM::kBytesI, kBytesF = SM::kBytesF;
  constexpr uint32_t kOffG = FIRST ? kBytesI : 2 * kBytesF;   // G's block in a forward stage
  constexpr uint32_t kOffH = kOffG + kBytesF;                // H's block in the twist stage

  const Group grp = b.groups[blockIdx.x >> 1];
  // both CTAs of the cluster see the same case: both leave here, or neither
  if (!case_live(b, grp.cs, a.need)) return;
  const int h = (int)cluster_rank();           // 0: from the wall, 1: from the far field
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const CaseDev cs = b.cases[grp.cs];
  const int ni = cs.g.ni, nc = cs.g.nc;
  const int k = nc / 2;                        // twist row (as in k_factor)
  const int nf0 = k, nf1 = nc - 1 - k;         // forward steps of the wall / far-field half
  const int nf = h == 0 ? nf0 : nf1;
  const int nsteps = h == 0 ? 2 * k + 1 : 2 * nf1;   // this half's steps
  const int tb0 = h == 0 ? k + 1 : nf1;              // this half's first back-substitution step
  const int nslots = tb0 + (nsteps - tb0 + kPack - 1) / kPack;   // ring slots: one per forward step, one per pack
  // step t of the half: forward rows first; the wall half's step k is the twist
  // row; then the back substitution outward from the twist row
  auto row_of = [&](int t) {
    if (h == 0) return t <= k ? t : 2 * k - t;
    return t < nf1 ? nc - 1 - t : k + 1 + (t - nf1);
  };
  const size_t vbase = 4 * (size_t)cs.cell_off;
  const size_t comp = (size_t)nc * ni;         // stride between the components of a case vector
  const size_t blk0 = lbidx(cs.rows_nc, nc, grp.g, 0, 0, 0);   // row j's block at blk0 + j * kBlockEntries

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) {
      mbar_init(&sm.full[s], 1);        // the producer's arrival with the bulk-copy bytes
      mbar_init(&sm.empty[s], 4);       // one arrival per consumer warp
    }
    mbar_init(&sm.xbar, 1);
    sm.failed = 0;
    mbar_init_fence();
  }
  if (warp < kProducerWarp) {
    sm.xchg[0][lane][warp] = TC(0);
    sm.xchg[1][lane][warp] = TC(0);   // d_{-1} = d'_{nc} = 0
  }
  __syncthreads();
  cluster_sync();   // the other CTA's mbarriers are initialised before any arrival on them

  // ======================= producer warp (as in the rows variant, one half) =======================
  if (warp == kProducerWarp) {
    const TI* INV = static_cast<const TI*>(a.INV);
    const TF* PQG = static_cast<const TF*>(a.PQG);
    const TF* CF = static_cast<const TF*>(a.CF);
    const uint64_t pol = l2_evict_first();   // factor blocks are read once per sweep
    int issued = 0;
    bool ok = true;
#pragma unroll 1
    for (int n = 0; n < nslots && ok; ++n) {
      const int s = n % S;
      if (n >= S && !mbar_wait(&sm.empty[s], ((n / S) - 1) & 1)) {
        ok = false;
        break;
      }
      const bool fwd = n < tb0;                  // forward steps and the twist: one step per slot
      const int t = fwd ? n : tb0 + (n - tb0) * kPack;
      const bool twist = h == 0 && t == k;
      uint64_t* bar = &sm.full[s];
      if (lane == 0) {
        unsigned char* m = sm.mat[s];
        if (fwd) {
          const size_t o = blk0 + (size_t)row_of(t) * kBlockEntries;
          if constexpr (FIRST) {
            mbar_arrive_expect(bar, kBytesI + (twist ? 2 : 1) * kBytesF);
            bulk_load_hint(m, INV + o, kBytesI, bar, pol);
            bulk_load_hint(m + kBytesI, PQG + 3 * o + 2 * kBlockEntries, kBytesF, bar, pol);
            if (twist) bulk_load_hint(m + kOffH, CF + o, kBytesF, bar, pol);
          } else {
            mbar_arrive_expect(bar, (twist ? 4 : 3) * kBytesF);
            bulk_load_hint(m, PQG + 3 * o, 3 * kBytesF, bar, pol);   // P, Q, G: one run
            if (twist) bulk_load_hint(m + kOffH, CF + o, kBytesF, bar, pol);
          }
        } else {
          // a pack of up to kPack back steps: their rows are consecutive, so their C
          // blocks are one run starting at the lowest row
          const int c = min(kPack, nsteps - t);
          const int jlo = h == 0 ? row_of(t + c - 1) : row_of(t);
          const size_t o = blk0 + (size_t)jlo * kBlockEntries;
          mbar_arrive_expect(bar, c * kBytesF);
          bulk_load_hint(m, CF + o, c * kBytesF, bar, pol);
        }
      }
      issued = n + 1;
    }
    if (!ok) {
      // the consumers stopped: record it, and give the copies still in flight
      // a bounded time to land before the CTA's shared memory goes away
      if (lane == 0 && a.err != nullptr) atomicExch(a.err, 1u);
#pragma unroll 1
      for (int u = issued > S ? issued - S : 0; u < issued; ++u) (void)mbar_wait(&sm.full[u % S], (u / S) & 1);
    }
    return;
  }

  // ======================= consumers (one half, as in the rows variant) =======================
  const int q = warp;                          // row of the blocks owned by this warp
  const int l = lane;                          // line within the group
  const bool owner = l < grp.n;                // lanes past the group's last line only compute
  const int i = grp.i0 + (owner ? l : grp.n - 1);
  const int im = (i == 0) ? ni - 1 : i - 1;
  const int ip = (i + 1 == ni) ? 0 : i + 1;
  const size_t vq = vbase + (size_t)q * comp;  // component q of the case's vectors
  TX* x = reinterpret_cast<TX*>(a.x) + vq;
  // d_j in the compute type: in x itself, or (last sweep, FP64 x) in the scratch
  TC* dv = reinterpret_cast<TC*>(LAST ? a.dtmp : a.x) + vq;
  const int eo = (q * kLanes + l) * 4;         // this thread's entries in a block
  const TC* e0v = reinterpret_cast<const TC*>(a.e0) + vq;
  const TC* xpv = reinterpret_cast<const TC*>(a.xprev) + vq;
  const double* rv = a.r + vq;
  const int rstep = h == 0 ? ni : -ni;
  const int rf0 = h == 0 ? 0 : (nc - 1) * ni;
  const TC* e0b = e0v + i;
  const TC* xmb = xpv + im;
  const TC* xpb = xpv + ip;
  const double* rb = rv + i;
  TC* dvb = dv + i;
  TX* xb = x + i;
  const int nvec = h == 0 ? k + 1 : nf1;       // steps with vector entries (forward, and the twist)

  constexpr int L = kAhead;
  double rr[L];
  TC re[L], rm[L], rp[L];
  auto load_vec = [&](bool has, int off, int sl) {
    if (has) {
      if constexpr (FIRST) {
        rr[sl] = __ldcg(rb + off);
      } else {
        re[sl] = __ldcg(e0b + off);
        rm[sl] = __ldcg(xmb + off);
        rp[sl] = __ldcg(xpb + off);
      }
    }
  };
  auto store_vec = [&](bool has, int par, int sl) {
    if (has) {
      if constexpr (FIRST) {
        reinterpret_cast<double*>(sm.vec[par])[l * 4 + q] = rr[sl];
      } else {
        TC* v = reinterpret_cast<TC*>(sm.vec[par]) + l * 4 + q;
        v[0] = re[sl];
        v[kLanes * 4] = rm[sl];
        v[2 * kLanes * 4] = rp[sl];
      }
    }
  };
  bool wfail = false;
  auto wait_full = [&](int t) {
    if (!mbar_wait(&sm.full[t % S], (t / S) & 1)) wfail = true;
  };
  auto release = [&](int t) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[t % S]);
  };
  auto rhs = [&](int t, int s, int off) -> TC {
    const unsigned char* m = sm.mat[s];
    const unsigned char* vsb = sm.vec[t & 1];
    TC e;
    if constexpr (FIRST) {
      TC iv[4], rvv[4];
      load4(reinterpret_cast<const TI*>(m) + eo, iv);
      load4(reinterpret_cast<const double*>(vsb) + l * 4, rvv);
      e = iv[0] * rvv[0];
#pragma unroll
      for (int c = 1; c < 4; ++c) e += iv[c] * rvv[c];
      if (a.e0 != nullptr && owner) reinterpret_cast<TC*>(a.e0)[vq + i + off] = e;
    } else {
      const TC* vs = reinterpret_cast<const TC*>(vsb);
      TC pv[4], qv[4], xm[4], xp[4];
      load4(reinterpret_cast<const TF*>(m) + eo, pv);
      load4(reinterpret_cast<const TF*>(m + kBytesF) + eo, qv);
      load4(vs + kLanes * 4 + l * 4, xm);
      load4(vs + 2 * kLanes * 4 + l * 4, xp);
      TC s1 = pv[0] * xm[0];
      TC s2 = qv[0] * xp[0];
#pragma unroll
      for (int c = 1; c < 4; ++c) {
        s1 += pv[c] * xm[c];
        s2 += qv[c] * xp[c];
      }
      e = vs[l * 4 + q] + s1 - s2;
    }
    return e;
  };

  int done = 0;     // stages of the ring this warp has released
  int voff = rf0;   // row of the latest vector load
  load_vec(0 < nvec, voff, 0);
  store_vec(0 < nvec, 0, 0);
#pragma unroll
  for (int u = 1; u <= L; ++u) {
    voff += rstep;
    load_vec(u < nvec, voff, u % L);
  }
  consumers_sync();

  int tstop = -1;
  int roff = rf0;
  // ---- forward elimination of this half ----
#pragma unroll 1
  for (int tb = 0; tb < nf && tstop < 0; tb += L) {
#pragma unroll
    for (int uu = 0; uu < L; ++uu) {
      const int t = tb + uu;
      if (t < nf && tstop < 0) {
        const int s = t % S;
        wait_full(t);
        const TC e = rhs(t, s, roff);
        TC gv[4], dp[4];
        load4(reinterpret_cast<const TF*>(sm.mat[s] + kOffG) + eo, gv);
        release(t);
        ++done;
        load4(&sm.xchg[(t + 1) & 1][l][0], dp);
        TC d = e;
#pragma unroll
        for (int c = 0; c < 4; ++c) d += gv[c] * dp[c];
        sm.xchg[t & 1][l][q] = d;
        if (owner) dvb[roff] = d;
        roff += rstep;
        store_vec(t + 1 < nvec, (t + 1) & 1, (uu + 1) % L);
        voff += rstep;
        load_vec(t + 1 + L < nvec, voff, (uu + 1) % L);
        if (consumers_sync_or(wfail)) tstop = t;
      }
    }
  }
  if (tstop >= 0 && l == 0 && q == 0) sm.failed = 1;

  // ---- the halves meet: d'_{k+1} to the wall CTA, the twist row there, x_k back ----
  const uint32_t peer = 1u - (uint32_t)h;
  const int koff = k * ni;
  if (h == 1) {
    // the far-field half's last forward vector (zero without forward steps), into the
    // wall CTA's dfar; the fences and the barrier put every store before the arrival
    const TC dlast = nf1 > 0 ? sm.xchg[(nf1 + 1) & 1][l][q] : TC(0);
    peer_store(peer_addr(&sm.dfar[l][q], peer), dlast);
    fence_cluster();
    consumers_sync();
    if (tid == 0) peer_arrive(peer_addr(&sm.xbar, peer));
    // x_k from the wall CTA
    if (consumers_sync_or(!xbar_wait(&sm.xbar)) && tstop < 0) tstop = nf1;
  } else {
    if (consumers_sync_or(!xbar_wait(&sm.xbar)) && tstop < 0) tstop = k;
    if (tstop < 0) {
      // twist row k (as the rows variant's wall half computes it)
      const int t = k;
      const int s = t % S;
      wait_full(t);
      const TC e = rhs(t, s, koff);
      TC gv[4], hv[4], dm[4], dpl[4];
      load4(reinterpret_cast<const TF*>(sm.mat[s] + kOffG) + eo, gv);
      load4(reinterpret_cast<const TF*>(sm.mat[s] + kOffH) + eo, hv);
      release(t);
      ++done;
      load4(&sm.xchg[(k + 1) & 1][l][0], dm);                 // d_{k-1}
      if (nf1 > 0) load4(&sm.dfar[l][0], dpl);                // d'_{k+1}
      else dpl[0] = dpl[1] = dpl[2] = dpl[3] = TC(0);
      TC xv = e;
#pragma unroll
      for (int c = 0; c < 4; ++c) xv += gv[c] * dm[c];
#pragma unroll
      for (int c = 0; c < 4; ++c) xv += hv[c] * dpl[c];
      sm.xk[l][q] = xv;
      peer_store(peer_addr(&sm.xk[l][q], peer), xv);
      if (owner) xb[koff] = TX(xv);
      fence_cluster();
      if (consumers_sync_or(wfail)) tstop = t;
    }
    // the far-field CTA is released even after a failure (its x_k is then not used)
    if (tid == 0) peer_arrive(peer_addr(&sm.xbar, peer));
  }

  // ---- back substitution of this half, outward from the twist row ----
  if (tstop < 0) {
    const int t0 = h == 0 ? k + 1 : nf;
    const int bstep = -rstep;
    int boff = (h == 0 ? k - 1 : k + 1) * ni;   // row of back step t0
    int poff = boff;                            // row of the next prefetch
    TC dbuf[kBackAhead];
    int pslot = 0;                              // wall half: the pack's first step's block in the stage
#pragma unroll
    for (int u = 0; u < kBackAhead; ++u) {
      dbuf[u] = t0 + u < nsteps ? dvb[poff] : TC(0);
      poff += bstep;
    }
#pragma unroll 1
    for (int b0 = t0; b0 < nsteps && tstop < 0; b0 += kBackAhead) {
#pragma unroll
      for (int u = 0; u < kBackAhead; ++u) {
        const int t = b0 + u;
        if (t < nsteps && tstop < 0) {
          // t - t0 = (b0 - t0) + u with b0 - t0 a multiple of kPack: the step's place
          // in its pack is u % kPack, known at compile time
          const int n = tb0 + (t - tb0) / kPack;   // ring slot of the pack
          const int s = n % S;
          if (u % kPack == 0) {
            wait_full(n);
            // the pack's run starts at its lowest row: the wall half walks down
            const int c = min(kPack, nsteps - (t - u % kPack));
            pslot = h == 0 ? c - 1 : 0;
          }
          TC cv[4], xn[4];
          load4(reinterpret_cast<const TF*>(sm.mat[s] + (h == 0 ? pslot - u % kPack : u % kPack) * kBytesF) + eo, cv);
          if (u % kPack == kPack - 1 || t + 1 == nsteps) {
            release(n);
            ++done;
          }
          load4(t == t0 ? &sm.xk[l][0] : &sm.xchg[(t + 1) & 1][l][0], xn);
          TC acc = cv[0] * xn[0];
#pragma unroll
          for (int c = 1; c < 4; ++c) acc += cv[c] * xn[c];
          const TC xv = dbuf[u] - acc;
          sm.xchg[t & 1][l][q] = xv;
          if (owner) xb[boff] = TX(xv);
          boff += bstep;
          if (t + kBackAhead < nsteps) dbuf[u] = dvb[poff];
          poff += bstep;
          if (consumers_sync_or(wfail)) tstop = t;
        }
      }
    }
  }
  if (tstop >= 0 && tid == 0) {
    // a wait ran out: record it, and give the copies that may still be in flight (the
    // last released stage, whose wait may have run out, and the ones after it) a
    // bounded time to land
    if (a.err != nullptr) atomicExch(a.err, 1u);
#pragma unroll 1
    for (int u = done > 0 ? done - 1 : 0; u < done + S && u < nslots; ++u) (void)mbar_wait(&sm.full[u % S], (u / S) & 1);
  }
  cluster_sync();   // neither CTA leaves while the other may still store into its shared memory
}

}  // namespace halves

template <bool FIRST>
void launch_sweep_halves(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s) {
  using namespace halves;
  if (b.ngroups == 0) return;
  const int grid = 2 * b.ngroups;   // a cluster of two CTAs per 32-line group
  if (last) k_sweep<FIRST, true><<<grid, kSweepThreads, sizeof(SweepSmem), s>>>(b, a);
  else k_sweep<FIRST, false><<<grid, kSweepThreads, sizeof(SweepSmem), s>>>(b, a);
}

cudaError_t sweep_halves_init() {
  using namespace halves;
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SweepSmem));
  };
  set(reinterpret_cast<const void*>(&k_sweep<true, true>));
  set(reinterpret_cast<const void*>(&k_sweep<true, false>));
  set(reinterpret_cast<const void*>(&k_sweep<false, true>));
  set(reinterpret_cast<const void*>(&k_sweep<false, false>));
  return e;
}

template void launch_sweep_halves<true>(const Batch&, const SweepArgs&, bool, cudaStream_t);
template void launch_sweep_halves<false>(const Batch&, const SweepArgs&, bool, cudaStream_t);

}  // namespace a2d
