// The row-warp variant of the line-Jacobi sweep (sweep.cu has the kernel's
// mathematics and the lane-per-line variant): one CTA of nine warps per 32-line
// group, warp-specialised.  Warps 0-3 solve the wall half and warps 4-7 the
// far-field half, in parallel (lane = line, warp = row of the 4x4 blocks, so a
// line's 4-vector passes between the four row warps of a half through a two-slot
// shared exchange buffer, one named barrier per step); warp 8 is the producer:
// for every step of each half its lane 0 brings the step's blocks by TMA bulk
// copies (the back substitution's C blocks four consecutive rows to a copy) into
// a ring of kStages stages per half with two mbarriers per stage,
// "full" (the bulk-copy bytes) and "empty" (one arrival per consumer warp done
// with the stage).  Each consumer thread loads its own vector entries of the
// forward steps (component q of its line) through L2 into registers kAhead
// steps ahead and stores them into a two-slot shared buffer the step before
// they are used; the halves meet twice around the twist row.  Four warps per
// line half spread a step's arithmetic over more threads than the lane variant
// (a plan's tuning knob picks one, aero2d_b200.autotune).  The row arithmetic is
// the same as the lane variant's, in the same order.  Mixed-precision plans only:
// an FP64 form gave results that depended on which other cases shared the batch
// (deterministic for a given batch; the cause was not found), so FP64 plans run
// the lane or pair variants, whose results are independent of the batch.  Every wait is bounded; a
// wait that runs out records an error and the CTA drains its copies in flight
// (bounded again) before exit.
#include <type_traits>

#include "batch.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace a2d {
namespace rows {

constexpr int kHalfThreads = 128;                       // consumer threads of one half
constexpr int kConsumerThreads = 2 * kHalfThreads;
constexpr int kProducerWarp = kConsumerThreads / 32;    // warp 8
constexpr int kSweepThreads = kConsumerThreads + 32;
constexpr int kBlockEntries = 16 * kLanes;              // one 4x4 block for the 32 lines of a group
constexpr int kBackAhead = 8;                           // register prefetch depth of d in the back substitution
constexpr int kPack = 4;                                // back-substitution steps per ring stage (their rows are contiguous)
static_assert(kBackAhead % kPack == 0, "a back prefetch block holds whole packs");

// TI: pivot inverses (the Jacobian type); TF: the other factors (FactorStore);
// TC: arithmetic and intermediate vectors
template <typename TI> struct SweepTypes;
template <> struct SweepTypes<float> {
  using TF = __half;
  using TC = float;
  static constexpr int kStages = 4;   // bulk-copy ring stages per half
  static constexpr int kAhead = 4;    // steps between loading a vector entry and its use
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
  alignas(16) unsigned char vec[2][2][kVecBytes];   // per half, by step parity
  alignas(16) TC xchg[2][2][kLanes][4];   // per half: the previous step's 4-vector of every line
  alignas(16) TC xk[kLanes][4];           // the twist row's solution
  uint64_t full[2][kS];
  uint64_t empty[2][kS];
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

// barrier of the 128 consumer threads of one half (ids 1, 2) and of all 256
// consumer threads (id 3); the producer warp takes part in none
__device__ __forceinline__ void half_sync(int h) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + h), "r"(kHalfThreads) : "memory");
}
// the same barrier of one half, OR-reducing a per-thread flag over its 128 threads
__device__ __forceinline__ bool half_sync_or(int h, bool flag) {
  uint32_t r;
  asm volatile(
      "{\n"
      " .reg .pred pi, po;\n"
      " setp.ne.u32 pi, %1, 0;\n"
      " bar.red.or.pred po, %2, %3, pi;\n"
      " selp.u32 %0, 1, 0, po;\n"
      "}\n"
      : "=r"(r)
      : "r"((uint32_t)flag), "r"(1 + h), "r"(kHalfThreads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void consumers_sync() {
  asm volatile("bar.sync 3, %0;" ::"r"(kConsumerThreads) : "memory");
}

template <typename TI, bool FIRST, bool LAST>
__global__ void __launch_bounds__(kSweepThreads, 4) k_sweep(Batch b, SweepArgs a) {
  using SM = SweepSmem<TI>;
  using TF = typename SM::TF;
  using TC = typename SM::TC;
  using TX = typename std::conditional<LAST, double, TC>::type;   // type of x
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SM& sm = *reinterpret_cast<SM*>(smem_raw);
  constexpr int S = SM::kS;
  constexpr uint32_t kBytesI = SM::kBytesI, kBytesF = SM::kBytesF;
  constexpr uint32_t kOffG = FIRST ? kBytesI : 2 * kBytesF;   // G's block in a forward stage
  constexpr uint32_t kOffH = kOffG + kBytesF;                // H's block in the twist stage

  const Group grp = b.groups[blockIdx.x];
  if (!case_live(b, grp.cs, a.need)) return;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const CaseDev cs = b.cases[grp.cs];
  const int ni = cs.g.ni, nc = cs.g.nc;
  const int k = nc / 2;                        // twist row (as in k_factor)
  const int nf0 = k, nf1 = nc - 1 - k;         // forward steps of the wall / far-field half
  const int ns0 = 2 * k + 1, ns1 = 2 * nf1;    // steps of each half
  // ring slots of each half: one per forward step (and the twist), then one per
  // pack of up to kPack back-substitution steps, from the half's first back step
  const int nsl0 = k + 1 + (ns0 - k - 1 + kPack - 1) / kPack;
  const int nsl1 = nf1 + (ns1 - nf1 + kPack - 1) / kPack;
  // step t of half h: forward rows first; the wall half's step k is the twist
  // row; then the back substitution outward from the twist row
  auto row_of = [&](int h, int t) {
    if (h == 0) return t <= k ? t : 2 * k - t;
    return t < nf1 ? nc - 1 - t : k + 1 + (t - nf1);
  };
  const size_t vbase = 4 * (size_t)cs.cell_off;
  const size_t comp = (size_t)nc * ni;         // stride between the components of a case vector
  const size_t blk0 = lbidx(cs.rows_nc, nc, grp.g, 0, 0, 0);   // row j's block at blk0 + j * kBlockEntries

  if (tid == 0) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
      for (int s = 0; s < S; ++s) {
        mbar_init(&sm.full[h][s], 1);        // the producer's arrival with the bulk-copy bytes
        mbar_init(&sm.empty[h][s], 4);       // one arrival per consumer warp of the half
      }
      sm.failed[h] = 0;
    }
    mbar_init_fence();
  }
  if (warp < kProducerWarp) {
    const int h = warp >> 2, q = warp & 3;
    sm.xchg[h][0][lane][q] = TC(0);
    sm.xchg[h][1][lane][q] = TC(0);   // d_{-1} = d'_{nc} = 0
  }
  __syncthreads();

  // ======================= producer warp =======================
  if (warp == kProducerWarp) {
    const TI* INV = static_cast<const TI*>(a.INV);
    const TF* PQG = static_cast<const TF*>(a.PQG);
    const TF* CF = static_cast<const TF*>(a.CF);
    const uint64_t pol = l2_evict_first();   // factor blocks are read once per sweep
    int issued[2] = {0, 0};
    bool ok = true;
    const int nmax = nsl0 > nsl1 ? nsl0 : nsl1;
#pragma unroll 1
    for (int n = 0; n < nmax && ok; ++n) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (!ok || n >= (h == 0 ? nsl0 : nsl1)) continue;
        const int s = n % S;
        if (n >= S && !mbar_wait(&sm.empty[h][s], ((n / S) - 1) & 1)) {
          ok = false;
          continue;
        }
        const int tb = h == 0 ? k + 1 : nf1;      // the half's first back step
        const bool fwd = n < tb;                  // forward steps and the twist: one step per slot
        const int t = fwd ? n : tb + (n - tb) * kPack;
        const bool twist = h == 0 && t == k;
        uint64_t* bar = &sm.full[h][s];
        if (lane == 0) {
          unsigned char* m = sm.mat[h][s];
          if (fwd) {
            const size_t o = blk0 + (size_t)row_of(h, t) * kBlockEntries;
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
            // a pack of up to kPack back steps: their rows are consecutive, so
            // their C blocks are one run starting at the lowest row
            const int c = min(kPack, (h == 0 ? ns0 : ns1) - t);
            const int jlo = h == 0 ? row_of(h, t + c - 1) : row_of(h, t);
            const size_t o = blk0 + (size_t)jlo * kBlockEntries;
            mbar_arrive_expect(bar, c * kBytesF);
            bulk_load_hint(m, CF + o, c * kBytesF, bar, pol);
          }
        }
        issued[h] = n + 1;
      }
    }
    if (!ok) {
      // the consumers stopped: record it, and give the copies still in flight
      // a bounded time to land before the CTA's shared memory goes away
      if (lane == 0 && a.err != nullptr) atomicExch(a.err, 1u);
#pragma unroll 1
      for (int h = 0; h < 2; ++h)
        for (int u = issued[h] > S ? issued[h] - S : 0; u < issued[h]; ++u)
          (void)mbar_wait(&sm.full[h][u % S], (u / S) & 1);
    }
    return;
  }

  // ======================= consumers =======================
  const int h = warp >> 2;                     // 0: from the wall, 1: from the far field
  const int q = warp & 3;                      // row of the blocks owned by this warp
  const int l = lane;                          // line within the group
  const bool owner = l < grp.n;                // lanes past the group's last line only compute
  const int i = grp.i0 + (owner ? l : grp.n - 1);
  const int im = (i == 0) ? ni - 1 : i - 1;
  const int ip = (i + 1 == ni) ? 0 : i + 1;
  const int nf = h == 0 ? nf0 : nf1;
  const int nsteps = h == 0 ? ns0 : ns1;
  const size_t vq = vbase + (size_t)q * comp;  // component q of the case's vectors
  TX* x = reinterpret_cast<TX*>(a.x) + vq;
  // d_j in the compute type: in x itself, or (last sweep, FP64 x) in the scratch
  TC* dv = reinterpret_cast<TC*>(LAST ? a.dtmp : a.x) + vq;
  const int eo = (q * kLanes + l) * 4;         // this thread's entries in a block
  const TC* e0v = reinterpret_cast<const TC*>(a.e0) + vq;
  const TC* xpv = reinterpret_cast<const TC*>(a.xprev) + vq;
  const double* rv = a.r + vq;

  // rows as offsets into a component plane: forward step t of the half is row
  // jf0 + t * jdir (the wall half's twist row k continues the sequence); the
  // back substitution runs outward from the twist row
  const int rstep = h == 0 ? ni : -ni;
  const int rf0 = h == 0 ? 0 : (nc - 1) * ni;
  // per-thread bases: offsets within a component plane stay 32-bit
  const TC* e0b = e0v + i;
  const TC* xmb = xpv + im;
  const TC* xpb = xpv + ip;
  const double* rb = rv + i;
  TC* dvb = dv + i;
  TX* xb = x + i;
  const int nvec = h == 0 ? k + 1 : nf1;       // steps with vector entries (forward, and the twist)

  // the vector entries of step u: each thread loads component q of its line (r,
  // or e0 and x' of both neighbour lines) into register slot sl and later stores
  // it into the step's parity slot
  constexpr int L = SweepTypes<TI>::kAhead;
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
        reinterpret_cast<double*>(sm.vec[h][par])[l * 4 + q] = rr[sl];
      } else {
        TC* v = reinterpret_cast<TC*>(sm.vec[h][par]) + l * 4 + q;
        v[0] = re[sl];
        v[kLanes * 4] = rm[sl];
        v[2 * kLanes * 4] = rp[sl];
      }
    }
  };

  // waits for stage t of the half; a wait that runs out is remembered and
  // OR-reduced over the half by the step's barrier
  bool wfail = false;
  auto wait_full = [&](int t) {
    if (!mbar_wait(&sm.full[h][t % S], (t / S) & 1)) wfail = true;
  };
  // this warp is done with stage t % S
  auto release = [&](int t) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[h][t % S]);
  };
  // e of step t from the forward blocks of stage s and the step's vector entries;
  // the first sweep also keeps e (row offset off) for the later sweeps
  auto rhs = [&](int t, int s, int off) -> TC {
    const unsigned char* m = sm.mat[h][s];
    const unsigned char* vsb = sm.vec[h][t & 1];
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

  // step 0's entries stored, steps 1 .. L in flight
  int voff = rf0;   // row of the latest vector load
  load_vec(0 < nvec, voff, 0);
  store_vec(0 < nvec, 0, 0);
#pragma unroll
  for (int u = 1; u <= L; ++u) {
    voff += rstep;
    load_vec(u < nvec, voff, u % L);
  }
  half_sync(h);

  int tstop = -1;     // step at which a wait ran out
  int roff = rf0;   // row of the current forward step
  // ---- forward eliminations of both halves (unrolled by L: register slots are static) ----
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
        load4(reinterpret_cast<const TF*>(sm.mat[h][s] + kOffG) + eo, gv);
        release(t);
        load4(&sm.xchg[h][(t + 1) & 1][l][0], dp);
        TC d = e;
#pragma unroll
        for (int c = 0; c < 4; ++c) d += gv[c] * dp[c];
        sm.xchg[h][t & 1][l][q] = d;
        if (owner) dvb[roff] = d;
        roff += rstep;
        store_vec(t + 1 < nvec, (t + 1) & 1, (uu + 1) % L);   // step t+1's entries, published by the barrier
        voff += rstep;
        load_vec(t + 1 + L < nvec, voff, (uu + 1) % L);       // and the slot refilled L steps ahead
        if (half_sync_or(h, wfail)) tstop = t;
      }
    }
  }
  if (tstop >= 0 && l == 0 && q == 0) sm.failed[h] = 1;
  consumers_sync();   // (A) both forward eliminations done
  // ---- twist row k (wall half) ----
  if (!(sm.failed[0] || sm.failed[1]) && h == 0) {
    const int t = k;
    const int s = t % S;
    const int koff = k * ni;
    wait_full(t);
    const TC e = rhs(t, s, koff);
    TC gv[4], hv[4], dm[4], dpl[4];
    load4(reinterpret_cast<const TF*>(sm.mat[h][s] + kOffG) + eo, gv);
    load4(reinterpret_cast<const TF*>(sm.mat[h][s] + kOffH) + eo, hv);
    release(t);
    load4(&sm.xchg[0][(k + 1) & 1][l][0], dm);                        // d_{k-1}
    if (nf1 > 0) load4(&sm.xchg[1][(nf1 + 1) & 1][l][0], dpl);        // d'_{k+1}
    else dpl[0] = dpl[1] = dpl[2] = dpl[3] = TC(0);
    TC xv = e;
#pragma unroll
    for (int c = 0; c < 4; ++c) xv += gv[c] * dm[c];
#pragma unroll
    for (int c = 0; c < 4; ++c) xv += hv[c] * dpl[c];
    sm.xk[l][q] = xv;
    if (owner) xb[koff] = TX(xv);
    if (half_sync_or(h, wfail)) {
      tstop = t;
      if (l == 0 && q == 0) sm.failed[h] = 1;
    }
  }
  consumers_sync();   // (B) x_k visible to both halves
  // ---- back substitutions of both halves, outward from the twist row ----
  const int t0 = h == 0 ? k + 1 : nf;
  if (!(sm.failed[0] || sm.failed[1])) {
    const int bstep = -rstep;                               // outward from the twist row
    int boff = (h == 0 ? k - 1 : k + 1) * ni;               // row of back step t0
    int poff = boff;                                        // row of the next prefetch
    TC dbuf[kBackAhead];
    int pslot = 0;                                          // wall half: the pack's first step's block in the stage
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
          // b0 - t0 is a multiple of kPack: the step's place in its pack is u % kPack
          const int n = t0 + (t - t0) / kPack;     // ring slot of the pack
          const int s = n % S;
          if (u % kPack == 0) {
            wait_full(n);
            // the pack's run starts at its lowest row: the wall half walks down
            const int c = min(kPack, nsteps - (t - u % kPack));
            pslot = h == 0 ? c - 1 : 0;
          }
          TC cv[4], xn[4];
          load4(reinterpret_cast<const TF*>(sm.mat[h][s] + (h == 0 ? pslot - u % kPack : u % kPack) * kBytesF) + eo, cv);
          if (u % kPack == kPack - 1 || t + 1 == nsteps) release(n);
          load4(t == t0 ? &sm.xk[l][0] : &sm.xchg[h][(t + 1) & 1][l][0], xn);
          TC acc = cv[0] * xn[0];
#pragma unroll
          for (int c = 1; c < 4; ++c) acc += cv[c] * xn[c];
          const TC xv = dbuf[u] - acc;
          sm.xchg[h][t & 1][l][q] = xv;
          if (owner) xb[boff] = TX(xv);
          boff += bstep;
          if (t + kBackAhead < nsteps) dbuf[u] = dvb[poff];
          poff += bstep;
          if (half_sync_or(h, wfail)) tstop = t;
        }
      }
    }
  }
  if (tstop >= 0 && l == 0 && q == 0) {
    // a copy never landed: record it, and give the copies that may still be in
    // flight for this half (issued for ring slots n .. n+S-1 from the slot of step
    // tstop) a bounded time
    if (a.err != nullptr) atomicExch(a.err, 1u);
    const int n0 = tstop < t0 ? tstop : t0 + (tstop - t0) / kPack;
#pragma unroll 1
    for (int u = n0; u < n0 + S && u < (h == 0 ? nsl0 : nsl1); ++u) (void)mbar_wait(&sm.full[h][u % S], (u / S) & 1);
  }
}

}  // namespace rows

template <typename TI, bool FIRST>
void launch_sweep_rows(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s) {
  using namespace rows;
  if (b.ngroups == 0) return;
  if (last) k_sweep<TI, FIRST, true><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
  else k_sweep<TI, FIRST, false><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
}

cudaError_t sweep_rows_init() {
  using namespace rows;
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f, size_t bytes) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  };
#define A2D_SWEEP_ATTR(TI, F, L) set(reinterpret_cast<const void*>(&k_sweep<TI, F, L>), sizeof(SweepSmem<TI>));
  A2D_SWEEP_ATTR(float, true, true) A2D_SWEEP_ATTR(float, true, false)
  A2D_SWEEP_ATTR(float, false, true) A2D_SWEEP_ATTR(float, false, false)
#undef A2D_SWEEP_ATTR
  return e;
}

template void launch_sweep_rows<float, true>(const Batch&, const SweepArgs&, bool, cudaStream_t);
template void launch_sweep_rows<float, false>(const Batch&, const SweepArgs&, bool, cudaStream_t);

}  // namespace a2d
