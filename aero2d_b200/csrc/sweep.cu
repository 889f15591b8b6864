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
// One CTA of two warps per 32-line group: warp 0 solves the wall half and
// warp 1 the far-field half, in parallel; each lane owns one line and all four
// rows of its 4x4 blocks, so a step needs no barrier: the recurrence's 4-vector
// stays in the lane's registers.  Each warp streams its own factor blocks: lane
// 0 keeps kStages steps in flight, one TMA bulk copy per factor run (a group's
// blocks of one row are one contiguous run: fbidx/fbidx3, a lane's block row is
// one vector load) into a ring of kStages stages, each with one mbarrier that
// counts the copy's bytes; once the warp is done with a stage, lane 0 refills
// it with the step kStages ahead.  Each lane loads its line's vector entries
// (r, or e0 and x' of both neighbour lines) through L2 into registers kAhead
// steps before their use (the vectors written by the preceding sweep bypass
// L1).  The halves meet at the twist row through shared memory, two named
// barriers of the CTA's 64 threads.  d_j goes to x (the last sweep, whose x is
// FP64: to a scratch vector) and comes back, register-prefetched, in the back
// substitution.  Every wait is bounded; a wait that runs out records an error,
// both warps still meet at both barriers, and each drains the copies it issued
// (bounded again) before it exits.
//
// Arithmetic and intermediate vectors are in the sweep's compute type: FP64
// in the FP64 path; FP32 in the mixed path, whose factors are FP16 and pivot
// inverses FP32 (a preconditioner only steers GMRES; the Newton residual and
// the Krylov reductions stay FP64).  The operation order of every row is fixed
// (products summed over the columns in order), so results are bitwise
// repeatable.
#include <type_traits>
#include <utility>

#include "batch.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace a2d {

constexpr int kSweepThreads = 64;                       // warp 0: wall half, warp 1: far-field half
constexpr int kBlockEntries = 16 * kLanes;              // one 4x4 block for the 32 lines of a group

// TI: pivot inverses (the Jacobian type); TF: the other factors (FactorStore);
// TC: arithmetic and intermediate vectors
template <typename TI> struct SweepTypes;
template <> struct SweepTypes<float> {
  using TF = __half;
  using TC = float;
  static constexpr int kStages = 6;     // bulk-copy ring stages per half
  static constexpr int kAhead = 8;      // steps between loading a vector entry and its use
  static constexpr int kBackAhead = 8;  // register prefetch depth of d in the back substitution
};
template <> struct SweepTypes<double> {
  using TF = double;
  using TC = double;
  static constexpr int kStages = 2;
  static constexpr int kAhead = 4;
  static constexpr int kBackAhead = 4;
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
  alignas(128) unsigned char mat[2][kS][kMatBytes];
  alignas(16) TC dk[kLanes][4];           // the far-field half's d'_{k+1}
  alignas(16) TC xk[kLanes][4];           // the twist row's solution
  uint64_t full[2][kS];
  int failed[2];                          // per half: a wait ran out
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
__device__ __forceinline__ void load4(const double* p, double (&v)[4]) {
  const double2 t0 = *reinterpret_cast<const double2*>(p);
  const double2 t1 = *reinterpret_cast<const double2*>(p + 2);
  v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
}

// f(integral_constant<int, sl>) for the runtime slot sl in [0, L): register
// arrays indexed through it keep static indices (a runtime index would put them
// in local memory)
template <typename F, int... I>
__device__ __forceinline__ void slot_dispatch(int sl, F&& f, std::integer_sequence<int, I...>) {
  ((sl == I ? f(std::integral_constant<int, I>{}) : void()), ...);
}

// the 64 threads of the CTA (named barrier 1)
__device__ __forceinline__ void halves_sync() { asm volatile("bar.sync 1, %0;" ::"r"(kSweepThreads) : "memory"); }

// orders this warp's reads of a ring stage before the bulk copy that refills it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

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
  constexpr uint32_t kOffG = FIRST ? kBytesI : 2 * kBytesF;   // G's block in a forward stage
  constexpr uint32_t kOffH = kOffG + kBytesF;                // H's block in the twist stage
  constexpr int L = SweepTypes<TI>::kAhead;
  constexpr int LB = SweepTypes<TI>::kBackAhead;

  const Group grp = b.groups[blockIdx.x];
  if (!case_live(b, grp.cs, a.need)) return;
  const int h = threadIdx.x >> 5;              // 0: from the wall, 1: from the far field
  const int l = threadIdx.x & 31;              // line within the group
  const CaseDev cs = b.cases[grp.cs];
  const int ni = cs.g.ni, nc = cs.g.nc;
  const int k = nc / 2;                        // twist row (as in k_factor)
  const int nf0 = k, nf1 = nc - 1 - k;         // forward steps of the wall / far-field half
  const int nf = h == 0 ? nf0 : nf1;
  const int nsteps = h == 0 ? 2 * k + 1 : 2 * nf1;
  // step t of the half: forward rows first; the wall half's step k is the twist
  // row; then the back substitution outward from the twist row
  auto row_of = [&](int t) {
    if (h == 0) return t <= k ? t : 2 * k - t;
    return t < nf1 ? nc - 1 - t : k + 1 + (t - nf1);
  };
  const size_t blk0 = lbidx(cs.rows_nc, nc, grp.g, 0, 0, 0);   // row j's block at blk0 + j * kBlockEntries

  if (l == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(&sm.full[h][s], 1);   // lane 0's arrival with the copy's bytes
    sm.failed[h] = 0;
    mbar_init_fence();
  }
  __syncthreads();

  // lane 0: bulk copies of step t's factor blocks into stage t % S
  const TI* INV = static_cast<const TI*>(a.INV);
  const TF* PQG = static_cast<const TF*>(a.PQG);
  const TF* CF = static_cast<const TF*>(a.CF);
  const uint64_t pol = l2_evict_first();   // factor blocks are read once per sweep
  int issued = 0;
  auto issue = [&](int t) {
    const int j = row_of(t);
    const bool twist = h == 0 && t == k;
    const bool fwd = twist || t < nf;
    uint64_t* bar = &sm.full[h][t % S];
    unsigned char* m = sm.mat[h][t % S];
    const size_t o = blk0 + (size_t)j * kBlockEntries;
    if (fwd) {
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
      mbar_arrive_expect(bar, kBytesF);
      bulk_load_hint(m, CF + o, kBytesF, bar, pol);
    }
  };
  if (l == 0)
    for (; issued < S && issued < nsteps; ++issued) issue(issued);
  // the warp is done with stage t: lane 0 refills it with step t + S
  auto advance = [&](int t) {
    __syncwarp();
    if (l == 0 && issued < nsteps) {
      fence_proxy_async();
      issue(issued);
      ++issued;
    }
  };
  // waits for step t's stage; false (on every lane) once any lane's wait ran out
  auto wait_full = [&](int t) -> bool {
    const bool ok = mbar_wait(&sm.full[h][t % S], (t / S) & 1);
    return __all_sync(0xffffffffu, ok);
  };

  const bool owner = l < grp.n;                // lanes past the group's last line only compute
  const int i = grp.i0 + (owner ? l : grp.n - 1);
  const int im = (i == 0) ? ni - 1 : i - 1;
  const int ip = (i + 1 == ni) ? 0 : i + 1;
  const size_t vbase = 4 * (size_t)cs.cell_off;
  const size_t comp = (size_t)nc * ni;         // stride between the components of a case vector
  // per-line bases: row offsets within a component plane stay 32-bit
  const TC* e0b = reinterpret_cast<const TC*>(a.e0) + vbase + i;
  const TC* xcb = reinterpret_cast<const TC*>(a.xprev) + vbase + i;
  const TC* xmb = reinterpret_cast<const TC*>(a.xprev) + vbase + im;
  const TC* xpb = reinterpret_cast<const TC*>(a.xprev) + vbase + ip;
  // x' of the neighbour lines comes from the neighbour lanes by shuffles; the
  // group's first lane and its last line's lane load the neighbour outside the group
  const int lastl = grp.n - 1;
  const double* rb = a.r + vbase + i;
  TC* e0w = reinterpret_cast<TC*>(a.e0) + vbase + i;
  // d_j in the compute type: in x itself, or (last sweep, FP64 x) in the scratch
  TC* dvb = reinterpret_cast<TC*>(LAST ? a.dtmp : a.x) + vbase + i;
  TX* xb = reinterpret_cast<TX*>(a.x) + vbase + i;
  const int eo = l * 4;                        // this lane's entries in block row r: eo + r * kLanes * 4
  const int rstep = h == 0 ? ni : -ni;
  const int rf0 = h == 0 ? 0 : (nc - 1) * ni;
  const int nvec = h == 0 ? k + 1 : nf1;       // steps with vector entries (forward, and the twist)

  // vector entries of step u in register slot sl: r (first sweep) or e0, and x'
  // of this line (rx), of the line before the group (rl, lane 0) and of the line
  // after the group's last (rr, lane lastl)
  TC re[L][4], rx[L][4], rl[L][4] = {}, rr[L][4] = {};   // rl / rr: loaded by the edge lanes only
  auto load_vec = [&](int u, int off, int sl) {
    if (u < nvec) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if constexpr (FIRST) {
          re[sl][c] = TC(__ldcg(rb + c * comp + off));
        } else {
          re[sl][c] = __ldcg(e0b + c * comp + off);
          rx[sl][c] = __ldcg(xcb + c * comp + off);
          if (l == 0) rl[sl][c] = __ldcg(xmb + c * comp + off);
          if (l == lastl) rr[sl][c] = __ldcg(xpb + c * comp + off);
        }
      }
    }
  };
  // e of a step from stage s and the step's vector entries (first sweep: va = r;
  // later sweeps: va = e0, vx = x' of the line, vl / vr the outside neighbours);
  // the first sweep also keeps e (row offset off).  All lanes call it (shuffles)
  auto rhs = [&](int s, int off, const TC (&va)[4], const TC (&vx)[4], const TC (&vl)[4], const TC (&vr)[4],
                 TC (&e)[4]) {
    const unsigned char* m = sm.mat[h][s];
    TC vm[4], vp[4];   // x'[i-1], x'[i+1]
    if constexpr (!FIRST) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const TC up = __shfl_up_sync(0xffffffffu, vx[c], 1);
        const TC dn = __shfl_down_sync(0xffffffffu, vx[c], 1);
        vm[c] = l == 0 ? vl[c] : up;
        vp[c] = l == lastl ? vr[c] : dn;
      }
    }
    if constexpr (FIRST) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        TC iv[4];
        load4(reinterpret_cast<const TI*>(m) + eo + r * kLanes * 4, iv);
        e[r] = iv[0] * va[0];
#pragma unroll
        for (int c = 1; c < 4; ++c) e[r] += iv[c] * va[c];
      }
      if (a.e0 != nullptr && owner) {
#pragma unroll
        for (int r = 0; r < 4; ++r) e0w[r * comp + off] = e[r];
      }
    } else {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        TC pv[4], qv[4];
        load4(reinterpret_cast<const TF*>(m) + eo + r * kLanes * 4, pv);
        load4(reinterpret_cast<const TF*>(m + kBytesF) + eo + r * kLanes * 4, qv);
        TC s1 = pv[0] * vm[0];
        TC s2 = qv[0] * vp[0];
#pragma unroll
        for (int c = 1; c < 4; ++c) {
          s1 += pv[c] * vm[c];
          s2 += qv[c] * vp[c];
        }
        e[r] = va[r] + s1 - s2;
      }
    }
  };
  // y += B x for the block at byte offset boff of stage s
  auto addmv = [&](int s, uint32_t boff, const TC (&xv)[4], TC (&y)[4]) {
    const TF* B = reinterpret_cast<const TF*>(sm.mat[h][s] + boff) + eo;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      TC bv[4];
      load4(B + r * kLanes * 4, bv);
#pragma unroll
      for (int c = 0; c < 4; ++c) y[r] += bv[c] * xv[c];
    }
  };

  bool fail = false;
  int consumed = 0;   // steps of this half whose stage has been consumed
  TC dprev[4] = {TC(0), TC(0), TC(0), TC(0)};   // d_{-1} = d'_{nc} = 0

  // ---- forward elimination of this half (unrolled by L: register slots are static) ----
  int voff = rf0;   // row of the latest vector load
#pragma unroll
  for (int u = 0; u < L; ++u) {
    load_vec(u, voff, u);
    voff += rstep;
  }
  int roff = rf0;   // row of the current forward step
#pragma unroll 1
  for (int tb = 0; tb < nf && !fail; tb += L) {
#pragma unroll
    for (int uu = 0; uu < L; ++uu) {
      const int t = tb + uu;
      if (t < nf && !fail) {
        const int s = t % S;
        if (!wait_full(t)) {
          fail = true;
        } else {
          TC d[4];
          rhs(s, roff, re[uu], rx[uu], rl[uu], rr[uu], d);
          addmv(s, kOffG, dprev, d);
          consumed = t + 1;
          advance(t);
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            if (owner) dvb[r * comp + roff] = d[r];
            dprev[r] = d[r];
          }
          roff += rstep;
          load_vec(t + L, voff, uu);   // refill the slot L steps ahead
          voff += rstep;
        }
      }
    }
  }
  // (A): the far-field half's d'_{k+1} to the wall half
  if (h == 1) {
#pragma unroll
    for (int r = 0; r < 4; ++r) sm.dk[l][r] = dprev[r];
  }
  if (fail && l == 0) sm.failed[h] = 1;
  halves_sync();
  // ---- twist row k (wall half): its vector entries are in slot k % L ----
  if (h == 0 && !(sm.failed[0] || sm.failed[1])) {
    const int t = k;
    const int s = t % S;
    if (!wait_full(t)) {
      fail = true;
    } else {
      TC xv[4], dpl[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) dpl[r] = sm.dk[l][r];
      // the twist's vector entries from register slot k % L (static indices)
      TC ve[4], vx[4], vl[4], vr[4];
      slot_dispatch(k % L, [&](auto slot) {
        constexpr int sl = decltype(slot)::value;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          ve[c] = re[sl][c];
          vx[c] = rx[sl][c];
          vl[c] = rl[sl][c];
          vr[c] = rr[sl][c];
        }
      }, std::make_integer_sequence<int, L>{});
      rhs(s, k * ni, ve, vx, vl, vr, xv);
      addmv(s, kOffG, dprev, xv);
      addmv(s, kOffH, dpl, xv);
      consumed = t + 1;
      advance(t);
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        sm.xk[l][r] = xv[r];
        if (owner) xb[r * comp + k * ni] = TX(xv[r]);
      }
    }
    if (fail && l == 0) sm.failed[0] = 1;
  }
  halves_sync();   // (B) x_k visible to both halves
  // ---- back substitution of this half, outward from the twist row ----
  if (!(sm.failed[0] || sm.failed[1])) {
    const int t0 = h == 0 ? k + 1 : nf;
    const int bstep = -rstep;
    int boff = (h == 0 ? k - 1 : k + 1) * ni;   // row of back step t0
    int poff = boff;                           // row of the next prefetch
    TC xn[4], dbuf[LB][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) xn[r] = sm.xk[l][r];
#pragma unroll
    for (int u = 0; u < LB; ++u) {
#pragma unroll
      for (int r = 0; r < 4; ++r) dbuf[u][r] = t0 + u < nsteps ? dvb[r * comp + poff] : TC(0);
      poff += bstep;
    }
#pragma unroll 1
    for (int b0 = t0; b0 < nsteps && !fail; b0 += LB) {
#pragma unroll
      for (int u = 0; u < LB; ++u) {
        const int t = b0 + u;
        if (t < nsteps && !fail) {
          const int s = t % S;
          if (!wait_full(t)) {
            fail = true;
          } else {
            const TF* Cb = reinterpret_cast<const TF*>(sm.mat[h][s]) + eo;
            TC xv[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              TC cv[4];
              load4(Cb + r * kLanes * 4, cv);
              TC acc = cv[0] * xn[0];
#pragma unroll
              for (int c = 1; c < 4; ++c) acc += cv[c] * xn[c];
              xv[r] = dbuf[u][r] - acc;
            }
            consumed = t + 1;
            advance(t);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              if (owner) xb[r * comp + boff] = TX(xv[r]);
              xn[r] = xv[r];
              if (t + LB < nsteps) dbuf[u][r] = dvb[r * comp + poff];
            }
            boff += bstep;
            poff += bstep;
          }
        }
      }
    }
  }
  if (fail || sm.failed[0] || sm.failed[1]) {
    // a copy never landed (here or in the other half): record it, and give the
    // copies this warp issued and has not consumed a bounded time to land
    // before the CTA's shared memory goes away
    if (l == 0) {
      if (a.err != nullptr) atomicExch(a.err, 1u);
#pragma unroll 1
      for (int u = consumed; u < issued; ++u) (void)mbar_wait(&sm.full[h][u % S], (u / S) & 1);
    }
  }
}

template <typename TI, bool FIRST>
void launch_sweep(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s, int variant) {
  if (b.ngroups == 0) return;
  if constexpr (sizeof(TI) == 4) {   // the rows and halves variants run mixed-precision plans only
    if (variant == kSweepRows) {
      launch_sweep_rows<TI, FIRST>(b, a, last, s);
      return;
    }
    if (variant == kSweepHalves) {
      launch_sweep_halves<FIRST>(b, a, last, s);
      return;
    }
  }
  if (variant == kSweepPairs) {
    launch_sweep_pairs<TI, FIRST>(b, a, last, s);
    return;
  }
  if (last) k_sweep<TI, FIRST, true><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
  else k_sweep<TI, FIRST, false><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
}

cudaError_t sweep_init() {
  cudaError_t e = sweep_rows_init();
  if (e == cudaSuccess) e = sweep_pairs_init();
  if (e == cudaSuccess) e = sweep_halves_init();
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

template void launch_sweep<float, true>(const Batch&, const SweepArgs&, bool, cudaStream_t, int);
template void launch_sweep<float, false>(const Batch&, const SweepArgs&, bool, cudaStream_t, int);
template void launch_sweep<double, true>(const Batch&, const SweepArgs&, bool, cudaStream_t, int);
template void launch_sweep<double, false>(const Batch&, const SweepArgs&, bool, cudaStream_t, int);

}  // namespace a2d
