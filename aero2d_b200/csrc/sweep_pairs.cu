// The pairs variant of the line-Jacobi sweep (sweep.cu has the kernel's
// mathematics and the lanes variant, sweep_rows.cu the rows variant).
//
// One CTA of five warps per 32-line group.  Warps 0-1 solve the wall half and
// warps 2-3 the far-field half, 16 lines per warp; the two lanes of a line
// (lane = 2 * line + p) own block rows 2p and 2p+1 of its 4x4 blocks, so a
// step's arithmetic is split two ways and the line's 4-vector is completed by
// one shuffle with the partner lane: no barrier between steps.  x' of the
// neighbour lines comes from the lanes two apart by shuffles; the lines at a
// warp's edges load theirs.  Warp 4 is the producer: for every step of each half
// its lane 0 brings the step's blocks (a group's blocks of one row are one
// contiguous run) by TMA bulk copies, L2 evict-first, into a ring of kStages
// stages per half with two mbarriers per stage: "full" (the copy's bytes) and
// "empty" (one arrival per consumer warp of the half done with the stage).
// Each lane prefetches its two components of the step's vector entries (r, or
// e0 and x') into registers kAhead steps ahead.  The halves meet at the twist
// row through shared memory and two named barriers of the 128 consumer
// threads.  The row arithmetic is the lanes variant's, in the same order, so the
// variants give bitwise the same results.  Every wait is bounded; a wait that
// runs out records an error, the consumers still meet at both barriers, and the
// producer gives its copies in flight a bounded time to land before exit.
#include <type_traits>
#include <utility>

#include "batch.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace a2d {
namespace pairs {

constexpr int kConsumerWarps = 4;                        // two per half, 16 lines each
constexpr int kConsumerThreads = kConsumerWarps * 32;
constexpr int kProducerWarp = kConsumerWarps;            // warp 4
constexpr int kSweepThreads = kConsumerThreads + 32;
constexpr int kBlockEntries = 16 * kLanes;               // one 4x4 block for the 32 lines of a group

template <typename TI> struct SweepTypes;
template <> struct SweepTypes<float> {
  using TF = __half;
  using TC = float;
  static constexpr int kStages = 6;
  static constexpr int kAhead = 8;
  static constexpr int kBackAhead = 8;
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
  static constexpr uint32_t kMatBytes = (kBytesI + 2 * kBytesF > 4 * kBytesF) ? kBytesI + 2 * kBytesF : 4 * kBytesF;
  alignas(128) unsigned char mat[2][kS][kMatBytes];
  alignas(16) TC dk[kLanes][4];           // the far-field half's d'_{k+1}
  alignas(16) TC xk[kLanes][4];           // the twist row's solution
  uint64_t full[2][kS];
  uint64_t empty[2][kS];
  int failed[2];
};

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

template <typename F, int... I>
__device__ __forceinline__ void slot_dispatch(int sl, F&& f, std::integer_sequence<int, I...>) {
  ((sl == I ? f(std::integral_constant<int, I>{}) : void()), ...);
}

// the 128 consumer threads (named barrier 1)
__device__ __forceinline__ void consumers_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(kConsumerThreads) : "memory");
}

// the line's 4-vector from this lane's two components (rows 2p, 2p+1) and the partner's
template <typename TC>
__device__ __forceinline__ void full4(int p, const TC (&own)[2], TC (&v)[4]) {
  const TC q0 = __shfl_xor_sync(0xffffffffu, own[0], 1);
  const TC q1 = __shfl_xor_sync(0xffffffffu, own[1], 1);
  v[0] = p ? q0 : own[0];
  v[1] = p ? q1 : own[1];
  v[2] = p ? own[0] : q0;
  v[3] = p ? own[1] : q1;
}

template <typename TI, bool FIRST, bool LAST>
__global__ void __launch_bounds__(kSweepThreads) k_sweep(Batch b, SweepArgs a) {
  using SM = SweepSmem<TI>;
  using TF = typename SM::TF;
  using TC = typename SM::TC;
  using TX = typename std::conditional<LAST, double, TC>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SM& sm = *reinterpret_cast<SM*>(smem_raw);
  constexpr int S = SM::kS;
  constexpr uint32_t kBytesI = SM::kBytesI, kBytesF = SM::kBytesF;
  constexpr uint32_t kOffG = FIRST ? kBytesI : 2 * kBytesF;
  constexpr uint32_t kOffH = kOffG + kBytesF;
  constexpr int L = SweepTypes<TI>::kAhead;
  constexpr int LB = SweepTypes<TI>::kBackAhead;

  const Group grp = b.groups[blockIdx.x];
  if (!case_live(b, grp.cs, a.need)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const CaseDev cs = b.cases[grp.cs];
  const int ni = cs.g.ni, nc = cs.g.nc;
  const int k = nc / 2;
  const int nf0 = k, nf1 = nc - 1 - k;
  const int ns0 = 2 * k + 1, ns1 = 2 * nf1;
  auto row_of = [&](int h, int t) {
    if (h == 0) return t <= k ? t : 2 * k - t;
    return t < nf1 ? nc - 1 - t : k + 1 + (t - nf1);
  };
  const size_t blk0 = lbidx(cs.rows_nc, nc, grp.g, 0, 0, 0);

  if (threadIdx.x == 0) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
      for (int s = 0; s < S; ++s) {
        mbar_init(&sm.full[h][s], 1);
        mbar_init(&sm.empty[h][s], 2);   // one arrival per consumer warp of the half
      }
      sm.failed[h] = 0;
    }
    mbar_init_fence();
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
    const int smax = ns0 > ns1 ? ns0 : ns1;
#pragma unroll 1
    for (int t = 0; t < smax && ok; ++t) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (!ok || t >= (h == 0 ? ns0 : ns1)) continue;
        const int s = t % S;
        if (t >= S && !mbar_wait(&sm.empty[h][s], ((t / S) - 1) & 1)) {
          ok = false;
          continue;
        }
        const int j = row_of(h, t);
        const bool twist = h == 0 && t == k;
        const bool fwd = twist || t < (h == 0 ? nf0 : nf1);
        uint64_t* bar = &sm.full[h][s];
        if (lane == 0) {
          unsigned char* m = sm.mat[h][s];
          const size_t o = blk0 + (size_t)j * kBlockEntries;
          if (fwd) {
            if constexpr (FIRST) {
              mbar_arrive_expect(bar, kBytesI + (twist ? 2 : 1) * kBytesF);
              bulk_load_hint(m, INV + o, kBytesI, bar, pol);
              bulk_load_hint(m + kBytesI, PQG + 3 * o + 2 * kBlockEntries, kBytesF, bar, pol);
              if (twist) bulk_load_hint(m + kOffH, CF + o, kBytesF, bar, pol);
            } else {
              mbar_arrive_expect(bar, (twist ? 4 : 3) * kBytesF);
              bulk_load_hint(m, PQG + 3 * o, 3 * kBytesF, bar, pol);
              if (twist) bulk_load_hint(m + kOffH, CF + o, kBytesF, bar, pol);
            }
          } else {
            mbar_arrive_expect(bar, kBytesF);
            bulk_load_hint(m, CF + o, kBytesF, bar, pol);
          }
        }
        issued[h] = t + 1;
      }
    }
    if (!ok) {
      if (lane == 0 && a.err != nullptr) atomicExch(a.err, 1u);
#pragma unroll 1
      for (int h = 0; h < 2; ++h)
        for (int u = issued[h] > S ? issued[h] - S : 0; u < issued[h]; ++u)
          (void)mbar_wait(&sm.full[h][u % S], (u / S) & 1);
    }
    return;
  }

  // ======================= consumers =======================
  const int h = warp >> 1;                     // 0: from the wall, 1: from the far field
  const int ln = lane >> 1;                    // line within the warp's 16
  const int p = lane & 1;                      // block rows 2p, 2p+1
  const int l = (warp & 1) * 16 + ln;          // line within the group
  const int r0 = 2 * p;
  const bool owner = l < grp.n;
  const int i = grp.i0 + (owner ? l : grp.n - 1);
  const int im = (i == 0) ? ni - 1 : i - 1;
  const int ip = (i + 1 == ni) ? 0 : i + 1;
  const bool left_edge = ln == 0;              // x'[i-1] is outside the warp
  const bool right_edge = ln == 15 || l == grp.n - 1;
  const int nf = h == 0 ? nf0 : nf1;
  const int nsteps = h == 0 ? ns0 : ns1;
  const size_t vbase = 4 * (size_t)cs.cell_off;
  const size_t comp = (size_t)nc * ni;
  const size_t c0 = (size_t)r0 * comp;         // this lane's first component plane
  const TC* e0b = reinterpret_cast<const TC*>(a.e0) + vbase + c0 + i;
  const TC* xcb = reinterpret_cast<const TC*>(a.xprev) + vbase + c0 + i;
  const TC* xmb = reinterpret_cast<const TC*>(a.xprev) + vbase + c0 + im;
  const TC* xpb = reinterpret_cast<const TC*>(a.xprev) + vbase + c0 + ip;
  const double* rb = a.r + vbase + c0 + i;
  TC* e0w = reinterpret_cast<TC*>(a.e0) + vbase + c0 + i;
  TC* dvb = reinterpret_cast<TC*>(LAST ? a.dtmp : a.x) + vbase + c0 + i;
  TX* xb = reinterpret_cast<TX*>(a.x) + vbase + c0 + i;
  const int rstep = h == 0 ? ni : -ni;
  const int rf0 = h == 0 ? 0 : (nc - 1) * ni;
  const int nvec = h == 0 ? k + 1 : nf1;
  const int eo = l * 4;                        // entries of line l in block row r: eo + r * kLanes * 4

  // this lane's two components of step u's vector entries, in slot sl
  TC re[L][2], rx[L][2], rl[L][2] = {}, rr[L][2] = {};   // rl / rr: loaded by the edge lanes only
  auto load_vec = [&](int u, int off, int sl) {
    if (u < nvec) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const size_t o = q * comp + off;
        if constexpr (FIRST) {
          re[sl][q] = TC(__ldcg(rb + o));
        } else {
          re[sl][q] = __ldcg(e0b + o);
          rx[sl][q] = __ldcg(xcb + o);
          if (left_edge) rl[sl][q] = __ldcg(xmb + o);
          if (right_edge) rr[sl][q] = __ldcg(xpb + o);
        }
      }
    }
  };
  // e of this lane's two rows (first sweep: va = r; later: va = e0, vx = x' of the
  // line, vl / vr the neighbours outside the warp); all lanes call it (shuffles)
  auto rhs = [&](int s, int off, const TC (&va)[2], const TC (&vx)[2], const TC (&vl)[2], const TC (&vr)[2],
                 TC (&e)[2]) {
    const unsigned char* m = sm.mat[h][s];
    if constexpr (FIRST) {
      TC rv[4];
      full4(p, va, rv);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        TC iv[4];
        load4(reinterpret_cast<const TI*>(m) + eo + (r0 + q) * kLanes * 4, iv);
        e[q] = iv[0] * rv[0];
#pragma unroll
        for (int c = 1; c < 4; ++c) e[q] += iv[c] * rv[c];
      }
      if (a.e0 != nullptr && owner) {
#pragma unroll
        for (int q = 0; q < 2; ++q) e0w[q * comp + off] = e[q];
      }
    } else {
      TC xo[4], xl[4], xr[4], vm[4], vp[4];
      full4(p, vx, xo);
      full4(p, vl, xl);
      full4(p, vr, xr);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const TC up = __shfl_up_sync(0xffffffffu, xo[c], 2);
        const TC dn = __shfl_down_sync(0xffffffffu, xo[c], 2);
        vm[c] = left_edge ? xl[c] : up;
        vp[c] = right_edge ? xr[c] : dn;
      }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        TC pv[4], qv[4];
        load4(reinterpret_cast<const TF*>(m) + eo + (r0 + q) * kLanes * 4, pv);
        load4(reinterpret_cast<const TF*>(m + kBytesF) + eo + (r0 + q) * kLanes * 4, qv);
        TC s1 = pv[0] * vm[0];
        TC s2 = qv[0] * vp[0];
#pragma unroll
        for (int c = 1; c < 4; ++c) {
          s1 += pv[c] * vm[c];
          s2 += qv[c] * vp[c];
        }
        e[q] = va[q] + s1 - s2;
      }
    }
  };
  // y += B x for this lane's two rows of the block at byte offset boff of stage s
  auto addmv = [&](int s, uint32_t boff, const TC (&xv)[4], TC (&y)[2]) {
    const TF* B = reinterpret_cast<const TF*>(sm.mat[h][s] + boff) + eo;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      TC bv[4];
      load4(B + (r0 + q) * kLanes * 4, bv);
#pragma unroll
      for (int c = 0; c < 4; ++c) y[q] += bv[c] * xv[c];
    }
  };
  auto wait_full = [&](int t) -> bool {
    const bool ok = mbar_wait(&sm.full[h][t % S], (t / S) & 1);
    return __all_sync(0xffffffffu, ok);
  };
  auto release = [&](int t) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[h][t % S]);
  };

  bool fail = false;
  TC dprev[4] = {TC(0), TC(0), TC(0), TC(0)};   // d_{-1} = d'_{nc} = 0

  // ---- forward elimination of this half ----
  int voff = rf0;
#pragma unroll
  for (int u = 0; u < L; ++u) {
    load_vec(u, voff, u);
    voff += rstep;
  }
  int roff = rf0;
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
          TC d[2];
          rhs(s, roff, re[uu], rx[uu], rl[uu], rr[uu], d);
          addmv(s, kOffG, dprev, d);
          release(t);
#pragma unroll
          for (int q = 0; q < 2; ++q)
            if (owner) dvb[q * comp + roff] = d[q];
          full4(p, d, dprev);
          roff += rstep;
          load_vec(t + L, voff, uu);
          voff += rstep;
        }
      }
    }
  }
  // (A): the far-field half's d'_{k+1} to the wall half
  if (h == 1) {
#pragma unroll
    for (int q = 0; q < 2; ++q) sm.dk[l][r0 + q] = p ? dprev[2 + q] : dprev[q];   // static register indices
  }
  if (fail && lane == 0) sm.failed[h] = 1;
  consumers_sync();
  // ---- twist row k (wall half) ----
  if (h == 0 && !(sm.failed[0] || sm.failed[1])) {
    const int t = k;
    const int s = t % S;
    if (!wait_full(t)) {
      fail = true;
    } else {
      TC xv[2], dpl[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) dpl[c] = sm.dk[l][c];
      TC ve[2], vx[2], vl[2], vr[2];
      slot_dispatch(k % L, [&](auto slot) {
        constexpr int sl = decltype(slot)::value;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          ve[q] = re[sl][q];
          vx[q] = rx[sl][q];
          vl[q] = rl[sl][q];
          vr[q] = rr[sl][q];
        }
      }, std::make_integer_sequence<int, L>{});
      rhs(s, k * ni, ve, vx, vl, vr, xv);
      addmv(s, kOffG, dprev, xv);
      addmv(s, kOffH, dpl, xv);
      release(t);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        sm.xk[l][r0 + q] = xv[q];
        if (owner) xb[q * comp + k * ni] = TX(xv[q]);
      }
    }
    if (fail && lane == 0) sm.failed[0] = 1;
  }
  consumers_sync();   // (B) x_k visible to both halves
  // ---- back substitution, outward from the twist row ----
  if (!(sm.failed[0] || sm.failed[1])) {
    const int t0 = h == 0 ? k + 1 : nf;
    const int bstep = -rstep;
    int boff = (h == 0 ? k - 1 : k + 1) * ni;
    int poff = boff;
    TC xn[4], dbuf[LB][2];
#pragma unroll
    for (int c = 0; c < 4; ++c) xn[c] = sm.xk[l][c];
#pragma unroll
    for (int u = 0; u < LB; ++u) {
#pragma unroll
      for (int q = 0; q < 2; ++q) dbuf[u][q] = t0 + u < nsteps ? dvb[q * comp + poff] : TC(0);
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
            TC xv[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              TC cv[4];
              load4(Cb + (r0 + q) * kLanes * 4, cv);
              TC acc = cv[0] * xn[0];
#pragma unroll
              for (int c = 1; c < 4; ++c) acc += cv[c] * xn[c];
              xv[q] = dbuf[u][q] - acc;
            }
            release(t);
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              if (owner) xb[q * comp + boff] = TX(xv[q]);
              if (t + LB < nsteps) dbuf[u][q] = dvb[q * comp + poff];
            }
            full4(p, xv, xn);
            boff += bstep;
            poff += bstep;
          }
        }
      }
    }
  }
  if (fail && lane == 0 && a.err != nullptr) atomicExch(a.err, 1u);
}

}  // namespace pairs

template <typename TI, bool FIRST>
void launch_sweep_pairs(const Batch& b, const SweepArgs& a, bool last, cudaStream_t s) {
  using namespace pairs;
  if (b.ngroups == 0) return;
  if (last) k_sweep<TI, FIRST, true><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
  else k_sweep<TI, FIRST, false><<<b.ngroups, kSweepThreads, sizeof(SweepSmem<TI>), s>>>(b, a);
}

cudaError_t sweep_pairs_init() {
  using namespace pairs;
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

template void launch_sweep_pairs<float, true>(const Batch&, const SweepArgs&, bool, cudaStream_t);
template void launch_sweep_pairs<float, false>(const Batch&, const SweepArgs&, bool, cudaStream_t);
template void launch_sweep_pairs<double, true>(const Batch&, const SweepArgs&, bool, cudaStream_t);
template void launch_sweep_pairs<double, false>(const Batch&, const SweepArgs&, bool, cudaStream_t);

}  // namespace a2d
