// fk_mark.cuh -- the marking sieve for long lanes (stage S1 + marking).
//
// A weak sieve (small n: every prime kills only a few residues) leaves many
// candidates alive deep into the prime list, and testing each of them
// against every remaining prime costs tens of tests per candidate.  Long
// lanes are therefore sieved the Eratosthenes way instead: one CTA owns one
// lane over kSeg * kSegPerTask consecutive periods, and per segment of
// kSeg periods it
//   (a) ORs the compile-time pattern primes into a 512-word bitmap (the
//       stage-1a pattern sieve of fk_sieve.cuh, two words per thread),
//   (b) marks every other prime below 2^16 into a kSeg-byte shared map:
//       for each (prime, forbidden residue) the hits are an arithmetic
//       progression of step q in u, written with plain byte stores (a mark
//       is idempotent, so there is no read-modify-write and no atomic), and
//   (c) extracts the periods that neither marked, tests any primes beyond
//       the marked range one by one, and appends the survivors to the
//       candidate list.
// This is the reference AP engine's bitmap marking (primorial-ap/ap_gpu.py:
// 204-369: tabulated small primes, shared-memory marks for mid primes,
// global atomics for the rest) re-laid out per lane, so no mark needs an
// atomic and every engine kind can use it.
#pragma once
#include "fk_sieve.cuh"

namespace fk {

struct MarkSmem {
  unsigned char bytes[kSeg];
  u64 patw[kSeg / 64];
  unsigned short s16[8192];
  u32 warp[kBlock / 32];
  u32 minv[kNS];
  u32 sbits[512];
  u64 task;
  u32 item;
  u32 eng;
  u32 status;
  u32 pad;
  unsigned long long mbar;
};

template <int P0, int I, int NS>
struct PatSkip {
  // advance every phase by a compile-time number of periods
  template <u32 STEP>
  static __device__ __forceinline__ void skip(u32* rho) {
    constexpr u32 q = fk_nth_prime(P0 + I);
    constexpr u32 st = STEP % q;
    const u32 a = rho[I] + st;
    rho[I] = min(a, a - q);
    PatSkip<P0, I + 1, NS>::template skip<STEP>(rho);
  }
};
template <int P0, int NS>
struct PatSkip<P0, NS, NS> {
  template <u32 STEP>
  static __device__ __forceinline__ void skip(u32*) {}
};

// Stage an engine's pattern table into shared memory with a bulk async
// copy, bounded wait.  Returns false (and flags the counters) on timeout.
template <int P0>
__device__ __forceinline__ bool stage_patterns(u64* spat, const DevEngine& eg,
                                               unsigned long long* mbar,
                                               u32* status, u32& phase,
                                               DevCounters* ctr) {
  __syncthreads();
  if (threadIdx.x == 0) {
    *status = 0;
    const u32 mb = smem_u32(mbar);
    const u32 bytes = pat_bytes<P0>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile(
        "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb),
        "r"(bytes)
        : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1], %2, [%3];" ::"r"(smem_u32(spat)),
        "l"((u64)__cvta_generic_to_global(eg.pat)), "r"(bytes), "r"(mb)
        : "memory");
    u32 done = 0, spins = 0;
    while (!done) {
      asm volatile(
          "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, "
          "[%1], %2; selp.u32 %0, 1, 0, p; }"
          : "=r"(done)
          : "r"(mb), "r"(phase)
          : "memory");
      if (!done && ++spins > kWaitSpins) break;
    }
    if (!done) {
      *status = 1;
      atomicOr(&ctr->overflow, 4u);
    }
  }
  phase ^= 1u;
  __syncthreads();
  return *status == 0;
}

template <int KIND>
__device__ __forceinline__ bool tail_alive(u64 v, const DevEngine& e,
                                           const u32* __restrict__ xq,
                                           const u32* s_sbits, u64& ntest) {
  for (u32 i = e.NPm; i < e.NP; ++i) {
    const PrimeRec pr = e.recs[i];
    u32 rr = fk_bmod(v, pr.q, pr.magic) + __ldg(xq + i);
    rr = min(rr, rr - pr.q);
    ++ntest;
    if (kill_test<KIND>(pr, rr, e.lists, s_sbits, e.xxmax, e.n)) return false;
  }
  return true;
}

template <int P0>
__global__ void __launch_bounds__(kBlock, 2) k_mark(SieveArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  u64* spat = reinterpret_cast<u64*>(smem_raw);
  MarkSmem& S = *reinterpret_cast<MarkSmem*>(smem_raw + pat_bytes<P0>());
  const int tid = threadIdx.x;
  if (tid == 0) {
    S.eng = 0xFFFFFFFFu;
    const u32 mb = smem_u32(&S.mbar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  u32 phase = 0;
  u64 nmark = 0, ntest = 0, nword = 0;

  for (;;) {
    if (tid == 0) {
      const u64 t = atomicAdd(a.task_ctr, 1ull);
      S.task = t;
      if (t < a.ntask) {
        u32 lo = 0, hi = a.nitems;
        while (hi - lo > 1) {
          const u32 mid = (lo + hi) >> 1;
          if (a.task_prefix[mid] <= t) lo = mid; else hi = mid;
        }
        S.item = lo;
      }
    }
    __syncthreads();
    const u64 task = S.task;
    if (task >= a.ntask) break;
    const u32 gitem = a.item_index[S.item];
    const DevItem it = a.items[gitem];
    const u32 eidx = it.engine;
    const DevEngine& eg = a.engines[eidx];
    if (S.eng != eidx) {
      if (!stage_patterns<P0>(spat, eg, &S.mbar, &S.status, phase, a.ctr))
        return;
      for (u32 i = tid; i < kNS; i += kBlock) S.minv[i] = eg.pat_minv[i];
      for (u32 i = tid; i < eg.sbits_words && i < 512; i += kBlock)
        S.sbits[i] = eg.sbits[i];
      __syncthreads();
      if (tid == 0) S.eng = eidx;
    }
    const DevEngine e = eg;
    const u32* __restrict__ xq = a.xq + it.xq_off;
    const u64 tl = task - a.task_prefix[S.item];
    const u32 lane = (u32)(tl % e.L);
    const u64 chunk = tl / e.L;
    const u64 R = e.lanes[lane];
    const u64 u_start = chunk * (u64)(kSeg * kSegPerTask);
    const u64 u_end = min((u64)it.U, u_start + (u64)(kSeg * kSegPerTask));
    // the lane's shift for every marked prime
    for (u32 i = e.NS + tid; i < e.NPm; i += kBlock) {
      const PrimeRec pr = e.recs[i];
      const u32 rq = fk_bmod(R, pr.q, pr.magic);
      u32 x = xq[i] + rq;
      x = min(x, x - pr.q);
      S.s16[i - e.NS] =
          (unsigned short)fk_mulmod(x, __ldg(e.minv_all + i), pr.q, pr.magic);
    }
    u32 rho[kNS];
    Pat<P0, 0, kNS>::setup(rho, R, u_start + 128ull * tid, xq, S.minv);
    __syncthreads();
    for (u64 useg = u_start; useg < u_end; useg += kSeg) {
      const u32 seg_len = (u32)min((u64)kSeg, u_end - useg);
      // (a) pattern words 2*tid and 2*tid + 1
      {
        u64 acc0 = 0, acc1 = 0;
        Pat<P0, 0, kNS>::word(spat, rho, acc0);
        Pat<P0, 0, kNS>::word(spat, rho, acc1);
        PatSkip<P0, 0, kNS>::template skip<(u32)(kSeg - 128)>(rho);
        S.patw[2 * tid] = acc0;
        S.patw[2 * tid + 1] = acc1;
        nword += 2;
      }
      // zero the byte map
      {
        uint4* b4 = reinterpret_cast<uint4*>(S.bytes);
        const uint4 z = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int k = 0; k < kSeg / 16 / kBlock; ++k) b4[tid + k * kBlock] = z;
      }
      __syncthreads();
      // (b) mark.  Primes below NPw (at least 16 hits per residue and
      // segment) one warp each, the lanes splitting every progression
      // (stride 32q), warps taking primes round robin so the heavy small
      // primes spread over all warps; larger primes one thread each.
      {
        const u32 lane = tid & 31, wid = tid >> 5;
        for (u32 i = e.NS + wid; i < e.NPw; i += kBlock / 32) {
          const PrimeRec pr = e.recs[i];
          const u32 q = pr.q;
          u32 off = fk_bmod(useg, q, pr.magic) + S.s16[i - e.NS];
          off = min(off, off - q);
          const u32 ga = __ldg(e.gaux + i);
          const u32 go = ga & 0x00FFFFFFu, gc = ga >> 24;
          for (u32 c = 0; c < gc; ++c) {
            const u32 g = __ldg(e.glist + go + c);
            const u32 h0 = g >= off ? g - off : g + q - off;
            for (u32 h = h0 + lane * q; h < seg_len; h += 32 * q) {
              S.bytes[h] = 1;
              ++nmark;
            }
          }
        }
      }
      for (u32 i = e.NPw + tid; i < e.NPm; i += kBlock) {
        const PrimeRec pr = e.recs[i];
        const u32 q = pr.q;
        u32 off = fk_bmod(useg, q, pr.magic) + S.s16[i - e.NS];
        off = min(off, off - q);
        const u32 ga = __ldg(e.gaux + i);
        const u32 go = ga & 0x00FFFFFFu, gc = ga >> 24;
        for (u32 c = 0; c < gc; ++c) {
          const u32 g = __ldg(e.glist + go + c);
          u32 h = g >= off ? g - off : g + q - off;
          for (; h < seg_len; h += q) {
            S.bytes[h] = 1;
            ++nmark;
          }
        }
      }
      __syncthreads();
      // (c) extract
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const u32 w = 2 * tid + k;
        const u64 uw = useg + 64ull * w;
        if (uw >= u_end) continue;
        const uint2* bw = reinterpret_cast<const uint2*>(S.bytes + 64 * w);
        u64 m = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const uint2 b = bw[j];
          const u64 x = ((u64)b.y << 32) | b.x;  // bytes are 0 or 1
          m |= ((x * 0x0102040810204080ull) >> 56) << (8 * j);
        }
        const u64 left = u_end - uw;
        u64 valid = left >= 64 ? ~0ull : ((1ull << left) - 1ull);
        if (uw == 0 && R < it.lo_off) valid &= ~1ull;
        if (it.U - uw <= 64 && R >= it.hi_last)
          valid &= ~(1ull << (it.U - uw - 1));
        u64 surv = ~S.patw[w] & ~m & valid;
        while (surv) {
          const int b = __ffsll((long long)surv) - 1;
          surv &= surv - 1;
          const u64 v = (uw + b) * e.M + R;
          bool alive = true;
          if (e.NPm < e.NP) {
            switch (e.kind) {
              case KIND_EULER:
                alive = tail_alive<KIND_EULER>(v, e, xq, S.sbits, ntest); break;
              case KIND_DICKSON:
                alive = tail_alive<KIND_DICKSON>(v, e, xq, S.sbits, ntest); break;
              default:
                alive = tail_alive<KIND_AP>(v, e, xq, S.sbits, ntest); break;
            }
          }
          if (!alive) continue;
          const unsigned long long p = atomicAdd(&a.ctr->ncand, 1ull);
          if (p < a.cand_cap) {
            a.cand_key[p] = v;
            a.cand_item[p] = gitem;
          } else {
            atomicOr(&a.ctr->overflow, 1u);
          }
        }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nmark += __shfl_down_sync(0xffffffffu, nmark, o);
    ntest += __shfl_down_sync(0xffffffffu, ntest, o);
    nword += __shfl_down_sync(0xffffffffu, nword, o);
  }
  if ((tid & 31) == 0) {
    if (nmark) atomicAdd(&a.ctr->marks, (unsigned long long)nmark);
    if (ntest) atomicAdd(&a.ctr->s2_tests, (unsigned long long)ntest);
    if (nword) atomicAdd(&a.ctr->s1_words, (unsigned long long)nword);
  }
}

}  // namespace fk
