// fk_mark.cuh -- the marking sieve for long lanes (stage S1 + marking).
//
// A weak sieve (small n: every prime kills only a few residues) leaves many
// candidates alive deep into the prime list, and testing each of them
// against every remaining prime costs tens of tests per candidate.  Long
// lanes are therefore sieved the Eratosthenes way instead: one CTA owns one
// lane over SEG * seg_per_task consecutive periods, and per segment of SEG
// periods (16384, 32768 or 65536: a template variant chosen per batch) it
//   (a) ORs the NS compile-time pattern primes into SEG / 16384 words per
//       thread (the stage-1a pattern sieve of fk_sieve.cuh),
//   (b) marks every other prime below 2^16 into a SEG-byte shared map.
//       Each (prime, forbidden residue) progression of step q is one or
//       more work entries of at least kMarkHits hits (the large primes:
//       one entry of at most two hits), built once per engine and
//       segment length and ordered by prime; the threads take the entries
//       round robin, so the heavy small primes spread over every warp and
//       a warp's entries share q and trip count.  Marks are plain byte
//       stores (a mark is idempotent: no read-modify-write, no atomic),
//       four per loop trip, and
//   (c) extracts the periods that neither marked, tests any primes beyond
//       the marked range one by one, and appends the survivors to the
//       candidate list.
// Each prime's first hit offset lives in shared memory and steps by the
// tabulated SEG mod q from one segment to the next.
// This is the reference AP engine's bitmap marking (primorial-ap/ap_gpu.py:
// 204-369: tabulated small primes, shared-memory marks for mid primes,
// global atomics for the rest) re-laid out per lane, so no mark needs an
// atomic and every engine kind can use it.
#pragma once
#include "fk_sieve.cuh"

namespace fk {

template <int SEG>
struct MarkSmem {
  unsigned char bytes[SEG];
  unsigned short off16[kMarkPrimes];  // first hit offset of each prime from
                                      // index kNSMin (marked ones are used)
  u32 ph[kNSMax];                     // table index at the segment start
  u32 lsh[kNSMax];                    // the lane's index shift per prime
  u32 warp[kBlock / 32];
  u32 minv[kNSMax];
  u32 sbits[512];
  u64 task;
  u32 item;
  u32 eng;
  u32 status;
  u32 pad;
  unsigned long long mbar;
};

// The WPT pattern words of thread t in a segment (words WPT*t ...
// WPT*t + WPT - 1), from each prime's table index at the segment start in
// shared memory (ph[I]; consecutive words are consecutive entries): no
// per-prime index occupies a register while the segment is marked.
template <int P0, int I, int NS, int WPT>
struct PatSeg {
  static __device__ __forceinline__ void words(const u64* __restrict__ spat,
                                               const u32* ph, u32 tw,
                                               u64* acc) {
    constexpr u32 q = fk_nth_prime(P0 + I);
    constexpr u32 off = fk_pat_prefix(P0, I);
    u32 r = ph[I] + tw % q;
    r = min(r, r - q);
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
      acc[k] |= spat[off + r];
      r += 1;
      r = min(r, r - q);
    }
    PatSeg<P0, I + 1, NS, WPT>::words(spat, ph, tw, acc);
  }
};
template <int P0, int NS, int WPT>
struct PatSeg<P0, NS, NS, WPT> {
  static __device__ __forceinline__ void words(const u64*, const u32*, u32,
                                               u64*) {}
};

template <int KIND>
__device__ __forceinline__ bool tail_alive(u64 v, const DevEngine& e,
                                           const u32* __restrict__ xq,
                                           const u32* s_sbits, u64& ntest) {
  for (u32 i = e.NPm; i < e.NP; ++i) {
    const PrimeRec pr = e.recs[i];
    u32 rr = fk_bmod(v, pr.q, pr.magic) + __ldg(xq + i);
    rr = min(rr, rr - pr.q);
    ++ntest;
    const u64 hm = KIND == KIND_DICKSON ? __ldg(e.hmask + i) : 0ull;
    if (kill_test<KIND>(pr, rr, e.lists, s_sbits, e.xxmax, e.n, hm))
      return false;
  }
  return true;
}

// NS pattern primes, SEG periods per segment; the engine descriptor's NS
// and marking tables (mq, mitems) must be the ones of this variant.
template <int P0, int NS, int SEG>
__global__ void __launch_bounds__(kBlock, 3) k_mark(SieveArgs a) {
  constexpr int WPT = SEG / (64 * kBlock);  // pattern words per thread
  static_assert(WPT * 64 * kBlock == SEG, "segment must be 1-4 words per thread");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  u64* spat = reinterpret_cast<u64*>(smem_raw);
  MarkSmem<SEG>& S =
      *reinterpret_cast<MarkSmem<SEG>*>(smem_raw + pat_bytes<P0, NS>());
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
      if (!stage_patterns<P0, NS>(spat, eg, &S.mbar, &S.status, phase, a.ctr))
        return;
      for (u32 i = tid; i < (u32)NS; i += kBlock) S.minv[i] = eg.pat_minv[i];
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
    const u64 u_start = chunk * (u64)SEG * a.seg_per_task;
    const u64 u_end = min((u64)it.U, u_start + (u64)SEG * a.seg_per_task);
    // marked primes: indices [NS, NPm), off16 / mq slots [pbeg, pend)
    const u32 pbeg = (u32)(NS - kNSMin), pend = e.NPm - kNSMin;
    // the lane's index shift and first-segment table index for every
    // pattern prime: ((u + s_l) * 64^-1) mod q, s_l carrying 64^-1 already
    if (tid < NS) {
      const PrimeRec pr = e.recs[tid];
      u32 x = xq[tid] + fk_bmod(R, pr.q, pr.magic);
      x = min(x, x - pr.q);
      const u32 sh = fk_mulmod(x, S.minv[tid], pr.q, pr.magic);
      S.lsh[tid] = sh;
      u32 p = fk_mulmod(fk_bmod(u_start, pr.q, pr.magic),
                        __ldg(e.pat_i64 + tid), pr.q, pr.magic) + sh;
      S.ph[tid] = min(p, p - pr.q);
    }
    // the first hit offset of every marked prime in the first segment
    for (u32 pi = pbeg + tid; pi < pend; pi += kBlock) {
      const u32 i = kNSMin + pi;
      const PrimeRec pr = e.recs[i];
      u32 x = xq[i] + fk_bmod(R, pr.q, pr.magic);
      x = min(x, x - pr.q);
      const u32 sh = fk_mulmod(x, __ldg(e.minv_all + i), pr.q, pr.magic);
      u32 o = fk_bmod(u_start, pr.q, pr.magic) + sh;
      S.off16[pi] = (unsigned short)min(o, o - pr.q);
    }
    __syncthreads();
    for (u64 useg = u_start; useg < u_end; useg += SEG) {
      const u32 seg_len = (u32)min((u64)SEG, u_end - useg);
      // (a) the pattern words WPT*tid ... WPT*tid + WPT - 1
      // (a thread whose words all lie past the segment's end skips it:
      // a short lane's last segment leaves most threads idle)
      u64 acc[WPT];
#pragma unroll
      for (int k = 0; k < WPT; ++k) acc[k] = 0;
      if (64u * WPT * (u32)tid < seg_len) {
        PatSeg<P0, 0, NS, WPT>::words(spat, S.ph, (u32)(WPT * tid), acc);
        nword += WPT;
      }
      // zero the byte map up to the segment's end
      {
        uint4* b4 = reinterpret_cast<uint4*>(S.bytes);
        const uint4 z = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int k = 0; k < SEG / 16 / kBlock; ++k) {
          const u32 idx = tid + k * kBlock;
          if (16u * idx < seg_len) b4[idx] = z;
        }
      }
      __syncthreads();
      // (b) mark: the work entries round robin over the threads, the next
      // two entries' loads in flight while this one's progression is
      // written (an entry carries its prime and sub-range length: one load
      // each).
      // Entries come ordered by prime, so a warp's 32 consecutive entries
      // share a hit class: from index nm2 on, a residue hits the segment
      // at most twice (q >= SEG / 2), from nm1 on at most once (q >= SEG),
      // and those are written by a fixed predicated sequence instead of
      // the loops
      {
        const u32 nm = e.nmitems, nm2 = e.nm2, nm1 = e.nm1;
        const u64* __restrict__ mit = reinterpret_cast<const u64*>(e.mitems);
        unsigned char* __restrict__ B = S.bytes;
        u32 cnt = 0;
        u32 i = tid;
        // two entries' loads in flight ahead of the one being written: a
        // large prime's entry is a handful of instructions, too few to
        // cover one L2 round trip
        u64 w = i < nm ? __ldg(mit + i) : 0ull;
        u64 w1 = i + kBlock < nm ? __ldg(mit + i + kBlock) : 0ull;
        while (i < nm) {
          const u32 inext = i + kBlock;
          const u64 wn = w1;
          w1 = inext + kBlock < nm ? __ldg(mit + inext + kBlock) : 0ull;
          const u32 wl = (u32)w, wh = (u32)(w >> 32);
          const u32 g = wl & 0xFFFFu, pi = (wl >> 16) & 0x1FFFu;
          const u32 q = wh & 0xFFFFu;
          const u32 off = S.off16[pi];
          const u32 d = g - off;
          u32 h = min(d, d + q);   // (g - off) mod q: the first hit
          if (i >= nm2) {
            // whole-segment entries of large primes: h < q, so h + q is
            // the last possible hit (h + 2q >= 2q >= SEG)
            if (h < seg_len) { B[h] = 1; ++cnt; }
            if (i < nm1) {
              h += q;
              if (h < seg_len) { B[h] = 1; ++cnt; }
            }
          } else {
            const u32 k = wl >> 29, sl = wh >> 16;
            h += k * sl;
            const u32 end = sl ? min(seg_len, (k + 1) * sl) : seg_len;
            const u32 q2 = 2 * q, q3 = 3 * q, q4 = 4 * q;
            for (; h + q3 < end; h += q4, cnt += 4) {
              B[h] = 1;
              B[h + q] = 1;
              B[h + q2] = 1;
              B[h + q3] = 1;
            }
            for (; h < end; h += q, ++cnt) B[h] = 1;
          }
          i = inext;
          w = wn;
        }
        nmark += cnt;
      }
      __syncthreads();
      // advance the offsets and phases to the next segment (nothing below
      // reads them before the next segment's barrier)
      if (useg + SEG < u_end) {
        for (u32 pi = pbeg + tid; pi < pend; pi += kBlock) {
          const u64 m = __ldg(reinterpret_cast<const u64*>(e.mq) + pi);
          const u32 q = (u32)m & 0xFFFFu;
          const u32 o = S.off16[pi] + (((u32)m >> 16) & 0xFFFFu);
          S.off16[pi] = (unsigned short)min(o, o - q);
        }
        if (tid < NS) {
          const PrimeRec pr = e.recs[tid];
          const u32 p = S.ph[tid] + (u32)(SEG / 64) % pr.q;
          S.ph[tid] = min(p, p - pr.q);
        }
      }
      // (c) extract
#pragma unroll
      for (int k = 0; k < WPT; ++k) {
        const u32 w = WPT * tid + k;
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
        u64 surv = ~acc[k] & ~m & valid;
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
