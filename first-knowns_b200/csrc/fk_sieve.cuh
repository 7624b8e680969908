// fk_sieve.cuh -- the fused sieve kernel (stages S1 and S2).
//
// The line of one item is x = X0 + u*M + R[l]: period u in [0, U), lane l
// over the wheel's admissible residues R mod M.  A CHAIN is one lane over
// Tc 64-period words per thread: either one thread per lane on Tc
// consecutive words, or -- for long lanes -- one warp per lane, thread t
// on words t, t + 32, ... (so a warp's pattern loads are 32 consecutive
// table entries).  A CTA runs 256 threads' chains (a TASK), and a
// persistent grid pulls tasks from a device counter, so thousands of
// items of uneven length run in one launch.  Inside a task the warps claim
// blocks of 32 threads' chains (warp tasks) from a shared counter.
//
// S1 (pattern sieve).  For the NS pattern primes starting at prime index
// P0 (NS = 24, 32 or 40: a template variant chosen per batch) --
// compile-time constants, so each prime's modulus, word step and
// table offset are immediates -- the kill pattern of 64 consecutive
// periods of a lane is one 64-bit word of a per-prime table of q words,
// indexed by the lane's rotating phase rho (u + s_l) mod q.  The tables
// sit in shared memory, staged from HBM by a bulk async copy (TMA).  This
// is the reference's stage-1a bit-sieve (euler-prime-runs/euler_gpu.py:
// 438-520, dickson-ladders/ladder_gpu.py:254-317, and the AP register
// gather primorial-ap/ap_gpu.py:204-313), re-indexed so that one table per
// prime serves every lane of every wheel.
//
// S2 (compaction rounds).  S1 survivors go to a per-WARP shared-memory
// queue (ballot/prefix compaction inside the warp, so the word loop has no
// block-wide barrier).  When it fills, the warp drains it through rounds
// over the remaining primes: every live candidate is tested against a
// round's primes (Barrett residue plus the engine's kill test), then the
// survivors are compacted with ballots so the next round starts with every
// lane busy; a short queue instead goes one candidate per warp, the lanes
// splitting the primes -- the reference's stage 1b / stage 2 rounds
// (euler-prime-runs/euler_gpu.py:523-709, dickson-ladders/ladder_gpu.py:
// 349-407) without a host-visible queue.  Final survivors are appended to
// a global candidate list with warp-aggregated atomics.
#pragma once
#include "fk_arith.cuh"
#include "fk_types.h"

namespace fk {

constexpr u32 kWaitSpins = 1u << 20;
constexpr int kRoundUnroll = 2;  // primes per trip of the compaction rounds

__device__ __forceinline__ u32 smem_u32(const void* p) {
  return (u32)__cvta_generic_to_shared(p);
}

// Block-wide exclusive scan of one u32 per thread; returns the prefix and
// sets *total.  Two barriers.
__device__ __forceinline__ u32 block_scan(u32 v, u32* s_warp, u32* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  u32 x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    u32 y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  u32 base = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < kBlock / 32; ++w) {
    u32 t = s_warp[w];
    base += (w < wid) ? t : 0;
    tot += t;
  }
  __syncthreads();
  *total = tot;
  return base + x - v;
}

// ---- per-candidate kill tests ------------------------------------------
// aux bit 31 set: explicit list, offset in bits 0..23, count in 24..30.
__device__ __forceinline__ bool list_kill(u32 aux, u32 r,
                                          const u32* __restrict__ lists) {
  const u32 off = aux & 0x00FFFFFFu, cnt = (aux >> 24) & 0x7Fu;
  bool k = false;
  for (u32 c = 0; c < cnt; ++c) k |= (__ldg(lists + off + c) == r);
  return k;
}

template <int KIND>
__device__ __forceinline__ bool kill_test(const PrimeRec& pr, u32 r,
                                          const u32* __restrict__ lists,
                                          const u32* s_sbits, u32 xxmax,
                                          u32 n, u64 hm) {
  if (KIND == KIND_DICKSON) {
    // the forbidden residues come in pairs r, q - r: h = min(r, q - r)
    // must be on the half list, which a 64-bit filter of h mod 64
    // screens first
    const u32 h = min(r, pr.q - r);
    if (!((hm >> (h & 63)) & 1ull)) return false;
    return list_kill(pr.aux, h, lists);
  }
  if (pr.aux & 0x80000000u) return list_kill(pr.aux, r, lists);
  if (KIND == KIND_EULER) {
    // q > max(x^2+x): r is killed iff q - r (mod q) is one of the x^2+x.
    if (r == 0) return true;
    const u32 t = pr.q - r;
    return t <= xxmax && ((s_sbits[t >> 5] >> (t & 31)) & 1u);
  } else if (KIND == KIND_AP) {
    // killed iff r + j*d == 0 (mod q) for some j < n, i.e.
    // j = (q - r) * d^-1 mod q is below n; aux = d^-1 (0 when q | d).
    if (r == 0) return true;
    if (pr.aux == 0) return false;
    // for q < 2^16 the product (q - r) * d^-1 < q^2 fits 32 bits: a
    // 32-bit Barrett with floor(2^32 / q); deeper primes take 64 bits
    u32 t;
    if (pr.q < 65536u) {
      const u32 x = (pr.q - r) * pr.aux;
      t = x - __umulhi(x, (u32)(pr.magic >> 32)) * pr.q;
      t = min(t, t - pr.q);
    } else {
      t = fk_mulmod(pr.q - r, pr.aux, pr.q, pr.magic);
    }
    return t < n;
  }
  return false;  // Dickson primes always carry a list
}

// ---- S1 helpers, unrolled over the compile-time pattern primes ----------
// k[I] is the lane's current TABLE INDEX for pattern prime I (entry k =
// phase 64k mod q), so one word forward is k + 1 and STRIDE words forward
// is k + STRIDE (mod q).
template <int P0, int I, int NS>
struct Pat {
  // Two words of the chain, STRIDE words apart, each OR-ed into two
  // accumulators by prime parity, so the loads and ORs of one prime do not
  // wait on the previous prime's; the index then moves 2 * STRIDE words.
  template <u32 STRIDE>
  static __device__ __forceinline__ void word2(const u64* __restrict__ spat,
                                               u32* k, u64* acc) {
    constexpr u32 q = fk_nth_prime(P0 + I);
    constexpr u32 off = fk_pat_prefix(P0, I);
    constexpr u32 st = STRIDE % q;
    const u32 r0 = k[I];
    u32 r1 = r0 + st;
    r1 = min(r1, r1 - q);  // unsigned: r1 - q wraps when r1 < q
    u32 r2 = r1 + st;
    r2 = min(r2, r2 - q);
    acc[I & 1] |= spat[off + r0];
    acc[2 + (I & 1)] |= spat[off + r1];
    k[I] = r2;
    Pat<P0, I + 1, NS>::template word2<STRIDE>(spat, k, acc);
  }
  // The table index of period u0 of lane R: phase (u0 + s_l) mod q with
  // s_l = (X0 + R) * (M mod q)^-1, times 64^-1 (s_minv already carries it).
  static __device__ __forceinline__ void setup(u32* k, u64 R, u64 u0,
                                               const u32* __restrict__ xq,
                                               const u32* s_minv) {
    constexpr u32 q = fk_nth_prime(P0 + I);
    constexpr u32 i64 = fk_inv64(q);
    const u32 rq = (u32)(R % q);
    const u32 s = (u32)(((xq[I] + rq) % q) * (u64)s_minv[I] % q);
    k[I] = (u32)(((u32)(u0 % q) * i64 + s) % q);
    Pat<P0, I + 1, NS>::setup(k, R, u0, xq, s_minv);
  }
  // The table indexes of a group of GW threads sweeping one lane, thread
  // t of the group from word base + t: (base_I + t) mod q, base_I held in
  // v[I / GW] by thread I mod GW of the group.
  template <int GW>
  static __device__ __forceinline__ void spread(u32* k, const u32* v,
                                                u32 t) {
    constexpr u32 q = fk_nth_prime(P0 + I);
    const u32 b = __shfl_sync(0xffffffffu, v[I / GW], I % GW, GW);
    // t < GW: below q for every prime when GW = 8 and from the 37 up when
    // GW = 32; the 17 ... 31 of the 13# and 17# families reduce it first,
    // so one subtraction still ends in [0, q)
    const u32 r = b + (q >= (u32)GW ? t : t % q);
    k[I] = min(r, r - q);
    Pat<P0, I + 1, NS>::template spread<GW>(k, v, t);
  }
};
template <int P0, int NS>
struct Pat<P0, NS, NS> {
  template <u32 STRIDE>
  static __device__ __forceinline__ void word2(const u64*, u32*, u64*) {}
  static __device__ __forceinline__ void setup(u32*, u64, u64, const u32*,
                                               const u32*) {}
  template <int GW>
  static __device__ __forceinline__ void spread(u32*, const u32*, u32) {}
};

// Pattern prime I's table index at word wb of lane R: (wb + s) mod q with
// s = (X0 + R) * (M mod q)^-1 * 64^-1 mod q the lane's phase (xq holds X0
// mod q, s_minv the product of the two inverses), from the prime's record.
__device__ __forceinline__ u32 lane_base(const DevEngine& e,
                                         const u32* __restrict__ xq,
                                         const u32* s_minv, u64 R, u64 wb,
                                         u32 I) {
  const PrimeRec pr = e.recs[I];
  u32 x = xq[I] + fk_bmod(R, pr.q, pr.magic);
  x = min(x, x - pr.q);
  const u32 s = fk_mulmod(x, s_minv[I], pr.q, pr.magic);
  const u32 t = s + fk_bmod(wb, pr.q, pr.magic);
  return min(t, t - pr.q);
}

// The table indexes of a group of GW threads sweeping one lane from word
// wb, thread t at word wb + t: thread t computes the base index of the
// pattern primes t, t + GW, ... and the group shares them by shuffle.
template <int P0, int NS, int GW>
__device__ __forceinline__ void shared_setup(u32* rho, const DevEngine& e,
                                             const u32* __restrict__ xq,
                                             const u32* s_minv, u64 R,
                                             u64 wb, u32 t) {
  constexpr int K = (NS + GW - 1) / GW;
  u32 v[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const u32 I = t + (u32)(j * GW);
    v[j] = I < (u32)NS ? lane_base(e, xq, s_minv, R, wb, I) : 0u;
  }
  Pat<P0, 0, NS>::template spread<GW>(rho, v, t);
}

struct SieveArgs {
  const DevEngine* engines;
  const DevItem* items;
  const u64* task_prefix;  // [nitems + 1] for this kernel's items
  const u32* item_index;   // [nitems] global item index of each entry
  u32 nitems;
  u32 pad;
  u64 ntask;
  const u32* xq;
  u64* cand_key;
  u32* cand_item;
  u64 cand_cap;
  DevCounters* ctr;
  unsigned long long* task_ctr;
  u32 warp_queue;     // compaction: warp queues below this go one
                      // candidate per warp
  u32 seg_per_task;   // marking: segments per task
  u32 warp_tasks;     // pattern sieve: warp tasks per CTA task (8, 16 or
                      // 32); a warp task is one warp's 32 threads' chains
  u32 pad2;
};

// The entry of the item holding task t: the last i with task_prefix[i] <=
// t, searched forward from `from` (a CTA's claims only grow, so its next
// task's item is at or after its last one): a few steps, then bisection.
__device__ __forceinline__ u32 task_item(const SieveArgs& a, u64 t, u32 from) {
  u32 lo = from;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (lo + 1 < a.nitems && a.task_prefix[lo + 1] <= t) ++lo;
    else return lo;
  }
  u32 hi = a.nitems;
  while (hi - lo > 1) {
    const u32 mid = (lo + hi) >> 1;
    if (a.task_prefix[mid] <= t) lo = mid; else hi = mid;
  }
  return lo;
}

// Per-warp candidate queues: kQcap / 8 entries per warp, two buffers.
constexpr u32 kWq = kQcap / (kBlock / 32);

struct SieveSmem {
  u32 qa[kQcap];
  u32 qb[kQcap];
  u64 chain_R[kBlock];
  u64 chain_w0[kBlock];   // the thread's first word; word j is w0 + j*stride
  u32 stride;             // 1, or 32 when a warp sweeps one lane
  u32 wnext;              // the CTA task's next warp task
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

// Shared bytes of the first NS pattern primes' tables (the prefix a kernel
// variant stages), padded to 16 bytes.
template <int P0, int NS = kNS>
__host__ __device__ constexpr u32 pat_bytes() {
  return ((fk_pat_prefix(P0, NS) + 1) / 2) * 16;
}

// A queued candidate: the chain (thread of the CTA), the word within the
// chain and the bit within the word.
__device__ __forceinline__ u64 cand_value(const SieveSmem& S, u32 code,
                                          u64 M) {
  const u32 t = code >> 22;
  const u64 u = 64ull * (S.chain_w0[t] +
                         (u64)((code >> 6) & 0xFFFFu) * S.stride) +
                (code & 63u);
  return u * M + S.chain_R[t];
}

__device__ __forceinline__ void emit_cand(const SieveArgs& a, u64 v,
                                          u32 gitem, u64 p) {
  if (p < a.cand_cap) {
    a.cand_key[p] = v;
    a.cand_item[p] = gitem;
  } else {
    atomicOr(&a.ctr->overflow, 1u);
  }
}

// Drain one warp's queue (n candidates in qin; qout is the second buffer):
// rounds over the per-candidate primes with ballot compaction, a short
// queue one candidate per warp over every remaining prime, then the
// survivors appended to the global list.  Warp-synchronous: every lane of
// the warp calls it with the same n.
template <int KIND>
__device__ void warp_drain(u32* qin, u32* qout, u32 n, const SieveSmem& S,
                           const DevEngine& e, const DevItem& it, u32 gitem,
                           const SieveArgs& a, u32 wq_short, u32& ntest) {
  const u32 lane = threadIdx.x & 31;
  const u32 lt = (1u << lane) - 1u;
  const u32* __restrict__ xq = a.xq + it.xq_off;
  const u64 M = e.M;
  for (u32 r = 0; r < e.nrounds && n > 0; ++r) {
    const u32 i0 = __ldg(e.rounds + r), i1 = __ldg(e.rounds + r + 1);
    if (n < wq_short) {
      // one candidate per warp, the lanes splitting the primes 32 at a
      // time and voting after each group (the reference's warp-per-
      // candidate deep rounds, dickson-ladders/ladder_gpu.py:378-407)
      for (u32 idx = 0; idx < n; ++idx) {
        const u64 v = cand_value(S, qin[idx], M);
        bool dead = false;
        for (u32 b = i0; b < e.NP && !dead; b += 32) {
          const u32 i = b + lane;
          bool kill = false;
          if (i < e.NP) {
            const PrimeRec pr = e.recs[i];
            u32 rr = fk_bmod(v, pr.q, pr.magic) + __ldg(xq + i);
            rr = min(rr, rr - pr.q);
            const u64 hm = KIND == KIND_DICKSON ? __ldg(e.hmask + i) : 0ull;
            kill = kill_test<KIND>(pr, rr, e.lists, S.sbits, e.xxmax, e.n, hm);
            ++ntest;
          }
          dead = __any_sync(0xffffffffu, kill);
        }
        if (!dead && lane == 0)
          emit_cand(a, v, gitem, atomicAdd(&a.ctr->ncand, 1ull));
      }
      __syncwarp();
      return;
    }
    u32 out = 0;
    for (u32 base = 0; base < n; base += 32) {
      const u32 idx = base + lane;
      bool alive = false;
      u32 code = 0;
      if (idx < n) {
        code = qin[idx];
        const u64 v = cand_value(S, code, M);
        alive = true;
        u32 i = i0;
        // kRoundUnroll primes per trip, every load issued before any test
        // (a kill ends the round; tests past it in the trip are not counted)
        for (; i + kRoundUnroll <= i1; i += kRoundUnroll) {
          PrimeRec pr[kRoundUnroll];
          u32 xo[kRoundUnroll];
          u64 hm[kRoundUnroll];
#pragma unroll
          for (int k = 0; k < kRoundUnroll; ++k) {
            pr[k] = e.recs[i + k];
            xo[k] = __ldg(xq + i + k);
            hm[k] = KIND == KIND_DICKSON ? __ldg(e.hmask + i + k) : 0ull;
          }
          u32 kill = 0;
#pragma unroll
          for (int k = 0; k < kRoundUnroll; ++k) {
            u32 rr = fk_bmod(v, pr[k].q, pr[k].magic) + xo[k];
            rr = min(rr, rr - pr[k].q);
            if (kill_test<KIND>(pr[k], rr, e.lists, S.sbits, e.xxmax, e.n,
                                hm[k]))
              kill |= 1u << k;
          }
          if (kill) {
            i += __ffs((int)kill) - 1;
            alive = false;
            break;
          }
        }
        for (; alive && i < i1; ++i) {
          const PrimeRec pr = e.recs[i];
          u32 rr = fk_bmod(v, pr.q, pr.magic) + __ldg(xq + i);
          rr = min(rr, rr - pr.q);
          const u64 hm = KIND == KIND_DICKSON ? __ldg(e.hmask + i) : 0ull;
          if (kill_test<KIND>(pr, rr, e.lists, S.sbits, e.xxmax, e.n, hm)) {
            alive = false;
            break;
          }
        }
        ntest += (i - i0) + (alive ? 0 : 1);
      }
      const u32 bal = __ballot_sync(0xffffffffu, alive);
      if (alive) qout[out + __popc(bal & lt)] = code;
      out += __popc(bal);
    }
    __syncwarp();
    u32* t = qin;
    qin = qout;
    qout = t;
    n = out;
  }
  // emit survivors: one atomic per warp
  if (n) {
    u64 base = 0;
    if (lane == 0) base = atomicAdd(&a.ctr->ncand, (unsigned long long)n);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (u32 idx = lane; idx < n; idx += 32)
      emit_cand(a, cand_value(S, qin[idx], M), gitem, base + idx);
  }
  __syncwarp();
}

__device__ __forceinline__ void drain_any(u32* qin, u32* qout, u32 n,
                                          const SieveSmem& S,
                                          const DevEngine& e,
                                          const DevItem& it, u32 gitem,
                                          const SieveArgs& a, u32 wq_short,
                                          u32& ntest) {
  switch (e.kind) {
    case KIND_EULER:
      warp_drain<KIND_EULER>(qin, qout, n, S, e, it, gitem, a, wq_short, ntest);
      break;
    case KIND_DICKSON:
      warp_drain<KIND_DICKSON>(qin, qout, n, S, e, it, gitem, a, wq_short, ntest);
      break;
    default:
      warp_drain<KIND_AP>(qin, qout, n, S, e, it, gitem, a, wq_short, ntest);
      break;
  }
}

// Polls the CTA's mbarrier for the given phase, at most `spins` times.
__device__ __forceinline__ bool mbar_wait(u32 mb, u32 phase, u32 spins) {
  u32 done = 0;
  for (u32 i = 0; i < spins && !done; ++i)
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, "
        "[%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(mb), "r"(phase)
        : "memory");
  return done != 0;
}

// Stage the first NS primes' pattern tables of an engine (a prefix of its
// table) into shared memory with one bulk async
// copy (TMA) completing on the CTA's mbarrier, waiting a bounded number of
// polls.  On a timeout it flags the counters (the host reports
// FK_ERR_TIMEOUT) and returns false, after a second bounded wait for the
// copy to land: the CTA then exits, and a copy still writing into the
// shared memory of an exited CTA is what the second wait avoids.  Every
// thread of the CTA calls it.
template <int P0, int NS>
__device__ __forceinline__ bool stage_patterns(u64* spat, const DevEngine& eg,
                                               unsigned long long* mbar,
                                               u32* status, u32& phase,
                                               DevCounters* ctr) {
  __syncthreads();
  if (threadIdx.x == 0) {
    *status = 0;
    const u32 mb = smem_u32(mbar);
    const u32 bytes = pat_bytes<P0, NS>();
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
    if (!mbar_wait(mb, phase, kWaitSpins)) {
      *status = 1;
      atomicOr(&ctr->overflow, 4u);
      mbar_wait(mb, phase, kWaitSpins);  // let the copy in flight land
    }
  }
  phase ^= 1u;
  __syncthreads();
  return *status == 0;
}

// One block of 32 threads' chains (a warp task): thread wl of the warp
// sweeps chain gw + (wl >> gsh) of the item, pushes its pattern survivors
// into the warp's queue and drains it through the compaction rounds; the
// queue is empty again on return.
template <int P0, int NS>
__device__ __forceinline__ void sieve_block(
    const u64* __restrict__ spat, SieveSmem& S, const SieveArgs& a,
    const DevEngine& e, const DevItem& it, u32 gitem, u64 gw, u64 nchain,
    u32 G, u32 gsh, u32 wq_short, u64 wfull, u32& ntest, u32& nword) {
  const int tid = threadIdx.x;
  const u32 wl = tid & 31, wid = tid >> 5;
  const u64 U = it.U;
  const u32 stride = G;
  u32* wq = S.qa + wid * kWq;
  u32* wq2 = S.qb + wid * kWq;
  // ---- this thread's chain -----------------------------------------
  const u64 g = gw + (wl >> gsh);
  const bool active = g < nchain;
  const u64 chunk = active ? g / e.L : 0;
  const u32 lane = active ? (u32)(g % e.L) : 0;
  const u64 R = active ? e.lanes[lane] : 0;
  const u64 w0 = chunk * (u64)G * it.Tc + (wl & (G - 1));
  S.chain_R[tid] = R;
  S.chain_w0[tid] = w0;
  u32 rho[NS];
  if (G == 32) {
    // the whole warp sweeps one lane: thread I works out prime I's base
    // index once and the warp shares it (instead of every thread
    // computing all NS of them)
    shared_setup<P0, NS, 32>(rho, e, a.xq + it.xq_off, S.minv, R,
                             chunk * 32ull * it.Tc, wl);
  } else if (G == 8) {
    // the same within each group of eight threads sweeping one lane
    shared_setup<P0, NS, 8>(rho, e, a.xq + it.xq_off, S.minv, R,
                            chunk * 8ull * it.Tc, wl & 7u);
  } else {
    Pat<P0, 0, NS>::setup(rho, R, 64ull * w0, a.xq + it.xq_off, S.minv);
  }
  u32 qn = 0;
  if (active) {
    // the chain's words in range: j < Tc with w0 + j*stride < ceil(U/64)
    const u64 wend = (U + 63) >> 6;
    if (w0 < wend)
      nword += (u32)min((u64)it.Tc, (wend - w0 + stride - 1) / stride);
  }
  __syncwarp();
  for (u32 wi = 0; wi < it.Tc; wi += 2) {
    // two words of the chain: j = wi and wi + 1
    u64 sv[2] = {0, 0};
    if (active) {
      u64 acc[4] = {0, 0, 0, 0};
      if (G == 32)
        Pat<P0, 0, NS>::template word2<32>(spat, rho, acc);
      else if (G == 8)
        Pat<P0, 0, NS>::template word2<8>(spat, rho, acc);
      else
        Pat<P0, 0, NS>::template word2<1>(spat, rho, acc);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const u64 w = w0 + (u64)(wi + k) * stride;
        const u64 s = ~(acc[k * 2] | acc[k * 2 + 1]);
        if (w != 0 && w < wfull && wi + k < it.Tc) {
          sv[k] = s;  // an interior word: every period is in range
          continue;
        }
        if (wi + k >= it.Tc || 64ull * w >= U) continue;
        const u64 left = U - 64ull * w;
        u64 valid = left >= 64 ? ~0ull : ((1ull << left) - 1ull);
        if (w == 0 && R < it.lo_off) valid &= ~1ull;
        if (left <= 64 && R >= it.hi_last) valid &= ~(1ull << (left - 1));
        sv[k] = s & valid;
      }
    }
    // push the survivors into the warp's queue; drain first when they
    // do not fit, and when one step alone overfills an empty queue
    // push the prefix that fits and drain again (every pass pushes or
    // drains, so it ends)
    for (;;) {
      const u32 c = __popcll(sv[0]) + __popcll(sv[1]);
      const u32 tot = __reduce_add_sync(0xffffffffu, c);
      if (tot == 0) break;
      if (qn + tot > kWq && qn > 0) {
        drain_any(wq, wq2, qn, S, e, it, gitem, a, wq_short, ntest);
        qn = 0;
        continue;
      }
      // exclusive prefix of c over the warp
      u32 x = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (wl >= (u32)o) x += y;
      }
      u32 pos = qn + x - c;
      const u32 end = min(qn + tot, (u32)kWq);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        while (sv[k] && pos < end) {
          const int b = __ffsll((long long)sv[k]) - 1;
          sv[k] &= sv[k] - 1;
          wq[pos++] = ((u32)tid << 22) | ((wi + k) << 6) | (u32)b;
        }
      }
      __syncwarp();
      if (qn + tot <= (u32)kWq) {
        qn += tot;
        break;
      }
      drain_any(wq, wq2, kWq, S, e, it, gitem, a, wq_short, ntest);
      qn = 0;
    }
  }
  // every queued code refers to this warp task's chains: drain them
  // before the warp's threads take the next task's chains
  drain_any(wq, wq2, qn, S, e, it, gitem, a, wq_short, ntest);
}

// NS: the pattern primes this variant stages (the engine descriptor's NS
// and round cuts must match it).  DYN: the CTA's warps claim blocks of
// chains from a shared counter (a.warp_tasks blocks per task); without it
// each warp takes exactly its own block (a.warp_tasks = 8), which holds
// fewer registers across the word loop.
template <int P0, int NS, bool DYN>
__global__ void __launch_bounds__(kBlock, 3) k_sieve(SieveArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  u64* spat = reinterpret_cast<u64*>(smem_raw);
  SieveSmem& S = *reinterpret_cast<SieveSmem*>(smem_raw + pat_bytes<P0, NS>());
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

  for (;;) {
    if (tid == 0) {
      const u64 t = atomicAdd(a.task_ctr, 1ull);
      S.task = t;
      S.wnext = 0;
      if (t < a.ntask) {
        // binary search: last entry with task_prefix[i] <= t
        u32 lo = 0, hi = a.nitems;
        while (hi - lo > 1) {
          const u32 mid = (lo + hi) >> 1;
          if (a.task_prefix[mid] <= t) lo = mid; else hi = mid;
        }
        S.item = lo;
        S.stride = a.items[a.item_index[lo]].lane_threads;
      }
    }
    __syncthreads();
    const u64 task = S.task;
    if (task >= a.ntask) break;
    const u32 gitem = a.item_index[S.item];
    const DevItem it = a.items[gitem];
    const u32 eidx = it.engine;
    const DevEngine& eg = a.engines[eidx];
    // ---- engine switch: stage its pattern table into shared memory ----
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
    // ---- warp tasks ------------------------------------------------------
    // A CTA task is a.warp_tasks blocks of 32 threads' chains; each warp
    // claims blocks from the CTA's counter until none is left, so a warp
    // held up by a long queue drain takes fewer of them and the barrier
    // that ends the CTA task comes once per a.warp_tasks blocks.
    // G = lane_threads threads sweep one lane: thread t of the group takes
    // words t, t + G, ... of a G * Tc word block, so a group's pattern
    // loads are G consecutive table entries (G = 1: one lane per thread,
    // Tc consecutive words; 8: four lanes per warp; 32: one per warp)
    const u32 G = it.lane_threads;
    const u32 gsh = G == 32 ? 5u : (G == 8 ? 3u : 0u);
    const u32 wl = tid & 31, wid = tid >> 5;
    const u64 nchain = it.nchunk * e.L;
    const u64 wt0 = (task - a.task_prefix[S.item]) * (u64)a.warp_tasks;
    const u32 cpw = 32u >> gsh;  // chains per warp task
    const u32 wq_short = a.warp_queue;
    // words below wfull end before the item's last period, so only the
    // first word (lo_off) and the last (hi_last, U) need a validity mask
    const u64 wfull = it.U ? (it.U - 1) >> 6 : 0;
    u32 ntest = 0, nword = 0;  // this CTA task's counts
    if (DYN) {
      for (;;) {
        u32 wt = 0;
        if (wl == 0) wt = atomicAdd(&S.wnext, 1u);
        wt = __shfl_sync(0xffffffffu, wt, 0);
        if (wt >= a.warp_tasks) break;
        const u64 gw = (wt0 + wt) * cpw;     // the warp task's first chain
        if (gw >= nchain) break;             // and every later one's too
        sieve_block<P0, NS>(spat, S, a, e, it, gitem, gw, nchain, G, gsh,
                            wq_short, wfull, ntest, nword);
      }
    } else {
      // this warp's own block (a block past the item's chains runs with
      // every thread inactive and emits nothing)
      sieve_block<P0, NS>(spat, S, a, e, it, gitem, (wt0 + wid) * cpw,
                          nchain, G, gsh, wq_short, wfull, ntest, nword);
    }
    u64 nt = ntest, nw = nword;  // warp sums in 64 bits
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      nt += __shfl_down_sync(0xffffffffu, nt, o);
      nw += __shfl_down_sync(0xffffffffu, nw, o);
    }
    if (wl == 0) {
      if (nt) atomicAdd(&a.ctr->s2_tests, (unsigned long long)nt);
      if (nw) atomicAdd(&a.ctr->s1_words, (unsigned long long)nw);
    }
    __syncthreads();
  }
}

}  // namespace fk
