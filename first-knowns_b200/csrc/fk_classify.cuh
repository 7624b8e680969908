// fk_classify.cuh -- base residues, chain classification and ordering.
//
// k_xq        X0 mod q for every (item, sieve prime): the per-launch
//             "(k_base mod q)" tables of the reference
//             (euler-prime-runs/euler_gpu.py:1474-1477,
//             primorial-ap/ap_gpu.py:586-593), computed on the device from
//             the 128-bit base.
// k_dense     fills the candidate list with every x of a DENSE item (the
//             launchers' low passes below the engine floors).
// k_classify  the on-device SPRP stage: each candidate's chain depth by
//             the reference's definition for its engine (Euler
//             mr_run_length, Dickson run_length / sprp_run, AP two-pass
//             chain_depth), kept when it reaches the item's threshold.
// k_scan / k_scatter / k_sort_seg
//             order the kept entries per item ascending in x without a
//             host sort: counting scatter by item, then a bitonic sort of
//             each item's segment.
#pragma once
#include "fk_sprp.cuh"
#include "fk_types.h"

namespace fk {

struct ClassArgs {
  const DevEngine* engines;
  const DevItem* items;
  const u32* nitems_p;      // device scalar
  const u32* xq_items;      // unused here
  const u64* cand_key;
  const u32* cand_item;
  u64 cand_cap;
  DevCounters* ctr;
  OutRec* out;
  u64 out_cap;
  u32* item_count;
};

__device__ __forceinline__ void emit_out(const ClassArgs& a, u32 item,
                                         u64 packed) {
  const unsigned long long p = atomicAdd(&a.ctr->nout, 1ull);
  if (p < a.out_cap) {
    a.out[p].packed = packed;
    a.out[p].item = item;
    atomicAdd(a.item_count + item, 1u);
  } else {
    atomicOr(&a.ctr->overflow, 2u);
  }
}

// The values of one candidate's chain (Euler x^2 + x + p for x = t, Dickson
// (t + 1) * k^2 + 1, AP p + t * d).
struct Chain {
  u32 kind;
  u128 x;   // Euler / AP: p
  V3 kk;    // Dickson: k^2
  V3 d;     // AP: difference
};

__device__ __forceinline__ V3 chain_value(const Chain& c, u32 t) {
  if (c.kind == KIND_EULER) return v3_from_u128(c.x + (u128)((u64)t * t + t));
  if (c.kind == KIND_DICKSON) {
    V3 v = v3_mul_u64(c.kk, (u64)(t + 1));
    const V3 one = {{1, 0, 0}};
    return v3_add(v, one);
  }
  return v3_add(v3_from_u128(c.x), v3_mul_u64(c.d, (u64)t));
}

// First t < lim whose value fails sprp_base2 (lim when none does): an
// upper bound on every engine's depth, because mr_is_prime implies
// sprp_base2 (huntlib/primes.py:38-46 tests base 2 first).
__device__ u32 chain_base2(const Chain& c, u32 lim, u64* imad, u64* nval) {
  u32 t = 0;
  while (t < lim) {
    ++*nval;
    if (!sprp(chain_value(c, t), true, imad)) break;
    ++t;
  }
  return t;
}

// Every value below d2 passed base 2; the exact mr_is_prime chain ends at
// the first of them that fails one of the other six bases.
__device__ u32 chain_exact(const Chain& c, u32 d2, u64* imad, u64* nval) {
  u32 t = 0;
  while (t < d2) {
    ++*nval;
    if (!sprp_rest(chain_value(c, t), imad)) break;
    ++t;
  }
  return t;
}

// Depth by the reference's definition for the engine, or -1 when the
// base-2 bound already proves it below the threshold:
//   Euler    mr_run_length (euler_search.py:258-262), searched to
//            max(threshold, cap); hunt keeps f >= threshold, reports
//            min(f, cap); the dense low pass keeps min(f, cap) >= thr
//   Dickson  run_length (ladder_search.py:143-148), or the launcher's
//            two-pass sprp_run (dickson-ladders/launch.py:310-343)
//   AP       two-pass chain_depth (ap_search.py:160-194)
__device__ int chain_depth_thr(const Chain& c, u32 mode, u32 thr, u32 cap,
                               bool two_pass, u64* imad, u64* nval) {
  if (c.kind == KIND_EULER) {
    const u32 lim = max(thr, cap);
    const u32 d2 = chain_base2(c, lim, imad, nval);
    const bool dense = mode == MODE_DENSE;
    if ((dense ? min(d2, cap) : d2) < thr) return -1;
    const u32 f = chain_exact(c, d2, imad, nval);
    const u32 depth = min(f, cap);
    return ((dense ? depth : f) >= thr) ? (int)depth : -1;
  }
  const u32 d2 = chain_base2(c, cap, imad, nval);
  const u32 pass = (c.kind == KIND_AP) ? 6u : (two_pass ? 5u : 0u);
  u32 depth;
  if (d2 < pass) {
    depth = d2;
  } else {
    if (d2 < thr) return -1;
    depth = chain_exact(c, d2, imad, nval);
  }
  return depth >= thr ? (int)depth : -1;
}

// The SPRP stage as a step interpreter.  Each lane holds the state of one
// candidate's chain and performs exactly ONE strong test per step -- one
// value, one base -- then advances its own state machine:
//   phase 0  base-2 chain: test value t to base 2; pass -> t + 1 (until the
//            limit), fail -> d2 = t, the base-2 depth, an upper bound on
//            every engine's depth (mr_is_prime implies sprp_base2)
//   decide   by the engine's rules (chain_depth_thr): drop the candidate
//            when d2 already proves it below the threshold, report d2 for
//            the two-pass engines below their exact-from depth, else
//   phase 1  the exact chain: values t < d2 tested to the six other bases,
//            one base per step; the first failure ends the chain
// A lane whose candidate is finished takes the next one at once from a
// chunk its warp fetched, so a warp never waits for its longest chain, and
// lanes of one warp run the same loop shape on same-sized values.
struct LaneState {
  Chain c;
  u64 v;
  u32 item, mode, thr, cap;
  u32 phase, t, bi, lim, d2, pass;
};

__device__ __forceinline__ bool lane_init(LaneState& s, const ClassArgs& a,
                                          u64 i) {
  s.item = a.cand_item[i];
  const DevItem it = a.items[s.item];
  const DevEngine& e = a.engines[it.engine];
  s.v = a.cand_key[i];
  if (it.mode == MODE_SIEVE) {
    emit_out(a, s.item, s.v << 8);
    return false;
  }
  s.mode = it.mode;
  s.thr = it.threshold;
  s.cap = it.cap;
  s.c.kind = e.kind;
  s.c.x = (((u128)it.X0_hi << 64) | it.X0_lo) + s.v;
  if (e.kind == KIND_DICKSON) {
    const u64 W = (it.mode == MODE_DENSE) ? 1ull : e.W;
    bool of = false;
    const u128 k = s.c.x * (u128)W;
    s.c.kk = v3_mul_128(k, k, &of);
    if (of) {
      atomicOr(&a.ctr->overflow, 8u);
      return false;
    }
  } else if (e.kind == KIND_AP) {
    s.c.d = V3{{e.d_lo, e.d_hi, 0}};
  }
  s.pass = (e.kind == KIND_AP) ? 6u
           : (e.kind == KIND_DICKSON ? (e.two_pass ? 5u : 0u) : 0u);
  s.lim = (e.kind == KIND_EULER) ? max(s.thr, s.cap) : s.cap;
  s.phase = 0;
  s.t = 0;
  s.bi = 0;
  return true;
}

// Finish with the exact depth: emit when it reaches the threshold.
__device__ __forceinline__ void lane_final(const LaneState& s,
                                           const ClassArgs& a, u32 exact) {
  if (s.c.kind == KIND_EULER) {
    const u32 depth = min(exact, s.cap);
    const u32 test = (s.mode == MODE_DENSE) ? depth : exact;
    if (test >= s.thr) emit_out(a, s.item, (s.v << 8) | (u64)min(depth, 255u));
  } else if (exact >= s.thr) {
    emit_out(a, s.item, (s.v << 8) | (u64)min(exact, 255u));
  }
}

// After the base-2 chain: returns true when the exact phase must run.
__device__ __forceinline__ bool lane_decide(LaneState& s, const ClassArgs& a) {
  const u32 d2 = s.d2;
  if (s.c.kind == KIND_EULER) {
    const u32 bound = (s.mode == MODE_DENSE) ? min(d2, s.cap) : d2;
    if (bound < s.thr) return false;
  } else {
    if (d2 < s.pass) {
      if (d2 >= s.thr) emit_out(a, s.item, (s.v << 8) | (u64)min(d2, 255u));
      return false;
    }
    if (d2 < s.thr) return false;
  }
  if (d2 == 0) {
    lane_final(s, a, 0);
    return false;
  }
  s.phase = 1;
  s.t = 0;
  s.bi = 1;
  return true;
}

__global__ void __launch_bounds__(kBlock) k_classify(ClassArgs a) {
  u64 n = a.ctr->ncand;
  if (n > a.cand_cap) n = a.cand_cap;
  const u32 lane = threadIdx.x & 31;
  const u32 lt = (1u << lane) - 1u;
  u64 chunk_pos = 0, chunk_end = 0;  // warp-uniform
  bool active = false, drained = false;
  LaneState st;
  u64 imad = 0, nval = 0;
  for (;;) {
    // hand new candidates to idle lanes
    while (!drained) {
      const u32 idle = __ballot_sync(0xffffffffu, !active);
      if (!idle) break;
      if (chunk_pos >= chunk_end) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&a.ctr->class_next, (u64)kClassChunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) {
          drained = true;
          break;
        }
        chunk_pos = base;
        chunk_end = min(base + (u64)kClassChunk, n);
      }
      const u32 rank = __popc(idle & lt);
      const u32 take = (u32)min((u64)__popc(idle), chunk_end - chunk_pos);
      if (!active && rank < take) active = lane_init(st, a, chunk_pos + rank);
      chunk_pos += take;
    }
    if (__ballot_sync(0xffffffffu, active) == 0) break;
    if (active) {
      ++nval;
      const bool pass = sprp_step(chain_value(st.c, st.t), st.bi, &imad);
      if (st.phase == 0) {
        if (pass && st.t + 1 < st.lim) {
          ++st.t;
        } else {
          st.d2 = pass ? st.lim : st.t;
          active = lane_decide(st, a);
        }
      } else {
        if (!pass) {
          lane_final(st, a, st.t);
          active = false;
        } else if (st.bi < 6) {
          ++st.bi;
        } else if (st.t + 1 < st.d2) {
          ++st.t;
          st.bi = 1;
        } else {
          lane_final(st, a, st.d2);
          active = false;
        }
      }
    }
  }
  // one atomic per warp for the work counters
  u64 s1 = imad, s2 = nval;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (s1) atomicAdd(&a.ctr->imad_alg, (unsigned long long)s1);
    if (s2) atomicAdd(&a.ctr->sprp_values, (unsigned long long)s2);
  }
}

// Every x of dense items, into the candidate list.
__global__ void k_dense(const DevItem* items, const u32* dense_idx,
                        u32 ndense, u64* cand_key, u32* cand_item,
                        u64 cand_cap, DevCounters* ctr) {
  for (u32 d = 0; d < ndense; ++d) {
    const u32 item = dense_idx[d];
    const u64 cnt = items[item].U;
    for (u64 v = (u64)blockIdx.x * blockDim.x + threadIdx.x; v < cnt;
         v += (u64)gridDim.x * blockDim.x) {
      const unsigned long long p = atomicAdd(&ctr->ncand, 1ull);
      if (p < cand_cap) {
        cand_key[p] = v;
        cand_item[p] = item;
      } else {
        atomicOr(&ctr->overflow, 1u);
      }
    }
  }
}

// X0 mod q for every (item, prime) of sieve items.
__global__ void k_xq(const DevEngine* engines, const DevItem* items,
                     const u32* sieve_idx, u32 nsieve, u32* xq) {
  for (u32 s = blockIdx.y; s < nsieve; s += gridDim.y) {
    const DevItem it = items[sieve_idx[s]];
    const DevEngine& e = engines[it.engine];
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < e.NP;
         i += gridDim.x * blockDim.x) {
      const PrimeRec pr = e.recs[i];
      xq[it.xq_off + i] =
          fk_bmod128(it.X0_lo, it.X0_hi, pr.q, pr.magic, e.c64[i]);
    }
  }
}

// Exclusive scan of the per-item counts (one CTA).  With n_dev set, the
// count is read from device memory (graph replays of varying sizes).
__global__ void k_scan(const u32* count, u32 n, u64* off,
                       const u32* n_dev = nullptr) {
  if (n_dev) n = *n_dev;
  __shared__ u64 s_carry;
  __shared__ u64 s_warp[kBlock / 32];
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (u32 base = 0; base < n; base += kBlock) {
    const u32 i = base + threadIdx.x;
    const u64 v = i < n ? count[i] : 0;
    u64 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u64 y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    u64 pre = 0, tot = 0;
    for (int w = 0; w < kBlock / 32; ++w) {
      pre += (w < wid) ? s_warp[w] : 0;
      tot += s_warp[w];
    }
    if (i < n) off[i] = s_carry + pre + x - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) off[n] = s_carry;
}

__global__ void k_scatter(const OutRec* out, const DevCounters* ctr,
                          u64 out_cap, const u64* off, u32* fill,
                          u64* sorted) {
  u64 n = ctr->nout;
  if (n > out_cap) n = out_cap;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const OutRec r = out[i];
    const u32 p = atomicAdd(fill + r.item, 1u);
    sorted[off[r.item] + p] = r.packed;
  }
}

// Buckets for ordering: every item's entries are split by key range into
// nb = ceil(count / kBucketFill) buckets (the entries of one interval are
// spread over its span, so a bucket holds about kBucketFill of them), and
// each bucket is then sorted on its own (k_sort_seg).  nb[i] per item:
__global__ void k_bucket_nb(const u32* count, u32 n, u32* nb) {
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    nb[i] = count[i] ? (count[i] + kBucketFill - 1) / kBucketFill : 0;
}

__device__ __forceinline__ u32 bucket_of(const OutRec& r, const DevItem* items,
                                         const DevEngine* engines,
                                         const u64* bucket_base,
                                         const u32* nb) {
  const DevItem it = items[r.item];
  const u64 span = (it.mode == MODE_DENSE)
                       ? it.U
                       : it.U * engines[it.engine].M;  // keys are below U*M
  const u32 k = nb[r.item];
  const u64 key = r.packed >> 8;
  u64 b = (u64)(((u128)key * k) / (span ? span : 1));
  if (b >= k) b = k - 1;
  return (u32)(bucket_base[r.item] + b);
}

__global__ void k_bucket_count(const OutRec* out, const DevCounters* ctr,
                               u64 out_cap, const DevItem* items,
                               const DevEngine* engines,
                               const u64* bucket_base, const u32* nb,
                               u32* bcount) {
  u64 n = ctr->nout;
  if (n > out_cap) n = out_cap;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x)
    atomicAdd(bcount + bucket_of(out[i], items, engines, bucket_base, nb), 1u);
}

__global__ void k_bucket_scatter(const OutRec* out, const DevCounters* ctr,
                                 u64 out_cap, const DevItem* items,
                                 const DevEngine* engines,
                                 const u64* bucket_base, const u32* nb,
                                 const u64* boff, u32* bfill, u64* sorted) {
  u64 n = ctr->nout;
  if (n > out_cap) n = out_cap;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const OutRec r = out[i];
    const u32 b = bucket_of(r, items, engines, bucket_base, nb);
    sorted[boff[b] + atomicAdd(bfill + b, 1u)] = r.packed;
  }
}

// The bucket count, for k_sort_seg's device-side segment count.
__global__ void k_bucket_total(const u64* bucket_base, u32 nitems,
                               u32* nbuckets) {
  *nbuckets = (u32)bucket_base[nitems];
}

// Bitonic sort of buf[0, npow) ascending, npow a power of two, by one CTA.
__device__ void cta_bitonic(u64* buf, u32 npow) {
  for (u32 k = 2; k <= npow; k <<= 1) {
    for (u32 j = k >> 1; j > 0; j >>= 1) {
      for (u32 i = threadIdx.x; i < npow; i += blockDim.x) {
        const u32 l = i ^ j;
        if (l > i) {
          const u64 x = buf[i], y = buf[l];
          const bool up = (i & k) == 0;
          if ((x > y) == up) {
            buf[i] = y;
            buf[l] = x;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Sort every item's segment of `sorted` (keys unique per item).
__global__ void __launch_bounds__(kBlock) k_sort_seg(
    u64* sorted, const u64* off, const u32* nitems_p, u64* scratch) {
  __shared__ u64 s_buf[kSortSmem];
  const u32 nitems = *nitems_p;
  for (u32 item = blockIdx.x; item < nitems; item += gridDim.x) {
    const u64 o = off[item];
    const u32 n = (u32)(off[item + 1] - o);
    if (n < 2) continue;
    u32 npow = 1;
    while (npow < n) npow <<= 1;
    u64* buf = (npow <= (u32)kSortSmem) ? s_buf : scratch + 2 * o;
    for (u32 i = threadIdx.x; i < npow; i += blockDim.x)
      buf[i] = i < n ? sorted[o + i] : ~0ull;
    __syncthreads();
    cta_bitonic(buf, npow);
    for (u32 i = threadIdx.x; i < n; i += blockDim.x) sorted[o + i] = buf[i];
    __syncthreads();
  }
}

}  // namespace fk
