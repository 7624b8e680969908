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

__global__ void __launch_bounds__(kBlock) k_classify(ClassArgs a) {
  u64 n = a.ctr->ncand;
  if (n > a.cand_cap) n = a.cand_cap;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  u64 imad = 0, nval = 0;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += stride) {
    const u32 item = a.cand_item[i];
    const DevItem it = a.items[item];
    const DevEngine& e = a.engines[it.engine];
    const u64 v = a.cand_key[i];
    if (it.mode == MODE_SIEVE) {
      emit_out(a, item, v << 8);
      continue;
    }
    Chain c;
    c.kind = e.kind;
    c.x = (((u128)it.X0_hi << 64) | it.X0_lo) + v;
    if (e.kind == KIND_DICKSON) {
      // the line variable is j (k = W*j); a dense item carries k itself
      const u64 W = (it.mode == MODE_DENSE) ? 1ull : e.W;
      bool of = false;
      const u128 k = c.x * (u128)W;
      c.kk = v3_mul_128(k, k, &of);
      if (of) {
        atomicOr(&a.ctr->overflow, 8u);
        continue;
      }
    } else if (e.kind == KIND_AP) {
      c.d = V3{{e.d_lo, e.d_hi, 0}};
    }
    const int depth = chain_depth_thr(c, it.mode, it.threshold, it.cap,
                                      e.two_pass != 0, &imad, &nval);
    if (depth >= 0) emit_out(a, item, (v << 8) | (u64)min((u32)depth, 255u));
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

// Exclusive scan of the per-item counts (one CTA).
__global__ void k_scan(const u32* count, u32 n, u64* off) {
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
