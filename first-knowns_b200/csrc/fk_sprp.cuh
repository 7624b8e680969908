// fk_sprp.cuh -- multi-limb Montgomery strong-probable-prime tests.
//
// Device restatement of huntlib/primes.py:23-80 (mr_is_prime and
// sprp_base2) for values of one to three 64-bit limbs (up to 192 bits):
// trial division by the primes to 37 returning m == sp, then the strong
// test to the bases (2, 325, 9375, 28178, 450775, 9780504, 1795265022)
// with a %= m and a zero base skipped.  Verdicts are bit-identical to the
// reference's on every input; above 3.317e24 they are strong-probable-
// prime verdicts, exactly as the reference's are.
//
// Multiplication is CIOS Montgomery (Koc, Acar, Kaliski 1996) over
// 32-bit limbs with PTX carry chains (fk_mont32.cuh), two to six limbs by
// the value's size; reduction constants are -m^-1 mod 2^32 by Newton
// iteration and R mod m, R^2 mod m by modular doubling.
#pragma once
#include "fk_arith.cuh"
#include "fk_mont32.cuh"

namespace fk {

__device__ __constant__ u32 kMrBases[7] = {2u, 325u, 9375u, 28178u, 450775u,
                                           9780504u, 1795265022u};

// A value of up to three 64-bit limbs, little-endian.
struct V3 {
  u64 w[3];
};

__device__ __forceinline__ V3 v3_from_u128(u128 x) {
  V3 v;
  v.w[0] = (u64)x;
  v.w[1] = (u64)(x >> 64);
  v.w[2] = 0;
  return v;
}

// a + b (no overflow past 192 bits assumed by callers)
__device__ __forceinline__ V3 v3_add(const V3& a, const V3& b) {
  V3 r;
  u64 c = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    u64 s = a.w[i] + b.w[i];
    u64 c1 = s < a.w[i];
    u64 t = s + c;
    u64 c2 = t < s;
    r.w[i] = t;
    c = c1 | c2;
  }
  return r;
}

// a * small (a < 2^192 / small assumed)
__device__ __forceinline__ V3 v3_mul_u64(const V3& a, u64 s) {
  V3 r;
  u64 c = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    u128 p = (u128)a.w[i] * s + c;
    r.w[i] = (u64)p;
    c = (u64)(p >> 64);
  }
  return r;
}

// a (two limbs) * b (two limbs) -> low three limbs; *overflow set if the
// product needs a fourth limb.
__device__ __forceinline__ V3 v3_mul_128(u128 a, u128 b, bool* overflow) {
  u64 a0 = (u64)a, a1 = (u64)(a >> 64), b0 = (u64)b, b1 = (u64)(b >> 64);
  u128 p00 = (u128)a0 * b0;
  u128 p01 = (u128)a0 * b1;
  u128 p10 = (u128)a1 * b0;
  u128 p11 = (u128)a1 * b1;
  V3 r;
  r.w[0] = (u64)p00;
  u128 mid = (p00 >> 64) + (u64)p01 + (u64)p10;
  r.w[1] = (u64)mid;
  u128 hi = (mid >> 64) + (p01 >> 64) + (p10 >> 64) + (u64)p11;
  r.w[2] = (u64)hi;
  *overflow = ((hi >> 64) + (p11 >> 64)) != 0;
  return r;
}

// ---- Montgomery arithmetic on 64-bit limbs (one-limb values) -----------

template <int L>
__device__ __forceinline__ int bitlen64(const u64* m) {
  return 64 * (L - 1) + (64 - __clzll(m[L - 1]));
}

// x = 2x mod m for x < m.
template <int L>
__device__ __forceinline__ void mdbl64(u64* x, const u64* m) {
  u64 y[L];
  u64 top = x[L - 1] >> 63;
#pragma unroll
  for (int i = L - 1; i > 0; --i) y[i] = (x[i] << 1) | (x[i - 1] >> 63);
  y[0] = x[0] << 1;
  // y (+ top * 2^(64L)) >= m ?
  u64 d[L];
  u64 br = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    u64 t = y[i] - m[i];
    u64 b1 = y[i] < m[i];
    u64 t2 = t - br;
    u64 b2 = t < br;
    d[i] = t2;
    br = b1 | b2;
  }
  bool ge = top || !br;
#pragma unroll
  for (int i = 0; i < L; ++i) x[i] = ge ? d[i] : y[i];
}

// r = a * b * 2^(-64L) mod m for a, b < m, m odd.  CIOS.
template <int L>
__device__ __forceinline__ void mmul64(u64* r, const u64* a, const u64* b,
                                         const u64* m, u64 minv) {
  u64 t[L + 2];
#pragma unroll
  for (int i = 0; i < L + 2; ++i) t[i] = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    u64 c = 0;
#pragma unroll
    for (int j = 0; j < L; ++j) {
      u128 p = (u128)a[j] * b[i] + t[j] + c;
      t[j] = (u64)p;
      c = (u64)(p >> 64);
    }
    u128 s = (u128)t[L] + c;
    t[L] = (u64)s;
    t[L + 1] = (u64)(s >> 64);
    u64 q = t[0] * minv;
    u128 p = (u128)q * m[0] + t[0];
    c = (u64)(p >> 64);
#pragma unroll
    for (int j = 1; j < L; ++j) {
      p = (u128)q * m[j] + t[j] + c;
      t[j - 1] = (u64)p;
      c = (u64)(p >> 64);
    }
    s = (u128)t[L] + c;
    t[L - 1] = (u64)s;
    t[L] = t[L + 1] + (u64)(s >> 64);
  }
  u64 d[L];
  u64 br = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    u64 x = t[i] - m[i];
    u64 b1 = t[i] < m[i];
    u64 x2 = x - br;
    u64 b2 = x < br;
    d[i] = x2;
    br = b1 | b2;
  }
  bool ge = t[L] || !br;
#pragma unroll
  for (int i = 0; i < L; ++i) r[i] = ge ? d[i] : t[i];
}

template <int L>
__device__ __forceinline__ bool eq64(const u64* a, const u64* b) {
  bool e = true;
#pragma unroll
  for (int i = 0; i < L; ++i) e &= (a[i] == b[i]);
  return e;
}

// Residue of the multi-limb m modulo a small modulus s (s < 2^31), from
// the limbs top down with c = 2^64 mod s.
template <int L>
__device__ __forceinline__ u32 small_mod64(const u64* m, u32 s, u32 c) {
  u64 r = 0;
#pragma unroll
  for (int i = L - 1; i >= 0; --i) r = (r * c + (m[i] % s)) % s;
  return (u32)r;
}

// Trial division of huntlib/primes.py:31-33 by the primes 2..37:
// returns 0 (composite: divisible by a small prime it is not), 1 (m is one
// of those primes, prime), or 2 (no small factor: go on).  Uses two
// composite moduli, 223092870 = 2*3*5*7*11*13*17*19*23 and 33263 = 29*31*37.
template <int L>
__device__ __forceinline__ int trial64(const u64* m) {
  if (L == 1 && m[0] < 2) return 0;
  const u32 r1 = small_mod64<L>(
      m, 223092870u, (u32)((18446744073709551615ull % 223092870ull + 1) % 223092870ull));
  const u32 r2 = small_mod64<L>(
      m, 33263u, (u32)((18446744073709551615ull % 33263ull + 1) % 33263ull));
  const u32 sp1[9] = {2, 3, 5, 7, 11, 13, 17, 19, 23};
  const u32 sp2[3] = {29, 31, 37};
#pragma unroll
  for (int i = 0; i < 9; ++i)
    if (r1 % sp1[i] == 0) return (L == 1 && m[0] == sp1[i]) ? 1 : 0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (r2 % sp2[i] == 0) return (L == 1 && m[0] == sp2[i]) ? 1 : 0;
  return 2;
}

// Montgomery context over 64-bit limbs (used for one-limb values, where
// one 64 x 64-bit product beats two 32-bit CIOS rounds).
template <int L>
struct Ctx64 {
  u64 m[L], one[L], mone[L], d[L];
  u64 minv;
  int bl, s, dtop;
};

template <int L>
__device__ __forceinline__ void ctx_init64(Ctx64<L>& c, const u64* m) {
#pragma unroll
  for (int i = 0; i < L; ++i) c.m[i] = m[i];
  u64 minv = m[0];  // m * m == 1 mod 8: correct to 3 bits
#pragma unroll
  for (int i = 0; i < 5; ++i) minv *= 2 - m[0] * minv;
  c.minv = (u64)0 - minv;  // -m^-1 mod 2^64
  c.bl = bitlen64<L>(m);
#pragma unroll
  for (int i = 0; i < L; ++i) c.one[i] = 0;
  c.one[(c.bl - 1) >> 6] = 1ull << ((c.bl - 1) & 63);  // 2^(bl-1) < m
  for (int i = 0; i < 64 * L - c.bl + 1; ++i) mdbl64<L>(c.one, m);
  u64 br = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {  // m - (R mod m): -1 in Montgomery form
    const u64 x = m[i] - c.one[i];
    const u64 b1 = m[i] < c.one[i];
    const u64 x2 = x - br;
    const u64 b2 = x < br;
    c.mone[i] = x2;
    br = b1 | b2;
  }
#pragma unroll
  for (int i = 0; i < L; ++i) c.d[i] = m[i];
  c.d[0] -= 1;  // m odd
  int lz = 0;
  while (c.d[lz] == 0) ++lz;
  c.s = 64 * lz + __ffsll((long long)c.d[lz]) - 1;
  const int ws = c.s >> 6, bs = c.s & 63;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    const u64 lo = (i + ws < L) ? c.d[i + ws] : 0;
    const u64 hi = (i + ws + 1 < L) ? c.d[i + ws + 1] : 0;
    c.d[i] = bs ? ((lo >> bs) | (hi << (64 - bs))) : lo;
  }
  c.dtop = 0;
#pragma unroll
  for (int i = L - 1; i >= 0; --i)
    if (c.d[i] && c.dtop == 0) c.dtop = 64 * i + 63 - __clzll(c.d[i]);
}

// Algorithmic 32-bit multiply-adds of one strong test (CIOS on 32-bit
// limbs): (bits - 1) squarings of 2l^2 + l word products, lo and hi each.
template <int L>
__device__ __forceinline__ u64 imad64(const Ctx64<L>& c) {
  const u64 l32 = (u64)((c.bl + 31) >> 5);
  return (u64)(c.bl - 1) * (4 * l32 * l32 + 2 * l32);
}

// The strong-test tail: x = a^d already in Montgomery form.
template <int L>
__device__ __forceinline__ bool tail64(const Ctx64<L>& c, u64* x) {
  if (eq64<L>(x, c.one) || eq64<L>(x, c.mone)) return true;
  for (int r = 1; r < c.s; ++r) {
    mmul64<L>(x, x, x, c.m, c.minv);
    if (eq64<L>(x, c.mone)) return true;
  }
  return false;
}

// One strong test of m to base kMrBases[bi] (bi = 0 is base 2), with the
// trial division first: the unit of work of the step interpreter in
// k_classify.  Every base runs the same loop shape -- square, then on a set
// bit of d multiply by the base (a modular doubling for base 2) -- so lanes
// testing different bases of same-sized values stay converged.
template <int L>
__device__ __forceinline__ bool step64(const u64* m, int bi, u64* imad) {
  const int t = trial64<L>(m);
  if (t != 2) return t == 1;
  Ctx64<L> c;
  ctx_init64<L>(c, m);
  u64 at[L];
  bool is2 = bi == 0;
  if (!is2) {
    u64 a = kMrBases[bi];
    if (L == 1 && c.m[0] <= a) {
      a %= c.m[0];
      if (a == 0) return true;  // huntlib skips a zero base
    }
    u64 r2m[L], av[L];
#pragma unroll
    for (int i = 0; i < L; ++i) { r2m[i] = c.one[i]; av[i] = 0; }
    for (int i = 0; i < 64 * L; ++i) mdbl64<L>(r2m, c.m);
    av[0] = a;
    mmul64<L>(at, av, r2m, c.m, c.minv);  // a * R mod m
  }
  *imad += imad64<L>(c);
  u64 x[L];
#pragma unroll
  for (int i = 0; i < L; ++i) x[i] = c.one[i];
  for (int b = c.dtop; b >= 0; --b) {
    mmul64<L>(x, x, x, c.m, c.minv);
    if ((c.d[b >> 6] >> (b & 63)) & 1) {
      if (is2) mdbl64<L>(x, c.m);
      else mmul64<L>(x, x, at, c.m, c.minv);
    }
  }
  return tail64<L>(c, x);
}


// ---- Montgomery arithmetic on N 32-bit limbs (N = 2..6) -----------------
// A value below 2^(32N) as N little-endian 32-bit words.  Products use the
// carry-chained multiply-accumulate pass of fk_mont32.cuh, so one word
// product is one mad.lo and one mad.hi -- the two IMADs per product the
// algorithmic count charges.

template <int N>
__device__ __forceinline__ int bitlen32(const u32* m) {
#pragma unroll
  for (int i = N - 1; i > 0; --i)
    if (m[i]) return 32 * i + 32 - __clz(m[i]);
  return 32 - __clz(m[0]);
}

// d = x - y over N words; returns the borrow out.
template <int N>
__device__ __forceinline__ u32 sub_n(u32* d, const u32* x, const u32* y) {
  u32 br = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const u64 t = (u64)x[i] - y[i] - br;
    d[i] = (u32)t;
    br = (u32)(t >> 63);
  }
  return br;
}

// x = 2x mod m for x < m.
template <int N>
__device__ __forceinline__ void mdbl32(u32* x, const u32* m) {
  u32 y[N], d[N];
  const u32 top = x[N - 1] >> 31;
#pragma unroll
  for (int i = N - 1; i > 0; --i) y[i] = (x[i] << 1) | (x[i - 1] >> 31);
  y[0] = x[0] << 1;
  const u32 br = sub_n<N>(d, y, m);
  const bool ge = top || !br;
#pragma unroll
  for (int i = 0; i < N; ++i) x[i] = ge ? d[i] : y[i];
}

// r = a * b * 2^(-32N) mod m for a, b < m, m odd (CIOS; r may alias a/b).
template <int N>
__device__ __forceinline__ void mmul32(u32* r, const u32* a, const u32* b,
                                       const u32* m, u32 minv) {
  u32 t[N + 2];
#pragma unroll
  for (int i = 0; i < N + 2; ++i) t[i] = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    Mont32<N>::mac(t, a, b[i]);
    const u32 q = t[0] * minv;
    Mont32<N>::mac(t, m, q);       // t[0] becomes 0
#pragma unroll
    for (int j = 0; j < N + 1; ++j) t[j] = t[j + 1];
    t[N + 1] = 0;
  }
  u32 d[N];
  const u32 br = sub_n<N>(d, t, m);
  const bool ge = t[N] || !br;
#pragma unroll
  for (int i = 0; i < N; ++i) r[i] = ge ? d[i] : t[i];
}

template <int N>
__device__ __forceinline__ bool eq32(const u32* a, const u32* b) {
  bool e = true;
#pragma unroll
  for (int i = 0; i < N; ++i) e &= (a[i] == b[i]);
  return e;
}

// Residue of m modulo a small modulus s (s < 2^31), from the top word
// down with c = 2^32 mod s.
template <int N>
__device__ __forceinline__ u32 small_mod32(const u32* m, u32 s, u32 c) {
  u64 r = 0;
#pragma unroll
  for (int i = N - 1; i >= 0; --i) r = (r * c + m[i] % s) % s;
  return (u32)r;
}

// Trial division of huntlib/primes.py:31-33 by the primes 2..37:
// returns 0 (composite: divisible by a small prime it is not), 1 (m is one
// of those primes, prime), or 2 (no small factor: go on).  Uses two
// composite moduli, 223092870 = 2*3*5*7*11*13*17*19*23 and 33263 = 29*31*37.
template <int N>
__device__ __forceinline__ int trial_small(const u32* m) {
  bool small = true;
#pragma unroll
  for (int i = 1; i < N; ++i) small &= (m[i] == 0);
  if (small && m[0] < 2) return 0;
  const u32 r1 = small_mod32<N>(m, 223092870u,
                                (u32)((1ull << 32) % 223092870ull));
  const u32 r2 = small_mod32<N>(m, 33263u, (u32)((1ull << 32) % 33263ull));
  const u32 sp1[9] = {2, 3, 5, 7, 11, 13, 17, 19, 23};
  const u32 sp2[3] = {29, 31, 37};
#pragma unroll
  for (int i = 0; i < 9; ++i)
    if (r1 % sp1[i] == 0) return (small && m[0] == sp1[i]) ? 1 : 0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (r2 % sp2[i] == 0) return (small && m[0] == sp2[i]) ? 1 : 0;
  return 2;
}

// Montgomery context of an odd m > 37 with no small factor: R = 2^(32N).
template <int N>
struct Ctx {
  u32 m[N], one[N], mone[N], d[N];
  u32 minv;
  int bl, s, dtop;
};

template <int N>
__device__ __forceinline__ void ctx_init(Ctx<N>& c, const u32* m) {
#pragma unroll
  for (int i = 0; i < N; ++i) c.m[i] = m[i];
  u32 inv = m[0];  // m * m == 1 mod 8: correct to 3 bits
#pragma unroll
  for (int i = 0; i < 4; ++i) inv *= 2u - m[0] * inv;
  c.minv = 0u - inv;  // -m^-1 mod 2^32
  c.bl = bitlen32<N>(m);
#pragma unroll
  for (int i = 0; i < N; ++i) c.one[i] = 0;
  c.one[(c.bl - 1) >> 5] = 1u << ((c.bl - 1) & 31);  // 2^(bl-1) < m
  for (int i = 0; i < 32 * N - c.bl + 1; ++i) mdbl32<N>(c.one, m);
  sub_n<N>(c.mone, m, c.one);  // -1 in Montgomery form
#pragma unroll
  for (int i = 0; i < N; ++i) c.d[i] = m[i];
  c.d[0] -= 1;  // m odd
  int lz = 0;
  while (c.d[lz] == 0) ++lz;
  c.s = 32 * lz + __ffs((int)c.d[lz]) - 1;
  const int ws = c.s >> 5, bs = c.s & 31;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const u32 lo = (i + ws < N) ? c.d[i + ws] : 0;
    const u32 hi = (i + ws + 1 < N) ? c.d[i + ws + 1] : 0;
    c.d[i] = bs ? ((lo >> bs) | (hi << (32 - bs))) : lo;
  }
  c.dtop = 0;
#pragma unroll
  for (int i = N - 1; i >= 0; --i)
    if (c.d[i] && c.dtop == 0) c.dtop = 32 * i + 31 - __clz(c.d[i]);
}

// Algorithmic 32-bit multiply-adds of one strong test (CIOS on 32-bit
// limbs): (bits - 1) squarings of 2l^2 + l word products, lo and hi each.
template <int N>
__device__ __forceinline__ u64 imad_per_base(const Ctx<N>& c) {
  const u64 l32 = (u64)((c.bl + 31) >> 5);
  return (u64)(c.bl - 1) * (4 * l32 * l32 + 2 * l32);
}

// The strong-test tail: x = a^d already in Montgomery form.
template <int N>
__device__ __forceinline__ bool strong_tail(const Ctx<N>& c, u32* x) {
  if (eq32<N>(x, c.one) || eq32<N>(x, c.mone)) return true;
  for (int r = 1; r < c.s; ++r) {
    mmul32<N>(x, x, x, c.m, c.minv);
    if (eq32<N>(x, c.mone)) return true;
  }
  return false;
}

// One strong test of m to base kMrBases[bi] (bi = 0 is base 2), with the
// trial division first.  Every base runs the same loop shape -- square,
// then on a set bit of d multiply by the base (a modular doubling for base
// 2, so base 2 needs no R^2) -- so lanes testing different bases of
// same-sized values stay converged.
template <int N>
__device__ __forceinline__ bool step_N(const u32* m, int bi, u64* imad) {
  const int t = trial_small<N>(m);
  if (t != 2) return t == 1;
  Ctx<N> c;
  ctx_init<N>(c, m);
  u32 at[N];
  const bool is2 = bi == 0;
  if (!is2) {
    u32 a = kMrBases[bi];
    bool small = true;
#pragma unroll
    for (int i = 1; i < N; ++i) small &= (c.m[i] == 0);
    if (small && c.m[0] <= a) {
      a %= c.m[0];
      if (a == 0) return true;  // huntlib skips a zero base
    }
    u32 r2m[N], av[N];
#pragma unroll
    for (int i = 0; i < N; ++i) { r2m[i] = c.one[i]; av[i] = 0; }
    for (int i = 0; i < 32 * N; ++i) mdbl32<N>(r2m, c.m);  // R^2 mod m
    av[0] = a;
    mmul32<N>(at, av, r2m, c.m, c.minv);  // a * R mod m
  }
  *imad += imad_per_base<N>(c);
  u32 x[N];
#pragma unroll
  for (int i = 0; i < N; ++i) x[i] = c.one[i];
  u32 dw = 0;
  for (int b = c.dtop; b >= 0; --b) {
    if (b == c.dtop || (b & 31) == 31) dw = c.d[b >> 5];  // once a word
    mmul32<N>(x, x, x, c.m, c.minv);
    if ((dw >> (b & 31)) & 1u) {
      if (is2) mdbl32<N>(x, c.m);
      else mmul32<N>(x, x, at, c.m, c.minv);
    }
  }
  return strong_tail<N>(c, x);
}

// The value's 32-bit words and the limb count it needs (at least 2).
__device__ __forceinline__ int to_words(const V3& v, u32* w) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    w[2 * i] = (u32)v.w[i];
    w[2 * i + 1] = (u32)(v.w[i] >> 32);
  }
  int n = 6;
  while (n > 2 && w[n - 1] == 0) --n;
  return n;
}

__device__ __noinline__ bool sprp_step(const V3& v, int bi, u64* imad) {
  if (v.w[1] == 0 && v.w[2] == 0) return step64<1>(v.w, bi, imad);
  u32 w[6];
  switch (to_words(v, w)) {
    case 6: return step_N<6>(w, bi, imad);
    case 5: return step_N<5>(w, bi, imad);
    case 4: return step_N<4>(w, bi, imad);
    case 3: return step_N<3>(w, bi, imad);
    default: return step_N<2>(w, bi, imad);
  }
}

// which = 0: mr_is_prime, 1: sprp_base2, 2: the six bases after 2 only
// (callers that already know m passes base 2).
__device__ __noinline__ bool sprp_which(const V3& v, int which, u64* imad) {
  if (which != 2 && !sprp_step(v, 0, imad)) return false;
  if (which == 1) return true;
  for (int bi = 1; bi < 7; ++bi)
    if (!sprp_step(v, bi, imad)) return false;
  return true;
}

// mr_is_prime (base2_only = false) or sprp_base2 (true).
__device__ __forceinline__ bool sprp(const V3& v, bool base2_only, u64* imad) {
  return sprp_which(v, base2_only ? 1 : 0, imad);
}

// The six bases after 2 (v already passed base 2 and trial division).
__device__ __forceinline__ bool sprp_rest(const V3& v, u64* imad) {
  return sprp_which(v, 2, imad);
}

}  // namespace fk
