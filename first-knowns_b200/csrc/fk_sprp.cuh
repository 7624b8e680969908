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
// Arithmetic is Montgomery's (Montgomery 1985): one 64-bit word for
// m < 2^62, else CIOS (Koc, Acar, Kaliski 1996) over three to six 32-bit
// limbs with PTX carry chains (fk_mont32.cuh).  The word count is chosen
// so that 4m < R, which lets every residue stay in [0, 2m) between
// products (lazy reduction: no conditional subtraction per product,
// Walter's bound); residues are made canonical only to be compared.
// -m^-1 mod 2^w comes by Newton iteration, R mod m by modular doubling
// from 2^(bits-1), and a*R mod m for a base a by double-and-add.
//
// The exponent d of m - 1 = d * 2^s is read in bit pairs aligned to even
// positions (they never straddle a 32-bit word): two squarings per pair,
// then one product by a, a^2 or a^3 (precomputed) -- or, for base 2, up
// to three modular doublings -- so lanes testing different bases of
// same-sized values share the squarings and the loop shape.
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

// ---- trial division (huntlib/primes.py:31-33) ---------------------------

// Divisibility of a residue r < 2^32 by an odd prime p, by multiplying
// with pinv = p^-1 mod 2^32 (Granlund and Montgomery 1994): p | r iff
// r * pinv mod 2^32 <= lim = (2^32 - 1) / p.
__device__ __forceinline__ bool divides(u32 r, u32 pinv, u32 lim) {
  return r * pinv <= lim;
}

// x mod s for a value of three 64-bit limbs, c = 2^64 mod s, s < 2^28.
__device__ __forceinline__ u32 mod3(const V3& v, u64 s, u64 c) {
  u64 r = v.w[2] % s;
  r = (r * c + v.w[1] % s) % s;
  r = (r * c + v.w[0] % s) % s;
  return (u32)r;
}

// Trial division of huntlib/primes.py:31-33 by the primes 2..37: 0 when m
// is divisible by one of them and is not that prime (composite), 1 when m
// is one of them (prime), 2 when none divides m (the strong tests decide).
// Residues modulo 223092870 = 2*3*...*23 and 33263 = 29*31*37 carry it.
__device__ __forceinline__ int sprp_trial(const V3& v) {
  const bool small = (v.w[1] | v.w[2]) == 0;
  if (small && v.w[0] < 2) return 0;
  u32 r1, r2;
  if (small) {
    r1 = (u32)(v.w[0] % 223092870ull);
    r2 = (u32)(v.w[0] % 33263ull);
  } else {
    r1 = mod3(v, 223092870ull, (~0ull % 223092870ull + 1) % 223092870ull);
    r2 = mod3(v, 33263ull, (~0ull % 33263ull + 1) % 33263ull);
  }
  const u64 m = v.w[0];
  if ((r1 & 1u) == 0) return (small && m == 2) ? 1 : 0;
  // the odd primes to 23 and their inverses mod 2^32, then 29, 31, 37
  constexpr u32 P1[8] = {3, 5, 7, 11, 13, 17, 19, 23};
  constexpr u32 I1[8] = {0xAAAAAAABu, 0xCCCCCCCDu, 0xB6DB6DB7u, 0xBA2E8BA3u,
                         0xC4EC4EC5u, 0xF0F0F0F1u, 0x286BCA1Bu, 0xE9BD37A7u};
  constexpr u32 P2[3] = {29, 31, 37};
  constexpr u32 I2[3] = {0x4F72C235u, 0xBDEF7BDFu, 0x914C1BADu};
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if (divides(r1, I1[i], 0xFFFFFFFFu / P1[i]))
      return (small && m == P1[i]) ? 1 : 0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (divides(r2, I2[i], 0xFFFFFFFFu / P2[i]))
      return (small && m == P2[i]) ? 1 : 0;
  return 2;
}

// Algorithmic 32-bit multiply-adds of one strong test (CIOS on 32-bit
// limbs): (bits - 1) squarings of 2l^2 + l word products, lo and hi each,
// l = ceil(bits / 32) -- whatever representation the test actually uses.
__device__ __forceinline__ u64 imad_alg(int bl) {
  const u64 l = (u64)((bl + 31) >> 5);
  return (u64)(bl - 1) * (4 * l * l + 2 * l);
}

// ---- one 64-bit word: m odd, 37 < m < 2^62, R = 2^64 ---------------------

struct M64 {
  u64 m, m2, minv;
};

// a * b / R mod m in [0, 2m) for a, b < 2m: the low word of a*b + q*m is
// zero by the choice of q, so only its carry (lo != 0) is needed.
__device__ __forceinline__ u64 mul64(const M64& c, u64 a, u64 b) {
  const u64 lo = a * b;
  const u64 hi = __umul64hi(a, b);
  const u64 q = lo * c.minv;
  return hi + __umul64hi(q, c.m) + (lo != 0 ? 1ull : 0ull);
}

__device__ __forceinline__ u64 dbl64(const M64& c, u64 x) {  // [0, 2m)
  const u64 y = x << 1;
  return y >= c.m2 ? y - c.m2 : y;
}

__device__ __forceinline__ bool strong64(u64 m, u32 a, u64* imad) {
  M64 c;
  c.m = m;
  c.m2 = m << 1;
  u64 inv = m;  // m * m == 1 mod 8: correct to 3 bits, doubling each step
#pragma unroll
  for (int i = 0; i < 5; ++i) inv *= 2 - m * inv;
  c.minv = 0 - inv;
  const int bl = 64 - __clzll((long long)m);
  u64 one = 1ull << (bl - 1);  // < m, doubled to 2^64 mod m
  for (int i = 0; i < 64 - bl + 1; ++i) {
    one <<= 1;
    one = one >= m ? one - m : one;
  }
  const u64 dm = m - 1;
  const int s = __ffsll((long long)dm) - 1;
  const u64 d = dm >> s;
  const int dtop = 63 - __clzll((long long)d);
  *imad += imad_alg(bl);
  const bool b2 = a == 2;
  if (m <= a) {  // huntlib: a %= m, a zero base is skipped
    a = (u32)(a % m);
    if (a == 0) return true;
  }
  u64 t1 = one, t2 = one, t3 = one;
  if (!b2) {  // a * R mod m by double-and-add, then a^2, a^3
    u64 r = one;
    for (int b = 30 - __clz(a); b >= 0; --b) {
      r <<= 1;
      r = r >= m ? r - m : r;
      if ((a >> b) & 1u) {
        r += one;
        r = r >= m ? r - m : r;
      }
    }
    t1 = r;
    t2 = mul64(c, t1, t1);
    t3 = mul64(c, t2, t1);
  }
  int b = dtop | 1;  // the aligned pair (b, b - 1) holding the top bit
  u32 w = (u32)(d >> (b - 1)) & 3u;
  u64 x;
  if (b2) {
    x = one;
    for (u32 k = 0; k < w; ++k) x = dbl64(c, x);
  } else {
    x = w == 1 ? t1 : (w == 2 ? t2 : t3);
  }
  for (b -= 2; b >= 1; b -= 2) {
    x = mul64(c, x, x);
    x = mul64(c, x, x);
    w = (u32)(d >> (b - 1)) & 3u;
    if (b2) {
      for (u32 k = 0; k < w; ++k) x = dbl64(c, x);
    } else if (w) {
      x = mul64(c, x, w == 1 ? t1 : (w == 2 ? t2 : t3));
    }
  }
  const u64 mone = m - one;
  x = x >= m ? x - m : x;
  if (x == one || x == mone) return true;
  for (int r = 1; r < s; ++r) {
    x = mul64(c, x, x);
    x = x >= m ? x - m : x;
    if (x == mone) return true;
  }
  return false;
}

// ---- N 32-bit words (N = 3..6): m odd, 4m < 2^(32N) ----------------------

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

// x = x - y when x >= y (in place).
template <int N>
__device__ __forceinline__ void csub_n(u32* x, const u32* y) {
  u32 d[N];
  const u32 br = sub_n<N>(d, x, y);
#pragma unroll
  for (int i = 0; i < N; ++i) x[i] = br ? x[i] : d[i];
}

// x = x - m when `carry` (a bit above the N words) is set or x >= m.
template <int N>
__device__ __forceinline__ void csub_c(u32* x, u32 carry, const u32* m) {
  u32 d[N];
  const u32 br = sub_n<N>(d, x, m);
  const bool ge = carry || !br;
#pragma unroll
  for (int i = 0; i < N; ++i) x[i] = ge ? d[i] : x[i];
}

// x = 2x mod m for x < m (the bit shifted out of the top word counts).
template <int N>
__device__ __forceinline__ void dbl_n(u32* x, const u32* m) {
  const u32 top = x[N - 1] >> 31;
#pragma unroll
  for (int i = N - 1; i > 0; --i) x[i] = (x[i] << 1) | (x[i - 1] >> 31);
  x[0] <<= 1;
  csub_c<N>(x, top, m);
}

// r = a * b / R mod m for R = 2^(32N), by CIOS.  Lazy (4m < R): a, b < 2m
// give r < 2m with no final subtraction (the top word stays zero).
// Strict: a, b < m give r < m after one conditional subtraction.
template <int N, bool Strict = false>
__device__ __forceinline__ void mul_n(u32* r, const u32* a, const u32* b,
                                      const u32* m, u32 minv) {
  u32 t[N + 2];
#pragma unroll
  for (int i = 0; i < N + 2; ++i) t[i] = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    Mont32<N>::mac(t, a, b[i]);
    const u32 q = t[0] * minv;
    Mont32<N>::mac(t, m, q);  // t[0] becomes 0
#pragma unroll
    for (int j = 0; j < N + 1; ++j) t[j] = t[j + 1];
    t[N + 1] = 0;
  }
  if (Strict) csub_c<N>(t, t[N], m);
#pragma unroll
  for (int i = 0; i < N; ++i) r[i] = t[i];
}

template <int N>
__device__ __forceinline__ bool eq_n(const u32* a, const u32* b) {
  bool e = true;
#pragma unroll
  for (int i = 0; i < N; ++i) e &= (a[i] == b[i]);
  return e;
}

template <int N>
__device__ __forceinline__ void sel_n(u32* r, u32 w, const u32* t1,
                                      const u32* t2, const u32* t3) {
#pragma unroll
  for (int i = 0; i < N; ++i) r[i] = w == 1 ? t1[i] : (w == 2 ? t2[i] : t3[i]);
}

// One strong test on N words.  Lazy residues need 4m < R (bits <= 32N -
// 2); Strict keeps every residue canonical and serves the 191- and 192-bit
// values that six words hold without that margin.
template <int N, bool Strict = false>
__device__ __forceinline__ bool strong_n(const u32* m, u32 a, u64* imad) {
  u32 inv = m[0];
#pragma unroll
  for (int i = 0; i < 4; ++i) inv *= 2u - m[0] * inv;
  const u32 minv = 0u - inv;
  int bl = 0;
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (m[i]) bl = 32 * i + 32 - __clz(m[i]);
  *imad += imad_alg(bl);
  // R mod m: 2^(bl - 1) doubled 32N - bl + 1 times, canonical
  u32 one[N];
#pragma unroll
  for (int i = 0; i < N; ++i)
    one[i] = ((bl - 1) >> 5) == i ? 1u << ((bl - 1) & 31) : 0u;
  for (int i = 0; i < 32 * N - bl + 1; ++i) dbl_n<N>(one, m);
  // m - 1 = d * 2^s
  u32 d[N];
#pragma unroll
  for (int i = 0; i < N; ++i) d[i] = m[i];
  d[0] -= 1;  // m odd: no borrow
  int s = 0;
  while (d[0] == 0) {  // whole zero words: shift down (indices stay static)
#pragma unroll
    for (int i = 0; i < N - 1; ++i) d[i] = d[i + 1];
    d[N - 1] = 0;
    s += 32;
  }
  const int bs = __ffs((int)d[0]) - 1;
  s += bs;
  if (bs) {
#pragma unroll
    for (int i = 0; i < N - 1; ++i) d[i] = (d[i] >> bs) | (d[i + 1] << (32 - bs));
    d[N - 1] >>= bs;
  }
  int dtop = 0;
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (d[i]) dtop = 32 * i + 31 - __clz(d[i]);
  const bool b2 = a == 2;
  u32 t1[N], t2[N], t3[N];
  if (!b2) {  // a * R mod m by double-and-add (a < 2^31 < m), then a^2, a^3
#pragma unroll
    for (int i = 0; i < N; ++i) t1[i] = one[i];
    for (int b = 30 - __clz(a); b >= 0; --b) {
      dbl_n<N>(t1, m);
      if ((a >> b) & 1u) {
        u32 c = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const u64 x = (u64)t1[i] + one[i] + c;
          t1[i] = (u32)x;
          c = (u32)(x >> 32);
        }
        csub_c<N>(t1, c, m);
      }
    }
    mul_n<N, Strict>(t2, t1, t1, m, minv);
    mul_n<N, Strict>(t3, t2, t1, m, minv);
  }
  // the aligned bit pairs of d, top down; pairs never straddle a word
  u32 x[N];
  bool started = false;
#pragma unroll
  for (int wi = N - 1; wi >= 0; --wi) {
    if (32 * wi > dtop) continue;
    const u32 dw = d[wi];
    const int top = (32 * wi + 31 > dtop) ? (dtop & 31) : 31;
    for (int b = top | 1; b >= 1; b -= 2) {
      const u32 w = (dw >> (b - 1)) & 3u;
      if (started) {
        mul_n<N, Strict>(x, x, x, m, minv);
        mul_n<N, Strict>(x, x, x, m, minv);
        if (b2) {  // canonical first, then doublings mod m stay below m
          if (w) csub_n<N>(x, m);
          for (u32 k = 0; k < w; ++k) dbl_n<N>(x, m);
        } else if (w) {
          u32 y[N];
          sel_n<N>(y, w, t1, t2, t3);
          mul_n<N, Strict>(x, x, y, m, minv);
        }
      } else {
        started = true;
        if (b2) {
#pragma unroll
          for (int i = 0; i < N; ++i) x[i] = one[i];
          for (u32 k = 0; k < w; ++k) dbl_n<N>(x, m);
        } else {
          sel_n<N>(x, w, t1, t2, t3);
        }
      }
    }
  }
  u32 mone[N];
  sub_n<N>(mone, m, one);
  csub_n<N>(x, m);
  if (eq_n<N>(x, one) || eq_n<N>(x, mone)) return true;
  for (int r = 1; r < s; ++r) {
    mul_n<N, Strict>(x, x, x, m, minv);
    csub_n<N>(x, m);
    if (eq_n<N>(x, mone)) return true;
  }
  return false;
}

// The strong test of a value of 2^62 or more (three 64-bit limbs) to base
// a, on N = ceil((bits + 2) / 32) 32-bit words, which keeps 4m < R, or on
// six words with canonical residues for 191 and 192 bits.  Kept
// out of line, with scalars in and out, so the common one-word path of the
// callers keeps its registers: returns the algorithmic IMADs << 1 | pass.
__device__ __noinline__ u64 strong_wide(u64 w0, u64 w1, u64 w2, u32 a) {
  u32 w[6] = {(u32)w0, (u32)(w0 >> 32), (u32)w1, (u32)(w1 >> 32), (u32)w2,
              (u32)(w2 >> 32)};
  int bl = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i)
    if (w[i]) bl = 32 * i + 32 - __clz(w[i]);
  const int n = (bl + 2 + 31) >> 5;
  u64 im = 0;
  bool pass;
  if (n <= 3) pass = strong_n<3>(w, a, &im);
  else if (n == 4) pass = strong_n<4>(w, a, &im);
  else if (n == 5) pass = strong_n<5>(w, a, &im);
  else if (n == 6) pass = strong_n<6>(w, a, &im);
  else pass = strong_n<6, true>(w, a, &im);
  return (im << 1) | (pass ? 1ull : 0ull);
}

// One strong test of v to base kMrBases[bi] (bi = 0 is base 2), for a v
// that trial division left undecided (odd, above 37, no factor <= 37).
// Values below 2^62 take one 64-bit word, larger ones strong_wide.
__device__ __forceinline__ bool sprp_strong(const V3& v, int bi, u64* imad) {
  const u32 a = kMrBases[bi];
  if (v.w[1] == 0 && v.w[2] == 0 && v.w[0] < (1ull << 62))
    return strong64(v.w[0], a, imad);
  const u64 r = strong_wide(v.w[0], v.w[1], v.w[2], a);
  *imad += r >> 1;
  return (r & 1) != 0;
}

// One base of huntlib's test: the trial division, then the strong test.
__device__ __forceinline__ bool sprp_step(const V3& v, int bi, u64* imad) {
  const int t = sprp_trial(v);
  if (t != 2) return t == 1;
  return sprp_strong(v, bi, imad);
}

// mr_is_prime (base2_only = false) or sprp_base2 (true).
__device__ __forceinline__ bool sprp(const V3& v, bool base2_only, u64* imad) {
  const int t = sprp_trial(v);
  if (t != 2) return t == 1;
  const int nb = base2_only ? 1 : 7;
  for (int bi = 0; bi < nb; ++bi)
    if (!sprp_strong(v, bi, imad)) return false;
  return true;
}

// The six bases after 2 (v already passed base 2 and trial division).
__device__ __forceinline__ bool sprp_rest(const V3& v, u64* imad) {
  const int t = sprp_trial(v);
  if (t != 2) return t == 1;
  for (int bi = 1; bi < 7; ++bi)
    if (!sprp_strong(v, bi, imad)) return false;
  return true;
}

}  // namespace fk
