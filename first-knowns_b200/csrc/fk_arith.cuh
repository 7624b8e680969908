// fk_arith.cuh -- integer arithmetic shared by the sieve and SPRP kernels.
//
// Barrett reduction by a u32 prime (Barrett 1986) with the magic
// floor(2^64 / q), as huntlib/gpu.py:33-36 describes it, and the
// compile-time prime table the pattern sieve bakes its constants from.
#pragma once
#include <cstdint>

typedef unsigned long long u64;
typedef unsigned int u32;
typedef unsigned __int128 u128;

#if defined(__CUDACC__)
#define FK_HD __host__ __device__ __forceinline__
#else
#define FK_HD inline
#endif

FK_HD u64 fk_mulhi64(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (u64)(((u128)a * b) >> 64);
#endif
}

// v mod q for v < 2^64 and 2 <= q < 2^30.  With magic = floor(2^64/q),
// qhat = floor(v*magic / 2^64) >= floor(v/q) - 1, so the remainder before
// the correction is below 2q < 2^31 and one conditional subtract finishes.
FK_HD u32 fk_bmod(u64 v, u32 q, u64 magic) {
  u64 qh = fk_mulhi64(v, magic);
  u32 r = (u32)v - (u32)qh * q;
  return r >= q ? r - q : r;
}

// (a * b) mod q for a, b < q < 2^30.
FK_HD u32 fk_mulmod(u32 a, u32 b, u32 q, u64 magic) {
  return fk_bmod((u64)a * b, q, magic);
}

// x mod q for a 128-bit x, given c64 = 2^64 mod q.
FK_HD u32 fk_bmod128(u64 lo, u64 hi, u32 q, u64 magic, u32 c64) {
  u32 h = fk_bmod(hi, q, magic);
  u32 l = fk_bmod(lo, q, magic);
  u32 t = fk_bmod((u64)h * c64 + l, q, magic);
  return t;
}

// The i-th prime (0 -> 2), evaluated at compile time for the pattern
// sieve's baked constants.
__host__ __device__ constexpr u32 fk_nth_prime(int i) {
  u32 c = 1;
  int k = -1;
  while (k < i) {
    ++c;
    bool pr = c >= 2;
    for (u32 d = 2; d * d <= c; ++d)
      if (c % d == 0) { pr = false; break; }
    if (pr) ++k;
  }
  return c;
}

// 64^-1 mod q for an odd prime q, at compile time: the pattern tables are
// stored in the order of 64-period steps, so a word's table index is its
// phase times this inverse.
__host__ __device__ constexpr u32 fk_inv64(u32 q) {
  u32 x = 1;
  while ((64u * x) % q != 1u) ++x;
  return x;
}

// Word offset of pattern prime I (counted from prime index P0) in the
// concatenated pattern table: the sum of the I primes before it.
__host__ __device__ constexpr u32 fk_pat_prefix(int P0, int I) {
  u32 s = 0;
  for (int k = 0; k < I; ++k) s += fk_nth_prime(P0 + k);
  return s;
}
