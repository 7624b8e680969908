// fk_mont32.cuh -- GENERATED by gen_mont32.py; do not edit by hand.
//
// The multiply-accumulate pass of CIOS Montgomery multiplication on 32-bit
// limbs: t[0..N+1] += a[0..N-1] * x in one carry chain (low halves into
// words 0..N-1, high halves into words 1..N, carries into N and N+1).
// Method: Koc, Acar, Kaliski, IEEE Micro 1996 (CIOS).
#pragma once
#include "fk_arith.cuh"

namespace fk {

template <int N>
struct Mont32;


template <>
struct Mont32<2> {
  // t[0..3] += a * x
  static __device__ __forceinline__ void mac(u32* t, const u32* a, u32 x) {
    asm("mad.lo.cc.u32 %0, %4, %6, %0;\n\tmadc.lo.cc.u32 %1, %5, %6, %1;\n\taddc.cc.u32 %2, %2, 0;\n\taddc.u32 %3, %3, 0;\n\tmad.hi.cc.u32 %1, %4, %6, %1;\n\tmadc.hi.cc.u32 %2, %5, %6, %2;\n\taddc.u32 %3, %3, 0;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3])
        : "r"(a[0]), "r"(a[1]), "r"(x));
  }
};

template <>
struct Mont32<3> {
  // t[0..4] += a * x
  static __device__ __forceinline__ void mac(u32* t, const u32* a, u32 x) {
    asm("mad.lo.cc.u32 %0, %5, %8, %0;\n\tmadc.lo.cc.u32 %1, %6, %8, %1;\n\tmadc.lo.cc.u32 %2, %7, %8, %2;\n\taddc.cc.u32 %3, %3, 0;\n\taddc.u32 %4, %4, 0;\n\tmad.hi.cc.u32 %1, %5, %8, %1;\n\tmadc.hi.cc.u32 %2, %6, %8, %2;\n\tmadc.hi.cc.u32 %3, %7, %8, %3;\n\taddc.u32 %4, %4, 0;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(x));
  }
};

template <>
struct Mont32<4> {
  // t[0..5] += a * x
  static __device__ __forceinline__ void mac(u32* t, const u32* a, u32 x) {
    asm("mad.lo.cc.u32 %0, %6, %10, %0;\n\tmadc.lo.cc.u32 %1, %7, %10, %1;\n\tmadc.lo.cc.u32 %2, %8, %10, %2;\n\tmadc.lo.cc.u32 %3, %9, %10, %3;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.u32 %5, %5, 0;\n\tmad.hi.cc.u32 %1, %6, %10, %1;\n\tmadc.hi.cc.u32 %2, %7, %10, %2;\n\tmadc.hi.cc.u32 %3, %8, %10, %3;\n\tmadc.hi.cc.u32 %4, %9, %10, %4;\n\taddc.u32 %5, %5, 0;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(x));
  }
};

template <>
struct Mont32<5> {
  // t[0..6] += a * x
  static __device__ __forceinline__ void mac(u32* t, const u32* a, u32 x) {
    asm("mad.lo.cc.u32 %0, %7, %12, %0;\n\tmadc.lo.cc.u32 %1, %8, %12, %1;\n\tmadc.lo.cc.u32 %2, %9, %12, %2;\n\tmadc.lo.cc.u32 %3, %10, %12, %3;\n\tmadc.lo.cc.u32 %4, %11, %12, %4;\n\taddc.cc.u32 %5, %5, 0;\n\taddc.u32 %6, %6, 0;\n\tmad.hi.cc.u32 %1, %7, %12, %1;\n\tmadc.hi.cc.u32 %2, %8, %12, %2;\n\tmadc.hi.cc.u32 %3, %9, %12, %3;\n\tmadc.hi.cc.u32 %4, %10, %12, %4;\n\tmadc.hi.cc.u32 %5, %11, %12, %5;\n\taddc.u32 %6, %6, 0;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(x));
  }
};

template <>
struct Mont32<6> {
  // t[0..7] += a * x
  static __device__ __forceinline__ void mac(u32* t, const u32* a, u32 x) {
    asm("mad.lo.cc.u32 %0, %8, %14, %0;\n\tmadc.lo.cc.u32 %1, %9, %14, %1;\n\tmadc.lo.cc.u32 %2, %10, %14, %2;\n\tmadc.lo.cc.u32 %3, %11, %14, %3;\n\tmadc.lo.cc.u32 %4, %12, %14, %4;\n\tmadc.lo.cc.u32 %5, %13, %14, %5;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.u32 %7, %7, 0;\n\tmad.hi.cc.u32 %1, %8, %14, %1;\n\tmadc.hi.cc.u32 %2, %9, %14, %2;\n\tmadc.hi.cc.u32 %3, %10, %14, %3;\n\tmadc.hi.cc.u32 %4, %11, %14, %4;\n\tmadc.hi.cc.u32 %5, %12, %14, %5;\n\tmadc.hi.cc.u32 %6, %13, %14, %6;\n\taddc.u32 %7, %7, 0;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(x));
  }
};


}  // namespace fk
