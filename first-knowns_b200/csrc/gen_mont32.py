"""Generate fk_mont32.cuh: CIOS Montgomery multiplication on 32-bit limbs
with PTX carry chains, one specialization per limb count N = 2..6.

    python first-knowns_b200/csrc/gen_mont32.py

Each pass (t += a * b_i, then t += q * m and the one-word shift) is a single
asm statement, so the carry flag never crosses a statement boundary: the
low halves of the N products go in with mad.lo.cc / madc.lo.cc, the high
halves one word up with mad.hi.cc / madc.hi.cc, and the chain ends in the
two top words.  Method: Koc, Acar, Kaliski, "Analyzing and comparing
Montgomery multiplication algorithms", IEEE Micro 1996 (CIOS).
"""

import pathlib

HERE = pathlib.Path(__file__).resolve().parent


def pass_code(n, name_a):
    """asm body for t[0..n+1] += A[0..n-1] * x, with t %0..%(n+1),
    A %(n+2)..%(2n+1), x %(2n+2)."""
    t = [f"%{i}" for i in range(n + 2)]
    a = [f"%{n + 2 + i}" for i in range(n)]
    x = f"%{2 * n + 2}"
    lines = []
    for j in range(n):
        op = "mad.lo.cc.u32" if j == 0 else "madc.lo.cc.u32"
        lines.append(f"{op} {t[j]}, {a[j]}, {x}, {t[j]};")
    lines.append(f"addc.cc.u32 {t[n]}, {t[n]}, 0;")
    lines.append(f"addc.u32 {t[n + 1]}, {t[n + 1]}, 0;")
    for j in range(n):
        op = "mad.hi.cc.u32" if j == 0 else "madc.hi.cc.u32"
        lines.append(f"{op} {t[j + 1]}, {a[j]}, {x}, {t[j + 1]};")
    lines.append(f"addc.u32 {t[n + 1]}, {t[n + 1]}, 0;")
    return lines


def asm_block(n, lines, arr):
    body = "\\n\\t".join(lines)
    outs = ", ".join(f'"+r"(t[{i}])' for i in range(n + 2))
    ins = ", ".join(f'"r"({arr}[{i}])' for i in range(n)) + ', "r"(x)'
    return f'    asm("{body}"\n        : {outs}\n        : {ins});'


def spec(n):
    out = []
    out.append(f"template <>\nstruct Mont32<{n}> {{")
    out.append(f"  // t[0..{n + 1}] += a * x")
    out.append(f"  static __device__ __forceinline__ void mac(u32* t, const u32* a, u32 x) {{")
    out.append(asm_block(n, pass_code(n, "a"), "a"))
    out.append("  }")
    out.append("};")
    return "\n".join(out)


def main():
    parts = ['''// fk_mont32.cuh -- GENERATED by gen_mont32.py; do not edit by hand.
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
''']
    for n in range(2, 7):
        parts.append(spec(n))
    parts.append("\n}  // namespace fk\n")
    (HERE / "fk_mont32.cuh").write_text("\n\n".join(parts))


if __name__ == "__main__":
    main()
