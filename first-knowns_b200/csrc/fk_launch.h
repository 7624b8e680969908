// fk_launch.h -- launchers of the sieve kernels' template variants.
//
// k_sieve<P0, NS, DYN> and k_mark<P0, NS, SEG> come in one variant per
// wheel family P0 (6, 7, 9, 11), pattern-prime count NS (24, 32, 40), for
// the rounds kernel with or without warps claiming blocks of chains (DYN),
// and for the marking sieve per segment length SEG (16384, 32768, 65536
// periods): 24 and 36 kernels.  They are instantiated in their own translation units
// (fk_sieve_k.cu, fk_mark_k6.cu ... fk_mark_k11.cu), which the build
// compiles in parallel, and reached through the plain functions below.
#pragma once
#include <cuda_runtime.h>

#include "fk_sieve.cuh"

namespace fk {

// The variant values; anything else is rejected by the tuning checks
// before a launch.
inline bool valid_pattern_primes(u32 ns) {
  return ns == 24 || ns == 32 || ns == 40;
}
inline bool valid_mark_segment(u32 seg) {
  return seg == 16384 || seg == 32768 || seg == 65536;
}
inline int seg_index(u32 seg) {
  return seg == 16384 ? 0 : (seg == 65536 ? 2 : 1);
}

// Dynamic shared bytes a variant launches with.
size_t sieve_smem_bytes(u32 P0, u32 NS);
size_t mark_smem_bytes(u32 P0, u32 NS, u32 SEG);

// Raise every variant's dynamic shared-memory limit on the current device.
cudaError_t sieve_set_smem_limits();
cudaError_t mark_set_smem_limits();

// Launch one variant: grid CTAs of kBlock threads on stream s.  Returns
// the launch's error (cudaGetLastError).
cudaError_t launch_sieve(u32 P0, u32 NS, u32 grid, cudaStream_t s,
                         const SieveArgs& a);
cudaError_t launch_mark(u32 P0, u32 NS, u32 SEG, u32 grid, cudaStream_t s,
                        const SieveArgs& a);

// Per-family halves of the marking launchers (one translation unit each).
template <int P0>
size_t mark_smem_p0(u32 NS, u32 SEG);
template <int P0>
cudaError_t mark_limits_p0();
template <int P0>
cudaError_t mark_launch_p0(u32 NS, u32 SEG, u32 grid, cudaStream_t s,
                           const SieveArgs& a);

}  // namespace fk
