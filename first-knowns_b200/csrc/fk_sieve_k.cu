// fk_sieve_k.cu -- the pattern-sieve kernel variants k_sieve<P0, NS, DYN>
// and the dispatch of every sieve launch (fk_launch.h).
#include "fk_launch.h"

namespace fk {
namespace {

template <int P0, int NS>
size_t sieve_smem() {
  return pat_bytes<P0, NS>() + sizeof(SieveSmem);
}

template <int P0, int NS>
cudaError_t sieve_limit() {
  cudaError_t r = cudaFuncSetAttribute(
      k_sieve<P0, NS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
      (int)sieve_smem<P0, NS>());
  if (r != cudaSuccess) return r;
  return cudaFuncSetAttribute(k_sieve<P0, NS, true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sieve_smem<P0, NS>());
}

// Eight blocks per task is one per warp: the variant without the shared
// counter; more blocks per task take the claiming variant.
template <int P0, int NS>
cudaError_t sieve_launch(u32 grid, cudaStream_t s, const SieveArgs& a) {
  if (a.warp_tasks == kBlock / 32)
    k_sieve<P0, NS, false><<<grid, kBlock, sieve_smem<P0, NS>(), s>>>(a);
  else
    k_sieve<P0, NS, true><<<grid, kBlock, sieve_smem<P0, NS>(), s>>>(a);
  return cudaGetLastError();
}

template <int P0>
size_t sieve_smem_ns(u32 NS) {
  return NS == 24 ? sieve_smem<P0, 24>()
                  : NS == 40 ? sieve_smem<P0, 40>() : sieve_smem<P0, 32>();
}

template <int P0>
cudaError_t sieve_limits_p0() {
  cudaError_t r = sieve_limit<P0, 24>();
  if (r == cudaSuccess) r = sieve_limit<P0, 32>();
  if (r == cudaSuccess) r = sieve_limit<P0, 40>();
  return r;
}

template <int P0>
cudaError_t sieve_launch_ns(u32 NS, u32 grid, cudaStream_t s,
                            const SieveArgs& a) {
  switch (NS) {
    case 24: return sieve_launch<P0, 24>(grid, s, a);
    case 40: return sieve_launch<P0, 40>(grid, s, a);
    default: return sieve_launch<P0, 32>(grid, s, a);
  }
}

}  // namespace

size_t sieve_smem_bytes(u32 P0, u32 NS) {
  switch (P0) {
    case 6: return sieve_smem_ns<6>(NS);
    case 7: return sieve_smem_ns<7>(NS);
    case 9: return sieve_smem_ns<9>(NS);
    default: return sieve_smem_ns<11>(NS);
  }
}

size_t mark_smem_bytes(u32 P0, u32 NS, u32 SEG) {
  switch (P0) {
    case 6: return mark_smem_p0<6>(NS, SEG);
    case 7: return mark_smem_p0<7>(NS, SEG);
    case 9: return mark_smem_p0<9>(NS, SEG);
    default: return mark_smem_p0<11>(NS, SEG);
  }
}

cudaError_t sieve_set_smem_limits() {
  cudaError_t r = sieve_limits_p0<6>();
  if (r == cudaSuccess) r = sieve_limits_p0<7>();
  if (r == cudaSuccess) r = sieve_limits_p0<9>();
  if (r == cudaSuccess) r = sieve_limits_p0<11>();
  return r;
}

cudaError_t mark_set_smem_limits() {
  cudaError_t r = mark_limits_p0<6>();
  if (r == cudaSuccess) r = mark_limits_p0<7>();
  if (r == cudaSuccess) r = mark_limits_p0<9>();
  if (r == cudaSuccess) r = mark_limits_p0<11>();
  return r;
}

cudaError_t launch_sieve(u32 P0, u32 NS, u32 grid, cudaStream_t s,
                         const SieveArgs& a) {
  switch (P0) {
    case 6: return sieve_launch_ns<6>(NS, grid, s, a);
    case 7: return sieve_launch_ns<7>(NS, grid, s, a);
    case 9: return sieve_launch_ns<9>(NS, grid, s, a);
    default: return sieve_launch_ns<11>(NS, grid, s, a);
  }
}

cudaError_t launch_mark(u32 P0, u32 NS, u32 SEG, u32 grid, cudaStream_t s,
                        const SieveArgs& a) {
  switch (P0) {
    case 6: return mark_launch_p0<6>(NS, SEG, grid, s, a);
    case 7: return mark_launch_p0<7>(NS, SEG, grid, s, a);
    case 9: return mark_launch_p0<9>(NS, SEG, grid, s, a);
    default: return mark_launch_p0<11>(NS, SEG, grid, s, a);
  }
}

}  // namespace fk
