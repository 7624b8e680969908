// fk_mark_k.cuh -- the marking-sieve variants of one wheel family: the
// per-family launchers of fk_launch.h, instantiated for P0 = FK_MARK_P0 by
// fk_mark_k6.cu ... fk_mark_k11.cu (one translation unit per family, so
// the 36 variants compile in parallel).
#pragma once
#include "fk_launch.h"
#include "fk_mark.cuh"

namespace fk {
namespace mark_detail {

template <int P0, int NS, int SEG>
size_t smem() {
  return pat_bytes<P0, NS>() + sizeof(MarkSmem<SEG>);
}

template <int P0, int NS, int SEG>
cudaError_t limit() {
  return cudaFuncSetAttribute(k_mark<P0, NS, SEG>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem<P0, NS, SEG>());
}

template <int P0, int NS, int SEG>
cudaError_t launch(u32 grid, cudaStream_t s, const SieveArgs& a) {
  k_mark<P0, NS, SEG><<<grid, kBlock, smem<P0, NS, SEG>(), s>>>(a);
  return cudaGetLastError();
}

template <int P0, int NS>
size_t smem_seg(u32 SEG) {
  return SEG == 16384 ? smem<P0, NS, 16384>()
                      : SEG == 65536 ? smem<P0, NS, 65536>()
                                     : smem<P0, NS, 32768>();
}

template <int P0, int NS>
cudaError_t limits_seg() {
  cudaError_t r = limit<P0, NS, 16384>();
  if (r == cudaSuccess) r = limit<P0, NS, 32768>();
  if (r == cudaSuccess) r = limit<P0, NS, 65536>();
  return r;
}

template <int P0, int NS>
cudaError_t launch_seg(u32 SEG, u32 grid, cudaStream_t s, const SieveArgs& a) {
  switch (SEG) {
    case 16384: return launch<P0, NS, 16384>(grid, s, a);
    case 65536: return launch<P0, NS, 65536>(grid, s, a);
    default: return launch<P0, NS, 32768>(grid, s, a);
  }
}

}  // namespace mark_detail

template <int P0>
size_t mark_smem_p0(u32 NS, u32 SEG) {
  using namespace mark_detail;
  return NS == 24 ? smem_seg<P0, 24>(SEG)
                  : NS == 40 ? smem_seg<P0, 40>(SEG) : smem_seg<P0, 32>(SEG);
}

template <int P0>
cudaError_t mark_limits_p0() {
  using namespace mark_detail;
  cudaError_t r = limits_seg<P0, 24>();
  if (r == cudaSuccess) r = limits_seg<P0, 32>();
  if (r == cudaSuccess) r = limits_seg<P0, 40>();
  return r;
}

template <int P0>
cudaError_t mark_launch_p0(u32 NS, u32 SEG, u32 grid, cudaStream_t s,
                           const SieveArgs& a) {
  using namespace mark_detail;
  switch (NS) {
    case 24: return launch_seg<P0, 24>(SEG, grid, s, a);
    case 40: return launch_seg<P0, 40>(SEG, grid, s, a);
    default: return launch_seg<P0, 32>(SEG, grid, s, a);
  }
}

template size_t mark_smem_p0<FK_MARK_P0>(u32, u32);
template cudaError_t mark_limits_p0<FK_MARK_P0>();
template cudaError_t mark_launch_p0<FK_MARK_P0>(u32, u32, u32, cudaStream_t,
                                                const SieveArgs&);

}  // namespace fk
