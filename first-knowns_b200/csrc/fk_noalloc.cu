// fk_noalloc.cu -- fk_sieve_noalloc: the pre-primality sieve of one
// interval for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc when they sweep: a real-time loop
// whose memory budget is fixed up front, a host framework that owns every
// allocation through its own pool and forbids the library from growing
// the heap behind its back, or code that must not trigger the implicit
// synchronisation an allocation can cause.  fk_sieve (fk_engine.cu) grows
// its buffers on demand; this entry point instead keeps every piece of
// per-call scratch -- the item descriptor, the base-residue table, the
// candidate list, the counters and the ordering buffers -- in one fixed array
// in device memory, declared below, and writes its result into buffers
// the caller owns.  It calls no cudaMalloc, cudaFree or other allocating
// routine; the engine's own tables were uploaded when the engine was
// created.
//
// Limits (rejected with FK_ERR_DOMAIN and a message before any launch):
//   * at most kMaxPrimes sieve primes (q2 up to about 821,000);
//   * the interval must fit one device item (periods * M below 2^55, the
//     same bound fk_sieve cuts its items at: item_periods_max), on top of
//     the domain checks every sweep applies (check_interval);
// the current device must be the one the engine was created on
// (FK_ERR_DEVICE otherwise, before any launch); and at run time the
// caller's count receives, instead of a result,
//   UINT64_MAX      more than kMaxCand pre-primality survivors, or more
//                   than the caller's capacity (split the interval);
//   UINT64_MAX - 1  a bounded device wait gave up (the pattern staging);
//                   splitting the interval does not help -- the device is
//                   stalled or faulty.
//
// Sharing: every call, from any thread, uses the same array on a given
// device, and the array keeps the previous call's contents; each call
// clears its counters first.  Two calls whose work overlaps on the GPU
// (different streams, or different host threads) race on the array and
// both results are undefined.  Serialize them, e.g. on one stream.
//
// Set-up: the first call on a device, with that device current, looks up
// the array's device address (cudaGetSymbolAddress) and sets the sieve
// kernels' shared-memory limits; make that first call before any stream
// capture is active.  Every GPU that loads the library holds the array
// (kScratchBytes, about 5.3 MiB) until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fk.h"
#include "fk_internal.h"
#include "fk_launch.h"
#include "fk_sieve.cuh"

using namespace fk;

namespace {

constexpr uint64_t kMaxCand = 1ull << 18;   // survivors one call may emit
constexpr uint32_t kMaxPrimes = 1u << 16;   // sieve primes of the engine

// byte layout of the scratch array
constexpr size_t kOffCtr = 0;
constexpr size_t kOffTaskCtr = 256;
constexpr size_t kOffItem = 512;
constexpr size_t kOffEngine = 1024;
constexpr size_t kOffPrefix = 2048;
constexpr size_t kOffIndex = 2304;
constexpr size_t kOffXq = 4096;
constexpr size_t kOffKey = kOffXq + 4ull * kMaxPrimes;
constexpr size_t kOffCandItem = kOffKey + 8ull * kMaxCand;
constexpr size_t kOffSort = kOffCandItem + 4ull * kMaxCand;
// ordering: survivors are bucketed by key range (key >> shift, kNaBuckets
// buckets), scattered into the sort region bucket by bucket, and each
// bucket is sorted in shared memory by its own CTA
constexpr uint32_t kNaBuckets = 2048;
constexpr size_t kOffBucketCnt = kOffSort + 8ull * kMaxCand;
constexpr size_t kOffBucketStart = kOffBucketCnt + 4ull * kNaBuckets;
constexpr size_t kOffBucketFill = kOffBucketStart + 4ull * kNaBuckets;
constexpr size_t kScratchBytes = kOffBucketFill + 4ull * kNaBuckets;

static_assert(sizeof(DevCounters) <= kOffTaskCtr - kOffCtr, "layout");
static_assert(sizeof(DevItem) <= kOffEngine - kOffItem, "layout");
static_assert(sizeof(DevEngine) <= kOffPrefix - kOffEngine, "layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char* g_scratch_addr[64] = {nullptr};

template <typename T>
T* at(unsigned char* base, size_t off) {
  return reinterpret_cast<T*>(base + off);
}

// Writes this call's descriptors into the scratch array and zeroes its
// counters (the array keeps the last call's contents otherwise).
__global__ void k_na_init(unsigned char* s, DevEngine eng, DevItem item,
                          unsigned long long ntask) {
  u32* cnt = reinterpret_cast<u32*>(s + kOffBucketCnt);
  for (u32 b = threadIdx.x; b < kNaBuckets; b += blockDim.x) cnt[b] = 0u;
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    DevCounters* c = reinterpret_cast<DevCounters*>(s + kOffCtr);
    *c = DevCounters{};
    *reinterpret_cast<unsigned long long*>(s + kOffTaskCtr) = 0ull;
    *reinterpret_cast<DevItem*>(s + kOffItem) = item;
    *reinterpret_cast<DevEngine*>(s + kOffEngine) = eng;
    u64* pre = reinterpret_cast<u64*>(s + kOffPrefix);
    pre[0] = 0;
    pre[1] = ntask;
    *reinterpret_cast<u32*>(s + kOffIndex) = 0u;
  }
}

// X0 mod q for every sieve prime of the call's item, into the array.
__global__ void k_na_xq(unsigned char* s) {
  const DevItem* it = reinterpret_cast<const DevItem*>(s + kOffItem);
  const DevEngine* e = reinterpret_cast<const DevEngine*>(s + kOffEngine);
  u32* xq = reinterpret_cast<u32*>(s + kOffXq);
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < e->NP;
       i += gridDim.x * blockDim.x) {
    const PrimeRec pr = e->recs[i];
    xq[i] = fk_bmod128(it->X0_lo, it->X0_hi, pr.q, pr.magic, e->c64[i]);
  }
}

// The call's outcome once the sieve is done: 0 the survivors fit, 1 too
// many (more than kMaxCand or than the caller's capacity), 2 the pattern
// staging gave up a bounded wait.
__device__ __forceinline__ int na_outcome(const unsigned char* s,
                                          u64 capacity) {
  const DevCounters* c = reinterpret_cast<const DevCounters*>(s + kOffCtr);
  if (c->overflow & 4u) return 2;
  const u64 n = c->ncand;
  if (n > kMaxCand || n > capacity || (c->overflow & 1u)) return 1;
  return 0;
}

// Survivors per bucket: bucket (key - lo_shift) >> shift, i.e. by the
// offset from the caller's lo.
__global__ void __launch_bounds__(kBlock) k_na_count(unsigned char* s,
                                                     u64 capacity, u64 lo_shift,
                                                     u32 shift) {
  if (na_outcome(s, capacity)) return;
  const u64 n = reinterpret_cast<const DevCounters*>(s + kOffCtr)->ncand;
  const u64* key = reinterpret_cast<const u64*>(s + kOffKey);
  u32* cnt = reinterpret_cast<u32*>(s + kOffBucketCnt);
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 b = (key[i] - lo_shift) >> shift;
    atomicAdd(&cnt[b < kNaBuckets ? b : kNaBuckets - 1], 1u);
  }
}

// Exclusive scan of the bucket counts (one CTA): each bucket's first slot
// in the sort region, twice (start, and the fill cursor the scatter
// advances).
__global__ void __launch_bounds__(kBlock) k_na_scan(unsigned char* s,
                                                    u64 capacity) {
  if (na_outcome(s, capacity)) return;
  constexpr u32 per = kNaBuckets / kBlock;
  const u32* cnt = reinterpret_cast<const u32*>(s + kOffBucketCnt);
  u32* start = reinterpret_cast<u32*>(s + kOffBucketStart);
  u32* fill = reinterpret_cast<u32*>(s + kOffBucketFill);
  __shared__ u32 warp_sum[kBlock / 32];
  const u32 t = threadIdx.x, lane = t & 31, w = t >> 5;
  u32 local[per];
  u32 sum = 0;
#pragma unroll
  for (u32 k = 0; k < per; ++k) {
    local[k] = cnt[t * per + k];
    sum += local[k];
  }
  // inclusive scan of the per-thread sums: within the warp, then across
  u32 inc = sum;
#pragma unroll
  for (u32 d = 1; d < 32; d <<= 1) {
    const u32 o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) warp_sum[w] = inc;
  __syncthreads();
  u32 before = 0;
  for (u32 k = 0; k < w; ++k) before += warp_sum[k];
  u32 at = before + inc - sum;
#pragma unroll
  for (u32 k = 0; k < per; ++k) {
    start[t * per + k] = at;
    fill[t * per + k] = at;
    at += local[k];
  }
}

// Survivor keys into their buckets' slots of the sort region.
__global__ void __launch_bounds__(kBlock) k_na_scatter(unsigned char* s,
                                                       u64 capacity,
                                                       u64 lo_shift,
                                                       u32 shift) {
  if (na_outcome(s, capacity)) return;
  const u64 n = reinterpret_cast<const DevCounters*>(s + kOffCtr)->ncand;
  const u64* key = reinterpret_cast<const u64*>(s + kOffKey);
  u32* fill = reinterpret_cast<u32*>(s + kOffBucketFill);
  u64* buf = reinterpret_cast<u64*>(s + kOffSort);
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 k = key[i];
    const u64 b = (k - lo_shift) >> shift;
    buf[atomicAdd(&fill[b < kNaBuckets ? b : kNaBuckets - 1], 1u)] = k;
  }
}

// Sorts the c keys at `a` ascending, by one CTA (shared or device
// memory).  A bitonic network in the form whose blocks all sort upward
// (the first step of each merge compares mirror positions i and
// i ^ (k - 1)); positions at or past c act as +infinity and their
// compare-exchanges are skipped, so c need not be a power of two.
__device__ void na_sort(u64* a, u32 c) {
  for (u32 k = 2; (k >> 1) < c; k <<= 1) {
    for (u32 j = k >> 1; j > 0; j >>= 1) {
      for (u32 i = threadIdx.x; i < c; i += blockDim.x) {
        if (i & j) continue;
        const u32 l = j == (k >> 1) ? i ^ (k - 1) : i | j;
        if (l < c) {
          const u64 x = a[i], y = a[l];
          if (x > y) {
            a[i] = y;
            a[l] = x;
          }
        }
      }
      __syncthreads();
    }
  }
}

// One CTA per bucket: the bucket's keys sorted in shared memory (in place
// in the sort region when the bucket outgrows the tile) and written, as
// offsets from the caller's lo, to the caller's buffer at the bucket's
// start.  Buckets hold disjoint, increasing key ranges, so the
// concatenation is the sorted stream.
__global__ void __launch_bounds__(kBlock) k_na_finish(
    unsigned char* s, u64* out, u64 capacity, u64* count, u64 lo_shift) {
  const int outcome = na_outcome(s, capacity);
  if (outcome) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
      *count = outcome == 2 ? ~0ull - 1 : ~0ull;
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0)
    *count = reinterpret_cast<const DevCounters*>(s + kOffCtr)->ncand;
  u64* buf = reinterpret_cast<u64*>(s + kOffSort);
  __shared__ u64 tile[kSortSmem];
  for (u32 b = blockIdx.x; b < kNaBuckets; b += gridDim.x) {
    const u32 c = reinterpret_cast<const u32*>(s + kOffBucketCnt)[b];
    if (c == 0) continue;
    const u32 at0 = reinterpret_cast<const u32*>(s + kOffBucketStart)[b];
    u64* a = tile;
    if (c <= (u32)kSortSmem) {
      for (u32 i = threadIdx.x; i < c; i += blockDim.x) tile[i] = buf[at0 + i];
    } else {
      a = buf + at0;
    }
    __syncthreads();
    na_sort(a, c);
    for (u32 i = threadIdx.x; i < c; i += blockDim.x)
      out[at0 + i] = a[i] - lo_shift;
    __syncthreads();
  }
}

}  // namespace

extern "C" fk_status fk_sieve_noalloc(fk_engine* e, const uint64_t lo[2],
                                      const uint64_t hi[2], uint64_t* d_offsets,
                                      uint64_t capacity, uint64_t* d_count,
                                      void* stream) {
  if (!e || !lo || !hi || !d_offsets || !d_count)
    return set_error(FK_ERR_ARG, "fk_sieve_noalloc: null argument");
  const EngineView v = engine_view(e);
  if (v.NP > kMaxPrimes)
    return set_error(FK_ERR_DOMAIN,
                     "fk_sieve_noalloc: the engine has more than 65536 sieve "
                     "primes (q2 too deep for the fixed scratch array)");
  const u128 L0 = ((u128)lo[1] << 64) | lo[0];
  const u128 H0 = ((u128)hi[1] << 64) | hi[0];
  if (H0 <= L0)
    return set_error(FK_ERR_DOMAIN, "fk_sieve_noalloc: empty interval");
  fk_status cs = check_interval(e, lo, hi, 0, false);
  if (cs) return cs;
  const u64 M = v.M;
  const u128 X0 = L0 / M * M;
  const u128 periods = (H0 - X0 + M - 1) / M;
  if (periods > (u128)item_periods_max(M))
    return set_error(FK_ERR_DOMAIN,
                     "fk_sieve_noalloc: interval too long for one call "
                     "(periods * M must stay below 2^55)");
  // the engine's tables must live on the current device
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return set_error(FK_ERR_DEVICE, cudaGetErrorString(ce));
  {
    char msg[192];
    if (check_engine_device(v.device, dev, msg, sizeof msg))
      return set_error(FK_ERR_DEVICE, msg);
  }
  // per-device set-up: the array's device address and kernel attributes
  if (dev < 0 || dev >= 64) return set_error(FK_ERR_DEVICE, "device index above 63");
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (ce != cudaSuccess)
        return set_error(FK_ERR_DEVICE, cudaGetErrorString(ce));
      const cudaError_t r = sieve_set_smem_limits();
      if (r != cudaSuccess) return set_error(FK_ERR_DEVICE, cudaGetErrorString(r));
      g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    base = g_scratch_addr[dev];
  }
  int nsm = 0;
  ce = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (ce != cudaSuccess) return set_error(FK_ERR_DEVICE, cudaGetErrorString(ce));
  // the one device item: the same line geometry the batch pipeline uses
  const u64 U = (u64)periods;
  DevItem it{};
  it.engine = 0;
  it.mode = MODE_SIEVE;
  it.X0_lo = (u64)X0;
  it.X0_hi = (u64)(X0 >> 64);
  it.U = U;
  it.lo_off = (u64)(L0 - X0);
  it.hi_last = (u64)(H0 - (X0 + (u128)(U - 1) * M));
  const u64 words = (U + 63) / 64;
  const u64 target = (u64)nsm * 2 * kBlock * 4;
  u64 tc = (words * v.L + target - 1) / target;
  tc = tc < 1 ? 1 : (tc > 256 ? 256 : tc);
  it.Tc = (u32)tc;
  it.lane_threads = 1;  // one lane per thread, Tc consecutive words
  it.nchunk = (words + tc - 1) / tc;
  const u64 ntask = (it.nchunk * v.L + kBlock - 1) / kBlock;
  it.ntask = ntask;
  it.xq_off = 0;
  it.marked = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_na_init<<<1, kBlock, 0, s>>>(base, v.dev, it, ntask);
  k_na_xq<<<64, kBlock, 0, s>>>(base);
  SieveArgs a{};
  a.engines = at<DevEngine>(base, kOffEngine);
  a.items = at<DevItem>(base, kOffItem);
  a.task_prefix = at<u64>(base, kOffPrefix);
  a.item_index = at<u32>(base, kOffIndex);
  a.nitems = 1;
  a.ntask = ntask;
  a.xq = at<u32>(base, kOffXq);
  a.cand_key = at<u64>(base, kOffKey);
  a.cand_item = at<u32>(base, kOffCandItem);
  a.cand_cap = kMaxCand;
  a.ctr = at<DevCounters>(base, kOffCtr);
  a.task_ctr = at<unsigned long long>(base, kOffTaskCtr);
  a.warp_queue = kWarpMode;
  a.seg_per_task = kSegPerTask;
  a.warp_tasks = kBlock / 32;  // ntask above counts kBlock chains per task
  const u32 grid = (u32)(ntask < (u64)nsm * 2 ? ntask : (u64)nsm * 2);
  // the engine's own descriptor is the default variant: kNS pattern primes
  ce = launch_sieve(v.P0, kNS, grid, s, a);
  if (ce != cudaSuccess) return set_error(FK_ERR_DEVICE, cudaGetErrorString(ce));
  const u64 lo_shift = (u64)(L0 - X0);
  // bucket = (key - lo_shift) >> shift over the interval's length: at
  // most kNaBuckets buckets, spread evenly over [lo, hi)
  const u64 span = (u64)(H0 - L0);
  u32 shift = 0;
  while (((span - 1) >> shift) >= kNaBuckets) ++shift;
  const u32 sgrid = (u32)nsm * 2;
  k_na_count<<<sgrid, kBlock, 0, s>>>(base, capacity, lo_shift, shift);
  k_na_scan<<<1, kBlock, 0, s>>>(base, capacity);
  k_na_scatter<<<sgrid, kBlock, 0, s>>>(base, capacity, lo_shift, shift);
  k_na_finish<<<sgrid, kBlock, 0, s>>>(base, reinterpret_cast<u64*>(d_offsets),
                                       capacity,
                                       reinterpret_cast<u64*>(d_count),
                                       lo_shift);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return set_error(FK_ERR_DEVICE, cudaGetErrorString(ce));
  return FK_OK;
}
