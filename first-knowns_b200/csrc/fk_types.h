// fk_types.h -- device-side descriptors shared by host and kernels.
#pragma once
#include <cstdint>

namespace fk {

enum Kind : uint32_t { KIND_EULER = 0, KIND_DICKSON = 1, KIND_AP = 2 };

// What an item asks for.
enum Mode : uint32_t {
  MODE_SIEVE = 0,   // pre-primality survivors only
  MODE_HUNT = 1,    // survivors classified; keep depth >= threshold
  MODE_DENSE = 2,   // no sieve: every x in the range is classified
};

// Per-prime record for the per-candidate stage (16 bytes).
struct PrimeRec {
  uint32_t q;
  uint32_t aux;     // kind test data (see fk_engine.cu, build_tests)
  uint64_t magic;   // floor(2^64 / q)
};

constexpr int kBlock = 256;       // threads per CTA, every kernel
constexpr int kQcap = 4096;       // candidate queue entries per CTA (8 warps)
constexpr int kNS = 32;           // pattern primes per CTA (default)
constexpr int kNSMin = 24;        // fewest pattern primes a kernel variant
                                  // stages; marking tables start here
constexpr int kNSMax = 40;        // most: the engine's pattern tables hold
                                  // this many primes
constexpr int kMaxRounds = 64;
constexpr int kSortSmem = 4096;   // entries a CTA sorts in shared memory
constexpr int kClassChunk = 128;  // candidates a warp fetches at once
constexpr int kBucketFill = 1024; // expected entries per ordering bucket
constexpr int kWarpMode = 32;     // warp queue below which a candidate
                                  // takes a whole warp
constexpr int kSeg = 32768;       // marking: periods per shared segment
                                  // (default; variants 16384 and 65536)
constexpr int kNumSeg = 3;        // marking segment variants
constexpr int kSegOf(int i) { return 16384 << i; }
constexpr int kSegPerTask = 8;    // marking: segments per task
constexpr int kMarkPrimes = 6528; // marking: most primes one engine marks,
                                  // counted from pattern prime kNSMin
                                  // (every prime from 7 to 2^16 fits)
constexpr int kMarkHits = 16;     // marking: least hits per work entry

// Immutable per-engine tables (device-resident for the engine's life).
struct DevEngine {
  uint32_t kind, n, L, NP;        // NP: sieve primes (pattern + per-candidate)
  uint32_t P0, NS, nrounds, xxmax;  // NS: pattern primes of this batch's
                                    // kernel variant (kNSMin..kNSMax)
  uint32_t pat_words, sbits_words, two_pass, pad0;
  uint64_t M;                     // wheel period (x units)
  uint64_t W;                     // Dickson: k = W * j
  uint64_t d_lo, d_hi;            // AP difference
  const uint64_t* lanes;          // [L] admissible residues mod M, ascending
  // pattern words, compile-time layout: prime q's table holds q words,
  // entry k = the kill mask of the 64 periods from phase 64k mod q, so
  // consecutive words of a lane are consecutive entries
  const uint64_t* pat;
  const uint32_t* pat_minv;       // [kNSMax] (M mod q)^-1 * 64^-1 mod q
  const uint32_t* pat_i64;        // [kNSMax] 64^-1 mod q
  const PrimeRec* recs;           // [NP]
  const uint32_t* c64;            // [NP] 2^64 mod q
  const uint32_t* lists;          // explicit forbidden-residue lists
  const uint64_t* hmask;          // [NP] Dickson: bit (h mod 64) set for
                                  // each half residue h on the prime's list
  const uint32_t* rounds;         // [nrounds + 1] prime-index cuts
  const uint32_t* sbits;          // Euler: bitset of {x^2 + x : x < n}
  // marking sieve (long lanes): primes [NS, NPm) are marked in a per-lane
  // byte map; G lists hold each prime's forbidden residues of the PERIOD
  // u for lane offset 0 (f * (M mod q)^-1 mod q)
  uint32_t NPm, use_mark;
  uint32_t nmitems;               // marking work entries of this batch
  uint32_t nm2, nm1;              // entries before the first prime with
                                  // q >= SEG / 2 (at most two hits per
                                  // segment) and with q >= SEG (at most
                                  // one); both relative to mitems
  uint32_t pad3;
  const uint32_t* minv_all;       // [NP] (M mod q)^-1 mod q
  const uint32_t* gaux;           // [NP] offset | count << 24 into glist
  const uint32_t* glist;
  // tables of this batch's segment length SEG (one set per variant):
  // [NPm - kNSMin] per prime from index kNSMin: q | (SEG mod q) << 16
  const uint64_t* mq;
  // [nmitems] work entries g | (prime - kNSMin) << 16 | sub-range k << 29 |
  // q << 32 | S << 48: the hits u = g (mod q), shifted by the lane, of one
  // forbidden period residue g inside sub-range k of length S (a multiple
  // of q; S = 0 when the entry covers the whole segment), one 8-byte load
  // per entry; ordered by prime, and the batch's pointer starts at the
  // first prime past its pattern primes
  const uint64_t* mitems;
};

// One unit of work: a sub-range of one engine's line.
struct DevItem {
  uint32_t engine, mode, threshold, cap;
  uint64_t X0_lo, X0_hi;          // line base (a multiple of M for sieves)
  uint64_t U;                     // periods (sieve) or x count (dense)
  uint64_t lo_off;                // first valid x - X0 (in period 0)
  uint64_t hi_last;               // valid iff R < hi_last in period U-1
  uint32_t Tc;                    // words per chain (per thread)
  uint32_t lane_threads;          // threads sweeping one lane: 1, 8 or 32;
                                  // thread t of a group takes words t,
                                  // t + lane_threads, ... of its block
  uint64_t nchunk;                // chains per lane
  uint64_t task0, ntask;          // first task, task count
  uint64_t xq_off;                // this item's base-residue table
  uint32_t marked, pad2;          // 1: the marking kernel sweeps this item
  uint64_t nchunk_u;              // marking: u-chunks per lane
};

// Output entry before ordering: item index + (key << 8 | depth).
struct OutRec {
  uint64_t packed;
  uint32_t item;
  uint32_t pad;
};

struct DevCounters {
  unsigned long long task_next;   // persistent task counter
  unsigned long long ncand;       // candidates written
  unsigned long long nout;        // outputs written
  unsigned int overflow;          // bit 0 cand, bit 1 out, bit 2 timeout,
                                  // bit 3 value past 192 bits
  unsigned int pad;
  unsigned long long s1_words;    // pattern-sieve words processed
  unsigned long long s2_tests;    // per-candidate prime tests
  unsigned long long imad_alg;    // algorithmic IMADs of the SPRP stage
  unsigned long long sprp_values; // values strong-tested
  unsigned long long marks;       // marking-sieve byte marks
  unsigned long long class_next;  // SPRP stage: next candidate chunk
};

}  // namespace fk
