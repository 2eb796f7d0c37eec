// Stable LSD radix sort of 32-bit keys with 32-bit values, for the
// particle sort of mass assignment.  The reference's MassAssignor merge-sorts
// each buffer of particles by x before its slab-parallel scatter
// (cc/particle_mesh/mass_assignor.h:137-148, merge_sort_omp.h); here the
// particles are ordered by scatter unit, and a stable sort keeps each cell's
// particles in input order, so the grid is the same bits on every run.
//
// Each pass sorts by one digit of up to kMaxBits bits in three steps, with
// no inter-block waits:
//   upsweep   one block per tile of kSortTile keys counts the tile's digits
//             into a count matrix laid out digit-major (cnt[d * ntiles + t]);
//   scan      an exclusive scan of the whole matrix in that order gives, for
//             every (digit, tile), the first output position of the tile's
//             keys of that digit;
//   downsweep one block per tile ranks its keys stably by digit (each warp
//             takes a contiguous segment of the tile in rounds of 32, in
//             order, with running per-warp digit counters), stages them in
//             shared memory in digit order and writes each digit's run to
//             its output position in coalesced stores.
// The first pass takes implicit values (the key's own index), so the key
// kernel writes no index array.  Keys equal to `invalid` (particles outside
// the grid) take a digit of their own above every other in each pass, so
// they end last whatever their bits, and the passes cover only the bits of
// the valid keys.  Peers of equal digits within a warp are found with one
// ballot per digit bit.
#pragma once

#include <cstdint>

namespace fc {
namespace radix {

constexpr int kSortThreads = 512;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per tile
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kMaxBits = 10;
constexpr int kMaxBins = 1 << kMaxBits;
constexpr int kBinsCap = kMaxBins + 1;  // digits and the invalid keys' digit
constexpr int kRow = kMaxBins + 2;      // 16-bit counters per warp row
constexpr int kScanPer = (kBinsCap + kSortThreads - 1) / kSortThreads;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kSortThreads * kScanItems;  // matrix entries per scan block

// Passes and digit width for valid keys whose bits [begin_bit, end_bit)
// vary.
struct SortPlan {
  int passes = 0;
  int bits = 0;
  int64_t ntiles = 0;
  int64_t m = 0;        // count-matrix entries: ((1 << bits) + 1) * ntiles
  int64_t nchunks = 0;  // scan blocks over the matrix
  size_t scratch_bytes() const {
    return (size_t)(m + nchunks + 64) * sizeof(uint32_t);
  }
};

inline SortPlan sort_plan(int64_t n, int begin_bit, int end_bit) {
  SortPlan p;
  const int nbits = end_bit - begin_bit > 0 ? end_bit - begin_bit : 1;
  p.passes = (nbits + kMaxBits - 1) / kMaxBits;
  p.bits = (nbits + p.passes - 1) / p.passes;
  p.ntiles = n > 0 ? (n + kSortTile - 1) / kSortTile : 0;
  p.m = ((int64_t(1) << p.bits) + 1) * p.ntiles;
  p.nchunks = (p.m + kScanChunk - 1) / kScanChunk;
  return p;
}

// Dynamic shared memory of the downsweep: per-warp digit counters (16-bit),
// the tile's digit starts and output positions, the staged keys and values.
constexpr size_t kDownSmem = (size_t)kSortWarps * kRow * sizeof(uint16_t) +
                             2 * (size_t)kBinsCap * sizeof(uint32_t) +
                             2 * (size_t)kSortTile * sizeof(uint32_t);

// Exclusive prefix sum over a block of kSortThreads threads; sh holds 32
// words.  Every thread must call it.
__device__ __forceinline__ uint32_t sort_block_scan(uint32_t v, uint32_t *sh,
                                                    uint32_t *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kSortWarps ? sh[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kSortWarps) sh[lane] = w;
  }
  __syncthreads();
  const uint32_t before = warp ? sh[warp - 1] : 0u;
  if (total) *total = sh[kSortWarps - 1];
  __syncthreads();  // sh may be reused by the caller's next scan
  return before + x - v;
}

// The digit of a key in a pass: (key >> shift) & mask, or mask + 1 for the
// invalid key.
__device__ __forceinline__ uint32_t sort_digit(uint32_t key, uint32_t invalid,
                                               int shift, uint32_t mask) {
  return key == invalid ? mask + 1u : (key >> shift) & mask;
}

// Upsweep: the digit counts of tile blockIdx.x into cnt[d * ntiles + t].
__global__ void __launch_bounds__(kSortThreads)
    k_sort_upsweep(const uint32_t *__restrict__ keys, int64_t n, uint32_t invalid,
                   int shift, int bits, int64_t ntiles,
                   uint32_t *__restrict__ cnt) {
  __shared__ uint32_t h[kBinsCap];
  const int bins = 1 << bits;
  const int nd = bins + 1;
  const uint32_t mask = (uint32_t)bins - 1u;
  for (int b = threadIdx.x; b < nd; b += kSortThreads) h[b] = 0u;
  __syncthreads();
  const int64_t t = blockIdx.x;
  const int64_t base = t * kSortTile;
  const int cnt_tile = (int)min((int64_t)kSortTile, n - base);
  uint32_t k[kSortItems];
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const int i = threadIdx.x + j * kSortThreads;
    k[j] = i < cnt_tile ? keys[base + i] : 0u;
  }
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const int i = threadIdx.x + j * kSortThreads;
    if (i < cnt_tile) atomicAdd(&h[sort_digit(k[j], invalid, shift, mask)], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nd; b += kSortThreads)
    cnt[(int64_t)b * ntiles + t] = h[b];
}

// Scan step 1: the sum of each chunk of kScanChunk matrix entries.
__global__ void __launch_bounds__(kSortThreads)
    k_sort_scan_reduce(const uint32_t *__restrict__ a, int64_t m,
                       uint32_t *__restrict__ sums) {
  __shared__ uint32_t sh[32];
  const int64_t base = (int64_t)blockIdx.x * kScanChunk;
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const int64_t i = base + threadIdx.x + j * kSortThreads;
    if (i < m) s += a[i];
  }
  uint32_t total = 0;
  sort_block_scan(s, sh, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Scan step 2 (one block): exclusive scan of the chunk sums in place.
__global__ void __launch_bounds__(kSortThreads)
    k_sort_scan_top(uint32_t *__restrict__ sums, int64_t nchunks) {
  __shared__ uint32_t sh[32];
  uint32_t carry = 0;
  for (int64_t b0 = 0; b0 < nchunks; b0 += kSortThreads) {
    const int64_t i = b0 + threadIdx.x;
    const uint32_t v = i < nchunks ? sums[i] : 0u;
    uint32_t total = 0;
    const uint32_t ex = sort_block_scan(v, sh, &total);
    if (i < nchunks) sums[i] = carry + ex;
    carry += total;
  }
}

// Scan step 3: each chunk's entries become exclusive prefix sums, in place.
// Thread t holds kScanItems consecutive entries.
__global__ void __launch_bounds__(kSortThreads)
    k_sort_scan_apply(uint32_t *__restrict__ a, int64_t m,
                      const uint32_t *__restrict__ sums) {
  __shared__ uint32_t sh[32];
  const int64_t base = (int64_t)blockIdx.x * kScanChunk +
                       (int64_t)threadIdx.x * kScanItems;
  static_assert(kScanItems == 8, "two 16-byte accesses per thread");
  const bool whole = base + kScanItems <= m;  // base is 32-byte aligned
  uint32_t v[kScanItems];
  if (whole) {
    const uint4 x = *reinterpret_cast<const uint4 *>(a + base);
    const uint4 y = *reinterpret_cast<const uint4 *>(a + base + 4);
    v[0] = x.x, v[1] = x.y, v[2] = x.z, v[3] = x.w;
    v[4] = y.x, v[5] = y.y, v[6] = y.z, v[7] = y.w;
  } else {
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) v[j] = base + j < m ? a[base + j] : 0u;
  }
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) s += v[j];
  uint32_t run = sums[blockIdx.x] + sort_block_scan(s, sh, nullptr);
  uint32_t o[kScanItems];
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    o[j] = run;
    run += v[j];
  }
  if (whole) {
    *reinterpret_cast<uint4 *>(a + base) = make_uint4(o[0], o[1], o[2], o[3]);
    *reinterpret_cast<uint4 *>(a + base + 4) = make_uint4(o[4], o[5], o[6], o[7]);
  } else {
#pragma unroll
    for (int j = 0; j < kScanItems; ++j)
      if (base + j < m) a[base + j] = o[j];
  }
}

// Downsweep: tile blockIdx.x's keys (and values; implicit indices when
// vals_in is null) to their stable sorted positions by sort_digit.  off is
// the scanned count matrix.  BITS is the pass's digit width.
template <int BITS>
__global__ void __launch_bounds__(kSortThreads, 2)
    k_sort_downsweep(const uint32_t *__restrict__ keys_in,
                     const uint32_t *__restrict__ vals_in, int64_t n,
                     uint32_t invalid, int shift, int64_t ntiles,
                     const uint32_t *__restrict__ off,
                     uint32_t *__restrict__ keys_out,
                     uint32_t *__restrict__ vals_out) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint16_t *wc = reinterpret_cast<uint16_t *>(sm);  // [kSortWarps][kRow]
  uint32_t *lstart = sm + kSortWarps * kRow / 2;      // [kBinsCap]
  uint32_t *gstart = lstart + kBinsCap;               // [kBinsCap]: then
                                                      // output - staged position
  uint32_t *skeys = gstart + kBinsCap;                // [kSortTile]
  uint32_t *svals = skeys + kSortTile;                // [kSortTile]
  __shared__ uint32_t sh[32];
  constexpr int bins = 1 << BITS;
  constexpr int nd = bins + 1;
  constexpr uint32_t mask = (uint32_t)bins - 1u;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t t = blockIdx.x;
  const int64_t base = t * kSortTile;
  const int cnt_tile = (int)min((int64_t)kSortTile, n - base);
  // Warp w's items are [w * 32 * kSortItems, (w + 1) * 32 * kSortItems) of
  // the tile, in rounds of 32: the tile's order is (warp, round, lane).
  const int wbase = warp * 32 * kSortItems;
  uint16_t *mine = wc + warp * kRow;
  for (int b = lane; b < nd; b += 32) mine[b] = 0;
  uint32_t k[kSortItems], v[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int i = wbase + r * 32 + lane;
    k[r] = i < cnt_tile ? keys_in[base + i] : 0u;
  }
  __syncwarp();
  uint32_t rk[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int i = wbase + r * 32 + lane;
    const bool valid = i < cnt_tile;
    const uint32_t d = valid ? sort_digit(k[r], invalid, shift, mask) : 0u;
    // Lanes holding the same digit: bits 0 .. BITS of d (bit BITS marks
    // the invalid keys' digit), one ballot each.
    unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int q = 0; q <= BITS; ++q) {
      const unsigned bit = (d >> q) & 1u;
      peers &= __ballot_sync(0xffffffffu, bit) ^ (bit - 1u);
    }
    const int leader = valid ? __ffs(peers) - 1 : lane;
    uint32_t b = 0;
    if (valid && lane == leader) {
      b = mine[d];
      mine[d] = (uint16_t)(b + __popc(peers));
    }
    b = __shfl_sync(0xffffffffu, b, leader);
    rk[r] = b + __popc(peers & lt);
    __syncwarp();
  }
  // The values are read now, in flight while the digits are counted.
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int i = wbase + r * 32 + lane;
    v[r] = i < cnt_tile ? (vals_in ? vals_in[base + i] : (uint32_t)(base + i)) : 0u;
  }
  __syncthreads();
  // Per digit: each warp's first rank among the tile's keys of the digit,
  // the tile's count of the digit, and its output position.
  for (int b = threadIdx.x; b < nd; b += kSortThreads) {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = wc[w * kRow + b];
      wc[w * kRow + b] = (uint16_t)run;
      run += c;
    }
    lstart[b] = run;
    gstart[b] = off[(int64_t)b * ntiles + t];
  }
  __syncthreads();
  // Tile-local digit starts: thread t scans digits [kScanPer t, kScanPer (t + 1)).
  {
    const int b0 = kScanPer * threadIdx.x;
    uint32_t c[kScanPer], s = 0;
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) {
      c[j] = b0 + j < nd ? lstart[b0 + j] : 0u;
      s += c[j];
    }
    uint32_t ex = sort_block_scan(s, sh, nullptr);
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) {
      if (b0 + j < nd) {
        lstart[b0 + j] = ex;
        gstart[b0 + j] -= ex;  // modulo 2^32: output = staged + this
      }
      ex += c[j];
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int i = wbase + r * 32 + lane;
    if (i < cnt_tile) {
      const uint32_t d = sort_digit(k[r], invalid, shift, mask);
      const uint32_t lp = lstart[d] + wc[warp * kRow + d] + rk[r];
      skeys[lp] = k[r];
      svals[lp] = v[r];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < cnt_tile; i += kSortThreads) {
    const uint32_t key = skeys[i];
    const uint32_t d = sort_digit(key, invalid, shift, mask);
    const uint32_t gp = gstart[d] + (uint32_t)i;
    keys_out[gp] = key;
    vals_out[gp] = svals[i];
  }
}

using DownsweepFn = void (*)(const uint32_t *, const uint32_t *, int64_t,
                             uint32_t, int, int64_t, const uint32_t *,
                             uint32_t *, uint32_t *);

// The downsweep for a digit width of 1 .. kMaxBits bits.
inline DownsweepFn downsweep_kernel(int bits) {
  switch (bits) {
    case 1: return k_sort_downsweep<1>;
    case 2: return k_sort_downsweep<2>;
    case 3: return k_sort_downsweep<3>;
    case 4: return k_sort_downsweep<4>;
    case 5: return k_sort_downsweep<5>;
    case 6: return k_sort_downsweep<6>;
    case 7: return k_sort_downsweep<7>;
    case 8: return k_sort_downsweep<8>;
    case 9: return k_sort_downsweep<9>;
    case 10: return k_sort_downsweep<10>;
    default: return nullptr;
  }
}
static_assert(kMaxBits == 10, "one downsweep instance per digit width");

}  // namespace radix
}  // namespace fc
