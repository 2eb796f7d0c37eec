// fc_assign.cu -- MassAssignor on the GPU: radix sort by cell, then a
// deterministic tiled stencil scatter.
//
// Reference: cc/particle_mesh/mass_assignor.h:30-234 (buffering, counters,
// sort, coloured slab scatter), distribution_functions.h:17-236 (NGP, TSC,
// D12 stencils), d12.h:13-155 (D12 table), config_space_grid.h:31-46
// (survey -> grid coordinates).  Cloud-in-cell (scheme 3) is new.
//
// Pipeline per flush:
//   K-key     grid coordinates, skip/wrap, tile-major cell key, counters
//   K-sort    CUB radix sort of (key, particle index): stable, so the order
//             of particles inside a cell is their input order
//   K-units   first sorted position of every scatter unit (binary search)
//             and, per colour, the list of non-empty units
//   K-scatter NGP/CIC/TSC: persistent CTAs per colour pass draw 2x8x8-cell
//             units; a thread per home cell sums its particles' stencil
//             products in registers, and the footprint (unit + stencil
//             halo) takes the home cells' sums in W^3 ordered rounds.  D12
//             (8^3 taps): one CTA per 8^3 tile; particles are staged in
//             shared memory with their 1-D weights and every footprint cell
//             sums its contributions in a fixed order (home cell, then
//             sorted particle order).  Either way each footprint total is
//             added to the grid once.  Units are processed in colour passes
//             chosen so that footprints within one pass never overlap, so
//             there are no atomics on the grid and the result is
//             bit-reproducible run to run.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "fc_common.cuh"
#include "fc_internal.h"
#include "fc_sort.cuh"

#if __has_include("_gen/d12_table.inc")
#define FC_HAVE_D12 1
#else
#define FC_HAVE_D12 0
#endif

namespace fc {
namespace {

constexpr int kTile = 8;         // tile edge in cells
constexpr int kTileCells = 512;  // cells per tile
// A scatter unit with more particles than this is drawn before the others
// of its colour pass (a quarter of the narrow stencils' staging chunk).
constexpr uint32_t kHeavyUnit = 128;
constexpr int kScatterThreads = 256;
constexpr int kChunk = 256;      // particles staged per shared-memory chunk

#if FC_HAVE_D12
// Transposed D12 table wave[sub * 8 + offset] (d12.h:149-155), generated at
// build time from the reference header.
__constant__ double c_wave[8 * 64] = {
#include "_gen/d12_table.inc"
};
#else
__constant__ double c_wave[8 * 64];
#endif

struct AssignGeom {
  int n[3];
  int nt[3];  // tiles per axis
  double posmin[3];
  double cell;
  double rcell;  // 1 / cell, correctly rounded
  int fast_div;  // cell and rcell are in [2^-400, 2^400]
  int periodic;
};

// a / g.cell, correctly rounded.  For |a| in [2^-400, 2^400] and a cell in
// the same range the quotient is formed from the correctly rounded
// reciprocal with one fused residual correction (Markstein, IBM J. Res.
// Dev. 34(1), 1990: q = a*r, e = fma(-q, cell, a), q + e*r rounds to
// nearest), which is the IEEE quotient; elsewhere it is a plain division.
__device__ __forceinline__ double div_cell(double a, const AssignGeom &g) {
  const double m = fabs(a);
  if (g.fast_div && m >= 0x1p-400 && m <= 0x1p400) {
    const double q = a * g.rcell;
    return fma(fma(-q, g.cell, a), g.rcell, q);
  }
  return a / g.cell;
}

// config_space_grid.h:31-46 on the device.
__device__ __forceinline__ bool dev_grid_coords(const double *p,
                                                const AssignGeom &g,
                                                double x[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double xi = div_cell(p[i] - g.posmin[i], g);
    const double xmax = (double)g.n[i];
    if (xi < 0 || xi >= xmax) {
      if (!g.periodic) return false;
      xi = fmod(xi, xmax);
      if (xi < 0) xi += xmax;
    }
    x[i] = xi;
  }
  return true;
}

// floor(x) as a cell index.  A periodically wrapped coordinate can round up
// to exactly n, which is the periodic image of 0: cell 0 with offset 0, as
// the reference's wrapped stencil indices place it.  Offsets within the cell
// are x - floor(x).
__device__ __forceinline__ int home_cell(double x, int n) {
  int i = (int)floor(x);
  return i >= n ? i - n : (i < 0 ? 0 : i);
}

// 1-D stencil weights per scheme; the particle weight is folded into the x
// weights as the reference does (distribution_functions.h:73-81, 191-205).
template <int S>
struct Stencil;

template <>
struct Stencil<0> {  // nearest cell
  static constexpr int W = 1, OMIN = 0;
  __device__ static void weights(double rx, double ry, double rz, double w,
                                 double *wx, double *wy, double *wz) {
    wx[0] = w;
    wy[0] = 1.0;
    wz[0] = 1.0;
  }
};

template <>
struct Stencil<1> {  // triangular shaped cloud, offsets -1..1
  static constexpr int W = 3, OMIN = -1;
  __device__ static void weights(double rx, double ry, double rz, double w,
                                 double *wx, double *wy, double *wz) {
    wx[0] = 0.5 * (1 - rx) * (1 - rx) * w;
    wx[1] = (0.5 + rx - rx * rx) * w;
    wx[2] = 0.5 * rx * rx * w;
    wy[0] = 0.5 * (1 - ry) * (1 - ry);
    wy[1] = 0.5 + ry - ry * ry;
    wy[2] = 0.5 * ry * ry;
    wz[0] = 0.5 * (1 - rz) * (1 - rz);
    wz[1] = 0.5 + rz - rz * rz;
    wz[2] = 0.5 * rz * rz;
  }
};

template <>
struct Stencil<2> {  // D12 wavelet, offsets -1..6, 64 sub-cell samples
  static constexpr int W = 8, OMIN = -1;
  __device__ static void weights(double rx, double ry, double rz, double w,
                                 double *wx, double *wy, double *wz) {
    const int sx = min((int)floor(rx * 64), 63);
    const int sy = min((int)floor(ry * 64), 63);
    const int sz = min((int)floor(rz * 64), 63);
#pragma unroll
    for (int o = 0; o < 8; ++o) {
      wx[o] = c_wave[sx * 8 + o] * w;
      wy[o] = c_wave[sy * 8 + o];
      wz[o] = c_wave[sz * 8 + o];
    }
  }
};

template <>
struct Stencil<3> {  // cloud in cell (trilinear), offsets 0..1
  static constexpr int W = 2, OMIN = 0;
  __device__ static void weights(double rx, double ry, double rz, double w,
                                 double *wx, double *wy, double *wz) {
    wx[0] = (1 - rx) * w;
    wx[1] = rx * w;
    wy[0] = 1 - ry;
    wy[1] = ry;
    wz[0] = 1 - rz;
    wz[1] = rz;
  }
};

// K-key: one key per particle of [base, base+n) plus counters.
template <typename KeyT>
__global__ void k_keys(const double *posw, int64_t base, int64_t n,
                       AssignGeom g, KeyT invalid_key, KeyT *keys,
                       uint32_t *vals, double *partials,
                       unsigned long long *counts) {
  __shared__ double red[32];
  double sw = 0.0, sw2 = 0.0;
  unsigned long long added = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pi = base + i;
    const double *p = posw + 4 * pi;
    double x[3];
    KeyT key = invalid_key;
    if (dev_grid_coords(p, g, x)) {
      const int ix = home_cell(x[0], g.n[0]);
      const int iy = home_cell(x[1], g.n[1]);
      const int iz = home_cell(x[2], g.n[2]);
      const KeyT tile =
          ((KeyT)(ix >> 3) * g.nt[1] + (KeyT)(iy >> 3)) * g.nt[2] + (iz >> 3);
      key = tile * kTileCells + (KeyT)((ix & 7) * 64 + (iy & 7) * 8 + (iz & 7));
      const double w = p[3];
      sw += w;
      sw2 += w * w;
      ++added;
    }
    keys[pi] = key;
    if (vals) vals[pi] = (uint32_t)pi;
  }
  // Integer counts are exact whatever the order.
  unsigned long long a = added;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0 && a) atomicAdd(&counts[0], a);
  sw = block_sum(sw, red);
  sw2 = block_sum(sw2, red);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = sw;
    partials[2 * blockIdx.x + 1] = sw2;
  }
}

// Folds the K-key block partials into the running totals in block order.
__global__ void k_fold_totals(const double *partials, int nparts,
                              double *totals) {
  __shared__ double red[32];
  double s = 0.0, q = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    s += partials[2 * i];
    q += partials[2 * i + 1];
  }
  s = block_sum(s, red);
  q = block_sum(q, red);
  if (threadIdx.x == 0) {
    totals[0] += s;
    totals[1] += q;
  }
}

// Packs (n,3) positions with per-particle or constant weights into posw.
__global__ void k_pack(const double *pos, const double *w, double wconst,
                       int64_t n, double *posw) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    posw[4 * i + 0] = pos[3 * i + 0];
    posw[4 * i + 1] = pos[3 * i + 1];
    posw[4 * i + 2] = pos[3 * i + 2];
    posw[4 * i + 3] = w ? w[i] : wconst;
  }
}

// K-units: start[u] = first sorted index whose key >= u * unit_cells, for
// u in [0, nunits]; invalid keys (== nunits * unit_cells) sort last.
template <typename KeyT>
__global__ void k_unit_starts(const KeyT *keys, int64_t n, int64_t nunits,
                              int unit_cells, uint32_t *start) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t <= nunits;
       t += (int64_t)gridDim.x * blockDim.x) {
    const KeyT target = (KeyT)t * (KeyT)unit_cells;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < target)
        lo = mid + 1;
      else
        hi = mid;
    }
    start[t] = (uint32_t)lo;
  }
}

// The non-empty units of every colour as (unit, first particle, end),
// packed at the front of the colour's slice of `ranges`; cnt[c] counts
// them.  `units` lists the units in colour order, colour c owning
// [coff[c], coff[c + 1]).  The order inside a slice does not matter: units
// of one colour have disjoint footprints.
__global__ void k_unit_ranges(const uint32_t *__restrict__ units, int64_t nu,
                              const uint32_t *__restrict__ start,
                              const int64_t *__restrict__ coff, int ncolors,
                              unsigned *__restrict__ cnt,
                              uint4 *__restrict__ ranges) {
  // The loop is warp-uniform so that the lanes of a warp that hold
  // non-empty units of the same colour and class take their slots with one
  // atomic.  Units of more than kHeavyUnit particles fill the colour's slice
  // from its end (counter cnt[2 ncolors + c]), the others from its start
  // (cnt[c]); the scatter draws the heavy ones first, so that no long unit
  // starts near the end of a pass.
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < nu;
       i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    uint32_t u = 0, ts = 0, te = 0;
    int c = 0;
    if (i < nu) {
      u = units[i];
      ts = start[u];
      te = start[u + 1];
      while (c + 1 < ncolors && i >= coff[c + 1]) ++c;
    }
    const bool ne = i < nu && ts < te;
    const unsigned act = __ballot_sync(0xffffffffu, ne);
    if (!ne) continue;
    const bool heavy = te - ts > kHeavyUnit;
    const unsigned grp = __match_any_sync(act, 2 * c + (heavy ? 1 : 0));
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(grp) - 1;
    unsigned *ctr = heavy ? &cnt[2 * ncolors + c] : &cnt[c];
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(ctr, (unsigned)__popc(grp));
    base = __shfl_sync(grp, base, leader);
    const unsigned slot = base + (unsigned)__popc(grp & ((1u << lane) - 1u));
    const int64_t at = heavy ? coff[c + 1] - 1 - (int64_t)slot : coff[c] + slot;
    ranges[at] = make_uint4(u, ts, te, 0u);
  }
}

// Unit i of a colour pass: the heavy units (nh of them, stored from the
// slice's end backwards) first, then the others from the slice's start.
__device__ __forceinline__ uint4 pass_unit(const uint4 *__restrict__ front,
                                           const uint4 *__restrict__ back,
                                           unsigned nh, unsigned i) {
  return i < nh ? back[-1 - (int64_t)i] : front[i - nh];
}

// Exclusive prefix sum over the block (blockDim.x a multiple of 32, at most
// 1024); sh32 holds 32 words.  Every thread must call it.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v,
                                                         uint32_t *sh32) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh32[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    uint32_t w = lane < nw ? sh32[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) sh32[lane] = w;
  }
  __syncthreads();
  const uint32_t before = warp ? sh32[warp - 1] : 0u;
  return before + x - v;
}

// K-scatter for one colour pass.  Shared memory layout:
//   acc[F^3] footprint sums | wts[kChunk][3W] | pcell[kChunk] | cstart[513]
template <int S, typename KeyT, typename GT>
__global__ void __launch_bounds__(kScatterThreads)
    k_scatter(const double *__restrict__ posw, const KeyT *__restrict__ keys,
              const uint32_t *__restrict__ vals,
              const uint32_t *__restrict__ tile_start,
              const uint32_t *__restrict__ tiles, AssignGeom g,
              GT *__restrict__ grid) {
  constexpr int W = Stencil<S>::W;
  constexpr int OMIN = Stencil<S>::OMIN;
  constexpr int F = kTile + W - 1;
  constexpr int F3 = F * F * F;
  extern __shared__ double smem[];
  double *acc = smem;
  double *wts = acc + F3;
  int *pcell = reinterpret_cast<int *>(wts + kChunk * 3 * W);
  int *cstart = pcell + kChunk;

  const uint32_t tile = tiles[blockIdx.x];
  const uint32_t ts = tile_start[tile];
  const uint32_t te = tile_start[tile + 1];
  if (ts >= te) return;
  const int tz = tile % g.nt[2];
  const int ty = (tile / g.nt[2]) % g.nt[1];
  const int tx = tile / (g.nt[2] * g.nt[1]);
  const int o0 = tx * kTile, o1 = ty * kTile, o2 = tz * kTile;

  for (int f = threadIdx.x; f < F3; f += blockDim.x) acc[f] = 0.0;

  for (uint32_t c0 = ts; c0 < te; c0 += kChunk) {
    const int nch = (int)min((uint32_t)kChunk, te - c0);
    __syncthreads();
    if ((int)threadIdx.x < nch) {
      const uint32_t idx = vals[c0 + threadIdx.x];
      const double *p = posw + 4 * (size_t)idx;
      double x[3];
      dev_grid_coords(p, g, x);
      pcell[threadIdx.x] = (int)(keys[c0 + threadIdx.x] & (kTileCells - 1));
      double *wt = wts + threadIdx.x * 3 * W;
      Stencil<S>::weights(x[0] - floor(x[0]), x[1] - floor(x[1]),
                          x[2] - floor(x[2]), p[3], wt, wt + W, wt + 2 * W);
    }
    __syncthreads();
    for (int c = threadIdx.x; c <= kTileCells; c += blockDim.x) {
      int lo = 0, hi = nch;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (pcell[mid] < c)
          lo = mid + 1;
        else
          hi = mid;
      }
      cstart[c] = lo;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < F3; f += blockDim.x) {
      const int fx = f / (F * F);
      const int fy = (f / F) % F;
      const int fz = f % F;
      double a = acc[f];
      const int hx0 = max(0, fx - (W - 1)), hx1 = min(kTile - 1, fx);
      const int hy0 = max(0, fy - (W - 1)), hy1 = min(kTile - 1, fy);
      const int hz0 = max(0, fz - (W - 1)), hz1 = min(kTile - 1, fz);
      for (int hx = hx0; hx <= hx1; ++hx) {
        const int ox = fx - hx;
        for (int hy = hy0; hy <= hy1; ++hy) {
          const int oy = fy - hy;
          const int cbase = hx * 64 + hy * 8;
          for (int hz = hz0; hz <= hz1; ++hz) {
            const int oz = fz - hz;
            const int c = cbase + hz;
            const int pe = cstart[c + 1];
            for (int q = cstart[c]; q < pe; ++q) {
              const double *wt = wts + q * 3 * W;
              a += (wt[ox] * wt[W + oy]) * wt[2 * W + oz];
            }
          }
        }
      }
      acc[f] = a;
    }
  }
  __syncthreads();
  // Each global cell is written by one footprint cell (its smallest alias
  // when the footprint wraps onto itself on grids narrower than F).
  for (int f = threadIdx.x; f < F3; f += blockDim.x) {
    const int fx = f / (F * F);
    const int fy = (f / F) % F;
    const int fz = f % F;
    if (fx >= g.n[0] || fy >= g.n[1] || fz >= g.n[2]) continue;
    double v = 0.0;
    for (int ax = fx; ax < F; ax += g.n[0])
      for (int ay = fy; ay < F; ay += g.n[1])
        for (int az = fz; az < F; az += g.n[2]) v += acc[(ax * F + ay) * F + az];
    if (v == 0.0) continue;
    int gx = (o0 + fx + OMIN) % g.n[0];
    int gy = (o1 + fy + OMIN) % g.n[1];
    int gz = (o2 + fz + OMIN) % g.n[2];
    if (gx < 0) gx += g.n[0];
    if (gy < 0) gy += g.n[1];
    if (gz < 0) gz += g.n[2];
    GT &cell = grid[((size_t)gx * g.n[1] + gy) * g.n[2] + gz];
    cell = (GT)((double)cell + v);
  }
}

// K-scatter for stencils of width <= 3 (NGP, CIC, TSC).  The work unit is
// a sub-tile of TX x 8 x 8 home cells (TX = 2, 4 or 8: a contiguous range
// of tile-major keys), one thread per home cell, and a colour pass is run
// by persistent CTAs that draw the non-empty units of the colour from a
// counter.  A unit's particles (contiguous in sorted order) are staged in
// chunks: all threads gather positions and weights in parallel into shared
// memory (fractional cell offsets and weight), then each thread walks its
// own cell's particles of the chunk in sorted order and accumulates the W^3
// products wx[a]*wy[b]*wz[c] in registers (S_h[a][b][c]).  The home cells'
// sums then go to a shared table S[o][h], and each footprint cell f adds
// the terms S[o][f - o] of the home cells that reach it in the order o
// (one barrier, where a scatter into the footprint would need one per o).
// Each cell's particles are summed in sorted order whatever the chunking,
// so the grid is the same bits on every run.
// Scatter unit width along x for the narrow stencils: 2 x 8 x 8 home cells
// per CTA of 128 threads, five CTAs per SM.
constexpr int kUnitX = 2;

template <int S, int TX>
struct ScatterP {
  static constexpr int W = Stencil<S>::W;
  static constexpr int W3 = W * W * W;
  static constexpr int THREADS = TX * 64;
  static constexpr int MIN_BLOCKS = TX == 2 ? 5 : kTile / TX;
  static constexpr int FX = TX + W - 1;     // footprint extent along x
  static constexpr int FY = kTile + W - 1;  // ... along y and z
  static constexpr int F3 = FX * FY * FY;
  static constexpr int C = TX * 256;  // particles staged per chunk
  static constexpr int NW = THREADS / 32;
  static constexpr int ROUNDS = C / THREADS;  // rounds of 32 items per warp
  // The staged particles pd[C][4] and, once a unit's particles are summed,
  // the home-cell table S[W3][THREADS] share the first region.
  static constexpr size_t REGION0 =
      (size_t)C * 4 > (size_t)W3 * THREADS ? (size_t)C * 4 : (size_t)W3 * THREADS;
  // region0 | acc[F3] | gfoot[F3] doubles,
  // perm[C] | wc[NW][THREADS] | cstart[THREADS + 1] ints
  static constexpr size_t smem = REGION0 * 8 + (size_t)F3 * 16 + (size_t)C * 4 +
                                 (size_t)NW * THREADS * 4 +
                                 (size_t)(THREADS + 1) * 4;
};


// Global cell of footprint cell (fx, fy, fz) of a unit at (o0, o1, o2) on a
// grid at least a footprint wide (one wrap at most per axis).
template <int OMIN>
__device__ __forceinline__ size_t foot_cell(int fx, int fy, int fz, int o0,
                                            int o1, int o2,
                                            const AssignGeom &g) {
  int gx = o0 + fx + OMIN, gy = o1 + fy + OMIN, gz = o2 + fz + OMIN;
  gx += gx < 0 ? g.n[0] : (gx >= g.n[0] ? -g.n[0] : 0);
  gy += gy < 0 ? g.n[1] : (gy >= g.n[1] ? -g.n[1] : 0);
  gz += gz < 0 ? g.n[2] : (gz >= g.n[2] ? -g.n[2] : 0);
  return ((size_t)gx * g.n[1] + gy) * g.n[2] + gz;
}

// [ranges, ranges_end): this colour's slice of (unit, first, end) records,
// `count` non-empty units from its start and `count_heavy` heavy ones from
// its end; `next` is this colour's work counter (zero before the pass).
// GT is the grid's cell type: each footprint cell's FP64 sum for the unit is
// added to the cell in FP64 and rounded to GT once.
template <int S, typename KeyT, int TX, typename GT>
__global__ void __launch_bounds__(TX * 64, ScatterP<S, TX>::MIN_BLOCKS)
    k_scatter_p(const double *__restrict__ posw, const KeyT *__restrict__ keys,
                const uint32_t *__restrict__ vals,
                const uint4 *__restrict__ ranges,
                const uint4 *__restrict__ ranges_end,
                const unsigned *__restrict__ count,
                const unsigned *__restrict__ count_heavy, unsigned *next,
                AssignGeom g, GT *__restrict__ grid) {
  using Q = ScatterP<S, TX>;
  constexpr int W = Q::W;
  constexpr int W3 = Q::W3;
  constexpr int T = Q::THREADS;
  constexpr int FX = Q::FX;
  constexpr int FY = Q::FY;
  constexpr int F3 = Q::F3;
  constexpr int C = Q::C;
  constexpr int NS = kTile / TX;
  constexpr int OMIN = Stencil<S>::OMIN;
  constexpr int kSlots = C / T;
  constexpr int NW = Q::NW;
  constexpr int R = Q::ROUNDS;
  static_assert(C % T == 0, "whole staging slots per thread");
  extern __shared__ __align__(16) double smem[];
  double *pd = smem;                                     // [C][4]
  double *stab = smem;                                   // [W3][T], after pd
  double *acc = smem + Q::REGION0;                       // [F3]
  GT *gfoot = reinterpret_cast<GT *>(acc + F3);          // [F3]
  int *perm = reinterpret_cast<int *>(acc + 2 * F3);     // [C]
  int *wcs = perm + C;                                   // [NW][T]
  int *cstart = wcs + NW * T;                            // [T + 1]
  __shared__ uint4 s_rg;
  __shared__ unsigned s_next;
  __shared__ uint32_t s_scan[32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;

  const unsigned nh = *count_heavy;
  const unsigned n = *count + nh;
  if (threadIdx.x == 0) {
    const unsigned i0 = atomicAdd(next, 1u);
    s_next = atomicAdd(next, 1u);
    s_rg = i0 < n ? pass_unit(ranges, ranges_end, nh, i0) : make_uint4(0u, 0u, 0u, 0u);
  }
  __syncthreads();
  uint4 rg = s_rg;
  unsigned inext = s_next;
  const int h = threadIdx.x;
  const bool direct = g.n[0] >= FX && g.n[1] >= FY && g.n[2] >= FY;
  const bool a16 = (reinterpret_cast<uintptr_t>(posw) & 15) == 0;
  while (rg.y < rg.z) {
    // Thread 0 fetches the next unit's range and draws the index after it;
    // neither is needed before the end of this unit.
    uint4 rgn = make_uint4(0u, 0u, 0u, 0u);
    unsigned inn = 0;
    if (threadIdx.x == 0) {
      inn = atomicAdd(next, 1u);
      if (inext < n) rgn = pass_unit(ranges, ranges_end, nh, inext);
    }
    const uint32_t unit = rg.x, ts = rg.y, te = rg.z;
    const uint32_t tile = unit / NS;
    const int tz = tile % g.nt[2];
    const int ty = (tile / g.nt[2]) % g.nt[1];
    const int tx = tile / (g.nt[2] * g.nt[1]);
    const int o0 = tx * kTile + (int)(unit % NS) * TX;
    const int o1 = ty * kTile, o2 = tz * kTile;
    const KeyT kbase = (KeyT)unit * (KeyT)T;
    // When no footprint wraps onto itself, each footprint cell has one
    // global cell: copy its current value now, so the latency of the final
    // read-modify-write overlaps the particle gather.  (No other CTA of this
    // colour pass touches these cells.)  The first chunk's wait covers it.
    if (direct) {
      for (int f = h; f < F3; f += T)
        cp_async_cell(gfoot + f, grid + foot_cell<OMIN>(f / (FY * FY), (f / FY) % FY,
                                                    f % FY, o0, o1, o2, g));
    }

    double sacc[W3];
#pragma unroll
    for (int o = 0; o < W3; ++o) sacc[o] = 0.0;
    for (uint32_t c0 = ts; c0 < te; c0 += C) {
      const int m = (int)min((uint32_t)C, te - c0);
      if (c0 != ts) __syncthreads();  // the previous chunk has been consumed
      // Each thread stages up to kSlots particles: the index loads first,
      // then the catalog rows as asynchronous copies, so the gathers of one
      // thread overlap.
      // The keys this thread's warp ranks below are read here, together
      // with the indices, so that both loads are in flight at once.
      KeyT kr[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = warp * 32 * R + r * 32 + lane;
        kr[r] = i < m ? keys[c0 + i] : kbase + (KeyT)T;
      }
      uint32_t idx[kSlots];
#pragma unroll
      for (int j = 0; j < kSlots; ++j) {
        const int i = h + j * T;
        idx[j] = i < m ? vals[c0 + i] : 0u;
      }
#pragma unroll
      for (int j = 0; j < kSlots; ++j) {
        const int i = h + j * T;
        if (i >= m) continue;
        const double *p = posw + 4 * (size_t)idx[j];
        double *d = pd + 4 * i;
        if (a16) {
          cp_async16(d, p);
          cp_async16(d + 2, p + 2);
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) cp_async8(d + k, p + k);
        }
      }
      // Stable order by home cell: warp w ranks its R rounds of 32 items
      // (items [w*32R, (w+1)*32R)) among equal cells with a running count
      // per cell in its row of wcs.
      int *wc = wcs + warp * T;
      for (int k = lane; k < T; k += 32) wc[k] = 0;
      __syncwarp();
      int lcell[R], lrank[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        // (A key outside this unit cannot occur in a correct sort; it is
        // dropped rather than indexing outside the unit's cells.)
        const KeyT kd = kr[r] - kbase;
        const int cell = kd < (KeyT)T ? (int)kd : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, cell);
        const int leader = __ffs(peers) - 1;
        int b = 0;
        if (lane == leader && cell >= 0) {
          b = wc[cell];
          wc[cell] = b + __popc(peers);
        }
        b = __shfl_sync(0xffffffffu, b, leader);
        lcell[r] = cell;
        lrank[r] = b + __popc(peers & lt);
        __syncwarp();
      }
      cp_async_wait_all();
      // Each thread converts its own rows to (rx, ry, rz, w).
#pragma unroll
      for (int j = 0; j < kSlots; ++j) {
        const int i = h + j * T;
        if (i >= m) continue;
        double *d = pd + 4 * i;
        double x[3];
        dev_grid_coords(d, g, x);
        d[0] = x[0] - floor(x[0]);
        d[1] = x[1] - floor(x[1]);
        d[2] = x[2] - floor(x[2]);
      }
      __syncthreads();
      // Cell h: its first position, then each warp's first position in it.
      int tot = 0;
#pragma unroll
      for (int w = 0; w < NW; ++w) tot += wcs[w * T + h];
      int run = (int)block_exclusive_scan((uint32_t)tot, s_scan);
      cstart[h] = run;
      if (h == T - 1) cstart[T] = run + tot;
#pragma unroll
      for (int w = 0; w < NW; ++w) {
        const int c = wcs[w * T + h];
        wcs[w * T + h] = run;
        run += c;
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (lcell[r] >= 0)
          perm[wc[lcell[r]] + lrank[r]] = warp * 32 * R + r * 32 + lane;
      __syncthreads();
      const int lo = cstart[h], hi = cstart[h + 1];
      for (int q = lo; q < hi; ++q) {
        const int i = perm[q];
        double wx[W], wy[W], wz[W];
        Stencil<S>::weights(pd[4 * i + 0], pd[4 * i + 1], pd[4 * i + 2],
                            pd[4 * i + 3], wx, wy, wz);
#pragma unroll
        for (int a = 0; a < W; ++a)
#pragma unroll
          for (int b = 0; b < W; ++b) {
            const double wxy = wx[a] * wy[b];
#pragma unroll
            for (int c = 0; c < W; ++c)
              sacc[(a * W + b) * W + c] = fma(wxy, wz[c], sacc[(a * W + b) * W + c]);
          }
      }
    }
    __syncthreads();  // every thread is done with the staged particles
#pragma unroll
    for (int o = 0; o < W3; ++o) stab[o * T + h] = sacc[o];
    __syncthreads();
    // Footprint cell f = h + o takes S[o][h] for every home cell h in the
    // unit, in the order o, starting from 0.0.
    for (int f = h; f < F3; f += T) {
      const int fx = f / (FY * FY), fy = (f / FY) % FY, fz = f % FY;
      double v = 0.0;
#pragma unroll
      for (int o = 0; o < W3; ++o) {
        const int qx = fx - o / (W * W), qy = fy - (o / W) % W, qz = fz - o % W;
        if (qx >= 0 && qx < TX && qy >= 0 && qy < kTile && qz >= 0 && qz < kTile)
          v += stab[o * T + (qx * kTile + qy) * kTile + qz];
      }
      if (direct) {
        if (v != 0.0)
          grid[foot_cell<OMIN>(fx, fy, fz, o0, o1, o2, g)] =
              (GT)((double)gfoot[f] + v);
      } else {
        acc[f] = v;
      }
    }
    if (!direct) {
      __syncthreads();
      // Each global cell is written by one footprint cell (its smallest
      // alias when the footprint wraps onto itself on narrow grids).
      for (int f = h; f < F3; f += T) {
        const int fx = f / (FY * FY);
        const int fy = (f / FY) % FY;
        const int fz = f % FY;
        if (fx >= g.n[0] || fy >= g.n[1] || fz >= g.n[2]) continue;
        double v = 0.0;
        for (int ax = fx; ax < FX; ax += g.n[0])
          for (int ay = fy; ay < FY; ay += g.n[1])
            for (int az = fz; az < FY; az += g.n[2])
              v += acc[(ax * FY + ay) * FY + az];
        if (v == 0.0) continue;
        int gx = (o0 + fx + OMIN) % g.n[0];
        int gy = (o1 + fy + OMIN) % g.n[1];
        int gz = (o2 + fz + OMIN) % g.n[2];
        if (gx < 0) gx += g.n[0];
        if (gy < 0) gy += g.n[1];
        if (gz < 0) gz += g.n[2];
        GT &cell = grid[((size_t)gx * g.n[1] + gy) * g.n[2] + gz];
        cell = (GT)((double)cell + v);
      }
    }
    if (threadIdx.x == 0) {
      s_rg = rgn;
      s_next = inn;
    }
    __syncthreads();  // acc and the staging buffers are free again
    rg = s_rg;
    inext = s_next;
  }
}

template <int S>
size_t scatter_smem() {
  constexpr int W = Stencil<S>::W;
  constexpr int F = kTile + W - 1;
  return sizeof(double) * (F * F * F + kChunk * 3 * W) +
         sizeof(int) * (kChunk + kTileCells + 1);
}

// Greedy colouring along one axis of units `unit` cells wide, so that
// units sharing a colour have disjoint (periodically wrapped) footprints.
// Units past the end of the axis hold no cells and take colour 0.
std::vector<int> color_axis(int n, int nunits, int unit, int W, int omin) {
  std::vector<std::vector<char>> used;  // per colour: cells covered so far
  std::vector<int> color(nunits, 0);
  std::vector<char> cover(n);
  for (int t = 0; t < nunits; ++t) {
    const int lo = t * unit;
    if (lo >= n) continue;
    const int hi = std::min(n, lo + unit) - 1;
    std::fill(cover.begin(), cover.end(), 0);
    for (int c = lo + omin; c <= hi + omin + W - 1; ++c)
      cover[((c % n) + n) % n] = 1;
    int c = 0;
    for (;; ++c) {
      if (c == (int)used.size()) used.emplace_back(n, 0);
      bool ok = true;
      for (int k = 0; k < n && ok; ++k) ok = !(cover[k] && used[c][k]);
      if (ok) break;
    }
    for (int k = 0; k < n; ++k) used[c][k] |= cover[k];
    color[t] = c;
  }
  return color;
}

int stencil_width(int scheme, int *omin) {
  switch (scheme) {
    case 0:
      *omin = 0;
      return 1;
    case 1:
      *omin = -1;
      return 3;
    case 2:
      *omin = -1;
      return 8;
    default:
      *omin = 0;
      return 2;
  }
}

// Scatter kernel for scheme 0, 1 or 3, a key type and a cell type.
template <typename KeyT, typename GT>
void scatter_p_kernel(int scheme, const void **fn, size_t *smem) {
  switch (scheme) {
    case 0:
      *fn = (const void *)k_scatter_p<0, KeyT, kUnitX, GT>;
      *smem = ScatterP<0, kUnitX>::smem;
      break;
    case 1:
      *fn = (const void *)k_scatter_p<1, KeyT, kUnitX, GT>;
      *smem = ScatterP<1, kUnitX>::smem;
      break;
    default:
      *fn = (const void *)k_scatter_p<3, KeyT, kUnitX, GT>;
      *smem = ScatterP<3, kUnitX>::smem;
      break;
  }
}

}  // namespace

// MassAssignor state (mass_assignor.h:30-234) with a device-side buffer.
struct Assignor {
  Grid *grid;
  std::weak_ptr<int> grid_alive;
  int scheme;
  bool periodic;
  int64_t buffer_size;
  AssignGeom geom;
  int64_t ntiles;
  int unit_x;      // scatter unit: unit_x x 8 x 8 cells
  int64_t nunits;  // ntiles * (8 / unit_x)
  bool wide_keys;  // 64-bit keys when the key space exceeds 32 bits
  int end_bit;

  // Buffered particles.
  int64_t count = 0;
  int64_t capacity = 0;
  DeviceBuffer posw, keys, keys_alt, vals, vals_alt, sort_temp;
  // NGP/CIC/TSC sort by unit only (key bits from unit_shift up): the
  // scatter orders each unit's particles by cell itself.
  int unit_shift = 0;
  DeviceBuffer unit_start;             // first sorted particle per unit
  DeviceBuffer color_units;            // units in colour order
  DeviceBuffer unit_ranges;            // uint4 per unit, colour slices
  DeviceBuffer color_off_dev;          // color_offsets on the device
  DeviceBuffer pass_counters;          // per colour: light units, work, heavy units
  std::vector<int64_t> color_offsets;  // per colour, into color_units
  const void *scatter_fn = nullptr;    // k_scatter_p for this scheme / keys
  size_t scatter_smem_bytes = 0;
  int scatter_threads = 0;
  unsigned scatter_ctas = 0;           // persistent CTAs per colour pass
  DeviceBuffer partials;               // K-key block partials
  DeviceBuffer totals;                 // [totw, totwsq]
  DeviceBuffer counts;                 // [num_added]
  DeviceBuffer staging;                // pos / weights for the (pos, w) forms
  // Particles being keyed and scattered: the internal buffer, or a caller's
  // device array that is assigned in place without a copy.
  const double *src_posw = nullptr;
  uint64_t num_seen = 0;               // particles passed to add calls
  PhaseTimer sort_timer, window_timer;
  double sort_seconds = 0.0, window_seconds = 0.0;
  // Graph mode (batched form): work goes to stream_override, nothing
  // synchronises the host, nothing is allocated, phases are not timed.
  bool graph_mode = false;
  cudaStream_t stream_override = nullptr;

  Assignor(Grid *g, int scheme_, bool periodic_, int64_t buffer_size_)
      : grid(g), grid_alive(g->alive), scheme(scheme_), periodic(periodic_),
        buffer_size(buffer_size_) {
    FC_REQUIRE(scheme >= 0 && scheme <= 3, FC_ERR_INVALID,
               "unknown distribution scheme");
    FC_REQUIRE(scheme != 2 || FC_HAVE_D12, FC_ERR_UNSUPPORTED,
               "this build has no D12 wavelet table (build with the "
               "reference tree available)");
    FC_REQUIRE(buffer_size >= 0, FC_ERR_INVALID, "buffer_size must be >= 0");
    for (int i = 0; i < 3; ++i) {
      geom.n[i] = g->shape[i];
      geom.nt[i] = (g->shape[i] + kTile - 1) / kTile;
      geom.posmin[i] = g->posmin[i];
    }
    geom.cell = g->cell_size;
    geom.rcell = 1.0 / geom.cell;
    geom.fast_div = geom.cell >= 0x1p-400 && geom.cell <= 0x1p400;
    geom.periodic = periodic ? 1 : 0;
    ntiles = (int64_t)geom.nt[0] * geom.nt[1] * geom.nt[2];
    unit_x = scheme == 2 ? kTile : kUnitX;
    nunits = ntiles * (kTile / unit_x);
    const uint64_t max_key = (uint64_t)ntiles * kTileCells;  // invalid key
    wide_keys = max_key >= 0xffffffffull;
    end_bit = 1;
    while (end_bit < 64 && (max_key >> end_bit) != 0) ++end_bit;
    unit_start.resize((nunits + 1) * sizeof(uint32_t));
    if (scheme != 2) unit_ranges.resize(std::max<int64_t>(nunits, 1) * sizeof(uint4));
    partials.resize(2 * kSumBlocks * sizeof(double));
    totals.resize(2 * sizeof(double));
    counts.resize(sizeof(unsigned long long));
    build_colors();
    FC_CUDA(cudaMemsetAsync(totals.get(), 0, totals.bytes(), grid->stream));
    FC_CUDA(cudaMemsetAsync(counts.get(), 0, counts.bytes(), grid->stream));
    if (scheme != 2) {
      while ((1 << unit_shift) < unit_x * kTile * kTile) ++unit_shift;
      if (wide_keys && grid->fp32())
        scatter_p_kernel<uint64_t, float>(scheme, &scatter_fn, &scatter_smem_bytes);
      else if (wide_keys)
        scatter_p_kernel<uint64_t, double>(scheme, &scatter_fn, &scatter_smem_bytes);
      else if (grid->fp32())
        scatter_p_kernel<uint32_t, float>(scheme, &scatter_fn, &scatter_smem_bytes);
      else
        scatter_p_kernel<uint32_t, double>(scheme, &scatter_fn, &scatter_smem_bytes);
      scatter_threads = unit_x * 64;
      FC_CUDA(cudaFuncSetAttribute(scatter_fn,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)scatter_smem_bytes));
      int per_sm = 0;
      FC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, scatter_fn, scatter_threads, scatter_smem_bytes));
      scatter_ctas = (unsigned)std::max(1, per_sm) * (unsigned)sm_count();
    }
    for (int b = 1; b <= radix::kMaxBits; ++b)
      FC_CUDA(cudaFuncSetAttribute(radix::downsweep_kernel(b),
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)radix::kDownSmem));
    if (scheme == 2) {
      FC_CUDA(cudaFuncSetAttribute(k_scatter<2, uint32_t, double>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)scatter_smem<2>()));
      FC_CUDA(cudaFuncSetAttribute(k_scatter<2, uint64_t, double>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)scatter_smem<2>()));
      FC_CUDA(cudaFuncSetAttribute(k_scatter<2, uint32_t, float>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)scatter_smem<2>()));
      FC_CUDA(cudaFuncSetAttribute(k_scatter<2, uint64_t, float>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)scatter_smem<2>()));
    }
  }

  ~Assignor() {
    // The grid may have gone first (its destructor drains its stream).
    if (!grid_alive.expired() && grid->stream) cudaStreamSynchronize(grid->stream);
  }

  cudaStream_t stream() const {
    return stream_override ? stream_override : grid->stream;
  }

  void build_colors() {
    int omin = 0;
    const int W = stencil_width(scheme, &omin);
    const int ns = kTile / unit_x;
    const int nux[3] = {geom.nt[0] * ns, geom.nt[1], geom.nt[2]};
    const int unit[3] = {unit_x, kTile, kTile};
    std::vector<int> col[3];
    int ncol[3];
    for (int a = 0; a < 3; ++a) {
      col[a] = color_axis(geom.n[a], nux[a], unit[a], W, omin);
      ncol[a] = 1 + *std::max_element(col[a].begin(), col[a].end());
    }
    const int ncolors = ncol[0] * ncol[1] * ncol[2];
    std::vector<std::vector<uint32_t>> lists(ncolors);
    for (int ux = 0; ux < nux[0]; ++ux)
      for (int ty = 0; ty < geom.nt[1]; ++ty)
        for (int tz = 0; tz < geom.nt[2]; ++tz) {
          const int c = (col[0][ux] * ncol[1] + col[1][ty]) * ncol[2] + col[2][tz];
          const int64_t tile = ((int64_t)(ux / ns) * geom.nt[1] + ty) * geom.nt[2] + tz;
          lists[c].push_back((uint32_t)(tile * ns + ux % ns));
        }
    std::vector<uint32_t> flat;
    flat.reserve(nunits);
    color_offsets.assign(1, 0);
    for (auto &l : lists) {
      flat.insert(flat.end(), l.begin(), l.end());
      color_offsets.push_back((int64_t)flat.size());
    }
    color_units.resize(flat.size() * sizeof(uint32_t));
    FC_CUDA(cudaMemcpy(color_units.get(), flat.data(),
                       flat.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    color_off_dev.resize(color_offsets.size() * sizeof(int64_t));
    FC_CUDA(cudaMemcpy(color_off_dev.get(), color_offsets.data(),
                       color_offsets.size() * sizeof(int64_t),
                       cudaMemcpyHostToDevice));
    pass_counters.resize(3 * ncolors * sizeof(unsigned));
  }

  size_t key_bytes() const { return wide_keys ? 8 : 4; }

  // Key/index buffers for assigning `need` particles straight from a
  // caller's device array (nothing is buffered).
  void reserve_keys(int64_t need) {
    FC_REQUIRE(count == 0, FC_ERR_STATE, "particles are still buffered");
    FC_REQUIRE(need < (int64_t)0xffffffffll, FC_ERR_INVALID,
               "too many particles in one call (limit 2^32-1)");
    if ((size_t)need * key_bytes() <= keys.bytes()) return;
    keys.release();
    vals.release();
    keys_alt.release();
    vals_alt.release();
    keys.resize(need * key_bytes());
    vals.resize(need * sizeof(uint32_t));
    keys_alt.resize(need * key_bytes());
    vals_alt.resize(need * sizeof(uint32_t));
  }

  // Grows the particle buffer to hold `need` particles, keeping the
  // buffered ones.
  void reserve(int64_t need) {
    if (need <= capacity) return;
    FC_REQUIRE(need < (int64_t)0xffffffffll, FC_ERR_INVALID,
               "too many buffered particles (limit 2^32-1 per flush)");
    int64_t cap = std::max<int64_t>(need, capacity + capacity / 2);
    cap = std::min<int64_t>(cap, (int64_t)0xfffffffell);
    DeviceBuffer np(cap * 4 * sizeof(double));
    DeviceBuffer nk(cap * key_bytes());
    DeviceBuffer nv(cap * sizeof(uint32_t));
    if (count > 0) {
      FC_CUDA(cudaMemcpyAsync(np.get(), posw.get(), count * 4 * sizeof(double),
                              cudaMemcpyDeviceToDevice, stream()));
      FC_CUDA(cudaMemcpyAsync(nk.get(), keys.get(), count * key_bytes(),
                              cudaMemcpyDeviceToDevice, stream()));
      // Only wide keys keep an index array before the sort (the 32-bit
      // sort's first pass takes each key's position as its index).
      if (wide_keys)
        FC_CUDA(cudaMemcpyAsync(nv.get(), vals.get(), count * sizeof(uint32_t),
                                cudaMemcpyDeviceToDevice, stream()));
      FC_CUDA(cudaStreamSynchronize(stream()));
    }
    posw = std::move(np);
    keys = std::move(nk);
    vals = std::move(nv);
    keys_alt.release();
    vals_alt.release();
    keys_alt.resize(cap * key_bytes());
    vals_alt.resize(cap * sizeof(uint32_t));
    capacity = cap;
  }

  // K-key over the particles just placed at [count, count+n).
  void key_new(int64_t n) {
    if (n == 0) return;
    src_posw = posw.as<double>();
    const unsigned blocks = std::min<unsigned>(kSumBlocks, grid_for(n, 256));
    double *parts = partials.as<double>();
    if (wide_keys) {
      k_keys<uint64_t><<<blocks, 256, 0, stream()>>>(
          src_posw, count, n, geom, (uint64_t)ntiles * kTileCells,
          keys.as<uint64_t>(), vals.as<uint32_t>(), parts,
          counts.as<unsigned long long>());
    } else {
      k_keys<uint32_t><<<blocks, 256, 0, stream()>>>(
          src_posw, count, n, geom, (uint32_t)(ntiles * kTileCells),
          keys.as<uint32_t>(), nullptr, parts, counts.as<unsigned long long>());
    }
    FC_LAUNCH_CHECK();
    k_fold_totals<<<1, 256, 0, stream()>>>(parts, blocks, totals.as<double>());
    FC_LAUNCH_CHECK();
    count += n;
    num_seen += n;
  }

  void add_device_posw(const double *src, int64_t n, cudaMemcpyKind kind) {
    FC_REQUIRE(n >= 0, FC_ERR_INVALID, "negative particle count");
    if (kind == cudaMemcpyDeviceToDevice && count == 0 && n > 0 &&
        n < (int64_t)0xffffffffll && (buffer_size == 0 || n >= buffer_size)) {
      // Assigned at once: key, sort and scatter straight from the caller's
      // array instead of copying it into the buffer first.
      reserve_keys(n);
      const double *keep = src_posw;
      key_device(src, n);
      flush();
      src_posw = keep;
      return;
    }
    int64_t done = 0;
    // Large inputs are assigned in pieces so the buffer stays bounded.
    const int64_t piece_max = (int64_t)1 << 28;
    while (done < n) {
      const int64_t piece = std::min(n - done, piece_max);
      reserve(count + piece);
      FC_CUDA(cudaMemcpyAsync(posw.as<double>() + 4 * count, src + 4 * done,
                              piece * 4 * sizeof(double), kind, stream()));
      key_new(piece);
      done += piece;
      maybe_flush();
    }
  }

  // K-key over an external device array of n particles (buffer empty).
  void key_device(const double *src, int64_t n) {
    src_posw = src;
    const unsigned blocks = std::min<unsigned>(kSumBlocks, grid_for(n, 256));
    double *parts = partials.as<double>();
    if (wide_keys) {
      k_keys<uint64_t><<<blocks, 256, 0, stream()>>>(
          src, 0, n, geom, (uint64_t)ntiles * kTileCells, keys.as<uint64_t>(),
          vals.as<uint32_t>(), parts, counts.as<unsigned long long>());
    } else {
      k_keys<uint32_t><<<blocks, 256, 0, stream()>>>(
          src, 0, n, geom, (uint32_t)(ntiles * kTileCells), keys.as<uint32_t>(),
          nullptr, parts, counts.as<unsigned long long>());
    }
    FC_LAUNCH_CHECK();
    k_fold_totals<<<1, 256, 0, stream()>>>(parts, blocks, totals.as<double>());
    FC_LAUNCH_CHECK();
    count = n;
    num_seen += n;
  }

  void add_pos(const double *pos, const double *w, double wconst, int64_t n) {
    FC_REQUIRE(n >= 0, FC_ERR_INVALID, "negative particle count");
    int64_t done = 0;
    const int64_t piece_max = (int64_t)1 << 26;
    while (done < n) {
      const int64_t piece = std::min(n - done, piece_max);
      reserve(count + piece);
      staging.resize(piece * 4 * sizeof(double));
      double *sp = staging.as<double>();
      FC_CUDA(cudaMemcpyAsync(sp, pos + 3 * done, piece * 3 * sizeof(double),
                              cudaMemcpyHostToDevice, stream()));
      const double *dw = nullptr;
      if (w) {
        FC_CUDA(cudaMemcpyAsync(sp + 3 * piece, w + done, piece * sizeof(double),
                                cudaMemcpyHostToDevice, stream()));
        dw = sp + 3 * piece;
      }
      k_pack<<<grid_for(piece, 256), 256, 0, stream()>>>(
          sp, dw, wconst, piece, posw.as<double>() + 4 * count);
      FC_LAUNCH_CHECK();
      // The pack reads staging before the next piece overwrites it.
      key_new(piece);
      FC_CUDA(cudaStreamSynchronize(stream()));
      done += piece;
      maybe_flush();
    }
  }

  void maybe_flush() {
    if (buffer_size == 0 || count >= buffer_size) flush();
  }

  // K-sort: stable radix sort of (key, particle index) on key bits
  // [begin_bit, end_bit).  Returns the sorted arrays.
  template <typename KeyT>
  void sort_keys(int begin_bit, const KeyT **sk, const uint32_t **sv) {
    if constexpr (std::is_same_v<KeyT, uint32_t>) {
      radix_sort(begin_bit, sk, sv);
    } else {
      // Keys wider than 32 bits (grids of more than 2^32 cells).
      const int64_t n = count;
      cub::DoubleBuffer<KeyT> dk(keys.as<KeyT>(), keys_alt.as<KeyT>());
      cub::DoubleBuffer<uint32_t> dv(vals.as<uint32_t>(), vals_alt.as<uint32_t>());
      size_t temp = 0;
      FC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, dk, dv, n, begin_bit,
                                              end_bit, stream()));
      if (graph_mode)
        FC_REQUIRE(temp <= sort_temp.bytes(), FC_ERR_STATE,
                   "sort scratch was not prepared for this many particles");
      sort_temp.resize(temp);
      if (!graph_mode) sort_timer.start(stream());
      FC_CUDA(cub::DeviceRadixSort::SortPairs(sort_temp.get(), temp, dk, dv, n,
                                              begin_bit, end_bit, stream()));
      if (!graph_mode) sort_timer.stop(stream());
      *sk = dk.Current();
      *sv = dv.Current();
    }
  }

  // The key of particles outside the grid, and the bits of the valid keys
  // (the invalid key sorts last through a digit of its own).
  uint32_t invalid_key32() const { return (uint32_t)(ntiles * kTileCells); }
  int valid_end_bit() const {
    const uint64_t max_valid = (uint64_t)invalid_key32() - 1;
    int e = 1;
    while (e < 32 && (max_valid >> e) != 0) ++e;
    return e;
  }

  // Scratch of the 32-bit-key sort for n particles, either sort range.
  size_t radix_scratch(int64_t n) const {
    return std::max(radix::sort_plan(n, 0, valid_end_bit()).scratch_bytes(),
                    radix::sort_plan(n, unit_shift, valid_end_bit()).scratch_bytes());
  }

  // The stable LSD radix sort of the 32-bit keys (fc_sort.cuh): the first
  // pass reads the keys in place with implicit indices, later passes
  // alternate between the two key and index buffers.
  void radix_sort(int begin_bit, const uint32_t **sk, const uint32_t **sv) {
    using namespace radix;
    const int64_t n = count;
    const SortPlan p = sort_plan(n, begin_bit, valid_end_bit());
    const uint32_t invalid = invalid_key32();
    if (graph_mode)
      FC_REQUIRE(p.scratch_bytes() <= sort_temp.bytes(), FC_ERR_STATE,
                 "sort scratch was not prepared for this many particles");
    sort_temp.resize(p.scratch_bytes());
    uint32_t *cnt = sort_temp.as<uint32_t>();
    uint32_t *sums = cnt + p.m;
    cudaStream_t st = stream();
    if (!graph_mode) sort_timer.start(st);
    const uint32_t *kin = keys.as<uint32_t>();
    const uint32_t *vin = nullptr;
    uint32_t *kbuf[2] = {keys_alt.as<uint32_t>(), keys.as<uint32_t>()};
    uint32_t *vbuf[2] = {vals_alt.as<uint32_t>(), vals.as<uint32_t>()};
    for (int pass = 0; pass < p.passes; ++pass) {
      const int shift = begin_bit + pass * p.bits;
      k_sort_upsweep<<<(unsigned)p.ntiles, kSortThreads, 0, st>>>(
          kin, n, invalid, shift, p.bits, p.ntiles, cnt);
      FC_LAUNCH_CHECK();
      k_sort_scan_reduce<<<(unsigned)p.nchunks, kSortThreads, 0, st>>>(cnt, p.m, sums);
      FC_LAUNCH_CHECK();
      k_sort_scan_top<<<1, kSortThreads, 0, st>>>(sums, p.nchunks);
      FC_LAUNCH_CHECK();
      k_sort_scan_apply<<<(unsigned)p.nchunks, kSortThreads, 0, st>>>(cnt, p.m, sums);
      FC_LAUNCH_CHECK();
      uint32_t *kout = kbuf[pass & 1], *vout = vbuf[pass & 1];
      downsweep_kernel(p.bits)<<<(unsigned)p.ntiles, kSortThreads, kDownSmem, st>>>(
          kin, vin, n, invalid, shift, p.ntiles, cnt, kout, vout);
      FC_LAUNCH_CHECK();
      kin = kout;
      vin = vout;
    }
    if (!graph_mode) sort_timer.stop(st);
    *sk = kin;
    *sv = vin;
  }

  // D12: sort by cell key, then the tile scatter.
  template <typename KeyT>
  void flush_d12() {
    const int64_t n = count;
    const KeyT *sk;
    const uint32_t *sv;
    sort_keys<KeyT>(0, &sk, &sv);
    if (!graph_mode) window_timer.start(stream());
    const int unit_cells = unit_x * kTile * kTile;
    k_unit_starts<KeyT><<<grid_for(nunits + 1, 256), 256, 0, stream()>>>(
        sk, n, nunits, unit_cells, unit_start.as<uint32_t>());
    FC_LAUNCH_CHECK();
    const uint32_t *units = color_units.as<uint32_t>();
    const int ncolors = (int)color_offsets.size() - 1;
    for (int c = 0; c < ncolors; ++c) {
      const int64_t nu = color_offsets[c + 1] - color_offsets[c];
      if (nu == 0) continue;
      if (grid->fp32())
        k_scatter<2, KeyT, float><<<(unsigned)nu, kScatterThreads,
                                    scatter_smem<2>(), stream()>>>(
            src_posw, sk, sv, unit_start.as<uint32_t>(), units + color_offsets[c],
            geom, static_cast<float *>(grid->raw()));
      else
        k_scatter<2, KeyT, double><<<(unsigned)nu, kScatterThreads,
                                     scatter_smem<2>(), stream()>>>(
            src_posw, sk, sv, unit_start.as<uint32_t>(), units + color_offsets[c],
            geom, grid->ptr());
      FC_LAUNCH_CHECK();
    }
    if (!graph_mode) window_timer.stop(stream());
  }

  // NGP / CIC / TSC: sort by unit, then the persistent unit scatter in
  // colour passes.
  template <typename KeyT>
  void flush_units() {
    const int64_t n = count;
    const KeyT *sk;
    const uint32_t *sv;
    sort_keys<KeyT>(unit_shift, &sk, &sv);
    cudaStream_t st = stream();
    if (!graph_mode) window_timer.start(st);
    const int unit_cells = unit_x * kTile * kTile;
    k_unit_starts<KeyT><<<grid_for(nunits + 1, 256), 256, 0, st>>>(
        sk, n, nunits, unit_cells, unit_start.as<uint32_t>());
    FC_LAUNCH_CHECK();
    const uint32_t *units = color_units.as<uint32_t>();
    const int ncolors = (int)color_offsets.size() - 1;
    unsigned *counters = pass_counters.as<unsigned>();
    FC_CUDA(cudaMemsetAsync(counters, 0, pass_counters.bytes(), st));
    k_unit_ranges<<<grid_for(nunits, 256), 256, 0, st>>>(
        units, nunits, unit_start.as<uint32_t>(), color_off_dev.as<int64_t>(),
        ncolors, counters, unit_ranges.as<uint4>());
    FC_LAUNCH_CHECK();
    void *gp = grid->raw();
    AssignGeom ga = geom;
    const double *pw = src_posw;
    for (int c = 0; c < ncolors; ++c) {
      const int64_t nu = color_offsets[c + 1] - color_offsets[c];
      if (nu == 0) continue;
      const uint4 *cr = unit_ranges.as<uint4>() + color_offsets[c];
      const uint4 *cre = unit_ranges.as<uint4>() + color_offsets[c + 1];
      const unsigned *cnt = counters + c;
      const unsigned *cnth = counters + 2 * ncolors + c;
      unsigned *nxt = counters + ncolors + c;
      void *args[] = {(void *)&pw, (void *)&sk,  (void *)&sv,  (void *)&cr,
                      (void *)&cre, (void *)&cnt, (void *)&cnth, (void *)&nxt,
                      (void *)&ga, (void *)&gp};
      const unsigned ctas = (unsigned)std::min<int64_t>(nu, scatter_ctas);
      FC_CUDA(cudaLaunchKernel(scatter_fn, dim3(ctas), dim3(scatter_threads),
                               args, scatter_smem_bytes, st));
      FC_LAUNCH_CHECK();
    }
    if (!graph_mode) window_timer.stop(st);
  }

  template <typename KeyT>
  void flush_typed() {
    if (scheme == 2)
      flush_d12<KeyT>();
    else
      flush_units<KeyT>();
  }

  // MassAssignor::flush (mass_assignor.h:127-191).
  void flush() {
    if (count == 0) return;
    if (wide_keys)
      flush_typed<uint64_t>();
    else
      flush_typed<uint32_t>();
    count = 0;
    if (graph_mode) return;
    // Keep the timers' running totals current.
    sort_seconds += sort_timer.seconds();
    sort_timer.clear();
    window_seconds += window_timer.seconds();
    window_timer.clear();
  }

  // Batched form: size every buffer for up to max_n particles assigned
  // straight from a device array, so later enqueues allocate nothing.
  void prepare_graph(int64_t max_n) {
    graph_mode = true;
    reserve_keys(std::max<int64_t>(max_n, 1));
    size_t temp = 0;
    if (wide_keys) {
      cub::DoubleBuffer<uint64_t> dk(keys.as<uint64_t>(), keys_alt.as<uint64_t>());
      cub::DoubleBuffer<uint32_t> dv(vals.as<uint32_t>(), vals_alt.as<uint32_t>());
      FC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, dk, dv, max_n, 0,
                                              end_bit, stream()));
    } else {
      temp = radix_scratch(std::max<int64_t>(max_n, 1));
    }
    sort_temp.resize(temp + 1024);
  }

  // Batched form: clear the running totals and assign n particles from a
  // device array, all enqueued on stream().
  void enqueue_graph(const double *posw_dev, int64_t n) {
    FC_CUDA(cudaMemsetAsync(totals.get(), 0, totals.bytes(), stream()));
    FC_CUDA(cudaMemsetAsync(counts.get(), 0, counts.bytes(), stream()));
    count = 0;
    num_seen = 0;
    if (n == 0) return;
    FC_REQUIRE((size_t)n * key_bytes() <= keys.bytes(), FC_ERR_STATE,
               "more particles than the batch was prepared for");
    key_device(posw_dev, n);
    flush();
  }

  // add_random_particles (fftcorr/catalog/random_catalog.py:8-87) with the
  // positions drawn on the device: uniform over the grid's box, optionally
  // displaced by a gridded field, weight w each, in batches of `batch`.
  void add_random(int64_t n, double w, const double *disp_host, uint64_t seed,
                  int64_t batch) {
    FC_REQUIRE(n >= 0, FC_ERR_INVALID, "negative particle count");
    if (n == 0) return;
    if (batch <= 0) batch = (int64_t)1 << 26;
    const int64_t nb_max = std::min(batch, n);
    DeviceBuffer gen((size_t)nb_max * 4 * sizeof(double));
    DeviceBuffer ddisp, dflag(sizeof(int));
    AssignGeomLite lite;
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lite.n[a] = geom.n[a];
      lite.posmin[a] = geom.posmin[a];
      lo[a] = geom.posmin[a];
      hi[a] = geom.posmin[a] + geom.n[a] * geom.cell;
    }
    lite.cell = geom.cell;
    lite.periodic = geom.periodic;
    FC_CUDA(cudaMemsetAsync(dflag.get(), 0, sizeof(int), stream()));
    if (disp_host) {
      const size_t nd = (size_t)geom.n[0] * geom.n[1] * geom.n[2] * 3;
      ddisp.resize(nd * sizeof(double));
      FC_CUDA(cudaMemcpyAsync(ddisp.get(), disp_host, nd * sizeof(double),
                              cudaMemcpyHostToDevice, stream()));
    }
    for (int64_t done = 0; done < n;) {
      const int64_t nb = std::min(nb_max, n - done);
      catalog_uniform(gen.as<double>(), done, nb, lo, hi, w, w, seed, stream());
      if (disp_host)
        displace(gen.as<double>(), 4, nb, ddisp.as<double>(), lite,
                 gen.as<double>(), 4, dflag.as<int>(), stream());
      add_device_posw(gen.as<double>(), nb, cudaMemcpyDeviceToDevice);
      done += nb;
    }
    int flag = 0;
    FC_CUDA(cudaMemcpyAsync(&flag, dflag.get(), sizeof(int),
                            cudaMemcpyDeviceToHost, stream()));
    FC_CUDA(cudaStreamSynchronize(stream()));
    FC_REQUIRE(!flag, FC_ERR_INVALID,
               "Failed to apply displacement field: coordinates out of bounds? "
               "Try setting periodic_wrap=True.");
  }

  void clear() {
    FC_CUDA(cudaStreamSynchronize(stream()));
    count = 0;
    num_seen = 0;
    FC_CUDA(cudaMemsetAsync(totals.get(), 0, totals.bytes(), stream()));
    FC_CUDA(cudaMemsetAsync(counts.get(), 0, counts.bytes(), stream()));
    FC_CUDA(cudaStreamSynchronize(stream()));
    sort_seconds = window_seconds = 0.0;
  }

  void stats(fc_assign_stats *s) {
    double tot[2];
    unsigned long long added = 0;
    FC_CUDA(cudaMemcpyAsync(tot, totals.get(), sizeof(tot),
                            cudaMemcpyDeviceToHost, stream()));
    FC_CUDA(cudaMemcpyAsync(&added, counts.get(), sizeof(added),
                            cudaMemcpyDeviceToHost, stream()));
    FC_CUDA(cudaStreamSynchronize(stream()));
    s->num_added = added;
    s->num_skipped = num_seen - added;
    s->totw = tot[0];
    s->totwsq = tot[1];
    s->sort_time = sort_seconds;
    s->window_time = window_seconds;
  }
};

Assignor *assignor_new(Grid *g, int scheme, bool periodic) {
  return new Assignor(g, scheme, periodic, 0);
}
void assignor_delete(Assignor *a) { delete a; }
void assignor_prepare_graph(Assignor *a, int64_t max_n, cudaStream_t s) {
  a->stream_override = s;
  a->prepare_graph(max_n);
}
void assignor_enqueue_graph(Assignor *a, const double *posw, int64_t n,
                            cudaStream_t s) {
  a->stream_override = s;
  a->enqueue_graph(posw, n);
}
void assignor_add_device(Assignor *a, const double *posw, int64_t n) {
  a->add_device_posw(posw, n, cudaMemcpyDeviceToDevice);
  a->flush();
  FC_CUDA(cudaStreamSynchronize(a->stream()));
}
void assignor_clear(Assignor *a) { a->clear(); }
bool assignor_has_d12() { return FC_HAVE_D12 != 0; }
void assignor_stats(Assignor *a, fc_assign_stats *s) { a->stats(s); }
size_t assignor_bytes(const int shape[3], int64_t n) {
  // Keys, indices and their sort copies, plus the sort's scratch.
  int64_t nt = 1;
  for (int i = 0; i < 3; ++i) nt *= (shape[i] + kTile - 1) / kTile;
  const bool wide = (uint64_t)nt * kTileCells >= 0xffffffffull;
  const size_t per = (wide ? 8 : 4) * 2 + 4 * 2 + 8;
  // Per unit (up to 4 per tile): start, colour list entry and range.
  return (size_t)std::max<int64_t>(n, 1) * per + (size_t)nt * 4 * 24 + (1 << 20);
}
const double *assignor_totals(const Assignor *a) { return a->totals.as<double>(); }
const unsigned long long *assignor_counts(const Assignor *a) {
  return a->counts.as<unsigned long long>();
}

}  // namespace fc

using namespace fc;

namespace {
Assignor *as_assignor(fc_assignor *a) {
  FC_REQUIRE(a, FC_ERR_INVALID, "null assignor handle");
  return reinterpret_cast<Assignor *>(a);
}
}  // namespace

extern "C" {

int fc_assignor_create(fc_grid *grid, int scheme, int periodic_wrap,
                       int64_t buffer_size, fc_assignor **out) {
  return guard([&] {
    FC_REQUIRE(out, FC_ERR_INVALID, "null argument");
    *out = nullptr;
    Assignor *a =
        new Assignor(as_grid(grid), scheme, periodic_wrap != 0, buffer_size);
    FC_CUDA(cudaStreamSynchronize(a->stream()));
    *out = reinterpret_cast<fc_assignor *>(a);
  });
}

int fc_assignor_destroy(fc_assignor *ma) {
  return guard([&] { delete reinterpret_cast<Assignor *>(ma); });
}

int fc_assignor_add_posw(fc_assignor *ma, const double *posw, int64_t n) {
  return guard([&] {
    Assignor *a = as_assignor(ma);
    FC_REQUIRE(posw || n == 0, FC_ERR_INVALID, "null particle array");
    a->add_device_posw(posw, n, cudaMemcpyHostToDevice);
    FC_CUDA(cudaStreamSynchronize(a->stream()));
  });
}

int fc_assignor_add_posw_device(fc_assignor *ma, const double *posw_device,
                                int64_t n) {
  return guard([&] {
    Assignor *a = as_assignor(ma);
    FC_REQUIRE(posw_device || n == 0, FC_ERR_INVALID, "null particle array");
    a->add_device_posw(posw_device, n, cudaMemcpyDeviceToDevice);
    FC_CUDA(cudaStreamSynchronize(a->stream()));
  });
}

int fc_assignor_add_random(fc_assignor *ma, int64_t n, double particle_weight,
                           const double *disp, uint64_t seed, int64_t batch_size) {
  return guard([&] {
    as_assignor(ma)->add_random(n, particle_weight, disp, seed, batch_size);
  });
}

int fc_assignor_add_pos_weights(fc_assignor *ma, const double *pos,
                                const double *weights, int64_t n) {
  return guard([&] {
    Assignor *a = as_assignor(ma);
    FC_REQUIRE((pos && weights) || n == 0, FC_ERR_INVALID,
               "null particle array");
    a->add_pos(pos, weights, 0.0, n);
    FC_CUDA(cudaStreamSynchronize(a->stream()));
  });
}

int fc_assignor_add_pos_weight(fc_assignor *ma, const double *pos,
                               double weight, int64_t n) {
  return guard([&] {
    Assignor *a = as_assignor(ma);
    FC_REQUIRE(pos || n == 0, FC_ERR_INVALID, "null particle array");
    a->add_pos(pos, nullptr, weight, n);
    FC_CUDA(cudaStreamSynchronize(a->stream()));
  });
}

int fc_assignor_flush(fc_assignor *ma) {
  return guard([&] {
    Assignor *a = as_assignor(ma);
    a->flush();
    FC_CUDA(cudaStreamSynchronize(a->stream()));
  });
}

int fc_assignor_clear(fc_assignor *ma) {
  return guard([&] { as_assignor(ma)->clear(); });
}

int fc_assignor_stats(fc_assignor *ma, fc_assign_stats *stats) {
  return guard([&] {
    FC_REQUIRE(stats, FC_ERR_INVALID, "null argument");
    as_assignor(ma)->stats(stats);
  });
}

int fc_assignor_buffer_size(const fc_assignor *ma, int64_t *buffer_size) {
  return guard([&] {
    FC_REQUIRE(ma && buffer_size, FC_ERR_INVALID, "null argument");
    *buffer_size = reinterpret_cast<const Assignor *>(ma)->buffer_size;
  });
}

}  // extern "C"
