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
//   K-tiles   first sorted position of every 8x8x8 tile (binary search)
//   K-scatter one CTA per tile.  NGP/CIC/TSC: a thread per home cell sums
//             its particles' stencil products in registers, and every cell
//             of the tile's footprint (tile + stencil halo) adds the home
//             cells' sums in a fixed order.  D12 (8^3 taps): particles are
//             staged in shared memory with their 1-D weights and every
//             footprint cell sums its contributions in a fixed order (home
//             cell, then sorted particle order).  Either way each footprint
//             total is added to the grid once.  Tiles are processed in colour
//             passes chosen so that footprints within one pass never
//             overlap, so there are no atomics and the result is
//             bit-reproducible run to run.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "fc_common.cuh"
#include "fc_internal.h"

#if __has_include("_gen/d12_table.inc")
#define FC_HAVE_D12 1
#else
#define FC_HAVE_D12 0
#endif

namespace fc {
namespace {

constexpr int kTile = 8;         // tile edge in cells
constexpr int kTileCells = 512;  // cells per tile
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
  int periodic;
};

// config_space_grid.h:31-46 on the device.
__device__ __forceinline__ bool dev_grid_coords(const double *p,
                                                const AssignGeom &g,
                                                double x[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double xi = (p[i] - g.posmin[i]) / g.cell;
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

// floor(x) as a cell index.  A wrapped coordinate can round up to exactly
// n; that point is the upper edge of cell n-1, which is where it goes.
__device__ __forceinline__ int home_cell(double x, int n) {
  int i = (int)floor(x);
  return i >= n ? n - 1 : (i < 0 ? 0 : i);
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
    vals[pi] = (uint32_t)pi;
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

// K-tiles: tile_start[t] = first sorted index whose key >= t*512, for
// t in [0, ntiles]; invalid keys (== ntiles*512) sort last.
template <typename KeyT>
__global__ void k_tile_starts(const KeyT *keys, int64_t n, int64_t ntiles,
                              uint32_t *tile_start) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t <= ntiles;
       t += (int64_t)gridDim.x * blockDim.x) {
    const KeyT target = (KeyT)t * kTileCells;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < target)
        lo = mid + 1;
      else
        hi = mid;
    }
    tile_start[t] = (uint32_t)lo;
  }
}

// (tile, first particle, end) of every tile in colour order, so a scatter
// CTA finds its work with one load.
__global__ void k_tile_ranges(const uint32_t *__restrict__ tiles, int64_t nt,
                              const uint32_t *__restrict__ tile_start,
                              uint4 *__restrict__ ranges) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nt;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t t = tiles[i];
    ranges[i] = make_uint4(t, tile_start[t], tile_start[t + 1], 0u);
  }
}

// K-scatter for one colour pass.  Shared memory layout:
//   acc[F^3] footprint sums | wts[kChunk][3W] | pcell[kChunk] | cstart[513]
template <int S, typename KeyT>
__global__ void __launch_bounds__(kScatterThreads)
    k_scatter(const double *__restrict__ posw, const KeyT *__restrict__ keys,
              const uint32_t *__restrict__ vals,
              const uint32_t *__restrict__ tile_start,
              const uint32_t *__restrict__ tiles, AssignGeom g,
              double *__restrict__ grid) {
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
      const int ix = home_cell(x[0], g.n[0]);
      const int iy = home_cell(x[1], g.n[1]);
      const int iz = home_cell(x[2], g.n[2]);
      pcell[threadIdx.x] = (int)(keys[c0 + threadIdx.x] & (kTileCells - 1));
      double *wt = wts + threadIdx.x * 3 * W;
      Stencil<S>::weights(x[0] - ix, x[1] - iy, x[2] - iz, p[3], wt, wt + W,
                          wt + 2 * W);
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
    grid[((size_t)gx * g.n[1] + gy) * g.n[2] + gz] += v;
  }
}

// K-scatter for stencils of width <= 3 (NGP, CIC, TSC): one thread per
// home cell of the 8x8x8 tile.  The tile's particles (contiguous in sorted
// order) are staged in chunks: all threads gather positions and weights in
// parallel into shared memory (fractional cell offsets and weight), then
// each thread walks its own cell's particles of the chunk in sorted order
// and accumulates the W^3 products wx[a]*wy[b]*wz[c] in registers
// (S_h[a][b][c]).  The sums go to shared memory, and every footprint cell
// then adds the S_h[o] of the home cells h = f - o in a fixed order.  Each
// cell's particles are summed in sorted order whatever the chunking, so the
// grid is the same bits on every run.
template <int S>
struct ScatterS {
  static constexpr int W = Stencil<S>::W;
  static constexpr int W3 = W * W * W;
  static constexpr int F = kTile + W - 1;
  static constexpr int F3 = F * F * F;
  // Staged particles per chunk: at least 1024, more when the S_h buffer the
  // chunk shares memory with is larger (TSC).
  static constexpr int C0 = (W3 * kTileCells * 8) / 36 / 32 * 32;
  static constexpr int C = C0 > 1024 ? C0 : 1024;
  static constexpr size_t region =
      (size_t)W3 * kTileCells * 8 > (size_t)C * 36 ? (size_t)W3 * kTileCells * 8
                                                   : (size_t)C * 36;
  static constexpr size_t smem = region + (size_t)F3 * 8;
};

__device__ __forceinline__ int lower_bound_smem(const int *a, int n, int v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

template <int S, typename KeyT>
__global__ void __launch_bounds__(kTileCells)
    k_scatter_s(const double *__restrict__ posw, const KeyT *__restrict__ keys,
                const uint32_t *__restrict__ vals,
                const uint4 *__restrict__ ranges, AssignGeom g,
                double *__restrict__ grid) {
  using Q = ScatterS<S>;
  constexpr int W = Q::W;
  constexpr int OMIN = Stencil<S>::OMIN;
  constexpr int W3 = Q::W3;
  constexpr int F = Q::F;
  constexpr int F3 = Q::F3;
  constexpr int C = Q::C;
  extern __shared__ double smem[];
  double *sh = smem;                                   // [W3][512], last
  double *pd = smem;                                   // [C][4], per chunk
  int *pc = reinterpret_cast<int *>(smem + 4 * C);     // [C], per chunk
  double *acc = smem + Q::region / 8;                  // [F3]

  const uint4 rg = ranges[blockIdx.x];
  const uint32_t tile = rg.x;
  const uint32_t ts = rg.y;
  const uint32_t te = rg.z;
  if (ts >= te) return;
  const int tz = tile % g.nt[2];
  const int ty = (tile / g.nt[2]) % g.nt[1];
  const int tx = tile / (g.nt[2] * g.nt[1]);
  const int o0 = tx * kTile, o1 = ty * kTile, o2 = tz * kTile;
  const int h = threadIdx.x;
  const KeyT kbase = (KeyT)tile * kTileCells;
  // When no footprint wraps onto itself, each footprint cell has one
  // global cell: load its current value now, so the latency of the final
  // read-modify-write overlaps the particle gather.  (No other CTA of this
  // colour pass touches these cells.)
  constexpr int kFPer = (F3 + kTileCells - 1) / kTileCells;
  const bool direct = g.n[0] >= F && g.n[1] >= F && g.n[2] >= F;
  size_t gidx[kFPer];
  double gval[kFPer];
#pragma unroll
  for (int r = 0; r < kFPer; ++r) {
    const int f = threadIdx.x + r * kTileCells;
    gidx[r] = 0;
    gval[r] = 0.0;
    if (direct && f < F3) {
      int gx = (o0 + f / (F * F) + OMIN) % g.n[0];
      int gy = (o1 + (f / F) % F + OMIN) % g.n[1];
      int gz = (o2 + f % F + OMIN) % g.n[2];
      if (gx < 0) gx += g.n[0];
      if (gy < 0) gy += g.n[1];
      if (gz < 0) gz += g.n[2];
      gidx[r] = ((size_t)gx * g.n[1] + gy) * g.n[2] + gz;
      gval[r] = grid[gidx[r]];
    }
  }

  double sacc[W3];
#pragma unroll
  for (int o = 0; o < W3; ++o) sacc[o] = 0.0;
  for (uint32_t c0 = ts; c0 < te; c0 += C) {
    const int m = (int)min((uint32_t)C, te - c0);
    if (c0 != ts) __syncthreads();  // the previous chunk has been consumed
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      const uint32_t q = c0 + i;
      const double *p = posw + 4 * (size_t)vals[q];
      double x[3];
      dev_grid_coords(p, g, x);
      pd[4 * i + 0] = x[0] - home_cell(x[0], g.n[0]);
      pd[4 * i + 1] = x[1] - home_cell(x[1], g.n[1]);
      pd[4 * i + 2] = x[2] - home_cell(x[2], g.n[2]);
      pd[4 * i + 3] = p[3];
      pc[i] = (int)(keys[q] - kbase);
    }
    __syncthreads();
    const int lo = lower_bound_smem(pc, m, h);
    const int hi = lower_bound_smem(pc, m, h + 1);
    for (int i = lo; i < hi; ++i) {
      double wx[W], wy[W], wz[W];
      Stencil<S>::weights(pd[4 * i + 0], pd[4 * i + 1], pd[4 * i + 2],
                          pd[4 * i + 3], wx, wy, wz);
#pragma unroll
      for (int a = 0; a < W; ++a)
#pragma unroll
        for (int b = 0; b < W; ++b) {
          const double wxy = wx[a] * wy[b];
#pragma unroll
          for (int c = 0; c < W; ++c) sacc[(a * W + b) * W + c] += wxy * wz[c];
        }
    }
  }
  __syncthreads();  // the chunk buffer becomes S_h
#pragma unroll
  for (int o = 0; o < W3; ++o) sh[o * kTileCells + h] = sacc[o];
  __syncthreads();
  for (int f = threadIdx.x; f < F3; f += blockDim.x) {
    const int fx = f / (F * F);
    const int fy = (f / F) % F;
    const int fz = f % F;
    double a = 0.0;
#pragma unroll
    for (int ox = 0; ox < W; ++ox) {
      const int hx = fx - ox;
      if (hx < 0 || hx >= kTile) continue;
#pragma unroll
      for (int oy = 0; oy < W; ++oy) {
        const int hy = fy - oy;
        if (hy < 0 || hy >= kTile) continue;
#pragma unroll
        for (int oz = 0; oz < W; ++oz) {
          const int hz = fz - oz;
          if (hz < 0 || hz >= kTile) continue;
          a += sh[((ox * W + oy) * W + oz) * kTileCells + (hx * 64 + hy * 8 + hz)];
        }
      }
    }
    acc[f] = a;
  }
  __syncthreads();
  if (direct) {
#pragma unroll
    for (int r = 0; r < kFPer; ++r) {
      const int f = threadIdx.x + r * kTileCells;
      if (f >= F3) continue;
      const double v = 0.0 + acc[f];
      if (v != 0.0) grid[gidx[r]] = gval[r] + v;
    }
    return;
  }
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
    grid[((size_t)gx * g.n[1] + gy) * g.n[2] + gz] += v;
  }
}

template <int S>
size_t scatter_s_smem() {
  return ScatterS<S>::smem;
}

template <int S>
size_t scatter_smem() {
  constexpr int W = Stencil<S>::W;
  constexpr int F = kTile + W - 1;
  return sizeof(double) * (F * F * F + kChunk * 3 * W) +
         sizeof(int) * (kChunk + kTileCells + 1);
}

// Greedy colouring of the tiles along one axis so that tiles sharing a
// colour have disjoint (periodically wrapped) footprints.
std::vector<int> color_axis(int n, int ntiles, int W, int omin) {
  std::vector<std::vector<char>> cover(ntiles, std::vector<char>(n, 0));
  for (int t = 0; t < ntiles; ++t) {
    const int lo = t * kTile;
    const int hi = std::min(n, lo + kTile) - 1;
    for (int c = lo + omin; c <= hi + omin + W - 1; ++c)
      cover[t][((c % n) + n) % n] = 1;
  }
  std::vector<int> color(ntiles, -1);
  for (int t = 0; t < ntiles; ++t) {
    for (int c = 0;; ++c) {
      bool ok = true;
      for (int u = 0; u < t && ok; ++u) {
        if (color[u] != c) continue;
        for (int k = 0; k < n; ++k)
          if (cover[t][k] && cover[u][k]) {
            ok = false;
            break;
          }
      }
      if (ok) {
        color[t] = c;
        break;
      }
    }
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

}  // namespace

// MassAssignor state (mass_assignor.h:30-234) with a device-side buffer.
struct Assignor {
  Grid *grid;
  int scheme;
  bool periodic;
  int64_t buffer_size;
  AssignGeom geom;
  int64_t ntiles;
  bool wide_keys;  // 64-bit keys when the key space exceeds 32 bits
  int end_bit;

  // Buffered particles.
  int64_t count = 0;
  int64_t capacity = 0;
  DeviceBuffer posw, keys, keys_alt, vals, vals_alt, cub_temp;
  DeviceBuffer tile_start;
  DeviceBuffer color_tiles;
  DeviceBuffer tile_ranges;            // uint4 per tile, colour order
  std::vector<int64_t> color_offsets;  // per colour, into color_tiles
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
      : grid(g), scheme(scheme_), periodic(periodic_), buffer_size(buffer_size_) {
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
    geom.periodic = periodic ? 1 : 0;
    ntiles = (int64_t)geom.nt[0] * geom.nt[1] * geom.nt[2];
    const uint64_t max_key = (uint64_t)ntiles * kTileCells;  // invalid key
    wide_keys = max_key >= 0xffffffffull;
    end_bit = 1;
    while (end_bit < 64 && (max_key >> end_bit) != 0) ++end_bit;
    tile_start.resize((ntiles + 1) * sizeof(uint32_t));
    tile_ranges.resize(std::max<int64_t>(ntiles, 1) * sizeof(uint4));
    partials.resize(2 * kSumBlocks * sizeof(double));
    totals.resize(2 * sizeof(double));
    counts.resize(sizeof(unsigned long long));
    build_colors();
    FC_CUDA(cudaMemsetAsync(totals.get(), 0, totals.bytes(), grid->stream));
    FC_CUDA(cudaMemsetAsync(counts.get(), 0, counts.bytes(), grid->stream));
    for (auto fn : {(const void *)k_scatter_s<0, uint32_t>,
                    (const void *)k_scatter_s<0, uint64_t>,
                    (const void *)k_scatter_s<1, uint32_t>,
                    (const void *)k_scatter_s<1, uint64_t>,
                    (const void *)k_scatter_s<3, uint32_t>,
                    (const void *)k_scatter_s<3, uint64_t>})
      FC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)scatter_s_smem<1>()));
    if (scheme == 2) {
      FC_CUDA(cudaFuncSetAttribute(k_scatter<2, uint32_t>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)scatter_smem<2>()));
      FC_CUDA(cudaFuncSetAttribute(k_scatter<2, uint64_t>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)scatter_smem<2>()));
    }
  }

  ~Assignor() {
    if (grid && grid->stream) cudaStreamSynchronize(grid->stream);
  }

  cudaStream_t stream() const {
    return stream_override ? stream_override : grid->stream;
  }

  void build_colors() {
    int omin = 0;
    const int W = stencil_width(scheme, &omin);
    std::vector<int> col[3];
    int ncol[3];
    for (int a = 0; a < 3; ++a) {
      col[a] = color_axis(geom.n[a], geom.nt[a], W, omin);
      ncol[a] = 1 + *std::max_element(col[a].begin(), col[a].end());
    }
    const int ncolors = ncol[0] * ncol[1] * ncol[2];
    std::vector<std::vector<uint32_t>> lists(ncolors);
    for (int tx = 0; tx < geom.nt[0]; ++tx)
      for (int ty = 0; ty < geom.nt[1]; ++ty)
        for (int tz = 0; tz < geom.nt[2]; ++tz) {
          const int c = (col[0][tx] * ncol[1] + col[1][ty]) * ncol[2] + col[2][tz];
          lists[c].push_back(
              (uint32_t)(((int64_t)tx * geom.nt[1] + ty) * geom.nt[2] + tz));
        }
    std::vector<uint32_t> flat;
    flat.reserve(ntiles);
    color_offsets.assign(1, 0);
    for (auto &l : lists) {
      flat.insert(flat.end(), l.begin(), l.end());
      color_offsets.push_back((int64_t)flat.size());
    }
    color_tiles.resize(flat.size() * sizeof(uint32_t));
    FC_CUDA(cudaMemcpy(color_tiles.get(), flat.data(),
                       flat.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
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
          keys.as<uint32_t>(), vals.as<uint32_t>(), parts,
          counts.as<unsigned long long>());
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
          vals.as<uint32_t>(), parts, counts.as<unsigned long long>());
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

  template <typename KeyT>
  void flush_typed() {
    const int64_t n = count;
    // K-sort.
    cub::DoubleBuffer<KeyT> dk(keys.as<KeyT>(), keys_alt.as<KeyT>());
    cub::DoubleBuffer<uint32_t> dv(vals.as<uint32_t>(), vals_alt.as<uint32_t>());
    size_t temp = 0;
    FC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, dk, dv, n, 0,
                                            end_bit, stream()));
    if (graph_mode)
      FC_REQUIRE(temp <= cub_temp.bytes(), FC_ERR_STATE,
                 "sort scratch was not prepared for this many particles");
    cub_temp.resize(temp);
    if (!graph_mode) sort_timer.start(stream());
    FC_CUDA(cub::DeviceRadixSort::SortPairs(cub_temp.get(), temp, dk, dv, n, 0,
                                            end_bit, stream()));
    if (!graph_mode) sort_timer.stop(stream());
    const KeyT *sk = dk.Current();
    const uint32_t *sv = dv.Current();
    // K-tiles + K-scatter.
    if (!graph_mode) window_timer.start(stream());
    k_tile_starts<KeyT><<<grid_for(ntiles + 1, 256), 256, 0, stream()>>>(
        sk, n, ntiles, tile_start.as<uint32_t>());
    FC_LAUNCH_CHECK();
    const uint32_t *tiles = color_tiles.as<uint32_t>();
    if (scheme != 2) {
      k_tile_ranges<<<grid_for(ntiles, 256), 256, 0, stream()>>>(
          tiles, ntiles, tile_start.as<uint32_t>(), tile_ranges.as<uint4>());
      FC_LAUNCH_CHECK();
    }
    for (size_t c = 0; c + 1 < color_offsets.size(); ++c) {
      const int64_t nt = color_offsets[c + 1] - color_offsets[c];
      if (nt == 0) continue;
      const uint32_t *ct = tiles + color_offsets[c];
      const uint4 *cr = tile_ranges.as<uint4>() + color_offsets[c];
      switch (scheme) {
        case 0:
          k_scatter_s<0, KeyT><<<(unsigned)nt, kTileCells, scatter_s_smem<0>(),
                                 stream()>>>(src_posw, sk, sv, cr, geom,
                                             grid->ptr());
          break;
        case 1:
          k_scatter_s<1, KeyT><<<(unsigned)nt, kTileCells, scatter_s_smem<1>(),
                                 stream()>>>(src_posw, sk, sv, cr, geom,
                                             grid->ptr());
          break;
        case 2:
          k_scatter<2, KeyT><<<(unsigned)nt, kScatterThreads, scatter_smem<2>(),
                               stream()>>>(src_posw, sk, sv,
                                           tile_start.as<uint32_t>(), ct, geom,
                                           grid->ptr());
          break;
        default:
          k_scatter_s<3, KeyT><<<(unsigned)nt, kTileCells, scatter_s_smem<3>(),
                                 stream()>>>(src_posw, sk, sv, cr, geom,
                                             grid->ptr());
          break;
      }
      FC_LAUNCH_CHECK();
    }
    if (!graph_mode) window_timer.stop(stream());
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
      cub::DoubleBuffer<uint32_t> dk(keys.as<uint32_t>(), keys_alt.as<uint32_t>());
      cub::DoubleBuffer<uint32_t> dv(vals.as<uint32_t>(), vals_alt.as<uint32_t>());
      FC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, dk, dv, max_n, 0,
                                              end_bit, stream()));
    }
    cub_temp.resize(temp + 1024);
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
  return (size_t)std::max<int64_t>(n, 1) * per + (size_t)nt * 8 + (1 << 20);
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
