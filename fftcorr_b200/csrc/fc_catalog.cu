// fc_catalog.cu -- synthetic catalogs generated in device memory, and the
// displacement of positions by a gridded field.
//
// add_random_particles (fftcorr/catalog/random_catalog.py:8-87) draws
// uniform positions over the grid's box with numpy and feeds them to a
// MassAssignor; apply_displacement_field (fftcorr/grid/utils.pyx:21-55)
// adds the displacement of each position's cell.  Here both run on the GPU
// so randoms never cross PCIe.  The generator is counter-based: Philox4x32
// with 10 rounds (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011), so particle i's values depend only on (seed,
// i) and any split of the work into batches gives the same catalog.  The
// streams differ from numpy's PCG64, so a device catalog matches the
// reference's only in distribution, not value by value.
#include <cmath>
#include <cstring>

#include "fc_internal.h"

namespace fc {
namespace {

struct U4 {
  uint32_t v[4];
};

// Philox4x32-10: the round function and key schedule of the SC'11 paper.
__device__ __forceinline__ U4 philox(uint64_t counter, uint32_t stream,
                                     uint64_t seed) {
  uint32_t c0 = (uint32_t)counter, c1 = (uint32_t)(counter >> 32);
  uint32_t c2 = stream, c3 = 0x2545F491u;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
    const uint32_t hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += W0;
    k1 += W1;
  }
  return U4{{c0, c1, c2, c3}};
}

// Uniform double in [0, 1) with 53 random bits.
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) *
         (1.0 / 9007199254740992.0);
}

// Two independent standard normals by the Box-Muller transform.
__device__ __forceinline__ void box_muller(double ua, double ub, double *z0,
                                           double *z1) {
  const double r = sqrt(-2.0 * log(1.0 - ua));  // 1 - ua in (0, 1]
  double s, c;
  sincospi(2.0 * ub, &s, &c);
  *z0 = r * c;
  *z1 = r * s;
}

// Streams of the generator.
enum : uint32_t {
  kStreamUniform = 1,
  kStreamUniform2 = 2,
  kStreamCentre = 3,
  kStreamMember = 4,
  kStreamMember2 = 5,
  kStreamMember3 = 6,
  kStreamSector = 7,
  kStreamSector2 = 8
};

__device__ __forceinline__ double wrap_box(double x, double len) {
  x -= len * floor(x / len);
  return x >= len ? 0.0 : x;
}

// Uniform positions over [lo, hi) per axis, weights w0 + (w1 - w0) u.
__global__ void k_uniform(double *__restrict__ posw, int64_t first, int64_t n,
                          double3 lo, double3 hi, double w0, double w1,
                          uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t id = (uint64_t)(first + i);
    const U4 a = philox(id, kStreamUniform, seed);
    const U4 b = philox(id, kStreamUniform2, seed);
    double *p = posw + 4 * i;
    p[0] = lo.x + (hi.x - lo.x) * u53(a.v[0], a.v[1]);
    p[1] = lo.y + (hi.y - lo.y) * u53(a.v[2], a.v[3]);
    p[2] = lo.z + (hi.z - lo.z) * u53(b.v[0], b.v[1]);
    p[3] = w0 == w1 ? w0 : w0 + (w1 - w0) * u53(b.v[2], b.v[3]);
  }
}

// Cluster centres uniform in the periodic box [0, len)^3.
__global__ void k_centres(double *__restrict__ c, int nc, double len,
                          uint64_t seed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc;
       i += gridDim.x * blockDim.x) {
    const U4 a = philox((uint64_t)i, kStreamCentre, seed);
    const U4 b = philox((uint64_t)i, kStreamUniform2, seed ^ 0x5bd1e995ull);
    c[3 * i + 0] = len * u53(a.v[0], a.v[1]);
    c[3 * i + 1] = len * u53(a.v[2], a.v[3]);
    c[3 * i + 2] = len * u53(b.v[0], b.v[1]);
  }
}

// Each point: a uniformly chosen centre plus N(0, sigma^2 I), wrapped into
// the periodic box.
__global__ void k_clustered(double *__restrict__ posw, int64_t first,
                            int64_t n, const double *__restrict__ centres,
                            int nc, double len, double sigma, double w0,
                            double w1, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t id = (uint64_t)(first + i);
    const U4 a = philox(id, kStreamMember, seed);
    const U4 b = philox(id, kStreamMember2, seed);
    const U4 d = philox(id, kStreamMember3, seed);
    int ci = (int)(u53(a.v[0], a.v[1]) * nc);
    if (ci >= nc) ci = nc - 1;
    double z0, z1, z2, z3;
    box_muller(u53(a.v[2], a.v[3]), u53(b.v[0], b.v[1]), &z0, &z1);
    box_muller(u53(b.v[2], b.v[3]), u53(d.v[0], d.v[1]), &z2, &z3);
    double *p = posw + 4 * i;
    p[0] = wrap_box(centres[3 * ci + 0] + sigma * z0, len);
    p[1] = wrap_box(centres[3 * ci + 1] + sigma * z1, len);
    p[2] = wrap_box(centres[3 * ci + 2] + sigma * z2, len);
    p[3] = w0 == w1 ? w0 : w0 + (w1 - w0) * u53(d.v[2], d.v[3]);
  }
}

// Uniform in the volume of a spherical-shell sector about the origin:
// r^3 uniform in [rmin^3, rmax^3), RA uniform in [-ra, ra] about +x,
// sin(Dec) uniform in [-sin(dec), sin(dec)].
__global__ void k_sector(double *__restrict__ posw, int64_t first, int64_t n,
                         double rmin, double rmax, double ra, double dec,
                         double w0, double w1, double wsign, uint64_t seed) {
  const double r3a = rmin * rmin * rmin, r3b = rmax * rmax * rmax;
  const double sd = sin(dec);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t id = (uint64_t)(first + i);
    const U4 a = philox(id, kStreamSector, seed);
    const U4 b = philox(id, kStreamSector2, seed);
    const double r = cbrt(r3a + (r3b - r3a) * u53(a.v[0], a.v[1]));
    const double phi = ra * (2.0 * u53(a.v[2], a.v[3]) - 1.0);
    const double sdec = sd * (2.0 * u53(b.v[0], b.v[1]) - 1.0);
    const double cdec = sqrt(1.0 - sdec * sdec);
    double sp, cp;
    sincos(phi, &sp, &cp);
    double *p = posw + 4 * i;
    p[0] = r * cdec * cp;
    p[1] = r * cdec * sp;
    p[2] = r * sdec;
    p[3] = wsign * (w0 == w1 ? w0 : w0 + (w1 - w0) * u53(b.v[2], b.v[3]));
  }
}

__device__ __forceinline__ bool in_sector(double x, double y, double z,
                                          double rmin, double rmax, double ra,
                                          double sdec) {
  const double r = sqrt(x * x + y * y + z * z);
  if (!(r >= rmin && r < rmax)) return false;
  if (fabs(atan2(y, x)) > ra) return false;
  return fabs(z) <= sdec * r;
}

// Clustered points in the sector: a uniformly chosen centre (from k_sector)
// plus N(0, sigma^2 I), redrawn until inside the sector (at most 64 draws;
// then the centre itself).
__global__ void k_sector_clustered(double *__restrict__ posw, int64_t n,
                                   const double *__restrict__ centres, int nc,
                                   double sigma, double rmin, double rmax,
                                   double ra, double dec, double w0, double w1,
                                   double wsign, uint64_t seed) {
  const double sdec = sin(dec);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const U4 a = philox((uint64_t)i, kStreamMember, seed);
    int ci = (int)(u53(a.v[0], a.v[1]) * nc);
    if (ci >= nc) ci = nc - 1;
    const double *c = centres + 4 * ci;
    double x = c[0], y = c[1], z = c[2];
    for (uint32_t t = 0; t < 64; ++t) {
      const U4 b = philox((uint64_t)i, 16 + 2 * t, seed);
      const U4 d = philox((uint64_t)i, 17 + 2 * t, seed);
      double z0, z1, z2, z3;
      box_muller(u53(b.v[0], b.v[1]), u53(b.v[2], b.v[3]), &z0, &z1);
      box_muller(u53(d.v[0], d.v[1]), u53(d.v[2], d.v[3]), &z2, &z3);
      const double px = c[0] + sigma * z0, py = c[1] + sigma * z1,
                   pz = c[2] + sigma * z2;
      if (in_sector(px, py, pz, rmin, rmax, ra, sdec)) {
        x = px;
        y = py;
        z = pz;
        break;
      }
    }
    double *p = posw + 4 * i;
    p[0] = x;
    p[1] = y;
    p[2] = z;
    p[3] = wsign * (w0 == w1 ? w0 : w0 + (w1 - w0) * u53(a.v[2], a.v[3]));
  }
}

// out = pos + disp[cell of pos] (utils.pyx:21-40); flag[0] = 1 when a
// position has no cell (outside the grid without periodic wrap).
__global__ void k_displace(const double *__restrict__ pos, int stride,
                           int64_t n, const double *__restrict__ disp,
                           AssignGeomLite g, double *__restrict__ out,
                           int out_stride, int *flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double *p = pos + stride * i;
    int c[3];
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      double x = (p[a] - g.posmin[a]) / g.cell;
      const double xmax = g.n[a];
      if (x < 0 || x >= xmax) {
        if (!g.periodic) {
          ok = false;
          break;
        }
        x = fmod(x, xmax);
        if (x < 0) x += xmax;
      }
      c[a] = (int)x;
    }
    if (!ok) {
      flag[0] = 1;
      continue;
    }
    const double *d =
        disp + 3 * (((int64_t)c[0] * g.n[1] + c[1]) * g.n[2] + c[2]);
    double *o = out + out_stride * i;
    o[0] = p[0] + d[0];
    o[1] = p[1] + d[1];
    o[2] = p[2] + d[2];
  }
}

unsigned gen_blocks(int64_t n) { return grid_for((size_t)std::max<int64_t>(n, 1), 256); }

}  // namespace

void catalog_uniform(double *posw, int64_t first, int64_t n, const double lo[3],
                     const double hi[3], double w0, double w1, uint64_t seed,
                     cudaStream_t s) {
  if (n <= 0) return;
  k_uniform<<<gen_blocks(n), 256, 0, s>>>(posw, first, n,
                                          make_double3(lo[0], lo[1], lo[2]),
                                          make_double3(hi[0], hi[1], hi[2]), w0,
                                          w1, seed);
  FC_LAUNCH_CHECK();
}

size_t catalog_scratch_bytes(const fc_catalog_spec &c) {
  const bool clustered =
      c.kind == FC_CAT_CLUSTERED_BOX || c.kind == FC_CAT_SECTOR_CLUSTERED;
  return clustered && c.ncentres > 0 ? (size_t)c.ncentres * 4 * sizeof(double)
                                     : 0;
}

void catalog_generate(const fc_catalog_spec &c, double *posw, cudaStream_t s,
                      double *scratch, size_t scratch_bytes) {
  // Cluster centres go to the caller's scratch when it is large enough, else
  // to a stream-ordered allocation.
  auto centres_buffer = [&](size_t bytes) {
    double *p = nullptr;
    if (scratch && scratch_bytes >= bytes) return scratch;
    FC_CUDA(cudaMallocAsync(&p, bytes, s));
    return p;
  };
  auto release = [&](double *p) {
    if (p != scratch) FC_CUDA(cudaFreeAsync(p, s));
  };
  const int64_t n = c.n;
  if (n <= 0) return;
  switch (c.kind) {
    case FC_CAT_DEVICE:
      FC_REQUIRE(c.posw, FC_ERR_INVALID, "null particle array");
      FC_CUDA(cudaMemcpyAsync(posw, c.posw, (size_t)n * 32,
                              cudaMemcpyDeviceToDevice, s));
      return;
    case FC_CAT_HOST:
      FC_REQUIRE(c.posw, FC_ERR_INVALID, "null particle array");
      FC_CUDA(cudaMemcpyAsync(posw, c.posw, (size_t)n * 32,
                              cudaMemcpyHostToDevice, s));
      return;
    case FC_CAT_UNIFORM_BOX: {
      const double lo[3] = {0, 0, 0};
      const double hi[3] = {c.boxsize, c.boxsize, c.boxsize};
      catalog_uniform(posw, 0, n, lo, hi, c.wmin, c.wmax, c.seed, s);
      return;
    }
    case FC_CAT_CLUSTERED_BOX: {
      FC_REQUIRE(c.ncentres > 0, FC_ERR_INVALID, "ncentres must be positive");
      // Stream-ordered scratch: no device-wide synchronisation.
      double *centres = centres_buffer((size_t)c.ncentres * 3 * sizeof(double));
      k_centres<<<gen_blocks(c.ncentres), 256, 0, s>>>(centres, c.ncentres,
                                                       c.boxsize, c.seed);
      FC_LAUNCH_CHECK();
      k_clustered<<<gen_blocks(n), 256, 0, s>>>(posw, 0, n, centres, c.ncentres,
                                                c.boxsize, c.sigma, c.wmin,
                                                c.wmax, c.seed);
      FC_LAUNCH_CHECK();
      release(centres);
      return;
    }
    case FC_CAT_SECTOR_UNIFORM:
      k_sector<<<gen_blocks(n), 256, 0, s>>>(posw, 0, n, c.rmin, c.rmax,
                                             c.ra_half, c.dec_half, c.wmin,
                                             c.wmax, c.wsign, c.seed);
      FC_LAUNCH_CHECK();
      return;
    case FC_CAT_SECTOR_CLUSTERED: {
      FC_REQUIRE(c.ncentres > 0, FC_ERR_INVALID, "ncentres must be positive");
      double *centres = centres_buffer((size_t)c.ncentres * 4 * sizeof(double));
      k_sector<<<gen_blocks(c.ncentres), 256, 0, s>>>(
          centres, 0, c.ncentres, c.rmin, c.rmax, c.ra_half, c.dec_half, 1.0,
          1.0, 1.0, c.seed ^ 0x3c6ef372fe94f82bull);
      FC_LAUNCH_CHECK();
      k_sector_clustered<<<gen_blocks(n), 256, 0, s>>>(
          posw, n, centres, c.ncentres, c.sigma, c.rmin, c.rmax, c.ra_half,
          c.dec_half, c.wmin, c.wmax, c.wsign, c.seed);
      FC_LAUNCH_CHECK();
      release(centres);
      return;
    }
  }
  FC_THROW(FC_ERR_INVALID, "unknown catalog kind");
}

void displace(const double *pos, int stride, int64_t n, const double *disp,
              const AssignGeomLite &g, double *out, int out_stride, int *flag,
              cudaStream_t s) {
  if (n <= 0) return;
  k_displace<<<gen_blocks(n), 256, 0, s>>>(pos, stride, n, disp, g, out,
                                           out_stride, flag);
  FC_LAUNCH_CHECK();
}

}  // namespace fc

using namespace fc;

extern "C" {

int fc_catalog_uniform(double *posw_device, int64_t n, const double lo[3],
                       const double hi[3], double wmin, double wmax,
                       uint64_t seed) {
  return guard([&] {
    FC_REQUIRE(lo && hi && (n == 0 || posw_device), FC_ERR_INVALID,
               "null argument");
    FC_REQUIRE(n >= 0, FC_ERR_INVALID, "negative count");
    for (int a = 0; a < 3; ++a)
      FC_REQUIRE(hi[a] > lo[a], FC_ERR_INVALID, "empty box");
    catalog_uniform(posw_device, 0, n, lo, hi, wmin, wmax, seed, 0);
    FC_CUDA(cudaStreamSynchronize(0));
  });
}

int fc_catalog_clustered_box(double *posw_device, int64_t n, double boxsize,
                             int ncentres, double sigma, double wmin,
                             double wmax, uint64_t seed) {
  return guard([&] {
    FC_REQUIRE(n >= 0 && (n == 0 || posw_device), FC_ERR_INVALID,
               "null argument");
    FC_REQUIRE(boxsize > 0 && ncentres > 0 && sigma >= 0, FC_ERR_INVALID,
               "boxsize and ncentres must be positive, sigma >= 0");
    if (n == 0) return;
    DeviceBuffer centres((size_t)ncentres * 3 * sizeof(double));
    k_centres<<<gen_blocks(ncentres), 256>>>(centres.as<double>(), ncentres,
                                            boxsize, seed);
    FC_LAUNCH_CHECK();
    k_clustered<<<gen_blocks(n), 256>>>(posw_device, 0, n, centres.as<double>(),
                                       ncentres, boxsize, sigma, wmin, wmax,
                                       seed);
    FC_LAUNCH_CHECK();
    FC_CUDA(cudaStreamSynchronize(0));
  });
}

int fc_catalog_sector(double *posw_device, int64_t n, double rmin, double rmax,
                      double ra_half, double dec_half, double wmin, double wmax,
                      double wsign, uint64_t seed) {
  return guard([&] {
    FC_REQUIRE(n >= 0 && (n == 0 || posw_device), FC_ERR_INVALID,
               "null argument");
    FC_REQUIRE(rmax > rmin && rmin >= 0, FC_ERR_INVALID, "need 0 <= rmin < rmax");
    if (n == 0) return;
    k_sector<<<gen_blocks(n), 256>>>(posw_device, 0, n, rmin, rmax, ra_half,
                                    dec_half, wmin, wmax, wsign, seed);
    FC_LAUNCH_CHECK();
    FC_CUDA(cudaStreamSynchronize(0));
  });
}

int fc_catalog_generate(const fc_catalog_spec *spec, double *posw_device) {
  return guard([&] {
    FC_REQUIRE(spec, FC_ERR_INVALID, "null argument");
    FC_REQUIRE(spec->n >= 0, FC_ERR_INVALID, "negative count");
    FC_REQUIRE(spec->n == 0 || posw_device, FC_ERR_INVALID, "null output");
    catalog_generate(*spec, posw_device, 0);
    FC_CUDA(cudaStreamSynchronize(0));
  });
}

int fc_apply_displacement(const fc_grid *grid, const double *pos, int64_t n,
                          const double *disp, int periodic_wrap, double *out) {
  return guard([&] {
    const Grid *g = as_grid(grid);
    FC_REQUIRE(n >= 0, FC_ERR_INVALID, "negative count");
    FC_REQUIRE(n == 0 || (pos && disp && out), FC_ERR_INVALID, "null argument");
    if (n == 0) return;
    AssignGeomLite geo;
    for (int a = 0; a < 3; ++a) {
      geo.n[a] = g->shape[a];
      geo.posmin[a] = g->posmin[a];
    }
    geo.cell = g->cell_size;
    geo.periodic = periodic_wrap ? 1 : 0;
    const size_t nd = g->size() * 3;
    DeviceBuffer dpos((size_t)n * 3 * sizeof(double)), dout((size_t)n * 3 * sizeof(double));
    DeviceBuffer ddisp(nd * sizeof(double)), dflag(sizeof(int));
    cudaStream_t s = g->stream;
    FC_CUDA(cudaMemcpyAsync(dpos.get(), pos, (size_t)n * 3 * sizeof(double),
                            cudaMemcpyHostToDevice, s));
    FC_CUDA(cudaMemcpyAsync(ddisp.get(), disp, nd * sizeof(double),
                            cudaMemcpyHostToDevice, s));
    FC_CUDA(cudaMemsetAsync(dflag.get(), 0, sizeof(int), s));
    displace(dpos.as<double>(), 3, n, ddisp.as<double>(), geo, dout.as<double>(),
             3, dflag.as<int>(), s);
    int flag = 0;
    FC_CUDA(cudaMemcpyAsync(&flag, dflag.get(), sizeof(int),
                            cudaMemcpyDeviceToHost, s));
    FC_CUDA(cudaMemcpyAsync(out, dout.get(), (size_t)n * 3 * sizeof(double),
                            cudaMemcpyDeviceToHost, s));
    FC_CUDA(cudaStreamSynchronize(s));
    FC_REQUIRE(!flag, FC_ERR_INVALID,
               "Failed to apply displacement field: coordinates out of bounds? "
               "Try setting periodic_wrap=True.");
  });
}

}  // extern "C"
