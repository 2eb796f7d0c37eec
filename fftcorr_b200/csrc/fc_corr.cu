// fc_corr.cu -- PeriodicCorrelator and Correlator (survey, Y_lm about the
// observer) on the GPU.
//
// Reference: cc/correlate/correlator.h:18-505 (geometry, loops,
// normalisations), cc/grid/fft_grid.cc:10-258 (padded in-place r2c/c2r
// layout and the centred subgrid extractions), spherical_harmonics.h:32-179,
// window_correct.h:14-60, histogram_list.h:33-45.
//
// Layout in HBM (per correlator):
//   work  [N0][N1][N2p] real == [N0][N1][N2p/2] complex, N2p = 2(N2/2+1),
//         the FftGrid layout; FP64 or FP32 (mixed precision)
//   g2    [N0][N1][N2/2+1] complex: FFT of grid2 (BaseCorrelator::grid2_fft_)
//   rsub  [R][R][R] FP64, ksub [K0][K1][K2] FP64 subgrid accumulators
//   BinIndex per subgrid: cells sorted by histogram bin
// Per (ell, m) of a survey correlation:
//   k_weight   work = Y_lm(cell) * rho        (make_ylm on the full grid)
//   cuFFT r2c  in place
//   k_conj_mul work *= conj(g2)                (multiply_with_conjugation)
//   k_ksub     ksub += Y_lm(k)*W^-2*4pi*Re(work) on the k-subgrid
//   cuFFT c2r  in place
//   k_rsub     rsub += Y_lm(r)*4pi/N*work on the r-subgrid
// then per ell the two deterministic histograms (fc_hist.cuh).
#include <cufft.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include <cstdlib>
#include <memory>

#include "fc_common.cuh"
#include "fc_fused.h"
#include "fc_hist.cuh"
#include "fc_internal.h"

namespace fc {
namespace {

template <typename T>
struct Cplx;
template <>
struct Cplx<double> {
  using type = double2;
};
template <>
struct Cplx<float> {
  using type = float2;
};

// ----------------------------------------------------------------- kernels

// work[i][j][k] = (T) Y_lm(x_i, y_j, z_k) * (rho[i][j][k] - shift), with cell
// coordinates x_i = x0 + i (correlator.h:399-401: sequence(0.5 - obs, 1, n)).
template <typename T>
__global__ void k_weight(const double *__restrict__ rho, T *__restrict__ work,
                         int n0, int n1, int n2, int n2p, double x0, double y0,
                         double z0, YlmParams p, double shift) {
  const size_t nrows = (size_t)n0 * n1;
  for (size_t row = blockIdx.x; row < nrows; row += gridDim.x) {
    const int i = (int)(row / n1);
    const int j = (int)(row % n1);
    const double x = x0 + i * 1.0;
    const double y = y0 + j * 1.0;
    const double *src = rho + row * n2;
    T *dst = work + row * n2p;
    for (int k = threadIdx.x; k < n2; k += blockDim.x) {
      const double z = z0 + k * 1.0;
      dst[k] = (T)ylm_eval(p, src[k] - shift, x, y, z);
    }
  }
}

// copy_into_padded_array (array_ops.cc:35-53), with an optional shift and a
// precision cast.
template <typename TI, typename T>
__global__ void k_copy_pad(const TI *__restrict__ rho, T *__restrict__ work,
                           int n0, int n1, int n2, int n2p, double shift) {
  const size_t nrows = (size_t)n0 * n1;
  for (size_t row = blockIdx.x; row < nrows; row += gridDim.x) {
    const TI *src = rho + row * n2;
    T *dst = work + row * n2p;
    for (int k = threadIdx.x; k < n2; k += blockDim.x)
      dst[k] = (T)((double)src[k] - shift);
  }
}

// out[i] *= conj(in[i]) (array_ops.cc:139-163).
template <typename C>
__global__ void k_conj_mul(C *__restrict__ out, const C *__restrict__ in,
                           size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const C a = out[i];
    const C b = in[i];
    C r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.y * b.x - a.x * b.y;
    out[i] = r;
  }
}

// |out[i]|^2, the autocorrelation case of k_conj_mul (imaginary part 0).
template <typename C>
__global__ void k_abs2(C *__restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const C a = out[i];
    C r;
    r.x = a.x * a.x + a.y * a.y;
    r.y = a.y * a.x - a.x * a.y;
    out[i] = r;
  }
}

// k-subgrid accumulation: extract_fft_submatrix_c2r (fft_grid.cc:215-258)
// times make_ylm(ell, m, kx, ky, kz, coeff, 0, &inv_window)
// (correlator.h:309-314, 453-466).  inv_window = 1/(Wx*Wy*Wz)
// (correlator.h:193-204) from per-axis |W|^2 tables computed on the host.
template <typename C>
__global__ void k_ksub(const C *__restrict__ cgrid, double *__restrict__ ksub,
                       int k0, int k1, int k2, int c0, int c1, int c2p,
                       const double *__restrict__ kx,
                       const double *__restrict__ ky,
                       const double *__restrict__ kz,
                       const double *__restrict__ wx,
                       const double *__restrict__ wy,
                       const double *__restrict__ wz, YlmParams p) {
  const size_t n = (size_t)k0 * k1 * k2;
  const int ox = k0 / 2, oy = k1 / 2, oz = k2 / 2;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n;
       c += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(c % k2);
    const int j = (int)((c / k2) % k1);
    const int i = (int)(c / ((size_t)k2 * k1));
    const int ii = (c0 - ox + i) % c0;
    const int jj = (c1 - oy + j) % c1;
    size_t src;
    if (k < oz) {
      const int iin = (c0 - ii) % c0;
      const int jjn = (c1 - jj) % c1;
      src = ((size_t)iin * c1 + jjn) * c2p + (oz - k);
    } else {
      src = ((size_t)ii * c1 + jj) * c2p + (k - oz);
    }
    const double re = (double)cgrid[src].x;
    const double inv_w = 1.0 / (wx[i] * wy[j] * wz[k]);
    const double y = ylm_eval(p, inv_w, kx[i], ky[j], kz[k]);
    ksub[c] += y * re;
  }
}

// r-subgrid accumulation: extract_submatrix (fft_grid.cc:182-210) times
// make_ylm(ell, m, rx, ry, rz, coeff, 0, NULL) (correlator.h:342-349, 477-483).
template <typename T>
__global__ void k_rsub(const T *__restrict__ work, double *__restrict__ rsub,
                       int rs, int n0, int n1, int n2, int n2p,
                       const double *__restrict__ raxis, YlmParams p) {
  const size_t n = (size_t)rs * rs * rs;
  const int o = rs / 2;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n;
       c += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(c % rs);
    const int j = (int)((c / rs) % rs);
    const int i = (int)(c / ((size_t)rs * rs));
    const int ii = (n0 - o + i) % n0;
    const int jj = (n1 - o + j) % n1;
    const int kk = (n2 - o + k) % n2;
    const double v = (double)work[((size_t)ii * n1 + jj) * n2p + kk];
    const double y = ylm_eval(p, 1.0, raxis[i], raxis[j], raxis[k]);
    rsub[c] += y * v;
  }
}

// Bin of every subgrid cell: |r| or |k| (correlator.h:123-136, 172-188)
// through HistogramList::to_bin_index (histogram_list.h:57), exactly.
__global__ void k_cell_bins(const double *__restrict__ ax,
                            const double *__restrict__ ay,
                            const double *__restrict__ az, int n0, int n1,
                            int n2, double binsize, int nbins, int *bins) {
  const size_t n = (size_t)n0 * n1 * n2;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n;
       c += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(c % n2);
    const int j = (int)((c / n2) % n1);
    const int i = (int)(c / ((size_t)n2 * n1));
    bins[c] = bin_of(norm3(ax[i], ay[j], az[k]), 0.0, binsize, nbins);
  }
}

// Converts an FP64 complex grid to FP32 (set_grid2_fft in mixed precision).
// rows of h complex values, written `pitch` elements apart.
__global__ void k_z2c(const double2 *in, float2 *out, size_t n, int h,
                      int pitch) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t row = i / h;
    out[row * pitch + (i - row * h)] = make_float2((float)in[i].x, (float)in[i].y);
  }
}

// ------------------------------------------------------------------ host

// array_ops::sequence (array_ops.cc:7-13).
std::vector<double> sequence(double start, double step, int size) {
  std::vector<double> s(size);
  for (int i = 0; i < size; ++i) s[i] = start + i * step;
  return s;
}

double sinc(double x) { return x == 0 ? 1.0 : sin(x) / x; }

// WindowSquaredNorm::evaluate (window_correct.h:22-44).
double window_sq(int kind, double k, double cell) {
  switch (kind) {
    case FC_NO_CORRECTION:
      return 1.0;
    case FC_TSC_CORRECTION:
      return pow(sinc(k * cell / 2.0), 6);
    case FC_TSC_ALIASED_CORRECTION: {
      double sinsq = sin(k * cell / 2.0);
      sinsq *= sinsq;
      return 1 - sinsq + 2.0 / 15.0 * sinsq * sinsq;
    }
  }
  FC_THROW(FC_ERR_INVALID, "unknown window correction");
}

unsigned rows_grid(size_t nrows) {
  return (unsigned)std::min<size_t>(nrows, (size_t)sm_count() * 64);
}

int row_threads(int n2) {
  if (n2 >= 256) return 256;
  return std::max(32, ((n2 + 31) / 32) * 32);
}

}  // namespace

// Per-kernel-family device time of a correlator's launches (off by
// default).  Events come from a pool; intervals are folded in when read.
struct Profiler {
  bool on = false;
  std::vector<std::string> names;
  std::vector<int> launches;
  std::vector<double> seconds;
  struct Rec {
    int fam;
    cudaEvent_t a, b;
  };
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;

  ~Profiler() {
    for (auto &r : pending) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
  }
  int family(const char *n) {
    for (size_t i = 0; i < names.size(); ++i)
      if (names[i] == n) return (int)i;
    names.push_back(n);
    launches.push_back(0);
    seconds.push_back(0.0);
    return (int)names.size() - 1;
  }
  cudaEvent_t event() {
    if (pool.empty()) {
      cudaEvent_t e;
      FC_CUDA(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  void settle() {
    for (auto &r : pending) {
      cudaEventSynchronize(r.b);
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
        seconds[r.fam] += ms * 1e-3;
        launches[r.fam] += 1;
      }
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    pending.clear();
  }
  void reset() {
    settle();
    std::fill(launches.begin(), launches.end(), 0);
    std::fill(seconds.begin(), seconds.end(), 0.0);
  }
  // Brackets the launches made during its lifetime.
  struct Scope {
    Profiler *p;
    cudaStream_t s;
    int fam;
    cudaEvent_t a;
    Scope(Profiler *p_, cudaStream_t s_, const char *name) : p(p_), s(s_) {
      if (!p->on) return;
      fam = p->family(name);
      a = p->event();
      cudaEventRecord(a, s);
    }
    ~Scope() {
      if (!p->on) return;
      cudaEvent_t b = p->event();
      cudaEventRecord(b, s);
      p->pending.push_back({fam, a, b});
    }
  };
};

struct Geometry {
  int shape[3];
  double cell;
  int rmax_cells, rsize;
  int kshape[3];
  int nrows, nr, nk;
  std::vector<double> raxis, kx, ky, kz, wx, wy, wz;

  Geometry(const int shp[3], double cell_size, int window, double rmax,
           double dr, double kmax, double dk, int maxell) {
    FC_REQUIRE(cell_size > 0, FC_ERR_INVALID, "cell_size must be positive");
    FC_REQUIRE(maxell >= 0 && maxell % 2 == 0 && maxell <= 4, FC_ERR_INVALID,
               "maxell must be 0, 2 or 4");
    FC_REQUIRE(window >= 0 && window <= 2, FC_ERR_INVALID,
               "unknown window correction");
    // HistogramList validation (histogram_list.h:20-24).
    FC_REQUIRE(rmax > 0 && kmax > 0, FC_ERR_INVALID,
               "maxval must be greater than minval.");
    FC_REQUIRE(dr > 0 && dk > 0, FC_ERR_INVALID, "binsize must be positive.");
    for (int i = 0; i < 3; ++i) {
      FC_REQUIRE(shp[i] > 0, FC_ERR_INVALID, "shape must be positive");
      shape[i] = shp[i];
    }
    cell = cell_size;
    nrows = maxell / 2 + 1;
    nr = (int)floor((rmax - 0.0) / dr);
    nk = (int)floor((kmax - 0.0) / dk);
    // setup_r_subgrid (correlator.h:109-140).
    rmax_cells = (int)ceil(rmax / cell);
    rsize = 2 * rmax_cells + 1;
    raxis = sequence(-cell * rmax_cells, cell, rsize);
    // setup_k_subgrid (correlator.h:142-205).
    const double k_nyq = M_PI / cell;
    for (int i = 0; i < 3; ++i) {
      kshape[i] = (int)(2 * ceil(kmax / (2.0 * k_nyq / shape[i])) + 1);
      if (kshape[i] > shape[i]) kshape[i] = 2 * (shape[i] / 2) + 1;
    }
    kx = sequence((-kshape[0] / 2) * 2.0 * k_nyq / shape[0],
                  2.0 * k_nyq / shape[0], kshape[0]);
    ky = sequence((-kshape[1] / 2) * 2.0 * k_nyq / shape[1],
                  2.0 * k_nyq / shape[1], kshape[1]);
    kz = sequence((-kshape[2] / 2) * 2.0 * k_nyq / shape[2],
                  2.0 * k_nyq / shape[2], kshape[2]);
    for (double k : kx) wx.push_back(window_sq(window, k, cell));
    for (double k : ky) wy.push_back(window_sq(window, k, cell));
    for (double k : kz) wz.push_back(window_sq(window, k, cell));
    // The centred extraction indexes (n - rmax_cells + i) mod n, which the
    // reference only defines for rmax_cells <= n (fft_grid.cc:192-200).
    FC_REQUIRE(rmax_cells <= shape[0] && rmax_cells <= shape[1] &&
                   rmax_cells <= shape[2],
               FC_ERR_INVALID, "rmax exceeds the grid extent");
  }

  size_t ncells() const { return (size_t)shape[0] * shape[1] * shape[2]; }
  int n2p() const { return 2 * (shape[2] / 2 + 1); }
  size_t nreal_padded() const { return (size_t)shape[0] * shape[1] * n2p(); }
  size_t ncomplex() const {
    return (size_t)shape[0] * shape[1] * (shape[2] / 2 + 1);
  }
  size_t rcells() const { return (size_t)rsize * rsize * rsize; }
  size_t kcells() const { return (size_t)kshape[0] * kshape[1] * kshape[2]; }
};

struct Correlator {
  int kind;
  int precision;
  Geometry geo;
  double posmin[3] = {0, 0, 0};
  double xyz0[3] = {0, 0, 0};  // survey cell-centre coordinates of cell 0
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;

  DeviceBuffer work, g2, input, rsub, ksub;
  DeviceBuffer d_raxis, d_kaxes, d_kwin;
  DeviceBuffer d_rhist, d_khist, d_zerolag;
  BinIndex rbins, kbins;
  bool have_g2 = false;
  bool have_result = false;
  double shift_value = 0.0;  // mean removed before FP32 transforms

  Profiler prof;
  // Hand-written fused FFT passes for the survey loop (null: cuFFT path).
  std::unique_ptr<FusedSurvey> fused;
  cufftHandle plan_r2c = 0, plan_c2r = 0;
  DeviceBuffer fft_area;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  cudaEvent_t ev_fft0 = nullptr, ev_fft1 = nullptr;
  double last_total = 0.0;
  int n_fft = 0;
  // Survey (ell, m) terms this correlator computes: term i of the loop order
  // (ell ascending, then m ascending) when i % term_world == term_rank.
  int term_rank = 0, term_world = 1;
  bool owns_term(int i) const { return i % term_world == term_rank; }
  // Launch shapes of the grid-stride kernels; results do not depend on them
  // (every cell is computed independently), so the autotuner may change them.
  LaunchShape ls_abs2{256, 8}, ls_ksub{256, 8}, ls_rsub{256, 8};
  // Deferred-histogram mode (batched form): each multipole keeps its own
  // subgrids and the histograms are reduced later, for many correlators at
  // once.
  bool deferred = false;
  std::vector<DeviceBuffer> rsub_l, ksub_l;

  Correlator(int kind_, const int shape[3], double cell, const double pmin[3],
             int window, double rmax, double dr, double kmax, double dk,
             int maxell, int precision_)
      : kind(kind_),
        precision(precision_),
        geo(shape, cell, window, rmax, dr, kmax, dk, maxell) {
    FC_REQUIRE(kind == FC_PERIODIC || kind == FC_SURVEY, FC_ERR_INVALID,
               "unknown correlator kind");
    FC_REQUIRE(precision == FC_FP64 || precision == FC_FP32_MIXED,
               FC_ERR_INVALID, "unknown precision");
    dr_binsize = dr;
    dk_binsize = dk;
    if (kind == FC_SURVEY) {
      FC_REQUIRE(pmin, FC_ERR_INVALID, "survey correlator needs posmin");
      // setup_cell_coords (correlator.h:381-402).
      for (int i = 0; i < 3; ++i) {
        posmin[i] = pmin[i];
        const double observer = -posmin[i] / cell;
        xyz0[i] = 0.5 - observer;
      }
    }
    FC_CUDA(cudaGetDevice(&device));
    try {
      FC_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
      stream = own_stream;
      FC_CUDA(cudaEventCreate(&ev_start));
      FC_CUDA(cudaEventCreate(&ev_stop));
      const char *mode = std::getenv("FFTCORR_B200_FFT");
      const bool want_fused = !(mode && std::string(mode) == "cufft");
      if (kind == FC_SURVEY && want_fused &&
          FusedSurvey::supported(geo.shape, geo.rsize))
        fused.reset(new FusedSurvey(geo.shape, geo.rsize, geo.kshape, fp64()));
      allocate();
      if (!fused) make_plans();
      build_bins();
      // Every (ell, m) weight table now: a correlation (a served job on a
      // resident correlator in particular) then allocates nothing.
      if (fused)
        fused->prepare_tables(2 * (geo.nrows - 1), (double)geo.ncells(),
                              d_raxis.as<double>(), kaxes(),
                              ksub.as<double>() != nullptr, stream);
    } catch (...) {
      // A failed construction leaves no stream, event or plan behind (the
      // buffers free themselves).
      release_handles();
      throw;
    }
  }

  ~Correlator() { release_handles(); }

  void release_handles() {
    if (stream) cudaStreamSynchronize(stream);
    if (plan_r2c) cufftDestroy(plan_r2c);
    if (plan_c2r) cufftDestroy(plan_c2r);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    if (own_stream) cudaStreamDestroy(own_stream);
    plan_r2c = plan_c2r = 0;
    ev_start = ev_stop = nullptr;
    own_stream = stream = nullptr;
  }

  bool fp64() const { return precision == FC_FP64; }
  size_t real_bytes() const { return fp64() ? 8 : 4; }

  void allocate() {
    if (!fused) work.resize(geo.nreal_padded() * real_bytes());
    rsub.resize(geo.rcells() * sizeof(double));
    ksub.resize(geo.kcells() * sizeof(double));
    d_raxis.resize(geo.rsize * sizeof(double));
    FC_CUDA(cudaMemcpy(d_raxis.get(), geo.raxis.data(),
                       geo.rsize * sizeof(double), cudaMemcpyHostToDevice));
    const size_t nk = geo.kshape[0] + geo.kshape[1] + geo.kshape[2];
    std::vector<double> ax, wn;
    ax.insert(ax.end(), geo.kx.begin(), geo.kx.end());
    ax.insert(ax.end(), geo.ky.begin(), geo.ky.end());
    ax.insert(ax.end(), geo.kz.begin(), geo.kz.end());
    wn.insert(wn.end(), geo.wx.begin(), geo.wx.end());
    wn.insert(wn.end(), geo.wy.begin(), geo.wy.end());
    wn.insert(wn.end(), geo.wz.begin(), geo.wz.end());
    d_kaxes.resize(nk * sizeof(double));
    d_kwin.resize(nk * sizeof(double));
    FC_CUDA(cudaMemcpy(d_kaxes.get(), ax.data(), nk * sizeof(double),
                       cudaMemcpyHostToDevice));
    FC_CUDA(cudaMemcpy(d_kwin.get(), wn.data(), nk * sizeof(double),
                       cudaMemcpyHostToDevice));
    d_rhist.resize(std::max(1, geo.nrows * geo.nr) * sizeof(double));
    d_khist.resize(std::max(1, geo.nrows * geo.nk) * sizeof(double));
    d_zerolag.resize(sizeof(double));
    FC_CUDA(cudaMemset(d_rhist.get(), 0, d_rhist.bytes()));
    FC_CUDA(cudaMemset(d_khist.get(), 0, d_khist.bytes()));
    FC_CUDA(cudaMemset(d_zerolag.get(), 0, d_zerolag.bytes()));
  }

  // Creates both plans; on a failure neither is left behind (the
  // constructor that calls this does not run the destructor when it throws).
  void make_plans() {
    try {
      make_plans_unguarded();
    } catch (...) {
      if (plan_r2c) cufftDestroy(plan_r2c);
      if (plan_c2r) cufftDestroy(plan_c2r);
      plan_r2c = plan_c2r = 0;
      throw;
    }
  }

  void make_plans_unguarded() {
    // In-place padded r2c / c2r, FftGrid::plan_fft (fft_grid.cc:69-84).
    int n[3] = {geo.shape[0], geo.shape[1], geo.shape[2]};
    int rembed[3] = {geo.shape[0], geo.shape[1], geo.n2p()};
    int cembed[3] = {geo.shape[0], geo.shape[1], geo.n2p() / 2};
    const long long rdist = (long long)geo.nreal_padded();
    const long long cdist = (long long)geo.ncomplex();
    FC_CUFFT(cufftCreate(&plan_r2c));
    FC_CUFFT(cufftCreate(&plan_c2r));
    FC_CUFFT(cufftSetAutoAllocation(plan_r2c, 0));
    FC_CUFFT(cufftSetAutoAllocation(plan_c2r, 0));
    size_t ws1 = 0, ws2 = 0;
    if (fault_fires(kFaultFftPlan))
      FC_THROW(FC_ERR_CUFFT, "injected cuFFT plan creation failure");
    FC_CUFFT(cufftMakePlanMany(plan_r2c, 3, n, rembed, 1, (int)std::min<long long>(rdist, 1LL << 30),
                               cembed, 1, (int)std::min<long long>(cdist, 1LL << 30),
                               fp64() ? CUFFT_D2Z : CUFFT_R2C, 1, &ws1));
    FC_CUFFT(cufftMakePlanMany(plan_c2r, 3, n, cembed, 1, (int)std::min<long long>(cdist, 1LL << 30),
                               rembed, 1, (int)std::min<long long>(rdist, 1LL << 30),
                               fp64() ? CUFFT_Z2D : CUFFT_C2R, 1, &ws2));
    fft_area.resize(std::max<size_t>(std::max(ws1, ws2), 256));
    FC_CUFFT(cufftSetWorkArea(plan_r2c, fft_area.get()));
    FC_CUFFT(cufftSetWorkArea(plan_c2r, fft_area.get()));
    FC_CUFFT(cufftSetStream(plan_r2c, stream));
    FC_CUFFT(cufftSetStream(plan_c2r, stream));
  }

  void build_bins() {
    const double *kaxes = d_kaxes.as<double>();
    {
      DeviceBuffer b(geo.rcells() * sizeof(int) + 16);
      const double *ra = d_raxis.as<double>();
      k_cell_bins<<<grid_for(geo.rcells(), 256), 256, 0, stream>>>(
          ra, ra, ra, geo.rsize, geo.rsize, geo.rsize, dr_(), geo.nr,
          b.as<int>());
      FC_LAUNCH_CHECK();
      rbins.build(b.as<int>(), geo.rcells(), geo.nr, stream);
    }
    {
      DeviceBuffer b(geo.kcells() * sizeof(int) + 16);
      k_cell_bins<<<grid_for(geo.kcells(), 256), 256, 0, stream>>>(
          kaxes, kaxes + geo.kshape[0], kaxes + geo.kshape[0] + geo.kshape[1],
          geo.kshape[0], geo.kshape[1], geo.kshape[2], dk_(), geo.nk,
          b.as<int>());
      FC_LAUNCH_CHECK();
      kbins.build(b.as<int>(), geo.kcells(), geo.nk, stream);
    }
  }

  double dr_binsize = 0, dk_binsize = 0;
  double dr_() const { return dr_binsize; }
  double dk_() const { return dk_binsize; }

  void set_stream(cudaStream_t s) {
    stream = s ? s : own_stream;
    if (plan_r2c) FC_CUFFT(cufftSetStream(plan_r2c, stream));
    if (plan_c2r) FC_CUFFT(cufftSetStream(plan_c2r, stream));
  }

  KAxes kaxes() const {
    const double *ax = d_kaxes.as<double>();
    const double *wn = d_kwin.as<double>();
    const int a = geo.kshape[0], b = geo.kshape[1];
    return KAxes{ax, ax + a, ax + a + b, wn, wn + a, wn + a + b};
  }

  // Adapter from the fused passes' hooks to the profiler.
  struct ProfHook : PhaseHook {
    Profiler *p;
    cudaStream_t s;
    std::unique_ptr<Profiler::Scope> cur;
    ProfHook(Profiler *p_, cudaStream_t s_) : p(p_), s(s_) {}
    void begin(const char *name) override { cur.reset(new Profiler::Scope(p, s, name)); }
    void end() override { cur.reset(); }
  };

  // ------------------------------------------------------------ kernels

  template <typename T>
  T *work_real() const {
    return work.as<T>();
  }

  void exec_r2c(void *in, void *out) {
    Profiler::Scope ps(&prof, stream, "r2c");
    if (fp64())
      FC_CUFFT(cufftExecD2Z(plan_r2c, (cufftDoubleReal *)in,
                            (cufftDoubleComplex *)out));
    else
      FC_CUFFT(cufftExecR2C(plan_r2c, (cufftReal *)in, (cufftComplex *)out));
    ++n_fft;
  }

  void exec_c2r(void *in, void *out) {
    Profiler::Scope ps(&prof, stream, "c2r");
    if (fp64())
      FC_CUFFT(cufftExecZ2D(plan_c2r, (cufftDoubleComplex *)in,
                            (cufftDoubleReal *)out));
    else
      FC_CUFFT(cufftExecC2R(plan_c2r, (cufftComplex *)in, (cufftReal *)out));
    ++n_fft;
  }

  template <typename T>
  void copy_pad(Density d, double shift) {
    Profiler::Scope ps(&prof, stream, "copy_pad");
    const size_t nrows = (size_t)geo.shape[0] * geo.shape[1];
    if (d.f32)
      k_copy_pad<float, T><<<rows_grid(nrows), row_threads(geo.shape[2]), 0,
                             stream>>>(static_cast<const float *>(d.p), work.as<T>(),
                                       geo.shape[0], geo.shape[1], geo.shape[2],
                                       geo.n2p(), shift);
    else
      k_copy_pad<double, T><<<rows_grid(nrows), row_threads(geo.shape[2]), 0,
                              stream>>>(static_cast<const double *>(d.p),
                                        work.as<T>(), geo.shape[0], geo.shape[1],
                                        geo.shape[2], geo.n2p(), shift);
    FC_LAUNCH_CHECK();
  }

  template <typename T>
  void weight(const double *rho, int ell, int m, double shift) {
    Profiler::Scope ps(&prof, stream, "weight");
    const size_t nrows = (size_t)geo.shape[0] * geo.shape[1];
    k_weight<T><<<rows_grid(nrows), row_threads(geo.shape[2]), 0, stream>>>(
        rho, work.as<T>(), geo.shape[0], geo.shape[1], geo.shape[2], geo.n2p(),
        xyz0[0], xyz0[1], xyz0[2], make_ylm_params(ell, m, 1.0), shift);
    FC_LAUNCH_CHECK();
  }

  template <typename T>
  void conj_mul(bool autocorr) {
    Profiler::Scope ps(&prof, stream, "conj_mul");
    using C = typename Cplx<T>::type;
    const size_t nc = geo.ncomplex();
    // The work grid has padded rows of n2p/2 complex = ncomplex overall.
    if (autocorr) {
      k_abs2<C><<<ls_abs2.grid(nc), ls_abs2.threads, 0, stream>>>(work.as<C>(),
                                                                   nc);
    } else {
      k_conj_mul<C><<<grid_for(nc, 256), 256, 0, stream>>>(work.as<C>(),
                                                           g2.as<C>(), nc);
    }
    FC_LAUNCH_CHECK();
  }

  template <typename T>
  void ksub_acc(int ell, int m, double coeff, double *dst = nullptr) {
    Profiler::Scope ps(&prof, stream, "ksub");
    using C = typename Cplx<T>::type;
    const double *ax = d_kaxes.as<double>();
    const double *wn = d_kwin.as<double>();
    const int a = geo.kshape[0], b = geo.kshape[1];
    k_ksub<C><<<ls_ksub.grid(geo.kcells()), ls_ksub.threads, 0, stream>>>(
        work.as<C>(), dst ? dst : ksub.as<double>(), geo.kshape[0], geo.kshape[1],
        geo.kshape[2], geo.shape[0], geo.shape[1], geo.n2p() / 2, ax, ax + a,
        ax + a + b, wn, wn + a, wn + a + b, make_ylm_params(ell, m, coeff));
    FC_LAUNCH_CHECK();
  }

  template <typename T>
  void rsub_acc(int ell, int m, double coeff, double *dst = nullptr) {
    Profiler::Scope ps(&prof, stream, "rsub");
    k_rsub<T><<<ls_rsub.grid(geo.rcells()), ls_rsub.threads, 0, stream>>>(
        work.as<T>(), dst ? dst : rsub.as<double>(), geo.rsize, geo.shape[0], geo.shape[1],
        geo.shape[2], geo.n2p(), d_raxis.as<double>(),
        make_ylm_params(ell, m, coeff));
    FC_LAUNCH_CHECK();
  }

  void hist_rows(int ell, bool do_r, bool do_k) {
    Profiler::Scope ps(&prof, stream, "hist");
    const int ih = ell / 2;
    if (do_r) rbins.reduce(rsub.as<double>(), d_rhist.as<double>() + ih * geo.nr, stream);
    if (do_k) kbins.reduce(ksub.as<double>(), d_khist.as<double>() + ih * geo.nk, stream);
  }

  void zero_sub(bool r, bool k) {
    if (r) FC_CUDA(cudaMemsetAsync(rsub.get(), 0, geo.rcells() * sizeof(double), stream));
    if (k) FC_CUDA(cudaMemsetAsync(ksub.get(), 0, geo.kcells() * sizeof(double), stream));
  }

  void save_zerolag() {
    const size_t rz = ((size_t)geo.rmax_cells * geo.rsize + geo.rmax_cells) *
                          geo.rsize + geo.rmax_cells;
    FC_CUDA(cudaMemcpyAsync(d_zerolag.get(), rsub.as<double>() + rz,
                            sizeof(double), cudaMemcpyDeviceToDevice, stream));
  }

  // ----------------------------------------------------------- grid2

  template <typename T>
  void set_grid2_dev(Density d) {
    using C = typename Cplx<T>::type;
    if (fused) {
      ProfHook hook(&prof, stream);
      hook.begin("grid2");
      fused->grid2(fused->prepare_input(d.p, d.f32, stream), stream, kaxes());
      hook.end();
      ++n_fft;
      have_g2 = true;
      return;
    }
    g2.resize(geo.ncomplex() * sizeof(C));
    copy_pad<T>(d, shift_for(d));
    exec_r2c(work.get(), g2.get());
    have_g2 = true;
  }

  // The FP64 cells of a density that accept() has passed through.
  static const double *fp64_cells(Density d) {
    FC_REQUIRE(!d.f32, FC_ERR_STATE, "FP32 cells on an FP64 input path");
    return static_cast<const double *>(d.p);
  }

  // FP32 cells go straight into the FP32 fused passes and the periodic
  // copy into the FP32 work grid; every other path reads FP64 cells,
  // widened here into the staging buffer.
  Density accept(Density d) {
    if (!d.f32 || (!fp64() && (fused || kind == FC_PERIODIC))) return d;
    input.resize(geo.ncells() * sizeof(double));
    device_widen(static_cast<const float *>(d.p), input.as<double>(),
                 geo.ncells(), stream);
    return {input.get(), false};
  }

  // Mean of the grid, removed before FP32 transforms of periodic grids.
  double shift_for(Density d) {
    (void)d;
    return 0.0;
  }

  void set_grid2_fft_host(const double *host_complex) {
    const size_t nc = geo.ncomplex();
    if (fused) {
      const int h = fused->g.h, hp = fused->g.hp;
      if (fp64()) {
        FC_CUDA(cudaMemcpy2DAsync(fused->g_data(), hp * sizeof(double2),
                                  host_complex, h * sizeof(double2),
                                  h * sizeof(double2), nc / h,
                                  cudaMemcpyHostToDevice, stream));
      } else {
        DeviceBuffer tmp(nc * sizeof(double2));
        FC_CUDA(cudaMemcpyAsync(tmp.get(), host_complex, nc * sizeof(double2),
                                cudaMemcpyHostToDevice, stream));
        k_z2c<<<grid_for(nc, 256), 256, 0, stream>>>(
            tmp.as<double2>(), static_cast<float2 *>(fused->g_data()), nc, h,
            hp);
        FC_LAUNCH_CHECK();
        FC_CUDA(cudaStreamSynchronize(stream));
      }
      have_g2 = true;
      return;
    }
    if (fp64()) {
      g2.resize(nc * sizeof(double2));
      FC_CUDA(cudaMemcpyAsync(g2.get(), host_complex, nc * sizeof(double2),
                              cudaMemcpyHostToDevice, stream));
    } else {
      DeviceBuffer tmp(nc * sizeof(double2));
      g2.resize(nc * sizeof(float2));
      FC_CUDA(cudaMemcpyAsync(tmp.get(), host_complex, nc * sizeof(double2),
                              cudaMemcpyHostToDevice, stream));
      const int h = (int)(nc / ((size_t)geo.shape[0] * geo.shape[1]));
      k_z2c<<<grid_for(nc, 256), 256, 0, stream>>>(tmp.as<double2>(),
                                                   g2.as<float2>(), nc, h, h);
      FC_LAUNCH_CHECK();
      FC_CUDA(cudaStreamSynchronize(stream));
    }
    have_g2 = true;
  }

  // -------------------------------------------------------- correlate

  // PeriodicCorrelator::correlate_internal (correlator.h:273-357).
  template <typename T>
  void periodic_run(Density d, bool cross) {
    const size_t ncells = geo.ncells();
    copy_pad<T>(d, 0.0);
    exec_r2c(work.get(), work.get());
    conj_mul<T>(!cross);
    const double k_rescale = geo.cell * geo.cell * geo.cell / (double)ncells;
    const int maxell = 2 * (geo.nrows - 1);
    for (int ell = 0; ell <= maxell; ell += 2) {
      zero_sub(false, true);
      const double coeff = sqrt((4.0 * M_PI) * (2 * ell + 1)) * k_rescale;
      ksub_acc<T>(ell, 0, coeff);
      hist_rows(ell, false, true);
    }
    exec_c2r(work.get(), work.get());
    const double r_rescale = (1.0 / ncells / ncells);
    for (int ell = 0; ell <= maxell; ell += 2) {
      zero_sub(true, false);
      const double coeff = sqrt((4.0 * M_PI) * (2 * ell + 1)) * r_rescale;
      rsub_acc<T>(ell, 0, coeff);
      hist_rows(ell, true, false);
      if (ell == 0) save_zerolag();
    }
  }

  // Deferred-histogram mode: one r- and one k-subgrid per multipole.
  void make_deferred() {
    FC_REQUIRE(kind == FC_PERIODIC && !fused, FC_ERR_UNSUPPORTED,
               "deferred histograms are built for the periodic correlator");
    deferred = true;
    rsub_l.resize(geo.nrows);
    ksub_l.resize(geo.nrows);
    for (int r = 0; r < geo.nrows; ++r) {
      rsub_l[r].resize(geo.rcells() * sizeof(double));
      ksub_l[r].resize(geo.kcells() * sizeof(double));
    }
  }

  // PeriodicCorrelator::correlate_internal (correlator.h:273-357) on a
  // density the caller has already written into the padded work grid, with
  // the histograms deferred (hist_work).  Enqueue only: no allocation, no
  // host synchronisation, so it can be captured into a CUDA graph.
  template <typename T>
  void periodic_prepared() {
    const size_t ncells = geo.ncells();
    exec_r2c(work.get(), work.get());
    conj_mul<T>(true);
    const double k_rescale = geo.cell * geo.cell * geo.cell / (double)ncells;
    const int maxell = 2 * (geo.nrows - 1);
    for (int ell = 0; ell <= maxell; ell += 2) {
      double *dst = ksub_l[ell / 2].as<double>();
      FC_CUDA(cudaMemsetAsync(dst, 0, geo.kcells() * sizeof(double), stream));
      const double coeff = sqrt((4.0 * M_PI) * (2 * ell + 1)) * k_rescale;
      ksub_acc<T>(ell, 0, coeff, dst);
    }
    exec_c2r(work.get(), work.get());
    const double r_rescale = (1.0 / ncells / ncells);
    for (int ell = 0; ell <= maxell; ell += 2) {
      double *dst = rsub_l[ell / 2].as<double>();
      FC_CUDA(cudaMemsetAsync(dst, 0, geo.rcells() * sizeof(double), stream));
      const double coeff = sqrt((4.0 * M_PI) * (2 * ell + 1)) * r_rescale;
      rsub_acc<T>(ell, 0, coeff, dst);
    }
    const size_t rz = ((size_t)geo.rmax_cells * geo.rsize + geo.rmax_cells) *
                          geo.rsize + geo.rmax_cells;
    FC_CUDA(cudaMemcpyAsync(d_zerolag.get(), rsub_l[0].as<double>() + rz,
                            sizeof(double), cudaMemcpyDeviceToDevice, stream));
    have_result = true;
  }

  // The histogram reductions of the deferred subgrids as work items.
  void hist_work(std::vector<HistItem> &items, std::vector<FoldItem> &folds) {
    FC_REQUIRE(deferred, FC_ERR_STATE, "correlator is not in deferred mode");
    for (int r = 0; r < geo.nrows; ++r) {
      rbins.append_work(rsub_l[r].as<double>(), d_rhist.as<double>() + r * geo.nr,
                        items, folds);
      kbins.append_work(ksub_l[r].as<double>(), d_khist.as<double>() + r * geo.nk,
                        items, folds);
    }
  }

  // Correlator::correlate_internal (correlator.h:406-497).  The reference
  // first transforms grid1 and then overwrites the result (:412-417); that
  // transform has no effect on any output and is not repeated here.
  // prepared: the fused passes' input already holds rho (set_grid2 of the
  // same grid has just converted it).
  template <typename T>
  void survey_run(Density d, bool prepared = false) {
    const size_t ncells = geo.ncells();
    const int maxell = 2 * (geo.nrows - 1);
    if (fused) {
      const void *in = prepared ? fused->input(d.p, d.f32)
                                : fused->prepare_input(d.p, d.f32, stream);
      ProfHook hook(&prof, stream);
      PhaseHook *ph = prof.on ? &hook : nullptr;
      const KAxes ka = kaxes();
      // This correlator's terms in order.  Consecutive weighted terms
      // (ell > 0) share one z pass where the passes allow it; the second
      // term's z result waits in the fused passes' second buffer.
      std::vector<std::array<int, 2>> owned;
      int term = 0;
      for (int ell = 0; ell <= maxell; ell += 2)
        for (int m = -ell; m <= ell; ++m)
          if (owns_term(term++)) owned.push_back({ell, m});
      size_t next = 0;
      bool second_ready = false;
      for (int ell = 0; ell <= maxell; ell += 2) {
        zero_sub(true, true);
        for (; next < owned.size() && owned[next][0] == ell; ++next) {
          const int m = owned[next][1];
          bool z_done = false;
          if (second_ready) {
            fused->take_second();
            z_done = true;
            second_ready = false;
          } else if (ell > 0 && next + 1 < owned.size() && fused->pairs()) {
            fused->zfwd_pair(in, ell, m, owned[next + 1][0], owned[next + 1][1],
                             xyz0, stream, ph);
            z_done = true;
            second_ready = true;
          }
          // One forward and one (pruned) inverse transform, or the inverse
          // alone for the ell = 0 term of an autocorrelation.
          n_fft += fused->term(in, ell, m, xyz0, (double)ncells,
                               ksub.as<double>(), rsub.as<double>(),
                               d_raxis.as<double>(), ka, stream, ph, prepared,
                               z_done);
        }
        hist_rows(ell, true, true);
        if (ell == 0) save_zerolag();
      }
      return;
    }
    const double *rho = fp64_cells(d);
    int term = 0;
    for (int ell = 0; ell <= maxell; ell += 2) {
      zero_sub(true, true);
      for (int m = -ell; m <= ell; ++m) {
        if (!owns_term(term++)) continue;
        weight<T>(rho, ell, m, 0.0);
        exec_r2c(work.get(), work.get());
        conj_mul<T>(false);
        ksub_acc<T>(ell, m, 4.0 * M_PI);
        exec_c2r(work.get(), work.get());
        rsub_acc<T>(ell, m, 4.0 * M_PI / ncells);
      }
      hist_rows(ell, true, true);
      if (ell == 0) save_zerolag();
    }
  }

  template <typename T>
  void run_typed(Density d, bool cross) {
    if (kind == FC_PERIODIC) {
      FC_REQUIRE(!cross || have_g2, FC_ERR_STATE,
                 "cross_correlate needs set_grid2 or set_grid2_fft first");
      periodic_run<T>(d, cross);
    } else {
      if (!cross) set_grid2_dev<T>(d);
      FC_REQUIRE(have_g2, FC_ERR_STATE,
                 "cross_correlate needs set_grid2 or set_grid2_fft first");
      survey_run<T>(d, !cross);
    }
  }

  // Enqueues one correlation of a device density.
  void enqueue(Density d, bool cross) {
    n_fft = 0;
    FC_CUDA(cudaEventRecord(ev_start, stream));
    d = accept(d);
    if (fp64())
      run_typed<double>(d, cross);
    else
      run_typed<float>(d, cross);
    FC_CUDA(cudaEventRecord(ev_stop, stream));
    have_result = true;
  }

  void synchronize() {
    FC_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.f;
    if (have_result && cudaEventElapsedTime(&ms, ev_start, ev_stop) == cudaSuccess)
      last_total = ms * 1e-3;
  }

  const double *stage_host(const double *host) {
    input.resize(geo.ncells() * sizeof(double));
    FC_CUDA(cudaMemcpyAsync(input.get(), host, geo.ncells() * sizeof(double),
                            cudaMemcpyHostToDevice, stream));
    return input.as<double>();
  }

  void set_grid2_device(Density d) {
    d = accept(d);
    if (fp64())
      set_grid2_dev<double>(d);
    else
      set_grid2_dev<float>(d);
  }

  void results(double *rbins_out, int *rcounts, double *rhist, double *kbins_out,
               int *kcounts, double *khist, double *zerolag) {
    FC_CUDA(cudaStreamSynchronize(stream));
    const int nr = geo.nr, nk = geo.nk, nrows = geo.nrows;
    if (rbins_out)
      for (int i = 0; i < nr; ++i) rbins_out[i] = 0.0 + (i + 0.5) * dr_binsize;
    if (kbins_out)
      for (int i = 0; i < nk; ++i) kbins_out[i] = 0.0 + (i + 0.5) * dk_binsize;
    // A finished correlation added every in-range subgrid cell once per row.
    if (rcounts)
      for (int r = 0; r < nrows; ++r)
        for (int i = 0; i < nr; ++i)
          rcounts[r * nr + i] = have_result ? rbins.counts[i] : 0;
    if (kcounts)
      for (int r = 0; r < nrows; ++r)
        for (int i = 0; i < nk; ++i)
          kcounts[r * nk + i] = have_result ? kbins.counts[i] : 0;
    if (rhist)
      FC_CUDA(cudaMemcpy(rhist, d_rhist.get(), (size_t)nrows * nr * sizeof(double),
                         cudaMemcpyDeviceToHost));
    if (khist)
      FC_CUDA(cudaMemcpy(khist, d_khist.get(), (size_t)nrows * nk * sizeof(double),
                         cudaMemcpyDeviceToHost));
    if (zerolag)
      FC_CUDA(cudaMemcpy(zerolag, d_zerolag.get(), sizeof(double),
                         cudaMemcpyDeviceToHost));
  }
};

Correlator *correlator_new(int kind, const int shape[3], double cell,
                           const double posmin[3], int window, double rmax,
                           double dr, double kmax, double dk, int maxell,
                           int precision) {
  Correlator *c = new Correlator(kind, shape, cell, posmin, window, rmax, dr,
                                 kmax, dk, maxell, precision);
  try {
    FC_CUDA(cudaStreamSynchronize(c->stream));
  } catch (...) {
    delete c;
    throw;
  }
  return c;
}
void correlator_delete(Correlator *c) { delete c; }
void correlator_autocorrelate(Correlator *c, const Grid *g) {
  for (int i = 0; i < 3; ++i)
    FC_REQUIRE(g->shape[i] == c->geo.shape[i], FC_ERR_INVALID,
               "grid shape does not match the correlator");
  stream_after(c->stream, g->stream);
  c->enqueue(density_of(g), false);
  c->synchronize();
}
void correlator_make_deferred(Correlator *c) { c->make_deferred(); }
void *correlator_work(Correlator *c) { return c->work.get(); }
void correlator_set_stream(Correlator *c, cudaStream_t s) { c->set_stream(s); }
void correlator_enqueue_prepared(Correlator *c) {
  if (c->fp64())
    c->periodic_prepared<double>();
  else
    c->periodic_prepared<float>();
}
void correlator_hist_work(Correlator *c, std::vector<HistItem> &items,
                          std::vector<FoldItem> &folds) {
  c->hist_work(items, folds);
}
void correlator_results(Correlator *c, double *rbins, int *rcounts,
                        double *rhist, double *kbins, int *kcounts,
                        double *khist, double *zerolag) {
  c->results(rbins, rcounts, rhist, kbins, kcounts, khist, zerolag);
}
void correlator_dims(const Correlator *c, int *nrows, int *nr, int *nk) {
  if (nrows) *nrows = c->geo.nrows;
  if (nr) *nr = c->geo.nr;
  if (nk) *nk = c->geo.nk;
}
CorrShapes correlator_shapes(Correlator *c) {
  return CorrShapes{&c->ls_abs2, &c->ls_ksub, &c->ls_rsub};
}
void correlator_time_kernels(Correlator *c, int which, cudaStream_t s) {
  c->set_stream(s);
  const int ell = c->geo.nrows > 1 ? 2 : 0;
  double *k = c->deferred ? c->ksub_l[0].as<double>() : c->ksub.as<double>();
  double *r = c->deferred ? c->rsub_l[0].as<double>() : c->rsub.as<double>();
  if (c->fp64()) {
    if (which == 0) c->conj_mul<double>(true);
    if (which == 1) c->ksub_acc<double>(ell, 0, 1.0, k);
    if (which == 2) c->rsub_acc<double>(ell, 0, 1.0, r);
  } else {
    if (which == 0) c->conj_mul<float>(true);
    if (which == 1) c->ksub_acc<float>(ell, 0, 1.0, k);
    if (which == 2) c->rsub_acc<float>(ell, 0, 1.0, r);
  }
}

// Device bytes of a correlator (see Correlator::allocate and make_plans);
// the cuFFT work area is estimated as one complex grid.
size_t correlator_footprint(int kind, const int shape[3], double cell,
                            double rmax, double kmax, int maxell,
                            int precision) {
  Geometry g(shape, cell, FC_NO_CORRECTION, rmax, rmax, kmax, kmax, maxell);
  const size_t rb = precision == FC_FP64 ? 8 : 4;
  const size_t eb = 2 * rb;
  size_t bytes = 0;
  const char *mode = std::getenv("FFTCORR_B200_FFT");
  const bool want_fused = !(mode && std::string(mode) == "cufft");
  if (kind == FC_SURVEY && want_fused && FusedSurvey::supported(g.shape, g.rsize)) {
    const size_t h = (g.shape[2] / 2 + 1 + 15) / 16 * 16;   // row pitch
    bytes += 2 * (size_t)g.shape[0] * g.shape[1] * h * eb;   // W, G
    bytes += (size_t)g.rsize * g.shape[1] * h * eb;          // Wr
    bytes += (size_t)g.rsize * g.rsize * h * eb;             // Wry
    if (precision != FC_FP64) {                              // FP32 density,
      bytes += g.ncells() * 4 + (size_t)g.shape[0] * g.shape[1] * 32;  // row table
      const int m = g.shape[2] / 2;
      if (m >= 64 && m <= 2048 && (m & (m - 1)) == 0)        // paired z pass:
        bytes += (size_t)g.shape[0] * g.shape[1] * (h * eb + 32);  // W2, table
    }
    const int nlm = maxell == 0 ? 1 : maxell == 2 ? 6 : 15;
    bytes += (size_t)nlm * g.kcells() * rb;                  // k weights
    bytes += (size_t)nlm * g.rsize * g.rsize * g.rsize * rb; // r weights
  } else {
    bytes += g.nreal_padded() * rb;                          // work
    if (kind == FC_SURVEY) bytes += g.ncomplex() * eb;       // grid2 FFT
    bytes += g.ncomplex() * eb;                              // cuFFT work area
  }
  bytes += g.rcells() * (8 + 4) + g.kcells() * (8 + 4);    // subgrids + perms
  return bytes + (4 << 20);
}

}  // namespace fc

using namespace fc;

namespace {
Correlator *as_corr(fc_correlator *c) {
  FC_REQUIRE(c, FC_ERR_INVALID, "null correlator handle");
  return reinterpret_cast<Correlator *>(c);
}
const Correlator *as_corr(const fc_correlator *c) {
  FC_REQUIRE(c, FC_ERR_INVALID, "null correlator handle");
  return reinterpret_cast<const Correlator *>(c);
}
}  // namespace

extern "C" {

int fc_corr_create(int kind, const int shape[3], double cell_size,
                   const double posmin[3], int window_correct, double rmax,
                   double dr, double kmax, double dk, int maxell,
                   unsigned fft_flags, int precision, fc_correlator **out) {
  (void)fft_flags;
  return guard([&] {
    FC_REQUIRE(shape && out, FC_ERR_INVALID, "null argument");
    *out = nullptr;
    struct Holder {
      Correlator *c = nullptr;
      ~Holder() { delete c; }
    } h;
    Correlator *c;
    c = new Correlator(kind, shape, cell_size, posmin, window_correct, rmax, dr,
                       kmax, dk, maxell, precision);
    h.c = c;
    FC_CUDA(cudaStreamSynchronize(c->stream));
    h.c = nullptr;
    *out = reinterpret_cast<fc_correlator *>(c);
  });
}

int fc_corr_destroy(fc_correlator *corr) {
  return guard([&] { delete reinterpret_cast<Correlator *>(corr); });
}

int fc_corr_dims(const fc_correlator *corr, int *nrows, int *nr, int *nk,
                 int rshape[3], int kshape[3]) {
  return guard([&] {
    const Correlator *c = as_corr(corr);
    if (nrows) *nrows = c->geo.nrows;
    if (nr) *nr = c->geo.nr;
    if (nk) *nk = c->geo.nk;
    if (rshape)
      for (int i = 0; i < 3; ++i) rshape[i] = c->geo.rsize;
    if (kshape)
      for (int i = 0; i < 3; ++i) kshape[i] = c->geo.kshape[i];
  });
}

int fc_corr_set_grid2(fc_correlator *corr, const double *host_grid) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    FC_REQUIRE(host_grid, FC_ERR_INVALID, "null grid");
    c->set_grid2_device({c->stage_host(host_grid), false});
    FC_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int fc_corr_set_grid2_grid(fc_correlator *corr, const fc_grid *grid2) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    const Grid *g = as_grid(grid2);
    for (int i = 0; i < 3; ++i)
      FC_REQUIRE(g->shape[i] == c->geo.shape[i], FC_ERR_INVALID,
                 "grid shape does not match the correlator");
    stream_after(c->stream, g->stream);
    c->set_grid2_device(density_of(g));
    FC_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int fc_corr_set_grid2_fft(fc_correlator *corr, const double *host_complex) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    FC_REQUIRE(host_complex, FC_ERR_INVALID, "null grid");
    c->set_grid2_fft_host(host_complex);
    FC_CUDA(cudaStreamSynchronize(c->stream));
  });
}

int fc_corr_autocorrelate(fc_correlator *corr, const double *host_grid) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    FC_REQUIRE(host_grid, FC_ERR_INVALID, "null grid");
    c->enqueue({c->stage_host(host_grid), false}, false);
    c->synchronize();
  });
}

int fc_corr_autocorrelate_grid(fc_correlator *corr, const fc_grid *grid) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    const Grid *g = as_grid(grid);
    for (int i = 0; i < 3; ++i)
      FC_REQUIRE(g->shape[i] == c->geo.shape[i], FC_ERR_INVALID,
                 "grid shape does not match the correlator");
    stream_after(c->stream, g->stream);
    c->enqueue(density_of(g), false);
    c->synchronize();
  });
}

int fc_corr_autocorrelate_grid_async(fc_correlator *corr, const fc_grid *grid) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    const Grid *g = as_grid(grid);
    for (int i = 0; i < 3; ++i)
      FC_REQUIRE(g->shape[i] == c->geo.shape[i], FC_ERR_INVALID,
                 "grid shape does not match the correlator");
    stream_after(c->stream, g->stream);
    c->enqueue(density_of(g), false);
  });
}

int fc_corr_synchronize(fc_correlator *corr) {
  return guard([&] { as_corr(corr)->synchronize(); });
}

int fc_corr_cross_correlate(fc_correlator *corr, const double *host_grid1) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    FC_REQUIRE(host_grid1, FC_ERR_INVALID, "null grid");
    FC_REQUIRE(c->have_g2, FC_ERR_STATE,
               "cross_correlate needs set_grid2 or set_grid2_fft first");
    c->enqueue({c->stage_host(host_grid1), false}, true);
    c->synchronize();
  });
}

int fc_corr_cross_correlate_grid(fc_correlator *corr, const fc_grid *grid1) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    const Grid *g = as_grid(grid1);
    FC_REQUIRE(c->have_g2, FC_ERR_STATE,
               "cross_correlate needs set_grid2 or set_grid2_fft first");
    for (int i = 0; i < 3; ++i)
      FC_REQUIRE(g->shape[i] == c->geo.shape[i], FC_ERR_INVALID,
                 "grid shape does not match the correlator");
    stream_after(c->stream, g->stream);
    c->enqueue(density_of(g), true);
    c->synchronize();
  });
}

int fc_corr_results(const fc_correlator *corr, double *rbins, int *rcounts,
                    double *rhist, double *kbins, int *kcounts, double *khist,
                    double *zerolag) {
  return guard([&] {
    Correlator *c = const_cast<Correlator *>(as_corr(corr));
    c->results(rbins, rcounts, rhist, kbins, kcounts, khist, zerolag);
  });
}

int fc_corr_timings_get(const fc_correlator *corr, fc_corr_timings *t) {
  return guard([&] {
    FC_REQUIRE(t, FC_ERR_INVALID, "null argument");
    const Correlator *c = as_corr(corr);
    std::memset(t, 0, sizeof(*t));
    t->total_time = c->last_total;
    t->n_fft = c->n_fft;
  });
}

int fc_corr_footprint(int kind, const int shape[3], double cell_size,
                      double rmax, double kmax, int maxell, int precision,
                      size_t *bytes) {
  return guard([&] {
    FC_REQUIRE(shape && bytes, FC_ERR_INVALID, "null argument");
    *bytes = correlator_footprint(kind, shape, cell_size, rmax, kmax, maxell,
                                  precision);
  });
}

int fc_corr_set_term_shard(fc_correlator *corr, int rank, int world) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    FC_REQUIRE(world >= 1 && rank >= 0 && rank < world, FC_ERR_INVALID,
               "term shard needs 0 <= rank < world");
    FC_REQUIRE(world == 1 || c->kind == FC_SURVEY, FC_ERR_UNSUPPORTED,
               "only the survey correlator has per-(ell, m) transforms to shard");
    FC_CUDA(cudaStreamSynchronize(c->stream));
    c->term_rank = rank;
    c->term_world = world;
  });
}

int fc_corr_set_profiling(fc_correlator *corr, int enable) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    FC_CUDA(cudaStreamSynchronize(c->stream));
    c->prof.reset();
    c->prof.on = enable != 0;
  });
}

int fc_corr_profile(fc_correlator *corr, fc_kernel_time *out, int max,
                    int *n) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    FC_CUDA(cudaStreamSynchronize(c->stream));
    c->prof.settle();
    const int nf = (int)c->prof.names.size();
    if (n) *n = nf;
    for (int i = 0; i < nf && i < max && out; ++i) {
      std::memset(out[i].name, 0, sizeof(out[i].name));
      std::strncpy(out[i].name, c->prof.names[i].c_str(),
                   sizeof(out[i].name) - 1);
      out[i].launches = c->prof.launches[i];
      out[i].seconds = c->prof.seconds[i];
    }
  });
}

int fc_corr_set_stream(fc_correlator *corr, void *cuda_stream) {
  return guard([&] {
    Correlator *c = as_corr(corr);
    FC_CUDA(cudaStreamSynchronize(c->stream));
    c->set_stream(static_cast<cudaStream_t>(cuda_stream));
  });
}

}  // extern "C"
