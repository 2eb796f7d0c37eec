// fc_fused.h -- fused hand-written FFT passes of the survey correlator
// (see fc_fused.cu for the algorithm).
#pragma once

#include <map>
#include <utility>
#include <vector>

#include "fc_common.cuh"
#include "fc_fft.cuh"

namespace fc {

// Geometry shared by the fused kernels (passed by value).
struct FusedGeom {
  int n0, n1, n2;  // grid shape
  int m;           // N2 / 2: complex length of the z transform
  int h;           // N2 / 2 + 1: half-complex z extent
  int hp;          // row pitch of W, G, Wr, Wry: h rounded up to 16, so
                   // every 16-column group starts on a 128-byte line
  int rs, ro;      // r-subgrid edge and its centre offset (rs / 2)
  int ks0, ks1, ks2;  // k-subgrid shape
  FftPlan px, py, pz;
};

// Device pointers of the k axes and the per-axis |W|^2 window tables.
struct KAxes {
  const double *kx, *ky, *kz, *wx, *wy, *wz;
};

// Optional per-pass timing callbacks (the correlator's profiler).
struct PhaseHook {
  virtual void begin(const char *name) = 0;
  virtual void end() = 0;
  virtual ~PhaseHook() {}
};

class FusedSurvey {
 public:
  // True when every transform length factors into 2, 3, 5, 7, N2 is even
  // and the shared-memory tiles fit.
  static bool supported(const int shape[3], int rsize);

  FusedSurvey(const int shape[3], int rsize, const int kshape[3], bool fp64);

  // The grid in the arithmetic of the passes: rho itself when its cells
  // already have the passes' type (f32: FP32 cells, in mixed precision
  // only), else an FP32 copy of FP64 cells.
  const void *prepare_input(const void *rho, bool f32, cudaStream_t s);
  // What prepare_input(rho, f32) last returned -- valid only while that
  // density is unchanged.
  const void *input(const void *rho, bool f32) const {
    return fp64_ || f32 ? rho : rho32.get();
  }
  // G = 3-D DFT of the prepared grid (BaseCorrelator::set_grid2).
  void grid2(const void *rho_in, cudaStream_t s, const KAxes &ka);
  // Builds the r- (and, with with_k, k-) subgrid weight tables of every
  // (ell, m) up to maxell, so that later correlations allocate nothing.
  void prepare_tables(int maxell, double ncells, const double *raxis,
                      const KAxes &ka, bool with_k, cudaStream_t s);
  // One (ell, m) term of Correlator::correlate_internal, accumulated into
  // the FP64 subgrids.
  // Returns the number of full-grid transforms run (1 or 2).
  int term(const void *rho_in, int ell, int m, const double xyz0[3],
            double ncells, double *ksub, double *rsub, const double *raxis,
            const KAxes &ka, cudaStream_t s, PhaseHook *hook,
            bool g_of_input = false, bool z_done = false);
  // Whether two weighted terms can share one z pass (FP32, power-of-two
  // rows).  zfwd_pair runs the z pass of terms a and b (both ell > 0) in
  // one launch: term a's result lands in W, term b's in a second buffer
  // that take_second() swaps into W before term b runs with z_done.
  bool pairs() const;
  // 1 when the last group of B columns holds only the last column (kz =
  // N2/2), which the paired column passes then take for B planes per CTA;
  // with k_extract, only when that column lies outside the k-subgrid.
  template <int B>
  int nyq_group(bool k_extract) const {
    return (g.h - 1) % B == 0 && (!k_extract || g.ks2 / 2 < g.h - 1) ? 1 : 0;
  }
  void zfwd_pair(const void *rho_in, int ell_a, int m_a, int ell_b, int m_b,
                 const double xyz0[3], cudaStream_t s, PhaseHook *hook);
  void take_second() { std::swap(W, W2); }

  // G in the half-complex layout [N0][N1][N2/2+1] with rows g.hp elements
  // apart (FP64 or FP32 complex).
  void *g_data() const { return G.get(); }
  bool fp64() const { return fp64_; }

  FusedGeom g;

 private:
  template <typename V>
  void upload(DeviceBuffer &dst, const std::vector<V> &v);
  size_t smem(int L) const;
  void set_smem_limits();
  template <typename T>
  void zfwd(const void *rho, bool weight, const YlmParams &p,
            const double xyz0[3], cudaStream_t s);
  template <typename T>
  void yfwd(cudaStream_t s);
  template <typename T>
  void xcorr(bool product, double *ksub, const void *ktab, cudaStream_t s);
  template <typename T>
  void xcorr00(double *ksub, const void *ktab, double w00, cudaStream_t s);
  // Weights of the k-subgrid cells for (ell, m), built on first use.
  // (FP64 for the FP64 form, FP32 for the FP32-mixed form)
  const void *k_table(int ell, int m, const KAxes &ka, cudaStream_t s);
  // Y_lm(r) of the r-subgrid cells for (ell, m), built on first use, in
  // the same type as the k weights.
  const void *r_table(int ell, int m, const double *raxis,
                      const YlmParams &pr, cudaStream_t s);
  template <typename T>
  void yinv(cudaStream_t s);
  template <typename T>
  void zinv(double *rsub, const void *rtab, cudaStream_t s);

  bool fp64_;
  DeviceBuffer tabx, taby, tabz;
  DeviceBuffer W, G, Wr, Wry, rho32;
  DeviceBuffer W2, rowtab2;  // the second term of a paired z pass
  std::map<int, DeviceBuffer> ktabs;
  std::map<int, DeviceBuffer> rtabs;
  DeviceBuffer rowtab;  // per-row z-pass weight coefficients (FP32 form)
};

}  // namespace fc
