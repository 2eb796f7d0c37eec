// fc_fused.cu -- the survey correlator's per-(ell, m) work as five fused,
// hand-written FFT passes over HBM (no cuFFT), with the Y_lm weighting, the
// conjugate product, the k-subgrid extraction and the r-subgrid extraction
// folded into them, and the inverse transform pruned to the rows the
// r-subgrid needs.
//
// Per (ell, m), for the half-complex work array W[x][y][kz] (kz < N2/2+1):
//   zfwd   W[x][y][:] = R2C_z( Y_lm(cell) * rho[x][y][:] )   (make_ylm + r2c
//          along z; spherical_harmonics.h:32-179, fft_grid.cc:125-150)
//   yfwd   W = DFT_y(W)
//   xcorr  per (ky, kz) column: F = DFT_x(W); P = F * conj(G)
//          (array_ops.cc:139-163); ksub += Y_lm(k) W(k)^-2 4 pi Re P on the
//          k-subgrid (fft_grid.cc:215-258); Wr[ri][ky][kz] = IDFT_x(P) only
//          at the rs rows x = (N0 - rs/2 + ri) mod N0 of the r-subgrid
//   yinv   Wry[ri][rj][kz] = IDFT_y(Wr) at the rs rows of the r-subgrid
//   zinv   rsub[ri][rj][rk] += Y_lm(r) 4 pi/N * C2R_z(Wry)[rk] (fft_grid.cc:
//          182-210)
// grid2's transform G (correlator.h:53-77) is zfwd (no weighting) + yfwd +
// DFT_x.  Bytes per (ell, m) at 512^3 FP32: ~4 GB instead of ~11 GB for
// separate make_ylm / cuFFT r2c / multiply / extract / cuFFT c2r passes.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "fc_common.cuh"
#include "fc_fft.cuh"
#include "fc_fused.h"
#include "fc_internal.h"

namespace fc {
namespace {

template <typename T>
using C2 = typename Vec2<T>::type;

// Columns (or rows) per CTA: 64-byte segments of complex values.
template <typename T>
struct Tile {
  static constexpr int B = 64 / (2 * sizeof(T));  // 8 for FP32, 4 for FP64
};

// Y_lm * D in the arithmetic of the pass: the reference's FP64 evaluation
// for the FP64 form, the FP32 evaluator (FP64 coordinates and
// normalisation) for the FP32-mixed form.
template <typename T>
__device__ __forceinline__ T weight_value(const YlmParams &p, T D, double x,
                                          double y, double z);
template <>
__device__ __forceinline__ double weight_value<double>(const YlmParams &p,
                                                       double D, double x,
                                                       double y, double z) {
  return ylm_eval(p, D, x, y, z);
}
template <>
__device__ __forceinline__ float weight_value<float>(const YlmParams &p,
                                                     float D, double x,
                                                     double y, double z) {
  return ylm_eval_f32(p, D, x, y, z);
}

// FP32-mixed weighting of one grid row: with (x, y) fixed, Y_lm * r^ell is
// a polynomial in z, so the row's coefficients (normalisation folded in)
// are formed once in FP64 and each cell costs a Horner evaluation and one
// reciprocal:  Y = D * (c0 + c1 z + c2 z^2 + c3 z^3 + c4 z^4) / r^ell.
struct RowPoly {
  float c[5];
  float rxy2;  // x^2 + y^2
  int ell;
  float value0;
};

__device__ __forceinline__ RowPoly row_poly(const YlmParams &p, double x,
                                            double y) {
  RowPoly r;
  r.ell = p.ell;
  r.value0 = (float)p.value0;
  const double x2 = x * x, y2 = y * y, s = x2 + y2, n = p.norm;
  double c[5] = {0, 0, 0, 0, 0};
  if (p.ell == 2) {
    switch (p.m) {
      case 2: c[0] = x2 - y2; break;
      case 1: c[1] = x; break;
      case 0: c[0] = -s; c[2] = 2.0; break;
      case -1: c[1] = y; break;
      default: c[0] = x * y; break;
    }
  } else if (p.ell == 4) {
    switch (p.m) {
      case 4: c[0] = x2 * x2 - 6.0 * x2 * y2 + y2 * y2; break;
      case 3: c[1] = x * (x2 - 3.0 * y2); break;
      case 2: c[0] = y2 * y2 - x2 * x2; c[2] = 6.0 * (x2 - y2); break;
      case 1: c[1] = -x * s; c[3] = 4.0 / 3.0 * x; break;
      case 0: c[0] = 0.375 * s * s; c[2] = -3.0 * s; c[4] = 1.0; break;
      case -1: c[1] = -y * s; c[3] = 4.0 / 3.0 * y; break;
      case -2: c[0] = -2.0 * x * y * s; c[2] = 12.0 * x * y; break;
      case -3: c[1] = 3.0 * x2 * y - y2 * y; break;
      default: c[0] = 4.0 * x * (x2 * y - y2 * y); break;
    }
  }
  for (int i = 0; i < 5; ++i) r.c[i] = (float)(n * c[i]);
  r.rxy2 = (float)s;
  return r;
}

// z is the cell's z coordinate rounded to FP32 (the polynomial is FP32).
// 1/r^2 uses the fast reciprocal-divide intrinsic: r^2 lies between 1e-20
// and 1e10 here, where its error is 2 ulp, far inside the FP32 budget.
__device__ __forceinline__ float row_weight(const RowPoly &r, float D,
                                            float z) {
  if (r.ell == 0) return D * r.value0;
  const float z2 = z * z;
  const float poly =
      (((r.c[4] * z + r.c[3]) * z + r.c[2]) * z + r.c[1]) * z + r.c[0];
  const float ir2 = __fdividef(1.0f, r.rxy2 + z2 + 1e-20f);
  return r.ell == 2 ? D * poly * ir2 : D * poly * (ir2 * ir2);
}

// The row polynomial of an (ell, m) term has only the powers of z of one
// parity up to ell - |m| (spherical_harmonics.h:100-176): its form is one
// of five (POLY, below), chosen once per thread instead of a full Horner
// evaluation per cell.
//   0: c0    1: c1 z    2: c0 + c2 z^2    3: (c1 + c3 z^2) z
//   4: c0 + (c2 + c4 z^2) z^2
__host__ __device__ __forceinline__ int row_poly_form(int ell, int m) {
  const int a = m < 0 ? -m : m;
  if (ell == 2) return a == 2 ? 0 : a == 1 ? 1 : 2;
  return a == 4 ? 0 : a == 3 ? 1 : a == 2 ? 2 : a == 1 ? 3 : 4;
}

template <int POLY, int ELL>
__device__ __forceinline__ float row_weight_form(const RowPoly &r, float D,
                                                 float z) {
  const float z2 = z * z;
  float poly;
  if constexpr (POLY == 0) poly = r.c[0];
  else if constexpr (POLY == 1) poly = r.c[1] * z;
  else if constexpr (POLY == 2) poly = r.c[2] * z2 + r.c[0];
  else if constexpr (POLY == 3) poly = (r.c[3] * z2 + r.c[1]) * z;
  else poly = (r.c[4] * z2 + r.c[2]) * z2 + r.c[0];
  const float ir2 = __fdividef(1.0f, r.rxy2 + z2 + 1e-20f);
  if constexpr (ELL == 2) return D * poly * ir2;
  else return D * poly * (ir2 * ir2);
}

__device__ __forceinline__ RowPoly load_row_poly(const float4 *__restrict__ tab,
                                                 int64_t row,
                                                 const YlmParams &p) {
  const float4 a = __ldg(&tab[2 * row]);
  const float4 b = __ldg(&tab[2 * row + 1]);
  RowPoly r;
  r.c[0] = a.x;
  r.c[1] = a.y;
  r.c[2] = a.z;
  r.c[3] = a.w;
  r.c[4] = b.x;
  r.rxy2 = b.y;
  r.ell = p.ell;
  r.value0 = (float)p.value0;
  return r;
}

// ------------------------------------------------------------------ zfwd
// B rows of N2 reals per CTA: (optionally Y_lm-weighted) packed as
// z_j = x_2j + i x_2j+1, length-M complex DFT, then the real-to-complex
// split X_k = E_k + e^{-2 pi i k/N2} O_k for k <= M.
template <typename T, bool WEIGHT>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 ? 3 : 2))
    k_zfwd(const T *__restrict__ rho, C2<T> *__restrict__ W, FusedGeom g,
           YlmParams p, double x0, double y0, double z0,
           const C2<T> *__restrict__ tabz) {
  using C = C2<T>;
  constexpr int B = Tile<T>::B;
  constexpr int BP = B + 1;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int M = g.m;
  C *buf2 = buf + M * BP;
  const int64_t nrows = (int64_t)g.n0 * g.n1;
  const int64_t row0 = (int64_t)blockIdx.x * B;
  for (int idx = threadIdx.x; idx < M * B; idx += blockDim.x) {
    const int b = idx / M;
    const int j = idx - b * M;
    const int64_t row = row0 + b;
    C z;
    z.x = 0;
    z.y = 0;
    if (row < nrows) {
      const typename Vec2<T>::type v =
          reinterpret_cast<const typename Vec2<T>::type *>(rho + row * g.n2)[j];
      z = v;
      if (WEIGHT) {
        const int x = (int)(row / g.n1);
        const int y = (int)(row - (int64_t)x * g.n1);
        const double cx = x0 + x * 1.0;
        const double cy = y0 + y * 1.0;
        z.x = weight_value<T>(p, v.x, cx, cy, z0 + (2 * j) * 1.0);
        z.y = weight_value<T>(p, v.y, cx, cy, z0 + (2 * j + 1) * 1.0);
      }
    }
    buf[j * BP + b] = z;
  }
  __syncthreads();
  buf = fft_columns<B>(buf, buf2, g.pz, tabz, -1);
  const int H = M + 1;
  for (int idx = threadIdx.x; idx < H * B; idx += blockDim.x) {
    const int b = idx / H;
    const int k = idx - b * H;
    const int64_t row = row0 + b;
    if (row >= nrows) continue;
    const C a = buf[(k == M ? 0 : k) * BP + b];
    const C c = cconj(buf[(k == 0 ? 0 : M - k) * BP + b]);
    C e, d, o;
    e.x = (T)0.5 * (a.x + c.x);
    e.y = (T)0.5 * (a.y + c.y);
    d = csub(a, c);
    o.x = (T)0.5 * d.y;  // -i (a - c) / 2
    o.y = (T)-0.5 * d.x;
    W[row * g.hp + k] = cadd(e, cmul(__ldg(&tabz[k]), o));
  }
}

// Loads a B-column tile of a strided axis into shared memory.
// Loads are issued in groups of 8 before any shared-memory store so each
// thread keeps eight global reads in flight.
template <int B, typename C>
__device__ __forceinline__ void load_columns(C *buf, const C *__restrict__ src,
                                             int64_t base, int64_t stride,
                                             int L, int kz0, int h) {
  constexpr int BP = B + 1;
  const int n = L * B;
  for (int idx0 = threadIdx.x; idx0 < n; idx0 += 8 * blockDim.x) {
    C v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = idx0 + u * blockDim.x;
      const int i = idx / B;
      const int b = idx - i * B;
      v[u].x = 0;
      v[u].y = 0;
      if (idx < n && kz0 + b < h) v[u] = src[base + i * stride + kz0 + b];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = idx0 + u * blockDim.x;
      if (idx < n) {
        const int i = idx / B;
        buf[i * BP + (idx - i * B)] = v[u];
      }
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------ yfwd
template <typename T>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 ? 3 : 2))
    k_yfwd(C2<T> *__restrict__ W, FusedGeom g, const C2<T> *__restrict__ taby) {
  using C = C2<T>;
  constexpr int B = Tile<T>::B;
  constexpr int BP = B + 1;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int kz0 = blockIdx.x * B;
  const int x = blockIdx.y;
  const int64_t base = (int64_t)x * g.n1 * g.hp;
  load_columns<B>(buf, W, base, g.hp, g.n1, kz0, g.h);
  buf = fft_columns<B>(buf, buf + g.n1 * BP, g.py, taby, -1);
  for (int idx = threadIdx.x; idx < g.n1 * B; idx += blockDim.x) {
    const int i = idx / B;
    const int b = idx - i * B;
    if (kz0 + b < g.h) W[base + (int64_t)i * g.hp + kz0 + b] = buf[i * BP + b];
  }
}

// ----------------------------------------------------------------- xcorr
// MODE 0: G = DFT_x(W) (grid2's transform).  MODE 1: the fused product,
// k-subgrid extraction, inverse and pruning described at the top.
template <typename T, int MODE>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 ? 3 : 2))
    k_xcorr(const C2<T> *__restrict__ W, const C2<T> *__restrict__ G,
            C2<T> *__restrict__ out, double *__restrict__ ksub, FusedGeom g,
            const C2<T> *__restrict__ tabx, const T *__restrict__ ktab) {
  using C = C2<T>;
  constexpr int B = Tile<T>::B;
  constexpr int BP = B + 1;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int kz0 = blockIdx.x * B;
  const int yy = blockIdx.y;
  const int64_t stride = (int64_t)g.n1 * g.hp;
  const int64_t base = (int64_t)yy * g.hp;
  C *other = buf + g.n0 * BP;
  load_columns<B>(buf, W, base, stride, g.n0, kz0, g.h);
  {
    C *res = fft_columns<B>(buf, other, g.px, tabx, -1);
    other = res == buf ? other : buf;
    buf = res;
  }
  if constexpr (MODE == 0) {
    for (int idx = threadIdx.x; idx < g.n0 * B; idx += blockDim.x) {
      const int i = idx / B;
      const int b = idx - i * B;
      if (kz0 + b < g.h) out[base + i * stride + kz0 + b] = buf[i * BP + b];
    }
  } else {
    // P = F * conj(G).
    for (int idx = threadIdx.x; idx < g.n0 * B; idx += blockDim.x) {
      const int i = idx / B;
      const int b = idx - i * B;
      if (kz0 + b < g.h)
        buf[i * BP + b] = cmulc(buf[i * BP + b], G[base + i * stride + kz0 + b]);
    }
    __syncthreads();
    // k-subgrid: this CTA owns the sources with ky index yy and kz in its
    // block.  Direct targets k = kz + oz read P[(i - ox) mod N0][yy][kz];
    // reflected targets k = oz - kz (kz >= 1) read P[(ox - i) mod N0][yy][kz]
    // for j with (oy - j) mod N1 == yy.  Every ksub cell has exactly one
    // source element, so these read-modify-writes never collide.
    if (ksub != nullptr) {
      const int ox = g.ks0 / 2, oy = g.ks1 / 2, oz = g.ks2 / 2;
      if (kz0 <= oz) {
        for (int refl = 0; refl < 2; ++refl) {
          int j = refl == 0 ? (yy + oy) % g.n1 : ((oy - yy) % g.n1 + g.n1) % g.n1;
          for (; j < g.ks1; j += g.n1) {
            for (int idx = threadIdx.x; idx < g.ks0 * B; idx += blockDim.x) {
              const int i = idx / B;
              const int b = idx - i * B;
              const int kzi = kz0 + b;
              if (kzi >= g.h || kzi > oz || (refl == 1 && kzi == 0)) continue;
              const int k = refl == 0 ? kzi + oz : oz - kzi;
              const int x = refl == 0 ? ((i - ox) % g.n0 + g.n0) % g.n0
                                      : ((ox - i) % g.n0 + g.n0) % g.n0;
              const double re = (double)buf[x * BP + b].x;
              const size_t cell = ((size_t)i * g.ks1 + j) * g.ks2 + k;
              ksub[cell] += (double)ktab[cell] * re;
            }
          }
        }
      }
      __syncthreads();
    }
    buf = fft_columns<B>(buf, other, g.px, tabx, +1);
    const int64_t obase = (int64_t)yy * g.hp;
    const int64_t ostride = (int64_t)g.n1 * g.hp;
    for (int idx = threadIdx.x; idx < g.rs * B; idx += blockDim.x) {
      const int ri = idx / B;
      const int b = idx - ri * B;
      if (kz0 + b >= g.h) continue;
      const int x = ((ri - g.ro) % g.n0 + g.n0) % g.n0;
      out[obase + ri * ostride + kz0 + b] = buf[x * BP + b];
    }
  }
}

// ------------------------------------------------------------------ yinv
template <typename T>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 ? 3 : 2))
    k_yinv(const C2<T> *__restrict__ Wr, C2<T> *__restrict__ Wry, FusedGeom g,
           const C2<T> *__restrict__ taby) {
  using C = C2<T>;
  constexpr int B = Tile<T>::B;
  constexpr int BP = B + 1;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int kz0 = blockIdx.x * B;
  const int ri = blockIdx.y;
  const int64_t base = (int64_t)ri * g.n1 * g.hp;
  load_columns<B>(buf, Wr, base, g.hp, g.n1, kz0, g.h);
  buf = fft_columns<B>(buf, buf + g.n1 * BP, g.py, taby, +1);
  const int64_t obase = (int64_t)ri * g.rs * g.hp;
  for (int idx = threadIdx.x; idx < g.rs * B; idx += blockDim.x) {
    const int rj = idx / B;
    const int b = idx - rj * B;
    if (kz0 + b >= g.h) continue;
    const int y = ((rj - g.ro) % g.n1 + g.n1) % g.n1;
    Wry[obase + (int64_t)rj * g.hp + kz0 + b] = buf[y * BP + b];
  }
}

// ----------------------------------------------------------------- zinv
// B rows (ri, rj) per CTA: complex-to-real inverse along z (unnormalised,
// the imaginary parts of the DC and Nyquist terms ignored), then
// rsub[ri][rj][rk] += Y_lm(r) * value at z = (N2 - rs/2 + rk) mod N2.
template <typename T>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 ? 3 : 2))
    k_zinv_rsub(const C2<T> *__restrict__ Wry, double *__restrict__ rsub,
                FusedGeom g, const C2<T> *__restrict__ tabz,
                const T *__restrict__ rtab) {
  using C = C2<T>;
  constexpr int B = Tile<T>::B;
  constexpr int BP = B + 1;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int M = g.m;
  const int nrows = g.rs * g.rs;
  const int row0 = blockIdx.x * B;
  C *buf2 = buf + M * BP;
  for (int idx = threadIdx.x; idx < M * B; idx += blockDim.x) {
    const int b = idx / M;
    const int k = idx - b * M;
    const int row = row0 + b;
    C z;
    z.x = 0;
    z.y = 0;
    if (row < nrows) {
      const C *X = Wry + (int64_t)row * g.hp;
      C a = X[k];
      C c = cconj(X[M - k]);
      if (k == 0) {
        a.y = 0;
        c.y = 0;  // X[M] is the Nyquist term
      }
      const C e = cadd(a, c);
      const C o = cmul(csub(a, c), cconj(__ldg(&tabz[k])));  // e^{+2 pi i k/N2}
      z.x = e.x - o.y;
      z.y = e.y + o.x;
    }
    buf[k * BP + b] = z;
  }
  __syncthreads();
  buf = fft_columns<B>(buf, buf2, g.pz, tabz, +1);
  for (int idx = threadIdx.x; idx < g.rs * B; idx += blockDim.x) {
    const int b = idx / g.rs;
    const int rk = idx - b * g.rs;
    const int row = row0 + b;
    if (row >= nrows) continue;
    const int z = ((rk - g.ro) % g.n2 + g.n2) % g.n2;
    const C zz = buf[(z >> 1) * BP + b];
    const double v = (double)((z & 1) ? zz.y : zz.x);
    const size_t cell = (size_t)row * g.rs + rk;
    rsub[cell] += (double)rtab[cell] * v;
  }
}

// --------------------------------------------------------------------------
// Power-of-two lengths: the same passes with the register-resident engine
// (reg_fft in fc_fft.cuh).  B2 columns per CTA keep the CTA at <= 1024
// threads (TPC = L/8 threads per column).
template <typename T, int L>
struct P2 {
  static constexpr int B = (Tile<T>::B < 8192 / L) ? Tile<T>::B : 8192 / L;
  static constexpr int TPC = L / 8;
  static constexpr int THREADS = TPC * B;
  // Exchange rows of B elements: a 128-byte shared-memory line holds R of
  // them.  Row i is stored at row i ^ ((i >> 3) & (R - 1)), which spreads
  // the rows a warp touches in every Stockham write and read evenly over
  // the line's R parts (bank-conflict free), with no padding.
  static constexpr int RB = B * (int)sizeof(C2<T>);
  static constexpr int R = RB >= 128 ? 1 : 128 / RB;
  __device__ static __forceinline__ int row(int i) {
    return i ^ ((i >> 3) & (R - 1));
  }
  // Element index of row t + TPC u, column b: when TPC / 8 is a multiple
  // of R the swizzle only depends on t, so it is a per-thread base plus u
  // times a constant.
  static constexpr bool kFastRead = (TPC / 8) % R == 0;
  __device__ static __forceinline__ int rd_base(int t, int b) {
    return kFastRead ? row(t) * B + b : 0;
  }
  __device__ static __forceinline__ int rd(int base, int t, int b, int u) {
    return kFastRead ? base + u * TPC * B : row(t + TPC * u) * B + b;
  }
};

template <typename T, int L>
__global__ void __launch_bounds__(P2<T, L>::THREADS)
    k_yfwd_p2(C2<T> *__restrict__ W, FusedGeom g,
              const C2<T> *__restrict__ taby) {
  using C = C2<T>;
  using Q = P2<T, L>;
  extern __shared__ unsigned char smem_raw[];
  C *ex = reinterpret_cast<C *>(smem_raw);
  const int t = threadIdx.x / Q::B;
  const int b = threadIdx.x - t * Q::B;
  const int kz0 = blockIdx.x * Q::B;
  const bool valid = kz0 + b < g.h;
  const int64_t base = (int64_t)blockIdx.y * L * g.hp + kz0 + b;
  C v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    v[u].x = 0;
    v[u].y = 0;
    if (valid) v[u] = W[base + (int64_t)(t + Q::TPC * u) * g.hp];
  }
  const int rb = Q::rd_base(t, b);
  reg_fft<L>(v, t, [&](int i) { return &ex[Q::row(i) * Q::B + b]; },
             [&](int u) { return &ex[Q::rd(rb, t, b, u)]; }, taby, -1);
  if (valid) {
#pragma unroll
    for (int u = 0; u < 8; ++u) W[base + (int64_t)(t + Q::TPC * u) * g.hp] = v[u];
  }
}

template <typename T, int L>
__global__ void __launch_bounds__(P2<T, L>::THREADS)
    k_yinv_p2(const C2<T> *__restrict__ Wr, C2<T> *__restrict__ Wry,
              FusedGeom g, const C2<T> *__restrict__ taby) {
  using C = C2<T>;
  using Q = P2<T, L>;
  extern __shared__ unsigned char smem_raw[];
  C *ex = reinterpret_cast<C *>(smem_raw);
  const int t = threadIdx.x / Q::B;
  const int b = threadIdx.x - t * Q::B;
  const int kz0 = blockIdx.x * Q::B;
  const int ri = blockIdx.y;
  const bool valid = kz0 + b < g.h;
  const int64_t base = (int64_t)ri * L * g.hp + kz0 + b;
  C v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    v[u].x = 0;
    v[u].y = 0;
    if (valid) v[u] = Wr[base + (int64_t)(t + Q::TPC * u) * g.hp];
  }
  const int rb = Q::rd_base(t, b);
  reg_fft<L>(v, t, [&](int i) { return &ex[Q::row(i) * Q::B + b]; },
             [&](int u) { return &ex[Q::rd(rb, t, b, u)]; }, taby, +1);
  if (!valid) return;
  const int64_t obase = (int64_t)ri * g.rs * g.hp + kz0 + b;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int y = t + Q::TPC * u;
    for (int rj = (y + g.ro) & (L - 1); rj < g.rs; rj += L)
      Wry[obase + (int64_t)rj * g.hp] = v[u];
  }
}

template <typename T, int L, int MODE>
__global__ void __launch_bounds__(P2<T, L>::THREADS)
    k_xcorr_p2(const C2<T> *__restrict__ W, const C2<T> *__restrict__ G,
               C2<T> *__restrict__ out, double *__restrict__ ksub, FusedGeom g,
               const C2<T> *__restrict__ tabx, const T *__restrict__ ktab,
               T w00) {
  using C = C2<T>;
  using Q = P2<T, L>;
  extern __shared__ unsigned char smem_raw[];
  C *ex = reinterpret_cast<C *>(smem_raw);
  const int t = threadIdx.x / Q::B;
  const int b = threadIdx.x - t * Q::B;
  const int kz0 = blockIdx.x * Q::B;
  const int yy = blockIdx.y;
  const int kzi = kz0 + b;
  const bool valid = kzi < g.h;
  const int64_t stride = (int64_t)g.n1 * g.hp;
  const int64_t base = (int64_t)yy * g.hp + kzi;
  auto exf = [&](int i) { return &ex[Q::row(i) * Q::B + b]; };
  C v[8];
  // In product mode the G column is loaded together with the W column, so
  // both streams are in flight during the forward transform.
  C gv[MODE == 1 ? 8 : 1];
  if constexpr (MODE == 2) {
    // ell = 0 of an autocorrelation: the weighted field is w00 * rho, whose
    // transform is w00 * G, so the product is w00 |G|^2 and neither W nor a
    // forward transform is needed.
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      C gg;
      gg.x = 0;
      gg.y = 0;
      if (valid) gg = G[base + (t + Q::TPC * u) * stride];
      v[u].x = w00 * (gg.x * gg.x + gg.y * gg.y);
      v[u].y = 0;
    }
  } else {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      v[u].x = 0;
      v[u].y = 0;
      if (valid) v[u] = W[base + (t + Q::TPC * u) * stride];
    }
  }
  if constexpr (MODE == 1) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      gv[u].x = 0;
      gv[u].y = 0;
      if (valid) gv[u] = G[base + (t + Q::TPC * u) * stride];
    }
  }
  const int rb = Q::rd_base(t, b);
  auto exr = [&](int u) { return &ex[Q::rd(rb, t, b, u)]; };
  if constexpr (MODE != 2) reg_fft<L>(v, t, exf, exr, tabx, -1);
  if constexpr (MODE == 0) {
    if (valid) {
#pragma unroll
      for (int u = 0; u < 8; ++u) out[base + (t + Q::TPC * u) * stride] = v[u];
    }
  } else {
    if constexpr (MODE == 1) {
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = cmulc(v[u], gv[u]);
    }
    // k-subgrid extraction (see k_xcorr): needs P at arbitrary rows.  Only
    // CTAs whose y feeds a k-subgrid row (for either sign of ky) and whose
    // kz range reaches it stage P in shared memory.
    const int ox = g.ks0 / 2, oy = g.ks1 / 2, oz = g.ks2 / 2;
    const int jr0 = (yy + oy) % g.n1;
    const int jr1 = ((oy - yy) % g.n1 + g.n1) % g.n1;
    if (ksub != nullptr && kz0 <= oz && (jr0 < g.ks1 || jr1 < g.ks1)) {
#pragma unroll
      for (int u = 0; u < 8; ++u) *exf(t + Q::TPC * u) = v[u];
      __syncthreads();
      if (valid && kzi <= oz) {
        if (g.ks0 <= 3 * Q::TPC && g.ks1 <= g.n1) {
          // At most three x rows per thread and one row j per reflection:
          // each reflection's loads are issued together.
#pragma unroll
          for (int refl = 0; refl < 2; ++refl) {
            const int j = refl == 0 ? jr0 : jr1;
            if (j >= g.ks1 || (refl == 1 && kzi == 0)) continue;
            const int k = refl == 0 ? kzi + oz : oz - kzi;
            size_t cell[3];
            double acc[3], w[3], re[3];
#pragma unroll
            for (int s = 0; s < 3; ++s) {
              const int i = t + s * Q::TPC;
              cell[s] = ((size_t)i * g.ks1 + j) * g.ks2 + k;
              if (i < g.ks0) {
                const int x = refl == 0 ? (i - ox) & (L - 1)
                                        : (ox - i) & (L - 1);
                re[s] = (double)exf(x)->x;
                w[s] = (double)ktab[cell[s]];
                acc[s] = ksub[cell[s]];
              }
            }
#pragma unroll
            for (int s = 0; s < 3; ++s)
              if (t + s * Q::TPC < g.ks0) ksub[cell[s]] = acc[s] + w[s] * re[s];
          }
        } else {
          for (int refl = 0; refl < 2; ++refl) {
            if (refl == 1 && kzi == 0) continue;
            const int k = refl == 0 ? kzi + oz : oz - kzi;
            for (int j = refl == 0 ? jr0 : jr1; j < g.ks1; j += g.n1) {
              for (int i = t; i < g.ks0; i += Q::TPC) {
                const int x = refl == 0 ? (i - ox) & (L - 1)
                                        : (ox - i) & (L - 1);
                const double re = (double)exf(x)->x;
                const size_t cell = ((size_t)i * g.ks1 + j) * g.ks2 + k;
                ksub[cell] += (double)ktab[cell] * re;
              }
            }
          }
        }
      }
      __syncthreads();
    }
    reg_fft<L>(v, t, exf, exr, tabx, +1);
    if (valid) {
      const int64_t obase = (int64_t)yy * g.hp + kzi;
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int x = t + Q::TPC * u;
        for (int ri = (x + g.ro) & (L - 1); ri < g.rs; ri += L)
          out[obase + ri * stride] = v[u];
      }
    }
  }
}

// Rows of the z transform: thread t of row b holds z[t + TPC u].
template <typename T, int L, bool WEIGHT>
__global__ void __launch_bounds__(P2<T, L>::THREADS)
    k_zfwd_p2(const T *__restrict__ rho, C2<T> *__restrict__ W, FusedGeom g,
              YlmParams p, double x0, double y0, double z0,
              const C2<T> *__restrict__ tabz) {
  using C = C2<T>;
  using Q = P2<T, L>;
  // Row pitch in shared memory, with one pad slot every 8 elements so the
  // strided Stockham writes spread over the banks.
  constexpr int RP = L + L / 8 + 1;
  extern __shared__ unsigned char smem_raw[];
  C *ex = reinterpret_cast<C *>(smem_raw);
  const int b = threadIdx.x / Q::TPC;
  const int t = threadIdx.x - b * Q::TPC;
  const int64_t nrows = (int64_t)g.n0 * g.n1;
  const int64_t row = (int64_t)blockIdx.x * Q::B + b;
  const bool valid = row < nrows;
  C v[8];
  int x = 0, y = 0;
  if (valid) {
    x = (int)(row / g.n1);
    y = (int)(row - (int64_t)x * g.n1);
  }
  const double cx = x0 + x * 1.0;
  const double cy = y0 + y * 1.0;
  const C *src = reinterpret_cast<const C *>(rho + row * g.n2);
  RowPoly rp;
  // z of this thread's first element in FP64; the elements u step by the
  // exact integer 2 TPC, added in FP32.
  float zt = 0.f;
  if constexpr (WEIGHT && sizeof(T) == 4) {
    rp = row_poly(p, cx, cy);
    zt = (float)(z0 + (2 * t) * 1.0);
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    v[u].x = 0;
    v[u].y = 0;
    if (valid) {
      const int jj = t + Q::TPC * u;
      const C pr = src[jj];
      v[u] = pr;
      if constexpr (WEIGHT && sizeof(T) == 4) {
        const float zu = zt + (float)(2 * Q::TPC * u);
        v[u].x = row_weight(rp, pr.x, zu);
        v[u].y = row_weight(rp, pr.y, zu + 1.0f);
      } else if constexpr (WEIGHT) {
        v[u].x = weight_value<T>(p, pr.x, cx, cy, z0 + (2 * jj) * 1.0);
        v[u].y = weight_value<T>(p, pr.y, cx, cy, z0 + (2 * jj + 1) * 1.0);
      }
    }
  }
  auto exf = [&](int i) { return &ex[b * RP + i + (i >> 3)]; };
  reg_fft<L>(v, t, exf, tabz, -1, 2);
  // Real-to-complex split needs Z_k and Z_{M-k}.
#pragma unroll
  for (int u = 0; u < 8; ++u) *exf(t + Q::TPC * u) = v[u];
  __syncthreads();
  if (!valid) return;
  C *dst = W + row * g.hp;
  for (int k = t; k <= L; k += Q::TPC) {
    const C a = *exf(k == L ? 0 : k);
    const C c = cconj(*exf(k == 0 ? 0 : L - k));
    C e, d, o;
    e.x = (T)0.5 * (a.x + c.x);
    e.y = (T)0.5 * (a.y + c.y);
    d = csub(a, c);
    o.x = (T)0.5 * d.y;
    o.y = (T)-0.5 * d.x;
    dst[k] = cadd(e, cmul(__ldg(&tabz[k]), o));
  }
}

template <typename T, int L>
__global__ void __launch_bounds__(P2<T, L>::THREADS)
    k_zinv_p2(const C2<T> *__restrict__ Wry, double *__restrict__ rsub,
              FusedGeom g, const C2<T> *__restrict__ tabz,
              const T *__restrict__ rtab) {
  using C = C2<T>;
  using Q = P2<T, L>;
  constexpr int RP = L + L / 8 + 1;
  extern __shared__ unsigned char smem_raw[];
  C *ex = reinterpret_cast<C *>(smem_raw);
  const int b = threadIdx.x / Q::TPC;
  const int t = threadIdx.x - b * Q::TPC;
  const int nrows = g.rs * g.rs;
  const int row = blockIdx.x * Q::B + b;
  const bool valid = row < nrows;
  C v[8];
  const C *X = Wry + (int64_t)(valid ? row : 0) * g.hp;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int k = t + Q::TPC * u;
    v[u].x = 0;
    v[u].y = 0;
    if (valid) {
      C a = X[k];
      C c = cconj(X[L - k]);
      if (k == 0) {
        a.y = 0;
        c.y = 0;
      }
      const C e = cadd(a, c);
      const C o = cmul(csub(a, c), cconj(__ldg(&tabz[k])));
      v[u].x = e.x - o.y;
      v[u].y = e.y + o.x;
    }
  }
  auto exf = [&](int i) { return &ex[b * RP + i + (i >> 3)]; };
  reg_fft<L>(v, t, exf, tabz, +1, 2);
  if (!valid) return;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int jj = t + Q::TPC * u;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int z = 2 * jj + h;
      const double val = (double)(h ? v[u].y : v[u].x);
      for (int rk = (z + g.ro) % g.n2; rk < g.rs; rk += g.n2) {
        const size_t cell = (size_t)row * g.rs + rk;
        rsub[cell] += (double)rtab[cell] * val;
      }
    }
  }
}

// ------------------------------------------------- FP32 two-per-thread
// FP32 y and z passes with two independent transforms per thread: the same
// B columns (or rows) per CTA as the kernels above with half the threads.
// The two transforms share every twiddle load and index computation and the
// shared-memory exchanges move 16 bytes per access.  The y passes carry the
// pair as CPair (packed two-lane instructions), the z pass as CPairS
// (one-lane instructions), whichever measured faster for the pass.
// Thread (t, p) holds columns p and p + PB of the CTA's B, so each global
// access of a warp stays contiguous per row.  (The FP32 x passes pair
// adjacent columns like the y passes, below.)
template <int L>
struct PP {
  static constexpr int B = P2<float, L>::B;
  static constexpr int PB = B / 2;
  static constexpr int TPC = L / 8;
  static constexpr int THREADS = TPC * PB;
  static constexpr int RB = PB * (int)sizeof(CPair);
  static constexpr int R = RB >= 128 ? 1 : 128 / RB;
  __device__ static __forceinline__ int row(int i) {
    return i ^ ((i >> 3) & (R - 1));
  }
  static constexpr bool kFastRead = (TPC / 8) % R == 0;
  __device__ static __forceinline__ int rd_base(int t, int p) {
    return kFastRead ? row(t) * PB + p : 0;
  }
  __device__ static __forceinline__ int rd(int base, int t, int p, int u) {
    return kFastRead ? base + u * TPC * PB : row(t + TPC * u) * PB + p;
  }
};

// The FP32 y passes pair ADJACENT columns: thread (t, p) holds columns 2p
// and 2p + 1 of the CTA's B and moves both with one 16-byte access, and B
// is 16 where the CTA allows it, so a warp's access covers whole 128-byte
// row segments.  (Row pitches are multiples of 16 columns, so the pair of
// the last valid column lies in the padding and is read but never stored.)
template <int L, int BW = 16>
struct PY {
  static constexpr int B = BW < 8192 / L ? BW : 8192 / L;
  static constexpr int PB = B / 2;
  static constexpr int TPC = L / 8;
  static constexpr int THREADS = TPC * PB;
  static constexpr int RB = PB * (int)sizeof(CPair);
  static constexpr int R = RB >= 128 ? 1 : 128 / RB;
  __device__ static __forceinline__ int row(int i) {
    return i ^ ((i >> 3) & (R - 1));
  }
  static constexpr bool kFastRead = (TPC / 8) % R == 0;
  __device__ static __forceinline__ int rd_base(int t, int p) {
    return kFastRead ? row(t) * PB + p : 0;
  }
  __device__ static __forceinline__ int rd(int base, int t, int p, int u) {
    return kFastRead ? base + u * TPC * PB : row(t + TPC * u) * PB + p;
  }
  static constexpr size_t smem = (size_t)L * PB * sizeof(CPair);
};

__device__ __forceinline__ CPair load_pair(const float2 *p) {
  const float4 q = *reinterpret_cast<const float4 *>(p);
  return cpack(make_float2(q.x, q.y), make_float2(q.z, q.w));
}
__device__ __forceinline__ void store_pair(float2 *p, const CPair &v, bool v0,
                                           bool v1) {
  if (v1) {
    const float2 a = clane0(v), b = clane1(v);
    *reinterpret_cast<float4 *>(p) = make_float4(a.x, a.y, b.x, b.y);
  } else if (v0) {
    *p = clane0(v);
  }
}

// The column pair of thread p in a column pass.  Ordinary CTAs hold
// adjacent columns c0, c0 + 1 of one plane (one 16-byte access).  When the
// pass runs with `nyq`, the CTAs of the last column group (SPLIT) instead
// hold the last column (kz = N2/2, alone in its 16-column group) of planes
// 2p and 2p + 1 of their group of B planes, so that column does not take a
// whole group of mostly padding columns per plane.  The kernels branch once
// per CTA between the two forms, each compiled separately.
template <bool SPLIT>
struct ColPair {
  int64_t b0, b1;  // element offsets of the two columns' first rows
  bool v0, v1;     // whether each column exists
  __device__ CPair load(const float2 *a, int64_t row) const {
    if constexpr (!SPLIT) return load_pair(a + b0 + row);
    else return cpack(a[b0 + row], a[b1 + row]);
  }
  __device__ void store(float2 *a, int64_t row, const CPair &v) const {
    if constexpr (!SPLIT) {
      store_pair(a + b0 + row, v, v0, v1);
    } else {
      if (v0) a[b0 + row] = clane0(v);
      if (v1) a[b1 + row] = clane1(v);
    }
  }
  // Asynchronous copy of the pair at `row` into a 16-byte shared slot, laid
  // out as in memory (re, im of each column).
  __device__ void copy_async(CPair *slot, const float2 *a, int64_t row) const {
    if constexpr (!SPLIT) {
      cp_async16(slot, a + b0 + row);
    } else {
      float2 *d = reinterpret_cast<float2 *>(slot);
      cp_async8(d, a + b0 + row);
      cp_async8(d + 1, a + b1 + row);
    }
  }
};

// Column pair of thread p in the CTA of group blockIdx.x and plane (or, for
// SPLIT, plane group) `plane`, in a pass whose `nplanes` planes are `pitch`
// elements apart.  Returns false when a SPLIT CTA has no planes left.
template <int B, bool SPLIT>
__device__ __forceinline__ bool col_pair(ColPair<SPLIT> &c, int p, int plane,
                                         int64_t pitch, int nplanes,
                                         const FusedGeom &g) {
  if constexpr (SPLIT) {
    const int pl0 = plane * B;
    if (pl0 >= nplanes) return false;
    const int pa = pl0 + 2 * p;
    c.v0 = pa < nplanes;
    c.v1 = pa + 1 < nplanes;
    c.b0 = (int64_t)(c.v0 ? pa : 0) * pitch + g.h - 1;
    c.b1 = (int64_t)(c.v1 ? pa + 1 : 0) * pitch + g.h - 1;
  } else {
    const int c0 = blockIdx.x * B + 2 * p;
    c.v0 = c0 < g.h;
    c.v1 = c0 + 1 < g.h;
    c.b0 = (int64_t)plane * pitch + c0;
    c.b1 = c.b0 + 1;
  }
  return true;
}

// Whether this CTA takes the last column of a group of planes.
__device__ __forceinline__ bool split_cta(int nyq) {
  return nyq != 0 && blockIdx.x == gridDim.x - 1;
}

template <int L, bool SPLIT>
__device__ __forceinline__ void yfwd_pp_body(float2 *__restrict__ W,
                                             const FusedGeom &g,
                                             const float2 *__restrict__ taby) {
  using Q = PY<L>;
  extern __shared__ unsigned char smem_raw[];
  CPair *ex = reinterpret_cast<CPair *>(smem_raw);
  const int t = threadIdx.x / Q::PB;
  const int p = threadIdx.x - t * Q::PB;
  // Planes are x, L * g.hp elements apart.
  ColPair<SPLIT> cp;
  if (!col_pair<Q::B>(cp, p, blockIdx.y, (int64_t)L * g.hp, g.n0, g)) return;
  CPair v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) v[u] = cp.load(W, (int64_t)(t + Q::TPC * u) * g.hp);
  const int rb = Q::rd_base(t, p);
  reg_fft<L>(v, t, [&](int i) { return &ex[Q::row(i) * Q::PB + p]; },
             [&](int u) { return &ex[Q::rd(rb, t, p, u)]; }, taby, -1);
#pragma unroll
  for (int u = 0; u < 8; ++u) cp.store(W, (int64_t)(t + Q::TPC * u) * g.hp, v[u]);
}

template <int L>
__global__ void __launch_bounds__(PY<L>::THREADS, 1024 / PY<L>::THREADS)
    k_yfwd_pp(float2 *__restrict__ W, FusedGeom g,
              const float2 *__restrict__ taby) {
  // (Splitting off the last column measured slower here: 194 vs 183 us.)
  yfwd_pp_body<L, false>(W, g, taby);
}

// grid2's x transform in the FP32 form: G = DFT_x(W), the same column
// pairing as the y passes, with rows N1 * hp elements apart.
template <int L, bool SPLIT>
__device__ __forceinline__ void xfwd_pp_body(const float2 *__restrict__ W,
                                             float2 *__restrict__ G,
                                             const FusedGeom &g,
                                             const float2 *__restrict__ tabx) {
  using Q = PY<L>;
  extern __shared__ unsigned char smem_raw[];
  CPair *ex = reinterpret_cast<CPair *>(smem_raw);
  const int t = threadIdx.x / Q::PB;
  const int p = threadIdx.x - t * Q::PB;
  const int64_t stride = (int64_t)g.n1 * g.hp;
  // Planes are y, g.hp elements apart.
  ColPair<SPLIT> cp;
  if (!col_pair<Q::B>(cp, p, blockIdx.y, g.hp, g.n1, g)) return;
  CPair v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) v[u] = cp.load(W, (t + Q::TPC * u) * stride);
  const int rb = Q::rd_base(t, p);
  reg_fft<L>(v, t, [&](int i) { return &ex[Q::row(i) * Q::PB + p]; },
             [&](int u) { return &ex[Q::rd(rb, t, p, u)]; }, tabx, -1);
#pragma unroll
  for (int u = 0; u < 8; ++u) cp.store(G, (t + Q::TPC * u) * stride, v[u]);
}

template <int L>
__global__ void __launch_bounds__(PY<L>::THREADS, 1024 / PY<L>::THREADS)
    k_xfwd_pp(const float2 *__restrict__ W, float2 *__restrict__ G, FusedGeom g,
              const float2 *__restrict__ tabx) {
  xfwd_pp_body<L, false>(W, G, g, tabx);
}

// The FP32 x pass of one (ell, m) term with the same column pairing.
// MODE 1: P = DFT_x(W) conj(G); MODE 2 (ell = 0 of an autocorrelation):
// P = w00 |G|^2 with no forward transform (see k_xcorr_p2).  Then the
// k-subgrid extraction and the inverse transform, stored only at the
// r-subgrid's rows.  G is read after the forward transform, so a thread
// holds one pair of columns at a time and two CTAs fit an SM; the other
// CTA's warps cover those loads.
constexpr int kXB = 16;  // columns per CTA of the FP32 x passes

// k-subgrid extraction of k_xcorr_pp (as in k_xcorr_p2) for the columns c0
// and c0 + 1 of thread (t, p), from P staged in the exchange slots.  Not
// inlined, so that its registers do not weigh on the kernel's transforms;
// only the CTAs whose y and kz reach the k-subgrid call it.
template <int L>
__device__ __noinline__ void xcorr_pp_extract(const CPair *ex, int t, int p,
                                              int c0, int jr0, int jr1, int ks0,
                                              int ks1, int ks2, int n1,
                                              double *__restrict__ ksub,
                                              const float *__restrict__ ktab) {
  using Q = PY<L, kXB>;
  const int ox = ks0 / 2, oz = ks2 / 2;
  auto exf = [&](int i) { return &ex[Q::row(i) * Q::PB + p]; };
  if (ks0 <= 3 * Q::TPC && ks1 <= n1) {
    // At most three x rows per thread and one row j per reflection: each
    // reflection's loads are issued together.
#pragma unroll
    for (int refl = 0; refl < 2; ++refl) {
      const int j = refl == 0 ? jr0 : jr1;
      if (j >= ks1) continue;
      size_t cell[3][2];
      double acc[3][2], w[3][2], re[3][2];
      bool on[3][2];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const int i = t + s * Q::TPC;
        const int x = refl == 0 ? (i - ox) & (L - 1) : (ox - i) & (L - 1);
#pragma unroll
        for (int ln = 0; ln < 2; ++ln) {
          const int kzi = c0 + ln;
          on[s][ln] = i < ks0 && kzi <= oz && !(refl == 1 && kzi == 0);
          const int k = refl == 0 ? kzi + oz : oz - kzi;
          cell[s][ln] = ((size_t)i * ks1 + j) * ks2 + k;
          if (on[s][ln]) {
            re[s][ln] = (double)(ln ? exf(x)->x.y : exf(x)->x.x);
            w[s][ln] = (double)ktab[cell[s][ln]];
            acc[s][ln] = ksub[cell[s][ln]];
          }
        }
      }
#pragma unroll
      for (int s = 0; s < 3; ++s)
#pragma unroll
        for (int ln = 0; ln < 2; ++ln)
          if (on[s][ln]) ksub[cell[s][ln]] = acc[s][ln] + w[s][ln] * re[s][ln];
    }
    return;
  }
  for (int ln = 0; ln < 2; ++ln) {
    const int kzi = c0 + ln;
    if (kzi > oz) continue;
    for (int refl = 0; refl < 2; ++refl) {
      if (refl == 1 && kzi == 0) continue;
      const int k = refl == 0 ? kzi + oz : oz - kzi;
      for (int j = refl == 0 ? jr0 : jr1; j < ks1; j += n1) {
        for (int i = t; i < ks0; i += Q::TPC) {
          const int x = refl == 0 ? (i - ox) & (L - 1) : (ox - i) & (L - 1);
          const double re = (double)(ln ? exf(x)->x.y : exf(x)->x.x);
          const size_t cell = ((size_t)i * ks1 + j) * ks2 + k;
          ksub[cell] += (double)ktab[cell] * re;
        }
      }
    }
  }
}

template <int L, int MODE, bool SPLIT>
__device__ __forceinline__ void xcorr_pp_body(
    const float2 *__restrict__ W, const float2 *__restrict__ G,
    float2 *__restrict__ out, double *__restrict__ ksub, const FusedGeom &g,
    const float2 *__restrict__ tabx, const float *__restrict__ ktab, float w00) {
  using Q = PY<L, kXB>;
  extern __shared__ unsigned char smem_raw[];
  CPair *ex = reinterpret_cast<CPair *>(smem_raw);
  const int t = threadIdx.x / Q::PB;
  const int p = threadIdx.x - t * Q::PB;
  const int yy = blockIdx.y;
  const int64_t stride = (int64_t)g.n1 * g.hp;
  // Planes are y, g.hp elements apart; with nyq the host has made sure the
  // last column lies outside the k-subgrid.
  ColPair<SPLIT> cp;
  if (!col_pair<Q::B>(cp, p, yy, g.hp, g.n1, g)) return;
  const int cb = SPLIT ? g.h - 1 : blockIdx.x * Q::B;
  const int c0 = SPLIT ? g.h - 1 : cb + 2 * p;
  auto exf = [&](int i) { return &ex[Q::row(i) * Q::PB + p]; };
  const int rb = Q::rd_base(t, p);
  auto exr = [&](int u) { return &ex[Q::rd(rb, t, p, u)]; };
  CPair v[8];
  if constexpr (MODE == 2) {
    const float2 w = f2splat(w00);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const CPair q = cp.load(G, (t + Q::TPC * u) * stride);
      v[u].x = w * __ffma2_rn(q.x, q.x, q.y * q.y);
      v[u].y = f2splat(0.f);
    }
  } else {
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = cp.load(W, (t + Q::TPC * u) * stride);
    // G's pairs are copied into this thread's own exchange slots while the
    // last pass of the forward transform computes.  A slot then holds the
    // two columns as stored in memory, (re, im) of each, so it is read back
    // with load_pair like a global pair.
    reg_fft<L>(v, t, exf, exr, tabx, -1, 1, [&] {
#pragma unroll
      for (int u = 0; u < 8; ++u)
        cp.copy_async(exr(u), G, (t + Q::TPC * u) * stride);
    });
    cp_async_wait_all();
#pragma unroll
    for (int u = 0; u < 8; ++u)
      v[u] = cmulc(v[u], load_pair(reinterpret_cast<const float2 *>(exr(u))));
  }
  // k-subgrid extraction, as in k_xcorr_p2, for both columns of the pair.
  const int oy = g.ks1 / 2, oz = g.ks2 / 2;
  const int jr0 = (yy + oy) % g.n1;
  const int jr1 = ((oy - yy) % g.n1 + g.n1) % g.n1;
  if (ksub != nullptr && cb <= oz && (jr0 < g.ks1 || jr1 < g.ks1)) {
    // P goes through shared memory and is read back afterwards, so the
    // registers of the pair are free while the extraction runs.
#pragma unroll
    for (int u = 0; u < 8; ++u) *exr(u) = v[u];
    __syncthreads();
    if (c0 <= oz)
      xcorr_pp_extract<L>(ex, t, p, c0, jr0, jr1, g.ks0, g.ks1, g.ks2, g.n1,
                          ksub, ktab);
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = *exr(u);
    __syncthreads();
  } else if constexpr (MODE == 1) {
    // Every thread has read G from its slots before the inverse transform's
    // first exchange writes over them.
    __syncthreads();
  }
  // Rows x whose r-subgrid row (x + ro) mod L is below rs; when they all lie
  // in the first and last TPC rows, only outputs u = 0 and 7 are computed.
  const bool edges = g.ro <= Q::TPC && g.rs - g.ro <= Q::TPC;
  reg_fft<L>(v, t, exf, exr, tabx, +1, 1, NoHook{}, edges);
  if (edges) {
#pragma unroll
    for (int u = 0; u < 8; u += 7) {
      const int ri = (t + Q::TPC * u + g.ro) & (L - 1);
      if (ri < g.rs) cp.store(out, ri * stride, v[u]);
    }
    return;
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int x = t + Q::TPC * u;
    for (int ri = (x + g.ro) & (L - 1); ri < g.rs; ri += L)
      cp.store(out, ri * stride, v[u]);
  }
}

template <int L, int MODE>
__global__ void __launch_bounds__(PY<L, kXB>::THREADS, 1024 / PY<L, kXB>::THREADS)
    k_xcorr_pp(const float2 *__restrict__ W, const float2 *__restrict__ G,
               float2 *__restrict__ out, double *__restrict__ ksub, FusedGeom g,
               const float2 *__restrict__ tabx, const float *__restrict__ ktab,
               float w00, int nyq) {
  // The last column split off (nyq) pays in the product mode only; the
  // ell = 0 mode compiles without it (with it: 215 vs 188 us).
  if constexpr (MODE == 1) {
    if (split_cta(nyq)) {
      xcorr_pp_body<L, MODE, true>(W, G, out, ksub, g, tabx, ktab, w00);
      return;
    }
  }
  xcorr_pp_body<L, MODE, false>(W, G, out, ksub, g, tabx, ktab, w00);
}

template <int L, bool SPLIT>
__device__ __forceinline__ void yinv_pp_body(const float2 *__restrict__ Wr,
                                             float2 *__restrict__ Wry,
                                             const FusedGeom &g,
                                             const float2 *__restrict__ taby) {
  using Q = PY<L>;
  extern __shared__ unsigned char smem_raw[];
  CPair *ex = reinterpret_cast<CPair *>(smem_raw);
  const int t = threadIdx.x / Q::PB;
  const int p = threadIdx.x - t * Q::PB;
  // Planes are the r-subgrid's x rows ri: L * g.hp elements apart in Wr,
  // rs * g.hp in Wry.
  ColPair<SPLIT> cp;
  if (!col_pair<Q::B>(cp, p, blockIdx.y, (int64_t)L * g.hp, g.rs, g)) return;
  CPair v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) v[u] = cp.load(Wr, (int64_t)(t + Q::TPC * u) * g.hp);
  const int rb = Q::rd_base(t, p);
  const bool edges = g.ro <= Q::TPC && g.rs - g.ro <= Q::TPC;  // see k_xcorr_pp
  reg_fft<L>(v, t, [&](int i) { return &ex[Q::row(i) * Q::PB + p]; },
             [&](int u) { return &ex[Q::rd(rb, t, p, u)]; }, taby, +1, 1,
             NoHook{}, edges);
  ColPair<SPLIT> co;  // the same columns of the same planes in Wry
  col_pair<Q::B>(co, p, blockIdx.y, (int64_t)g.rs * g.hp, g.rs, g);
  if (edges) {
#pragma unroll
    for (int u = 0; u < 8; u += 7) {
      const int rj = (t + Q::TPC * u + g.ro) & (L - 1);
      if (rj < g.rs) co.store(Wry, (int64_t)rj * g.hp, v[u]);
    }
    return;
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int y = t + Q::TPC * u;
    for (int rj = (y + g.ro) & (L - 1); rj < g.rs; rj += L)
      co.store(Wry, (int64_t)rj * g.hp, v[u]);
  }
}

template <int L>
__global__ void __launch_bounds__(PY<L>::THREADS, 1024 / PY<L>::THREADS)
    k_yinv_pp(const float2 *__restrict__ Wr, float2 *__restrict__ Wry,
              FusedGeom g, const float2 *__restrict__ taby, int nyq) {
  if (split_cta(nyq))
    yinv_pp_body<L, true>(Wr, Wry, g, taby);
  else
    yinv_pp_body<L, false>(Wr, Wry, g, taby);
}

// Rows of the z transform, two rows per thread: rows b and b + PB of the
// CTA's B, thread t of a row pair holding z[t + TPC u] of both.
template <int L, bool WEIGHT>
__global__ void __launch_bounds__(PP<L>::THREADS)
    k_zfwd_pp(const float *__restrict__ rho, float2 *__restrict__ W, FusedGeom g,
              YlmParams p, double x0, double y0, double z0,
              const float2 *__restrict__ tabz,
              const float4 *__restrict__ rowtab) {
  using Q = PP<L>;
  constexpr int RP = L + L / 8 + 1;
  extern __shared__ unsigned char smem_raw[];
  CPairS *ex = reinterpret_cast<CPairS *>(smem_raw);
  const int pb = threadIdx.x / Q::TPC;
  const int t = threadIdx.x - pb * Q::TPC;
  const int64_t nrows = (int64_t)g.n0 * g.n1;
  const int64_t row0 = (int64_t)blockIdx.x * Q::B + pb;
  const int64_t row1 = row0 + Q::PB;
  const bool v0 = row0 < nrows, v1 = row1 < nrows;
  const float2 *src0 = reinterpret_cast<const float2 *>(rho + (v0 ? row0 : 0) * g.n2);
  const float2 *src1 = reinterpret_cast<const float2 *>(rho + (v1 ? row1 : 0) * g.n2);
  RowPoly rp0, rp1;
  float zt = 0.f;
  if constexpr (WEIGHT) {
    if (rowtab != nullptr) {
      // Per-row coefficients from k_rowpoly (the same FP64 evaluation).
      rp0 = load_row_poly(rowtab, v0 ? row0 : 0, p);
      rp1 = load_row_poly(rowtab, v1 ? row1 : 0, p);
    } else {
      const int xa = (int)(row0 / g.n1), ya = (int)(row0 - (int64_t)xa * g.n1);
      const int xb = (int)(row1 / g.n1), yb = (int)(row1 - (int64_t)xb * g.n1);
      rp0 = row_poly(p, x0 + xa * 1.0, y0 + ya * 1.0);
      rp1 = row_poly(p, x0 + xb * 1.0, y0 + yb * 1.0);
    }
    zt = (float)(z0 + (2 * t) * 1.0);
  }
  const float2 zero = make_float2(0.f, 0.f);
  float2 a[8], b[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int jj = t + Q::TPC * u;
    a[u] = v0 ? src0[jj] : zero;
    b[u] = v1 ? src1[jj] : zero;
  }
  if constexpr (WEIGHT) {
    // One uniform branch per thread picks the weight's form.
    auto weigh = [&](auto poly, auto ellc) {
      constexpr int POLY = decltype(poly)::value, ELL = decltype(ellc)::value;
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const float zu = zt + (float)(2 * Q::TPC * u);
        a[u].x = row_weight_form<POLY, ELL>(rp0, a[u].x, zu);
        a[u].y = row_weight_form<POLY, ELL>(rp0, a[u].y, zu + 1.0f);
        b[u].x = row_weight_form<POLY, ELL>(rp1, b[u].x, zu);
        b[u].y = row_weight_form<POLY, ELL>(rp1, b[u].y, zu + 1.0f);
      }
    };
    using std::integral_constant;
    using I2 = integral_constant<int, 2>;
    using I4 = integral_constant<int, 4>;
    if (p.ell == 0) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        a[u] = make_float2(a[u].x * rp0.value0, a[u].y * rp0.value0);
        b[u] = make_float2(b[u].x * rp1.value0, b[u].y * rp1.value0);
      }
    } else if (p.ell == 2) {
      switch (row_poly_form(2, p.m)) {
        case 0: weigh(integral_constant<int, 0>(), I2()); break;
        case 1: weigh(integral_constant<int, 1>(), I2()); break;
        default: weigh(integral_constant<int, 2>(), I2()); break;
      }
    } else {
      switch (row_poly_form(4, p.m)) {
        case 0: weigh(integral_constant<int, 0>(), I4()); break;
        case 1: weigh(integral_constant<int, 1>(), I4()); break;
        case 2: weigh(integral_constant<int, 2>(), I4()); break;
        case 3: weigh(integral_constant<int, 3>(), I4()); break;
        default: weigh(integral_constant<int, 4>(), I4()); break;
      }
    }
  }
  CPairS v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) v[u] = cpack_s(a[u], b[u]);
  auto exf = [&](int i) { return &ex[pb * RP + i + (i >> 3)]; };
  reg_fft<L>(v, t, exf, tabz, -1, 2);
#pragma unroll
  for (int u = 0; u < 8; ++u) *exf(t + Q::TPC * u) = v[u];
  __syncthreads();
  float2 *dst0 = W + row0 * g.hp;
  float2 *dst1 = W + row1 * g.hp;
  // Real-to-complex split, outputs k and L - k together: with
  // e = (Z_k + conj Z_{L-k}) / 2 and o = -i (Z_k - conj Z_{L-k}) / 2,
  // X_k = e + o w_k and X_{L-k} = conj(e - o w_k) (w_{L-k} = -conj w_k).
  // Unrolled so the twiddle loads of all outputs issue together.
#pragma unroll
  for (int i = 0; i <= L / 2 / Q::TPC; ++i) {
    const int k = t + Q::TPC * i;
    if (k > L / 2) break;
    const CPairS za = *exf(k);
    const CPairS c = cconj(*exf(k == 0 ? 0 : L - k));
    CPairS e, o;
    e.x = 0.5f * (za.x + c.x);
    e.y = 0.5f * (za.y + c.y);
    const CPairS d = csub(za, c);
    o.x = 0.5f * d.y;
    o.y = -0.5f * d.x;
    const CPairS ow = cmul(o, __ldg(&tabz[k]));
    const CPairS r = cadd(e, ow);
    if (v0) dst0[k] = clane0(r);
    if (v1) dst1[k] = clane1(r);
    if (k != L / 2) {
      const CPairS q = cconj(csub(e, ow));
      if (v0) dst0[L - k] = clane0(q);
      if (v1) dst1[L - k] = clane1(q);
    }
  }
}

// Calls f(POLY, ELL) with the compile-time form of an (ell > 0, m) term's
// row polynomial (row_poly_form).
template <typename F>
__device__ __forceinline__ void with_row_form(const YlmParams &p, F &&f) {
  using std::integral_constant;
  using I2 = integral_constant<int, 2>;
  using I4 = integral_constant<int, 4>;
  if (p.ell == 2) {
    switch (row_poly_form(2, p.m)) {
      case 0: f(integral_constant<int, 0>(), I2()); break;
      case 1: f(integral_constant<int, 1>(), I2()); break;
      default: f(integral_constant<int, 2>(), I2()); break;
    }
  } else {
    switch (row_poly_form(4, p.m)) {
      case 0: f(integral_constant<int, 0>(), I4()); break;
      case 1: f(integral_constant<int, 1>(), I4()); break;
      case 2: f(integral_constant<int, 2>(), I4()); break;
      case 3: f(integral_constant<int, 3>(), I4()); break;
      default: f(integral_constant<int, 4>(), I4()); break;
    }
  }
}

// The row polynomial of form POLY at z (z2 = z^2), as row_weight_form.
template <int POLY>
__device__ __forceinline__ float row_poly_at(const RowPoly &r, float z, float z2) {
  if constexpr (POLY == 0) return r.c[0];
  else if constexpr (POLY == 1) return r.c[1] * z;
  else if constexpr (POLY == 2) return r.c[2] * z2 + r.c[0];
  else if constexpr (POLY == 3) return (r.c[3] * z2 + r.c[1]) * z;
  else return (r.c[4] * z2 + r.c[2]) * z2 + r.c[0];
}

// One row weighted for two terms a and q: b = Y_q * a, then a = Y_a * a,
// with the same operations as row_weight_form; z^2 and 1/r^2 depend only
// on the row and z, so they are computed once for both terms.
template <int TPC>
__device__ __forceinline__ void weigh_row_pair(const RowPoly &ra,
                                               const YlmParams &pa,
                                               const RowPoly &rq,
                                               const YlmParams &pq, float zt,
                                               float2 *a, float2 *b) {
  with_row_form(pa, [&](auto polya, auto ella) {
    with_row_form(pq, [&](auto polyq, auto ellq) {
      constexpr int PA = decltype(polya)::value, EA = decltype(ella)::value;
      constexpr int PQ = decltype(polyq)::value, EQ = decltype(ellq)::value;
      auto one = [&](float d, float z, float &wa, float &wq) {
        const float z2 = z * z;
        const float ir2 = __fdividef(1.0f, ra.rxy2 + z2 + 1e-20f);
        const float fa = EA == 2 ? ir2 : ir2 * ir2;
        const float fq = EQ == 2 ? ir2 : ir2 * ir2;
        wq = d * row_poly_at<PQ>(rq, z, z2) * fq;
        wa = d * row_poly_at<PA>(ra, z, z2) * fa;
      };
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const float zu = zt + (float)(2 * TPC * u);
        one(a[u].x, zu, a[u].x, b[u].x);
        one(a[u].y, zu + 1.0f, a[u].y, b[u].y);
      }
    });
  });
}

// The weighted z pass of two (ell > 0, m) terms at once: thread t of row
// group pb holds z[t + TPC u] of one row, and its two transforms are that
// row weighted for term a and for term b.  The density row is read once
// for both terms and each term's W gets its row, so a pair of terms reads
// the density once instead of twice; the transform and the real-to-complex
// split are those of k_zfwd_pp.
template <int L>
__global__ void __launch_bounds__(PP<L>::THREADS, 1024 / PP<L>::THREADS)
    k_zfwd_pp2(const float *__restrict__ rho, float2 *__restrict__ Wa,
               float2 *__restrict__ Wb, FusedGeom g, YlmParams pa, YlmParams pq,
               double z0, const float2 *__restrict__ tabz,
               const float4 *__restrict__ rowtab_a,
               const float4 *__restrict__ rowtab_b) {
  using Q = PP<L>;
  constexpr int RP = L + L / 8 + 1;
  extern __shared__ unsigned char smem_raw[];
  CPairS *ex = reinterpret_cast<CPairS *>(smem_raw);
  const int pb = threadIdx.x / Q::TPC;
  const int t = threadIdx.x - pb * Q::TPC;
  const int64_t nrows = (int64_t)g.n0 * g.n1;
  const int64_t row = (int64_t)blockIdx.x * Q::PB + pb;
  const bool valid = row < nrows;
  const int64_t r = valid ? row : 0;
  const float2 *src = reinterpret_cast<const float2 *>(rho + r * g.n2);
  const RowPoly ra = load_row_poly(rowtab_a, r, pa);
  const RowPoly rq = load_row_poly(rowtab_b, r, pq);
  const float zt = (float)(z0 + (2 * t) * 1.0);
  const float2 zero = make_float2(0.f, 0.f);
  float2 a[8], b[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) a[u] = valid ? src[t + Q::TPC * u] : zero;
  weigh_row_pair<Q::TPC>(ra, pa, rq, pq, zt, a, b);
  CPairS v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) v[u] = cpack_s(a[u], b[u]);
  auto exf = [&](int i) { return &ex[pb * RP + i + (i >> 3)]; };
  reg_fft<L>(v, t, exf, tabz, -1, 2);
#pragma unroll
  for (int u = 0; u < 8; ++u) *exf(t + Q::TPC * u) = v[u];
  __syncthreads();
  if (!valid) return;
  float2 *dst0 = Wa + row * g.hp;
  float2 *dst1 = Wb + row * g.hp;
#pragma unroll
  for (int i = 0; i <= L / 2 / Q::TPC; ++i) {
    const int k = t + Q::TPC * i;
    if (k > L / 2) break;
    const CPairS za = *exf(k);
    const CPairS c = cconj(*exf(k == 0 ? 0 : L - k));
    CPairS e, o;
    e.x = 0.5f * (za.x + c.x);
    e.y = 0.5f * (za.y + c.y);
    const CPairS d = csub(za, c);
    o.x = 0.5f * d.y;
    o.y = -0.5f * d.x;
    const CPairS ow = cmul(o, __ldg(&tabz[k]));
    const CPairS rr = cadd(e, ow);
    dst0[k] = clane0(rr);
    dst1[k] = clane1(rr);
    if (k != L / 2) {
      const CPairS q = cconj(csub(e, ow));
      dst0[L - k] = clane0(q);
      dst1[L - k] = clane1(q);
    }
  }
}

// Per-row Horner coefficients of one (ell, m) (row_poly), two float4 per
// row, so the z pass does no FP64 work per row.
__global__ void k_rowpoly(float4 *__restrict__ tab, int64_t nrows, int n1,
                          YlmParams p, double x0, double y0) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
       row < nrows; row += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(row / n1);
    const int y = (int)(row - (int64_t)x * n1);
    const RowPoly r = row_poly(p, x0 + x * 1.0, y0 + y * 1.0);
    tab[2 * row] = make_float4(r.c[0], r.c[1], r.c[2], r.c[3]);
    tab[2 * row + 1] = make_float4(r.c[4], r.rxy2, 0.f, 0.f);
  }
}

// Per-cell r-subgrid weight of one (ell, m): Y_lm(r) with the r-subgrid
// normalisation (make_ylm, correlator.h:477-480), computed once per
// correlator and multipole so the z inverse pass does a multiply-add.
template <typename RT>
__global__ void k_rtable(RT *__restrict__ tab, int rs,
                         const double *__restrict__ raxis, YlmParams pr) {
  const size_t n = (size_t)rs * rs * rs;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int rk = (int)(i % rs);
    const int rj = (int)((i / rs) % rs);
    const int ri = (int)(i / ((size_t)rs * rs));
    tab[i] = (RT)ylm_eval(pr, 1.0, raxis[ri], raxis[rj], raxis[rk]);
  }
}

// Per-cell k-subgrid weight of one (ell, m): Y_lm(k) * 4 pi / (W(kx) W(ky)
// W(kz)) with make_ylm's arithmetic (correlator.h:453-466), computed once
// per correlator and multipole so the extraction in the x pass is a
// multiply-add.
template <typename KT>
__global__ void k_ktable(KT *__restrict__ tab, int k0, int k1, int k2,
                         const double *__restrict__ kx,
                         const double *__restrict__ ky,
                         const double *__restrict__ kz,
                         const double *__restrict__ wx,
                         const double *__restrict__ wy,
                         const double *__restrict__ wz, YlmParams pk) {
  const size_t n = (size_t)k0 * k1 * k2;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n;
       c += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(c % k2);
    const int j = (int)((c / k2) % k1);
    const int i = (int)(c / ((size_t)k2 * k1));
    const double inv_w = 1.0 / (wx[i] * wy[j] * wz[k]);
    tab[c] = (KT)ylm_eval(pk, inv_w, kx[i], ky[j], kz[k]);
  }
}

__global__ void k_to_float(const double *__restrict__ in, float *__restrict__ out,
                           size_t n, double shift) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)(in[i] - shift);
}

// Radices of a length, largest first (8, 4, 2, 3, 5, 7); false if L has a
// prime factor above 7.
bool plan_length(int L, int tab_scale, FftPlan *p) {
  p->L = L;
  p->tab_scale = tab_scale;
  p->npass = 0;
  int n = L;
  const int radices[] = {8, 4, 2, 3, 5, 7};
  for (int r : radices) {
    while (n % r == 0) {
      if (p->npass == 12) return false;
      p->radix[p->npass++] = r;
      n /= r;
    }
  }
  if (n != 1) return false;
  int ns = 1;
  for (int s = 0; s < p->npass; ++s) {
    p->ns[s] = ns;
    p->nsmask[s] = (ns & (ns - 1)) == 0 ? ns - 1 : -1;
    ns *= p->radix[s];
  }
  return true;
}

template <typename C>
std::vector<C> root_table(int order) {
  std::vector<C> t(order);
  for (int m = 0; m < order; ++m) {
    // e^{-2 pi i m / order}, argument reduced exactly before the FP64 call.
    const double a = 2.0 * M_PI * (double)m / (double)order;
    t[m].x = (decltype(t[m].x))cos(a);
    t[m].y = (decltype(t[m].y))(-sin(a));
  }
  return t;
}

// Threads per CTA for a pass of length L over B columns: one thread per
// radix-8 butterfly where possible, between 128 and 256.
int threads_for(int L, int B) {
  int t = (L / 8) * B;
  t = ((t + 31) / 32) * 32;
  return std::max(128, std::min(256, t));
}

// ----------------------------------------------------- power-of-two dispatch

bool is_p2(int L) { return L >= 64 && L <= 2048 && (L & (L - 1)) == 0; }

template <typename T, int L>
size_t p2_col_smem() {
  return (size_t)L * P2<T, L>::B * sizeof(C2<T>);
}
template <typename T, int L>
size_t p2_row_smem() {
  return (size_t)P2<T, L>::B * (L + L / 8 + 1) * sizeof(C2<T>);
}

// Calls f.template operator()<L>() for the power-of-two L.
template <typename F>
void with_p2(int L, F &&f) {
  switch (L) {
    case 64: f.template operator()<64>(); break;
    case 128: f.template operator()<128>(); break;
    case 256: f.template operator()<256>(); break;
    case 512: f.template operator()<512>(); break;
    case 1024: f.template operator()<1024>(); break;
    default: f.template operator()<2048>(); break;
  }
}

template <typename T, int L>
void p2_set_limits() {
  const int big = 200 * 1024;
  FC_CUDA(cudaFuncSetAttribute(k_yfwd_p2<T, L>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_yinv_p2<T, L>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_xcorr_p2<T, L, 0>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_xcorr_p2<T, L, 1>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_xcorr_p2<T, L, 2>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_zfwd_p2<T, L, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_zfwd_p2<T, L, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_zinv_p2<T, L>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  if constexpr (std::is_same_v<T, float>) {
    FC_CUDA(cudaFuncSetAttribute(k_yfwd_pp<L>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_yinv_pp<L>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_xfwd_pp<L>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_xcorr_pp<L, 1>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_xcorr_pp<L, 2>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_zfwd_pp<L, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_zfwd_pp<L, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_zfwd_pp2<L>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  }
}

}  // namespace

bool FusedSurvey::supported(const int shape[3], int rsize) {
  if (shape[2] % 2 != 0) return false;
  FftPlan p;
  if (!plan_length(shape[0], 1, &p) || !plan_length(shape[1], 1, &p) ||
      !plan_length(shape[2] / 2, 2, &p))
    return false;
  // Two shared tiles of L x (B+1) complex must fit in 200 KB.
  for (int a = 0; a < 3; ++a) {
    const int L = a == 2 ? shape[2] / 2 : shape[a];
    if (2 * (size_t)L * 5 * 16 > 200 * 1024 || 2 * (size_t)L * 9 * 8 > 200 * 1024)
      return false;
  }
  return rsize > 0;
}

FusedSurvey::FusedSurvey(const int shape[3], int rsize, const int kshape[3],
                         bool fp64)
    : fp64_(fp64) {
  g.n0 = shape[0];
  g.n1 = shape[1];
  g.n2 = shape[2];
  g.m = shape[2] / 2;
  g.h = g.m + 1;
  g.hp = (g.h + 15) / 16 * 16;
  g.rs = rsize;
  g.ro = rsize / 2;
  g.ks0 = kshape[0];
  g.ks1 = kshape[1];
  g.ks2 = kshape[2];
  FC_REQUIRE(plan_length(g.n0, 1, &g.px) && plan_length(g.n1, 1, &g.py) &&
                 plan_length(g.m, 2, &g.pz),
             FC_ERR_UNSUPPORTED, "grid size has a prime factor above 7");
  const size_t eb = fp64 ? 16 : 8;
  if (fp64) {
    upload(tabx, root_table<double2>(g.n0));
    upload(taby, root_table<double2>(g.n1));
    upload(tabz, root_table<double2>(g.n2));
  } else {
    upload(tabx, root_table<float2>(g.n0));
    upload(taby, root_table<float2>(g.n1));
    upload(tabz, root_table<float2>(g.n2));
  }
  const size_t nc = (size_t)g.n0 * g.n1 * g.hp;
  W.resize(nc * eb);
  G.resize(nc * eb);
  Wr.resize((size_t)g.rs * g.n1 * g.hp * eb);
  Wry.resize((size_t)g.rs * g.rs * g.hp * eb);
  if (!fp64) {
    rho32.resize((size_t)g.n0 * g.n1 * g.n2 * sizeof(float));
    rowtab.resize((size_t)g.n0 * g.n1 * 2 * sizeof(float4));
    if (pairs()) {
      W2.resize(nc * eb);
      rowtab2.resize((size_t)g.n0 * g.n1 * 2 * sizeof(float4));
    }
  }
  set_smem_limits();
}

template <typename V>
void FusedSurvey::upload(DeviceBuffer &dst, const std::vector<V> &v) {
  dst.resize(v.size() * sizeof(V));
  FC_CUDA(cudaMemcpy(dst.get(), v.data(), v.size() * sizeof(V),
                     cudaMemcpyHostToDevice));
}

size_t FusedSurvey::smem(int L) const {
  const int B = fp64_ ? Tile<double>::B : Tile<float>::B;
  return 2 * (size_t)L * (B + 1) * (fp64_ ? 16 : 8);
}

template <typename T>
static void set_limits_for() {
  const int big = 200 * 1024;
  FC_CUDA(cudaFuncSetAttribute(k_zfwd<T, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_zfwd<T, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_yfwd<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_xcorr<T, 0>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_xcorr<T, 1>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_yinv<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FC_CUDA(cudaFuncSetAttribute(k_zinv_rsub<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, big));
}

void FusedSurvey::set_smem_limits() {
  if (fp64_)
    set_limits_for<double>();
  else
    set_limits_for<float>();
  for (int L : {g.n0, g.n1, g.m}) {
    if (!is_p2(L)) continue;
    if (fp64_)
      with_p2(L, [&]<int LL>() { p2_set_limits<double, LL>(); });
    else
      with_p2(L, [&]<int LL>() { p2_set_limits<float, LL>(); });
  }
}

const void *FusedSurvey::prepare_input(const void *rho, bool f32,
                                       cudaStream_t s) {
  FC_REQUIRE(!(fp64_ && f32), FC_ERR_INVALID,
             "the FP64 passes take FP64 cells");
  if (fp64_ || f32) return rho;
  const size_t n = (size_t)g.n0 * g.n1 * g.n2;
  k_to_float<<<grid_for(n, 256), 256, 0, s>>>(static_cast<const double *>(rho),
                                              rho32.as<float>(), n, 0.0);
  FC_LAUNCH_CHECK();
  return rho32.get();
}

template <typename T>
void FusedSurvey::zfwd(const void *rho, bool weight, const YlmParams &p,
                       const double xyz0[3], cudaStream_t s) {
  if (is_p2(g.m)) {
    with_p2(g.m, [&]<int L>() {
      using Q = P2<T, L>;
      const int64_t nrows = (int64_t)g.n0 * g.n1;
      const unsigned blocks = (unsigned)((nrows + Q::B - 1) / Q::B);
      if constexpr (std::is_same_v<T, float>) {
        using PQ = PP<L>;
        const float4 *rt = nullptr;
        if (weight && p.ell != 0) {
          rowtab.resize((size_t)nrows * 2 * sizeof(float4));
          k_rowpoly<<<grid_for(nrows, 256), 256, 0, s>>>(
              rowtab.as<float4>(), nrows, g.n1, p, xyz0[0], xyz0[1]);
          FC_LAUNCH_CHECK();
          rt = rowtab.as<float4>();
        }
        if (weight)
          k_zfwd_pp<L, true><<<blocks, PQ::THREADS, p2_row_smem<T, L>(), s>>>(
              (const float *)rho, W.as<float2>(), g, p, xyz0[0], xyz0[1],
              xyz0[2], tabz.as<float2>(), rt);
        else
          k_zfwd_pp<L, false><<<blocks, PQ::THREADS, p2_row_smem<T, L>(), s>>>(
              (const float *)rho, W.as<float2>(), g, p, xyz0[0], xyz0[1],
              xyz0[2], tabz.as<float2>(), nullptr);
        return;
      }
      if (weight)
        k_zfwd_p2<T, L, true><<<blocks, Q::THREADS, p2_row_smem<T, L>(), s>>>(
            (const T *)rho, W.as<C2<T>>(), g, p, xyz0[0], xyz0[1], xyz0[2],
            tabz.as<C2<T>>());
      else
        k_zfwd_p2<T, L, false><<<blocks, Q::THREADS, p2_row_smem<T, L>(), s>>>(
            (const T *)rho, W.as<C2<T>>(), g, p, xyz0[0], xyz0[1], xyz0[2],
            tabz.as<C2<T>>());
    });
    FC_LAUNCH_CHECK();
    return;
  }
  constexpr int B = Tile<T>::B;
  const int64_t nrows = (int64_t)g.n0 * g.n1;
  const unsigned blocks = (unsigned)((nrows + B - 1) / B);
  const int threads = threads_for(g.m, B);
  const size_t sm = smem(g.m);
  if (weight)
    k_zfwd<T, true><<<blocks, threads, sm, s>>>(
        (const T *)rho, W.as<C2<T>>(), g, p, xyz0[0], xyz0[1], xyz0[2],
        tabz.as<C2<T>>());
  else
    k_zfwd<T, false><<<blocks, threads, sm, s>>>(
        (const T *)rho, W.as<C2<T>>(), g, p, xyz0[0], xyz0[1], xyz0[2],
        tabz.as<C2<T>>());
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::yfwd(cudaStream_t s) {
  if (is_p2(g.n1)) {
    with_p2(g.n1, [&]<int L>() {
      using Q = P2<T, L>;
      if constexpr (std::is_same_v<T, float>) {
        using Y = PY<L>;
        dim3 grid((g.h + Y::B - 1) / Y::B, g.n0);
        k_yfwd_pp<L><<<grid, Y::THREADS, Y::smem, s>>>(W.as<float2>(), g,
                                                        taby.as<float2>());
      } else {
        dim3 grid((g.h + Q::B - 1) / Q::B, g.n0);
        k_yfwd_p2<T, L><<<grid, Q::THREADS, p2_col_smem<T, L>(), s>>>(
            W.as<C2<T>>(), g, taby.as<C2<T>>());
      }
    });
    FC_LAUNCH_CHECK();
    return;
  }
  constexpr int B = Tile<T>::B;
  dim3 grid((g.h + B - 1) / B, g.n0);
  k_yfwd<T><<<grid, threads_for(g.n1, B), smem(g.n1), s>>>(W.as<C2<T>>(), g,
                                                           taby.as<C2<T>>());
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::xcorr(bool product, double *ksub, const void *ktab_v,
                        cudaStream_t s) {
  const T *ktab = static_cast<const T *>(ktab_v);
  if (is_p2(g.n0)) {
    with_p2(g.n0, [&]<int L>() {
      using Q = P2<T, L>;
      dim3 grid((g.h + Q::B - 1) / Q::B, g.n1);
      if (!product && std::is_same_v<T, float>) {
        using Y = PY<L>;
        dim3 gy((g.h + Y::B - 1) / Y::B, g.n1);
        k_xfwd_pp<L><<<gy, Y::THREADS, Y::smem, s>>>(
            W.as<float2>(), G.as<float2>(), g, tabx.as<float2>());
      } else if (!product)
        k_xcorr_p2<T, L, 0><<<grid, Q::THREADS, p2_col_smem<T, L>(), s>>>(
            W.as<C2<T>>(), nullptr, G.as<C2<T>>(), nullptr, g, tabx.as<C2<T>>(),
            nullptr, T(0));
      else if constexpr (std::is_same_v<T, float>) {
        using Y = PY<L, kXB>;
        dim3 gy((g.h + Y::B - 1) / Y::B, g.n1);
        k_xcorr_pp<L, 1><<<gy, Y::THREADS, Y::smem, s>>>(
            W.as<float2>(), G.as<float2>(), Wr.as<float2>(), ksub, g,
            tabx.as<float2>(), ktab, 0.f, nyq_group<Y::B>(ksub != nullptr));
      } else
        k_xcorr_p2<T, L, 1><<<grid, Q::THREADS, p2_col_smem<T, L>(), s>>>(
            W.as<C2<T>>(), G.as<C2<T>>(), Wr.as<C2<T>>(), ksub, g,
            tabx.as<C2<T>>(), ktab, T(0));
    });
    FC_LAUNCH_CHECK();
    return;
  }
  constexpr int B = Tile<T>::B;
  dim3 grid((g.h + B - 1) / B, g.n1);
  const int threads = threads_for(g.n0, B);
  const size_t sm = smem(g.n0);
  if (!product) {
    k_xcorr<T, 0><<<grid, threads, sm, s>>>(
        W.as<C2<T>>(), nullptr, G.as<C2<T>>(), nullptr, g, tabx.as<C2<T>>(),
        nullptr);
  } else {
    k_xcorr<T, 1><<<grid, threads, sm, s>>>(
        W.as<C2<T>>(), G.as<C2<T>>(), Wr.as<C2<T>>(), ksub, g, tabx.as<C2<T>>(),
        ktab);
  }
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::xcorr00(double *ksub, const void *ktab_v, double w00,
                          cudaStream_t s) {
  const T *ktab = static_cast<const T *>(ktab_v);
  with_p2(g.n0, [&]<int L>() {
    using Q = P2<T, L>;
    if constexpr (std::is_same_v<T, float>) {
      using Y = PY<L, kXB>;
      dim3 gy((g.h + Y::B - 1) / Y::B, g.n1);
      k_xcorr_pp<L, 2><<<gy, Y::THREADS, Y::smem, s>>>(
          nullptr, G.as<float2>(), Wr.as<float2>(), ksub, g, tabx.as<float2>(),
          ktab, (float)w00, 0);
    } else {
      dim3 grid((g.h + Q::B - 1) / Q::B, g.n1);
      k_xcorr_p2<T, L, 2><<<grid, Q::THREADS, p2_col_smem<T, L>(), s>>>(
          nullptr, G.as<C2<T>>(), Wr.as<C2<T>>(), ksub, g, tabx.as<C2<T>>(),
          ktab, (T)w00);
    }
  });
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::yinv(cudaStream_t s) {
  if (is_p2(g.n1)) {
    with_p2(g.n1, [&]<int L>() {
      using Q = P2<T, L>;
      if constexpr (std::is_same_v<T, float>) {
        using Y = PY<L>;
        dim3 grid((g.h + Y::B - 1) / Y::B, g.rs);
        k_yinv_pp<L><<<grid, Y::THREADS, Y::smem, s>>>(
            Wr.as<float2>(), Wry.as<float2>(), g, taby.as<float2>(),
            nyq_group<Y::B>(false));
      } else {
        dim3 grid((g.h + Q::B - 1) / Q::B, g.rs);
        k_yinv_p2<T, L><<<grid, Q::THREADS, p2_col_smem<T, L>(), s>>>(
            Wr.as<C2<T>>(), Wry.as<C2<T>>(), g, taby.as<C2<T>>());
      }
    });
    FC_LAUNCH_CHECK();
    return;
  }
  constexpr int B = Tile<T>::B;
  dim3 grid((g.h + B - 1) / B, g.rs);
  k_yinv<T><<<grid, threads_for(g.n1, B), smem(g.n1), s>>>(
      Wr.as<C2<T>>(), Wry.as<C2<T>>(), g, taby.as<C2<T>>());
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::zinv(double *rsub, const void *rtab_v, cudaStream_t s) {
  const T *rtab = static_cast<const T *>(rtab_v);
  if (is_p2(g.m)) {
    with_p2(g.m, [&]<int L>() {
      using Q = P2<T, L>;
      const int nrows = g.rs * g.rs;
      const unsigned blocks = (unsigned)((nrows + Q::B - 1) / Q::B);
      k_zinv_p2<T, L><<<blocks, Q::THREADS, p2_row_smem<T, L>(), s>>>(
          Wry.as<C2<T>>(), rsub, g, tabz.as<C2<T>>(), rtab);
    });
    FC_LAUNCH_CHECK();
    return;
  }
  constexpr int B = Tile<T>::B;
  const int nrows = g.rs * g.rs;
  const unsigned blocks = (unsigned)((nrows + B - 1) / B);
  k_zinv_rsub<T><<<blocks, threads_for(g.m, B), smem(g.m), s>>>(
      Wry.as<C2<T>>(), rsub, g, tabz.as<C2<T>>(), rtab);
  FC_LAUNCH_CHECK();
}

const void *FusedSurvey::r_table(int ell, int m, const double *raxis,
                                 const YlmParams &pr, cudaStream_t s) {
  const int key = ell * 16 + (m + ell);
  auto it = rtabs.find(key);
  if (it != rtabs.end()) return it->second.get();
  const size_t n = (size_t)g.rs * g.rs * g.rs;
  DeviceBuffer &b = rtabs[key];
  // FP64 for the FP64 form, FP32 for the FP32-mixed form (the product with
  // the transform and the accumulation stay FP64).
  if (fp64_) {
    b.resize(std::max<size_t>(n, 1) * sizeof(double));
    k_rtable<double><<<grid_for(n, 256), 256, 0, s>>>(b.as<double>(), g.rs, raxis, pr);
  } else {
    b.resize(std::max<size_t>(n, 1) * sizeof(float));
    k_rtable<float><<<grid_for(n, 256), 256, 0, s>>>(b.as<float>(), g.rs, raxis, pr);
  }
  FC_LAUNCH_CHECK();
  return b.get();
}

void FusedSurvey::prepare_tables(int maxell, double ncells, const double *raxis,
                                 const KAxes &ka, bool with_k, cudaStream_t s) {
  for (int ell = 0; ell <= maxell; ell += 2)
    for (int m = -ell; m <= ell; ++m) {
      r_table(ell, m, raxis, make_ylm_params(ell, m, 4.0 * M_PI / ncells), s);
      if (with_k) k_table(ell, m, ka, s);
    }
}

const void *FusedSurvey::k_table(int ell, int m, const KAxes &ka,
                                 cudaStream_t s) {
  const int key = ell * 16 + (m + ell);
  auto it = ktabs.find(key);
  if (it != ktabs.end()) return it->second.get();
  const size_t n = (size_t)g.ks0 * g.ks1 * g.ks2;
  DeviceBuffer &b = ktabs[key];
  const YlmParams pk = make_ylm_params(ell, m, 4.0 * M_PI);
  // FP64 weights for the FP64 form; the FP32 form keeps them in FP32 (a
  // relative rounding of 6e-8, far inside its precision).
  if (fp64_) {
    b.resize(std::max<size_t>(n, 1) * sizeof(double));
    k_ktable<double><<<grid_for(n, 256), 256, 0, s>>>(
        b.as<double>(), g.ks0, g.ks1, g.ks2, ka.kx, ka.ky, ka.kz, ka.wx, ka.wy,
        ka.wz, pk);
  } else {
    b.resize(std::max<size_t>(n, 1) * sizeof(float));
    k_ktable<float><<<grid_for(n, 256), 256, 0, s>>>(
        b.as<float>(), g.ks0, g.ks1, g.ks2, ka.kx, ka.ky, ka.kz, ka.wx, ka.wy,
        ka.wz, pk);
  }
  FC_LAUNCH_CHECK();
  return b.get();
}

void FusedSurvey::grid2(const void *rho_in, cudaStream_t s, const KAxes &ka) {
  (void)ka;
  YlmParams none = make_ylm_params(0, 0, 1.0);
  const double zero[3] = {0, 0, 0};
  if (fp64_) {
    zfwd<double>(rho_in, false, none, zero, s);
    yfwd<double>(s);
    xcorr<double>(false, nullptr, nullptr, s);
  } else {
    zfwd<float>(rho_in, false, none, zero, s);
    yfwd<float>(s);
    xcorr<float>(false, nullptr, nullptr, s);
  }
}

bool FusedSurvey::pairs() const { return !fp64_ && is_p2(g.m); }

void FusedSurvey::zfwd_pair(const void *rho_in, int ell_a, int m_a, int ell_b,
                            int m_b, const double xyz0[3], cudaStream_t s,
                            PhaseHook *hook) {
  FC_REQUIRE(pairs() && ell_a > 0 && ell_b > 0, FC_ERR_STATE,
             "paired z pass needs two weighted FP32 terms");
  const YlmParams pa = make_ylm_params(ell_a, m_a, 1.0);
  const YlmParams pb = make_ylm_params(ell_b, m_b, 1.0);
  const int64_t nrows = (int64_t)g.n0 * g.n1;
  k_rowpoly<<<grid_for(nrows, 256), 256, 0, s>>>(rowtab.as<float4>(), nrows,
                                                 g.n1, pa, xyz0[0], xyz0[1]);
  FC_LAUNCH_CHECK();
  k_rowpoly<<<grid_for(nrows, 256), 256, 0, s>>>(rowtab2.as<float4>(), nrows,
                                                 g.n1, pb, xyz0[0], xyz0[1]);
  FC_LAUNCH_CHECK();
  if (hook) hook->begin("zfwd2");
  with_p2(g.m, [&]<int L>() {
    using PQ = PP<L>;
    const unsigned blocks = (unsigned)((nrows + PQ::PB - 1) / PQ::PB);
    k_zfwd_pp2<L><<<blocks, PQ::THREADS, p2_row_smem<float, L>(), s>>>(
        static_cast<const float *>(rho_in), W.as<float2>(), W2.as<float2>(), g,
        pa, pb, xyz0[2], tabz.as<float2>(), rowtab.as<float4>(),
        rowtab2.as<float4>());
  });
  FC_LAUNCH_CHECK();
  if (hook) hook->end();
}

int FusedSurvey::term(const void *rho_in, int ell, int m, const double xyz0[3],
                       double ncells, double *ksub, double *rsub,
                       const double *raxis, const KAxes &ka, cudaStream_t s,
                       PhaseHook *hook, bool g_of_input, bool z_done) {
  const YlmParams pw = make_ylm_params(ell, m, 1.0);
  const YlmParams pr = make_ylm_params(ell, m, 4.0 * M_PI / ncells);
  const void *ktab = ksub ? k_table(ell, m, ka, s) : nullptr;
  const void *rtab = r_table(ell, m, raxis, pr, s);
  const bool from_g = ell == 0 && g_of_input && is_p2(g.n0);
  auto run = [&](auto tag) {
    using T = decltype(tag);
    if (from_g) {
      // The weight is the constant pw.value0, so the term's transform is
      // value0 * G (see k_xcorr_p2, MODE 2).
      if (hook) hook->begin("xcorr00");
      xcorr00<T>(ksub, ktab, pw.value0, s);
      if (hook) hook->end();
    } else {
      if (!z_done) {
        if (hook) hook->begin("zfwd");
        zfwd<T>(rho_in, true, pw, xyz0, s);
        if (hook) hook->end();
      }
      if (hook) hook->begin("yfwd");
      yfwd<T>(s);
      if (hook) hook->end();
      if (hook) hook->begin("xcorr");
      xcorr<T>(true, ksub, ktab, s);
      if (hook) hook->end();
    }
    if (hook) hook->begin("yinv");
    yinv<T>(s);
    if (hook) hook->end();
    if (hook) hook->begin("zinv");
    zinv<T>(rsub, rtab, s);
    if (hook) hook->end();
  };
  if (fp64_)
    run(double());
  else
    run(float());
  return from_g ? 1 : 2;
}

}  // namespace fc
