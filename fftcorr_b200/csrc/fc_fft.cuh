// fc_fft.cuh -- shared-memory Stockham FFT engine for the fused correlator
// passes.
//
// A CTA transforms B columns of length L held in shared memory as
// buf[i * BP + b] (row i of column b, BP = B + 1 to spread banks).  The
// transform is an iterative mixed-radix Stockham autosort (radices 8, 4, 2,
// 3, 5, 7) between two shared buffers: each pass reads a butterfly's R
// inputs, applies the twiddles and the radix-R DFT in registers and writes
// the outputs to their Stockham positions in the other buffer.  Twiddles come from a table of e^{-2 pi i m / Lt} (Lt a
// multiple of L) computed in FP64 on the host.  Forward is sign -1 and the
// inverse is unnormalised, as in FFTW and cuFFT.
#pragma once

#include <cuda_runtime.h>

namespace fc {

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

// Arithmetic on float2 as a vector of two lanes (used by CPair below), in
// the packed two-lane FP32 instructions of sm_100 (one issue for both
// lanes; each lane rounds as the scalar operation does).
__device__ __forceinline__ float2 f2splat(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) {
  return __fadd2_rn(a, b);
}
// Packed subtract (PTX sub.rn.f32x2; there is no intrinsic for it): one
// rounding of a - b per lane, with no register pair of -1 constants.
__device__ __forceinline__ float2 operator-(float2 a, float2 b) {
  unsigned long long ra, rb, rd;
  asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(rd));
  return r;
}
__device__ __forceinline__ float2 operator-(float2 a) {
  return make_float2(-a.x, -a.y);
}
__device__ __forceinline__ float2 operator*(float2 a, float s) {
  return __fmul2_rn(a, f2splat(s));
}
__device__ __forceinline__ float2 operator*(float s, float2 a) {
  return __fmul2_rn(f2splat(s), a);
}
__device__ __forceinline__ float2 operator*(float2 a, float2 b) {
  return __fmul2_rn(a, b);  // lane by lane
}

// Two complex numbers of two independent transforms (columns or rows)
// carried through one FFT together: x holds both real parts, y both
// imaginary parts.  Twiddles are shared, shared-memory exchanges move 16
// bytes at a time.
struct __align__(16) CPair {
  float2 x, y;
};
__device__ __forceinline__ CPair cpack(float2 a, float2 b) {
  CPair r;
  r.x = make_float2(a.x, b.x);
  r.y = make_float2(a.y, b.y);
  return r;
}
__device__ __forceinline__ float2 clane0(const CPair &v) {
  return make_float2(v.x.x, v.y.x);
}
__device__ __forceinline__ float2 clane1(const CPair &v) {
  return make_float2(v.x.y, v.y.y);
}

// The same pair with one-lane FP32 instructions (for kernels where the packed
// forms measure slower).
struct SF2 {
  float x, y;
};
__device__ __forceinline__ SF2 operator+(SF2 a, SF2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ SF2 operator-(SF2 a, SF2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ SF2 operator-(SF2 a) { return {-a.x, -a.y}; }
__device__ __forceinline__ SF2 operator*(SF2 a, float s) { return {a.x * s, a.y * s}; }
__device__ __forceinline__ SF2 operator*(float s, SF2 a) { return {s * a.x, s * a.y}; }
struct __align__(16) CPairS {
  SF2 x, y;
};
__device__ __forceinline__ CPairS cpack_s(float2 a, float2 b) {
  CPairS r;
  r.x = {a.x, b.x};
  r.y = {a.y, b.y};
  return r;
}
__device__ __forceinline__ float2 clane0(const CPairS &v) {
  return make_float2(v.x.x, v.y.x);
}
__device__ __forceinline__ float2 clane1(const CPairS &v) {
  return make_float2(v.x.y, v.y.y);
}

// Scalar type of a complex (or complex-pair) type.
template <typename C>
struct Real;
template <>
struct Real<float2> {
  using type = float;
};
template <>
struct Real<double2> {
  using type = double;
};
template <>
struct Real<CPair> {
  using type = float;
};
template <>
struct Real<CPairS> {
  using type = float;
};

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
  C r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
  C r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a * conj(b)
template <typename C>
__device__ __forceinline__ C cmulc(C a, C b) {
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}
template <typename C>
__device__ __forceinline__ C cconj(C a) {
  C r;
  r.x = a.x;
  r.y = -a.y;
  return r;
}
// A pair times one shared complex twiddle.
__device__ __forceinline__ CPair cmul(CPair a, float2 w) {
  CPair r;
  r.x = __ffma2_rn(a.y, f2splat(-w.y), __fmul2_rn(a.x, f2splat(w.x)));
  r.y = __ffma2_rn(a.y, f2splat(w.x), __fmul2_rn(a.x, f2splat(w.y)));
  return r;
}
__device__ __forceinline__ CPairS cmul(CPairS a, float2 w) {
  CPairS r;
  r.x = a.x * w.x - a.y * w.y;
  r.y = a.x * w.y + a.y * w.x;
  return r;
}
// (sign * i) * a
template <typename C>
__device__ __forceinline__ C cmuli(C a, int sign) {
  C r;
  if (sign > 0) {
    r.x = -a.y;
    r.y = a.x;
  } else {
    r.x = a.y;
    r.y = -a.x;
  }
  return r;
}
template <typename C, typename T>
__device__ __forceinline__ C cscale(C a, T s) {
  C r;
  r.x = a.x * s;
  r.y = a.y * s;
  return r;
}

// Radix-R DFT in registers: out[q] = sum_u v[u] * e^{sign 2 pi i u q / R}.
template <int R, typename C>
struct Dft;

template <typename C>
struct Dft<2, C> {
  __device__ static void run(C *v, int) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <typename C>
struct Dft<4, C> {
  __device__ static void run(C *v, int sign) {
    const C a0 = cadd(v[0], v[2]);
    const C a1 = csub(v[0], v[2]);
    const C a2 = cadd(v[1], v[3]);
    const C d = cmuli(csub(v[1], v[3]), sign);
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, d);
    v[3] = csub(a1, d);
  }
};

template <typename C>
struct Dft<8, C> {
  // Radix 2 across stride 4, then two radix-4 DFTs (even and odd outputs).
  __device__ static void run(C *v, int sign) {
    using T = typename Real<C>::type;
    const T h = (T)0.70710678118654752440;
    const T sg = (T)sign;
    C a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = cadd(v[u], v[u + 4]);
      b[u] = csub(v[u], v[u + 4]);
    }
    // b[u] *= e^{sign 2 pi i u / 8}
    {
      C t = b[1];
      b[1].x = h * (t.x - sg * t.y);
      b[1].y = h * (t.y + sg * t.x);
      b[2] = cmuli(b[2], sign);
      t = b[3];
      b[3].x = h * (-t.x - sg * t.y);
      b[3].y = h * (-t.y + sg * t.x);
    }
    Dft<4, C>::run(a, sign);
    Dft<4, C>::run(b, sign);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      v[2 * p] = a[p];
      v[2 * p + 1] = b[p];
    }
  }
};

template <typename C>
struct Dft<3, C> {
  __device__ static void run(C *v, int sign) {
    using T = decltype(v[0].x);
    const T s3 = (T)0.86602540378443864676 * sign;
    const C t = cadd(v[1], v[2]);
    const C d = csub(v[1], v[2]);
    C m;
    m.x = v[0].x - (T)0.5 * t.x;
    m.y = v[0].y - (T)0.5 * t.y;
    C sd;
    sd.x = -s3 * d.y;
    sd.y = s3 * d.x;
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, sd);
    v[2] = csub(m, sd);
  }
};

// Generic odd prime radix (5, 7): O(R^2) complex products with the R-th
// roots of unity evaluated once per butterfly by sincospi (correctly
// rounded to within an ulp); these radices are rare in practice.
template <int R, typename C>
struct DftGeneric {
  __device__ static void run(C *v, int sign) {
    using T = decltype(v[0].x);
    C w[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
      double s, c;
      sincospi(2.0 * m / R, &s, &c);
      w[m].x = (T)c;
      w[m].y = (T)(sign * s);
    }
    C in[R];
#pragma unroll
    for (int u = 0; u < R; ++u) in[u] = v[u];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      C acc = in[0];
#pragma unroll
      for (int u = 1; u < R; ++u) acc = cadd(acc, cmul(in[u], w[(u * q) % R]));
      v[q] = acc;
    }
  }
};
template <typename C>
struct Dft<5, C> : DftGeneric<5, C> {};
template <typename C>
struct Dft<7, C> : DftGeneric<7, C> {};

// Plan of one transform length: up to 12 passes.
struct FftPlan {
  int L;          // transform length
  int npass;
  int radix[12];
  int ns[12];     // product of the radices before each pass
  int nsmask[12]; // ns - 1 when ns is a power of two, else -1
  int tab_scale;  // root-table order / L
};

// One Stockham pass of radix R: reads the B columns from src, writes the
// result to dst (both [L][BP] in shared memory).  Each thread handles one
// butterfly at a time, so only R complex values live in registers.  B is a
// compile-time constant so the butterfly decomposition is shifts and masks.
template <int R, int B, typename C>
__device__ __forceinline__ void stockham_pass(const C *src, C *dst, int L,
                                              int Ns, int nsmask,
                                              const C *__restrict__ tab,
                                              int tab_scale, int sign) {
  constexpr int BP = B + 1;
  const int LR = L / R;
  const int nbf = LR * B;
  const int step = (L / (Ns * R)) * tab_scale;
  for (int bf = threadIdx.x; bf < nbf; bf += blockDim.x) {
    const int j = bf / B;
    const int b = bf - j * B;
    const int k = nsmask >= 0 ? (j & nsmask) : (j % Ns);
    C v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = src[(j + q * LR) * BP + b];
    if (Ns > 1) {
      // q * k * step < L * tab_scale: no reduction needed.
      const int ks = k * step;
#pragma unroll
      for (int q = 1; q < R; ++q) {
        C w = __ldg(&tab[q * ks]);
        if (sign > 0) w.y = -w.y;
        v[q] = cmul(v[q], w);
      }
    }
    Dft<R, C>::run(v, sign);
    const int o = ((j - k) * R + k) * BP + b;
#pragma unroll
    for (int q = 0; q < R; ++q) dst[o + q * Ns * BP] = v[q];
  }
  __syncthreads();
}

// Transforms the B columns in a (the caller has synchronised after filling
// it), ping-ponging with b; returns the buffer that holds the result
// (synchronised).
template <int B, typename C>
__device__ C *fft_columns(C *a, C *b, const FftPlan &p,
                          const C *__restrict__ tab, int sign) {
  C *src = a, *dst = b;
  for (int s = 0; s < p.npass; ++s) {
    const int R = p.radix[s];
    const int Ns = p.ns[s];
    const int m = p.nsmask[s];
    switch (R) {
      case 8:
        stockham_pass<8, B>(src, dst, p.L, Ns, m, tab, p.tab_scale, sign);
        break;
      case 4:
        stockham_pass<4, B>(src, dst, p.L, Ns, m, tab, p.tab_scale, sign);
        break;
      case 2:
        stockham_pass<2, B>(src, dst, p.L, Ns, m, tab, p.tab_scale, sign);
        break;
      case 3:
        stockham_pass<3, B>(src, dst, p.L, Ns, m, tab, p.tab_scale, sign);
        break;
      case 5:
        stockham_pass<5, B>(src, dst, p.L, Ns, m, tab, p.tab_scale, sign);
        break;
      default:
        stockham_pass<7, B>(src, dst, p.L, Ns, m, tab, p.tab_scale, sign);
        break;
    }
    C *t = src;
    src = dst;
    dst = t;
  }
  return src;
}

}  // namespace fc

namespace fc {

// ---------------------------------------------------------------------------
// Register-resident FFT for power-of-two lengths 64 <= L <= 4096.
//
// A column of length L is owned by TPC = L/8 threads; thread t holds the
// eight elements v[u] = x[t + TPC*u].  That is exactly the input of the
// Stockham radix-8 butterfly j = t, so every pass is a DFT8 in registers and
// the passes exchange data through shared memory (write, barrier, read,
// barrier).  A radix-2 or radix-4 pass comes first when L is not a power of
// 8.  After the last radix-8 pass (Ns = L/8, k = t) thread t holds the
// natural-order outputs x[t + TPC*q], so the result is stored straight from
// registers.  Twiddles of a pass are w^q, w = e^{sign 2 pi i k/(8 Ns)}: w,
// w^2 and w^4 come from the order-L root table and the rest are products.
// ---------------------------------------------------------------------------

template <typename Tw>
__device__ __forceinline__ Tw tw_load(const Tw *__restrict__ tab, int idx,
                                      int sign) {
  Tw w = __ldg(&tab[idx]);
  if (sign > 0) w.y = -w.y;
  return w;
}

// One radix-8 pass with Ns > 1 for butterfly j = t on registers v.
template <typename C, typename Tw>
__device__ __forceinline__ void r8_twiddle(C *v, int k, int step,
                                           const Tw *__restrict__ tab, int sign) {
  const Tw w1 = tw_load(tab, k * step, sign);
  const Tw w2 = tw_load(tab, 2 * k * step, sign);
  const Tw w4 = tw_load(tab, 4 * k * step, sign);
  const Tw w3 = cmul(w1, w2);
  v[1] = cmul(v[1], w1);
  v[2] = cmul(v[2], w2);
  v[3] = cmul(v[3], w3);
  v[4] = cmul(v[4], w4);
  v[5] = cmul(v[5], cmul(w1, w4));
  v[6] = cmul(v[6], cmul(w2, w4));
  v[7] = cmul(v[7], cmul(w3, w4));
}

// Outputs 0 and 7 of Dft<8> only (into v[0] and v[7]), by the same
// operations, for transforms whose later use reads only the first and the
// last TPC rows.
template <typename C>
__device__ __forceinline__ void dft8_edges(C *v, int sign) {
  using T = typename Real<C>::type;
  const T h = (T)0.70710678118654752440;
  const T sg = (T)sign;
  C a[4], b[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    a[u] = cadd(v[u], v[u + 4]);
    b[u] = csub(v[u], v[u + 4]);
  }
  C t = b[1];
  b[1].x = h * (t.x - sg * t.y);
  b[1].y = h * (t.y + sg * t.x);
  b[2] = cmuli(b[2], sign);
  t = b[3];
  b[3].x = h * (-t.x - sg * t.y);
  b[3].y = h * (-t.y + sg * t.x);
  v[0] = cadd(cadd(a[0], a[2]), cadd(a[1], a[3]));
  v[7] = csub(csub(b[0], b[2]), cmuli(csub(b[1], b[3]), sign));
}

// Transform of one column held in registers (layout above).  ex(i) gives the
// shared-memory slot of row i of this thread's column; all TPC threads of
// every column in the CTA must call this together.
// rd(u) must return ex(t + TPC * u): kernels pass one that adds constant
// offsets to a per-thread base instead of recomputing the layout's index.
// before_last() runs once the last exchange is complete, before the last
// pass: from there on the transform no longer touches shared memory, so a
// kernel may start asynchronous copies into it.  With edges_only the last
// pass computes only outputs t and t + 7 TPC (v[0] and v[7]).
struct NoHook {
  __device__ void operator()() const {}
};
template <int L, typename C, typename Tw, typename Ex, typename Rd,
          typename Hook = NoHook>
__device__ __forceinline__ void reg_fft(C *v, int t, Ex ex, Rd rd,
                                        const Tw *__restrict__ tab, int sign,
                                        int tab_scale = 1, Hook before_last = {},
                                        bool edges_only = false) {
  constexpr int TPC = L / 8;
  // Number of radix-8 passes and the leading radix (1, 2 or 4).
  constexpr int LOG = __builtin_ctz(L);
  constexpr int P8 = LOG / 3;
  constexpr int R0 = 1 << (LOG - 3 * P8);
  int Ns = 1;
  if constexpr (R0 == 2) {
    // Four radix-2 butterflies j = t + TPC c, inputs x[j + (L/2) q] = v[c + 4q].
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      C a = v[c], b = v[c + 4];
      v[c] = cadd(a, b);
      v[c + 4] = csub(a, b);
    }
    // Outputs y[2j + q]: write, then read x[t + TPC u].
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int j = t + TPC * c;
      *ex(2 * j) = v[c];
      *ex(2 * j + 1) = v[c + 4];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = *rd(u);
    __syncthreads();
    Ns = 2;
  } else if constexpr (R0 == 4) {
    // Two radix-4 butterflies j = t + TPC c, inputs x[j + (L/4) q] = v[c + 2q].
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      C w[4] = {v[c], v[c + 2], v[c + 4], v[c + 6]};
      Dft<4, C>::run(w, sign);
      v[c] = w[0];
      v[c + 2] = w[1];
      v[c + 4] = w[2];
      v[c + 6] = w[3];
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int j = t + TPC * c;
#pragma unroll
      for (int q = 0; q < 4; ++q) *ex(4 * j + q) = v[c + 2 * q];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = *rd(u);
    __syncthreads();
    Ns = 4;
  }
#pragma unroll
  for (int p = 0; p < P8; ++p) {
    if (p + 1 == P8) before_last();
    const int k = t & (Ns - 1);
    if (Ns > 1) r8_twiddle(v, k, (L / (8 * Ns)) * tab_scale, tab, sign);
    if (p + 1 == P8 && edges_only)
      dft8_edges(v, sign);
    else
      Dft<8, C>::run(v, sign);
    if (p + 1 < P8) {
      const int o = (t - k) * 8 + k;
#pragma unroll
      for (int q = 0; q < 8; ++q) *ex(o + q * Ns) = v[q];
      __syncthreads();
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = *rd(u);
      __syncthreads();
    }
    Ns *= 8;
  }
}

template <int L, typename C, typename Tw, typename Ex>
__device__ __forceinline__ void reg_fft(C *v, int t, Ex ex,
                                        const Tw *__restrict__ tab, int sign,
                                        int tab_scale = 1) {
  reg_fft<L>(v, t, ex, [&](int u) { return ex(t + (L / 8) * u); }, tab, sign,
             tab_scale);
}

}  // namespace fc
