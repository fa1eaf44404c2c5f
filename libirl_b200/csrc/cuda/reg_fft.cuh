// reg_fft.cuh -- DFTs held in registers, for the one-CTA-per-plane form of
// the Fourier-domain DRF convolution (k_drf_fft.cu).
//
// RDft<N, INV> transforms N complex values in a thread's registers, in
// natural order in and out.  N = 2, 3, 4, 5, 7, 8 use the small DFTs of
// fft_core.cuh; a composite N = A * B runs as A-point DFTs, twiddles and
// B-point DFTs, all with compile-time indices, so the values never leave
// registers.  Twiddles inside a composite DFT are compile-time constants:
// cos and sin of 2 pi m / N come from a reduction of the fraction m / N to
// the first octant and Taylor series in double, evaluated by the compiler.
// INV = false is the forward transform (exp(-i ...)), INV = true the
// unscaled inverse.
//
// A line of length L = N1 * N2 is then transformed by N2 threads holding
// x[n2 + N2 n1] (n1 < N1), an N1-point register DFT, the twiddle
// W_L^(n2 k1), one exchange through shared memory and an N2-point register
// DFT in the N1 threads holding Y[n2][k1] (n2 < N2), which leaves
// X[k1 + N1 k2] in thread k1.
#pragma once

#include "fft_core.cuh"

namespace irlcu {

// ------------------------------------------------- compile-time roots

constexpr double kPiD = 3.14159265358979323846264338327950288;

// sin x and cos x for |x| <= pi / 4 (13 terms: error far below 1e-20)
constexpr double ce_sin_small(double x) {
  const double x2 = x * x;
  double t = x, s = x;
  for (int k = 1; k <= 12; ++k) {
    t *= -x2 / (double)((2 * k) * (2 * k + 1));
    s += t;
  }
  return s;
}
constexpr double ce_cos_small(double x) {
  const double x2 = x * x;
  double t = 1.0, s = 1.0;
  for (int k = 1; k <= 12; ++k) {
    t *= -x2 / (double)((2 * k - 1) * (2 * k));
    s += t;
  }
  return s;
}

struct CeRoot {
  double c, s;
};

// cos and sin of 2 pi m / N: the angle pi a / d (a = 2m mod 2N, d = N) is
// folded into [0, pi/4] with exact integer arithmetic
constexpr CeRoot ce_root(int m, int N) {
  long long a = (2LL * m) % (2LL * N), d = N;
  if (a < 0) a += 2LL * N;
  double sc = 1.0, ss = 1.0;
  if (a > d) {  // 2 pi - theta
    a = 2 * d - a;
    ss = -1.0;
  }
  if (2 * a > d) {  // pi - theta
    a = d - a;
    sc = -1.0;
  }
  bool swap = false;
  if (4 * a > d) {  // pi/2 - theta
    a = d - 2 * a;
    d = 2 * d;
    swap = true;
  }
  const double x = kPiD * (double)a / (double)d;
  double c = ce_cos_small(x), s = ce_sin_small(x);
  if (swap) {
    const double t = c;
    c = s;
    s = t;
  }
  return CeRoot{sc * c, ss * s};
}

template <int N, int M>
struct Root {
  static constexpr float c = (float)ce_root(M, N).c;
  static constexpr float s = (float)ce_root(M, N).s;
};

// x * W_N^M (forward, W = exp(-2 pi i / N)) or x * conj(W_N^M) (inverse)
template <int N, int M, bool INV>
__device__ __forceinline__ float2 rot(float2 x) {
  constexpr int m = ((M % N) + N) % N;
  if constexpr (m == 0) {
    return x;
  } else if constexpr (2 * m == N) {
    return make_float2(-x.x, -x.y);
  } else if constexpr (4 * m == N) {  // W = -i (forward), +i (inverse)
    return INV ? make_float2(-x.y, x.x) : make_float2(x.y, -x.x);
  } else if constexpr (4 * m == 3 * N) {  // W = +i (forward), -i (inverse)
    return INV ? make_float2(x.y, -x.x) : make_float2(-x.y, x.x);
  } else {
    constexpr float c = Root<N, m>::c, s = Root<N, m>::s;
    return INV ? make_float2(x.x * c - x.y * s, x.y * c + x.x * s)
               : make_float2(x.x * c + x.y * s, x.y * c - x.x * s);
  }
}

// x * w (forward) or x * conj(w) (inverse) for a runtime twiddle w
template <bool INV>
__device__ __forceinline__ float2 twiddle(float2 x, float2 w) {
  return INV ? make_float2(x.x * w.x + x.y * w.y, x.y * w.x - x.x * w.y)
             : make_float2(x.x * w.x - x.y * w.y, x.x * w.y + x.y * w.x);
}

// ------------------------------------------------- register DFTs

__host__ __device__ constexpr bool rdft_base(int N) {
  return N == 2 || N == 3 || N == 4 || N == 5 || N == 7 || N == 8;
}
// first factor A of a composite N = A * B
__host__ __device__ constexpr int rdft_split(int N) {
  return (N % 8 == 0 && N > 8) ? 8
         : (N % 4 == 0 && N > 4) ? 4
         : N % 2 == 0 ? 2
         : N % 5 == 0 ? 5
         : N % 3 == 0 ? 3
                      : 7;
}

// y[n2 * A + k1] *= W_N^(n2 k1), I = n2 * A + k1
template <int N, int A, bool INV, int I>
struct TwApply {
  static __device__ __forceinline__ void run(float2 *y) {
    if constexpr (I < N) {
      y[I] = rot<N, (I / A) * (I % A), INV>(y[I]);
      TwApply<N, A, INV, I + 1>::run(y);
    }
  }
};

template <int N, bool INV>
struct RDft {
  static __device__ __forceinline__ void run(float2 *v) {
    if constexpr (rdft_base(N)) {
      dft_r<N>(v, INV ? -1.f : 1.f);
    } else {
      // n = n2 + B n1, k = k1 + A k2
      constexpr int A = rdft_split(N), B = N / A;
      float2 y[N];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) {
        float2 t[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) t[n1] = v[n2 + B * n1];
        RDft<A, INV>::run(t);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) y[n2 * A + k1] = t[k1];
      }
      TwApply<N, A, INV, 0>::run(y);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) {
        float2 u[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) u[n2] = y[n2 * A + k1];
        RDft<B, INV>::run(u);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = u[k2];
      }
    }
  }
};

// split of a line length L = N1 * N2 for the two-level line transforms
template <int L>
struct LineSplit {
  static constexpr int N1 = (L % 16 == 0 && L >= 32) ? 16 : 8;
  static constexpr int N2 = L / N1;
  static_assert(N1 * N2 == L && N2 >= 2, "line length must be a multiple of 8 or 16");
};

}  // namespace irlcu
