// fft_core.cuh -- batched complex line DFTs in shared memory, shared by the
// ESSE scatter model (k_esse.cu) and the FFT form of the DRF convolution
// (k_drf_fft.cu).
//
// A transform of length L runs as a sequence of Stockham autosort passes
// of radix R in {8, 4, 2, 5, 3, 7} (largest power-of-two radix first), so L
// may be any product of 2, 3, 5 and 7.  Each pass reads one buffer and
// writes the other; twiddles tw[m] = exp(-2 pi i m / L) come from a table
// computed in double on the host.  s = +1 is the forward transform
// (exp(-i ...)), s = -1 the unscaled inverse.
#pragma once

#include <cuda_runtime.h>

namespace irlcu {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float f) { return make_float2(a.x * f, a.y * f); }
// multiply by -i*s (s = +1 forward, -1 inverse): (x, y) -> (s*y, -s*x)
__device__ __forceinline__ float2 mul_mis(float2 a, float s) { return make_float2(s * a.y, -s * a.x); }

template <int R>
__device__ __forceinline__ void dft_r(float2 *v, float s);  // in place, R points

template <>
__device__ __forceinline__ void dft_r<2>(float2 *v, float) {
  const float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <>
__device__ __forceinline__ void dft_r<4>(float2 *v, float s) {
  const float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
  const float2 c = cadd(v[1], v[3]), d = mul_mis(csub(v[1], v[3]), s);
  v[0] = cadd(a, c);
  v[2] = csub(a, c);
  v[1] = cadd(b, d);
  v[3] = csub(b, d);
}

template <>
__device__ __forceinline__ void dft_r<8>(float2 *v, float s) {
  // two 4-point DFTs on even and odd samples, then the radix-2 combine
  float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  dft_r<4>(e, s);
  dft_r<4>(o, s);
  const float h = 0.70710678118654752440f;
  // W8^k = exp(-i*s*pi*k/4)
  const float2 w1 = make_float2(h, -s * h), w3 = make_float2(-h, -s * h);
  const float2 o1 = cmul(o[1], w1), o2 = mul_mis(o[2], s), o3 = cmul(o[3], w3);
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}

// cos(2 pi k / R), sin(2 pi k / R) for the odd radices
template <int R>
__device__ __forceinline__ float root_cos(int k);
template <int R>
__device__ __forceinline__ float root_sin(int k);
template <>
__device__ __forceinline__ float root_cos<3>(int) { return -0.5f; }
template <>
__device__ __forceinline__ float root_sin<3>(int) { return 0.86602540378443864676f; }
template <>
__device__ __forceinline__ float root_cos<5>(int k) {
  return k == 1 ? 0.30901699437494742410f : -0.80901699437494742410f;
}
template <>
__device__ __forceinline__ float root_sin<5>(int k) {
  return k == 1 ? 0.95105651629515357212f : 0.58778525229247312917f;
}
template <>
__device__ __forceinline__ float root_cos<7>(int k) {
  return k == 1 ? 0.62348980185873353053f : (k == 2 ? -0.22252093395631440429f : -0.90096886790241912624f);
}
template <>
__device__ __forceinline__ float root_sin<7>(int k) {
  return k == 1 ? 0.78183148246802980871f : (k == 2 ? 0.97492791218182360702f : 0.43388373911755812048f);
}

// odd R: out[m] = v0 + sum_j (v_j + v_{R-j}) cos(2 pi j m / R)
//                    - i s sum_j (v_j - v_{R-j}) sin(2 pi j m / R),
// and out[R-m] with the sine part negated (j, m = 1 .. (R-1)/2)
template <int R>
__device__ __forceinline__ void dft_odd(float2 *v, float s) {
  constexpr int Q = (R - 1) / 2;
  float2 a[Q + 1], b[Q + 1];
  float2 sum = v[0];
#pragma unroll
  for (int j = 1; j <= Q; ++j) {
    a[j] = cadd(v[j], v[R - j]);
    b[j] = csub(v[j], v[R - j]);
    sum = cadd(sum, a[j]);
  }
  float2 out[R];
  out[0] = sum;
#pragma unroll
  for (int m = 1; m <= Q; ++m) {
    float2 A = v[0], B = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 1; j <= Q; ++j) {
      int k = (j * m) % R;                  // angle index in [1, R)
      const bool neg = k > Q;               // sin(2 pi (R-k) / R) = -sin(2 pi k / R)
      k = neg ? R - k : k;
      const float c = root_cos<R>(k), sn = neg ? -root_sin<R>(k) : root_sin<R>(k);
      A = make_float2(A.x + c * a[j].x, A.y + c * a[j].y);
      B = make_float2(B.x + sn * b[j].x, B.y + sn * b[j].y);
    }
    const float2 iB = mul_mis(B, s);
    out[m] = cadd(A, iB);
    out[R - m] = csub(A, iB);
  }
#pragma unroll
  for (int m = 0; m < R; ++m) v[m] = out[m];
}
template <>
__device__ __forceinline__ void dft_r<3>(float2 *v, float s) { dft_odd<3>(v, s); }
template <>
__device__ __forceinline__ void dft_r<5>(float2 *v, float s) { dft_odd<5>(v, s); }
template <>
__device__ __forceinline__ void dft_r<7>(float2 *v, float s) { dft_odd<7>(v, s); }

// one Stockham pass of radix R over W lines of length L held in shared
// memory (element (w, i) at base[w*lstride + i]); NS, the length of the
// sub-transforms already done, is a compile-time constant so that every
// index division is by a constant
template <int L, int R, int NS>
__device__ __forceinline__ void stockham_pass(const float2 *in, float2 *out, int W, int lstride, const float2 *tw,
                                              float s) {
  constexpr int J = L / R;
  constexpr int STEP = L / (NS * R);  // twiddle index stride; r*k*STEP < L
  const int jobs = W * J;
  for (int q = threadIdx.x; q < jobs; q += blockDim.x) {
    const int w = q / J, j = q - w * J;
    const float2 *src = in + w * lstride;
    float2 v[R];
    const int k = j % NS;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 x = src[j + r * J];
      if (r > 0 && k > 0) {
        float2 t = tw[r * k * STEP];
        t.y *= s;  // conjugate for the inverse
        x = cmul(x, t);
      }
      v[r] = x;
    }
    dft_r<R>(v, s);
    float2 *dst = out + w * lstride;
    const int idxD = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[idxD + r * NS] = v[r];
  }
}

// radix of the next pass when rem = L / NS points remain: the largest
// power-of-two radix first, then 5, 3, 7
__host__ __device__ constexpr int next_radix(int rem) {
  return rem % 8 == 0 ? 8 : rem % 4 == 0 ? 4 : rem % 2 == 0 ? 2 : rem % 5 == 0 ? 5 : rem % 3 == 0 ? 3 : 7;
}

template <int L, int NS>
struct FftPlan {
  static __device__ __forceinline__ void run(float2 *&in, float2 *&out, int W, int lstride, const float2 *tw,
                                             float s) {
    if constexpr (NS < L) {
      constexpr int R = next_radix(L / NS);
      stockham_pass<L, R, NS>(in, out, W, lstride, tw, s);
      __syncthreads();
      float2 *t = in;
      in = out;
      out = t;
      FftPlan<L, NS * R>::run(in, out, W, lstride, tw, s);
    }
  }
};

// full transform of W lines; returns the buffer holding the result (a or b).
// Ends with a barrier.
template <int L>
__device__ float2 *fft_lines(float2 *a, float2 *b, int W, int lstride, const float2 *tw, float s) {
  float2 *in = a, *out = b;
  FftPlan<L, 1>::run(in, out, W, lstride, tw, s);
  return in;
}

// host: lengths the line transforms accept
inline bool fft_len_ok(int L) {
  if (L < 2) return false;
  int r = L;
  for (int p : {2, 3, 5, 7})
    while (r % p == 0) r /= p;
  return r == 1;
}

// host: twiddle table exp(-2 pi i m / L), m < L, in device memory
int upload_twiddle_table(cudaStream_t st, float2 **d, int L);

}  // namespace irlcu
