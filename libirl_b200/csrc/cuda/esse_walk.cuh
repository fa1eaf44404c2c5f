// esse_walk.cuh -- ExpandByFac's expansion and recursive smoothing along
// one line (krnlprj3d.c:595-673), shared by the ESSE kernels of k_esse.cu
// and their host test.
//
// The expansion by c replicates each coarse value (scaled by 1/c^3) over c
// fine entries along every axis.  coarse_walk runs the in-place smoothing
// along one line whose nc coarse entries stand for nf = c nc fine ones,
// reading the coarse values (each once, WALK_PF ahead) and writing the nf
// smoothed fine values.  The in-place walk only ever reads entries it has
// not yet overwritten, so its inputs are the expanded values themselves.
#pragma once

namespace irlcu {

// x / D for the odd window lengths D = 2h+1 of the smoothing and for odd
// collapse factors: q0 = x * RN(1/D), then one correction with the exact
// residual r = x - q0*D (Markstein, IBM J. Res. Dev. 34(1), 1990).  For
// D = 3, 5, 7 this equals the correctly rounded x / D for every finite x
// except -0 (checked over all float inputs; tests/test_const_division.py
// repeats it over the binades where under- and overflow could matter).
// The sums divided here start from +0, so they are never -0.
template <int D>
__device__ __forceinline__ float div_const(float x) {
  if constexpr (D == 1) {
    return x;
  } else if constexpr (D == 3 || D == 5 || D == 7) {
    const float y = __int_as_float(D == 3 ? 0x3eaaaaab : (D == 5 ? 0x3e4ccccd : 0x3e124925));
    const float q0 = __fmul_rn(x, y);
    const float r = __fmaf_rn(-q0, (float)D, x);
    return __fmaf_rn(r, y, q0);
  } else if constexpr ((D & (D - 1)) == 0) {
    return __fmul_rn(x, 1.0f / (float)D);  // exact for powers of two
  } else {
    return __fdiv_rn(x, (float)D);
  }
}

// ExpandByFac's smoothing (krnlprj3d.c:636-670) walks each line once in
// increasing order and overwrites it in place, so every output is
//   out[k] = (out[k-h] + .. + out[k-1] + in[k] + .. + in[k+h]) / (2h+1)
// summed left to right from 0, for h <= k < len-h (other entries keep
// their input value), h = c/2.  The line walkers below keep the last h
// outputs and the next h+1 inputs in registers.
template <int H>
struct LineSmoother {
  float outp[H > 0 ? H : 1];   // out[k-H..k-1]
  float in[H + 1];             // in[k..k+H]
  // push in[k+H] after in[k..k+H-1] are loaded, return out[k]
  __device__ __forceinline__ float step(int k, int len) {
    float v;
    if (k < H || k >= len - H) {
      v = in[0];
    } else {
      float s = 0.f;
#pragma unroll
      for (int q = 0; q < H; ++q) s = __fadd_rn(s, outp[q]);
#pragma unroll
      for (int q = 0; q <= H; ++q) s = __fadd_rn(s, in[q]);
      v = div_const<2 * H + 1>(s);
    }
#pragma unroll
    for (int q = 0; q + 1 < H; ++q) outp[q] = outp[q + 1];
    if (H > 0) outp[H - 1] = v;
#pragma unroll
    for (int q = 0; q < H; ++q) in[q] = in[q + 1];
    return v;
  }
};

// fine value of the expansion: coarse / c / c / c in libirl's order
template <int C>
__device__ __forceinline__ float expand_scale(float v) {
  return div_const<C>(div_const<C>(div_const<C>(v)));
}


// loads issued ahead of the dependent walk along a line
constexpr int WALK_PF = 8;

#ifdef __CUDA_ARCH__
template <bool GLOBAL>
__device__ __forceinline__ float ew_ld(const float *p) {
  if constexpr (GLOBAL) return __ldg(p);
  else return *p;
}
#else
template <bool GLOBAL>
inline float ew_ld(const float *p) { return *p; }
#endif

// one line: coarse values in[i * is] (i < nc; SCALE: scaled by expand_scale
// on load), fine outputs out[f * os] (f < C nc); GLOBAL: in is global
// memory (read through the read-only path), else shared memory.  The
// look-ahead input of fine entry f is coarse entry min(f + H, nf - 1) / C,
// which is this coarse entry or the next one.
template <int C, bool SCALE, bool GLOBAL>
__device__ __forceinline__ void coarse_walk(const float *in, size_t is, int nc, float *out, size_t os) {
  constexpr int H = C / 2;
  const int nf = nc * C;
  auto val = [&](float v) { return SCALE ? expand_scale<C>(v) : v; };
  LineSmoother<H> L;
  float cv[WALK_PF];
#pragma unroll
  for (int q = 0; q < WALK_PF; ++q) cv[q] = val(ew_ld<GLOBAL>(in + (size_t)min(q, nc - 1) * is));
#pragma unroll
  for (int q = 0; q < H; ++q) L.in[q] = cv[0];
  for (int c0 = 0; c0 < nc; c0 += WALK_PF) {
    float nx[WALK_PF];
#pragma unroll
    for (int q = 0; q < WALK_PF; ++q) nx[q] = ew_ld<GLOBAL>(in + (size_t)min(c0 + WALK_PF + q, nc - 1) * is);
    const float cnext = val(nx[0]);
#pragma unroll
    for (int r = 0; r < WALK_PF; ++r) {
      const int cc = c0 + r;
      if (cc < nc) {
        const float ca = cv[r], cb = r + 1 < WALK_PF ? cv[r + 1] : cnext;
#pragma unroll
        for (int q = 0; q < C; ++q) {
          const int f = cc * C + q;
          L.in[H] = ((q + H) / C == 0) ? ca : cb;
          out[(size_t)f * os] = L.step(f, nf);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < WALK_PF; ++q) cv[q] = val(nx[q]);
  }
}

}  // namespace irlcu
