// Host test of the ESSE expansion and smoothing at coarse resolution
// (esse_walk.cuh, as k_expand_y, k_smooth_z and k_smooth_x_combine run it):
// against ExpandByFac's full-resolution form -- replicate every coarse value
// (scaled by 1/c^3) over a c x c x c block, then smooth in place along y,
// then z, then x -- bit for bit.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <vector>
#include <random>
#include <algorithm>
#include <cuda_runtime.h>
using std::min;
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fmul_rn(float a, float b) { return a * b; }
static inline float __fmaf_rn(float a, float b, float c) { return std::fmaf(a, b, c); }
static inline float __fdiv_rn(float a, float b) { return a / b; }
static inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
#include "esse_walk.cuh"
using namespace irlcu;

// the in-place smoothing of one line (krnlprj3d.c:636-670) restated from its
// formula: out[k] = (out[k-h] + .. + out[k-1] + in[k] + .. + in[k+h]) / (2h+1)
// summed left to right from 0 for h <= k < len-h, else out[k] = in[k]
template <int H> static void smooth_line(float *v, size_t stride, int len) {
  std::vector<float> in(len), out(len);
  for (int k = 0; k < len; ++k) in[k] = v[k * stride];
  for (int k = 0; k < len; ++k) {
    if (k < H || k >= len - H) { out[k] = in[k]; continue; }
    float s = 0.f;
    for (int q = k - H; q < k; ++q) s = __fadd_rn(s, out[q]);
    for (int q = k; q <= k + H; ++q) s = __fadd_rn(s, in[q]);
    out[k] = div_const<2 * H + 1>(s);
  }
  for (int k = 0; k < len; ++k) v[k * stride] = out[k];
}

static long long g_bad = 0;

template <int C> static void test(int nyv, int nzv, int nxv, unsigned seed) {
  constexpr int H = C / 2;
  const int n = C * nyv, nz = C * nzv, nx = C * nxv;  // fine y, z, x
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> U(-1, 1);
  std::vector<float> g((size_t)nyv * nzv * nxv);
  for (auto &v : g) v = U(rng);
  g[0] = -0.f;  // a signed zero travels through both forms alike
  // full resolution
  std::vector<float> T((size_t)n * nz * nx);
  for (int y = 0; y < n; ++y)
    for (int z = 0; z < nz; ++z)
      for (int x = 0; x < nx; ++x)
        T[((size_t)y * nz + z) * nx + x] = expand_scale<C>(g[((size_t)(y / C) * nzv + z / C) * nxv + x / C]);
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) smooth_line<H>(&T[(size_t)z * nx + x], (size_t)nz * nx, n);
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < nx; ++x) smooth_line<H>(&T[(size_t)y * nz * nx + x], nx, nz);
  for (int y = 0; y < n; ++y)
    for (int z = 0; z < nz; ++z) smooth_line<H>(&T[((size_t)y * nz + z) * nx], 1, nx);
  // coarse form: y pass at coarse (z, x), z pass at coarse x, x pass fine
  const size_t gs = (size_t)nzv * nxv;
  std::vector<float> Tc((size_t)n * gs, NAN), Uz((size_t)n * nz * nxv, NAN), F((size_t)n * nz * nx, NAN);
  for (size_t i = 0; i < gs; ++i) coarse_walk<C, true, true>(&g[i], gs, nyv, &Tc[i], gs);
  for (int y = 0; y < n; ++y)
    for (int xc = 0; xc < nxv; ++xc)
      coarse_walk<C, false, true>(&Tc[(size_t)y * gs + xc], nxv, nzv, &Uz[(size_t)y * nz * nxv + xc], nxv);
  for (int y = 0; y < n; ++y)
    for (int z = 0; z < nz; ++z)
      coarse_walk<C, false, false>(&Uz[((size_t)y * nz + z) * nxv], 1, nxv, &F[((size_t)y * nz + z) * nx], 1);
  long long bad = 0;
  for (size_t e = 0; e < F.size(); ++e)
    if (std::memcmp(&F[e], &T[e], 4) != 0) ++bad;
  g_bad += bad;
  printf("c=%d coarse %dx%dx%d: %lld of %zu differ\n", C, nyv, nzv, nxv, bad, F.size());
}

int main() {
  test<2>(5, 6, 7, 1);
  test<2>(16, 16, 16, 2);
  test<2>(33, 20, 17, 3);
  test<3>(9, 3, 4, 4);
  test<3>(12, 11, 10, 5);
  test<4>(8, 5, 9, 6);
  test<4>(2, 1, 3, 7);
  printf("worst %lld differing values\n", g_bad);
  return g_bad == 0 ? 0 : 1;
}
