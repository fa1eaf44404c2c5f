// k_orbit.cu -- body-contour orbit edges (libirl ComputeOrbit,
// computeorbit.c:81-147).
//
// For every view, the thresholded 2D body image is rotated onto an m x m
// grid (m ~ sqrt(2) n, so an off-centre body stays on the grid) by the
// bilinear rotator of rot3dpar.c:19-198.  The rows are then searched from
// the detector side for the first one that holds any positive sample.
// libirl rotates the whole image and sums rows until a sum is positive.
// Thresholded pixels are 0 or above a non-negative threshold, so every
// sample is >= 0.  A row sum is therefore positive exactly when one sample
// is, and the search can stop at that row without rotating the rest.
//
// One CTA per view.  Its threads cover a row's pixels and vote with
// __syncthreads_or.  The samples are the exact float expressions of
// rot3dpar (products and sums each rounded once, truncating conversions);
// sin/cos come from the host's libm, as in libirl.
#include "irlcu_internal.cuh"

namespace irlcu {

__global__ void k_orbit_edge(const float *__restrict__ img, int n, int m, const float *__restrict__ sn,
                             const float *__restrict__ cs, int *__restrict__ consumed) {
  const int v = blockIdx.x;
  const float Sin = sn[v], Cos = cs[v];
  const float new_axis = (float)(0.5 * (double)(m - 1));
  const float old_axis = (float)(0.5 * (double)(n - 1));
  const float radius = (float)(0.5 * (double)m);
  for (int row = 0; row < m / 2; ++row) {
    // the row's extent inside the circle (rot3dpar.c:98-101)
    const double t = __dsub_rn((double)__fsub_rn(radius, (float)row), 0.5);
    const int np = 2 * (int)__dadd_rn(sqrt(__dsub_rn((double)__fmul_rn(radius, radius), __dmul_rn(t, t))), 0.5);
    const int head = (int)(0.5 * (double)(m - np));
    const int tail = head + np - 1;
    const float Y = __fsub_rn((float)row, new_axis);
    int hit = 0;
    for (int x = head + (int)threadIdx.x; x <= tail && !hit; x += blockDim.x) {
      const float X = __fsub_rn((float)x, new_axis);
      const float fx = __fadd_rn(__fsub_rn(__fmul_rn(X, Cos), __fmul_rn(Y, Sin)), old_axis);
      const float fy = __fadd_rn(__fadd_rn(__fmul_rn(X, Sin), __fmul_rn(Y, Cos)), old_axis);
      const int ox = (int)fx, oy = (int)fy;
      const bool xin0 = ox >= 0 && ox < n, xin1 = ox + 1 >= 0 && ox + 1 < n;
      const bool yin0 = oy >= 0 && oy < n, yin1 = oy + 1 >= 0 && oy + 1 < n;
      const float z0 = (xin0 && yin0) ? __ldg(img + (size_t)oy * n + ox) : 0.f;
      const float z1 = (xin0 && yin1) ? __ldg(img + (size_t)(oy + 1) * n + ox) : 0.f;
      const float z2 = (xin1 && yin0) ? __ldg(img + (size_t)oy * n + ox + 1) : 0.f;
      const float z3 = (xin1 && yin1) ? __ldg(img + (size_t)(oy + 1) * n + ox + 1) : 0.f;
      const float wy = __fsub_rn(fy, (float)oy), wx = __fsub_rn(fx, (float)ox);
      float z01 = __fadd_rn(z0, __fmul_rn(wy, __fsub_rn(z1, z0)));
      float z23 = __fadd_rn(z2, __fmul_rn(wy, __fsub_rn(z3, z2)));
      if (fy < 0.f) {
        z01 = z0;
        z23 = z2;
      }
      float s = __fadd_rn(z01, __fmul_rn(wx, __fsub_rn(z23, z01)));
      if (fx < 0.f) s = z01;
      hit = s > 0.f;
    }
    if (__syncthreads_or(hit)) {
      // libirl's row loop increments past the row it stopped on
      if (threadIdx.x == 0) consumed[v] = row + 1;
      return;
    }
  }
  if (threadIdx.x == 0) consumed[v] = m / 2;
}

}  // namespace irlcu

using namespace irlcu;

// Synchronous, on a stream of its own (every copy stream-ordered, like the
// rest of the library); needs no library context.
extern "C" int irlcu_orbit_edges(const float *img, int n, int m, const float *sn, const float *cs, int nviews,
                                 int *consumed) {
  if (!img || !sn || !cs || !consumed || n < 1 || m < n || nviews < 1)
    return set_error(IRLCU_EARG, "irlcu_orbit_edges: bad arguments (n = %d, m = %d, views = %d)", n, m, nviews);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(IRLCU_ECUDA, "no CUDA device is available; libirl_b200 has no CPU path");
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
    return set_error(IRLCU_ECUDA, "irlcu_orbit_edges: no stream");
  float *d_img = nullptr, *d_sc = nullptr;
  int *d_rows = nullptr;
  int rc = IRLCU_OK;
  const size_t img_bytes = sizeof(float) * (size_t)n * n;
  do {
    if (dev_alloc((void **)&d_img, img_bytes, st) != cudaSuccess ||
        dev_alloc((void **)&d_sc, sizeof(float) * 2 * nviews, st) != cudaSuccess ||
        dev_alloc((void **)&d_rows, sizeof(int) * nviews, st) != cudaSuccess) {
      rc = set_error(IRLCU_ENOMEM, "irlcu_orbit_edges: device allocation failed");
      break;
    }
    cudaError_t e = cudaMemcpyAsync(d_img, img, img_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_sc, sn, sizeof(float) * nviews, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_sc + nviews, cs, sizeof(float) * nviews, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
      k_orbit_edge<<<nviews, 256, 0, st>>>(d_img, n, m, d_sc, d_sc + nviews, d_rows);
      ++g_launch_count;
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(consumed, d_rows, sizeof(int) * nviews, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = set_error(IRLCU_ECUDA, "irlcu_orbit_edges: %s", cudaGetErrorString(e));
  } while (0);
  dev_free(d_img, st);
  dev_free(d_sc, st);
  dev_free(d_rows, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return rc;
}
