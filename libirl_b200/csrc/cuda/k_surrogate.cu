// k_surrogate.cu -- the learned scatter surrogate: a small 3D-conv encoder
// and 2D decoder that maps a view's rotated activity and attenuation to the
// view's ESSE scatter projection (the difference between the projection with
// and without the scatter model, osemrecon.c:757-786).
//
// Network (BF16 weights and activations, FP32 accumulation), per view:
//   input  [32][32][32][3]: the rotated activity, mu and exp(-depth) of the
//          128^3 view frame, each 4x4x4 average-pooled ([y][z][x][c],
//          channels last); activity and target are divided by the view's
//          mean activity s (the scatter projection is linear in activity)
//   E1 conv3d 3->32  k3 s1 + ReLU       [32][32][32][32]
//   E2 conv3d 32->32 k3 s2 + ReLU       [16][16][16][32]
//   E3 conv3d 32->64 k3 s2 + ReLU       [8][8][8][64]
//   fold depth into channels            [8][8][512]
//   D1 conv2d 512->256 k3 + ReLU, x2 nearest upsample   [16][16][256]
//   D2 conv2d 256->128 k3 + ReLU, x2                    [32][32][128]
//   D3 conv2d 128->64  k3 + ReLU, x2                    [64][64][64]
//   D4 conv2d 64->32   k3 + ReLU, x2                    [128][128][32]
//   D5 conv2d 32->1    k3 (linear)                      [128][128]
// 1,653,153 parameters.  Every convolution is a BF16 tensor-core GEMM on
// tcgen05 (TMEM accumulator, FP32) with the bias and ReLU in its epilogue:
// forward as an implicit GEMM that gathers the channels-last input directly
// (k_conv0_tc, k_conv_tc); backward (k_gemm_tc) on explicit im2col columns,
// transposed for the weight gradient, and on the input-gradient columns,
// folded back by a gather-form col2im.  The last layer (one output
// channel) keeps direct kernels and, for its input gradient, the
// mma.sync m16n8k16 GEMM, which IRLCU_SUR_TC=0 also selects everywhere.
// Long reductions are split over K and summed in a fixed order, so results
// are deterministic.
// Training: Adam on FP32 master weights, BF16 copies for the GEMMs.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "irlcu_internal.cuh"

namespace irlcu {

typedef __nv_bfloat16 bf16;

// activations are channels-last: [b][d][h][w][c]; 2D layers use d = 1.
struct ConvGeom {
  int b, di, hi, wi, ci;   // input (hi, wi: after the optional upsampling)
  int kd, kh, kw, s;       // kernel (odd sides, "same" padding k/2), stride
  int dout, hout, wout, co;
  int up;                  // 1: the input is the x2 nearest upsampling of a
                           // stored [b][di][hi/2][wi/2][ci] tensor
};

// element offset of input (b, id, ih, iw, c), upsampling folded in
__device__ __forceinline__ size_t in_off(const ConvGeom &g, int b, int id, int ih, int iw, int c) {
  const int ph = g.up ? ih >> 1 : ih, pw = g.up ? iw >> 1 : iw;
  const int H = g.up ? g.hi >> 1 : g.hi, Wd = g.up ? g.wi >> 1 : g.wi;
  return ((((size_t)b * g.di + id) * H + ph) * Wd + pw) * g.ci + c;
}

// ------------------------------------------------------------------ GEMM
// C(m, n) = sum_k A(m, k) B(k, n) over BF16 operands with FP32
// accumulation; A(m, k) = A[m*sam + k*sak], B(k, n) = B[k*sbk + n*sbn].
// Epilogue: + bias[n] (optional), ReLU (optional), then C = v (FP32 and/or
// BF16 output at C[m*scm + n*scn]).
struct GemmArgs {
  const bf16 *A, *B;
  long long sam, sak, sbk, sbn;
  int M, N, K;
  const float *bias;
  int relu;
  float *Cf;       // FP32 output or null
  bf16 *Cb;        // BF16 output or null
  long long scm, scn;
  // split-K: grid.z slices of kper each write raw sums to ws[z][M][N];
  // k_splitk_reduce adds them in slice order and applies the epilogue
  int splits, kper;
  float *ws;
};

constexpr int GBM = 64, GBN = 64, GBK = 32, GPAD = 8, GNT = 128;

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// tile [64 rows][GBK] of a strided operand into shared memory (k
// contiguous); entries outside rows x [.., K) are zero
__device__ __forceinline__ void load_tile(bf16 (*s)[GBK + GPAD], const bf16 *src, long long s_row, long long s_k,
                                          int row0, int k0, int rows, int K) {
  const bf16 zero = __float2bfloat16(0.f);
  if (s_k == 1 && (K & 7) == 0 && (s_row & 7) == 0 && ((uintptr_t)src & 15) == 0) {
    // 8 consecutive k per 16-byte load (k0 and K are multiples of 8)
    for (int e = threadIdx.x; e < GBM * (GBK / 8); e += GNT) {
      const int r = e / (GBK / 8), kk = (e % (GBK / 8)) * 8;
      const int row = row0 + r, k = k0 + kk;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (row < rows && k < K) v = *reinterpret_cast<const uint4 *>(src + row * s_row + k);
      *reinterpret_cast<uint4 *>(&s[r][kk]) = v;
    }
  } else if (s_row == 1) {
    // transposed operand: consecutive threads take consecutive rows
    for (int e = threadIdx.x; e < GBM * GBK; e += GNT) {
      const int r = e % GBM, kk = e / GBM;
      const int row = row0 + r, k = k0 + kk;
      s[r][kk] = (row < rows && k < K) ? src[row + k * s_k] : zero;
    }
  } else {
    for (int e = threadIdx.x; e < GBM * GBK; e += GNT) {
      const int r = e / GBK, kk = e % GBK;
      const int row = row0 + r, k = k0 + kk;
      s[r][kk] = (row < rows && k < K) ? src[row * s_row + k * s_k] : zero;
    }
  }
}

__global__ void __launch_bounds__(GNT) k_gemm_bf16(GemmArgs a) {
  __shared__ __align__(16) bf16 As[GBM][GBK + GPAD];
  __shared__ __align__(16) bf16 Bs[GBN][GBK + GPAD];  // [n][k]
  const int m0 = blockIdx.y * GBM, n0 = blockIdx.x * GBN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
  const int kb = a.splits > 1 ? blockIdx.z * a.kper : 0;
  const int ke = a.splits > 1 ? min(a.K, kb + a.kper) : a.K;
  for (int k0 = kb; k0 < ke; k0 += GBK) {
    __syncthreads();
    load_tile(As, a.A, a.sam, a.sak, m0, k0, a.M, ke);
    load_tile(Bs, a.B, a.sbn, a.sbk, n0, k0, a.N, ke);
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GBK; kk += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + g;
        af[i][0] = *reinterpret_cast<const uint32_t *>(&As[r][kk + 2 * t]);
        af[i][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + 2 * t]);
        af[i][2] = *reinterpret_cast<const uint32_t *>(&As[r][kk + 2 * t + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + j * 8 + g;
        bfr[j][0] = *reinterpret_cast<const uint32_t *>(&Bs[c][kk + 2 * t]);
        bfr[j][1] = *reinterpret_cast<const uint32_t *>(&Bs[c][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm + i * 16 + g + (q >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + 2 * t + (q & 1);
        if (m >= a.M || n >= a.N) continue;
        float v = acc[i][j][q];
        if (a.splits > 1) {
          a.ws[((size_t)blockIdx.z * a.M + m) * a.N + n] = v;
          continue;
        }
        if (a.bias) v += a.bias[n];
        if (a.relu) v = fmaxf(v, 0.f);
        const long long o = (long long)m * a.scm + (long long)n * a.scn;
        if (a.Cf) a.Cf[o] = v;
        if (a.Cb) a.Cb[o] = __float2bfloat16(v);
      }
}

// Convolution as an implicit GEMM (forward): C(m, n) = sum_k A(m, k) W[n][k]
// with A(m, k) read straight from the channels-last input, m = output
// position (b, od, oh, ow), k = tap*ci + c.  The CTA's 64 output positions
// are decoded once into shared memory; with ci a multiple of 8 every
// 8-wide k chunk is one tap's contiguous channels (a 16-byte load).
template <bool VEC>
__global__ void __launch_bounds__(GNT) k_conv_gemm(GemmArgs a, ConvGeom g, const bf16 *__restrict__ X) {
  __shared__ __align__(16) bf16 As[GBM][GBK + GPAD];
  __shared__ __align__(16) bf16 Bs[GBN][GBK + GPAD];
  __shared__ int rb[GBM], rd[GBM], rh[GBM], rw[GBM];
  const int m0 = blockIdx.y * GBM, n0 = blockIdx.x * GBN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int gq = lane >> 2, t = lane & 3;
  if (threadIdx.x < GBM) {
    const int m = m0 + threadIdx.x;
    if (m < a.M) {
      int r = m;
      const int ow = r % g.wout; r /= g.wout;
      const int oh = r % g.hout; r /= g.hout;
      const int od = r % g.dout;
      rb[threadIdx.x] = r / g.dout;
      rd[threadIdx.x] = od * g.s - g.kd / 2;
      rh[threadIdx.x] = oh * g.s - g.kh / 2;
      rw[threadIdx.x] = ow * g.s - g.kw / 2;
    } else {
      rb[threadIdx.x] = -1;
    }
  }
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
  const int kb = a.splits > 1 ? blockIdx.z * a.kper : 0;
  const int ke = a.splits > 1 ? min(a.K, kb + a.kper) : a.K;
  const int khw = g.kh * g.kw;
  for (int k0 = kb; k0 < ke; k0 += GBK) {
    __syncthreads();
    if (VEC) {
      for (int e = threadIdx.x; e < GBM * (GBK / 8); e += GNT) {
        const int r = e / (GBK / 8), kk = (e % (GBK / 8)) * 8, k = k0 + kk;
        uint4 v = make_uint4(0, 0, 0, 0);
        const int b = rb[r];
        if (b >= 0 && k < ke) {
          const int tap = k / g.ci, c = k - tap * g.ci;
          const int td = tap / khw, th = (tap - td * khw) / g.kw, tw = tap - td * khw - th * g.kw;
          const int id = rd[r] + td, ih = rh[r] + th, iw = rw[r] + tw;
          if (id >= 0 && id < g.di && ih >= 0 && ih < g.hi && iw >= 0 && iw < g.wi)
            v = *reinterpret_cast<const uint4 *>(X + in_off(g, b, id, ih, iw, c));
        }
        *reinterpret_cast<uint4 *>(&As[r][kk]) = v;
      }
    } else {
      const bf16 zero = __float2bfloat16(0.f);
      for (int e = threadIdx.x; e < GBM * GBK; e += GNT) {
        const int r = e / GBK, kk = e % GBK, k = k0 + kk;
        bf16 v = zero;
        const int b = rb[r];
        if (b >= 0 && k < ke) {
          const int tap = k / g.ci, c = k - tap * g.ci;
          const int td = tap / khw, th = (tap - td * khw) / g.kw, tw = tap - td * khw - th * g.kw;
          const int id = rd[r] + td, ih = rh[r] + th, iw = rw[r] + tw;
          if (id >= 0 && id < g.di && ih >= 0 && ih < g.hi && iw >= 0 && iw < g.wi)
            v = X[in_off(g, b, id, ih, iw, c)];
        }
        As[r][kk] = v;
      }
    }
    load_tile(Bs, a.B, a.sbn, a.sbk, n0, k0, a.N, ke);
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GBK; kk += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + gq;
        af[i][0] = *reinterpret_cast<const uint32_t *>(&As[r][kk + 2 * t]);
        af[i][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + 2 * t]);
        af[i][2] = *reinterpret_cast<const uint32_t *>(&As[r][kk + 2 * t + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + j * 8 + gq;
        bfr[j][0] = *reinterpret_cast<const uint32_t *>(&Bs[c][kk + 2 * t]);
        bfr[j][1] = *reinterpret_cast<const uint32_t *>(&Bs[c][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm + i * 16 + gq + (q >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + 2 * t + (q & 1);
        if (m >= a.M || n >= a.N) continue;
        float v = acc[i][j][q];
        if (a.splits > 1) {
          a.ws[((size_t)blockIdx.z * a.M + m) * a.N + n] = v;
          continue;
        }
        if (a.bias) v += a.bias[n];
        if (a.relu) v = fmaxf(v, 0.f);
        const long long o = (long long)m * a.scm + (long long)n * a.scn;
        if (a.Cf) a.Cf[o] = v;
        if (a.Cb) a.Cb[o] = __float2bfloat16(v);
      }
}

// ------------------------------------------------ tcgen05 implicit GEMM
// Forward convolution on the 5th-generation tensor cores: one CTA of 128
// threads per 128 output positions (rows) x all N = co output channels.
//   * operands: the CTA gathers A (the implicit im2col of the channels-last
//     input, 16-byte chunks of 8 channels of one tap) and B (the weights
//     [co][K], K contiguous) for a k tile of TC_BK into shared memory in
//     the K-major, no-swizzle canonical layout: core matrices of 8 rows x
//     16 bytes, row r of k chunk q at byte q * (R * 16) + r * 16, so the
//     descriptor's stride byte offset (between 8-row groups) is 128 and its
//     leading byte offset (between the two k chunks of one MMA) is R * 16;
//   * one elected thread issues tcgen05.mma (M 128, N, K 16, BF16 x BF16 ->
//     FP32) into a TMEM accumulator of N columns and commits to the
//     stage's mbarrier; two stages, so the gather of tile t + 1 overlaps
//     the MMAs of tile t;
//   * epilogue: warp w reads TMEM lanes 32w .. 32w+31 (its rows) with
//     tcgen05.ld, adds the bias, applies ReLU and stores 8 channels per
//     16-byte vector, or writes raw split-K partial sums.
// Every mbarrier wait is bounded; on a timeout the CTA records the error in
// g_tc_error, issues no further copies or MMAs, waits for its copies in
// flight and (bounded) for its last commit, and frees its TMEM.
constexpr int TC_BM = 128, TC_BK = 64, TC_NT = 128, TC_S = 4;
static_assert(TC_BM == TC_NT && TC_NT == 128 && TC_BK % 32 == 0, "k_conv_tc's copy mapping: 4 threads per row");
constexpr int TC_MAXCH = 640;  // k chunks (of 8) of one CTA's k range: K / 8 <= 576 here
constexpr unsigned TC_WAIT_LIMIT = 1u << 22;

__device__ int g_tc_error;
unsigned g_tc_refill_limit = TC_WAIT_LIMIT;  // host: polls of a stage-refill wait

template <int N>
struct TcCfg {
  static constexpr int A_BYTES = TC_BM * TC_BK * 2;
  static constexpr int B_BYTES = N * TC_BK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int TMEM_COLS = N < 32 ? 32 : N;
  // stages, the k-chunk tap table, barriers, alignment slack
  static constexpr size_t SMEM = TC_S * (size_t)STAGE + TC_MAXCH * 8 + 256 + 128;
  // kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major,
  // N >> 3 at bit 17, M >> 4 at bit 24
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
                                    ((uint32_t)(TC_BM >> 4) << 24);
  static_assert(N % 16 == 0 && N >= 16 && N <= 256, "M = 128 needs N a multiple of 16 up to 256");
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start, leading and stride byte offsets
// (16-byte units), version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned limit = TC_WAIT_LIMIT) {
  for (unsigned it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16-byte asynchronous copy global -> shared; ok = false fills zeros
__device__ __forceinline__ void cp16(uint32_t dst, const void *src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(ok ? 16 : 0) : "memory");
}

// refill_limit: polls of a stage-refill wait (TC_WAIT_LIMIT; a test sets 0,
// which makes those waits run out at once); the final wait for the last
// MMAs always polls up to TC_WAIT_LIMIT, so no MMA is in flight when the
// TMEM is freed
template <int N>
__global__ void __launch_bounds__(TC_NT) k_conv_tc(GemmArgs a, ConvGeom g, const bf16 *__restrict__ X,
                                                   unsigned refill_limit) {
  using Cfg = TcCfg<N>;
  extern __shared__ __align__(128) unsigned char tcs[];
  unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)tcs + 127) & ~(uintptr_t)127);
  int2 *ktab = reinterpret_cast<int2 *>(base + TC_S * Cfg::STAGE);     // per k chunk: packed tap, channel
  uint64_t *bars = reinterpret_cast<uint64_t *>(ktab + TC_MAXCH);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + TC_S);
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * TC_BM;
  const int kb = a.splits > 1 ? blockIdx.z * a.kper : 0;
  const int ke = a.splits > 1 ? min(a.K, kb + a.kper) : a.K;
  const int nk = (ke - kb + TC_BK - 1) / TC_BK;
  // A rows this thread copies: rows rg * 32 + tid / 4 (rg < TC_BM / 32),
  // output positions decoded once
  constexpr int TC_RG = TC_BM / 32;
  int rb[TC_RG], rd[TC_RG], rh[TC_RG], rw[TC_RG];
#pragma unroll
  for (int rg = 0; rg < TC_RG; ++rg) {
    rb[rg] = -1;
    rd[rg] = rh[rg] = rw[rg] = 0;
    const int m = m0 + rg * 32 + (tid >> 2);
    if (m < a.M) {
      int r = m;
      const int ow = r % g.wout;
      r /= g.wout;
      const int oh = r % g.hout;
      r /= g.hout;
      const int od = r % g.dout;
      rb[rg] = r / g.dout;
      rd[rg] = od * g.s - g.kd / 2;
      rh[rg] = oh * g.s - g.kh / 2;
      rw[rg] = ow * g.s - g.kw / 2;
    }
  }
  // tap offsets of the k chunks of [kb, kb + nk TC_BK) (c = -1 past ke)
  const int nch = nk * (TC_BK / 8);
  const int khw = g.kh * g.kw;
  for (int q = tid; q < nch; q += TC_NT) {
    const int k = kb + q * 8;
    int2 t = make_int2(0, -1);
    if (k < ke) {
      const int tap = k / g.ci, c = k - tap * g.ci;
      const int td = tap / khw, th = (tap - td * khw) / g.kw, tw = tap - td * khw - th * g.kw;
      t = make_int2(td | (th << 8) | (tw << 16), c);
    }
    ktab[q] = t;
  }
  if (tid == 0) {
    for (int i = 0; i < TC_S; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[i])));
    asm volatile("fence.mbarrier_init.release.cluster;");
    abort_flag = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(Cfg::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  const uint32_t sbase = smem_addr(base);
  // issue the copies of k tile t into stage t % TC_S
  auto load_tile = [&](int t) {
    const uint32_t As = sbase + (t % TC_S) * Cfg::STAGE, Bs = As + Cfg::A_BYTES;
    const int k0 = kb + t * TC_BK;
    // A: four consecutive threads copy four consecutive 16-byte chunks of
    // one row (64 bytes of one tap's channels, contiguous in the input), so
    // a warp's copies are 8 rows x 64 bytes of whole sectors, and its
    // shared-memory stores of one chunk column cover the 32 banks once
#pragma unroll
    for (int hq = 0; hq < TC_BK / 32; ++hq) {
      const int q = hq * 4 + (tid & 3);
      const int2 e = ktab[t * (TC_BK / 8) + q];
#pragma unroll
      for (int rg = 0; rg < TC_RG; ++rg) {
        const int row = rg * 32 + (tid >> 2);
        const int id = rd[rg] + (e.x & 0xff), ih = rh[rg] + ((e.x >> 8) & 0xff), iw = rw[rg] + (e.x >> 16);
        const bool ok =
            rb[rg] >= 0 && e.y >= 0 && id >= 0 && id < g.di && ih >= 0 && ih < g.hi && iw >= 0 && iw < g.wi;
        cp16(As + q * (TC_BM * 16) + row * 16,
             ok ? (const void *)(X + in_off(g, rb[rg], id, ih, iw, e.y)) : (const void *)X, ok);
      }
    }
    // B: 8 consecutive threads read one weight row's 8 chunks (128 bytes)
    for (int e = tid; e < N * (TC_BK / 8); e += TC_NT) {
      const int n = e >> 3, q = e & 7, k = k0 + q * 8;
      const bool ok = n < a.N && k < ke;
      cp16(Bs + q * (N * 16) + n * 16, ok ? (const void *)(a.B + (size_t)n * a.sbn + k) : (const void *)a.B, ok);
    }
  };
#pragma unroll
  for (int p = 0; p < TC_S - 1; ++p) {
    if (p < nk) load_tile(p);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  int last_it = -1;  // last tile whose MMAs were committed
  for (int it = 0; it < nk; ++it) {
    const int st = it % TC_S;
    asm volatile("cp.async.wait_group %0;" ::"n"(TC_S - 2) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (abort_flag) break;  // a wait ran out (flag set before the barrier): issue nothing more
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = sbase + st * Cfg::STAGE, b0 = a0 + Cfg::A_BYTES;
#pragma unroll
      for (int kk = 0; kk < TC_BK / 16; ++kk) {
        const uint64_t ad = umma_desc(a0 + kk * 2 * (TC_BM * 16), TC_BM * 16, 128);
        const uint64_t bd = umma_desc(b0 + kk * 2 * (N * 16), N * 16, 128);
        const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(Cfg::IDESC), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&bars[st]))
                   : "memory");
    }
    last_it = it;
    // refill the stage of tile it - 1 with tile it + TC_S - 1 once the MMAs
    // of tile it - 1 have read it
    const int nt = it + TC_S - 1;
    if (nt < nk) {
      if (it >= 1) {
        const int pt = it - 1;
        if (!mbar_wait(smem_addr(&bars[pt % TC_S]), (pt / TC_S) & 1, refill_limit)) {
          if (tid == 0) atomicExch(&g_tc_error, 1);
          abort_flag = 1;
        }
      }
      load_tile(nt);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  // all MMAs done: the last commit tracks every earlier one
  if (last_it >= 0 && !mbar_wait(smem_addr(&bars[last_it % TC_S]), (last_it / TC_S) & 1)) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
    abort_flag = 1;
  }
  __syncthreads();
  const bool ok = !abort_flag;  // uniform: the TMEM loads below are warp-collective
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (ok && last_it >= 0) {
    const int row = warp * 32 + lane, m = m0 + row;
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 8) {
      uint32_t v[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < a.M) {
        float f[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) f[q] = __uint_as_float(v[q]);
        if (a.splits > 1) {
          float *w = a.ws + ((size_t)blockIdx.z * a.M + m) * a.N + c0;
#pragma unroll
          for (int q = 0; q < 8; ++q) w[q] = f[q];
        } else {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            if (a.bias) f[q] += a.bias[c0 + q];
            if (a.relu) f[q] = fmaxf(f[q], 0.f);
          }
          __align__(16) bf16 h[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16(f[q]);
          *reinterpret_cast<uint4 *>(a.Cb + (long long)m * a.scm + c0) = *reinterpret_cast<const uint4 *>(h);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS));
}

// Plain tcgen05 GEMM for training's backward pass, both operands K-major:
// C(m, n) = sum_k A[m*sam + k] B[n*sbn + k] (sak = sbk = 1; K, sam, sbn
// multiples of 8 and 16-byte aligned rows), FP32 output at
// Cf[m*scm + n*scn], or raw split-K partials ws[z][M][N] that
// k_splitk_reduce adds in slice order.  One CTA of 128 threads per 128
// rows x NT columns (grid.y tiles N); the stage layout, the MMA issue, the
// bounded waits and the TMEM epilogue are k_conv_tc's, with the gather
// replaced by row copies: eight consecutive threads copy one row's 128
// bytes of a k tile.  Rows past M or N and k past the CTA's range read 0.
template <int NT>
__global__ void __launch_bounds__(TC_NT) k_gemm_tc(GemmArgs a, unsigned refill_limit) {
  using Cfg = TcCfg<NT>;
  extern __shared__ __align__(128) unsigned char tcs[];
  unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)tcs + 127) & ~(uintptr_t)127);
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + TC_S * Cfg::STAGE);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + TC_S);
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * NT;
  const int kb = a.splits > 1 ? blockIdx.z * a.kper : 0;
  const int ke = a.splits > 1 ? min(a.K, kb + a.kper) : a.K;
  const int nk = (ke - kb + TC_BK - 1) / TC_BK;
  if (tid == 0) {
    for (int i = 0; i < TC_S; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[i])));
    asm volatile("fence.mbarrier_init.release.cluster;");
    abort_flag = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(Cfg::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  const uint32_t sbase = smem_addr(base);
  auto load_tile = [&](int t) {
    const uint32_t As = sbase + (t % TC_S) * Cfg::STAGE, Bs = As + Cfg::A_BYTES;
    const int k0 = kb + t * TC_BK;
    for (int e = tid; e < TC_BM * (TC_BK / 8); e += TC_NT) {
      const int row = e >> 3, q = e & 7, k = k0 + q * 8, m = m0 + row;
      const bool ok = m < a.M && k < ke;
      cp16(As + q * (TC_BM * 16) + row * 16, ok ? (const void *)(a.A + (size_t)m * a.sam + k) : (const void *)a.A,
           ok);
    }
    for (int e = tid; e < NT * (TC_BK / 8); e += TC_NT) {
      const int n = e >> 3, q = e & 7, k = k0 + q * 8, nn = n0 + n;
      const bool ok = nn < a.N && k < ke;
      cp16(Bs + q * (NT * 16) + n * 16, ok ? (const void *)(a.B + (size_t)nn * a.sbn + k) : (const void *)a.B, ok);
    }
  };
#pragma unroll
  for (int p = 0; p < TC_S - 1; ++p) {
    if (p < nk) load_tile(p);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  int last_it = -1;
  for (int it = 0; it < nk; ++it) {
    const int st = it % TC_S;
    asm volatile("cp.async.wait_group %0;" ::"n"(TC_S - 2) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (abort_flag) break;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = sbase + st * Cfg::STAGE, b0 = a0 + Cfg::A_BYTES;
#pragma unroll
      for (int kk = 0; kk < TC_BK / 16; ++kk) {
        const uint64_t ad = umma_desc(a0 + kk * 2 * (TC_BM * 16), TC_BM * 16, 128);
        const uint64_t bd = umma_desc(b0 + kk * 2 * (NT * 16), NT * 16, 128);
        const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(Cfg::IDESC), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&bars[st]))
                   : "memory");
    }
    last_it = it;
    const int nt = it + TC_S - 1;
    if (nt < nk) {
      if (it >= 1) {
        const int pt = it - 1;
        if (!mbar_wait(smem_addr(&bars[pt % TC_S]), (pt / TC_S) & 1, refill_limit)) {
          if (tid == 0) atomicExch(&g_tc_error, 1);
          abort_flag = 1;
        }
      }
      load_tile(nt);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (last_it >= 0 && !mbar_wait(smem_addr(&bars[last_it % TC_S]), (last_it / TC_S) & 1)) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
    abort_flag = 1;
  }
  __syncthreads();
  const bool ok = !abort_flag;
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (ok && last_it >= 0) {
    const int m = m0 + warp * 32 + lane;
#pragma unroll
    for (int c0 = 0; c0 < NT; c0 += 8) {
      if (n0 + c0 >= a.N) break;  // uniform over the CTA
      uint32_t v[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      // eight consecutive columns of a row-major FP32 output (the split-K
      // partials, or Cf with scn = 1) go out as two 16-byte stores: one
      // whole 32-byte sector per thread instead of eight scalar stores
      float *vrow = nullptr;
      if (m < a.M && n0 + c0 + 8 <= a.N) {
        if (a.splits > 1) {
          if ((a.N & 3) == 0) vrow = a.ws + ((size_t)blockIdx.z * a.M + m) * a.N + n0 + c0;
        } else if (a.scn == 1 && (a.scm & 3) == 0 && a.Cf && !a.Cb && !a.bias && !a.relu &&
                   ((uintptr_t)a.Cf & 15) == 0) {
          vrow = a.Cf + (long long)m * a.scm + n0 + c0;
        }
      }
      if (vrow) {
        reinterpret_cast<float4 *>(vrow)[0] =
            make_float4(__uint_as_float(v[0]), __uint_as_float(v[1]), __uint_as_float(v[2]), __uint_as_float(v[3]));
        reinterpret_cast<float4 *>(vrow)[1] =
            make_float4(__uint_as_float(v[4]), __uint_as_float(v[5]), __uint_as_float(v[6]), __uint_as_float(v[7]));
      } else if (m < a.M) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int n = n0 + c0 + q;
          if (n >= a.N) break;
          float f = __uint_as_float(v[q]);
          if (a.splits > 1) {
            a.ws[((size_t)blockIdx.z * a.M + m) * a.N + n] = f;
          } else {
            if (a.bias) f += a.bias[n];
            if (a.relu) f = fmaxf(f, 0.f);
            const long long o = (long long)m * a.scm + (long long)n * a.scn;
            if (a.Cf) a.Cf[o] = f;
            if (a.Cb) a.Cb[o] = __float2bfloat16(f);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS));
}

__global__ void k_splitk_reduce(GemmArgs a) {
  const size_t tot = (size_t)a.M * a.N;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(e / a.N), n = (int)(e % a.N);
    float v = 0.f;
    for (int z = 0; z < a.splits; ++z) v += a.ws[(size_t)z * tot + e];
    if (a.bias) v += a.bias[n];
    if (a.relu) v = fmaxf(v, 0.f);
    const long long o = (long long)m * a.scm + (long long)n * a.scn;
    if (a.Cf) a.Cf[o] = v;
    if (a.Cb) a.Cb[o] = __float2bfloat16(v);
  }
}

// split-K workspace of a network (FP32 elements)
constexpr size_t GEMM_WS_ELEMS = (size_t)16 << 20;

// the tcgen05 convolution takes 16-byte channel chunks (ci a multiple of
// 8, aligned input and weights), N = co in {32, 64, 128, 256} and a
// channels-last output; IRLCU_SUR_TC=0 keeps the mma.sync kernel
static bool tc_usable(const GemmArgs &a, const ConvGeom &g, const bf16 *X) {
  static int env = -1;
  if (env < 0) {
    const char *e = getenv("IRLCU_SUR_TC");
    env = (e && e[0] == '0') ? 0 : 1;
  }
  if (!env) return false;
  const bool n_ok = a.N == 32 || a.N == 64 || a.N == 128 || a.N == 256;
  const int kspan = a.splits > 1 ? a.kper : a.K;  // one CTA's k range, in chunks of 8 for the tap table
  return n_ok && g.ci % 8 == 0 && a.K % 8 == 0 && a.sbk == 1 && a.sbn == a.K && ((uintptr_t)X & 15) == 0 &&
         ((uintptr_t)a.B & 15) == 0 && a.scn == 1 && a.scm == a.N && !a.Cf && a.Cb &&
         (kspan + TC_BK - 1) / TC_BK * (TC_BK / 8) <= TC_MAXCH && g.kd < 256 && g.kh < 256 && g.kw < 256;
}

#define TC_TRY(x)          \
  do {                     \
    const int rc_ = (x);   \
    if (rc_) return rc_;   \
  } while (0)

template <int N>
static int tc_attr() {
  static bool done = false;
  if (done) return IRLCU_OK;
  CU_TRY(cudaFuncSetAttribute(k_conv_tc<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TcCfg<N>::SMEM));
  done = true;
  return IRLCU_OK;
}

static int gemm(cudaStream_t st, GemmArgs a, float *ws, const ConvGeom *conv = nullptr, const bf16 *X = nullptr) {
  if (a.M <= 0 || a.N <= 0 || a.K <= 0) return IRLCU_OK;
  const int tiles_m = (a.M + GBM - 1) / GBM, tiles_n = (a.N + GBN - 1) / GBN;
  if (tiles_m > 65535) return set_error(IRLCU_EARG, "GEMM with M = %d too large", a.M);
  // split the reduction when the tile grid is small and K long
  const long long tiles = (long long)tiles_m * tiles_n;
  long long sp = std::min<long long>(592 / std::max<long long>(tiles, 1), a.K / 512);
  int splits = (int)std::max<long long>(1, std::min<long long>(sp, 64));
  while (splits > 1 && (size_t)splits * a.M * a.N > GEMM_WS_ELEMS) --splits;
  a.splits = 1;
  a.kper = a.K;
  if (splits > 1) {
    a.kper = ((a.K + splits - 1) / splits + GBK - 1) / GBK * GBK;
    a.splits = (a.K + a.kper - 1) / a.kper;  // slices actually populated
    a.ws = ws;
  }
  if (conv && tc_usable(a, *conv, X)) {
    const dim3 tgrid((a.M + TC_BM - 1) / TC_BM, 1, a.splits);
    switch (a.N) {
      case 32: TC_TRY(tc_attr<32>()); k_conv_tc<32><<<tgrid, TC_NT, TcCfg<32>::SMEM, st>>>(a, *conv, X, g_tc_refill_limit); break;
      case 64: TC_TRY(tc_attr<64>()); k_conv_tc<64><<<tgrid, TC_NT, TcCfg<64>::SMEM, st>>>(a, *conv, X, g_tc_refill_limit); break;
      case 128: TC_TRY(tc_attr<128>()); k_conv_tc<128><<<tgrid, TC_NT, TcCfg<128>::SMEM, st>>>(a, *conv, X, g_tc_refill_limit); break;
      default: TC_TRY(tc_attr<256>()); k_conv_tc<256><<<tgrid, TC_NT, TcCfg<256>::SMEM, st>>>(a, *conv, X, g_tc_refill_limit); break;
    }
    CU_LAUNCHED();
  } else {
  const dim3 grid(tiles_n, tiles_m, a.splits);
  if (conv) {
    if (conv->ci % 8 == 0 && ((uintptr_t)X & 15) == 0)
      k_conv_gemm<true><<<grid, GNT, 0, st>>>(a, *conv, X);
    else
      k_conv_gemm<false><<<grid, GNT, 0, st>>>(a, *conv, X);
  } else {
    k_gemm_bf16<<<grid, GNT, 0, st>>>(a);
  }
  CU_LAUNCHED();
  }
  if (a.splits > 1) {
    const size_t tot = (size_t)a.M * a.N;
    k_splitk_reduce<<<(unsigned)std::min<size_t>((tot + 255) / 256, 148 * 32), 256, 0, st>>>(a);
    CU_LAUNCHED();
  }
  return IRLCU_OK;
}

template <int NT>
static int gemm_tc_attr() {
  static bool done = false;
  if (done) return IRLCU_OK;
  CU_TRY(cudaFuncSetAttribute(k_gemm_tc<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TcCfg<NT>::SMEM));
  done = true;
  return IRLCU_OK;
}

// the backward GEMMs on tcgen05 unless IRLCU_SUR_TC=0
static bool bwd_tc_on() {
  static int env = -1;
  if (env < 0) {
    const char *e = getenv("IRLCU_SUR_TC");
    env = (e && e[0] == '0') ? 0 : 1;
  }
  return env == 1;
}

// k_gemm_tc over a GEMM with K-major operands (see there); the reduction
// is split when the tile grid is small, summed by k_splitk_reduce in slice
// order, so the result does not depend on scheduling
static int gemm_tc(cudaStream_t st, GemmArgs a, float *ws) {
  if (a.M <= 0 || a.N <= 0 || a.K <= 0) return IRLCU_OK;
  if (a.sak != 1 || a.sbk != 1 || a.K % 8 || a.sam % 8 || a.sbn % 8 || ((uintptr_t)a.A & 15) ||
      ((uintptr_t)a.B & 15))
    return set_error(IRLCU_EARG, "tcgen05 GEMM needs K-major operands with 16-byte rows (K = %d)", a.K);
  const int NT = a.N <= 32 ? 32 : a.N <= 64 ? 64 : a.N <= 128 ? 128 : 256;
  const long long tm = (a.M + TC_BM - 1) / TC_BM, tn = (a.N + NT - 1) / NT;
  if (tn > 65535) return set_error(IRLCU_EARG, "tcgen05 GEMM with N = %d too wide", a.N);
  const long long per_sm = NT <= 64 ? 2 : 1;  // resident CTAs per SM (shared memory)
  long long sp = std::min<long long>(per_sm * 148 / std::max<long long>(tm * tn, 1), a.K / 256);
  int splits = (int)std::max<long long>(1, std::min<long long>(sp, 64));
  while (splits > 1 && (size_t)splits * a.M * a.N > GEMM_WS_ELEMS) --splits;
  a.splits = 1;
  a.kper = a.K;
  if (splits > 1) {
    a.kper = ((a.K + splits - 1) / splits + TC_BK - 1) / TC_BK * TC_BK;
    a.splits = (a.K + a.kper - 1) / a.kper;
    a.ws = ws;
  }
  const dim3 grid((unsigned)tm, (unsigned)tn, a.splits);
  switch (NT) {
    case 32: TC_TRY(gemm_tc_attr<32>()); k_gemm_tc<32><<<grid, TC_NT, TcCfg<32>::SMEM, st>>>(a, g_tc_refill_limit); break;
    case 64: TC_TRY(gemm_tc_attr<64>()); k_gemm_tc<64><<<grid, TC_NT, TcCfg<64>::SMEM, st>>>(a, g_tc_refill_limit); break;
    case 128: TC_TRY(gemm_tc_attr<128>()); k_gemm_tc<128><<<grid, TC_NT, TcCfg<128>::SMEM, st>>>(a, g_tc_refill_limit); break;
    default: TC_TRY(gemm_tc_attr<256>()); k_gemm_tc<256><<<grid, TC_NT, TcCfg<256>::SMEM, st>>>(a, g_tc_refill_limit); break;
  }
  CU_LAUNCHED();
  if (a.splits > 1) {
    const size_t tot = (size_t)a.M * a.N;
    k_splitk_reduce<<<(unsigned)std::min<size_t>((tot + 255) / 256, 148 * 32), 256, 0, st>>>(a);
    CU_LAUNCHED();
  }
  return IRLCU_OK;
}

// out[c][r] = in[r][c] for a rows x cols BF16 matrix: 32 x 32 tiles through
// shared memory, grid (ceil(rows / 32), ceil(cols / 32)), block (32, 8)
__global__ void k_transpose_bf16(const bf16 *__restrict__ in, bf16 *__restrict__ out, long long rows, int cols) {
  __shared__ bf16 t[32][33];
  const long long r0 = (long long)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const long long r = r0 + i;
    const int c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[i][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = c0 + i;
    const long long r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(long long)c * rows + r] = t[threadIdx.x][i];
  }
}

static int transpose_bf16(cudaStream_t st, const bf16 *in, bf16 *out, long long rows, int cols) {
  const long long bx = (rows + 31) / 32;
  if (bx > 0x7fffffffLL || (cols + 31) / 32 > 65535) return set_error(IRLCU_EARG, "transpose of %lld x %d", rows, cols);
  k_transpose_bf16<<<dim3((unsigned)bx, (unsigned)((cols + 31) / 32)), dim3(32, 8), 0, st>>>(in, out, rows, cols);
  CU_LAUNCHED();
  return IRLCU_OK;
}

// ---------------------------------------------------------- conv helpers

__host__ __device__ inline int conv_out(int in, int k, int s) { return (in + 2 * (k / 2) - k) / s + 1; }

// im2col: row m = output position (b, od, oh, ow), column k = tap*ci + c
// with tap = (td*kh + th)*kw + tw
__global__ void k_im2col(ConvGeom g, const bf16 *__restrict__ x, bf16 *__restrict__ col) {
  const long long K = (long long)g.kd * g.kh * g.kw * g.ci;
  const long long M = (long long)g.b * g.dout * g.hout * g.wout;
  const long long tot = M * K;
  const bf16 zero = __float2bfloat16(0.f);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const long long m = e / K;
    const int k = (int)(e - m * K);
    const int c = k % g.ci, tap = k / g.ci;
    const int tw = tap % g.kw, th = (tap / g.kw) % g.kh, td = tap / (g.kw * g.kh);
    long long r = m;
    const int ow = (int)(r % g.wout); r /= g.wout;
    const int oh = (int)(r % g.hout); r /= g.hout;
    const int od = (int)(r % g.dout);
    const int b = (int)(r / g.dout);
    const int id = od * g.s + td - g.kd / 2, ih = oh * g.s + th - g.kh / 2, iw = ow * g.s + tw - g.kw / 2;
    bf16 v = zero;
    if (id >= 0 && id < g.di && ih >= 0 && ih < g.hi && iw >= 0 && iw < g.wi)
      v = x[in_off(g, b, id, ih, iw, c)];
    col[e] = v;
  }
}

// the same columns transposed, colT[k][m] (m contiguous): the K-major
// operand of the weight-gradient GEMM, whose reduction runs over m
__global__ void k_im2colT(ConvGeom g, const bf16 *__restrict__ x, bf16 *__restrict__ colT) {
  const long long K = (long long)g.kd * g.kh * g.kw * g.ci;
  const long long M = (long long)g.b * g.dout * g.hout * g.wout;
  const long long tot = M * K;
  const bf16 zero = __float2bfloat16(0.f);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e / M);
    const long long m = e - (long long)k * M;
    const int c = k % g.ci, tap = k / g.ci;
    const int tw = tap % g.kw, th = (tap / g.kw) % g.kh, td = tap / (g.kw * g.kh);
    long long r = m;
    const int ow = (int)(r % g.wout); r /= g.wout;
    const int oh = (int)(r % g.hout); r /= g.hout;
    const int od = (int)(r % g.dout);
    const int b = (int)(r / g.dout);
    const int id = od * g.s + td - g.kd / 2, ih = oh * g.s + th - g.kh / 2, iw = ow * g.s + tw - g.kw / 2;
    bf16 v = zero;
    if (id >= 0 && id < g.di && ih >= 0 && ih < g.hi && iw >= 0 && iw < g.wi)
      v = x[in_off(g, b, id, ih, iw, c)];
    colT[e] = v;
  }
}

// col2im in gather form: dx(b, id, ih, iw, c) = sum over the taps whose
// output position lies on the stride grid of dcol(m, tap*ci + c)
__global__ void k_col2im(ConvGeom g, const float *__restrict__ dcol, float *__restrict__ dx) {
  const long long K = (long long)g.kd * g.kh * g.kw * g.ci;
  const long long tot = (long long)g.b * g.di * g.hi * g.wi * g.ci;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e;
    const int c = (int)(r % g.ci); r /= g.ci;
    const int iw = (int)(r % g.wi); r /= g.wi;
    const int ih = (int)(r % g.hi); r /= g.hi;
    const int id = (int)(r % g.di);
    const int b = (int)(r / g.di);
    float s = 0.f;
    for (int td = 0; td < g.kd; ++td) {
      const int nd = id - td + g.kd / 2;
      if (nd < 0 || nd % g.s) continue;
      const int od = nd / g.s;
      if (od >= g.dout) continue;
      for (int th = 0; th < g.kh; ++th) {
        const int nh = ih - th + g.kh / 2;
        if (nh < 0 || nh % g.s) continue;
        const int oh = nh / g.s;
        if (oh >= g.hout) continue;
        for (int tw = 0; tw < g.kw; ++tw) {
          const int nw = iw - tw + g.kw / 2;
          if (nw < 0 || nw % g.s) continue;
          const int ow = nw / g.s;
          if (ow >= g.wout) continue;
          const long long m = (((long long)b * g.dout + od) * g.hout + oh) * g.wout + ow;
          const int tap = (td * g.kh + th) * g.kw + tw;
          s += dcol[m * K + (long long)tap * g.ci + c];
        }
      }
    }
    dx[e] = s;
  }
}

// First layer (3 input channels) as a direct convolution: one thread per
// output position, all 32 output channels in registers, FP32 products of the
// BF16 weights and inputs; + bias, ReLU, BF16 store
constexpr int FIRST_CI = 3, FIRST_CO = 32, FIRST_TAPS = 27;
__global__ void __launch_bounds__(128) k_conv_first(ConvGeom g, const bf16 *__restrict__ x,
                                                    const bf16 *__restrict__ w, const float *__restrict__ bias,
                                                    bf16 *__restrict__ y) {
  __shared__ __align__(16) float ws[FIRST_TAPS * FIRST_CI][FIRST_CO];
  __shared__ float bs[FIRST_CO];
  for (int e = threadIdx.x; e < FIRST_TAPS * FIRST_CI * FIRST_CO; e += blockDim.x) {
    const int co = e / (FIRST_TAPS * FIRST_CI), k = e % (FIRST_TAPS * FIRST_CI);
    ws[k][co] = __bfloat162float(w[e]);
  }
  if (threadIdx.x < FIRST_CO) bs[threadIdx.x] = bias[threadIdx.x];
  __syncthreads();
  const long long M = (long long)g.b * g.dout * g.hout * g.wout;
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  long long r = m;
  const int ow = (int)(r % g.wout); r /= g.wout;
  const int oh = (int)(r % g.hout); r /= g.hout;
  const int od = (int)(r % g.dout);
  const int b = (int)(r / g.dout);
  float acc[FIRST_CO];
#pragma unroll
  for (int co = 0; co < FIRST_CO; ++co) acc[co] = bs[co];
  for (int tap = 0; tap < FIRST_TAPS; ++tap) {
    const int td = tap / 9, th = (tap / 3) % 3, tw = tap % 3;
    const int id = od * g.s + td - 1, ih = oh * g.s + th - 1, iw = ow * g.s + tw - 1;
    if (id < 0 || id >= g.di || ih < 0 || ih >= g.hi || iw < 0 || iw >= g.wi) continue;
    const bf16 *px = x + in_off(g, b, id, ih, iw, 0);
#pragma unroll
    for (int c = 0; c < FIRST_CI; ++c) {
      const float v = __bfloat162float(px[c]);
      // one 16-byte (broadcast) shared load per 4 output channels
      const float4 *wr = reinterpret_cast<const float4 *>(ws[tap * FIRST_CI + c]);
#pragma unroll
      for (int q = 0; q < FIRST_CO / 4; ++q) {
        const float4 w4 = wr[q];
        acc[4 * q] = fmaf(w4.x, v, acc[4 * q]);
        acc[4 * q + 1] = fmaf(w4.y, v, acc[4 * q + 1]);
        acc[4 * q + 2] = fmaf(w4.z, v, acc[4 * q + 2]);
        acc[4 * q + 3] = fmaf(w4.w, v, acc[4 * q + 3]);
      }
    }
  }
  uint4 *o = reinterpret_cast<uint4 *>(y + m * FIRST_CO);
#pragma unroll
  for (int q = 0; q < FIRST_CO / 8; ++q) {
    __align__(16) bf16 h[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) h[j] = __float2bfloat16(fmaxf(acc[q * 8 + j], 0.f));
    o[q] = *reinterpret_cast<const uint4 *>(h);
  }
}

// The first layer (3 input channels, 27 taps: K = 81) on the tensor cores.
// Its 3-channel rows do not come in the 16-byte channel chunks that
// k_conv_tc gathers, so each thread builds its output position's whole A
// row in registers (the 27 taps x 3 channels, zero outside the input and
// past K, padded to K = 96) and stores it in the K-major no-swizzle
// layout; the weights [32][81] are staged the same way.  Thread 0 issues
// six M128 x N32 x K16 BF16 MMAs into a 32-column TMEM accumulator and
// commits to an mbarrier (bounded wait, as in k_conv_tc); the epilogue adds
// the bias, applies the ReLU and stores BF16.  One CTA of 128 threads per
// 128 output positions.  The products are summed in the tensor cores'
// order, not the direct kernels', so the outputs agree with them to FP32
// rounding.
constexpr int C0_KC = 12;                    // K chunks of 8: K = 96 >= 81
constexpr int C0_A = TC_BM * C0_KC * 16;     // A tile bytes
constexpr int C0_B = 32 * C0_KC * 16;        // B tile bytes
constexpr size_t C0_SMEM = (size_t)C0_A + C0_B + 64 + 128;

__global__ void __launch_bounds__(TC_NT) k_conv0_tc(ConvGeom g, const bf16 *__restrict__ x,
                                                    const bf16 *__restrict__ w, const float *__restrict__ bias,
                                                    bf16 *__restrict__ y) {
  extern __shared__ __align__(128) unsigned char c0s[];
  unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)c0s + 127) & ~(uintptr_t)127);
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + C0_A + C0_B);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long M = (long long)g.b * g.dout * g.hout * g.wout;
  const long long m = (long long)blockIdx.x * TC_BM + tid;
  const uint32_t sA = smem_addr(base), sB = sA + C0_A;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(32));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // this thread's A row: the 81 inputs of output position m, k = tap * 3 + c
  {
    uint32_t pk[C0_KC * 4];
#pragma unroll
    for (int q = 0; q < C0_KC * 4; ++q) pk[q] = 0u;
    if (m < M) {
      long long r = m;
      const int ow = (int)(r % g.wout);
      r /= g.wout;
      const int oh = (int)(r % g.hout);
      r /= g.hout;
      const int od = (int)(r % g.dout);
      const int b = (int)(r / g.dout);
#pragma unroll
      for (int tap = 0; tap < FIRST_TAPS; ++tap) {
        const int td = tap / 9, th = (tap / 3) % 3, tw = tap % 3;
        const int id = od * g.s + td - 1, ih = oh * g.s + th - 1, iw = ow * g.s + tw - 1;
        if (id < 0 || id >= g.di || ih < 0 || ih >= g.hi || iw < 0 || iw >= g.wi) continue;
        const unsigned short *px = reinterpret_cast<const unsigned short *>(x + in_off(g, b, id, ih, iw, 0));
#pragma unroll
        for (int c = 0; c < FIRST_CI; ++c) {
          const int k = tap * FIRST_CI + c;
          const uint32_t v = __ldg(px + c);
          pk[k >> 1] |= (k & 1) ? (v << 16) : v;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < C0_KC; ++q)
      asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sA + q * (TC_BM * 16) + tid * 16),
                   "r"(pk[4 * q]), "r"(pk[4 * q + 1]), "r"(pk[4 * q + 2]), "r"(pk[4 * q + 3]));
  }
  // B: weight row n, chunk q (k = 8q .. 8q+7; zero at k >= 81)
  {
    const unsigned short *wu = reinterpret_cast<const unsigned short *>(w);
    for (int e = tid; e < 32 * C0_KC; e += TC_NT) {
      const int n = e / C0_KC, q = e - n * C0_KC;
      uint32_t h[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = 8 * q + i;
        const uint32_t v = k < FIRST_TAPS * FIRST_CI ? (uint32_t)__ldg(wu + n * (FIRST_TAPS * FIRST_CI) + k) : 0u;
        h[i >> 1] |= (i & 1) ? (v << 16) : v;
      }
      asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sB + q * (32 * 16) + n * 16), "r"(h[0]),
                   "r"(h[1]), "r"(h[2]), "r"(h[3]));
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  if (tid == 0) {
#pragma unroll
    for (int kk = 0; kk < C0_KC / 2; ++kk) {
      const uint64_t ad = umma_desc(sA + kk * 2 * (TC_BM * 16), TC_BM * 16, 128);
      const uint64_t bd = umma_desc(sB + kk * 2 * (32 * 16), 32 * 16, 128);
      asm volatile(
          "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
          "l"(ad), "l"(bd), "r"(TcCfg<32>::IDESC), "r"(kk > 0 ? 1u : 0u), "r"(0), "r"(0), "r"(0), "r"(0));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
  }
  const bool ok = mbar_wait(smem_addr(bar), 0);
  if (!ok && lane == 0) atomicExch(&g_tc_error, 1);
  const bool all_ok = __syncthreads_and(ok);  // uniform: the TMEM loads are warp-collective
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (all_ok) {
#pragma unroll
    for (int c0 = 0; c0 < 32; c0 += 8) {
      uint32_t v[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < M) {
        __align__(16) bf16 h[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16(fmaxf(__uint_as_float(v[q]) + bias[c0 + q], 0.f));
        *reinterpret_cast<uint4 *>(y + m * 32 + c0) = *reinterpret_cast<const uint4 *>(h);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32));
}

// The first layer for an even output width: two adjacent output positions
// (ow, ow + 1) per thread, so that every shared-memory weight load feeds
// both.  Each output accumulates its products in the order k_conv_first does
// (taps, then channels), and a tap outside the input is skipped for that
// output alone, so the results are the same bit for bit.
__global__ void __launch_bounds__(128) k_conv_first2(ConvGeom g, const bf16 *__restrict__ x,
                                                     const bf16 *__restrict__ w, const float *__restrict__ bias,
                                                     bf16 *__restrict__ y) {
  __shared__ __align__(16) float ws[FIRST_TAPS * FIRST_CI][FIRST_CO];
  __shared__ float bs[FIRST_CO];
  for (int e = threadIdx.x; e < FIRST_TAPS * FIRST_CI * FIRST_CO; e += blockDim.x) {
    const int co = e / (FIRST_TAPS * FIRST_CI), k = e % (FIRST_TAPS * FIRST_CI);
    ws[k][co] = __bfloat162float(w[e]);
  }
  if (threadIdx.x < FIRST_CO) bs[threadIdx.x] = bias[threadIdx.x];
  __syncthreads();
  const int wh = g.wout >> 1;
  const long long M2 = (long long)g.b * g.dout * g.hout * wh;
  const long long m2 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m2 >= M2) return;
  long long r = m2;
  const int ow = (int)(r % wh) * 2;
  r /= wh;
  const int oh = (int)(r % g.hout);
  r /= g.hout;
  const int od = (int)(r % g.dout);
  const int b = (int)(r / g.dout);
  float a0[FIRST_CO], a1[FIRST_CO];
#pragma unroll
  for (int co = 0; co < FIRST_CO; ++co) a0[co] = a1[co] = bs[co];
  for (int tap = 0; tap < FIRST_TAPS; ++tap) {
    const int td = tap / 9, th = (tap / 3) % 3, tw = tap % 3;
    const int id = od * g.s + td - 1, ih = oh * g.s + th - 1, iw0 = ow * g.s + tw - 1, iw1 = iw0 + g.s;
    const bool dh = id >= 0 && id < g.di && ih >= 0 && ih < g.hi;
    const bool v0 = dh && iw0 >= 0 && iw0 < g.wi, v1 = dh && iw1 >= 0 && iw1 < g.wi;
    if (!v0 && !v1) continue;
    const bf16 *p0 = v0 ? x + in_off(g, b, id, ih, iw0, 0) : x;
    const bf16 *p1 = v1 ? x + in_off(g, b, id, ih, iw1, 0) : x;
#pragma unroll
    for (int c = 0; c < FIRST_CI; ++c) {
      const float x0 = v0 ? __bfloat162float(p0[c]) : 0.f, x1 = v1 ? __bfloat162float(p1[c]) : 0.f;
      const float4 *wr = reinterpret_cast<const float4 *>(ws[tap * FIRST_CI + c]);
#pragma unroll
      for (int q = 0; q < FIRST_CO / 4; ++q) {
        const float4 w4 = wr[q];
        if (v0) {
          a0[4 * q] = fmaf(w4.x, x0, a0[4 * q]);
          a0[4 * q + 1] = fmaf(w4.y, x0, a0[4 * q + 1]);
          a0[4 * q + 2] = fmaf(w4.z, x0, a0[4 * q + 2]);
          a0[4 * q + 3] = fmaf(w4.w, x0, a0[4 * q + 3]);
        }
        if (v1) {
          a1[4 * q] = fmaf(w4.x, x1, a1[4 * q]);
          a1[4 * q + 1] = fmaf(w4.y, x1, a1[4 * q + 1]);
          a1[4 * q + 2] = fmaf(w4.z, x1, a1[4 * q + 2]);
          a1[4 * q + 3] = fmaf(w4.w, x1, a1[4 * q + 3]);
        }
      }
    }
  }
  const long long m = (((long long)b * g.dout + od) * g.hout + oh) * g.wout + ow;
  uint4 *o = reinterpret_cast<uint4 *>(y + m * FIRST_CO);
#pragma unroll
  for (int q = 0; q < FIRST_CO / 8; ++q) {
    __align__(16) bf16 h0[8], h1[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      h0[j] = __float2bfloat16(fmaxf(a0[q * 8 + j], 0.f));
      h1[j] = __float2bfloat16(fmaxf(a1[q * 8 + j], 0.f));
    }
    o[q] = *reinterpret_cast<const uint4 *>(h0);
    o[FIRST_CO / 8 + q] = *reinterpret_cast<const uint4 *>(h1);
  }
}

// Last layer (one output channel, 2D, input 32 channels) as a direct
// convolution: one thread per output pixel, FP32 output
constexpr int LAST_CI = 32;
__global__ void __launch_bounds__(256) k_conv_last(ConvGeom g, const bf16 *__restrict__ x,
                                                   const bf16 *__restrict__ w, const float *__restrict__ bias,
                                                   float *__restrict__ y) {
  __shared__ float ws[9 * LAST_CI];
  for (int e = threadIdx.x; e < 9 * LAST_CI; e += blockDim.x) ws[e] = __bfloat162float(w[e]);
  __syncthreads();
  const long long M = (long long)g.b * g.hout * g.wout;
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  const int ow = (int)(m % g.wout), oh = (int)((m / g.wout) % g.hout), b = (int)(m / ((long long)g.wout * g.hout));
  float acc = bias[0];
  for (int tap = 0; tap < 9; ++tap) {
    const int ih = oh + tap / 3 - 1, iw = ow + tap % 3 - 1;
    if (ih < 0 || ih >= g.hi || iw < 0 || iw >= g.wi) continue;
    const uint4 *px = reinterpret_cast<const uint4 *>(x + in_off(g, b, 0, ih, iw, 0));
#pragma unroll
    for (int q = 0; q < LAST_CI / 8; ++q) {
      const uint4 u = px[q];
      const bf16 *h = reinterpret_cast<const bf16 *>(&u);
#pragma unroll
      for (int j = 0; j < 8; ++j) acc = fmaf(ws[tap * LAST_CI + q * 8 + j], __bfloat162float(h[j]), acc);
    }
  }
  y[m] = acc;
}

// gradient through ReLU: g = dy * (y > 0), to BF16 for the next GEMMs
__global__ void k_relu_grad(const float *__restrict__ dy, const bf16 *__restrict__ y, bf16 *__restrict__ g,
                            long long n, int relu) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    float v = dy[e];
    if (relu && !(__bfloat162float(y[e]) > 0.f)) v = 0.f;
    g[e] = __float2bfloat16(v);
  }
}

// bias gradient: column sums of g [M][N], fixed order
__global__ void k_bias_grad(const bf16 *__restrict__ g, long long M, int N, float *__restrict__ db) {
  const int n = blockIdx.x;
  __shared__ float red[256];
  float s = 0.f;
  for (long long m = threadIdx.x; m < M; m += blockDim.x) s += __bfloat162float(g[m * N + n]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[n] = red[0];
}

// fold depth into channels: [b][d][h][w][c] -> [b][h][w][d*c]; and the
// gradient back
__global__ void k_fold(const bf16 *__restrict__ x, bf16 *__restrict__ y, int b, int d, int h, int w, int c) {
  const long long tot = (long long)b * d * h * w * c;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e;
    const int cc = (int)(r % c); r /= c;
    const int ww = (int)(r % w); r /= w;
    const int hh = (int)(r % h); r /= h;
    const int dd = (int)(r % d);
    const int bb = (int)(r / d);
    y[(((long long)bb * h + hh) * w + ww) * (d * c) + dd * c + cc] = x[e];
  }
}
__global__ void k_unfold_f(const float *__restrict__ y, float *__restrict__ x, int b, int d, int h, int w, int c) {
  const long long tot = (long long)b * d * h * w * c;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e;
    const int cc = (int)(r % c); r /= c;
    const int ww = (int)(r % w); r /= w;
    const int hh = (int)(r % h); r /= h;
    const int dd = (int)(r % d);
    const int bb = (int)(r / d);
    x[e] = y[(((long long)bb * h + hh) * w + ww) * (d * c) + dd * c + cc];
  }
}

// x2 nearest upsampling of [b][h][w][c] and its gradient (sum of 4)
__global__ void k_up2(const bf16 *__restrict__ x, bf16 *__restrict__ y, int b, int h, int w, int c) {
  const long long tot = (long long)b * 4 * h * w * c;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e;
    const int cc = (int)(r % c); r /= c;
    const int X = (int)(r % (2 * w)); r /= 2 * w;
    const int Y = (int)(r % (2 * h));
    const int bb = (int)(r / (2 * h));
    y[e] = x[(((long long)bb * h + Y / 2) * w + X / 2) * c + cc];
  }
}
__global__ void k_up2_grad(const float *__restrict__ dy, float *__restrict__ dx, int b, int h, int w, int c) {
  const long long tot = (long long)b * h * w * c;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e;
    const int cc = (int)(r % c); r /= c;
    const int xx = (int)(r % w); r /= w;
    const int yy = (int)(r % h);
    const int bb = (int)(r / h);
    float s = 0.f;
    for (int q = 0; q < 4; ++q) {
      const int Y = 2 * yy + (q >> 1), X = 2 * xx + (q & 1);
      s += dy[(((long long)bb * 2 * h + Y) * 2 * w + X) * c + cc];
    }
    dx[e] = s;
  }
}

// mean squared error over [B][P]: grad = 2 (y - t) / (B P); per-sample
// squared-error sums in part[b] (fixed-order block reduction)
__global__ void k_mse(const float *__restrict__ y, const float *__restrict__ t, float *__restrict__ grad,
                      float *__restrict__ part, int P, float inv_count) {
  const int b = blockIdx.x;
  __shared__ float red[256];
  float s = 0.f;
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    const float d = y[(size_t)b * P + i] - t[(size_t)b * P + i];
    grad[(size_t)b * P + i] = 2.f * d * inv_count;
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[b] = red[0];
}

// Adam on FP32 master weights; refreshes the BF16 copy
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       bf16 *__restrict__ wb, long long n, float lr, float b1, float b2, float c1, float c2, float eps) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.f - b1) * gg;
    const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    const float nw = w[e] - lr * (mm * c1) / (sqrtf(vv * c2) + eps);
    w[e] = nw;
    wb[e] = __float2bfloat16(nw);
  }
}

__global__ void k_to_bf16(const float *__restrict__ x, bf16 *__restrict__ y, long long n) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    y[e] = __float2bfloat16(x[e]);
}

// Network input from the rotated volumes of a batch, channels last: 4x4x4
// means of the activity / s, of mu * 10 (per pixel -> order 1) and of
// exp(-S); s = the view's mean activity.  Pass 1 writes the mu and depth
// channels, the pooled activity means (pa) and one partial sum of them per
// CTA; pass 2 forms s from the partial sums (fixed order) and writes the
// normalised activity channel.
constexpr int POOL_NT = 256;
__global__ void __launch_bounds__(POOL_NT) k_pool_inputs(const float *__restrict__ act, size_t act_stride,
                                                         const float *__restrict__ mu, const float *__restrict__ S,
                                                         const int *__restrict__ views, size_t vox, int n,
                                                         float *__restrict__ pa, float *__restrict__ part,
                                                         bf16 *__restrict__ out) {
  const int P = SUR_P, f = n / SUR_P;
  const int tot = P * P * P;
  const float inv = 1.f / (float)(f * f * f);
  const int b = blockIdx.y;
  const int view = views[b];
  const float *a = act + (size_t)b * act_stride;
  const float *m = mu + (size_t)view * vox;
  const float *sd = S + (size_t)view * vox;
  __shared__ float red[POOL_NT];
  float psum = 0.f;
  for (int e = blockIdx.x * POOL_NT + threadIdx.x; e < tot; e += gridDim.x * POOL_NT) {
    const int px = e % P, pz = (e / P) % P, py = e / (P * P);
    float sa = 0.f, sm = 0.f, se = 0.f;
    for (int dy = 0; dy < f; ++dy)
      for (int dz = 0; dz < f; ++dz)
        for (int dx = 0; dx < f; dx += 4) {
          const size_t i = ((size_t)(f * py + dy) * n + (f * pz + dz)) * n + f * px + dx;
          const float4 va = __ldg(reinterpret_cast<const float4 *>(a + i));
          const float4 vm = __ldg(reinterpret_cast<const float4 *>(m + i));
          const float4 vs = __ldg(reinterpret_cast<const float4 *>(sd + i));
          sa += (va.x + va.y) + (va.z + va.w);
          sm += (vm.x + vm.y) + (vm.z + vm.w);
          se += (__expf(-vs.x) + __expf(-vs.y)) + (__expf(-vs.z) + __expf(-vs.w));
        }
    const float mean_a = sa * inv;
    pa[(size_t)b * tot + e] = mean_a;
    psum += mean_a;
    bf16 *o = out + ((size_t)b * tot + e) * 3;
    o[1] = __float2bfloat16(sm * (10.f * inv));
    o[2] = __float2bfloat16(se * inv);
  }
  red[threadIdx.x] = psum;
  __syncthreads();
  for (int w = POOL_NT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(size_t)b * gridDim.x + blockIdx.x] = red[0];
}

// the iteration-invariant channels (mu * 10 and exp(-S), 4^3 means) of
// every view, [view][P^3][2], pooled once per reconstruction
__global__ void __launch_bounds__(POOL_NT) k_pool_static(const float *__restrict__ mu, const float *__restrict__ S,
                                                         size_t vox, int n, bf16 *__restrict__ stat) {
  const int P = SUR_P, f = n / SUR_P;
  const int tot = P * P * P;
  const float inv = 1.f / (float)(f * f * f);
  const int view = blockIdx.y;
  const float *m = mu + (size_t)view * vox;
  const float *sd = S + (size_t)view * vox;
  for (int e = blockIdx.x * POOL_NT + threadIdx.x; e < tot; e += gridDim.x * POOL_NT) {
    const int px = e % P, pz = (e / P) % P, py = e / (P * P);
    float sm = 0.f, se = 0.f;
    for (int dy = 0; dy < f; ++dy)
      for (int dz = 0; dz < f; ++dz)
        for (int dx = 0; dx < f; dx += 4) {
          const size_t i = ((size_t)(f * py + dy) * n + (f * pz + dz)) * n + f * px + dx;
          const float4 vm = __ldg(reinterpret_cast<const float4 *>(m + i));
          const float4 vs = __ldg(reinterpret_cast<const float4 *>(sd + i));
          sm += (vm.x + vm.y) + (vm.z + vm.w);
          se += (__expf(-vs.x) + __expf(-vs.y)) + (__expf(-vs.z) + __expf(-vs.w));
        }
    bf16 *o = stat + ((size_t)view * tot + e) * 2;
    o[0] = __float2bfloat16(sm * (10.f * inv));
    o[1] = __float2bfloat16(se * inv);
  }
}

// activity channel only: 4^3 means and their partial sums
__global__ void __launch_bounds__(POOL_NT) k_pool_act(const float *__restrict__ act, size_t act_stride, int n,
                                                      float *__restrict__ pa, float *__restrict__ part) {
  const int P = SUR_P, f = n / SUR_P;
  const int tot = P * P * P;
  const float inv = 1.f / (float)(f * f * f);
  const int b = blockIdx.y;
  const float *a = act + (size_t)b * act_stride;
  __shared__ float red[POOL_NT];
  float psum = 0.f;
  for (int e = blockIdx.x * POOL_NT + threadIdx.x; e < tot; e += gridDim.x * POOL_NT) {
    const int px = e % P, pz = (e / P) % P, py = e / (P * P);
    float sa = 0.f;
    for (int dy = 0; dy < f; ++dy)
      for (int dz = 0; dz < f; ++dz)
        for (int dx = 0; dx < f; dx += 4) {
          const size_t i = ((size_t)(f * py + dy) * n + (f * pz + dz)) * n + f * px + dx;
          const float4 va = __ldg(reinterpret_cast<const float4 *>(a + i));
          sa += (va.x + va.y) + (va.z + va.w);
        }
    const float mean_a = sa * inv;
    pa[(size_t)b * tot + e] = mean_a;
    psum += mean_a;
  }
  red[threadIdx.x] = psum;
  __syncthreads();
  for (int w = POOL_NT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(size_t)b * gridDim.x + blockIdx.x] = red[0];
}

// channel 0 = activity / its mean; channels 1, 2 from the per-view cache
__global__ void __launch_bounds__(POOL_NT) k_pool_normalise_static(const float *__restrict__ pa,
                                                                   const float *__restrict__ part, int nparts,
                                                                   int tot, const int *__restrict__ views,
                                                                   const bf16 *__restrict__ stat,
                                                                   float *__restrict__ scale, bf16 *__restrict__ out) {
  const int b = blockIdx.y;
  float s = 0.f;
  for (int j = 0; j < nparts; ++j) s += part[(size_t)b * nparts + j];
  s /= (float)tot;
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[b] = s;
  const float inv = s > 0.f ? 1.f / s : 0.f;
  const bf16 *st = stat + (size_t)views[b] * tot * 2;
  for (int e = blockIdx.x * POOL_NT + threadIdx.x; e < tot; e += gridDim.x * POOL_NT) {
    bf16 *o = out + ((size_t)b * tot + e) * 3;
    o[0] = __float2bfloat16(pa[(size_t)b * tot + e] * inv);
    o[1] = st[2 * e];
    o[2] = st[2 * e + 1];
  }
}

__global__ void __launch_bounds__(POOL_NT) k_pool_normalise(const float *__restrict__ pa,
                                                            const float *__restrict__ part, int nparts, int tot,
                                                            float *__restrict__ scale, bf16 *__restrict__ out) {
  const int b = blockIdx.y;
  float s = 0.f;
  for (int j = 0; j < nparts; ++j) s += part[(size_t)b * nparts + j];
  s /= (float)tot;
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[b] = s;
  const float inv = s > 0.f ? 1.f / s : 0.f;
  for (int e = blockIdx.x * POOL_NT + threadIdx.x; e < tot; e += gridDim.x * POOL_NT)
    out[((size_t)b * tot + e) * 3] = __float2bfloat16(pa[(size_t)b * tot + e] * inv);
}

// out = a - c, elementwise
__global__ void k_sub(const float *__restrict__ a, const float *__restrict__ c, float *__restrict__ out, size_t n) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    out[e] = a[e] - c[e];
}

// y[b] = x[b] * s[b] (+ y[b] when accumulate)
__global__ void k_scale_views(const float *__restrict__ x, const float *__restrict__ s, float *__restrict__ y,
                              int P, int nb, int accumulate) {
  const size_t tot = (size_t)nb * P;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const float v = x[e] * s[e / P];
    y[e] = accumulate ? y[e] + v : v;
  }
}

// out[b] = a[b] / s[b]
__global__ void k_div_views(const float *__restrict__ a, const float *__restrict__ s, float *__restrict__ out, int P,
                            int nb) {
  const size_t tot = (size_t)nb * P;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const float sc = s[e / P];
    out[e] = sc > 0.f ? a[e] / sc : 0.f;
  }
}

// Projections larger than the network's SUR_OUT x SUR_OUT output (n = 256):
// y[b][z][x] (+)= s[b] * the output bilinearly interpolated at the pixel's
// centre ((u + 0.5) / f - 0.5 in output pixels, clamped at the edges)
constexpr int SUR_OUT = 128;
__global__ void k_scale_views_up(const float *__restrict__ x, const float *__restrict__ s, float *__restrict__ y,
                                 int n, int nb, int accumulate) {
  const int f = n / SUR_OUT;
  const size_t P = (size_t)n * n, tot = (size_t)nb * P;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(e / P), r = (int)(e - (size_t)b * P), zz = r / n, xx = r - zz * n;
    const float tz = fminf(fmaxf((zz + 0.5f) / f - 0.5f, 0.f), (float)(SUR_OUT - 1));
    const float tx = fminf(fmaxf((xx + 0.5f) / f - 0.5f, 0.f), (float)(SUR_OUT - 1));
    const int z0 = min((int)tz, SUR_OUT - 2), x0 = min((int)tx, SUR_OUT - 2);
    const float wz = tz - z0, wx = tx - x0;
    const float *q = x + (size_t)b * SUR_OUT * SUR_OUT + (size_t)z0 * SUR_OUT + x0;
    const float v0 = q[0] + wx * (q[1] - q[0]), v1 = q[SUR_OUT] + wx * (q[SUR_OUT + 1] - q[SUR_OUT]);
    const float v = (v0 + wz * (v1 - v0)) * s[b];
    y[e] = accumulate ? y[e] + v : v;
  }
}

// training targets of projections larger than the output: f x f means / s[b]
__global__ void k_div_views_down(const float *__restrict__ a, const float *__restrict__ s, float *__restrict__ out,
                                 int n, int nb) {
  const int f = n / SUR_OUT;
  const size_t P = (size_t)SUR_OUT * SUR_OUT, tot = (size_t)nb * P;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(e / P), r = (int)(e - (size_t)b * P), zz = r / SUR_OUT, xx = r - zz * SUR_OUT;
    const float *q = a + (size_t)b * n * n + (size_t)zz * f * n + (size_t)xx * f;
    float acc = 0.f;
    for (int i = 0; i < f; ++i)
      for (int j = 0; j < f; ++j) acc += q[(size_t)i * n + j];
    const float sc = s[b];
    out[e] = sc > 0.f ? acc / (float)(f * f) / sc : 0.f;
  }
}

static unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  return (unsigned)(g > 148 * 64 ? 148 * 64 : (g < 1 ? 1 : g));
}

struct Layer {
  ConvGeom g;
  bool relu, up;           // ReLU; x2 upsampling after the layer (decoder)
  size_t woff, boff;       // weights [co][K] and bias [co] in the parameter vector
  long long K;
};

}  // namespace irlcu

struct irlcu_sur {
  int max_batch = 0;
  std::vector<irlcu::Layer> L;
  size_t nparams = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // FP32 master, gradient, Adam moments
  irlcu::bf16 *wb = nullptr;                                     // BF16 weights
  long long step = 0;
  // act[0] = input, act[i+1] = output of layer i after ReLU (the next layer
  // reads it upsampled where it is); fold = E3 output, depth folded
  std::vector<irlcu::bf16 *> act;
  irlcu::bf16 *fold = nullptr;
  irlcu::bf16 *col = nullptr;     // im2col buffer (largest layer)
  float *dcol = nullptr;          // input-gradient columns
  float *gf = nullptr, *gf2 = nullptr;   // FP32 activation gradients
  irlcu::bf16 *gb = nullptr;      // BF16 gradient of the current layer output
  irlcu::bf16 *gbT = nullptr;     // gb transposed [co][M] (tcgen05 weight gradient)
  irlcu::bf16 *wT = nullptr;      // a layer's BF16 weights transposed [K][co] (tcgen05 input gradient)
  float *out = nullptr;           // network output [B][128*128]
  float *dout = nullptr;
  float *loss_part = nullptr;
  float *ws = nullptr;            // split-K workspace
  cudaStream_t st = nullptr;      // stream of the current work
  cudaStream_t own = nullptr;     // the network's own stream
};

namespace irlcu {

static void build_layers(irlcu_sur &s) {
  struct Spec {
    int di, hi, wi, ci, k3d, s, co;
    bool relu, up;
  };
  const Spec sp[] = {
      {32, 32, 32, 3, 1, 1, 32, true, false},  {32, 32, 32, 32, 1, 2, 32, true, false},
      {16, 16, 16, 32, 1, 2, 64, true, false}, {1, 8, 8, 512, 0, 1, 256, true, true},
      {1, 16, 16, 256, 0, 1, 128, true, true}, {1, 32, 32, 128, 0, 1, 64, true, true},
      {1, 64, 64, 64, 0, 1, 32, true, true},   {1, 128, 128, 32, 0, 1, 1, false, false}};
  size_t off = 0;
  s.L.clear();
  for (const Spec &p : sp) {
    Layer l{};
    l.g.di = p.di;
    l.g.hi = p.hi;
    l.g.wi = p.wi;
    l.g.ci = p.ci;
    l.g.kd = p.k3d ? 3 : 1;
    l.g.kh = 3;
    l.g.kw = 3;
    l.g.s = p.s;
    l.g.dout = conv_out(p.di, l.g.kd, p.s);
    l.g.hout = conv_out(p.hi, 3, p.s);
    l.g.wout = conv_out(p.wi, 3, p.s);
    l.g.co = p.co;
    l.relu = p.relu;
    l.up = p.up;
    l.g.up = (!s.L.empty() && s.L.back().up) ? 1 : 0;
    l.K = (long long)l.g.kd * 9 * p.ci;
    l.woff = off;
    off += (size_t)l.K * p.co;
    l.boff = off;
    off += p.co;
    s.L.push_back(l);
  }
  s.nparams = off;
}

// He-uniform initialisation from a seed (splitmix64), biases zero
static void init_weights(const irlcu_sur &s, unsigned long long seed, std::vector<float> &w) {
  w.assign(s.nparams, 0.f);
  unsigned long long x = seed;
  auto next = [&]() {
    x += 0x9E3779B97F4A7C15ULL;
    unsigned long long z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  };
  for (const Layer &l : s.L) {
    const double bound = std::sqrt(6.0 / (double)l.K);
    for (long long i = 0; i < l.K * l.g.co; ++i) {
      const double u = (double)(next() >> 11) / 9007199254740992.0;  // [0, 1)
      w[l.woff + i] = (float)((2.0 * u - 1.0) * bound);
    }
  }
}

static size_t layer_in_elems(const Layer &l, int B) { return (size_t)B * l.g.di * l.g.hi * l.g.wi * l.g.ci; }
static size_t layer_out_elems(const Layer &l, int B) {
  return (size_t)B * l.g.dout * l.g.hout * l.g.wout * l.g.co;
}

template <class T>
static int dmalloc(T **p, size_t n) {
  *p = nullptr;
  if (cudaMalloc(p, sizeof(T) * (n ? n : 1)) != cudaSuccess)
    return set_error(IRLCU_ENOMEM, "surrogate: device allocation of %zu bytes failed", sizeof(T) * n);
  return IRLCU_OK;
}

static void sur_free(irlcu_sur *s) {
  if (!s) return;
  cudaFree(s->w);
  cudaFree(s->g);
  cudaFree(s->m);
  cudaFree(s->v);
  cudaFree(s->wb);
  for (auto p : s->act) cudaFree(p);
  cudaFree(s->fold);
  cudaFree(s->col);
  cudaFree(s->dcol);
  cudaFree(s->gf);
  cudaFree(s->gf2);
  cudaFree(s->gb);
  cudaFree(s->gbT);
  cudaFree(s->wT);
  cudaFree(s->out);
  cudaFree(s->dout);
  cudaFree(s->loss_part);
  cudaFree(s->ws);
  if (s->own) cudaStreamDestroy(s->own);
  delete s;
}

#define STRY(x)            \
  do {                     \
    int rc_ = (x);         \
    if (rc_) return rc_;   \
  } while (0)

// input of layer i as im2col sees it
static const bf16 *layer_input(const irlcu_sur &s, int i) {
  if (i == 3) return s.fold;
  return s.act[i];  // layers after an upsampling read it through ConvGeom::up
}

// forward over the B samples in act[0]; FP32 output [B][128*128] in s.out
// the first layer on the tensor cores unless IRLCU_SUR_TC=0 (then the
// direct FP32 kernels k_conv_first / k_conv_first2)
static bool conv0_tc_usable() {
  static int env = -1;
  if (env < 0) {
    const char *e = getenv("IRLCU_SUR_TC");
    env = (e && e[0] == '0') ? 0 : 1;
  }
  return env == 1;
}

static int sur_forward(irlcu_sur &s, int B) {
  const int nl = (int)s.L.size();
  for (int i = 0; i < nl; ++i) {
    Layer l = s.L[i];
    l.g.b = B;
    if (i == 3) {  // fold the encoder's depth into channels
      const Layer &p = s.L[2];
      k_fold<<<grid_for((long long)layer_out_elems(p, B)), 256, 0, s.st>>>(s.act[3], s.fold, B, p.g.dout, p.g.hout,
                                                                            p.g.wout, p.g.co);
      CU_LAUNCHED();
    }
    const long long M = (long long)B * l.g.dout * l.g.hout * l.g.wout;
    if (i == 0 && l.g.ci == FIRST_CI && l.g.co == FIRST_CO && l.g.kd == 3) {
      if (conv0_tc_usable()) {
        static bool attr = false;
        if (!attr) {
          CU_TRY(cudaFuncSetAttribute(k_conv0_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C0_SMEM));
          attr = true;
        }
        k_conv0_tc<<<(unsigned)((M + TC_BM - 1) / TC_BM), TC_NT, C0_SMEM, s.st>>>(l.g, s.act[0], s.wb + l.woff,
                                                                               s.w + l.boff, s.act[1]);
      } else if ((l.g.wout & 1) == 0)
        k_conv_first2<<<(unsigned)((M / 2 + 127) / 128), 128, 0, s.st>>>(l.g, s.act[0], s.wb + l.woff,
                                                                        s.w + l.boff, s.act[1]);
      else
        k_conv_first<<<(unsigned)((M + 127) / 128), 128, 0, s.st>>>(l.g, s.act[0], s.wb + l.woff, s.w + l.boff,
                                                                   s.act[1]);
      CU_LAUNCHED();
      continue;
    }
    if (i == nl - 1 && l.g.co == 1 && l.g.ci == LAST_CI && l.g.kd == 1) {
      k_conv_last<<<(unsigned)((M + 255) / 256), 256, 0, s.st>>>(l.g, layer_input(s, i), s.wb + l.woff,
                                                                 s.w + l.boff, s.out);
      CU_LAUNCHED();
      continue;
    }
    GemmArgs a{};  // A read straight from the layer input (implicit im2col)
    a.B = s.wb + l.woff;  // weights [co][K]: B(k, n) = W[n*K + k]
    a.sbk = 1;
    a.sbn = l.K;
    a.M = (int)M;
    a.N = l.g.co;
    a.K = (int)l.K;
    a.bias = s.w + l.boff;
    a.relu = l.relu;
    if (i == nl - 1)
      a.Cf = s.out;
    else
      a.Cb = s.act[i + 1];
    a.scm = l.g.co;
    a.scn = 1;
    STRY(gemm(s.st, a, s.ws, &l.g, layer_input(s, i)));
  }
  return IRLCU_OK;
}

// backward from s.dout (dLoss / d output); parameter gradients into s.g
static int sur_backward(irlcu_sur &s, int B) {
  const int nl = (int)s.L.size();
  float *gcur = s.gf, *gnext = s.gf2;  // dLoss / d(layer output after ReLU)
  CU_TRY(cudaMemcpyAsync(gcur, s.dout, sizeof(float) * (size_t)B * 128 * 128, cudaMemcpyDeviceToDevice, s.st));
  for (int i = nl - 1; i >= 0; --i) {
    Layer l = s.L[i];
    l.g.b = B;
    const long long M = (long long)B * l.g.dout * l.g.hout * l.g.wout;
    const long long nout = M * l.g.co;
    const bf16 *yact = (i == nl - 1) ? nullptr : s.act[i + 1];
    k_relu_grad<<<grid_for(nout), 256, 0, s.st>>>(gcur, yact, s.gb, nout, (yact && l.relu) ? 1 : 0);
    CU_LAUNCHED();
    // the tcgen05 GEMMs take K-major operands: the weight gradient reduces
    // over the M output positions, so it reads the columns and the layer
    // gradient transposed (M a multiple of 8 keeps their rows 16-byte
    // aligned); the input gradient reduces over the co output channels
    const bool tc_w = bwd_tc_on() && M % 8 == 0;
    const bool tc_d = bwd_tc_on() && l.g.co % 8 == 0;
    if (tc_w) {
      k_im2colT<<<grid_for(M * l.K), 256, 0, s.st>>>(l.g, layer_input(s, i), s.col);
      CU_LAUNCHED();
      STRY(transpose_bf16(s.st, s.gb, s.gbT, M, l.g.co));
      // dW[n][k] = sum_m colT[k][m] gT[n][m]
      GemmArgs a{};
      a.A = s.col;
      a.sam = M;
      a.sak = 1;
      a.B = s.gbT;
      a.sbn = M;
      a.sbk = 1;
      a.M = (int)l.K;
      a.N = l.g.co;
      a.K = (int)M;
      a.Cf = s.g + l.woff;  // dW[n*K + k]
      a.scm = 1;
      a.scn = l.K;
      STRY(gemm_tc(s.st, a, s.ws));
    } else {
      k_im2col<<<grid_for(M * l.K), 256, 0, s.st>>>(l.g, layer_input(s, i), s.col);
      CU_LAUNCHED();
      // dW[n][k] = sum_m col[m][k] g[m][n]
      GemmArgs a{};
      a.A = s.col;  // A'(k, m) = col[m*K + k]
      a.sam = 1;
      a.sak = l.K;
      a.B = s.gb;   // B'(m, n) = g[m*co + n]
      a.sbk = l.g.co;
      a.sbn = 1;
      a.M = (int)l.K;
      a.N = l.g.co;
      a.K = (int)M;
      a.Cf = s.g + l.woff;  // dW[n*K + k]
      a.scm = 1;
      a.scn = l.K;
      STRY(gemm(s.st, a, s.ws));
    }
    k_bias_grad<<<l.g.co, 256, 0, s.st>>>(s.gb, M, l.g.co, s.g + l.boff);
    CU_LAUNCHED();
    if (i == 0) break;  // no gradient for the input
    // dcol[m][k] = sum_n g[m][n] W[n][k]
    GemmArgs d{};
    d.A = s.gb;
    d.sam = l.g.co;
    d.sak = 1;
    d.M = (int)M;
    d.N = (int)l.K;
    d.K = l.g.co;
    d.Cf = s.dcol;
    d.scm = l.K;
    d.scn = 1;
    if (tc_d) {
      STRY(transpose_bf16(s.st, s.wb + l.woff, s.wT, l.g.co, (int)l.K));
      d.B = s.wT;  // B(k, n) = WT[k*co + n]
      d.sbn = l.g.co;
      d.sbk = 1;
      STRY(gemm_tc(s.st, d, s.ws));
    } else {
      d.B = s.wb + l.woff;  // B(n, k) = W[n*K + k]
      d.sbk = l.K;
      d.sbn = 1;
      STRY(gemm(s.st, d, s.ws));
    }
    const long long nin = (long long)layer_in_elems(l, B);
    k_col2im<<<grid_for(nin), 256, 0, s.st>>>(l.g, s.dcol, gnext);
    CU_LAUNCHED();
    // gnext = dLoss / d(layer i input): map it to layer i-1's output
    if (i == 3) {
      const Layer &p = s.L[2];
      k_unfold_f<<<grid_for(nin), 256, 0, s.st>>>(gnext, gcur, B, p.g.dout, p.g.hout, p.g.wout, p.g.co);
      CU_LAUNCHED();
    } else if (i > 3 && s.L[i - 1].up) {
      const Layer &p = s.L[i - 1];
      k_up2_grad<<<grid_for((long long)layer_out_elems(p, B)), 256, 0, s.st>>>(gnext, gcur, B, p.g.hout, p.g.wout,
                                                                              p.g.co);
      CU_LAUNCHED();
    } else {
      std::swap(gcur, gnext);
    }
  }
  return IRLCU_OK;
}

static int sur_loss(irlcu_sur &s, int B, const float *t, float *loss) {
  const int P = 128 * 128;
  k_mse<<<B, 256, 0, s.st>>>(s.out, t, s.dout, s.loss_part, P, 1.f / ((float)B * P));
  CU_LAUNCHED();
  if (loss) {
    std::vector<float> part(B);
    CU_TRY(cudaMemcpyAsync(part.data(), s.loss_part, sizeof(float) * B, cudaMemcpyDeviceToHost, s.st));
    CU_TRY(cudaStreamSynchronize(s.st));
    double sum = 0.0;
    for (float p : part) sum += p;
    *loss = (float)(sum / ((double)B * P));
  }
  return IRLCU_OK;
}

static int sur_check_batch(const irlcu_sur *s, int B) {
  if (!s) return set_error(IRLCU_EARG, "surrogate: null network");
  if (B < 1 || B > s->max_batch) return set_error(IRLCU_EARG, "surrogate: batch %d outside 1..%d", B, s->max_batch);
  return IRLCU_OK;
}

// ------------------------------------------- use inside the projector

// a tcgen05 pipeline wait that ran out leaves g_tc_error set (the kernel
// freed its TMEM and returned); the host reads and clears the flag after it
// has synchronised with st and reports it as an error
int sur_tc_status(cudaStream_t st) {
  int v = 0;
  CU_TRY(cudaMemcpyFromSymbolAsync(&v, g_tc_error, sizeof(int), 0, cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  if (!v) return IRLCU_OK;
  const int zero = 0;
  CU_TRY(cudaMemcpyToSymbolAsync(g_tc_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st));
  CU_TRY(cudaStreamSynchronize(st));
  return set_error(IRLCU_ECUDA, "surrogate: a tensor-core pipeline wait timed out");
}

int sur_max_batch(const irlcu_sur *s) { return s ? s->max_batch : 0; }
void *sur_input(irlcu_sur *s) { return s->act[0]; }

// forward of the B samples already in sur_input(s), on stream st; FP32
// output [B][128*128] in *y (the network's buffer, valid until its next use)
int sur_infer(irlcu_sur *s, cudaStream_t st, int B, const float **y) {
  STRY(sur_check_batch(s, B));
  s->st = st;
  const int rc = sur_forward(*s, B);
  s->st = s->own;
  *y = s->out;
  return rc;
}

// pooled network inputs of nv rotated volumes (act, stride act_stride) with
// the per-view mu and depth tables; the activity means go to scale
int launch_sur_static(cudaStream_t st, const float *mu, const float *S, int nviews, int n, size_t vox, void *stat) {
  k_pool_static<<<dim3(SUR_POOL_PARTS, nviews), POOL_NT, 0, st>>>(mu, S, vox, n, static_cast<bf16 *>(stat));
  CU_LAUNCHED();
  return IRLCU_OK;
}

int launch_sur_inputs_static(cudaStream_t st, const float *act, size_t act_stride, const void *stat,
                             const int *dviews, int nv, int n, float *scale, void *out, float *work) {
  const int P = SUR_P, tot = P * P * P;
  const int nparts = SUR_POOL_PARTS;
  float *pa = work, *part = work + (size_t)nv * tot;
  dim3 grid(nparts, nv);
  k_pool_act<<<grid, POOL_NT, 0, st>>>(act, act_stride, n, pa, part);
  CU_LAUNCHED();
  k_pool_normalise_static<<<grid, POOL_NT, 0, st>>>(pa, part, nparts, tot, dviews,
                                                    static_cast<const bf16 *>(stat), scale, static_cast<bf16 *>(out));
  CU_LAUNCHED();
  return IRLCU_OK;
}

int launch_sur_inputs(cudaStream_t st, const float *act, size_t act_stride, const float *mu, const float *S,
                      const int *dviews, int nv, int n, size_t vox, float *scale, void *out, float *work) {
  const int P = SUR_P, tot = P * P * P;
  const int nparts = SUR_POOL_PARTS;
  float *pa = work, *part = work + (size_t)nv * tot;
  dim3 grid(nparts, nv);
  k_pool_inputs<<<grid, POOL_NT, 0, st>>>(act, act_stride, mu, S, dviews, vox, n, pa, part, static_cast<bf16 *>(out));
  CU_LAUNCHED();
  k_pool_normalise<<<grid, POOL_NT, 0, st>>>(pa, part, nparts, tot, scale, static_cast<bf16 *>(out));
  CU_LAUNCHED();
  return IRLCU_OK;
}

int launch_sub(cudaStream_t st, const float *a, const float *b, float *out, size_t n) {
  k_sub<<<grid_for((long long)n), 256, 0, st>>>(a, b, out, n);
  CU_LAUNCHED();
  return IRLCU_OK;
}

int launch_scale_views(cudaStream_t st, const float *x, const float *s, float *y, int P, int nb, int accumulate) {
  k_scale_views<<<grid_for((long long)P * nb), 256, 0, st>>>(x, s, y, P, nb, accumulate);
  CU_LAUNCHED();
  return IRLCU_OK;
}

int launch_scale_views_up(cudaStream_t st, const float *x, const float *s, float *y, int n, int nb, int accumulate) {
  if (n == SUR_OUT) return launch_scale_views(st, x, s, y, n * n, nb, accumulate);
  if (n % SUR_OUT) return set_error(IRLCU_EARG, "surrogate output: n = %d is not a multiple of %d", n, SUR_OUT);
  k_scale_views_up<<<grid_for((long long)n * n * nb), 256, 0, st>>>(x, s, y, n, nb, accumulate);
  CU_LAUNCHED();
  return IRLCU_OK;
}

int launch_div_views_down(cudaStream_t st, const float *a, const float *s, float *out, int n, int nb) {
  if (n == SUR_OUT) return launch_div_views(st, a, s, out, n * n, nb);
  if (n % SUR_OUT) return set_error(IRLCU_EARG, "surrogate targets: n = %d is not a multiple of %d", n, SUR_OUT);
  k_div_views_down<<<grid_for((long long)SUR_OUT * SUR_OUT * nb), 256, 0, st>>>(a, s, out, n, nb);
  CU_LAUNCHED();
  return IRLCU_OK;
}

int launch_div_views(cudaStream_t st, const float *a, const float *s, float *out, int P, int nb) {
  k_div_views<<<grid_for((long long)P * nb), 256, 0, st>>>(a, s, out, P, nb);
  CU_LAUNCHED();
  return IRLCU_OK;
}

}  // namespace irlcu

using namespace irlcu;

extern "C" {

int irlcu_sur_create(int max_batch, unsigned long long seed, irlcu_sur **out) {
  *out = nullptr;
  if (max_batch < 1 || max_batch > 256) return set_error(IRLCU_EARG, "surrogate: batch %d outside 1..256", max_batch);
  irlcu_sur *s = new irlcu_sur;
  s->max_batch = max_batch;
  build_layers(*s);
  int rc = IRLCU_OK;
  auto fail = [&](int r) {
    sur_free(s);
    return r;
  };
  if (cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error(IRLCU_ECUDA, "surrogate: stream creation failed"));
  s->st = s->own;
  const size_t P = s->nparams;
  if ((rc = dmalloc(&s->w, P)) || (rc = dmalloc(&s->g, P)) || (rc = dmalloc(&s->m, P)) || (rc = dmalloc(&s->v, P)) ||
      (rc = dmalloc(&s->wb, P)))
    return fail(rc);
  const int B = max_batch;
  size_t colmax = 0, actmax = 0, wmax = 0;
  s->act.assign(s->L.size() + 1, nullptr);
  for (size_t i = 0; i < s->L.size(); ++i) {
    const Layer &l = s->L[i];
    wmax = std::max(wmax, (size_t)l.K * l.g.co);
    const size_t M = (size_t)B * l.g.dout * l.g.hout * l.g.wout;
    colmax = std::max(colmax, M * (size_t)l.K);
    actmax = std::max(actmax, std::max(layer_in_elems(l, B), layer_out_elems(l, B)));
    if (i == 0 && (rc = dmalloc(&s->act[0], layer_in_elems(l, B)))) return fail(rc);
    if ((rc = dmalloc(&s->act[i + 1], layer_out_elems(l, B)))) return fail(rc);
    if (l.up) actmax = std::max(actmax, layer_out_elems(l, B) * 4);
  }
  if ((rc = dmalloc(&s->fold, layer_out_elems(s->L[2], B))) || (rc = dmalloc(&s->col, colmax)) ||
      (rc = dmalloc(&s->dcol, colmax)) || (rc = dmalloc(&s->gf, actmax)) || (rc = dmalloc(&s->gf2, actmax)) ||
      (rc = dmalloc(&s->gb, actmax)) || (rc = dmalloc(&s->gbT, actmax)) || (rc = dmalloc(&s->wT, wmax)) ||
      (rc = dmalloc(&s->out, (size_t)B * 128 * 128)) ||
      (rc = dmalloc(&s->dout, (size_t)B * 128 * 128)) || (rc = dmalloc(&s->loss_part, (size_t)B)) ||
      (rc = dmalloc(&s->ws, GEMM_WS_ELEMS)))
    return fail(rc);
  std::vector<float> w;
  init_weights(*s, seed, w);
  if (cudaMemcpyAsync(s->w, w.data(), sizeof(float) * P, cudaMemcpyHostToDevice, s->st) != cudaSuccess ||
      cudaMemsetAsync(s->m, 0, sizeof(float) * P, s->st) != cudaSuccess ||
      cudaMemsetAsync(s->v, 0, sizeof(float) * P, s->st) != cudaSuccess)
    return fail(set_error(IRLCU_ECUDA, "surrogate: initial upload failed"));
  k_to_bf16<<<grid_for((long long)P), 256, 0, s->st>>>(s->w, s->wb, (long long)P);
  ++g_launch_count;
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s->st) != cudaSuccess)
    return fail(set_error(IRLCU_ECUDA, "surrogate: initialisation failed"));
  *out = s;
  return IRLCU_OK;
}

void irlcu_sur_destroy(irlcu_sur *s) {
  if (s) cudaStreamSynchronize(s->own);
  sur_free(s);
}

size_t irlcu_sur_nparams(const irlcu_sur *s) { return s ? s->nparams : 0; }

int irlcu_sur_get_weights(irlcu_sur *s, float *host, size_t n) {
  if (!s || n != s->nparams) return set_error(IRLCU_EARG, "surrogate: expected %zu parameters", s ? s->nparams : 0);
  CU_TRY(cudaStreamSynchronize(s->st));
  CU_TRY(cudaMemcpyAsync(host, s->w, sizeof(float) * n, cudaMemcpyDeviceToHost, s->st));
  CU_TRY(cudaStreamSynchronize(s->st));
  return IRLCU_OK;
}

int irlcu_sur_set_weights(irlcu_sur *s, const float *host, size_t n) {
  if (!s || n != s->nparams) return set_error(IRLCU_EARG, "surrogate: expected %zu parameters", s ? s->nparams : 0);
  CU_TRY(cudaStreamSynchronize(s->st));
  CU_TRY(cudaMemcpyAsync(s->w, host, sizeof(float) * n, cudaMemcpyHostToDevice, s->st));
  CU_TRY(cudaMemsetAsync(s->m, 0, sizeof(float) * n, s->st));
  CU_TRY(cudaMemsetAsync(s->v, 0, sizeof(float) * n, s->st));
  s->step = 0;
  k_to_bf16<<<grid_for((long long)n), 256, 0, s->st>>>(s->w, s->wb, (long long)n);
  CU_LAUNCHED();
  CU_TRY(cudaStreamSynchronize(s->st));
  return IRLCU_OK;
}

unsigned irlcu_sur_test_refill_wait(unsigned polls) {
  const unsigned prev = g_tc_refill_limit;
  g_tc_refill_limit = polls < TC_WAIT_LIMIT ? polls : TC_WAIT_LIMIT;
  return prev;
}

int irlcu_sur_forward(irlcu_sur *s, int B, const void *x, float *y) {
  STRY(sur_check_batch(s, B));
  CU_TRY(cudaMemcpyAsync(s->act[0], x, sizeof(bf16) * layer_in_elems(s->L[0], B), cudaMemcpyDeviceToDevice, s->st));
  STRY(sur_forward(*s, B));
  CU_TRY(cudaMemcpyAsync(y, s->out, sizeof(float) * (size_t)B * 128 * 128, cudaMemcpyDeviceToDevice, s->st));
  return sur_tc_status(s->st);
}

int irlcu_sur_gradient(irlcu_sur *s, int B, const void *x, const float *t, float *loss, float *grad_host) {
  STRY(sur_check_batch(s, B));
  CU_TRY(cudaMemcpyAsync(s->act[0], x, sizeof(bf16) * layer_in_elems(s->L[0], B), cudaMemcpyDeviceToDevice, s->st));
  STRY(sur_forward(*s, B));
  STRY(sur_loss(*s, B, t, loss));
  STRY(sur_backward(*s, B));
  STRY(sur_tc_status(s->st));
  if (grad_host) {
    CU_TRY(cudaMemcpyAsync(grad_host, s->g, sizeof(float) * s->nparams, cudaMemcpyDeviceToHost, s->st));
    CU_TRY(cudaStreamSynchronize(s->st));
  }
  return IRLCU_OK;
}

int irlcu_sur_train_step(irlcu_sur *s, int B, const void *x, const float *t, float lr, float *loss) {
  STRY(irlcu_sur_gradient(s, B, x, t, loss, nullptr));
  s->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, (double)s->step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, (double)s->step)));
  k_adam<<<grid_for((long long)s->nparams), 256, 0, s->st>>>(s->w, s->g, s->m, s->v, s->wb, (long long)s->nparams, lr,
                                                             b1, b2, c1, c2, 1e-8f);
  CU_LAUNCHED();
  CU_TRY(cudaStreamSynchronize(s->st));
  return IRLCU_OK;
}

}  // extern "C"
