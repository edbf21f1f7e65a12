// Kernels of the learned surrogate: a U-Net on (N, H, W, C) BF16 activations
// with FP32 accumulation.
//
// conv3x3_kernel is an implicit GEMM on the tensor cores (mma.sync
// m16n8k16, BF16 in, FP32 accumulate): rows are output pixels, columns output
// channels, the reduction runs over (tap, input channel) in chunks of 32,
// staged through shared memory with cp.async double buffering (zero fill at
// the image border). Its epilogue adds the bias and applies GELU, writes the
// pre-activation for the backward pass, and can scale by GELU'(gate) (the
// backward of a preceding GELU). The input gradient of a 3x3 convolution is
// the same kernel on the output gradient with the taps flipped and the
// channel roles swapped (weights packed by unet_pack_weights).
//
// wgrad3x3_kernel is the weight gradient, a GEMM over pixels:
// dW[(tap, ci)][co] = sum_p x[p + tap][ci] g[p][co], split over pixel ranges
// into FP32 partials that reduce_partials_kernel adds in a fixed order.
//
// Activations may be channel slices of a wider buffer (the U-Net's
// concatenations): element (p, c) of a slice is ptr[p * stride + offset + c].
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace clv {
namespace unet {

typedef __nv_bfloat16 bf16;

// GELU(z) = z Phi(z) (exact form, with the error function) and its derivative
__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

struct ConvArgs {
  const bf16* in;
  int in_cs, in_co;  // input channel stride and offset
  const bf16* w;     // [9][Cin][Cout]
  const float* bias;  // Cout, or null
  bf16* out;
  int out_cs, out_co;
  bf16* pre;  // pre-activation [P][Cout], or null
  const bf16* gate;  // scale by gelu_grad(gate[p][c]) (stride gate_cs, offset gate_co), or null
  int gate_cs, gate_co;
  int N, H, W, Cin, Cout;
  int gelu;  // apply GELU to the output
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void ldsm_x4(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ------------------------------------------------------------ conv 3x3
// block: 128 pixels x BN channels, 256 threads; BN = 64: warps 4 x 2 of
// 32 x 32; BN = 32: warps 8 x 1 of 16 x 32. K chunk 32 = (tap, 32 channels).
constexpr int CONV_BM = 128, CONV_BK = 32, A_LD = CONV_BK + 8;

template <int BN> __global__ void __launch_bounds__(256) conv3x3_kernel(ConvArgs a) {
  constexpr int B_LD = BN + 8;
  constexpr int WARPS_M = BN == 64 ? 4 : 8;
  constexpr int WM = CONV_BM / WARPS_M;  // 32 or 16
  constexpr int MI = WM / 16;            // m16 tiles per warp
  __shared__ __align__(16) bf16 sA[2][CONV_BM][A_LD];
  __shared__ __align__(16) bf16 sB[2][CONV_BK][B_LD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WARPS_M, wn = warp / WARPS_M;
  const long long P = (long long)a.N * a.H * a.W;
  const long long m0 = (long long)blockIdx.x * CONV_BM;
  const int n0 = blockIdx.y * BN;
  const int kchunks = 9 * (a.Cin / CONV_BK);
  // this thread's A rows: r = tid / 2, vectors (tid % 2) * 2 + {0, 1}
  const int ar = tid >> 1, av0 = (tid & 1) * 2;
  const long long ap = m0 + ar;
  int an = 0, ah = 0, aw = 0;
  if (ap < P) {
    an = (int)(ap / ((long long)a.H * a.W));
    const int rem = (int)(ap % ((long long)a.H * a.W));
    ah = rem / a.W;
    aw = rem % a.W;
  }
  auto load = [&](int chunk, int buf) {
    const int tap = chunk / (a.Cin / CONV_BK), c0 = (chunk % (a.Cin / CONV_BK)) * CONV_BK;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    const int hh = ah + dy, ww = aw + dx;
    const bool ok = ap < P && hh >= 0 && hh < a.H && ww >= 0 && ww < a.W;
    const bf16* src = ok ? a.in + ((long long)(an * a.H + hh) * a.W + ww) * a.in_cs + a.in_co + c0 : a.in;
#pragma unroll
    for (int v = 0; v < 2; v++) cp_async16(&sA[buf][ar][(av0 + v) * 8], ok ? src + (av0 + v) * 8 : a.in, ok);
    constexpr int BV = BN / 8;  // vectors per B row
    if (tid < CONV_BK * BV) {
      const int br = tid / BV, bv = tid % BV;
      const int col = n0 + bv * 8;
      const bool okb = col < a.Cout;
      const bf16* bsrc = okb ? a.w + ((long long)(tap * a.Cin + c0 + br)) * a.Cout + col : a.w;
      cp_async16(&sB[buf][br][bv * 8], bsrc, okb);
    }
    cp_async_commit();
  };
  float acc[MI][4][4];
#pragma unroll
  for (int i = 0; i < MI; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0f;
  load(0, 0);
  for (int ch = 0; ch < kchunks; ch++) {
    const int buf = ch & 1;
    if (ch + 1 < kchunks) {
      load(ch + 1, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < CONV_BK; ks += 16) {
      uint32_t af[MI][4];
#pragma unroll
      for (int i = 0; i < MI; i++)
        ldsm_x4(af[i][0], af[i][1], af[i][2], af[i][3], &sA[buf][wm * WM + i * 16 + (lane & 15)][ks + (lane >> 4) * 8]);
      uint32_t bfr[4][2];
#pragma unroll
      for (int jj = 0; jj < 2; jj++) {
        uint32_t r0, r1, r2, r3;
        ldsm_x4_t(r0, r1, r2, r3, &sB[buf][ks + (lane & 15)][wn * 32 + jj * 16 + (lane >> 4) * 8]);
        bfr[2 * jj][0] = r0;
        bfr[2 * jj][1] = r1;
        bfr[2 * jj + 1][0] = r2;
        bfr[2 * jj + 1][1] = r3;
      }
#pragma unroll
      for (int i = 0; i < MI; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], af[i], bfr[j][0], bfr[j][1]);
    }
    __syncthreads();
  }
  // epilogue
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int i = 0; i < MI; i++)
#pragma unroll
    for (int h2 = 0; h2 < 2; h2++) {
      const long long p = m0 + wm * WM + i * 16 + g + h2 * 8;
      if (p >= P) continue;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int c = n0 + wn * 32 + j * 8 + t4 * 2;
        if (c >= a.Cout) continue;
        float v0 = acc[i][j][h2 * 2], v1 = acc[i][j][h2 * 2 + 1];
        if (a.bias) {
          v0 += a.bias[c];
          v1 += a.bias[c + 1];
        }
        if (a.gate) {
          const __nv_bfloat162 gz = *reinterpret_cast<const __nv_bfloat162*>(a.gate + p * a.gate_cs + a.gate_co + c);
          v0 *= gelu_grad(__bfloat162float(gz.x));
          v1 *= gelu_grad(__bfloat162float(gz.y));
        }
        if (a.pre)
          *reinterpret_cast<__nv_bfloat162*>(a.pre + p * a.Cout + c) = __floats2bfloat162_rn(v0, v1);
        if (a.gelu) {
          v0 = gelu_f(v0);
          v1 = gelu_f(v1);
        }
        *reinterpret_cast<__nv_bfloat162*>(a.out + p * a.out_cs + a.out_co + c) = __floats2bfloat162_rn(v0, v1);
      }
    }
}

// ------------------------------------------------------------ wgrad 3x3
struct WgradArgs {
  const bf16* x;  // layer input slice
  int x_cs, x_co;
  const bf16* g;  // gradient wrt the pre-activation [P][Cout]
  float* part;    // [S][9 Cin][Cout]
  int N, H, W, Cin, Cout;
  long long pix_per_split;
};
constexpr int WG_BM = 64, WG_BN = 64, WG_BK = 32, WG_LD = 64 + 8;

// grid (ceil(9 Cin / 64), ceil(Cout / 64), S); warps 2 (m) x 4 (n) of 32 x 16
__global__ void __launch_bounds__(256) wgrad3x3_kernel(WgradArgs a) {
  __shared__ __align__(16) bf16 sA[2][WG_BK][WG_LD];  // [pixel][(tap, ci)]
  __shared__ __align__(16) bf16 sB[2][WG_BK][WG_LD];  // [pixel][co]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int M = 9 * a.Cin;
  const int mb = blockIdx.x * WG_BM, nb = blockIdx.y * WG_BN;
  const long long P = (long long)a.N * a.H * a.W;
  const long long p_lo = (long long)blockIdx.z * a.pix_per_split;
  const long long p_hi = p_lo + a.pix_per_split < P ? p_lo + a.pix_per_split : P;
  // this thread loads pixel row r = tid / 8 and vector v = tid % 8 of both tiles
  const int r = tid >> 3, v = tid & 7;
  const int m_v = mb + v * 8;  // 8 consecutive (tap, ci) rows: one tap, as Cin % 8 == 0
  const int tap = m_v < M ? m_v / a.Cin : 0, ci0 = m_v < M ? m_v % a.Cin : 0;
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;
  auto load = [&](long long k0, int buf) {
    const long long p = k0 + r;
    bool okp = p < p_hi;
    int n = 0, h = 0, w = 0;
    if (okp) {
      n = (int)(p / ((long long)a.H * a.W));
      const int rem = (int)(p % ((long long)a.H * a.W));
      h = rem / a.W;
      w = rem % a.W;
    }
    const int hh = h + dy, ww = w + dx;
    const bool oka = okp && m_v < M && hh >= 0 && hh < a.H && ww >= 0 && ww < a.W;
    cp_async16(&sA[buf][r][v * 8],
               oka ? a.x + ((long long)(n * a.H + hh) * a.W + ww) * a.x_cs + a.x_co + ci0 : a.x, oka);
    const int co = nb + v * 8;
    const bool okb = okp && co < a.Cout;
    cp_async16(&sB[buf][r][v * 8], okb ? a.g + p * a.Cout + co : a.g, okb);
    cp_async_commit();
  };
  float acc[2][2][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0f;
  const long long nk = (p_hi - p_lo + WG_BK - 1) / WG_BK;
  if (nk > 0) load(p_lo, 0);
  for (long long kc = 0; kc < nk; kc++) {
    const int buf = (int)(kc & 1);
    if (kc + 1 < nk) {
      load(p_lo + (kc + 1) * WG_BK, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < WG_BK; ks += 16) {
      uint32_t af[2][4];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        // A (m x k) from sA[k][m]: rows k, transposed loads
        const int k = ks + (lane & 7) + ((lane >> 4) << 3);
        const int m = wm * 32 + i * 16 + ((lane >> 3) & 1) * 8;
        ldsm_x4_t(af[i][0], af[i][1], af[i][2], af[i][3], &sA[buf][k][m]);
      }
      uint32_t r0, r1, r2, r3;
      ldsm_x4_t(r0, r1, r2, r3, &sB[buf][ks + (lane & 15)][wn * 16 + (lane >> 4) * 8]);
#pragma unroll
      for (int i = 0; i < 2; i++) {
        mma_bf16(acc[i][0], af[i], r0, r1);
        mma_bf16(acc[i][1], af[i], r2, r3);
      }
    }
    __syncthreads();
  }
  const int g = lane >> 2, t4 = lane & 3;
  float* out = a.part + (long long)blockIdx.z * M * a.Cout;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int h2 = 0; h2 < 2; h2++) {
      const int m = mb + wm * 32 + i * 16 + g + h2 * 8;
      if (m >= M) continue;
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int c = nb + wn * 16 + j * 8 + t4 * 2;
        if (c >= a.Cout) continue;
        out[(long long)m * a.Cout + c] = acc[i][j][h2 * 2];
        out[(long long)m * a.Cout + c + 1] = acc[i][j][h2 * 2 + 1];
      }
    }
}

// out[i] (+)= sum_s part[s][i], in s order
__global__ void reduce_partials_kernel(const float* part, int S, long long n, float* out, int accumulate) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.0f;
  for (int k = 0; k < S; k++) s += part[(long long)k * n + i];
  out[i] = accumulate ? out[i] + s : s;
}

// column sums of g[P][C] (bias gradient): block b sums rows [b*rows, ...) into part[b][C]
__global__ void colsum_kernel(const bf16* g, int g_cs, long long P, int C, long long rows, float* part) {
  const long long p0 = (long long)blockIdx.x * rows;
  const long long p1 = p0 + rows < P ? p0 + rows : P;
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    float s = 0.0f;
    for (long long p = p0; p < p1; p++) s += __bfloat162float(g[p * g_cs + c]);
    part[(long long)blockIdx.x * C + c] = s;
  }
}

// --------------------------------------------------- small layers (CUDA cores)
// first layer: 1 input channel (FP32 image) -> C channels, bias, GELU
__global__ void conv_first_kernel(const float* x, const float* w /*[9][C]*/, const float* bias, int N, int H, int W,
                                  int C, bf16* pre, bf16* out, int out_cs, int out_co) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long P = (long long)N * H * W;
  if (t >= P * C) return;
  const long long p = t / C;
  const int c = (int)(t % C);
  const int n = (int)(p / ((long long)H * W)), rem = (int)(p % ((long long)H * W)), h = rem / W, wq = rem % W;
  float s = bias[c];
  for (int tap = 0; tap < 9; tap++) {
    const int hh = h + tap / 3 - 1, ww = wq + tap % 3 - 1;
    if (hh < 0 || hh >= H || ww < 0 || ww >= W) continue;
    s += x[((long long)n * H + hh) * W + ww] * w[tap * C + c];
  }
  pre[p * C + c] = __float2bfloat16_rn(s);
  out[p * out_cs + out_co + c] = __float2bfloat16_rn(gelu_f(s));
}
// its weight gradient: part[b][tap][c] = sum over pixel block b of x[p + tap] g[p][c]
__global__ void wgrad_first_kernel(const float* x, const bf16* g, int N, int H, int W, int C, long long rows,
                                   float* part) {
  const long long P = (long long)N * H * W;
  const long long p0 = (long long)blockIdx.x * rows, p1 = p0 + rows < P ? p0 + rows : P;
  for (int q = threadIdx.x; q < 9 * C; q += blockDim.x) {
    const int tap = q / C, c = q % C;
    float s = 0.0f;
    for (long long p = p0; p < p1; p++) {
      const int n = (int)(p / ((long long)H * W)), rem = (int)(p % ((long long)H * W));
      const int hh = rem / W + tap / 3 - 1, ww = rem % W + tap % 3 - 1;
      if (hh < 0 || hh >= H || ww < 0 || ww >= W) continue;
      s += x[((long long)n * H + hh) * W + ww] * __bfloat162float(g[p * C + c]);
    }
    part[(long long)blockIdx.x * 9 * C + q] = s;
  }
}

// head: 1x1 convolution C -> K (FP32 out)
__global__ void head_fwd_kernel(const bf16* y, int y_cs, int y_co, const float* w /*[C][K]*/, const float* b,
                                long long P, int C, int K, float* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P * K) return;
  const long long p = t / K;
  const int k = (int)(t % K);
  float s = b[k];
  for (int c = 0; c < C; c++) s += __bfloat162float(y[p * y_cs + y_co + c]) * w[c * K + k];
  out[t] = s;
}
// head backward to its input, times GELU'(z): gy[p][c] = gelu'(z[p][c]) sum_k g[p][k] w[c][k]
__global__ void head_dgrad_kernel(const float* g, const float* w, const bf16* z, long long P, int C, int K, bf16* gz) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P * C) return;
  const long long p = t / C;
  const int c = (int)(t % C);
  float s = 0.0f;
  for (int k = 0; k < K; k++) s += g[p * K + k] * w[c * K + k];
  gz[t] = __float2bfloat16_rn(s * gelu_grad(__bfloat162float(z[t])));
}
// head weight and bias gradients: part[b][c][k] and part[b][C][k] over pixel block b
__global__ void head_wgrad_kernel(const bf16* y, int y_cs, int y_co, const float* g, long long P, int C, int K,
                                  long long rows, float* part) {
  const long long p0 = (long long)blockIdx.x * rows, p1 = p0 + rows < P ? p0 + rows : P;
  for (int q = threadIdx.x; q < (C + 1) * K; q += blockDim.x) {
    const int c = q / K, k = q % K;
    float s = 0.0f;
    for (long long p = p0; p < p1; p++)
      s += (c < C ? __bfloat162float(y[p * y_cs + y_co + c]) : 1.0f) * g[p * K + k];
    part[(long long)blockIdx.x * (C + 1) * K + q] = s;
  }
}

// 2x2 average pooling of a channel slice
__global__ void pool_kernel(const bf16* x, int x_cs, int x_co, int N, int H, int W, int C, bf16* out) {
  const int Ho = H / 2, Wo = W / 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * Ho * Wo * C) return;
  const int c = (int)(t % C);
  const long long q = t / C;
  const int n = (int)(q / ((long long)Ho * Wo)), rem = (int)(q % ((long long)Ho * Wo)), h = rem / Wo, w = rem % Wo;
  float s = 0.0f;
  for (int d = 0; d < 4; d++) {
    const long long p = ((long long)n * H + 2 * h + d / 2) * W + 2 * w + d % 2;
    s += __bfloat162float(x[p * x_cs + x_co + c]);
  }
  out[t] = __float2bfloat16_rn(0.25f * s);
}
// nearest 2x upsampling into a channel slice
__global__ void up_kernel(const bf16* x, int N, int H, int W, int C, bf16* out, int out_cs, int out_co) {
  const int Ho = 2 * H, Wo = 2 * W;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * Ho * Wo * C) return;
  const int c = (int)(t % C);
  const long long q = t / C;
  const int n = (int)(q / ((long long)Ho * Wo)), rem = (int)(q % ((long long)Ho * Wo)), h = rem / Wo, w = rem % Wo;
  out[q * out_cs + out_co + c] = x[(((long long)n * H + h / 2) * W + w / 2) * C + c];
}
// gradient of an encoder output used twice (skip slice of the concatenation
// and input of the pooling): gz = (gcat[p][co + c] + gpool[p/2][c] / 4) gelu'(z)
__global__ void skip_grad_kernel(const bf16* gcat, int gcat_cs, int gcat_co, const bf16* gpool, const bf16* z, int N,
                                 int H, int W, int C, bf16* gz) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * H * W * C) return;
  const int c = (int)(t % C);
  const long long p = t / C;
  const int n = (int)(p / ((long long)H * W)), rem = (int)(p % ((long long)H * W)), h = rem / W, w = rem % W;
  float s = __bfloat162float(gcat[p * gcat_cs + gcat_co + c]);
  if (gpool) s += 0.25f * __bfloat162float(gpool[(((long long)n * (H / 2) + h / 2) * (W / 2) + w / 2) * C + c]);
  gz[t] = __float2bfloat16_rn(s * gelu_grad(__bfloat162float(z[t])));
}
// upsampling backward (sum of the 4 children of a channel slice) times gelu'(z)
__global__ void up_grad_kernel(const bf16* gcat, int gcat_cs, int gcat_co, const bf16* z, int N, int H, int W, int C,
                               bf16* gz) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * H * W * C) return;
  const int c = (int)(t % C);
  const long long q = t / C;
  const int n = (int)(q / ((long long)H * W)), rem = (int)(q % ((long long)H * W)), h = rem / W, w = rem % W;
  float s = 0.0f;
  for (int d = 0; d < 4; d++) {
    const long long p = ((long long)n * 2 * H + 2 * h + d / 2) * (2 * W) + 2 * w + d % 2;
    s += __bfloat162float(gcat[p * gcat_cs + gcat_co + c]);
  }
  gz[t] = __float2bfloat16_rn(s * gelu_grad(__bfloat162float(z[t])));
}

// weighted squared error: loss partials per block, gradient dL/dout
__global__ void mse_kernel(const float* out, const float* target, const float* wch, long long P, int K, float scale,
                           float* grad, float* part) {
  __shared__ float sh[256];
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float s = 0.0f;
  for (long long t = t0; t < P * K; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % K);
    const float d = out[t] - target[t];
    s += wch[k] * d * d;
    grad[t] = 2.0f * wch[k] * d * scale;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0] * scale;
}

// Adam on FP32 master weights (Kingma and Ba, 2015), bias-corrected step size given
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, long long n, float lr_t, float b1, float b2,
                            float eps) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr_t * mi / (sqrtf(vi) + eps);
}

// BF16 weights of a 3x3 layer from FP32 [9][Cin][Cout]: w (same layout) and,
// for the input gradient, wt[tap][co][ci] = w[8 - tap][ci][co]
__global__ void pack_weights_kernel(const float* wf, int Cin, int Cout, bf16* w, bf16* wt) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 9LL * Cin * Cout) return;
  const int co = (int)(t % Cout);
  const long long q = t / Cout;
  const int ci = (int)(q % Cin), tap = (int)(q / Cin);
  const bf16 b = __float2bfloat16_rn(wf[t]);
  w[t] = b;
  wt[((long long)(8 - tap) * Cout + co) * Cin + ci] = b;
}

}  // namespace unet
}  // namespace clv
