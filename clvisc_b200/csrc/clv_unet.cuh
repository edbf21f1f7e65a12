// Kernels of the learned surrogate: a U-Net on (N, H, W, C) BF16 activations
// with FP32 accumulation.
//
// conv3x3_tma_kernel and conv3x3_tc_kernel (the default path) are implicit
// GEMMs on the 5th-generation tensor cores (tcgen05.mma, accumulator in tensor
// memory), described at the kernels; conv3x3_kernel is the same GEMM on
// mma.sync m16n8k16 (BF16 in, FP32 accumulate), kept as a selectable variant: rows are output pixels, columns output
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
#include <cuda.h>
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

// ------------------------------------------------- conv 3x3, tcgen05 path
// The same implicit GEMM on the 5th-generation tensor cores, for images that
// do not tile into 128-pixel blocks (conv3x3_tma_kernel takes the others). A
// CTA of 128 threads owns 128 output pixels x BN output channels; the FP32
// accumulator (128 lanes x BN columns) lives in tensor memory. Per K chunk of
// 32 (one tap, 32 input channels) the threads stage, with cp.async into a ring
// of TC_STAGES buffers TC_AHEAD chunks ahead, the A tile (pixels x channels,
// K-major 8x16-byte core matrices, zero fill at the image border) and the B
// tile (weights rows of [tap][Cin][Cout], MN-major core matrices); one thread
// issues two tcgen05.mma (M 128, N BN, K 16, BF16 in, FP32 accumulate) and
// commits them to the stage's mbarrier; a stage is refilled once the MMAs
// that read it are done. The epilogue reads the accumulator with tcgen05.ld
// (warp w: lanes 32w..32w+31, one pixel a thread) and applies the same bias /
// gate / GELU as conv3x3_kernel. Every mbarrier wait is bounded; a wait that
// runs out counts in g_tc_timeouts and the kernel stops issuing, waits
// (bounded) for the MMAs it issued and frees its tensor memory.
#ifndef CLV_TC_STAGES
#define CLV_TC_STAGES 4
#endif
#ifndef CLV_TC_AHEAD
#define CLV_TC_AHEAD 2
#endif
constexpr int TC_BM = 128, TC_BK = 32, TC_STAGES = CLV_TC_STAGES, TC_AHEAD = CLV_TC_AHEAD;
static_assert(TC_AHEAD >= 1 && TC_AHEAD < TC_STAGES, "pipeline depth");

__device__ int g_tc_timeouts;  // bounded waits that ran out (read by clv_unet_timeouts)

// shared-memory matrix descriptor: byte offsets lbo (leading-dimension
// stride) and sbo (stride-dimension stride), descriptor version 1 (sm_100),
// layout 0 (no swizzle) or 4 (64-byte swizzle)
__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout = 0) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}
// instruction descriptor of kind::f16: BF16 A and B, FP32 D, A K-major,
// B MN-major, M x N
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); i++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void tc_mma(uint32_t dtm, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtm),
      "l"(da), "l"(db), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }

// the epilogue of one pixel (thread) over 8 accumulator columns starting at
// output channel c0: bias, gate, pre-activation, GELU, BF16 store
__device__ __forceinline__ void tc_epilogue8(const ConvArgs& a, long long p, int c0, const uint32_t (&v)[8]) {
  // 16-byte accesses when every row of 8 channels starts 16-byte aligned
  const bool vec = c0 + 8 <= a.Cout && ((a.out_cs | a.out_co) & 7) == 0 &&
                   ((reinterpret_cast<uintptr_t>(a.out) | reinterpret_cast<uintptr_t>(a.pre) |
                     reinterpret_cast<uintptr_t>(a.gate)) & 15) == 0 &&
                   (!a.gate || ((a.gate_cs | a.gate_co) & 7) == 0);
  if (vec) {
    float f[8];
#pragma unroll
    for (int jj = 0; jj < 8; jj++) f[jj] = __uint_as_float(v[jj]);
    if (a.bias)
#pragma unroll
      for (int jj = 0; jj < 8; jj++) f[jj] += a.bias[c0 + jj];
    if (a.gate) {
      const uint4 g4 = *reinterpret_cast<const uint4*>(a.gate + p * a.gate_cs + a.gate_co + c0);
      const __nv_bfloat162* gz = reinterpret_cast<const __nv_bfloat162*>(&g4);
#pragma unroll
      for (int jj = 0; jj < 4; jj++) {
        f[2 * jj] *= gelu_grad(__bfloat162float(gz[jj].x));
        f[2 * jj + 1] *= gelu_grad(__bfloat162float(gz[jj].y));
      }
    }
    uint4 o;
    __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(&o);
    if (a.pre) {
#pragma unroll
      for (int jj = 0; jj < 4; jj++) ob[jj] = __floats2bfloat162_rn(f[2 * jj], f[2 * jj + 1]);
      *reinterpret_cast<uint4*>(a.pre + p * a.Cout + c0) = o;
    }
    if (a.gelu)
#pragma unroll
      for (int jj = 0; jj < 8; jj++) f[jj] = gelu_f(f[jj]);
#pragma unroll
    for (int jj = 0; jj < 4; jj++) ob[jj] = __floats2bfloat162_rn(f[2 * jj], f[2 * jj + 1]);
    *reinterpret_cast<uint4*>(a.out + p * a.out_cs + a.out_co + c0) = o;
    return;
  }
#pragma unroll
  for (int jj = 0; jj < 8; jj += 2) {
    const int c = c0 + jj;
    if (c >= a.Cout) continue;
    float v0 = __uint_as_float(v[jj]), v1 = __uint_as_float(v[jj + 1]);
    if (a.bias) {
      v0 += a.bias[c];
      v1 += a.bias[c + 1];
    }
    if (a.gate) {
      const __nv_bfloat162 gz = *reinterpret_cast<const __nv_bfloat162*>(a.gate + p * a.gate_cs + a.gate_co + c);
      v0 *= gelu_grad(__bfloat162float(gz.x));
      v1 *= gelu_grad(__bfloat162float(gz.y));
    }
    if (a.pre) *reinterpret_cast<__nv_bfloat162*>(a.pre + p * a.Cout + c) = __floats2bfloat162_rn(v0, v1);
    if (a.gelu) {
      v0 = gelu_f(v0);
      v1 = gelu_f(v1);
    }
    *reinterpret_cast<__nv_bfloat162*>(a.out + p * a.out_cs + a.out_co + c) = __floats2bfloat162_rn(v0, v1);
  }
}
__device__ __forceinline__ void tc_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

template <int BN> struct TcSmem {
  bf16 A[TC_STAGES][TC_BM * TC_BK];
  bf16 B[TC_STAGES][BN * TC_BK];
  uint64_t bar[TC_STAGES];
  uint32_t tmem;
};

template <int BN> __global__ void __launch_bounds__(128) conv3x3_tc_kernel(ConvArgs a) {
  static_assert(BN == 32 || BN == 64 || BN == 128, "BN");
  constexpr int TCOLS = BN;                    // tensor-memory columns (a power of two >= 32)
  constexpr uint32_t LBO_A = TC_BM / 8 * 128;  // A: K-adjacent core matrices (8 channels apart)
  constexpr uint32_t LBO_B = BN / 8 * 128;     // B: K-adjacent core matrices (8 rows apart)
  constexpr uint32_t IDESC = tc_idesc(TC_BM, BN);
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem<BN>& s = *reinterpret_cast<TcSmem<BN>*>(tc_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long P = (long long)a.N * a.H * a.W;
  const long long m0 = (long long)blockIdx.x * TC_BM;
  const int n0 = blockIdx.y * BN;
  const int cpt = a.Cin / TC_BK;  // K chunks per tap
  const int kchunks = 9 * cpt;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s.tmem)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
#pragma unroll
    for (int st = 0; st < TC_STAGES; st++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s.bar[st])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem;

  // this thread's A row (pixel m0 + tid)
  const long long ap = m0 + tid;
  int an = 0, ah = 0, aw = 0;
  if (ap < P) {
    an = (int)(ap / ((long long)a.H * a.W));
    const int rem = (int)(ap % ((long long)a.H * a.W));
    ah = rem / a.W;
    aw = rem % a.W;
  }
  auto load = [&](int chunk, int st) {
    const int tap = chunk / cpt, c0 = (chunk % cpt) * TC_BK;
    const int hh = ah + tap / 3 - 1, ww = aw + tap % 3 - 1;
    const bool ok = ap < P && hh >= 0 && hh < a.H && ww >= 0 && ww < a.W;
    const bf16* src = ok ? a.in + ((long long)(an * a.H + hh) * a.W + ww) * a.in_cs + a.in_co + c0 : a.in;
    unsigned char* A = reinterpret_cast<unsigned char*>(s.A[st]);
#pragma unroll
    for (int v = 0; v < TC_BK / 8; v++)  // core matrix (row group tid/8, channel group v), row tid%8
      cp_async16(A + v * LBO_A + (tid >> 3) * 128 + (tid & 7) * 16, ok ? src + v * 8 : a.in, ok);
    unsigned char* B = reinterpret_cast<unsigned char*>(s.B[st]);
#pragma unroll
    for (int q = tid; q < BN * TC_BK / 8; q += 128) {  // weight row kk, output channels ng*8 .. ng*8+7
      const int kk = q / (BN / 8), ng = q % (BN / 8);
      const int col = n0 + ng * 8;
      const bool okb = col < a.Cout;
      const bf16* bsrc = okb ? a.w + ((long long)(tap * a.Cin + c0 + kk)) * a.Cout + col : a.w;
      cp_async16(B + (kk >> 3) * LBO_B + ng * 128 + (kk & 7) * 16, bsrc, okb);
    }
  };

  bool live = true;  // no bounded wait has run out
#pragma unroll
  for (int c = 0; c < TC_AHEAD; c++) {
    if (c < kchunks) load(c, c);
    cp_async_commit();
  }
  for (int ch = 0; ch < kchunks; ch++) {
    const int st = ch % TC_STAGES;
    const int nxt = ch + TC_AHEAD;
    if (nxt < kchunks) {
      // the stage of chunk nxt was last read by the MMAs of chunk old
      const int old = nxt - TC_STAGES;
      if (old >= 0 && live && !tc_wait(smem_u32(&s.bar[old % TC_STAGES]), (old / TC_STAGES) & 1)) {
        live = false;
        atomicAdd(&g_tc_timeouts, 1);
      }
      if (live) load(nxt, nxt % TC_STAGES);
    }
    cp_async_commit();
    cp_async_wait<TC_AHEAD>();  // chunk ch has landed
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0 && live) {
      tc_fence_after();
      const uint32_t sa = smem_u32(s.A[st]), sb = smem_u32(s.B[st]);
#pragma unroll
      for (int kh = 0; kh < TC_BK / 16; kh++)
        tc_mma(tmem, tc_smem_desc(sa + kh * 2 * LBO_A, LBO_A, 128), tc_smem_desc(sb + kh * 2 * LBO_B, LBO_B, 128),
               IDESC, (ch > 0 || kh > 0) ? 1u : 0u);
      tc_commit(smem_u32(&s.bar[st]));
    }
  }
  cp_async_wait<0>();
  // the last chunk's commit completes when every MMA of the tile has
  const int last = kchunks - 1;
  bool ready = tc_wait(smem_u32(&s.bar[last % TC_STAGES]), (last / TC_STAGES) & 1);
  if (!ready) atomicAdd(&g_tc_timeouts, 1);
  tc_fence_after();
  live = live && ready;
  live = __syncthreads_and(live);

  if (live) {
    const long long p = m0 + warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c8 = 0; c8 < BN / 8; c8++) {
      uint32_t v[8];
      tc_ld8(trow + c8 * 8, v);
      if (p < P) tc_epilogue8(a, p, n0 + c8 * 8, v);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
  }
}

// ------------------------------------------ conv 3x3, TMA + tcgen05 path
// For images that tile evenly into blocks of 128 pixels (W divides 128 and H
// is a multiple of 128 / W, or W is a multiple of 128). Persistent and warp
// specialised: a CTA of 6 warps takes tiles (a (128 / bw) x bw pixel block of
// one image, BN output channels) blockIdx.x, blockIdx.x + gridDim.x, ...
//   * warp 0 (one thread) loads each K chunk (one tap, 32 input channels)
//     with the tensor memory accelerator into a ring of TC_STAGES stages, the
//     image border as TMA's zero fill. With SW (the default), one box of
//     [32 channels, bw, 128 / bw, 1] of the activation tensor at the tap's
//     offset lands as the K-major operand in the 64-byte swizzled layout
//     (128 pixel rows of 64 bytes; 8-row atoms 512 bytes apart) and BN / 32
//     boxes of [32 output channels, 32 rows] of the weights as the MN-major
//     operand in the same swizzle; without SW, boxes 16 bytes wide fill the
//     no-swizzle core-matrix layouts (four [8, bw, 128 / bw, 1] activation
//     boxes, BN / 8 [8, 32] weight boxes);
//   * warp 1 (one thread) issues the chunk's two tcgen05.mma (M 128, N BN,
//     K 16) into one of two tensor-memory accumulators, commits them to the
//     stage's empty barrier and, after a tile's last chunk, to the
//     accumulator's full barrier;
//   * warps 2-5 drain a full accumulator (warp w: lanes 32 (w % 4) ..,
//     one pixel a thread) through the bias / gate / GELU epilogue while the
//     next tile accumulates in the other one, then free it.
// Every wait is bounded (g_tc_timeouts); a role whose wait runs out stops.
constexpr int TMA_THREADS = 192;

template <int BN> struct TmaSmem {
  bf16 A[TC_STAGES][TC_BM * TC_BK];
  bf16 B[TC_STAGES][BN * TC_BK];
  uint64_t full[TC_STAGES], empty[TC_STAGES], acc_full[2], acc_empty[2];
  uint32_t tmem;
};

__device__ __forceinline__ void tma_load4(uint32_t dst, const void* map, int c0, int c1, int c2, int c3, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(
          dst),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_load2(uint32_t dst, const void* map, int c0, int c1, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(map), "r"(c0), "r"(c1), "r"(bar)
      : "memory");
}

template <int BN, bool SW>
__global__ void __launch_bounds__(TMA_THREADS)
    conv3x3_tma_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, ConvArgs a, int bw) {
  static_assert(BN == 32 || BN == 64 || BN == 128, "BN");
  constexpr int TCOLS = 2 * BN;  // two accumulators
  constexpr uint32_t A_BYTES = TC_BM * TC_BK * 2, B_BYTES = BN * TC_BK * 2;
  // no swizzle: A 8-channel groups (LBO) 2048 B apart, 8-row groups (SBO) 128 B; B 8-row groups (LBO) 128 B,
  // 8-channel groups (SBO) 512 B. 64-byte swizzle: A 8-row atoms (SBO) 512 B apart, K step of 16 channels
  // +32 B; B 32-channel groups (LBO) 2048 B apart, 8-row atoms (SBO) 512 B, K step of 16 rows +1024 B
  constexpr uint32_t LAYOUT = SW ? 4u : 0u;
  constexpr uint32_t LBO_A = SW ? 16 : TC_BM * 16, SBO_A = SW ? 512 : 128;
  constexpr uint32_t LBO_B = SW ? 2048 : 128, SBO_B = SW ? 512 : TC_BK * 16;
  constexpr uint32_t KSTEP_A = SW ? 32 : 2 * TC_BM * 16, KSTEP_B = SW ? 1024 : 2 * 128;
  constexpr uint32_t IDESC = tc_idesc(TC_BM, BN);
  extern __shared__ __align__(1024) unsigned char tma_raw[];
  TmaSmem<BN>& s = *reinterpret_cast<TmaSmem<BN>*>(tma_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int bh = TC_BM / bw;
  const int tiles_w = a.W / bw, tiles_h = a.H / bh;
  const int ntn = a.Cout / BN;
  const long long ntiles = (long long)a.N * tiles_h * tiles_w * ntn;
  const int cpt = a.Cin / TC_BK, kchunks = 9 * cpt;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s.tmem)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 32) {
#pragma unroll
    for (int st = 0; st < TC_STAGES; st++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s.full[st])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s.empty[st])) : "memory");
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s.acc_full[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;\n" ::"r"(smem_u32(&s.acc_empty[q])) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem;

  // tile q -> (image, pixel block, output-channel block); channel blocks of
  // one pixel block are consecutive, so they share its activations in L2
  auto tile = [&](long long q, int& img, int& h0, int& w0, int& n0) {
    n0 = (int)(q % ntn) * BN;
    q /= ntn;
    w0 = (int)(q % tiles_w) * bw;
    q /= tiles_w;
    h0 = (int)(q % tiles_h) * bh;
    img = (int)(q / tiles_h);
  };

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      long long it = 0;
      bool ok = true;
      for (long long q = blockIdx.x; q < ntiles && ok; q += gridDim.x) {
        int img, h0, w0, n0;
        tile(q, img, h0, w0, n0);
        for (int ch = 0; ch < kchunks; ch++, it++) {
          const int st = (int)(it % TC_STAGES);
          const long long j = it / TC_STAGES;
          if (j >= 1 && !tc_wait(smem_u32(&s.empty[st]), (uint32_t)((j - 1) & 1))) {
            ok = false;
            atomicAdd(&g_tc_timeouts, 1);
            break;
          }
          const int tap = ch / cpt, c0 = (ch % cpt) * TC_BK;
          const uint32_t fb = smem_u32(&s.full[st]);
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(A_BYTES + B_BYTES)
                       : "memory");
          const uint32_t sa = smem_u32(s.A[st]), sb = smem_u32(s.B[st]);
          if (SW) {
            tma_load4(sa, &ta, a.in_co + c0, w0 + tap % 3 - 1, h0 + tap / 3 - 1, img, fb);
#pragma unroll
            for (int ng = 0; ng < BN / 32; ng++) tma_load2(sb + ng * 2048, &tb, n0 + 32 * ng, tap * a.Cin + c0, fb);
          } else {
#pragma unroll
            for (int g = 0; g < TC_BK / 8; g++)
              tma_load4(sa + g * TC_BM * 16, &ta, a.in_co + c0 + 8 * g, w0 + tap % 3 - 1, h0 + tap / 3 - 1, img, fb);
#pragma unroll
            for (int ng = 0; ng < BN / 8; ng++)
              tma_load2(sb + ng * TC_BK * 16, &tb, n0 + 8 * ng, tap * a.Cin + c0, fb);
          }
        }
      }
      // the loads in flight land before the CTA can exit
      for (long long c = it - 1; c >= 0 && c >= it - TC_STAGES; c--)
        tc_wait(smem_u32(&s.full[c % TC_STAGES]), (uint32_t)((c / TC_STAGES) & 1));
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      long long it = 0;
      int t = 0;
      bool ok = true;
      for (long long q = blockIdx.x; q < ntiles && ok; q += gridDim.x, t++) {
        const int acc = t & 1;
        if (t >= 2 && !tc_wait(smem_u32(&s.acc_empty[acc]), (uint32_t)(((t >> 1) - 1) & 1))) {
          ok = false;
          atomicAdd(&g_tc_timeouts, 1);
          break;
        }
        tc_fence_after();
        const uint32_t dtm = tmem + acc * BN;
        for (int ch = 0; ch < kchunks; ch++, it++) {
          const int st = (int)(it % TC_STAGES);
          if (!tc_wait(smem_u32(&s.full[st]), (uint32_t)((it / TC_STAGES) & 1))) {
            ok = false;
            atomicAdd(&g_tc_timeouts, 1);
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(s.A[st]), sb = smem_u32(s.B[st]);
#pragma unroll
          for (int kh = 0; kh < TC_BK / 16; kh++)
            tc_mma(dtm, tc_smem_desc(sa + kh * KSTEP_A, LBO_A, SBO_A, LAYOUT),
                   tc_smem_desc(sb + kh * KSTEP_B, LBO_B, SBO_B, LAYOUT), IDESC, (ch > 0 || kh > 0) ? 1u : 0u);
          tc_commit(smem_u32(&s.empty[st]));
        }
        if (ok) tc_commit(smem_u32(&s.acc_full[acc]));
      }
    }
  } else {  // epilogue warps 2-5
    const int quarter = warp & 3;  // tensor-memory lanes 32 quarter .. 32 quarter + 31
    const int r = quarter * 32 + lane;
    int t = 0;
    for (long long q = blockIdx.x; q < ntiles; q += gridDim.x, t++) {
      const int acc = t & 1;
      const bool ok = __all_sync(0xffffffffu, tc_wait(smem_u32(&s.acc_full[acc]), (uint32_t)((t >> 1) & 1)));
      if (!ok) {
        if (lane == 0) atomicAdd(&g_tc_timeouts, 1);
        break;
      }
      tc_fence_after();
      int img, h0, w0, n0;
      tile(q, img, h0, w0, n0);
      const long long p = ((long long)img * a.H + h0 + r / bw) * a.W + w0 + r % bw;
      const uint32_t trow = tmem + ((uint32_t)(quarter * 32) << 16) + acc * BN;
#pragma unroll 1
      for (int c8 = 0; c8 < BN / 8; c8++) {
        uint32_t v[8];
        tc_ld8(trow + c8 * 8, v);
        tc_epilogue8(a, p, n0 + c8 * 8, v);
      }
      tc_fence_before();
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&s.acc_empty[acc])) : "memory");
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
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
// ------------------------------------------ wgrad 3x3, TMA + tcgen05 path
// (the default path; wgrad3x3_kernel takes images that do not tile and the
// mma.sync paths.) The weight gradient on the
// 5th-generation tensor cores, for images whose pixels tile into blocks of 32
// (bw = min(W, 64) columns x 64 / bw rows):
// D[(tap, ci)][co] = sum over pixels p of x[p + tap][ci] g[p][co], the rows
// r = tap * Cin + ci of the [9 Cin][Cout] result in tiles of M = 128 (four
// 32-channel groups, each a [32 channels, bw, 64 / bw, 1] box of x shifted by
// its tap, the image border as zero fill), N = up to 128 output channels
// ([32, bw, 64 / bw, 1] boxes of g), K = 64-pixel blocks; both operands are
// MN-major in the 64-byte swizzled layout. A CTA of 128 threads takes one
// (row tile, channel tile) and a contiguous range of pixel blocks (split K):
// thread 0 loads with TMA into WGT_STAGES stages, thread 32 issues the
// tcgen05.mma and commits each stage back, and all four warps write the
// accumulator (one row a thread) as an FP32 partial [split][9 Cin][Cout] that
// reduce_partials_kernel adds in a fixed order.
constexpr int WGT_BM = 128, WGT_BN = 128, WGT_BK = 64, WGT_STAGES = 3;

struct WgTmaSmem {
  bf16 A[WGT_STAGES][WGT_BM * WGT_BK];
  bf16 B[WGT_STAGES][WGT_BN * WGT_BK];
  uint64_t full[WGT_STAGES], empty[WGT_STAGES], done;
  uint32_t tmem;
};

__global__ void __launch_bounds__(128)
    wgrad3x3_tma_kernel(const __grid_constant__ CUtensorMap tg, const __grid_constant__ CUtensorMap tx, WgradArgs a,
                        int bw, int chunks_per_split) {
  // MN-major, 64-byte swizzle: 32-channel groups (one box each) WGT_BK x 64 B apart, 8-row atoms 512 B,
  // K step of 16 pixel rows 1024 B
  constexpr uint32_t LBO = WGT_BK * 64, SBO = 512, KSTEP = 1024, LAYOUT = 4;
  extern __shared__ __align__(1024) unsigned char wgt_raw[];
  WgTmaSmem& s = *reinterpret_cast<WgTmaSmem*>(wgt_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int rows = 9 * a.Cin;
  const int mblocks = (rows + WGT_BM - 1) / WGT_BM;
  const int m0 = (blockIdx.x % mblocks) * WGT_BM, co0 = (blockIdx.x / mblocks) * WGT_BN;
  const int nn = min(WGT_BN, a.Cout - co0);        // a multiple of 32
  const int groups = min(4, (rows - m0) / 32);     // 32-row groups with data
  const int split = blockIdx.y;
  const int bh = WGT_BK / bw;
  const int per_row = a.W / bw, per_img = per_row * (a.H / bh);
  const long long nchunks = (long long)a.N * per_img;
  const long long c0 = (long long)split * chunks_per_split;
  const long long c1 = min(nchunks, c0 + chunks_per_split);
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(nn >> 3) << 17) |
                         ((uint32_t)(WGT_BM >> 4) << 24);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s.tmem)),
                 "r"(WGT_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 32) {
#pragma unroll
    for (int st = 0; st < WGT_STAGES; st++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s.full[st])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s.empty[st])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s.done)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem;

  if (tid == 0) {  // TMA producer
    long long it = 0;
    for (long long c = c0; c < c1; c++, it++) {
      const int st = (int)(it % WGT_STAGES);
      const long long j = it / WGT_STAGES;
      if (j >= 1 && !tc_wait(smem_u32(&s.empty[st]), (uint32_t)((j - 1) & 1))) {
        atomicAdd(&g_tc_timeouts, 1);
        break;
      }
      const int img = (int)(c / per_img), q = (int)(c % per_img);
      const int h0 = (q / per_row) * bh, w0 = (q % per_row) * bw;
      const uint32_t fb = smem_u32(&s.full[st]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb),
                   "r"((uint32_t)(groups * 32 + nn) * WGT_BK * 2)
                   : "memory");
      const uint32_t sa = smem_u32(s.A[st]), sb = smem_u32(s.B[st]);
      for (int gi = 0; gi < groups; gi++) {  // rows m0 + 32 gi ..: one tap, 32 input channels
        const int r0 = m0 + 32 * gi, tap = r0 / a.Cin, ci = r0 % a.Cin;
        tma_load4(sa + gi * LBO, &tx, a.x_co + ci, w0 + tap % 3 - 1, h0 + tap / 3 - 1, img, fb);
      }
      for (int ng = 0; ng < nn / 32; ng++) tma_load4(sb + ng * LBO, &tg, co0 + 32 * ng, w0, h0, img, fb);
    }
    // the loads in flight land before the CTA can exit
    for (long long c = it - 1; c >= 0 && c >= it - WGT_STAGES; c--)
      tc_wait(smem_u32(&s.full[c % WGT_STAGES]), (uint32_t)((c / WGT_STAGES) & 1));
  } else if (tid == 32) {  // MMA issuer
    long long it = 0;
    bool ok = true;
    for (long long c = c0; c < c1; c++, it++) {
      const int st = (int)(it % WGT_STAGES);
      if (!tc_wait(smem_u32(&s.full[st]), (uint32_t)((it / WGT_STAGES) & 1))) {
        ok = false;
        atomicAdd(&g_tc_timeouts, 1);
        break;
      }
      tc_fence_after();
      const uint32_t sa = smem_u32(s.A[st]), sb = smem_u32(s.B[st]);
#pragma unroll
      for (int kh = 0; kh < WGT_BK / 16; kh++)
        tc_mma(tmem, tc_smem_desc(sa + kh * KSTEP, LBO, SBO, LAYOUT), tc_smem_desc(sb + kh * KSTEP, LBO, SBO, LAYOUT),
               idesc, (it > 0 || kh > 0) ? 1u : 0u);
      tc_commit(smem_u32(&s.empty[st]));
    }
    if (ok && c1 > c0) tc_commit(smem_u32(&s.done));
  }
  bool ready = c1 > c0 ? tc_wait(smem_u32(&s.done), 0) : true;
  tc_fence_after();
  ready = __syncthreads_and(ready);
  if (!ready && tid == 0) atomicAdd(&g_tc_timeouts, 1);
  if (ready) {
    const int r = m0 + warp * 32 + lane;  // (tap, ci) row of this thread
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    float* out = a.part + ((long long)split * rows + r) * a.Cout + co0;
#pragma unroll 1
    for (int c8 = 0; c8 < nn / 8; c8++) {
      uint32_t v[8];
      tc_ld8(trow + c8 * 8, v);
      if (r < rows) {
        float4 lo, hi;
        const bool any = c1 > c0;
        lo.x = any ? __uint_as_float(v[0]) : 0.0f;
        lo.y = any ? __uint_as_float(v[1]) : 0.0f;
        lo.z = any ? __uint_as_float(v[2]) : 0.0f;
        lo.w = any ? __uint_as_float(v[3]) : 0.0f;
        hi.x = any ? __uint_as_float(v[4]) : 0.0f;
        hi.y = any ? __uint_as_float(v[5]) : 0.0f;
        hi.z = any ? __uint_as_float(v[6]) : 0.0f;
        hi.w = any ? __uint_as_float(v[7]) : 0.0f;
        *reinterpret_cast<float4*>(out + c8 * 8) = lo;
        *reinterpret_cast<float4*>(out + c8 * 8 + 4) = hi;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(WGT_BN));
  }
}

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
