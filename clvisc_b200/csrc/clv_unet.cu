// extern "C" entry points of the learned surrogate's kernels (declared in
// include/clvisc_b200.h). No counterpart in the reference.
#include <algorithm>
#include <cstring>
#include <string>

#include <cudaTypedefs.h>

#include "../../include/clvisc_b200.h"
#include "clv_unet.cuh"

namespace clv_host {
int set_error(int code, const std::string& msg);
int check_cuda(const char* where);
}  // namespace clv_host

using namespace clv::unet;

namespace {
inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// the current device (launch set-up is cached per device), or -1
constexpr int kMaxDevices = 64;
inline int current_device() {
  int d = 0;
  return (cudaGetDevice(&d) == cudaSuccess && d >= 0 && d < kMaxDevices) ? d : -1;
}
inline unsigned nb(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }
inline bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
static_assert(sizeof(clv_unet_conv) == sizeof(ConvArgs), "clv_unet_conv layout");

// pixel ranges of the weight-gradient split: enough blocks to fill the GPU
int wgrad_splits(long long P, int Cin, int Cout) {
  const long long tiles = (long long)((9 * Cin + WG_BM - 1) / WG_BM) * ((Cout + WG_BN - 1) / WG_BN);
  long long s = (148 * 4 + tiles - 1) / tiles;
  const long long most = (P + 1023) / 1024;
  if (s > most) s = most;
  if (s < 1) s = 1;
  if (s > 256) s = 256;
  return (int)s;
}
constexpr int kRowBlocks = 148 * 2;

// clv_unet_set_conv_path: 1 tcgen05 convolutions and weight gradient (default), 2 tcgen05 convolutions
// with no-swizzle TMA operands and the mma.sync weight gradient, 3 tcgen05 convolutions and the mma.sync
// weight gradient, 0 mma.sync for both
int g_conv_path = 1;

// cuTensorMapEncodeTiled from the driver (through the runtime, no link-time
// dependency on libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

// pixel-block width of the TMA path, or 0 if the image does not tile into
// 128-pixel blocks
int tma_block_width(const ConvArgs& a) {
  if (a.W % TC_BM == 0) return TC_BM;
  if (TC_BM % a.W == 0 && a.H % (TC_BM / a.W) == 0) return a.W;
  return 0;
}

template <int BN, bool SW> int launch_conv_tma(const ConvArgs& a, int bw, cudaStream_t s) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return clv_host::set_error(CLV_ERR_CUDA, "unet_conv3x3: cuTensorMapEncodeTiled unavailable");
  CUtensorMap ta, tb;
  {  // activations [N][H][W][in_cs] BF16
    const cuuint64_t dims[4] = {(cuuint64_t)a.in_cs, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.N};
    const cuuint64_t strides[3] = {(cuuint64_t)a.in_cs * 2, (cuuint64_t)a.W * a.in_cs * 2,
                                   (cuuint64_t)a.H * a.W * a.in_cs * 2};
    const cuuint32_t box[4] = {SW ? 32u : 8u, (cuuint32_t)bw, (cuuint32_t)(TC_BM / bw), 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(a.in), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, SW ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return clv_host::set_error(CLV_ERR_INVALID, "unet_conv3x3: activation tensor map rejected");
  }
  {  // weights [9 * Cin][Cout] BF16
    const cuuint64_t dims[2] = {(cuuint64_t)a.Cout, (cuuint64_t)9 * a.Cin};
    const cuuint64_t strides[1] = {(cuuint64_t)a.Cout * 2};
    const cuuint32_t box[2] = {SW ? 32u : 8u, TC_BK};
    const cuuint32_t es[2] = {1, 1};
    if (enc(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(a.w), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, SW ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return clv_host::set_error(CLV_ERR_INVALID, "unet_conv3x3: weight tensor map rejected");
  }
  auto kern = conv3x3_tma_kernel<BN, SW>;
  static int grids[kMaxDevices] = {};  // resident CTAs of this device
  const int gdev = current_device();
  if (gdev < 0) return clv_host::check_cuda("cudaGetDevice");
  int& grid = grids[gdev];
  if (!grid) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TmaSmem<BN>)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
      return clv_host::check_cuda("cudaFuncSetAttribute(conv3x3_tma_kernel)");
    // persistent: shared memory (228 KB an SM, 1 KB reserved per block),
    // threads and tensor-memory columns (512 an SM) bound the resident CTAs
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int by_smem = (228 * 1024) / ((int)sizeof(TmaSmem<BN>) + 1024);
    const int per_sm = std::min(std::min(by_smem, 2048 / TMA_THREADS), 512 / (2 * BN));
    grid = sms * std::max(per_sm, 1);
  }
  const long long tiles = (long long)a.N * (a.H / (TC_BM / bw)) * (a.W / bw) * (a.Cout / BN);
  kern<<<(unsigned)std::min<long long>(grid, tiles), TMA_THREADS, sizeof(TmaSmem<BN>), s>>>(ta, tb, a, bw);
  return clv_host::check_cuda("conv3x3_tma_kernel");
}

// the weight gradient on tcgen05 when the pixels tile into 64-pixel blocks
// (bw = min(W, 64) columns) and the channel counts are multiples of 32;
// returns -1 when it does not apply
int wgrad_tma(const WgradArgs& a, float* dw, int accumulate, int max_splits, cudaStream_t s) {
  const int bw = a.W >= WGT_BK ? WGT_BK : a.W;
  if (a.W % bw || WGT_BK % bw || a.H % (WGT_BK / bw) || a.Cin % 32 || a.Cout % 32) return -1;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return -1;
  const int bh = WGT_BK / bw;
  CUtensorMap tg, tx;
  const cuuint32_t box[4] = {32, (cuuint32_t)bw, (cuuint32_t)bh, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  {
    const cuuint64_t dims[4] = {(cuuint64_t)a.Cout, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.N};
    const cuuint64_t strides[3] = {(cuuint64_t)a.Cout * 2, (cuuint64_t)a.W * a.Cout * 2,
                                   (cuuint64_t)a.H * a.W * a.Cout * 2};
    if (enc(&tg, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(a.g), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return clv_host::set_error(CLV_ERR_INVALID, "unet_wgrad3x3: gradient tensor map rejected");
  }
  {
    const cuuint64_t dims[4] = {(cuuint64_t)a.x_cs, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.N};
    const cuuint64_t strides[3] = {(cuuint64_t)a.x_cs * 2, (cuuint64_t)a.W * a.x_cs * 2,
                                   (cuuint64_t)a.H * a.W * a.x_cs * 2};
    if (enc(&tx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(a.x), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return clv_host::set_error(CLV_ERR_INVALID, "unet_wgrad3x3: activation tensor map rejected");
  }
  static bool configured[kMaxDevices] = {};  // launch attributes are per device
  const int cdev = current_device();
  if (cdev < 0) return clv_host::check_cuda("cudaGetDevice");
  if (!configured[cdev]) {
    if (cudaFuncSetAttribute(wgrad3x3_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(WgTmaSmem)) != cudaSuccess)
      return clv_host::check_cuda("cudaFuncSetAttribute(wgrad3x3_tma_kernel)");
    configured[cdev] = true;
  }
  const long long nchunks = (long long)a.N * (a.H / bh) * (a.W / bw);
  const int blocks = ((9 * a.Cin + WGT_BM - 1) / WGT_BM) * ((a.Cout + WGT_BN - 1) / WGT_BN);
  // one wave of resident CTAs (two an SM: shared memory), within the scratch
  // the caller sized for max_splits
  static int residents[kMaxDevices] = {};  // per device: SM counts differ
  const int rdev = current_device();
  if (rdev < 0) return clv_host::check_cuda("cudaGetDevice");
  int& resident = residents[rdev];
  if (!resident) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    resident = std::max(1, sms) * std::max(1, (228 * 1024) / ((int)sizeof(WgTmaSmem) + 1024));
  }
  const long long want = std::max(1, std::min(max_splits, resident / blocks));
  const long long cps = (nchunks + want - 1) / want;
  const int splits = (int)((nchunks + cps - 1) / cps);  // every split has pixel blocks
  WgradArgs b = a;
  wgrad3x3_tma_kernel<<<dim3(blocks, splits), 128, sizeof(WgTmaSmem), s>>>(tg, tx, b, bw, (int)cps);
  int rc = clv_host::check_cuda("wgrad3x3_tma_kernel");
  if (rc) return rc;
  const long long n = 9LL * a.Cin * a.Cout;
  reduce_partials_kernel<<<nb(n, 256), 256, 0, s>>>(a.part, splits, n, dw, accumulate);
  return clv_host::check_cuda("reduce_partials_kernel");
}

template <int BN> int launch_conv_tc(const ConvArgs& a, long long P, cudaStream_t s) {
  auto kern = conv3x3_tc_kernel<BN>;
  static bool configured[kMaxDevices] = {};  // launch attributes are per device
  const int cdev = current_device();
  if (cdev < 0) return clv_host::check_cuda("cudaGetDevice");
  if (!configured[cdev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem<BN>)) !=
        cudaSuccess)
      return clv_host::check_cuda("cudaFuncSetAttribute(conv3x3_tc_kernel)");
    configured[cdev] = true;
  }
  dim3 grid(nb(P, TC_BM), a.Cout / BN);
  kern<<<grid, 128, sizeof(TcSmem<BN>), s>>>(a);
  return clv_host::check_cuda("conv3x3_tc_kernel");
}
}  // namespace

extern "C" {

int clv_unet_conv3x3(const clv_unet_conv* args, void* stream) {
  if (!args) return clv_host::set_error(CLV_ERR_INVALID, "unet_conv3x3: null args");
  ConvArgs a;
  memcpy(&a, args, sizeof(a));
  if (!a.in || !a.w || !a.out || a.N < 1 || a.H < 1 || a.W < 1 || a.Cin % 32 || a.Cout % 32 || a.Cin < 32 ||
      a.in_cs % 8 || a.in_co % 8 || a.out_cs % 2 || a.out_co % 2 || !al16(a.in) || !al16(a.w) ||
      (a.gate && (a.gate_cs % 2 || a.gate_co % 2)))
    return clv_host::set_error(CLV_ERR_INVALID,
                               "unet_conv3x3: Cin and Cout must be multiples of 32, input strides/offsets of 8, "
                               "pointers 16-byte aligned");
  const long long P = (long long)a.N * a.H * a.W;
  if (g_conv_path >= 1) {
    // images that tile into 128-pixel blocks: operands by TMA; others: cp.async
    const int bw = tma_block_width(a);
    if (bw && g_conv_path != 2) {
      if (a.Cout % 128 == 0) return launch_conv_tma<128, true>(a, bw, S(stream));
      if (a.Cout % 64 == 0) return launch_conv_tma<64, true>(a, bw, S(stream));
      return launch_conv_tma<32, true>(a, bw, S(stream));
    }
    if (bw) {
      if (a.Cout % 128 == 0) return launch_conv_tma<128, false>(a, bw, S(stream));
      if (a.Cout % 64 == 0) return launch_conv_tma<64, false>(a, bw, S(stream));
      return launch_conv_tma<32, false>(a, bw, S(stream));
    }
    if (a.Cout % 128 == 0) return launch_conv_tc<128>(a, P, S(stream));
    if (a.Cout % 64 == 0) return launch_conv_tc<64>(a, P, S(stream));
    return launch_conv_tc<32>(a, P, S(stream));
  }
  if (a.Cout % 64 == 0) {
    dim3 grid(nb(P, CONV_BM), a.Cout / 64);
    conv3x3_kernel<64><<<grid, 256, 0, S(stream)>>>(a);
  } else {
    dim3 grid(nb(P, CONV_BM), a.Cout / 32);
    conv3x3_kernel<32><<<grid, 256, 0, S(stream)>>>(a);
  }
  return clv_host::check_cuda("conv3x3_kernel");
}

size_t clv_unet_wgrad_scratch_bytes(int N, int H, int W, int Cin, int Cout) {
  const long long P = (long long)N * H * W;
  return (size_t)wgrad_splits(P, Cin, Cout) * 9 * Cin * Cout * sizeof(float);
}

int clv_unet_wgrad3x3(const void* x, int x_cs, int x_co, const void* g, int N, int H, int W, int Cin, int Cout,
                      float* dw, int accumulate, void* scratch, size_t scratch_bytes, void* stream) {
  if (!x || !g || !dw || !scratch || Cin % 8 || Cout % 8 || x_cs % 8 || x_co % 8 || !al16(x) || !al16(g))
    return clv_host::set_error(CLV_ERR_INVALID, "unet_wgrad3x3: bad argument");
  if (scratch_bytes < clv_unet_wgrad_scratch_bytes(N, H, W, Cin, Cout))
    return clv_host::set_error(CLV_ERR_INVALID, "unet_wgrad3x3: scratch too small");
  WgradArgs a;
  a.x = (const bf16*)x;
  a.x_cs = x_cs;
  a.x_co = x_co;
  a.g = (const bf16*)g;
  a.part = (float*)scratch;
  a.N = N;
  a.H = H;
  a.W = W;
  a.Cin = Cin;
  a.Cout = Cout;
  const long long P = (long long)N * H * W;
  const int s = wgrad_splits(P, Cin, Cout);
  if (g_conv_path == 1) {  // tcgen05 where the pixels tile into 64-pixel blocks
    const int rc = wgrad_tma(a, dw, accumulate, s, S(stream));
    if (rc != -1) return rc;
  }
  a.pix_per_split = (P + s - 1) / s;
  dim3 grid((9 * Cin + WG_BM - 1) / WG_BM, (Cout + WG_BN - 1) / WG_BN, s);
  wgrad3x3_kernel<<<grid, 256, 0, S(stream)>>>(a);
  const long long n = 9LL * Cin * Cout;
  reduce_partials_kernel<<<nb(n, 256), 256, 0, S(stream)>>>(a.part, s, n, dw, accumulate);
  return clv_host::check_cuda("wgrad3x3_kernel");
}

size_t clv_unet_rows_scratch_bytes(int width) { return (size_t)kRowBlocks * width * sizeof(float); }

int clv_unet_bias_grad(const void* g, int g_cs, long long P, int C, float* db, void* scratch, size_t scratch_bytes,
                       void* stream) {
  if (!g || !db || !scratch || scratch_bytes < clv_unet_rows_scratch_bytes(C))
    return clv_host::set_error(CLV_ERR_INVALID, "unet_bias_grad: bad argument");
  const long long rows = (P + kRowBlocks - 1) / kRowBlocks;
  colsum_kernel<<<kRowBlocks, 128, 0, S(stream)>>>((const bf16*)g, g_cs, P, C, rows, (float*)scratch);
  reduce_partials_kernel<<<nb(C, 256), 256, 0, S(stream)>>>((const float*)scratch, kRowBlocks, C, db, 0);
  return clv_host::check_cuda("colsum_kernel");
}

int clv_unet_first_fwd(const float* x, const float* w, const float* bias, int N, int H, int W, int C, void* pre,
                       void* out, int out_cs, int out_co, void* stream) {
  if (!x || !w || !bias || !pre || !out) return clv_host::set_error(CLV_ERR_INVALID, "unet_first_fwd: null");
  const long long n = (long long)N * H * W * C;
  conv_first_kernel<<<nb(n, 256), 256, 0, S(stream)>>>(x, w, bias, N, H, W, C, (bf16*)pre, (bf16*)out, out_cs, out_co);
  return clv_host::check_cuda("conv_first_kernel");
}

int clv_unet_first_wgrad(const float* x, const void* g, int N, int H, int W, int C, float* dw, void* scratch,
                         size_t scratch_bytes, void* stream) {
  if (!x || !g || !dw || !scratch || scratch_bytes < clv_unet_rows_scratch_bytes(9 * C))
    return clv_host::set_error(CLV_ERR_INVALID, "unet_first_wgrad: bad argument");
  const long long P = (long long)N * H * W;
  const long long rows = (P + kRowBlocks - 1) / kRowBlocks;
  wgrad_first_kernel<<<kRowBlocks, 288, 0, S(stream)>>>(x, (const bf16*)g, N, H, W, C, rows, (float*)scratch);
  reduce_partials_kernel<<<nb(9 * C, 256), 256, 0, S(stream)>>>((const float*)scratch, kRowBlocks, 9LL * C, dw, 0);
  return clv_host::check_cuda("wgrad_first_kernel");
}

int clv_unet_head_fwd(const void* y, int y_cs, int y_co, const float* w, const float* b, long long P, int C, int K,
                      float* out, void* stream) {
  if (!y || !w || !b || !out) return clv_host::set_error(CLV_ERR_INVALID, "unet_head_fwd: null");
  head_fwd_kernel<<<nb(P * K, 256), 256, 0, S(stream)>>>((const bf16*)y, y_cs, y_co, w, b, P, C, K, out);
  return clv_host::check_cuda("head_fwd_kernel");
}

int clv_unet_head_bwd(const void* y, int y_cs, int y_co, const void* z, const float* g, const float* w, long long P,
                      int C, int K, void* gz, float* dwb, void* scratch, size_t scratch_bytes, void* stream) {
  if (!y || !z || !g || !w || !gz || !dwb || !scratch || scratch_bytes < clv_unet_rows_scratch_bytes((C + 1) * K))
    return clv_host::set_error(CLV_ERR_INVALID, "unet_head_bwd: bad argument");
  head_dgrad_kernel<<<nb(P * C, 256), 256, 0, S(stream)>>>(g, w, (const bf16*)z, P, C, K, (bf16*)gz);
  const long long rows = (P + kRowBlocks - 1) / kRowBlocks;
  head_wgrad_kernel<<<kRowBlocks, 224, 0, S(stream)>>>((const bf16*)y, y_cs, y_co, g, P, C, K, rows,
                                                       (float*)scratch);
  reduce_partials_kernel<<<nb((C + 1) * K, 256), 256, 0, S(stream)>>>((const float*)scratch, kRowBlocks,
                                                                       (long long)(C + 1) * K, dwb, 0);
  return clv_host::check_cuda("head_bwd");
}

int clv_unet_pool(const void* x, int x_cs, int x_co, int N, int H, int W, int C, void* out, void* stream) {
  if (!x || !out || H % 2 || W % 2) return clv_host::set_error(CLV_ERR_INVALID, "unet_pool: bad argument");
  pool_kernel<<<nb((long long)N * (H / 2) * (W / 2) * C, 256), 256, 0, S(stream)>>>((const bf16*)x, x_cs, x_co, N, H,
                                                                                      W, C, (bf16*)out);
  return clv_host::check_cuda("pool_kernel");
}

int clv_unet_up(const void* x, int N, int H, int W, int C, void* out, int out_cs, int out_co, void* stream) {
  if (!x || !out) return clv_host::set_error(CLV_ERR_INVALID, "unet_up: null");
  up_kernel<<<nb((long long)N * 4 * H * W * C, 256), 256, 0, S(stream)>>>((const bf16*)x, N, H, W, C, (bf16*)out,
                                                                          out_cs, out_co);
  return clv_host::check_cuda("up_kernel");
}

int clv_unet_skip_grad(const void* gcat, int gcat_cs, int gcat_co, const void* gpool, const void* z, int N, int H,
                       int W, int C, void* gz, void* stream) {
  if (!gcat || !z || !gz) return clv_host::set_error(CLV_ERR_INVALID, "unet_skip_grad: null");
  skip_grad_kernel<<<nb((long long)N * H * W * C, 256), 256, 0, S(stream)>>>(
      (const bf16*)gcat, gcat_cs, gcat_co, (const bf16*)gpool, (const bf16*)z, N, H, W, C, (bf16*)gz);
  return clv_host::check_cuda("skip_grad_kernel");
}

int clv_unet_up_grad(const void* gcat, int gcat_cs, int gcat_co, const void* z, int N, int H, int W, int C, void* gz,
                     void* stream) {
  if (!gcat || !z || !gz) return clv_host::set_error(CLV_ERR_INVALID, "unet_up_grad: null");
  up_grad_kernel<<<nb((long long)N * H * W * C, 256), 256, 0, S(stream)>>>((const bf16*)gcat, gcat_cs, gcat_co,
                                                                           (const bf16*)z, N, H, W, C, (bf16*)gz);
  return clv_host::check_cuda("up_grad_kernel");
}

int clv_unet_mse(const float* out, const float* target, const float* wch, long long P, int K, float scale,
                 float* grad, float* part, int nparts, void* stream) {
  if (!out || !target || !wch || !grad || !part || nparts < 1)
    return clv_host::set_error(CLV_ERR_INVALID, "unet_mse: bad argument");
  mse_kernel<<<nparts, 256, 0, S(stream)>>>(out, target, wch, P, K, scale, grad, part);
  return clv_host::check_cuda("mse_kernel");
}

int clv_unet_adam(float* w, const float* g, float* m, float* v, long long n, float lr_t, float b1, float b2,
                  float eps, void* stream) {
  if (!w || !g || !m || !v) return clv_host::set_error(CLV_ERR_INVALID, "unet_adam: null");
  adam_kernel<<<nb(n, 256), 256, 0, S(stream)>>>(w, g, m, v, n, lr_t, b1, b2, eps);
  return clv_host::check_cuda("adam_kernel");
}

int clv_unet_set_conv_path(int path) {
  if (path < 0 || path > 3) return clv_host::set_error(CLV_ERR_INVALID, "unet_set_conv_path: 0, 1, 2 or 3");
  g_conv_path = path;
  return CLV_OK;
}

int clv_unet_timeouts(int* count, int reset) {
  if (!count) return clv_host::set_error(CLV_ERR_INVALID, "unet_timeouts: null");
  if (cudaMemcpyFromSymbol(count, g_tc_timeouts, sizeof(int)) != cudaSuccess)
    return clv_host::check_cuda("unet_timeouts");
  if (reset) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(g_tc_timeouts, &zero, sizeof(int)) != cudaSuccess)
      return clv_host::check_cuda("unet_timeouts");
  }
  return CLV_OK;
}

int clv_unet_pack(const float* wf, int Cin, int Cout, void* w, void* wt, void* stream) {
  if (!wf || !w || !wt) return clv_host::set_error(CLV_ERR_INVALID, "unet_pack: null");
  pack_weights_kernel<<<nb(9LL * Cin * Cout, 256), 256, 0, S(stream)>>>(wf, Cin, Cout, (bf16*)w, (bf16*)wt);
  return clv_host::check_cuda("pack_weights_kernel");
}

}  // extern "C"
