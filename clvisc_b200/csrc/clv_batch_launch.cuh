// Launchers of the batched stage kernels, shared by the exact translation
// unit (clv_batch.cu) and the tolerance-arithmetic one (clv_fast.cu): each
// instantiates the kernels of its own arithmetic (clv::exact or clv::fast).
#pragma once
#include <string>

#include "clv_batch.cuh"

namespace clv_host {
int set_error(int code, const std::string& msg);
int check_cuda(const char* where);
}  // namespace clv_host

namespace clv {
inline namespace CLV_ARITH {
namespace batch_launch {

// the current device (launch set-up is cached per device), or -1
constexpr int kMaxDevices = 64;
inline int current_device() {
  int d = 0;
  return (cudaGetDevice(&d) == cudaSuccess && d >= 0 && d < kMaxDevices) ? d : -1;
}

template <class real, bool BULK, int BS, int MINB>
int launch_stage(const Params& p, const BatchArgs<real>& a, int step, int grid, cudaStream_t s) {
  auto kern = batch_stage_kernel<real, BULK, BS, MINB>;
  if (grid <= 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BS, 0);
    grid = sms * (per_sm > 0 ? per_sm : 1);
  }
  kern<<<grid, BS, 0, s>>>(p, a, step);
  return clv_host::check_cuda("batch_stage_kernel");
}

// the register caps are offered in FP32 only (FP64 spills heavily under
// them): 128 registers a thread (512 threads per SM) or, for 64- and
// 128-thread blocks, 168 (384 threads per SM)
template <class real> constexpr int capped_minb(int bs) { return sizeof(real) == 4 ? 512 / bs : 1; }
template <class real> constexpr int capped168_minb(int bs) { return sizeof(real) == 4 ? 384 / bs : 1; }

template <class real, bool BULK>
int stage_bs(const Params& p, const BatchArgs<real>& a, int step, int bs, int grid, int cap,
             cudaStream_t s) {
  if (cap && sizeof(real) == 8) return clv_host::set_error(CLV_ERR_INVALID, "batch: max_registers is FP32 only");
  if (cap == 168 && bs == 256)
    return clv_host::set_error(CLV_ERR_INVALID, "batch: max_registers 168 needs 64- or 128-thread blocks");
  if (bs == 64 && cap == 168) return launch_stage<real, BULK, 64, capped168_minb<real>(64)>(p, a, step, grid, s);
  if (bs == 128 && cap == 168) return launch_stage<real, BULK, 128, capped168_minb<real>(128)>(p, a, step, grid, s);
  if (bs == 64)
    return cap ? launch_stage<real, BULK, 64, capped_minb<real>(64)>(p, a, step, grid, s)
               : launch_stage<real, BULK, 64, 1>(p, a, step, grid, s);
  if (bs == 128)
    return cap ? launch_stage<real, BULK, 128, capped_minb<real>(128)>(p, a, step, grid, s)
               : launch_stage<real, BULK, 128, 1>(p, a, step, grid, s);
  if (bs == 256)
    return cap ? launch_stage<real, BULK, 256, capped_minb<real>(256)>(p, a, step, grid, s)
               : launch_stage<real, BULK, 256, 1>(p, a, step, grid, s);
  return clv_host::set_error(CLV_ERR_INVALID, "batch: block_size must be 64, 128 or 256");
}

template <class real, bool BULK, int TB>
int launch_tiled(const Params& p, const BatchArgs<real>& a, int step, int chunk, int grid, cudaStream_t s) {
  typedef Tile2Smem<real, BULK, TB> SM;
  auto kern = batch_tiled2d_kernel<real, BULK, TB, tiled2d_minb<real, TB>()>;
  static bool configured[kMaxDevices] = {};  // launch attributes are per device
  const int cdev = current_device();
  if (cdev < 0) return clv_host::check_cuda("cudaGetDevice");
  if (!configured[cdev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SM)) != cudaSuccess)
      return clv_host::check_cuda("cudaFuncSetAttribute(batch_tiled2d_kernel)");
    configured[cdev] = true;
  }
  if (grid <= 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TB, sizeof(SM));
    grid = sms * (per_sm > 0 ? per_sm : 1);
  }
  kern<<<grid, TB, sizeof(SM), s>>>(p, a, step, chunk);
  return clv_host::check_cuda("batch_tiled2d_kernel");
}

// resident blocks per SM of the stage kernel of one launch shape (this also
// loads the kernel and, for the tiled one, raises its shared-memory limit, so
// that a later stream capture needs neither)
template <class real, bool BULK>
int occupancy(int bs, int cap, int* n) {
  const void* f = nullptr;
  if (bs == 64) f = cap == 168 ? (const void*)batch_stage_kernel<real, BULK, 64, capped168_minb<real>(64)>
                 : cap ? (const void*)batch_stage_kernel<real, BULK, 64, capped_minb<real>(64)>
                       : (const void*)batch_stage_kernel<real, BULK, 64, 1>;
  else if (bs == 128) f = cap == 168 ? (const void*)batch_stage_kernel<real, BULK, 128, capped168_minb<real>(128)>
                     : cap ? (const void*)batch_stage_kernel<real, BULK, 128, capped_minb<real>(128)>
                           : (const void*)batch_stage_kernel<real, BULK, 128, 1>;
  else f = cap ? (const void*)batch_stage_kernel<real, BULK, 256, capped_minb<real>(256)>
               : (const void*)batch_stage_kernel<real, BULK, 256, 1>;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, f, bs, 0) != cudaSuccess)
    return clv_host::check_cuda("batch_occupancy");
  return 0;
}
template <class real, bool BULK, int TB> int occupancy_tiled(int* n) {
  typedef Tile2Smem<real, BULK, TB> SM;
  auto kern = batch_tiled2d_kernel<real, BULK, TB, tiled2d_minb<real, TB>()>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SM)) != cudaSuccess)
    return clv_host::check_cuda("cudaFuncSetAttribute(batch_tiled2d_kernel)");
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, kern, TB, sizeof(SM)) != cudaSuccess)
    return clv_host::check_cuda("batch_occupancy_tiled");
  return 0;
}

template <class real>
int stage_tiled(const Params& p, const BatchArgs<real>& a, int step, int rows, int chunk, int grid, cudaStream_t s) {
  const bool bulk = p.flags & FLAG_BULK;
  if (rows == 64)
    return bulk ? launch_tiled<real, true, 64>(p, a, step, chunk, grid, s)
                : launch_tiled<real, false, 64>(p, a, step, chunk, grid, s);
  return bulk ? launch_tiled<real, true, 128>(p, a, step, chunk, grid, s)
              : launch_tiled<real, false, 128>(p, a, step, chunk, grid, s);
}

}  // namespace batch_launch
}  // namespace CLV_ARITH
}  // namespace clv
