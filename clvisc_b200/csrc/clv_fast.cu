// The fused viscous stage in tolerance arithmetic (CLV_FLAG_FAST).
//
// This translation unit compiles the same stage headers as the exact build
// with CLV_FAST=1 and --fmad=true -prec-div=false -prec-sqrt=false, which
// selects the fast branches of clv_device.cuh (division by run constants as a
// product with the reciprocal, sign-test minmod, the KT speed max(lambda, 1)
// as 1, one atomic per warp and event for the max energy density). Its functions and kernels live in clv::fast, so
// they link beside the exact ones in clv::exact. The batched stage kernels
// (clv_batch.cuh) come in this arithmetic too.
#define CLV_FAST 1
#include <string>

#include "../../include/clvisc_b200.h"
#include "clv_fast.h"
#include "clv_batch_launch.cuh"
#include "clv_stage_tiled.cuh"

namespace clv_fastpath {
namespace {

constexpr int kTiledMinNz = 24;  // fewer cells along eta: per-cell kernel

// per-device "dynamic shared memory raised" flags of each tiled instantiation
constexpr int kMaxDev = 64;

template <class real, bool CPL, int MINB, int TJ, int TK>
int launch_tiled(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, const clv::TauConst<real>& tc,
                 int chunk, cudaStream_t s) {
  typedef clv::TileSmem<real, TJ, TK> SM;
  auto kern = clv::visc_stage_tiled_kernel<real, true, true, CPL, TJ, TK, MINB>;
  static bool configured[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return clv_host::check_cuda("cudaGetDevice");
  if (!configured[dev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SM)) != cudaSuccess)
      return clv_host::check_cuda("cudaFuncSetAttribute(fast visc_stage_tiled_kernel)");
    configured[dev] = true;
  }
  dim3 grid((p.nz + TK - 1) / TK, (p.ny + TJ - 1) / TJ, (p.nx + chunk - 1) / chunk);
  kern<<<grid, TJ * TK, sizeof(SM), s>>>(p, v, step, tc, chunk);
  return clv_host::check_cuda("fast visc_stage_tiled_kernel");
}

template <class real, bool BULK, int TB>
int launch_tiled2d(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, const clv::TauConst<real>& tc,
                   int chunk, cudaStream_t s) {
  typedef clv::Tile2Smem<real, BULK, TB> SM;
  auto kern = clv::visc_stage_tiled2d_kernel<real, BULK, TB, clv::tiled2d_minb<real, TB>()>;
  static bool configured[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return clv_host::check_cuda("cudaGetDevice");
  if (!configured[dev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SM)) != cudaSuccess)
      return clv_host::check_cuda("cudaFuncSetAttribute(fast visc_stage_tiled2d_kernel)");
    configured[dev] = true;
  }
  dim3 grid((p.ny + TB - 5) / (TB - 4), (p.nx + chunk - 1) / chunk);
  kern<<<grid, TB, sizeof(SM), s>>>(p, v, step, tc, chunk);
  return clv_host::check_cuda("fast visc_stage_tiled2d_kernel");
}

}  // namespace

template <class real>
int visc_stage(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, const clv::TauConst<real>& tc,
               const clv::StageOpts& o, cudaStream_t s) {
  const bool bulk = p.flags & clv::FLAG_BULK;
  const bool cpl = p.flags & (clv::FLAG_GUBSER_VISC | clv::FLAG_PIMN_OMEGA | clv::FLAG_OMEGA_OMEGA);
  if (o.chunk < 1) return clv_host::set_error(CLV_ERR_INVALID, "fast visc stage: chunk must be >= 1");
  if (!bulk && (o.stage_kernel == 2 || (o.stage_kernel != 1 && p.nz >= kTiledMinNz))) {
    if (cpl) return launch_tiled<real, true, 1, 8, 32>(p, v, step, tc, o.chunk, s);
    // 16 x 16 and 8 x 16 (y, eta) tiles as in the exact build (CLV_OPT_TILE 1, 2)
    if (o.tile == 1) {
      if (sizeof(real) == 8 || o.minb == 1) return launch_tiled<real, false, 1, 16, 16>(p, v, step, tc, o.chunk, s);
      if constexpr (sizeof(real) == 4) return launch_tiled<real, false, 2, 16, 16>(p, v, step, tc, o.chunk, s);
    }
    if (o.tile == 2) {
      if (sizeof(real) == 8 || o.minb == 1) return launch_tiled<real, false, 2, 8, 16>(p, v, step, tc, o.chunk, s);
      if constexpr (sizeof(real) == 4) return launch_tiled<real, false, 4, 8, 16>(p, v, step, tc, o.chunk, s);
    }
    if constexpr (sizeof(real) == 8) return launch_tiled<real, false, 1, 8, 32>(p, v, step, tc, o.chunk, s);
    else {
      // 16 x 32 (y, eta) tiles, one 512-thread CTA an SM: less halo than two 8 x 32 CTAs
      if (o.tile == 3) return launch_tiled<real, false, 1, 16, 32>(p, v, step, tc, o.chunk, s);
      if (o.minb == 1) return launch_tiled<real, false, 1, 8, 32>(p, v, step, tc, o.chunk, s);
      return launch_tiled<real, false, 2, 8, 32>(p, v, step, tc, o.chunk, s);
    }
  }
  // (2+1)D grids: the tiled (2+1)D kernel (CLV_OPT_STAGE_KERNEL 3), with
  // or without the bulk sector; not the coupling terms
  if (p.nz == 1 && !cpl && o.stage_kernel == 3) {
    if (o.chunk2d < 1) return clv_host::set_error(CLV_ERR_INVALID, "fast visc stage: chunk2d must be >= 1");
    if (o.rows2d == 128)
      return bulk ? launch_tiled2d<real, true, 128>(p, v, step, tc, o.chunk2d, s)
                  : launch_tiled2d<real, false, 128>(p, v, step, tc, o.chunk2d, s);
    return bulk ? launch_tiled2d<real, true, 64>(p, v, step, tc, o.chunk2d, s)
                : launch_tiled2d<real, false, 64>(p, v, step, tc, o.chunk2d, s);
  }
  // one thread per cell: (2+1)D grids, short eta axes, the bulk sector
  const int bs = 128;
  const long long n = (long long)p.nx * p.ny * p.nz;
  dim3 grid((unsigned int)((n + bs - 1) / bs));
  if (bulk) {
    if (cpl) clv::visc_stage_kernel<real, true, true, true, true><<<grid, bs, 0, s>>>(p, v, step, tc);
    else clv::visc_stage_kernel<real, true, true, false, true><<<grid, bs, 0, s>>>(p, v, step, tc);
  } else {
    if (cpl) clv::visc_stage_kernel<real, true, true, true, false><<<grid, bs, 0, s>>>(p, v, step, tc);
    else clv::visc_stage_kernel<real, true, true, false, false><<<grid, bs, 0, s>>>(p, v, step, tc);
  }
  return clv_host::check_cuda("fast visc_stage_kernel");
}

template <class real>
int batch_stage(const clv::Params& p, const clv::BatchArgs<real>& a, int step, int bs, int grid, int cap,
                cudaStream_t s) {
  if (p.flags & clv::FLAG_BULK) return clv::batch_launch::stage_bs<real, true>(p, a, step, bs, grid, cap, s);
  return clv::batch_launch::stage_bs<real, false>(p, a, step, bs, grid, cap, s);
}

template <class real>
int batch_stage_tiled(const clv::Params& p, const clv::BatchArgs<real>& a, int step, int rows, int chunk, int grid,
                      cudaStream_t s) {
  return clv::batch_launch::stage_tiled<real>(p, a, step, rows, chunk, grid, s);
}

template <class real> int batch_occupancy(bool bulk, int bs, int cap, int* n) {
  return bulk ? clv::batch_launch::occupancy<real, true>(bs, cap, n)
              : clv::batch_launch::occupancy<real, false>(bs, cap, n);
}
template <class real> int batch_occupancy_tiled(bool bulk, int rows, int* n) {
  if (rows == 64)
    return bulk ? clv::batch_launch::occupancy_tiled<real, true, 64>(n)
                : clv::batch_launch::occupancy_tiled<real, false, 64>(n);
  return bulk ? clv::batch_launch::occupancy_tiled<real, true, 128>(n)
              : clv::batch_launch::occupancy_tiled<real, false, 128>(n);
}
template int batch_occupancy<float>(bool, int, int, int*);
template int batch_occupancy<double>(bool, int, int, int*);
template int batch_occupancy_tiled<float>(bool, int, int*);
template int batch_occupancy_tiled<double>(bool, int, int*);

template int batch_stage<float>(const clv::Params&, const clv::BatchArgs<float>&, int, int, int, int, cudaStream_t);
template int batch_stage<double>(const clv::Params&, const clv::BatchArgs<double>&, int, int, int, int, cudaStream_t);
template int batch_stage_tiled<float>(const clv::Params&, const clv::BatchArgs<float>&, int, int, int, int,
                                      cudaStream_t);
template int batch_stage_tiled<double>(const clv::Params&, const clv::BatchArgs<double>&, int, int, int, int,
                                       cudaStream_t);

template int visc_stage<float>(const clv::Params&, const clv::ViscBuffers<float>&, int, const clv::TauConst<float>&,
                               const clv::StageOpts&, cudaStream_t);
template int visc_stage<double>(const clv::Params&, const clv::ViscBuffers<double>&, int,
                                const clv::TauConst<double>&, const clv::StageOpts&, cudaStream_t);

}  // namespace clv_fastpath
