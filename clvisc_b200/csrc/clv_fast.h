// Interface of the tolerance-arithmetic translation unit (clv_fast.cu) to the
// C ABI's dispatcher (clv_capi.cu): the fused viscous stage compiled with
// CLV_FAST=1 (fused multiply-add contraction, approximate division and square
// root, reciprocal products for division by run constants).
#pragma once
#include <cuda_runtime.h>

#include "clv_device.cuh"

namespace clv {
template <class real> struct ViscBuffers;
template <class real> struct BatchArgs;
}

namespace clv_fastpath {
// one fused (IS + KT) Runge-Kutta stage; returns CLV_OK or a CLV_ERR_* code
template <class real>
int visc_stage(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, const clv::TauConst<real>& tc,
               const clv::StageOpts& o, cudaStream_t s);
// one stage of a batch of events, one thread per cell (block size bs, grid
// blocks, register cap 0 / 128 / 168) or (2+1)D tiles of rows - 4 rows
template <class real>
int batch_stage(const clv::Params& p, const clv::BatchArgs<real>& a, int step, int bs, int grid, int cap,
                cudaStream_t s);
template <class real>
int batch_stage_tiled(const clv::Params& p, const clv::BatchArgs<real>& a, int step, int rows, int chunk, int grid,
                      cudaStream_t s);
// resident blocks per SM of the fast batched stage kernels (loads them)
template <class real> int batch_occupancy(bool bulk, int bs, int cap, int* n);
template <class real> int batch_occupancy_tiled(bool bulk, int rows, int* n);
}  // namespace clv_fastpath
