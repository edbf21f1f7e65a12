// Interface of the tolerance-arithmetic translation unit (clv_fast.cu) to the
// C ABI's dispatcher (clv_capi.cu): the fused viscous stage compiled with
// CLV_FAST=1 (fused multiply-add contraction, approximate division and square
// root, reciprocal products for division by run constants).
#pragma once
#include <cuda_runtime.h>

#include "clv_device.cuh"

namespace clv {
template <class real> struct ViscBuffers;
}

namespace clv_fastpath {
// one fused (IS + KT) Runge-Kutta stage; returns CLV_OK or a CLV_ERR_* code
template <class real>
int visc_stage(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, const clv::TauConst<real>& tc,
               const clv::StageOpts& o, cudaStream_t s);
}  // namespace clv_fastpath
