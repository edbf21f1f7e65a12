// extern "C" entry points of the batched event runner (declared in
// include/clvisc_b200.h). The reference runs events one at a time; these have
// no counterpart in it.
#include <string>

#include "../../include/clvisc_b200.h"
#include "clv_batch.cuh"

namespace clv_host {
int params_from_abi(const clv_params* in, clv::Params* out);
int set_error(int code, const std::string& msg);
int check_cuda(const char* where);
}  // namespace clv_host

namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

static_assert(sizeof(clv_batch_event) == sizeof(clv::BatchEvent), "clv_batch_event layout");
static_assert(sizeof(clv_batch_ctl) == sizeof(clv::BatchCtl), "clv_batch_ctl layout");

template <class real>
int make_args(const clv_params* pp, const clv_batch* b, clv::Params* p, clv::BatchArgs<real>* a) {
  int rc = clv_host::params_from_abi(pp, p);
  if (rc) return rc;
  if (!b) return clv_host::set_error(CLV_ERR_INVALID, "batch: null clv_batch");
  if (b->n_events < 1 || b->n_events > clv::BATCH_MAX_EVENTS)
    return clv_host::set_error(CLV_ERR_INVALID, "batch: n_events must be in 1.." +
                                                    std::to_string(clv::BATCH_MAX_EVENTS));
  if (!b->events || !b->src || !b->udiff || !b->goodcell || !b->keys || !b->ctl || !b->active || !b->prefix ||
      !b->loops || (b->hist_cap > 0 && !b->history))
    return clv_host::set_error(CLV_ERR_INVALID, "batch: null buffer");
  for (int k = 0; k < 3; k++)
    if (!b->ev[k] || !b->pi[k]) return clv_host::set_error(CLV_ERR_INVALID, "batch: null ev/pi slot");
  if (b->ntskip < 1) return clv_host::set_error(CLV_ERR_INVALID, "batch: ntskip must be >= 1");
  a->events = reinterpret_cast<const clv::BatchEvent*>(b->events);
  a->n_events = b->n_events;
  for (int k = 0; k < 3; k++) {
    a->ev[k] = (real*)b->ev[k];
    a->pi[k] = (real*)b->pi[k];
  }
  a->src = (real*)b->src;
  a->udiff = (real*)b->udiff;
  a->goodcell = b->goodcell;
  a->keys = (typename clv::KeyT<real>::type*)b->keys;
  a->ctl = reinterpret_cast<clv::BatchCtl*>(b->ctl);
  a->active = b->active;
  a->prefix = b->prefix;
  a->loops = b->loops;
  a->history = b->history;
  a->hist_cap = b->hist_cap;
  a->tau0 = b->tau0;
  a->dt = b->dt;
  a->efrz = b->efrz;
  a->ntskip = b->ntskip;
  a->max_loops = b->max_loops;
  return CLV_OK;
}

template <class real, bool BULK, int BS>
int launch_stage(const clv::Params& p, const clv::BatchArgs<real>& a, int step, int grid, cudaStream_t s) {
  auto kern = clv::batch_stage_kernel<real, BULK, BS>;
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

template <class real, bool BULK>
int stage_bs(const clv::Params& p, const clv::BatchArgs<real>& a, int step, int bs, int grid, cudaStream_t s) {
  if (bs == 64) return launch_stage<real, BULK, 64>(p, a, step, grid, s);
  if (bs == 128) return launch_stage<real, BULK, 128>(p, a, step, grid, s);
  if (bs == 256) return launch_stage<real, BULK, 256>(p, a, step, grid, s);
  return clv_host::set_error(CLV_ERR_INVALID, "batch: block_size must be 64, 128 or 256");
}

template <class real>
int batch_stage_t(const clv_params* pp, int step, const clv_batch* b, int bs, int grid, cudaStream_t s) {
  clv::Params p;
  clv::BatchArgs<real> a;
  int rc = make_args<real>(pp, b, &p, &a);
  if (rc) return rc;
  if (step != 1 && step != 2) return clv_host::set_error(CLV_ERR_INVALID, "batch: step must be 1 or 2");
  if (p.flags & (clv::FLAG_GUBSER_VISC | clv::FLAG_PIMN_OMEGA | clv::FLAG_OMEGA_OMEGA | clv::FLAG_RIEMANN))
    return clv_host::set_error(CLV_ERR_INVALID, "batch: test flags (Gubser, couplings, Riemann) are not batched");
  if (p.flags & clv::FLAG_BULK) return stage_bs<real, true>(p, a, step, bs, grid, s);
  return stage_bs<real, false>(p, a, step, bs, grid, s);
}

template <class real> int batch_advance_t(const clv_params* pp, const clv_batch* b, int first, cudaStream_t s) {
  clv::Params p;
  clv::BatchArgs<real> a;
  int rc = make_args<real>(pp, b, &p, &a);
  if (rc) return rc;
  clv::batch_advance_kernel<real><<<1, 1024, 0, s>>>(a, first ? 1 : 0);
  return clv_host::check_cuda("batch_advance_kernel");
}

}  // namespace

extern "C" {

int clv_batch_stage(const clv_params* p, int step, const clv_batch* b, int block_size, int grid_blocks,
                    void* stream) {
  if (!p) return clv_host::set_error(CLV_ERR_INVALID, "batch: null clv_params");
  if (p->precision == 4) return batch_stage_t<float>(p, step, b, block_size, grid_blocks, S(stream));
  return batch_stage_t<double>(p, step, b, block_size, grid_blocks, S(stream));
}

int clv_batch_advance(const clv_params* p, const clv_batch* b, int first, void* stream) {
  if (!p) return clv_host::set_error(CLV_ERR_INVALID, "batch: null clv_params");
  if (p->precision == 4) return batch_advance_t<float>(p, b, first, S(stream));
  return batch_advance_t<double>(p, b, first, S(stream));
}

int clv_batch_occupancy(const clv_params* p, int block_size, int* blocks_per_sm) {
  if (!p || !blocks_per_sm || (p->precision != 4 && p->precision != 8))
    return clv_host::set_error(CLV_ERR_INVALID, "batch_occupancy: bad argument");
  const bool bulk = p->flags & CLV_FLAG_BULK;
  cudaError_t e = cudaErrorInvalidValue;
  int n = 0;
#define CLV_OCC(real, B, BS) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, clv::batch_stage_kernel<real, B, BS>, BS, 0)
  if (block_size != 64 && block_size != 128 && block_size != 256)
    return clv_host::set_error(CLV_ERR_INVALID, "batch_occupancy: block_size must be 64, 128 or 256");
  if (p->precision == 4) {
    if (bulk) { if (block_size == 64) CLV_OCC(float, true, 64); else if (block_size == 128) CLV_OCC(float, true, 128); else CLV_OCC(float, true, 256); }
    else { if (block_size == 64) CLV_OCC(float, false, 64); else if (block_size == 128) CLV_OCC(float, false, 128); else CLV_OCC(float, false, 256); }
  } else {
    if (bulk) { if (block_size == 64) CLV_OCC(double, true, 64); else if (block_size == 128) CLV_OCC(double, true, 128); else CLV_OCC(double, true, 256); }
    else { if (block_size == 64) CLV_OCC(double, false, 64); else if (block_size == 128) CLV_OCC(double, false, 128); else CLV_OCC(double, false, 256); }
  }
#undef CLV_OCC
  if (e != cudaSuccess) return clv_host::set_error(CLV_ERR_CUDA, std::string("batch_occupancy: ") + cudaGetErrorString(e));
  *blocks_per_sm = n;
  return CLV_OK;
}

}  // extern "C"
