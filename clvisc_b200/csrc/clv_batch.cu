// extern "C" entry points of the batched event runner (declared in
// include/clvisc_b200.h). The reference runs events one at a time; these have
// no counterpart in it.
#include <string>

#include "../../include/clvisc_b200.h"
#include "clv_batch.cuh"
#include "clv_batch_launch.cuh"
#include "clv_fast.h"

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

template <class real>
int batch_stage_t(const clv_params* pp, int step, const clv_batch* b, int bs, int grid, int max_regs,
                  cudaStream_t s) {
  clv::Params p;
  clv::BatchArgs<real> a;
  int rc = make_args<real>(pp, b, &p, &a);
  if (rc) return rc;
  if (step != 1 && step != 2) return clv_host::set_error(CLV_ERR_INVALID, "batch: step must be 1 or 2");
  if (p.flags & (clv::FLAG_GUBSER_VISC | clv::FLAG_PIMN_OMEGA | clv::FLAG_OMEGA_OMEGA | clv::FLAG_RIEMANN))
    return clv_host::set_error(CLV_ERR_INVALID, "batch: test flags (Gubser, couplings, Riemann) are not batched");
  if (max_regs != 0 && max_regs != 128 && max_regs != 168)
    return clv_host::set_error(CLV_ERR_INVALID, "batch: max_registers must be 0, 128 or 168");
  const int cap = max_regs;
  if (p.flags & clv::FLAG_FAST) return clv_fastpath::batch_stage<real>(p, a, step, bs, grid, cap, s);
  if (p.flags & clv::FLAG_BULK) return clv::batch_launch::stage_bs<real, true>(p, a, step, bs, grid, cap, s);
  return clv::batch_launch::stage_bs<real, false>(p, a, step, bs, grid, cap, s);
}

template <class real>
int batch_stage_tiled_t(const clv_params* pp, int step, const clv_batch* b, int rows, int chunk, int grid,
                        cudaStream_t s) {
  clv::Params p;
  clv::BatchArgs<real> a;
  int rc = make_args<real>(pp, b, &p, &a);
  if (rc) return rc;
  if (step != 1 && step != 2) return clv_host::set_error(CLV_ERR_INVALID, "batch: step must be 1 or 2");
  if (p.flags & (clv::FLAG_GUBSER_VISC | clv::FLAG_PIMN_OMEGA | clv::FLAG_OMEGA_OMEGA | clv::FLAG_RIEMANN))
    return clv_host::set_error(CLV_ERR_INVALID, "batch: test flags (Gubser, couplings, Riemann) are not batched");
  if (chunk < 1 || chunk > 4096) return clv_host::set_error(CLV_ERR_INVALID, "batch: chunk must be in 1..4096");
  if (rows != 64 && rows != 128) return clv_host::set_error(CLV_ERR_INVALID, "batch: rows must be 64 or 128");
  if (p.flags & clv::FLAG_FAST) return clv_fastpath::batch_stage_tiled<real>(p, a, step, rows, chunk, grid, s);
  return clv::batch_launch::stage_tiled<real>(p, a, step, rows, chunk, grid, s);
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
                    int max_registers, void* stream) {
  if (!p) return clv_host::set_error(CLV_ERR_INVALID, "batch: null clv_params");
  if (p->precision == 4) return batch_stage_t<float>(p, step, b, block_size, grid_blocks, max_registers, S(stream));
  return batch_stage_t<double>(p, step, b, block_size, grid_blocks, max_registers, S(stream));
}

int clv_batch_advance(const clv_params* p, const clv_batch* b, int first, void* stream) {
  if (!p) return clv_host::set_error(CLV_ERR_INVALID, "batch: null clv_params");
  if (p->precision == 4) return batch_advance_t<float>(p, b, first, S(stream));
  return batch_advance_t<double>(p, b, first, S(stream));
}

int clv_batch_stage_tiled(const clv_params* p, int step, const clv_batch* b, int rows, int chunk, int grid_blocks,
                          void* stream) {
  if (!p) return clv_host::set_error(CLV_ERR_INVALID, "batch: null clv_params");
  if (p->precision == 4) return batch_stage_tiled_t<float>(p, step, b, rows, chunk, grid_blocks, S(stream));
  return batch_stage_tiled_t<double>(p, step, b, rows, chunk, grid_blocks, S(stream));
}

int clv_batch_occupancy_tiled(const clv_params* p, int rows, int* blocks_per_sm) {
  if (!p || !blocks_per_sm || (p->precision != 4 && p->precision != 8))
    return clv_host::set_error(CLV_ERR_INVALID, "batch_occupancy_tiled: bad argument");
  if (rows != 64 && rows != 128) return clv_host::set_error(CLV_ERR_INVALID, "batch_occupancy_tiled: rows must be 64 or 128");
  const bool bulk = p->flags & CLV_FLAG_BULK;
  int n = 0, rc;
  if (p->flags & CLV_FLAG_FAST)
    rc = p->precision == 4 ? clv_fastpath::batch_occupancy_tiled<float>(bulk, rows, &n)
                           : clv_fastpath::batch_occupancy_tiled<double>(bulk, rows, &n);
  else if (p->precision == 4)
    rc = rows == 64 ? (bulk ? clv::batch_launch::occupancy_tiled<float, true, 64>(&n)
                            : clv::batch_launch::occupancy_tiled<float, false, 64>(&n))
                    : (bulk ? clv::batch_launch::occupancy_tiled<float, true, 128>(&n)
                            : clv::batch_launch::occupancy_tiled<float, false, 128>(&n));
  else
    rc = rows == 64 ? (bulk ? clv::batch_launch::occupancy_tiled<double, true, 64>(&n)
                            : clv::batch_launch::occupancy_tiled<double, false, 64>(&n))
                    : (bulk ? clv::batch_launch::occupancy_tiled<double, true, 128>(&n)
                            : clv::batch_launch::occupancy_tiled<double, false, 128>(&n));
  if (rc) return rc;
  *blocks_per_sm = n;
  return CLV_OK;
}

int clv_batch_occupancy(const clv_params* p, int block_size, int max_registers, int* blocks_per_sm) {
  if (!p || !blocks_per_sm || (p->precision != 4 && p->precision != 8))
    return clv_host::set_error(CLV_ERR_INVALID, "batch_occupancy: bad argument");
  if (block_size != 64 && block_size != 128 && block_size != 256)
    return clv_host::set_error(CLV_ERR_INVALID, "batch_occupancy: block_size must be 64, 128 or 256");
  if (max_registers != 0 && ((max_registers != 128 && max_registers != 168) || p->precision != 4 ||
                             (max_registers == 168 && block_size == 256)))
    return clv_host::set_error(CLV_ERR_INVALID,
                               "batch_occupancy: max_registers must be 0 (or 128, or 168 below 256 threads, in FP32)");
  const bool bulk = p->flags & CLV_FLAG_BULK;
  int n = 0, rc;
  if (p->flags & CLV_FLAG_FAST)
    rc = p->precision == 4 ? clv_fastpath::batch_occupancy<float>(bulk, block_size, max_registers, &n)
                           : clv_fastpath::batch_occupancy<double>(bulk, block_size, max_registers, &n);
  else if (p->precision == 4)
    rc = bulk ? clv::batch_launch::occupancy<float, true>(block_size, max_registers, &n)
              : clv::batch_launch::occupancy<float, false>(block_size, max_registers, &n);
  else
    rc = bulk ? clv::batch_launch::occupancy<double, true>(block_size, max_registers, &n)
              : clv::batch_launch::occupancy<double, false>(block_size, max_registers, &n);
  if (rc) return rc;
  *blocks_per_sm = n;
  return CLV_OK;
}

}  // extern "C"
