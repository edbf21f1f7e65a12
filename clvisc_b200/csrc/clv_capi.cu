// extern "C" entry points of libclvisc_b200.so (declared in include/clvisc_b200.h).
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/clvisc_b200.h"
#include "clv_device.cuh"
#include "clv_hypersf.cuh"
#include "clv_misc.cuh"
#include "clv_stage.cuh"
#include "clv_stage_tiled.cuh"
#include "clv_stage_tiled2d.cuh"
#include "clv_fast.h"

namespace clv_host {
thread_local std::string g_err;  // message behind clv_last_error()
}
using clv_host::g_err;

namespace {

int g_stage_kernel = 0;  // CLV_OPT_STAGE_KERNEL: 0 automatic, 1 per-cell, 2 tiled (3+1)D, 3 tiled (2+1)D
constexpr int kTiledMinNz = 24;  // fewer cells along eta: per-cell kernel
constexpr int kTiled2dMin = 4;   // (2+1)D tiles: at least this many cells along x and y
int g_chunk = 32;        // CLV_OPT_CHUNK: x planes per tiled CTA
int g_minb = 2;          // CLV_OPT_TILED_BLOCKS: resident tiled CTAs per SM (FP32)
int g_tile = 0;          // CLV_OPT_TILE: 0 = 8 x 32, 1 = 16 x 16, 2 = 8 x 16 (y, eta) tile of the fused stage
int g_rows2d = 64;       // CLV_OPT_TILE2D_ROWS: threads of a (2+1)D tile block (64 or 128)
int g_chunk2d = 8;       // CLV_OPT_CHUNK2D: x planes per (2+1)D tile

int fail(int code, const char* fmt, const char* what = "") {
  char buf[256];
  snprintf(buf, sizeof(buf), fmt, what);
  g_err = buf;
  return code;
}
int cuda_check(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return CLV_ERR_CUDA;
  }
  return CLV_OK;
}
inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kAlign = 16;
constexpr int kMaxDev = 64;  // devices tracked by the per-device launch set-up
inline bool aligned(const void* q) { return (reinterpret_cast<uintptr_t>(q) % kAlign) == 0; }

int to_params(const clv_params* in, clv::Params* out) {
  if (!in) return fail(CLV_ERR_INVALID, "null clv_params%s");
  if (in->precision != 4 && in->precision != 8) return fail(CLV_ERR_INVALID, "precision must be 4 or 8%s");
  if (in->nx < 1 || in->ny < 1 || in->nz < 1) return fail(CLV_ERR_INVALID, "grid sizes must be >= 1%s");
  long long n = (long long)in->nx * in->ny * in->nz;
  if (in->ld < n) return fail(CLV_ERR_INVALID, "ld must be >= nx*ny*nz%s");
  if ((in->ld * in->precision) % kAlign) return fail(CLV_ERR_INVALID, "ld*precision must be a multiple of 16%s");
  if (10 * in->ld >= (1ll << 40)) return fail(CLV_ERR_INVALID, "grid too large%s");
  if (!in->eos_table || in->eos_nrow < 1 || in->eos_ncol < 1) return fail(CLV_ERR_INVALID, "EOS table missing%s");
  if (!aligned(in->eos_table)) return fail(CLV_ERR_INVALID, "EOS table must be 16-byte aligned%s");
  if (!(in->eos_ed_step > 0.0f)) return fail(CLV_ERR_INVALID, "eos_ed_step must be > 0%s");
  if (in->nxskip < 1 || in->nyskip < 1 || in->nzskip < 1) return fail(CLV_ERR_INVALID, "skips must be >= 1%s");
  clv::Params& p = *out;
  p.nx = in->nx; p.ny = in->ny; p.nz = in->nz; p.ld = in->ld;
  p.DT = in->dt; p.DX = in->dx; p.DY = in->dy; p.DZ = in->dz; p.TAU0 = in->tau0;
  p.ETAOS_XMIN = in->etaos_xmin; p.ETAOS_YMIN = in->etaos_ymin;
  p.ETAOS_LEFT_SLOP = in->etaos_left_slop; p.ETAOS_RIGHT_SLOP = in->etaos_right_slop; p.LAM1 = in->lam1;
  p.EFRZ = in->efrz;
  p.nxskip = in->nxskip; p.nyskip = in->nyskip; p.nzskip = in->nzskip;
  p.eos_start = in->eos_ed_start; p.eos_step = in->eos_ed_step;
  p.eos_num = in->eos_num_ed; p.eos_nrow = in->eos_nrow; p.eos_ncol = in->eos_ncol;
  p.eos = in->eos_table;
  p.eos_p2 = reinterpret_cast<const float2*>(in->eos_p2);
  if (in->eos_p2 && (reinterpret_cast<uintptr_t>(in->eos_p2) % 8))
    return fail(CLV_ERR_INVALID, "eos_p2 must be 8-byte aligned%s");
  p.flags = in->flags;
  p.ZETAOS_MAX = in->zetaos_max; p.ZETAOS_T0 = in->zetaos_t0;
  p.ZETAOS_WIDTH = in->zetaos_width; p.ZETAOS_SKEW = in->zetaos_skew; p.ZETAOS_TMIN = in->zetaos_tmin;
  p.opt[0] = in->opt_stage_kernel; p.opt[1] = in->opt_chunk; p.opt[2] = in->opt_tiled_blocks; p.opt[3] = in->opt_tile;
  if (in->opt_stage_kernel < 0 || in->opt_stage_kernel > 4 || in->opt_chunk < 0 || in->opt_chunk > 4096 ||
      in->opt_tiled_blocks < 0 || in->opt_tiled_blocks > 2 || in->opt_tile < 0 || in->opt_tile > 4)
    return fail(CLV_ERR_INVALID, "opt_* fields out of range%s");
  if ((in->flags & CLV_FLAG_BULK) && (!(in->zetaos_width > 0.0f) || !(in->zetaos_max >= 0.0f)))
    return fail(CLV_ERR_INVALID, "bulk sector: zetaos_width must be > 0 and zetaos_max >= 0%s");
  // correctly rounded reciprocals in each precision (host IEEE arithmetic, no
  // contraction): the kernels divide by these constants with clv::div_by
  const float epr = in->eos_ed_step * in->eos_ncol;  // as the kernels form it
  p.rf.eos_step = 1.0f / in->eos_ed_step;
  p.rf.eos_epr = 1.0f / epr;
  p.rf.DT = 1.0f / in->dt;
  p.rf.DX = 1.0f / in->dx;
  p.rf.DY = 1.0f / in->dy;
  p.rf.DZ = 1.0f / in->dz;
  p.rf.three = 1.0f / 3.0f;
  p.rd.eos_step = 1.0 / (double)in->eos_ed_step;
  p.rd.eos_epr = 1.0 / (double)epr;
  p.rd.DT = 1.0 / (double)in->dt;
  p.rd.DX = 1.0 / (double)in->dx;
  p.rd.DY = 1.0 / (double)in->dy;
  p.rd.DZ = 1.0 / (double)in->dz;
  p.rd.three = 1.0 / 3.0;
  if (!(in->dt > 0.0f) || !(in->dx > 0.0f) || !(in->dy > 0.0f) || !(in->dz > 0.0f))
    return fail(CLV_ERR_INVALID, "dt, dx, dy, dz must be > 0%s");
  return CLV_OK;
}

// tau of a stage launch in the run precision, DZ*tau as the kernels form it,
// and the correctly rounded reciprocals of both
template <class real>
clv::TauConst<real> tau_const(const clv::Params& p, double tau_d) {
  clv::TauConst<real> t;
  t.tau = (real)tau_d;
  t.rtau = (real)1 / t.tau;
  t.dzt = (real)p.DZ * t.tau;
  t.rdzt = (real)1 / t.dzt;
  return t;
}
inline long long ncell(const clv::Params& p) { return (long long)p.nx * p.ny * p.nz; }
inline unsigned int nblk(long long n, int bs) { return (unsigned int)((n + bs - 1) / bs); }

// the stage launch choices of a run: its own opt_* fields where set, else the
// process-wide settings of clv_set_option
clv::StageOpts stage_opts(const clv::Params& p) {
  clv::StageOpts o;
  o.stage_kernel = p.opt[0] ? p.opt[0] - 1 : g_stage_kernel;
  o.chunk = p.opt[1] ? p.opt[1] : g_chunk;
  o.minb = p.opt[2] ? p.opt[2] : g_minb;
  o.tile = p.opt[3] ? p.opt[3] - 1 : g_tile;
  o.rows2d = g_rows2d;
  o.chunk2d = g_chunk2d;
  return o;
}

template <class real, bool IS, bool KT, bool CPL, int MINB, int TJ = 8, int TK = 32>
int launch_tiled_b(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, double tau, cudaStream_t s,
                   const clv::StageOpts& o) {
  typedef clv::TileSmem<real, TJ, TK> SM;
  auto kern = clv::visc_stage_tiled_kernel<real, IS, KT, CPL, TJ, TK, MINB>;
  static bool configured[kMaxDev] = {};  // the attribute is per device
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return cuda_check("cudaGetDevice");
  if (!configured[dev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SM)) != cudaSuccess)
      return cuda_check("cudaFuncSetAttribute(visc_stage_tiled_kernel)");
    configured[dev] = true;
  }
  const int chunk = o.chunk;
  dim3 grid((p.nz + TK - 1) / TK, (p.ny + TJ - 1) / TJ, (p.nx + chunk - 1) / chunk);
  kern<<<grid, TJ * TK, sizeof(SM), s>>>(p, v, step, tau_const<real>(p, tau), chunk);
  return cuda_check("visc_stage_tiled_kernel");
}

template <class real, bool BULK, int TB>
int launch_tiled2d_b(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, double tau, cudaStream_t s) {
  typedef clv::Tile2Smem<real, BULK, TB> SM;
  auto kern = clv::visc_stage_tiled2d_kernel<real, BULK, TB, clv::tiled2d_minb<real, TB>()>;
  static bool configured[kMaxDev] = {};  // the attribute is per device
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return cuda_check("cudaGetDevice");
  if (!configured[dev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SM)) != cudaSuccess)
      return cuda_check("cudaFuncSetAttribute(visc_stage_tiled2d_kernel)");
    configured[dev] = true;
  }
  const int chunk = g_chunk2d;
  dim3 grid((p.ny + TB - 5) / (TB - 4), (p.nx + chunk - 1) / chunk);
  kern<<<grid, TB, sizeof(SM), s>>>(p, v, step, tau_const<real>(p, tau), chunk);
  return cuda_check("visc_stage_tiled2d_kernel");
}

template <class real, bool BULK>
int launch_tiled2d(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, double tau, cudaStream_t s) {
  if (g_rows2d == 128) return launch_tiled2d_b<real, BULK, 128>(p, v, step, tau, s);
  return launch_tiled2d_b<real, BULK, 64>(p, v, step, tau, s);
}

template <class real, bool IS, bool KT>
int launch_tiled(const clv::Params& p, const clv::ViscBuffers<real>& v, int step, double tau, cudaStream_t s,
                 const clv::StageOpts& o) {
  // the coupling terms (GUBSER_VISC_TEST, PIMUNU_OMEGA_COUPLING,
  // OMEGA_OMEGA_COUPLING) live in a separate instantiation so that the
  // default kernel does not carry their code
  const bool cpl = IS && (p.flags & (clv::FLAG_GUBSER_VISC | clv::FLAG_PIMN_OMEGA | clv::FLAG_OMEGA_OMEGA));
  if (cpl) return launch_tiled_b<real, IS, KT, IS, 1>(p, v, step, tau, s, o);
  // the fused stage also comes with 16 x 16 and 8 x 16 (y, eta) tiles
  // (CLV_OPT_TILE); the 128-thread 8 x 16 tile keeps 4 CTAs an SM at 128
  // registers (FP32; 2 at 255 with CLV_OPT_TILED_BLOCKS = 1, and in FP64)
  constexpr bool dbl = sizeof(real) == 8;
  if (IS && KT && o.tile == 2) {
    if (dbl || o.minb == 1) return launch_tiled_b<real, IS, KT, false, 2, 8, 16>(p, v, step, tau, s, o);
    if constexpr (!dbl) return launch_tiled_b<real, IS, KT, false, 4, 8, 16>(p, v, step, tau, s, o);
  }
  if (IS && KT && o.tile == 1) {
    if (dbl || o.minb == 1) return launch_tiled_b<real, IS, KT, false, 1, 16, 16>(p, v, step, tau, s, o);
    if constexpr (!dbl) return launch_tiled_b<real, IS, KT, false, 2, 16, 16>(p, v, step, tau, s, o);
  }
  if (dbl || o.minb == 1) return launch_tiled_b<real, IS, KT, false, 1>(p, v, step, tau, s, o);
  if constexpr (!dbl) return launch_tiled_b<real, IS, KT, false, 2>(p, v, step, tau, s, o);
  return CLV_ERR_INVALID;  // not reached
}

template <class real>
int visc_stage_t(const clv::Params& p, int step, double tau, int parts, const clv_visc_buffers* b, cudaStream_t s) {
  clv::ViscBuffers<real> v;
  v.ev_st = (const real*)b->ev_st; v.pi_st = (const real*)b->pi_st;
  v.ev1 = (const real*)b->ev1; v.ev2e = (const real*)b->ev2_ed;
  v.pi1 = (const real*)b->pi1; v.pin = (const real*)b->pi_n; v.pi2in = (const real*)b->pi_new_in;
  v.evnew = (real*)b->ev_new; v.pinew = (real*)b->pi_new;
  v.src = (real*)b->src; v.udiff = (real*)b->udiff; v.goodcell = b->goodcell;
  v.edmax_key = (typename clv::KeyT<real>::type*)b->edmax_key;
  v.write_src = b->write_src; v.write_udiff = b->write_udiff;
  const bool is = parts & CLV_PART_IS, kt = parts & CLV_PART_KT;
  const clv::StageOpts o = stage_opts(p);
  if (!v.ev_st || !v.pi_st || !v.ev1 || !v.src) return fail(CLV_ERR_INVALID, "visc stage: null stencil/src buffer%s");
  if (is && (!v.pi1 || !v.pinew || !v.udiff || !v.goodcell || (step == 1 && !v.ev2e)))
    return fail(CLV_ERR_INVALID, "visc stage: null buffer for the pi update%s");
  if (kt && (!v.evnew || !v.pin || (!is && !v.pi2in))) return fail(CLV_ERR_INVALID, "visc stage: null buffer for update_ev%s");
  if (v.write_udiff && (!kt || !v.udiff)) return fail(CLV_ERR_INVALID, "visc stage: write_udiff needs CLV_PART_KT%s");
  const bool bulk = p.flags & clv::FLAG_BULK;
  const bool cpl0 = p.flags & (clv::FLAG_GUBSER_VISC | clv::FLAG_PIMN_OMEGA | clv::FLAG_OMEGA_OMEGA);
  // tolerance arithmetic (CLV_FLAG_FAST) for the fused stage
  if ((p.flags & clv::FLAG_FAST) && is && kt) return clv_fastpath::visc_stage<real>(p, v, step, tau_const<real>(p, tau), o, s);
  // the tiled (2+1)D kernel (bulk sector, no coupling terms) when asked for:
  // on B200 the per-cell kernel is faster on the (2+1)D grids of this code
  const bool fit2d = p.nz == 1 && p.nx >= kTiled2dMin && p.ny >= kTiled2dMin && is && kt && !cpl0;
  if (fit2d && o.stage_kernel == 3)
    return bulk ? launch_tiled2d<real, true>(p, v, step, tau, s) : launch_tiled2d<real, false>(p, v, step, tau, s);
  // The tiled kernel has no bulk sector, and its 8 x 32 (y, eta) tile leaves
  // most threads idle on grids with few cells along eta ((2+1)D runs have
  // one): those runs take the per-cell kernel, which gives the same bits.
  if (!bulk && (o.stage_kernel == 2 || (o.stage_kernel == 0 && p.nz >= kTiledMinNz))) {
    if (is && kt) return launch_tiled<real, true, true>(p, v, step, tau, s, o);
    if (is) return launch_tiled<real, true, false>(p, v, step, tau, s, o);
    return launch_tiled<real, false, true>(p, v, step, tau, s, o);
  }
  const int bs = 128;
  dim3 grid(nblk(ncell(p), bs));
  const clv::TauConst<real> t = tau_const<real>(p, tau);
  const bool cpl = p.flags & (clv::FLAG_GUBSER_VISC | clv::FLAG_PIMN_OMEGA | clv::FLAG_OMEGA_OMEGA);
  if (bulk) {
    if (is && kt && cpl) clv::visc_stage_kernel<real, true, true, true, true><<<grid, bs, 0, s>>>(p, v, step, t);
    else if (is && kt) clv::visc_stage_kernel<real, true, true, false, true><<<grid, bs, 0, s>>>(p, v, step, t);
    else if (is && cpl) clv::visc_stage_kernel<real, true, false, true, true><<<grid, bs, 0, s>>>(p, v, step, t);
    else if (is) clv::visc_stage_kernel<real, true, false, false, true><<<grid, bs, 0, s>>>(p, v, step, t);
    else clv::visc_stage_kernel<real, false, true, false, true><<<grid, bs, 0, s>>>(p, v, step, t);
  } else {
    if (is && kt && cpl) clv::visc_stage_kernel<real, true, true, true, false><<<grid, bs, 0, s>>>(p, v, step, t);
    else if (is && kt) clv::visc_stage_kernel<real, true, true, false, false><<<grid, bs, 0, s>>>(p, v, step, t);
    else if (is && cpl) clv::visc_stage_kernel<real, true, false, true, false><<<grid, bs, 0, s>>>(p, v, step, t);
    else if (is) clv::visc_stage_kernel<real, true, false, false, false><<<grid, bs, 0, s>>>(p, v, step, t);
    else clv::visc_stage_kernel<real, false, true, false, false><<<grid, bs, 0, s>>>(p, v, step, t);
  }
  return cuda_check("visc_stage_kernel");
}

template <class real>
int ideal_stage_t(const clv::Params& p, int step, double tau, const void* ev_st, const void* ev1, void* ev_new,
                  void* src, int write_src, void* key, cudaStream_t s) {
  clv::IdealBuffers<real> b;
  b.ev_st = (const real*)ev_st; b.ev1 = (const real*)ev1; b.evnew = (real*)ev_new; b.src = (real*)src;
  b.edmax_key = (typename clv::KeyT<real>::type*)key; b.write_src = write_src;
  const int bs = 128;
  clv::ideal_stage_kernel<real><<<nblk(ncell(p), bs), bs, 0, s>>>(p, b, step, tau_const<real>(p, tau));
  return cuda_check("ideal_stage_kernel");
}

template <class real>
size_t hsf_scratch(const clv::Params& p) {
  clv::CubeGrid g = clv::cube_grid(p);
  long long nc = (long long)g.nx * g.ny * g.nz;
  long long nb = (nc + 255) / 256;
  size_t bytes = 0;
  bytes += ((nc + 255) / 256) * 256;          // marks
  bytes += (size_t)nb * sizeof(int) + 256;    // block counts / offsets
  bytes += (size_t)nc * sizeof(int) + 256;    // cube list
  bytes += 2 * sizeof(long long) + 256;       // count
  return bytes;
}

template <class real>
int hypersf_t(const clv::Params& p, int visc, double tau_old, double tau_new, const void* ev_old,
              const void* ev_new, const void* pi_old, const void* pi_new, void* sf, void* txyz, void* pisf,
              long long capacity, long long* total, void* scratch, size_t scratch_bytes, cudaStream_t s) {
  if (!ev_old || !ev_new || !sf || !txyz || !total || !scratch) return fail(CLV_ERR_INVALID, "hypersf: null pointer%s");
  if (visc && (!pi_old || !pi_new)) return fail(CLV_ERR_INVALID, "hypersf: visc needs pi_old and pi_new%s");
  if (scratch_bytes < hsf_scratch<real>(p)) return fail(CLV_ERR_INVALID, "hypersf: scratch too small%s");
  clv::CubeGrid g = clv::cube_grid(p);
  long long nc = (long long)g.nx * g.ny * g.nz;
  unsigned int nb = nblk(nc, 256);
  char* sp = (char*)scratch;
  uint8_t* mark = (uint8_t*)sp; sp += ((nc + 255) / 256) * 256;
  int* bcount = (int*)sp; sp += (((size_t)nb * sizeof(int) + 255) / 256) * 256;
  int* list = (int*)sp; sp += (((size_t)nc * sizeof(int) + 255) / 256) * 256;
  long long* count = (long long*)sp;
  clv::hsf_mark_kernel<real><<<nb, 256, 0, s>>>(p, (const real*)ev_old, (const real*)ev_new, visc, mark, bcount);
  clv::hsf_scan_kernel<<<1, 1024, 0, s>>>(bcount, (int)nb, count);
  clv::hsf_compact_kernel<<<nb, 256, 0, s>>>(nc, mark, bcount, list);
  clv::hsf_element_kernel<real><<<148 * 4, 128, 0, s>>>(
      p, (const real*)ev_old, (const real*)ev_new, (const real*)pi_old, (const real*)pi_new, (real)tau_old,
      (real)tau_new, visc, list, count, total, (real*)sf, (real*)txyz, (real*)pisf, capacity);
  clv::hsf_advance_kernel<<<1, 1, 0, s>>>(count, total);
  return cuda_check("hypersf kernels");
}

}  // namespace

// shared with the library's other translation units
namespace clv_host {
int params_from_abi(const clv_params* in, clv::Params* out) { return to_params(in, out); }
int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int check_cuda(const char* where) { return cuda_check(where); }
}  // namespace clv_host

extern "C" {

int clv_version(void) { return 0x000104; }
const char* clv_last_error(void) { return g_err.c_str(); }
int clv_alignment(void) { return kAlign; }

int clv_set_option(int option, int value) {
  if (option == CLV_OPT_TILE2D_ROWS && (value == 64 || value == 128)) {
    g_rows2d = value;
    return CLV_OK;
  }
  if (option == CLV_OPT_CHUNK2D && value >= 1 && value <= 4096) {
    g_chunk2d = value;
    return CLV_OK;
  }
  if (option == CLV_OPT_STAGE_KERNEL && value >= 0 && value <= 3) {
    g_stage_kernel = value;
    return CLV_OK;
  }
  if (option == CLV_OPT_TILED_BLOCKS && (value == 1 || value == 2)) {
    g_minb = value;
    return CLV_OK;
  }
  if (option == CLV_OPT_TILE && value >= 0 && value <= 3) {
    g_tile = value;
    return CLV_OK;
  }
  if (option == CLV_OPT_CHUNK && value >= 1 && value <= 4096) {
    g_chunk = value;
    return CLV_OK;
  }
  return fail(CLV_ERR_INVALID, "clv_set_option: unknown option or value%s");
}

int clv_ideal_stage(const clv_params* pp, int step, double tau, const void* ev_st, const void* ev1, void* ev_new,
                    void* src, int write_src, void* edmax_key, void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (step != 1 && step != 2) return fail(CLV_ERR_INVALID, "step must be 1 or 2%s");
  if (!ev_st || !ev1 || !ev_new || !src) return fail(CLV_ERR_INVALID, "ideal stage: null buffer%s");
  if (!aligned(ev_st) || !aligned(ev1) || !aligned(ev_new) || !aligned(src)) return fail(CLV_ERR_INVALID, "ideal stage: misaligned buffer%s");
  if (pp->precision == 4) return ideal_stage_t<float>(p, step, tau, ev_st, ev1, ev_new, src, write_src, edmax_key, S(stream));
  return ideal_stage_t<double>(p, step, tau, ev_st, ev1, ev_new, src, write_src, edmax_key, S(stream));
}

int clv_visc_stage(const clv_params* pp, int step, double tau, int parts, const clv_visc_buffers* b, void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (step != 1 && step != 2) return fail(CLV_ERR_INVALID, "step must be 1 or 2%s");
  if (!b || !(parts & (CLV_PART_IS | CLV_PART_KT)) || (parts & ~3)) return fail(CLV_ERR_INVALID, "bad parts or buffers%s");
  if (pp->precision == 4) return visc_stage_t<float>(p, step, tau, parts, b, S(stream));
  return visc_stage_t<double>(p, step, tau, parts, b, S(stream));
}

int clv_visc_initialize(const clv_params* pp, void* pi1, unsigned char* goodcell, void* udiff, const void* ev,
                        double tau, void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (!pi1 || !goodcell || !udiff || !ev) return fail(CLV_ERR_INVALID, "visc_initialize: null buffer%s");
  const int bs = 256;
  if (pp->precision == 4)
    clv::visc_initialize_kernel<float><<<nblk(ncell(p), bs), bs, 0, S(stream)>>>(p, (float*)pi1, goodcell, (float*)udiff, (const float*)ev, (float)tau);
  else
    clv::visc_initialize_kernel<double><<<nblk(ncell(p), bs), bs, 0, S(stream)>>>(p, (double*)pi1, goodcell, (double*)udiff, (const double*)ev, tau);
  return cuda_check("visc_initialize_kernel");
}

int clv_get_udiff(const clv_params* pp, void* udiff, const void* ev0, const void* ev1, void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (!udiff || !ev0 || !ev1) return fail(CLV_ERR_INVALID, "get_udiff: null buffer%s");
  const int bs = 256;
  if (pp->precision == 4)
    clv::get_udiff_kernel<float><<<nblk(ncell(p), bs), bs, 0, S(stream)>>>(p, (float*)udiff, (const float*)ev0, (const float*)ev1);
  else
    clv::get_udiff_kernel<double><<<nblk(ncell(p), bs), bs, 0, S(stream)>>>(p, (double*)udiff, (const double*)ev0, (const double*)ev1);
  return cuda_check("get_udiff_kernel");
}

int clv_max_ed_reset(const clv_params* pp, void* key, void* stream) {
  if (!pp || !key || (pp->precision != 4 && pp->precision != 8)) return fail(CLV_ERR_INVALID, "max_ed_reset: bad argument%s");
  cudaMemsetAsync(key, 0, pp->precision, S(stream));
  return cuda_check("cudaMemsetAsync");
}

int clv_max_ed(const clv_params* pp, const void* ev, void* key, void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (!ev || !key) return fail(CLV_ERR_INVALID, "max_ed: null buffer%s");
  const long long n = ncell(p);
  unsigned int g = (unsigned int)((n + 255) / 256);
  if (g > 148u * 16u) g = 148u * 16u;
  if (pp->precision == 4)
    clv::max_key_kernel<float><<<g, 256, 0, S(stream)>>>((const float*)ev, n, (unsigned int*)key);
  else
    clv::max_key_kernel<double><<<g, 256, 0, S(stream)>>>((const double*)ev, n, (unsigned long long*)key);
  return cuda_check("max_key_kernel");
}

int clv_max_ed_read(const clv_params* pp, const void* key, double* out, void* stream) {
  if (!pp || !key || !out) return fail(CLV_ERR_INVALID, "max_ed_read: null argument%s");
  if (pp->precision == 4) {
    unsigned int k = 0;
    cudaMemcpyAsync(&k, key, sizeof(k), cudaMemcpyDeviceToHost, S(stream));
    cudaStreamSynchronize(S(stream));
    int rc = cuda_check("max_ed_read");
    if (rc) return rc;
    if (k == 0) { *out = -FLT_MAX; return CLV_OK; }
    unsigned int b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    memcpy(&f, &b, 4);
    *out = f;
  } else {
    unsigned long long k = 0;
    cudaMemcpyAsync(&k, key, sizeof(k), cudaMemcpyDeviceToHost, S(stream));
    cudaStreamSynchronize(S(stream));
    int rc = cuda_check("max_ed_read");
    if (rc) return rc;
    if (k == 0) { *out = -FLT_MAX; return CLV_OK; }
    unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    double f;
    memcpy(&f, &b, 8);
    *out = f;
  }
  return CLV_OK;
}

int clv_status(const clv_params* pp, const void* ev, const void* pi, int npi, const unsigned char* goodcell,
               const long long* sf_total, long long sf_capacity, long long* counts_dev, long long* counts_host,
               void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (!ev || !counts_dev || (pi && (npi < 1 || npi > 11)) || sf_capacity < 0)
    return fail(CLV_ERR_INVALID, "status: bad argument%s");
  const long long n = ncell(p);
  unsigned int g = nblk(n, 256);
  if (g > 148u * 8u) g = 148u * 8u;
  unsigned long long* out = reinterpret_cast<unsigned long long*>(counts_dev);
  cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), S(stream));
  if (pp->precision == 4) {
    clv::status_kernel<float><<<g, 256, 0, S(stream)>>>((const float*)ev, 4, p.ld, n, goodcell, sf_total, sf_capacity, out);
    if (pi) clv::status_kernel<float><<<g, 256, 0, S(stream)>>>((const float*)pi, npi, p.ld, n, nullptr, nullptr, 0, out);
  } else {
    clv::status_kernel<double><<<g, 256, 0, S(stream)>>>((const double*)ev, 4, p.ld, n, goodcell, sf_total, sf_capacity, out);
    if (pi) clv::status_kernel<double><<<g, 256, 0, S(stream)>>>((const double*)pi, npi, p.ld, n, nullptr, nullptr, 0, out);
  }
  rc = cuda_check("status_kernel");
  if (rc || !counts_host) return rc;
  cudaMemcpyAsync(counts_host, counts_dev, 3 * sizeof(long long), cudaMemcpyDeviceToHost, S(stream));
  cudaStreamSynchronize(S(stream));
  return cuda_check("status readback");
}

size_t clv_params_size(void) { return sizeof(clv_params); }

size_t clv_hypersf_scratch_bytes(const clv_params* pp) {
  clv::Params p;
  if (to_params(pp, &p)) return 0;
  return pp->precision == 4 ? hsf_scratch<float>(p) : hsf_scratch<double>(p);
}

int clv_hypersf_append(const clv_params* pp, int visc, double tau_old, double tau_new, const void* ev_old,
                       const void* ev_new, const void* pi_old, const void* pi_new, void* sf, void* txyz, void* pisf,
                       long long capacity, long long* total, void* scratch, size_t scratch_bytes, void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (capacity < 0) return fail(CLV_ERR_INVALID, "hypersf: negative capacity%s");
  if (pp->precision == 4)
    return hypersf_t<float>(p, visc, tau_old, tau_new, ev_old, ev_new, pi_old, pi_new, sf, txyz, pisf, capacity,
                            total, scratch, scratch_bytes, S(stream));
  return hypersf_t<double>(p, visc, tau_old, tau_new, ev_old, ev_new, pi_old, pi_new, sf, txyz, pisf, capacity,
                           total, scratch, scratch_bytes, S(stream));
}

int clv_aos_to_soa(const clv_params* pp, const void* aos, void* soa, long long n, int w, void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (!aos || !soa || n < 0 || n > p.ld || w < 1 || w > 16) return fail(CLV_ERR_INVALID, "aos_to_soa: bad argument%s");
  if (n == 0) return CLV_OK;
  if (pp->precision == 4)
    clv::aos_to_soa_kernel<float><<<nblk(n * w, 256), 256, 0, S(stream)>>>((const float*)aos, (float*)soa, n, w, p.ld);
  else
    clv::aos_to_soa_kernel<double><<<nblk(n * w, 256), 256, 0, S(stream)>>>((const double*)aos, (double*)soa, n, w, p.ld);
  return cuda_check("aos_to_soa_kernel");
}

int clv_soa_to_aos(const clv_params* pp, const void* soa, void* aos, long long n, int w, void* stream) {
  clv::Params p;
  int rc = to_params(pp, &p);
  if (rc) return rc;
  if (!aos || !soa || n < 0 || n > p.ld || w < 1 || w > 16) return fail(CLV_ERR_INVALID, "soa_to_aos: bad argument%s");
  if (n == 0) return CLV_OK;
  if (pp->precision == 4)
    clv::soa_to_aos_kernel<float><<<nblk(n * w, 256), 256, 0, S(stream)>>>((const float*)soa, (float*)aos, n, w, p.ld);
  else
    clv::soa_to_aos_kernel<double><<<nblk(n * w, 256), 256, 0, S(stream)>>>((const double*)soa, (double*)aos, n, w, p.ld);
  return cuda_check("soa_to_aos_kernel");
}

}  // extern "C"
