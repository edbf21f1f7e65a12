// clv_hypersf_append_noalloc: the freeze-out surface finder for callers that
// cannot allocate device memory.
//
// Who needs it: a host application that owns all device memory through its own
// pool and does not let libraries allocate, or a time-critical loop where a
// cudaMalloc (which may synchronise the whole device) is not acceptable. Such a
// caller cannot provide the scratch buffer clv_hypersf_append asks for, so this
// entry point keeps its scratch in a fixed array inside the library instead.
//
// The scratch is a file-scope __device__ array of NOALLOC_MAX_BLOCKS block
// counts plus two counters (about 1 MB). Every GPU that loads the library holds
// it until the process exits. It limits one call to NOALLOC_MAX_CUBES coarse
// cubes ((NX-1)/nxskip+1) x ((NY-1)/nyskip+1) x ((NZ-1)/nzskip+1); larger grids
// are rejected with CLV_ERR_INVALID.
//
// To need no per-cube storage, this variant does not keep the marks and the
// cube list of clv_hypersf_append: it counts emitting cubes per block, scans the
// counts, and then every cube decides again whether it emits and, if so, writes
// its element at (elements already present) + (block offset) + (rank inside the
// block). The marks and the elements are computed by the same device functions
// as in clv_hypersf_append, so the output is identical, element for element.
//
// Calls share the array: two calls whose launches overlap on the GPU (for
// example on two streams) race and corrupt each other's results; serialise them.
// Each call writes every block count and both counters it reads before reading
// them, so nothing left from a previous call is used.
//
// The array's device address is looked up with cudaGetSymbolAddress, with the
// call's device current, on every call made outside stream capture (so it is
// right again after a cudaDeviceReset); a call during capture reuses the
// address of the last call outside capture on that device. The first call on
// each device should therefore come before any stream capture.
#include <mutex>
#include <string>

#include "../../include/clvisc_b200.h"
#include "clv_device.cuh"
#define CLV_HSF_NO_SHARED_KERNELS  // the library's other unit defines the shared kernels
#include "clv_hypersf.cuh"

namespace clv_host {
extern thread_local std::string g_err;  // message behind clv_last_error()
}

namespace {

constexpr long long NOALLOC_MAX_CUBES = 1ll << 26;
constexpr int NOALLOC_BLOCK = 256;
constexpr long long NOALLOC_MAX_BLOCKS = NOALLOC_MAX_CUBES / NOALLOC_BLOCK;

struct NoallocScratch {
  int block_count[NOALLOC_MAX_BLOCKS];  // emitting cubes per block, then offsets
  long long count;                      // elements emitted by this call
  long long pad[31];
};
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

std::mutex g_noalloc_mu;
NoallocScratch* g_noalloc_addr[256] = {nullptr};

int noalloc_fail(int code, const std::string& msg) {
  clv_host::g_err = msg;
  return code;
}

// exclusive scan of n block counts in one block of 1024 threads; sum -> *total
__global__ void noalloc_scan_kernel(int* block_count, int n, long long* total) {
  __shared__ long long warp_sum[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    int t = base + threadIdx.x;
    long long v = t < n ? block_count[t] : 0;
    long long x = v;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    if (w == 0) {
      long long sum = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, sum, o);
        if (lane >= o) sum += y;
      }
      warp_sum[lane] = sum;
    }
    __syncthreads();
    long long excl = carry + (w > 0 ? warp_sum[w - 1] : 0) + x - v;
    if (t < n) block_count[t] = (int)excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void noalloc_advance_kernel(const long long* count, long long* total) { *total += *count; }

// device address of the scratch array on the current device. Outside stream
// capture the address is looked up again on every call, so a context that was
// torn down and rebuilt (cudaDeviceReset) never leaves a stale pointer behind;
// during capture, where that lookup is best avoided, the address cached by the
// last call outside capture on this device is used.
int noalloc_scratch(NoallocScratch** out, cudaStream_t s) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256)
    return noalloc_fail(CLV_ERR_CUDA, "hypersf_noalloc: no current CUDA device");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess)
    return noalloc_fail(CLV_ERR_CUDA, "hypersf_noalloc: cudaStreamIsCapturing failed");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (cap == cudaStreamCaptureStatusNone || !g_noalloc_addr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      return noalloc_fail(CLV_ERR_CUDA, std::string("hypersf_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_addr[dev] = static_cast<NoallocScratch*>(ptr);
  }
  *out = g_noalloc_addr[dev];
  return CLV_OK;
}

// whether coarse cube q emits an element (the test of hsf_mark_kernel)
template <class real>
__device__ __forceinline__ int cube_emits(const clv::Params& p, const real* ev_old, const real* ev_new, int visc,
                                          long long q, const clv::CubeGrid& g) {
  int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.ny * g.nz));
  real ed[16];
  const real efrz = p.EFRZ;
  if (!clv::load_cube(p, ev_old, ev_new, i, j, k, ed) || !clv::crosses(ed, efrz)) return 0;
  if (visc) {
    clv::R4<real> all[32];
    int n;
    clv::all_intersections(ed, efrz, all, &n);
    clv::R4<real> mc = clv::mass_center(all, n);
    if (isnan(mc.x)) return 0;
  }
  return 1;
}

template <class real>
__global__ void noalloc_count_kernel(clv::Params p, const real* ev_old, const real* ev_new, int visc, int* block_count) {
  const clv::CubeGrid g = clv::cube_grid(p);
  const long long nc = (long long)g.nx * g.ny * g.nz;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int emit = (q < nc) ? cube_emits(p, ev_old, ev_new, visc, q, g) : 0;
  int c = __syncthreads_count(emit);
  if (threadIdx.x == 0) block_count[blockIdx.x] = c;
}

// each emitting cube writes its element at total + block offset + rank in block
template <class real>
__global__ void noalloc_element_kernel(clv::Params p, const real* ev_old, const real* ev_new, const real* pi_old,
                                       const real* pi_new, real time_old, real time_new, int visc,
                                       const int* block_offset, const long long* total_in, real* sf, real* txyz,
                                       real* pisf, long long capacity) {
  __shared__ int warp_tot[NOALLOC_BLOCK / 32];
  const clv::CubeGrid g = clv::cube_grid(p);
  const long long nc = (long long)g.nx * g.ny * g.nz;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int emit = (q < nc) ? cube_emits(p, ev_old, ev_new, visc, q, g) : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned int bal = __ballot_sync(0xffffffffu, emit);
  if (lane == 0) warp_tot[w] = __popc(bal);
  __syncthreads();
  if (!emit) return;
  int rank = __popc(bal & ((1u << lane) - 1u));
  for (int u = 0; u < w; u++) rank += warp_tot[u];
  const long long o = *total_in + block_offset[blockIdx.x] + rank;
  if (o >= capacity) return;
  const long long ld = p.ld;
  const real efrz = p.EFRZ;
  int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.ny * g.nz));
  real ed[16];
  clv::load_cube(p, ev_old, ev_new, i, j, k, ed);
  clv::R4<real> all[32];
  int n;
  clv::all_intersections(ed, efrz, all, &n);
  clv::R4<real> flow = clv::energy_flow(ed, efrz);
  clv::R4<real> mc = clv::mass_center(all, n);
  clv::R4<real> dS = clv::calc_area(all, flow, n, i * j * k);
  real dtd = time_new - time_old;
  real dxd = p.nxskip * p.DX;
  real dyd = p.nyskip * p.DY;
  real dzd = p.nzskip * p.DZ;
  real tau = time_old + mc.x * dtd;
  real x = (-p.nx) / 2 * p.DX + i * dxd + mc.y * dxd;
  real y = (-p.ny) / 2 * p.DY + j * dyd + mc.z * dyd;
  real eta = (-p.nz) / 2 * p.DZ + k * dzd + mc.w * dzd;
  real v[4];
#pragma unroll
  for (int c = 1; c < 4; c++) {
    real acc = 0.0f;
    for (int qq = 0; qq < 16; qq++) {
      const real* src = qq < 8 ? ev_old : ev_new;
      real t = clv::corner_weight(mc, qq) * src[c * ld + clv::corner_cell(p, i, j, k, qq & 7)];
      acc = (qq == 0) ? t : acc + t;
    }
    v[c] = acc;
  }
  real* r8 = sf + 8 * o;
  r8[0] = tau * dxd * dyd * dzd * dS.x;
  r8[1] = -tau * dtd * dyd * dzd * dS.y;
  r8[2] = -tau * dtd * dxd * dzd * dS.z;
  r8[3] = -dtd * dxd * dyd * dS.w;
  r8[4] = v[1];
  r8[5] = v[2];
  r8[6] = v[3];
  r8[7] = eta;
  real* r4 = txyz + 4 * o;
  r4[0] = tau * cosh(eta);
  r4[1] = x;
  r4[2] = y;
  r4[3] = tau * sinh(eta);
  if (visc && pisf) {
    for (int mn = 0; mn < 10; mn++) {
      real acc = 0.0f;
      for (int qq = 0; qq < 16; qq++) {
        const real* src = qq < 8 ? pi_old : pi_new;
        real t = clv::corner_weight(mc, qq) * src[mn * ld + clv::corner_cell(p, i, j, k, qq & 7)];
        acc = (qq == 0) ? t : acc + t;
      }
      pisf[10 * o + mn] = acc;
    }
  }
}

template <class real>
int noalloc_run(const clv_params* pp, int visc, double tau_old, double tau_new, const void* ev_old, const void* ev_new,
                const void* pi_old, const void* pi_new, void* sf, void* txyz, void* pisf, long long capacity,
                long long* total, cudaStream_t s) {
  clv::Params p;
  p.nx = pp->nx; p.ny = pp->ny; p.nz = pp->nz; p.ld = pp->ld;
  p.DT = pp->dt; p.DX = pp->dx; p.DY = pp->dy; p.DZ = pp->dz; p.TAU0 = pp->tau0;
  p.ETAOS_XMIN = pp->etaos_xmin; p.ETAOS_YMIN = pp->etaos_ymin;
  p.ETAOS_LEFT_SLOP = pp->etaos_left_slop; p.ETAOS_RIGHT_SLOP = pp->etaos_right_slop; p.LAM1 = pp->lam1;
  p.EFRZ = pp->efrz;
  p.nxskip = pp->nxskip; p.nyskip = pp->nyskip; p.nzskip = pp->nzskip;
  p.eos_start = pp->eos_ed_start; p.eos_step = pp->eos_ed_step;
  p.eos_num = pp->eos_num_ed; p.eos_nrow = pp->eos_nrow; p.eos_ncol = pp->eos_ncol;
  p.eos = pp->eos_table;
  p.eos_p2 = nullptr;  // the surface kernels use the exact lookup
  for (int q = 0; q < 4; q++) p.opt[q] = 0;
  p.flags = pp->flags;
  const clv::CubeGrid g = clv::cube_grid(p);
  const long long nc = (long long)g.nx * g.ny * g.nz;
  if (nc > NOALLOC_MAX_CUBES)
    return noalloc_fail(CLV_ERR_INVALID, "hypersf_noalloc: " + std::to_string(nc) + " coarse cubes exceed the limit of " +
                                             std::to_string(NOALLOC_MAX_CUBES) + "; use clv_hypersf_append");
  NoallocScratch* scr = nullptr;
  int rc = noalloc_scratch(&scr, s);
  if (rc) return rc;
  const unsigned int nb = (unsigned int)((nc + NOALLOC_BLOCK - 1) / NOALLOC_BLOCK);
  noalloc_count_kernel<real><<<nb, NOALLOC_BLOCK, 0, s>>>(p, (const real*)ev_old, (const real*)ev_new, visc,
                                                          scr->block_count);
  noalloc_scan_kernel<<<1, 1024, 0, s>>>(scr->block_count, (int)nb, &scr->count);
  noalloc_element_kernel<real><<<nb, NOALLOC_BLOCK, 0, s>>>(
      p, (const real*)ev_old, (const real*)ev_new, (const real*)pi_old, (const real*)pi_new, (real)tau_old,
      (real)tau_new, visc, scr->block_count, total, (real*)sf, (real*)txyz, (real*)pisf, capacity);
  noalloc_advance_kernel<<<1, 1, 0, s>>>(&scr->count, total);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(CLV_ERR_CUDA, std::string("hypersf_noalloc: ") + cudaGetErrorString(e));
  return CLV_OK;
}

}  // namespace

extern "C" int clv_hypersf_append_noalloc(const clv_params* p, int visc, double tau_old, double tau_new,
                                          const void* ev_old, const void* ev_new, const void* pi_old,
                                          const void* pi_new, void* sf, void* txyz, void* pisf, long long capacity,
                                          long long* total, void* stream) {
  if (!p || (p->precision != 4 && p->precision != 8)) return noalloc_fail(CLV_ERR_INVALID, "hypersf_noalloc: bad params");
  if (p->nx < 1 || p->ny < 1 || p->nz < 1 || p->nxskip < 1 || p->nyskip < 1 || p->nzskip < 1 ||
      p->ld < (long long)p->nx * p->ny * p->nz || !p->eos_table)
    return noalloc_fail(CLV_ERR_INVALID, "hypersf_noalloc: bad grid");
  if (!ev_old || !ev_new || !sf || !txyz || !total || capacity < 0)
    return noalloc_fail(CLV_ERR_INVALID, "hypersf_noalloc: null pointer or negative capacity");
  if (visc && (!pi_old || !pi_new)) return noalloc_fail(CLV_ERR_INVALID, "hypersf_noalloc: visc needs pi_old and pi_new");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (p->precision == 4)
    return noalloc_run<float>(p, visc, tau_old, tau_new, ev_old, ev_new, pi_old, pi_new, sf, txyz, pisf, capacity,
                              total, s);
  return noalloc_run<double>(p, visc, tau_old, tau_new, ev_old, ev_new, pi_old, pi_new, sf, txyz, pisf, capacity,
                             total, s);
}
