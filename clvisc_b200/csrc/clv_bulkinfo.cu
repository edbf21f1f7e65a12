// extern "C" entry points of the bulk-evolution diagnostics (declared in
// include/clvisc_b200.h).
#include <algorithm>
#include <string>

#include "../../include/clvisc_b200.h"
#include "clv_bulkinfo.cuh"

namespace clv_host {
int params_from_abi(const clv_params* in, clv::Params* out);
int set_error(int code, const std::string& msg);
int check_cuda(const char* where);
}  // namespace clv_host

namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }
constexpr int kLabBlocks = 148 * 8;

// sums the per-block partials of bulk_lab_kernel in block order, times the cell volume
__global__ void lab_finish_kernel(const double* part, int n, double volume, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double e = 0.0, s = 0.0;
  for (int b = 0; b < n; b++) {
    e += part[2 * b];
    s += part[2 * b + 1];
  }
  out[0] = e * volume;
  out[1] = s * volume;
}

}  // namespace

extern "C" {

long long clv_bulk_slices_size(const clv_params* p) {
  if (!p) return 0;
  const long long X = p->nx, Y = p->ny, Z = p->nz;
  return 4 * (X + Y + Z + X * Y + X * Z + Y * Z) + 3 * X * Y;
}

int clv_bulk_slices(const clv_params* pp, const void* ev, const void* pi, void* out, void* stream) {
  clv::Params p;
  int rc = clv_host::params_from_abi(pp, &p);
  if (rc) return rc;
  if (!ev || !out) return clv_host::set_error(CLV_ERR_INVALID, "bulk_slices: null buffer");
  const long long X = p.nx, Y = p.ny, Z = p.nz;
  const long long off[10] = {0, 4 * X, 4 * (X + Y), 4 * (X + Y + Z), 4 * (X + Y + Z + X * Y),
                             4 * (X + Y + Z + X * Y + X * Z), 4 * (X + Y + Z + X * Y + X * Z + Y * Z),
                             4 * (X + Y + Z + X * Y + X * Z + Y * Z) + X * Y,
                             4 * (X + Y + Z + X * Y + X * Z + Y * Z) + 2 * X * Y, 0};
  const int n = (int)std::max(X, std::max(Y, Z));
  cudaStream_t s = S(stream);
  dim3 g2((p.ny + 127) / 128, p.nx);
  if (pp->precision == 4) {
    float* o = (float*)out;
    clv::bulk_slices_kernel<float><<<(n + 127) / 128, 128, 0, s>>>(p, (const float*)ev, o + off[0], o + off[1],
                                                                    o + off[2], o + off[3], o + off[4], o + off[5]);
    if (pi) clv::bulk_pimn_kernel<float><<<g2, 128, 0, s>>>(p, (const float*)pi, o + off[6], o + off[7], o + off[8]);
  } else {
    double* o = (double*)out;
    clv::bulk_slices_kernel<double><<<(n + 127) / 128, 128, 0, s>>>(p, (const double*)ev, o + off[0], o + off[1],
                                                                     o + off[2], o + off[3], o + off[4], o + off[5]);
    if (pi) clv::bulk_pimn_kernel<double><<<g2, 128, 0, s>>>(p, (const double*)pi, o + off[6], o + off[7], o + off[8]);
  }
  return clv_host::check_cuda("bulk_slices");
}

int clv_bulk_sums(const clv_params* pp, const void* ev, const void* pi, double* out, void* stream) {
  clv::Params p;
  int rc = clv_host::params_from_abi(pp, &p);
  if (rc) return rc;
  if (!ev || !out) return clv_host::set_error(CLV_ERR_INVALID, "bulk_sums: null buffer");
  if (pp->precision == 4)
    clv::bulk_sums_kernel<float><<<p.nz, clv::BULK_SUM_THREADS, 0, S(stream)>>>(p, (const float*)ev,
                                                                                (const float*)pi, out);
  else
    clv::bulk_sums_kernel<double><<<p.nz, clv::BULK_SUM_THREADS, 0, S(stream)>>>(p, (const double*)ev,
                                                                                 (const double*)pi, out);
  return clv_host::check_cuda("bulk_sums_kernel");
}

size_t clv_bulk_lab_scratch_bytes(void) { return (size_t)kLabBlocks * 2 * sizeof(double); }

int clv_bulk_lab_totals(const clv_params* pp, const void* ev, double tau, double volume, double* out, void* scratch,
                        size_t scratch_bytes, void* stream) {
  clv::Params p;
  int rc = clv_host::params_from_abi(pp, &p);
  if (rc) return rc;
  if (!ev || !out || !scratch || scratch_bytes < clv_bulk_lab_scratch_bytes())
    return clv_host::set_error(CLV_ERR_INVALID, "bulk_lab_totals: null buffer or scratch too small");
  const long long N = (long long)p.nx * p.ny * p.nz;
  const long long chunk = (N + kLabBlocks - 1) / kLabBlocks;
  double* part = (double*)scratch;
  cudaStream_t s = S(stream);
  if (pp->precision == 4)
    clv::bulk_lab_kernel<float><<<kLabBlocks, clv::BULK_SUM_THREADS, 0, s>>>(p, (const float*)ev, (float)tau, chunk,
                                                                             part);
  else
    clv::bulk_lab_kernel<double><<<kLabBlocks, clv::BULK_SUM_THREADS, 0, s>>>(p, (const double*)ev, tau, chunk,
                                                                              part);
  lab_finish_kernel<<<1, 32, 0, s>>>(part, kLabBlocks, volume, out);
  return clv_host::check_cuda("bulk_lab_kernel");
}

}  // extern "C"
