// extern "C" entry points of the initial-condition generators (declared in
// include/clvisc_b200.h).
#include <string>

#include "../../include/clvisc_b200.h"
#include "clv_initial.cuh"

namespace clv_host {
int params_from_abi(const clv_params* in, clv::Params* out);
int set_error(int code, const std::string& msg);
int check_cuda(const char* where);
}  // namespace clv_host

namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }
static_assert(sizeof(clv_glauber) == sizeof(clv::GlauberConsts), "clv_glauber layout");

clv::GlauberConsts glauber_consts(const clv_glauber* g) {
  clv::GlauberConsts c;
  c.NumOfNucleons = g->num_of_nucleons;
  c.SQRTS = g->sqrts;
  c.Ro0 = g->ro0;
  c.R = g->r;
  c.Eta = g->eta;
  c.Si0 = g->si0;
  c.ImpactParameter = g->impact_parameter;
  c.Edmax = g->edmax;
  c.Hwn = g->hwn;
  c.Eta_flat = g->eta_flat;
  c.Eta_gw = g->eta_gw;
  return c;
}

inline size_t align256(size_t n) { return (n + 255) / 256 * 256; }

size_t hotspot_bytes(long long nx, long long ny, long long n) {
  return align256((size_t)(n * nx) * 8) + align256((size_t)(n * ny) * 8) + align256((size_t)(nx * ny) * 8) + 256;
}

}  // namespace

extern "C" {

int clv_glauber_ini(const clv_params* pp, const clv_glauber* g, void* ev, void* stream) {
  clv::Params p;
  int rc = clv_host::params_from_abi(pp, &p);
  if (rc) return rc;
  if (!g || !ev) return clv_host::set_error(CLV_ERR_INVALID, "glauber_ini: null argument");
  const clv::GlauberConsts c = glauber_consts(g);
  dim3 grid((p.ny + 127) / 128, p.nx);
  if (pp->precision == 4) clv::glauber_ini_kernel<float><<<grid, 128, 0, S(stream)>>>(p, c, (float*)ev);
  else clv::glauber_ini_kernel<double><<<grid, 128, 0, S(stream)>>>(p, c, (double*)ev);
  return clv_host::check_cuda("glauber_ini_kernel");
}

int clv_glauber_nbinary(const clv_params* pp, const clv_glauber* g, void* out, double xlow, double ylow, double dx,
                        double dy, int nx, int ny, void* stream) {
  if (!pp || !g || !out || nx < 1 || ny < 1 || (pp->precision != 4 && pp->precision != 8))
    return clv_host::set_error(CLV_ERR_INVALID, "glauber_nbinary: bad argument");
  const clv::GlauberConsts c = glauber_consts(g);
  dim3 grid((ny + 127) / 128, nx);
  if (pp->precision == 4)
    clv::glauber_nbinary_kernel<float><<<grid, 128, 0, S(stream)>>>(c, (float*)out, (float)xlow, (float)ylow,
                                                                     (float)dx, (float)dy, nx, ny);
  else
    clv::glauber_nbinary_kernel<double><<<grid, 128, 0, S(stream)>>>(c, (double*)out, xlow, ylow, dx, dy, nx, ny);
  return clv_host::check_cuda("glauber_nbinary_kernel");
}

size_t clv_hotspot_scratch_bytes(const clv_params* pp, int n_parts) {
  if (!pp || n_parts < 0 || pp->nx < 1 || pp->ny < 1) return 0;
  return hotspot_bytes(pp->nx, pp->ny, n_parts);
}

int clv_hotspot_ini(const clv_params* pp, void* ev, const double* parts, int n_parts, double dx, double dy,
                    double dz, double width, double plateau, double sigma_eta, double edmax, void* scratch,
                    size_t scratch_bytes, void* stream) {
  clv::Params p;
  int rc = clv_host::params_from_abi(pp, &p);
  if (rc) return rc;
  if (!ev || !scratch || (n_parts > 0 && !parts) || n_parts < 1)
    return clv_host::set_error(CLV_ERR_INVALID, "hotspot_ini: null buffer or no participants");
  if (!(width > 0.0) || !(sigma_eta > 0.0) || !(edmax > 0.0))
    return clv_host::set_error(CLV_ERR_INVALID, "hotspot_ini: width, sigma_eta and edmax must be > 0");
  if (scratch_bytes < hotspot_bytes(p.nx, p.ny, n_parts) || (reinterpret_cast<uintptr_t>(scratch) % 256))
    return clv_host::set_error(CLV_ERR_INVALID, "hotspot_ini: scratch too small or not 256-byte aligned");
  char* base = static_cast<char*>(scratch);
  double* gx = reinterpret_cast<double*>(base);
  double* gy = reinterpret_cast<double*>(base + align256((size_t)n_parts * p.nx * 8));
  double* exy = reinterpret_cast<double*>(reinterpret_cast<char*>(gy) + align256((size_t)n_parts * p.ny * 8));
  unsigned long long* key =
      reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(exy) + align256((size_t)p.nx * p.ny * 8));
  cudaStream_t s = S(stream);
  cudaMemsetAsync(key, 0, 8, s);
  const double inv = 1.0 / (2.0 * width * width);
  const long long nf = (long long)n_parts * (p.nx + p.ny);
  clv::hotspot_factor_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(parts, n_parts, p.nx, p.ny, dx, dy, inv, gx,
                                                                          gy);
  dim3 g2((p.ny + 127) / 128, p.nx);
  clv::hotspot_sum_kernel<<<g2, 128, 0, s>>>(parts, n_parts, p.nx, p.ny, gx, gy, exy, key);
  const long long N = (long long)p.nx * p.ny * p.nz;
  const unsigned nb = (unsigned)((N + 255) / 256);
  if (pp->precision == 4)
    clv::hotspot_fill_kernel<float><<<nb, 256, 0, s>>>(p, exy, key, edmax, dz, plateau, sigma_eta, (float*)ev);
  else
    clv::hotspot_fill_kernel<double><<<nb, 256, 0, s>>>(p, exy, key, edmax, dz, plateau, sigma_eta, (double*)ev);
  return clv_host::check_cuda("hotspot kernels");
}

}  // extern "C"
