// extern "C" entry points of the Cooper-Frye smooth spectra (declared in
// include/clvisc_b200.h).
#include <algorithm>
#include <string>

#include "../../include/clvisc_b200.h"
#include "clv_spectra.cuh"

namespace clv_host {
int set_error(int code, const std::string& msg);
int check_cuda(const char* where);
}  // namespace clv_host

namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// surface chunks per rapidity: enough blocks to fill the GPU a few times
int spectra_chunks(long long n, int ny) {
  long long want = (148LL * 4 + ny - 1) / ny;
  long long most = std::max(1LL, (n + clv::SPEC_TILE - 1) / clv::SPEC_TILE);
  return (int)std::max(1LL, std::min(want, most));
}

template <class real>
int spectra_t(const clv_spectra_args* a, void* out, void* scratch, cudaStream_t s) {
  const long long np = (long long)a->ny * a->npt * a->nphi;
  const int nchunk = spectra_chunks(a->n, a->ny);
  const long long chunk = (a->n + nchunk - 1) / nchunk;
  double* part = (double*)scratch;
  clv::SpecHadron h{a->mass, a->gspin, a->fermi_boson, a->mu};
  dim3 grid(nchunk, a->ny);
  const int threads = ((a->npt * a->nphi + 31) / 32) * 32;
  if (a->pisf)
    clv::spectra_kernel<real, true><<<grid, threads, 0, s>>>(
        (const real*)a->sf, (const real*)a->pisf, a->n, chunk, h, (real)a->tfrz, (real)a->tcoeff, (const real*)a->y,
        (const real*)a->pt, (const real*)a->cphi, (const real*)a->sphi, a->npt, a->nphi, part);
  else
    clv::spectra_kernel<real, false><<<grid, threads, 0, s>>>(
        (const real*)a->sf, nullptr, a->n, chunk, h, (real)a->tfrz, (real)0, (const real*)a->y, (const real*)a->pt,
        (const real*)a->cphi, (const real*)a->sphi, a->npt, a->nphi, part);
  clv::spectra_finish_kernel<real><<<(unsigned)((np + 255) / 256), 256, 0, s>>>(part, nchunk, np, (real*)out);
  return clv_host::check_cuda("spectra_kernel");
}

}  // namespace

extern "C" {

size_t clv_spectra_scratch_bytes(long long n, int ny, int npt, int nphi) {
  if (n < 0 || ny < 1 || npt < 1 || nphi < 1) return 0;
  return (size_t)spectra_chunks(n, ny) * ny * npt * nphi * sizeof(double);
}

int clv_spectra(const clv_spectra_args* a, void* out, void* scratch, size_t scratch_bytes, void* stream) {
  if (!a || !out || !scratch || (a->n > 0 && !a->sf) || !a->y || !a->pt || !a->cphi || !a->sphi)
    return clv_host::set_error(CLV_ERR_INVALID, "spectra: null argument");
  if (a->precision != 4 && a->precision != 8) return clv_host::set_error(CLV_ERR_INVALID, "spectra: precision must be 4 or 8");
  if (a->ny < 1 || a->npt < 1 || a->nphi < 1 || a->npt * a->nphi > 1024 || a->n < 0)
    return clv_host::set_error(CLV_ERR_INVALID, "spectra: grid sizes must be >= 1 with npt * nphi <= 1024");
  if (!(a->tfrz > 0.0)) return clv_host::set_error(CLV_ERR_INVALID, "spectra: tfrz must be > 0");
  if (scratch_bytes < clv_spectra_scratch_bytes(a->n, a->ny, a->npt, a->nphi))
    return clv_host::set_error(CLV_ERR_INVALID, "spectra: scratch too small");
  if (a->precision == 4) return spectra_t<float>(a, out, scratch, S(stream));
  return spectra_t<double>(a, out, scratch, S(stream));
}

}  // extern "C"
