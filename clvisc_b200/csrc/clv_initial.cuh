// Initial conditions on the device.
//
// glauber_ini_kernel restates the reference's optical Glauber model
// (kernel_glauber.cl:9-102): Woods-Saxon thickness functions integrated along
// z with 10 x 5-point Gauss-Legendre, wounded-nucleon / binary-collision
// two-component energy density scaled so that the centre of a head-on
// collision has Edmax, times the plateau-with-Gaussian-tails profile in
// eta_s. It uses exp and pow, so it matches a CPU evaluation to a few ulp,
// not bit for bit.
//
// hotspot kernels build the seeded Monte Carlo Glauber profile: the
// participants and their Gamma weights are sampled on the host; each cell
// sums w_p * gx_p(i) * gy_p(j) over the participants in the host's order, with
// the one-dimensional Gaussian factors tabulated once per participant, in
// double precision like the host construction (initial.py).
#pragma once
#include "clv_device.cuh"

namespace clv {

struct GlauberConsts {  // layout of clv_glauber: the -D literals of glauber.py:79-90
  float NumOfNucleons, SQRTS, Ro0, R, Eta, Si0, ImpactParameter, Edmax, Hwn, Eta_flat, Eta_gw;
};

// kernel_glauber.cl:10-32
template <class real> __device__ real glauber_thickness(const GlauberConsts& g, real x, real y) {
  const real zk[5] = {-0.9061798f, -0.5386492f, 0.0f, 0.5386493f, 0.9061798f};
  const real Ak[5] = {0.2369269f, 0.4786287f, 0.5688889f, 0.4786287f, 0.2369269f};
  real thickness = 0.0f;
  real cut = 5.0f * g.R;
  for (int j = 0; j != 10; ++j) {
    real a = j * cut / 10.0f;
    real b = (j + 1) * cut / 10.0f;
    for (int i = 0; i != 5; ++i) {
      real z = (a + b) / 2.0f + (b - a) / 2.0f * zk[i];
      real r = sqrt(x * x + y * y + z * z);
      real f = g.Ro0 / (1.0f + exp((r - g.R) / g.Eta));
      thickness = thickness + Ak[i] * f * (b - a) / 2.0f;
    }
  }
  return 2.0f * thickness;
}

// kernel_glauber.cl:75-83
template <class real> __device__ real glauber_nw(const GlauberConsts& g, real Ta, real Tb) {
  return Ta * (1.0f - pow(1.0f - g.Si0 * Tb / g.NumOfNucleons, (real)g.NumOfNucleons)) +
         Tb * (1.0f - pow(1.0f - g.Si0 * Ta / g.NumOfNucleons, (real)g.NumOfNucleons));
}
template <class real> __device__ real glauber_nb(const GlauberConsts& g, real Ta, real Tb) {
  return g.Si0 * Ta * Tb;
}
// kernel_glauber.cl:50-52
template <class real> __device__ real glauber_ed_transverse(const GlauberConsts& g, real Ta, real Tb) {
  return (g.Hwn * glauber_nw<real>(g, Ta, Tb) + (1.0f - g.Hwn) * glauber_nb<real>(g, Ta, Tb));
}
// kernel_glauber.cl:35-47 (without BJORKEN_SCALING, which glauber.py never sets)
template <class real> __device__ real glauber_weight_along_eta(const GlauberConsts& g, real z, real etas0) {
  real heta;
  if (fabs(z - etas0) > g.Eta_flat) {
    heta = exp(-pow(fabs(z - etas0) - g.Eta_flat, (real)2.0f) / (2.0f * g.Eta_gw * g.Eta_gw));
  } else {
    heta = 1.0f;
  }
  return heta;
}

// kernel_glauber.cl:86-102: one thread per (i, j), all k; ev in SoA planes.
// The rapidity twist etas0() of kernel_glauber.cl:57-67 returns 0.
template <class real> __global__ void glauber_ini_kernel(Params p, GlauberConsts g, real* ev) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nx || j >= p.ny) return;
  const long long ld = p.ld;
  real x = (i - p.nx / 2) * (real)p.DX;
  real y = (j - p.ny / 2) * (real)p.DY;
  real Tcent = glauber_thickness<real>(g, 0.0f, 0.0f);
  real ed_central = glauber_ed_transverse<real>(g, Tcent, Tcent);
  real kFactor = g.Edmax / ed_central;
  real b = g.ImpactParameter;
  real Ta = glauber_thickness<real>(g, x - 0.5f * b, y);
  real Tb = glauber_thickness<real>(g, x + 0.5f * b, y);
  real edxy = kFactor * glauber_ed_transverse<real>(g, Ta, Tb);
  real etas0 = 0.0f;
  for (int k = 0; k < p.nz; k++) {
    real etas = (k - p.nz / 2) * (real)p.DZ;
    real heta = glauber_weight_along_eta<real>(g, etas, etas0);
    const long long I = ((long long)i * p.ny + j) * p.nz + k;
    ev[I] = edxy * heta;
    ev[ld + I] = 0.0f;
    ev[2 * ld + I] = 0.0f;
    ev[3 * ld + I] = 0.0f;
  }
}

// kernel_glauber.cl:104-121: binary collisions on an (nx, ny) grid from (xlow, ylow)
template <class real>
__global__ void glauber_nbinary_kernel(GlauberConsts g, real* out, real xlow, real ylow, real dx, real dy, int nx,
                                       int ny) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx || j >= ny) return;
  real x = xlow + i * dx;
  real y = ylow + j * dy;
  real b = g.ImpactParameter;
  real Ta = glauber_thickness<real>(g, x - 0.5f * b, y);
  real Tb = glauber_thickness<real>(g, x + 0.5f * b, y);
  out[(long long)i * ny + j] = glauber_nb<real>(g, Ta, Tb);
}

// ------------------------------------------------------------- hotspots
// Gaussian factors gx[p][i] = exp(-((i - nx/2) dx - px)^2 inv) for i < nx and
// gy[p][j] likewise, with inv = 1 / (2 width^2); parts = (x, y, w) per participant.
__global__ void hotspot_factor_kernel(const double* parts, int n, int nx, int ny, double dx, double dy, double inv,
                                      double* gx, double* gy) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)nx + ny;
  if (t >= per * n) return;
  const int p = (int)(t / per);
  const int q = (int)(t % per);
  if (q < nx) {
    double x = (double)(q - nx / 2) * dx;
    double d = x - parts[3 * p];
    gx[(long long)p * nx + q] = exp(-(d * d) * inv);
  } else {
    const int j = q - nx;
    double y = (double)(j - ny / 2) * dy;
    double d = y - parts[3 * p + 1];
    gy[(long long)p * ny + j] = exp(-(d * d) * inv);
  }
}

// exy[i][j] = sum_p w_p (gx[p][i] gy[p][j]) in participant order; the running
// maximum of exy goes into *key (ordered bits of a non-negative double).
__global__ void hotspot_sum_kernel(const double* parts, int n, int nx, int ny, const double* gx, const double* gy,
                                   double* exy, unsigned long long* key) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (j < ny) {
    for (int p = 0; p < n; p++) acc = acc + parts[3 * p + 2] * (gx[(long long)p * nx + i] * gy[(long long)p * ny + j]);
    exy[(long long)i * ny + j] = acc;
  }
  unsigned long long k = (j < ny && acc == acc) ? fkey(acc) : 0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long other = __shfl_xor_sync(0xffffffffu, k, o);
    k = other > k ? other : k;
  }
  if ((threadIdx.x & 31) == 0 && k) atomicMax(key, k);
}

// ev = (exy * h(eta_k) * (edmax / max exy), 0, 0, 0), eta_k = (k - nz/2) dz in
// double, with the plateau profile
// h = 1 for |eta| <= plateau, exp(-(|eta| - plateau)^2 / (2 sigma^2)) beyond.
template <class real>
__global__ void hotspot_fill_kernel(Params p, const double* exy, const unsigned long long* key, double edmax,
                                    double dz, double plateau, double sigma, real* ev) {
  const long long N = (long long)p.nx * p.ny * p.nz;
  const long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= N) return;
  const int k = (int)(I % p.nz);
  const long long ij = I / p.nz;
  const unsigned long long kb = *key;
  const unsigned long long bits = (kb & 0x8000000000000000ull) ? (kb & 0x7fffffffffffffffull) : ~kb;
  const double mx = __longlong_as_double((long long)bits);
  double eta = (double)(k - p.nz / 2) * dz;
  double h = 1.0;
  if (fabs(eta) > plateau) {
    double d = fabs(eta) - plateau;
    h = exp(-(d * d) / (2.0 * sigma * sigma));
  }
  const long long ld = p.ld;
  ev[I] = (real)((exy[ij] * h) * (edmax / mx));
  ev[ld + I] = 0.0f;
  ev[2 * ld + I] = 0.0f;
  ev[3 * ld + I] = 0.0f;
}

}  // namespace clv
