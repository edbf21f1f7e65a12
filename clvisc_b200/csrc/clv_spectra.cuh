// Cooper-Frye smooth spectra dN/(dY pt dpt dphi) of one hadron species on the
// freeze-out surface (CLSmoothSpec/src/kernel_spec.cl:4-141 for ideal
// surfaces, kernel_spec_csc.cl:4-101 with the viscous correction delta f).
//
// Layout: block (c, k) takes the rapidity Y[k] and the c-th contiguous chunk
// of surface elements; its NPT x NPHI threads each own one (pt, phi) point.
// Elements are staged through shared memory in tiles, with the per-element
// factors that do not depend on (pt, phi) (gamma or u^mu, cosh and sinh of
// Y - eta_s) computed once per tile. Each thread sums its point over the chunk
// in double, in element order; spectra_finish adds the chunks in order, so
// the result does not depend on scheduling.
#pragma once
#include "clv_device.cuh"

namespace clv {

constexpr int SPEC_TILE = 64;

struct SpecHadron {
  double mass, gspin, fermi_boson, muB;
};

template <class real, bool VISCOUS>
__global__ void spectra_kernel(const real* sf, const real* pisf, long long n, long long chunk, SpecHadron h,
                               real tfrz, real tcoeff, const real* Y, const real* Pt, const real* cphi,
                               const real* sphi, int npt, int nphi, double* part) {
  __shared__ real s_sf[SPEC_TILE][8];
  __shared__ real s_g[SPEC_TILE][4];  // gamma (ideal) or u^0..u^3 (viscous)
  __shared__ real s_ch[SPEC_TILE], s_sh[SPEC_TILE];
  __shared__ real s_pi[VISCOUS ? SPEC_TILE : 1][10];
  const int c = blockIdx.x, k = blockIdx.y, ny = gridDim.y;
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const bool active = tid < npt * nphi;
  const int l = active ? tid / nphi : 0, m = active ? tid % nphi : 0;
  const real mass = (real)h.mass, fb = (real)h.fermi_boson, muB = (real)h.muB;
  // dof = gspin / (2 pi)^3 (kernel_spec.cl:30)
  const real dof = (real)(h.gspin / ((2.0 * 3.14159265358979323846) * (2.0 * 3.14159265358979323846) *
                                     (2.0 * 3.14159265358979323846)));
  const real rapidity = Y[k];
  const real pt = Pt[l];
  const real mt = sqrt(mass * mass + pt * pt);
  const real px = pt * cphi[m], py = pt * sphi[m];
  double acc = 0.0;
  const long long lo = (long long)c * chunk, hi = min(n, lo + chunk);
  for (long long t0 = lo; t0 < hi; t0 += SPEC_TILE) {
    const int nt = (int)min((long long)SPEC_TILE, hi - t0);
    __syncthreads();
    for (int q = tid; q < nt * 8; q += nthr) s_sf[q / 8][q % 8] = sf[(t0 + q / 8) * 8 + q % 8];
    if (VISCOUS)
      for (int q = tid; q < nt * 10; q += nthr) s_pi[q / 10][q % 10] = pisf[(t0 + q / 10) * 10 + q % 10];
    __syncthreads();
    for (int e = tid; e < nt; e += nthr) {
      const real vx = s_sf[e][4], vy = s_sf[e][5], vh = s_sf[e][6];
      if (VISCOUS) {  // kernel_spec_csc.cl:55-57
        const real g = (real)1.0f / sqrt(cmax<real>((real)1.0E-15f, (real)(1.0f - vx * vx - vy * vy - vh * vh)));
        s_g[e][0] = (real)1.0f * g;
        s_g[e][1] = vx * g;
        s_g[e][2] = vy * g;
        s_g[e][3] = vh * g;
      } else {  // kernel_spec.cl:40
        s_g[e][0] = (real)(1.0 / sqrt(cmax<double>(1.0E-30, 1.0 - vx * vx - vy * vy - vh * vh)));
      }
      s_ch[e] = cosh(rapidity - s_sf[e][7]);
      s_sh[e] = sinh(rapidity - s_sf[e][7]);
    }
    __syncthreads();
    if (!active) continue;
    for (int e = 0; e < nt; e++) {
      const real mtcy = mt * s_ch[e], mtsy = mt * s_sh[e];
      const real* S = s_sf[e];
      if (!VISCOUS) {  // kernel_spec.cl:41-55
        const real gamma = s_g[e][0];
        const real efkt = (gamma * (mtcy - px * S[4] - py * S[5] - mtsy * S[6]) - muB) / tfrz;
        const real volum = mtcy * S[0] - px * S[1] - py * S[2] - mtsy * S[3];
        acc += (double)(dof * volum / (exp(efkt) + fb));
      } else {  // kernel_spec_csc.cl:58-78
        const real p0 = mtcy, p1 = -pt * cphi[m], p2 = -pt * sphi[m], p3 = -mtsy;
        const real pu = p0 * s_g[e][0] + p1 * s_g[e][1] + p2 * s_g[e][2] + p3 * s_g[e][3];
        double feq = 1.0 / ((double)exp((real)((pu - muB) / tfrz)) + (double)fb);
        const real* pm = s_pi[e];
        // the reference's contraction, with pi^{03} and pi^{13} where the
        // p_3 p_1 and p_3 p_2 terms take pi^{13} and pi^{23} (kept as written)
        const real p2pi = tcoeff * (p0 * p0 * pm[0] + p3 * p3 * pm[9] + 2.0f * p0 * (p1 * pm[1] + p2 * pm[2] + p3 * pm[3]) +
                                    (p1 * p1 * pm[4] + 2 * p1 * p2 * pm[5] + p2 * p2 * pm[7]) +
                                    2.0f * p3 * (p1 * pm[3] + p2 * pm[6]));
        const double df = feq * (1.0 - (double)fb * feq) * (double)p2pi;
        feq += fabs(df) > feq ? (df > 0 ? 1.0 : (df < 0 ? -1.0 : 0.0)) * feq * 0.999 : df;
        const real pdsig = p0 * S[0] + p1 * S[1] + p2 * S[2] + p3 * S[3];
        acc += (double)dof * (double)pdsig * feq;
      }
    }
  }
  if (active) part[((long long)c * ny + k) * (npt * nphi) + tid] = acc;
}

template <class real>
__global__ void spectra_finish_kernel(const double* part, int nchunk, long long npoint, real* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npoint) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; c++) s += part[(long long)c * npoint + i];
  out[i] = (real)s;
}

}  // namespace clv
