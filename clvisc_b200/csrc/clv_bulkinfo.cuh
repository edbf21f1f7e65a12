// Bulk-evolution diagnostics on the device (pyvisc/bulkinfo.py,
// pyvisc/bulkinfo_h5.py, kernel_bulkinfo.cl).
//
// bulk_slices_kernel restates bulkinfo.py's get_ed and get_pimn kernels
// (bulkinfo.py:62-117): the lines through the grid centre along x, y and
// eta_s, the planes k = NZ/2, j = NY/2 and i = NX/2 of (e, vx, vy, veta), and
// pi^{xx}, pi^{yy}, pi^{tx} "in the transverse plane" with get_pimn's own
// index oid = i*NY*(NZ/2) + j*(NZ/2) + NZ/2, which is not the cell
// (i, j, NZ/2) of the plane (for NZ = 1 it is cell 0 everywhere); the index
// is kept as the reference computes it.
//
// bulk_sums_kernel replaces the host sums the reference makes after copying
// the whole state to the host (bulkinfo.py:184-257): per eta_s slice the
// momentum-anisotropy sums of T^{xx}, T^{yy}, T^{tx} (ecc_vs_rapidity,
// bulkinfo.py:259-271), and in the plane k = NZ/2 the sums behind eccp, the
// viscous eccp, <v_r> and the mid-rapidity entropy (bulkinfo.py:184-257, with
// their floors e >= 1e-10 and v^2 <= 0.999999 and their vz = 0 in the plane).
// One block per slice reduces in a fixed order in double, so the results do
// not depend on scheduling. The equation of state is the run's table.
//
// bulk_lab_kernel is kernel_bulkinfo.cl:18-45 (total_energy_and_entropy)
// with the sums over all cells (bulkinfo_h5.py:264-277) done per block in a
// fixed order.
#pragma once
#include "clv_device.cuh"

namespace clv {

constexpr int BULK_SUM_THREADS = 256;
// per-slice sums: Txx, Tyy, T0x (with veta)
constexpr int BULK_NSLICE = 3;
// plane sums: Txx, Tyy, T0x (veta = 0), u0 e v_r, u0 e, u0 s, pi^xx + pi^yy, pi^xx - pi^yy
constexpr int BULK_NPLANE = 8;

template <class real>
__global__ void bulk_slices_kernel(Params p, const real* ev, real* x0, real* y0, real* z0, real* xy, real* xz,
                                   real* yz) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int NX = p.nx, NY = p.ny, NZ = p.nz;
  const long long ld = p.ld;
  auto cp = [&](real* dst, long long d, long long I) {
#pragma unroll
    for (int c = 0; c < 4; c++) dst[4 * d + c] = ev[c * ld + I];
  };
  if (gid < NX) {
    int j = NY / 2;
    int k = NZ / 2;
    cp(x0, gid, (long long)gid * NY * NZ + j * NZ + k);
    int i = gid;
    for (j = 0; j < NY; j++) cp(xy, (long long)i * NY + j, (long long)i * NY * NZ + (long long)j * NZ + k);
    j = NY / 2;
    for (k = 0; k < NZ; k++) cp(xz, (long long)i * NZ + k, (long long)i * NY * NZ + (long long)j * NZ + k);
  }
  if (gid < NY) {
    int i = NX / 2;
    int k = NZ / 2;
    cp(y0, gid, (long long)i * NY * NZ + (long long)gid * NZ + k);
    int j = gid;
    for (k = 0; k < NZ; k++) cp(yz, (long long)j * NZ + k, (long long)i * NY * NZ + (long long)j * NZ + k);
  }
  if (gid < NZ) {
    int i = NX / 2;
    int j = NY / 2;
    cp(z0, gid, (long long)i * NY * NZ + (long long)j * NZ + gid);
  }
}

// get_pimn, bulkinfo.py:103-117 (pi planes 4 = xx, 7 = yy, 1 = tx)
template <class real>
__global__ void bulk_pimn_kernel(Params p, const real* pi, real* pixx, real* piyy, real* pitx) {
  const int gx = blockIdx.y;
  const int gy = blockIdx.x * blockDim.x + threadIdx.x;
  if (gx >= p.nx || gy >= p.ny) return;
  const int NY = p.ny, NZ = p.nz;
  const long long oid = (long long)gx * NY * (NZ / 2) + (long long)gy * (NZ / 2) + NZ / 2;
  const long long nid = (long long)gx * NY + gy;
  pixx[nid] = pi[4 * p.ld + oid];
  piyy[nid] = pi[7 * p.ld + oid];
  pitx[nid] = pi[1 * p.ld + oid];
}

template <int N> __device__ void block_sum(double (&v)[N], double (*sh)[BULK_SUM_THREADS]) {
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < N; q++) sh[q][t] = v[q];
  __syncthreads();
  for (int s = BULK_SUM_THREADS / 2; s > 0; s >>= 1) {
    if (t < s)
#pragma unroll
      for (int q = 0; q < N; q++) sh[q][t] += sh[q][t + s];
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < N; q++) v[q] = sh[q][0];
}

// the reference's host floors: e >= 1e-10, v^2 > 1 -> 0.999999
__device__ __forceinline__ double floor_ed(double e) { return e < 1.0E-10 ? 1.0E-10 : e; }
__device__ __forceinline__ double u0_of(double vr2) { return 1.0 / sqrt(1.0 - (vr2 > 1.0 ? 0.999999 : vr2)); }

// blockIdx.x = k; out[3k .. 3k+2] per slice; the block of k = NZ/2 also
// writes out[3 NZ .. 3 NZ + 7] (pi terms only when pi != nullptr)
template <class real>
__global__ void __launch_bounds__(BULK_SUM_THREADS) bulk_sums_kernel(Params p, const real* ev, const real* pi,
                                                                      double* out) {
  __shared__ double sh[BULK_NSLICE + BULK_NPLANE][BULK_SUM_THREADS];
  const int k = blockIdx.x;
  const int NX = p.nx, NY = p.ny, NZ = p.nz;
  const long long ld = p.ld;
  const bool plane = (k == NZ / 2);
  double s[BULK_NSLICE + BULK_NPLANE];
#pragma unroll
  for (int q = 0; q < BULK_NSLICE + BULK_NPLANE; q++) s[q] = 0.0;
  for (int id = threadIdx.x; id < NX * NY; id += BULK_SUM_THREADS) {
    const long long I = (long long)id * NZ + k;
    const double ed = floor_ed((double)ev[I]);
    const double vx = ev[ld + I], vy = ev[2 * ld + I], vz = ev[3 * ld + I];
    const double pre = (double)eosP<real>(p, (real)ed);
    const double u0 = u0_of(vx * vx + vy * vy + vz * vz);
    s[0] += (ed + pre) * u0 * u0 * vx * vx + pre;
    s[1] += (ed + pre) * u0 * u0 * vy * vy + pre;
    s[2] += (ed + pre) * u0 * u0 * vx;
    if (plane) {
      const double w0 = u0_of(vx * vx + vy * vy);
      s[3] += (ed + pre) * w0 * w0 * vx * vx + pre;
      s[4] += (ed + pre) * w0 * w0 * vy * vy + pre;
      s[5] += (ed + pre) * w0 * w0 * vx;
      s[6] += w0 * ed * sqrt(vx * vx + vy * vy);
      s[7] += w0 * ed;
      s[8] += w0 * (double)eos_comp<real>(p, (real)ed, 3);
      if (pi) {
        const int i = id / NY, j = id % NY;
        const long long oid = (long long)i * NY * (NZ / 2) + (long long)j * (NZ / 2) + NZ / 2;
        const double xx = pi[4 * ld + oid], yy = pi[7 * ld + oid];
        s[9] += xx + yy;
        s[10] += xx - yy;
      }
    }
  }
  block_sum<BULK_NSLICE + BULK_NPLANE>(s, sh);
  if (threadIdx.x == 0) {
    for (int q = 0; q < BULK_NSLICE; q++) out[BULK_NSLICE * k + q] = s[q];
    if (plane)
      for (int q = 0; q < BULK_NPLANE; q++) out[BULK_NSLICE * NZ + q] = s[BULK_NSLICE + q];
  }
}

// kernel_bulkinfo.cl:18-45 summed: block b adds cells [b*chunk, (b+1)*chunk)
// into part[2b], part[2b+1] (lab-frame energy and entropy density)
template <class real>
__global__ void __launch_bounds__(BULK_SUM_THREADS) bulk_lab_kernel(Params p, const real* ev, real tau, long long chunk,
                                                                     double* part) {
  __shared__ double sh[2][BULK_SUM_THREADS];
  const long long N = (long long)p.nx * p.ny * p.nz;
  const long long lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  const long long ld = p.ld;
  double s[2] = {0.0, 0.0};
  for (long long I = lo + threadIdx.x; I < hi; I += BULK_SUM_THREADS) {
    const int K = (int)(I % p.nz);
    real ed = ev[I], vx = ev[ld + I], vy = ev[2 * ld + I], vz = ev[3 * ld + I];
    real pr = eosP<real>(p, ed);
    real u0 = gamma3<real>(vx, vy, vz);
    real etas = (K - p.nz / 2) * (real)p.DZ;
    real cosh_etas = cosh(etas);
    real ed_lab = (ed + pr) * u0 * u0 * (cosh_etas + vz * sinh(etas)) - pr * cosh_etas;
    real s_lab = u0 * eos_comp<real>(p, ed, 3);
    s[0] += (double)ed_lab;
    s[1] += (double)s_lab;
  }
  block_sum<2>(s, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s[0];
    part[2 * blockIdx.x + 1] = s[1];
  }
}

}  // namespace clv
