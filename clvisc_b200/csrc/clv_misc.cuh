// Point-wise kernels of the hydro step: Israel-Stewart initialisation,
// the u^mu difference, the maximum energy density and the AoS <-> SoA
// transposes used at the host boundary.
#pragma once
#include "clv_device.cuh"

namespace clv {

// kernel_IS.cl:10-36: Navier-Stokes Bjorken pi, udiff = 0, goodcell = 1
template <class real>
__global__ void visc_initialize_kernel(Params p, real* pi1, uint8_t* goodcell, real* udiff, const real* ev, real tau) {
  const long long N = (long long)p.nx * p.ny * p.nz;
  const long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= N) return;
  const long long ld = p.ld;
  real e = ev[I];
  real T = eos_comp<real>(p, e, 2);
  real s = eos_comp<real>(p, e, 3);
  real etav = etaos<real>(p, T) * s * CLV_HBARC;
  real tmp = 2.0f / 3.0f * etav / tau;
  pi1[pidx(1, 1) * ld + I] = tmp;
  pi1[pidx(2, 2) * ld + I] = tmp;
  pi1[pidx(3, 3) * ld + I] = -2.0f * tmp;
  if (p.flags & FLAG_BULK) {  // bulk sector: Navier-Stokes Pi of Bjorken flow, theta = 1/tau, regulated
    real zetav = zetaos<real>(p, T) * s * CLV_HBARC;
    real b0 = -zetav / tau;
    real pb = eos_comp<real>(p, e, 1);
    if (b0 < -pb) b0 = -pb;
    else if (b0 > pb) b0 = pb;
    if (T < p.ZETAOS_TMIN) b0 = 0.0f;
    pi1[10 * ld + I] = b0;
  }
#pragma unroll
  for (int c = 0; c < 4; c++) udiff[c * ld + I] = 0.0f;
  goodcell[I] = 1;
}

// kernel_IS.cl:714-724: udiff = u(ev1) - u(ev0)
template <class real> __global__ void get_udiff_kernel(Params p, real* udiff, const real* ev0, const real* ev1) {
  const long long N = (long long)p.nx * p.ny * p.nz;
  const long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= N) return;
  const long long ld = p.ld;
  real a1 = ev1[ld + I], a2 = ev1[2 * ld + I], a3 = ev1[3 * ld + I];
  real b1 = ev0[ld + I], b2 = ev0[2 * ld + I], b3 = ev0[3 * ld + I];
  real gn = gamma3<real>(a1, a2, a3);
  real go = gamma3<real>(b1, b2, b3);
  udiff[I] = gn * 1.0f - go * 1.0f;
  udiff[ld + I] = gn * a1 - go * b1;
  udiff[2 * ld + I] = gn * a2 - go * b2;
  udiff[3 * ld + I] = gn * a3 - go * b3;
}

// max over a plane of n values (NaN ignored), as an ordered key: warp
// shuffle, one atomic per warp
template <class real>
__global__ void max_key_kernel(const real* x, long long n, typename KeyT<real>::type* key) {
  typedef typename KeyT<real>::type K;
  K best = 0;
  for (long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x; I < n; I += (long long)gridDim.x * blockDim.x) {
    real v = x[I];
    if (v == v) {
      K kv = fkey(v);
      best = kv > best ? kv : best;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    K other = __shfl_xor_sync(0xffffffffu, best, o);
    best = other > best ? other : best;
  }
  if ((threadIdx.x & 31) == 0 && best) atomicMax(key, best);
}

// Health of a state (clv_status): counts of non-finite values over w planes of
// n cells, and of cells whose goodcell flag is 0 (the reference's bad-cell
// reset, kernel_IS.cl:697-708), added into out[0] and out[1]; block 0 also
// sets out[2] to the surface elements beyond the capacity (0 if none).
template <class real>
__global__ void status_kernel(const real* f, int w, long long ld, long long n, const uint8_t* goodcell,
                              const long long* sf_total, long long capacity, unsigned long long* out) {
  unsigned long long nonfinite = 0, bad = 0;
  for (long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x; I < n; I += (long long)gridDim.x * blockDim.x) {
    if (f)
      for (int c = 0; c < w; c++) nonfinite += isfinite(f[c * ld + I]) ? 0ull : 1ull;
    if (goodcell) bad += goodcell[I] == 0 ? 1ull : 0ull;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nonfinite += __shfl_xor_sync(0xffffffffu, nonfinite, o);
    bad += __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (nonfinite) atomicAdd(out, nonfinite);
    if (bad) atomicAdd(out + 1, bad);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && sf_total)
    out[2] = *sf_total > capacity ? (unsigned long long)(*sf_total - capacity) : 0ull;
}

// (n, w) row-major  <->  w planes of stride ld
template <class real>
__global__ void aos_to_soa_kernel(const real* aos, real* soa, long long n, int w, long long ld) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * w) return;
  long long I = t / w;
  int c = (int)(t % w);
  soa[c * ld + I] = aos[t];
}
template <class real>
__global__ void soa_to_aos_kernel(const real* soa, real* aos, long long n, int w, long long ld) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * w) return;
  long long I = t / w;
  int c = (int)(t % w);
  aos[t] = soa[c * ld + I];
}

}  // namespace clv
