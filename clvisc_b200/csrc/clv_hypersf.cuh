// Freeze-out hypersurface finder (kernel_hypersf.cl:98-660) with
// deterministic output order.
//
// The reference appends surface elements with atomic_inc, so their order
// changes from run to run. Here a first pass marks the coarse cubes that emit
// an element, a block scan turns the marks into offsets, and the element pass
// writes cube q's element at (elements already in the buffer) + (number of
// emitting cubes before q in (i, j, k) order). The element count and the
// per-element arithmetic are those of the reference kernel.
#pragma once
#include "clv_device.cuh"

namespace clv {

template <class real> struct R4 { real x, y, z, w; };  // (tau, x, y, eta) / dSigma components
template <class real> __device__ __forceinline__ R4<real> add4(R4<real> a, R4<real> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class real> __device__ __forceinline__ R4<real> sub4(R4<real> a, R4<real> b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
template <class real> __device__ __forceinline__ R4<real> scl4(real s, R4<real> a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
template <class real> __device__ __forceinline__ R4<real> mul4s(R4<real> a, real s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class real> __device__ __forceinline__ R4<real> div4(R4<real> a, real s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
template <class real> __device__ __forceinline__ real dotr4(R4<real> a, R4<real> b) {
  real r = a.x * b.x;
  r = r + a.y * b.y;
  r = r + a.z * b.z;
  r = r + a.w * b.w;
  return r;
}
// corner n of the unit 4-cube: (tau, x, y, eta) bits (3, 0, 1, 2) (kernel_hypersf.cl:33-54)
template <class real> __device__ __forceinline__ R4<real> cube_corner(int n) {
  return R4<real>{(real)((n >> 3) & 1), (real)(n & 1), (real)((n >> 1) & 1), (real)((n >> 2) & 1)};
}

template <class real> struct SurfPiece {
  int id[4];
  R4<real> center, norm;
};

// kernel_hypersf.cl:98-122
template <class real>
__device__ SurfPiece<real> construct_hypersf(int id0, int id1, int id2, int id3, const R4<real>* ints, R4<real> mc) {
  SurfPiece<real> s;
  s.id[0] = id0; s.id[1] = id1; s.id[2] = id2; s.id[3] = id3;
  s.center = scl4<real>(0.25f, add4(add4(add4(ints[id0], ints[id1]), ints[id2]), ints[id3]));
  R4<real> vo = sub4(s.center, mc);
  R4<real> a = sub4(ints[id1], ints[id0]);
  R4<real> b = sub4(ints[id2], ints[id0]);
  R4<real> c = sub4(ints[id3], ints[id0]);
  R4<real> n;
  n.x = a.y * (b.z * c.w - b.w * c.z) + a.z * (b.w * c.y - b.y * c.w) + a.w * (b.y * c.z - b.z * c.y);
  n.y = -(a.x * (b.z * c.w - b.w * c.z) + a.z * (b.w * c.x - b.x * c.w) + a.w * (b.x * c.z - b.z * c.x));
  n.z = a.x * (b.y * c.w - b.w * c.y) + a.y * (b.w * c.x - b.x * c.w) + a.w * (b.x * c.y - b.y * c.x);
  n.w = -(a.x * (b.y * c.z - b.z * c.y) + a.y * (b.z * c.x - b.x * c.z) + a.z * (b.x * c.y - b.y * c.x));
  real projection = dotr4(vo, n);
  if (projection < 0) n = R4<real>{-n.x, -n.y, -n.z, -n.w};
  s.norm = n;
  return s;
}

// kernel_hypersf.cl:126-132 (the 32-bit product wraps as on any GPU)
template <class real> __device__ __forceinline__ real sf_rand(int* seed) {
  const int a = 16807;
  const int m = 2147483647;
  int prod = (int)((unsigned int)(*seed) * (unsigned int)a);
  *seed = (int)(((long long)prod) % m);
  return (*seed) / ((real)m);
}

template <class real> __device__ R4<real> mass_center(const R4<real>* ints, int n) {  // :226-232
  R4<real> c{0.0f, 0.0f, 0.0f, 0.0f};
  for (int i = 0; i < n; i++) c = add4(c, ints[i]);
  return div4(c, (real)n);
}

// :135-159. The reference builds the piece (i, j, k, l) inside the m loop;
// it depends only on the intersections and their centre, which change only
// at a hit, after which the m loop ends, so it is built once per (i, j, k, l)
// here: the same values, n - l - 1 times fewer constructions.
template <class real> __device__ void tiny_move_if_coplanar(R4<real>* ints, int n, R4<real>* mc, int gid) {
  int seed = (int)(32117u * (unsigned int)(gid + 1));
  for (int i = 0; i < n - 4; i++)
    for (int j = i + 1; j < n - 3; j++)
      for (int k = j + 1; k < n - 2; k++)
        for (int l = k + 1; l < n - 1; l++) {
          const SurfPiece<real> sf = construct_hypersf(i, j, k, l, ints, *mc);
          for (int m = l + 1; m < n; m++) {
            if (dotr4(sf.norm, sub4(ints[m], sf.center)) == 0.0f) {
              for (int q = 0; q < n; q++) {
                real r0 = sf_rand<real>(&seed), r1 = sf_rand<real>(&seed), r2 = sf_rand<real>(&seed),
                     r3 = sf_rand<real>(&seed);
                R4<real> sh{(r0 - 0.5f) * 1.0E-7f, (r1 - 0.5f) * 1.0E-7f, (r2 - 0.5f) * 1.0E-7f, (r3 - 0.5f) * 1.0E-7f};
                ints[q] = add4(ints[q], sh);
              }
              *mc = mass_center(ints, n);
              break;
            }
          }
        }
}

template <class real> __device__ bool on_convex_hull(const SurfPiece<real>& sf, const R4<real>* ints, int n) {  // :163-176
  for (int q = 0; q < n; q++) {
    if (q != sf.id[0] && q != sf.id[1] && q != sf.id[2] && q != sf.id[3]) {
      if (dotr4(sub4(ints[q], sf.center), sf.norm) >= 0.0f) return false;
    }
  }
  return true;
}

// :195-223 with contribution_from (:180-192)
template <class real> __device__ R4<real> energy_flow(const real ed[16], real efrz) {
  R4<real> vl{0.0f, 0.0f, 0.0f, 0.0f}, vh{0.0f, 0.0f, 0.0f, 0.0f};
  real elsum = 0.0f, ehsum = 0.0f;
#pragma unroll
  for (int n = 0; n < 2; n++)
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++)
#pragma unroll
        for (int k = 0; k < 2; k++) {
          int id = 8 * n + 4 * k + 2 * j + i;
          real dek = efrz - ed[id];
          real adek = fabs(dek);
          R4<real> w = mul4s(R4<real>{(real)n, (real)i, (real)j, (real)k}, adek);
          if (dek > 0.0f) {
            elsum += adek;
            vl = add4(vl, w);
          } else {
            ehsum += adek;
            vh = add4(vh, w);
          }
        }
  if (fabs(elsum) > Acu<real>::v) vl = div4(vl, elsum);
  if (fabs(ehsum) > Acu<real>::v) vh = div4(vh, ehsum);
  return sub4(vl, vh);
}

// :237-266
template <class real> __device__ R4<real> calc_area(R4<real>* ints, R4<real> flow, int n, int gid) {
  R4<real> mc = mass_center(ints, n);
  R4<real> area{0.0f, 0.0f, 0.0f, 0.0f};
  if (n == 4) {
    SurfPiece<real> sf = construct_hypersf(0, 1, 2, 3, ints, mc);
    if (dotr4(flow, sf.norm) < 0.0f) sf.norm = R4<real>{-sf.norm.x, -sf.norm.y, -sf.norm.z, -sf.norm.w};
    area = sf.norm;
  } else if (n > 4) {
    tiny_move_if_coplanar(ints, n, &mc, gid);
    for (int i = 0; i < n - 3; i++)
      for (int j = i + 1; j < n - 2; j++)
        for (int k = j + 1; k < n - 1; k++)
          for (int l = k + 1; l < n; l++) {
            SurfPiece<real> sf = construct_hypersf(i, j, k, l, ints, mc);
            // both tests are pure: the cheap one first (the reference
            // evaluates the hull test first; the sum is the same)
            if (dotr4(sf.norm, flow) > 0.0f && on_convex_hull(sf, ints, n)) area = add4(area, sf.norm);
          }
  }
  return div4(area, (real)6.0f);
}

// :269-314
template <class real>
__device__ __forceinline__ void ints_between(real el, real er, int cl, int cr, real efrz, R4<real>* all, int* n) {
  real dE1 = efrz - el;
  real dE2 = efrz - er;
  real dE12 = el - er;
  if (dE1 * dE2 < 0) {
    real ratio = fabs(dE1) / fabs(dE12);
    all[*n] = add4(scl4<real>(ratio, cube_corner<real>(cr)), scl4<real>((real)(1 - ratio), cube_corner<real>(cl)));
    *n += 1;
  }
}
template <class real> __device__ void all_intersections(const real ed[16], real efrz, R4<real>* all, int* n) {
  *n = 0;
  for (int s = 0; s < 16; s += 4) {
    ints_between(ed[s + 0], ed[s + 1], s + 0, s + 1, efrz, all, n);
    ints_between(ed[s + 0], ed[s + 2], s + 0, s + 2, efrz, all, n);
    ints_between(ed[s + 2], ed[s + 3], s + 2, s + 3, efrz, all, n);
    ints_between(ed[s + 1], ed[s + 3], s + 1, s + 3, efrz, all, n);
  }
  for (int s = 0; s < 16; s += 8) {
    ints_between(ed[s + 0], ed[s + 4], s + 0, s + 4, efrz, all, n);
    ints_between(ed[s + 1], ed[s + 5], s + 1, s + 5, efrz, all, n);
    ints_between(ed[s + 2], ed[s + 6], s + 2, s + 6, efrz, all, n);
    ints_between(ed[s + 3], ed[s + 7], s + 3, s + 7, efrz, all, n);
  }
  for (int s = 0; s < 8; s++) ints_between(ed[s + 0], ed[s + 8], s + 0, s + 8, efrz, all, n);
}

struct CubeGrid {
  int nx, ny, nz;  // coarse cube counts per axis
};
__host__ __device__ inline CubeGrid cube_grid(const Params& p) {
  return CubeGrid{(p.nx - 1) / p.nxskip + 1, (p.ny - 1) / p.nyskip + 1, (p.nz - 1) / p.nzskip + 1};
}
__device__ __forceinline__ long long corner_cell(const Params& p, int i, int j, int k, int q) {
  int ii = (i + (q & 1)) * p.nxskip, jj = (j + ((q >> 1) & 1)) * p.nyskip, kk = (k + ((q >> 2) & 1)) * p.nzskip;
  return ((long long)ii * p.ny + jj) * p.nz + kk;
}
// centroid weight of corner q (kernel_hypersf.cl:329-348)
template <class real> __device__ __forceinline__ real corner_weight(R4<real> mc, int q) {
  real a = (q & 8) ? mc.x : (real)(1.0f - mc.x);
  real b = (q & 1) ? mc.y : (real)(1.0f - mc.y);
  real c = (q & 2) ? mc.z : (real)(1.0f - mc.z);
  real d = (q & 4) ? mc.w : (real)(1.0f - mc.w);
  return a * b * c * d;
}

// energy densities of the 16 corners; false when the cube is outside the
// grid (kernel_hypersf.cl:536)
template <class real>
__device__ __forceinline__ bool load_cube(const Params& p, const real* ev_old, const real* ev_new, int i, int j, int k,
                                          real ed[16]) {
  if (!((i + 1) * p.nxskip < p.nx && (j + 1) * p.nyskip < p.ny && (k + 1) * p.nzskip < p.nz)) return false;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    long long c = corner_cell(p, i, j, k, q);
    ed[q] = ev_old[c];
    ed[8 + q] = ev_new[c];
  }
  return true;
}
template <class real> __device__ __forceinline__ bool crosses(const real ed[16], real efrz) {  // :562-571
  return !((ed[0] - efrz) * (ed[15] - efrz) > 0 && (ed[1] - efrz) * (ed[14] - efrz) > 0 &&
           (ed[2] - efrz) * (ed[13] - efrz) > 0 && (ed[3] - efrz) * (ed[12] - efrz) > 0 &&
           (ed[4] - efrz) * (ed[11] - efrz) > 0 && (ed[5] - efrz) * (ed[10] - efrz) > 0 &&
           (ed[6] - efrz) * (ed[9] - efrz) > 0 && (ed[7] - efrz) * (ed[8] - efrz) > 0);
}

// pass 1: does cube q emit an element?  (visc: mass centre not NaN, :604)
template <class real>
__global__ void hsf_mark_kernel(Params p, const real* ev_old, const real* ev_new, int visc, uint8_t* mark,
                                int* block_count) {
  const CubeGrid g = cube_grid(p);
  const long long nc = (long long)g.nx * g.ny * g.nz;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int emit = 0;
  if (q < nc) {
    int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.ny * g.nz));
    real ed[16];
    const real efrz = p.EFRZ;
    if (load_cube(p, ev_old, ev_new, i, j, k, ed) && crosses(ed, efrz)) {
      emit = 1;
      if (visc) {
        R4<real> all[32];
        int n;
        all_intersections(ed, efrz, all, &n);
        R4<real> mc = mass_center(all, n);
        if (isnan(mc.x)) emit = 0;
      }
    }
    mark[q] = (uint8_t)emit;
  }
  int c = __syncthreads_count(emit);
  if (threadIdx.x == 0) block_count[blockIdx.x] = c;
}

#ifndef CLV_HSF_NO_SHARED_KERNELS
// pass 2: exclusive scan of the block counts in one block; total -> *total
__global__ void hsf_scan_kernel(int* block_count, int nblocks, long long* total) {
  __shared__ long long warp_sum[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nblocks; base += blockDim.x) {
    int t = base + threadIdx.x;
    long long v = t < nblocks ? block_count[t] : 0;
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
      long long s = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      warp_sum[lane] = s;
    }
    __syncthreads();
    long long excl = carry + (w > 0 ? warp_sum[w - 1] : 0) + x - v;
    if (t < nblocks) block_count[t] = (int)excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// pass 3: cube list in order
__global__ void hsf_compact_kernel(long long ncube, const uint8_t* mark, const int* block_offset, int* list) {
  __shared__ int warp_tot[32];
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int m = (q < ncube) ? mark[q] : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned int bal = __ballot_sync(0xffffffffu, m);
  int before = __popc(bal & ((1u << lane) - 1u));
  if (lane == 0) warp_tot[w] = __popc(bal);
  __syncthreads();
  int wbase = 0;
  for (int u = 0; u < w; u++) wbase += warp_tot[u];
  if (m) list[block_offset[blockIdx.x] + wbase + before] = (int)q;
}

#endif  // CLV_HSF_NO_SHARED_KERNELS

// pass 4: one thread per emitted element
template <class real>
__global__ void hsf_element_kernel(Params p, const real* ev_old, const real* ev_new, const real* pi_old,
                                   const real* pi_new, real time_old, real time_new, int visc, const int* list,
                                   const long long* count, long long* total_inout, real* sf, real* txyz,
                                   real* pisf, long long capacity) {
  const long long n_here = *count;
  const long long base = *total_inout;
  const CubeGrid g = cube_grid(p);
  const long long ld = p.ld;
  const real efrz = p.EFRZ;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n_here;
       e += (long long)gridDim.x * blockDim.x) {
    const long long q = list[e];
    int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.ny * g.nz));
    real ed[16];
    load_cube(p, ev_old, ev_new, i, j, k, ed);
    R4<real> all[32];
    int n;
    all_intersections(ed, efrz, all, &n);
    R4<real> flow = energy_flow(ed, efrz);
    R4<real> mc = mass_center(all, n);
    R4<real> dS = calc_area(all, flow, n, i * j * k);
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
        real t = corner_weight(mc, qq) * src[c * ld + corner_cell(p, i, j, k, qq & 7)];
        acc = (qq == 0) ? t : acc + t;
      }
      v[c] = acc;
    }
    const long long o = base + e;
    if (o < capacity) {
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
            real t = corner_weight(mc, qq) * src[mn * ld + corner_cell(p, i, j, k, qq & 7)];
            acc = (qq == 0) ? t : acc + t;
          }
          pisf[10 * o + mn] = acc;
        }
      }
    }
  }
}

#ifndef CLV_HSF_NO_SHARED_KERNELS
__global__ void hsf_advance_kernel(const long long* count, long long* total_inout) { *total_inout += *count; }
#endif

}  // namespace clv
