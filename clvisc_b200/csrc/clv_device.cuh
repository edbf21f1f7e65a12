// Device-side building blocks of the CLVisc hydro step for sm_100a.
//
// Every floating-point expression keeps the operand order and the
// float-literal constants of the reference OpenCL kernels
// (pyvisc/kernel/helper.h, eos_table.h, kernel_*.cl), and the library is
// compiled with --fmad=false and IEEE division/square root, so each cell's
// result is bit-identical to a straightforward evaluation of the reference
// source in the same precision.
//
// Compiled with CLV_FAST=1 (the tolerance build, clv_fast.cu: FMA
// contraction, approximate division and square root) the same headers give the
// fast arithmetic: division by run constants through their reciprocals (the
// EOS lookup included: the reference's row and column arithmetic, with its
// float-rounded row width, is kept), the limiters in sign-test form and
// the KT speed max(lambda, 1) taken as 1 (lambda <= 1 for |v| < 1 and
// c_s^2 <= 1). Functions and kernels live in an inline namespace named after
// the arithmetic (clv::exact or clv::fast), so both builds link into one
// library; plain structs are shared.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef CLV_FAST
#define CLV_FAST 0
#endif
#if CLV_FAST
#define CLV_ARITH fast
#else
#define CLV_ARITH exact
#endif

namespace clv {

// correctly rounded reciprocals of run constants in one precision
template <class real> struct Recips {
  real eos_step, eos_epr;  // EOS grid step and energy density per image row
  real DT, DX, DY, DZ;     // DT, DX, DY, DZ as reals
  real three;              // 3
};

// run constants, passed by value to every kernel
struct Params {
  int nx, ny, nz;
  long long ld;  // plane stride of every SoA field, in elements
  float DT, DX, DY, DZ, TAU0;
  float ETAOS_XMIN, ETAOS_YMIN, ETAOS_LEFT_SLOP, ETAOS_RIGHT_SLOP, LAM1;
  float EFRZ;
  int nxskip, nyskip, nzskip;
  float eos_start, eos_step;
  int eos_num, eos_nrow, eos_ncol;
  const float* eos;  // nrow*ncol texels of (cs2, p, T, s)
  const float2* eos_p2;  // optional: pairs (p[t], p[t+1]) of the pressure column (tolerance build)
  int flags;
  // bulk sector (FLAG_BULK): zeta/s(T) peak, position, width, skewness
  float ZETAOS_MAX, ZETAOS_T0, ZETAOS_WIDTH, ZETAOS_SKEW;
  float ZETAOS_TMIN;  // Pi = 0 in cells colder than this
  Recips<float> rf;   // reciprocals for float kernels
  Recips<double> rd;  // reciprocals for double kernels
  int opt[4];         // the run's own stage_kernel+1, chunk, tiled blocks, tile+1 (0: process-wide)
};
inline namespace CLV_ARITH {
template <class real> __device__ __forceinline__ const Recips<real>& recips(const Params& p);
template <> __device__ __forceinline__ const Recips<float>& recips<float>(const Params& p) { return p.rf; }
template <> __device__ __forceinline__ const Recips<double>& recips<double>(const Params& p) { return p.rd; }
}  // namespace CLV_ARITH

// tau-dependent divisors of one stage launch and their reciprocals
template <class real> struct TauConst {
  real tau, rtau;  // tau, 1/tau
  real dzt, rdzt;  // DZ*tau, 1/(DZ*tau)
};

enum : int {
  FLAG_RIEMANN = 1,
  FLAG_GUBSER_VISC = 2,
  FLAG_PIMN_OMEGA = 4,
  FLAG_OMEGA_OMEGA = 8,
  FLAG_BULK = 16,
  FLAG_FAST = 32,
};

// launch choices of the viscous stage (clv_set_option, or a run's own)
struct StageOpts {
  int stage_kernel;  // 0 automatic, 1 per-cell, 2 tiled (3+1)D, 3 tiled (2+1)D
  int chunk;         // x planes per tiled (3+1)D CTA
  int minb;          // resident tiled CTAs per SM (FP32)
  int tile;          // 0 = 8 x 32, 1 = 16 x 16, 2 = 8 x 16 (y, eta)
  int rows2d;        // threads of a tiled (2+1)D block (64 or 128)
  int chunk2d;       // x planes per tiled (2+1)D block
};

template <class real> struct Acu;
template <> struct Acu<float> { static constexpr float v = 1.0E-7f; };
template <> struct Acu<double> { static constexpr double v = 1.0E-14; };

#define CLV_THETA 1.1f
#define CLV_HBARC 0.19733f

template <class real> struct DivRange;
template <> struct DivRange<float> {
  static constexpr float lo = 0x1p-80f, hi = 0x1p+80f;
};
template <> struct DivRange<double> {
  static constexpr double lo = 0x1p-900, hi = 0x1p+900;
};
// the two texels (as texel indices) and the interpolation weight at eps
template <class real> struct EosSpot {
  long long t0, t1;
  real r;
};
template <class real> struct KeyT;
template <> struct KeyT<float> { typedef unsigned int type; };
template <> struct KeyT<double> { typedef unsigned long long type; };

inline namespace CLV_ARITH {

// OpenCL min/max/sign semantics (helper.h uses the builtins)
template <class real> __device__ __forceinline__ real cmin(real x, real y) { return (y < x) ? y : x; }
template <class real> __device__ __forceinline__ real cmax(real x, real y) { return (x < y) ? y : x; }
template <class real> __device__ __forceinline__ real csign(real x) {
  return x > (real)0 ? (real)1 : (x < (real)0 ? (real)-1 : (x != x ? (real)0 : x));
}

// ------------------------------------------------------- exact division
// a/b rounded to nearest (the IEEE quotient) from y = RN(1/b), by Markstein's
// method (P. Markstein, IBM J. Res. Dev. 34 (1990) 111): q = RN(a*y) is within
// a few ulps of a/b, r = a - b*q is formed exactly with a fused multiply-add,
// and q + r*y rounded once corrects q; applied twice, the second correction
// starts from a faithful quotient, for which the theorem gives the correctly
// rounded a/b when nothing under- or overflows. Outside the range where that
// holds (|a| below 2^-80 / 2^-900 or above 2^80 / 2^900, infinities, NaN) the
// IEEE division is used; a = 0 gives a*y, the correctly signed zero. Only used
// with divisors and reciprocals that are normal numbers well inside the range.
static __device__ __noinline__ float ieee_div(float a, float b) { return a / b; }
static __device__ __noinline__ double ieee_div(double a, double b) { return a / b; }
template <class real> __device__ __forceinline__ real div_by(real a, real b, real y) {
#if CLV_FAST
  (void)b;
  return a * y;  // tolerance build: the reciprocal's product
#endif
  real q0 = a * y;
  real r = fma(-q0, b, a);
  real q = fma(r, y, q0);
  r = fma(-q, b, a);
  q = fma(r, y, q);
  real aa = fabs(a);
  if (!(aa >= DivRange<real>::lo && aa <= DivRange<real>::hi)) q = (a == (real)0) ? q0 : ieee_div(a, b);
  return q;
}

// x / step for the Runge-Kutta stage index step (1 or 2): dividing by 1 or 2
// is exact, as is multiplying by 1 or 0.5, so this equals the division bit for
// bit (subnormal results included)
template <class real> __device__ __forceinline__ real div_step(real x, int step) {
  return step == 2 ? x * (real)0.5f : x;
}

// ------------------------------------------------------------------ EOS
// Table lookup of eos_table.h:39-62: row/col from the energy density, two
// nearest texels (the second wraps to the next row), clamp-to-edge, lerp.
// CLV_EOS_INLINE (default 1): inline the lookup at every call site, or keep
// one out-of-line copy per precision to shrink the kernels' code
#ifndef CLV_EOS_INLINE
#define CLV_EOS_INLINE 1
#endif
#if CLV_EOS_INLINE
#define CLV_EOS_ATTR __forceinline__
#else
#define CLV_EOS_ATTR __noinline__
#endif
template <class real> __device__ __forceinline__ EosSpot<real> eos_spot(const Params& p, real eps) {
  const Recips<real>& rc = recips<real>(p);
  real ed_per_row = p.eos_step * p.eos_ncol;
  int row = (int)div_by<real>(eps, ed_per_row, rc.eos_epr);
  int col = (int)div_by<real>(eps - p.eos_start - row * ed_per_row, (real)p.eos_step, rc.eos_step);
  real eps_low = p.eos_start + row * ed_per_row + col * p.eos_step;
  int col2 = col + 1, row2 = row;
  if (col2 == p.eos_ncol) {
    row2 += 1;
    col2 = 0;
  }
  int c0 = min(max(col, 0), p.eos_ncol - 1), r0 = min(max(row, 0), p.eos_nrow - 1);
  int c1 = min(max(col2, 0), p.eos_ncol - 1), r1 = min(max(row2, 0), p.eos_nrow - 1);
  EosSpot<real> s;
  s.t0 = (long long)r0 * p.eos_ncol + c0;
  s.t1 = (long long)r1 * p.eos_ncol + c1;
  s.r = div_by<real>(eps - eps_low, (real)p.eos_step, rc.eos_step);
  return s;
}
template <class real> __device__ __forceinline__ real eos_lerp(real r, float lo, float hi) {
  return (real)(1.0f - r) * (real)lo + r * (real)hi;
}
template <class real>
__device__ CLV_EOS_ATTR real eos_comp(const Params& p, real eps, int c) {
  const EosSpot<real> s = eos_spot<real>(p, eps);
#if CLV_FAST
  // tolerance build: the pressure from one 8-byte read of the pair table
  // when the two texels are neighbours (everywhere inside the table)
  if (c == 1 && p.eos_p2 && s.t1 == s.t0 + 1) {
    const float2 q = __ldg(p.eos_p2 + s.t0);
    return eos_lerp<real>(s.r, q.x, q.y);
  }
#endif
  float lo = __ldg(p.eos + 4 * s.t0 + c);
  float hi = __ldg(p.eos + 4 * s.t1 + c);
  return eos_lerp<real>(s.r, lo, hi);
}
// the four components (cs2, p, T, s) of the table at eps from one pair of
// 16-byte texel reads; component c equals eos_comp(p, eps, c) bit for bit
// (the table is 16-byte aligned: the library checks it)
template <class real> __device__ __forceinline__ void eos_texel4(const Params& p, real eps, real out[4]) {
  const EosSpot<real> s = eos_spot<real>(p, eps);
  const float4 lo = __ldg(reinterpret_cast<const float4*>(p.eos) + s.t0);
  const float4 hi = __ldg(reinterpret_cast<const float4*>(p.eos) + s.t1);
  out[0] = eos_lerp<real>(s.r, lo.x, hi.x);
  out[1] = eos_lerp<real>(s.r, lo.y, hi.y);
  out[2] = eos_lerp<real>(s.r, lo.z, hi.z);
  out[3] = eos_lerp<real>(s.r, lo.w, hi.w);
}
template <class real> __device__ __forceinline__ bool eos_in_table(const Params& p, real eps) {
  return eps < p.eos_start + p.eos_num * p.eos_step;
}
// P(e): eos_table.h:65-71
template <class real> __device__ __forceinline__ real eosP(const Params& p, real eps) {
  if (eos_in_table(p, eps)) return eos_comp(p, eps, 1);
  return 0.3327f * eps - 0.3223f * pow(eps, (real)0.4585f) - 0.003906f * eps * exp(-0.05697f * eps);
}
// CS2(e): eos_table.h:94-100
template <class real> __device__ __forceinline__ real eosCS2(const Params& p, real eps) {
  if (eos_in_table(p, eps)) return eos_comp(p, eps, 0);
  return 0.333333333f;
}

// ---------------------------------------------------------------- helper.h
template <class real> __device__ __forceinline__ real gamma3(real vx, real vy, real vz) {  // helper.h:46-48
#if CLV_FAST
  return rsqrt(cmax<real>(1.0f - vx * vx - vy * vy - vz * vz, Acu<real>::v));
#else
  return 1.0f / sqrt(cmax<real>(1.0f - vx * vx - vy * vy - vz * vz, Acu<real>::v));
#endif
}
template <class real> __device__ __forceinline__ real minmod(real x, real y) {  // helper.h:74-77
  real res = cmin<real>(fabs(x), fabs(y));
  return res * (csign(x) + csign(y)) * 0.5f;
}
#if CLV_FAST
// tolerance build: the generalised minmod of the two one-sided differences
// a = R - C, b = C - L: zero unless they have the same sign, else that sign
// times min(TH |a|, TH |b|, |a + b| / 2) -- the value of the nested minmods
// below, in a few instructions
template <class real> __device__ __forceinline__ real gminmod(real a, real b) {
  const real TH = CLV_THETA;
  const real m = fmin(TH * fmin(fabs(a), fabs(b)), (real)0.5f * fabs(a + b));
  return (a * b > (real)0) ? copysign(m, a) : (real)0;
}
template <class real> __device__ __forceinline__ real slope(real L, real C, real R) { return gminmod<real>(R - C, C - L); }
template <class real> __device__ __forceinline__ real grad_limit(real L, real C, real R) {
  return gminmod<real>(R - C, C - L);
}
#else
// slope limiter of kt1d (helper.h:213-217): minmod(0.5(R-L), minmod(TH(R-C), TH(C-L)))
template <class real> __device__ __forceinline__ real slope(real L, real C, real R) {
  const real TH = CLV_THETA;
  return minmod<real>(0.5f * (R - L), minmod<real>(TH * (R - C), TH * (C - L)));
}
// velocity-gradient limiter of kernel_IS.cl:134-137 (argument order differs)
template <class real> __device__ __forceinline__ real grad_limit(real L, real C, real R) {
  const real TH = CLV_THETA;
  return minmod<real>(0.5f * (R - L), minmod<real>(TH * (C - L), TH * (R - C)));
}
#endif

// helper.h:94-105, with edv = 0.5*(ev_L + ev_R)
template <class real>
__device__ __forceinline__ real max_speed(const Params& p, real e, real vx, real vy, real vz, real vk) {
#if CLV_FAST
  // tolerance build: lambda, the larger characteristic speed of flow plus
  // sound, is below 1 for |v| < 1 and c_s^2 <= 1, so max(lambda, 1) is 1
  (void)p; (void)e; (void)vx; (void)vy; (void)vz; (void)vk;
  return (real)1.0f;
#endif
  real ut = gamma3<real>(vx, vy, vz);
  real uk = ut * vk;
  real ut2 = ut * ut;
  real uk2 = uk * uk;
  real cs2 = eosCS2<real>(p, e);
  real lam = (fabs(ut * uk * (1.0f - cs2)) + sqrt((ut2 - uk2 - (ut2 - uk2 - 1.0f) * cs2) * cs2)) /
             (ut2 - (ut2 - 1.0f) * cs2);
  return cmax<real>(lam, 1.0f);
}

// helper.h:128-167; returns the energy density. With BULK the pressure is
// P(e) + bulk, the bulk viscous pressure of the cell.
template <class real, bool BULK = false>
__device__ __forceinline__ real root_newton(const Params& p, real T00, real M, real bulk = (real)0.0f,
                                            real v_start = (real)-1.0f) {
  real vl = 0.0f;
  real vh = 1.0f;
  real dpe = 1.0f / 3.0f;
  // the reference starts at the middle of the bracket; a start in [0, 1)
  // (the tolerance build passes the cell's speed at the start of the step)
  // leaves the bracket and the safeguards as they are
  real v = v_start >= (real)0.0f ? v_start : 0.5f * (vl + vh);
  real ed = T00 - M * v;
  real pr = eosP<real>(p, ed);
  if (BULK) pr = pr + bulk;
  real f = (T00 + pr) * v - M;
  real df = (T00 + pr) - M * v * dpe;
  real dvold = vh - vl;
  real dv = dvold;
  int i = 0;
  while (true) {
    if ((f + df * (vh - v)) * (f + df * (vl - v)) > 0.0f || fabs(2.f * f) > fabs(dvold * df)) {
      dvold = dv;
      dv = 0.5f * (vh - vl);
      v = vl + dv;
    } else {
      dvold = dv;
      dv = f / df;
      v -= dv;
    }
    i++;
    if (fabs(dv) < 0.00001f || i > 100) break;
    ed = T00 - M * v;
    pr = eosP<real>(p, ed);
    if (BULK) pr = pr + bulk;
    f = (T00 + pr) * v - M;
    df = (T00 + pr) - M * v * dpe;
    if (f > 0.0f) {
      vh = v;
    } else {
      vl = v;
    }
  }
  return T00 - M * v;
}

// Bulk sector (no counterpart in the reference): zeta/s(T) as a skewed Cauchy
// peak, ZETAOS_MAX w^2 / (w^2 + (T - T0)^2), w = WIDTH (1 + SKEW sign(T - T0))
// (the JETSCAPE parametrisation, Everett et al., PRC 103, 054904 (2021)).
template <class real> __device__ __forceinline__ real zetaos(const Params& p, real T) {
  real dT = T - p.ZETAOS_T0;
  real w = p.ZETAOS_WIDTH * (1.0f + p.ZETAOS_SKEW * csign<real>(dT));
  return p.ZETAOS_MAX * (w * w) / (w * w + dT * dT);
}

// helper.h:23-26
template <class real> __device__ __forceinline__ real etaos(const Params& p, real T) {
  return (T < p.ETAOS_XMIN) ? (p.ETAOS_LEFT_SLOP * (T - p.ETAOS_XMIN) + p.ETAOS_YMIN)
                            : (p.ETAOS_RIGHT_SLOP * (T - p.ETAOS_XMIN) + p.ETAOS_YMIN);
}

// kernel_IS.cl:3-6 and helper.h:59-63 as scalar lookups
template <class real> __device__ __forceinline__ real gmn(int a, int b) {
  return a != b ? (real)0.0f : (a == 0 ? (real)1.0f : (real)-1.0f);
}
__host__ __device__ constexpr int pidx(int i, int j) {  // helper.h:31
  return (i < j) ? ((7 * i + 2 * j - i * i) / 2) : ((7 * j + 2 * i - j * j) / 2);
}

// OpenCL dot(): left to right, separate multiply and add
template <class real> __device__ __forceinline__ real dot4(const real a[4], const real b[4]) {
  real r = a[0] * b[0];
  r = r + a[1] * b[1];
  r = r + a[2] * b[2];
  r = r + a[3] * b[3];
  return r;
}

// Delta^{k c} = g^{k c} - u^k u^c (kernel_IS.cl:333-334)
template <class real> __device__ __forceinline__ void delta4(const real u[4], real D[4][4]) {
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int c = 0; c < 4; c++) D[k][c] = gmn<real>(k, c) - u[k] * u[c];
}
// pi_{mu}^{lam} as a lowered 4-vector (kernel_IS.cl:328-329)
template <class real> __device__ __forceinline__ void pi_low(int lam, const real pimn[10], real A[4]) {
  A[0] = pimn[pidx(0, lam)];
  A[1] = -pimn[pidx(1, lam)];
  A[2] = -pimn[pidx(2, lam)];
  A[3] = -pimn[pidx(3, lam)];
}
// omega_{a}^{lam} (kernel_IS.cl:406-417)
template <class real> __device__ __forceinline__ void omega_col(int lam, const real om[6], real B[4]) {
  if (lam == 0) { B[0] = 0.0f; B[1] = om[0]; B[2] = om[1]; B[3] = om[2]; }
  else if (lam == 1) { B[0] = om[0]; B[1] = 0.0f; B[2] = om[3]; B[3] = om[4]; }
  else if (lam == 2) { B[0] = om[1]; B[1] = -om[3]; B[2] = 0.0f; B[3] = om[5]; }
  else { B[0] = om[2]; B[1] = -om[4]; B[2] = -om[5]; B[3] = 0.0f; }
}
// pi^{<mu}_{lam} pi^{nu>lam} (kernel_IS.cl:324-346), GUBSER_VISC_TEST only
template <class real> __device__ real pipi(int lam, int mu, int nu, const real pimn[10], const real u[4]) {
  real A[4], D[4][4], temp[4];
  pi_low<real>(lam, pimn, A);
  delta4<real>(u, D);
  real firstTerm = dot4<real>(D[mu], A) * dot4<real>(D[nu], A);
#pragma unroll
  for (int q = 0; q < 4; q++) temp[q] = dot4<real>(D[q], A);
  real secondTerm = -1.0f / 3.0f * (gmn<real>(mu, nu) - u[mu] * u[nu]) * dot4<real>(temp, A);
  return firstTerm + secondTerm;
}
// Omega^{mu nu} (kernel_IS.cl:355-377)
template <class real> __device__ real omega_munu(int mu, int nu, const real om[6], const real u[4]) {
  real ua[4] = {u[0], -u[1], -u[2], -u[3]};
  real D[4][4], A[4][4], temp[4];
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int c = 0; c < 4; c++) D[k][c] = (k == c ? (real)1.0f : (real)0.0f) - u[k] * ua[c];
  A[0][0] = 0.0f;   A[0][1] = om[0];  A[0][2] = om[1];  A[0][3] = om[2];
  A[1][0] = -om[0]; A[1][1] = 0.0f;   A[1][2] = om[3];  A[1][3] = om[4];
  A[2][0] = -om[1]; A[2][1] = -om[3]; A[2][2] = 0.0f;   A[2][3] = om[5];
  A[3][0] = -om[2]; A[3][1] = -om[4]; A[3][2] = -om[5]; A[3][3] = 0.0f;
#pragma unroll
  for (int q = 0; q < 4; q++) temp[q] = dot4<real>(D[nu], A[q]);
  return 0.5f * dot4<real>(D[mu], temp);
}
// the six Omega components from the velocity gradients (kernel_IS.cl:637-651)
template <class real>
__device__ void omega_tensor(const real udt[4], const real g[3][4], const real u[4], real Om[6]) {
  real om[6];
  om[0] = udt[1] - g[0][0];
  om[1] = udt[2] - g[1][0];
  om[2] = udt[3] - g[2][0];
  om[3] = g[0][2] - g[1][1];
  om[4] = g[0][3] - g[2][1];
  om[5] = g[1][3] - g[2][2];
  Om[0] = omega_munu<real>(0, 1, om, u);
  Om[1] = omega_munu<real>(0, 2, om, u);
  Om[2] = omega_munu<real>(0, 3, om, u);
  Om[3] = omega_munu<real>(1, 2, om, u);
  Om[4] = omega_munu<real>(1, 3, om, u);
  Om[5] = omega_munu<real>(2, 3, om, u);
}
// pi^{<mu}_{lam} omega^{nu>lam} (kernel_IS.cl:390-437)
template <class real>
__device__ real pi_omega(int lam, int mu, int nu, const real pimn[10], const real Om[6], const real u[4]) {
  real A[4], B[4], D[4][4], temp[4];
  pi_low<real>(lam, pimn, A);
  omega_col<real>(lam, Om, B);
  delta4<real>(u, D);
  real firstTerm = 0.5f * (dot4<real>(D[mu], A) * dot4<real>(D[nu], B) + dot4<real>(D[mu], B) * dot4<real>(D[nu], A));
#pragma unroll
  for (int q = 0; q < 4; q++) temp[q] = dot4<real>(D[q], A);
  real secondTerm = -1.0f / 3.0f * (gmn<real>(mu, nu) - u[mu] * u[nu]) * dot4<real>(temp, B);
  return firstTerm + secondTerm;
}
// omega^{<mu}_{lam} omega^{nu>lam} (kernel_IS.cl:449-487)
template <class real> __device__ real omega_omega(int lam, int mu, int nu, const real Om[6], const real u[4]) {
  real B[4], D[4][4], temp[4];
  omega_col<real>(lam, Om, B);
  delta4<real>(u, D);
  real firstTerm = dot4<real>(D[mu], B) * dot4<real>(D[nu], B);
#pragma unroll
  for (int q = 0; q < 4; q++) temp[q] = dot4<real>(D[q], B);
  real secondTerm = -1.0f / 3.0f * (gmn<real>(mu, nu) - u[mu] * u[nu]) * dot4<real>(temp, B);
  return firstTerm + secondTerm;
}

// ordered-integer keys for an atomic max over floating values
__device__ __forceinline__ unsigned int fkey(float f) {
  unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ unsigned long long fkey(double f) {
  unsigned long long b = (unsigned long long)__double_as_longlong(f);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
// atomicMax of the ordered key of f into *key; the tolerance build first takes
// the maximum over the active lanes of the warp that update the same key (a
// warp of the batched kernel can span several events), by hardware warp
// reductions over the lanes __match_any_sync groups (64-bit keys as the high
// word, then the low word among the lanes holding the largest high word), so
// that one lane of each group issues the atomic
__device__ __forceinline__ unsigned int warp_max_key(unsigned int m, unsigned int k) { return __reduce_max_sync(m, k); }
__device__ __forceinline__ unsigned long long warp_max_key(unsigned int m, unsigned long long k) {
  const unsigned int hi = __reduce_max_sync(m, (unsigned int)(k >> 32));
  const unsigned int lo = __reduce_max_sync(m, (unsigned int)(k >> 32) == hi ? (unsigned int)k : 0u);
  return ((unsigned long long)hi << 32) | lo;
}
template <class real> __device__ __forceinline__ void key_max(typename KeyT<real>::type* key, real f) {
  typedef typename KeyT<real>::type K;
  const bool ok = (f == f);
  K k = ok ? fkey(f) : (K)0;
#if CLV_FAST
  const unsigned int m = __match_any_sync(__activemask(), (unsigned long long)key);
  k = warp_max_key(m, k);
  if ((threadIdx.x & 31) == (unsigned int)(__ffs(m) - 1) && k != (K)0) atomicMax(key, k);
#else
  if (ok) atomicMax(key, k);
#endif
}
}  // namespace CLV_ARITH
}  // namespace clv
