// TEST INFRASTRUCTURE ONLY -- the oracle.
//
// A CPU restatement, expression by expression, of CLVisc's OpenCL hot path:
//   pyvisc/kernel/real_type.h, helper.h, eos_table.h, kernel_ideal.cl,
//   kernel_visc.cl, kernel_IS.cl, kernel_reduction.cl, kernel_hypersf.cl.
// Every function cites the reference file:line it follows. It keeps the
// reference's float-literal constants (THETA 1.1f, hbarc 0.19733f, the -D
// defines DT/DX/... which the host emits as "%sf" literals), its float32 EOS
// table read with clamp-to-edge nearest sampling and a manual lerp, and its
// operation order (no FMA contraction: build with -ffp-contract=off).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
// this code, as the checker and the timed CPU baseline. The product
// (clvisc_b200/) never links or calls it.
#pragma once
#include <cmath>
#include <cstdint>
#include <climits>

namespace clvo {

// ---------------------------------------------------------------- constants
// The reference's compile-time defines (ideal.py:146-171, visc.py:111-121,
// eos.py:194-201, ideal.py:190-194). Floating values are float literals.
struct Consts {
  int NX, NY, NZ;
  float DT, DX, DY, DZ, TAU0;
  float ETAOS_XMIN, ETAOS_YMIN, ETAOS_LEFT_SLOP, ETAOS_RIGHT_SLOP, LAM1;
  float EFRZ;
  int nxskip, nyskip, nzskip;
  int eos_kind;  // 0: EOS_TABLE branch, 1: EOSI branch (eos_table.h:8-31)
  float EOS_ED_START, EOS_ED_STEP;
  int EOS_NUM_ED, EOS_NUM_OF_ROWS, EOS_NUM_OF_COLS;
  const float* eos_table;  // nrow*ncol*4 floats: (cs2, p, T, s) per texel
  int riemann_test;        // -D RIEMANN_TEST
  int gubser_visc_test;    // -D GUBSER_VISC_TEST
  int pimn_omega_coupling; // -D PIMUNU_OMEGA_COUPLING
  int omega_omega_coupling;// -D OMEGA_OMEGA_COUPLING
  // Bulk viscosity. The reference has none (kernel_visc.cl:31-33 keeps a
  // zero placeholder); these fields select the bulk sector specified below.
  int bulk;
  float ZETAOS_MAX, ZETAOS_T0, ZETAOS_WIDTH, ZETAOS_SKEW;
  float ZETAOS_TMIN;  // Pi = 0 in cells colder than this
};

// real_type.h:9,16
template <class real> struct Acu;
template <> struct Acu<float> { static constexpr float v = 1.0E-7f; };
template <> struct Acu<double> { static constexpr double v = 1.0E-14; };

// helper.h:7-8
#define CLVO_THETA 1.1f
#define CLVO_HBARC 0.19733f

// ------------------------------------------------------------ vector type
template <class real> struct V4 { real s0, s1, s2, s3; };
template <class real> inline V4<real> v4(real a, real b, real c, real d) { return V4<real>{a, b, c, d}; }
template <class real> inline V4<real> operator+(V4<real> a, V4<real> b) { return {a.s0 + b.s0, a.s1 + b.s1, a.s2 + b.s2, a.s3 + b.s3}; }
template <class real> inline V4<real> operator-(V4<real> a, V4<real> b) { return {a.s0 - b.s0, a.s1 - b.s1, a.s2 - b.s2, a.s3 - b.s3}; }
template <class real> inline V4<real> operator-(V4<real> a) { return {-a.s0, -a.s1, -a.s2, -a.s3}; }
template <class real> inline V4<real> operator*(V4<real> a, V4<real> b) { return {a.s0 * b.s0, a.s1 * b.s1, a.s2 * b.s2, a.s3 * b.s3}; }
template <class real> inline V4<real> smul(real s, V4<real> a) { return {s * a.s0, s * a.s1, s * a.s2, s * a.s3}; }
template <class real> inline V4<real> vmul(V4<real> a, real s) { return {a.s0 * s, a.s1 * s, a.s2 * s, a.s3 * s}; }
template <class real> inline V4<real> vdiv(V4<real> a, real s) { return {a.s0 / s, a.s1 / s, a.s2 / s, a.s3 / s}; }
template <class real> inline real comp(V4<real> a, int i) { return i == 0 ? a.s0 : i == 1 ? a.s1 : i == 2 ? a.s2 : a.s3; }
// OpenCL dot(): evaluated left to right, no fused multiply-add.
template <class real> inline real dot(V4<real> a, V4<real> b) {
  real r = a.s0 * b.s0;
  r = r + a.s1 * b.s1;
  r = r + a.s2 * b.s2;
  r = r + a.s3 * b.s3;
  return r;
}

// OpenCL builtins (min/max: "y if y < x" / "y if x < y"; sign: +-1, +-0, 0 for NaN)
template <class real> inline real cl_min(real x, real y) { return (y < x) ? y : x; }
template <class real> inline real cl_max(real x, real y) { return (x < y) ? y : x; }
template <class real> inline real cl_sign(real x) {
  if (x > (real)0) return (real)1;
  if (x < (real)0) return (real)-1;
  if (x != x) return (real)0;
  return x;  // +0 or -0
}
// float -> int conversion with the GPU's saturating semantics (NaN -> 0);
// the reference only ever converts in-range non-negative values here.
template <class real> inline int f2i(real x) {
  if (x != x) return 0;
  if (x >= (real)2147483647.0) return INT_MAX;
  if (x <= (real)-2147483648.0) return INT_MIN;
  return (int)x;
}

// g^{tau mu} ... without tau*tau (helper.h:59-63)
template <class real> inline V4<real> gm(int a) {
  switch (a) {
    case 0: return V4<real>{(real)1.0f, (real)0.0f, (real)0.0f, (real)0.0f};
    case 1: return V4<real>{(real)0.0f, (real)-1.0f, (real)0.0f, (real)0.0f};
    case 2: return V4<real>{(real)0.0f, (real)0.0f, (real)-1.0f, (real)0.0f};
    default: return V4<real>{(real)0.0f, (real)0.0f, (real)0.0f, (real)-1.0f};
  }
}
// kernel_IS.cl:3-6
template <class real> inline real gmn(int a, int b) { return a != b ? (real)0.0f : (a == 0 ? (real)1.0f : (real)-1.0f); }

// helper.h:31
inline int idx(int i, int j) { return (i < j) ? ((7 * i + 2 * j - i * i) / 2) : ((7 * j + 2 * i - j * j) / 2); }

// ----------------------------------------------------------------- EOS
// eos_table.h:33-104 (EOS_TABLE) and eos_table.h:8-31 (EOSI).
template <class real> struct Eos {
  const Consts& c;
  explicit Eos(const Consts& cc) : c(cc) {}

  V4<real> texel(int col, int row) const {  // clamp-to-edge nearest sampler
    if (col < 0) col = 0;
    if (col > c.EOS_NUM_OF_COLS - 1) col = c.EOS_NUM_OF_COLS - 1;
    if (row < 0) row = 0;
    if (row > c.EOS_NUM_OF_ROWS - 1) row = c.EOS_NUM_OF_ROWS - 1;
    const float* t = c.eos_table + 4 * ((size_t)row * c.EOS_NUM_OF_COLS + col);
    return V4<real>{(real)t[0], (real)t[1], (real)t[2], (real)t[3]};
  }
  // eos_table.h:39-62
  V4<real> eos(real eps) const {
    real ed_per_row = c.EOS_ED_STEP * c.EOS_NUM_OF_COLS;
    int row = f2i<real>(eps / ed_per_row);
    int col = f2i<real>((eps - c.EOS_ED_START - row * ed_per_row) / c.EOS_ED_STEP);
    real eps_low = c.EOS_ED_START + row * ed_per_row + col * c.EOS_ED_STEP;
    V4<real> eos_low = texel(col, row);
    col = col + 1;
    if (col == c.EOS_NUM_OF_COLS) {
      row += 1;
      col = 0;
    }
    V4<real> eos_high = texel(col, row);
    real r = (eps - eps_low) / c.EOS_ED_STEP;
    return smul<real>((real)(1.0f - r), eos_low) + smul<real>(r, eos_high);
  }
  bool in_table(real eps) const { return eps < c.EOS_ED_START + c.EOS_NUM_ED * c.EOS_ED_STEP; }

  // EOSI constants, eos_table.h:10-13
  static real eosi_T(real eps) {
    const float dof = 169.0f / 4.0f;
    const float hbarc1 = 0.1973269f;
    const float pi_f = (float)M_PI;                   // M_PI_F
    const float coef = (pi_f * pi_f / 30.0f);
    return hbarc1 * std::pow((real)1.0f / (dof * coef) * eps / hbarc1, (real)0.25f);
  }

  real P(real eps) const {  // eos_table.h:65-71
    if (c.eos_kind == 1) return eps / 3.0f;
    if (in_table(eps)) return eos(eps).s1;
    return 0.3327f * eps - 0.3223f * std::pow(eps, (real)0.4585f) - 0.003906f * eps * std::exp(-0.05697f * eps);
  }
  real S(real eps) const {  // eos_table.h:74-81
    if (c.eos_kind == 1) {
      real t = eosi_T(eps);
      return (eps + P(eps)) / std::fmax((real)1.0E-10f, t);
    }
    if (in_table(eps)) return eos(eps).s3;
    return 18.202f * eps - 63.0218f - 4.85479f * std::exp(-2.72407E-11f * std::pow(eps, (real)4.54886f)) +
           65.1272f * std::pow(eps, -(real)0.128012f) * std::exp(-0.00369624f * std::pow(eps, (real)1.18735f));
  }
  real T(real eps) const {  // eos_table.h:85-91
    if (c.eos_kind == 1) return eosi_T(eps);
    if (in_table(eps)) return eos(eps).s2;
    return (eps + P(eps)) / S(eps);
  }
  real CS2(real eps) const {  // eos_table.h:94-100
    if (c.eos_kind == 1) return 0.33333333f;
    if (in_table(eps)) return eos(eps).s0;
    return 0.333333333f;
  }
};

// -------------------------------------------------------------- helper.h
template <class real> struct Helper {
  const Consts& c;
  Eos<real> E;
  static constexpr real acu = Acu<real>::v;
  explicit Helper(const Consts& cc) : c(cc), E(cc) {}

  real etaos(real temperature) const {  // helper.h:23-26
    return (temperature < c.ETAOS_XMIN) ? (c.ETAOS_LEFT_SLOP * (temperature - c.ETAOS_XMIN) + c.ETAOS_YMIN)
                                        : (c.ETAOS_RIGHT_SLOP * (temperature - c.ETAOS_XMIN) + c.ETAOS_YMIN);
  }
  // Bulk sector (no counterpart in the reference). zeta/s(T) is a skewed
  // Cauchy peak, (zeta/s)_max w^2 / (w^2 + (T - T0)^2) with
  // w = width * (1 + skew * sign(T - T0)), the parametrisation of the
  // JETSCAPE Bayesian analysis (Everett et al., PRC 103, 054904 (2021));
  // it needs only +, -, *, /, so both sides evaluate it to the same bits.
  real zetaos(real temperature) const {
    real dT = temperature - c.ZETAOS_T0;
    real w = c.ZETAOS_WIDTH * (1.0f + c.ZETAOS_SKEW * cl_sign<real>(dT));
    return c.ZETAOS_MAX * (w * w) / (w * w + dT * dT);
  }
  static real gamma(real vx, real vy, real vz) {  // helper.h:46-48
    return 1.0f / std::sqrt(cl_max<real>(1.0f - vx * vx - vy * vy - vz * vz, acu));
  }
  static real gamma_real4(V4<real> ev) {  // helper.h:51-53
    return 1.0f / std::sqrt(cl_max<real>(1.0f - ev.s1 * ev.s1 - ev.s2 * ev.s2 - ev.s3 * ev.s3, acu));
  }
  static V4<real> umu4(V4<real> ev) {  // helper.h:56-58
    real g = gamma_real4(ev);
    return smul<real>(g, V4<real>{(real)1.0f, ev.s1, ev.s2, ev.s3});
  }
  static real minmod(real x, real y) {  // helper.h:74-77
    real res = cl_min<real>(std::fabs(x), std::fabs(y));
    return res * (cl_sign(x) + cl_sign(y)) * 0.5f;
  }
  static V4<real> minmod4(V4<real> x, V4<real> y) {  // helper.h:79-82
    return V4<real>{minmod(x.s0, y.s0), minmod(x.s1, y.s1), minmod(x.s2, y.s2), minmod(x.s3, y.s3)};
  }
  real maxPropagationSpeed(V4<real> edv, real vk) const {  // helper.h:94-105
    real ut = gamma(edv.s1, edv.s2, edv.s3);
    real uk = ut * vk;
    real ut2 = ut * ut;
    real uk2 = uk * uk;
    real cs2 = E.CS2(edv.s0);
    real lam = (std::fabs(ut * uk * (1.0f - cs2)) + std::sqrt((ut2 - uk2 - (ut2 - uk2 - 1.0f) * cs2) * cs2)) /
               (ut2 - (ut2 - 1.0f) * cs2);
    return cl_max<real>(lam, 1.0f);
  }
  // helper.h:112-125 (fixed-point root finder; used by test_kernel_helper.py)
  void rootFinding(real* EdFind, real T00, real M) const {
    real E0, E1;
    E1 = T00;
    real K2 = M * M;
    int i = 0;
    while (true) {
      E0 = E1;
      E1 = T00 - K2 / (T00 + E.P(E1));
      i++;
      if (i > 100 || std::fabs(E1 - E0) / cl_max<real>(std::fabs(E1), (real)acu) < acu) break;
    }
    *EdFind = E1;
  }
  // helper.h:128-167
  // With bulk != nullptr the pressure is P(e) + Pi (the bulk sector).
  void rootFinding_newton(real* ed_find, real T00, real M, int* iters = nullptr, const real* bulk = nullptr) const {
    real vl = 0.0f;
    real vh = 1.0f;
    real dpe = 1.0f / 3.0f;
    real v = 0.5f * (vl + vh);
    real ed = T00 - M * v;
    real pr = E.P(ed);
    if (bulk) pr = pr + *bulk;
    real f = (T00 + pr) * v - M;
    real df = (T00 + pr) - M * v * dpe;
    real dvold = vh - vl;
    real dv = dvold;
    int i = 0;
    while (true) {
      if ((f + df * (vh - v)) * (f + df * (vl - v)) > 0.0f || std::fabs(2.f * f) > std::fabs(dvold * df)) {
        dvold = dv;
        dv = 0.5f * (vh - vl);
        v = vl + dv;
      } else {
        dvold = dv;
        dv = f / df;
        v -= dv;
      }
      i++;
      if (std::fabs(dv) < 0.00001f || i > 100) break;
      ed = T00 - M * v;
      pr = E.P(ed);
      if (bulk) pr = pr + *bulk;
      f = (T00 + pr) * v - M;
      df = (T00 + pr) - M * v * dpe;
      if (f > 0.0f) {
        vh = v;
      } else {
        vl = v;
      }
    }
    if (iters) *iters = i;
    *ed_find = T00 - M * v;
  }
  // helper.h:172-177
  static V4<real> t0m(V4<real> edv, real pr) {
    real u0 = gamma(edv.s1, edv.s2, edv.s3);
    real ed = edv.s0;
    V4<real> u4 = vmul<real>(V4<real>{(real)1.0f, edv.s1, edv.s2, edv.s3}, u0);
    return smul<real>((ed + pr) * u0, u4) - vmul<real>(gm<real>(0), pr);
  }
  // helper.h:179-242
  V4<real> kt1d(V4<real> ev_im2, V4<real> ev_im1, V4<real> ev_i, V4<real> ev_ip1, V4<real> ev_ip2, real tau,
                int along) const {
    (void)tau;
    const real TH = CLVO_THETA;
    real pr_im1 = E.P(ev_im1.s0);
    real pr_i = E.P(ev_i.s0);
    real pr_ip1 = E.P(ev_ip1.s0);
    real pr_ip2 = E.P(ev_ip2.s0);
    V4<real> T0m_im1 = t0m(ev_im1, pr_im1);
    V4<real> T0m_i = t0m(ev_i, pr_i);
    V4<real> T0m_ip1 = t0m(ev_ip1, pr_ip1);
    V4<real> T0m_ip2 = t0m(ev_ip2, pr_ip2);
    V4<real> DA0, DA1;
    DA0 = minmod4(smul<real>(0.5f, T0m_ip1 - T0m_im1), minmod4(smul<real>(TH, T0m_ip1 - T0m_i), smul<real>(TH, T0m_i - T0m_im1)));
    DA1 = minmod4(smul<real>(0.5f, T0m_ip2 - T0m_i), minmod4(smul<real>(TH, T0m_ip2 - T0m_ip1), smul<real>(TH, T0m_ip1 - T0m_i)));
    real vim1[3] = {ev_im1.s1, ev_im1.s2, ev_im1.s3};
    real vi[3] = {ev_i.s1, ev_i.s2, ev_i.s3};
    real vip1[3] = {ev_ip1.s1, ev_ip1.s2, ev_ip1.s3};
    V4<real> AL = T0m_i + smul<real>(0.5f, DA0);
    V4<real> AR = T0m_ip1 - smul<real>(0.5f, DA1);
    real pr_half = 0.5f * (pr_ip1 + pr_i);
    real vi_half = 0.5f * (vi[along] + vip1[along]);
    V4<real> Jp = vmul<real>(AR + smul<real>(pr_half, gm<real>(0)), vi_half) - smul<real>(pr_half, gm<real>(along + 1));
    V4<real> Jm = vmul<real>(AL + smul<real>(pr_half, gm<real>(0)), vi_half) - smul<real>(pr_half, gm<real>(along + 1));
    V4<real> ev_half = smul<real>(0.5f, ev_i + ev_ip1);
    real lam = maxPropagationSpeed(ev_half, vi_half);
    V4<real> src = smul<real>(0.5f, Jp + Jm) - smul<real>((real)0.5f * lam, AR - AL);
    real pr_im2 = E.P(ev_im2.s0);
    V4<real> T0m_im2 = t0m(ev_im2, pr_im2);
    DA1 = DA0;
    DA0 = minmod4(smul<real>(0.5f, T0m_i - T0m_im2), minmod4(smul<real>(TH, T0m_i - T0m_im1), smul<real>(TH, T0m_im1 - T0m_im2)));
    AL = T0m_im1 + smul<real>(0.5f, DA0);
    AR = T0m_i - smul<real>(0.5f, DA1);
    pr_half = 0.5f * (pr_im1 + pr_i);
    vi_half = 0.5f * (vim1[along] + vi[along]);
    Jp = vmul<real>(AR + smul<real>(pr_half, gm<real>(0)), vi_half) - smul<real>(pr_half, gm<real>(along + 1));
    Jm = vmul<real>(AL + smul<real>(pr_half, gm<real>(0)), vi_half) - smul<real>(pr_half, gm<real>(along + 1));
    ev_half = smul<real>(0.5f, ev_i + ev_im1);
    lam = maxPropagationSpeed(ev_half, vi_half);
    src = src - (smul<real>(0.5f, Jp + Jm) - smul<real>((real)0.5f * lam, AR - AL));
    return src;
  }
  // helper.h:249-285
  static real kt1d_real(real Q_im2, real Q_im1, real Q_i, real Q_ip1, real Q_ip2, real v_mh, real v_ph, real lam_mh,
                        real lam_ph) {
    const real TH = CLVO_THETA;
    real DA0, DA1;
    DA0 = minmod(0.5f * (Q_ip1 - Q_im1), minmod(TH * (Q_ip1 - Q_i), TH * (Q_i - Q_im1)));
    DA1 = minmod(0.5f * (Q_ip2 - Q_i), minmod(TH * (Q_ip2 - Q_ip1), TH * (Q_ip1 - Q_i)));
    real AL = Q_i + 0.5f * DA0;
    real AR = Q_ip1 - 0.5f * DA1;
    real Jp = AR * v_ph;
    real Jm = AL * v_ph;
    real src = 0.5f * (Jp + Jm) - 0.5f * lam_ph * (AR - AL);
    DA1 = DA0;
    DA0 = minmod(0.5f * (Q_i - Q_im2), minmod(TH * (Q_i - Q_im1), TH * (Q_im1 - Q_im2)));
    AL = Q_im1 + 0.5f * DA0;
    AR = Q_i - 0.5f * DA1;
    Jp = AR * v_mh;
    Jm = AL * v_mh;
    src -= 0.5f * (Jp + Jm) - 0.5f * lam_mh * (AR - AL);
    return src;
  }
};

// Reference cell index I = i*NY*NZ + j*NZ + k (kernel_visc.cl:145)
inline size_t cell(const Consts& c, int i, int j, int k) { return ((size_t)i * c.NY + j) * c.NZ + k; }

}  // namespace clvo
