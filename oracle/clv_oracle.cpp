// TEST INFRASTRUCTURE ONLY -- the oracle (see clv_oracle.hpp).
//
// One function per reference OpenCL kernel, over the reference's own buffer
// layout: ev = real4 per cell (ed, vx, vy, veta), pi = 10 reals per cell packed
// by idx(), Src = real4 per cell (KT) or 10 reals per cell (IS). Work-item
// loops become OpenMP loops; a work-group's __local line buffer with two ghost
// cells of constant extrapolation becomes a clamped neighbour index. The
// hypersurface kernels append in cube order (count, prefix, write) instead of
// the reference's atomic_inc, so their output order is deterministic.
#include <vector>
#include <algorithm>
#include <cstring>
#include "clv_oracle.hpp"

namespace clvo {

inline int clampi(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }
template <class real> inline V4<real> ld4(const real* p, size_t I) { return V4<real>{p[4 * I], p[4 * I + 1], p[4 * I + 2], p[4 * I + 3]}; }
template <class real> inline void st4(real* p, size_t I, V4<real> v) { p[4 * I] = v.s0; p[4 * I + 1] = v.s1; p[4 * I + 2] = v.s2; p[4 * I + 3] = v.s3; }

// neighbour d along axis of cell (i,j,k), clamped: the ghost cells of
// kernel_ideal.cl:166-172 repeat the edge cell.
inline size_t nbr(const Consts& c, int i, int j, int k, int axis, int d) {
  if (axis == 0) i = clampi(i + d, 0, c.NX - 1);
  else if (axis == 1) j = clampi(j + d, 0, c.NY - 1);
  else k = clampi(k + d, 0, c.NZ - 1);
  return cell(c, i, j, k);
}
inline size_t ncells(const Consts& c) { return (size_t)c.NX * c.NY * c.NZ; }

// ============================================================ kernel_ideal.cl
// kernel_ideal.cl:3-36
template <class real>
void ideal_christoffel(const Consts& c, real* Src, const real* ev, real tau, int step) {
  Helper<real> H(c);
  const long N = (long)ncells(c);
#pragma omp parallel for schedule(static)
  for (long I = 0; I < N; I++) {
    if (step == 1) st4(Src, I, V4<real>{0.0f, 0.0f, 0.0f, 0.0f});
    V4<real> e_v = ld4(ev, I);
    real ed = e_v.s0, vx = e_v.s1, vy = e_v.s2, vz = e_v.s3;
    real pressure = H.E.P(ed);
    real u0 = Helper<real>::gamma(vx, vy, vz);
    real Tzz_tilde = (ed + pressure) * u0 * u0 * vz * vz + pressure;
    real Ttz_tilde = (ed + pressure) * u0 * u0 * vz;
    if (!c.riemann_test) st4(Src, I, ld4(Src, I) - V4<real>{Tzz_tilde, 0.0f, 0.0f, Ttz_tilde});
  }
}

// kernel_ideal.cl:39-165 (kt_src_alongx/y/z)
template <class real>
void ideal_along(const Consts& c, int axis, real* Src, const real* ev, real tau) {
  Helper<real> H(c);
  const int n0 = axis == 0 ? c.NY : c.NX;
  const int n1 = axis == 2 ? c.NY : c.NZ;
  const int L = axis == 0 ? c.NX : (axis == 1 ? c.NY : c.NZ);
#pragma omp parallel for collapse(2) schedule(static)
  for (int a = 0; a < n0; a++)
    for (int b = 0; b < n1; b++)
      for (int t = 0; t < L; t++) {
        int i, j, k;
        if (axis == 0) { i = t; j = a; k = b; }
        else if (axis == 1) { i = a; j = t; k = b; }
        else { i = a; j = b; k = t; }
        size_t IND = cell(c, i, j, k);
        V4<real> e[5];
        for (int d = -2; d <= 2; d++) e[d + 2] = ld4(ev, nbr(c, i, j, k, axis, d));
        V4<real> f = H.kt1d(e[0], e[1], e[2], e[3], e[4], tau, axis);
        V4<real> s = ld4(Src, IND);
        if (c.riemann_test) {
          real D = axis == 0 ? c.DX : (axis == 1 ? c.DY : c.DZ);
          st4(Src, IND, s - vdiv<real>(f, D));
        } else if (axis == 0) {
          st4(Src, IND, s - vdiv<real>(smul<real>(tau, f), c.DX));
        } else if (axis == 1) {
          st4(Src, IND, s - vdiv<real>(smul<real>(tau, f), c.DY));
        } else {
          st4(Src, IND, s - vdiv<real>(smul<real>(tau, f), tau * c.DZ));
        }
      }
}

// kernel_ideal.cl:165-231
template <class real>
void ideal_update_ev(const Consts& c, real* evnew, const real* ev1, const real* Src, real tau, int step) {
  Helper<real> H(c);
  const real acu = Acu<real>::v;
  const long N = (long)ncells(c);
#pragma omp parallel for schedule(static)
  for (long I = 0; I < N; I++) {
    V4<real> e_v = ld4(ev1, I);
    real ed = e_v.s0, vx = e_v.s1, vy = e_v.s2, vz = e_v.s3;
    real pressure = H.E.P(ed);
    real u0 = Helper<real>::gamma(vx, vy, vz);
    V4<real> umu = smul<real>(u0, V4<real>{1.0f, vx, vy, vz});
    real old_time = tau - (step - 1) * c.DT;
    V4<real> T0m = smul<real>((ed + pressure) * u0, umu) - smul<real>(pressure, gm<real>(0));
    if (!c.riemann_test) T0m = vmul<real>(T0m, old_time);
    T0m = T0m + vdiv<real>(vmul<real>(ld4(Src, I), (real)c.DT), (real)step);
    real T00, T01, T02, T03;
    if (c.riemann_test) {
      T00 = cl_max<real>(acu, T0m.s0);
      T01 = (std::fabs(T0m.s1) < acu) ? (real)0.0f : T0m.s1;
      T02 = (std::fabs(T0m.s2) < acu) ? (real)0.0f : T0m.s2;
      T03 = (std::fabs(T0m.s3) < acu) ? (real)0.0f : T0m.s3;
    } else {
      T00 = cl_max<real>(acu, T0m.s0) / tau;
      T01 = (std::fabs(T0m.s1) < acu) ? (real)0.0f : T0m.s1 / tau;
      T02 = (std::fabs(T0m.s2) < acu) ? (real)0.0f : T0m.s2 / tau;
      T03 = (std::fabs(T0m.s3) < acu) ? (real)0.0f : T0m.s3 / tau;
    }
    real M = std::sqrt(T01 * T01 + T02 * T02 + T03 * T03);
    real SCALE_COEF = 0.999f;
    if (M > T00) {
      T01 *= SCALE_COEF * T00 / M;
      T02 *= SCALE_COEF * T00 / M;
      T03 *= SCALE_COEF * T00 / M;
      M = SCALE_COEF * T00;
    }
    real ed_find;
    H.rootFinding_newton(&ed_find, T00, M);
    ed_find = cl_max<real>(0.0f, ed_find);
    real pr = H.E.P(ed_find);
    real epv = cl_max<real>(acu, T00 + pr);
    st4(evnew, I, V4<real>{ed_find, T01 / epv, T02 / epv, T03 / epv});
  }
}

// ============================================================= kernel_visc.cl
// kernel_visc.cl:11-53
template <class real>
void visc_christoffel(const Consts& c, real* SrcT, const real* ev, const real* pi, real tau, int step,
                      const real* bulk = nullptr) {
  Helper<real> H(c);
  (void)tau;
  const long N = (long)ncells(c);
#pragma omp parallel for schedule(static)
  for (long I = 0; I < N; I++) {
    if (step == 1) st4(SrcT, I, V4<real>{0.0f, 0.0f, 0.0f, 0.0f});
    V4<real> e_v = ld4(ev, I);
    real ed = e_v.s0, vx = e_v.s1, vy = e_v.s2, vz = e_v.s3;
    real u0 = Helper<real>::gamma(vx, vy, vz);
    real bulkpi = bulk ? bulk[I] : (real)0.0f;  // the bulk sector fills the reference's placeholder
    real pressure = H.E.P(ed) + bulkpi;
    real Tzz_tilde = (ed + pressure) * u0 * u0 * vz * vz + pressure + pi[10 * I + idx(3, 3)];
    real Ttz_tilde = (ed + pressure) * u0 * u0 * vz + pi[10 * I + idx(0, 3)];
    st4(SrcT, I, ld4(SrcT, I) - V4<real>{Tzz_tilde, 0.0f, 0.0f, Ttz_tilde});
    if (c.riemann_test) {
      real Ttt_tilde = (ed + pressure) * u0 * u0 - pressure;
      real Ttx_tilde = (ed + pressure) * u0 * u0 * vx;
      real Tty_tilde = (ed + pressure) * u0 * u0 * vy;
      st4(SrcT, I, ld4(SrcT, I) + V4<real>{Tzz_tilde + Ttt_tilde, Ttx_tilde, Tty_tilde, 3.0f * Ttz_tilde});
    }
  }
}

// kernel_visc.cl:68-127
template <class real>
V4<real> kt1d_visc(const Helper<real>& H, const V4<real> ev[5], const V4<real> pim0[5], const V4<real> pimi[5],
                   real vip_half, real vim_half, real tau, int along, const real* bulk5 = nullptr) {
  const real TH = CLVO_THETA;
  real pr[5];
  V4<real> Q[5];
  for (int i = 0; i < 5; i++) {
    pr[i] = H.E.P(ev[i].s0);
    if (bulk5) pr[i] = pr[i] + bulk5[i];  // bulk sector: P -> P + Pi
    Q[i] = smul<real>(tau, Helper<real>::t0m(ev[i], pr[i]) + pim0[i]);
  }
  V4<real> DA0, DA1;
  int i = 2;
  DA0 = Helper<real>::minmod4(smul<real>(0.5f, Q[i + 1] - Q[i - 1]),
                              Helper<real>::minmod4(smul<real>(TH, Q[i + 1] - Q[i]), smul<real>(TH, Q[i] - Q[i - 1])));
  i = 3;
  DA1 = Helper<real>::minmod4(smul<real>(0.5f, Q[i + 1] - Q[i - 1]),
                              Helper<real>::minmod4(smul<real>(TH, Q[i + 1] - Q[i]), smul<real>(TH, Q[i] - Q[i - 1])));
  V4<real> AL = Q[2] + smul<real>(0.5f, DA0);
  V4<real> AR = Q[3] - smul<real>(0.5f, DA1);
  real pr_half = 0.5f * (pr[2] + pr[3]);
  V4<real> pim0_half = smul<real>(0.5f, pim0[2] + pim0[3]);
  V4<real> pimi_half = smul<real>(0.5f, pimi[2] + pimi[3]);
  V4<real> g0 = gm<real>(0), ga = gm<real>(along + 1);
  V4<real> Jp = vmul<real>(AR + smul<real>(pr_half * tau, g0) - smul<real>(tau, pim0_half), vip_half) -
                smul<real>(pr_half * tau, ga) + smul<real>(tau, pimi_half);
  V4<real> Jm = vmul<real>(AL + smul<real>(pr_half * tau, g0) - smul<real>(tau, pim0_half), vip_half) -
                smul<real>(pr_half * tau, ga) + smul<real>(tau, pimi_half);
  V4<real> ev_half = smul<real>(0.5f, ev[2] + ev[3]);
  real lam = H.maxPropagationSpeed(ev_half, vip_half);
  V4<real> src = smul<real>(0.5f, Jp + Jm) - smul<real>((real)0.5f * lam, AR - AL);
  DA1 = DA0;
  i = 1;
  DA0 = Helper<real>::minmod4(smul<real>(0.5f, Q[i + 1] - Q[i - 1]),
                              Helper<real>::minmod4(smul<real>(TH, Q[i + 1] - Q[i]), smul<real>(TH, Q[i] - Q[i - 1])));
  AL = Q[1] + smul<real>(0.5f, DA0);
  AR = Q[2] - smul<real>(0.5f, DA1);
  pr_half = 0.5f * (pr[1] + pr[2]);
  pim0_half = smul<real>(0.5f, pim0[1] + pim0[2]);
  pimi_half = smul<real>(0.5f, pimi[1] + pimi[2]);
  Jp = vmul<real>(AR + smul<real>(pr_half * tau, g0) - smul<real>(tau, pim0_half), vim_half) -
       smul<real>(pr_half * tau, ga) + smul<real>(tau, pimi_half);
  Jm = vmul<real>(AL + smul<real>(pr_half * tau, g0) - smul<real>(tau, pim0_half), vim_half) -
       smul<real>(pr_half * tau, ga) + smul<real>(tau, pimi_half);
  ev_half = smul<real>(0.5f, ev[2] + ev[1]);
  lam = H.maxPropagationSpeed(ev_half, vim_half);
  src = src - (smul<real>(0.5f, Jp + Jm) - smul<real>((real)0.5f * lam, AR - AL));
  return src;
}

// kernel_visc.cl:131-318 (kt_src_alongx/y/z)
template <class real>
void visc_along(const Consts& c, int axis, real* Src, const real* ev, const real* pi, real tau,
                const real* bulk = nullptr) {
  Helper<real> H(c);
  const int n0 = axis == 0 ? c.NY : c.NX;
  const int n1 = axis == 2 ? c.NY : c.NZ;
  const int L = axis == 0 ? c.NX : (axis == 1 ? c.NY : c.NZ);
  const int r = axis + 1;  // pimi = pi^{r mu}
#pragma omp parallel for collapse(2) schedule(static)
  for (int a = 0; a < n0; a++)
    for (int b = 0; b < n1; b++)
      for (int t = 0; t < L; t++) {
        int i, j, k;
        if (axis == 0) { i = t; j = a; k = b; }
        else if (axis == 1) { i = a; j = t; k = b; }
        else { i = a; j = b; k = t; }
        size_t IND = cell(c, i, j, k);
        V4<real> e[5], p0[5], pr_[5];
        real b5[5];
        for (int d = -2; d <= 2; d++) {
          size_t J = nbr(c, i, j, k, axis, d);
          e[d + 2] = ld4(ev, J);
          b5[d + 2] = bulk ? bulk[J] : (real)0.0f;
          const real* p = pi + 10 * J;
          p0[d + 2] = V4<real>{p[0], p[1], p[2], p[3]};
          pr_[d + 2] = V4<real>{p[idx(r, 0)], p[idx(r, 1)], p[idx(r, 2)], p[idx(r, 3)]};
        }
        real vip_half = 0.5f * (comp(e[2], r) + comp(e[3], r));
        real vim_half = 0.5f * (comp(e[1], r) + comp(e[2], r));
        V4<real> f = kt1d_visc(H, e, p0, pr_, vip_half, vim_half, tau, axis, bulk ? b5 : nullptr);
        V4<real> s = ld4(Src, IND);
        if (axis == 0) st4(Src, IND, s - vdiv<real>(f, (real)c.DX));
        else if (axis == 1) st4(Src, IND, s - vdiv<real>(f, (real)c.DY));
        else st4(Src, IND, s - vdiv<real>(f, tau * c.DZ));
      }
}

// kernel_visc.cl:322-393
template <class real>
void visc_update_ev(const Consts& c, real* evnew, const real* ev1, const real* pi1, const real* pi2, const real* Src,
                    real tau, int step, const real* bulk1 = nullptr, const real* bulk2 = nullptr) {
  Helper<real> H(c);
  const real acu = Acu<real>::v;
  const long N = (long)ncells(c);
#pragma omp parallel for schedule(static)
  for (long I = 0; I < N; I++) {
    V4<real> e_v = ld4(ev1, I);
    real ed = e_v.s0, vx = e_v.s1, vy = e_v.s2, vz = e_v.s3;
    real pressure = H.E.P(ed);
    if (bulk1) pressure = pressure + bulk1[I];  // bulk sector
    real u0 = Helper<real>::gamma(vx, vy, vz);
    V4<real> umu = smul<real>(u0, V4<real>{1.0f, vx, vy, vz});
    V4<real> pim0 = V4<real>{pi1[10 * I + 0], pi1[10 * I + 1], pi1[10 * I + 2], pi1[10 * I + 3]};
    real old_time = tau - (step - 1) * c.DT;
    V4<real> T0m = vmul<real>(smul<real>((ed + pressure) * u0, umu) - smul<real>(pressure, gm<real>(0)) + pim0, old_time);
    pim0 = V4<real>{pi2[10 * I + 0], pi2[10 * I + 1], pi2[10 * I + 2], pi2[10 * I + 3]};
    T0m = T0m + vdiv<real>(vmul<real>(ld4(Src, I), (real)c.DT), (real)step) - vmul<real>(pim0, tau);
    real T00 = cl_max<real>(acu, T0m.s0) / tau;
    real T01 = (std::fabs(T0m.s1) < acu) ? (real)0.0f : T0m.s1 / tau;
    real T02 = (std::fabs(T0m.s2) < acu) ? (real)0.0f : T0m.s2 / tau;
    real T03 = (std::fabs(T0m.s3) < acu) ? (real)0.0f : T0m.s3 / tau;
    real M = std::sqrt(T01 * T01 + T02 * T02 + T03 * T03);
    real SCALE_COEF = 0.999f;
    if (M > T00) {
      T01 *= SCALE_COEF * T00 / M;
      T02 *= SCALE_COEF * T00 / M;
      T03 *= SCALE_COEF * T00 / M;
      M = SCALE_COEF * T00;
    }
    real ed_find;
    H.rootFinding_newton(&ed_find, T00, M, nullptr, bulk2 ? bulk2 + I : nullptr);
    if (ed_find < acu) {
      T01 = 0.0f;
      T02 = 0.0f;
      T03 = 0.0f;
    }
    ed_find = cl_max<real>(0.0f, ed_find);
    real pr = H.E.P(ed_find);
    if (bulk2) pr = pr + bulk2[I];
    real epv = cl_max<real>(acu, T00 + pr);
    st4(evnew, I, V4<real>{ed_find, T01 / epv, T02 / epv, T03 / epv});
  }
}

// =============================================================== kernel_IS.cl
// kernel_IS.cl:10-36
template <class real>
void visc_initialize(const Consts& c, real* pi1, real* goodcell, real* udiff, const real* ev, real tau,
                     real* bulk1 = nullptr) {
  Helper<real> H(c);
  const long N = (long)ncells(c);
#pragma omp parallel for schedule(static)
  for (long I = 0; I < N; I++) {
    V4<real> e = ld4(ev, I);
    V4<real> cpTs = H.E.eos(e.s0);
    real etav = H.etaos(cpTs.s2) * cpTs.s3 * CLVO_HBARC;
    real tmp = 2.0f / 3.0f * etav / tau;
    pi1[10 * I + idx(1, 1)] = tmp;
    pi1[10 * I + idx(2, 2)] = tmp;
    pi1[10 * I + idx(3, 3)] = -2.0f * tmp;
    if (bulk1) {  // bulk sector: Navier-Stokes value for Bjorken flow, theta = 1/tau, regulated
      real zetav = H.zetaos(cpTs.s2) * cpTs.s3 * CLVO_HBARC;
      real b0 = -zetav / tau;
      real pb = cpTs.s1;
      if (b0 < -pb) b0 = -pb;
      else if (b0 > pb) b0 = pb;
      if (cpTs.s2 < c.ZETAOS_TMIN) b0 = 0.0f;
      bulk1[I] = b0;
    }
    st4(udiff, I, V4<real>{0.0f, 0.0f, 0.0f, 0.0f});
    goodcell[I] = 1.0f;
  }
}

// kernel_IS.cl:41-67
template <class real>
void visc_src_christoffel(const Consts& c, real* Src, const real* pi1, const real* ev, real tau, int step,
                          real* SrcB = nullptr) {
  const long N = (long)ncells(c);
#pragma omp parallel for schedule(static)
  for (long I = 0; I < N; I++) {
    real* S = Src + 10 * I;
    const real* p = pi1 + 10 * I;
    if (step == 1)
      for (int mn = 0; mn < 10; mn++) S[mn] = 0.0f;
    if (SrcB && step == 1) SrcB[I] = 0.0f;  // bulk sector: no Christoffel term
    V4<real> e_v = ld4(ev, I);
    real uz = e_v.s3 * Helper<real>::gamma(e_v.s1, e_v.s2, e_v.s3);
    S[0] -= 2.0f * uz * p[idx(0, 3)] / tau;
    S[1] -= uz * p[idx(1, 3)] / tau;
    S[2] -= uz * p[idx(2, 3)] / tau;
    S[3] -= uz * (p[idx(0, 0)] + p[idx(3, 3)]) / tau;
    S[6] -= uz * p[idx(0, 1)] / tau;
    S[8] -= uz * p[idx(0, 2)] / tau;
    S[9] -= 2.0f * uz * p[idx(0, 3)] / tau;
  }
}

// kernel_IS.cl:74-318 (visc_src_alongx/y/z)
template <class real>
void visc_src_along(const Consts& c, int axis, real* Src, real* ud, const real* pi1, const real* ev, real tau,
                    real* SrcB = nullptr, const real* bulk1 = nullptr) {
  Helper<real> H(c);
  const real TH = CLVO_THETA;
  const int n0 = axis == 0 ? c.NY : c.NX;
  const int n1 = axis == 2 ? c.NY : c.NZ;
  const int L = axis == 0 ? c.NX : (axis == 1 ? c.NY : c.NZ);
  const int r = axis + 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int a = 0; a < n0; a++)
    for (int b = 0; b < n1; b++)
      for (int t = 0; t < L; t++) {
        int i, j, k;
        if (axis == 0) { i = t; j = a; k = b; }
        else if (axis == 1) { i = a; j = t; k = b; }
        else { i = a; j = b; k = t; }
        size_t IND = cell(c, i, j, k);
        size_t Jn[5];
        V4<real> e[5];
        for (int d = -2; d <= 2; d++) {
          Jn[d + 2] = nbr(c, i, j, k, axis, d);
          e[d + 2] = ld4(ev, Jn[d + 2]);
        }
        real u0[5];
        for (int d = 0; d < 5; d++) u0[d] = Helper<real>::gamma_real4(e[d]);
        real v_mh = 0.5f * (comp(e[1], r) + comp(e[2], r));
        real v_ph = 0.5f * (comp(e[3], r) + comp(e[2], r));
        real lam_mh = H.maxPropagationSpeed(smul<real>(0.5f, e[1] + e[2]), v_mh);
        real lam_ph = H.maxPropagationSpeed(smul<real>(0.5f, e[3] + e[2]), v_ph);
        V4<real> g = Helper<real>::minmod4(
            smul<real>(0.5f, Helper<real>::umu4(e[3]) - Helper<real>::umu4(e[1])),
            Helper<real>::minmod4(smul<real>(TH, Helper<real>::umu4(e[2]) - Helper<real>::umu4(e[1])),
                                  smul<real>(TH, Helper<real>::umu4(e[3]) - Helper<real>::umu4(e[2]))));
        if (axis == 0) g = vdiv<real>(g, (real)c.DX);
        else if (axis == 1) g = vdiv<real>(g, (real)c.DY);
        else {
          V4<real> christoffel_term = vdiv<real>(vmul<real>(V4<real>{e[2].s3, 0.0f, 0.0f, 1.0f}, u0[2]), tau);
          g = vdiv<real>(g, c.DZ * tau) + christoffel_term;
        }
        st4(ud, IND, g);
        for (int mn = 0; mn < 10; mn++) {
          real f = Helper<real>::kt1d_real(u0[0] * pi1[10 * Jn[0] + mn], u0[1] * pi1[10 * Jn[1] + mn],
                                           u0[2] * pi1[10 * Jn[2] + mn], u0[3] * pi1[10 * Jn[3] + mn],
                                           u0[4] * pi1[10 * Jn[4] + mn], v_mh, v_ph, lam_mh, lam_ph);
          real D = axis == 0 ? (real)c.DX : (axis == 1 ? (real)c.DY : tau * c.DZ);
          Src[10 * IND + mn] = Src[10 * IND + mn] - f / D;
        }
        if (SrcB) {  // bulk sector: KT flux of u0 * Pi, the eleventh component
          real f = Helper<real>::kt1d_real(u0[0] * bulk1[Jn[0]], u0[1] * bulk1[Jn[1]], u0[2] * bulk1[Jn[2]],
                                           u0[3] * bulk1[Jn[3]], u0[4] * bulk1[Jn[4]], v_mh, v_ph, lam_mh, lam_ph);
          real D = axis == 0 ? (real)c.DX : (axis == 1 ? (real)c.DY : tau * c.DZ);
          SrcB[IND] = SrcB[IND] - f / D;
        }
      }
}

// kernel_IS.cl:324-346
template <class real>
real PiPi(int lam, int mu, int nu, const real pimn[10], const real u[4]) {
  V4<real> A{pimn[idx(0, lam)], -pimn[idx(1, lam)], -pimn[idx(2, lam)], -pimn[idx(3, lam)]};
  V4<real> umu{u[0], u[1], u[2], u[3]};
  V4<real> D[4] = {gm<real>(0) - smul<real>(u[0], umu), gm<real>(1) - smul<real>(u[1], umu),
                   gm<real>(2) - smul<real>(u[2], umu), gm<real>(3) - smul<real>(u[3], umu)};
  real firstTerm = dot(D[mu], A) * dot(D[nu], A);
  V4<real> temp{dot(D[0], A), dot(D[1], A), dot(D[2], A), dot(D[3], A)};
  real secondTerm = -1.0f / 3.0f * (gmn<real>(mu, nu) - u[mu] * u[nu]) * dot(temp, A);
  return firstTerm + secondTerm;
}
// kernel_IS.cl:355-377
template <class real>
real OmegaMuNu(int mu, int nu, const real omega[6], const real u[4]) {
  V4<real> u_alpha{u[0], -u[1], -u[2], -u[3]};
  V4<real> D[4] = {V4<real>{1.0f, 0.0f, 0.0f, 0.0f} - smul<real>(u[0], u_alpha),
                   V4<real>{0.0f, 1.0f, 0.0f, 0.0f} - smul<real>(u[1], u_alpha),
                   V4<real>{0.0f, 0.0f, 1.0f, 0.0f} - smul<real>(u[2], u_alpha),
                   V4<real>{0.0f, 0.0f, 0.0f, 1.0f} - smul<real>(u[3], u_alpha)};
  V4<real> A[4] = {V4<real>{0.0f, omega[0], omega[1], omega[2]}, V4<real>{-omega[0], 0.0f, omega[3], omega[4]},
                   V4<real>{-omega[1], -omega[3], 0.0f, omega[5]}, V4<real>{-omega[2], -omega[4], -omega[5], 0.0f}};
  V4<real> temp{dot(D[nu], A[0]), dot(D[nu], A[1]), dot(D[nu], A[2]), dot(D[nu], A[3])};
  return 0.5f * dot(D[mu], temp);
}
template <class real>
V4<real> omegaB(int lam, const real om[6]) {
  if (lam == 0) return V4<real>{0.0f, om[0], om[1], om[2]};
  if (lam == 1) return V4<real>{om[0], 0.0f, om[3], om[4]};
  if (lam == 2) return V4<real>{om[1], -om[3], 0.0f, om[5]};
  if (lam == 3) return V4<real>{om[2], -om[4], -om[5], 0.0f};
  return V4<real>{0.0f, 0.0f, 0.0f, 0.0f};
}
// kernel_IS.cl:390-437
template <class real>
real pi_omega(int lam, int mu, int nu, const real pimn[10], const real omega[6], const real u[4]) {
  V4<real> A{pimn[idx(0, lam)], -pimn[idx(1, lam)], -pimn[idx(2, lam)], -pimn[idx(3, lam)]};
  V4<real> B = omegaB<real>(lam, omega);
  V4<real> umu{u[0], u[1], u[2], u[3]};
  V4<real> D[4] = {gm<real>(0) - smul<real>(u[0], umu), gm<real>(1) - smul<real>(u[1], umu),
                   gm<real>(2) - smul<real>(u[2], umu), gm<real>(3) - smul<real>(u[3], umu)};
  real firstTerm = 0.5f * (dot(D[mu], A) * dot(D[nu], B) + dot(D[mu], B) * dot(D[nu], A));
  V4<real> temp{dot(D[0], A), dot(D[1], A), dot(D[2], A), dot(D[3], A)};
  real secondTerm = -1.0f / 3.0f * (gmn<real>(mu, nu) - u[mu] * u[nu]) * dot(temp, B);
  return firstTerm + secondTerm;
}
// kernel_IS.cl:449-487
template <class real>
real omega_omega(int lam, int mu, int nu, const real omega[6], const real u[4]) {
  V4<real> B = omegaB<real>(lam, omega);
  V4<real> umu{u[0], u[1], u[2], u[3]};
  V4<real> D[4] = {gm<real>(0) - smul<real>(u[0], umu), gm<real>(1) - smul<real>(u[1], umu),
                   gm<real>(2) - smul<real>(u[2], umu), gm<real>(3) - smul<real>(u[3], umu)};
  real firstTerm = dot(D[mu], B) * dot(D[nu], B);
  V4<real> temp{dot(D[0], B), dot(D[1], B), dot(D[2], B), dot(D[3], B)};
  real secondTerm = -1.0f / 3.0f * (gmn<real>(mu, nu) - u[mu] * u[nu]) * dot(temp, B);
  return firstTerm + secondTerm;
}

// kernel_IS.cl:501-709
template <class real>
void update_pimn(const Consts& c, real* pinew, real* goodcell, const real* pi1, const real* pistep, const real* ev1,
                 const real* ev2, const real* udiff, const real* udx, const real* udy, const real* udz, real* Src,
                 real tau, int step, real* bulknew = nullptr, const real* bulk1 = nullptr,
                 const real* bulkstep = nullptr, real* SrcB = nullptr) {
  Helper<real> H(c);
  const real acu = Acu<real>::v;
  const long N = (long)ncells(c);
#pragma omp parallel for schedule(static)
  for (long I = 0; I < N; I++) {
    V4<real> e_v1 = ld4(ev1, I);
    V4<real> e_v2 = ld4(ev2, I);
    V4<real> u_old = Helper<real>::umu4(e_v1);
    V4<real> u_new = Helper<real>::umu4(e_v2);
    V4<real> udt = vdiv<real>(u_new - u_old, (real)c.DT);
    if (step == 1) {
      udt = vdiv<real>(ld4(udiff, I), (real)c.DT);
      u_new = u_old + ld4(udiff, I);
    }
    V4<real> ux = ld4(udx, I), uy = ld4(udy, I), uz = ld4(udz, I);
    V4<real> da[4] = {V4<real>{udt.s0, ux.s0, uy.s0, uz.s0}, V4<real>{udt.s1, ux.s1, uy.s1, uz.s1},
                      V4<real>{udt.s2, ux.s2, uy.s2, uz.s2}, V4<real>{udt.s3, ux.s3, uy.s3, uz.s3}};
    real DU[4], u[4];
    real ed_step = 0.0f;
    V4<real> us = (step == 1) ? u_old : u_new;
    for (int i = 0; i < 4; i++) DU[i] = dot(us, da[i]);
    u[0] = us.s0; u[1] = us.s1; u[2] = us.s2; u[3] = us.s3;
    ed_step = (step == 1) ? e_v1.s0 : e_v2.s0;
    real theta = udt.s0 + ux.s1 + uy.s2 + uz.s3;
    V4<real> cpTs = H.E.eos(ed_step);
    real temperature = cpTs.s2;
    real local_etaos = H.etaos(temperature);
    real etav = local_etaos * cpTs.s3 * CLVO_HBARC;
    real one_over_taupi = temperature / (3.0f * cl_max<real>(acu, local_etaos) * CLVO_HBARC);
    real coef_pipi = 0.0f;
    if (c.gubser_visc_test) {
      real ETAOS = c.ETAOS_YMIN;
      real etavH = ETAOS * 4.0f / 3.0f;
      real taupiH = c.LAM1 * c.LAM1 * etavH / 3.0f;
      one_over_taupi = 1.0f / (taupiH * std::pow(ed_step, (real)-0.25f));
      coef_pipi = c.LAM1 / ed_step;
      etav = ETAOS * 4.0f / 3.0f * std::pow(ed_step, (real)0.75f);
    }
    real pi2[10];
    for (int mn = 0; mn < 10; mn++) pi2[mn] = pistep[10 * I + mn];
    real Omega[6] = {0, 0, 0, 0, 0, 0};
    if (c.pimn_omega_coupling || c.omega_omega_coupling) {
      real omega[6];
      omega[0] = udt.s1 - ux.s0;
      omega[1] = udt.s2 - uy.s0;
      omega[2] = udt.s3 - uz.s0;
      omega[3] = ux.s2 - uy.s1;
      omega[4] = ux.s3 - uz.s1;
      omega[5] = uy.s3 - uz.s2;
      Omega[0] = OmegaMuNu<real>(0, 1, omega, u);
      Omega[1] = OmegaMuNu<real>(0, 2, omega, u);
      Omega[2] = OmegaMuNu<real>(0, 3, omega, u);
      Omega[3] = OmegaMuNu<real>(1, 2, omega, u);
      Omega[4] = OmegaMuNu<real>(1, 3, omega, u);
      Omega[5] = OmegaMuNu<real>(2, 3, omega, u);
    }
    real sigma;
    real max_pimn_abs = 0.0f;
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu; nu < 4; nu++) {
        sigma = dot(gm<real>(mu), da[nu]) + dot(gm<real>(nu), da[mu]) - (u[mu] * DU[nu] + u[nu] * DU[mu]) -
                2.0f / 3.0f * (gmn<real>(mu, nu) - u[mu] * u[nu]) * theta;
        int mn = idx(mu, nu);
        if (u[0] > 10000.0f) sigma = 0.0f;
        real piNS = etav * sigma;
        real pi_old = pi1[10 * I + mn] * u_old.s0;
        real src = -pi2[mn] * theta / 3.0f - pi2[mn] * u[0] / tau;
        src -= (u[mu] * pi2[idx(nu, 0)] + u[nu] * pi2[idx(mu, 0)]) * DU[0] * gmn<real>(0, 0);
        src -= (u[mu] * pi2[idx(nu, 1)] + u[nu] * pi2[idx(mu, 1)]) * DU[1] * gmn<real>(1, 1);
        src -= (u[mu] * pi2[idx(nu, 2)] + u[nu] * pi2[idx(mu, 2)]) * DU[2] * gmn<real>(2, 2);
        src -= (u[mu] * pi2[idx(nu, 3)] + u[nu] * pi2[idx(mu, 3)]) * DU[3] * gmn<real>(3, 3);
        if (c.gubser_visc_test) {
          src -= one_over_taupi * coef_pipi *
                 (PiPi<real>(0, mu, nu, pi2, u) - PiPi<real>(1, mu, nu, pi2, u) - PiPi<real>(2, mu, nu, pi2, u) -
                  PiPi<real>(3, mu, nu, pi2, u));
        }
        if (c.pimn_omega_coupling) {
          src += 2.0f * (pi_omega<real>(0, mu, nu, pi2, Omega, u) - pi_omega<real>(1, mu, nu, pi2, Omega, u) -
                         pi_omega<real>(2, mu, nu, pi2, Omega, u) - pi_omega<real>(3, mu, nu, pi2, Omega, u));
        }
        if (c.omega_omega_coupling) {
          src -= 1.0f * one_over_taupi *
                 (omega_omega<real>(0, mu, nu, Omega, u) - omega_omega<real>(1, mu, nu, Omega, u) -
                  omega_omega<real>(2, mu, nu, Omega, u) - omega_omega<real>(3, mu, nu, Omega, u));
        }
        Src[10 * I + mn] += src;
        pi_old = (pi_old + Src[10 * I + mn] * c.DT / step + c.DT * one_over_taupi * piNS) /
                 (u_new.s0 + c.DT * one_over_taupi);
        if (std::fabs(pi_old) > max_pimn_abs) max_pimn_abs = std::fabs(pi_old);
        pinew[10 * I + mn] = pi_old;
      }
    if (bulknew) {
      // Bulk sector (no counterpart in the reference): the relaxation
      // equation tau_Pi D Pi + Pi = -zeta theta - delta_PiPi Pi theta with the
      // 14-moment coefficients of Denicol, Niemi, Molnar and Rischke (PRD 85,
      // 114047 (2012)), delta_PiPi = 2/3 tau_Pi and
      // tau_Pi = zeta / (14.55 (1/3 - cs2)^2 (e + P)), written like the shear
      // update above for the conserved density u0 * Pi:
      // d(u0 Pi) + div(v u0 Pi) = Pi theta / 3 - Pi u0 / tau - (Pi - Pi_NS) / tau_Pi.
      // The shear-bulk coupling lambda_Pipi pi^{mu nu} sigma_{mu nu} is left
      // out: in dilute cells at the edge of a fireball, where |pi| >> e, it
      // drove Pi past -P and the step became unstable (so did the regulated
      // equation without the cut at ZETAOS_TMIN below).
      real local_zetaos = H.zetaos(temperature);
      real zetav = local_zetaos * cpTs.s3 * CLVO_HBARC;
      real dcs = 1.0f / 3.0f - cpTs.s0;
      real one_over_taubulk = 14.55f * dcs * dcs * temperature / (cl_max<real>(acu, local_zetaos) * CLVO_HBARC);
      real bulkNS = -zetav * theta;
      if (u[0] > 10000.0f) bulkNS = 0.0f;
      real bc = bulkstep[I];
      real srcB = bc * theta / 3.0f - bc * u[0] / tau;
      SrcB[I] += srcB;
      real b_old = bulk1[I] * u_old.s0;
      b_old = (b_old + SrcB[I] * c.DT / step + c.DT * one_over_taubulk * bulkNS) /
              (u_new.s0 + c.DT * one_over_taubulk);
      // regulators: |Pi| <= P, so that the effective pressure P + Pi stays
      // >= 0, and Pi = 0 in cells colder than ZETAOS_TMIN. In dilute cells at
      // the edge of a fireball (|pi| >> e, T far below freeze-out) the
      // relaxation equation otherwise drives Pi past -P, the T^{tau mu} ->
      // (e, v) root find has no physical solution and the step runs away.
      real pb = H.E.P(e_v2.s0);
      if (b_old < -pb) b_old = -pb;
      else if (b_old > pb) b_old = pb;
      if (temperature < c.ZETAOS_TMIN) b_old = 0.0f;
      bulknew[I] = b_old;
    }
    real pre = H.E.P(e_v2.s0);
    real T00 = (e_v2.s0 + pre) * u_new.s0 * u_new.s0 - pre;
    goodcell[I] = 1.0f;
    if (max_pimn_abs > T00) {
      for (int mn = 0; mn < 10; mn++) pinew[10 * I + mn] = 0.0f;
      if (bulknew) bulknew[I] = 0.0f;
      goodcell[I] = 0.0f;
    }
  }
}

// kernel_IS.cl:714-724
template <class real>
void get_udiff(const Consts& c, real* udiff, const real* ev0, const real* ev1) {
  const long N = (long)ncells(c);
#pragma omp parallel for schedule(static)
  for (long I = 0; I < N; I++)
    st4(udiff, I, Helper<real>::umu4(ld4(ev1, I)) - Helper<real>::umu4(ld4(ev0, I)));
}

// ========================================================= kernel_reduction.cl
// kernel_reduction.cl:7-39 with 64 groups of 256 work-items; the host takes
// the max of the 64 partials (ideal.py:257-262).
template <class real>
void reduction_stage1(const real* x, real* semi, int size) {
  const int BSZ = 256, NB = 64, G = BSZ * NB;
  for (int g = 0; g < NB; g++) {
    real xmax[BSZ];
    for (int lid = 0; lid < BSZ; lid++) {
      int gid = g * BSZ + lid;
      xmax[lid] = (real)(-3.40282346638528859812e+38F);  // -MAXFLOAT
      if (gid < size) xmax[lid] = x[4 * (size_t)gid];
      while (gid + G < size) {
        gid += G;
        real new_x = x[4 * (size_t)gid];
        if (new_x > xmax[lid]) xmax[lid] = new_x;
      }
    }
    for (int s = BSZ >> 1; s > 0; s >>= 1)
      for (int lid = 0; lid < s; lid++) xmax[lid] = (xmax[lid] > xmax[s + lid]) ? xmax[lid] : xmax[s + lid];
    semi[g] = xmax[0];
  }
}

// ========================================================== kernel_hypersf.cl
template <class real> struct Hypersf {
  const Consts& c;
  static constexpr real acu = Acu<real>::v;
  explicit Hypersf(const Consts& cc) : c(cc) {}

  static V4<real> cube(int n) {  // kernel_hypersf.cl:33-54
    return V4<real>{(real)((n >> 3) & 1), (real)(n & 1), (real)((n >> 1) & 1), (real)((n >> 2) & 1)};
  }
  struct SF { int id[4]; V4<real> center, norm; };

  static SF construct_hypersf(int id0, int id1, int id2, int id3, const V4<real>* ints, V4<real> mass_center) {  // :98-122
    SF surf;
    surf.id[0] = id0; surf.id[1] = id1; surf.id[2] = id2; surf.id[3] = id3;
    surf.center = smul<real>(0.25f, ints[id0] + ints[id1] + ints[id2] + ints[id3]);
    V4<real> vector_out = surf.center - mass_center;
    V4<real> a = ints[id1] - ints[id0];
    V4<real> b = ints[id2] - ints[id0];
    V4<real> cc = ints[id3] - ints[id0];
    V4<real> norm_vector{
        a.s1 * (b.s2 * cc.s3 - b.s3 * cc.s2) + a.s2 * (b.s3 * cc.s1 - b.s1 * cc.s3) + a.s3 * (b.s1 * cc.s2 - b.s2 * cc.s1),
        -(a.s0 * (b.s2 * cc.s3 - b.s3 * cc.s2) + a.s2 * (b.s3 * cc.s0 - b.s0 * cc.s3) + a.s3 * (b.s0 * cc.s2 - b.s2 * cc.s0)),
        a.s0 * (b.s1 * cc.s3 - b.s3 * cc.s1) + a.s1 * (b.s3 * cc.s0 - b.s0 * cc.s3) + a.s3 * (b.s0 * cc.s1 - b.s1 * cc.s0),
        -(a.s0 * (b.s1 * cc.s2 - b.s2 * cc.s1) + a.s1 * (b.s2 * cc.s0 - b.s0 * cc.s2) + a.s2 * (b.s0 * cc.s1 - b.s1 * cc.s0))};
    real projection = dot(vector_out, norm_vector);
    if (projection < 0) norm_vector = -norm_vector;
    surf.norm = norm_vector;
    return surf;
  }
  // :126-132; the int product wraps as on the device
  static real rnd(int* seed) {
    const int a = 16807;
    const int m = 2147483647;
    int prod = (int)((uint32_t)(*seed) * (uint32_t)a);
    *seed = (int)(((long long)prod) % m);
    return (*seed) / ((real)m);
  }
  static V4<real> get_mass_center(const V4<real>* ints, int n) {  // :226-232
    V4<real> center{0.0f, 0.0f, 0.0f, 0.0f};
    for (int i = 0; i < n; i++) center = center + ints[i];
    return vdiv<real>(center, (real)n);
  }
  static void tiny_move_if_coplanar(V4<real>* ints, int n, V4<real>* mass_center, int gid) {  // :135-159
    SF sf;
    int seed = (int)(32117u * (uint32_t)(gid + 1));
    for (int i = 0; i < n - 4; i++)
      for (int j = i + 1; j < n - 3; j++)
        for (int k = j + 1; k < n - 2; k++)
          for (int l = k + 1; l < n - 1; l++)
            for (int m = l + 1; m < n; m++) {
              sf = construct_hypersf(i, j, k, l, ints, *mass_center);
              if (dot(sf.norm, ints[m] - sf.center) == 0.0f) {
                for (int q = 0; q < n; q++) {
                  real r0 = rnd(&seed), r1 = rnd(&seed), r2 = rnd(&seed), r3 = rnd(&seed);
                  V4<real> tiny_shift{(r0 - 0.5f) * 1.0E-7f, (r1 - 0.5f) * 1.0E-7f, (r2 - 0.5f) * 1.0E-7f,
                                      (r3 - 0.5f) * 1.0E-7f};
                  ints[q] = ints[q] + tiny_shift;
                }
                *mass_center = get_mass_center(ints, n);
                break;
              }
            }
  }
  static bool is_on_convex_hull(const SF& sf, const V4<real>* ints, int n) {  // :163-176
    for (int q = 0; q < n; q++) {
      if (q != sf.id[0] && q != sf.id[1] && q != sf.id[2] && q != sf.id[3]) {
        V4<real> test_vector = ints[q] - sf.center;
        if (dot(test_vector, sf.norm) >= 0.0f) return false;
      }
    }
    return true;
  }
  void contribution_from(const real ed[16], int n, int i, int j, int k, V4<real>* vl, V4<real>* vh, real* elsum,
                         real* ehsum) const {  // :180-192
    int id = 8 * n + 4 * k + 2 * j + i;
    real dek = c.EFRZ - ed[id];
    real adek = std::fabs(dek);
    if (dek > 0.0f) {
      *elsum += adek;
      *vl = *vl + vmul<real>(V4<real>{(real)n, (real)i, (real)j, (real)k}, adek);
    } else {
      *ehsum += adek;
      *vh = *vh + vmul<real>(V4<real>{(real)n, (real)i, (real)j, (real)k}, adek);
    }
  }
  V4<real> energy_flow(const real ed[16]) const {  // :195-223
    V4<real> vl{0.0f, 0.0f, 0.0f, 0.0f}, vh{0.0f, 0.0f, 0.0f, 0.0f};
    real elsum = 0.0f, ehsum = 0.0f;
    for (int n = 0; n < 2; n++)
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
          for (int k = 0; k < 2; k++) contribution_from(ed, n, i, j, k, &vl, &vh, &elsum, &ehsum);
    if (std::fabs(elsum) > acu) vl = vdiv<real>(vl, elsum);
    if (std::fabs(ehsum) > acu) vh = vdiv<real>(vh, ehsum);
    return vl - vh;
  }
  static V4<real> calc_area(V4<real>* ints, V4<real> energy_flow, int n, int gid) {  // :237-266
    V4<real> mass_center = get_mass_center(ints, n);
    V4<real> area{0.0f, 0.0f, 0.0f, 0.0f};
    SF sf;
    if (n == 4) {
      sf = construct_hypersf(0, 1, 2, 3, ints, mass_center);
      if (dot(energy_flow, sf.norm) < 0.0f) sf.norm = -sf.norm;
      area = sf.norm;
    } else if (n > 4) {
      tiny_move_if_coplanar(ints, n, &mass_center, gid);
      for (int i = 0; i < n - 3; i++)
        for (int j = i + 1; j < n - 2; j++)
          for (int k = j + 1; k < n - 1; k++)
            for (int l = k + 1; l < n; l++) {
              sf = construct_hypersf(i, j, k, l, ints, mass_center);
              if (is_on_convex_hull(sf, ints, n) && dot(sf.norm, energy_flow) > 0.0f) area = area + sf.norm;
            }
    }
    return vdiv<real>(area, (real)6.0f);
  }
  void ints_between(real ed_left, real ed_right, V4<real> pos_left, V4<real> pos_right, V4<real>* all, int* n) const {
    real dE1 = c.EFRZ - ed_left;  // :269-280
    real dE2 = c.EFRZ - ed_right;
    real dE12 = ed_left - ed_right;
    if (dE1 * dE2 < 0) {
      real ratio = std::fabs(dE1) / std::fabs(dE12);
      all[*n] = smul<real>(ratio, pos_right) + smul<real>((real)(1 - ratio), pos_left);
      *n += 1;
    }
  }
  void get_all_intersections(const real ed[16], V4<real> all[32], int* n) const {  // :283-314
    *n = 0;
    for (int s = 0; s < 16; s += 4) {
      ints_between(ed[s + 0], ed[s + 1], cube(s + 0), cube(s + 1), all, n);
      ints_between(ed[s + 0], ed[s + 2], cube(s + 0), cube(s + 2), all, n);
      ints_between(ed[s + 2], ed[s + 3], cube(s + 2), cube(s + 3), all, n);
      ints_between(ed[s + 1], ed[s + 3], cube(s + 1), cube(s + 3), all, n);
    }
    for (int s = 0; s < 16; s += 8) {
      ints_between(ed[s + 0], ed[s + 4], cube(s + 0), cube(s + 4), all, n);
      ints_between(ed[s + 1], ed[s + 5], cube(s + 1), cube(s + 5), all, n);
      ints_between(ed[s + 2], ed[s + 6], cube(s + 2), cube(s + 6), all, n);
      ints_between(ed[s + 3], ed[s + 7], cube(s + 3), cube(s + 7), all, n);
    }
    for (int s = 0; s < 8; s++) ints_between(ed[s + 0], ed[s + 8], cube(s + 0), cube(s + 8), all, n);
  }
  size_t idn(int I, int J, int K) const {  // :320-325
    return cell(c, I * c.nxskip, J * c.nyskip, K * c.nzskip);
  }
  // centroid weight of cube corner q (kernel_hypersf.cl:329-348)
  static real wgt(V4<real> mc, int q) {
    real a = (q & 8) ? mc.s0 : (real)(1.0f - mc.s0);
    real b = (q & 1) ? mc.s1 : (real)(1.0f - mc.s1);
    real d = (q & 2) ? mc.s2 : (real)(1.0f - mc.s2);
    real e = (q & 4) ? mc.s3 : (real)(1.0f - mc.s3);
    return a * b * d * e;
  }
  size_t corner(int i, int j, int k, int q) const {
    return idn(i + (q & 1), j + ((q >> 1) & 1), k + ((q >> 2) & 1));
  }

  // One coarse cube; returns true and fills the outputs when it emits an
  // element. visc: NaN-centroid filter of kernel_hypersf.cl:604.
  bool cube_element(const real* ev_old, const real* ev_new, const real* pi_old, const real* pi_new, real time_old,
                    real time_new, int i, int j, int k, bool visc, real out8[8], real out4[4], real outpi[10]) const {
    if (!((i + 1) * c.nxskip < c.NX && (j + 1) * c.nyskip < c.NY && (k + 1) * c.nzskip < c.NZ)) return false;
    V4<real> ev_cube[16];
    real ed_cube[16];
    for (int q = 0; q < 8; q++) ev_cube[q] = ld4(ev_old, corner(i, j, k, q));
    for (int q = 0; q < 8; q++) ev_cube[8 + q] = ld4(ev_new, corner(i, j, k, q));
    for (int g = 0; g < 16; g++) ed_cube[g] = ev_cube[g].s0;
    if ((ed_cube[0] - c.EFRZ) * (ed_cube[15] - c.EFRZ) > 0 && (ed_cube[1] - c.EFRZ) * (ed_cube[14] - c.EFRZ) > 0 &&
        (ed_cube[2] - c.EFRZ) * (ed_cube[13] - c.EFRZ) > 0 && (ed_cube[3] - c.EFRZ) * (ed_cube[12] - c.EFRZ) > 0 &&
        (ed_cube[4] - c.EFRZ) * (ed_cube[11] - c.EFRZ) > 0 && (ed_cube[5] - c.EFRZ) * (ed_cube[10] - c.EFRZ) > 0 &&
        (ed_cube[6] - c.EFRZ) * (ed_cube[9] - c.EFRZ) > 0 && (ed_cube[7] - c.EFRZ) * (ed_cube[8] - c.EFRZ) > 0)
      return false;
    V4<real> all_ints[32];
    int nint;
    get_all_intersections(ed_cube, all_ints, &nint);
    V4<real> efv = energy_flow(ed_cube);
    V4<real> mass_center = get_mass_center(all_ints, nint);
    V4<real> dS = calc_area(all_ints, efv, nint, i * j * k);
    real dtd = time_new - time_old;
    real dxd = c.nxskip * c.DX;
    real dyd = c.nyskip * c.DY;
    real dzd = c.nzskip * c.DZ;
    real tau = time_old + mass_center.s0 * dtd;
    real x = (-c.NX) / 2 * c.DX + i * dxd + mass_center.s1 * dxd;
    real y = (-c.NY) / 2 * c.DY + j * dyd + mass_center.s2 * dyd;
    real eta = (-c.NZ) / 2 * c.DZ + k * dzd + mass_center.s3 * dzd;
    V4<real> ev{0.0f, 0.0f, 0.0f, 0.0f};
    for (int q = 0; q < 16; q++) {
      V4<real> t = smul<real>(wgt(mass_center, q), ev_cube[q]);
      ev = (q == 0) ? t : ev + t;
    }
    if (visc && std::isnan(mass_center.s0)) return false;
    out8[0] = tau * dxd * dyd * dzd * dS.s0;
    out8[1] = -tau * dtd * dyd * dzd * dS.s1;
    out8[2] = -tau * dtd * dxd * dzd * dS.s2;
    out8[3] = -dtd * dxd * dyd * dS.s3;
    out8[4] = ev.s1; out8[5] = ev.s2; out8[6] = ev.s3; out8[7] = eta;
    out4[0] = tau * std::cosh(eta); out4[1] = x; out4[2] = y; out4[3] = tau * std::sinh(eta);
    if (visc) {
      for (int mn = 0; mn < 10; mn++) {
        real acc = 0.0f;
        for (int q = 0; q < 16; q++) {
          const real* src = (q < 8) ? pi_old : pi_new;
          real t = wgt(mass_center, q) * src[corner(i, j, k, q & 7) * 10 + mn];
          acc = (q == 0) ? t : acc + t;
        }
        outpi[mn] = acc;
      }
    }
    return true;
  }

  // get_hypersf (kernel_hypersf.cl:404-496) / visc_hypersf (:501-660).
  // Elements are appended in (i, j, k) cube order. Returns the number of
  // elements (or, if it exceeds capacity, the number that would be written).
  long run(const real* ev_old, const real* ev_new, const real* pi_old, const real* pi_new, real time_old,
           real time_new, bool visc, real* sf, real* txyz, real* pisf, long capacity) const {
    const int nx = (c.NX - 1) / c.nxskip + 1, ny = (c.NY - 1) / c.nyskip + 1, nz = (c.NZ - 1) / c.nzskip + 1;
    const long ncube = (long)nx * ny * nz;
    std::vector<unsigned char> emits(ncube, 0);
    std::vector<real> b8(8 * ncube), b4(4 * ncube), bp(visc ? 10 * ncube : 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (long q = 0; q < ncube; q++) {
      int i = (int)(q / ((long)ny * nz)), j = (int)((q / nz) % ny), k = (int)(q % nz);
      emits[q] = cube_element(ev_old, ev_new, pi_old, pi_new, time_old, time_new, i, j, k, visc, &b8[8 * q],
                              &b4[4 * q], visc ? &bp[10 * q] : nullptr);
    }
    long n = 0;
    for (long q = 0; q < ncube; q++) {
      if (!emits[q]) continue;
      if (n < capacity) {
        std::memcpy(sf + 8 * n, &b8[8 * q], 8 * sizeof(real));
        std::memcpy(txyz + 4 * n, &b4[4 * q], 4 * sizeof(real));
        if (visc) std::memcpy(pisf + 10 * n, &bp[10 * q], 10 * sizeof(real));
      }
      n++;
    }
    return n;
  }
};

// ============================================================ kernel_glauber.cl
// The -D literals of glauber.py:79-90, as floats.
struct GlauberC {
  float NumOfNucleons, SQRTS, Ro0, R, Eta, Si0, ImpactParameter, Edmax, Hwn, Eta_flat, Eta_gw;
};
// kernel_glauber.cl:10-32
template <class real> real thickness(const GlauberC& g, real x, real y) {
  real r, th, f, z, cut, a[10], b[10];
  const real zk[5] = {-0.9061798f, -0.5386492f, 0.0f, 0.5386493f, 0.9061798f};
  const real Ak[5] = {0.2369269f, 0.4786287f, 0.5688889f, 0.4786287f, 0.2369269f};
  th = 0.0f;
  cut = 5.0f * g.R;
  for (int j = 0; j != 10; ++j) {
    a[j] = j * cut / 10.0f;
    b[j] = (j + 1) * cut / 10.0f;
    for (int i = 0; i != 5; ++i) {
      z = (a[j] + b[j]) / 2.0f + (b[j] - a[j]) / 2.0f * zk[i];
      r = std::sqrt(x * x + y * y + z * z);
      f = g.Ro0 / (1.0f + std::exp((r - g.R) / g.Eta));
      th = th + Ak[i] * f * (b[j] - a[j]) / 2.0f;
    }
  }
  return 2.0f * th;
}
// kernel_glauber.cl:75-83
template <class real> real Nw(const GlauberC& g, real Ta, real Tb) {
  return Ta * (1.0f - std::pow(1.0f - g.Si0 * Tb / g.NumOfNucleons, (real)g.NumOfNucleons)) +
         Tb * (1.0f - std::pow(1.0f - g.Si0 * Ta / g.NumOfNucleons, (real)g.NumOfNucleons));
}
template <class real> real Nb(const GlauberC& g, real Ta, real Tb) { return g.Si0 * Ta * Tb; }
// kernel_glauber.cl:50-52
template <class real> real ed_transverse(const GlauberC& g, real Ta, real Tb) {
  return (g.Hwn * Nw<real>(g, Ta, Tb) + (1.0f - g.Hwn) * Nb<real>(g, Ta, Tb));
}
// kernel_glauber.cl:35-47
template <class real> real weight_along_eta(const GlauberC& g, real z, real etas0_) {
  real heta;
  if (std::fabs(z - etas0_) > g.Eta_flat)
    heta = std::exp(-std::pow(std::fabs(z - etas0_) - g.Eta_flat, (real)2.0f) / (2.0f * g.Eta_gw * g.Eta_gw));
  else
    heta = 1.0f;
  return heta;
}
// kernel_glauber.cl:86-102 (etas0() returns 0)
template <class real> void glauber_ini(const Consts& c, const GlauberC& g, real* ev1) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < c.NX; i++)
    for (int j = 0; j < c.NY; j++) {
      real x = (i - c.NX / 2) * (real)c.DX;
      real y = (j - c.NY / 2) * (real)c.DY;
      real Tcent = thickness<real>(g, 0.0f, 0.0f);
      real ed_central = ed_transverse<real>(g, Tcent, Tcent);
      real kFactor = g.Edmax / ed_central;
      real b = g.ImpactParameter;
      real Ta = thickness<real>(g, x - 0.5f * b, y);
      real Tb = thickness<real>(g, x + 0.5f * b, y);
      real edxy = kFactor * ed_transverse<real>(g, Ta, Tb);
      real etas0_ = 0.0f;
      for (int k = 0; k < c.NZ; k++) {
        real etas = (k - c.NZ / 2) * (real)c.DZ;
        real heta = weight_along_eta<real>(g, etas, etas0_);
        st4(ev1, ((size_t)i * c.NY + j) * c.NZ + k, V4<real>{edxy * heta, 0.0f, 0.0f, 0.0f});
      }
    }
}
// kernel_glauber.cl:104-121
template <class real> void glauber_nbinary(const GlauberC& g, real* out, real xlow, real ylow, real dx, real dy,
                                           int nx, int ny) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) {
      real x = xlow + i * dx;
      real y = ylow + j * dy;
      real b = g.ImpactParameter;
      real Ta = thickness<real>(g, x - 0.5f * b, y);
      real Tb = thickness<real>(g, x + 0.5f * b, y);
      out[(size_t)i * ny + j] = Nb<real>(g, Ta, Tb);
    }
}

// ===================================================== CLSmoothSpec kernels
// Cooper-Frye: kernel_spec.cl:4-70 (ideal) and kernel_spec_csc.cl:4-88
// (viscous delta f, its contraction kept as written), every (y, pt, phi)
// point summed over the elements in order, in double.
template <class real, bool VISC>
void spectra(const real* sf, const real* pisf, long n, double mass_d, double gspin, double fb_d, double mu_d,
             double tfrz_d, double tcoeff_d, const real* Y, const real* Pt, const real* cphi, const real* sphi,
             int ny, int npt, int nphi, real* out) {
  const real mass = (real)mass_d, fb = (real)fb_d, muB = (real)mu_d, tfrz = (real)tfrz_d, tcoeff = (real)tcoeff_d;
  const double twopi = 2.0 * 3.14159265358979323846;
  const real dof = (real)(gspin / (twopi * twopi * twopi));
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < ny; k++)
    for (int l = 0; l < npt; l++) {
      const real rapidity = Y[k], pt = Pt[l];
      const real mt = std::sqrt(mass * mass + pt * pt);
      for (int m = 0; m < nphi; m++) {
        const real px = pt * cphi[m], py = pt * sphi[m];
        double acc = 0.0;
        for (long e = 0; e < n; e++) {
          const real* S = sf + 8 * e;
          const real vx = S[4], vy = S[5], vh = S[6];
          const real ch = std::cosh(rapidity - S[7]), sh = std::sinh(rapidity - S[7]);
          const real mtcy = mt * ch, mtsy = mt * sh;
          if (!VISC) {
            const real gamma = (real)(1.0 / std::sqrt(cl_max<double>(1.0E-30, 1.0 - vx * vx - vy * vy - vh * vh)));
            const real efkt = (gamma * (mtcy - px * S[4] - py * S[5] - mtsy * S[6]) - muB) / tfrz;
            const real volum = mtcy * S[0] - px * S[1] - py * S[2] - mtsy * S[3];
            acc += (double)(dof * volum / (std::exp(efkt) + fb));
          } else {
            const real g = (real)1.0f / std::sqrt(cl_max<real>((real)1.0E-15f, (real)(1.0f - vx * vx - vy * vy - vh * vh)));
            const real u0 = (real)1.0f * g, u1 = vx * g, u2 = vy * g, u3 = vh * g;
            const real p0 = mtcy, p1 = -pt * cphi[m], p2 = -pt * sphi[m], p3 = -mtsy;
            const real pu = p0 * u0 + p1 * u1 + p2 * u2 + p3 * u3;
            double feq = 1.0 / ((double)std::exp((real)((pu - muB) / tfrz)) + (double)fb);
            const real* pm = pisf + 10 * e;
            const real p2pi = tcoeff * (p0 * p0 * pm[0] + p3 * p3 * pm[9] + 2.0f * p0 * (p1 * pm[1] + p2 * pm[2] + p3 * pm[3]) +
                                        (p1 * p1 * pm[4] + 2 * p1 * p2 * pm[5] + p2 * p2 * pm[7]) +
                                        2.0f * p3 * (p1 * pm[3] + p2 * pm[6]));
            const double df = feq * (1.0 - (double)fb * feq) * (double)p2pi;
            feq += std::fabs(df) > feq ? (df > 0 ? 1.0 : (df < 0 ? -1.0 : 0.0)) * feq * 0.999 : df;
            const real pdsig = p0 * S[0] + p1 * S[1] + p2 * S[2] + p3 * S[3];
            acc += (double)dof * (double)pdsig * feq;
          }
        }
        out[((size_t)k * npt + l) * nphi + m] = (real)acc;
      }
    }
}

}  // namespace clvo

// ================================================================= C ABI
using clvo::Consts;
extern "C" {

#define DEF(real, sfx)                                                                                                  \
  void clvo_ideal_christoffel_##sfx(const Consts* c, real* Src, const real* ev, real tau, int step) {                 \
    clvo::ideal_christoffel<real>(*c, Src, ev, tau, step);                                                             \
  }                                                                                                                     \
  void clvo_ideal_along_##sfx(const Consts* c, int axis, real* Src, const real* ev, real tau) {                       \
    clvo::ideal_along<real>(*c, axis, Src, ev, tau);                                                                    \
  }                                                                                                                     \
  void clvo_ideal_update_ev_##sfx(const Consts* c, real* evnew, const real* ev1, const real* Src, real tau, int step) { \
    clvo::ideal_update_ev<real>(*c, evnew, ev1, Src, tau, step);                                                        \
  }                                                                                                                     \
  void clvo_visc_christoffel_##sfx(const Consts* c, real* Src, const real* ev, const real* pi, real tau, int step,   \
                                   const real* bulk) {                                                                 \
    clvo::visc_christoffel<real>(*c, Src, ev, pi, tau, step, bulk);                                                     \
  }                                                                                                                     \
  void clvo_visc_along_##sfx(const Consts* c, int axis, real* Src, const real* ev, const real* pi, real tau,         \
                             const real* bulk) {                                                                       \
    clvo::visc_along<real>(*c, axis, Src, ev, pi, tau, bulk);                                                           \
  }                                                                                                                     \
  void clvo_visc_update_ev_##sfx(const Consts* c, real* evnew, const real* ev1, const real* pi1, const real* pi2,     \
                                 const real* Src, real tau, int step, const real* bulk1, const real* bulk2) {          \
    clvo::visc_update_ev<real>(*c, evnew, ev1, pi1, pi2, Src, tau, step, bulk1, bulk2);                                 \
  }                                                                                                                     \
  void clvo_visc_initialize_##sfx(const Consts* c, real* pi1, real* goodcell, real* udiff, const real* ev, real tau,  \
                                  real* bulk1) {                                                                       \
    clvo::visc_initialize<real>(*c, pi1, goodcell, udiff, ev, tau, bulk1);                                              \
  }                                                                                                                     \
  void clvo_visc_src_christoffel_##sfx(const Consts* c, real* Src, const real* pi1, const real* ev, real tau,        \
                                       int step, real* SrcB) {                                                         \
    clvo::visc_src_christoffel<real>(*c, Src, pi1, ev, tau, step, SrcB);                                                \
  }                                                                                                                     \
  void clvo_visc_src_along_##sfx(const Consts* c, int axis, real* Src, real* ud, const real* pi1, const real* ev,     \
                                 real tau, real* SrcB, const real* bulk1) {                                            \
    clvo::visc_src_along<real>(*c, axis, Src, ud, pi1, ev, tau, SrcB, bulk1);                                           \
  }                                                                                                                     \
  void clvo_update_pimn_##sfx(const Consts* c, real* pinew, real* goodcell, const real* pi1, const real* pistep,       \
                              const real* ev1, const real* ev2, const real* udiff, const real* udx, const real* udy,   \
                              const real* udz, real* Src, real tau, int step, real* bulknew, const real* bulk1,        \
                              const real* bulkstep, real* SrcB) {                                                      \
    clvo::update_pimn<real>(*c, pinew, goodcell, pi1, pistep, ev1, ev2, udiff, udx, udy, udz, Src, tau, step, bulknew, \
                            bulk1, bulkstep, SrcB);                                                                    \
  }                                                                                                                     \
  void clvo_get_udiff_##sfx(const Consts* c, real* udiff, const real* ev0, const real* ev1) {                          \
    clvo::get_udiff<real>(*c, udiff, ev0, ev1);                                                                         \
  }                                                                                                                     \
  void clvo_reduction_stage1_##sfx(const real* x, real* semi, int size) { clvo::reduction_stage1<real>(x, semi, size); } \
  long clvo_hypersf_##sfx(const Consts* c, const real* ev_old, const real* ev_new, const real* pi_old,                 \
                          const real* pi_new, real time_old, real time_new, int visc, real* sf, real* txyz, real* pisf, \
                          long capacity) {                                                                             \
    clvo::Hypersf<real> H(*c);                                                                                          \
    return H.run(ev_old, ev_new, pi_old, pi_new, time_old, time_new, visc != 0, sf, txyz, pisf, capacity);              \
  }                                                                                                                     \
  real clvo_P_##sfx(const Consts* c, real e) { return clvo::Eos<real>(*c).P(e); }                                      \
  real clvo_T_##sfx(const Consts* c, real e) { return clvo::Eos<real>(*c).T(e); }                                      \
  real clvo_S_##sfx(const Consts* c, real e) { return clvo::Eos<real>(*c).S(e); }                                      \
  real clvo_CS2_##sfx(const Consts* c, real e) { return clvo::Eos<real>(*c).CS2(e); }                                  \
  void clvo_minmod4_##sfx(const real* a, const real* b, real* out) {                                                    \
    clvo::V4<real> r = clvo::Helper<real>::minmod4(clvo::V4<real>{a[0], a[1], a[2], a[3]},                              \
                                                   clvo::V4<real>{b[0], b[1], b[2], b[3]});                             \
    out[0] = r.s0; out[1] = r.s1; out[2] = r.s2; out[3] = r.s3;                                                         \
  }                                                                                                                     \
  real clvo_root_fixed_##sfx(const Consts* c, real T00, real M) {                                                       \
    real e; clvo::Helper<real>(*c).rootFinding(&e, T00, M); return e;                                                   \
  }                                                                                                                     \
  real clvo_root_newton_##sfx(const Consts* c, real T00, real M, int* iters) {                                          \
    real e; clvo::Helper<real>(*c).rootFinding_newton(&e, T00, M, iters); return e;                                     \
  }                                                                                                                     \
  real clvo_zetaos_##sfx(const Consts* c, real T) { return clvo::Helper<real>(*c).zetaos(T); }                          \
  void clvo_test_hypersf_##sfx(const Consts* c, real* out4) {                                                           \
    clvo::Hypersf<real> H(*c);                                                                                          \
    real ed[16]; for (int q = 0; q < 8; q++) { ed[q] = 3.0f; ed[8 + q] = 2.0f; }                                        \
    clvo::V4<real> all[32]; int n; H.get_all_intersections(ed, all, &n);                                                \
    clvo::V4<real> efv = H.energy_flow(ed);                                                                             \
    clvo::V4<real> d = clvo::Hypersf<real>::calc_area(all, efv, n, 0);                                                  \
    out4[0] = d.s0; out4[1] = d.s1; out4[2] = d.s2; out4[3] = d.s3;                                                     \
  }

DEF(float, f32)
DEF(double, f64)

#define DEFG(real, sfx)                                                                                  \
  void clvo_glauber_ini_##sfx(const Consts* c, const clvo::GlauberC* g, real* ev1) {                     \
    clvo::glauber_ini<real>(*c, *g, ev1);                                                                \
  }                                                                                                      \
  void clvo_glauber_nbinary_##sfx(const clvo::GlauberC* g, real* out, real xlow, real ylow, real dx, real dy, \
                                  int nx, int ny) {                                                     \
    clvo::glauber_nbinary<real>(*g, out, xlow, ylow, dx, dy, nx, ny);                                   \
  }                                                                                                      \
  real clvo_thickness_##sfx(const clvo::GlauberC* g, real x, real y) { return clvo::thickness<real>(*g, x, y); }
DEFG(float, f32)
DEFG(double, f64)

#define DEFS(real, sfx)                                                                                          \
  void clvo_spectra_##sfx(const real* sf, const real* pisf, long n, double mass, double gspin, double fb, double mu, \
                          double tfrz, double tcoeff, const real* Y, const real* Pt, const real* cphi,          \
                          const real* sphi, int ny, int npt, int nphi, real* out) {                             \
    if (pisf)                                                                                                    \
      clvo::spectra<real, true>(sf, pisf, n, mass, gspin, fb, mu, tfrz, tcoeff, Y, Pt, cphi, sphi, ny, npt, nphi, out); \
    else                                                                                                         \
      clvo::spectra<real, false>(sf, pisf, n, mass, gspin, fb, mu, tfrz, tcoeff, Y, Pt, cphi, sphi, ny, npt, nphi, out); \
  }
DEFS(float, f32)
DEFS(double, f64)

int clvo_abi_version(void) { return 2; }
}
