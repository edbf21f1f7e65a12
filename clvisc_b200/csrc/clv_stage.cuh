// Fused Runge-Kutta stage kernels of the CLVisc hydro step.
//
// One thread owns one cell and produces, in a single pass over HBM, what the
// reference computes with ten separate launches per stage
// (visc.py:232-314): the Christoffel sources, the three directional
// Kurganov-Tadmor flux differences of T^{tau mu} (kernel_visc.cl:68-318) and
// of u0*pi^{mu nu} (kernel_IS.cl:74-318) with the minmod-limited velocity
// gradients, the implicit Israel-Stewart update (kernel_IS.cl:501-709) and
// the T^{tau mu} -> (e, v) root find (kernel_visc.cl:322-393). The ideal
// variant covers kernel_ideal.cl.
//
// Fields are structure-of-arrays planes of Params::ld elements in the
// reference's cell order I = i*NY*NZ + j*NZ + k. A face flux is evaluated from
// the two cells that share the face, so the value at face i+1/2 is the same
// for cells i and i+1, as in the reference.
#pragma once
#include "clv_device.cuh"

namespace clv {

template <class real> struct ViscBuffers {
  const real* ev_st;   // 4 planes: d_ev[step], stencil input
  const real* pi_st;   // 10 planes (11 with the bulk sector: plane 10 is Pi): d_pi[step], stencil input
  const real* ev1;     // 4 planes: d_ev[1]
  const real* ev2e;    // plane 0 of d_ev[2] (read at stage 1)
  const real* pi1;     // 10 planes: d_pi[1], start point of the pi update
  const real* pin;     // 10 planes: pi at the start of the step (update_ev base)
  const real* pi2in;   // 10 planes: new pi, read when the pi update is not fused
  real* evnew;         // 4 planes
  real* pinew;         // 10 planes
  real* src;           // 14 planes: KT sources 0..3, IS sources 4..13 (14: bulk source)
  real* udiff;         // 4 planes
  uint8_t* goodcell;   // 1 byte per cell
  typename KeyT<real>::type* edmax_key;  // optional max of evnew energy density
  int write_src;       // keep the accumulated sources for the next stage
  int write_udiff;     // udiff = u(evnew) - u(ev1) (fused second stage)
};

template <class real> struct IdealBuffers {
  const real* ev_st;  // d_ev[step]
  const real* ev1;    // d_ev[1]
  real* evnew;        // d_ev[3-step]
  real* src;          // 4 planes
  typename KeyT<real>::type* edmax_key;
  int write_src;
};

// neighbour offsets along one axis, clamped at the edges: the reference's
// two ghost cells repeat the edge cell (kernel_ideal.cl:166-172)
struct Stencil {
  long long off[5];
};
// Grid of one event: sizes and plane stride (the single-event kernels take
// them from Params, the batch kernel from its event table).
struct GridDims {
  int nx, ny, nz;
  long long ld;
};
// Values of one cell that the Christoffel terms, the pi update and update_ev
// share, each evaluated once: the stage input ev (d_ev[step]) and d_ev[1] at
// the cell, with their gamma and table pressure P(e) (no bulk part).
template <class real> struct CellIn {
  real e0[4], g0, p0;
  real e1[4], g1, p1;
};

inline namespace CLV_ARITH {
__device__ __forceinline__ Stencil make_stencil(int q, int L, long long stride) {
  Stencil s;
#pragma unroll
  for (int d = -2; d <= 2; d++) {
    int qq = min(max(q + d, 0), L - 1);
    s.off[d + 2] = (long long)(qq - q) * stride;
  }
  return s;
}

// e0, g0 and p0 set: fills e1, g1, p1. At stage 1 the stencil input is d_ev[1]
// itself (same buffer), so its values are e0's; otherwise they are read.
template <class real>
__device__ __forceinline__ void cell_in_ev1(const Params& p, const ViscBuffers<real>& b, long long I, long long ld,
                                            CellIn<real>& c) {
  if (b.ev1 == b.ev_st) {
#pragma unroll
    for (int q = 0; q < 4; q++) c.e1[q] = c.e0[q];
    c.g1 = c.g0;
    c.p1 = c.p0;
  } else {
#pragma unroll
    for (int q = 0; q < 4; q++) c.e1[q] = b.ev1[q * ld + I];
    c.g1 = gamma3<real>(c.e1[1], c.e1[2], c.e1[3]);
    c.p1 = eosP<real>(p, c.e1[0]);
  }
}

// update_pimn (kernel_IS.cl:501-709) for cell I: c holds the stage input ev
// and d_ev[1] at the cell, pc the stage input pi, grad the velocity gradients,
// S10 the IS sources (updated in place); writes pi_new and goodcell, returns
// the new pi in pinew. With BULK, component 10 of pc, S10 and pinew is the
// bulk pressure Pi.
template <class real, bool COUPLED, bool BULK>
__device__ __forceinline__ void pi_update(const Params& p, const ViscBuffers<real>& b, int step,
                                          const TauConst<real>& tc, long long I, long long ld, const CellIn<real>& cin,
                                          const real pc[11], const real grad[3][4], real S10[11], real pinew[11]) {
  const real acu = Acu<real>::v;
  const real tau = tc.tau;
  const Recips<real>& rc = recips<real>(p);
  const real* e0 = cin.e0;
  const real* e1 = cin.e1;
  real g1 = cin.g1;
  real u_old[4] = {g1 * 1.0f, g1 * e1[1], g1 * e1[2], g1 * e1[3]};
  real u_new[4], udt[4];
  real e2s0;
  if (step == 1) {
#pragma unroll
    for (int c = 0; c < 4; c++) {
      real ud = b.udiff[c * ld + I];
      udt[c] = div_by<real>(ud, (real)p.DT, rc.DT);
      u_new[c] = u_old[c] + ud;
    }
    e2s0 = b.ev2e[I];
  } else {
    real g2 = cin.g0;
    u_new[0] = g2 * 1.0f;
    u_new[1] = g2 * e0[1];
    u_new[2] = g2 * e0[2];
    u_new[3] = g2 * e0[3];
#pragma unroll
    for (int c = 0; c < 4; c++) udt[c] = div_by<real>(u_new[c] - u_old[c], (real)p.DT, rc.DT);
    e2s0 = e0[0];
  }
  real da[4][4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    da[c][0] = udt[c];
    da[c][1] = grad[0][c];
    da[c][2] = grad[1][c];
    da[c][3] = grad[2][c];
  }
  real u[4], DU[4];
#pragma unroll
  for (int c = 0; c < 4; c++) u[c] = (step == 1) ? u_old[c] : u_new[c];
#pragma unroll
  for (int c = 0; c < 4; c++) DU[c] = dot4<real>(u, da[c]);
  real ed_step = (step == 1) ? e1[0] : e2s0;
  real theta = udt[0] + grad[0][1] + grad[1][2] + grad[2][3];
  real tex[4];  // cs2, P, T, s at ed_step
  eos_texel4<real>(p, ed_step, tex);
  real temperature = tex[2];
  real sdens = tex[3];
  real local_etaos = etaos<real>(p, temperature);
  real etav = local_etaos * sdens * CLV_HBARC;
  real one_over_taupi = temperature / (3.0f * cmax<real>(acu, local_etaos) * CLV_HBARC);
  real coef_pipi = 0.0f;
  if (COUPLED && (p.flags & FLAG_GUBSER_VISC)) {  // kernel_IS.cl:581-590
    real ETAOS = p.ETAOS_YMIN;
    real etavH = ETAOS * 4.0f / 3.0f;
    real taupiH = p.LAM1 * p.LAM1 * etavH / 3.0f;
    one_over_taupi = 1.0f / (taupiH * pow(ed_step, (real)-0.25f));
    coef_pipi = p.LAM1 / ed_step;
    etav = ETAOS * 4.0f / 3.0f * pow(ed_step, (real)0.75f);
  }
  real Omega[6] = {0, 0, 0, 0, 0, 0};
  if (COUPLED && (p.flags & (FLAG_PIMN_OMEGA | FLAG_OMEGA_OMEGA))) omega_tensor<real>(udt, grad, u, Omega);

  // the implicit update's denominator, shared by the ten components
  const real den = u_new[0] + p.DT * one_over_taupi;
  const real rden = (real)1.0f / den;
  real max_pimn_abs = 0.0f;
#if CLV_FAST
  // tolerance build: the transversality terms of every component,
  // (u^mu pi^{nu lam} + u^nu pi^{mu lam}) Du_lam, from the lowered vector
  // W^mu = pi^{mu lam} g_{lam lam} Du^lam, formed once
  real Wv[4];
#pragma unroll
  for (int q = 0; q < 4; q++)
    Wv[q] = pc[pidx(q, 0)] * DU[0] - pc[pidx(q, 1)] * DU[1] - pc[pidx(q, 2)] * DU[2] - pc[pidx(q, 3)] * DU[3];
  const real r3 = (real)1.0f / 3.0f;
#endif
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
#pragma unroll
    for (int nu = mu; nu < 4; nu++) {
      real gmu[4] = {gmn<real>(mu, 0), gmn<real>(mu, 1), gmn<real>(mu, 2), gmn<real>(mu, 3)};
      real gnu[4] = {gmn<real>(nu, 0), gmn<real>(nu, 1), gmn<real>(nu, 2), gmn<real>(nu, 3)};
      real sigma = dot4<real>(gmu, da[nu]) + dot4<real>(gnu, da[mu]) - (u[mu] * DU[nu] + u[nu] * DU[mu]) -
                   2.0f / 3.0f * (gmn<real>(mu, nu) - u[mu] * u[nu]) * theta;
      const int mn = pidx(mu, nu);
      if (u[0] > 10000.0f) sigma = 0.0f;
      real piNS = etav * sigma;
      real pi_old = b.pi1[mn * ld + I] * u_old[0];
#if CLV_FAST
      real src = -pc[mn] * (theta * r3 + u[0] * tc.rtau) - (u[mu] * Wv[nu] + u[nu] * Wv[mu]);
#else
      real src = div_by<real>(-pc[mn] * theta, (real)3.0f, rc.three) - div_by<real>(pc[mn] * u[0], tau, tc.rtau);
      src -= (u[mu] * pc[pidx(nu, 0)] + u[nu] * pc[pidx(mu, 0)]) * DU[0] * gmn<real>(0, 0);
      src -= (u[mu] * pc[pidx(nu, 1)] + u[nu] * pc[pidx(mu, 1)]) * DU[1] * gmn<real>(1, 1);
      src -= (u[mu] * pc[pidx(nu, 2)] + u[nu] * pc[pidx(mu, 2)]) * DU[2] * gmn<real>(2, 2);
      src -= (u[mu] * pc[pidx(nu, 3)] + u[nu] * pc[pidx(mu, 3)]) * DU[3] * gmn<real>(3, 3);
#endif
      if (COUPLED && (p.flags & FLAG_GUBSER_VISC))
        src -= one_over_taupi * coef_pipi *
               (pipi<real>(0, mu, nu, pc, u) - pipi<real>(1, mu, nu, pc, u) - pipi<real>(2, mu, nu, pc, u) -
                pipi<real>(3, mu, nu, pc, u));
      if (COUPLED && (p.flags & FLAG_PIMN_OMEGA))
        src += 2.0f * (pi_omega<real>(0, mu, nu, pc, Omega, u) - pi_omega<real>(1, mu, nu, pc, Omega, u) -
                       pi_omega<real>(2, mu, nu, pc, Omega, u) - pi_omega<real>(3, mu, nu, pc, Omega, u));
      if (COUPLED && (p.flags & FLAG_OMEGA_OMEGA))
        src -= 1.0f * one_over_taupi *
               (omega_omega<real>(0, mu, nu, Omega, u) - omega_omega<real>(1, mu, nu, Omega, u) -
                omega_omega<real>(2, mu, nu, Omega, u) - omega_omega<real>(3, mu, nu, Omega, u));
      S10[mn] += src;
      pi_old = div_by<real>(pi_old + div_step(S10[mn] * p.DT, step) + p.DT * one_over_taupi * piNS, den, rden);
      if (fabs(pi_old) > max_pimn_abs) max_pimn_abs = fabs(pi_old);
      pinew[mn] = pi_old;
    }
  if (BULK) {
    // Bulk sector (no counterpart in the reference): the relaxation equation
    // tau_Pi D Pi + Pi = -zeta theta - 2/3 tau_Pi Pi theta with the 14-moment
    // tau_Pi = zeta / (14.55 (1/3 - cs2)^2 (e + P)) of Denicol, Niemi, Molnar
    // and Rischke (PRD 85, 114047 (2012)), for the density u0 Pi with the same
    // implicit relaxation step as the shear components. No shear-bulk
    // coupling; |Pi| <= P and Pi = 0 below ZETAOS_TMIN, which keep dilute
    // cells at the edge of a fireball (|pi| >> e, far below freeze-out) from
    // running away.
    real cs2 = tex[0];
    real local_zetaos = zetaos<real>(p, temperature);
    real zetav = local_zetaos * sdens * CLV_HBARC;
    real dcs = 1.0f / 3.0f - cs2;
    real one_over_taubulk = 14.55f * dcs * dcs * temperature / (cmax<real>(acu, local_zetaos) * CLV_HBARC);
    real bulkNS = -zetav * theta;
    if (u[0] > 10000.0f) bulkNS = 0.0f;
    real bc = pc[10];
    real srcB = div_by<real>(bc * theta, (real)3.0f, rc.three) - div_by<real>(bc * u[0], tau, tc.rtau);
    S10[10] += srcB;
    real b_old = b.pi1[10 * ld + I] * u_old[0];
    b_old = (b_old + div_step(S10[10] * p.DT, step) + p.DT * one_over_taubulk * bulkNS) /
            (u_new[0] + p.DT * one_over_taubulk);
    const real pb = (step == 1) ? eosP<real>(p, e2s0) : cin.p0;
    if (b_old < -pb) b_old = -pb;
    else if (b_old > pb) b_old = pb;
    if (temperature < p.ZETAOS_TMIN) b_old = 0.0f;
    pinew[10] = b_old;
  }
  real pre = (step == 1) ? eosP<real>(p, e2s0) : cin.p0;  // stage 2: e2s0 is e0[0]
  real T00 = (e2s0 + pre) * u_new[0] * u_new[0] - pre;
  uint8_t good = 1;
  constexpr int NPI = BULK ? 11 : 10;
  if (max_pimn_abs > T00) {
#pragma unroll
    for (int m = 0; m < NPI; m++) pinew[m] = 0.0f;
    good = 0;
  }
#pragma unroll
  for (int m = 0; m < NPI; m++) b.pinew[m * ld + I] = pinew[m];
  b.goodcell[I] = good;
}

// update_ev (kernel_visc.cl:322-393) for cell I: cin holds d_ev[1] at the
// cell, pin = pi^{tau mu} at the start of the step, S4 the KT sources; the new
// pi^{tau mu} comes from pinew (fused pi update) or from pi_new_in. Also
// get_udiff and the edmax key. With BULK, pin[4] is Pi at the start of the
// step and the pressure of the old and the new state is P(e) + Pi.
template <class real, bool FUSED_PI, bool BULK>
__device__ __forceinline__ void ev_update(const Params& p, const ViscBuffers<real>& b, int step,
                                          const TauConst<real>& tc, long long I, long long ld, const CellIn<real>& cin,
                                          const real pin[5], const real S4[4], const real pinew[11]) {
  const real acu = Acu<real>::v;
  const real tau = tc.tau;
  const real* e1 = cin.e1;
  real ed = e1[0], vx = e1[1], vy = e1[2], vz = e1[3];
  real pressure = cin.p1;
  if (BULK) pressure = pressure + pin[4];
  real u0 = cin.g1;
  real umu[4] = {u0 * 1.0f, u0 * vx, u0 * vy, u0 * vz};
  real old_time = tau - (step - 1) * p.DT;
  real T0m[4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    real g0 = c == 0 ? (real)1.0f : (real)0.0f;
    T0m[c] = ((ed + pressure) * u0 * umu[c] - pressure * g0 + pin[c]) * old_time;
  }
  real bnew = 0.0f;
  if (BULK) bnew = FUSED_PI ? pinew[10] : b.pi2in[10 * ld + I];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    real pim2 = FUSED_PI ? pinew[c] : b.pi2in[c * ld + I];
    T0m[c] = T0m[c] + div_step(S4[c] * p.DT, step) - pim2 * tau;
  }
  real T00 = div_by<real>(cmax<real>(acu, T0m[0]), tau, tc.rtau);
  real T01 = (fabs(T0m[1]) < acu) ? (real)0.0f : div_by<real>(T0m[1], tau, tc.rtau);
  real T02 = (fabs(T0m[2]) < acu) ? (real)0.0f : div_by<real>(T0m[2], tau, tc.rtau);
  real T03 = (fabs(T0m[3]) < acu) ? (real)0.0f : div_by<real>(T0m[3], tau, tc.rtau);
  real M = sqrt(T01 * T01 + T02 * T02 + T03 * T03);
  real SCALE_COEF = 0.999f;
  if (M > T00) {
    T01 *= SCALE_COEF * T00 / M;
    T02 *= SCALE_COEF * T00 / M;
    T03 *= SCALE_COEF * T00 / M;
    M = SCALE_COEF * T00;
  }
  // tolerance build, FP32: Newton from the cell's speed at the start of the
  // step, which is near the root, instead of from 1/2 (fewer EOS lookups).
  // The finder stops at a step below 1e-5, so where it ends depends on where
  // it starts: about 1e-9 of the energy density, inside the FP32 tolerance
  // but not the FP64 one, which keeps the reference's start.
  real v_start = -1.0f;
#if CLV_FAST
  if constexpr (sizeof(real) == 4) v_start = fmin(sqrt(vx * vx + vy * vy + vz * vz), (real)0.999f);
#endif
  real ed_find = root_newton<real, BULK>(p, T00, M, bnew, v_start);
  if (ed_find < acu) {
    T01 = 0.0f;
    T02 = 0.0f;
    T03 = 0.0f;
  }
  ed_find = cmax<real>(0.0f, ed_find);
  real pr = eosP<real>(p, ed_find);
  if (BULK) pr = pr + bnew;
  real epv = cmax<real>(acu, T00 + pr);
  const real repv = (real)1.0f / epv;
  real en[4] = {ed_find, div_by<real>(T01, epv, repv), div_by<real>(T02, epv, repv), div_by<real>(T03, epv, repv)};
#pragma unroll
  for (int c = 0; c < 4; c++) b.evnew[c * ld + I] = en[c];
  if (b.write_udiff) {  // get_udiff, kernel_IS.cl:714-724
    real gn = gamma3<real>(en[1], en[2], en[3]);
    real go = cin.g1;
    b.udiff[0 * ld + I] = gn * 1.0f - go * 1.0f;
    b.udiff[1 * ld + I] = gn * en[1] - go * e1[1];
    b.udiff[2 * ld + I] = gn * en[2] - go * e1[2];
    b.udiff[3 * ld + I] = gn * en[3] - go * e1[3];
  }
  if (b.edmax_key) key_max<real>(b.edmax_key, en[0]);
}

// --------------------------------------------------------------- viscous

// One cell of the fused viscous stage. With BULK the pi fields carry an
// eleventh plane, the bulk pressure Pi, and the sources an eleventh IS term.
template <class real, bool DO_IS, bool DO_KT, bool COUPLED, bool BULK>
__device__ __forceinline__ void visc_stage_cell(const Params& p, const GridDims gd, const ViscBuffers<real>& b,
                                                int step, const TauConst<real>& tc, long long I) {
  const real tau = tc.tau;
  const Recips<real>& rc = recips<real>(p);
  constexpr int NPI = BULK ? 11 : 10;
  const long long ld = gd.ld;
  const int k = (int)(I % gd.nz);
  const long long t = I / gd.nz;
  const int j = (int)(t % gd.ny);
  const int i = (int)(t / gd.ny);
  const real acu = Acu<real>::v;

  // centre cell of the stage input
  CellIn<real> cin;
  real* e0 = cin.e0;
#pragma unroll
  for (int c = 0; c < 4; c++) e0[c] = b.ev_st[c * ld + I];
  cin.g0 = gamma3<real>(e0[1], e0[2], e0[3]);
  cin.p0 = eosP<real>(p, e0[0]);
  real pc[11];
#pragma unroll
  for (int m = 0; m < NPI; m++) pc[m] = b.pi_st[m * ld + I];
  if (!BULK) pc[10] = 0.0f;
  // pi at the start of the step: read before this thread's pi_new store,
  // which may alias it (in-place second stage)
  real pin[5];
#pragma unroll
  for (int c = 0; c < 4; c++) pin[c] = DO_KT ? b.pin[c * ld + I] : (real)0.0f;
  pin[4] = (BULK && DO_KT) ? b.pin[10 * ld + I] : (real)0.0f;

  real S4[4], S10[11];
  if (step == 1) {
#pragma unroll
    for (int c = 0; c < 4; c++) S4[c] = 0.0f;
#pragma unroll
    for (int m = 0; m < 11; m++) S10[m] = 0.0f;
  } else {
#pragma unroll
    for (int c = 0; c < 4; c++) S4[c] = DO_KT ? b.src[c * ld + I] : (real)0.0f;
#pragma unroll
    for (int m = 0; m < NPI; m++) S10[m] = DO_IS ? b.src[(4 + m) * ld + I] : (real)0.0f;
    if (!BULK) S10[10] = 0.0f;
  }

  // Christoffel terms
  if (DO_IS) {  // kernel_IS.cl:56-65
    real uz = e0[3] * cin.g0;
    S10[0] -= div_by<real>(2.0f * uz * pc[pidx(0, 3)], tau, tc.rtau);
    S10[1] -= div_by<real>(uz * pc[pidx(1, 3)], tau, tc.rtau);
    S10[2] -= div_by<real>(uz * pc[pidx(2, 3)], tau, tc.rtau);
    S10[3] -= div_by<real>(uz * (pc[pidx(0, 0)] + pc[pidx(3, 3)]), tau, tc.rtau);
    S10[6] -= div_by<real>(uz * pc[pidx(0, 1)], tau, tc.rtau);
    S10[8] -= div_by<real>(uz * pc[pidx(0, 2)], tau, tc.rtau);
    S10[9] -= div_by<real>(2.0f * uz * pc[pidx(0, 3)], tau, tc.rtau);
  }
  if (DO_KT) {  // kernel_visc.cl:24-50
    real ed = e0[0], vx = e0[1], vy = e0[2], vz = e0[3];
    real u0 = cin.g0;
    real bulkpi = BULK ? pc[10] : (real)0.0f;  // fills the reference's placeholder, kernel_visc.cl:31-33
    real pressure = cin.p0 + bulkpi;
    real Tzz_tilde = (ed + pressure) * u0 * u0 * vz * vz + pressure + pc[pidx(3, 3)];
    real Ttz_tilde = (ed + pressure) * u0 * u0 * vz + pc[pidx(0, 3)];
    S4[0] = S4[0] - Tzz_tilde;
    S4[1] = S4[1] - (real)0.0f;
    S4[2] = S4[2] - (real)0.0f;
    S4[3] = S4[3] - Ttz_tilde;
    if (p.flags & FLAG_RIEMANN) {
      real Ttt_tilde = (ed + pressure) * u0 * u0 - pressure;
      real Ttx_tilde = (ed + pressure) * u0 * u0 * vx;
      real Tty_tilde = (ed + pressure) * u0 * u0 * vy;
      S4[0] = S4[0] + (Tzz_tilde + Ttt_tilde);
      S4[1] = S4[1] + Ttx_tilde;
      S4[2] = S4[2] + Tty_tilde;
      S4[3] = S4[3] + 3.0f * Ttz_tilde;
    }
  }

  real grad[3][4];  // d_udx, d_udy, d_udz of kernel_IS.cl

#pragma unroll 1
  for (int a = 0; a < 3; a++) {
    const int q = a == 0 ? i : (a == 1 ? j : k);
    const int L = a == 0 ? gd.nx : (a == 1 ? gd.ny : gd.nz);
    if (L == 1) {
      // One cell along this axis (a (2+1)D event along eta): the five stencil
      // cells are this cell, so both face fluxes are the same value and their
      // difference is +0, which leaves every source unchanged, and the limited
      // velocity difference is +0. Only the Christoffel part of the eta
      // gradient remains. For a finite state this gives the bits of the full
      // evaluation; a non-finite state already turns the x or y terms to NaN.
      if (DO_IS) {
#pragma unroll
        for (int c = 0; c < 4; c++) grad[a][c] = 0.0f;
        if (a == 2) {
          const real u0c = cin.g0;
          grad[2][0] = grad[2][0] + div_by<real>(e0[3] * u0c, tau, tc.rtau);
          grad[2][1] = grad[2][1] + div_by<real>((real)0.0f * u0c, tau, tc.rtau);
          grad[2][2] = grad[2][2] + div_by<real>((real)0.0f * u0c, tau, tc.rtau);
          grad[2][3] = grad[2][3] + div_by<real>((real)1.0f * u0c, tau, tc.rtau);
        }
      }
      continue;
    }
    const long long stride = a == 0 ? (long long)gd.ny * gd.nz : (a == 1 ? (long long)gd.nz : 1ll);
    const Stencil st = make_stencil(q, L, stride);
    const real D = a == 0 ? (real)p.DX : (a == 1 ? (real)p.DY : tc.dzt);
    const real rD = a == 0 ? rc.DX : (a == 1 ? rc.DY : tc.rdzt);

    real E[5][4];
#pragma unroll
    for (int d = 0; d < 5; d++)
#pragma unroll
      for (int c = 0; c < 4; c++) E[d][c] = (d == 2) ? e0[c] : b.ev_st[c * ld + I + st.off[d]];
    real u0[5];
#pragma unroll
    for (int d = 0; d < 5; d++) u0[d] = (d == 2) ? cin.g0 : gamma3<real>(E[d][1], E[d][2], E[d][3]);

    // face (i-1/2) uses cells 1,2 and face (i+1/2) cells 2,3 of the stencil
    real vh[2], lam[2];
#pragma unroll
    for (int f = 0; f < 2; f++) {
      const int l = 1 + f, r = 2 + f;
      real h[4];
#pragma unroll
      for (int c = 0; c < 4; c++) h[c] = 0.5f * (E[l][c] + E[r][c]);
      vh[f] = h[a + 1];
      lam[f] = max_speed<real>(p, h[0], h[1], h[2], h[3], vh[f]);
    }

    if (DO_KT) {  // kt1d_visc, kernel_visc.cl:68-127
      real pr[5], Q[5][4];
#pragma unroll
      for (int d = 0; d < 5; d++) {
        const long long J = I + st.off[d];
        pr[d] = (d == 2) ? cin.p0 : eosP<real>(p, E[d][0]);
        if (BULK) pr[d] = pr[d] + ((d == 2) ? pc[10] : b.pi_st[10 * ld + J]);
        real A = (E[d][0] + pr[d]) * u0[d];
        real u4[4] = {(real)1.0f * u0[d], E[d][1] * u0[d], E[d][2] * u0[d], E[d][3] * u0[d]};
#pragma unroll
        for (int c = 0; c < 4; c++) {
          real g0 = c == 0 ? (real)1.0f : (real)0.0f;
          real T0m = A * u4[c] - g0 * pr[d];
          real pim0 = (d == 2) ? pc[c] : b.pi_st[c * ld + J];
          Q[d][c] = tau * (T0m + pim0);
        }
      }
      // limited slopes at stencil cells 1, 2, 3 (each face uses two of them)
      real DA[3][4];
#pragma unroll
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int c = 0; c < 4; c++) DA[d][c] = slope<real>(Q[d][c], Q[d + 1][c], Q[d + 2][c]);
      real F[2][4];
#pragma unroll
      for (int f = 0; f < 2; f++) {
        const int l = 1 + f, r = 2 + f;
        const long long Jl = I + st.off[l], Jr = I + st.off[r];
        real pr_half = 0.5f * (pr[l] + pr[r]);
        real pt = pr_half * tau;
#pragma unroll
        for (int c = 0; c < 4; c++) {
          real DAl = DA[l - 1][c];
          real DAr = DA[r - 1][c];
          real AL = Q[l][c] + 0.5f * DAl;
          real AR = Q[r][c] - 0.5f * DAr;
          real p0l = (l == 2) ? pc[c] : b.pi_st[c * ld + Jl];
          real p0r = (r == 2) ? pc[c] : b.pi_st[c * ld + Jr];
          const int mi = pidx(a + 1, c);
          real pil = (l == 2) ? pc[mi] : b.pi_st[mi * ld + Jl];
          real pir = (r == 2) ? pc[mi] : b.pi_st[mi * ld + Jr];
          real pim0_half = 0.5f * (p0l + p0r);
          real pimi_half = 0.5f * (pil + pir);
          real g0 = c == 0 ? (real)1.0f : (real)0.0f;
          real ga = c == a + 1 ? (real)-1.0f : (real)0.0f;
          real Jp = (AR + pt * g0 - tau * pim0_half) * vh[f] - pt * ga + tau * pimi_half;
          real Jm = (AL + pt * g0 - tau * pim0_half) * vh[f] - pt * ga + tau * pimi_half;
          F[f][c] = 0.5f * (Jp + Jm) - 0.5f * lam[f] * (AR - AL);
        }
      }
#pragma unroll
      for (int c = 0; c < 4; c++) {
        real src = F[1][c];
        src -= F[0][c];
        S4[c] = S4[c] - div_by<real>(src, D, rD);
      }
    }

    if (DO_IS) {
      // velocity gradient, kernel_IS.cl:134-137 / 217-220 / 299-304
      real um[3][4];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        um[d][0] = u0[d + 1] * 1.0f;
        um[d][1] = u0[d + 1] * E[d + 1][1];
        um[d][2] = u0[d + 1] * E[d + 1][2];
        um[d][3] = u0[d + 1] * E[d + 1][3];
      }
#pragma unroll
      for (int c = 0; c < 4; c++) grad[a][c] = div_by<real>(grad_limit<real>(um[0][c], um[1][c], um[2][c]), D, rD);
      if (a == 2) {
        grad[2][0] = grad[2][0] + div_by<real>(E[2][3] * u0[2], tau, tc.rtau);
        grad[2][1] = grad[2][1] + div_by<real>((real)0.0f * u0[2], tau, tc.rtau);
        grad[2][2] = grad[2][2] + div_by<real>((real)0.0f * u0[2], tau, tc.rtau);
        grad[2][3] = grad[2][3] + div_by<real>((real)1.0f * u0[2], tau, tc.rtau);
      }
      // KT flux of u0*pi^{mn}, kt1d_real (helper.h:249-285); with BULK also of u0*Pi
#pragma unroll 2
      for (int m = 0; m < NPI; m++) {
        real U[5];
#pragma unroll
        for (int d = 0; d < 5; d++) U[d] = u0[d] * ((d == 2) ? pc[m] : b.pi_st[m * ld + I + st.off[d]]);
        real DU[3];
#pragma unroll
        for (int d = 0; d < 3; d++) DU[d] = slope<real>(U[d], U[d + 1], U[d + 2]);
        real Fm[2];
#pragma unroll
        for (int f = 0; f < 2; f++) {
          const int l = 1 + f, r = 2 + f;
          real DAl = DU[l - 1];
          real DAr = DU[r - 1];
          real AL = U[l] + 0.5f * DAl;
          real AR = U[r] - 0.5f * DAr;
          real Jp = AR * vh[f];
          real Jm = AL * vh[f];
          Fm[f] = 0.5f * (Jp + Jm) - 0.5f * lam[f] * (AR - AL);
        }
        real src = Fm[1];
        src -= Fm[0];
        S10[m] = S10[m] - div_by<real>(src, D, rD);
      }
    }
  }

  real pinew[11];
  cell_in_ev1<real>(p, b, I, ld, cin);
  if (DO_IS) pi_update<real, COUPLED, BULK>(p, b, step, tc, I, ld, cin, pc, grad, S10, pinew);
  if (DO_KT) ev_update<real, DO_IS, BULK>(p, b, step, tc, I, ld, cin, pin, S4, pinew);

  if (b.write_src) {
    if (DO_KT)
#pragma unroll
      for (int c = 0; c < 4; c++) b.src[c * ld + I] = S4[c];
    if (DO_IS)
#pragma unroll
      for (int m = 0; m < NPI; m++) b.src[(4 + m) * ld + I] = S10[m];
  }
}

template <class real, bool DO_IS, bool DO_KT, bool COUPLED, bool BULK>
__global__ void __launch_bounds__(128) visc_stage_kernel(Params p, ViscBuffers<real> b, int step, TauConst<real> tc) {
  const long long N = (long long)p.nx * p.ny * p.nz;
  const long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= N) return;
  visc_stage_cell<real, DO_IS, DO_KT, COUPLED, BULK>(p, GridDims{p.nx, p.ny, p.nz, p.ld}, b, step, tc, I);
}

// ----------------------------------------------------------------- ideal
template <class real>
__global__ void __launch_bounds__(128) ideal_stage_kernel(Params p, IdealBuffers<real> b, int step, TauConst<real> tc) {
  const real tau = tc.tau;
  const Recips<real>& rc = recips<real>(p);
  const long long N = (long long)p.nx * p.ny * p.nz;
  const long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= N) return;
  const long long ld = p.ld;
  const int k = (int)(I % p.nz);
  const long long t = I / p.nz;
  const int j = (int)(t % p.ny);
  const int i = (int)(t / p.ny);
  const real acu = Acu<real>::v;
  const bool riemann = (p.flags & FLAG_RIEMANN) != 0;

  real e0[4];
#pragma unroll
  for (int c = 0; c < 4; c++) e0[c] = b.ev_st[c * ld + I];
  real S[4];
#pragma unroll
  for (int c = 0; c < 4; c++) S[c] = (step == 1) ? (real)0.0f : b.src[c * ld + I];

  {  // kernel_ideal.cl:125-143
    real ed = e0[0], vz = e0[3];
    real pressure = eosP<real>(p, ed);
    real u0 = gamma3<real>(e0[1], e0[2], vz);
    real Tzz_tilde = (ed + pressure) * u0 * u0 * vz * vz + pressure;
    real Ttz_tilde = (ed + pressure) * u0 * u0 * vz;
    if (!riemann) {
      S[0] = S[0] - Tzz_tilde;
      S[1] = S[1] - (real)0.0f;
      S[2] = S[2] - (real)0.0f;
      S[3] = S[3] - Ttz_tilde;
    }
  }

#pragma unroll 1
  for (int a = 0; a < 3; a++) {
    const int q = a == 0 ? i : (a == 1 ? j : k);
    const int L = a == 0 ? p.nx : (a == 1 ? p.ny : p.nz);
    // one cell along this axis: both face fluxes are equal, their difference
    // is +0 and leaves the sources unchanged (finite states; see visc_stage_cell)
    if (L == 1) continue;
    const long long stride = a == 0 ? (long long)p.ny * p.nz : (a == 1 ? (long long)p.nz : 1ll);
    const Stencil st = make_stencil(q, L, stride);
    real E[5][4], pr[5], T[5][4];
#pragma unroll
    for (int d = 0; d < 5; d++) {
#pragma unroll
      for (int c = 0; c < 4; c++) E[d][c] = (d == 2) ? e0[c] : b.ev_st[c * ld + I + st.off[d]];
      pr[d] = eosP<real>(p, E[d][0]);
      real u0 = gamma3<real>(E[d][1], E[d][2], E[d][3]);
      real A = (E[d][0] + pr[d]) * u0;
      real u4[4] = {(real)1.0f * u0, E[d][1] * u0, E[d][2] * u0, E[d][3] * u0};
#pragma unroll
      for (int c = 0; c < 4; c++) {
        real g0 = c == 0 ? (real)1.0f : (real)0.0f;
        T[d][c] = A * u4[c] - g0 * pr[d];
      }
    }
    real F[2][4];
#pragma unroll
    for (int f = 0; f < 2; f++) {  // kt1d, helper.h:199-262
      const int l = 1 + f, r = 2 + f;
      real h[4];
#pragma unroll
      for (int c = 0; c < 4; c++) h[c] = 0.5f * (E[l][c] + E[r][c]);
      real vh = h[a + 1];
      real lam = max_speed<real>(p, h[0], h[1], h[2], h[3], vh);
      real pr_half = 0.5f * (pr[l] + pr[r]);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        real DAl = slope<real>(T[l - 1][c], T[l][c], T[l + 1][c]);
        real DAr = slope<real>(T[r - 1][c], T[r][c], T[r + 1][c]);
        real AL = T[l][c] + 0.5f * DAl;
        real AR = T[r][c] - 0.5f * DAr;
        real g0 = c == 0 ? (real)1.0f : (real)0.0f;
        real ga = c == a + 1 ? (real)-1.0f : (real)0.0f;
        real Jp = (AR + pr_half * g0) * vh - pr_half * ga;
        real Jm = (AL + pr_half * g0) * vh - pr_half * ga;
        F[f][c] = 0.5f * (Jp + Jm) - 0.5f * lam * (AR - AL);
      }
    }
    const real D = a == 0 ? (real)p.DX : (a == 1 ? (real)p.DY : (real)p.DZ);
    const real rD = a == 0 ? rc.DX : (a == 1 ? rc.DY : rc.DZ);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      real src = F[1][c];
      src -= F[0][c];
      if (riemann) S[c] = S[c] - div_by<real>(src, D, rD);
      else if (a < 2) S[c] = S[c] - div_by<real>(tau * src, D, rD);
      else S[c] = S[c] - div_by<real>(tau * src, tc.dzt, tc.rdzt);
    }
  }

  // update_ev, kernel_ideal.cl:283-339
  real e1[4];
#pragma unroll
  for (int c = 0; c < 4; c++) e1[c] = b.ev1[c * ld + I];
  real ed = e1[0], vx = e1[1], vy = e1[2], vz = e1[3];
  real pressure = eosP<real>(p, ed);
  real u0 = gamma3<real>(vx, vy, vz);
  real umu[4] = {u0 * 1.0f, u0 * vx, u0 * vy, u0 * vz};
  real old_time = tau - (step - 1) * p.DT;
  real T0m[4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    real g0 = c == 0 ? (real)1.0f : (real)0.0f;
    T0m[c] = (ed + pressure) * u0 * umu[c] - pressure * g0;
    if (!riemann) T0m[c] = T0m[c] * old_time;
    T0m[c] = T0m[c] + div_step(S[c] * p.DT, step);
  }
  real T00, T01, T02, T03;
  if (riemann) {
    T00 = cmax<real>(acu, T0m[0]);
    T01 = (fabs(T0m[1]) < acu) ? (real)0.0f : T0m[1];
    T02 = (fabs(T0m[2]) < acu) ? (real)0.0f : T0m[2];
    T03 = (fabs(T0m[3]) < acu) ? (real)0.0f : T0m[3];
  } else {
    T00 = div_by<real>(cmax<real>(acu, T0m[0]), tau, tc.rtau);
    T01 = (fabs(T0m[1]) < acu) ? (real)0.0f : div_by<real>(T0m[1], tau, tc.rtau);
    T02 = (fabs(T0m[2]) < acu) ? (real)0.0f : div_by<real>(T0m[2], tau, tc.rtau);
    T03 = (fabs(T0m[3]) < acu) ? (real)0.0f : div_by<real>(T0m[3], tau, tc.rtau);
  }
  real M = sqrt(T01 * T01 + T02 * T02 + T03 * T03);
  real SCALE_COEF = 0.999f;
  if (M > T00) {
    T01 *= SCALE_COEF * T00 / M;
    T02 *= SCALE_COEF * T00 / M;
    T03 *= SCALE_COEF * T00 / M;
    M = SCALE_COEF * T00;
  }
  real ed_find = root_newton<real>(p, T00, M);
  ed_find = cmax<real>(0.0f, ed_find);
  real pr = eosP<real>(p, ed_find);
  real epv = cmax<real>(acu, T00 + pr);
  const real repv = (real)1.0f / epv;
  real en[4] = {ed_find, div_by<real>(T01, epv, repv), div_by<real>(T02, epv, repv), div_by<real>(T03, epv, repv)};
#pragma unroll
  for (int c = 0; c < 4; c++) b.evnew[c * ld + I] = en[c];
  if (b.write_src)
#pragma unroll
    for (int c = 0; c < 4; c++) b.src[c * ld + I] = S[c];
  if (b.edmax_key) key_max<real>(b.edmax_key, en[0]);
}

}  // namespace CLV_ARITH
}  // namespace clv
