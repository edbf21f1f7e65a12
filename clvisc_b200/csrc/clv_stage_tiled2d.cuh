// Tiled fused Runge-Kutta stage for (2+1)D grids (one cell along eta), with
// the bulk sector.
//
// Same arithmetic as visc_stage_cell (clv_stage.cuh) on a grid with NZ = 1,
// reorganised so that nothing is computed twice:
//   * A thread block of TB threads owns TB consecutive rows j0-2 .. j0+TB-3
//     of one event and marches along i over a chunk of x planes. Thread t
//     keeps row j0-2+t; the TB-4 rows j0 .. j0+TB-5 are the tile's cells, the
//     two rows either side are its y halo (recomputed by the neighbouring
//     tile), so each phase below gives every thread one item of work.
//   * Per cell, a record (ev, P(e) + Pi, gamma, Q = tau*(T0m + pi^{tau mu}),
//     pi, Pi, P(e)) is computed once per plane into shared memory; the two
//     planes ahead (i+1, i+2) of the thread's own row sit in per-thread
//     shared-memory slots. Records, slopes and faces are stored as 16-byte
//     groups (clv_smem16.cuh), one shared-memory access a group.
//   * The limited slope of every cell is computed once per direction and the
//     flux through every face once; a cell's flux difference subtracts its
//     minus face from its plus face, exactly the two values the reference
//     evaluates for that cell (kernel_visc.cl:68-127, helper.h:249-285). The
//     x face and slope travel in registers from one plane to the next.
//   * Along eta (one cell) nothing but the Christoffel part of the velocity
//     gradient remains, as in visc_stage_cell's one-cell-axis branch.
// Each record, slope and face flux is the per-cell kernel's expression, so the
// results are identical bit for bit.
#pragma once
#include "clv_smem16.cuh"
#include "clv_stage.cuh"

namespace clv {

// record fields (planes of a shared-memory region) and slope/face components
template <bool BULK> struct Rec2 {
  enum : int {
    E = 0, VX, VY, VZ,
    PR,                       // P(e) + Pi: the pressure of the KT flux
    U0,                       // gamma
    Q0,                       // Q0..Q3 = tau*(T^{tau mu} + pi^{tau mu})
    PI = Q0 + 4,              // the ten pi^{mu nu}, then Pi with the bulk sector
    NPI = BULK ? 11 : 10,
    P0 = BULK ? PI + NPI : PR,  // P(e) alone (the same plane as PR without bulk)
    N = BULK ? PI + NPI + 1 : PI + NPI,
    NCOMP = 4 + NPI           // components 0..3: Q (KT), 4..: u0*pi (IS)
  };
};

// a record (and the slope and face components) padded to whole 16-byte
// groups of U = 16 / sizeof(real) values
template <class real, bool BULK> struct Rec2L {
  static constexpr int U = Smem16<real>::U;
  static constexpr int NP = Smem16<real>::pad(Rec2<BULK>::N), RG = NP / U;
  static constexpr int CP = Smem16<real>::pad(Rec2<BULK>::NCOMP), CG = CP / U;
};

// each region stores its values as 16-byte groups, each group row by row
// ([value / U][row][value % U]): a group moves in one access
template <class real, bool BULK, int TB> struct Tile2Smem {
  typedef Rec2L<real, BULK> L;
  __align__(16) real C[L::RG][TB][L::U];   // plane i, every row of the block
  __align__(16) real A[L::RG][TB][L::U];   // plane i+1, own row
  __align__(16) real B[L::RG][TB][L::U];   // plane i+2, own row
  __align__(16) real SY[L::CG][TB][L::U];  // y slope of row t
  __align__(16) real FY[L::CG][TB][L::U];  // flux through the y face between rows t and t+1
};

inline namespace CLV_ARITH {

// record of the (clamped) cell (i, j) of the stage input, NZ = 1, into dst
template <class real, bool BULK>
__device__ __forceinline__ void rec2_make(const Params& p, const GridDims& gd, const ViscBuffers<real>& b, real tau,
                                          int i, int j, real dst[Rec2L<real, BULK>::NP]) {
  typedef Rec2<BULK> R;
  constexpr int stride = 1;
#pragma unroll
  for (int f = R::N; f < Rec2L<real, BULK>::NP; f++) dst[f] = 0.0f;  // padding
  i = min(max(i, 0), gd.nx - 1);
  j = min(max(j, 0), gd.ny - 1);
  const long long I = (long long)i * gd.ny + j;
  const long long ld = gd.ld;
  real e = b.ev_st[I], vx = b.ev_st[ld + I], vy = b.ev_st[2 * ld + I], vz = b.ev_st[3 * ld + I];
  real pv[R::NPI];
#pragma unroll
  for (int m = 0; m < R::NPI; m++) pv[m] = b.pi_st[m * ld + I];
  real p0 = eosP<real>(p, e);
  real pr = p0;
  if (BULK) pr = pr + pv[R::NPI - 1];
  real u0 = gamma3<real>(vx, vy, vz);
  real A = (e + pr) * u0;
  real u4[4] = {(real)1.0f * u0, vx * u0, vy * u0, vz * u0};
  dst[R::E * stride] = e;
  dst[R::VX * stride] = vx;
  dst[R::VY * stride] = vy;
  dst[R::VZ * stride] = vz;
  dst[R::PR * stride] = pr;
  dst[R::U0 * stride] = u0;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    real g0 = c == 0 ? (real)1.0f : (real)0.0f;
    real T0m = A * u4[c] - g0 * pr;
    dst[(R::Q0 + c) * stride] = tau * (T0m + pv[c]);
  }
#pragma unroll
  for (int m = 0; m < R::NPI; m++) dst[(R::PI + m) * stride] = pv[m];
  if (BULK) dst[R::P0 * stride] = p0;
}

// limited slopes of every component at the middle of three records
template <class real, bool BULK>
__device__ __forceinline__ void rec2_slopes(const real* L, const real* M, const real* R_, real* out) {
  typedef Rec2<BULK> R;
  constexpr int sl = 1, sm = 1, sr = 1, so = 1;
#pragma unroll
  for (int c = R::NCOMP; c < Rec2L<real, BULK>::CP; c++) out[c] = 0.0f;  // padding
#pragma unroll
  for (int c = 0; c < 4; c++) out[c * so] = slope<real>(L[(R::Q0 + c) * sl], M[(R::Q0 + c) * sm], R_[(R::Q0 + c) * sr]);
  real uL = L[R::U0 * sl], uM = M[R::U0 * sm], uR = R_[R::U0 * sr];
#pragma unroll
  for (int m = 0; m < R::NPI; m++)
    out[(4 + m) * so] =
        slope<real>(uL * L[(R::PI + m) * sl], uM * M[(R::PI + m) * sm], uR * R_[(R::PI + m) * sr]);
}

// flux through the face between records L and R along axis a (0: x, 1: y)
template <class real, bool BULK>
__device__ __forceinline__ void rec2_face(const Params& p, real tau, int a, const real* L, const real* sL,
                                          const real* R_, const real* sR, real F[Rec2L<real, BULK>::CP]) {
  typedef Rec2<BULK> R;
  constexpr int sl = 1, ssl = 1, sr = 1, ssr = 1;
#pragma unroll
  for (int c = R::NCOMP; c < Rec2L<real, BULK>::CP; c++) F[c] = 0.0f;  // padding
#if CLV_FAST
  // tolerance build, KT speed 1: the weighted form of the (3+1)D kernel's
  // face_flux (cp = (v+1)/2 on the left state, cm = (v-1)/2 on the right)
  {
    const int va = R::VX + a;
    const real vh = 0.5f * (L[va * sl] + R_[va * sr]);
    const real cp = 0.5f * (vh + (real)1.0f), cm = 0.5f * (vh - (real)1.0f);
    const real hp = 0.5f * cp, hm = 0.5f * cm;
    const real pt = 0.5f * (L[R::PR * sl] + R_[R::PR * sr]) * tau;
    const real th = 0.5f * tau;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int mi = a == 0 ? pidx(1, c) : pidx(2, c);
      const real p0s = L[(R::PI + c) * sl] + R_[(R::PI + c) * sr];
      const real pis = L[(R::PI + mi) * sl] + R_[(R::PI + mi) * sr];
      real k = (c == 0 ? pt - th * p0s : -th * p0s) * vh + th * pis;
      if (c == a + 1) k += pt;
      real f = cm * R_[(R::Q0 + c) * sr] + k;
      f = f - hm * sR[c * ssr];
      f = f + cp * L[(R::Q0 + c) * sl];
      F[c] = f + hp * sL[c * ssl];
    }
    const real cmR = cm * R_[R::U0 * sr], cpL = cp * L[R::U0 * sl];
#pragma unroll
    for (int m = 0; m < R::NPI; m++) {
      real f = cmR * R_[(R::PI + m) * sr] - hm * sR[(4 + m) * ssr];
      f = f + cpL * L[(R::PI + m) * sl];
      F[4 + m] = f + hp * sL[(4 + m) * ssl];
    }
    (void)p;
  }
#else
  real h[4];
#pragma unroll
  for (int c = 0; c < 4; c++) h[c] = 0.5f * (L[(R::E + c) * sl] + R_[(R::E + c) * sr]);
  const real vh = a == 0 ? h[1] : h[2];
  const real lam = max_speed<real>(p, h[0], h[1], h[2], h[3], vh);
  real pr_half = 0.5f * (L[R::PR * sl] + R_[R::PR * sr]);
  real pt = pr_half * tau;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    real AL = L[(R::Q0 + c) * sl] + 0.5f * sL[c * ssl];
    real AR = R_[(R::Q0 + c) * sr] - 0.5f * sR[c * ssr];
    const int mi = a == 0 ? pidx(1, c) : pidx(2, c);
    real pim0_half = 0.5f * (L[(R::PI + c) * sl] + R_[(R::PI + c) * sr]);
    real pimi_half = 0.5f * (L[(R::PI + mi) * sl] + R_[(R::PI + mi) * sr]);
    real g0 = c == 0 ? (real)1.0f : (real)0.0f;
    real ga = c == a + 1 ? (real)-1.0f : (real)0.0f;
    real Jp = (AR + pt * g0 - tau * pim0_half) * vh - pt * ga + tau * pimi_half;
    real Jm = (AL + pt * g0 - tau * pim0_half) * vh - pt * ga + tau * pimi_half;
    F[c] = 0.5f * (Jp + Jm) - 0.5f * lam * (AR - AL);
  }
  real uL = L[R::U0 * sl], uR = R_[R::U0 * sr];
#pragma unroll
  for (int m = 0; m < R::NPI; m++) {
    real AL = uL * L[(R::PI + m) * sl] + 0.5f * sL[(4 + m) * ssl];
    real AR = uR * R_[(R::PI + m) * sr] - 0.5f * sR[(4 + m) * ssr];
    real Jp = AR * vh;
    real Jm = AL * vh;
    F[4 + m] = 0.5f * (Jp + Jm) - 0.5f * lam * (AR - AL);
  }
#endif
}

// One tile: rows j0 .. j0+TB-5 of planes i0 .. i1-1 of the event (gd, b).
// Every thread of the block calls it (it holds barriers).
template <class real, bool BULK, int TB>
__device__ __forceinline__ void tile2d(const Params& p, const GridDims& gd, const ViscBuffers<real>& b, int step,
                                       const TauConst<real>& tc, int j0, int i0, int i1, Tile2Smem<real, BULK, TB>& s) {
  typedef Rec2<BULK> R;
  typedef Rec2L<real, BULK> L;
  constexpr int NC = R::NCOMP, NP = L::NP, CP = L::CP, RG = L::RG, CG = L::CG;
  const real tau = tc.tau;
  const Recips<real>& rc = recips<real>(p);
  const long long ld = gd.ld;
  const int t = threadIdx.x;
  const int jj = j0 - 2 + t;                  // this thread's row
  const bool mid = (t >= 2) && (t < TB - 2);  // a row of the tile (not its halo)
  const bool inside = mid && (jj < gd.ny);
  real* const Cp = &s.C[0][0][0];  // plane i, slot t: row t
  real* A = &s.A[0][0][0];         // own slot t
  real* B = &s.B[0][0][0];
  real* const SYp = &s.SY[0][0][0];
  real* const FYp = &s.FY[0][0][0];

  // ------------------------------------------------------------ prologue
  real s_cur[CP], F_prev[CP], s_next[CP], umu_prev[4];
  if (mid) {
    real r0[NP], r1[NP], r2[NP], s_prev[CP];
    rec2_make<real, BULK>(p, gd, b, tau, i0 - 2, jj, r0);
    rec2_make<real, BULK>(p, gd, b, tau, i0 - 1, jj, r1);
    rec2_make<real, BULK>(p, gd, b, tau, i0, jj, r2);
    grp_store<real, RG>(Cp, TB, t, r2);
    rec2_slopes<real, BULK>(r0, r1, r2, s_prev);  // x slope at i0-1
    rec2_make<real, BULK>(p, gd, b, tau, i0 + 1, jj, r0);
    grp_store<real, RG>(A, TB, t, r0);
    rec2_slopes<real, BULK>(r1, r2, r0, s_cur);  // x slope at i0
    rec2_face<real, BULK>(p, tau, 0, r1, s_prev, r2, s_cur, F_prev);
    real u0 = r1[R::U0];
    umu_prev[0] = u0 * 1.0f;
    umu_prev[1] = u0 * r1[R::VX];
    umu_prev[2] = u0 * r1[R::VY];
    umu_prev[3] = u0 * r1[R::VZ];
    rec2_make<real, BULK>(p, gd, b, tau, i0 + 2, jj, r0);
    grp_store<real, RG>(B, TB, t, r0);
  } else {
    real r0[NP];
    rec2_make<real, BULK>(p, gd, b, tau, i0, jj, r0);
    grp_store<real, RG>(Cp, TB, t, r0);
  }
  __syncthreads();

  for (int i = i0; i < i1; i++) {
    // ------------------------------------------- slopes: y of row t, x at i+1
    if (t >= 1 && t <= TB - 2) {
      real rl[NP], rm[NP], rr[NP], sy[CP];
      grp_load<real, RG>(Cp, TB, t - 1, rl);
      grp_load<real, RG>(Cp, TB, t, rm);
      grp_load<real, RG>(Cp, TB, t + 1, rr);
      rec2_slopes<real, BULK>(rl, rm, rr, sy);
      grp_store<real, CG>(SYp, TB, t, sy);
    }
    if (mid) {
      real rl[NP], rm[NP], rr[NP];
      grp_load<real, RG>(Cp, TB, t, rl);
      grp_load<real, RG>(A, TB, t, rm);
      grp_load<real, RG>(B, TB, t, rr);
      rec2_slopes<real, BULK>(rl, rm, rr, s_next);
    }
    __syncthreads();

    // ------------------------------------- faces: y between t and t+1, x at i+1/2
    real Fx[CP];
    if (t >= 1 && t <= TB - 3) {
      real rl[NP], rr[NP], sl[CP], sr[CP], Fy[CP];
      grp_load<real, RG>(Cp, TB, t, rl);
      grp_load<real, RG>(Cp, TB, t + 1, rr);
      grp_load<real, CG>(SYp, TB, t, sl);
      grp_load<real, CG>(SYp, TB, t + 1, sr);
      rec2_face<real, BULK>(p, tau, 1, rl, sl, rr, sr, Fy);
      grp_store<real, CG>(FYp, TB, t, Fy);
    }
    if (mid) {
      real rl[NP], rr[NP];
      grp_load<real, RG>(Cp, TB, t, rl);
      grp_load<real, RG>(A, TB, t, rr);
      rec2_face<real, BULK>(p, tau, 0, rl, s_cur, rr, s_next, Fx);
    }
    __syncthreads();

    // ------------------------------------------------------ cell update
    if (inside && i < gd.nx) {
      const long long I = (long long)i * gd.ny + jj;
      real Cs[NP];
      grp_load<real, RG>(Cp, TB, t, Cs);
      CellIn<real> cin;
      real* e0 = cin.e0;
      e0[0] = Cs[R::E];
      e0[1] = Cs[R::VX];
      e0[2] = Cs[R::VY];
      e0[3] = Cs[R::VZ];
      cin.g0 = Cs[R::U0];
      cin.p0 = Cs[R::P0];
      real pc[11];
#pragma unroll
      for (int m = 0; m < R::NPI; m++) pc[m] = Cs[R::PI + m];
      if (!BULK) pc[10] = 0.0f;
      real pin[5];
#pragma unroll
      for (int c = 0; c < 4; c++) pin[c] = b.pin[c * ld + I];
      pin[4] = BULK ? b.pin[10 * ld + I] : (real)0.0f;
      real S4[4], S10[11];
      if (step == 1) {
#pragma unroll
        for (int c = 0; c < 4; c++) S4[c] = 0.0f;
#pragma unroll
        for (int m = 0; m < 11; m++) S10[m] = 0.0f;
      } else {
#pragma unroll
        for (int c = 0; c < 4; c++) S4[c] = b.src[c * ld + I];
#pragma unroll
        for (int m = 0; m < R::NPI; m++) S10[m] = b.src[(4 + m) * ld + I];
        if (!BULK) S10[10] = 0.0f;
      }
      {  // Christoffel terms, kernel_IS.cl:56-65
        real uz = e0[3] * cin.g0;
        S10[0] -= div_by<real>(2.0f * uz * pc[pidx(0, 3)], tau, tc.rtau);
        S10[1] -= div_by<real>(uz * pc[pidx(1, 3)], tau, tc.rtau);
        S10[2] -= div_by<real>(uz * pc[pidx(2, 3)], tau, tc.rtau);
        S10[3] -= div_by<real>(uz * (pc[pidx(0, 0)] + pc[pidx(3, 3)]), tau, tc.rtau);
        S10[6] -= div_by<real>(uz * pc[pidx(0, 1)], tau, tc.rtau);
        S10[8] -= div_by<real>(uz * pc[pidx(0, 2)], tau, tc.rtau);
        S10[9] -= div_by<real>(2.0f * uz * pc[pidx(0, 3)], tau, tc.rtau);
      }
      {  // kernel_visc.cl:24-50
        real ed = e0[0], vx = e0[1], vy = e0[2], vz = e0[3];
        real u0 = cin.g0;
        real bulkpi = BULK ? pc[10] : (real)0.0f;
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
      // flux differences in the reference's order x, y (eta: one cell, none)
      real Fyp[CP], Fym[CP];
      grp_load<real, CG>(FYp, TB, t, Fyp);
      grp_load<real, CG>(FYp, TB, t - 1, Fym);
#pragma unroll
      for (int a = 0; a < 2; a++) {
        const real D = a == 0 ? (real)p.DX : (real)p.DY;
        const real rD = a == 0 ? rc.DX : rc.DY;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          real fp = a == 0 ? Fx[c] : Fyp[c];
          real fm = a == 0 ? F_prev[c] : Fym[c];
          real src = fp;
          src -= fm;
          if (c < 4) S4[c] = S4[c] - div_by<real>(src, D, rD);
          else S10[c - 4] = S10[c - 4] - div_by<real>(src, D, rD);
        }
      }
      // velocity gradients, kernel_IS.cl:134-137 / 217-220 / 299-304
      real grad[3][4];
      {
        real Ax[NP], Cy0[NP], Cy1[NP];
        grp_load<real, RG>(A, TB, t, Ax);
        grp_load<real, RG>(Cp, TB, t - 1, Cy0);
        grp_load<real, RG>(Cp, TB, t + 1, Cy1);
        real u0c = cin.g0;
        real umc[4] = {u0c * 1.0f, u0c * e0[1], u0c * e0[2], u0c * e0[3]};
        real ua = Ax[R::U0];
        real umx1[4] = {ua * 1.0f, ua * Ax[R::VX], ua * Ax[R::VY], ua * Ax[R::VZ]};
        real uy0 = Cy0[R::U0], uy1 = Cy1[R::U0];
        real umy0[4] = {uy0 * 1.0f, uy0 * Cy0[R::VX], uy0 * Cy0[R::VY], uy0 * Cy0[R::VZ]};
        real umy1[4] = {uy1 * 1.0f, uy1 * Cy1[R::VX], uy1 * Cy1[R::VY], uy1 * Cy1[R::VZ]};
#pragma unroll
        for (int c = 0; c < 4; c++) {
          grad[0][c] = div_by<real>(grad_limit<real>(umu_prev[c], umc[c], umx1[c]), (real)p.DX, rc.DX);
          grad[1][c] = div_by<real>(grad_limit<real>(umy0[c], umc[c], umy1[c]), (real)p.DY, rc.DY);
          grad[2][c] = 0.0f;
        }
        grad[2][0] = grad[2][0] + div_by<real>(e0[3] * u0c, tau, tc.rtau);
        grad[2][1] = grad[2][1] + div_by<real>((real)0.0f * u0c, tau, tc.rtau);
        grad[2][2] = grad[2][2] + div_by<real>((real)0.0f * u0c, tau, tc.rtau);
        grad[2][3] = grad[2][3] + div_by<real>((real)1.0f * u0c, tau, tc.rtau);
#pragma unroll
        for (int c = 0; c < 4; c++) umu_prev[c] = umc[c];
      }
      real pinew[11];
      cell_in_ev1<real>(p, b, I, ld, cin);
      pi_update<real, false, BULK>(p, b, step, tc, I, ld, cin, pc, grad, S10, pinew);
      ev_update<real, true, BULK>(p, b, step, tc, I, ld, cin, pin, S4, pinew);
      if (b.write_src) {
#pragma unroll
        for (int c = 0; c < 4; c++) b.src[c * ld + I] = S4[c];
#pragma unroll
        for (int m = 0; m < R::NPI; m++) b.src[(4 + m) * ld + I] = S10[m];
      }
    } else if (mid) {
      real Cs[NP];
      grp_load<real, RG>(Cp, TB, t, Cs);
      real u0c = Cs[R::U0];
      umu_prev[0] = u0c * 1.0f;
      umu_prev[1] = u0c * Cs[R::VX];
      umu_prev[2] = u0c * Cs[R::VY];
      umu_prev[3] = u0c * Cs[R::VZ];
    }
    if (mid) {
#pragma unroll
      for (int c = 0; c < NC; c++) {
        F_prev[c] = Fx[c];
        s_cur[c] = s_next[c];
      }
    }
    __syncthreads();

    // --------------------------------------------------------- advance
    if (i + 1 < i1) {
      if (mid) {
        real r[NP];
        grp_load<real, RG>(A, TB, t, r);
        grp_store<real, RG>(Cp, TB, t, r);
        real* tmp = A;
        A = B;
        B = tmp;
        rec2_make<real, BULK>(p, gd, b, tau, i + 3, jj, r);
        grp_store<real, RG>(B, TB, t, r);
      } else {
        real r[NP];
        rec2_make<real, BULK>(p, gd, b, tau, i + 1, jj, r);
        grp_store<real, RG>(Cp, TB, t, r);
      }
      __syncthreads();
    }
  }
}

// resident blocks per SM the tiled (2+1)D kernels are compiled for: by
// default 384 threads per SM in FP32 (168 registers a thread; 512 threads at
// 128 registers spill and ran 25 % slower on B200), 256 in FP64;
// CLV_TILED2D_THREADS_F32 sets the FP32 threads per SM at build time
#ifndef CLV_TILED2D_THREADS_F32
#define CLV_TILED2D_THREADS_F32 384
#endif
template <class real, int TB> constexpr int tiled2d_minb() {
  return (sizeof(real) == 4 ? CLV_TILED2D_THREADS_F32 : 256) / TB;
}

// single event, grid (ceil(NY / (TB-4)), ceil(NX / chunk))
template <class real, bool BULK, int TB, int MINB>
__global__ void __launch_bounds__(TB, MINB)
    visc_stage_tiled2d_kernel(Params p, ViscBuffers<real> b, int step, TauConst<real> tc, int chunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Tile2Smem<real, BULK, TB>& s = *reinterpret_cast<Tile2Smem<real, BULK, TB>*>(smem_raw);
  const GridDims gd{p.nx, p.ny, p.nz, p.ld};
  const int i0 = blockIdx.y * chunk;
  tile2d<real, BULK, TB>(p, gd, b, step, tc, blockIdx.x * (TB - 4), i0, min(i0 + chunk, p.nx), s);
}

}  // namespace CLV_ARITH
}  // namespace clv
