// Tiled fused Runge-Kutta stage for the viscous step (the production kernel).
//
// Same arithmetic as visc_stage_kernel (clv_stage.cuh), reorganised so that
// nothing is computed twice:
//   * A CTA owns a TJ x TK tile of (j, k) columns and marches along i over a
//     chunk of x planes (2.5-D blocking), so every x plane is read from HBM
//     once per chunk.
//   * Per cell, a record (ev, P(e), u0, Q = tau*(T0m + pi^{tau mu}), pi) is
//     computed once, into shared memory: the centre plane with a 2-cell halo
//     in j and k, and the two planes ahead (i+1, i+2) for the x stencil.
//   * The limited slope of every cell is computed once per direction, and the
//     flux through every face once; a cell's flux difference subtracts the
//     flux of its minus face from that of its plus face, exactly the two
//     values the reference evaluates for that cell (helper.h:199-262,
//     kernel_visc.cl:68-127, helper.h:249-285). The x-direction face and
//     slope travel with the thread in registers from one plane to the next.
// Each face flux, slope and record is an expression-for-expression copy of
// the per-cell kernel's, so the results are identical bit for bit.
#pragma once
#include "clv_stage.cuh"

namespace clv {

#ifndef CLV_TILED_INLINE
#define CLV_TILED_INLINE 1
#endif
#if CLV_TILED_INLINE
#define CLV_TILED_ATTR __forceinline__
#else
#define CLV_TILED_ATTR __noinline__
#endif

// record fields (planes of the shared-memory region)
enum { RF_E = 0, RF_VX, RF_VY, RF_VZ, RF_PR, RF_U0, RF_Q0, RF_Q1, RF_Q2, RF_Q3, RF_PI, RF_N = RF_PI + 10 };
// slope / face-flux components: 0..3 KT (Q), 4..13 IS (u0*pi)
enum { NCOMP = 14 };

template <int TJ, int TK> struct TileGeom {
  static constexpr int CY = TJ + 4, CZ = TK + 4;     // centre region with halo
  static constexpr int NC = CY * CZ;                  // cells in the centre region
  static constexpr int NI = TJ * TK;                  // interior cells
  static constexpr int NSY = (TJ + 2) * TK;           // y slopes, rows -1..TJ
  static constexpr int NSZ = TJ * (TK + 2);           // z slopes, cols -1..TK
  static constexpr int NHALO = NC - NI;               // halo cells of the centre plane
};

template <class real, int TJ, int TK> struct TileSmem {
  typedef TileGeom<TJ, TK> G;
  real C[RF_N][G::NC];        // centre plane i
  real A[RF_N][G::NI];        // plane i+1 (interior)
  real B[RF_N][G::NI];        // plane i+2 (interior)
  real SY[NCOMP][G::NSY];     // y slopes, then y face fluxes
  real SZ[NCOMP][G::NSZ];     // z slopes, then z face fluxes
};

inline namespace CLV_ARITH {

// record of one (clamped) cell of the stage input
template <class real>
__device__ CLV_TILED_ATTR void make_record(const Params& p, const ViscBuffers<real>& b, real tau, int i, int j, int k,
                                            real* dst, int stride) {
  i = min(max(i, 0), p.nx - 1);
  j = min(max(j, 0), p.ny - 1);
  k = min(max(k, 0), p.nz - 1);
  const long long I = ((long long)i * p.ny + j) * p.nz + k;
  const long long ld = p.ld;
  real e = b.ev_st[I], vx = b.ev_st[ld + I], vy = b.ev_st[2 * ld + I], vz = b.ev_st[3 * ld + I];
  real pi[10];
#pragma unroll
  for (int m = 0; m < 10; m++) pi[m] = b.pi_st[m * ld + I];
  real pr = eosP<real>(p, e);
  real u0 = gamma3<real>(vx, vy, vz);
  real A = (e + pr) * u0;
  real u4[4] = {(real)1.0f * u0, vx * u0, vy * u0, vz * u0};
  dst[RF_E * stride] = e;
  dst[RF_VX * stride] = vx;
  dst[RF_VY * stride] = vy;
  dst[RF_VZ * stride] = vz;
  dst[RF_PR * stride] = pr;
  dst[RF_U0 * stride] = u0;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    real g0 = c == 0 ? (real)1.0f : (real)0.0f;
    real T0m = A * u4[c] - g0 * pr;
    dst[(RF_Q0 + c) * stride] = tau * (T0m + pi[c]);
  }
#pragma unroll
  for (int m = 0; m < 10; m++) dst[(RF_PI + m) * stride] = pi[m];
}

// limited slopes of the 14 components at the middle of three records
template <class real>
__device__ CLV_TILED_ATTR void slopes3(const real* L, int sl, const real* M, int sm, const real* R, int sr,
                                        real* out, int so) {
#pragma unroll
  for (int c = 0; c < 4; c++)
    out[c * so] = slope<real>(L[(RF_Q0 + c) * sl], M[(RF_Q0 + c) * sm], R[(RF_Q0 + c) * sr]);
  real uL = L[RF_U0 * sl], uM = M[RF_U0 * sm], uR = R[RF_U0 * sr];
#pragma unroll
  for (int m = 0; m < 10; m++)
    out[(4 + m) * so] = slope<real>(uL * L[(RF_PI + m) * sl], uM * M[(RF_PI + m) * sm], uR * R[(RF_PI + m) * sr]);
}

// flux through the face between records L and R along axis a, given their
// slopes (kt1d_visc face part and kt1d_real face part)
template <class real, bool DO_IS, bool DO_KT>
__device__ CLV_TILED_ATTR void face_flux(const Params& p, real tau, int a, const real* L, int sl, const real* sL,
                                          int ssl, const real* R, int sr, const real* sR, int ssr, real F[NCOMP]) {
#if CLV_FAST
  // tolerance build, with the KT speed 1: F = 0.5 (J(A_R) + J(A_L)) -
  // 0.5 (A_R - A_L) is, for J linear in A with slope v, the weighted sum
  // cp A_L + cm A_R + (the pressure and pi part), cp = (v+1)/2, cm = (v-1)/2;
  // A_L = Q_L + s_L/2, A_R = Q_R - s_R/2 expanded into fused multiply-adds
  {
    const int va = RF_VX + a;
    const real vh = 0.5f * (L[va * sl] + R[va * sr]);
    const real cp = 0.5f * (vh + (real)1.0f), cm = 0.5f * (vh - (real)1.0f);
    const real hp = 0.5f * cp, hm = 0.5f * cm;
    if (DO_KT) {
      const real pt = 0.5f * (L[RF_PR * sl] + R[RF_PR * sr]) * tau;
      const real th = 0.5f * tau;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int mi = a == 0 ? pidx(1, c) : (a == 1 ? pidx(2, c) : pidx(3, c));
        const real p0s = L[(RF_PI + c) * sl] + R[(RF_PI + c) * sr];
        const real pis = L[(RF_PI + mi) * sl] + R[(RF_PI + mi) * sr];
        real k = (c == 0 ? pt - th * p0s : -th * p0s) * vh + th * pis;
        if (c == a + 1) k += pt;
        real f = cm * R[(RF_Q0 + c) * sr] + k;
        f = f - hm * sR[c * ssr];
        f = f + cp * L[(RF_Q0 + c) * sl];
        F[c] = f + hp * sL[c * ssl];
      }
    }
    if (DO_IS) {
      const real cmR = cm * R[RF_U0 * sr], cpL = cp * L[RF_U0 * sl];
#pragma unroll
      for (int m = 0; m < 10; m++) {
        real f = cmR * R[(RF_PI + m) * sr] - hm * sR[(4 + m) * ssr];
        f = f + cpL * L[(RF_PI + m) * sl];
        F[4 + m] = f + hp * sL[(4 + m) * ssl];
      }
    }
    (void)p;
  }
#else
  real h[4];
#pragma unroll
  for (int c = 0; c < 4; c++) h[c] = 0.5f * (L[(RF_E + c) * sl] + R[(RF_E + c) * sr]);
  const real vh = a == 0 ? h[1] : (a == 1 ? h[2] : h[3]);
  const real lam = max_speed<real>(p, h[0], h[1], h[2], h[3], vh);
  if (DO_KT) {
    real pr_half = 0.5f * (L[RF_PR * sl] + R[RF_PR * sr]);
    real pt = pr_half * tau;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      real AL = L[(RF_Q0 + c) * sl] + 0.5f * sL[c * ssl];
      real AR = R[(RF_Q0 + c) * sr] - 0.5f * sR[c * ssr];
      const int mi = a == 0 ? pidx(1, c) : (a == 1 ? pidx(2, c) : pidx(3, c));
      real pim0_half = 0.5f * (L[(RF_PI + c) * sl] + R[(RF_PI + c) * sr]);
      real pimi_half = 0.5f * (L[(RF_PI + mi) * sl] + R[(RF_PI + mi) * sr]);
      real g0 = c == 0 ? (real)1.0f : (real)0.0f;
      real ga = c == a + 1 ? (real)-1.0f : (real)0.0f;
      real Jp = (AR + pt * g0 - tau * pim0_half) * vh - pt * ga + tau * pimi_half;
      real Jm = (AL + pt * g0 - tau * pim0_half) * vh - pt * ga + tau * pimi_half;
      F[c] = 0.5f * (Jp + Jm) - 0.5f * lam * (AR - AL);
    }
  }
  if (DO_IS) {
    real uL = L[RF_U0 * sl], uR = R[RF_U0 * sr];
#pragma unroll
    for (int m = 0; m < 10; m++) {
      real AL = uL * L[(RF_PI + m) * sl] + 0.5f * sL[(4 + m) * ssl];
      real AR = uR * R[(RF_PI + m) * sr] - 0.5f * sR[(4 + m) * ssr];
      real Jp = AR * vh;
      real Jm = AL * vh;
      F[4 + m] = 0.5f * (Jp + Jm) - 0.5f * lam * (AR - AL);
    }
  }
#endif
}

template <class real, bool DO_IS, bool DO_KT, bool COUPLED, int TJ, int TK, int MINB>
__global__ void __launch_bounds__(TJ * TK, MINB)
    visc_stage_tiled_kernel(Params p, ViscBuffers<real> b, int step, TauConst<real> tc, int chunk) {
  const real tau = tc.tau;
  const Recips<real>& rc = recips<real>(p);
  typedef TileGeom<TJ, TK> G;
  typedef TileSmem<real, TJ, TK> SM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SM& s = *reinterpret_cast<SM*>(smem_raw);
  real(*A)[G::NI] = s.A;
  real(*B)[G::NI] = s.B;

  const int tid = threadIdx.x;
  const int tj = tid / TK, tk = tid % TK;
  const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
  const int i0 = blockIdx.z * chunk;
  const int i1 = min(i0 + chunk, p.nx);
  const int jj = j0 + tj, kk = k0 + tk;
  const bool inside = (jj < p.ny) && (kk < p.nz);
  const int cself = (tj + 2) * G::CZ + (tk + 2);  // own cell in the centre region
  const long long ld = p.ld;
  const real acu = Acu<real>::v;

  // ------------------------------------------------------------ prologue
  // x window: records of planes i0-2 (A), i0-1 (B), i0 (own cell of C)
  make_record<real>(p, b, tau, i0 - 2, jj, kk, &A[0][tid], G::NI);
  make_record<real>(p, b, tau, i0 - 1, jj, kk, &B[0][tid], G::NI);
  make_record<real>(p, b, tau, i0, jj, kk, &s.C[0][cself], G::NC);
  real s_prev[NCOMP], s_cur[NCOMP], F_prev[NCOMP], s_next[NCOMP], umu_prev[4];
  slopes3<real>(&A[0][tid], G::NI, &B[0][tid], G::NI, &s.C[0][cself], G::NC, s_prev, 1);  // slope at i0-1
  make_record<real>(p, b, tau, i0 + 1, jj, kk, &A[0][tid], G::NI);
  slopes3<real>(&B[0][tid], G::NI, &s.C[0][cself], G::NC, &A[0][tid], G::NI, s_cur, 1);   // slope at i0
  face_flux<real, DO_IS, DO_KT>(p, tau, 0, &B[0][tid], G::NI, s_prev, 1, &s.C[0][cself], G::NC, s_cur, 1, F_prev);
  {
    real u0 = B[RF_U0][tid];
    umu_prev[0] = u0 * 1.0f;
    umu_prev[1] = u0 * B[RF_VX][tid];
    umu_prev[2] = u0 * B[RF_VY][tid];
    umu_prev[3] = u0 * B[RF_VZ][tid];
  }
  make_record<real>(p, b, tau, i0 + 2, jj, kk, &B[0][tid], G::NI);
  // halo of the centre plane i0
  for (int h = tid; h < G::NC; h += TJ * TK) {
    int r = h / G::CZ, c = h % G::CZ;
    if (r >= 2 && r < TJ + 2 && c >= 2 && c < TK + 2) continue;
    make_record<real>(p, b, tau, i0, j0 - 2 + r, k0 - 2 + c, &s.C[0][h], G::NC);
  }
  __syncthreads();

  for (int i = i0; i < i1; i++) {
    // ------------------------------------------------ slopes of plane i
    for (int q = tid; q < G::NSY + G::NSZ; q += TJ * TK) {
      if (q < G::NSY) {  // y slope at row yr-1, column zc
        int yr = q / TK, zc = q % TK;
        int cm = (yr + 1) * G::CZ + (zc + 2);
        slopes3<real>(&s.C[0][cm - G::CZ], G::NC, &s.C[0][cm], G::NC, &s.C[0][cm + G::CZ], G::NC, &s.SY[0][q], G::NSY);
      } else {  // z slope at row yr, column zc-1
        int qq = q - G::NSY;
        int yr = qq / (TK + 2), zc = qq % (TK + 2);
        int cm = (yr + 2) * G::CZ + (zc + 1);
        slopes3<real>(&s.C[0][cm - 1], G::NC, &s.C[0][cm], G::NC, &s.C[0][cm + 1], G::NC, &s.SZ[0][qq], G::NSZ);
      }
    }
    // x slope at i+1 (own column)
    slopes3<real>(&s.C[0][cself], G::NC, &A[0][tid], G::NI, &B[0][tid], G::NI, s_next, 1);
    __syncthreads();

    // ---------------------------------------------------- face fluxes
    real Fy[NCOMP], Fz[NCOMP], Fx[NCOMP], Fh[NCOMP];
    {
      const int sy = (tj + 1) * TK + tk;        // slope slot of own cell (y)
      const int sz = tj * (TK + 2) + (tk + 1);  // slope slot of own cell (z)
      face_flux<real, DO_IS, DO_KT>(p, tau, 1, &s.C[0][cself], G::NC, &s.SY[0][sy], G::NSY, &s.C[0][cself + G::CZ],
                                    G::NC, &s.SY[0][sy + TK], G::NSY, Fy);
      face_flux<real, DO_IS, DO_KT>(p, tau, 2, &s.C[0][cself], G::NC, &s.SZ[0][sz], G::NSZ, &s.C[0][cself + 1], G::NC,
                                    &s.SZ[0][sz + 1], G::NSZ, Fz);
      face_flux<real, DO_IS, DO_KT>(p, tau, 0, &s.C[0][cself], G::NC, s_cur, 1, &A[0][tid], G::NI, s_next, 1, Fx);
      if (tid < TK) {  // y face below row 0, column tid
        const int c0 = 1 * G::CZ + (tid + 2);
        face_flux<real, DO_IS, DO_KT>(p, tau, 1, &s.C[0][c0], G::NC, &s.SY[0][tid], G::NSY, &s.C[0][c0 + G::CZ], G::NC,
                                      &s.SY[0][TK + tid], G::NSY, Fh);
      } else if (tid < TK + TJ) {  // z face left of column 0, row tid-TK
        const int r = tid - TK;
        const int c0 = (r + 2) * G::CZ + 1;
        face_flux<real, DO_IS, DO_KT>(p, tau, 2, &s.C[0][c0], G::NC, &s.SZ[0][r * (TK + 2)], G::NSZ, &s.C[0][c0 + 1],
                                      G::NC, &s.SZ[0][r * (TK + 2) + 1], G::NSZ, Fh);
      }
    }
    __syncthreads();
    // faces replace slopes: y face j+1/2 in slot (j+1), z face k+1/2 in slot (k+1)
#pragma unroll
    for (int c = 0; c < NCOMP; c++) {
      if (c < 4 && !DO_KT) continue;
      if (c >= 4 && !DO_IS) continue;
      s.SY[c][(tj + 1) * TK + tk] = Fy[c];
      s.SZ[c][tj * (TK + 2) + (tk + 1)] = Fz[c];
      if (tid < TK) s.SY[c][tid] = Fh[c];
      else if (tid < TK + TJ) s.SZ[c][(tid - TK) * (TK + 2)] = Fh[c];
    }
    __syncthreads();

    // ------------------------------------------------------ cell update
    if (inside && i < p.nx) {
      const long long I = ((long long)i * p.ny + jj) * p.nz + kk;
      const real* Cc = &s.C[0][cself];
      CellIn<real> cin;  // the record holds gamma and P(e) of the stage input
      real* e0 = cin.e0;
      e0[0] = Cc[RF_E * G::NC];
      e0[1] = Cc[RF_VX * G::NC];
      e0[2] = Cc[RF_VY * G::NC];
      e0[3] = Cc[RF_VZ * G::NC];
      cin.g0 = Cc[RF_U0 * G::NC];
      cin.p0 = Cc[RF_PR * G::NC];
      real pc[11];  // component 10 (bulk) unused: this kernel has no bulk sector
#pragma unroll
      for (int m = 0; m < 10; m++) pc[m] = Cc[(RF_PI + m) * G::NC];
      real pin[5];
#pragma unroll
      for (int c = 0; c < 4; c++) pin[c] = DO_KT ? b.pin[c * ld + I] : (real)0.0f;
      pin[4] = 0.0f;
      pc[10] = 0.0f;
      real S4[4], S10[11];
      S10[10] = 0.0f;
      if (step == 1) {
#pragma unroll
        for (int c = 0; c < 4; c++) S4[c] = 0.0f;
#pragma unroll
        for (int m = 0; m < 10; m++) S10[m] = 0.0f;
      } else {
#pragma unroll
        for (int c = 0; c < 4; c++) S4[c] = DO_KT ? b.src[c * ld + I] : (real)0.0f;
#pragma unroll
        for (int m = 0; m < 10; m++) S10[m] = DO_IS ? b.src[(4 + m) * ld + I] : (real)0.0f;
      }
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
        real bulkpi = 0.0f;
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
      // flux differences in the reference's order x, y, z
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const real D = a == 0 ? (real)p.DX : (a == 1 ? (real)p.DY : tc.dzt);
        const real rD = a == 0 ? rc.DX : (a == 1 ? rc.DY : tc.rdzt);
#pragma unroll
        for (int c = 0; c < NCOMP; c++) {
          if (c < 4 && !DO_KT) continue;
          if (c >= 4 && !DO_IS) continue;
          real fp = a == 0 ? Fx[c] : (a == 1 ? Fy[c] : Fz[c]);
          real fm = a == 0 ? F_prev[c] : (a == 1 ? s.SY[c][tj * TK + tk] : s.SZ[c][tj * (TK + 2) + tk]);
          real src = fp;
          src -= fm;
          if (c < 4) S4[c] = S4[c] - div_by<real>(src, D, rD);
          else S10[c - 4] = S10[c - 4] - div_by<real>(src, D, rD);
        }
      }

      real pinew[11];
      cell_in_ev1<real>(p, b, I, ld, cin);
      if (DO_IS) {
        // velocity gradients, kernel_IS.cl:134-137 / 217-220 / 299-304
        real grad[3][4];
        {
          const real* Cy0 = Cc - G::CZ;
          const real* Cy1 = Cc + G::CZ;
          const real* Cz0 = Cc - 1;
          const real* Cz1 = Cc + 1;
          real u0c = Cc[RF_U0 * G::NC];
          real umc[4] = {u0c * 1.0f, u0c * e0[1], u0c * e0[2], u0c * e0[3]};
          real ua = A[RF_U0][tid];
          real umx1[4] = {ua * 1.0f, ua * A[RF_VX][tid], ua * A[RF_VY][tid], ua * A[RF_VZ][tid]};
          real uy0 = Cy0[RF_U0 * G::NC], uy1 = Cy1[RF_U0 * G::NC], uz0 = Cz0[RF_U0 * G::NC], uz1 = Cz1[RF_U0 * G::NC];
          real umy0[4] = {uy0 * 1.0f, uy0 * Cy0[RF_VX * G::NC], uy0 * Cy0[RF_VY * G::NC], uy0 * Cy0[RF_VZ * G::NC]};
          real umy1[4] = {uy1 * 1.0f, uy1 * Cy1[RF_VX * G::NC], uy1 * Cy1[RF_VY * G::NC], uy1 * Cy1[RF_VZ * G::NC]};
          real umz0[4] = {uz0 * 1.0f, uz0 * Cz0[RF_VX * G::NC], uz0 * Cz0[RF_VY * G::NC], uz0 * Cz0[RF_VZ * G::NC]};
          real umz1[4] = {uz1 * 1.0f, uz1 * Cz1[RF_VX * G::NC], uz1 * Cz1[RF_VY * G::NC], uz1 * Cz1[RF_VZ * G::NC]};
#pragma unroll
          for (int c = 0; c < 4; c++) {
            grad[0][c] = div_by<real>(grad_limit<real>(umu_prev[c], umc[c], umx1[c]), (real)p.DX, rc.DX);
            grad[1][c] = div_by<real>(grad_limit<real>(umy0[c], umc[c], umy1[c]), (real)p.DY, rc.DY);
            grad[2][c] = div_by<real>(grad_limit<real>(umz0[c], umc[c], umz1[c]), tc.dzt, tc.rdzt);
          }
          grad[2][0] = grad[2][0] + div_by<real>(e0[3] * u0c, tau, tc.rtau);
          grad[2][1] = grad[2][1] + div_by<real>((real)0.0f * u0c, tau, tc.rtau);
          grad[2][2] = grad[2][2] + div_by<real>((real)0.0f * u0c, tau, tc.rtau);
          grad[2][3] = grad[2][3] + div_by<real>((real)1.0f * u0c, tau, tc.rtau);
#pragma unroll
          for (int c = 0; c < 4; c++) umu_prev[c] = umc[c];
        }
        pi_update<real, COUPLED, false>(p, b, step, tc, I, ld, cin, pc, grad, S10, pinew);
      } else {
        real u0c = Cc[RF_U0 * G::NC];
        umu_prev[0] = u0c * 1.0f;
        umu_prev[1] = u0c * e0[1];
        umu_prev[2] = u0c * e0[2];
        umu_prev[3] = u0c * e0[3];
      }
      if (DO_KT) ev_update<real, DO_IS, false>(p, b, step, tc, I, ld, cin, pin, S4, pinew);
      if (b.write_src) {
        if (DO_KT)
#pragma unroll
          for (int c = 0; c < 4; c++) b.src[c * ld + I] = S4[c];
        if (DO_IS)
#pragma unroll
          for (int m = 0; m < 10; m++) b.src[(4 + m) * ld + I] = S10[m];
      }
    }
#pragma unroll
    for (int c = 0; c < NCOMP; c++) {
      F_prev[c] = Fx[c];
      s_cur[c] = s_next[c];
    }
    __syncthreads();

    // --------------------------------------------------------- advance
    if (i + 1 < i1) {
#pragma unroll
      for (int f = 0; f < RF_N; f++) s.C[f][cself] = A[f][tid];
      real(*t)[G::NI] = A;
      A = B;
      B = t;
      make_record<real>(p, b, tau, i + 3, jj, kk, &B[0][tid], G::NI);
      for (int h = tid; h < G::NC; h += TJ * TK) {
        int r = h / G::CZ, c = h % G::CZ;
        if (r >= 2 && r < TJ + 2 && c >= 2 && c < TK + 2) continue;
        make_record<real>(p, b, tau, i + 1, j0 - 2 + r, k0 - 2 + c, &s.C[0][h], G::NC);
      }
      __syncthreads();
    }
  }
  (void)acu;
}

}  // namespace CLV_ARITH
}  // namespace clv
