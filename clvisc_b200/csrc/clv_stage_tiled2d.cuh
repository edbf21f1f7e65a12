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
//     shared-memory slots.
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

template <class real, bool BULK, int TB> struct Tile2Smem {
  typedef Rec2<BULK> R;
  real C[R::N][TB];       // plane i, every row of the block
  real A[R::N][TB];       // plane i+1, own row
  real B[R::N][TB];       // plane i+2, own row
  real SY[R::NCOMP][TB];  // y slope of row t
  real FY[R::NCOMP][TB];  // flux through the y face between rows t and t+1
};

inline namespace CLV_ARITH {

// record of the (clamped) cell (i, j) of the stage input, NZ = 1
template <class real, bool BULK>
__device__ __forceinline__ void rec2_make(const Params& p, const GridDims& gd, const ViscBuffers<real>& b, real tau,
                                          int i, int j, real* dst, int stride) {
  typedef Rec2<BULK> R;
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
__device__ __forceinline__ void rec2_slopes(const real* L, int sl, const real* M, int sm, const real* R_, int sr,
                                            real* out, int so) {
  typedef Rec2<BULK> R;
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
__device__ __forceinline__ void rec2_face(const Params& p, real tau, int a, const real* L, int sl, const real* sL,
                                          int ssl, const real* R_, int sr, const real* sR, int ssr,
                                          real F[Rec2<BULK>::NCOMP]) {
  typedef Rec2<BULK> R;
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
  constexpr int NC = R::NCOMP;
  const real tau = tc.tau;
  const Recips<real>& rc = recips<real>(p);
  const long long ld = gd.ld;
  const int t = threadIdx.x;
  const int jj = j0 - 2 + t;                  // this thread's row
  const bool mid = (t >= 2) && (t < TB - 2);  // a row of the tile (not its halo)
  const bool inside = mid && (jj < gd.ny);
  real(*A)[TB] = s.A;
  real(*B)[TB] = s.B;
  real* const Cs = &s.C[0][t];  // own record in the plane region (stride TB)

  // ------------------------------------------------------------ prologue
  real s_cur[NC], F_prev[NC], s_next[NC], umu_prev[4];
  if (mid) {
    real s_prev[NC];
    rec2_make<real, BULK>(p, gd, b, tau, i0 - 2, jj, &A[0][t], TB);
    rec2_make<real, BULK>(p, gd, b, tau, i0 - 1, jj, &B[0][t], TB);
    rec2_make<real, BULK>(p, gd, b, tau, i0, jj, Cs, TB);
    rec2_slopes<real, BULK>(&A[0][t], TB, &B[0][t], TB, Cs, TB, s_prev, 1);  // x slope at i0-1
    rec2_make<real, BULK>(p, gd, b, tau, i0 + 1, jj, &A[0][t], TB);
    rec2_slopes<real, BULK>(&B[0][t], TB, Cs, TB, &A[0][t], TB, s_cur, 1);   // x slope at i0
    rec2_face<real, BULK>(p, tau, 0, &B[0][t], TB, s_prev, 1, Cs, TB, s_cur, 1, F_prev);
    real u0 = B[R::U0][t];
    umu_prev[0] = u0 * 1.0f;
    umu_prev[1] = u0 * B[R::VX][t];
    umu_prev[2] = u0 * B[R::VY][t];
    umu_prev[3] = u0 * B[R::VZ][t];
    rec2_make<real, BULK>(p, gd, b, tau, i0 + 2, jj, &B[0][t], TB);
  } else {
    rec2_make<real, BULK>(p, gd, b, tau, i0, jj, Cs, TB);
  }
  __syncthreads();

  for (int i = i0; i < i1; i++) {
    // ------------------------------------------- slopes: y of row t, x at i+1
    if (t >= 1 && t <= TB - 2) rec2_slopes<real, BULK>(Cs - 1, TB, Cs, TB, Cs + 1, TB, &s.SY[0][t], TB);
    if (mid) rec2_slopes<real, BULK>(Cs, TB, &A[0][t], TB, &B[0][t], TB, s_next, 1);
    __syncthreads();

    // ------------------------------------- faces: y between t and t+1, x at i+1/2
    real Fx[NC];
    if (t >= 1 && t <= TB - 3) {
      real Fy[NC];
      rec2_face<real, BULK>(p, tau, 1, Cs, TB, &s.SY[0][t], TB, Cs + 1, TB, &s.SY[0][t + 1], TB, Fy);
#pragma unroll
      for (int c = 0; c < NC; c++) s.FY[c][t] = Fy[c];
    }
    if (mid) rec2_face<real, BULK>(p, tau, 0, Cs, TB, s_cur, 1, &A[0][t], TB, s_next, 1, Fx);
    __syncthreads();

    // ------------------------------------------------------ cell update
    if (inside && i < gd.nx) {
      const long long I = (long long)i * gd.ny + jj;
      CellIn<real> cin;
      real* e0 = cin.e0;
      e0[0] = Cs[R::E * TB];
      e0[1] = Cs[R::VX * TB];
      e0[2] = Cs[R::VY * TB];
      e0[3] = Cs[R::VZ * TB];
      cin.g0 = Cs[R::U0 * TB];
      cin.p0 = Cs[R::P0 * TB];
      real pc[11];
#pragma unroll
      for (int m = 0; m < R::NPI; m++) pc[m] = Cs[(R::PI + m) * TB];
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
#pragma unroll
      for (int a = 0; a < 2; a++) {
        const real D = a == 0 ? (real)p.DX : (real)p.DY;
        const real rD = a == 0 ? rc.DX : rc.DY;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          real fp = a == 0 ? Fx[c] : s.FY[c][t];
          real fm = a == 0 ? F_prev[c] : s.FY[c][t - 1];
          real src = fp;
          src -= fm;
          if (c < 4) S4[c] = S4[c] - div_by<real>(src, D, rD);
          else S10[c - 4] = S10[c - 4] - div_by<real>(src, D, rD);
        }
      }
      // velocity gradients, kernel_IS.cl:134-137 / 217-220 / 299-304
      real grad[3][4];
      {
        const real* Cy0 = Cs - 1;
        const real* Cy1 = Cs + 1;
        real u0c = cin.g0;
        real umc[4] = {u0c * 1.0f, u0c * e0[1], u0c * e0[2], u0c * e0[3]};
        real ua = A[R::U0][t];
        real umx1[4] = {ua * 1.0f, ua * A[R::VX][t], ua * A[R::VY][t], ua * A[R::VZ][t]};
        real uy0 = Cy0[R::U0 * TB], uy1 = Cy1[R::U0 * TB];
        real umy0[4] = {uy0 * 1.0f, uy0 * Cy0[R::VX * TB], uy0 * Cy0[R::VY * TB], uy0 * Cy0[R::VZ * TB]};
        real umy1[4] = {uy1 * 1.0f, uy1 * Cy1[R::VX * TB], uy1 * Cy1[R::VY * TB], uy1 * Cy1[R::VZ * TB]};
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
      real u0c = Cs[R::U0 * TB];
      umu_prev[0] = u0c * 1.0f;
      umu_prev[1] = u0c * Cs[R::VX * TB];
      umu_prev[2] = u0c * Cs[R::VY * TB];
      umu_prev[3] = u0c * Cs[R::VZ * TB];
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
#pragma unroll
        for (int f = 0; f < R::N; f++) Cs[f * TB] = A[f][t];
        real(*tmp)[TB] = A;
        A = B;
        B = tmp;
        rec2_make<real, BULK>(p, gd, b, tau, i + 3, jj, &B[0][t], TB);
      } else {
        rec2_make<real, BULK>(p, gd, b, tau, i + 1, jj, Cs, TB);
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
