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
//     A record's 20 values are groups of 16 bytes (four floats or two
//     doubles), each group of a plane stored cell by cell, so a group moves
//     in one shared-memory access and a warp's accesses are contiguous;
//     slopes and face fluxes (14 components) likewise.
//   * The limited slope of every cell is computed once per direction, and the
//     flux through every face once; a cell's flux difference subtracts the
//     flux of its minus face from that of its plus face, exactly the two
//     values the reference evaluates for that cell (helper.h:199-262,
//     kernel_visc.cl:68-127, helper.h:249-285). The x-direction face and
//     slope travel with the thread in registers from one plane to the next.
// Each face flux, slope and record is an expression-for-expression copy of
// the per-cell kernel's, so the results are identical bit for bit.
#pragma once
#include "clv_smem16.cuh"
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

// record fields; in shared memory a plane's records are stored as groups of
// U = 16 / sizeof(real) fields (four floats or two doubles), each group cell
// by cell: field f of cell c at [f / U][c][f % U], so a group moves in one
// 16-byte access and a warp's accesses to one group are contiguous
enum { RF_E = 0, RF_VX, RF_VY, RF_VZ, RF_PR, RF_U0, RF_Q0, RF_Q1, RF_Q2, RF_Q3, RF_PI, RF_N = RF_PI + 10 };
// slope / face-flux components: 0..3 KT (Q), 4..13 IS (u0*pi); as groups of U
// and, for floats, a tail pair (12, 13)
enum { NCOMP = 14 };

template <class real> struct Lanes {
  static constexpr int U = 16 / (int)sizeof(real);  // reals in 16 bytes
  static constexpr int RG = RF_N / U;              // record groups: 5 (FP32), 10 (FP64)
  static constexpr int SG = NCOMP / U;             // slope groups: 3, 7
  static constexpr int ST = NCOMP % U;             // slope tail: 2, 0
};

template <int TJ, int TK> struct TileGeom {
  static constexpr int CY = TJ + 4, CZ = TK + 4;     // centre region with halo
  static constexpr int NC = CY * CZ;                  // cells in the centre region
  static constexpr int NI = TJ * TK;                  // interior cells
  static constexpr int NSY = (TJ + 2) * TK;           // y slopes, rows -1..TJ
  static constexpr int NSZ = TJ * (TK + 2);           // z slopes, cols -1..TK
  static constexpr int NHALO = NC - NI;               // halo cells of the centre plane
};

// slope tail of n slots (none for doubles: one unused element)
template <class real, int N, int ST> struct SlopeTail {
  __align__(16) real v[N][ST];
};
template <class real, int N> struct SlopeTail<real, N, 0> {
  real v[1][1];
};

template <class real, int TJ, int TK> struct TileSmem {
  typedef TileGeom<TJ, TK> G;
  typedef Lanes<real> L;
  __align__(16) real C[L::RG][G::NC][L::U];     // centre plane i
  __align__(16) real A[L::RG][G::NI][L::U];     // plane i+1 (interior)
  __align__(16) real B[L::RG][G::NI][L::U];     // plane i+2 (interior)
  __align__(16) real SY[L::SG][G::NSY][L::U];   // y slopes, then y face fluxes
  __align__(16) real SZ[L::SG][G::NSZ][L::U];   // z slopes, then z face fluxes
  SlopeTail<real, G::NSY, L::ST> SYT;
  SlopeTail<real, G::NSZ, L::ST> SZT;
};

// a record of cell c of a plane of n cells (plane = &X[0][0][0]); groups
// whose values go unused are dropped by the compiler
template <class real> __device__ __forceinline__ void rec_load(const real* plane, int n, int c, real r[RF_N]) {
  typedef Lanes<real> L;
#pragma unroll
  for (int g = 0; g < L::RG; g++) ld16<real>(plane + ((size_t)g * n + c) * L::U, r + L::U * g);
}
template <class real> __device__ __forceinline__ void rec_store(real* plane, int n, int c, const real r[RF_N]) {
  typedef Lanes<real> L;
#pragma unroll
  for (int g = 0; g < L::RG; g++) st16<real>(plane + ((size_t)g * n + c) * L::U, r + L::U * g);
}
// the 14 slope (or face) components of slot c of an array of n slots (sg:
// the groups, st: the tail)
template <class real>
__device__ __forceinline__ void cmp_load(const real* sg, const real* st, int n, int c, real v[NCOMP]) {
  typedef Lanes<real> L;
#pragma unroll
  for (int g = 0; g < L::SG; g++) ld16<real>(sg + ((size_t)g * n + c) * L::U, v + L::U * g);
  if constexpr (L::ST == 2) {
    const float2 t = *reinterpret_cast<const float2*>(st + (size_t)c * 2);
    v[NCOMP - 2] = t.x;
    v[NCOMP - 1] = t.y;
  }
  (void)st;
}
template <class real>
__device__ __forceinline__ void cmp_store(real* sg, real* st, int n, int c, const real v[NCOMP]) {
  typedef Lanes<real> L;
#pragma unroll
  for (int g = 0; g < L::SG; g++) st16<real>(sg + ((size_t)g * n + c) * L::U, v + L::U * g);
  if constexpr (L::ST == 2) *reinterpret_cast<float2*>(st + (size_t)c * 2) = make_float2(v[NCOMP - 2], v[NCOMP - 1]);
  (void)st;
}

inline namespace CLV_ARITH {

// record of one (clamped) cell of the stage input, into r
template <class real>
__device__ CLV_TILED_ATTR void make_record(const Params& p, const ViscBuffers<real>& b, real tau, int i, int j, int k,
                                            real r[RF_N]) {
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
  r[RF_E] = e;
  r[RF_VX] = vx;
  r[RF_VY] = vy;
  r[RF_VZ] = vz;
  r[RF_PR] = pr;
  r[RF_U0] = u0;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    real g0 = c == 0 ? (real)1.0f : (real)0.0f;
    real T0m = A * u4[c] - g0 * pr;
    r[RF_Q0 + c] = tau * (T0m + pi[c]);
  }
#pragma unroll
  for (int m = 0; m < 10; m++) r[RF_PI + m] = pi[m];
}
template <class real>
__device__ CLV_TILED_ATTR void store_record(const Params& p, const ViscBuffers<real>& b, real tau, int i, int j, int k,
                                             real* plane, int n, int c) {
  real r[RF_N];
  make_record<real>(p, b, tau, i, j, k, r);
  rec_store<real>(plane, n, c, r);
}

// records of the centre plane's halo: two rows above and below the tile
// (interior columns) and two columns left and right (interior rows). The
// corners of the (TJ+4) x (TK+4) region are never read (the y stencil stays
// in the interior columns, the z stencil in the interior rows) and are not
// computed.
template <class real, int TJ, int TK>
__device__ CLV_TILED_ATTR void halo_records(const Params& p, const ViscBuffers<real>& b, real tau, int i, int j0,
                                             int k0, int tid, real* C) {
  typedef TileGeom<TJ, TK> G;
  constexpr int NHY = 4 * TK, NHZ = 4 * TJ;
  for (int q = tid; q < NHY + NHZ; q += TJ * TK) {
    int r, c;
    if (q < NHY) {  // rows 0, 1, TJ+2, TJ+3; consecutive q along k
      const int rr = q / TK;
      r = rr < 2 ? rr : TJ + rr;
      c = 2 + q % TK;
    } else {  // columns 0, 1, TK+2, TK+3
      const int qq = q - NHY, cc = qq / TJ;
      c = cc < 2 ? cc : TK + cc;
      r = 2 + qq % TJ;
    }
    store_record<real>(p, b, tau, i, j0 - 2 + r, k0 - 2 + c, C, G::NC, r * G::CZ + c);
  }
}

// limited slopes of the 14 components at the middle of three records
template <class real>
__device__ CLV_TILED_ATTR void slopes3(const real L[RF_N], const real M[RF_N], const real R[RF_N], real out[NCOMP]) {
#pragma unroll
  for (int c = 0; c < 4; c++) out[c] = slope<real>(L[RF_Q0 + c], M[RF_Q0 + c], R[RF_Q0 + c]);
  real uL = L[RF_U0], uM = M[RF_U0], uR = R[RF_U0];
#pragma unroll
  for (int m = 0; m < 10; m++) out[4 + m] = slope<real>(uL * L[RF_PI + m], uM * M[RF_PI + m], uR * R[RF_PI + m]);
}

// flux through the face between records L and R along axis a, given their
// slopes (kt1d_visc face part and kt1d_real face part)
template <class real, bool DO_IS, bool DO_KT>
__device__ CLV_TILED_ATTR void face_flux(const Params& p, real tau, int a, const real L[RF_N], const real sL[NCOMP],
                                          const real R[RF_N], const real sR[NCOMP], real F[NCOMP]) {
  // components of a part this variant does not run: zero, stored and never used
  if (!DO_KT)
#pragma unroll
    for (int c = 0; c < 4; c++) F[c] = 0.0f;
  if (!DO_IS)
#pragma unroll
    for (int m = 0; m < 10; m++) F[4 + m] = 0.0f;
#if CLV_FAST
  // tolerance build, with the KT speed 1: F = 0.5 (J(A_R) + J(A_L)) -
  // 0.5 (A_R - A_L) is, for J linear in A with slope v, the weighted sum
  // cp A_L + cm A_R + (the pressure and pi part), cp = (v+1)/2, cm = (v-1)/2;
  // A_L = Q_L + s_L/2, A_R = Q_R - s_R/2 expanded into fused multiply-adds
  {
    const int va = RF_VX + a;
    const real vh = 0.5f * (L[va] + R[va]);
    const real cp = 0.5f * (vh + (real)1.0f), cm = 0.5f * (vh - (real)1.0f);
    const real hp = 0.5f * cp, hm = 0.5f * cm;
    if (DO_KT) {
      const real pt = 0.5f * (L[RF_PR] + R[RF_PR]) * tau;
      const real th = 0.5f * tau;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int mi = a == 0 ? pidx(1, c) : (a == 1 ? pidx(2, c) : pidx(3, c));
        const real p0s = L[RF_PI + c] + R[RF_PI + c];
        const real pis = L[RF_PI + mi] + R[RF_PI + mi];
        real k = (c == 0 ? pt - th * p0s : -th * p0s) * vh + th * pis;
        if (c == a + 1) k += pt;
        real f = cm * R[RF_Q0 + c] + k;
        f = f - hm * sR[c];
        f = f + cp * L[RF_Q0 + c];
        F[c] = f + hp * sL[c];
      }
    }
    if (DO_IS) {
      const real cmR = cm * R[RF_U0], cpL = cp * L[RF_U0];
#pragma unroll
      for (int m = 0; m < 10; m++) {
        real f = cmR * R[RF_PI + m] - hm * sR[4 + m];
        f = f + cpL * L[RF_PI + m];
        F[4 + m] = f + hp * sL[4 + m];
      }
    }
    (void)p;
  }
#else
  real h[4];
#pragma unroll
  for (int c = 0; c < 4; c++) h[c] = 0.5f * (L[RF_E + c] + R[RF_E + c]);
  const real vh = a == 0 ? h[1] : (a == 1 ? h[2] : h[3]);
  const real lam = max_speed<real>(p, h[0], h[1], h[2], h[3], vh);
  if (DO_KT) {
    real pr_half = 0.5f * (L[RF_PR] + R[RF_PR]);
    real pt = pr_half * tau;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      real AL = L[RF_Q0 + c] + 0.5f * sL[c];
      real AR = R[RF_Q0 + c] - 0.5f * sR[c];
      const int mi = a == 0 ? pidx(1, c) : (a == 1 ? pidx(2, c) : pidx(3, c));
      real pim0_half = 0.5f * (L[RF_PI + c] + R[RF_PI + c]);
      real pimi_half = 0.5f * (L[RF_PI + mi] + R[RF_PI + mi]);
      real g0 = c == 0 ? (real)1.0f : (real)0.0f;
      real ga = c == a + 1 ? (real)-1.0f : (real)0.0f;
      real Jp = (AR + pt * g0 - tau * pim0_half) * vh - pt * ga + tau * pimi_half;
      real Jm = (AL + pt * g0 - tau * pim0_half) * vh - pt * ga + tau * pimi_half;
      F[c] = 0.5f * (Jp + Jm) - 0.5f * lam * (AR - AL);
    }
  }
  if (DO_IS) {
    real uL = L[RF_U0], uR = R[RF_U0];
#pragma unroll
    for (int m = 0; m < 10; m++) {
      real AL = uL * L[RF_PI + m] + 0.5f * sL[4 + m];
      real AR = uR * R[RF_PI + m] - 0.5f * sR[4 + m];
      real Jp = AR * vh;
      real Jm = AL * vh;
      F[4 + m] = 0.5f * (Jp + Jm) - 0.5f * lam * (AR - AL);
    }
  }
#endif
}

// u^mu of a record
template <class real> __device__ __forceinline__ void umu_of(const real r[RF_N], real u[4]) {
  const real u0 = r[RF_U0];
  u[0] = u0 * 1.0f;
  u[1] = u0 * r[RF_VX];
  u[2] = u0 * r[RF_VY];
  u[3] = u0 * r[RF_VZ];
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
  real* const C = &s.C[0][0][0];
  real* A = &s.A[0][0][0];
  real* B = &s.B[0][0][0];
  real* const SY4 = &s.SY[0][0][0];
  real* const SY2 = &s.SYT.v[0][0];
  real* const SZ4 = &s.SZ[0][0][0];
  real* const SZ2 = &s.SZT.v[0][0];

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
  // x window: records of planes i0-2 and i0-1 (registers only), i0 (own cell
  // of C), i0+1 (A), i0+2 (B)
  real s_cur[NCOMP], F_prev[NCOMP], s_next[NCOMP], umu_prev[4];
  {
    real r0[RF_N], r1[RF_N], r2[RF_N], s_prev[NCOMP];
    make_record<real>(p, b, tau, i0 - 2, jj, kk, r0);
    make_record<real>(p, b, tau, i0 - 1, jj, kk, r1);
    make_record<real>(p, b, tau, i0, jj, kk, r2);
    rec_store<real>(C, G::NC, cself, r2);
    slopes3<real>(r0, r1, r2, s_prev);  // slope at i0-1
    make_record<real>(p, b, tau, i0 + 1, jj, kk, r0);
    rec_store<real>(A, G::NI, tid, r0);
    slopes3<real>(r1, r2, r0, s_cur);  // slope at i0
    face_flux<real, DO_IS, DO_KT>(p, tau, 0, r1, s_prev, r2, s_cur, F_prev);
    umu_of<real>(r1, umu_prev);
  }
  store_record<real>(p, b, tau, i0 + 2, jj, kk, B, G::NI, tid);
  // halo of the centre plane i0
  halo_records<real, TJ, TK>(p, b, tau, i0, j0, k0, tid, C);
  __syncthreads();

  for (int i = i0; i < i1; i++) {
    // ------------------------------------------------ slopes of plane i
    for (int q = tid; q < G::NSY + G::NSZ; q += TJ * TK) {
      real rl[RF_N], rm[RF_N], rr[RF_N], sl[NCOMP];
      if (q < G::NSY) {  // y slope at row yr-1, column zc
        int yr = q / TK, zc = q % TK;
        int cm = (yr + 1) * G::CZ + (zc + 2);
        rec_load<real>(C, G::NC, cm - G::CZ, rl);
        rec_load<real>(C, G::NC, cm, rm);
        rec_load<real>(C, G::NC, cm + G::CZ, rr);
        slopes3<real>(rl, rm, rr, sl);
        cmp_store<real>(SY4, SY2, G::NSY, q, sl);
      } else {  // z slope at row yr, column zc-1
        int qq = q - G::NSY;
        int yr = qq / (TK + 2), zc = qq % (TK + 2);
        int cm = (yr + 2) * G::CZ + (zc + 1);
        rec_load<real>(C, G::NC, cm - 1, rl);
        rec_load<real>(C, G::NC, cm, rm);
        rec_load<real>(C, G::NC, cm + 1, rr);
        slopes3<real>(rl, rm, rr, sl);
        cmp_store<real>(SZ4, SZ2, G::NSZ, qq, sl);
      }
    }
    // x slope at i+1 (own column)
    {
      real rl[RF_N], rm[RF_N], rr[RF_N];
      rec_load<real>(C, G::NC, cself, rl);
      rec_load<real>(A, G::NI, tid, rm);
      rec_load<real>(B, G::NI, tid, rr);
      slopes3<real>(rl, rm, rr, s_next);
    }
    __syncthreads();

    // ---------------------------------------------------- face fluxes
    real Fy[NCOMP], Fz[NCOMP], Fx[NCOMP];
    {
      const int sy = (tj + 1) * TK + tk;        // slope slot of own cell (y)
      const int sz = tj * (TK + 2) + (tk + 1);  // slope slot of own cell (z)
      real rs[RF_N], rn[RF_N], sa[NCOMP], sb[NCOMP], Fh[NCOMP];
      // the outer faces of the tile first, each stored at once: its slope
      // slots (row -1, column -1) are read by this thread alone, and nothing
      // of it stays live beside the three faces of the own cell
      if (tid < TK) {  // y face below row 0, column tid
        const int c0 = 1 * G::CZ + (tid + 2);
        rec_load<real>(C, G::NC, c0, rs);
        rec_load<real>(C, G::NC, c0 + G::CZ, rn);
        cmp_load<real>(SY4, SY2, G::NSY, tid, sa);
        cmp_load<real>(SY4, SY2, G::NSY, TK + tid, sb);
        face_flux<real, DO_IS, DO_KT>(p, tau, 1, rs, sa, rn, sb, Fh);
        cmp_store<real>(SY4, SY2, G::NSY, tid, Fh);
      } else if (tid < TK + TJ) {  // z face left of column 0, row tid-TK
        const int r = tid - TK;
        const int c0 = (r + 2) * G::CZ + 1;
        rec_load<real>(C, G::NC, c0, rs);
        rec_load<real>(C, G::NC, c0 + 1, rn);
        cmp_load<real>(SZ4, SZ2, G::NSZ, r * (TK + 2), sa);
        cmp_load<real>(SZ4, SZ2, G::NSZ, r * (TK + 2) + 1, sb);
        face_flux<real, DO_IS, DO_KT>(p, tau, 2, rs, sa, rn, sb, Fh);
        cmp_store<real>(SZ4, SZ2, G::NSZ, r * (TK + 2), Fh);
      }
      // the own record is read again for each face: holding its 20 values
      // across the three faces costs more registers than the reads
      rec_load<real>(C, G::NC, cself, rs);
      rec_load<real>(A, G::NI, tid, rn);
      face_flux<real, DO_IS, DO_KT>(p, tau, 0, rs, s_cur, rn, s_next, Fx);
      rec_load<real>(C, G::NC, cself, rs);
      rec_load<real>(C, G::NC, cself + G::CZ, rn);
      cmp_load<real>(SY4, SY2, G::NSY, sy, sa);
      cmp_load<real>(SY4, SY2, G::NSY, sy + TK, sb);
      face_flux<real, DO_IS, DO_KT>(p, tau, 1, rs, sa, rn, sb, Fy);
      rec_load<real>(C, G::NC, cself, rs);
      rec_load<real>(C, G::NC, cself + 1, rn);
      cmp_load<real>(SZ4, SZ2, G::NSZ, sz, sa);
      cmp_load<real>(SZ4, SZ2, G::NSZ, sz + 1, sb);
      face_flux<real, DO_IS, DO_KT>(p, tau, 2, rs, sa, rn, sb, Fz);
    }
    __syncthreads();
    // faces replace slopes: y face j+1/2 in slot (j+1), z face k+1/2 in slot (k+1)
    cmp_store<real>(SY4, SY2, G::NSY, (tj + 1) * TK + tk, Fy);
    cmp_store<real>(SZ4, SZ2, G::NSZ, tj * (TK + 2) + (tk + 1), Fz);
    __syncthreads();

    // ------------------------------------------------------ cell update
    if (inside && i < p.nx) {
      const long long I = ((long long)i * p.ny + jj) * p.nz + kk;
      real Cc[RF_N];
      rec_load<real>(C, G::NC, cself, Cc);
      CellIn<real> cin;  // the record holds gamma and P(e) of the stage input
      real* e0 = cin.e0;
      e0[0] = Cc[RF_E];
      e0[1] = Cc[RF_VX];
      e0[2] = Cc[RF_VY];
      e0[3] = Cc[RF_VZ];
      cin.g0 = Cc[RF_U0];
      cin.p0 = Cc[RF_PR];
      real pc[11];  // component 10 (bulk) unused: this kernel has no bulk sector
#pragma unroll
      for (int m = 0; m < 10; m++) pc[m] = Cc[RF_PI + m];
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
      // flux differences in the reference's order x, y, z; the y and z faces
      // (plus and minus) from shared memory, the x faces from registers
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const real D = a == 0 ? (real)p.DX : (a == 1 ? (real)p.DY : tc.dzt);
        const real rD = a == 0 ? rc.DX : (a == 1 ? rc.DY : tc.rdzt);
        real Fp[NCOMP], Fm[NCOMP];
        if (a == 1) {
          cmp_load<real>(SY4, SY2, G::NSY, (tj + 1) * TK + tk, Fp);
          cmp_load<real>(SY4, SY2, G::NSY, tj * TK + tk, Fm);
        } else if (a == 2) {
          cmp_load<real>(SZ4, SZ2, G::NSZ, tj * (TK + 2) + (tk + 1), Fp);
          cmp_load<real>(SZ4, SZ2, G::NSZ, tj * (TK + 2) + tk, Fm);
        }
#pragma unroll
        for (int c = 0; c < NCOMP; c++) {
          if (c < 4 && !DO_KT) continue;
          if (c >= 4 && !DO_IS) continue;
          real fp = a == 0 ? Fx[c] : Fp[c];
          real fm = a == 0 ? F_prev[c] : Fm[c];
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
          real rn[RF_N];
          real umc[4], umx1[4], umy0[4], umy1[4], umz0[4], umz1[4];
          umu_of<real>(Cc, umc);
          rec_load<real>(A, G::NI, tid, rn);
          umu_of<real>(rn, umx1);
          rec_load<real>(C, G::NC, cself - G::CZ, rn);
          umu_of<real>(rn, umy0);
          rec_load<real>(C, G::NC, cself + G::CZ, rn);
          umu_of<real>(rn, umy1);
          rec_load<real>(C, G::NC, cself - 1, rn);
          umu_of<real>(rn, umz0);
          rec_load<real>(C, G::NC, cself + 1, rn);
          umu_of<real>(rn, umz1);
          const real u0c = Cc[RF_U0];
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
        umu_of<real>(Cc, umu_prev);
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
      {
        real r[RF_N];
        rec_load<real>(A, G::NI, tid, r);
        rec_store<real>(C, G::NC, cself, r);
      }
      real* t = A;
      A = B;
      B = t;
      store_record<real>(p, b, tau, i + 3, jj, kk, B, G::NI, tid);
      halo_records<real, TJ, TK>(p, b, tau, i + 1, j0, k0, tid, C);
      __syncthreads();
    }
  }
  (void)acu;
}

}  // namespace CLV_ARITH
}  // namespace clv
