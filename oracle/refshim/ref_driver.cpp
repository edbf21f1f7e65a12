// The reference's own hydro kernels (pyvisc/kernel/kernel_ideal.cl,
// kernel_visc.cl, kernel_IS.cl, kernel_hypersf.cl, kernel_reduction.cl with
// helper.h, eos_table.h, real_type.h, kernel_vorticity.h),
// compiled on the CPU through cl_shim.hpp, with the launch geometry of the
// reference host (ideal.py:211-255, visc.py:232-314): one work-item per cell
// for the point-wise kernels; for the kt_src_along* / visc_src_along*
// kernels one work-group of BSZ work-items per grid line, run as an OpenMP
// team so that barrier() and the work-group's __local arrays behave as on a
// device; for the surface finder one work-item per cube of the skipped grid
// (ideal.py:279-287, visc.py:378-387), elements appended through atomic_inc
// in whatever order the threads reach them. Test infrastructure: the build recipe (oracle/ref_shim.py) copies
// the kernel sources from the reference tree into a per-configuration build
// directory, rewrites their vector literals and compiles this file with the
// reference's -D constants; nothing of it is part of the library.
#include <omp.h>

#include <cstdio>
#include <cstdlib>

#include "cl_shim.hpp"

namespace clshim {
thread_local int g_gid[3];
thread_local int g_lid[3];
thread_local int g_grp[3];
thread_local int g_gsize[3];
thread_local int g_lsize[3];
}  // namespace clshim

// Each OpenCL program is built on its own; here they share one translation
// unit, so the include guards and the object-like and function-like macros
// the kernel sources define are undone between programs.
namespace ideal_prg {
#include "kernel_ideal.cl.i"
}
#include "undef_program.h"
namespace visc_prg {
#include "kernel_visc.cl.i"
#include "kernel_IS.cl.i"
}
#include "undef_program.h"
namespace hsf_prg {
#include "kernel_hypersf.cl.i"
}
#undef __REAL_TYPE__
#undef acu
namespace red_prg {
#include "kernel_reduction.cl.i"
}

typedef visc_prg::real R;
typedef visc_prg::real4 R4;

namespace {
image2d_t g_eos;
int g_team_error = 0;

template <class F> void per_cell(F f) {
#pragma omp parallel for schedule(static)
  for (int I = 0; I < SIZE; I++) {
    clshim::g_gid[0] = I;
    clshim::g_gid[1] = clshim::g_gid[2] = 0;
    clshim::g_lid[0] = clshim::g_lid[1] = clshim::g_lid[2] = 0;
    f();
  }
}

// work-groups of BSZ work-items along `axis`, one per line of the other two
template <class F> void per_line(int axis, F f) {
  const int n1 = axis == 0 ? NY : NX;
  const int n2 = axis == 2 ? NY : NZ;
  for (int a = 0; a < n1; a++)
    for (int b = 0; b < n2; b++) {
#pragma omp parallel num_threads(BSZ)
      {
        if (omp_get_num_threads() != BSZ) {
#pragma omp atomic write
          g_team_error = 1;
        } else {
          const int t = omp_get_thread_num();
          int g[3], l[3] = {0, 0, 0};
          if (axis == 0) { g[0] = t; g[1] = a; g[2] = b; }
          else if (axis == 1) { g[0] = a; g[1] = t; g[2] = b; }
          else { g[0] = a; g[1] = b; g[2] = t; }
          l[axis] = t;
          for (int d = 0; d < 3; d++) { clshim::g_gid[d] = g[d]; clshim::g_lid[d] = l[d]; }
          f();
        }
      }
    }
}

// one work-item per cube (nx, ny, nz) of the skipped grid
template <class F> void per_cube(int nx, int ny, int nz, F f) {
#pragma omp parallel for collapse(3) schedule(dynamic, 64)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        clshim::g_gid[0] = i;
        clshim::g_gid[1] = j;
        clshim::g_gid[2] = k;
        clshim::g_lid[0] = clshim::g_lid[1] = clshim::g_lid[2] = 0;
        f();
      }
}

// a one-dimensional launch of ngroups work-groups of lsize work-items, each
// work-group an OpenMP team (its __local arrays shared, barrier() a team
// barrier), one work-group after another
template <class F> void per_group_1d(int ngroups, int lsize, F f) {
  for (int g = 0; g < ngroups; g++) {
#pragma omp parallel num_threads(lsize)
    {
      if (omp_get_num_threads() != lsize) {
#pragma omp atomic write
        g_team_error = 1;
      } else {
        const int t = omp_get_thread_num();
        for (int d = 0; d < 3; d++) {
          clshim::g_gid[d] = clshim::g_lid[d] = clshim::g_grp[d] = 0;
          clshim::g_gsize[d] = clshim::g_lsize[d] = 1;
        }
        clshim::g_gid[0] = g * lsize + t;
        clshim::g_lid[0] = t;
        clshim::g_grp[0] = g;
        clshim::g_gsize[0] = ngroups * lsize;
        clshim::g_lsize[0] = lsize;
        f();
      }
    }
  }
}
}  // namespace

extern "C" {

int ref_real_size(void) { return (int)sizeof(R); }
int ref_team_error(void) { return g_team_error; }
void ref_set_eos(const float* data, int ncol, int nrow) {
  omp_set_dynamic(0);
  g_eos.data = data;
  g_eos.width = ncol;
  g_eos.height = nrow;
}

// kernel_ideal.cl
void ref_ideal_christoffel(R4* Src, R4* ev, R tau, int step) {
  per_cell([&] { ideal_prg::kt_src_christoffel(Src, ev, g_eos, tau, step); });
}
void ref_ideal_along(int axis, R4* Src, R4* ev, R tau) {
  if (axis == 0) per_line(0, [&] { ideal_prg::kt_src_alongx(Src, ev, g_eos, tau); });
  else if (axis == 1) per_line(1, [&] { ideal_prg::kt_src_alongy(Src, ev, g_eos, tau); });
  else per_line(2, [&] { ideal_prg::kt_src_alongz(Src, ev, g_eos, tau); });
}
void ref_ideal_update_ev(R4* evnew, R4* ev1, R4* Src, R tau, int step) {
  per_cell([&] { ideal_prg::update_ev(evnew, ev1, Src, g_eos, tau, step); });
}

// kernel_visc.cl
void ref_visc_christoffel(R4* Src, R4* ev, R* pi, R tau, int step) {
  per_cell([&] { visc_prg::kt_src_christoffel(Src, ev, pi, g_eos, tau, step); });
}
void ref_visc_along(int axis, R4* Src, R4* ev, R* pi, R tau) {
  if (axis == 0) per_line(0, [&] { visc_prg::kt_src_alongx(Src, ev, pi, g_eos, tau); });
  else if (axis == 1) per_line(1, [&] { visc_prg::kt_src_alongy(Src, ev, pi, g_eos, tau); });
  else per_line(2, [&] { visc_prg::kt_src_alongz(Src, ev, pi, g_eos, tau); });
}
void ref_visc_update_ev(R4* evnew, R4* ev1, R* pi1, R* pi2, R4* Src, R tau, int step) {
  per_cell([&] { visc_prg::update_ev(evnew, ev1, pi1, pi2, Src, g_eos, tau, step); });
}

// kernel_IS.cl
void ref_visc_initialize(R* pi1, R* goodcell, R4* udiff, R4* ev, R tau) {
  per_cell([&] { visc_prg::visc_initialize(pi1, goodcell, udiff, ev, tau, g_eos); });
}
void ref_visc_src_christoffel(R* Src, R* pi1, R4* ev, R tau, int step) {
  per_cell([&] { visc_prg::visc_src_christoffel(Src, pi1, ev, tau, step); });
}
void ref_visc_src_along(int axis, R* Src, R4* ud, R* pi1, R4* ev, R tau) {
  if (axis == 0) per_line(0, [&] { visc_prg::visc_src_alongx(Src, ud, pi1, ev, g_eos, tau); });
  else if (axis == 1) per_line(1, [&] { visc_prg::visc_src_alongy(Src, ud, pi1, ev, g_eos, tau); });
  else per_line(2, [&] { visc_prg::visc_src_alongz(Src, ud, pi1, ev, g_eos, tau); });
}
void ref_update_pimn(R* pinew, R* goodcell, R* pi1, R* pistep, R4* ev1, R4* ev2, R4* udiff, R4* udx, R4* udy,
                     R4* udz, R* Src, R tau, int step) {
  per_cell([&] {
    visc_prg::update_pimn(pinew, goodcell, pi1, pistep, ev1, ev2, udiff, udx, udy, udz, Src, g_eos, tau, step);
  });
}
void ref_get_udiff(R4* udiff, R4* ev0, R4* ev1) {
  per_cell([&] { visc_prg::get_udiff(udiff, ev0, ev1); });
}

// kernel_reduction.cl's first stage with the reference's launch, 64
// work-groups of 256 (ideal.py:259-262): semi[64] gets each group's maximum
void ref_reduction_stage1(R4* x, R* semi, int size) {
  per_group_1d(REDUCTION_NBlocks, REDUCTION_BSZ, [&] { red_prg::reduction_stage1(x, semi, size); });
}

// kernel_hypersf.cl; sf, txyz, pisf (and the vorticity outputs) must hold one
// element per cube: the kernel has no capacity check
int ref_get_hypersf(hsf_prg::real8* sf, R4* txyz, R4* ev_old, R4* ev_new, R t_old, R t_new) {
  const int nx = (NX - 1) / nxskip + 1, ny = (NY - 1) / nyskip + 1, nz = (NZ - 1) / nzskip + 1;
  int n = 0;
  per_cube(nx, ny, nz, [&] { hsf_prg::get_hypersf(sf, txyz, &n, ev_old, ev_new, t_old, t_new); });
  return n;
}
int ref_visc_hypersf(hsf_prg::real8* sf, R4* txyz, R* pisf, R4* ev_old, R4* ev_new, R* pi_old, R* pi_new,
                     R* om_sf, R* om_old, R* om_new, R* s1_sf, R* s1_old, R* s1_new, R* s2_sf, R* s2_old,
                     R* s2_new, R* at_sf, R* at_old, R* at_new, R t_old, R t_new) {
  const int nx = (NX - 1) / nxskip + 1, ny = (NY - 1) / nyskip + 1, nz = (NZ - 1) / nzskip + 1;
  int n = 0;
  per_cube(nx, ny, nz, [&] {
    hsf_prg::visc_hypersf(sf, txyz, pisf, &n, ev_old, ev_new, pi_old, pi_new, om_sf, om_old, om_new, s1_sf, s1_old,
                          s1_new, s2_sf, s2_old, s2_new, at_sf, at_old, at_new, t_old, t_new);
  });
  return n;
}

}  // extern "C"
