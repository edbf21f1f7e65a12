// OpenCL C shim for compiling the reference's kernel sources with g++ (test
// infrastructure: the reference's own kernels run on the CPU, to check the
// oracle's restatement against them).
//
// What the reference's hydro kernels (pyvisc/kernel/helper.h, eos_table.h,
// kernel_ideal.cl, kernel_visc.cl, kernel_IS.cl, kernel_hypersf.cl,
// kernel_vorticity.h, kernel_reduction.cl) use of OpenCL C, given a C++
// meaning here:
//  * vector types float3/4/8, double3/4/8, int2 with .x..w / .s0..s3 / .s123
//    members and element-wise arithmetic; the literal (real4)(a, b, c, d) is
//    rewritten to the braced list real4{a, b, c, d} by the build recipe (C++
//    would read the literal as a cast of a comma expression; a braced list
//    also fixes the left-to-right evaluation of its elements);
//  * address-space and kernel qualifiers (empty), __local (static: one copy
//    shared by the work-group, whose work-items run as one OpenMP team);
//  * work-item functions (ids, sizes, group id) from per-thread state the
//    launcher sets; barrier() is an OpenMP barrier of the team; MAXFLOAT;
//  * min/max/sign with OpenCL's semantics; dot; the image read of the EOS
//    table (clamp-to-edge, nearest) returning its four float32 channels;
//  * atomic_inc (kernel_hypersf.cl's element counter).
// Arithmetic is IEEE: the recipe builds with -ffp-contract=off and no fast
// math, as the oracle is built, and -fwrapv (the 32-bit wrap of the surface
// finder's random-number step, kernel_hypersf.cl:126-132).
#pragma once
#include <cfloat>
#include <cmath>
#include <omp.h>

#define __kernel
#define __global
#define __private
#define __constant const
#define constant
#define read_only
#define __local static
#define M_PI_F 3.14159265358979323846f
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
#define CLK_NORMALIZED_COORDS_FALSE 0
#define CLK_ADDRESS_CLAMP_TO_EDGE 0
#define CLK_FILTER_NEAREST 0
typedef int sampler_t;

namespace clshim {
extern thread_local int g_gid[3];
extern thread_local int g_lid[3];
extern thread_local int g_grp[3];
extern thread_local int g_gsize[3];
extern thread_local int g_lsize[3];
}  // namespace clshim
inline int get_global_id(int d) { return clshim::g_gid[d]; }
inline int get_local_id(int d) { return clshim::g_lid[d]; }
inline int get_group_id(int d) { return clshim::g_grp[d]; }
inline int get_global_size(int d) { return clshim::g_gsize[d]; }
inline int get_local_size(int d) { return clshim::g_lsize[d]; }
#define MAXFLOAT FLT_MAX
inline void barrier(int) {
#pragma omp barrier
}

template <class T> struct vec3 {
  union {
    struct { T x, y, z; };
    struct { T s0, s1, s2; };
  };
};
template <class T> struct vec4 {
  union {
    struct { T x, y, z, w; };
    struct { T s0, s1, s2, s3; };
    struct { T s0_; vec3<T> s123; };
    T v[4];
  };
  vec4() = default;
  vec4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
  explicit vec4(T a) : x(a), y(a), z(a), w(a) {}
  vec4(T a, vec3<T> v) : x(a), y(v.x), z(v.y), w(v.z) {}
  template <class U> vec4(const vec4<U>& o) : x((T)o.x), y((T)o.y), z((T)o.z), w((T)o.w) {}
};
template <class T> struct vec8 {
  T s[8];
  vec8() = default;
  vec8(T a, T b, T c, T d, T e, T f, T g, T h) : s{a, b, c, d, e, f, g, h} {}
};
struct int2 {
  int x, y;
  int2(int a, int b) : x(a), y(b) {}
};

typedef vec3<float> float3;
typedef vec4<float> float4;
typedef vec8<float> float8;
typedef vec3<double> double3;
typedef vec4<double> double4;
typedef vec8<double> double8;

template <class T> inline vec4<T> operator+(vec4<T> a, vec4<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class T> inline vec4<T> operator-(vec4<T> a, vec4<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
template <class T> inline vec4<T> operator*(vec4<T> a, vec4<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
template <class T> inline vec4<T> operator/(vec4<T> a, vec4<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w}; }
template <class T> inline vec4<T> operator-(vec4<T> a) { return {-a.x, -a.y, -a.z, -a.w}; }
// scalar with vector: the scalar is converted to the element type first
// (OpenCL's widening of a scalar operand)
template <class T, class S> inline vec4<T> operator*(S s, vec4<T> a) { T t = (T)s; return {t * a.x, t * a.y, t * a.z, t * a.w}; }
template <class T, class S> inline vec4<T> operator*(vec4<T> a, S s) { T t = (T)s; return {a.x * t, a.y * t, a.z * t, a.w * t}; }
template <class T, class S> inline vec4<T> operator/(vec4<T> a, S s) { T t = (T)s; return {a.x / t, a.y / t, a.z / t, a.w / t}; }
template <class T, class S> inline vec4<T> operator+(vec4<T> a, S s) { T t = (T)s; return {a.x + t, a.y + t, a.z + t, a.w + t}; }
template <class T, class S> inline vec4<T> operator-(vec4<T> a, S s) { T t = (T)s; return {a.x - t, a.y - t, a.z - t, a.w - t}; }
template <class T> inline vec4<T>& operator+=(vec4<T>& a, vec4<T> b) { a = a + b; return a; }
template <class T> inline vec4<T>& operator-=(vec4<T>& a, vec4<T> b) { a = a - b; return a; }
template <class T, class S> inline vec4<T>& operator/=(vec4<T>& a, S s) { a = a / s; return a; }

// OpenCL dot(): sum of products, left to right, separate roundings
template <class T> inline T dot(vec4<T> a, vec4<T> b) {
  T r = a.x * b.x;
  r = r + a.y * b.y;
  r = r + a.z * b.z;
  r = r + a.w * b.w;
  return r;
}
template <class T> inline T dot(vec3<T> a, vec3<T> b) {
  T r = a.x * b.x;
  r = r + a.y * b.y;
  r = r + a.z * b.z;
  return r;
}

// OpenCL min / max (y if x < y, else x, for max) and sign
template <class A, class B> inline auto max(A a, B b) -> decltype(a + b) {
  typedef decltype(a + b) T;
  return ((T)a < (T)b) ? (T)b : (T)a;
}
template <class A, class B> inline auto min(A a, B b) -> decltype(a + b) {
  typedef decltype(a + b) T;
  return ((T)b < (T)a) ? (T)b : (T)a;
}
inline float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : (x != x ? 0.0f : x)); }
inline double sign(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : (x != x ? 0.0 : x)); }
using std::exp;
using std::fabs;
// the element-wise vector forms (minmod4 in helper.h)
template <class T> inline vec4<T> fabs(vec4<T> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z), std::fabs(a.w)}; }
template <class T> inline vec4<T> sign(vec4<T> a) { return {sign(a.x), sign(a.y), sign(a.z), sign(a.w)}; }
template <class T> inline vec4<T> min(vec4<T> a, vec4<T> b) {
  return {min(a.x, b.x), min(a.y, b.y), min(a.z, b.z), min(a.w, b.w)};
}
using std::fmax;
using std::pow;
using std::sqrt;
using std::atanh;
using std::cosh;
using std::isnan;
using std::sinh;
using std::tanh;
// atomic_inc on a global counter (the surface element index)
inline int atomic_inc(volatile int* p) { return __atomic_fetch_add(p, 1, __ATOMIC_RELAXED); }

// the EOS image: nrow x ncol texels of four float32 channels, row-major;
// clamp-to-edge, nearest
struct image2d_t {
  const float* data;
  int width, height;  // columns, rows
};
inline float4 read_imagef(image2d_t im, sampler_t, int2 c) {
  int x = c.x < 0 ? 0 : (c.x >= im.width ? im.width - 1 : c.x);
  int y = c.y < 0 ? 0 : (c.y >= im.height ? im.height - 1 : c.y);
  const float* t = im.data + 4 * ((long)y * im.width + x);
  return float4(t[0], t[1], t[2], t[3]);
}
