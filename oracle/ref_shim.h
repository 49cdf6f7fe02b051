/* OpenCL C builtins for compiling the reference's own kernel source
 * (cl-files/ImageProximity.cl) as host C++.
 *
 * TEST INFRASTRUCTURE ONLY: this header is part of the oracle. Nothing in the
 * shipped library includes it.
 *
 * The reference kernels are written against OpenCL C 1.1. They use address
 * space qualifiers (global/local), scalar and vector pixel types selected by
 * -D <TYPE> [-D NBCHAN=n] (cl-files/Buffers.h:28-101), convert_<type>(),
 * fabs/sqrt, get_global_id/get_local_id/get_local_size and one barrier() in
 * each _Cached kernel (cl-files/ImageProximity.cl:91 and siblings).
 *
 * Work-item ids live in thread_local variables set by the driver loop
 * (ref_proximity.cpp). `local` arrays become static thread_local so that the
 * work-items of an emulated work-group share them; the driver runs every
 * work-group twice (first pass fills the local cache, second pass computes),
 * which reproduces the barrier semantics of the _Cached kernels exactly because
 * the cache fill is a pure function of the template.
 */
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>

typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;

#define kernel
#define global
#define constant
#define local static thread_local
#define CLK_LOCAL_MEM_FENCE 0
#define CLK_GLOBAL_MEM_FENCE 0

namespace oclshim {
extern thread_local int g_gid[2];
extern thread_local int g_lid[2];
extern thread_local int g_lsize[2];
extern thread_local int g_grp[2];
}  // namespace oclshim

static inline int get_global_id(int d) { return oclshim::g_gid[d]; }
static inline int get_local_id(int d) { return oclshim::g_lid[d]; }
static inline int get_local_size(int d) { return oclshim::g_lsize[d]; }
static inline int get_group_id(int d) { return oclshim::g_grp[d]; }
static inline void barrier(int) {}

/* Single-precision overloads (the double ones come from <math.h>): a float
 * argument must give a float result, as in OpenCL C. */
static inline float fabs(float a) { return std::fabs(a); }
static inline float sqrt(float a) { return std::sqrt(a); }

/* OpenCL vector types: element-wise arithmetic, broadcast from a scalar,
 * .x/.y/.z/.w members and brace construction (`int2 Pos = {gx2, y};`). */
template <class T, int N>
struct clvec_storage;
template <class T>
struct clvec_storage<T, 2> {
  union {
    T s[2];
    struct { T x, y; };
  };
};
template <class T>
struct clvec_storage<T, 4> {
  union {
    T s[4];
    struct { T x, y, z, w; };
  };
};

template <class T, int N>
struct clvec : clvec_storage<T, N> {
  clvec() = default;
  template <class S>
  clvec(S v) {  // NOLINT: implicit broadcast, as `REAL sum = 0;` needs
    for (int i = 0; i < N; ++i) this->s[i] = T(v);
  }
  template <class U>
  clvec(const clvec<U, N>& o) {  // NOLINT: element-wise conversion
    for (int i = 0; i < N; ++i) this->s[i] = T(o.s[i]);
  }
  template <class A, class B, class... R>
  clvec(A a, B b, R... r) {
    const T v[N] = {T(a), T(b), T(r)...};
    for (int i = 0; i < N; ++i) this->s[i] = v[i];
  }
  template <class U>
  clvec& operator+=(const clvec<U, N>& b) {
    for (int i = 0; i < N; ++i) this->s[i] += b.s[i];
    return *this;
  }
};
#define CLVEC_OP(op)                                                       \
  template <class T, class U, int N>                                       \
  static inline auto operator op(const clvec<T, N>& a, const clvec<U, N>& b) \
      ->clvec<decltype(a.s[0] op b.s[0]), N> {                             \
    clvec<decltype(a.s[0] op b.s[0]), N> r;                                \
    for (int i = 0; i < N; ++i) r.s[i] = a.s[i] op b.s[i];                 \
    return r;                                                              \
  }
CLVEC_OP(+)
CLVEC_OP(-)
CLVEC_OP(*)
CLVEC_OP(/)
#undef CLVEC_OP

/* Contracted arithmetic (built with -DOCLSHIM_FUSED): `float` and `double`
 * in the reference source become freal<F>, whose product is kept unrounded
 * (fprod) until it is either added to an accumulator with `+=` -- one fused
 * multiply-add, fma(a, b, acc), which is how an OpenCL compiler contracts
 * `acc += a * b` -- or used in any other way, which rounds it first. */
#ifdef OCLSHIM_FUSED
template <class F>
struct fprod {
  F a, b;
  operator F() const { return a * b; }
};
template <class F>
struct freal {
  F v;
  freal() = default;
  template <class S>
  freal(S x) : v(F(x)) {}  // NOLINT
  freal(fprod<F> p) : v(p.a * p.b) {}  // NOLINT
  freal& operator+=(fprod<F> p) {
    v = std::fma(p.a, p.b, v);
    return *this;
  }
  freal& operator+=(freal o) {
    v = v + o.v;
    return *this;
  }
};
template <class F> static inline fprod<F> operator*(freal<F> a, freal<F> b) { return {a.v, b.v}; }
template <class F> static inline freal<F> operator-(freal<F> a, freal<F> b) { return freal<F>(a.v - b.v); }
template <class F> static inline freal<F> operator+(freal<F> a, freal<F> b) { return freal<F>(a.v + b.v); }
template <class F> static inline freal<F> operator/(freal<F> a, freal<F> b) { return freal<F>(a.v / b.v); }
template <class F> static inline freal<F> fabs(freal<F> a) { return freal<F>(std::fabs(a.v)); }
template <class F> static inline freal<F> sqrt(freal<F> a) { return freal<F>(std::sqrt(a.v)); }
template <class F> static inline freal<F> sqrt(fprod<F> p) { return freal<F>(std::sqrt(p.a * p.b)); }
#endif

#define CLVEC_TYPES(base)              \
  typedef clvec<base, 2> base##2;      \
  typedef clvec<base, 4> base##4;
CLVEC_TYPES(uchar)
CLVEC_TYPES(char)
CLVEC_TYPES(ushort)
CLVEC_TYPES(short)
CLVEC_TYPES(uint)
CLVEC_TYPES(int)
CLVEC_TYPES(float)
CLVEC_TYPES(double)
#undef CLVEC_TYPES

template <class T, int N>
static inline clvec<T, N> fabs(const clvec<T, N>& a) {
  clvec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = fabs(a.s[i]);
  return r;
}
template <class T, int N>
static inline auto sqrt(const clvec<T, N>& a) -> clvec<decltype(sqrt(a.s[0])), N> {
  clvec<decltype(sqrt(a.s[0])), N> r;
  for (int i = 0; i < N; ++i) r.s[i] = sqrt(a.s[i]);
  return r;
}

/* convert_<REAL>(value): plain value conversion (round-to-nearest for the
 * integer-to-float case, which is exact for every type narrower than 24 bits). */
template <class D, class S>
static inline D oclshim_convert(S v) { return D(v); }
template <class D, class S, int N>
static inline clvec<D, N> oclshim_convert_vec(const clvec<S, N>& v) {
  clvec<D, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = D(v.s[i]);
  return r;
}
#define CLCONV_SCALAR(D)                                              \
  template <class S>                                                  \
  static inline D convert_##D(S v) { return oclshim_convert<D>(v); }
CLCONV_SCALAR(float)
CLCONV_SCALAR(double)
#undef CLCONV_SCALAR
#define CLCONV_VEC(D, N)                                                   \
  template <class S>                                                       \
  static inline clvec<D, N> convert_##D##N(const clvec<S, N>& v) {         \
    return oclshim_convert_vec<D>(v);                                      \
  }
CLCONV_VEC(float, 2)
CLCONV_VEC(float, 4)
CLCONV_VEC(double, 2)
CLCONV_VEC(double, 4)
#undef CLCONV_VEC

#ifdef OCLSHIM_FUSED
/* The reference source's `float` and `double` (through REAL, SCALAR and
 * DOUBLE of cl-files/Buffers.h) name the contracted types from here on. The
 * macros expand to single identifiers so that the source's token pasting
 * (convert_##REAL, REAL##4) still forms valid names. */
typedef freal<float> oclf32;
typedef freal<double> oclf64;
typedef clvec<oclf32, 2> oclf322;
typedef clvec<oclf32, 4> oclf324;
typedef clvec<oclf64, 2> oclf642;
typedef clvec<oclf64, 4> oclf644;
template <class S> static inline oclf32 convert_oclf32(S v) { return oclf32(v); }
template <class S> static inline oclf64 convert_oclf64(S v) { return oclf64(v); }
template <class S> static inline oclf322 convert_oclf322(const clvec<S, 2>& v) { return oclf322(v); }
template <class S> static inline oclf324 convert_oclf324(const clvec<S, 4>& v) { return oclf324(v); }
template <class S> static inline oclf642 convert_oclf642(const clvec<S, 2>& v) { return oclf642(v); }
template <class S> static inline oclf644 convert_oclf644(const clvec<S, 4>& v) { return oclf644(v); }
#define float oclf32
#define double oclf64
#endif
