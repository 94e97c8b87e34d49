// cl_compat.hpp -- OpenCL C 1.2 compatibility layer for compiling bismit's
// kernel sources (cl/bismit.cl, cl/syns.cl, cl/control.cl, cl/tests.cl) as
// C++20 for the CPU. TEST INFRASTRUCTURE: it exists so the CPU oracle can be
// pinned against the reference's own kernel code.
//
// Everything lives in namespace clref; the prepared kernel text is included
// inside the same namespace so these builtins shadow the C library's.
//
// Semantics implemented (OpenCL C 1.2, section 6):
//  * scalar arithmetic follows C99 integer promotion; C++20 gives the same
//    wrap-around for signed left shifts and arithmetic right shifts;
//  * vector arithmetic happens in the element type (u8 vectors wrap at 8 bits);
//  * vector relational operators return -1 (all bits) / 0 in a signed vector of
//    the same element width;
//  * shift counts of vector shifts are taken modulo the element width;
//  * convert_* are plain (non-saturating) conversions;
//  * abs() returns the unsigned type of its argument;
//  * mul24/mad24 are exact 32-bit products (bismit only calls them with
//    operands inside the 24-bit range, where the two agree).
#pragma once
#include <cstddef>
#include <cstdint>
#include <type_traits>

namespace clref {

typedef unsigned char  uchar;
typedef unsigned short ushort;
typedef unsigned int   uint;

// ------------------------------------------------------------- NDRange ----
struct NDRange {
    size_t gsz[3] = {1, 1, 1};
    size_t lsz[3] = {1, 1, 1};
    size_t gid[3] = {0, 0, 0};
    size_t lid[3] = {0, 0, 0};
};
inline thread_local NDRange ndr;

inline size_t get_global_id(uint d) { return d < 3 ? ndr.gid[d] : 0; }
inline size_t get_global_size(uint d) { return d < 3 ? ndr.gsz[d] : 1; }
inline size_t get_local_id(uint d) { return d < 3 ? ndr.lid[d] : 0; }
inline size_t get_local_size(uint d) { return d < 3 ? ndr.lsz[d] : 1; }

// -------------------------------------------------------------- vectors ---
template <class T> struct vec4 {
    T s0, s1, s2, s3;
    vec4() = default;
    vec4(T a) : s0(a), s1(a), s2(a), s3(a) {}
    template <class A, class B, class C, class D>
    vec4(A a, B b, C c, D d) : s0((T)a), s1((T)b), s2((T)c), s3((T)d) {}
    T& operator[](int i) { return (&s0)[i]; }
    const T& operator[](int i) const { return (&s0)[i]; }
};

typedef vec4<char>  char4;
typedef vec4<uchar> uchar4;
typedef vec4<int>   int4;
typedef vec4<uint>  uint4;

// Signed vector type of the same element width (relational results).
template <class T> struct rel_of;
template <> struct rel_of<char> { typedef char type; };
template <> struct rel_of<uchar> { typedef char type; };
template <> struct rel_of<int> { typedef int type; };
template <> struct rel_of<uint> { typedef int type; };

template <class T> constexpr int bits_of() { return (int)sizeof(T) * 8; }

#define CLREF_VEC_BINOP(OP)                                                     \
    template <class T> inline vec4<T> operator OP(vec4<T> a, vec4<T> b) {       \
        vec4<T> r;                                                              \
        for (int i = 0; i < 4; i++) r[i] = (T)(a[i] OP b[i]);                   \
        return r;                                                               \
    }                                                                           \
    template <class T, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>> \
    inline vec4<T> operator OP(vec4<T> a, S b) { return a OP vec4<T>((T)b); }   \
    template <class T, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>> \
    inline vec4<T> operator OP(S a, vec4<T> b) { return vec4<T>((T)a) OP b; }

CLREF_VEC_BINOP(+)
CLREF_VEC_BINOP(-)
CLREF_VEC_BINOP(*)
CLREF_VEC_BINOP(&)
CLREF_VEC_BINOP(|)
CLREF_VEC_BINOP(^)
#undef CLREF_VEC_BINOP

template <class T> inline vec4<T> operator<<(vec4<T> a, vec4<T> b) {
    vec4<T> r;
    for (int i = 0; i < 4; i++) {
        typedef std::make_unsigned_t<T> U;
        r[i] = (T)(U)((U)a[i] << ((int)b[i] & (bits_of<T>() - 1)));
    }
    return r;
}
template <class T> inline vec4<T> operator>>(vec4<T> a, vec4<T> b) {
    vec4<T> r;
    for (int i = 0; i < 4; i++) r[i] = (T)(a[i] >> ((int)b[i] & (bits_of<T>() - 1)));
    return r;
}
template <class T, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>
inline vec4<T> operator<<(vec4<T> a, S b) { return a << vec4<T>((T)b); }
template <class T, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>
inline vec4<T> operator>>(vec4<T> a, S b) { return a >> vec4<T>((T)b); }

template <class T> inline vec4<T> operator-(vec4<T> a) {
    vec4<T> r;
    for (int i = 0; i < 4; i++) r[i] = (T)(-a[i]);
    return r;
}
template <class T> inline vec4<T> operator~(vec4<T> a) {
    vec4<T> r;
    for (int i = 0; i < 4; i++) r[i] = (T)(~a[i]);
    return r;
}

#define CLREF_VEC_REL(OP)                                                        \
    template <class T> inline vec4<typename rel_of<T>::type> operator OP(vec4<T> a, vec4<T> b) { \
        vec4<typename rel_of<T>::type> r;                                        \
        for (int i = 0; i < 4; i++) r[i] = (a[i] OP b[i]) ? -1 : 0;              \
        return r;                                                                \
    }                                                                            \
    template <class T, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>> \
    inline vec4<typename rel_of<T>::type> operator OP(vec4<T> a, S b) { return a OP vec4<T>((T)b); } \
    template <class T, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>> \
    inline vec4<typename rel_of<T>::type> operator OP(S a, vec4<T> b) { return vec4<T>((T)a) OP b; }

CLREF_VEC_REL(==)
CLREF_VEC_REL(!=)
CLREF_VEC_REL(<)
CLREF_VEC_REL(>)
CLREF_VEC_REL(<=)
CLREF_VEC_REL(>=)
#undef CLREF_VEC_REL

template <class D, class S> inline vec4<D> convert_vec(vec4<S> a) {
    return vec4<D>((D)a.s0, (D)a.s1, (D)a.s2, (D)a.s3);
}
template <class S> inline int4 convert_int4(vec4<S> a) { return convert_vec<int>(a); }
template <class S> inline uint4 convert_uint4(vec4<S> a) { return convert_vec<uint>(a); }
template <class S> inline uchar4 convert_uchar4(vec4<S> a) { return convert_vec<uchar>(a); }
template <class S> inline char4 convert_char4(vec4<S> a) { return convert_vec<char>(a); }

// ------------------------------------------------------------- builtins ---
template <class A, class B, class = std::enable_if_t<std::is_arithmetic_v<A> && std::is_arithmetic_v<B>>>
inline auto mul24(A a, B b) -> decltype(a * b) {
    typedef decltype(a * b) R;
    typedef std::make_unsigned_t<R> U;
    return (R)((U)(R)a * (U)(R)b);
}
template <class A, class B, class C,
          class = std::enable_if_t<std::is_arithmetic_v<A> && std::is_arithmetic_v<B> && std::is_arithmetic_v<C>>>
inline auto mad24(A a, B b, C c) -> decltype(a * b + c) {
    typedef decltype(a * b + c) R;
    typedef std::make_unsigned_t<R> U;
    return (R)((U)(R)a * (U)(R)b + (U)(R)c);
}
template <class T> inline vec4<T> mul24(vec4<T> a, vec4<T> b) {
    vec4<T> r;
    for (int i = 0; i < 4; i++) r[i] = mul24(a[i], b[i]);
    return r;
}
template <class T> inline vec4<T> mad24(vec4<T> a, vec4<T> b, vec4<T> c) {
    vec4<T> r;
    for (int i = 0; i < 4; i++) r[i] = mad24(a[i], b[i], c[i]);
    return r;
}

template <class T> inline T clamp(T x, T lo, T hi) { return x < lo ? lo : (x > hi ? hi : x); }
template <class T> inline T min(T a, T b) { return b < a ? b : a; }
template <class T> inline T max(T a, T b) { return a < b ? b : a; }

inline uchar abs(char x) { return (uchar)(x < 0 ? -(int)x : (int)x); }
inline uchar abs(uchar x) { return x; }
inline ushort abs(short x) { return (ushort)(x < 0 ? -(int)x : (int)x); }
inline uint abs(int x) { return x < 0 ? (uint)0 - (uint)x : (uint)x; }
inline uint abs(uint x) { return x; }

}  // namespace clref

// OpenCL address-space and function qualifiers compile to nothing.
#define __kernel
#define __global
#define __local
#define __private
#define __constant
