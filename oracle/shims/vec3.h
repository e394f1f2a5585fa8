/* Compile-only stand-in for the reference's missing "vec3.h" (oracle/_ref build
 * only).  warping.h needs geom::vec3<T> with element access, +, -, += and
 * scalar multiplication on either side. */
#ifndef STT_ORACLE_SHIM_VEC3_H
#define STT_ORACLE_SHIM_VEC3_H
namespace geom {
template <typename T> struct vec3 {
    T v[3];
    vec3() : v{T(0), T(0), T(0)} {}
    vec3(T a, T b, T c) : v{a, b, c} {}
    T &operator[](int i) { return v[i]; }
    const T &operator[](int i) const { return v[i]; }
    vec3 operator+(const vec3 &o) const { return vec3(v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]); }
    vec3 operator-(const vec3 &o) const { return vec3(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]); }
    vec3 &operator+=(const vec3 &o) { v[0] += o.v[0]; v[1] += o.v[1]; v[2] += o.v[2]; return *this; }
    vec3 &operator-=(const vec3 &o) { v[0] -= o.v[0]; v[1] -= o.v[1]; v[2] -= o.v[2]; return *this; }
};
template <typename T, typename S> vec3<T> operator*(S s, const vec3<T> &a) { return vec3<T>(T(s * a[0]), T(s * a[1]), T(s * a[2])); }
template <typename T, typename S> vec3<T> operator*(const vec3<T> &a, S s) { return vec3<T>(T(a[0] * s), T(a[1] * s), T(a[2] * s)); }
template <typename T, typename S> vec3<T> operator/(const vec3<T> &a, S s) { return vec3<T>(T(a[0] / s), T(a[1] / s), T(a[2] / s)); }
}
#endif
