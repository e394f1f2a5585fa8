/* Compile-only stand-in (oracle/_ref build only): the reference's cg.h names
 * these helpers inside a template that nothing instantiates. */
#ifndef STT_ORACLE_SHIM_IMAGE_BLAS_H
#define STT_ORACLE_SHIM_IMAGE_BLAS_H
namespace image_blas {
template <typename A> A scaled(const A &a, double) { return a; }
template <typename A, typename B> void add(const A &, B &) {}
template <typename A, typename B, typename C> void add(const A &, const B &, C &) {}
template <typename A, typename B> void copy(const A &, B &) {}
template <typename R, typename A, typename B> R dot(const A &, const B &) { return R(0); }
}
#endif
