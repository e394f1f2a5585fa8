/* Compile-only stand-in (oracle/_ref build only): optical_flow.h aliases this
 * namespace but calls nothing in it. */
#ifndef STT_ORACLE_SHIM_LINEAR_SOLVER_H
#define STT_ORACLE_SHIM_LINEAR_SOLVER_H
namespace linear_solver {}
#endif
