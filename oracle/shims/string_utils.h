/* Compile-only stand-in (oracle/_ref build only) for the reference's missing
 * "string_utils.h".  optical_flow.h includes it without using it; the joint
 * loop of ST_Tomography.cpp (:464-468) names its output files with
 * str_format(printf-format, ...) -> std::string, which this provides. */
#ifndef STT_ORACLE_SHIM_STRING_UTILS_H
#define STT_ORACLE_SHIM_STRING_UTILS_H
#include <cstdarg>
#include <cstdio>
#include <string>
static inline std::string str_format(const char *fmt, ...) {
    char buf[4096];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return std::string(buf);
}
#endif
