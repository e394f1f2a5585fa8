/* Compile-only stand-in (oracle/_ref build only) for the reference's missing
 * "scope.h".  optical_flow.h expands utilities_scope_defines at file scope and
 * then uses cout/endl and the imagelist type unqualified. */
#ifndef STT_ORACLE_SHIM_SCOPE_H
#define STT_ORACLE_SHIM_SCOPE_H
#include <iostream>
#define utilities_scope_defines \
    using std::cout;            \
    using std::endl;            \
    typedef cimg_library::CImgList<float> imagelist;
#endif
