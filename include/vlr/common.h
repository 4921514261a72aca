/* Host-side conveniences of the VLR public headers (namespace-free macros):
 * the constants and the debug assertion the C++ surface uses, as the
 * reference's libVLR/include/vlr/common.h provides them (VLR_M_PI,
 * VLR_INFINITY, VLR_NAN, VLRAssert; common.h:35-40).  VLRAssert checks only
 * when VLR_ENABLE_ASSERT is defined, and prints the message and aborts. */
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>

#if !defined(VLR_M_PI)
#define VLR_M_PI 3.14159265358979323846f
#endif
#define VLR_INFINITY (std::numeric_limits<float>::infinity())
#define VLR_NAN (std::numeric_limits<float>::quiet_NaN())

#include <limits>

#if defined(VLR_ENABLE_ASSERT)
#define VLRAssert(expr, ...) \
    do { \
        if (!(expr)) { \
            std::fprintf(stderr, "%s @%s:%d: ", #expr, __FILE__, __LINE__); \
            std::fprintf(stderr, __VA_ARGS__); \
            std::fprintf(stderr, "\n"); \
            std::abort(); \
        } \
    } while (0)
#else
#define VLRAssert(expr, ...) ((void)0)
#endif
#define VLRAssert_NotImplemented() VLRAssert(false, "Not implemented yet!")
#define VLRAssert_ShouldNotBeCalled() VLRAssert(false, "Should not be called!")
