// Host-only stand-in for the reference's OptiX/CUDA utility header.
//
// TEST INFRASTRUCTURE ONLY. This file lets the reference's own spectral and
// BSDF sources (libVLR/shared/*, libVLR/GPU_kernels/materials.cu) compile as
// plain host C++ so they can serve as the parity oracle.  It replaces
// libVLR/utils/optixu_on_cudau.h, which pulls in the OptiX SDK
// (libVLR/utils/optix_util.h:283-286) that does not exist here.
//
// Nothing in the shipped library includes this file.
#pragma once

#include <cstdint>
#include <cstddef>
#include <type_traits>
#include <cstring>
#include <cstdlib>
#include <cuda.h>
#include <vector_types.h>
#include <vector_functions.h>

// Host compilation: every device qualifier collapses to plain inline C++.
#define CUDA_SHARED_MEM
#define CUDA_CONSTANT_MEM
#define CUDA_DEVICE_MEM
#define CUDA_DEVICE_KERNEL extern "C"
#define CUDA_INLINE inline
#define CUDA_DEVICE_FUNCTION
#define CUDA_COMMON_FUNCTION
#define RT_DEVICE_FUNCTION inline
#define RT_COMMON_FUNCTION inline
#define RT_FUNCTION inline
#define RT_CALLABLE_PROGRAM static inline
#define RT_PIPELINE_LAUNCH_PARAMETERS
#define RT_DC_NAME(name) __direct_callable__ ## name
#define RT_AH_NAME(name) __anyhit__ ## name
#define RT_CH_NAME(name) __closesthit__ ## name
#define RT_MS_NAME(name) __miss__ ## name
#define RT_RG_NAME(name) __raygen__ ## name
#define RT_IS_NAME(name) __intersection__ ## name
#define RT_DC_NAME_STR(name) "__direct_callable__" name

typedef unsigned long long OptixTraversableHandle;

namespace optixu {
    // Callable IDs are only stored in descriptors on the host side of the
    // oracle; invoking one is never needed because the oracle calls the BSDF
    // classes directly.
    template <typename FuncType>
    class DirectCallableProgramID;

    template <typename R, typename... Args>
    class DirectCallableProgramID<R(Args...)> {
        uint32_t m_sbtIndex;
    public:
        DirectCallableProgramID() : m_sbtIndex(0) {}
        explicit DirectCallableProgramID(uint32_t sbtIndex) : m_sbtIndex(sbtIndex) {}
        explicit operator uint32_t() const { return m_sbtIndex; }
        // Only the Multi material dispatches through callables; the oracle
        // never builds one, so reaching this is a harness bug.
        template <typename... CallArgs>
        R operator()(CallArgs&&...) const { std::abort(); }
    };

    template <typename... PayloadTypes>
    struct PayloadSignature {};

    template <typename... AttributeTypes>
    struct AttributeSignature {};

    template <typename T>
    class NativeBlockBuffer2D {
        CUsurfObject m_surfObject;
    public:
        NativeBlockBuffer2D() : m_surfObject(0) {}
        NativeBlockBuffer2D(CUsurfObject s) : m_surfObject(s) {}
    };

    template <typename T, uint32_t log2BlockWidth>
    class BlockBuffer2D {
        T* m_rawBuffer;
        uint32_t m_width, m_height;
    public:
        BlockBuffer2D() : m_rawBuffer(nullptr), m_width(0), m_height(0) {}
    };
}
