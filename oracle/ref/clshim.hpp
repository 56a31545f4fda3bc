// OpenCL C on the host CPU: just enough of the OpenCL C language for the
// kernels that the reference's generators emit (KernelMatmulBuffer.hpp:174-342,
// KernelMatmulImage.hpp:190-314, KernelMatvecBuffer.hpp:180-325,
// KernelMatvecImage.hpp:185-297, KernelSaxpyBuffer.hpp:143-225) to compile
// as C++ and run one work group at a time.
//
// TEST INFRASTRUCTURE: gen_kernels.py rewrites each emitted kernel (address
// space qualifiers dropped, vector literals "(float4)(x)" turned into
// constructor calls) and compiles it against this header.  What it provides:
//  - vector types floatN / doubleN / intN / uintN with the .s0-.s3 fields the
//    generated code names, a splat constructor, and component-wise * and +;
//  - mad(): fused (one rounding, fma) when REFK_FUSED is 1, separately rounded
//    product and sum when it is 0 (built with -ffp-contract=off).  OpenCL
//    leaves the rounding of mad to the implementation; the two builds bracket
//    both choices;
//  - work-item functions answering from the running work item's ids;
//  - barrier(): a switch back to the work group's scheduler, which runs every
//    work item of the group up to the same barrier before any goes on
//    (ucontext fibers);
//  - RGBA images over row-major arrays: a texel is 16 bytes (four floats, or
//    two doubles read through read_imageui/as_double2), so an image of W/4
//    (float) or W/2 (double) texels by H rows is the row-major W x H array
//    itself (OCLAppUtil.hpp:266-286); reads use CLK_ADDRESS_NONE with
//    unnormalised coordinates, as every generated kernel does.
#pragma once

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <ucontext.h>

#ifndef REFK_FUSED
#error "define REFK_FUSED to 1 (fused mad) or 0 (separately rounded)"
#endif

namespace clshim {

// ---- vector types ---------------------------------------------------------
#define CLSHIM_VEC2(T, NAME)                                                       \
    struct NAME {                                                                  \
        T s0, s1;                                                                  \
        NAME() {}                                                                  \
        NAME(T v) : s0(v), s1(v) {}                                                \
        NAME(T a, T b) : s0(a), s1(b) {}                                           \
    };                                                                             \
    inline NAME operator*(const NAME &a, const NAME &b) { return NAME(a.s0 * b.s0, a.s1 * b.s1); } \
    inline NAME operator+(const NAME &a, const NAME &b) { return NAME(a.s0 + b.s0, a.s1 + b.s1); }

#define CLSHIM_VEC4(T, NAME)                                                       \
    struct NAME {                                                                  \
        T s0, s1, s2, s3;                                                          \
        NAME() {}                                                                  \
        NAME(T v) : s0(v), s1(v), s2(v), s3(v) {}                                  \
        NAME(T a, T b, T c, T d) : s0(a), s1(b), s2(c), s3(d) {}                   \
    };                                                                             \
    inline NAME operator*(const NAME &a, const NAME &b) {                          \
        return NAME(a.s0 * b.s0, a.s1 * b.s1, a.s2 * b.s2, a.s3 * b.s3);           \
    }                                                                              \
    inline NAME operator+(const NAME &a, const NAME &b) {                          \
        return NAME(a.s0 + b.s0, a.s1 + b.s1, a.s2 + b.s2, a.s3 + b.s3);           \
    }

CLSHIM_VEC2(float, float2)
CLSHIM_VEC4(float, float4)
CLSHIM_VEC2(double, double2)
CLSHIM_VEC4(double, double4)
CLSHIM_VEC2(int, int2)
CLSHIM_VEC4(unsigned, uint4)

// ---- mad ------------------------------------------------------------------
#if REFK_FUSED
inline float mad(float a, float b, float c) { return fmaf(a, b, c); }
inline double mad(double a, double b, double c) { return fma(a, b, c); }
#else
inline float mad(float a, float b, float c) {
    const float p = a * b;
    return p + c;
}
inline double mad(double a, double b, double c) {
    const double p = a * b;
    return p + c;
}
#endif
inline float2 mad(const float2 &a, const float2 &b, const float2 &c) {
    return float2(mad(a.s0, b.s0, c.s0), mad(a.s1, b.s1, c.s1));
}
inline float4 mad(const float4 &a, const float4 &b, const float4 &c) {
    return float4(mad(a.s0, b.s0, c.s0), mad(a.s1, b.s1, c.s1), mad(a.s2, b.s2, c.s2), mad(a.s3, b.s3, c.s3));
}
inline double2 mad(const double2 &a, const double2 &b, const double2 &c) {
    return double2(mad(a.s0, b.s0, c.s0), mad(a.s1, b.s1, c.s1));
}
inline double4 mad(const double4 &a, const double4 &b, const double4 &c) {
    return double4(mad(a.s0, b.s0, c.s0), mad(a.s1, b.s1, c.s1), mad(a.s2, b.s2, c.s2), mad(a.s3, b.s3, c.s3));
}

// ---- reinterpretation -----------------------------------------------------
inline double2 as_double2(const uint4 &u) {
    double2 d;
    memcpy(&d, &u, sizeof(d));
    return d;
}
inline uint4 as_uint4(const double2 &d) {
    uint4 u;
    memcpy(&u, &d, sizeof(u));
    return u;
}

// ---- work items -----------------------------------------------------------
struct WorkItem {
    size_t global_id[2], local_id[2], group_id[2];
    size_t local_size[2], global_size[2];
    ucontext_t ctx;
    int done;
};

struct GroupScheduler {
    ucontext_t sched;
};

extern thread_local WorkItem *tl_item;
extern thread_local GroupScheduler *tl_group;

inline size_t get_global_id(unsigned d) { return d < 2 ? tl_item->global_id[d] : 0; }
inline size_t get_local_id(unsigned d) { return d < 2 ? tl_item->local_id[d] : 0; }
inline size_t get_group_id(unsigned d) { return d < 2 ? tl_item->group_id[d] : 0; }
inline size_t get_local_size(unsigned d) { return d < 2 ? tl_item->local_size[d] : 1; }
inline size_t get_global_size(unsigned d) { return d < 2 ? tl_item->global_size[d] : 1; }
inline size_t get_num_groups(unsigned d) { return d < 2 ? tl_item->global_size[d] / tl_item->local_size[d] : 1; }

enum { CLK_LOCAL_MEM_FENCE = 1, CLK_GLOBAL_MEM_FENCE = 2 };

// Every work item of the group reaches this barrier before any goes past it:
// the item hands control back to the group's scheduler, which resumes the
// items in turn.
inline void barrier(int) { swapcontext(&tl_item->ctx, &tl_group->sched); }

// ---- images -----------------------------------------------------------------
struct Image {
    unsigned char *data;  // row-major texels of 16 bytes
    size_t width, height;  // in texels
};
typedef Image *image2d_t;
typedef int sampler_t;
enum { CLK_FILTER_NEAREST = 0, CLK_NORMALIZED_COORDS_FALSE = 0, CLK_ADDRESS_NONE = 0 };

inline const unsigned char *texel(const Image *im, const int2 &c) {
    return im->data + 16 * ((size_t)c.s1 * im->width + (size_t)c.s0);
}
inline float4 read_imagef(const Image *im, sampler_t, const int2 &c) {
    float4 v;
    memcpy(&v, texel(im, c), 16);
    return v;
}
inline uint4 read_imageui(const Image *im, sampler_t, const int2 &c) {
    uint4 v;
    memcpy(&v, texel(im, c), 16);
    return v;
}
inline void write_imagef(Image *im, const int2 &c, const float4 &v) {
    memcpy(const_cast<unsigned char *>(texel(im, c)), &v, 16);
}
inline void write_imageui(Image *im, const int2 &c, const uint4 &v) {
    memcpy(const_cast<unsigned char *>(texel(im, c)), &v, 16);
}

}  // namespace clshim
