/* Definitions for the compile-only OpenCL header in CL/cl.h.
 *
 * TEST INFRASTRUCTURE: the reference's print_* tools link against the
 * reference's OpenCL wrapper (OCLBase / OCLApp), which names these
 * functions, but only emit kernel source and never call them.  Every
 * function here fails (CL_INVALID_PLATFORM, or NULL with that error code),
 * so a tool that did reach the runtime would stop with an error instead of
 * touching any device.
 */
#include "CL/cl.h"

#define FAIL_HANDLE(T)                                      \
    do {                                                    \
        if (errcode_ret) *errcode_ret = CL_INVALID_PLATFORM; \
        return (T)0;                                        \
    } while (0)

cl_int clGetPlatformIDs(cl_uint n, cl_platform_id *p, cl_uint *np) {
    (void)n, (void)p;
    if (np) *np = 0;
    return CL_INVALID_PLATFORM;
}
cl_int clGetDeviceIDs(cl_platform_id p, cl_device_type t, cl_uint n, cl_device_id *d, cl_uint *nd) {
    (void)p, (void)t, (void)n, (void)d;
    if (nd) *nd = 0;
    return CL_INVALID_PLATFORM;
}
cl_int clGetDeviceInfo(cl_device_id d, cl_device_info i, size_t s, void *v, size_t *r) {
    (void)d, (void)i, (void)s, (void)v, (void)r;
    return CL_INVALID_PLATFORM;
}
cl_context clCreateContext(const cl_context_properties *p, cl_uint n, const cl_device_id *d,
                           void (*f)(const char *, const void *, size_t, void *), void *u, cl_int *errcode_ret) {
    (void)p, (void)n, (void)d, (void)f, (void)u;
    FAIL_HANDLE(cl_context);
}
cl_int clReleaseContext(cl_context c) { (void)c; return CL_INVALID_PLATFORM; }
cl_command_queue clCreateCommandQueue(cl_context c, cl_device_id d, cl_command_queue_properties p,
                                      cl_int *errcode_ret) {
    (void)c, (void)d, (void)p;
    FAIL_HANDLE(cl_command_queue);
}
cl_int clReleaseCommandQueue(cl_command_queue q) { (void)q; return CL_INVALID_PLATFORM; }
cl_mem clCreateBuffer(cl_context c, cl_mem_flags f, size_t s, void *h, cl_int *errcode_ret) {
    (void)c, (void)f, (void)s, (void)h;
    FAIL_HANDLE(cl_mem);
}
cl_mem clCreateImage2D(cl_context c, cl_mem_flags f, const cl_image_format *fmt, size_t w, size_t h, size_t p,
                       void *ptr, cl_int *errcode_ret) {
    (void)c, (void)f, (void)fmt, (void)w, (void)h, (void)p, (void)ptr;
    FAIL_HANDLE(cl_mem);
}
cl_int clReleaseMemObject(cl_mem m) { (void)m; return CL_INVALID_PLATFORM; }
cl_sampler clCreateSampler(cl_context c, cl_bool n, cl_addressing_mode a, cl_filter_mode f, cl_int *errcode_ret) {
    (void)c, (void)n, (void)a, (void)f;
    FAIL_HANDLE(cl_sampler);
}
cl_int clReleaseSampler(cl_sampler s) { (void)s; return CL_INVALID_PLATFORM; }
cl_program clCreateProgramWithSource(cl_context c, cl_uint n, const char **s, const size_t *l, cl_int *errcode_ret) {
    (void)c, (void)n, (void)s, (void)l;
    FAIL_HANDLE(cl_program);
}
cl_int clBuildProgram(cl_program p, cl_uint n, const cl_device_id *d, const char *o, void (*f)(cl_program, void *),
                      void *u) {
    (void)p, (void)n, (void)d, (void)o, (void)f, (void)u;
    return CL_INVALID_PLATFORM;
}
cl_int clGetProgramBuildInfo(cl_program p, cl_device_id d, cl_program_build_info i, size_t s, void *v, size_t *r) {
    (void)p, (void)d, (void)i, (void)s, (void)v, (void)r;
    return CL_INVALID_PLATFORM;
}
cl_int clReleaseProgram(cl_program p) { (void)p; return CL_INVALID_PLATFORM; }
cl_kernel clCreateKernel(cl_program p, const char *n, cl_int *errcode_ret) {
    (void)p, (void)n;
    FAIL_HANDLE(cl_kernel);
}
cl_int clGetKernelWorkGroupInfo(cl_kernel k, cl_device_id d, cl_kernel_work_group_info i, size_t s, void *v,
                                size_t *r) {
    (void)k, (void)d, (void)i, (void)s, (void)v, (void)r;
    return CL_INVALID_PLATFORM;
}
cl_int clSetKernelArg(cl_kernel k, cl_uint i, size_t s, const void *v) {
    (void)k, (void)i, (void)s, (void)v;
    return CL_INVALID_PLATFORM;
}
cl_int clReleaseKernel(cl_kernel k) { (void)k; return CL_INVALID_PLATFORM; }
cl_int clEnqueueNDRangeKernel(cl_command_queue q, cl_kernel k, cl_uint w, const size_t *o, const size_t *g,
                              const size_t *l, cl_uint n, const cl_event *wl, cl_event *e) {
    (void)q, (void)k, (void)w, (void)o, (void)g, (void)l, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clEnqueueReadBuffer(cl_command_queue q, cl_mem b, cl_bool bl, size_t o, size_t cb, void *p, cl_uint n,
                           const cl_event *wl, cl_event *e) {
    (void)q, (void)b, (void)bl, (void)o, (void)cb, (void)p, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clEnqueueWriteBuffer(cl_command_queue q, cl_mem b, cl_bool bl, size_t o, size_t cb, const void *p, cl_uint n,
                            const cl_event *wl, cl_event *e) {
    (void)q, (void)b, (void)bl, (void)o, (void)cb, (void)p, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clEnqueueCopyBuffer(cl_command_queue q, cl_mem s, cl_mem d, size_t so, size_t dof, size_t cb, cl_uint n,
                           const cl_event *wl, cl_event *e) {
    (void)q, (void)s, (void)d, (void)so, (void)dof, (void)cb, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clEnqueueReadImage(cl_command_queue q, cl_mem im, cl_bool bl, const size_t o[3], const size_t r[3],
                          size_t rp, size_t sp, void *p, cl_uint n, const cl_event *wl, cl_event *e) {
    (void)q, (void)im, (void)bl, (void)o, (void)r, (void)rp, (void)sp, (void)p, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clEnqueueWriteImage(cl_command_queue q, cl_mem im, cl_bool bl, const size_t o[3], const size_t r[3],
                           size_t rp, size_t sp, const void *p, cl_uint n, const cl_event *wl, cl_event *e) {
    (void)q, (void)im, (void)bl, (void)o, (void)r, (void)rp, (void)sp, (void)p, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clEnqueueCopyImage(cl_command_queue q, cl_mem s, cl_mem d, const size_t so[3], const size_t dof[3],
                          const size_t r[3], cl_uint n, const cl_event *wl, cl_event *e) {
    (void)q, (void)s, (void)d, (void)so, (void)dof, (void)r, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clEnqueueCopyBufferToImage(cl_command_queue q, cl_mem s, cl_mem d, size_t so, const size_t dof[3],
                                  const size_t r[3], cl_uint n, const cl_event *wl, cl_event *e) {
    (void)q, (void)s, (void)d, (void)so, (void)dof, (void)r, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clEnqueueCopyImageToBuffer(cl_command_queue q, cl_mem s, cl_mem d, const size_t so[3], const size_t r[3],
                                  size_t dof, cl_uint n, const cl_event *wl, cl_event *e) {
    (void)q, (void)s, (void)d, (void)so, (void)r, (void)dof, (void)n, (void)wl, (void)e;
    return CL_INVALID_PLATFORM;
}
cl_int clWaitForEvents(cl_uint n, const cl_event *l) { (void)n, (void)l; return CL_INVALID_PLATFORM; }
cl_int clReleaseEvent(cl_event e) { (void)e; return CL_INVALID_PLATFORM; }
cl_int clGetEventProfilingInfo(cl_event e, cl_profiling_info i, size_t s, void *v, size_t *r) {
    (void)e, (void)i, (void)s, (void)v, (void)r;
    return CL_INVALID_PLATFORM;
}
cl_int clFinish(cl_command_queue q) { (void)q; return CL_INVALID_PLATFORM; }
