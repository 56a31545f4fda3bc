// Per-thread error messages and status strings for the C ABI.
#include "status.hpp"

#include <cstdarg>
#include <cstdio>
#include <cstring>

namespace gatlas {

static thread_local char g_last_error[512] = {0};

int set_error(int status, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

void clear_error() { g_last_error[0] = 0; }

}  // namespace gatlas

extern "C" {

int gatlas_version(void) { return 100; }

const char *gatlas_status_string(int status) {
    switch (status) {
        case GATLAS_OK: return "ok";
        case GATLAS_ERR_INVALID: return "invalid argument";
        case GATLAS_ERR_CUDA: return "CUDA error";
        case GATLAS_ERR_UNSUPPORTED: return "unsupported parameter point";
        case GATLAS_ERR_TIMEOUT: return "bounded device wait expired";
        case GATLAS_ERR_NOMEM: return "out of memory";
        case GATLAS_ERR_CHECK: return "output check failed";
        case GATLAS_ERR_STATE: return "call out of order";
        default: return "unknown status";
    }
}

size_t gatlas_last_error(char *buf, size_t len) {
    const size_t n = std::strlen(gatlas::g_last_error);
    if (buf && len) {
        const size_t c = n < len - 1 ? n : len - 1;
        std::memcpy(buf, gatlas::g_last_error, c);
        buf[c] = 0;
    }
    return n;
}

}  // extern "C"
