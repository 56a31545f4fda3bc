// Status codes and the per-thread last-error message behind gatlas_last_error().
#pragma once

#include "../../include/gatlas.h"

namespace gatlas {

// Records a printf-style message for the calling thread and returns `status`.
int set_error(int status, const char *fmt, ...)
#if defined(__GNUC__)
    __attribute__((format(printf, 2, 3)))
#endif
    ;

void clear_error();

}  // namespace gatlas
