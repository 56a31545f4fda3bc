// C ABI over the plugin layer: KernelInterface objects and Bench::run.
#include <cstring>
#include <sstream>
#include <string>

#include "../../../include/gatlas.h"
#include "../status.hpp"
#include "bench.hpp"
#include "kernel.hpp"

using gatlas::set_error;
using namespace gatlas::host;

struct gatlas_kernel {
    KernelInterface *k;
};

static size_t copy_out(const std::string &s, char *buf, size_t len) {
    if (buf && len) {
        const size_t c = s.size() < len - 1 ? s.size() : len - 1;
        std::memcpy(buf, s.data(), c);
        buf[c] = 0;
    }
    return s.size();
}

static size_t copy_vec(const std::vector<size_t> &v, size_t *out, size_t cap) {
    for (size_t i = 0; i < v.size() && i < cap; ++i) out[i] = v[i];
    return v.size();
}

extern "C" {

int gatlas_kernel_create(const char *op, const char *type, gatlas_kernel **out) {
    if (!op || !type || !out) return set_error(GATLAS_ERR_INVALID, "kernel_create: null argument");
    KernelInterface *k = make_kernel(op, type);
    if (!k) return set_error(GATLAS_ERR_INVALID, "kernel_create: unknown op '%s' or type '%s'", op, type);
    *out = new gatlas_kernel{k};
    return GATLAS_OK;
}

void gatlas_kernel_destroy(gatlas_kernel *k) {
    if (!k) return;
    delete k->k;
    delete k;
}

size_t gatlas_kernel_name(const gatlas_kernel *k, char *buf, size_t len) {
    return k ? copy_out(k->k->kernelName(), buf, len) : 0;
}

int gatlas_kernel_set_params(gatlas_kernel *k, const size_t *params, size_t n) {
    if (!k || !params) return set_error(GATLAS_ERR_INVALID, "kernel_set_params: null argument");
    k->k->setParams(std::vector<size_t>(params, params + n));
    return GATLAS_OK;
}

int gatlas_kernel_get_params(const gatlas_kernel *k, size_t *params, size_t cap, size_t *n) {
    if (!k) return set_error(GATLAS_ERR_INVALID, "kernel_get_params: null kernel");
    std::vector<size_t> p;
    const bool ok = k->k->getParams(p);
    if (n) *n = ok ? p.size() : 0;
    if (ok && params) copy_vec(p, params, cap);
    return ok ? 1 : 0;
}

size_t gatlas_kernel_number_flops(const gatlas_kernel *k) { return k ? k->k->numberFlops() : 0; }

size_t gatlas_kernel_total_variations(const gatlas_kernel *k) { return k ? k->k->totalVariations() : 0; }

size_t gatlas_kernel_extra_param_detail(const gatlas_kernel *k, size_t *out, size_t cap) {
    return k ? copy_vec(k->k->extraParamDetail(), out, cap) : 0;
}

size_t gatlas_kernel_global_work_items(const gatlas_kernel *k, size_t *out, size_t cap) {
    return k ? copy_vec(k->k->globalWorkItems(), out, cap) : 0;
}

size_t gatlas_kernel_local_work_items(const gatlas_kernel *k, size_t *out, size_t cap) {
    return k ? copy_vec(k->k->localWorkItems(), out, cap) : 0;
}

size_t gatlas_kernel_print(const gatlas_kernel *k, char *buf, size_t len) {
    if (!k) return 0;
    std::stringstream ss;
    k->k->print(ss);
    return copy_out(ss.str(), buf, len);
}

void gatlas_kernel_paranoid_check(gatlas_kernel *k) {
    if (k) k->k->paranoidCheck();
}

void gatlas_kernel_paranoid_fused(gatlas_kernel *k, int fused) {
    if (k) k->k->paranoidFused(fused != 0);
}

double gatlas_kernel_last_check(const gatlas_kernel *k) { return k ? k->k->lastCheck() : 0.0; }

int gatlas_bench_run(gatlas_kernel *k, const char *journal, size_t trials, const size_t *params, size_t n,
                     int bus_to_device, int bus_from_device, size_t *usec) {
    if (!k || !params || !usec) return set_error(GATLAS_ERR_INVALID, "bench_run: null argument");
    std::vector<size_t> args(params, params + n);
    if (journal && journal[0]) {
        Journal j(journal);
        Bench b(*k->k, j, false);
        *usec = b.run(trials, args, bus_to_device != 0, bus_from_device != 0);
    } else {
        Bench b(*k->k, false);
        *usec = b.run(trials, args, bus_to_device != 0, bus_from_device != 0);
    }
    return GATLAS_OK;
}

}  // extern "C"
