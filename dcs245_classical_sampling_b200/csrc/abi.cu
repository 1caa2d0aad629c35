// ABI plumbing: error messages, device queries, version.
#include <stdarg.h>
#include <stdio.h>

#include <string>

#include "common.cuh"

namespace {
thread_local std::string g_last_error;
}

namespace dcs_host {
void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return DCS_OK;
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return DCS_E_CUDA;
}

int sm_count() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return check_cuda(e, "cudaGetDevice");
    static int cached[64] = {0};
    if (dev >= 0 && dev < 64 && cached[dev] > 0) return cached[dev];
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return check_cuda(e, "cudaDeviceGetAttribute");
    if (dev >= 0 && dev < 64) cached[dev] = sms;
    return sms;
}
}  // namespace dcs_host

extern "C" int dcs_abi_version(void) { return DCS_ABI_VERSION; }

extern "C" const char* dcs_last_error(void) { return g_last_error.c_str(); }

extern "C" int dcs_sm_count(void) { return dcs_host::sm_count(); }

extern "C" size_t dcs_struct_size(int which) {
    switch (which) {
        case 0: return sizeof(dcs_step);
        case 1: return sizeof(dcs_param);
        case 2: return sizeof(dcs_scale);
        case 3: return sizeof(dcs_group);
        case 4: return sizeof(dcs_tile_step);
        case 5: return sizeof(dcs_draw_result);
        case 6: return sizeof(dcs_tile_run);
        case 7: return sizeof(dcs_gather_step);
    }
    return 0;
}
