// Plan-specialised kernels: NVRTC compilation (sm_100a cubin), loading through the runtime
// library API, and launch of the group kernels that jit.py generates (device header
// runs_jit.cuh).
#include <nvrtc.h>
#include <stdlib.h>
#include <string.h>

#include "common.cuh"

namespace {

int nvrtc_check(nvrtcResult r, const char* what) {
    if (r == NVRTC_SUCCESS) return DCS_OK;
    dcs_host::set_error("%s: %s", what, nvrtcGetErrorString(r));
    return DCS_E_CUDA;
}

}  // namespace

extern "C" int dcs_jit_compile(const char* source, const char* name, const char* header_source,
                               const char* header_name, int lineinfo, void** image, size_t* image_size, char* log,
                               size_t log_capacity) {
    if (!source || !name || !image || !image_size || (header_source && !header_name)) {
        dcs_host::set_error("dcs_jit_compile: invalid arguments");
        return DCS_E_ARG;
    }
    *image = nullptr;
    *image_size = 0;
    if (log && log_capacity) log[0] = 0;
    nvrtcProgram prog;
    const char* hs[1] = {header_source};
    const char* hn[1] = {header_name};
    int rc = nvrtc_check(nvrtcCreateProgram(&prog, source, name, header_source ? 1 : 0, hs, hn), "nvrtcCreateProgram");
    if (rc != DCS_OK) return rc;
    const char* opts[4] = {"--gpu-architecture=sm_100a", "--std=c++17", "-DNDEBUG", "-lineinfo"};
    const nvrtcResult cr = nvrtcCompileProgram(prog, lineinfo ? 4 : 3, opts);
    size_t lsize = 0;
    if (log && log_capacity && nvrtcGetProgramLogSize(prog, &lsize) == NVRTC_SUCCESS && lsize > 1) {
        char* buf = (char*)malloc(lsize);
        if (buf && nvrtcGetProgramLog(prog, buf) == NVRTC_SUCCESS) {
            const size_t n = lsize < log_capacity ? lsize : log_capacity;
            memcpy(log, buf, n);
            log[n - 1] = 0;
        }
        free(buf);
    }
    if (cr != NVRTC_SUCCESS) {
        nvrtcDestroyProgram(&prog);
        return nvrtc_check(cr, "nvrtcCompileProgram");
    }
    size_t n = 0;
    rc = nvrtc_check(nvrtcGetCUBINSize(prog, &n), "nvrtcGetCUBINSize");
    if (rc == DCS_OK) {
        void* buf = malloc(n);
        if (!buf) {
            dcs_host::set_error("dcs_jit_compile: out of host memory");
            rc = DCS_E_ARG;
        } else {
            rc = nvrtc_check(nvrtcGetCUBIN(prog, (char*)buf), "nvrtcGetCUBIN");
            if (rc == DCS_OK) {
                *image = buf;
                *image_size = n;
            } else {
                free(buf);
            }
        }
    }
    nvrtcDestroyProgram(&prog);
    return rc;
}

extern "C" void dcs_jit_free(void* image) { free(image); }

extern "C" int dcs_jit_load(const void* image, void** library) {
    if (!image || !library) {
        dcs_host::set_error("dcs_jit_load: invalid arguments");
        return DCS_E_ARG;
    }
    cudaLibrary_t lib = nullptr;
    const cudaError_t e = cudaLibraryLoadData(&lib, image, nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) return dcs_host::check_cuda(e, "cudaLibraryLoadData");
    *library = (void*)lib;
    return DCS_OK;
}

extern "C" int dcs_jit_unload(void* library) {
    if (!library) return DCS_OK;
    const cudaError_t e = cudaLibraryUnload((cudaLibrary_t)library);
    return e == cudaSuccess ? DCS_OK : dcs_host::check_cuda(e, "cudaLibraryUnload");
}

extern "C" int dcs_jit_kernel(void* library, const char* name, size_t smem, int threads, void** kernel,
                              int* blocks_per_sm) {
    if (!library || !name || !kernel || !blocks_per_sm || threads < 32 || threads > 1024 || threads % 32) {
        dcs_host::set_error("dcs_jit_kernel: invalid arguments");
        return DCS_E_ARG;
    }
    cudaKernel_t k = nullptr;
    cudaError_t e = cudaLibraryGetKernel(&k, (cudaLibrary_t)library, name);
    if (e != cudaSuccess) return dcs_host::check_cuda(e, "cudaLibraryGetKernel");
    e = cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return dcs_host::check_cuda(e, "jit kernel smem attribute");
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, threads, smem);
    if (e != cudaSuccess) return dcs_host::check_cuda(e, "jit kernel occupancy");
    *kernel = (void*)k;
    *blocks_per_sm = per_sm;
    return DCS_OK;
}

extern "C" int dcs_jit_launch(void* kernel, unsigned grid, int threads, size_t smem, void* table,
                              const dcs_param* params, uint64_t* maxbits, dcs_scale* scale, void* stream) {
    if (!kernel || !grid || !table || !params || !maxbits || !scale || threads < 32 || threads > 1024 || threads % 32) {
        dcs_host::set_error("dcs_jit_launch: invalid arguments");
        return DCS_E_ARG;
    }
    void* args[4] = {&table, (void*)&params, &maxbits, &scale};
    const cudaError_t e =
        cudaLaunchKernel((const void*)kernel, dim3(grid), dim3(threads), args, smem, (cudaStream_t)stream);
    return e == cudaSuccess ? DCS_OK : dcs_host::check_cuda(e, "jit kernel launch");
}
