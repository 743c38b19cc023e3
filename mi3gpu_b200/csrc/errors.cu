// errors.cu -- host-side error plumbing of the C ABI.
#include "common.cuh"

namespace mi3 {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(MI3_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return MI3_OK;
}

}  // namespace mi3

extern "C" const char *mi3_last_error(void) { return mi3::g_last_error.c_str(); }

extern "C" int mi3_abi_version(void) { return 2; }

extern "C" uint64_t mi3_jrows_stride(uint32_t L, uint32_t q) { return mi3::jrow_stride(L, q); }
