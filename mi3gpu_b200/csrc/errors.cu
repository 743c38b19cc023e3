// errors.cu -- error plumbing of the C ABI: thread-local messages on the
// host, and a probe of the device-side bounded waits.
#include "common.cuh"

namespace mi3 {

// One thread waits on an mbarrier whose phase nothing completes, with the
// bounded wait every pipelined kernel of the library uses; when the limit
// passes it reports MI3_STATUS_TIMEOUT_FULL and returns.  When abort_after
// is nonzero a second warp sets the abort flag after that many nanoseconds,
// which must end the wait early (the path kernels take when another thread
// of the CTA gave up first).
__global__ void k_probe_bounded_wait(int32_t *status, uint64_t limit_ns, uint64_t abort_after_ns,
                                     unsigned long long *waited_ns) {
    __shared__ __align__(8) uint64_t bar;
    __shared__ volatile int abort_flag;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint64_t t0 = globaltimer_ns();
        const bool ok = mbar_wait_bounded(&bar, 0, &abort_flag, limit_ns);
        *waited_ns = globaltimer_ns() - t0;
        if (!ok) report(status, ST_TIMEOUT_FULL);
    } else if (threadIdx.x == 32 && abort_after_ns) {
        const uint64_t t0 = globaltimer_ns();
        while (globaltimer_ns() - t0 < abort_after_ns) {
        }
        abort_flag = 1;
    }
}

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

extern "C" int mi3_probe_bounded_wait(int32_t *status, uint64_t limit_ns, uint64_t abort_after_ns,
                                      unsigned long long *waited_ns, void *stream) {
    if (!status || !waited_ns) return mi3::fail(MI3_ERR_ARG, "mi3_probe_bounded_wait: null pointer");
    if (limit_ns == 0 || limit_ns > 2000000000ull || abort_after_ns > limit_ns)
        return mi3::fail(MI3_ERR_ARG, "mi3_probe_bounded_wait: limit must be in (0, 2 s], abort_after <= limit");
    mi3::k_probe_bounded_wait<<<1, 64, 0, mi3::as_stream(stream)>>>(status, limit_ns, abort_after_ns, waited_ns);
    return mi3::check_launch("mi3_probe_bounded_wait");
}
