// graph.cu -- CUDA-graph plumbing for whole quasi-Newton rounds.
//
// A round (sampling, counts, statistics, the Newton loop, the J update) of
// one or many independent problems is recorded once by stream capture and
// replayed with one graph launch per round.  The Newton loop's length is
// decided on the device: its steps form the body of a conditional WHILE
// node whose condition is written by k_newton_control after every step,
// from the FP64 weight sums, with the same stop rule as the host loop of
// NewtonSteps.iterNewton (NewtonSteps.py:217-246): stop after the step whose
// effective sample size falls below frac * N0, or after max_steps steps.
// The step counter bounds the loop, so a body always terminates.  The
// sampling phase can equilibrate on the device too: each checkpoint of the
// doubling schedule is a conditional IF node opened by the previous
// checkpoint's rank-correlation test (k_equil_control).
#include "common.cuh"

namespace mi3 {

// After a Newton step: count it, decide whether another one follows, and
// hand this step's min(0, dE) to the next step as its reference energy (the
// reference's one-step lag of ref_dE).  One thread.
__global__ void k_newton_control(cudaGraphConditionalHandle handle, const double *__restrict__ wstats64,
                                 const float *__restrict__ minout, float *ref, uint32_t *count,
                                 const uint32_t *__restrict__ max_steps, double neff_min, uint32_t *stopped) {
    const double s = wstats64[0], s2 = wstats64[1];
    const double neff = s * s / s2;
    const uint32_t c = *count + 1;
    *count = c;
    *ref = *minout;
    const bool diverged = !(s > 0.0) || !isfinite(s) || !isfinite(s2);
    const bool more = !diverged && neff >= neff_min && c < max(*max_steps, 1u);
    if (!more && stopped) *stopped = diverged ? 2u : 1u;
    cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// The per-round adaptation of the Newton-step budget (NewtonSteps.py:664-683):
// before the loop, shrink the budget by 1.5*delta when this round's SSR is
// above the mean of the last and the smallest SSR so far; after the loop,
// budget = min(2048, steps + delta).  state = {last SSR (NaN before the
// first round), smallest SSR}.  One thread.
__global__ void k_newton_adapt(uint32_t after, const double *__restrict__ stats, const uint32_t *__restrict__ count,
                               uint32_t *budget, double *state, uint32_t delta) {
    if (!after) {
        const double ssr = stats[0], last = state[0], mn = state[1];
        if (!isnan(last) && ssr > 0.5 * (last + mn)) {
            const uint32_t dec = (3 * delta) / 2;
            *budget = max(delta, *budget > dec ? *budget - dec : 0u);
        }
        state[0] = ssr;
        state[1] = fmin(mn, ssr);
    } else {
        const uint32_t steps = *count > 0 ? *count - 1 : 0;  // the reference's returned step index
        *budget = min(2048u, steps + delta);
    }
}

// After a checkpoint of the sampling phase (runMCMC's automatic
// equilibration, NewtonSteps.py:395-442, in the device's rank form):
// equilibrated when both rank correlations (last checkpoint against one
// and two checkpoints back) have p > 0.02, i.e. |r| < rcrit, and at least
// min_equil calls ran; stop at max_equil calls.  Opens the next checkpoint's
// IF node when neither holds (has_next), and records {calls, verdict}:
// verdict 1 equilibrated, 2 stopped at max_equil, 0 going on.  One thread.
__global__ void k_equil_control(cudaGraphConditionalHandle next, int has_next, const double *__restrict__ r1,
                                const double *__restrict__ r2, double rcrit, int test, uint32_t calls,
                                uint32_t min_equil, uint32_t max_equil, uint32_t *out) {
    bool eq = false;
    if (test) {
        const double a = fabs(*r1), b = fabs(*r2);
        eq = a < rcrit && b < rcrit && calls >= min_equil;  // false for NaN
    }
    const bool more = !eq && calls < max_equil;
    out[0] = calls;
    out[1] = eq ? 1u : (more ? 0u : 2u);
    if (has_next) cudaGraphSetConditional(next, more ? 1u : 0u);
}

}  // namespace mi3

using namespace mi3;

extern "C" int mi3_capture_begin(void *stream) {
    cudaError_t e = cudaStreamBeginCapture(as_stream(stream), cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("mi3_capture_begin: ") + cudaGetErrorString(e));
    return MI3_OK;
}

extern "C" int mi3_capture_end(void *stream, void **graph_out) {
    if (!graph_out) return fail(MI3_ERR_ARG, "mi3_capture_end: null pointer");
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(as_stream(stream), &g);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("mi3_capture_end: ") + cudaGetErrorString(e));
    *graph_out = g;
    return MI3_OK;
}

extern "C" int mi3_graph_instantiate(void *graph, void **exec_out) {
    if (!graph || !exec_out) return fail(MI3_ERR_ARG, "mi3_graph_instantiate: null pointer");
    cudaGraphExec_t x = nullptr;
    cudaError_t e = cudaGraphInstantiate(&x, reinterpret_cast<cudaGraph_t>(graph), 0);
    if (e != cudaSuccess)
        return fail(MI3_ERR_CUDA, std::string("mi3_graph_instantiate: ") + cudaGetErrorString(e));
    *exec_out = x;
    return MI3_OK;
}

extern "C" int mi3_graph_launch(void *exec, void *stream) {
    if (!exec) return fail(MI3_ERR_ARG, "mi3_graph_launch: null pointer");
    cudaError_t e = cudaGraphLaunch(reinterpret_cast<cudaGraphExec_t>(exec), as_stream(stream));
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("mi3_graph_launch: ") + cudaGetErrorString(e));
    return MI3_OK;
}

extern "C" int mi3_graph_destroy(void *graph, void *exec) {
    if (exec) cudaGraphExecDestroy(reinterpret_cast<cudaGraphExec_t>(exec));
    if (graph) cudaGraphDestroy(reinterpret_cast<cudaGraph_t>(graph));
    return check_launch("mi3_graph_destroy");
}

// At the current capture position of `stream`, add a conditional node of
// `type` driven by handle h and begin capturing its body on `body_stream`.
static int capture_cond_begin(void *stream, void *body_stream, cudaGraphConditionalNodeType type,
                              cudaGraphConditionalHandle h, const char *name) {
    cudaStream_t st = as_stream(stream);
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess || cs != cudaStreamCaptureStatusActive)
        return fail(MI3_ERR_CUDA, std::string(name) + ": stream is not capturing");
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = h;
    params.conditional.type = type;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, graph, deps, ndeps, &params);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string(name) + ": node: " + cudaGetErrorString(e));
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string(name) + ": deps: " + cudaGetErrorString(e));
    cudaGraph_t body = params.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(as_stream(body_stream), body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string(name) + ": body: " + cudaGetErrorString(e));
    return MI3_OK;
}

// A conditional handle of the graph `stream` is capturing into, reset to
// `value` at every launch of the graph.
extern "C" int mi3_cond_handle_create(void *stream, uint32_t value, unsigned long long *handle_out) {
    if (!handle_out) return fail(MI3_ERR_ARG, "mi3_cond_handle_create: null pointer");
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamGetCaptureInfo(as_stream(stream), &cs, nullptr, &graph, nullptr, nullptr);
    if (e != cudaSuccess || cs != cudaStreamCaptureStatusActive)
        return fail(MI3_ERR_CUDA, "mi3_cond_handle_create: stream is not capturing");
    cudaGraphConditionalHandle h;
    e = cudaGraphConditionalHandleCreate(&h, graph, value, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("mi3_cond_handle_create: ") + cudaGetErrorString(e));
    *handle_out = (unsigned long long)h;
    return MI3_OK;
}

// At the current capture position of `stream`, add a conditional WHILE node
// (condition 1 at every graph launch) and begin capturing its body on
// `body_stream`; everything issued on body_stream until mi3_capture_while_end
// forms one iteration.  `stream` continues after the node.
extern "C" int mi3_capture_while_begin(void *stream, void *body_stream, unsigned long long *handle_out) {
    if (!handle_out || stream == body_stream) return fail(MI3_ERR_ARG, "mi3_capture_while_begin: bad arguments");
    unsigned long long h = 0;
    int rc = mi3_cond_handle_create(stream, 1, &h);
    if (rc) return rc;
    rc = capture_cond_begin(stream, body_stream, cudaGraphCondTypeWhile, (cudaGraphConditionalHandle)h,
                            "mi3_capture_while_begin");
    if (rc) return rc;
    *handle_out = h;
    return MI3_OK;
}

// The same for a conditional IF node on an existing handle (from
// mi3_cond_handle_create): its body runs once when the handle is non-zero.
extern "C" int mi3_capture_if_begin(void *stream, void *body_stream, unsigned long long handle) {
    if (stream == body_stream) return fail(MI3_ERR_ARG, "mi3_capture_if_begin: bad arguments");
    return capture_cond_begin(stream, body_stream, cudaGraphCondTypeIf, (cudaGraphConditionalHandle)handle,
                              "mi3_capture_if_begin");
}

extern "C" int mi3_capture_if_end(void *body_stream) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(as_stream(body_stream), &g);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("mi3_capture_if_end: ") + cudaGetErrorString(e));
    return MI3_OK;
}

extern "C" int mi3_equil_control(unsigned long long next, int32_t has_next, const double *r1, const double *r2,
                                 double rcrit, int32_t test, uint32_t calls, uint32_t min_equil, uint32_t max_equil,
                                 uint32_t *out, void *stream) {
    if (!out || (test && (!r1 || !r2))) return fail(MI3_ERR_ARG, "mi3_equil_control: null pointer");
    k_equil_control<<<1, 1, 0, as_stream(stream)>>>((cudaGraphConditionalHandle)next, has_next, r1, r2, rcrit, test,
                                                    calls, min_equil, max_equil, out);
    return check_launch("mi3_equil_control");
}

extern "C" int mi3_capture_while_end(void *body_stream) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(as_stream(body_stream), &g);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("mi3_capture_while_end: ") + cudaGetErrorString(e));
    return MI3_OK;
}

extern "C" int mi3_newton_control(unsigned long long handle, const double *wstats64, const float *minout,
                                  float *ref, uint32_t *count, const uint32_t *max_steps, double neff_min,
                                  uint32_t *stopped, void *stream) {
    if (!wstats64 || !minout || !ref || !count || !max_steps)
        return fail(MI3_ERR_ARG, "mi3_newton_control: null pointer");
    k_newton_control<<<1, 1, 0, as_stream(stream)>>>((cudaGraphConditionalHandle)handle, wstats64, minout, ref,
                                                     count, max_steps, neff_min, stopped);
    return check_launch("mi3_newton_control");
}

extern "C" int mi3_newton_adapt(uint32_t after, const double *stats, const uint32_t *count, uint32_t *budget,
                                double *state, uint32_t delta, void *stream) {
    if (!stats || !count || !budget || !state) return fail(MI3_ERR_ARG, "mi3_newton_adapt: null pointer");
    k_newton_adapt<<<1, 1, 0, as_stream(stream)>>>(after, stats, count, budget, state, delta);
    return check_launch("mi3_newton_adapt");
}

// Dedicated non-blocking streams for capture (pooled streams of a framework
// may alias each other, and a stream cannot capture two graphs at once).
extern "C" int mi3_stream_create(void **stream_out) {
    if (!stream_out) return fail(MI3_ERR_ARG, "mi3_stream_create: null pointer");
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("mi3_stream_create: ") + cudaGetErrorString(e));
    *stream_out = st;
    return MI3_OK;
}

extern "C" int mi3_stream_destroy(void *stream) {
    if (stream) cudaStreamDestroy(as_stream(stream));
    return check_launch("mi3_stream_destroy");
}

extern "C" int mi3_memset(void *ptr, int value, size_t nbytes, void *stream) {
    if (!ptr && nbytes) return fail(MI3_ERR_ARG, "mi3_memset: null pointer");
    if (nbytes == 0) return MI3_OK;
    if (cudaMemsetAsync(ptr, value, nbytes, as_stream(stream)) != cudaSuccess) return check_launch("mi3_memset");
    return MI3_OK;
}
