// drift_tuning.cu -- captured launch graphs and the launch autotuner.
//
// Graphs: an integration is up to five stream operations (cursor reset, the
// three ordering kernels, the integration kernel).  drift_graph_create
// records them once by stream capture of drift_integrate; drift_graph_launch
// replays the whole sequence with one call, for loops that integrate the
// same buffers repeatedly (an optimiser updating initial states in place, a
// service re-running a fixed request).
//
// Autotuner: the tunable launch parameters of this path are the block size
// (32 to 128 threads) and the schedule (plain, persistent, ordered); the
// integrator has one particle per thread and writes samples directly, so
// there is no particles-per-warp or staging-depth dimension.  drift_autotune
// times every candidate on a particle sample of the request -- its own
// scratch buffers, the request's initial states and grid -- and returns the
// fastest, cached per workload class (method, precision, potential kind,
// shared or per-particle grid, nt and particle count rounded to powers of
// two).  No counterpart exists in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "drift_b200.h"

int drift_internal_fail(int code, const char *msg);

struct drift_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

std::mutex g_tune_mu;
using TuneKey = std::tuple<int, int, int, int, int, int, int>;
std::map<TuneKey, drift_tuning> g_tune_cache;

int ilog2_ceil(int64_t v)
{
    int k = 0;
    while ((int64_t(1) << k) < v && k < 62) k++;
    return k;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return drift_internal_fail(DRIFT_ERROR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

}  // namespace

extern "C" {

int drift_graph_create(const drift_launch *launch, void *stream, drift_graph **out)
{
    if (!launch || !out) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!s) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "graph capture needs a non-default stream");
    auto *g = new drift_graph();
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(e, "cudaStreamBeginCapture");
    }
    int rc = drift_integrate(launch, stream);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(s, &graph);
    if (rc != DRIFT_SUCCESS || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        delete g;
        if (rc != DRIFT_SUCCESS) return rc;
        return cuda_fail(e, "cudaStreamEndCapture");
    }
    g->graph = graph;
    e = cudaGraphInstantiate(&g->exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        delete g;
        return cuda_fail(e, "cudaGraphInstantiate");
    }
    *out = g;
    return DRIFT_SUCCESS;
}

int drift_graph_launch(drift_graph *graph, void *stream)
{
    if (!graph || !graph->exec) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "graph is NULL");
    cudaError_t e = cudaGraphLaunch(graph->exec, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    return DRIFT_SUCCESS;
}

int drift_graph_destroy(drift_graph *graph)
{
    if (!graph) return DRIFT_SUCCESS;
    if (graph->exec) cudaGraphExecDestroy(graph->exec);
    if (graph->graph) cudaGraphDestroy(graph->graph);
    delete graph;
    return DRIFT_SUCCESS;
}

int drift_autotune(const drift_launch *launch, int64_t sample, drift_tuning *best)
{
    if (!launch || !best) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (launch->n < 1 || !launch->y0 || (!launch->ts && !launch->t_end) || launch->nt < 2)
        return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "autotune needs y0, a grid, n >= 1, nt >= 2");
    if (launch->tape) return drift_internal_fail(DRIFT_ERROR_INVALID_ARGUMENT, "autotune a launch without tape");
    const int64_t n = std::min<int64_t>(launch->n, sample > 0 ? sample : 16384);
    const TuneKey key{launch->method, launch->precision, launch->potential.kind, launch->ts ? 1 : 0,
                      ilog2_ceil(launch->nt), ilog2_ceil(launch->n), launch->arbitrary_times};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            *best = it->second;
            best->cached = 1;
            return DRIFT_SUCCESS;
        }
    }
    // scratch outputs and workspace for the sample
    drift_launch L = *launch;
    if (L.y0_layout == DRIFT_Y0_COLUMNS && L.y0_stride == 0) L.y0_stride = L.n;  // the sample keeps the columns
    L.n = n;
    L.out = nullptr;
    L.y_final = nullptr;
    L.status = nullptr;
    L.err_code = nullptr;
    L.n_accepted = nullptr;
    L.n_rejected = nullptr;
    L.schedule = DRIFT_SCHEDULE_ORDERED;
    size_t ws_bytes = 0;
    drift_query_workspace(&L, &ws_bytes);
    const size_t out_bytes = (size_t)launch->nt * n * 6 * sizeof(double);
    void *out = nullptr, *ws = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&out, out_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ws, std::max<size_t>(ws_bytes, 256));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    int rc = e == cudaSuccess ? DRIFT_SUCCESS : cuda_fail(e, "autotune scratch");
    drift_tuning t{};
    t.seconds = INFINITY;
    const int schedules[3] = {DRIFT_SCHEDULE_PLAIN, DRIFT_SCHEDULE_PERSISTENT, DRIFT_SCHEDULE_ORDERED};
    int c = 0;
    for (int si = 0; rc == DRIFT_SUCCESS && si < 3; si++)
        for (int block = 32; rc == DRIFT_SUCCESS && block <= 128; block += 32, c++) {
            L.schedule = schedules[si];
            L.block_size = block;
            L.out = static_cast<double *>(out);
            L.workspace = ws;
            L.workspace_bytes = std::max<size_t>(ws_bytes, 256);
            float ms = 0.f, best_ms = INFINITY;
            for (int rep = 0; rc == DRIFT_SUCCESS && rep < 2; rep++) {  // first run warms up
                cudaEventRecord(e0, s);
                rc = drift_integrate(&L, s);
                cudaEventRecord(e1, s);
                if (rc == DRIFT_SUCCESS && (e = cudaEventSynchronize(e1)) != cudaSuccess)
                    rc = cuda_fail(e, "autotune run");
                if (rc == DRIFT_SUCCESS && rep == 1) {
                    cudaEventElapsedTime(&ms, e0, e1);
                    best_ms = ms;
                }
            }
            if (rc != DRIFT_SUCCESS) break;
            t.candidates[c] = best_ms * 1e-3;
            if (best_ms * 1e-3 < t.seconds) {
                t.seconds = best_ms * 1e-3;
                t.block_size = block;
                t.schedule = schedules[si];
            }
        }
    if (e1) cudaEventDestroy(e1);
    if (e0) cudaEventDestroy(e0);
    if (s) cudaStreamDestroy(s);
    if (ws) cudaFree(ws);
    if (out) cudaFree(out);
    if (rc != DRIFT_SUCCESS) return rc;
    t.sample = n;
    t.cached = 0;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = t;
    }
    *best = t;
    return DRIFT_SUCCESS;
}

}  // extern "C"
