// fx_ctl.h -- device-side control of a coupled step.
//
// A time step holds loops whose trip counts depend on device results: the
// Newton passes of ComputePhi_Rho (ElectrostaticSolver.cpp:690-742, until the
// L1 change of phi is below the tolerance) and, inside each pass, the
// multigrid V-cycles (until |r|_inf <= the MLMG target).  On the host path
// every one of those tests is a device-to-host read and a stream
// synchronisation.  Here the whole step is one CUDA graph: the loops are
// conditional WHILE / IF nodes whose conditions are set on the device by
// one-thread control kernels (cudaGraphSetConditional), with the loop state
// and the step's statistics in a StepCtl block in device memory that the host
// reads once at the end of the step.
//
// Every loop is bounded by its iteration cap (fx.mg_max_iter cycles per solve,
// fx.newton_max_iter passes per ComputePhi_Rho): a control kernel clears the
// loop condition once the cap is reached and records the failure in `status`.
#pragma once

#include <atomic>
#include <cuda_runtime.h>

namespace fx {

extern std::atomic<long long> g_launches;

// bodies of conditional nodes whose executions the control kernels count
enum CtlKind {
    KIND_MG_CYCLE = 0, KIND_MG_RESID, KIND_NEWTON_PASS, KIND_MX_FIRST, KIND_MX_SECOND, KIND_GATE_TDGL,
    KIND_GATE_CORRECTOR, KIND_N
};

// failure recorded on the device (first one wins)
enum CtlStatus { CTL_OK = 0, CTL_MG_NO_CONV = 1, CTL_MG_NONFINITE = 2, CTL_NEWTON_NO_CONV = 3, CTL_NEWTON_NONFINITE = 4 };

struct StepCtl {
    // the multigrid solve in progress
    double target;          // max(rtol, 1e-16) * max(|b|, |b'|)
    double rn;              // |r|_inf that the loop tests
    int it;                 // V-cycles (FP64) or FP32 cycles (mixed) of this solve
    int parity;             // mixed: 1 while the iterate sits in the second buffer
    // the ComputePhi_Rho in progress (the step's last one when the step ends)
    int passes, iter;
    double err;
    int mg_cycles_phirho;
    double mg_resid_last, mg_target_last;
    // step totals
    long long mg_cycles_step;
    int newton_passes_step;
    int status;
    int status_n;           // cycles or passes at the failure
    double status_val;      // |r| or Newton error at the failure
    double status_target;
    long long nexec[KIND_N];
};

// Builds conditional nodes while a stream is being captured.  node() adds a
// conditional node after the capture's current dependencies, captures the
// body on a dedicated stream per nesting depth, and continues the outer
// capture after the node.  It also attributes the kernel launches counted in
// g_launches during capture to the body kinds, so that the launches of one
// graph execution follow from the device's execution counts.
struct CondCapture {
    static constexpr int kDepth = 5;
    cudaStream_t sb[kDepth] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int depth = 0;
    long long in_bodies = 0;          // launches captured inside any body
    long long own[KIND_N] = {};       // launches per execution of each body kind
    cudaError_t err = cudaSuccess;

    cudaError_t init() {
        for (int d = 0; d < kDepth; ++d)
            if (!sb[d]) {
                cudaError_t e = cudaStreamCreateWithFlags(&sb[d], cudaStreamNonBlocking);
                if (e) return e;
            }
        return cudaSuccess;
    }
    void release() {
        for (int d = 0; d < kDepth; ++d)
            if (sb[d]) { cudaStreamDestroy(sb[d]); sb[d] = nullptr; }
    }
    void reset() { depth = 0; in_bodies = 0; err = cudaSuccess; for (int k = 0; k < KIND_N; ++k) own[k] = 0; }

    // a handle in the graph that `s` is capturing into (condition 0 at each launch)
    cudaGraphConditionalHandle handle(cudaStream_t s) {
        cudaGraphConditionalHandle h = 0;
        cudaStreamCaptureStatus st;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr);
        if (!e && st != cudaStreamCaptureStatusActive) e = cudaErrorStreamCaptureInvalidated;
        if (!e) e = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault);
        if (e && !err) err = e;
        return h;
    }

    template <typename F>
    void node(cudaStream_t s, cudaGraphConditionalNodeType type, cudaGraphConditionalHandle h, int kind, F&& body) {
        if (err) return;
        if (depth >= kDepth) { err = cudaErrorInvalidValue; return; }
        cudaStreamCaptureStatus st;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd);
        if (!e && st != cudaStreamCaptureStatusActive) e = cudaErrorStreamCaptureInvalidated;
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = type;
        np.conditional.size = 1;
        cudaGraphNode_t n = nullptr;
        if (!e) e = cudaGraphAddNode(&n, g, deps, nd, &np);
        if (e) { err = e; return; }
        cudaStream_t b = sb[depth];
        e = cudaStreamBeginCaptureToGraph(b, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
        if (e) { err = e; return; }
        const long long l0 = g_launches.load(), nested0 = in_bodies;
        ++depth;
        body(b);
        --depth;
        const long long mine = (g_launches.load() - l0) - (in_bodies - nested0);
        in_bodies += mine;
        own[kind] = mine;
        cudaGraph_t out = nullptr;
        e = cudaStreamEndCapture(b, &out);
        if (!e) e = cudaStreamUpdateCaptureDependencies(s, &n, 1, cudaStreamSetCaptureDependencies);
        if (e && !err) err = e;
    }
};

}  // namespace fx
