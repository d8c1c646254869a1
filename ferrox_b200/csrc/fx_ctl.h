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

// Programmatic dependent launch for the step kernels (fx.pdl, on by default):
// a kernel launched with programmatic stream serialisation may be scheduled
// while its predecessor drains; every kernel so launched calls pdl_entry()
// before it touches memory, which waits for the predecessor's completion and
// the visibility of its writes, then lets its own successor be scheduled.
// Without the attribute the wait returns at once, so the same kernels serve
// both forms.
extern bool g_pdl;
// the scalar Poisson right-hand side by row segments (k_rhs_p_seg; process-wide like g_pdl)
extern bool g_rhs_seg;

__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = g_pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

// bodies of conditional nodes whose executions the control kernels count
enum CtlKind {
    KIND_MG_CYCLE = 0, KIND_NEWTON_PASS, KIND_MX_FIRST, KIND_MX_SECOND, KIND_GATE_TDGL, KIND_GATE_CORRECTOR, KIND_N
};

// failure recorded on the device (first one wins)
enum CtlStatus { CTL_OK = 0, CTL_MG_NO_CONV = 1, CTL_MG_NONFINITE = 2, CTL_NEWTON_NO_CONV = 3, CTL_NEWTON_NONFINITE = 4 };

struct StepCtl {
    // the multigrid solve in progress
    double target;          // max(rtol, 1e-16) * max(|b|, |b'|)
    double rn;              // |r|_inf that the loop tests
    int it;                 // V-cycles (FP64) or FP32 cycles (mixed) of this solve
    int parity;             // mixed: 1 while the iterate sits in the second buffer
    int need;               // FP64: the exact residual is formed after this cycle
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
    double steady[2];       // CheckSteadyState: max|phi|, max|phi - phi_old|
};

// ---- loop control, run by one thread of the kernel that produces the tested
// quantity (the last block of a residual or charge kernel), or by a
// one-thread kernel

// the multigrid solve ended: its statistics and, short of the target, the failure
__device__ __forceinline__ void ctl_mg_end(StepCtl* ctl) {
    const int it = ctl->it;
    const double rn = ctl->rn, t = ctl->target;
    ctl->mg_cycles_phirho += it;
    ctl->mg_cycles_step += it;
    ctl->mg_resid_last = rn;
    ctl->mg_target_last = t;
    // a non-finite residual fails even against a non-finite target (a NaN in
    // the right-hand side makes both +inf)
    if ((!(rn <= t) || !isfinite(rn)) && ctl->status == CTL_OK) {
        ctl->status = isfinite(rn) ? CTL_MG_NO_CONV : CTL_MG_NONFINITE;
        ctl->status_n = it;
        ctl->status_val = rn;
        ctl->status_target = t;
    }
}

// the test of the ComputePhi_Rho loop (ElectrostaticSolver.cpp:690-742) after
// a pass from the L1 sums s1 = sum|phi - phi_prev|, s2 = sum|phi|: err = s1 / s2
// from the second pass on, as the host loop forms it; the pass cap turns a
// loop that would go on into a failure
__device__ __forceinline__ void ctl_newton(StepCtl* ctl, double s1, double s2, double tol, int max_iter,
                                           cudaGraphConditionalHandle h, int in_body) {
    if (in_body) ctl->nexec[KIND_NEWTON_PASS] += 1;
    const int passes = ctl->passes + 1;
    ctl->passes = passes;
    double err = ctl->err;
    if (ctl->iter > 0) err = s1 / s2;
    ctl->err = err;
    ctl->iter += 1;
    bool go = err > tol;
    if (ctl->status != CTL_OK) {
        go = false;
    } else if (!isfinite(err)) {
        ctl->status = CTL_NEWTON_NONFINITE;
        ctl->status_n = passes;
        ctl->status_val = err;
        go = false;
    } else if (go && passes >= max_iter) {
        ctl->status = isfinite(err) ? CTL_NEWTON_NO_CONV : CTL_NEWTON_NONFINITE;
        ctl->status_n = passes;
        ctl->status_val = err;
        go = false;
    }
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// control carried by the charge kernel's last block (null ctl: none)
struct RhoCtl {
    StepCtl* ctl;
    double tol;
    int max_iter;
    int in_body;
    int mg_end;            // first close the multigrid solve before it
    cudaGraphConditionalHandle h;
};

// control carried by the FP64 residual kernel's last block (null ctl: none)
enum ResidMode { RC_BEGIN = 1, RC_RN = 2, RC_MX = 3 };
struct ResidCtl {
    StepCtl* ctl;
    int mode;
    const double* nb;      // RC_BEGIN: max|b|, max|b'|
    double rtol;
    int maxit;
    int inner, parity, kind;   // RC_MX: FP32 cycles spent, buffer holding the iterate, body kind
    cudaGraphConditionalHandle h, h2;
    unsigned int* counter;
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
