// fx_mg.h -- geometric multigrid for the variable-permittivity Poisson
// operator that replaces AMReX MLABecLaplacian + MLMG
// (ElectrostaticSolver.cpp:562-611, solve at :719):
//
//   (-alpha - div beta grad) phi = rhs,   beta on faces = 0.5 (eps_L + eps_R),
//   x / y periodic, z Dirichlet through the maxorder-2 ghost 2 V - phi_0.
//
// Hierarchy: a direction is halved while its cell count is even and its
// spacing is within 1.5x of the finest spacing; while z is being coarsened a
// level uses red-black point Gauss-Seidel, once only x / y are coarsened it
// uses red-black z-line Gauss-Seidel (a tridiagonal solve per column), so the
// 1 x 1 x nz bottom level is solved exactly.  Prolongation is linear in the
// coarsened directions, restriction averages, coarse coefficients are face
// averages (beta) and cell averages (alpha).
#pragma once

#include <cstdint>
#include <initializer_list>
#include <vector>

#include <cuda_runtime.h>

#include "fx_ctl.h"
#include "fx_device.cuh"

namespace fx {

struct MGLevel {
    int n[3];
    double h[3];
    int cr[3];          // coarsening ratio from the finer level
    bool line;          // z-line smoother
    float* wf[3] = {nullptr, nullptr, nullptr};  // prolongation far-neighbour weight per finer cell
    size_t N;
    // device storage, FP64 and FP32 copies
    double *x64 = nullptr, *b64 = nullptr, *bw64 = nullptr, *bs64 = nullptr, *bb64 = nullptr, *a64 = nullptr, *cp64 = nullptr;
    float *x32 = nullptr, *b32 = nullptr, *bw32 = nullptr, *bs32 = nullptr, *bb32 = nullptr, *a32 = nullptr, *cp32 = nullptr;
    // smoother factors of the one-CTA levels (q, 1/pivot, cb/pivot), FP64 and
    // FP32, kept between calls while alpha is unchanged
    double* fac64[3] = {nullptr, nullptr, nullptr};
    float* fac32[3] = {nullptr, nullptr, nullptr};
    // coarse face beta that depends on z only (layered stacks): per plane
    // bw[nz], bs[nz], bb[nz + 1] in one array, else null
    double* zc64 = nullptr;
    float* zc32 = nullptr;
    // the FP32 cycle's face beta of a launched coarse level in FP16, scaled by
    // 1 / hscale (the largest face beta of the level); null on level 0, on
    // layered levels (per plane) and without fx.mg_half
    uint16_t *bwh = nullptr, *bsh = nullptr, *bbh = nullptr;
    double hscale = 1.0;
};

// Optional per-launch timing: CUDA events around each launch of a kernel
// class, on the launching stream, summed after the stream has synchronised.
enum ProfCat {
    PROF_TDGL = 0, PROF_RHS_P, PROF_NEWTON, PROF_RHO, PROF_STEADY, PROF_SMOOTH_L0, PROF_RESTRICT_L0,
    PROF_PROLONG_L0, PROF_MG_COARSE, PROF_RESID64, PROF_EFIELD, PROF_MG_L1, PROF_MG_L2, PROF_COARSE_CTA, PROF_NCAT
};

struct Prof {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    std::vector<int> cats;     // category of pending pair q: events 2q, 2q+1
    double ms[PROF_NCAT] = {0};
    long long cnt[PROF_NCAT] = {0};
    void begin(int cat, cudaStream_t s) {
        if (!on) return;
        const size_t q = cats.size();
        while (pool.size() < 2 * q + 2) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        cats.push_back(cat);
        cudaEventRecord(pool[2 * q], s);
    }
    void end(cudaStream_t s) {
        if (!on || cats.empty()) return;
        cudaEventRecord(pool[2 * (cats.size() - 1) + 1], s);
    }
    void collect() {
        for (size_t q = 0; q < cats.size(); ++q) {
            float t = 0.f;
            cudaEventSynchronize(pool[2 * q + 1]);
            if (cudaEventElapsedTime(&t, pool[2 * q], pool[2 * q + 1]) == cudaSuccess) {
                ms[cats[q]] += t;
                cnt[cats[q]] += 1;
            }
        }
        cats.clear();
    }
    void reset() { for (int c = 0; c < PROF_NCAT; ++c) { ms[c] = 0; cnt[c] = 0; } cats.clear(); }
    ~Prof() { for (auto e : pool) cudaEventDestroy(e); }
};

struct MGStats {
    int cycles = 0;
    double resid = 0.0;       // final |r|_inf
};

class Multigrid {
public:
    ~Multigrid();
    // builds the hierarchy and uploads the coarse face coefficients
    int setup(const DevParams& p, const std::vector<uint8_t>& code_host, bool want64, bool want32);
    // alpha changed on level 0 (device, FP64 and FP32 copies): average down
    int set_alpha(const double* a64, const float* a32, bool has_alpha, cudaStream_t s);
    // FP64 solve of A phi = rhs (+ electrode terms) to |r|_inf <= target
    int solve64(const DevParams& p, const uint8_t* code, double* phi, const double* rhs, double target, int maxit,
                cudaStream_t s, MGStats* st);
    // FP64 iterative refinement around FP32 V-cycles
    int solve_mixed(const DevParams& p, const uint8_t* code, double* phi, const double* rhs, double target,
                    int maxit, cudaStream_t s, MGStats* st);
    // The same two solves for a step graph being captured on s: the cycle
    // loop is a conditional WHILE node whose test runs on the device (fx_ctl.h).
    // nb points at max|b|, max|b'| on the device; the target, the cycles and a
    // failure are recorded in ctl.
    // end_in_next: the kernel that follows closes the solve's bookkeeping
    void enqueue_solve64_ctl(const DevParams& p, const uint8_t* code, double* phi, const double* rhs,
                             const double* nb, double rtol, int maxit, StepCtl* ctl, CondCapture& cap, cudaStream_t s,
                             bool end_in_next);
    void enqueue_solve_mixed_ctl(const DevParams& p, const uint8_t* code, double* phi, const double* rhs,
                                 const double* nb, double rtol, int maxit, StepCtl* ctl, CondCapture& cap,
                                 cudaStream_t s, bool end_in_next);
    // |b' - A phi|_inf with the electrode terms (FP64); r may be null
    int residual64(const DevParams& p, const uint8_t* code, const double* phi, const double* rhs, double* r,
                   cudaStream_t s, double* norm_out);
    size_t bytes() const { return bytes_; }
    const std::vector<MGLevel>& levels() const { return lev_; }
    int nu1 = 2, nu2 = 1, nu_bottom = 40;
    // sweeps on the levels below level 0, the one-CTA levels included (-1: nu1
    // / nu2).  One pre-smoothing sweep below level 0 measured fastest on the
    // polycrystal (both precisions) and the MFISM stack
    int nu1c = 1, nu2c = -1;
    int mixed_cycles = 2;    // FP32 V-cycles per FP64 refinement step
    bool alpha_tiles = true; // coarse alphas below level 1 in one launch (k_alpha_tiles)
    int seg_bytes = 16;      // point red-black half sweeps by row segments of 16 or 32 bytes where the shape allows (k_rbgs_seg); 0: one cell per thread
    long long seg_min_cells = 0;  // ... on levels of at least this many cells
    bool split_mode = true;  // level 0's FP32 correction and residual in the red-black split layout (mixed path)
    bool half_coarse = true; // the FP32 cycle's coarse face beta in FP16 (set before setup)
    // the one-CTA levels replaced, while alpha is absent, by the exact solve
    // with the dense inverse of the first one-CTA level's operator (built at
    // setup when that level has at most kDenseMax cells)
    bool dense_coarse = true;
    static constexpr int kDenseMax = 4096;

    static constexpr int kMaxLev = 24;
    Prof* prof = nullptr;
    int verbose = 0;
    void set_graphs(bool on) { use_graphs_ = on; }

private:
    std::vector<MGLevel> lev_;
    // level 0's FP32 arrays in the split layout for the solve being enqueued
    // (split0_ok at its start; every level-0 FP32 kernel and the FP64
    // residuals that write or read them follow it)
    bool split0_ok(const uint8_t* code, std::initializer_list<const void*> p64) const;
public:
    bool split_now_ = false;   // (read back as mg_level0_split: the last mixed solve used the split layout)
private:
    // the segment width for level 0's FP64 residual: 32 bytes whenever the
    // smoother runs by segments (measured faster than 16 for this kernel); 0:
    // one column of cells per thread
    int res_seg() const { return seg_bytes && !lev_.empty() && (long long)lev_[0].N >= seg_min_cells ? 32 : 0; }
    double eps_[8];
    const double* a0_64 = nullptr;
    const float* a0_32 = nullptr;
    bool has_alpha_ = false;
    double* d_norm_ = nullptr;       // device scalar
    double* h_norm_ = nullptr;       // pinned host
    float* e32_ = nullptr;           // level-0 FP32 correction
    float* r32_ = nullptr;           // level-0 FP32 residual
    double* alt64m_ = nullptr;       // second FP64 level-0 iterate of the mixed solve
    double* cp0_64_ = nullptr;       // level-0 line scratch
    float* cp0_32_ = nullptr;
    size_t bytes_ = 0;
    // one V-cycle (and its norm readback) captured as a CUDA graph, replayed
    // per cycle; re-captured when a captured launch parameter changes
    struct GraphCache {
        cudaGraphExec_t exec = nullptr;
        const void* x = nullptr;
        const void* rhs = nullptr;
        bool has_alpha = false;
        double vlo = 0, vhi = 0;
        int nu1 = 0, nu2 = 0, nu1c = 0, nu2c = 0;
        bool pdl = false, split = false, dense = false;
        int seg = 0;
        long long seg_min = 0;
        long long launches = 0;
    };
    GraphCache g64_, g32_, g32b_;   // g32b_: the refinement step from the second FP64 buffer
    bool use_graphs_ = true;
    template <typename F> int replay(GraphCache& g, const void* x, const void* rhs, const DevParams& p, cudaStream_t s, F&& enqueue);
    int coarse_top64_ = -1, coarse_top32_ = -1;   // first level run by the one-CTA kernel
    double* dinv64_ = nullptr;   // dense inverse of level coarse_top64_'s operator (alpha absent), or null
    float* dinv32_ = nullptr;    // ... of level coarse_top32_'s, FP32
    int build_dense(bool want64, bool want32);

    int* d_fvalid_ = nullptr;    // [0] FP64, [1] FP32: the one-CTA factors in global memory are current
    // k_alpha_tiles: tile level (0: per-level launches), level-l cells per
    // tile, the largest staged tile, and the last-block counter
    int at_T_ = 0;
    int at_tl_[kMaxLev][3] = {};
    int at_cap_ = 0;
    unsigned int* at_counter_ = nullptr;
    unsigned int* rc_counter_ = nullptr;   // last-block counter of the controlled residual kernel
    size_t coarse_smem64_ = 0, coarse_smem32_ = 0;
    void plan_coarse(bool want64, bool want32);
    double slots_max() const;
    template <typename T> int coarse_top() const;
    template <typename T> void launch_coarse(int top, cudaStream_t s);
    // zero: x starts at 0 (not read, not cleared by the caller)
    template <typename T> void vcycle(const DevParams& p, const uint8_t* code, int l, T* x0, const T* b0, bool inhom, cudaStream_t s,
                                      bool zero);
    template <typename T> void smooth(const DevParams& p, const uint8_t* code, int l, T* x, const T* b, bool inhom, int sweeps, cudaStream_t s,
                                      bool zero);
};

}  // namespace fx
