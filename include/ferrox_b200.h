/*
 * ferrox_b200.h -- C ABI of the B200 implementation of FerroX's coupled time
 * step (TDGL polarization update, semiconductor-charge Newton coupling,
 * variable-permittivity Poisson solve, E = -grad phi).
 *
 * The reference has no library API: its plugin surface is the inputs file,
 * the executable and the plotfile directory (Source/main.cpp:35-651), and its
 * hot path is a set of free functions on MultiFabs called from main_main.
 * Each entry point below names the reference function or loop section it
 * replaces.  All functions return FX_OK (0) or a negative FX_ERR_* status;
 * fx_last_error() gives the message.  The library owns all device memory.
 * Host pointers are borrowed for the duration of a call only.  One context
 * must not be used from two threads at once; all device work of a context is
 * ordered on one CUDA stream of the current device.
 *
 * Field layout everywhere: valid cells only, x fastest,
 * index = i + nx * (j + ny * k), FP64.
 */
#ifndef FERROX_B200_H
#define FERROX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FX_OK                   0
#define FX_ERR_INVALID_ARGUMENT (-1)
#define FX_ERR_INPUTS           (-2)   /* bad or missing inputs-file key (the reference's amrex::Abort) */
#define FX_ERR_UNSUPPORTED      (-3)
#define FX_ERR_CUDA             (-4)
#define FX_ERR_NO_CONVERGENCE   (-5)   /* multigrid or Newton iteration cap reached */
#define FX_ERR_NONFINITE        (-6)
#define FX_ERR_OUT_OF_MEMORY    (-7)
#define FX_ERR_IO               (-8)

/* Field ids: the plotfile variable order of Source/Plotfile.cpp:37-105, then
 * the Newton coefficient alpha_cc and the mobility Gamma. */
enum fx_field {
    FX_FIELD_PX = 0, FX_FIELD_PY, FX_FIELD_PZ, FX_FIELD_PHI, FX_FIELD_POISSON_RHS,
    FX_FIELD_EX, FX_FIELD_EY, FX_FIELD_EZ, FX_FIELD_HOLES, FX_FIELD_ELECTRONS,
    FX_FIELD_CHARGE, FX_FIELD_EPSILON, FX_FIELD_MASK, FX_FIELD_TPHASE,
    FX_FIELD_ANGLE_ALPHA, FX_FIELD_ANGLE_BETA, FX_FIELD_ANGLE_THETA, FX_FIELD_PHIDIFF,
    FX_FIELD_ALPHA_CC, FX_FIELD_GAMMA, FX_NFIELDS
};

typedef struct fx_ctx fx_ctx;

typedef struct fx_stats {
    int       step;                 /* last completed step of the main loop          */
    int       finished;             /* the reference loop's break condition was met  */
    int       newton_iters_last;    /* ComputePhi_Rho passes in the last call        */
    int       mg_cycles_last;       /* V-cycles (or refinement sweeps) in the last call */
    long long newton_iters_total;
    long long mg_cycles_total;
    long long kernel_launches;      /* this library's kernels launched so far         */
    double    mg_resid_last;        /* final |b - A phi|_inf of the last solve        */
    double    mg_target_last;       /* the stopping threshold it was held to          */
    double    phi_err_last;         /* Newton L1 change of the last ComputePhi_Rho    */
    double    steady_err_last;      /* CheckSteadyState norm of the last step         */
    double    Phi_Bc_hi;            /* present top-electrode value                    */
    double    time;
    int       steady_state_step;
    int       inc_step;
    int       num_Vapp;
    int       sign;
    double    device_bytes;         /* device memory held by the context              */
} fx_stats;

const char* fx_version(void);

/* Parse an inputs file (is_text = 0: path, 1: the text itself) and set up
 * masks, permittivity and the initial P on the host, as c_FerroX::InitData +
 * InitializeFerroXNamespace + InitializeMaterialMask + InitializePermittivity
 * + InitializePandRho do (Source/FerroX.cpp:150-572, main.cpp:65-226).
 * Device memory is allocated at the first call that needs the GPU.  An
 * embedded boundary (domain.embedded_boundary = 1, SetupMLMG_EB,
 * ElectrostaticSolver.cpp:613-676) is taken when it lies on grid faces: one
 * box with no fluid inside spanning x / y from a cell face to the top of z;
 * other geometries give FX_ERR_UNSUPPORTED.  On failure *out is NULL and
 * fx_create_error() holds the message. */
int         fx_create(const char* inputs, int is_text, fx_ctx** out);
/* message of the last failed fx_create (or fx_mean_P_noalloc) on this thread */
const char* fx_create_error(void);
void        fx_destroy(fx_ctx* ctx);
const char* fx_last_error(const fx_ctx* ctx);

int fx_get_dims(const fx_ctx* ctx, int n_cell[3], double dx[3]);
/* Scalar parameters by inputs-file key (FerroX namespace globals,
 * Source/FerroX_namespace.H:1-115), plus fx.* keys.  fx_get_param also
 * answers read-only diagnostics: contains_sc, num_variants, V_lo, V_hi,
 * phi_ref, intrinsic_carrier_concentration, adjoint_* (the last recorded
 * run), mg_level0_planes (1 when level 0's face coefficients depend on z
 * only and are read by plane) and step_graph_ran (1 when the last step ran
 * as one CUDA graph with its Newton and multigrid loop tests on the device,
 * fx.step_graph = 1; 0 when the host-driven loop ran it), eb_fluid_layers
 * and eb_surf_soln (domain.embedded_boundary = 1: the layers below the
 * embedded surface that the Poisson solve covers, 0 without one, and the
 * surface's Dirichlet value). */
int fx_get_param(const fx_ctx* ctx, const char* key, double* value);
int fx_set_param(fx_ctx* ctx, const char* key, double value);

/* Replaces the random initial P of InitializePandRho (Initialization.cpp:
 * 83-132); Px and Py may be NULL (zero). */
int fx_set_initial_P(fx_ctx* ctx, const double* Px, const double* Py, const double* Pz, size_t n);
/* Polycrystal input: per-cell grain id (255 = no grain), per-grain Euler
 * angles in degrees (3 per grain, the angle_alpha/beta/theta fields of
 * Initialize_Euler_angles, Initialization.cpp:297-383) and per-grain t-phase
 * flag (the tphase mask, :252-294).  Must precede the first device call. */
int fx_set_grains(fx_ctx* ctx, const uint8_t* grain_id, size_t n, const double* angles_deg,
                  const uint8_t* grain_tphase, int ngrains);
/* Per-grain Landau alpha (replaces the global alpha in grain cells). */
int fx_set_grain_alpha(fx_ctx* ctx, const double* alpha, int ngrains);
/* 0 = plain FP64; 1 = FP32 stencils and multigrid with FP64 refinement. */
int fx_set_precision(fx_ctx* ctx, int mode);

int fx_get_field(fx_ctx* ctx, int field, double* host_out, size_t n);
/* Px, Py, Pz, Phi only */
int fx_set_field(fx_ctx* ctx, int field, const double* host_in, size_t n);

/* -- the reference's hot-path functions, on the context's fields -------- */
int fx_compute_poisson_rhs(fx_ctx* ctx);  /* ComputePoissonRHS, ElectrostaticSolver.cpp:8-83       */
int fx_compute_rho(fx_ctx* ctx);          /* ComputeRho, ChargeDensity.cpp:15-102                   */
int fx_compute_phi_rho(fx_ctx* ctx);      /* ComputePhi_Rho, ElectrostaticSolver.cpp:678-747        */
int fx_compute_E(fx_ctx* ctx);            /* ComputeEfromPhi, ElectrostaticSolver.cpp:134-203       */
int fx_tdgl_euler(fx_ctx* ctx);           /* Calculate_Landau/Grad/Elec + CalculateTDGL_RHS +
                                             LinComb, TotalEnergyDensity.cpp:6-294, main.cpp:280-306 */
int fx_set_phi_bc(fx_ctx* ctx);           /* SetPhiBC_z + setLevelBC, ElectrostaticSolver.cpp:502-524 */
int fx_check_steady_state(fx_ctx* ctx, int step); /* CheckSteadyState, ElectrostaticSolver.cpp:526-560 */

/* nsteps passes of the main.cpp:261-621 loop body (coupled step, steady-state
 * check, voltage sweep, exit tests); stops early when the reference loop
 * would break.  *steps_done may be NULL. */
int fx_step(fx_ctx* ctx, int nsteps, int* steps_done);
/* The whole loop for the inputs' nsteps, with plotfiles at plot_int
 * (main.cpp:228-234, :563-570) and the reference's progress lines if verbose. */
int fx_run(fx_ctx* ctx, int* steps_done);
/* WritePlotfile (Source/Plotfile.cpp:5-178): <dir>/pltNNNNNNNN in AMReX
 * plotfile format (HyperCLaw-V1.1, one box, FP64). */
int fx_write_plotfile(fx_ctx* ctx, int step, const char* dir);
int fx_get_stats(const fx_ctx* ctx, fx_stats* out);
/* <Px>, <Py>, <Pz> over the ferroelectric (mask 0) cells: the hysteresis
 * observable a voltage sweep records each step (the reference writes P to
 * plotfiles and leaves the averaging to post-processing). */
int fx_mean_P(fx_ctx* ctx, double out[3]);
int fx_sync(fx_ctx* ctx);

/* Order the context's device work on the caller's cudaStream_t instead of
 * its own stream (the reference runs on AMReX's default stream). */
int fx_set_stream(fx_ctx* ctx, void* cuda_stream);

/* Per-launch CUDA-event timing of the kernel classes below, enabled with
 * fx_set_param(ctx, "fx.profile", 1): summed milliseconds and launch counts.
 * Returns the number of classes (FX_KT_COUNT). */
enum fx_kernel_class {
    FX_KT_TDGL = 0, FX_KT_RHS_P, FX_KT_NEWTON, FX_KT_RHO, FX_KT_STEADY, FX_KT_SMOOTH_L0,
    FX_KT_RESTRICT_L0, FX_KT_PROLONG_L0, FX_KT_MG_COARSE, FX_KT_RESID64, FX_KT_EFIELD, FX_KT_MG_L1,
    FX_KT_MG_L2, FX_KT_COARSE_CTA, FX_KT_COUNT
};
int fx_get_kernel_times(fx_ctx* ctx, double* ms, long long* counts, int n);
int fx_reset_kernel_times(fx_ctx* ctx);

/* ---- Gradients (no counterpart in the reference, which has no adjoint).
 *
 * A hysteresis loss over nsteps forward-Euler steps of the coupled step
 * (main.cpp:261-306 without the sweep logic): at step n (1-based) the top
 * electrode is held at Phi_Bc_hi = v_amp * v_shape[n-1], phi^n is solved
 * from P^{n-1} (ComputePhi_Rho) and P^n = P^{n-1} + dt f (CalculateTDGL_RHS);
 *     L = (1/nsteps) sum_n (<Pz>^n - target[n-1])^2,
 * <Pz> the mean over the ferroelectric cells (mask 0).  fx_forward_record
 * runs those steps from the context's current state, keeps FP64 checkpoints
 * of P and phi every checkpoint_every steps, and returns L; fx_backward then
 * recomputes each checkpoint segment and runs the hand-written adjoint (the
 * transposed TDGL step, the Poisson adjoint solved by the same multigrid with
 * rho'(phi) on the semiconductor cells) back to step 0.  Between the two calls
 * nothing may change the context (no fx_step, fx_set_param, fx_set_field ...);
 * after fx_backward the context holds the state at the end of the recorded
 * steps again.  TimeIntegratorOrder 2 is not supported (FX_ERR_UNSUPPORTED).
 */
typedef struct fx_loss_spec {
    int           nsteps;            /* >= 1 */
    int           checkpoint_every;  /* k >= 1: P and phi kept at steps 0, k, 2k, ... */
    double        v_amp;             /* volts */
    const double* v_shape;           /* nsteps values, or NULL for all ones */
    const double* target;            /* nsteps values of the target <Pz> (C/m^2) */
} fx_loss_spec;

/* gradient slots of fx_backward */
enum fx_grad {
    FX_GRAD_ALPHA = 0,   /* Landau alpha, over the cells that use the global alpha */
    FX_GRAD_BETA,        /* Landau beta */
    FX_GRAD_GAMMA,       /* Landau gamma */
    FX_GRAD_G11,         /* gradient coefficient g11 */
    FX_GRAD_G44,         /* gradient coefficient g44 */
    FX_GRAD_V_AMP,       /* the voltage amplitude v_amp */
    FX_GRAD_GRAIN_ALPHA  /* first of the per-grain alphas: slot 6 + g is dL/d alpha of grain g */
};

int fx_forward_record(fx_ctx* ctx, const fx_loss_spec* spec, double* loss);
/* grads: ngrads >= 6 slots (enum fx_grad); with grains set, slots 6 .. 6 +
 * ngrains - 1 receive the per-grain alpha gradients, further slots 0. */
int fx_backward(fx_ctx* ctx, double* grads, int ngrads);
/* dL/dP^0, the gradient with respect to the state fx_forward_record started
 * from, after fx_backward.  With scalar polarization (is_polarization_scalar
 * = 1 and Px = Py = 0) only dPz is available: pass NULL for dPx and dPy. */
int fx_get_grad_P0(fx_ctx* ctx, double* dPx, double* dPy, double* dPz, size_t n);

/* No counterpart in the reference.  fx_mean_P without any device allocation,
 * for callers that cannot call cudaMalloc where they need the number (memory
 * owned by another allocator, or code that must not synchronise the device).
 * Inputs are the caller's device arrays: Px and Py may be NULL, mask holds
 * one byte per cell with 0 for ferroelectric cells; d_out receives <Px>, <Py>,
 * <Pz> (3 doubles, device).  The work is enqueued on cuda_stream and the call
 * returns without waiting.  Scratch is a static device array of about 32 KB
 * that every GPU loading the library keeps until exit; n may be at most
 * 16,777,216 cells (larger n returns FX_ERR_INVALID_ARGUMENT).  The first call
 * on a device looks up that array's device address, so make the first call
 * before any stream capture.  Calls that overlap on the GPU share the scratch
 * and race: order them on one stream.  The looked-up address is kept for the
 * life of the process: do not call this after cudaDeviceReset (or after the
 * device's primary context was destroyed and made again) in the same
 * process, since the kept address then no longer names the array.  Errors are
 * reported through the return code and fx_create_error(). */
int fx_mean_P_noalloc(const double* d_Px, const double* d_Py, const double* d_Pz, const uint8_t* d_mask, size_t n,
                      double* d_out, void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif
