/*
 * ofx_oracle.h -- CPU oracle for the FerroX coupled time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain FP64 C++ restatement of the
 * reference's arithmetic (FerroX, the Source/Solver sources and Source/main.cpp), used
 * by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg as
 * the checker.  Nothing in the product library links or calls it.
 *
 * Pinning: the reference ships no tests, golden vectors or benchmark
 * plotfiles, and it cannot be compiled here (AMReX is absent), so the oracle is
 * pinned against closed-form known-answer cases (Landau polynomial, stencils on
 * polynomials, the lambda boundary forms, uniform-eps and two-layer capacitor
 * Poisson solutions, carrier densities at phi_ref, the Boltzmann limit of
 * FD_half).  The AMReX MLMG solve, amrex::Random and amrex::Parser are
 * third-party algorithms absent from the reference tree: for those the parity
 * is unpinned (the oracle solves the same discrete operator to a stated
 * relative residual).
 */
#ifndef OFX_ORACLE_H
#define OFX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* All physics keys of InitializeFerroXNamespace (Source/FerroX.cpp:273-572)
 * and the domain keys of c_GeometryProperties (GeometryProperties.cpp:86-173)
 * that the Order-1 / Order-2 time loop reads, plus the fx.* extensions. */
typedef struct ofx_params {
    int    n_cell[3];
    double prob_lo[3];
    double prob_hi[3];
    int    is_periodic[3];

    int    prob_type;
    int    TimeIntegratorOrder;
    int    nsteps;
    int    plot_int;
    double dt;

    int    P_BC_flag_lo[3];
    int    P_BC_flag_hi[3];
    double lambda;

    double epsilon_0, epsilonX_fe, epsilonX_fe_tphase, epsilonZ_fe, epsilon_de, epsilon_si;
    double alpha, beta, gamma, alpha_12, alpha_112, alpha_123;
    double BigGamma, g11, g44, g12, g44_p;

    double FE_lo[3], FE_hi[3], DE_lo[3], DE_hi[3], SC_lo[3], SC_hi[3];
    double Channel_lo[3], Channel_hi[3];
    double Remnant_P[3];

    double acceptor_doping, donor_doping;
    int    use_Fermi_Dirac, use_work_function;
    double metal_work_function;

    int    is_polarization_scalar;
    double delta;
    int    voltage_sweep, inc_step;
    double Phi_Bc_lo, Phi_Bc_hi, Phi_Bc_inc, Phi_Bc_hi_max, phi_tolerance;
    int    num_Vapp_max, random_seed;
    int    include_Landau, include_Grad, include_Elec;
    int    Coordinate_Transformation, use_Euler_angles;

    /* fx.* extensions */
    double mg_rtol;          /* relative residual target of each Poisson solve   */
    int    phi_ghost_mode;   /* 0 = extrap (2V - phi0), 1 = face (V), 2 = zero   */
    int    sweep_mode;       /* 0 = steady (reference), 1 = fixed cadence         */
    int    steps_per_voltage;
    int    newton_max_iter;
    int    mg_max_iter;
    int    verbose;
} ofx_params;

typedef struct ofx_ctx ofx_ctx;

/* field ids: same order as the plotfile (Source/Plotfile.cpp:37-105) */
enum {
    OFX_PX = 0, OFX_PY, OFX_PZ, OFX_PHI, OFX_POISSON_RHS, OFX_EX, OFX_EY, OFX_EZ,
    OFX_HOLES, OFX_ELECTRONS, OFX_CHARGE, OFX_EPSILON, OFX_MASK, OFX_TPHASE,
    OFX_ANGLE_ALPHA, OFX_ANGLE_BETA, OFX_ANGLE_THETA, OFX_PHIDIFF,
    OFX_ALPHA_CC, OFX_GAMMA, OFX_NFIELDS
};

/* tphase / angle arrays: valid cells, x fastest; NULL means all zero. */
ofx_ctx* ofx_create(const ofx_params* p, const double* tphase,
                    const double* ang_alpha, const double* ang_beta, const double* ang_theta);
void     ofx_destroy(ofx_ctx* c);
int      ofx_set_threads(int n);

/* valid-cell copies (x fastest); the mask additionally via ofx_get_mask_ghost */
int ofx_get_field(ofx_ctx* c, int id, double* out);
int ofx_set_field(ofx_ctx* c, int id, const double* in);
int ofx_get_mask_ghost(ofx_ctx* c, double* out);     /* (nx+2)(ny+2)(nz+2) */
int ofx_get_phi_ghost(ofx_ctx* c, double* out);      /* (nx+2)(ny+2)(nz+2) */
int ofx_get_beta_faces(ofx_ctx* c, double* bx, double* by, double* bz);

/* single reference functions, operating on the context's fields */
int ofx_compute_poisson_rhs(ofx_ctx* c);     /* ElectrostaticSolver.cpp:8-83   */
int ofx_compute_rho(ofx_ctx* c);             /* ChargeDensity.cpp:15-102       */
int ofx_compute_phi_rho(ofx_ctx* c);         /* ElectrostaticSolver.cpp:678-747 */
int ofx_compute_E(ofx_ctx* c);               /* ElectrostaticSolver.cpp:134-203 */
int ofx_tdgl_euler(ofx_ctx* c);              /* TotalEnergyDensity.cpp + main.cpp:280-306 */
int ofx_set_phi_bc(ofx_ctx* c);              /* ElectrostaticSolver.cpp:502-524 */
/* one pass of the main.cpp:261-621 loop body (with sweep and steady state).
 * Returns 1 when the loop would break, 0 to continue, <0 on error. */
int ofx_step(ofx_ctx* c, int step);
int ofx_run(ofx_ctx* c, int nsteps);          /* steps 1..nsteps, stops on break */

/* Poisson solve of (-alpha - div beta grad) phi = rhs with the context's
 * coefficients and z Dirichlet values; phi is the initial guess and result. */
int ofx_poisson_solve(ofx_ctx* c, const double* rhs, const double* alpha_cc,
                      double* phi, double rtol, int* iters_out, double* resid_out);
int ofx_poisson_apply(ofx_ctx* c, const double* alpha_cc, const double* phi,
                      int inhomogeneous, double* out);
// a grid-aligned embedded boundary covering the layers k >= nz_fluid (0:
// none): later Poisson solves run on the layers below it, their top face a
// Dirichlet face at V with the cell's own beta; call before the first solve
int ofx_set_eb(ofx_ctx* c, int nz_fluid, double V);

/* Calculate_Landau / Calculate_Grad / Calculate_Elec outputs for the current
 * P and E (3 x N each, x fastest) */
int ofx_tdgl_terms(ofx_ctx* c, double* landau, double* grad, double* elec);

/* scalar state */
double ofx_get_scalar(ofx_ctx* c, const char* name);
int    ofx_set_scalar(ofx_ctx* c, const char* name, double v);

/* deterministic seeded uniform in [0,1): the n-th draw (n >= 1) of a
 * splitmix64 stream started at `seed`, top 53 bits */
double ofx_uniform(unsigned long long seed, unsigned long long n);

#ifdef __cplusplus
}
#endif
#endif
