// fx_kernels.h -- launchers of the coupled-step kernels (fx_kernels.cu) and
// of the Poisson multigrid (fx_mg.cu).  All launches go to the given stream.
#pragma once

#include <cuda_runtime.h>

#include "fx_ctl.h"
#include "fx_device.cuh"

namespace fx {

// Pin/Pout: {Px, Py, Pz}; Px = Py = nullptr selects the scalar-P kernel.
// mode 0: Euler; 1: predictor (writes fbuf); 2: corrector (reads fbuf, Pold);
// skip (step graphs): a device flag; nonzero leaves the launch without effect
int launch_tdgl(const DevParams& p, int mixed, int mode, const uint8_t* code, const uint8_t* var, const Variant* vt,
                const double* const Pin[3], double* const Pout[3], const double* phi, double* const fbuf[3],
                const double* const Pold[3], cudaStream_t s, const int* skip = nullptr);
int launch_rhs_p(const DevParams& p, const uint8_t* code, const uint8_t* var, const Variant* vt,
                 const double* const P[3], double* rhs, double* norms, cudaStream_t s);
int launch_newton(const DevParams& p, const uint8_t* code, const double* phi, const double* rho,
                  const double* rhs_p, double* alpha, float* alpha32, double* rhs, double* norms, cudaStream_t s);
// rc (step graphs): the last block also runs the loop control of fx_ctl.h
int launch_rho(const DevParams& p, const uint8_t* code, const double* phi, double* phi_prev, double* rho,
               double* e_den, double* h_den, double* part, unsigned int* counter, double* out, int track,
               int carriers, cudaStream_t s, const RhoCtl* rc = nullptr);
// skip (step graphs): a device flag; nonzero leaves the launch without effect
int launch_steady(const DevParams& p, const double* phi, double* phi_old, double* dphi, double* out,
                  cudaStream_t s, const int* skip = nullptr);
int launch_mean_p(const DevParams& p, const uint8_t* code, const double* const P[3], double* part,
                  unsigned int* counter, double* out, cudaStream_t s);
// h: the history buffers, null beyond the configured order; order: the steps of
// history in use (1-6)
int launch_phi_extrap(const DevParams& p, int order, double* phi, double* const h[6], cudaStream_t s);
int launch_efield(const DevParams& p, const uint8_t* var, const Variant* vt, const double* phi, double* E[3],
                  cudaStream_t s);

// control of a step graph (fx_ctl.h): step and ComputePhi_Rho bookkeeping;
// phirho_end also opens the IF node `gate` (0: none) of body `kind` while no
// failure is recorded
// (both zero out[0..1], the norm accumulators of what follows)
int launch_ctl_step_begin(StepCtl* ctl, double* out, cudaStream_t s);
int launch_ctl_phirho_begin(StepCtl* ctl, double* out, cudaStream_t s);
int launch_ctl_phirho_end(StepCtl* ctl, int sc, cudaGraphConditionalHandle gate, int kind, cudaStream_t s);

// adjoint (fx_adjoint.cu).  lam = {lambda_x, lambda_y, lambda_z}; vec = the
// three-component kernels (else only lambda_z is read and written)
int launch_adj_init(const DevParams& p, const uint8_t* code, double* lam[3], double g, cudaStream_t s);
int launch_adj_phi(const DevParams& p, int mixed, bool vec, const uint8_t* code, const uint8_t* var, const Variant* vt,
                   double* const lam[3], double* mu, double* norm, double* dV, cudaStream_t s);
int launch_adj_P(const DevParams& p, int mixed, bool vec, const uint8_t* code, const uint8_t* var, const Variant* vt,
                 const uint8_t* gid, int ngalpha, const double* const P[3], double* const lam[3], const double* psi,
                 double gload, double* const lam_out[3], double* grad, double* dV, cudaStream_t s);
int launch_drho(const DevParams& p, const uint8_t* code, const double* phi, double* a64, float* a32, cudaStream_t s);
// psi = 0 when *nmu (the adjoint source's max) is not positive
int launch_zero_if_zero(double* psi, const double* nmu, long long n, cudaStream_t s);

}  // namespace fx
