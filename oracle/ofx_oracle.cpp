// ofx_oracle.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY, see ofx_oracle.h).
//
// A plain FP64 restatement of the FerroX reference arithmetic.  Every function
// names the reference file:line it follows.  Fields are held the way the
// reference's MultiFabs hold them: one box covering the domain with the same
// number of ghost cells, and FillBoundary with periodic images, so that every
// ghost-cell read of the reference stencils reads the same value here.
//
// The one piece that is not a restatement is the Poisson solve: the reference
// calls AMReX MLMG (MLABecLaplacian, ElectrostaticSolver.cpp:562-611, solve at
// :719), which is absent from the reference tree.  It is replaced by a
// residual-correction geometric multigrid in the style of MLMG (red-black
// Gauss-Seidel, 2+2 sweeps, averaging restriction, face-averaged coefficients,
// CG bottom solve, infinity-norm stopping rule |r| <= rtol * max(|r0|, |rhs|)),
// with semicoarsening of the finely spaced directions and linear
// cell-centred prolongation so that it converges for the stacks' dz != dx.
// It solves the same discrete operator; its parity is unpinned.
#include "ofx_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- Fab ------
struct Fab {
    int nx = 0, ny = 0, nz = 0, ng = 0;
    long sx = 0, sy = 0;
    std::vector<double> v;
    void define(int nx_, int ny_, int nz_, int ng_) {
        nx = nx_; ny = ny_; nz = nz_; ng = ng_;
        sx = nx + 2 * ng; sy = ny + 2 * ng;
        v.assign((size_t)sx * sy * (nz + 2 * ng), 0.0);
    }
    inline double& operator()(int i, int j, int k) {
        return v[(size_t)(i + ng) + (size_t)(j + ng) * sx + (size_t)(k + ng) * sx * sy];
    }
    inline double operator()(int i, int j, int k) const {
        return v[(size_t)(i + ng) + (size_t)(j + ng) * sx + (size_t)(k + ng) * sx * sy];
    }
    void setVal(double a) { std::fill(v.begin(), v.end(), a); }
};

// AMReX FillBoundary(geom.periodicity()) on a single box: a ghost cell takes
// the value of its periodic image when that image is a valid cell; all other
// ghost cells are left untouched.
void fill_boundary(Fab& f, const int per[3]) {
    const int n[3] = {f.nx, f.ny, f.nz};
    const int g = f.ng;
    if (g == 0) return;
    for (int k = -g; k < f.nz + g; ++k)
        for (int j = -g; j < f.ny + g; ++j)
            for (int i = -g; i < f.nx + g; ++i) {
                int c[3] = {i, j, k};
                bool ghost = false, ok = true;
                for (int d = 0; d < 3; ++d) {
                    if (c[d] < 0 || c[d] >= n[d]) {
                        ghost = true;
                        if (per[d]) c[d] = ((c[d] % n[d]) + n[d]) % n[d];
                        else ok = false;
                    }
                }
                if (ghost && ok) f(i, j, k) = f(c[0], c[1], c[2]);
            }
}

// Silicon constants, Source/FerroX.cpp:534-554.
struct SiConst {
    double Nc = 2.8e25, Nv = 1.83e25, bandgap = 1.12, affinity = 4.05;
    double q = 1.602e-19, kb = 1.38e-23, T = 300;
    double Ea = 44.0e-3, Ed = 46.0e-3;
    double ni = 0.0;
};

// ------------------------------------------------------------ multigrid ----
struct MGLevel {
    int n[3];
    double h[3];
    int cr[3] = {1, 1, 1};           // coarsening ratio from the finer level
    std::vector<double> wfar[3];     // prolongation weight of the far coarse cell, per fine cell of the finer level
    std::vector<double> a;           // alpha_cc (A = -1 multiplies it)
    std::vector<double> bx, by, bz;  // face coefficients (nx+1)*ny*nz etc.
    std::vector<double> x, r, t;     // correction, rhs, scratch
    size_t N() const { return (size_t)n[0] * n[1] * n[2]; }
};

} // namespace

struct ofx_ctx {
    ofx_params p;
    SiConst si;
    int n[3];
    double dx[3];
    size_t N;

    Fab mask, tphase, Gamma;
    Fab P[3], Pnew[3], Ppre[3];
    Fab GL[3], GLL[3], GLG[3], GLE[3], GLpre[3];
    Fab E[3];
    Fab phi, phi_old, phi_prev, phidiff;
    Fab rhs, rho, e_den, h_den, alpha_cc;
    Fab beta_cc;
    Fab ang[3];
    std::vector<double> bxf, byf, bzf;   // beta on faces
    // a grid-aligned embedded boundary covering the layers k >= eb_nz
    // (0: none): the solve runs on the layers below it with the Dirichlet
    // value eb_V on their top face (ofx_set_eb)
    int eb_nz = 0;
    double eb_V = 0.0;
    double V_lo = 0.0, V_hi = 0.0;       // Dirichlet values held by setLevelBC
    bool contains_sc = false;

    // loop state (main.cpp:238-242)
    int steady_state_step = 1000000;
    int sign = 1;
    int num_Vapp = 0;
    double time = 0.0;
    int inc_step = 0;
    double Phi_Bc_hi = 0.0;

    // statistics
    int last_newton_iters = 0;
    int last_mg_iters = 0;
    double last_phi_err = 0.0;
    double last_steady_err = 0.0;

    std::vector<MGLevel> mg;
};

namespace {

inline double pw(double x, double e) { return std::pow(x, e); }

// ------------------------------------------- DerivativeAlgorithm.H:8-497 --
// Faithful restatements; F is a P component or phi, mask the material mask.
struct Stencil {
    const ofx_params* p;
    double dx[3];
    double lambda;

    // DphiDz, DerivativeAlgorithm.H:8-22
    double DphiDz(const Fab& F, double z_hi, double z_lo, int i, int j, int k,
                  const double* prob_lo, const double* prob_hi) const {
        if (z_lo < prob_lo[2]) {
            return (-4. * F(i, j, k - 1) + 3. * F(i, j, k) + F(i, j, k + 1)) / (3. * dx[2]);
        } else if (z_hi > prob_hi[2]) {
            return (4. * F(i, j, k + 1) - 3. * F(i, j, k) - F(i, j, k - 1)) / (3. * dx[2]);
        } else {
            return (F(i, j, k + 1) - F(i, j, k - 1)) / (2. * dx[2]);
        }
    }
    // DFDx / DFDy, DerivativeAlgorithm.H:26-40
    double DFDx(const Fab& F, int i, int j, int k) const { return (F(i + 1, j, k) - F(i - 1, j, k)) / (2. * dx[0]); }
    double DFDy(const Fab& F, int i, int j, int k) const { return (F(i, j + 1, k) - F(i, j - 1, k)) / (2. * dx[1]); }

    // DPDx / DPDy / DPDz, DerivativeAlgorithm.H:45-252, written once over the
    // direction d with unit offsets (ox, oy, oz).
    double DPD(int d, const Fab& F, const Fab& mask, int i, int j, int k) const {
        const int ox = d == 0, oy = d == 1, oz = d == 2;
        const double h = dx[d];
        const int flo = p->P_BC_flag_lo[d], fhi = p->P_BC_flag_hi[d];
        if (mask(i - ox, j - oy, k - oz) != 0.0 && mask(i, j, k) == 0.0) {
            if (flo == 0) {
                double F_lo = 0.0;
                return (-4. * F_lo + 3. * F(i, j, k) + F(i + ox, j + oy, k + oz)) / (3. * h);
            } else if (flo == 1) {
                double F_lo = F(i, j, k) / (1 + h / 2 / lambda);
                return (h * F_lo / lambda - F(i, j, k) + F(i + ox, j + oy, k + oz)) / (2. * h);
            } else if (flo == 2) {
                return (-F(i, j, k) + F(i + ox, j + oy, k + oz)) / (2. * h);
            } else if (flo == 3) {
                return (-F(i - ox, j - oy, k - oz) + F(i + ox, j + oy, k + oz)) / (2. * h);
            } else if (flo == 4) {
                return (-F(i, j, k) + F(i + ox, j + oy, k + oz)) / (h);
            }
            return 0.0;
        } else if (mask(i + ox, j + oy, k + oz) != 0.0 && mask(i, j, k) == 0.0) {
            if (fhi == 0) {
                double F_hi = 0.0;
                return (4. * F_hi - 3. * F(i, j, k) - F(i - ox, j - oy, k - oz)) / (3. * h);
            } else if (fhi == 1) {
                double F_hi = F(i, j, k) / (1 - h / 2 / lambda);
                return (h * F_hi / lambda + F(i, j, k) - F(i - ox, j - oy, k - oz)) / (2. * h);
            } else if (fhi == 2) {
                return (F(i, j, k) - F(i - ox, j - oy, k - oz)) / (2. * h);
            } else if (fhi == 3) {
                return (F(i + ox, j + oy, k + oz) - F(i - ox, j - oy, k - oz)) / (2. * h);
            } else if (fhi == 4) {
                return (F(i, j, k) - F(i - ox, j - oy, k - oz)) / (h);
            }
            return 0.0;
        } else if (mask(i, j, k) == 0.0) {
            return (F(i + ox, j + oy, k + oz) - F(i - ox, j - oy, k - oz)) / (2. * h);
        } else {
            return 0.0;
        }
    }

    // DoubleDPDx / y / z, DerivativeAlgorithm.H:256-467
    double DDPD(int d, const Fab& F, const Fab& mask, int i, int j, int k) const {
        const int ox = d == 0, oy = d == 1, oz = d == 2;
        const double h = dx[d];
        const int flo = p->P_BC_flag_lo[d], fhi = p->P_BC_flag_hi[d];
        if (mask(i - ox, j - oy, k - oz) != 0.0 && mask(i, j, k) == 0.0) {
            if (flo == 0) {
                double F_lo = 0.0;
                return 4. * (2. * F_lo - 3. * F(i, j, k) + F(i + ox, j + oy, k + oz)) / 3. / h / h;
            } else if (flo == 1) {
                double F_lo = F(i, j, k) / (1 + h / 2 / lambda);
                return (-h * F_lo / lambda - F(i, j, k) + F(i + ox, j + oy, k + oz)) / h / h;
            } else if (flo == 2) {
                return (-F(i, j, k) + F(i + ox, j + oy, k + oz)) / h / h;
            } else if (flo == 3) {
                if (d == 2)   // :420 writes the z form as F(k-1) - 2F + F(k+1)
                    return (F(i - ox, j - oy, k - oz) - 2. * F(i, j, k) + F(i + ox, j + oy, k + oz)) / h / h;
                return (F(i + ox, j + oy, k + oz) - 2. * F(i, j, k) + F(i - ox, j - oy, k - oz)) / h / h;
            } else if (flo == 4) {
                if (d == 2)   // :423 orders F(k) - 2F(k+1) + F(k+2)
                    return (F(i, j, k) - 2. * F(i + ox, j + oy, k + oz) + F(i + 2 * ox, j + 2 * oy, k + 2 * oz)) / h / h;
                return (F(i + 2 * ox, j + 2 * oy, k + 2 * oz) - 2. * F(i + ox, j + oy, k + oz) + F(i, j, k)) / h / h;
            }
            return 0.0;
        } else if (mask(i + ox, j + oy, k + oz) != 0.0 && mask(i, j, k) == 0.0) {
            if (fhi == 0) {
                double F_hi = 0.0;
                return 4. * (2. * F_hi - 3. * F(i, j, k) + F(i - ox, j - oy, k - oz)) / 3. / h / h;
            } else if (fhi == 1) {
                double F_hi = F(i, j, k) / (1 - h / 2 / lambda);
                return (h * F_hi / lambda - F(i, j, k) + F(i - ox, j - oy, k - oz)) / h / h;
            } else if (fhi == 2) {
                return (-F(i, j, k) + F(i - ox, j - oy, k - oz)) / h / h;
            } else if (fhi == 3) {
                return (F(i + ox, j + oy, k + oz) - 2. * F(i, j, k) + F(i - ox, j - oy, k - oz)) / h / h;
            } else if (fhi == 4) {
                return (F(i, j, k) - 2. * F(i - ox, j - oy, k - oz) + F(i - 2 * ox, j - 2 * oy, k - 2 * oz)) / h / h;
            }
            return 0.0;
        } else if (mask(i, j, k) == 0.0) {
            return (F(i + ox, j + oy, k + oz) - 2. * F(i, j, k) + F(i - ox, j - oy, k - oz)) / (h * h);
        } else {
            return 0.0;
        }
    }
    // DoubleDPDxDy / DxDz / DyDz, DerivativeAlgorithm.H:471-497
    double DxDy(const Fab& F, const Fab& m, int i, int j, int k) const {
        return (DPD(1, F, m, i + 1, j, k) - DPD(1, F, m, i - 1, j, k)) / 2. / dx[0];
    }
    double DxDz(const Fab& F, const Fab& m, int i, int j, int k) const {
        return (DPD(2, F, m, i + 1, j, k) - DPD(2, F, m, i - 1, j, k)) / 2. / dx[0];
    }
    double DyDz(const Fab& F, const Fab& m, int i, int j, int k) const {
        return (DPD(2, F, m, i, j + 1, k) - DPD(2, F, m, i, j - 1, k)) / 2. / dx[1];
    }
};

// Rotation matrix from Euler angles in degrees, as computed per cell at
// TotalEnergyDensity.cpp:167-195 / ElectrostaticSolver.cpp:35-63 / :165-193.
void rotation(int use_euler, double a_deg, double b_deg, double t_deg, double R[9]) {
    double Pi = 3.14159265358979323846;
    double alpha_rad = Pi / 180. * a_deg;
    double beta_rad = Pi / 180. * b_deg;
    double theta_rad = Pi / 180. * t_deg;
    if (use_euler) {
        R[0] = cos(alpha_rad) * cos(theta_rad) - cos(beta_rad) * sin(alpha_rad) * sin(theta_rad);
        R[1] = sin(alpha_rad) * cos(theta_rad) + cos(beta_rad) * cos(alpha_rad) * sin(theta_rad);
        R[2] = sin(beta_rad) * sin(theta_rad);
        R[3] = -cos(beta_rad) * cos(theta_rad) * sin(alpha_rad) - cos(alpha_rad) * sin(theta_rad);
        R[4] = cos(beta_rad) * cos(alpha_rad) * cos(theta_rad) - sin(alpha_rad) * sin(theta_rad);
        R[5] = sin(beta_rad) * cos(theta_rad);
        R[6] = sin(alpha_rad) * sin(beta_rad);
        R[7] = -cos(alpha_rad) * sin(beta_rad);
        R[8] = cos(beta_rad);
    } else {
        R[0] = cos(beta_rad) * cos(theta_rad);
        R[1] = sin(alpha_rad) * sin(beta_rad) * cos(theta_rad) - cos(alpha_rad) * sin(theta_rad);
        R[2] = cos(alpha_rad) * sin(beta_rad) * cos(theta_rad) + sin(alpha_rad) * sin(theta_rad);
        R[3] = cos(beta_rad) * sin(theta_rad);
        R[4] = sin(beta_rad) * sin(alpha_rad) * sin(theta_rad) + cos(alpha_rad) * cos(theta_rad);
        R[5] = cos(alpha_rad) * sin(beta_rad) * sin(theta_rad) - sin(alpha_rad) * cos(theta_rad);
        R[6] = -sin(beta_rad);
        R[7] = sin(alpha_rad) * cos(beta_rad);
        R[8] = cos(alpha_rad) * cos(beta_rad);
    }
}

uint64_t splitmix_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

Stencil make_stencil(const ofx_ctx* c) {
    Stencil s;
    s.p = &c->p;
    for (int d = 0; d < 3; ++d) s.dx[d] = c->dx[d];
    s.lambda = c->p.lambda;
    return s;
}

// ----------------------------------------- ChargeDensity.cpp:4-11, 15-102 --
double FD_half(const double eta) {
    double nu = pw(eta, 4.0) + 50.0 + 33.6 * eta * (1.0 - 0.68 * exp(-0.17 * pw((eta + 1.0), 2.0)));
    double xi = 3.0 * sqrt(3.14) / (4.0 * pw(nu, 3. / 8.));
    double integral = pw(exp(-eta) + xi, -1.0);
    return integral;
}

void compute_rho(ofx_ctx* c, const Fab& phi, Fab& rho, Fab& e_den, Fab& p_den) {
    const SiConst& s = c->si;
    const ofx_params& P = c->p;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i) {
                if (c->mask(i, j, k) >= 2.0) {
                    double Ef = 0.0;
                    double Eg = s.bandgap;
                    double Chi = s.affinity;
                    double phi_ref = Chi + 0.5 * Eg + 0.5 * s.kb * s.T * log(s.Nc / s.Nv) / s.q;
                    double Ec_corr = -s.q * (phi(i, j, k) - phi_ref) - Chi * s.q;
                    double Ev_corr = Ec_corr - s.q * Eg;
                    double g_A = 4.0, g_D = 2.0;
                    double Ea = s.Ea, Ed = s.Ed;
                    double q = s.q, kb = s.kb, T = s.T;
                    double acc, don;
                    if (P.use_Fermi_Dirac == 1) {
                        double eta_n = -(Ec_corr - q * Ef) / (kb * T);
                        double eta_p = -(q * Ef - Ev_corr) / (kb * T);
                        e_den(i, j, k) = s.Nc * FD_half(eta_n);
                        p_den(i, j, k) = s.Nv * FD_half(eta_p);
                        acc = P.acceptor_doping / (1.0 + g_A * exp((-q * Ef + q * Ea + q * phi_ref - q * Chi - q * Eg - q * phi(i, j, k)) / (kb * T)));
                        don = P.donor_doping / (1.0 + g_D * exp((q * Ef + q * Ed - q * phi_ref + q * Chi + q * phi(i, j, k)) / (kb * T)));
                    } else {
                        e_den(i, j, k) = s.Nc * exp(-(Ec_corr - q * Ef) / (kb * T));
                        p_den(i, j, k) = s.Nv * exp(-(q * Ef - Ev_corr) / (kb * T));
                        acc = P.acceptor_doping / (1.0 + g_A * exp((-q * Ef + q * Ea + q * phi_ref - q * Chi - q * Eg - q * phi(i, j, k)) / (kb * T)));
                        don = P.donor_doping / (1.0 + g_D * exp((q * Ef + q * Ed - q * phi_ref + q * Chi + q * phi(i, j, k)) / (kb * T)));
                    }
                    rho(i, j, k) = q * (p_den(i, j, k) - e_den(i, j, k) - acc + don);
                } else {
                    rho(i, j, k) = 0.0;
                }
            }
}

// ------------------------------------- ElectrostaticSolver.cpp:8-83 ------
void compute_poisson_rhs(ofx_ctx* c, Fab& RHS, const Fab* Pf, const Fab& rho) {
    Stencil st = make_stencil(c);
    const Fab& mask = c->mask;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i) {
                double R[9];
                rotation(c->p.use_Euler_angles, c->ang[0](i, j, k), c->ang[1](i, j, k), c->ang[2](i, j, k), R);
                if (mask(i, j, k) >= 2.0) {
                    RHS(i, j, k) = rho(i, j, k);
                } else if (mask(i, j, k) == 1.0) {
                    RHS(i, j, k) = 0.;
                } else {
                    RHS(i, j, k) =
                        -(R[0] * st.DPD(0, Pf[0], mask, i, j, k) + R[1] * st.DPD(1, Pf[0], mask, i, j, k) + R[2] * st.DPD(2, Pf[0], mask, i, j, k))
                        - (R[3] * st.DPD(0, Pf[1], mask, i, j, k) + R[4] * st.DPD(1, Pf[1], mask, i, j, k) + R[5] * st.DPD(2, Pf[1], mask, i, j, k))
                        - (R[6] * st.DPD(0, Pf[2], mask, i, j, k) + R[7] * st.DPD(1, Pf[2], mask, i, j, k) + R[8] * st.DPD(2, Pf[2], mask, i, j, k));
                }
            }
}

// ------------------------------------------------ Poisson multigrid -----
// operator:  (A alpha - B div beta grad) phi with A = -1, B = 1
// (ElectrostaticSolver.cpp:603-605), z Dirichlet by the maxorder-2 ghost
// 2 V - phi_0, x/y periodic.
inline size_t L3(const MGLevel& l, int i, int j, int k) { return (size_t)i + (size_t)l.n[0] * ((size_t)j + (size_t)l.n[1] * k); }
inline size_t FX(const MGLevel& l, int i, int j, int k) { return (size_t)i + (size_t)(l.n[0] + 1) * ((size_t)j + (size_t)l.n[1] * k); }
inline size_t FY(const MGLevel& l, int i, int j, int k) { return (size_t)i + (size_t)l.n[0] * ((size_t)j + (size_t)(l.n[1] + 1) * k); }
inline size_t FZ(const MGLevel& l, int i, int j, int k) { return (size_t)i + (size_t)l.n[0] * ((size_t)j + (size_t)l.n[1] * k); }

// A x at one cell; vlo / vhi are the z Dirichlet values (0 for homogeneous)
inline double apply_cell(const MGLevel& l, const double* x, int i, int j, int k, double vlo, double vhi) {
    const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
    const double ihx = 1.0 / (l.h[0] * l.h[0]), ihy = 1.0 / (l.h[1] * l.h[1]), ihz = 1.0 / (l.h[2] * l.h[2]);
    const double xc = x[L3(l, i, j, k)];
    const int im = (i - 1 + nx) % nx, ip = (i + 1) % nx, jm = (j - 1 + ny) % ny, jp = (j + 1) % ny;
    double xzm = (k > 0) ? x[L3(l, i, j, k - 1)] : 2.0 * vlo - xc;
    double xzp = (k < nz - 1) ? x[L3(l, i, j, k + 1)] : 2.0 * vhi - xc;
    double s = -l.a[L3(l, i, j, k)] * xc;
    s += (l.bx[FX(l, i, j, k)] * (xc - x[L3(l, im, j, k)]) + l.bx[FX(l, i + 1, j, k)] * (xc - x[L3(l, ip, j, k)])) * ihx;
    s += (l.by[FY(l, i, j, k)] * (xc - x[L3(l, i, jm, k)]) + l.by[FY(l, i, j + 1, k)] * (xc - x[L3(l, i, jp, k)])) * ihy;
    s += (l.bz[FZ(l, i, j, k)] * (xc - xzm) + l.bz[FZ(l, i, j, k + 1)] * (xc - xzp)) * ihz;
    return s;
}

void mg_residual(const MGLevel& l, const double* x, const double* b, double* r, double vlo, double vhi) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < l.n[2]; ++k)
        for (int j = 0; j < l.n[1]; ++j)
            for (int i = 0; i < l.n[0]; ++i)
                r[L3(l, i, j, k)] = b[L3(l, i, j, k)] - apply_cell(l, x, i, j, k, vlo, vhi);
}

double norm_inf(const double* v, size_t n) {
    double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
    for (long q = 0; q < (long)n; ++q) m = std::max(m, std::fabs(v[q]));
    return m;
}

void gsrb(MGLevel& l, int sweeps) {
    const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
    const double ihx = 1.0 / (l.h[0] * l.h[0]), ihy = 1.0 / (l.h[1] * l.h[1]), ihz = 1.0 / (l.h[2] * l.h[2]);
    double* x = l.x.data();
    const double* b = l.r.data();
    for (int s = 0; s < sweeps; ++s)
        for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = (j + k + color) & 1; i < nx; i += 2) {
                        const int im = (i - 1 + nx) % nx, ip = (i + 1) % nx, jm = (j - 1 + ny) % ny, jp = (j + 1) % ny;
                        double bxm = l.bx[FX(l, i, j, k)], bxp = l.bx[FX(l, i + 1, j, k)];
                        double bym = l.by[FY(l, i, j, k)], byp = l.by[FY(l, i, j + 1, k)];
                        double bzm = l.bz[FZ(l, i, j, k)], bzp = l.bz[FZ(l, i, j, k + 1)];
                        double diag = -l.a[L3(l, i, j, k)] + (bxm + bxp) * ihx + (bym + byp) * ihy;
                        double off = (bxm * x[L3(l, im, j, k)] + bxp * x[L3(l, ip, j, k)]) * ihx +
                                     (bym * x[L3(l, i, jm, k)] + byp * x[L3(l, i, jp, k)]) * ihy;
                        if (k > 0) { diag += bzm * ihz; off += bzm * x[L3(l, i, j, k - 1)] * ihz; }
                        else diag += 2.0 * bzm * ihz;
                        if (k < nz - 1) { diag += bzp * ihz; off += bzp * x[L3(l, i, j, k + 1)] * ihz; }
                        else diag += 2.0 * bzp * ihz;
                        x[L3(l, i, j, k)] = (b[L3(l, i, j, k)] + off) / diag;
                    }
        }
}

// Coarsening: a direction is halved when its cell count is even, stays >= 2,
// and its spacing is within 1.5x of the finest spacing (semicoarsening keeps
// point smoothing effective when dz << dx or dx << dz).
void mg_build_coarse(std::vector<MGLevel>& mg) {
    while (true) {
        MGLevel& f = mg.back();
        double hmin = std::min(f.h[0], std::min(f.h[1], f.h[2]));
        int cr[3];
        bool any = false;
        for (int d = 0; d < 3; ++d) {
            cr[d] = (f.n[d] % 2 == 0) && (f.n[d] / 2 >= 2) && (f.h[d] <= 1.5 * hmin) ? 2 : 1;
            any = any || cr[d] == 2;
        }
        if (!any) break;
        MGLevel c;
        for (int d = 0; d < 3; ++d) { c.n[d] = f.n[d] / cr[d]; c.h[d] = f.h[d] * cr[d]; c.cr[d] = cr[d]; }
        size_t N = c.N();
        c.a.assign(N, 0.0);
        c.bx.assign((size_t)(c.n[0] + 1) * c.n[1] * c.n[2], 0.0);
        c.by.assign((size_t)c.n[0] * (c.n[1] + 1) * c.n[2], 0.0);
        c.bz.assign((size_t)c.n[0] * c.n[1] * (c.n[2] + 1), 0.0);
        c.x.assign(N, 0.0); c.r.assign(N, 0.0); c.t.assign(N, 0.0);
        mg.push_back(std::move(c));
    }
}

// coefficients of a coarse level: cell alpha averaged over the children,
// face beta averaged over the fine faces that make up the coarse face
void mg_average_coeffs(std::vector<MGLevel>& mg) {
    for (size_t l = 1; l < mg.size(); ++l) {
        const MGLevel& f = mg[l - 1];
        MGLevel& c = mg[l];
        const int rx = c.cr[0], ry = c.cr[1], rz = c.cr[2];
        for (int k = 0; k < c.n[2]; ++k)
            for (int j = 0; j < c.n[1]; ++j)
                for (int i = 0; i < c.n[0]; ++i) {
                    double s = 0.0;
                    for (int dk = 0; dk < rz; ++dk)
                        for (int dj = 0; dj < ry; ++dj)
                            for (int di = 0; di < rx; ++di) s += f.a[L3(f, rx * i + di, ry * j + dj, rz * k + dk)];
                    c.a[L3(c, i, j, k)] = s / (rx * ry * rz);
                }
        // along a coarsened direction the fine links between two coarse
        // centres act in series (half, full, half link), across the
        // transverse children in parallel; at a Dirichlet face the path runs
        // from the coarse centre to the electrode
        auto ser = [](double a, double b, double c2) { return 4.0 / (1.0 / a + 2.0 / b + 1.0 / c2); };
        const int fnx = f.n[0], fny = f.n[1], fnz = f.n[2];
        auto BX = [&](int i, int j, int k) { return f.bx[FX(f, ((i % fnx) + fnx) % fnx, j, k)]; };
        auto BY = [&](int i, int j, int k) { return f.by[FY(f, i, ((j % fny) + fny) % fny, k)]; };
        auto BZ = [&](int i, int j, int k) { return f.bz[FZ(f, i, j, k)]; };
        for (int k = 0; k < c.n[2]; ++k)
            for (int j = 0; j < c.n[1]; ++j)
                for (int i = 0; i <= c.n[0]; ++i) {
                    double s = 0.0;
                    for (int dk = 0; dk < rz; ++dk)
                        for (int dj = 0; dj < ry; ++dj) {
                            const int fj = ry * j + dj, fk = rz * k + dk;
                            s += rx == 2 ? ser(BX(2 * i - 1, fj, fk), BX(2 * i, fj, fk), BX(2 * i + 1, fj, fk)) : BX(i, fj, fk);
                        }
                    c.bx[FX(c, i, j, k)] = s / (ry * rz);
                }
        for (int k = 0; k < c.n[2]; ++k)
            for (int j = 0; j <= c.n[1]; ++j)
                for (int i = 0; i < c.n[0]; ++i) {
                    double s = 0.0;
                    for (int dk = 0; dk < rz; ++dk)
                        for (int di = 0; di < rx; ++di) {
                            const int fi = rx * i + di, fk = rz * k + dk;
                            s += ry == 2 ? ser(BY(fi, 2 * j - 1, fk), BY(fi, 2 * j, fk), BY(fi, 2 * j + 1, fk)) : BY(fi, j, fk);
                        }
                    c.by[FY(c, i, j, k)] = s / (rx * rz);
                }
        for (int k = 0; k <= c.n[2]; ++k)
            for (int j = 0; j < c.n[1]; ++j)
                for (int i = 0; i < c.n[0]; ++i) {
                    double s = 0.0;
                    for (int dj = 0; dj < ry; ++dj)
                        for (int di = 0; di < rx; ++di) {
                            const int fi = rx * i + di, fj = ry * j + dj;
                            double v;
                            if (rz == 1) v = BZ(fi, fj, k);
                            else if (k == 0) v = 2.0 / (1.0 / BZ(fi, fj, 0) + 1.0 / BZ(fi, fj, 1));
                            else if (k == c.n[2]) v = 2.0 / (1.0 / BZ(fi, fj, fnz) + 1.0 / BZ(fi, fj, fnz - 1));
                            else v = ser(BZ(fi, fj, 2 * k - 1), BZ(fi, fj, 2 * k), BZ(fi, fj, 2 * k + 1));
                            s += v;
                        }
                    c.bz[FZ(c, i, j, k)] = s / (rx * ry);
                }
    }
}

// Prolongation weights from the fine face coefficients: along a coarsened
// direction a fine cell lies between its parent's centre (near, h/2 away) and
// the neighbouring coarse centre (far, 3h/2 away); the weights are those of a
// 1-D resistor chain, G_near / G_far, so a thin low-eps layer between the two
// centres shifts the interpolated correction as the flux continuity demands.
// Uniform coefficients give the linear weights 3/4, 1/4 (1/2 at an electrode).
void mg_interp_weights(std::vector<MGLevel>& mg) {
    for (size_t l = 1; l < mg.size(); ++l) {
        const MGLevel& f = mg[l - 1];
        MGLevel& c = mg[l];
        const int nx = f.n[0], ny = f.n[1], nz = f.n[2];
        for (int d = 0; d < 3; ++d) {
            c.wfar[d].assign(f.N(), 0.25);
            if (c.cr[d] != 2) continue;
            const double h = f.h[d];
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        const int q = d == 0 ? i : d == 1 ? j : k;
                        const int n = f.n[d];
                        // face beta at fine face index t (between cells t-1 and t)
                        auto B = [&](int t) {
                            if (d == 0) return f.bx[FX(f, ((t % n) + n) % n, j, k)];
                            if (d == 1) return f.by[FY(f, i, ((t % n) + n) % n, k)];
                            return f.bz[FZ(f, i, j, t)];
                        };
                        double gn, gf;
                        if ((q & 1) == 0) {
                            gn = 2.0 * B(q + 1) / h;
                            if (d == 2 && q == 0) gf = 2.0 * B(0) / h;
                            else gf = 1.0 / (h / B(q) + h / (2.0 * B(q - 1)));
                        } else {
                            gn = 2.0 * B(q) / h;
                            if (d == 2 && q == n - 1) gf = 2.0 * B(n) / h;
                            else gf = 1.0 / (h / B(q + 1) + h / (2.0 * B(q + 2)));
                        }
                        c.wfar[d][L3(f, i, j, k)] = gf / (gn + gf);
                    }
        }
    }
}

// CG bottom solve (SPD operator), relative 2-norm reduction 1e-4, <= 200 its
void mg_bottom(MGLevel& l) {
    size_t N = l.N();
    std::vector<double> r(N), pv(N), Ap(N);
    std::fill(l.x.begin(), l.x.end(), 0.0);
    r = l.r;
    pv = r;
    double rr = 0; for (size_t q = 0; q < N; ++q) rr += r[q] * r[q];
    double rr0 = rr;
    if (rr0 == 0.0) return;
    for (int it = 0; it < 200 && rr > 1e-8 * rr0; ++it) {
        for (int k = 0; k < l.n[2]; ++k)
            for (int j = 0; j < l.n[1]; ++j)
                for (int i = 0; i < l.n[0]; ++i) Ap[L3(l, i, j, k)] = apply_cell(l, pv.data(), i, j, k, 0.0, 0.0);
        double pAp = 0; for (size_t q = 0; q < N; ++q) pAp += pv[q] * Ap[q];
        if (pAp <= 0) break;
        double a = rr / pAp;
        for (size_t q = 0; q < N; ++q) { l.x[q] += a * pv[q]; r[q] -= a * Ap[q]; }
        double rr2 = 0; for (size_t q = 0; q < N; ++q) rr2 += r[q] * r[q];
        double b = rr2 / rr; rr = rr2;
        for (size_t q = 0; q < N; ++q) pv[q] = r[q] + b * pv[q];
    }
}

void mg_vcycle(std::vector<MGLevel>& mg, size_t lev) {
    MGLevel& l = mg[lev];
    if (lev + 1 == mg.size()) { mg_bottom(l); return; }
    std::fill(l.x.begin(), l.x.end(), 0.0);
    gsrb(l, 2);
    mg_residual(l, l.x.data(), l.r.data(), l.t.data(), 0.0, 0.0);
    MGLevel& c = mg[lev + 1];
    const int rx = c.cr[0], ry = c.cr[1], rz = c.cr[2];
    const double inv = 1.0 / (rx * ry * rz);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c.n[2]; ++k)
        for (int j = 0; j < c.n[1]; ++j)
            for (int i = 0; i < c.n[0]; ++i) {
                double s = 0.0;
                for (int dk = 0; dk < rz; ++dk)
                    for (int dj = 0; dj < ry; ++dj)
                        for (int di = 0; di < rx; ++di) s += l.t[L3(l, rx * i + di, ry * j + dj, rz * k + dk)];
                c.r[L3(c, i, j, k)] = s * inv;
            }
    mg_vcycle(mg, lev + 1);
    // prolongation in the coarsened directions with the resistor-chain
    // weights (near parent / far neighbour); the far neighbour beyond an
    // electrode is the homogeneous Dirichlet value 0
#pragma omp parallel for schedule(static)
    for (int k = 0; k < l.n[2]; ++k)
        for (int j = 0; j < l.n[1]; ++j)
            for (int i = 0; i < l.n[0]; ++i) {
                const size_t fc = L3(l, i, j, k);
                int I[2], J[2], K[2];
                double wi[2], wj[2], wk[2];
                int ni = 1, nj = 1, nk = 1;
                I[0] = i / rx; wi[0] = 1.0;
                if (rx == 2) { ni = 2; wi[1] = c.wfar[0][fc]; wi[0] = 1.0 - wi[1]; I[1] = (i & 1) ? I[0] + 1 : I[0] - 1; I[1] = (I[1] + c.n[0]) % c.n[0]; }
                J[0] = j / ry; wj[0] = 1.0;
                if (ry == 2) { nj = 2; wj[1] = c.wfar[1][fc]; wj[0] = 1.0 - wj[1]; J[1] = (j & 1) ? J[0] + 1 : J[0] - 1; J[1] = (J[1] + c.n[1]) % c.n[1]; }
                K[0] = k / rz; wk[0] = 1.0;
                if (rz == 2) {
                    nk = 2; wk[1] = c.wfar[2][fc]; wk[0] = 1.0 - wk[1]; K[1] = (k & 1) ? K[0] + 1 : K[0] - 1;
                    if (K[1] < 0 || K[1] >= c.n[2]) { K[1] = K[0]; wk[1] = 0.0; }
                }
                double s = 0.0;
                for (int a = 0; a < nk; ++a)
                    for (int b = 0; b < nj; ++b)
                        for (int d = 0; d < ni; ++d) s += wk[a] * wj[b] * wi[d] * c.x[L3(c, I[d], J[b], K[a])];
                l.x[fc] += s;
            }
    gsrb(l, 2);
}

void mg_setup(ofx_ctx* c, const double* alpha_cc_valid) {
    if (c->mg.empty()) {
        MGLevel l0;
        for (int d = 0; d < 3; ++d) { l0.n[d] = c->n[d]; l0.h[d] = c->dx[d]; }
        if (c->eb_nz > 0) l0.n[2] = c->eb_nz;
        size_t N = l0.N();
        l0.a.assign(N, 0.0);
        l0.bx = c->bxf; l0.by = c->byf; l0.bz = c->bzf;
        if (c->eb_nz > 0) {
            // the fluid layers' faces; the embedded surface (their top face)
            // takes the cut cell's beta_cc, as setEBDirichlet is given beta_cc
            // (ElectrostaticSolver.cpp:668-672)
            const size_t nxy = (size_t)c->n[0] * c->n[1];
            l0.bx.resize((size_t)(c->n[0] + 1) * c->n[1] * c->eb_nz);
            l0.by.resize((size_t)c->n[0] * (c->n[1] + 1) * c->eb_nz);
            l0.bz.resize(nxy * (c->eb_nz + 1));
            for (int j = 0; j < c->n[1]; ++j)
                for (int i = 0; i < c->n[0]; ++i)
                    l0.bz[(size_t)i + (size_t)c->n[0] * j + nxy * c->eb_nz] = c->beta_cc(i, j, c->eb_nz - 1);
        }
        l0.x.assign(N, 0.0); l0.r.assign(N, 0.0); l0.t.assign(N, 0.0);
        c->mg.push_back(std::move(l0));
        mg_build_coarse(c->mg);
    }
    MGLevel& l0 = c->mg[0];
    for (size_t q = 0; q < l0.N(); ++q) l0.a[q] = alpha_cc_valid ? alpha_cc_valid[q] : 0.0;
    mg_average_coeffs(c->mg);
    mg_interp_weights(c->mg);
}

// returns 0 on convergence, -3 when the iteration cap is hit
int mg_solve(ofx_ctx* c, const double* b, double* sol, double rtol, int* iters, double* resid) {
    MGLevel& l0 = c->mg[0];
    size_t N = l0.N();
    std::vector<double> res(N);
    const double vhi = c->eb_nz > 0 ? c->eb_V : c->V_hi;   // the solve's top Dirichlet value
    mg_residual(l0, sol, b, res.data(), c->V_lo, vhi);
    double resnorm0 = norm_inf(res.data(), N);
    double rhsnorm0 = norm_inf(b, N);
    double target = std::max(rtol, 1e-16) * std::max(resnorm0, rhsnorm0);
    int it = 0;
    double rn = resnorm0;
    int maxit = c->p.mg_max_iter > 0 ? c->p.mg_max_iter : 200;
    while (rn > target && it < maxit) {
        l0.r = res;
        mg_vcycle(c->mg, 0);
        for (size_t q = 0; q < N; ++q) sol[q] += l0.x[q];
        mg_residual(l0, sol, b, res.data(), c->V_lo, vhi);
        rn = norm_inf(res.data(), N);
        ++it;
        if (c->p.verbose > 1) printf("  mg iter %d  |r|/|r0| = %g\n", it, rn / std::max(resnorm0, rhsnorm0));
    }
    if (iters) *iters = it;
    if (resid) *resid = (std::max(resnorm0, rhsnorm0) > 0) ? rn / std::max(resnorm0, rhsnorm0) : 0.0;
    return rn > target ? -3 : 0;
}

void fab_to_valid(const Fab& f, std::vector<double>& out) {
    out.resize((size_t)f.nx * f.ny * f.nz);
    for (int k = 0; k < f.nz; ++k)
        for (int j = 0; j < f.ny; ++j)
            for (int i = 0; i < f.nx; ++i) out[(size_t)i + (size_t)f.nx * ((size_t)j + (size_t)f.ny * k)] = f(i, j, k);
}
void valid_to_fab(const double* in, Fab& f) {
    for (int k = 0; k < f.nz; ++k)
        for (int j = 0; j < f.ny; ++j)
            for (int i = 0; i < f.nx; ++i) f(i, j, k) = in[(size_t)i + (size_t)f.nx * ((size_t)j + (size_t)f.ny * k)];
}

// ------------------------------------- ElectrostaticSolver.cpp:502-524 ---
void set_phi_bc_z(ofx_ctx* c) {
    const SiConst& s = c->si;
    double Eg = s.bandgap, Chi = s.affinity;
    double phi_ref = Chi + 0.5 * Eg + 0.5 * s.kb * s.T * log(s.Nc / s.Nv) / s.q;
    double phi_m = c->p.use_work_function ? c->p.metal_work_function : phi_ref;
    double vlo = c->p.Phi_Bc_lo;
    double vhi = c->Phi_Bc_hi - (phi_m - phi_ref);
    for (int k = -1; k <= c->n[2]; ++k)
        for (int j = -1; j <= c->n[1]; ++j)
            for (int i = -1; i <= c->n[0]; ++i) {
                if (k < 0) c->phi(i, j, k) = vlo;
                else if (k >= c->n[2]) c->phi(i, j, k) = vhi;
            }
    fill_boundary(c->phi, c->p.is_periodic);
    // setLevelBC (ElectrostaticSolver.cpp:601 / main.cpp:591) stores them
    c->V_lo = vlo;
    c->V_hi = vhi;
}

// ghost cells of phi after the MLMG solve (see the phi_ghost_mode key)
void phi_ghosts_after_solve(ofx_ctx* c) {
    Fab& phi = c->phi;
    for (int j = 0; j < c->n[1]; ++j)
        for (int i = 0; i < c->n[0]; ++i) {
            double glo, ghi;
            if (c->p.phi_ghost_mode == 0) {
                glo = 2.0 * c->V_lo + (-1.0) * phi(i, j, 0);
                ghi = 2.0 * c->V_hi + (-1.0) * phi(i, j, c->n[2] - 1);
            } else if (c->p.phi_ghost_mode == 1) {
                glo = c->V_lo; ghi = c->V_hi;
            } else {
                glo = 0.0; ghi = 0.0;
            }
            phi(i, j, -1) = glo;
            phi(i, j, c->n[2]) = ghi;
        }
    fill_boundary(phi, c->p.is_periodic);
}

// --------------------------------- ElectrostaticSolver.cpp:678-747 ------
int compute_phi_rho(ofx_ctx* c, const Fab* Pf) {
    const size_t N = c->N;
    double tol = 1.e-5;
    double err = 1.0;
    int iter = 0;
    int mg_total = 0;
    std::vector<double> rhs_v(N), alpha_v(N), phi_v(N);
    Fab phi_pd, rhs_pd;
    phi_pd.define(c->n[0], c->n[1], c->n[2], 0);
    rhs_pd.define(c->n[0], c->n[1], c->n[2], 0);
    int cap = c->p.newton_max_iter > 0 ? c->p.newton_max_iter : 50;
    int passes = 0;
    while (err > tol) {
        if (passes++ >= cap) return -3;
        compute_poisson_rhs(c, c->rhs, Pf, c->rho);
        // dF_dPhi, ElectrostaticSolver.cpp:85-113
        for (int k = 0; k < c->n[2]; ++k)
            for (int j = 0; j < c->n[1]; ++j)
                for (int i = 0; i < c->n[0]; ++i) phi_pd(i, j, k) = c->phi(i, j, k) + c->p.delta;
        compute_rho(c, phi_pd, c->rho, c->e_den, c->h_den);
        compute_poisson_rhs(c, rhs_pd, Pf, c->rho);
        for (int k = 0; k < c->n[2]; ++k)
            for (int j = 0; j < c->n[1]; ++j)
                for (int i = 0; i < c->n[0]; ++i)
                    c->alpha_cc(i, j, k) = (1. / c->p.delta) * rhs_pd(i, j, k) + (-1. / c->p.delta) * c->rhs(i, j, k);
        // ComputePoissonRHS_Newton, :114-132
        for (int k = 0; k < c->n[2]; ++k)
            for (int j = 0; j < c->n[1]; ++j)
                for (int i = 0; i < c->n[0]; ++i)
                    c->rhs(i, j, k) = c->rhs(i, j, k) - c->alpha_cc(i, j, k) * c->phi(i, j, k);
        fab_to_valid(c->rhs, rhs_v);
        fab_to_valid(c->alpha_cc, alpha_v);
        mg_setup(c, alpha_v.data());
        c->phi.setVal(0.);  // :716
        std::fill(phi_v.begin(), phi_v.end(), 0.0);
        int its = 0;
        double resid = 0;
        int st = mg_solve(c, rhs_v.data(), phi_v.data(), c->p.mg_rtol, &its, &resid);
        mg_total += its;
        if (st != 0) return st;
        valid_to_fab(phi_v.data(), c->phi);
        phi_ghosts_after_solve(c);
        compute_rho(c, c->phi, c->rho, c->e_den, c->h_den);
        if (!c->contains_sc) {
            err = 0.;
        } else {
            if (iter > 0) {
                double s1 = 0.0, s2 = 0.0;
                for (int k = 0; k < c->n[2]; ++k)
                    for (int j = 0; j < c->n[1]; ++j)
                        for (int i = 0; i < c->n[0]; ++i) {
                            s1 += std::fabs(c->phi(i, j, k) - c->phi_prev(i, j, k));
                            s2 += std::fabs(c->phi(i, j, k));
                        }
                err = s1 / s2;
            }
            for (int k = 0; k < c->n[2]; ++k)
                for (int j = 0; j < c->n[1]; ++j)
                    for (int i = 0; i < c->n[0]; ++i) c->phi_prev(i, j, k) = c->phi(i, j, k);
            iter = iter + 1;
            if (c->p.verbose) printf("%d iterations :: err = %g\n", iter, err);
        }
    }
    c->last_newton_iters = passes;
    c->last_mg_iters = mg_total;
    c->last_phi_err = err;
    return 0;
}

// ------------------------------------ ElectrostaticSolver.cpp:134-203 ----
void compute_E(ofx_ctx* c) {
    Stencil st = make_stencil(c);
    const double* prob_lo = c->p.prob_lo;
    const double* prob_hi = c->p.prob_hi;
    const double* dx = c->dx;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i) {
                double z_hi = prob_lo[2] + (k + 1.5) * dx[2];
                double z_lo = prob_lo[2] + (k - 0.5) * dx[2];
                double R[9];
                rotation(c->p.use_Euler_angles, c->ang[0](i, j, k), c->ang[1](i, j, k), c->ang[2](i, j, k), R);
                const Fab& phi = c->phi;
                c->E[0](i, j, k) = -(R[0] * st.DFDx(phi, i, j, k) + R[1] * st.DFDy(phi, i, j, k) + R[2] * st.DphiDz(phi, z_hi, z_lo, i, j, k, prob_lo, prob_hi));
                c->E[1](i, j, k) = -(R[3] * st.DFDx(phi, i, j, k) + R[4] * st.DFDy(phi, i, j, k) + R[5] * st.DphiDz(phi, z_hi, z_lo, i, j, k, prob_lo, prob_hi));
                c->E[2](i, j, k) = -(R[6] * st.DFDx(phi, i, j, k) + R[7] * st.DFDy(phi, i, j, k) + R[8] * st.DphiDz(phi, z_hi, z_lo, i, j, k, prob_lo, prob_hi));
            }
}

// ------------------------------------- TotalEnergyDensity.cpp:67-130 ----
void calculate_landau(ofx_ctx* c, Fab* GL, const Fab* Pf) {
    const ofx_params& p = c->p;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i) {
                double pp = Pf[0](i, j, k), pq = Pf[1](i, j, k), pr = Pf[2](i, j, k);
                double dFdPp_Landau = p.alpha * pp + p.beta * pw(pp, 3.) + p.gamma * pw(pp, 5.)
                    + 2. * p.alpha_12 * pp * pw(pq, 2.)
                    + 2. * p.alpha_12 * pp * pw(pr, 2.)
                    + 4. * p.alpha_112 * pw(pp, 3.) * (pw(pq, 2.) + pw(pr, 2.))
                    + 2. * p.alpha_112 * pp * pw(pq, 4.)
                    + 2. * p.alpha_112 * pp * pw(pr, 4.)
                    + 2. * p.alpha_123 * pp * pw(pq, 2.) * pw(pr, 2.);
                double dFdPq_Landau = p.alpha * pq + p.beta * pw(pq, 3.) + p.gamma * pw(pq, 5.)
                    + 2. * p.alpha_12 * pq * pw(pp, 2.)
                    + 2. * p.alpha_12 * pq * pw(pr, 2.)
                    + 4. * p.alpha_112 * pw(pq, 3.) * (pw(pp, 2.) + pw(pr, 2.))
                    + 2. * p.alpha_112 * pq * pw(pp, 4.)
                    + 2. * p.alpha_112 * pq * pw(pr, 4.)
                    + 2. * p.alpha_123 * pq * pw(pp, 2.) * pw(pr, 2.);
                double dFdPr_Landau = p.alpha * pr + p.beta * pw(pr, 3.) + p.gamma * pw(pr, 5.)
                    + 2. * p.alpha_12 * pr * pw(pp, 2.)
                    + 2. * p.alpha_12 * pr * pw(pq, 2.)
                    + 4. * p.alpha_112 * pw(pr, 3.) * (pw(pp, 2.) + pw(pq, 2.))
                    + 2. * p.alpha_112 * pr * pw(pp, 4.)
                    + 2. * p.alpha_112 * pr * pw(pq, 4.)
                    + 2. * p.alpha_123 * pr * pw(pp, 2.) * pw(pq, 2.);
                double G = c->Gamma(i, j, k);
                GL[0](i, j, k) = -1.0 * G * dFdPp_Landau;
                GL[1](i, j, k) = -1.0 * G * dFdPq_Landau;
                GL[2](i, j, k) = -1.0 * G * dFdPr_Landau;
                if (p.is_polarization_scalar == 1) { GL[0](i, j, k) = 0.0; GL[1](i, j, k) = 0.0; }
                if (c->tphase(i, j, k) == 1.0) { GL[0](i, j, k) = 0.0; GL[1](i, j, k) = 0.0; GL[2](i, j, k) = 0.0; }
            }
}

// ------------------------------------ TotalEnergyDensity.cpp:133-251 ----
void calculate_grad(ofx_ctx* c, Fab* GL, const Fab* Pf) {
    const ofx_params& p = c->p;
    Stencil st = make_stencil(c);
    const Fab& mask = c->mask;
    const Fab &pp = Pf[0], &pq = Pf[1], &pr = Pf[2];
    const double g11 = p.g11, g44 = p.g44, g44_p = p.g44_p, g12 = p.g12;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i) {
                double R[9];
                rotation(p.use_Euler_angles, c->ang[0](i, j, k), c->ang[1](i, j, k), c->ang[2](i, j, k), R);
                const double R_11 = R[0], R_12 = R[1], R_13 = R[2], R_21 = R[3], R_22 = R[4], R_23 = R[5], R_31 = R[6], R_32 = R[7], R_33 = R[8];
                double dFdPp_grad = -g11 * st.DDPD(0, pp, mask, i, j, k)
                    - (g44 + g44_p) * st.DDPD(1, pp, mask, i, j, k)
                    - (g44 + g44_p) * st.DDPD(2, pp, mask, i, j, k)
                    - (g12 + g44 - g44_p) * st.DxDy(pq, mask, i, j, k)
                    - (g12 + g44 - g44_p) * st.DxDz(pr, mask, i, j, k);
                double dFdPq_grad = -g11 * st.DDPD(1, pq, mask, i, j, k)
                    - (g44 - g44_p) * st.DDPD(0, pq, mask, i, j, k)
                    - (g44 - g44_p) * st.DDPD(2, pq, mask, i, j, k)
                    - (g12 + g44 + g44_p) * st.DxDy(pp, mask, i, j, k)
                    - (g12 + g44 - g44_p) * st.DyDz(pr, mask, i, j, k);
                double dFdPr_grad = -g11 * (R_31 * R_31 * st.DDPD(0, pr, mask, i, j, k)
                                            + R_32 * R_32 * st.DDPD(1, pr, mask, i, j, k)
                                            + R_33 * R_33 * st.DDPD(2, pr, mask, i, j, k)
                                            + 2. * R_31 * R_32 * st.DxDy(pr, mask, i, j, k)
                                            + 2. * R_32 * R_33 * st.DyDz(pr, mask, i, j, k)
                                            + 2. * R_33 * R_31 * st.DxDz(pr, mask, i, j, k))
                    - (g44 - g44_p) * (R_11 * R_11 * st.DDPD(0, pr, mask, i, j, k)
                                       + R_12 * R_12 * st.DDPD(1, pr, mask, i, j, k)
                                       + R_13 * R_13 * st.DDPD(2, pr, mask, i, j, k)
                                       + 2. * R_11 * R_12 * st.DxDy(pr, mask, i, j, k)
                                       + 2. * R_12 * R_13 * st.DyDz(pr, mask, i, j, k)
                                       + 2. * R_13 * R_11 * st.DxDz(pr, mask, i, j, k))
                    - (g44 - g44_p) * (R_21 * R_21 * st.DDPD(0, pr, mask, i, j, k)
                                       + R_22 * R_22 * st.DDPD(1, pr, mask, i, j, k)
                                       + R_23 * R_23 * st.DDPD(2, pr, mask, i, j, k)
                                       + 2. * R_21 * R_22 * st.DxDy(pr, mask, i, j, k)
                                       + 2. * R_22 * R_23 * st.DyDz(pr, mask, i, j, k)
                                       + 2. * R_23 * R_21 * st.DxDz(pr, mask, i, j, k))
                    - (g44 + g44_p + g12) * st.DyDz(pq, mask, i, j, k)
                    - (g44 + g44_p + g12) * st.DxDz(pp, mask, i, j, k);
                double G = c->Gamma(i, j, k);
                GL[0](i, j, k) = -1.0 * G * dFdPp_grad;
                GL[1](i, j, k) = -1.0 * G * dFdPq_grad;
                GL[2](i, j, k) = -1.0 * G * dFdPr_grad;
                if (p.is_polarization_scalar == 1) { GL[0](i, j, k) = 0.0; GL[1](i, j, k) = 0.0; }
                if (c->tphase(i, j, k) == 1.0) { GL[0](i, j, k) = 0.0; GL[1](i, j, k) = 0.0; GL[2](i, j, k) = 0.0; }
            }
}

// ------------------------------------ TotalEnergyDensity.cpp:254-294 ----
void calculate_elec(ofx_ctx* c, Fab* GL) {
    const ofx_params& p = c->p;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i) {
                double G = c->Gamma(i, j, k);
                GL[0](i, j, k) = -1.0 * G * (-c->E[0](i, j, k));
                GL[1](i, j, k) = -1.0 * G * (-c->E[1](i, j, k));
                GL[2](i, j, k) = -1.0 * G * (-c->E[2](i, j, k));
                if (p.is_polarization_scalar == 1) { GL[0](i, j, k) = 0.0; GL[1](i, j, k) = 0.0; }
                if (c->tphase(i, j, k) == 1.0) { GL[0](i, j, k) = 0.0; GL[1](i, j, k) = 0.0; GL[2](i, j, k) = 0.0; }
            }
}

// CalculateTDGL_RHS, TotalEnergyDensity.cpp:6-64 (GL starts at zero in all
// cells incl. ghosts, then the enabled terms are added in this order)
void tdgl_rhs(ofx_ctx* c, Fab* GL, const Fab* Pf) {
    const ofx_params& p = c->p;
    if (p.include_Landau == 1) calculate_landau(c, c->GLL, Pf);
    if (p.include_Grad == 1) calculate_grad(c, c->GLG, Pf);
    if (p.include_Elec == 1) calculate_elec(c, c->GLE);
    for (int d = 0; d < 3; ++d) GL[d].setVal(0.);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i)
                for (int d = 0; d < 3; ++d) {
                    if (p.include_Landau == 1) GL[d](i, j, k) += c->GLL[d](i, j, k);
                    if (p.include_Grad == 1) GL[d](i, j, k) += c->GLG[d](i, j, k);
                    if (p.include_Elec == 1) GL[d](i, j, k) += c->GLE[d](i, j, k);
                }
}

// MultiFab::LinComb(dst, a, x, b, y) over valid + ghost cells
void lincomb(Fab& dst, double a, const Fab& x, double b, const Fab& y) {
    for (size_t q = 0; q < dst.v.size(); ++q) dst.v[q] = a * x.v[q] + b * y.v[q];
}
void copy_valid(Fab& dst, const Fab& src) {
    for (int k = 0; k < dst.nz; ++k)
        for (int j = 0; j < dst.ny; ++j)
            for (int i = 0; i < dst.nx; ++i) dst(i, j, k) = src(i, j, k);
}

// ------------------------------------------- main.cpp:265-348 -----------
int tdgl_update(ofx_ctx* c) {
    tdgl_rhs(c, c->GL, c->P);
    for (int d = 0; d < 3; ++d) {
        lincomb(c->Ppre[d], 1.0, c->P[d], c->p.dt, c->GL[d]);
        fill_boundary(c->Ppre[d], c->p.is_periodic);
    }
    if (c->p.TimeIntegratorOrder == 1) {
        for (int d = 0; d < 3; ++d) {
            copy_valid(c->P[d], c->Ppre[d]);
            fill_boundary(c->P[d], c->p.is_periodic);
        }
        return 0;
    }
    int st = compute_phi_rho(c, c->Ppre);
    if (st) return st;
    compute_E(c);
    tdgl_rhs(c, c->GLpre, c->Ppre);
    for (int d = 0; d < 3; ++d) {
        Fab avg = c->GL[d];
        lincomb(avg, 0.5, c->GL[d], 0.5, c->GLpre[d]);
        lincomb(c->Pnew[d], 1.0, c->P[d], c->p.dt, avg);
    }
    for (int d = 0; d < 3; ++d) {
        copy_valid(c->P[d], c->Pnew[d]);
        fill_boundary(c->P[d], c->p.is_periodic);
    }
    return 0;
}

// ------------------------------------- ElectrostaticSolver.cpp:526-560 ---
void check_steady_state(ofx_ctx* c, int step) {
    double phi_max = 0.0;
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i) phi_max = std::max(phi_max, std::fabs(c->phi(i, j, k)));
    for (int k = -1; k <= c->n[2]; ++k)
        for (int j = -1; j <= c->n[1]; ++j)
            for (int i = -1; i <= c->n[0]; ++i)
                c->phidiff(i, j, k) = std::fabs(c->phi(i, j, k) - c->phi_old(i, j, k)) / phi_max;
    // norm0 keeps the running maximum under std::max, which passes over NaN
    // (the phi == 0 case, where 0/0 fills Phidiff)
    double max_phi_err = 0.0;
    for (int k = 0; k < c->n[2]; ++k)
        for (int j = 0; j < c->n[1]; ++j)
            for (int i = 0; i < c->n[0]; ++i) max_phi_err = std::max(max_phi_err, c->phidiff(i, j, k));
    if (step > 1) {
        if (max_phi_err < c->p.phi_tolerance) {
            c->steady_state_step = step;
            c->inc_step = step;
        }
    }
    copy_valid(c->phi_old, c->phi);
    c->last_steady_err = max_phi_err;
    if (c->p.verbose) printf("Steady state check : (phi(t) - phi(t-1)).norm0() = %g\n", max_phi_err);
}

} // namespace

// ============================================================ C API =====
extern "C" {

double ofx_uniform(unsigned long long seed, unsigned long long n) {
    uint64_t z = splitmix_mix((uint64_t)seed + (uint64_t)n * 0x9E3779B97F4A7C15ULL);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

int ofx_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

ofx_ctx* ofx_create(const ofx_params* pin, const double* tph, const double* aa, const double* ab, const double* at) {
    ofx_ctx* c = new ofx_ctx();
    c->p = *pin;
    const ofx_params& p = c->p;
    for (int d = 0; d < 3; ++d) {
        c->n[d] = p.n_cell[d];
        // Geometry::CellSize: (prob_hi - prob_lo) / n_cell
        c->dx[d] = (p.prob_hi[d] - p.prob_lo[d]) / p.n_cell[d];
    }
    if (!p.is_periodic[0] || !p.is_periodic[1] || p.is_periodic[2]) { delete c; return nullptr; }
    // DerivativeAlgorithm.H aborts on a flag outside 0..4 (e.g. :72)
    for (int d = 0; d < 3; ++d)
        if (p.P_BC_flag_lo[d] < 0 || p.P_BC_flag_lo[d] > 4 || p.P_BC_flag_hi[d] < 0 || p.P_BC_flag_hi[d] > 4) { delete c; return nullptr; }
    const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
    c->N = (size_t)nx * ny * nz;
    c->si.ni = std::sqrt(c->si.Nc * c->si.Nv) * exp(-0.5 * c->si.q * c->si.bandgap / (c->si.kb * c->si.T));
    c->inc_step = p.inc_step;
    c->Phi_Bc_hi = p.Phi_Bc_hi;

    // field allocation, main.cpp:73-173 (ghost counts as the reference)
    c->mask.define(nx, ny, nz, 1);
    c->tphase.define(nx, ny, nz, 1);
    c->Gamma.define(nx, ny, nz, 1);
    for (int d = 0; d < 3; ++d) {
        c->P[d].define(nx, ny, nz, 1); c->Pnew[d].define(nx, ny, nz, 1); c->Ppre[d].define(nx, ny, nz, 1);
        c->GL[d].define(nx, ny, nz, 1); c->GLL[d].define(nx, ny, nz, 1); c->GLG[d].define(nx, ny, nz, 1);
        c->GLE[d].define(nx, ny, nz, 1); c->GLpre[d].define(nx, ny, nz, 1);
        c->E[d].define(nx, ny, nz, 0);
        c->ang[d].define(nx, ny, nz, 0);
    }
    c->phi.define(nx, ny, nz, 1); c->phi_old.define(nx, ny, nz, 1); c->phi_prev.define(nx, ny, nz, 1);
    c->phidiff.define(nx, ny, nz, 1);
    c->rhs.define(nx, ny, nz, 0); c->rho.define(nx, ny, nz, 0); c->e_den.define(nx, ny, nz, 0);
    c->h_den.define(nx, ny, nz, 0); c->alpha_cc.define(nx, ny, nz, 0);
    c->beta_cc.define(nx, ny, nz, 1);

    // InitializeMaterialMask, Initialization.cpp:169-206 (grown box, then
    // FillBoundary)
    for (int k = -1; k <= nz; ++k)
        for (int j = -1; j <= ny; ++j)
            for (int i = -1; i <= nx; ++i) {
                double x = p.prob_lo[0] + (i + 0.5) * c->dx[0];
                double y = p.prob_lo[1] + (j + 0.5) * c->dx[1];
                double z = p.prob_lo[2] + (k + 0.5) * c->dx[2];
                double m;
                if (x <= p.FE_hi[0] && x >= p.FE_lo[0] && y <= p.FE_hi[1] && y >= p.FE_lo[1] && z <= p.FE_hi[2] && z >= p.FE_lo[2]) {
                    m = 0.;
                } else if (x <= p.DE_hi[0] && x >= p.DE_lo[0] && y <= p.DE_hi[1] && y >= p.DE_lo[1] && z <= p.DE_hi[2] && z >= p.DE_lo[2]) {
                    m = 1.;
                } else if (x <= p.SC_hi[0] && x >= p.SC_lo[0] && y <= p.SC_hi[1] && y >= p.SC_lo[1] && z <= p.SC_hi[2] && z >= p.SC_lo[2]) {
                    m = 2.;
                    if (x <= p.Channel_hi[0] && x >= p.Channel_lo[0] && y <= p.Channel_hi[1] && y >= p.Channel_lo[1] && z <= p.Channel_hi[2] && z >= p.Channel_lo[2])
                        m = 3.;
                } else {
                    m = 1.;
                }
                c->mask(i, j, k) = m;
            }
    fill_boundary(c->mask, p.is_periodic);

    // t-phase mask and Euler angles (main.cpp:178-181): valid cells from the
    // caller, ghosts via FillBoundary
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t q = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
                c->tphase(i, j, k) = tph ? tph[q] : 0.0;
                c->ang[0](i, j, k) = aa ? aa[q] : 0.0;
                c->ang[1](i, j, k) = ab ? ab[q] : 0.0;
                c->ang[2](i, j, k) = at ? at[q] : 0.0;
            }
    fill_boundary(c->tphase, p.is_periodic);

    // Contains_sc, FerroXUtil.cpp:12-41
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                if (c->mask(i, j, k) >= 2.0) c->contains_sc = true;

    // InitializePermittivity, ElectrostaticSolver.cpp:205-299
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double m = c->mask(i, j, k);
                double b;
                if (m == 0.0) {
                    b = p.epsilonX_fe * p.epsilon_0;
                    if (c->tphase(i, j, k) == 1.0) b = p.epsilonX_fe_tphase * p.epsilon_0;
                } else if (m == 1.0) {
                    b = p.epsilon_de * p.epsilon_0;
                } else if (m >= 2.0) {
                    b = p.epsilon_si * p.epsilon_0;
                } else {
                    b = p.epsilon_de * p.epsilon_0;
                }
                c->beta_cc(i, j, k) = b;
            }
    fill_boundary(c->beta_cc, p.is_periodic);
    for (int j = -1; j <= ny; ++j)
        for (int i = -1; i <= nx; ++i) {
            c->beta_cc(i, j, -1) = c->beta_cc(i, j, 0);        // z Dirichlet
            c->beta_cc(i, j, nz) = c->beta_cc(i, j, nz - 1);
        }
    // AverageCellCenteredMultiFabToCellFaces, eXstaticUtil.cpp:105-137
    c->bxf.assign((size_t)(nx + 1) * ny * nz, 0.0);
    c->byf.assign((size_t)nx * (ny + 1) * nz, 0.0);
    c->bzf.assign((size_t)nx * ny * (nz + 1), 0.0);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i)
                c->bxf[(size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k)] = 0.5 * (c->beta_cc(i, j, k) + c->beta_cc(i - 1, j, k));
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i < nx; ++i)
                c->byf[(size_t)i + (size_t)nx * ((size_t)j + (size_t)(ny + 1) * k)] = 0.5 * (c->beta_cc(i, j, k) + c->beta_cc(i, j - 1, k));
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                c->bzf[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)] = 0.5 * (c->beta_cc(i, j, k) + c->beta_cc(i, j, k - 1));

    // SetupMLMG -> SetPhiBC_z (ElectrostaticSolver.cpp:597-601)
    set_phi_bc_z(c);

    // InitializePandRho, Initialization.cpp:6-166
    const uint64_t seed = (uint64_t)(int64_t)p.random_seed;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
                double x = p.prob_lo[0] + (i + 0.5) * c->dx[0];
                double y = p.prob_lo[1] + (j + 0.5) * c->dx[1];
                double z = p.prob_lo[2] + (k + 0.5) * c->dx[2];
                double pp = 0, pq = 0, pr = 0, G = 0;
                if (c->mask(i, j, k) == 0.0) {
                    if (p.prob_type == 1) {
                        size_t r = (size_t)i + (size_t)k * nz;
                        double u = ofx_uniform(seed, r + 1);
                        pp = (-1.0 + 2.0 * u) * p.Remnant_P[0];
                        pq = (-1.0 + 2.0 * u) * p.Remnant_P[1];
                        pr = (-1.0 + 2.0 * u) * p.Remnant_P[2];
                    } else if (p.prob_type == 2) {
                        pp = (-1.0 + 2.0 * ofx_uniform(seed, 3 * idx + 1)) * p.Remnant_P[0];
                        pq = (-1.0 + 2.0 * ofx_uniform(seed, 3 * idx + 2)) * p.Remnant_P[1];
                        pr = (-1.0 + 2.0 * ofx_uniform(seed, 3 * idx + 3)) * p.Remnant_P[2];
                    } else if (p.prob_type == 3) {
                        double DEz = p.DE_hi[2];
                        double g = exp(-(x * x / (2.0 * 5.e-9 * 5.e-9) + y * y / (2.0 * 5.e-9 * 5.e-9) +
                                         (z - 1.5 * DEz) * (z - 1.5 * DEz) / (2.0 * 2.0e-9 * 2.0e-9)));
                        pp = p.Remnant_P[0] * g;
                        pq = p.Remnant_P[1] * g;
                        pr = p.Remnant_P[2] * g;
                    }
                    G = p.BigGamma;
                    if (c->tphase(i, j, k) == 1.0) pr = 0.0;
                }
                if (p.is_polarization_scalar == 1) { pp = 0.0; pq = 0.0; }
                c->P[0](i, j, k) = pp; c->P[1](i, j, k) = pq; c->P[2](i, j, k) = pr;
                c->Gamma(i, j, k) = G;
                (void)idx;
                // intrinsic charge: only SC cells carry n = p = n_i, N_A, N_D
                if (c->mask(i, j, k) >= 2.0) {
                    c->h_den(i, j, k) = c->si.ni;
                    c->e_den(i, j, k) = c->si.ni;
                    c->rho(i, j, k) = c->si.q * (c->si.ni - c->si.ni - p.acceptor_doping + p.donor_doping);
                } else {
                    c->rho(i, j, k) = 0.0;
                }
            }
    for (int d = 0; d < 3; ++d) fill_boundary(c->P[d], p.is_periodic);
    return c;
}

void ofx_destroy(ofx_ctx* c) { delete c; }

static Fab* field_ptr(ofx_ctx* c, int id) {
    switch (id) {
    case OFX_PX: return &c->P[0];
    case OFX_PY: return &c->P[1];
    case OFX_PZ: return &c->P[2];
    case OFX_PHI: return &c->phi;
    case OFX_POISSON_RHS: return &c->rhs;
    case OFX_EX: return &c->E[0];
    case OFX_EY: return &c->E[1];
    case OFX_EZ: return &c->E[2];
    case OFX_HOLES: return &c->h_den;
    case OFX_ELECTRONS: return &c->e_den;
    case OFX_CHARGE: return &c->rho;
    case OFX_EPSILON: return &c->beta_cc;
    case OFX_MASK: return &c->mask;
    case OFX_TPHASE: return &c->tphase;
    case OFX_ANGLE_ALPHA: return &c->ang[0];
    case OFX_ANGLE_BETA: return &c->ang[1];
    case OFX_ANGLE_THETA: return &c->ang[2];
    case OFX_PHIDIFF: return &c->phidiff;
    case OFX_ALPHA_CC: return &c->alpha_cc;
    case OFX_GAMMA: return &c->Gamma;
    }
    return nullptr;
}

int ofx_get_field(ofx_ctx* c, int id, double* out) {
    Fab* f = field_ptr(c, id);
    if (!f) return -1;
    std::vector<double> v;
    fab_to_valid(*f, v);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
    return 0;
}

int ofx_set_field(ofx_ctx* c, int id, const double* in) {
    Fab* f = field_ptr(c, id);
    if (!f) return -1;
    valid_to_fab(in, *f);
    if (id == OFX_PHI) phi_ghosts_after_solve(c);   // phi as left by a solve
    else if (id <= OFX_PZ || id == OFX_MASK || id == OFX_TPHASE) fill_boundary(*f, c->p.is_periodic);
    return 0;
}

static int get_ghosted(const Fab& f, double* out) {
    size_t q = 0;
    for (int k = -1; k <= f.nz; ++k)
        for (int j = -1; j <= f.ny; ++j)
            for (int i = -1; i <= f.nx; ++i) out[q++] = f(i, j, k);
    return 0;
}
int ofx_get_mask_ghost(ofx_ctx* c, double* out) { return get_ghosted(c->mask, out); }
int ofx_get_phi_ghost(ofx_ctx* c, double* out) { return get_ghosted(c->phi, out); }

int ofx_get_beta_faces(ofx_ctx* c, double* bx, double* by, double* bz) {
    std::memcpy(bx, c->bxf.data(), c->bxf.size() * sizeof(double));
    std::memcpy(by, c->byf.data(), c->byf.size() * sizeof(double));
    std::memcpy(bz, c->bzf.data(), c->bzf.size() * sizeof(double));
    return 0;
}

int ofx_compute_poisson_rhs(ofx_ctx* c) { compute_poisson_rhs(c, c->rhs, c->P, c->rho); return 0; }
int ofx_compute_rho(ofx_ctx* c) { compute_rho(c, c->phi, c->rho, c->e_den, c->h_den); return 0; }
int ofx_compute_phi_rho(ofx_ctx* c) { return compute_phi_rho(c, c->P); }
int ofx_compute_E(ofx_ctx* c) { compute_E(c); return 0; }
int ofx_tdgl_euler(ofx_ctx* c) { return tdgl_update(c); }
int ofx_set_phi_bc(ofx_ctx* c) { set_phi_bc_z(c); return 0; }

int ofx_tdgl_terms(ofx_ctx* c, double* landau, double* grad, double* elec) {
    calculate_landau(c, c->GLL, c->P);
    calculate_grad(c, c->GLG, c->P);
    calculate_elec(c, c->GLE);
    std::vector<double> v;
    for (int d = 0; d < 3; ++d) {
        fab_to_valid(c->GLL[d], v); std::memcpy(landau + d * c->N, v.data(), c->N * sizeof(double));
        fab_to_valid(c->GLG[d], v); std::memcpy(grad + d * c->N, v.data(), c->N * sizeof(double));
        fab_to_valid(c->GLE[d], v); std::memcpy(elec + d * c->N, v.data(), c->N * sizeof(double));
    }
    return 0;
}

int ofx_poisson_solve(ofx_ctx* c, const double* rhs, const double* alpha_cc, double* phi, double rtol, int* iters_out, double* resid_out) {
    mg_setup(c, alpha_cc);
    return mg_solve(c, rhs, phi, rtol, iters_out, resid_out);
}

int ofx_poisson_apply(ofx_ctx* c, const double* alpha_cc, const double* phi, int inh, double* out) {
    mg_setup(c, alpha_cc);
    const MGLevel& l = c->mg[0];
    for (int k = 0; k < l.n[2]; ++k)
        for (int j = 0; j < l.n[1]; ++j)
            for (int i = 0; i < l.n[0]; ++i)
                out[L3(l, i, j, k)] = apply_cell(l, phi, i, j, k, inh ? c->V_lo : 0.0,
                                                 inh ? (c->eb_nz > 0 ? c->eb_V : c->V_hi) : 0.0);
    return 0;
}

int ofx_set_eb(ofx_ctx* c, int nz_fluid, double V) {
    if (nz_fluid < 0 || nz_fluid >= c->n[2]) return -1;
    c->eb_nz = nz_fluid;
    c->eb_V = V;
    c->mg.clear();   // the hierarchy is built for the solve's layers
    return 0;
}

// one pass of the step loop, main.cpp:261-621
int ofx_step(ofx_ctx* c, int step) {
    const ofx_params& p = c->p;
    int st = compute_phi_rho(c, c->P);
    if (st) return st;
    compute_E(c);
    st = tdgl_update(c);
    if (st) return st;
    check_steady_state(c, step);
    compute_E(c);
    c->time = c->time + p.dt;
    const double tiny = 1.e-6;
    bool inc = false;
    if (p.voltage_sweep == 1) {
        if (p.sweep_mode == 1) inc = p.steps_per_voltage > 0 && step % p.steps_per_voltage == 0;
        else inc = c->inc_step > 0 && step == c->inc_step;
    }
    if (inc) {
        c->Phi_Bc_hi += c->sign * p.Phi_Bc_inc;
        c->num_Vapp += 1;
        if (std::fabs(std::fabs(c->Phi_Bc_hi) - p.Phi_Bc_hi_max) <= tiny) c->sign *= -1;
        set_phi_bc_z(c);
        st = compute_phi_rho(c, c->P);
        if (st) return st;
    }
    if (p.voltage_sweep == 0 && step == c->steady_state_step) return 1;
    if (p.voltage_sweep == 1 && c->Phi_Bc_hi > 0. && c->Phi_Bc_hi - p.Phi_Bc_hi_max > tiny) return 1;
    if (p.voltage_sweep == 1 && c->Phi_Bc_hi < 0. && -c->Phi_Bc_hi - p.Phi_Bc_hi_max > tiny) return 1;
    if (p.voltage_sweep == 1 && c->num_Vapp == p.num_Vapp_max) return 1;
    return 0;
}

int ofx_run(ofx_ctx* c, int nsteps) {
    for (int step = 1; step <= nsteps; ++step) {
        int st = ofx_step(c, step);
        if (st < 0) return st;
        if (st == 1) return step;
    }
    return nsteps;
}

double ofx_get_scalar(ofx_ctx* c, const char* name) {
    std::string s(name);
    if (s == "Phi_Bc_hi") return c->Phi_Bc_hi;
    if (s == "V_lo") return c->V_lo;
    if (s == "V_hi") return c->V_hi;
    if (s == "time") return c->time;
    if (s == "steady_state_step") return c->steady_state_step;
    if (s == "inc_step") return c->inc_step;
    if (s == "num_Vapp") return c->num_Vapp;
    if (s == "sign") return c->sign;
    if (s == "contains_sc") return c->contains_sc;
    if (s == "newton_iters") return c->last_newton_iters;
    if (s == "mg_iters") return c->last_mg_iters;
    if (s == "phi_err") return c->last_phi_err;
    if (s == "steady_err") return c->last_steady_err;
    if (s == "ni") return c->si.ni;
    if (s == "dx") return c->dx[0];
    if (s == "dy") return c->dx[1];
    if (s == "dz") return c->dx[2];
    return std::nan("");
}

int ofx_set_scalar(ofx_ctx* c, const char* name, double v) {
    std::string s(name);
    if (s == "Phi_Bc_hi") { c->Phi_Bc_hi = v; return 0; }
    if (s == "mg_rtol") { c->p.mg_rtol = v; return 0; }
    if (s == "phi_ghost_mode") { c->p.phi_ghost_mode = (int)v; return 0; }
    if (s == "verbose") { c->p.verbose = (int)v; return 0; }
    return -1;
}

} // extern "C"
