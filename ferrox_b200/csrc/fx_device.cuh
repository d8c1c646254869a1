// fx_device.cuh -- device data layout and the restated FerroX stencils.
//
// HBM layout (one GPU, one box covering the domain):
//   * every cell field is a flat array, x fastest: c = i + nx*(j + ny*k);
//     periodic x/y neighbours are wrapped in the index, no ghost storage;
//   * P components stay FP64 (the accumulated state); outside the z range a P
//     read returns 0, which is what the reference's never-filled z ghost cells
//     of P_old hold (main.cpp:157, :302-306);
//   * the material code is one byte per cell, code = mask | tphase << 2, with
//     one extra z layer below and above (nx*ny*(nz+2) bytes) so the stencils
//     can read the mask of the z ghost cells that InitializeMaterialMask fills
//     with the cell-centre rule (Initialization.cpp:177-202);
//   * an optional second byte per cell indexes a small table of rotation
//     matrices (per grain / per Euler-angle triple) and per-grain Landau alpha;
//   * phi has no ghost storage: its z ghost value follows from the electrode
//     value and the ghost mode (see phi_ghost()).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fx {

struct Variant {
    double R[9];
    double alpha;
    double pad[2];
};

struct DevParams {
    int nx, ny, nz;
    int ngrid_red;             // blocks of the reduction kernels
    long long nxy, N;
    double dx[3];
    double ih2[3];             // 1/dx^2
    double dt;
    double alpha, beta, gamma, a12, a112, a123;
    double BigGamma, g11, g44, g44p, g12, lambda;
    int flo[3], fhi[3];
    int incl_L, incl_G, incl_E;
    int scalar;
    double eps[8];             // eps_r * eps_0 by material code
    // semiconductor (ChargeDensity.cpp, FerroX.cpp:534-554)
    double q, kb, T, Nc, Nv, Eg, Chi, Ea, Ed, NA, ND, phi_ref;
    // Boltzmann statistics in product form: with E = exp(sc_qkT (phi - phi_ref)),
    // e = sc_Ce E, h = sc_Ch / E, acceptors NA / (1 + sc_Ca / E), donors
    // ND / (1 + sc_Cd E) (Ef = 0)
    double sc_qkT, sc_Ce, sc_Ch, sc_Ca, sc_Cd;
    int use_FD;
    double delta, inv_delta, neg_inv_delta;
    // z Dirichlet values of phi held by the solver and the ghost mode
    double V_lo, V_hi;
    int ghost_mode;
    // the Poisson solve's cells, a prefix of every cell array (N, or the
    // fluid layers below an embedded boundary), and the Dirichlet value on
    // their top face (V_hi, or the embedded surface's)
    long long Ns;
    double Vs_hi;
    // one byte per cell: 1 where the cell and its 18 face and edge neighbours
    // are ferroelectric and 1 <= k <= nz - 2, so that every mask test of the
    // P stencils passes (their central forms apply); null: none flagged
    const uint8_t* interior;
    // the planes holding every cell the TDGL update changes (ferroelectric,
    // not t-phase); P elsewhere never changes and both ping-pong buffers hold it
    int fe_k0, fe_k1;
};

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__device__ __forceinline__ size_t cidx(const DevParams& p, int i, int j, int k) {
    return (size_t)i + (size_t)p.nx * ((size_t)j + (size_t)p.ny * (size_t)k);
}

// material code at (i, j, k); i, j may be one or two cells outside (periodic),
// k in [-1, nz]
__device__ __forceinline__ int mcode(const uint8_t* __restrict__ code, const DevParams& p, int i, int j, int k) {
    i = wrap(i, p.nx);
    j = wrap(j, p.ny);
    return __ldg(code + (size_t)i + (size_t)p.nx * ((size_t)j + (size_t)p.ny * (size_t)(k + 1)));
}

template <typename T>
struct PView {
    const double* __restrict__ a;
    const DevParams* p;
    __device__ __forceinline__ T operator()(int i, int j, int k) const {
        if (k < 0 || k >= p->nz) return T(0);
        return T(__ldg(a + cidx(*p, wrap(i, p->nx), wrap(j, p->ny), k)));
    }
};

// unit impulse at cell (ci, cj, ck): evaluating a linear stencil on it gives
// that row's coefficient of the impulse cell (used for transposed stencils)
template <typename T>
struct DeltaView {
    int ci, cj, ck;
    const DevParams* p;
    __device__ __forceinline__ T operator()(int i, int j, int k) const {
        if (k < 0 || k >= p->nz) return T(0);
        return (wrap(i, p->nx) == ci && wrap(j, p->ny) == cj && k == ck) ? T(1) : T(0);
    }
};

struct MView {
    const uint8_t* __restrict__ code;
    const DevParams* p;
    __device__ __forceinline__ int operator()(int i, int j, int k) const { return mcode(code, *p, i, j, k) & 3; }
};

// The mask seen from an interior cell (DevParams::interior): every cell its
// stencils test is ferroelectric, so each derivative takes its central form.
// Evaluating the same stencil functions with this view gives the same
// arithmetic as with MView, without the mask loads and branches.
struct MInterior {
    __device__ __forceinline__ int operator()(int, int, int) const { return 0; }
};

// P read from an interior cell: every z index it reads is inside [0, nz)
template <typename T>
struct PViewIn {
    const double* __restrict__ a;
    const DevParams* p;
    __device__ __forceinline__ T operator()(int i, int j, int k) const {
        return T(__ldg(a + cidx(*p, wrap(i, p->nx), wrap(j, p->ny), k)));
    }
};

// DPDx / DPDy / DPDz, DerivativeAlgorithm.H:45-252 (direction D)
template <int D, typename T, typename FV, typename MV>
__device__ __forceinline__ T dpd(const FV& F, const MV& M, int i, int j, int k) {
    constexpr int ox = D == 0, oy = D == 1, oz = D == 2;
    const DevParams& p = *F.p;
    const T h = T(p.dx[D]);
    const T lam = T(p.lambda);
    const int mc = M(i, j, k);
    if (mc != 0) return T(0);
    if (M(i - ox, j - oy, k - oz) != 0) {
        const int f = p.flo[D];
        const T F0 = F(i, j, k), F1 = F(i + ox, j + oy, k + oz);
        if (f == 0) { T F_lo = T(0); return (T(-4.) * F_lo + T(3.) * F0 + F1) / (T(3.) * h); }
        if (f == 1) { T F_lo = F0 / (T(1) + h / T(2) / lam); return (h * F_lo / lam - F0 + F1) / (T(2.) * h); }
        if (f == 2) return (-F0 + F1) / (T(2.) * h);
        if (f == 3) return (-F(i - ox, j - oy, k - oz) + F1) / (T(2.) * h);
        return (-F0 + F1) / h;
    }
    if (M(i + ox, j + oy, k + oz) != 0) {
        const int f = p.fhi[D];
        const T F0 = F(i, j, k), Fm = F(i - ox, j - oy, k - oz);
        if (f == 0) { T F_hi = T(0); return (T(4.) * F_hi - T(3.) * F0 - Fm) / (T(3.) * h); }
        if (f == 1) { T F_hi = F0 / (T(1) - h / T(2) / lam); return (h * F_hi / lam + F0 - Fm) / (T(2.) * h); }
        if (f == 2) return (F0 - Fm) / (T(2.) * h);
        if (f == 3) return (F(i + ox, j + oy, k + oz) - Fm) / (T(2.) * h);
        return (F0 - Fm) / h;
    }
    return (F(i + ox, j + oy, k + oz) - F(i - ox, j - oy, k - oz)) / (T(2.) * h);
}

// a product that the compiler may not fuse into a neighbouring add: the
// second-derivative forms round 2 F the same way whichever branches survive
// inlining (and as the oracle, built without contraction, does)
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// DoubleDPDx / y / z, DerivativeAlgorithm.H:256-467 (direction D)
template <int D, typename T, typename FV, typename MV>
__device__ __forceinline__ T ddpd(const FV& F, const MV& M, int i, int j, int k) {
    constexpr int ox = D == 0, oy = D == 1, oz = D == 2;
    const DevParams& p = *F.p;
    const T h = T(p.dx[D]);
    const T lam = T(p.lambda);
    if (M(i, j, k) != 0) return T(0);
    const T F0 = F(i, j, k);
    if (M(i - ox, j - oy, k - oz) != 0) {
        const int f = p.flo[D];
        const T F1 = F(i + ox, j + oy, k + oz);
        if (f == 0) { T F_lo = T(0); return T(4.) * (T(2.) * F_lo - T(3.) * F0 + F1) / T(3.) / h / h; }
        if (f == 1) { T F_lo = F0 / (T(1) + h / T(2) / lam); return (-h * F_lo / lam - F0 + F1) / h / h; }
        if (f == 2) return (-F0 + F1) / h / h;
        if (f == 3) {
            const T Fm = F(i - ox, j - oy, k - oz);
            if (D == 2) return (Fm - mul_rn(T(2.), F0) + F1) / h / h;
            return (F1 - mul_rn(T(2.), F0) + Fm) / h / h;
        }
        const T F2 = F(i + 2 * ox, j + 2 * oy, k + 2 * oz);
        if (D == 2) return (F0 - mul_rn(T(2.), F1) + F2) / h / h;
        return (F2 - mul_rn(T(2.), F1) + F0) / h / h;
    }
    if (M(i + ox, j + oy, k + oz) != 0) {
        const int f = p.fhi[D];
        const T Fm = F(i - ox, j - oy, k - oz);
        if (f == 0) { T F_hi = T(0); return T(4.) * (T(2.) * F_hi - T(3.) * F0 + Fm) / T(3.) / h / h; }
        if (f == 1) { T F_hi = F0 / (T(1) - h / T(2) / lam); return (h * F_hi / lam - F0 + Fm) / h / h; }
        if (f == 2) return (-F0 + Fm) / h / h;
        if (f == 3) return (F(i + ox, j + oy, k + oz) - mul_rn(T(2.), F0) + Fm) / h / h;
        return (F0 - mul_rn(T(2.), Fm) + F(i - 2 * ox, j - 2 * oy, k - 2 * oz)) / h / h;
    }
    return (F(i + ox, j + oy, k + oz) - mul_rn(T(2.), F0) + F(i - ox, j - oy, k - oz)) / (h * h);
}

// DoubleDPDxDy / DxDz / DyDz, DerivativeAlgorithm.H:471-497
template <typename T, typename FV, typename MV>
__device__ __forceinline__ T dxdy(const FV& F, const MV& M, int i, int j, int k) {
    return (dpd<1, T>(F, M, i + 1, j, k) - dpd<1, T>(F, M, i - 1, j, k)) / T(2.) / T(F.p->dx[0]);
}
template <typename T, typename FV, typename MV>
__device__ __forceinline__ T dxdz(const FV& F, const MV& M, int i, int j, int k) {
    return (dpd<2, T>(F, M, i + 1, j, k) - dpd<2, T>(F, M, i - 1, j, k)) / T(2.) / T(F.p->dx[0]);
}
template <typename T, typename FV, typename MV>
__device__ __forceinline__ T dydz(const FV& F, const MV& M, int i, int j, int k) {
    return (dpd<2, T>(F, M, i, j + 1, k) - dpd<2, T>(F, M, i, j - 1, k)) / T(2.) / T(F.p->dx[1]);
}

// phi with its z ghost values: after the MLMG solve the ghost holds the
// maxorder-2 Dirichlet extrapolation 2 V - phi_0 (mode 0), or the face value V
// (mode 1), or 0 (mode 2)
__device__ __forceinline__ double phi_at(const double* __restrict__ phi, const DevParams& p, int i, int j, int k) {
    i = wrap(i, p.nx);
    j = wrap(j, p.ny);
    if (k < 0) {
        if (p.ghost_mode == 0) return 2.0 * p.V_lo + (-1.0) * __ldg(phi + cidx(p, i, j, 0));
        return p.ghost_mode == 1 ? p.V_lo : 0.0;
    }
    if (k >= p.nz) {
        if (p.ghost_mode == 0) return 2.0 * p.V_hi + (-1.0) * __ldg(phi + cidx(p, i, j, p.nz - 1));
        return p.ghost_mode == 1 ? p.V_hi : 0.0;
    }
    return __ldg(phi + cidx(p, i, j, k));
}

// grad phi as used by ComputeEfromPhi (ElectrostaticSolver.cpp:195-197):
// central in x / y, DphiDz (DerivativeAlgorithm.H:8-22) in z with the
// one-sided forms in the electrode-adjacent layers
// phi accessor with the ghost values (see phi_at)
struct PhiAt {
    const double* __restrict__ phi;
    const DevParams* p;
    __device__ __forceinline__ double operator()(int i, int j, int k) const { return phi_at(phi, *p, i, j, k); }
};

// derivative of phi_at(i, j, k) with respect to phi at cell (ci, cj, ck):
// the extrapolated ghost 2 V - phi_0 depends on the electrode-layer cell
struct PhiDelta {
    int ci, cj, ck;
    const DevParams* p;
    __device__ __forceinline__ double operator()(int i, int j, int k) const {
        i = wrap(i, p->nx);
        j = wrap(j, p->ny);
        if (k < 0) return (p->ghost_mode == 0 && i == ci && j == cj && ck == 0) ? -1.0 : 0.0;
        if (k >= p->nz) return (p->ghost_mode == 0 && i == ci && j == cj && ck == p->nz - 1) ? -1.0 : 0.0;
        return (i == ci && j == cj && k == ck) ? 1.0 : 0.0;
    }
};

template <typename T, typename A>
__device__ __forceinline__ void grad_phi_acc(const A& f, const DevParams& p, int i, int j, int k, T& gx, T& gy, T& gz) {
    // differences are taken in FP64 (phi is O(1 V) and its differences small)
    gx = T((f(i + 1, j, k) - f(i - 1, j, k)) / (2. * p.dx[0]));
    gy = T((f(i, j + 1, k) - f(i, j - 1, k)) / (2. * p.dx[1]));
    const double dz = p.dx[2];
    if (k == 0) {
        gz = T((-4. * f(i, j, k - 1) + 3. * f(i, j, k) + f(i, j, k + 1)) / (3. * dz));
    } else if (k == p.nz - 1) {
        gz = T((4. * f(i, j, k + 1) - 3. * f(i, j, k) - f(i, j, k - 1)) / (3. * dz));
    } else {
        gz = T((f(i, j, k + 1) - f(i, j, k - 1)) / (2. * dz));
    }
}

template <typename T>
__device__ __forceinline__ void grad_phi(const double* __restrict__ phi, const DevParams& p, int i, int j, int k,
                                         T& gx, T& gy, T& gz) {
    grad_phi_acc<T>(PhiAt{phi, &p}, p, i, j, k, gx, gy, gz);
}

// Landau derivative dF/dP_a (TotalEnergyDensity.cpp:88-110) for component a
// with the other two components b, c
template <typename T>
__device__ __forceinline__ T landau(const DevParams& p, T alpha, T a, T b, T c) {
    const T a2 = a * a, b2 = b * b, c2 = c * c;
    return alpha * a + T(p.beta) * (a2 * a) + T(p.gamma) * (a2 * a2 * a)
        + T(2.) * T(p.a12) * a * b2
        + T(2.) * T(p.a12) * a * c2
        + T(4.) * T(p.a112) * (a2 * a) * (b2 + c2)
        + T(2.) * T(p.a112) * a * (b2 * b2)
        + T(2.) * T(p.a112) * a * (c2 * c2)
        + T(2.) * T(p.a123) * a * b2 * c2;
}

// the six second derivatives of one component, for the rotated Pr term
template <typename T>
struct Hess { T xx, yy, zz, xy, yz, xz; };

template <typename T, bool ROT, typename FV, typename MV>
__device__ __forceinline__ Hess<T> hess(const FV& F, const MV& M, int i, int j, int k) {
    Hess<T> h;
    h.xx = ddpd<0, T>(F, M, i, j, k);
    h.yy = ddpd<1, T>(F, M, i, j, k);
    h.zz = ddpd<2, T>(F, M, i, j, k);
    if (ROT) {
        h.xy = dxdy<T>(F, M, i, j, k);
        h.yz = dydz<T>(F, M, i, j, k);
        h.xz = dxdz<T>(F, M, i, j, k);
    } else {
        h.xy = h.yz = h.xz = T(0);
    }
    return h;
}

// R_a1 R_a1 Dxx + ... + 2 R_a3 R_a1 Dxz, TotalEnergyDensity.cpp:209-228
template <typename T>
__device__ __forceinline__ T rot_quad(const T* R, int a, const Hess<T>& H) {
    const T r1 = R[3 * a], r2 = R[3 * a + 1], r3 = R[3 * a + 2];
    return r1 * r1 * H.xx + r2 * r2 * H.yy + r3 * r3 * H.zz + T(2.) * r1 * r2 * H.xy + T(2.) * r2 * r3 * H.yz +
           T(2.) * r3 * r1 * H.xz;
}

// ChargeDensity.cpp:4-11
__device__ __forceinline__ double fd_half(double eta) {
    double nu = pow(eta, 4.0) + 50.0 + 33.6 * eta * (1.0 - 0.68 * exp(-0.17 * pow((eta + 1.0), 2.0)));
    double xi = 3.0 * sqrt(3.14) / (4.0 * pow(nu, 3. / 8.));
    return pow(exp(-eta) + xi, -1.0);
}

// ChargeDensity.cpp:46-93: carrier densities and charge at potential phi.
// With Boltzmann statistics the four exponentials of the reference,
// exp(+-q (phi - phi_ref) / kT + const), are one exponential E and its
// reciprocal times constants formed on the host; the product form agrees with
// the reference's expressions to rounding (the exponent's own rounding,
// ~1e-14 relative at |exponent| ~ 150, dominates both).
__device__ __forceinline__ double sc_charge(const DevParams& p, double phi, double& e_den, double& h_den) {
    if (p.use_FD != 1) {
        const double E = exp(p.sc_qkT * (phi - p.phi_ref));
        const double r = 1.0 / E;
        e_den = p.sc_Ce * E;
        h_den = p.sc_Ch * r;
        const double acc = p.NA != 0.0 ? p.NA / (1.0 + p.sc_Ca * r) : 0.0;
        const double don = p.ND != 0.0 ? p.ND / (1.0 + p.sc_Cd * E) : 0.0;
        return p.q * (h_den - e_den - acc + don);
    }
    const double Ef = 0.0;
    const double q = p.q, kb = p.kb, T = p.T, Chi = p.Chi, Eg = p.Eg, phi_ref = p.phi_ref;
    double Ec_corr = -q * (phi - phi_ref) - Chi * q;
    double Ev_corr = Ec_corr - q * Eg;
    const double g_A = 4.0, g_D = 2.0;
    if (p.use_FD == 1) {
        double eta_n = -(Ec_corr - q * Ef) / (kb * T);
        double eta_p = -(q * Ef - Ev_corr) / (kb * T);
        e_den = p.Nc * fd_half(eta_n);
        h_den = p.Nv * fd_half(eta_p);
    } else {
        e_den = p.Nc * exp(-(Ec_corr - q * Ef) / (kb * T));
        h_den = p.Nv * exp(-(q * Ef - Ev_corr) / (kb * T));
    }
    double acc = p.NA / (1.0 + g_A * exp((-q * Ef + q * p.Ea + q * phi_ref - q * Chi - q * Eg - q * phi) / (kb * T)));
    double don = p.ND / (1.0 + g_D * exp((q * Ef + q * p.Ed - q * phi_ref + q * Chi + q * phi) / (kb * T)));
    return q * (h_den - e_den - acc + don);
}

}  // namespace fx
