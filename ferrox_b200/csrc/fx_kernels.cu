// fx_kernels.cu -- the coupled-step kernels other than the Poisson multigrid.
//
//   k_tdgl      Calculate_Landau + Calculate_Grad + Calculate_Elec +
//               CalculateTDGL_RHS + the forward-Euler LinComb in one pass
//               (TotalEnergyDensity.cpp:6-294, main.cpp:280-306); E is taken
//               on the fly from phi (ElectrostaticSolver.cpp:134-203)
//   k_rhs_p     the FE branch of ComputePoissonRHS (ElectrostaticSolver.cpp:
//               73-77) -- P does not change inside the Newton loop
//   k_newton    ComputeRho(phi+delta) + dF_dPhi + ComputePoissonRHS_Newton
//               (ElectrostaticSolver.cpp:85-132, ChargeDensity.cpp:15-102)
//   k_rho       ComputeRho(phi) after the solve, with the L1 norms of the
//               Newton error (ElectrostaticSolver.cpp:723-738)
//   k_steady    CheckSteadyState's two norm0 reductions and the copy
//               (ElectrostaticSolver.cpp:526-560)
//   k_efield    ComputeEfromPhi, materialised for output only
#include "fx_kernels.h"

#include <cmath>

namespace fx {

namespace {

constexpr int RED_THREADS = 256;

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    if (!(v == v)) return;  // NaN never wins a std::max
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// block sum in a fixed order (deterministic for a fixed launch shape); the
// result is valid in the block's first thread.  Warps are numbered by the
// linear thread index, so 2-D and 3-D blocks reduce every warp.
__device__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    const int lane = t & 31, w = t >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < nw ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}
__device__ double block_max(double v, double* sh) {
    v = warp_max(v);
    const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    const int lane = t & 31, w = t >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < nw ? sh[lane] : 0.0;
        r = warp_max(r);
    }
    __syncthreads();
    return r;
}

// The gradient-energy terms of CalculateTDGL_RHS (TotalEnergyDensity.cpp:
// 133-251) at cell (i, j, k): gr for the r (z) component and, with vector P,
// gp and gq.  M and the P views decide how neighbours are read: MView / PView
// in general, MInterior / PViewIn at interior cells (same arithmetic).
template <typename T, bool SCALAR, bool ROT, typename MV, typename PV>
__device__ __forceinline__ void grad_terms(const DevParams& p, const T* R, const MV& M, const PV& Fp, const PV& Fq,
                                           const PV& Fr, int i, int j, int k, T& gr, T& gp, T& gq) {
    const T g11 = T(p.g11), g44 = T(p.g44), g44p = T(p.g44p), g12 = T(p.g12);
    Hess<T> H = hess<T, ROT>(Fr, M, i, j, k);
    T g;
    if (ROT) {
        g = -g11 * rot_quad(R, 2, H) - (g44 - g44p) * rot_quad(R, 0, H) - (g44 - g44p) * rot_quad(R, 1, H);
    } else {
        g = -g11 * H.zz - (g44 - g44p) * H.xx - (g44 - g44p) * H.yy;
    }
    if (!SCALAR) g = g - (g44 + g44p + g12) * dydz<T>(Fq, M, i, j, k) - (g44 + g44p + g12) * dxdz<T>(Fp, M, i, j, k);
    gr = g;
    if (!SCALAR) {
        gp = -g11 * ddpd<0, T>(Fp, M, i, j, k) - (g44 + g44p) * ddpd<1, T>(Fp, M, i, j, k) -
             (g44 + g44p) * ddpd<2, T>(Fp, M, i, j, k) - (g12 + g44 - g44p) * dxdy<T>(Fq, M, i, j, k) -
             (g12 + g44 - g44p) * dxdz<T>(Fr, M, i, j, k);
        gq = -g11 * ddpd<1, T>(Fq, M, i, j, k) - (g44 - g44p) * ddpd<0, T>(Fq, M, i, j, k) -
             (g44 - g44p) * ddpd<2, T>(Fq, M, i, j, k) - (g12 + g44 + g44p) * dxdy<T>(Fp, M, i, j, k) -
             (g12 + g44 - g44p) * dydz<T>(Fr, M, i, j, k);
    }
}

// One forward-Euler TDGL update.  T is the stencil arithmetic (double for the
// FP64 path, float for the mixed path); the P state is read and written in
// FP64.  SCALAR: is_polarization_scalar == 1 with Px = Py = 0, so only Pz is
// read and updated.  ROT: a rotation table is present (else R = identity,
// whose zero entries contribute exact zeros in the reference's sums).
//
// MODE 0: forward Euler, P_out = P + dt f(P, phi)           (main.cpp:294-306)
// MODE 1: predictor, f_buf = f(P, phi), P_out = P + dt f     (main.cpp:291-297)
// MODE 2: corrector, f* = f(P, phi) with P the predictor state,
//         P_out = P_old + dt (0.5 f_buf + 0.5 f*)             (main.cpp:323-340)
// In MODE 2 P_out may alias P_old (each cell reads its own P_old first).
template <typename T, bool SCALAR, bool ROT, int MODE>
__global__ void __launch_bounds__(256) k_tdgl(DevParams p, const uint8_t* __restrict__ code,
                                              const uint8_t* __restrict__ var, const Variant* __restrict__ vt,
                                              const double* __restrict__ Pp, const double* __restrict__ Pq,
                                              const double* __restrict__ Pr, const double* __restrict__ phi,
                                              double* Pp_out, double* Pq_out, double* Pr_out,
                                              double* fbp, double* fbq, double* fbr,
                                              const double* Pp_old, const double* Pq_old, const double* Pr_old,
                                              const int* __restrict__ skip) {
    pdl_entry();
    if (skip && *skip) return;   // a step graph whose ComputePhi_Rho failed
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + p.fe_k0;   // the launch covers planes fe_k0 .. fe_k1
    if (i >= p.nx || j >= p.ny) return;
    const size_t c = cidx(p, i, j, k);
    const int m = mcode(code, p, i, j, k);
    // Gamma = 0 outside FE (Initialization.cpp:113, :125) and the t-phase
    // zeroing (TotalEnergyDensity.cpp:123-127) leave P unchanged there: both
    // ping-pong buffers already hold it (every write of P from the host fills
    // both), and the predictor's f buffer is zero there from its allocation
    if ((m & 3) != 0 || (m & 4) != 0) return;
    const double pr0 = Pr[c];
    const double pp0 = SCALAR ? 0.0 : Pp[c];
    const double pq0 = SCALAR ? 0.0 : Pq[c];
    T R[9] = {T(1), T(0), T(0), T(0), T(1), T(0), T(0), T(0), T(1)};
    T alpha = T(p.alpha);
    if (ROT) {
        const Variant& v = vt[__ldg(var + c)];
        for (int q = 0; q < 9; ++q) R[q] = T(v.R[q]);
        alpha = T(v.alpha);
    }
    const T Gam = T(p.BigGamma);
    // the gradient terms, through the interior views where the cell's whole
    // stencil is ferroelectric
    T g_r = T(0), g_p = T(0), g_q = T(0);
    if (p.incl_G) {
        if (p.interior && __ldg(p.interior + c))
            grad_terms<T, SCALAR, ROT>(p, R, MInterior{}, PViewIn<T>{Pp, &p}, PViewIn<T>{Pq, &p}, PViewIn<T>{Pr, &p},
                                       i, j, k, g_r, g_p, g_q);
        else
            grad_terms<T, SCALAR, ROT>(p, R, MView{code, &p}, PView<T>{Pp, &p}, PView<T>{Pq, &p}, PView<T>{Pr, &p},
                                       i, j, k, g_r, g_p, g_q);
    }

    // electric field from phi, ElectrostaticSolver.cpp:195-197
    T gx = T(0), gy = T(0), gz = T(0);
    if (p.incl_E) grad_phi<T>(phi, p, i, j, k, gx, gy, gz);

    // ---- r component
    const T r = T(pr0), pp = T(pp0), pq = T(pq0);
    T fr = T(0);
    if (p.incl_L) fr += T(-1.0) * Gam * landau<T>(p, alpha, r, pp, pq);
    if (p.incl_G) fr += T(-1.0) * Gam * g_r;
    if (p.incl_E) {
        const T Er = -(R[6] * gx + R[7] * gy + R[8] * gz);
        fr += T(-1.0) * Gam * (-Er);
    }
    if (MODE == 0) Pr_out[c] = 1.0 * pr0 + p.dt * (double)fr;
    if (MODE == 1) { fbr[c] = (double)fr; Pr_out[c] = 1.0 * pr0 + p.dt * (double)fr; }
    if (MODE == 2) Pr_out[c] = 1.0 * Pr_old[c] + p.dt * (0.5 * fbr[c] + 0.5 * (double)fr);

    if (!SCALAR) {
        T fp = T(0), fq = T(0);
        if (p.incl_L) {
            fp += T(-1.0) * Gam * landau<T>(p, alpha, pp, pq, r);
            fq += T(-1.0) * Gam * landau<T>(p, alpha, pq, pp, r);
        }
        if (p.incl_G) {
            fp += T(-1.0) * Gam * g_p;
            fq += T(-1.0) * Gam * g_q;
        }
        if (p.incl_E) {
            const T Ep = -(R[0] * gx + R[1] * gy + R[2] * gz);
            const T Eq = -(R[3] * gx + R[4] * gy + R[5] * gz);
            fp += T(-1.0) * Gam * (-Ep);
            fq += T(-1.0) * Gam * (-Eq);
        }
        if (p.scalar) { fp = T(0); fq = T(0); }
        if (MODE == 0) {
            Pp_out[c] = 1.0 * pp0 + p.dt * (double)fp;
            Pq_out[c] = 1.0 * pq0 + p.dt * (double)fq;
        }
        if (MODE == 1) {
            fbp[c] = (double)fp; fbq[c] = (double)fq;
            Pp_out[c] = 1.0 * pp0 + p.dt * (double)fp;
            Pq_out[c] = 1.0 * pq0 + p.dt * (double)fq;
        }
        if (MODE == 2) {
            const double op = Pp_old[c], oq = Pq_old[c];
            Pp_out[c] = 1.0 * op + p.dt * (0.5 * fbp[c] + 0.5 * (double)fp);
            Pq_out[c] = 1.0 * oq + p.dt * (0.5 * fbq[c] + 0.5 * (double)fq);
        }
    }
}

// R_z . grad Pz with every rounding fixed
__device__ __forceinline__ double rhs_r3(double r6, double r7, double r8, double d0, double d1, double d2) {
    return fma_rn(r8, d2, fma_rn(r7, d1, mul_rn(r6, d0)));
}

// -sum_ab R_ab dP_a/dx_b at a ferroelectric cell, ElectrostaticSolver.cpp:65-77
template <bool SCALAR, typename MV, typename PV>
__device__ __forceinline__ double rhs_fe(const double* R, const MV& M, const PV& Fp, const PV& Fq, const PV& Fr,
                                         int i, int j, int k) {
    if (SCALAR) {
        // roundings written out, shared with the row-segment kernel (k_rhs_p_seg)
        return -rhs_r3(R[6], R[7], R[8], dpd<0, double>(Fr, M, i, j, k), dpd<1, double>(Fr, M, i, j, k),
                       dpd<2, double>(Fr, M, i, j, k));
    }
    const double r3 = R[6] * dpd<0, double>(Fr, M, i, j, k) + R[7] * dpd<1, double>(Fr, M, i, j, k) + R[8] * dpd<2, double>(Fr, M, i, j, k);
    const double r1 = R[0] * dpd<0, double>(Fp, M, i, j, k) + R[1] * dpd<1, double>(Fp, M, i, j, k) + R[2] * dpd<2, double>(Fp, M, i, j, k);
    const double r2 = R[3] * dpd<0, double>(Fq, M, i, j, k) + R[4] * dpd<1, double>(Fq, M, i, j, k) + R[5] * dpd<2, double>(Fq, M, i, j, k);
    return -(r1) - (r2) - (r3);
}

// FE branch of ComputePoissonRHS, ElectrostaticSolver.cpp:65-77 (DE -> 0; the
// SC value rho is supplied by k_newton).  Also reduces max|rhs| and max|b'|
// where b' adds the Dirichlet electrode terms (the MLMG stopping rule's norms)
template <bool SCALAR, bool ROT>
__global__ void __launch_bounds__(256) k_rhs_p(DevParams p, const uint8_t* __restrict__ code,
                                               const uint8_t* __restrict__ var, const Variant* __restrict__ vt,
                                               const double* __restrict__ Pp, const double* __restrict__ Pq,
                                               const double* __restrict__ Pr, double* __restrict__ rhs,
                                               double* __restrict__ norms) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    __shared__ double sh[32];
    double nb = 0.0, nbp = 0.0;
    if (i < p.nx && j < p.ny) {
        const size_t c = cidx(p, i, j, k);
        const int m = mcode(code, p, i, j, k);
        double v = 0.0;
        if ((m & 3) == 0) {
            double R[9] = {1, 0, 0, 0, 1, 0, -0.0, 0, 1};
            if (ROT) {
                const Variant& vv = vt[__ldg(var + c)];
                for (int q = 0; q < 9; ++q) R[q] = vv.R[q];
            }
            // through the interior views where the cell's whole stencil is
            // ferroelectric (same arithmetic, no mask tests)
            if (p.interior && __ldg(p.interior + c))
                v = rhs_fe<SCALAR>(R, MInterior{}, PViewIn<double>{Pp, &p}, PViewIn<double>{Pq, &p},
                                   PViewIn<double>{Pr, &p}, i, j, k);
            else
                v = rhs_fe<SCALAR>(R, MView{code, &p}, PView<double>{Pp, &p}, PView<double>{Pq, &p},
                                   PView<double>{Pr, &p}, i, j, k);
        }
        rhs[c] = v;
        if ((long long)c < p.Ns) {   // the norms cover the cells of the solve
            nb = fabs(v);
            double bp = v;
            const double e = p.eps[m & 7];
            if (k == 0) bp += 2.0 * e * p.ih2[2] * p.V_lo;
            if ((long long)c >= p.Ns - p.nxy) bp += 2.0 * e * p.ih2[2] * p.Vs_hi;
            nbp = fabs(bp);
        }
    }
    if (norms) {
        const double a = block_max(nb, sh);
        const double b = block_max(nbp, sh);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            atomic_max_nonneg(norms, a);
            atomic_max_nonneg(norms + 1, b);
        }
    }
}

// k_rhs_p for scalar P by row segments: 4 cells of a row per thread.  Where
// all 4 are interior cells (the whole stencil ferroelectric) the central
// forms run on the segment's rows loaded once (two 16-byte loads per row);
// otherwise each cell takes k_rhs_p's own path.  Same operations per cell,
// so the same bits.
template <bool ROT>
__global__ void __launch_bounds__(256) k_rhs_p_seg(DevParams p, const uint8_t* __restrict__ code,
                                                   const uint8_t* __restrict__ var, const Variant* __restrict__ vt,
                                                   const double* __restrict__ Pr, double* __restrict__ rhs,
                                                   double* __restrict__ norms) {
    pdl_entry();
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    __shared__ double sh[32];
    double nb = 0.0, nbp = 0.0;
    if (j < p.ny) {
        const size_t c0 = cidx(p, i0, j, k);
        const unsigned cw = __ldg(reinterpret_cast<const unsigned*>(code + c0 + p.nxy));
        const unsigned iw = p.interior ? __ldg(reinterpret_cast<const unsigned*>(p.interior + c0)) : 0u;
        double v[4];
        bool fast = true;
#pragma unroll
        for (int m = 0; m < 4; ++m) fast = fast && ((iw >> (8 * m)) & 0xffu) != 0u && ((cw >> (8 * m)) & 3u) == 0u;
        if (fast) {
            const int jm = j == 0 ? p.ny - 1 : j - 1, jp = j == p.ny - 1 ? 0 : j + 1;
            const int il = i0 == 0 ? p.nx - 1 : i0 - 1, ir = i0 + 4 == p.nx ? 0 : i0 + 4;
            const size_t row = c0 - i0;
            double xc[4], xs[4], xn[4], xb[4], xt[4];
            auto ld4 = [](const double* q, double (&a)[4]) {
                const double2 u = __ldg(reinterpret_cast<const double2*>(q));
                const double2 w = __ldg(reinterpret_cast<const double2*>(q) + 1);
                a[0] = u.x; a[1] = u.y; a[2] = w.x; a[3] = w.y;
            };
            ld4(Pr + c0, xc);
            ld4(Pr + cidx(p, i0, jm, k), xs);
            ld4(Pr + cidx(p, i0, jp, k), xn);
            ld4(Pr + c0 - p.nxy, xb);   // interior cells are off the z faces
            ld4(Pr + c0 + p.nxy, xt);
            const double xl = __ldg(Pr + row + il), xr = __ldg(Pr + row + ir);
            const double hx = p.dx[0], hy = p.dx[1], hz = p.dx[2];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                double r6 = -0.0, r7 = 0.0, r8 = 1.0;
                if (ROT) {
                    const Variant& vv = vt[__ldg(var + c0 + m)];
                    r6 = vv.R[6]; r7 = vv.R[7]; r8 = vv.R[8];
                }
                const double d0 = ((m == 3 ? xr : xc[m + 1]) - (m == 0 ? xl : xc[m - 1])) / (2. * hx);
                const double d1 = (xn[m] - xs[m]) / (2. * hy);
                const double d2 = (xt[m] - xb[m]) / (2. * hz);
                v[m] = -rhs_r3(r6, r7, r8, d0, d1, d2);
            }
        } else {
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int i = i0 + m;
                v[m] = 0.0;
                if (((cw >> (8 * m)) & 3u) == 0u) {
                    double R[9] = {1, 0, 0, 0, 1, 0, -0.0, 0, 1};
                    if (ROT) {
                        const Variant& vv = vt[__ldg(var + c0 + m)];
                        for (int q = 0; q < 9; ++q) R[q] = vv.R[q];
                    }
                    if (p.interior && ((iw >> (8 * m)) & 0xffu))
                        v[m] = rhs_fe<true>(R, MInterior{}, PViewIn<double>{Pr, &p}, PViewIn<double>{Pr, &p},
                                            PViewIn<double>{Pr, &p}, i, j, k);
                    else
                        v[m] = rhs_fe<true>(R, MView{code, &p}, PView<double>{Pr, &p}, PView<double>{Pr, &p},
                                            PView<double>{Pr, &p}, i, j, k);
                }
            }
        }
        *reinterpret_cast<double2*>(rhs + c0) = make_double2(v[0], v[1]);
        *(reinterpret_cast<double2*>(rhs + c0) + 1) = make_double2(v[2], v[3]);
        if ((long long)c0 < p.Ns) {   // the norms cover the cells of the solve
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                nb = fmax(nb, fabs(v[m]));
                double bp = v[m];
                const double e = p.eps[(cw >> (8 * m)) & 7u];
                if (k == 0) bp += 2.0 * e * p.ih2[2] * p.V_lo;
                if ((long long)c0 >= p.Ns - p.nxy) bp += 2.0 * e * p.ih2[2] * p.Vs_hi;
                nbp = fmax(nbp, fabs(bp));
            }
        }
    }
    if (norms) {
        const double a = block_max(nb, sh);
        const double b = block_max(nbp, sh);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            atomic_max_nonneg(norms, a);
            atomic_max_nonneg(norms + 1, b);
        }
    }
}

// one Newton linearisation pass (FP64): alpha = (rho(phi+delta) - rho)/delta
// by the reference's LinComb, rhs = RHS - alpha phi; alpha is also written in
// FP32 for the mixed-precision multigrid.  One cell's arithmetic:
__device__ __forceinline__ void newton_cell(const DevParams& p, const double* seps, int m, double ph, double r0,
                                            double rp, long long c, double& a, double& v, double& bp) {
    const int mask = m & 3;
    a = 0.0;
    if (mask >= 2) {
        double e, h;
        const double rho_pd = sc_charge(p, ph + p.delta, e, h);
        a = p.inv_delta * rho_pd + p.neg_inv_delta * r0;
        v = r0 - a * ph;
    } else if (mask == 1) {
        v = 0.0;
    } else {
        v = rp;
    }
    bp = v;
    if (c < p.nxy) bp += 2.0 * seps[m & 7] * p.ih2[2] * p.V_lo;             // k == 0
    if (c >= p.Ns - p.nxy) bp += 2.0 * seps[m & 7] * p.ih2[2] * p.Vs_hi;    // the solve's top layer
}

// PAIR: each thread takes two neighbouring cells with vector loads and
// stores, every load issued before the arithmetic (N and nx ny even); the
// charge arithmetic is latency bound, so the loads of both cells overlap it
template <bool PAIR>
__global__ void __launch_bounds__(256) k_newton(DevParams p, const uint8_t* __restrict__ code,
                                                const double* __restrict__ phi, const double* __restrict__ rho,
                                                const double* __restrict__ rhs_p, double* __restrict__ alpha,
                                                float* __restrict__ alpha32, double* __restrict__ rhs,
                                                double* __restrict__ norms) {
    pdl_entry();
    __shared__ double sh[32];
    __shared__ double seps[8];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    if (tid == 0)
#pragma unroll
        for (int q = 0; q < 8; ++q) seps[q] = p.eps[q];
    __syncthreads();
    double nb = 0.0, nbp = 0.0;
    if (PAIR) {
        const long long np = p.N / 2;
        for (long long q = (long long)blockIdx.x * 256 + tid; q < np; q += (long long)gridDim.x * 256) {
            const long long c = 2 * q;
            // the code array carries one z ghost layer below: cell c is at c + nxy
            const uchar2 m2 = __ldg(reinterpret_cast<const uchar2*>(code + p.nxy + c));
            const double2 ph = __ldg(reinterpret_cast<const double2*>(phi + c));
            const double2 r0 = __ldg(reinterpret_cast<const double2*>(rho + c));
            const double2 rp = __ldg(reinterpret_cast<const double2*>(rhs_p + c));
            double a0, v0, bp0, a1, v1, bp1;
            newton_cell(p, seps, m2.x, ph.x, r0.x, rp.x, c, a0, v0, bp0);
            newton_cell(p, seps, m2.y, ph.y, r0.y, rp.y, c + 1, a1, v1, bp1);
            *reinterpret_cast<double2*>(alpha + c) = make_double2(a0, a1);
            *reinterpret_cast<float2*>(alpha32 + c) = make_float2((float)a0, (float)a1);
            *reinterpret_cast<double2*>(rhs + c) = make_double2(v0, v1);
            if (c < p.Ns) {   // the norms cover the cells of the solve (Ns, nxy even)
                nb = fmax(nb, fmax(fabs(v0), fabs(v1)));
                nbp = fmax(nbp, fmax(fabs(bp0), fabs(bp1)));
            }
        }
    } else {
        for (long long c = (long long)blockIdx.x * 256 + tid; c < p.N; c += (long long)gridDim.x * 256) {
            const int m = __ldg(code + c + p.nxy);
            double a, v, bp;
            newton_cell(p, seps, m, phi[c], rho[c], rhs_p[c], c, a, v, bp);
            alpha[c] = a;
            alpha32[c] = (float)a;
            rhs[c] = v;
            if (c < p.Ns) {
                nb = fmax(nb, fabs(v));
                nbp = fmax(nbp, fabs(bp));
            }
        }
    }
    const double x = block_max(nb, sh);
    const double y = block_max(nbp, sh);
    if (tid == 0) {
        atomic_max_nonneg(norms, x);
        atomic_max_nonneg(norms + 1, y);
    }
}

// ComputeRho at the new phi + the Newton error norms; partial sums go to
// part[2*block], the last block folds them in block order (deterministic)
template <bool PAIR>
__global__ void __launch_bounds__(256) k_rho(DevParams p, const uint8_t* __restrict__ code,
                                             const double* __restrict__ phi, double* __restrict__ phi_prev,
                                             double* __restrict__ rho, double* __restrict__ e_den,
                                             double* __restrict__ h_den, double* __restrict__ part,
                                             unsigned int* __restrict__ counter, double* __restrict__ out,
                                             int track, int carriers, RhoCtl rc) {
    pdl_entry();
    __shared__ double sh[32];
    __shared__ bool last;
    double s1 = 0.0, s2 = 0.0;
    if (PAIR) {
        // two neighbouring cells per thread with vector loads and stores,
        // every load issued before the exponentials (N and nx ny even)
        const long long np = p.N / 2;
        for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < np; q += (long long)gridDim.x * blockDim.x) {
            const long long c = 2 * q;
            const uchar2 m2 = __ldg(reinterpret_cast<const uchar2*>(code + p.nxy + c));   // one z ghost layer below
            const double2 ph = __ldg(reinterpret_cast<const double2*>(phi + c));
            const double2 pp = track ? *reinterpret_cast<const double2*>(phi_prev + c) : make_double2(0.0, 0.0);
            double e0 = 0.0, h0 = 0.0, e1 = 0.0, h1 = 0.0;
            const bool sc0 = (m2.x & 3) >= 2, sc1 = (m2.y & 3) >= 2;
            const double r0 = sc0 ? sc_charge(p, ph.x, e0, h0) : 0.0;
            const double r1 = sc1 ? sc_charge(p, ph.y, e1, h1) : 0.0;
            *reinterpret_cast<double2*>(rho + c) = make_double2(r0, r1);
            if (carriers) {
                if (sc0) { e_den[c] = e0; h_den[c] = h0; }
                if (sc1) { e_den[c + 1] = e1; h_den[c + 1] = h1; }
            }
            if (track) {
                s1 += fabs(ph.x - pp.x);
                s2 += fabs(ph.x);
                s1 += fabs(ph.y - pp.y);
                s2 += fabs(ph.y);
                *reinterpret_cast<double2*>(phi_prev + c) = ph;
            }
        }
    } else {
        for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < p.N; c += (long long)gridDim.x * blockDim.x) {
            const int m = __ldg(code + c + p.nxy) & 3;   // code has one z ghost layer below
            const double ph = phi[c];
            const double pp = track ? phi_prev[c] : 0.0;
            if (m >= 2) {
                double e, h;
                rho[c] = sc_charge(p, ph, e, h);
                if (carriers) {
                    e_den[c] = e;
                    h_den[c] = h;
                }
            } else {
                rho[c] = 0.0;
            }
            if (track) {
                s1 += fabs(ph - pp);
                s2 += fabs(ph);
                phi_prev[c] = ph;
            }
        }
    }
    if (!track) return;
    const double b1 = block_sum(s1, sh);
    const double b2 = block_sum(s2, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = b1;
        part[2 * blockIdx.x + 1] = b2;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        // fold the block partials with the whole block, in a fixed order
        __threadfence();
        double t1 = 0.0, t2 = 0.0;
        for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
            t1 += ((volatile double*)part)[2 * b];
            t2 += ((volatile double*)part)[2 * b + 1];
        }
        t1 = block_sum(t1, sh);
        t2 = block_sum(t2, sh);
        if (threadIdx.x == 0) {
            if (rc.ctl) {
                // a step graph: close the solve, test the Newton loop, and
                // leave out[] zeroed for the next linearisation's norms
                if (rc.mg_end) ctl_mg_end(rc.ctl);
                ctl_newton(rc.ctl, t1, t2, rc.tol, rc.max_iter, rc.h, rc.in_body);
                out[0] = 0.0;
                out[1] = 0.0;
            } else {
                out[0] = t1;
                out[1] = t2;
            }
            *counter = 0;
        }
    }
}

// CheckSteadyState: max|phi|, max|phi - phi_old| over valid cells, then
// phi_old := phi; optionally keeps |phi - phi_old| for the PhiDiff output
__global__ void __launch_bounds__(256) k_steady(DevParams p, const double* __restrict__ phi,
                                                double* __restrict__ phi_old, double* __restrict__ dphi,
                                                double* __restrict__ out, const int* __restrict__ skip) {
    pdl_entry();
    if (skip && *skip) return;
    __shared__ double sh[32];
    double m1 = 0.0, m2 = 0.0;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < p.N; c += (long long)gridDim.x * blockDim.x) {
        const double a = phi[c];
        const double d = fabs(a - phi_old[c]);
        if (dphi) dphi[c] = d;
        phi_old[c] = a;
        const double fa = fabs(a);
        if (fa == fa) m1 = fmax(m1, fa);
        if (d == d) m2 = fmax(m2, d);
    }
    const double x = block_max(m1, sh);
    const double y = block_max(m2, sh);
    if (threadIdx.x == 0) {
        atomic_max_nonneg(out, x);
        atomic_max_nonneg(out + 1, y);
    }
}

// mean of Px, Py, Pz over the ferroelectric cells (mask 0): the hysteresis
// observable; partial sums per block, folded in block order by the last block
__global__ void __launch_bounds__(256) k_mean_p(DevParams p, const uint8_t* __restrict__ code,
                                                const double* __restrict__ Px, const double* __restrict__ Py,
                                                const double* __restrict__ Pz, double* __restrict__ part,
                                                unsigned int* __restrict__ counter, double* __restrict__ out) {
    pdl_entry();
    __shared__ double sh[32];
    __shared__ bool last;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < p.N; c += (long long)gridDim.x * blockDim.x) {
        if ((__ldg(code + c + p.nxy) & 3) == 0) {
            if (Px) s[0] += Px[c];
            if (Py) s[1] += Py[c];
            s[2] += Pz[c];
            s[3] += 1.0;
        }
    }
    double b[4];
    for (int q = 0; q < 4; ++q) b[q] = block_sum(s[q], sh);
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; ++q) part[4 * blockIdx.x + q] = b[q];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (unsigned blk = threadIdx.x; blk < gridDim.x; blk += blockDim.x)
            for (int q = 0; q < 4; ++q) t[q] += ((volatile double*)part)[4 * blk + q];
        for (int q = 0; q < 4; ++q) t[q] = block_sum(t[q], sh);
        if (threadIdx.x == 0) {
            for (int q = 0; q < 3; ++q) out[q] = t[3] > 0 ? t[q] / t[3] : 0.0;
            *counter = 0;
        }
    }
}

template <bool ROT>
__global__ void __launch_bounds__(256) k_efield(DevParams p, const uint8_t* __restrict__ var,
                                                const Variant* __restrict__ vt, const double* __restrict__ phi,
                                                double* __restrict__ Ex, double* __restrict__ Ey,
                                                double* __restrict__ Ez) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= p.nx || j >= p.ny) return;
    const size_t c = cidx(p, i, j, k);
    double R[9] = {1, 0, 0, 0, 1, 0, -0.0, 0, 1};
    if (ROT) {
        const Variant& v = vt[__ldg(var + c)];
        for (int q = 0; q < 9; ++q) R[q] = v.R[q];
    }
    double gx, gy, gz;
    grad_phi<double>(phi, p, i, j, k, gx, gy, gz);
    Ex[c] = -(R[0] * gx + R[1] * gy + R[2] * gz);
    Ey[c] = -(R[3] * gx + R[4] * gy + R[5] * gz);
    Ez[c] = -(R[6] * gx + R[7] * gy + R[8] * gz);
}

dim3 cell_grid(const DevParams& p) { return dim3((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz); }

}  // namespace

// ------------------------------------------------------------ launchers --
int launch_tdgl(const DevParams& p, int mixed, int mode, const uint8_t* code, const uint8_t* var, const Variant* vt,
                const double* const Pin[3], double* const Pout[3], const double* phi, double* const fbuf[3],
                const double* const Pold[3], cudaStream_t s, const int* skip) {
    dim3 g = cell_grid(p);
    const dim3 b(32, 8);
    g.z = (unsigned)(p.fe_k1 - p.fe_k0 + 1);
    const bool scal = p.scalar && Pin[0] == nullptr;
    const bool rot = var != nullptr;
    double* fb[3] = {fbuf ? fbuf[0] : nullptr, fbuf ? fbuf[1] : nullptr, fbuf ? fbuf[2] : nullptr};
    const double* po[3] = {Pold ? Pold[0] : nullptr, Pold ? Pold[1] : nullptr, Pold ? Pold[2] : nullptr};
#define FX_TDGL(T, S, R, M) launch_k(k_tdgl<T, S, R, M>, g, b, 0, s, p, code, var, vt, Pin[0], Pin[1], Pin[2], phi, Pout[0], Pout[1], Pout[2], fb[0], fb[1], fb[2], po[0], po[1], po[2], skip)
#define FX_TDGL_M(T, S, R) do { if (mode == 0) FX_TDGL(T, S, R, 0); else if (mode == 1) FX_TDGL(T, S, R, 1); else FX_TDGL(T, S, R, 2); } while (0)
    if (!mixed) {
        if (scal) { if (rot) FX_TDGL_M(double, true, true); else FX_TDGL_M(double, true, false); }
        else { if (rot) FX_TDGL_M(double, false, true); else FX_TDGL_M(double, false, false); }
    } else {
        if (scal) { if (rot) FX_TDGL_M(float, true, true); else FX_TDGL_M(float, true, false); }
        else { if (rot) FX_TDGL_M(float, false, true); else FX_TDGL_M(float, false, false); }
    }
#undef FX_TDGL_M
#undef FX_TDGL
    return (int)cudaGetLastError();
}

int launch_rhs_p(const DevParams& p, const uint8_t* code, const uint8_t* var, const Variant* vt,
                 const double* const P[3], double* rhs, double* norms, cudaStream_t s) {
    const dim3 g = cell_grid(p), b(32, 8);
    const bool scal = p.scalar && P[0] == nullptr;
    const bool rot = var != nullptr;
    const int gx = p.nx / 4;
    auto al = [](const void* q, uintptr_t a) { return ((uintptr_t)q % a) == 0; };
    if (scal && g_rhs_seg && p.nx % 4 == 0 && (gx % 32 == 0 || 32 % gx == 0) && al(P[2], 16) && al(rhs, 16) &&
        al(code + p.nxy, 4) && (!p.interior || al(p.interior, 4))) {
        // 4 cells of a row per thread
        const int bx = gx < 32 ? gx : 32, by = 256 / bx;
        const dim3 bs(bx, by), gs(gx / bx, (p.ny + by - 1) / by, p.nz);
        if (rot) launch_k(k_rhs_p_seg<true>, gs, bs, 0, s, p, code, var, vt, P[2], rhs, norms);
        else launch_k(k_rhs_p_seg<false>, gs, bs, 0, s, p, code, var, vt, P[2], rhs, norms);
        return (int)cudaGetLastError();
    }
    if (scal) {
        if (rot) launch_k(k_rhs_p<true, true>, g, b, 0, s, p, code, var, vt, P[0], P[1], P[2], rhs, norms);
        else launch_k(k_rhs_p<true, false>, g, b, 0, s, p, code, var, vt, P[0], P[1], P[2], rhs, norms);
    } else {
        if (rot) launch_k(k_rhs_p<false, true>, g, b, 0, s, p, code, var, vt, P[0], P[1], P[2], rhs, norms);
        else launch_k(k_rhs_p<false, false>, g, b, 0, s, p, code, var, vt, P[0], P[1], P[2], rhs, norms);
    }
    return (int)cudaGetLastError();
}

// the paired kernels need whole cell pairs that start on an even cell of
// every array, the code array included (offset nx ny)
static bool pairs_ok(const DevParams& p) { return p.N % 2 == 0 && p.nxy % 2 == 0; }

int launch_newton(const DevParams& p, const uint8_t* code, const double* phi, const double* rho,
                  const double* rhs_p, double* alpha, float* alpha32, double* rhs, double* norms, cudaStream_t s) {
    if (pairs_ok(p)) launch_k(k_newton<true>, p.ngrid_red, dim3(256), 0, s, p, code, phi, rho, rhs_p, alpha, alpha32, rhs, norms);
    else launch_k(k_newton<false>, p.ngrid_red, dim3(256), 0, s, p, code, phi, rho, rhs_p, alpha, alpha32, rhs, norms);
    return (int)cudaGetLastError();
}

int launch_rho(const DevParams& p, const uint8_t* code, const double* phi, double* phi_prev, double* rho,
               double* e_den, double* h_den, double* part, unsigned int* counter, double* out, int track,
               int carriers, cudaStream_t s, const RhoCtl* rc) {
    RhoCtl none = {};
    if (pairs_ok(p))
        launch_k(k_rho<true>, p.ngrid_red, RED_THREADS, 0, s, p, code, phi, phi_prev, rho, e_den, h_den, part, counter,
                 out, track, carriers, rc ? *rc : none);
    else
        launch_k(k_rho<false>, p.ngrid_red, RED_THREADS, 0, s, p, code, phi, phi_prev, rho, e_den, h_den, part, counter,
                 out, track, carriers, rc ? *rc : none);
    return (int)cudaGetLastError();
}

namespace {

__global__ void k_ctl_step_begin(StepCtl* ctl, double* out) {
    pdl_entry();
    // the norm accumulators of the first linearisation (or of ComputePoissonRHS)
    out[0] = 0.0;
    out[1] = 0.0;
    ctl->steady[0] = 0.0;
    ctl->steady[1] = 0.0;
    ctl->mg_cycles_step = 0;
    ctl->newton_passes_step = 0;
    ctl->status = CTL_OK;
    ctl->status_n = 0;
    ctl->status_val = 0.0;
    ctl->status_target = 0.0;
    for (int k = 0; k < KIND_N; ++k) ctl->nexec[k] = 0;
    // and the step's first ComputePhi_Rho begins
    ctl->passes = 0;
    ctl->iter = 0;
    ctl->err = 1.0;
    ctl->mg_cycles_phirho = 0;
}

__global__ void k_ctl_phirho_begin(StepCtl* ctl, double* out) {
    pdl_entry();
    out[0] = 0.0;
    out[1] = 0.0;
    ctl->passes = 0;
    ctl->iter = 0;
    ctl->err = 1.0;
    ctl->mg_cycles_phirho = 0;
}

// without a semiconductor ComputePhi_Rho is one solve, counted as one pass
// (gate != 0: also opens the IF node `gate` of body `kind` while no failure
// is recorded, as k_ctl_gate)
__global__ void k_ctl_phirho_end(StepCtl* ctl, int sc, cudaGraphConditionalHandle gate, int kind) {
    pdl_entry();
    if (!sc) {
        ctl->passes = 1;
        ctl->err = 0.0;
    }
    ctl->newton_passes_step += ctl->passes;
    if (gate) {
        const bool ok = ctl->status == CTL_OK;
        if (ok) ctl->nexec[kind] += 1;
        cudaGraphSetConditional(gate, ok ? 1u : 0u);
    }
}

}  // namespace

int launch_ctl_step_begin(StepCtl* ctl, double* out, cudaStream_t s) {
    launch_k(k_ctl_step_begin, 1, 1, 0, s, ctl, out);
    return (int)cudaGetLastError();
}

int launch_ctl_phirho_begin(StepCtl* ctl, double* out, cudaStream_t s) {
    launch_k(k_ctl_phirho_begin, 1, 1, 0, s, ctl, out);
    return (int)cudaGetLastError();
}

int launch_ctl_phirho_end(StepCtl* ctl, int sc, cudaGraphConditionalHandle gate, int kind, cudaStream_t s) {
    launch_k(k_ctl_phirho_end, 1, 1, 0, s, ctl, sc, gate, kind);
    return (int)cudaGetLastError();
}

int launch_steady(const DevParams& p, const double* phi, double* phi_old, double* dphi, double* out,
                  cudaStream_t s, const int* skip) {
    launch_k(k_steady, p.ngrid_red, RED_THREADS, 0, s, p, phi, phi_old, dphi, out, skip);
    return (int)cudaGetLastError();
}

int launch_mean_p(const DevParams& p, const uint8_t* code, const double* const P[3], double* part,
                  unsigned int* counter, double* out, cudaStream_t s) {
    launch_k(k_mean_p, p.ngrid_red, RED_THREADS, 0, s, p, code, P[0], P[1], P[2], part, counter, out);
    return (int)cudaGetLastError();
}

// initial iterate of a step's first Poisson solve, extrapolated in time from
// the last steps' phi (h[0] the previous step's, h[1] the one before, ...):
// the polynomial of degree ORDER through the last ORDER + 1 steps, evaluated
// one step ahead, sum_m (-1)^m C(ORDER + 1, m + 1) phi^(n-m): order 1: 2 phi - h0;
// 2: 3 phi - 3 h0 + h1; 3: 4 phi - 6 h0 + 4 h1 - h2; 4: 5 phi - 10 h0 + 10 h1 -
// 5 h2 + h3; 5: 6, 15, 20, 15, 6, 1; 6: 7, 21, 35, 35, 21, 7, 1.  The
// histories shift by one step (the ones beyond ORDER take zeros).
struct PhiHist {
    double* h[6];   // null beyond the configured order
};

template <int ORDER>
__global__ void __launch_bounds__(256) k_phi_extrap(double* __restrict__ phi, PhiHist H, long long n) {
    pdl_entry();
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const double t = phi[c];
        double v[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) v[m] = m < ORDER ? H.h[m][c] : 0.0;
        const double a = v[0], b = v[1], d = v[2], e = v[3], f = v[4], g = v[5];
        if (ORDER == 1) phi[c] = 2.0 * t - a;
        if (ORDER == 2) phi[c] = 3.0 * t - 3.0 * a + b;
        if (ORDER == 3) phi[c] = 4.0 * t - 6.0 * a + 4.0 * b - d;
        if (ORDER == 4) phi[c] = 5.0 * t - 10.0 * a + 10.0 * b - 5.0 * d + e;
        if (ORDER == 5) phi[c] = 6.0 * t - 15.0 * a + 20.0 * b - 15.0 * d + 6.0 * e - f;
        if (ORDER == 6) phi[c] = 7.0 * t - 21.0 * a + 35.0 * b - 35.0 * d + 21.0 * e - 7.0 * f + g;
#pragma unroll
        for (int m = 5; m >= 1; --m)
            if (H.h[m]) H.h[m][c] = v[m - 1];
        H.h[0][c] = t;
    }
}

int launch_phi_extrap(const DevParams& p, int order, double* phi, double* const h[6], cudaStream_t s) {
    PhiHist H;
    for (int m = 0; m < 6; ++m) H.h[m] = h[m];
    switch (order >= 6 ? 6 : order) {
    case 6: launch_k(k_phi_extrap<6>, p.ngrid_red, RED_THREADS, 0, s, phi, H, p.N); break;
    case 5: launch_k(k_phi_extrap<5>, p.ngrid_red, RED_THREADS, 0, s, phi, H, p.N); break;
    case 4: launch_k(k_phi_extrap<4>, p.ngrid_red, RED_THREADS, 0, s, phi, H, p.N); break;
    case 3: launch_k(k_phi_extrap<3>, p.ngrid_red, RED_THREADS, 0, s, phi, H, p.N); break;
    case 2: launch_k(k_phi_extrap<2>, p.ngrid_red, RED_THREADS, 0, s, phi, H, p.N); break;
    default: launch_k(k_phi_extrap<1>, p.ngrid_red, RED_THREADS, 0, s, phi, H, p.N); break;
    }
    return (int)cudaGetLastError();
}

int launch_efield(const DevParams& p, const uint8_t* var, const Variant* vt, const double* phi, double* E[3],
                  cudaStream_t s) {
    const dim3 g = cell_grid(p), b(32, 8);
    if (var) launch_k(k_efield<true>, g, b, 0, s, p, var, vt, phi, E[0], E[1], E[2]);
    else launch_k(k_efield<false>, g, b, 0, s, p, var, vt, phi, E[0], E[1], E[2]);
    return (int)cudaGetLastError();
}

}  // namespace fx
