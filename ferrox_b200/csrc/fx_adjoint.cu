// fx_adjoint.cu -- reverse-mode kernels of the coupled time step, for the
// gradient of a polarization loss with respect to the Landau and gradient
// coefficients and the applied voltage.  The reference has no
// differentiation; these kernels transpose the forward step of
// fx_kernels.cu / fx_mg.cu exactly.
//
// Forward step n (Order 1):
//     phi^n = Phi(P^{n-1}, V_n)      solves F = A0 phi - bcv(V) - s(P) - rho(phi) = 0
//     P^n   = P^{n-1} + dt f(P^{n-1}, phi^n)
// with A0 = -div(eps grad) (the multigrid operator, symmetric), s(P) the FE
// right-hand side -div P (k_rhs_p) and rho the semiconductor charge.  With
// lambda^n = dL/dP^n one reverse step is
//     mu          = dt (df/dphi)^T lambda^n                          k_adj_phi
//     psi         : (A0 - diag(rho'(phi^n))) psi = mu, V = 0          the same multigrid
//     lambda^{n-1} = dL_{n-1}/dP + lambda^n + dt (df/dP)^T lambda^n
//                    + (ds/dP)^T psi                                  k_adj_P
//     dL/dV_n    += dt (df/dV)^T lambda^n + (dbcv/dV)^T psi
//     dL/dtheta  += dt lambda^n . df/dtheta  (theta = alpha, beta, gamma, g11, g44)
// The implicit-function form of the phi adjoint holds at a converged solve;
// rho' is the analytic derivative (the forward Newton's finite-difference
// slope only changes how fast phi converges, not phi itself).
//
// Transposed stencils: the forward stencil functions are linear in the field
// they read, so row c's coefficient of cell c' is the stencil at c evaluated
// on a unit impulse at c' (DeltaView, PhiDelta).  Every mask branch and
// boundary form of the forward is transposed that way without restating it.
#include "fx_kernels.h"

#include <cmath>
#include <utility>

namespace fx {

// which stencils evaluated at a cell c can read the cell c + (DI, DJ, DK):
// a second derivative along an axis reads up to two cells along it, a mixed
// one the first-derivative stencil (one cell along its axis) one cell to
// either side, a first derivative one cell along its axis
template <int DI, int DJ, int DK>
struct Reach {
    static constexpr bool xx = DJ == 0 && DK == 0;
    static constexpr bool yy = DI == 0 && DK == 0;
    static constexpr bool zz = DI == 0 && DJ == 0;
    static constexpr bool xy = (DI == 1 || DI == -1) && DK == 0;
    static constexpr bool xz = (DI == 1 || DI == -1) && DJ == 0;
    static constexpr bool yz = (DJ == 1 || DJ == -1) && DI == 0;
    static constexpr bool dx = DJ == 0 && DK == 0 && DI >= -1 && DI <= 1;
    static constexpr bool dy = DI == 0 && DK == 0 && DJ >= -1 && DJ <= 1;
    static constexpr bool dz = DI == 0 && DJ == 0 && DK >= -1 && DK <= 1;
    static constexpr bool gx = (DI == 1 || DI == -1) && DJ == 0 && DK == 0;   // central phi differences
    static constexpr bool gy = (DJ == 1 || DJ == -1) && DI == 0 && DK == 0;
    static constexpr bool gz = DI == 0 && DJ == 0;
};

namespace {

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block sum over a 2-D block (result valid in thread 0)
__device__ double block_sum2(double v, double* sh) {
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    const int nthr = blockDim.x * blockDim.y;
    v = warp_sum_d(v);
    if ((t & 31) == 0) sh[t >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (t < 32) {
        r = t < (nthr >> 5) ? sh[t] : 0.0;
        r = warp_sum_d(r);
    }
    __syncthreads();
    return r;
}

__device__ double block_max2(double v, double* sh) {
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    const int nthr = blockDim.x * blockDim.y;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((t & 31) == 0) sh[t >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (t < 32) {
        r = t < (nthr >> 5) ? sh[t] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    return r;
}

__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
    if (!(v == v)) v = __longlong_as_double(0x7ff0000000000000LL);
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// derivative of phi_at(i, j, k) with respect to the top electrode value V_hi
struct VDelta {
    const DevParams* p;
    __device__ __forceinline__ double operator()(int, int, int k) const {
        if (k < p->nz) return 0.0;
        return p->ghost_mode == 0 ? 2.0 : (p->ghost_mode == 1 ? 1.0 : 0.0);
    }
};

// TDGL-updated cell: ferroelectric and not t-phase (elsewhere f = 0)
__device__ __forceinline__ bool updated(int m) { return (m & 3) == 0 && (m & 4) == 0; }

template <typename T, bool ROT>
__device__ __forceinline__ void load_R(const uint8_t* __restrict__ var, const Variant* __restrict__ vt, size_t c, T* R,
                                       T& alpha, const DevParams& p) {
    if (ROT) {
        const Variant& v = vt[__ldg(var + c)];
#pragma unroll
        for (int q = 0; q < 9; ++q) R[q] = T(v.R[q]);
        alpha = T(v.alpha);
    } else {
#pragma unroll
        for (int q = 0; q < 9; ++q) R[q] = T(q % 4 == 0 ? 1 : 0);
        alpha = T(p.alpha);
    }
}

// adjoint weights of the rows of cell c: lambda_a for the components whose
// f is non-zero there (Px, Py are frozen when is_polarization_scalar = 1)
template <typename T, bool VEC>
__device__ __forceinline__ void load_lam(const DevParams& p, const double* __restrict__ lp, const double* __restrict__ lq,
                                         const double* __restrict__ lr, size_t c, T lam[3]) {
    lam[2] = T(lr[c]);
    if (VEC && !p.scalar) {
        lam[0] = T(lp[c]);
        lam[1] = T(lq[c]);
    } else {
        lam[0] = lam[1] = T(0);
    }
}

// offsets (di, dj, dk) of the cells whose TDGL stencil reads a given cell:
// the 13 axis offsets up to 2 (second derivatives, incl. the one-sided
// forms), then the 12 plane diagonals (mixed derivatives)
constexpr int kOff[25][3] = {
    {0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {2, 0, 0},  {-2, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 2, 0},  {0, -2, 0},
    {0, 0, 1},  {0, 0, -1}, {0, 0, 2},  {0, 0, -2}, {1, 1, 0},  {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1},
    {1, 0, -1}, {-1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};

// sum_a lambda_a d g_a(c) / d P_B(c') for the gradient-energy parts g_a of
// TotalEnergyDensity.cpp:133-251 (as in k_tdgl), D the impulse at c' =
// c + (DI, DJ, DK); stencils that cannot reach c' are skipped (they are zero)
template <typename T, bool VEC, bool ROT, int B, int DI, int DJ, int DK>
__device__ __forceinline__ T grad_rows_T(const DevParams& p, const MView& M, const T* R, const T lam[3],
                                         const DeltaView<T>& D, int i, int j, int k) {
    using Rc = Reach<DI, DJ, DK>;
    const T g11 = T(p.g11), g44 = T(p.g44), g44p = T(p.g44p), g12 = T(p.g12);
    T s = T(0);
    if constexpr (B == 2) {
        Hess<T> H;
        H.xx = Rc::xx ? ddpd<0, T>(D, M, i, j, k) : T(0);
        H.yy = Rc::yy ? ddpd<1, T>(D, M, i, j, k) : T(0);
        H.zz = Rc::zz ? ddpd<2, T>(D, M, i, j, k) : T(0);
        T A11, A44;
        if constexpr (ROT) {
            H.xy = Rc::xy ? dxdy<T>(D, M, i, j, k) : T(0);
            H.yz = Rc::yz ? dydz<T>(D, M, i, j, k) : T(0);
            H.xz = Rc::xz ? dxdz<T>(D, M, i, j, k) : T(0);
            A11 = rot_quad(R, 2, H);
            A44 = rot_quad(R, 0, H) + rot_quad(R, 1, H);
        } else {
            A11 = H.zz;
            A44 = H.xx + H.yy;
        }
        s = lam[2] * (-g11 * A11 - (g44 - g44p) * A44);
        if constexpr (VEC) {
            if constexpr (Rc::xz) s += lam[0] * (-(g12 + g44 - g44p) * dxdz<T>(D, M, i, j, k));
            if constexpr (Rc::yz) s += lam[1] * (-(g12 + g44 - g44p) * dydz<T>(D, M, i, j, k));
        }
    } else if constexpr (B == 0) {
        if constexpr (Rc::xz) s += lam[2] * (-(g44 + g44p + g12) * dxdz<T>(D, M, i, j, k));
        const T pxx = Rc::xx ? ddpd<0, T>(D, M, i, j, k) : T(0);
        const T pyy = Rc::yy ? ddpd<1, T>(D, M, i, j, k) : T(0);
        const T pzz = Rc::zz ? ddpd<2, T>(D, M, i, j, k) : T(0);
        s += lam[0] * (-g11 * pxx - (g44 + g44p) * (pyy + pzz));
        if constexpr (Rc::xy) s += lam[1] * (-(g12 + g44 + g44p) * dxdy<T>(D, M, i, j, k));
    } else {
        if constexpr (Rc::yz) s += lam[2] * (-(g44 + g44p + g12) * dydz<T>(D, M, i, j, k));
        if constexpr (Rc::xy) s += lam[0] * (-(g12 + g44 - g44p) * dxdy<T>(D, M, i, j, k));
        const T qxx = Rc::xx ? ddpd<0, T>(D, M, i, j, k) : T(0);
        const T qyy = Rc::yy ? ddpd<1, T>(D, M, i, j, k) : T(0);
        const T qzz = Rc::zz ? ddpd<2, T>(D, M, i, j, k) : T(0);
        s += lam[1] * (-g11 * qyy - (g44 - g44p) * (qxx + qzz));
    }
    return s;
}

// d L_a / d(a, b, c) of the Landau derivative L_a(a; b, c) (landau())
template <typename T>
__device__ __forceinline__ void landau_jac(const DevParams& p, T alpha, T a, T b, T c, T& Ja, T& Jb, T& Jc) {
    const T a2 = a * a, b2 = b * b, c2 = c * c;
    const T a12 = T(p.a12), a112 = T(p.a112), a123 = T(p.a123);
    Ja = alpha + T(3) * T(p.beta) * a2 + T(5) * T(p.gamma) * a2 * a2 + T(2) * a12 * (b2 + c2) +
         T(12) * a112 * a2 * (b2 + c2) + T(2) * a112 * (b2 * b2 + c2 * c2) + T(2) * a123 * b2 * c2;
    Jb = T(4) * a12 * a * b + T(8) * a112 * a2 * a * b + T(8) * a112 * a * b2 * b + T(4) * a123 * a * b * c2;
    Jc = T(4) * a12 * a * c + T(8) * a112 * a2 * a * c + T(8) * a112 * a * c2 * c + T(4) * a123 * a * b2 * c;
}

// the TDGL-updated cell c = c' + kOff[Q]: its rows' transposed gradient
// stencils at the impulse c' (the offset is a compile-time constant, so only
// the stencils that can reach c' are evaluated)
template <typename T, bool VEC, bool ROT, int Q>
__device__ __forceinline__ void grad_from(const DevParams& p, const MView& M, const uint8_t* __restrict__ code,
                                          const uint8_t* __restrict__ var, const Variant* __restrict__ vt,
                                          const double* __restrict__ lp, const double* __restrict__ lq,
                                          const double* __restrict__ lr, const DeltaView<T>& D, int i, int j, int k,
                                          T adj[3]) {
    constexpr int OX = kOff[Q][0], OY = kOff[Q][1], OZ = kOff[Q][2];
    const int ck = k + OZ;
    if (ck < 0 || ck >= p.nz) return;
    const int ci = wrap(i + OX, p.nx), cj = wrap(j + OY, p.ny);
    if (!updated(mcode(code, p, ci, cj, ck))) return;
    const size_t cc = cidx(p, ci, cj, ck);
    T R[9], al;
    load_R<T, ROT>(var, vt, cc, R, al, p);
    T lam[3];
    load_lam<T, VEC>(p, lp, lq, lr, cc, lam);
    adj[2] += grad_rows_T<T, VEC, ROT, 2, -OX, -OY, -OZ>(p, M, R, lam, D, ci, cj, ck);
    if constexpr (VEC) {
        adj[0] += grad_rows_T<T, VEC, ROT, 0, -OX, -OY, -OZ>(p, M, R, lam, D, ci, cj, ck);
        adj[1] += grad_rows_T<T, VEC, ROT, 1, -OX, -OY, -OZ>(p, M, R, lam, D, ci, cj, ck);
    }
}

template <typename T, bool VEC, bool ROT, int... Q>
__device__ __forceinline__ void grad_visit(std::integer_sequence<int, Q...>, const DevParams& p, const MView& M,
                                           const uint8_t* code, const uint8_t* var, const Variant* vt,
                                           const double* lp, const double* lq, const double* lr,
                                           const DeltaView<T>& D, int i, int j, int k, T adj[3]) {
    (grad_from<T, VEC, ROT, Q>(p, M, code, var, vt, lp, lq, lr, D, i, j, k, adj), ...);
}

// the seven cells whose first-derivative (dpd, grad phi) stencils can read a
// cell: itself and its face neighbours (entries of kOff)
constexpr int kFace[7] = {0, 1, 2, 5, 6, 9, 10};

// (ds/dP)^T psi from the FE cell c = c' + kOff[kFace[Q]] (k_rhs_p's
// -sum_a R_a . grad P_a, FP64)
template <bool VEC, bool ROT, int Q>
__device__ __forceinline__ void rhs_from(const DevParams& p, const MView& M, const uint8_t* __restrict__ code,
                                         const uint8_t* __restrict__ var, const Variant* __restrict__ vt,
                                         const double* __restrict__ psi, const DeltaView<double>& D, int i, int j,
                                         int k, double rs[3]) {
    constexpr int OX = kOff[kFace[Q]][0], OY = kOff[kFace[Q]][1], OZ = kOff[kFace[Q]][2];
    using Rc = Reach<-OX, -OY, -OZ>;
    const int ck = k + OZ;
    if (ck < 0 || ck >= p.nz) return;
    const int ci = wrap(i + OX, p.nx), cj = wrap(j + OY, p.ny);
    if ((mcode(code, p, ci, cj, ck) & 3) != 0) return;
    const size_t cc = cidx(p, ci, cj, ck);
    const double ps = psi[cc];
    if (ps == 0.0) return;
    double R[9], al;
    load_R<double, ROT>(var, vt, cc, R, al, p);
    const double d0 = Rc::dx ? dpd<0, double>(D, M, ci, cj, ck) : 0.0;
    const double d1 = Rc::dy ? dpd<1, double>(D, M, ci, cj, ck) : 0.0;
    const double d2 = Rc::dz ? dpd<2, double>(D, M, ci, cj, ck) : 0.0;
    rs[2] -= ps * (R[6] * d0 + R[7] * d1 + R[8] * d2);
    if constexpr (VEC) {
        rs[0] -= ps * (R[0] * d0 + R[1] * d1 + R[2] * d2);
        rs[1] -= ps * (R[3] * d0 + R[4] * d1 + R[5] * d2);
    }
}

template <bool VEC, bool ROT, int... Q>
__device__ __forceinline__ void rhs_visit(std::integer_sequence<int, Q...>, const DevParams& p, const MView& M,
                                          const uint8_t* code, const uint8_t* var, const Variant* vt,
                                          const double* psi, const DeltaView<double>& D, int i, int j, int k,
                                          double rs[3]) {
    (rhs_from<VEC, ROT, Q>(p, M, code, var, vt, psi, D, i, j, k, rs), ...);
}

// the components of grad_phi_acc that can depend on the accessor's cell
// c + (DI, DJ, DK); the others are left at zero (same formulas otherwise)
template <typename T, int DI, int DJ, int DK, typename A>
__device__ __forceinline__ void grad_phi_reach(const A& f, const DevParams& p, int i, int j, int k, T& gx, T& gy, T& gz) {
    using Rc = Reach<DI, DJ, DK>;
    gx = gy = gz = T(0);
    if constexpr (Rc::gx) gx = T((f(i + 1, j, k) - f(i - 1, j, k)) / (2. * p.dx[0]));
    if constexpr (Rc::gy) gy = T((f(i, j + 1, k) - f(i, j - 1, k)) / (2. * p.dx[1]));
    if constexpr (Rc::gz) {
        const double dz = p.dx[2];
        if (k == 0) gz = T((-4. * f(i, j, k - 1) + 3. * f(i, j, k) + f(i, j, k + 1)) / (3. * dz));
        else if (k == p.nz - 1) gz = T((4. * f(i, j, k + 1) - 3. * f(i, j, k) - f(i, j, k - 1)) / (3. * dz));
        else gz = T((f(i, j, k + 1) - f(i, j, k - 1)) / (2. * dz));
    }
}

// mu contribution of the TDGL-updated cell c = c' + kOff[kFace[Q]] (its E term
// reads phi at c'); the top-layer cell itself also carries the direct
// dependence on the electrode value
template <typename T, bool VEC, bool ROT, int Q>
__device__ __forceinline__ void phi_from(const DevParams& p, const uint8_t* __restrict__ code,
                                         const uint8_t* __restrict__ var, const Variant* __restrict__ vt,
                                         const double* __restrict__ lp, const double* __restrict__ lq,
                                         const double* __restrict__ lr, const PhiDelta& D, int i, int j, int k,
                                         T& acc, T& dvacc) {
    constexpr int OX = kOff[kFace[Q]][0], OY = kOff[kFace[Q]][1], OZ = kOff[kFace[Q]][2];
    const int ck = k + OZ;
    if (ck < 0 || ck >= p.nz) return;
    const int ci = wrap(i + OX, p.nx), cj = wrap(j + OY, p.ny);
    if (!updated(mcode(code, p, ci, cj, ck))) return;
    const size_t cc = cidx(p, ci, cj, ck);
    T R[9], al;
    load_R<T, ROT>(var, vt, cc, R, al, p);
    T lam[3];
    load_lam<T, VEC>(p, lp, lq, lr, cc, lam);
    T w[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) w[d] = lam[2] * R[6 + d] + (VEC ? lam[0] * R[d] + lam[1] * R[3 + d] : T(0));
    T gx, gy, gz;
    grad_phi_reach<T, -OX, -OY, -OZ>(D, p, ci, cj, ck, gx, gy, gz);
    acc += w[0] * gx + w[1] * gy + w[2] * gz;
    if constexpr (Q == 0) {
        if (k == p.nz - 1) {
            grad_phi_acc<T>(VDelta{&p}, p, ci, cj, ck, gx, gy, gz);
            dvacc = w[0] * gx + w[1] * gy + w[2] * gz;
        }
    }
}

template <typename T, bool VEC, bool ROT, int... Q>
__device__ __forceinline__ void phi_visit(std::integer_sequence<int, Q...>, const DevParams& p, const uint8_t* code,
                                          const uint8_t* var, const Variant* vt, const double* lp, const double* lq,
                                          const double* lr, const PhiDelta& D, int i, int j, int k, T& acc, T& dvacc) {
    (phi_from<T, VEC, ROT, Q>(p, code, var, vt, lp, lq, lr, D, i, j, k, acc, dvacc), ...);
}

// ---------------------------------------------------------------------------
// lambda^T: the loss weight on Pz of the FE cells, zero elsewhere
__global__ void __launch_bounds__(256) k_adj_init(DevParams p, const uint8_t* __restrict__ code, double* lp, double* lq,
                                                  double* lr, double g) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < p.N; c += (long long)gridDim.x * blockDim.x) {
        lr[c] = (__ldg(code + c + p.nxy) & 3) == 0 ? g : 0.0;
        if (lp) lp[c] = 0.0;
        if (lq) lq[c] = 0.0;
    }
}

// mu = dt (df/dphi)^T lambda: every cell collects from the TDGL-updated
// cells whose E stencil (grad_phi) reads it -- itself and the six face
// neighbours.  Also max|mu| (for the solve's stopping rule) and the direct
// voltage term dt (df/dV_hi)^T lambda of the top-layer cells.
template <typename T, bool VEC, bool ROT>
__global__ void __launch_bounds__(256) k_adj_phi(DevParams p, const uint8_t* __restrict__ code,
                                                 const uint8_t* __restrict__ var, const Variant* __restrict__ vt,
                                                 const double* __restrict__ lp, const double* __restrict__ lq,
                                                 const double* __restrict__ lr, double* __restrict__ mu,
                                                 double* __restrict__ norm, double* __restrict__ dV) {
    __shared__ double sh[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    double amax = 0.0, dv = 0.0;
    if (i < p.nx && j < p.ny) {
        const T mGam = T(-1.0) * T(p.BigGamma);
        T acc = T(0);
        const PhiDelta D{i, j, k, &p};
        T dvacc = T(0);
        phi_visit<T, VEC, ROT>(std::make_integer_sequence<int, 7>{}, p, code, var, vt, lp, lq, lr, D, i, j, k, acc, dvacc);
        dv = p.dt * (double)(mGam * dvacc);
        const double v = p.dt * (double)(mGam * acc);
        const size_t cc = cidx(p, i, j, k);
        mu[cc] = v;
        if ((long long)cc < p.Ns) amax = fabs(v);   // the solve reads mu on its own cells only
    }
    const double bm = block_max2(amax, sh);
    const double bs = block_sum2(dv, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        atomic_max_pos(norm, bm);
        if (bs != 0.0) atomicAdd(dV, bs);
    }
}

// lambda^{n-1} (see the file header) and the parameter sums of step n.
// grad layout: [0] alpha over the cells with the global alpha, [1] beta,
// [2] gamma, [3] g11, [4] g44, [8 + g] alpha of grain g.
template <typename T, bool VEC, bool ROT>
__global__ void __launch_bounds__(256) k_adj_P(DevParams p, const uint8_t* __restrict__ code,
                                               const uint8_t* __restrict__ var, const Variant* __restrict__ vt,
                                               const uint8_t* __restrict__ gid, int ngalpha,
                                               const double* __restrict__ Pp, const double* __restrict__ Pq,
                                               const double* __restrict__ Pr, const double* __restrict__ lp,
                                               const double* __restrict__ lq, const double* __restrict__ lr,
                                               const double* __restrict__ psi, double gload,
                                               double* __restrict__ lp_out, double* __restrict__ lq_out,
                                               double* __restrict__ lr_out, double* __restrict__ grad,
                                               double* __restrict__ dV) {
    __shared__ double sh[32];
    __shared__ double bins[256];
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    if (gid) {
        for (int q = t; q < 256; q += blockDim.x * blockDim.y) bins[q] = 0.0;
        __syncthreads();
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    double s_alpha = 0.0, s_beta = 0.0, s_gamma = 0.0, s_g11 = 0.0, s_g44 = 0.0, dv = 0.0;
    if (i < p.nx && j < p.ny) {
        const size_t c0 = cidx(p, i, j, k);
        const int m0 = mcode(code, p, i, j, k);
        const MView M{code, &p};
        const T mGam = T(-1.0) * T(p.BigGamma);
        double out[3];
        out[2] = lr[c0] + ((m0 & 3) == 0 ? gload : 0.0);
        out[0] = VEC ? lp[c0] : 0.0;
        out[1] = VEC ? lq[c0] : 0.0;
        T adj[3] = {T(0), T(0), T(0)};   // sum_a lambda_a d g_a / dP_b + Landau, before -Gamma dt

        // ---- local Landau Jacobian and the parameter sums at this cell
        if (updated(m0)) {
            T R[9], al;
            load_R<T, ROT>(var, vt, c0, R, al, p);
            T lam[3];
            load_lam<T, VEC>(p, lp, lq, lr, c0, lam);
            const T r = T(Pr[c0]), pp = VEC ? T(Pp[c0]) : T(0), pq = VEC ? T(Pq[c0]) : T(0);
            double sa = 0.0, sb = 0.0, sc = 0.0;
            if (p.incl_L) {
                T Ja, Jb, Jc;
                landau_jac<T>(p, al, r, pp, pq, Ja, Jb, Jc);       // row r: L(r; p, q)
                adj[2] += lam[2] * Ja;
                adj[0] += lam[2] * Jb;
                adj[1] += lam[2] * Jc;
                sa += (double)(lam[2] * r);
                sb += (double)(lam[2] * r * r * r);
                sc += (double)(lam[2] * r * r * r * r * r);
                if (VEC) {
                    landau_jac<T>(p, al, pp, pq, r, Ja, Jb, Jc);   // row p: L(p; q, r)
                    adj[0] += lam[0] * Ja;
                    adj[1] += lam[0] * Jb;
                    adj[2] += lam[0] * Jc;
                    landau_jac<T>(p, al, pq, pp, r, Ja, Jb, Jc);   // row q: L(q; p, r)
                    adj[1] += lam[1] * Ja;
                    adj[0] += lam[1] * Jb;
                    adj[2] += lam[1] * Jc;
                    sa += (double)(lam[0] * pp + lam[1] * pq);
                    sb += (double)(lam[0] * pp * pp * pp + lam[1] * pq * pq * pq);
                    sc += (double)(lam[0] * pp * pp * pp * pp * pp + lam[1] * pq * pq * pq * pq * pq);
                }
            }
            double s11 = 0.0, s44 = 0.0;
            if (p.incl_G) {
                const PView<T> Fr{Pr, &p};
                const Hess<T> H = hess<T, ROT>(Fr, M, i, j, k);
                T A11, A44;
                if (ROT) {
                    A11 = rot_quad(R, 2, H);
                    A44 = rot_quad(R, 0, H) + rot_quad(R, 1, H);
                } else {
                    A11 = H.zz;
                    A44 = H.xx + H.yy;
                }
                T d11 = lam[2] * (-A11), d44 = lam[2] * (-A44);
                if (VEC) {
                    const PView<T> Fp{Pp, &p}, Fq{Pq, &p};
                    d44 += lam[2] * (-(dydz<T>(Fq, M, i, j, k) + dxdz<T>(Fp, M, i, j, k)));
                    d11 += lam[0] * (-ddpd<0, T>(Fp, M, i, j, k));
                    d44 += lam[0] * (-(ddpd<1, T>(Fp, M, i, j, k) + ddpd<2, T>(Fp, M, i, j, k)) -
                                     (dxdy<T>(Fq, M, i, j, k) + dxdz<T>(Fr, M, i, j, k)));
                    d11 += lam[1] * (-ddpd<1, T>(Fq, M, i, j, k));
                    d44 += lam[1] * (-(ddpd<0, T>(Fq, M, i, j, k) + ddpd<2, T>(Fq, M, i, j, k)) -
                                     dxdy<T>(Fp, M, i, j, k) - dydz<T>(Fr, M, i, j, k));
                }
                s11 = (double)d11;
                s44 = (double)d44;
            }
            const double f = p.dt * (double)mGam;
            const double ga = f * sa;
            s_beta = f * sb;
            s_gamma = f * sc;
            s_g11 = f * s11;
            s_g44 = f * s44;
            const int g = gid ? (int)__ldg(gid + c0) : 255;
            if (g == 255 || g >= ngalpha) s_alpha = ga;
            if (gid && g != 255 && ga != 0.0) atomicAdd(&bins[g], ga);
        }

        // ---- transposed gradient-energy stencils of the cells that read this one
        if (p.incl_G) {
            const DeltaView<T> D{i, j, k, &p};
            if constexpr (VEC || ROT)
                grad_visit<T, VEC, ROT>(std::make_integer_sequence<int, 25>{}, p, M, code, var, vt, lp, lq, lr, D, i, j, k, adj);
            else   // without rotation or Px, Py only the axis second derivatives reach
                grad_visit<T, VEC, ROT>(std::make_integer_sequence<int, 13>{}, p, M, code, var, vt, lp, lq, lr, D, i, j, k, adj);
        }
        const double f = p.dt * (double)mGam;
        out[2] += f * (double)adj[2];
        if (VEC) {
            out[0] += f * (double)adj[0];
            out[1] += f * (double)adj[1];
        }

        // ---- (ds/dP)^T psi: the FE right-hand side -sum_a R_a . grad P_a
        // (k_rhs_p, FP64) of the cells whose dpd stencil reads this one
        if (psi) {
            const DeltaView<double> D{i, j, k, &p};
            double rs[3] = {0.0, 0.0, 0.0};
            rhs_visit<VEC, ROT>(std::make_integer_sequence<int, 7>{}, p, M, code, var, vt, psi, D, i, j, k, rs);
            out[2] += rs[2];
            if (VEC) {
                out[0] += rs[0];
                out[1] += rs[1];
            }
            // the electrode term 2 eps V / dz^2 of the top layer's right-hand side
            if (k == p.nz - 1) dv = 2.0 * p.eps[m0 & 7] * p.ih2[2] * psi[c0];
        }
        lr_out[c0] = out[2];
        if (VEC) {
            lp_out[c0] = out[0];
            lq_out[c0] = out[1];
        }
    }
    const double r0 = block_sum2(s_alpha, sh);
    const double r1 = block_sum2(s_beta, sh);
    const double r2 = block_sum2(s_gamma, sh);
    const double r3 = block_sum2(s_g11, sh);
    const double r4 = block_sum2(s_g44, sh);
    const double r5 = block_sum2(dv, sh);
    if (t == 0) {
        if (r0 != 0.0) atomicAdd(grad + 0, r0);
        if (r1 != 0.0) atomicAdd(grad + 1, r1);
        if (r2 != 0.0) atomicAdd(grad + 2, r2);
        if (r3 != 0.0) atomicAdd(grad + 3, r3);
        if (r4 != 0.0) atomicAdd(grad + 4, r4);
        if (r5 != 0.0) atomicAdd(dV, r5);
    }
    if (gid) {
        __syncthreads();
        for (int q = t; q < 256; q += blockDim.x * blockDim.y)
            if (bins[q] != 0.0) atomicAdd(grad + 8 + q, bins[q]);
    }
}

// d rho / d phi (ChargeDensity.cpp:46-93 differentiated in phi) on the
// semiconductor cells, zero elsewhere: the alpha of the adjoint Poisson
// operator A0 - diag(rho')
__device__ double fd_half_deriv(double eta, double& F) {
    // F(eta) = 1 / (exp(-eta) + xi(eta)), xi = 3 sqrt(3.14) / (4 nu^(3/8)),
    // nu = eta^4 + 50 + 33.6 eta (1 - 0.68 exp(-0.17 (eta + 1)^2))
    const double g = exp(-0.17 * pow((eta + 1.0), 2.0));
    const double nu = pow(eta, 4.0) + 50.0 + 33.6 * eta * (1.0 - 0.68 * g);
    const double dnu = 4.0 * pow(eta, 3.0) + 33.6 * (1.0 - 0.68 * g) + 33.6 * eta * (0.68 * 0.34 * (eta + 1.0) * g);
    const double c = 3.0 * sqrt(3.14) / 4.0;
    const double xi = c / pow(nu, 3. / 8.);
    const double dxi = c * (-3. / 8.) * pow(nu, -11. / 8.) * dnu;
    const double den = exp(-eta) + xi;
    F = 1.0 / den;
    return -(-exp(-eta) + dxi) / (den * den);
}

__global__ void __launch_bounds__(256) k_drho(DevParams p, const uint8_t* __restrict__ code, const double* __restrict__ phi,
                                              double* __restrict__ a64, float* __restrict__ a32) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < p.N; c += (long long)gridDim.x * blockDim.x) {
        double a = 0.0;
        if ((__ldg(code + c + p.nxy) & 3) >= 2) {
            const double q = p.q, kT = p.kb * p.T, ph = phi[c];
            const double Ef = 0.0, g_A = 4.0, g_D = 2.0;
            const double Ec_corr = -q * (ph - p.phi_ref) - p.Chi * q;
            const double Ev_corr = Ec_corr - q * p.Eg;
            double de, dh;   // d(e_den)/dphi, d(h_den)/dphi
            if (p.use_FD == 1) {
                const double eta_n = -(Ec_corr - q * Ef) / kT;   // d eta_n / dphi = q / kT
                const double eta_p = -(q * Ef - Ev_corr) / kT;   // d eta_p / dphi = -q / kT
                double F;
                de = p.Nc * fd_half_deriv(eta_n, F) * (q / kT);
                dh = p.Nv * fd_half_deriv(eta_p, F) * (-q / kT);
            } else {
                de = p.Nc * exp(-(Ec_corr - q * Ef) / kT) * (q / kT);
                dh = p.Nv * exp(-(q * Ef - Ev_corr) / kT) * (-q / kT);
            }
            const double xa = exp((-q * Ef + q * p.Ea + q * p.phi_ref - q * p.Chi - q * p.Eg - q * ph) / kT);
            const double xd = exp((q * Ef + q * p.Ed - q * p.phi_ref + q * p.Chi + q * ph) / kT);
            const double da = p.NA * g_A * xa * (q / kT) / ((1.0 + g_A * xa) * (1.0 + g_A * xa));
            const double dd = -p.ND * g_D * xd * (q / kT) / ((1.0 + g_D * xd) * (1.0 + g_D * xd));
            a = q * (dh - de - da + dd);
        }
        a64[c] = a;
        if (a32) a32[c] = (float)a;
    }
}

dim3 cell_grid2(const DevParams& p) { return dim3((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz); }

// psi = 0 when the reverse step's source is zero (max|mu| not positive):
// the adjoint solve then starts, and ends, at the exact answer
__global__ void __launch_bounds__(256) k_zero_if_zero(double* __restrict__ psi, const double* __restrict__ nmu,
                                                      long long n) {
    pdl_entry();
    if (*nmu > 0.0) return;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        psi[c] = 0.0;
}

}  // namespace

int launch_zero_if_zero(double* psi, const double* nmu, long long n, cudaStream_t s) {
    launch_k(k_zero_if_zero, 4 * 148, 256, 0, s, psi, nmu, n);
    return (int)cudaGetLastError();
}

int launch_adj_init(const DevParams& p, const uint8_t* code, double* lam[3], double g, cudaStream_t s) {
    k_adj_init<<<p.ngrid_red, 256, 0, s>>>(p, code, lam[0], lam[1], lam[2], g);
    return (int)cudaGetLastError();
}

int launch_adj_phi(const DevParams& p, int mixed, bool vec, const uint8_t* code, const uint8_t* var, const Variant* vt,
                   double* const lam[3], double* mu, double* norm, double* dV, cudaStream_t s) {
    const dim3 g = cell_grid2(p), b(32, 8);
    const bool rot = var != nullptr;
#define ADJ_PHI(T, V, R) k_adj_phi<T, V, R><<<g, b, 0, s>>>(p, code, var, vt, lam[0], lam[1], lam[2], mu, norm, dV)
    if (mixed) {
        if (vec) { if (rot) ADJ_PHI(float, true, true); else ADJ_PHI(float, true, false); }
        else { if (rot) ADJ_PHI(float, false, true); else ADJ_PHI(float, false, false); }
    } else {
        if (vec) { if (rot) ADJ_PHI(double, true, true); else ADJ_PHI(double, true, false); }
        else { if (rot) ADJ_PHI(double, false, true); else ADJ_PHI(double, false, false); }
    }
#undef ADJ_PHI
    return (int)cudaGetLastError();
}

int launch_adj_P(const DevParams& p, int mixed, bool vec, const uint8_t* code, const uint8_t* var, const Variant* vt,
                 const uint8_t* gid, int ngalpha, const double* const P[3], double* const lam[3], const double* psi,
                 double gload, double* const lam_out[3], double* grad, double* dV, cudaStream_t s) {
    const dim3 g = cell_grid2(p), b(32, 8);
    const bool rot = var != nullptr;
#define ADJ_P(T, V, R)                                                                                       \
    k_adj_P<T, V, R><<<g, b, 0, s>>>(p, code, var, vt, gid, ngalpha, P[0], P[1], P[2], lam[0], lam[1], lam[2], \
                                     psi, gload, lam_out[0], lam_out[1], lam_out[2], grad, dV)
    if (mixed) {
        if (vec) { if (rot) ADJ_P(float, true, true); else ADJ_P(float, true, false); }
        else { if (rot) ADJ_P(float, false, true); else ADJ_P(float, false, false); }
    } else {
        if (vec) { if (rot) ADJ_P(double, true, true); else ADJ_P(double, true, false); }
        else { if (rot) ADJ_P(double, false, true); else ADJ_P(double, false, false); }
    }
#undef ADJ_P
    return (int)cudaGetLastError();
}

int launch_drho(const DevParams& p, const uint8_t* code, const double* phi, double* a64, float* a32, cudaStream_t s) {
    k_drho<<<p.ngrid_red, 256, 0, s>>>(p, code, phi, a64, a32);
    return (int)cudaGetLastError();
}

}  // namespace fx
