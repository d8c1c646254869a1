// fx_mg.cu -- geometric multigrid for (-alpha - div beta grad) phi = rhs.
// See fx_mg.h for the hierarchy.  Level 0 reads the one-byte material code of
// each cell and forms beta_face = 0.5 (eps_L + eps_R) on the fly (the face
// average of eXstaticUtil.cpp:128-136 with the eps of
// ElectrostaticSolver.cpp:238-251); coarse levels store face beta and alpha.
#include "fx_mg.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>

#include <cuda_fp16.h>

namespace fx {

extern std::atomic<long long> g_launches;

namespace {

template <typename T>
struct Op {
    int nx, ny, nz;
    int nxy;               // cells per z plane (every level holds fewer than 2^31 cells)
    T ih2x, ih2y, ih2z;
    const uint8_t* code;   // level 0: material codes (with z ghost layers)
    T eps[8];
    const T* bw;           // coarse: beta on the low-x / low-y / low-z faces
    const T* bs;
    const T* bb;           // nz + 1 layers
    const T* a;            // alpha (may be null)
    const T* zc;           // coarse: face beta by plane (bw[nz], bs[nz], bb[nz+1]) when laterally uniform
    T vlo, vhi;            // electrode values (inhomogeneous level-0 operator only)
    // coarse, FP32 cycle: the face beta in FP16 scaled by 1 / hscale (ih2x..z
    // then carry hscale); null where the level keeps FP32 arrays
    const uint16_t* bwh;
    const uint16_t* bsh;
    const uint16_t* bbh;
};

// one FP16 face beta (read-only path)
__device__ __forceinline__ float hload(const uint16_t* p) { return __half2float(__ushort_as_half(__ldg(p))); }

// a coarse level whose FP32 kernels read the FP16 face arrays
template <typename T>
static bool half_faces(const Op<T>& o) { return sizeof(T) == 4 && o.bwh != nullptr && !o.zc; }

// couplings of cell (i,j,k) to its six neighbours (already divided by h^2),
// the diagonal and the electrode contribution to the right-hand side
// KIND: CK_FINE level 0 (material codes), CK_ARRAYS coarse face-beta arrays,
// CK_PLANES coarse face beta by plane (laterally uniform), CK_HALF coarse
// face-beta arrays in FP16 (FP32 cycle only)
constexpr int CK_ARRAYS = 0, CK_FINE = 1, CK_PLANES = 2, CK_HALF = 3;

// The per-cell arithmetic of the operator, every rounding written out (no
// product left for the compiler to fuse into a neighbouring add), so that
// each form of the smoother and residual that uses these helpers gives the
// same bits for a cell whatever surrounds it after inlining.
// a face coupling from the two cells' eps: 0.5 (e0 + e1) / h^2
template <typename T>
__device__ __forceinline__ T face_avg(T e0, T e1, T ih2) { return mul_rn(mul_rn(T(0.5), add_rn(e0, e1)), ih2); }
// a face coupling from a stored face beta
template <typename T>
__device__ __forceinline__ T face_beta(T f, T ih2) { return mul_rn(f, ih2); }
// an electrode face (maxorder-2 ghost 2 V - phi_0): 2 beta / h^2 into the
// diagonal, 2 beta V / h^2 into the right-hand side
template <typename T>
__device__ __forceinline__ void electrode(T beta, T ih2, T v, T& extra, T& bcv) {
    const T e2 = mul_rn(mul_rn(T(2), beta), ih2);
    extra = add_rn(extra, e2);
    bcv = add_rn(bcv, mul_rn(e2, v));
}
// the same on a coarse level (homogeneous electrode values: no right-hand-side term)
template <typename T>
__device__ __forceinline__ void electrode0(T beta, T ih2, T& extra) {
    extra = add_rn(extra, mul_rn(mul_rn(T(2), beta), ih2));
}
template <typename T>
__device__ __forceinline__ T diag_sum(T a, T cw, T ce, T cs, T cn, T cb, T ct, T extra) {
    T d = add_rn(-a, cw);
    d = add_rn(d, ce);
    d = add_rn(d, cs);
    d = add_rn(d, cn);
    d = add_rn(d, cb);
    d = add_rn(d, ct);
    return add_rn(d, extra);
}
// b + electrode terms + the off-diagonal couplings times the neighbours
template <typename T>
__device__ __forceinline__ T gs_rhs(T b, T bcv, T cw, T xw, T ce, T xe, T cs, T xs, T cn, T xn, bool lo, T cb, T xb,
                                    bool hi, T ct, T xt) {
    T s = add_rn(b, bcv);
    s = fma_rn(cw, xw, s);
    s = fma_rn(ce, xe, s);
    s = fma_rn(cs, xs, s);
    s = fma_rn(cn, xn, s);
    if (lo) s = fma_rn(cb, xb, s);
    if (hi) s = fma_rn(ct, xt, s);
    return s;
}

// the residual b + electrode terms - (diag x - the off-diagonal couplings times the neighbours)
template <typename T>
__device__ __forceinline__ T res_val(T b, T bcv, T diag, T xc, T cw, T xw, T ce, T xe, T cs, T xs, T cn, T xn, bool lo,
                                     T cb, T xb, bool hi, T ct, T xt) {
    T off = mul_rn(cw, xw);
    off = fma_rn(ce, xe, off);
    off = fma_rn(cs, xs, off);
    off = fma_rn(cn, xn, off);
    if (lo) off = fma_rn(cb, xb, off);
    if (hi) off = fma_rn(ct, xt, off);
    return add_rn(add_rn(b, bcv), -fma_rn(diag, xc, -off));
}

template <typename T, int KIND>
__device__ __forceinline__ void coeffs(const Op<T>& o, int i, int j, int k, int c, int im, int ip, int jm, int jp,
                                       T& cw, T& ce, T& cs, T& cn, T& cb, T& ct, T& diag, T& bcv, const T* eps) {
    T extra = T(0);
    bcv = T(0);
    if constexpr (KIND == CK_FINE) {
        const uint8_t* cd = o.code + o.nxy;   // skip the k = -1 ghost layer
        const int row = c - i;
        const T ec = eps[__ldg(cd + c) & 7];
        cw = face_avg(ec, eps[__ldg(cd + row + im) & 7], o.ih2x);
        ce = face_avg(ec, eps[__ldg(cd + row + ip) & 7], o.ih2x);
        cs = face_avg(ec, eps[__ldg(cd + c + (jm - j) * o.nx) & 7], o.ih2y);
        cn = face_avg(ec, eps[__ldg(cd + c + (jp - j) * o.nx) & 7], o.ih2y);
        if (k > 0) cb = face_avg(ec, eps[__ldg(cd + c - o.nxy) & 7], o.ih2z);
        else { cb = T(0); electrode(ec, o.ih2z, o.vlo, extra, bcv); }
        if (k < o.nz - 1) ct = face_avg(ec, eps[__ldg(cd + c + o.nxy) & 7], o.ih2z);
        else { ct = T(0); electrode(ec, o.ih2z, o.vhi, extra, bcv); }
    } else if constexpr (KIND == CK_PLANES) {
        // a layered stack: every face of a plane has the same beta
        cw = ce = face_beta(__ldg(o.zc + k), o.ih2x);
        cs = cn = face_beta(__ldg(o.zc + o.nz + k), o.ih2y);
        // (level 0: bb[0], bb[nz] are the eps of the electrode-layer cells)
        const T fb = __ldg(o.zc + 2 * o.nz + k), ft = __ldg(o.zc + 2 * o.nz + k + 1);
        if (k > 0) cb = face_beta(fb, o.ih2z);
        else { cb = T(0); electrode(fb, o.ih2z, o.vlo, extra, bcv); }
        if (k < o.nz - 1) ct = face_beta(ft, o.ih2z);
        else { ct = T(0); electrode(ft, o.ih2z, o.vhi, extra, bcv); }
    } else if constexpr (KIND == CK_HALF) {
        static_assert(sizeof(T) == 4, "FP16 faces in the FP32 cycle only");
        const int row = c - i;
        cw = face_beta(hload(o.bwh + c), o.ih2x);
        ce = face_beta(hload(o.bwh + row + ip), o.ih2x);
        cs = face_beta(hload(o.bsh + c), o.ih2y);
        cn = face_beta(hload(o.bsh + c + (jp - j) * o.nx), o.ih2y);
        const T fb = hload(o.bbh + c), ft = hload(o.bbh + c + o.nxy);
        if (k > 0) cb = face_beta(fb, o.ih2z);
        else { cb = T(0); electrode0(fb, o.ih2z, extra); }
        if (k < o.nz - 1) ct = face_beta(ft, o.ih2z);
        else { ct = T(0); electrode0(ft, o.ih2z, extra); }
    } else {
        // coarse levels: homogeneous electrode conditions (no right-hand-side term)
        const int row = c - i;
        cw = face_beta(__ldg(o.bw + c), o.ih2x);
        ce = face_beta(__ldg(o.bw + row + ip), o.ih2x);
        cs = face_beta(__ldg(o.bs + c), o.ih2y);
        cn = face_beta(__ldg(o.bs + c + (jp - j) * o.nx), o.ih2y);
        const T fb = __ldg(o.bb + c), ft = __ldg(o.bb + c + o.nxy);
        if (k > 0) cb = face_beta(fb, o.ih2z);
        else { cb = T(0); electrode0(fb, o.ih2z, extra); }
        if (k < o.nz - 1) ct = face_beta(ft, o.ih2z);
        else { ct = T(0); electrode0(ft, o.ih2z, extra); }
    }
    if (o.nx == 1) { cw = T(0); ce = T(0); }
    if (o.ny == 1) { cs = T(0); cn = T(0); }
    const T a = o.a ? o.a[c] : T(0);
    diag = diag_sum(a, cw, ce, cs, cn, cb, ct, extra);
}

__device__ __forceinline__ void nbr(int i, int n, int& m, int& p) {
    m = i == 0 ? n - 1 : i - 1;
    p = i == n - 1 ? 0 : i + 1;
}

// the max-norm reductions spread their block maxima over NORM_SLOTS addresses
// (one atomic per block, fewer collisions); the host takes the max of the slots
constexpr int NORM_SLOTS = 64;

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    if (!(v == v)) v = __longlong_as_double(0x7ff0000000000000LL);  // a NaN residual never converges
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// max that keeps a NaN (fmax would drop it): a NaN anywhere in a residual
// must reach the loop test, where it ends the solve as a failure
__device__ __forceinline__ double nan_max(double a, double b) { return (a > b || a != a) ? a : b; }

__device__ double block_max_all(double v) {
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_down_sync(0xffffffffu, v, o));
    const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nt = blockDim.x * blockDim.y * blockDim.z;
    if ((t & 31) == 0) sh[t >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (t < 32) {
        r = t < (nt + 31) / 32 ? sh[t] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r = nan_max(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    return r;
}

// red-black point Gauss-Seidel half sweep: color = parity of i + j + k
// the smoother's division: exact in FP64; in the FP32 correction cycle of
// the mixed path the fast single-precision divide (the update is a smoothing
// step; the FP64 outer residual decides convergence)
__device__ __forceinline__ double sdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float sdiv(float a, float b) { return __fdividef(a, b); }

// ZERO: the first half sweep (colour 0) from x = 0: the colour-0 value is
// (b + electrode terms) / diag and the colour-1 cell of the same x pair is
// set to 0, so the caller need not clear x first (even nx only)
// the update of one cell of a red-black half sweep: t indexes the x pair,
// the cell is the pair's one of this colour
template <typename T, int KIND, bool ZERO>
__device__ __forceinline__ void rbgs_update(const Op<T>& o, T* __restrict__ x, const T* __restrict__ b, int color,
                                            int t, int j, int k, const T* seps) {
    const int i = 2 * t + ((j + k + color) & 1);
    if (j >= o.ny || i >= o.nx) return;
    const int c = i + o.nx * (j + o.ny * k);
    int im, ip, jm, jp;
    nbr(i, o.nx, im, ip);
    nbr(j, o.ny, jm, jp);
    T cw, ce, cs, cn, cb, ct, diag, bcv;
    coeffs<T, KIND>(o, i, j, k, c, im, ip, jm, jp, cw, ce, cs, cn, cb, ct, diag, bcv, seps);
    const int row = c - i;
    if (ZERO) {
        x[c] = sdiv(add_rn(b[c], bcv), diag);
        x[c + ((i & 1) ? -1 : 1)] = T(0);
        return;
    }
    const bool lo = k > 0, hi = k < o.nz - 1;
    const T s = gs_rhs(b[c], bcv, cw, x[row + im], ce, x[row + ip], cs, x[c + (jm - j) * o.nx], cn,
                       x[c + (jp - j) * o.nx], lo, cb, lo ? x[c - o.nxy] : T(0), hi, ct, hi ? x[c + o.nxy] : T(0));
    x[c] = sdiv(s, diag);
}

template <typename T, int KIND, bool ZERO = false>
__global__ void __launch_bounds__(256) k_rbgs(Op<T> o, T* __restrict__ x, const T* __restrict__ b, int color) {
    pdl_entry();
    __shared__ T seps[8];
    if (KIND == CK_FINE) {
        if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
            for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
        __syncthreads();
    }
    rbgs_update<T, KIND, ZERO>(o, x, b, color, blockIdx.x * blockDim.x + threadIdx.x,
                               blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z, seps);
}

// ---- row-segment form of the point red-black half sweep
//
// Each thread owns a 32-byte segment of one x row (SEG = 8 FP32 or 4 FP64
// cells starting at a multiple of SEG) and updates the SEG / 2 cells of the
// colour in it.  Every row it needs -- the segment itself, the rows j - 1 and
// j + 1, the planes k - 1 and k + 1, b, alpha, the material codes or face
// coefficients -- arrives in two 16-byte loads (codes: one 8- or 4-byte load),
// and the index, wrap and plane tests are paid once per segment instead of
// once per cell.  The segment is written back whole: the other colour's
// cells with the bits they were read with (no thread of this half sweep
// writes them), so the result is bit-identical to k_rbgs, whose per-cell
// operations it repeats in the same order.  A warp never mixes the two
// parities of (j + k + colour): with fewer than 32 segments per row the
// block's rows are ordered even offsets first, so each warp's rows share one.
template <typename T, int SB> struct SegW { static constexpr int n = SB / (int)sizeof(T); };

// 16-byte vector accesses written as PTX: one 128-bit load or store per
// call (through float4 / double2 copies, ncu counted two load instructions
// per 16 bytes in this kernel).  The x accesses are volatile and the store
// clobbers memory, so they keep their order; the read-only loads (.nc) may move.
__device__ __forceinline__ void ld16(const float* p, float* v) {
    asm volatile("ld.global.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "l"(p));
}
__device__ __forceinline__ void ld16(const double* p, double* v) {
    asm volatile("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "l"(p));
}
__device__ __forceinline__ void ldg16(const float* p, float* v) {
    asm("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "l"(p));
}
__device__ __forceinline__ void ldg16(const double* p, double* v) {
    asm("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "l"(p));
}
__device__ __forceinline__ void st16(float* p, const float* v) {
    asm volatile("st.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3])
                 : "memory");
}
__device__ __forceinline__ void st16(double* p, const double* v) {
    asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v[0]), "d"(v[1]) : "memory");
}

template <typename T, int SB>
__device__ __forceinline__ void ld_seg(const T* p, T (&v)[SegW<T, SB>::n]) {
    constexpr int H = 16 / (int)sizeof(T);
    ld16(p, v);
    if constexpr (SB == 32) ld16(p + H, v + H);
}

template <typename T, int SB>
__device__ __forceinline__ void ldg_seg(const T* p, T (&v)[SegW<T, SB>::n]) {
    constexpr int H = 16 / (int)sizeof(T);
    ldg16(p, v);
    if constexpr (SB == 32) ldg16(p + H, v + H);
}

template <typename T, int SB>
__device__ __forceinline__ void st_seg(T* p, const T (&v)[SegW<T, SB>::n]) {
    constexpr int H = 16 / (int)sizeof(T);
    st16(p, v);
    if constexpr (SB == 32) st16(p + H, v + H);
}

// the material codes of a segment, one byte per cell
template <int SEG>
__device__ __forceinline__ unsigned long long ld_codes(const uint8_t* p) {
    if constexpr (SEG == 8) return __ldg(reinterpret_cast<const unsigned long long*>(p));
    else if constexpr (SEG == 4) return (unsigned long long)__ldg(reinterpret_cast<const unsigned int*>(p));
    else return (unsigned long long)__ldg(reinterpret_cast<const unsigned short*>(p));
}

__device__ __forceinline__ int code_at(unsigned long long w, int m) { return (int)(w >> (8 * m)) & 7; }

// The operator coefficients of one row segment: the material codes of the
// segment's row and of its four neighbour rows (level 0), the stored face
// beta (coarse levels) or the plane's face beta (layered stacks).  NL / NR:
// the cells left of the segment's first / right of its last are needed.
template <typename T, int SB, int KIND, bool NL, bool NR>
struct SegCoef {
    static constexpr int SEG = SegW<T, SB>::n;
    unsigned long long wc = 0, ws = 0, wn = 0, wb = 0, wt = 0;   // codes, one byte per cell
    int hl = 0, hr = 0;                                           // halo codes
    T pw = T(0), ps = T(0), pb = T(0), pt = T(0);                 // plane values
    T fw[SEG], fs[SEG], fn[SEG], fb[SEG], ft[SEG];                // face arrays
    T fr = T(0);                                                  // low-x face beta right of the segment

    // row: first cell of the row; c0 = row + i0; so / no: offsets of the rows j - 1 / j + 1;
    // il / ir: x index left of the segment / right of it
    __device__ __forceinline__ void load(const Op<T>& o, int row, int c0, int so, int no, int k, bool lo, bool hi,
                                         int il, int ir) {
        if constexpr (KIND == CK_FINE) {
            const uint8_t* cd = o.code + o.nxy;   // skip the k = -1 ghost layer
            wc = ld_codes<SEG>(cd + c0);
            ws = ld_codes<SEG>(cd + c0 + so);
            wn = ld_codes<SEG>(cd + c0 + no);
            if (lo) wb = ld_codes<SEG>(cd + c0 - o.nxy);
            if (hi) wt = ld_codes<SEG>(cd + c0 + o.nxy);
            if (NL) hl = __ldg(cd + row + il) & 7;
            if (NR) hr = __ldg(cd + row + ir) & 7;
        } else if constexpr (KIND == CK_PLANES) {
            pw = __ldg(o.zc + k);
            ps = __ldg(o.zc + o.nz + k);
            pb = __ldg(o.zc + 2 * o.nz + k);
            pt = __ldg(o.zc + 2 * o.nz + k + 1);
        } else if constexpr (KIND == CK_HALF) {
            static_assert(sizeof(T) == 4, "FP16 faces in the FP32 cycle only");
            ldh_seg(o.bwh + c0, fw);
            ldh_seg(o.bsh + c0, fs);
            ldh_seg(o.bsh + c0 + no, fn);
            ldh_seg(o.bbh + c0, fb);
            ldh_seg(o.bbh + c0 + o.nxy, ft);
            if (NR) fr = hload(o.bwh + row + ir);
        } else {
            ldg_seg<T, SB>(o.bw + c0, fw);
            ldg_seg<T, SB>(o.bs + c0, fs);
            ldg_seg<T, SB>(o.bs + c0 + no, fn);
            ldg_seg<T, SB>(o.bb + c0, fb);
            ldg_seg<T, SB>(o.bb + c0 + o.nxy, ft);
            if (NR) fr = __ldg(o.bw + row + ir);
        }
    }

    // SEG FP16 face betas (2 SEG bytes) as T
    template <int N>
    __device__ __forceinline__ static void ldh_seg(const uint16_t* p, T (&v)[N]) {
        auto h2f = [](unsigned w, int hi) {
            return __half2float(__ushort_as_half((unsigned short)(hi ? w >> 16 : w & 0xffffu)));
        };
        if constexpr (N == 4) {
            const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
            v[0] = h2f(q.x, 0); v[1] = h2f(q.x, 1); v[2] = h2f(q.y, 0); v[3] = h2f(q.y, 1);
        } else {
            static_assert(N == 8, "4 or 8 FP16 faces");
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(p));
            const unsigned w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int t = 0; t < 4; ++t) { v[2 * t] = h2f(w[t], 0); v[2 * t + 1] = h2f(w[t], 1); }
        }
    }

    // the couplings of cell m of the segment (the operations of coeffs<T, KIND>)
    __device__ __forceinline__ void cell(const Op<T>& o, const T* seps, int m, bool lo, bool hi, T& cw, T& ce, T& cs,
                                         T& cn, T& cb, T& ct, T& extra, T& bcv) const {
        extra = T(0);
        bcv = T(0);
        if constexpr (KIND == CK_FINE) {
            const T ec = seps[code_at(wc, m)];
            cw = face_avg(ec, seps[m == 0 ? hl : code_at(wc, m - 1)], o.ih2x);
            ce = face_avg(ec, seps[m == SEG - 1 ? hr : code_at(wc, m + 1)], o.ih2x);
            cs = face_avg(ec, seps[code_at(ws, m)], o.ih2y);
            cn = face_avg(ec, seps[code_at(wn, m)], o.ih2y);
            if (lo) cb = face_avg(ec, seps[code_at(wb, m)], o.ih2z);
            else { cb = T(0); electrode(ec, o.ih2z, o.vlo, extra, bcv); }
            if (hi) ct = face_avg(ec, seps[code_at(wt, m)], o.ih2z);
            else { ct = T(0); electrode(ec, o.ih2z, o.vhi, extra, bcv); }
        } else if constexpr (KIND == CK_PLANES) {
            cw = ce = face_beta(pw, o.ih2x);
            cs = cn = face_beta(ps, o.ih2y);
            if (lo) cb = face_beta(pb, o.ih2z);
            else { cb = T(0); electrode(pb, o.ih2z, o.vlo, extra, bcv); }
            if (hi) ct = face_beta(pt, o.ih2z);
            else { ct = T(0); electrode(pt, o.ih2z, o.vhi, extra, bcv); }
        } else {
            // face arrays, FP32 or FP16 (already converted)
            cw = face_beta(fw[m], o.ih2x);
            ce = face_beta(m == SEG - 1 ? fr : fw[m + 1], o.ih2x);
            cs = face_beta(fs[m], o.ih2y);
            cn = face_beta(fn[m], o.ih2y);
            if (lo) cb = face_beta(fb[m], o.ih2z);
            else { cb = T(0); electrode0(fb[m], o.ih2z, extra); }
            if (hi) ct = face_beta(ft[m], o.ih2z);
            else { ct = T(0); electrode0(ft[m], o.ih2z, extra); }
        }
        if (o.ny == 1) { cs = T(0); cn = T(0); }
    }
};

// the half sweep of one segment; PAR: the in-segment offset of this colour's cells
template <typename T, int SB, int KIND, bool ZERO, int PAR>
__device__ __forceinline__ void seg_update(const Op<T>& o, T* __restrict__ x, const T* __restrict__ b, int i0, int j,
                                           int k, const T* seps) {
    constexpr int SEG = SegW<T, SB>::n;
    const int row = o.nx * (j + o.ny * k);
    const int c0 = row + i0;
    int jm, jp;
    nbr(j, o.ny, jm, jp);
    const int so = (jm - j) * o.nx, no = (jp - j) * o.nx;
    const bool lo = k > 0, hi = k < o.nz - 1;
    // the x neighbour outside the segment: left of cell 0 (PAR 0) or right of cell SEG - 1 (PAR 1)
    const int il = i0 == 0 ? o.nx - 1 : i0 - 1, ir = i0 + SEG == o.nx ? 0 : i0 + SEG;
    T xc[SEG], bv[SEG];
    T xs[SEG], xn[SEG], xb[SEG], xt[SEG];
    ld_seg<T, SB>(x + c0, xc);
    ldg_seg<T, SB>(b + c0, bv);
    T xh = T(0);
    if (!ZERO) {
        xh = x[row + (PAR == 0 ? il : ir)];
        ld_seg<T, SB>(x + c0 + so, xs);
        ld_seg<T, SB>(x + c0 + no, xn);
        if (lo) ld_seg<T, SB>(x + c0 - o.nxy, xb);
        if (hi) ld_seg<T, SB>(x + c0 + o.nxy, xt);
    }
    T av[SEG];
    if (o.a) ldg_seg<T, SB>(o.a + c0, av);
    SegCoef<T, SB, KIND, PAR == 0, PAR == 1> cf;
    cf.load(o, row, c0, so, no, k, lo, hi, il, ir);
#pragma unroll
    for (int u = 0; u < SEG / 2; ++u) {
        const int m = 2 * u + PAR;
        T cw, ce, cs, cn, cb, ct, extra, bcv;
        cf.cell(o, seps, m, lo, hi, cw, ce, cs, cn, cb, ct, extra, bcv);
        const T diag = diag_sum(o.a ? av[m] : T(0), cw, ce, cs, cn, cb, ct, extra);
        if (ZERO) {
            xc[m] = sdiv(add_rn(bv[m], bcv), diag);
            xc[m ^ 1] = T(0);
            continue;
        }
        const T s = gs_rhs(bv[m], bcv, cw, m == 0 ? xh : xc[m - 1], ce, m == SEG - 1 ? xh : xc[m + 1], cs, xs[m], cn,
                           xn[m], lo, cb, xb[m], hi, ct, xt[m]);
        xc[m] = sdiv(s, diag);
    }
    st_seg<T, SB>(x + c0, xc);
}

// the residual b - A x of the SEG cells of one row segment (every cell; both
// halo cells read)
template <typename T, int SB, int KIND>
__device__ __forceinline__ void seg_resid_row(const Op<T>& o, const T* __restrict__ x, const T* __restrict__ b,
                                              int i0, int j, int k, const T* seps, T (&r)[SegW<T, SB>::n]) {
    constexpr int SEG = SegW<T, SB>::n;
    const int row = o.nx * (j + o.ny * k);
    const int c0 = row + i0;
    int jm, jp;
    nbr(j, o.ny, jm, jp);
    const int so = (jm - j) * o.nx, no = (jp - j) * o.nx;
    const bool lo = k > 0, hi = k < o.nz - 1;
    const int il = i0 == 0 ? o.nx - 1 : i0 - 1, ir = i0 + SEG == o.nx ? 0 : i0 + SEG;
    T xc[SEG], bv[SEG], xs[SEG], xn[SEG], xb[SEG], xt[SEG], av[SEG];
    ld_seg<T, SB>(x + c0, xc);
    ldg_seg<T, SB>(b + c0, bv);
    const T xl = x[row + il], xr = x[row + ir];
    ld_seg<T, SB>(x + c0 + so, xs);
    ld_seg<T, SB>(x + c0 + no, xn);
    if (lo) ld_seg<T, SB>(x + c0 - o.nxy, xb);
    if (hi) ld_seg<T, SB>(x + c0 + o.nxy, xt);
    if (o.a) ldg_seg<T, SB>(o.a + c0, av);
    SegCoef<T, SB, KIND, true, true> cf;
    cf.load(o, row, c0, so, no, k, lo, hi, il, ir);
#pragma unroll
    for (int m = 0; m < SEG; ++m) {
        T cw, ce, cs, cn, cb, ct, extra, bcv;
        cf.cell(o, seps, m, lo, hi, cw, ce, cs, cn, cb, ct, extra, bcv);
        const T diag = diag_sum(o.a ? av[m] : T(0), cw, ce, cs, cn, cb, ct, extra);
        r[m] = res_val(bv[m], bcv, diag, xc[m], cw, m == 0 ? xl : xc[m - 1], ce, m == SEG - 1 ? xr : xc[m + 1], cs,
                       xs[m], cn, xn[m], lo, cb, xb[m], hi, ct, xt[m]);
    }
}

template <typename T, int SB, int KIND, bool ZERO = false>
__global__ void __launch_bounds__(256) k_rbgs_seg(Op<T> o, T* __restrict__ x, const T* __restrict__ b, int color) {
    pdl_entry();
    __shared__ T seps[8];
    if (KIND == CK_FINE) {
        if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
            for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
        __syncthreads();
    }
    constexpr int SEG = SegW<T, SB>::n;
    // rows of the block: even offsets first, so that a warp's rows share a parity
    const int h = blockDim.y / 2;
    const int ty = threadIdx.y;
    const int j = blockIdx.y * blockDim.y + (ty < h ? 2 * ty : 2 * (ty - h) + 1);
    const int k = blockIdx.z;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * SEG;
    if (j >= o.ny) return;
    if (((j + k + color) & 1) == 0) seg_update<T, SB, KIND, ZERO, 0>(o, x, b, i0, j, k, seps);
    else seg_update<T, SB, KIND, ZERO, 1>(o, x, b, i0, j, k, seps);
}

// ---- the split (red-black) layout of level 0's FP32 arrays in the mixed path
//
// The FP32 correction x and right-hand side b of level 0 hold the cells of
// colour c = (i + j + k) & 1 at [c * N/2 + (n >> 1)], n = i + nx (j + ny k)
// the natural index (nx even: the two cells of an x pair share n >> 1, one
// of each colour).  A half sweep then reads only the other colour's values
// of its neighbours and writes only its own colour, every sector it moves
// fully used.  A thread takes 8 natural cells of a row (i0 a multiple of 8):
// its 4 cells of one colour are 16 contiguous bytes of that colour's array.

// the 8 natural-order values of cells n0 .. n0 + 7 (n0 a multiple of 8) of a
// split array; ce: the colour of the even positions
__device__ __forceinline__ void ld_split8(const float* a, int Nh, int n0, int ce, float (&v)[8]) {
    float e[4], o[4];
    ld16(a + ce * Nh + (n0 >> 1), e);
    ld16(a + (1 - ce) * Nh + (n0 >> 1), o);
#pragma unroll
    for (int u = 0; u < 4; ++u) { v[2 * u] = e[u]; v[2 * u + 1] = o[u]; }
}

// the same for 4 natural cells (n0 a multiple of 4): 8 bytes of each colour
__device__ __forceinline__ void ld_split4(const float* a, int Nh, int n0, int ce, float (&v)[4]) {
    const float2 e = *reinterpret_cast<const float2*>(a + ce * Nh + (n0 >> 1));
    const float2 o = *reinterpret_cast<const float2*>(a + (1 - ce) * Nh + (n0 >> 1));
    v[0] = e.x; v[1] = o.x; v[2] = e.y; v[3] = o.y;
}
template <int NC>
__device__ __forceinline__ void ld_splitn(const float* a, int Nh, int n0, int ce, float (&v)[NC]) {
    if constexpr (NC == 8) ld_split8(a, Nh, n0, ce, v);
    else ld_split4(a, Nh, n0, ce, v);
}

// one natural cell n of colour c
__device__ __forceinline__ float at_split(const float* a, int Nh, int n, int c) { return a[c * Nh + (n >> 1)]; }

// the half sweep of the 4 colour-`color` cells of 8 natural cells; PAR: their
// offset in the 8 (same operations as seg_update)
template <int KIND, bool ZERO, int PAR>
__device__ __forceinline__ void split_update(const Op<float>& o, float* __restrict__ x, const float* __restrict__ b,
                                             int i0, int j, int k, int color, int Nh, const float* seps) {
    const int row = o.nx * (j + o.ny * k);
    const int n0 = row + i0;
    const int m0 = n0 >> 1;
    int jm, jp;
    nbr(j, o.ny, jm, jp);
    const int so = (jm - j) * o.nx, no = (jp - j) * o.nx;
    const bool lo = k > 0, hi = k < o.nz - 1;
    const int il = i0 == 0 ? o.nx - 1 : i0 - 1, ir = i0 + 8 == o.nx ? 0 : i0 + 8;
    float* xo = x + color * Nh;            // this colour
    const float* xt = x + (1 - color) * Nh;  // the other colour: every neighbour
    float bv[4], oc[4], xs[4], xn[4], xb[4], xtp[4], av[8], nv[4];
    ld16(b + color * Nh + m0, bv);
    float xh = 0.f;
    if (!ZERO) {
        ld16(xt + m0, oc);
        xh = xt[(row + (PAR == 0 ? il : ir)) >> 1];
        ld16(xt + ((n0 + so) >> 1), xs);
        ld16(xt + ((n0 + no) >> 1), xn);
        if (lo) ld16(xt + ((n0 - o.nxy) >> 1), xb);
        if (hi) ld16(xt + ((n0 + o.nxy) >> 1), xtp);
    }
    if (o.a) {
        ldg16(o.a + n0, av);
        ldg16(o.a + n0 + 4, av + 4);
    }
    SegCoef<float, 32, KIND, PAR == 0, PAR == 1> cf;
    cf.load(o, row, n0, so, no, k, lo, hi, il, ir);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int m = 2 * u + PAR;
        float cw, ce, cs, cn, cb, ct, extra, bcv;
        cf.cell(o, seps, m, lo, hi, cw, ce, cs, cn, cb, ct, extra, bcv);
        const float diag = diag_sum(o.a ? av[m] : 0.f, cw, ce, cs, cn, cb, ct, extra);
        if (ZERO) {
            nv[u] = sdiv(add_rn(bv[u], bcv), diag);
            continue;
        }
        // the x neighbours: the other colour's cells of the 8, or the halo
        const float xw = PAR == 0 ? (u == 0 ? xh : oc[u - 1]) : oc[u];
        const float xe = PAR == 0 ? oc[u] : (u == 3 ? xh : oc[u + 1]);
        const float sum = gs_rhs(bv[u], bcv, cw, xw, ce, xe, cs, xs[u], cn, xn[u], lo, cb, xb[u], hi, ct, xtp[u]);
        nv[u] = sdiv(sum, diag);
    }
    st16(xo + m0, nv);
    if (ZERO) {
        const float z[4] = {0.f, 0.f, 0.f, 0.f};
        st16(x + (1 - color) * Nh + m0, z);
    }
}

template <int KIND, bool ZERO = false>
__global__ void __launch_bounds__(256) k_rbgs_split(Op<float> o, float* __restrict__ x, const float* __restrict__ b,
                                                    int color, int Nh) {
    pdl_entry();
    __shared__ float seps[8];
    if (KIND == CK_FINE) {
        if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
            for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
        __syncthreads();
    }
    // rows of the block: even offsets first, so that a warp's rows share a parity
    const int h = blockDim.y / 2;
    const int ty = threadIdx.y;
    const int j = blockIdx.y * blockDim.y + (ty < h ? 2 * ty : 2 * (ty - h) + 1);
    const int k = blockIdx.z;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 8;
    if (j >= o.ny) return;
    if (((j + k + color) & 1) == 0) split_update<KIND, ZERO, 0>(o, x, b, i0, j, k, color, Nh, seps);
    else split_update<KIND, ZERO, 1>(o, x, b, i0, j, k, color, Nh, seps);
}

// red-black z-line Gauss-Seidel half sweep: color = parity of i + j; each
// thread solves the tridiagonal system of one column (Thomas), q holds the
// forward-elimination ratios
template <typename T, int KIND>
__global__ void __launch_bounds__(128) k_line(Op<T> o, T* __restrict__ x, const T* __restrict__ b, T* __restrict__ q,
                                              int color) {
    pdl_entry();
    __shared__ T seps[8];
    if (KIND == CK_FINE) {
        if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
            for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
        __syncthreads();
    }
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((j + color) & 1);
    if (j >= o.ny || i >= o.nx) return;
    int im, ip, jm, jp;
    nbr(i, o.nx, im, ip);
    nbr(j, o.ny, jm, jp);
    T qprev = T(0), dprev = T(0);
    int c = i + o.nx * j;
    for (int k = 0; k < o.nz; ++k, c += o.nxy) {
        T cw, ce, cs, cn, cb, ct, diag, bcv;
        coeffs<T, KIND>(o, i, j, k, c, im, ip, jm, jp, cw, ce, cs, cn, cb, ct, diag, bcv, seps);
        const int row = c - i;
        const T r = b[c] + bcv + cw * x[row + im] + ce * x[row + ip] + cs * x[c + (jm - j) * o.nx] +
                    cn * x[c + (jp - j) * o.nx];
        const T den = diag - cb * qprev;
        const T qk = ct / den;
        const T dk = (r + cb * dprev) / den;
        q[c] = qk;
        x[c] = dk;
        qprev = qk;
        dprev = dk;
    }
    c -= o.nxy;   // top cell
    T xn = x[c];
    for (int k = o.nz - 2; k >= 0; --k) {
        c -= o.nxy;
        xn = x[c] + q[c] * xn;
        x[c] = xn;
    }
}

// residual b - A x at the children of each coarse cell, averaged into the
// coarse right-hand side; optionally the |r|_inf of the level.  RX, RY, RZ
// are the coarsening ratios (1 or 2).
// residual b - A x at the children of coarse cell (I, J, K), averaged into
// bc; returns the largest |r| among them
template <typename T, int KIND, int RX, int RY, int RZ>
__device__ __forceinline__ double rr_cell(const Op<T>& o, const T* __restrict__ x, const T* __restrict__ b,
                                          T* __restrict__ bc, int I, int J, int K, int ncx, int ncy, const T* seps) {
    double mx = 0.0;
    T s = T(0);
#pragma unroll
    for (int dk = 0; dk < RZ; ++dk)
#pragma unroll
        for (int dj = 0; dj < RY; ++dj)
#pragma unroll
            for (int di = 0; di < RX; ++di) {
                const int i = RX * I + di, j = RY * J + dj, k = RZ * K + dk;
                const int c = i + o.nx * (j + o.ny * k);
                int im, ip, jm, jp;
                nbr(i, o.nx, im, ip);
                nbr(j, o.ny, jm, jp);
                T cw, ce, cs, cn, cb, ct, diag, bcv;
                coeffs<T, KIND>(o, i, j, k, c, im, ip, jm, jp, cw, ce, cs, cn, cb, ct, diag, bcv, seps);
                const int row = c - i;
                const bool lo = k > 0, hi = k < o.nz - 1;
                const T r = res_val(b[c], bcv, diag, x[c], cw, x[row + im], ce, x[row + ip], cs, x[c + (jm - j) * o.nx],
                                    cn, x[c + (jp - j) * o.nx], lo, cb, lo ? x[c - o.nxy] : T(0), hi, ct,
                                    hi ? x[c + o.nxy] : T(0));
                s = add_rn(s, r);
                mx = nan_max(mx, fabs((double)r));
            }
    bc[I + ncx * (J + ncy * K)] = s / T(RX * RY * RZ);
    return mx;
}

// residual b - A x at the children of each coarse cell, averaged into the
// coarse right-hand side; optionally the |r|_inf of the level.  RX, RY, RZ
// are the coarsening ratios (1 or 2).
template <typename T, int KIND, int RX, int RY, int RZ>
__global__ void __launch_bounds__(256) k_resid_restrict(Op<T> o, const T* __restrict__ x, const T* __restrict__ b,
                                                        T* __restrict__ bc, int ncx, int ncy, int ncz,
                                                        double* __restrict__ norm) {
    pdl_entry();
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    const int K = blockIdx.z;
    __shared__ T seps[8];
    if (KIND == CK_FINE) {
        if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
            for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
        __syncthreads();
    }
    double mx = 0.0;
    if (I < ncx && J < ncy) mx = rr_cell<T, KIND, RX, RY, RZ>(o, x, b, bc, I, J, K, ncx, ncy, seps);
    if (norm) {
        const double m = block_max_all(mx);
        const int slot = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) & (NORM_SLOTS - 1);
        if (threadIdx.x == 0 && threadIdx.y == 0) atomic_max_nonneg(norm + slot, m);
    }
}

// FP64 residual of the level-0 operator with electrode terms; optional FP32
// copy for the mixed-precision correction solve.  With CORR the iterate is
// x + e (the FP32 correction added in FP64, at every stencil point) and is
// written to xout (out of place), so the update and the next residual take one
// pass.  Each thread walks R64_ZP
// consecutive cells of its z column, carrying the column's x and code values
// from one cell to the next (the coefficients are those of coeffs<double,
// true>, same operations); block maxima go to NORM_SLOTS spread slots.
constexpr int R64_ZP = 4;

// the loop test of a device-controlled solve on a residual norm (one thread):
// the max of the norm slots, which are left zeroed for their next user
__device__ void resid_ctl(const ResidCtl& rc, double* slots) {
    double rn = 0.0;
    for (int q = 0; q < NORM_SLOTS; ++q) {
        const double v = __ldcg(slots + q);
        rn = rn < v ? v : rn;
        slots[q] = 0.0;
    }
    StepCtl* ctl = rc.ctl;
    if (rc.mode == RC_BEGIN) {
        // the solve's target from the right-hand side norms, and the first test
        const double r = rc.rtol < 1e-16 ? 1e-16 : rc.rtol;
        const double m = rc.nb[0] < rc.nb[1] ? rc.nb[1] : rc.nb[0];
        const double target = r * m;
        ctl->target = target;
        ctl->rn = rn;
        ctl->it = 0;
        ctl->parity = 0;
        cudaGraphSetConditional(rc.h, (!(rn <= target) && isfinite(rn) && 0 < rc.maxit) ? 1u : 0u);
    } else if (rc.mode == RC_RN) {
        // the exact residual after a V-cycle
        ctl->rn = rn;
        cudaGraphSetConditional(rc.h, (!(rn <= ctl->target) && isfinite(rn) && ctl->it < rc.maxit) ? 1u : 0u);
    } else {
        // a mixed refinement step: `inner` FP32 cycles spent; h is the
        // condition of the next step in the same body (the IF node) or the
        // loop's own, h2 the loop's
        ctl->nexec[rc.kind] += 1;
        const int it = ctl->it + rc.inner;
        ctl->rn = rn;
        ctl->it = it;
        ctl->parity = rc.parity;
        cudaGraphSetConditional(rc.h, (!(rn <= ctl->target) && isfinite(rn) && it < rc.maxit) ? 1u : 0u);
        if (rc.h2 != rc.h) cudaGraphSetConditional(rc.h2, 0u);
    }
}

template <bool CORR, int KIND = CK_FINE>
__global__ void __launch_bounds__(256) k_resid64(Op<double> o, const double* __restrict__ x, const float* __restrict__ e,
                                                 const double* __restrict__ b, double* __restrict__ xout,
                                                 float* __restrict__ r32, double* __restrict__ norm, ResidCtl rc) {
    pdl_entry();
    // a step graph's exact residual after a V-cycle, not needed this time
    if (rc.mode == RC_RN && !rc.ctl->need) return;
    auto X = [&](int n) -> double { return CORR ? add_rn(x[n], (double)e[n]) : x[n]; };
    __shared__ double seps[8];
    if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
        for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = blockIdx.z * R64_ZP;
    double mx = 0.0;
    if (i < o.nx && j < o.ny) {
        int im, ip, jm, jp;
        nbr(i, o.nx, im, ip);
        nbr(j, o.ny, jm, jp);
        const int col = i + o.nx * j;
        const int row = col - i;
        const int dso = (jm - j) * o.nx, dno = (jp - j) * o.nx;
        const uint8_t* cd = o.code + o.nxy;   // the k = -1 ghost layer is cd - nxy
        double xm = k0 > 0 ? X(col + o.nxy * (k0 - 1)) : 0.0;
        double xc = X(col + o.nxy * k0);
        double em = KIND == CK_PLANES ? 0.0 : seps[__ldg(cd + col + o.nxy * (k0 - 1)) & 7];
        double ec = KIND == CK_PLANES ? 0.0 : seps[__ldg(cd + col + o.nxy * k0) & 7];
#pragma unroll
        for (int q = 0; q < R64_ZP; ++q) {
            const int k = k0 + q;
            if (k >= o.nz) break;
            const int c = col + o.nxy * k;
            const double xp = k < o.nz - 1 ? X(c + o.nxy) : 0.0;
            double extra = 0.0, bcv = 0.0, cb, ct, cw, ce, cs, cn;
            double ep = 0.0;
            if constexpr (KIND == CK_PLANES) {
                // a layered stack: the same face values per z plane, as the
                // setup formed them from the codes (same operations)
                cw = ce = face_beta(__ldg(o.zc + k), o.ih2x);
                cs = cn = face_beta(__ldg(o.zc + o.nz + k), o.ih2y);
                const double fb = __ldg(o.zc + 2 * o.nz + k), ft = __ldg(o.zc + 2 * o.nz + k + 1);
                if (k > 0) cb = face_beta(fb, o.ih2z);
                else { cb = 0.0; electrode(fb, o.ih2z, o.vlo, extra, bcv); }
                if (k < o.nz - 1) ct = face_beta(ft, o.ih2z);
                else { ct = 0.0; electrode(ft, o.ih2z, o.vhi, extra, bcv); }
            } else {
                ep = seps[__ldg(cd + c + o.nxy) & 7];
                cw = face_avg(ec, seps[__ldg(cd + row + o.nxy * k + im) & 7], o.ih2x);
                ce = face_avg(ec, seps[__ldg(cd + row + o.nxy * k + ip) & 7], o.ih2x);
                cs = face_avg(ec, seps[__ldg(cd + c + dso) & 7], o.ih2y);
                cn = face_avg(ec, seps[__ldg(cd + c + dno) & 7], o.ih2y);
                if (k > 0) cb = face_avg(ec, em, o.ih2z);
                else { cb = 0.0; electrode(ec, o.ih2z, o.vlo, extra, bcv); }
                if (k < o.nz - 1) ct = face_avg(ec, ep, o.ih2z);
                else { ct = 0.0; electrode(ec, o.ih2z, o.vhi, extra, bcv); }
            }
            if (o.nx == 1) { cw = 0.0; ce = 0.0; }
            if (o.ny == 1) { cs = 0.0; cn = 0.0; }
            const double diag = diag_sum(o.a ? o.a[c] : 0.0, cw, ce, cs, cn, cb, ct, extra);
            const int rk = row + o.nxy * k;
            const double r = res_val(b[c], bcv, diag, xc, cw, X(rk + im), ce, X(rk + ip), cs, X(c + dso), cn, X(c + dno),
                                     k > 0, cb, xm, k < o.nz - 1, ct, xp);
            if (r32) r32[c] = (float)r;
            if (CORR) xout[c] = xc;
            mx = nan_max(mx, fabs(r));
            xm = xc; xc = xp;
            em = ec; ec = ep;
        }
    }
    const double m = block_max_all(mx);
    const int slot = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) & (NORM_SLOTS - 1);
    if (threadIdx.x == 0 && threadIdx.y == 0) atomic_max_nonneg(norm + slot, m);
    if (rc.ctl) {
        // a step graph: the last block tests the solve's loop on the norm
        __shared__ bool last;
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            __threadfence();
            last = atomicAdd(rc.counter, 1u) == gridDim.x * gridDim.y * gridDim.z - 1;
        }
        __syncthreads();
        if (last && threadIdx.x == 0 && threadIdx.y == 0) {
            __threadfence();
            resid_ctl(rc, norm);
            *rc.counter = 0;
        }
    }
}

// the FP32 copies of a segment's residuals (SEG floats: 8 or 16 bytes)
template <int SEG>
__device__ __forceinline__ void st_r32(float* p, const double (&r)[SEG]) {
    if constexpr (SEG == 2) {
        *reinterpret_cast<float2*>(p) = make_float2((float)r[0], (float)r[1]);
    } else {
        float v[4] = {(float)r[0], (float)r[1], (float)r[2], (float)r[3]};
        asm volatile("st.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3])
                     : "memory");
    }
}

// the iterate of a segment: x, or x + e (the FP32 correction added in FP64);
// SPLIT: e in the split layout of level 0 (4 cells: the two of colour ce at
// even positions, the two of the other colour at odd ones, 8 bytes each)
template <bool CORR, int SB, bool SPLIT = false>
__device__ __forceinline__ void ld_iter(const double* x, const float* e, int c, double (&v)[SegW<double, SB>::n],
                                        int ce = 0, int Nh = 0) {
    constexpr int SEG = SegW<double, SB>::n;
    ldg_seg<double, SB>(x + c, v);
    if constexpr (CORR) {
        float f[SEG];
        if constexpr (SPLIT) {
            static_assert(SEG == 4, "split rows of 4 cells");
            const float2 a = __ldg(reinterpret_cast<const float2*>(e + ce * Nh + (c >> 1)));
            const float2 q = __ldg(reinterpret_cast<const float2*>(e + (1 - ce) * Nh + (c >> 1)));
            f[0] = a.x; f[1] = q.x; f[2] = a.y; f[3] = q.y;
        } else if constexpr (SEG == 2) {
            const float2 q = __ldg(reinterpret_cast<const float2*>(e + c));
            f[0] = q.x; f[1] = q.y;
        } else {
            ldg16(e + c, f);
        }
#pragma unroll
        for (int m = 0; m < SEG; ++m) v[m] = add_rn(v[m], (double)f[m]);
    }
}

// the FP32 copies of 4 residuals into the split layout (colour ce at the even positions)
__device__ __forceinline__ void st_r32_split(float* p, int c, int ce, int Nh, const double (&r)[4]) {
    *reinterpret_cast<float2*>(p + ce * Nh + (c >> 1)) = make_float2((float)r[0], (float)r[2]);
    *reinterpret_cast<float2*>(p + (1 - ce) * Nh + (c >> 1)) = make_float2((float)r[1], (float)r[3]);
}

// k_resid64 by row segments: each thread takes one SB-byte segment of a row
// (2 or 4 cells) through R64_ZP consecutive planes, the iterate of the planes
// k - 1, k, k + 1 carried in registers.  Same operations per cell as
// k_resid64, so the same bits.
template <bool CORR, int KIND, int SB, bool SPLIT = false>
__global__ void __launch_bounds__(256) k_resid64_seg(Op<double> o, const double* __restrict__ x,
                                                     const float* __restrict__ e, const double* __restrict__ b,
                                                     double* __restrict__ xout, float* __restrict__ r32,
                                                     double* __restrict__ norm, ResidCtl rc, int Nh) {
    pdl_entry();
    if (rc.mode == RC_RN && !rc.ctl->need) return;
    constexpr int SEG = SegW<double, SB>::n;
    __shared__ double seps[8];
    if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
        for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
    __syncthreads();
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * SEG;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = blockIdx.z * R64_ZP;
    double mx = 0.0;
    if (j < o.ny) {
        int jm, jp;
        nbr(j, o.ny, jm, jp);
        const int so = (jm - j) * o.nx, no = (jp - j) * o.nx;
        const int il = i0 == 0 ? o.nx - 1 : i0 - 1, ir = i0 + SEG == o.nx ? 0 : i0 + SEG;
        // one cell n of x (+ e), cl: its colour (the split layout's array)
        auto X = [&](int n, int cl) -> double {
            if (!CORR) return __ldg(x + n);
            return add_rn(__ldg(x + n), (double)__ldg(SPLIT ? e + cl * Nh + (n >> 1) : e + n));
        };
        double xm[SEG], xc[SEG], xp[SEG];
        const int col = i0 + o.nx * j;
        // the colour of a row's even positions at plane kk (i0 is even)
        auto cev = [&](int jj, int kk) { return (jj + kk) & 1; };
        if (k0 > 0) ld_iter<CORR, SB, SPLIT>(x, e, col + o.nxy * (k0 - 1), xm, cev(j, k0 - 1), Nh);
        ld_iter<CORR, SB, SPLIT>(x, e, col + o.nxy * k0, xc, cev(j, k0), Nh);
#pragma unroll
        for (int q = 0; q < R64_ZP; ++q) {
            const int k = k0 + q;
            if (k >= o.nz) break;
            const int row = o.nx * (j + o.ny * k);
            const int c0 = row + i0;
            const bool lo = k > 0, hi = k < o.nz - 1;
            if (hi) ld_iter<CORR, SB, SPLIT>(x, e, c0 + o.nxy, xp, cev(j, k + 1), Nh);
            double xs[SEG], xn[SEG], bv[SEG], av[SEG];
            ld_iter<CORR, SB, SPLIT>(x, e, c0 + so, xs, cev(j + 1, k), Nh);
            ld_iter<CORR, SB, SPLIT>(x, e, c0 + no, xn, cev(j + 1, k), Nh);
            // the halo cells: il is odd, ir even (nx even)
            const double xl = X(row + il, 1 - cev(j, k)), xr = X(row + ir, cev(j, k));
            ldg_seg<double, SB>(b + c0, bv);
            if (o.a) ldg_seg<double, SB>(o.a + c0, av);
            SegCoef<double, SB, KIND, true, true> cf;
            cf.load(o, row, c0, so, no, k, lo, hi, il, ir);
            double r[SEG];
#pragma unroll
            for (int m = 0; m < SEG; ++m) {
                double cw, ce, cs, cn, cb, ct, extra, bcv;
                cf.cell(o, seps, m, lo, hi, cw, ce, cs, cn, cb, ct, extra, bcv);
                const double diag = diag_sum(o.a ? av[m] : 0.0, cw, ce, cs, cn, cb, ct, extra);
                r[m] = res_val(bv[m], bcv, diag, xc[m], cw, m == 0 ? xl : xc[m - 1], ce, m == SEG - 1 ? xr : xc[m + 1],
                               cs, xs[m], cn, xn[m], lo, cb, xm[m], hi, ct, xp[m]);
                mx = nan_max(mx, fabs(r[m]));
            }
            if (r32) {
                if constexpr (SPLIT) st_r32_split(r32, c0, cev(j, k), Nh, r);
                else st_r32<SEG>(r32 + c0, r);
            }
            if (CORR) st_seg<double, SB>(xout + c0, xc);
#pragma unroll
            for (int m = 0; m < SEG; ++m) { xm[m] = xc[m]; xc[m] = xp[m]; }
        }
    }
    const double m = block_max_all(mx);
    const int slot = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) & (NORM_SLOTS - 1);
    if (threadIdx.x == 0 && threadIdx.y == 0) atomic_max_nonneg(norm + slot, m);
    if (rc.ctl) {
        // a step graph: the last block tests the solve's loop on the norm
        __shared__ bool last;
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            __threadfence();
            last = atomicAdd(rc.counter, 1u) == gridDim.x * gridDim.y * gridDim.z - 1;
        }
        __syncthreads();
        if (last && threadIdx.x == 0 && threadIdx.y == 0) {
            __threadfence();
            resid_ctl(rc, norm);
            *rc.counter = 0;
        }
    }
}

// k_resid64 with the face coefficients by plane when level 0 has them; by
// row segments of sb = 32 bytes where level 0's rows and the arrays'
// alignment allow (sb = 0: one column of cells per thread)
template <bool CORR>
void launch_resid64(const Op<double>& o, dim3 g, dim3 b, cudaStream_t s, const double* x, const float* e,
                    const double* rhs, double* xout, float* r32, double* norm, const ResidCtl& rc, int sb = 0,
                    bool split = false) {
    if (sb == 32) {
        const int seg = sb / 8;
        const int gx = o.nx / seg;
        auto al = [](const void* p, uintptr_t a) { return ((uintptr_t)p % a) == 0; };
        const bool ok = o.nx % seg == 0 && (gx % 32 == 0 || 32 % gx == 0) && al(x, 16) && al(rhs, 16) && al(o.a, 16) &&
                        al(e, 4 * seg) && al(xout, 16) && al(r32, 4 * seg) && (o.zc || al(o.code + o.nxy, seg));
        if (ok) {
            const int bx = gx < 32 ? gx : 32, by = 256 / bx;
            dim3 bs(bx, by), gs(gx / bx, (o.ny + by - 1) / by, (o.nz + R64_ZP - 1) / R64_ZP);
            const int Nh = (o.nxy * o.nz) / 2;
            if (split) {
                if (o.zc) launch_k(k_resid64_seg<CORR, CK_PLANES, 32, true>, gs, bs, 0, s, o, x, e, rhs, xout, r32, norm, rc, Nh);
                else launch_k(k_resid64_seg<CORR, CK_FINE, 32, true>, gs, bs, 0, s, o, x, e, rhs, xout, r32, norm, rc, Nh);
            } else {
                if (o.zc) launch_k(k_resid64_seg<CORR, CK_PLANES, 32>, gs, bs, 0, s, o, x, e, rhs, xout, r32, norm, rc, Nh);
                else launch_k(k_resid64_seg<CORR, CK_FINE, 32>, gs, bs, 0, s, o, x, e, rhs, xout, r32, norm, rc, Nh);
            }
            return;
        }
    }
    if (o.zc) launch_k(k_resid64<CORR, CK_PLANES>, g, b, 0, s, o, x, e, rhs, xout, r32, norm, rc);
    else launch_k(k_resid64<CORR, CK_FINE>, g, b, 0, s, o, x, e, rhs, xout, r32, norm, rc);
}

// prolongation in the coarsened directions with the per-cell resistor-chain
// weights (near parent, far neighbour), added to x; beyond an electrode the
// far neighbour is the homogeneous Dirichlet value 0.  RX, RY, RZ are the
// coarsening ratios (1 or 2), fixed at compile time.
// the z-only prolongation of one fine cell: (1 - w) x(K0) + w x(K1), the far
// term absent beyond an electrode (roundings written out: both launch forms
// give the same bits)
template <typename T>
__device__ __forceinline__ T prolong_z_val(T w, T x0, T x1, bool zin) {
    const T t0 = mul_rn(add_rn(T(1), -w), x0);
    return zin ? fma_rn(w, x1, t0) : t0;
}

template <typename T, int RX, int RY, int RZ>
__device__ __forceinline__ void prolong_cell(T* __restrict__ xf, const T* __restrict__ xc, const float* __restrict__ wx,
                                             const float* __restrict__ wy, const float* __restrict__ wz, int i, int j,
                                             int k, int nx, int ny, int nz, int ncx, int ncy, int ncz) {
    if (i >= nx || j >= ny) return;
    const int fc = i + nx * (j + ny * k);
    const int I0 = RX == 2 ? (i >> 1) : i, J0 = RY == 2 ? (j >> 1) : j, K0 = RZ == 2 ? (k >> 1) : k;
    int I1 = I0, J1 = J0, K1 = K0;
    T wxf = T(0), wyf = T(0), wzf = T(0);
    if (RX == 2) { wxf = T(__ldg(wx + fc)); I1 = (i & 1) ? (I0 + 1 == ncx ? 0 : I0 + 1) : (I0 == 0 ? ncx - 1 : I0 - 1); }
    if (RY == 2) { wyf = T(__ldg(wy + fc)); J1 = (j & 1) ? (J0 + 1 == ncy ? 0 : J0 + 1) : (J0 == 0 ? ncy - 1 : J0 - 1); }
    bool zin = true;
    if (RZ == 2) {
        wzf = T(__ldg(wz + fc));
        K1 = (k & 1) ? K0 + 1 : K0 - 1;
        zin = K1 >= 0 && K1 < ncz;
        if (!zin) K1 = K0;
    }
    const int ncxy = ncx * ncy;
    auto X = [&](int I, int J, int K) { return xc[I + ncx * J + ncxy * K]; };
    T s;
    if (RX == 2 && RY == 2 && RZ == 2) {
        const T wxn = T(1) - wxf, wyn = T(1) - wyf, wzn = T(1) - wzf, wzf2 = zin ? wzf : T(0);
        s = wzn * (wyn * (wxn * X(I0, J0, K0) + wxf * X(I1, J0, K0)) + wyf * (wxn * X(I0, J1, K0) + wxf * X(I1, J1, K0))) +
            wzf2 * (wyn * (wxn * X(I0, J0, K1) + wxf * X(I1, J0, K1)) + wyf * (wxn * X(I0, J1, K1) + wxf * X(I1, J1, K1)));
    } else if (RX == 2 && RY == 2) {
        const T wxn = T(1) - wxf, wyn = T(1) - wyf;
        s = wyn * (wxn * X(I0, J0, K0) + wxf * X(I1, J0, K0)) + wyf * (wxn * X(I0, J1, K0) + wxf * X(I1, J1, K0));
    } else if (RZ == 2 && RX == 1 && RY == 1) {
        s = prolong_z_val(wzf, X(I0, J0, K0), X(I0, J0, K1), zin);
    } else {
        // remaining ratio patterns (single x or y direction, x-z, y-z)
        T acc = T(0);
        for (int a = 0; a < (RZ == 2 ? 2 : 1); ++a) {
            const T wk = RZ == 2 ? (a ? (zin ? wzf : T(0)) : T(1) - wzf) : T(1);
            const int K = a ? K1 : K0;
            for (int b = 0; b < (RY == 2 ? 2 : 1); ++b) {
                const T wj = RY == 2 ? (b ? wyf : T(1) - wyf) : T(1);
                const int J = b ? J1 : J0;
                for (int d = 0; d < (RX == 2 ? 2 : 1); ++d) {
                    const T wi = RX == 2 ? (d ? wxf : T(1) - wxf) : T(1);
                    acc += wk * wj * wi * X(d ? I1 : I0, J, K);
                }
            }
        }
        s = acc;
    }
    xf[fc] = RZ == 2 && RX == 1 && RY == 1 ? add_rn(xf[fc], s) : xf[fc] + s;
}

// the coarse correction interpolated into the finer level and added
template <typename T, int RX, int RY, int RZ>
__global__ void __launch_bounds__(256) k_prolong(T* __restrict__ xf, const T* __restrict__ xc, const float* __restrict__ wx,
                                                 const float* __restrict__ wy, const float* __restrict__ wz, int nx, int ny,
                                                 int nz, int ncx, int ncy, int ncz) {
    pdl_entry();
    prolong_cell<T, RX, RY, RZ>(xf, xc, wx, wy, wz, blockIdx.x * blockDim.x + threadIdx.x,
                                blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z, nx, ny, nz, ncx, ncy, ncz);
}

// ---- row-segment forms of the z-semicoarsening transfers (ratios 1, 1, 2),
// one 16- or 32-byte segment of a row per thread, as k_rbgs_seg

// residual at the two fine cells of each coarse cell of a segment (fine
// planes 2K and 2K + 1, same x and y), averaged into the coarse right-hand
// side; optionally the |r|_inf of the level.  Same operations as
// k_resid_restrict<T, KIND, 1, 1, 2>.
template <typename T, int SB, int KIND>
__global__ void __launch_bounds__(256) k_rr_z_seg(Op<T> o, const T* __restrict__ x, const T* __restrict__ b,
                                                  T* __restrict__ bc, double* __restrict__ norm) {
    pdl_entry();
    __shared__ T seps[8];
    if (KIND == CK_FINE) {
        if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
            for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
        __syncthreads();
    }
    constexpr int SEG = SegW<T, SB>::n;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * SEG;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int K = blockIdx.z;
    double mx = 0.0;
    if (j < o.ny) {
        T acc[SEG], r[SEG];
#pragma unroll
        for (int m = 0; m < SEG; ++m) acc[m] = T(0);
#pragma unroll
        for (int dk = 0; dk < 2; ++dk) {
            seg_resid_row<T, SB, KIND>(o, x, b, i0, j, 2 * K + dk, seps, r);
#pragma unroll
            for (int m = 0; m < SEG; ++m) {
                acc[m] = add_rn(acc[m], r[m]);
                mx = nan_max(mx, fabs((double)r[m]));
            }
        }
#pragma unroll
        for (int m = 0; m < SEG; ++m) acc[m] = acc[m] / T(2);
        st_seg<T, SB>(bc + i0 + o.nx * (j + o.ny * K), acc);
    }
    if (norm) {
        const double m = block_max_all(mx);
        const int slot = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) & (NORM_SLOTS - 1);
        if (threadIdx.x == 0 && threadIdx.y == 0) atomic_max_nonneg(norm + slot, m);
    }
}

// the z-only prolongation of a row segment of fine plane k, added to xf
// (same operations as k_prolong<T, 1, 1, 2>)
template <typename T, int SB>
__global__ void __launch_bounds__(256) k_prolong_z_seg(T* __restrict__ xf, const T* __restrict__ xc,
                                                       const float* __restrict__ wz, int nx, int ny, int ncz) {
    pdl_entry();
    constexpr int SEG = SegW<T, SB>::n;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * SEG;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (j >= ny) return;
    const int K0 = k >> 1;
    int K1 = (k & 1) ? K0 + 1 : K0 - 1;
    const bool zin = K1 >= 0 && K1 < ncz;
    if (!zin) K1 = K0;
    const int fc = i0 + nx * (j + ny * k);
    const int cc = i0 + nx * j;
    T v[SEG], x0[SEG], x1[SEG];
    float w[SEG];
    ld_seg<T, SB>(xf + fc, v);
    ldg_seg<T, SB>(xc + cc + nx * ny * K0, x0);
    if (zin) ldg_seg<T, SB>(xc + cc + nx * ny * K1, x1);
    if constexpr (SEG == 4) {
        ldg16(wz + fc, w);
    } else if constexpr (SEG == 8) {
        ldg16(wz + fc, w);
        ldg16(wz + fc + 4, w + 4);
    } else {
        const float2 q = __ldg(reinterpret_cast<const float2*>(wz + fc));
        w[0] = q.x; w[1] = q.y;
    }
#pragma unroll
    for (int m = 0; m < SEG; ++m) v[m] = add_rn(v[m], prolong_z_val(T(w[m]), x0[m], zin ? x1[m] : T(0), zin));
    st_seg<T, SB>(xf + fc, v);
}

// the residual of NC = 4 or 8 natural cells of a row of level 0 with x and b
// in the split layout (same operations as seg_resid_row)
template <int KIND, int NC>
__device__ __forceinline__ void split_resid_row(const Op<float>& o, const float* __restrict__ x,
                                                const float* __restrict__ b, int i0, int j, int k, int Nh,
                                                const float* seps, float (&r)[NC]) {
    const int row = o.nx * (j + o.ny * k);
    const int n0 = row + i0;
    int jm, jp;
    nbr(j, o.ny, jm, jp);
    const int so = (jm - j) * o.nx, no = (jp - j) * o.nx;
    const bool lo = k > 0, hi = k < o.nz - 1;
    const int il = i0 == 0 ? o.nx - 1 : i0 - 1, ir = i0 + NC == o.nx ? 0 : i0 + NC;
    const int ce = (j + k) & 1;   // colour of the even positions (i0 is even)
    float xc[NC], bv[NC], xs[NC], xn[NC], xb[NC], xt[NC], av[NC];
    ld_splitn<NC>(x, Nh, n0, ce, xc);
    ld_splitn<NC>(b, Nh, n0, ce, bv);
    const float xl = at_split(x, Nh, row + il, 1 - ce), xr = at_split(x, Nh, row + ir, ce);
    ld_splitn<NC>(x, Nh, n0 + so, 1 - ce, xs);
    ld_splitn<NC>(x, Nh, n0 + no, 1 - ce, xn);
    if (lo) ld_splitn<NC>(x, Nh, n0 - o.nxy, 1 - ce, xb);
    if (hi) ld_splitn<NC>(x, Nh, n0 + o.nxy, 1 - ce, xt);
    if (o.a) {
        ldg16(o.a + n0, av);
        if constexpr (NC == 8) ldg16(o.a + n0 + 4, av + 4);
    }
    SegCoef<float, 4 * NC, KIND, true, true> cf;
    cf.load(o, row, n0, so, no, k, lo, hi, il, ir);
#pragma unroll
    for (int m = 0; m < NC; ++m) {
        float cw, ce_, cs, cn, cb, ct, extra, bcv;
        cf.cell(o, seps, m, lo, hi, cw, ce_, cs, cn, cb, ct, extra, bcv);
        const float diag = diag_sum(o.a ? av[m] : 0.f, cw, ce_, cs, cn, cb, ct, extra);
        r[m] = res_val(bv[m], bcv, diag, xc[m], cw, m == 0 ? xl : xc[m - 1], ce_, m == NC - 1 ? xr : xc[m + 1], cs,
                       xs[m], cn, xn[m], lo, cb, xb[m], hi, ct, xt[m]);
    }
}

// level 0 -> 1 z-semicoarsening restriction from the split layout: 4 coarse
// cells of a row per thread, written in the natural layout of level 1 (same
// operations as k_rr_z_seg)
template <int KIND>
__global__ void __launch_bounds__(256) k_rr_z_split(Op<float> o, const float* __restrict__ x,
                                                    const float* __restrict__ b, float* __restrict__ bc, int Nh) {
    pdl_entry();
    __shared__ float seps[8];
    if (KIND == CK_FINE) {
        if (threadIdx.x == 0 && threadIdx.y == 0)
#pragma unroll
            for (int q = 0; q < 8; ++q) seps[q] = o.eps[q];
        __syncthreads();
    }
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int K = blockIdx.z;
    if (j >= o.ny) return;
    float acc[4], r[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.f;
#pragma unroll
    for (int dk = 0; dk < 2; ++dk) {
        split_resid_row<KIND, 4>(o, x, b, i0, j, 2 * K + dk, Nh, seps, r);
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = add_rn(acc[m], r[m]);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = acc[m] / 2.f;
    st16(bc + i0 + o.nx * (j + o.ny * K), acc);
}

// level 1 -> 0 z-only prolongation into the split layout: 8 natural fine
// cells per thread (same operations as k_prolong_z_seg)
__global__ void __launch_bounds__(256) k_prolong_z_split(float* __restrict__ xf, const float* __restrict__ xc,
                                                         const float* __restrict__ wz, int nx, int ny, int ncz,
                                                         int Nh) {
    pdl_entry();
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 8;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (j >= ny) return;
    const int K0 = k >> 1;
    int K1 = (k & 1) ? K0 + 1 : K0 - 1;
    const bool zin = K1 >= 0 && K1 < ncz;
    if (!zin) K1 = K0;
    const int n0 = i0 + nx * (j + ny * k);
    const int cc = i0 + nx * j;
    const int ce = (j + k) & 1;
    float v[8], x0[8], x1[8], w[8];
    ld_split8(xf, Nh, n0, ce, v);
    ldg16(xc + cc + nx * ny * K0, x0);
    ldg16(xc + cc + nx * ny * K0 + 4, x0 + 4);
    if (zin) {
        ldg16(xc + cc + nx * ny * K1, x1);
        ldg16(xc + cc + nx * ny * K1 + 4, x1 + 4);
    }
    ldg16(wz + n0, w);
    ldg16(wz + n0 + 4, w + 4);
    float e[4], o[4];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const float t = add_rn(v[m], prolong_z_val(w[m], x0[m], zin ? x1[m] : 0.f, zin));
        if (m & 1) o[m >> 1] = t;
        else e[m >> 1] = t;
    }
    st16(xf + ce * Nh + (n0 >> 1), e);
    st16(xf + (1 - ce) * Nh + (n0 >> 1), o);
}

// ---------------------------------------------------------------------
// The small levels of the hierarchy in one CTA: every array of the levels
// from `top` down to the bottom lives in shared memory, and one launch runs
// their whole V-cycle (smoothing, restriction, prolongation, exact bottom
// line solve) with __syncthreads() between phases instead of one kernel
// launch per phase.
constexpr int MAXLEV = 24;
static_assert(MAXLEV == Multigrid::kMaxLev, "level tables");

struct CoarseLevelDesc {
    int nx, ny, nz, N, rx, ry, rz, line;   // r*: ratio to the next (coarser) level
    double ihx, ihy, ihz;
    long long ox, ob, obw, obs, obb, oa, oq, oi, op;   // offsets (elements of T) in shared memory
    long long ow[3];                            // offsets (floats) of the prolongation weights into this level
    const void* gbw;
    const void* gbs;
    const void* gbb;
    const void* ga;
    const float* gw[3];
    void* gf[3];                                // global copies of q, 1/pivot, cb/pivot
};

struct CoarseArgs {
    int nlev;
    int nu1, nu2, nu_bottom;
    long long wbase;                 // byte offset of the float region
    const void* b_in;                // right-hand side of the top level (global)
    void* x_out;                     // solution of the top level (global)
    int* fvalid;                     // the factors in gf are current (else computed and stored)
    CoarseLevelDesc L[MAXLEV];
};

template <typename T>
struct SV {
    int nx, ny, nz, N, nxy;
    T ihx, ihy, ihz;
    T *x, *b, *bw, *bs, *bb, *a, *q, *inv, *p;
};

template <typename T>
__device__ __forceinline__ SV<T> sview(const CoarseLevelDesc& d, T* sm) {
    SV<T> v;
    v.nx = d.nx; v.ny = d.ny; v.nz = d.nz; v.N = d.N; v.nxy = d.nx * d.ny;
    v.ihx = T(d.ihx); v.ihy = T(d.ihy); v.ihz = T(d.ihz);
    v.x = sm + d.ox; v.b = sm + d.ob; v.bw = sm + d.obw; v.bs = sm + d.obs; v.bb = sm + d.obb;
    v.a = d.oa >= 0 ? sm + d.oa : nullptr;
    v.q = d.oq >= 0 ? sm + d.oq : nullptr;
    v.inv = sm + d.oi;
    v.p = d.op >= 0 ? sm + d.op : nullptr;
    return v;
}

template <typename T>
__device__ __forceinline__ void s_coeffs(const SV<T>& o, int i, int j, int k, int c, int ip, int jp, T& cw, T& ce,
                                         T& cs, T& cn, T& cb, T& ct, T& diag) {
    T extra = T(0);
    const int row = c - i;
    cw = o.bw[c] * o.ihx;
    ce = o.bw[row + ip] * o.ihx;
    cs = o.bs[c] * o.ihy;
    cn = o.bs[c + (jp - j) * o.nx] * o.ihy;
    const T fb = o.bb[c], ft = o.bb[c + o.nxy];
    if (k > 0) cb = fb * o.ihz; else { cb = T(0); extra += T(2) * fb * o.ihz; }
    if (k < o.nz - 1) ct = ft * o.ihz; else { ct = T(0); extra += T(2) * ft * o.ihz; }
    if (o.nx == 1) { cw = T(0); ce = T(0); }
    if (o.ny == 1) { cs = T(0); cn = T(0); }
    const T a = o.a ? o.a[c] : T(0);
    diag = -a + cw + ce + cs + cn + cb + ct + extra;
}

// factor each z-line (den_k = diag_k - cb_k q_{k-1}: q_k = ct_k / den_k,
// inv_k = 1 / den_k, p_k = cb_k / den_k), or invert the point diagonal; the
// sweeps then need no division.  Recomputed only when alpha changes.
template <typename T>
__device__ void s_factor(const SV<T>& o, bool line) {
    if (line) {
        for (int col = threadIdx.x; col < o.nxy; col += blockDim.x) {
            const int i = col % o.nx, j = col / o.nx;
            const int ip = i == o.nx - 1 ? 0 : i + 1, jp = j == o.ny - 1 ? 0 : j + 1;
            T qprev = T(0);
            int c = col;
            for (int k = 0; k < o.nz; ++k, c += o.nxy) {
                T cw, ce, cs, cn, cb, ct, diag;
                s_coeffs(o, i, j, k, c, ip, jp, cw, ce, cs, cn, cb, ct, diag);
                const T inv = T(1) / (diag - cb * qprev);
                o.q[c] = ct * inv;
                o.inv[c] = inv;
                o.p[c] = cb * inv;
                qprev = o.q[c];
            }
        }
    } else {
        for (int c = threadIdx.x; c < o.N; c += blockDim.x) {
            const int i = c % o.nx, j = (c / o.nx) % o.ny, k = c / o.nxy;
            const int ip = i == o.nx - 1 ? 0 : i + 1, jp = j == o.ny - 1 ? 0 : j + 1;
            T cw, ce, cs, cn, cb, ct, diag;
            s_coeffs(o, i, j, k, c, ip, jp, cw, ce, cs, cn, cb, ct, diag);
            o.inv[c] = T(1) / diag;
        }
    }
}

template <typename T>
__device__ void s_smooth(const SV<T>& o, bool line, int sweeps) {
    const int nt = blockDim.x;
    for (int sw = 0; sw < sweeps; ++sw)
        for (int color = 0; color < 2; ++color) {
            if (line) {
                // the colour's columns in two phases: (1) every cell's
                // right-hand side with the x/y neighbours (the other colour),
                // scaled by 1/pivot, in parallel; (2) per column the
                // recurrences d_k = g_k + p_k d_{k-1}, x_k = d_k + q_k x_{k+1}
                for (int c = threadIdx.x; c < o.N; c += nt) {
                    const int i = c % o.nx, j = (c / o.nx) % o.ny;
                    if (((i + j) & 1) != color) continue;
                    const int im = i == 0 ? o.nx - 1 : i - 1, ip = i == o.nx - 1 ? 0 : i + 1;
                    const int jm = j == 0 ? o.ny - 1 : j - 1, jp = j == o.ny - 1 ? 0 : j + 1;
                    const int row = c - i;
                    T cw = o.bw[c] * o.ihx, ce = o.bw[row + ip] * o.ihx;
                    T cs = o.bs[c] * o.ihy, cn = o.bs[c + (jp - j) * o.nx] * o.ihy;
                    if (o.nx == 1) { cw = T(0); ce = T(0); }
                    if (o.ny == 1) { cs = T(0); cn = T(0); }
                    const T r = o.b[c] + cw * o.x[row + im] + ce * o.x[row + ip] + cs * o.x[c + (jm - j) * o.nx] +
                                cn * o.x[c + (jp - j) * o.nx];
                    o.x[c] = r * o.inv[c];
                }
                __syncthreads();
                for (int col = threadIdx.x; col < o.nxy; col += nt) {
                    const int i = col % o.nx, j = col / o.nx;
                    if (((i + j) & 1) != color) continue;
                    int c = col;
                    T d = o.x[c];
                    for (int k = 1; k < o.nz; ++k) {
                        c += o.nxy;
                        d = o.x[c] + o.p[c] * d;
                        o.x[c] = d;
                    }
                    T xn = d;
                    for (int k = o.nz - 2; k >= 0; --k) {
                        c -= o.nxy;
                        xn = o.x[c] + o.q[c] * xn;
                        o.x[c] = xn;
                    }
                }
            } else {
                for (int c = threadIdx.x; c < o.N; c += nt) {
                    const int i = c % o.nx, j = (c / o.nx) % o.ny, k = c / o.nxy;
                    if (((i + j + k) & 1) != color) continue;
                    const int im = i == 0 ? o.nx - 1 : i - 1, ip = i == o.nx - 1 ? 0 : i + 1;
                    const int jm = j == 0 ? o.ny - 1 : j - 1, jp = j == o.ny - 1 ? 0 : j + 1;
                    T cw, ce, cs, cn, cb, ct, diag;
                    s_coeffs(o, i, j, k, c, ip, jp, cw, ce, cs, cn, cb, ct, diag);
                    const int row = c - i;
                    T s = o.b[c] + cw * o.x[row + im] + ce * o.x[row + ip] + cs * o.x[c + (jm - j) * o.nx] +
                          cn * o.x[c + (jp - j) * o.nx];
                    if (k > 0) s += cb * o.x[c - o.nxy];
                    if (k < o.nz - 1) s += ct * o.x[c + o.nxy];
                    o.x[c] = s * o.inv[c];
                }
            }
            __syncthreads();
        }
}

template <typename T>
__device__ void s_restrict(const SV<T>& f, const SV<T>& c, int rx, int ry, int rz) {
    for (int cc = threadIdx.x; cc < c.N; cc += blockDim.x) {
        const int I = cc % c.nx, J = (cc / c.nx) % c.ny, K = cc / c.nxy;
        T s = T(0);
        for (int dk = 0; dk < rz; ++dk)
            for (int dj = 0; dj < ry; ++dj)
                for (int di = 0; di < rx; ++di) {
                    const int i = rx * I + di, j = ry * J + dj, k = rz * K + dk;
                    const int fc = i + f.nx * (j + f.ny * k);
                    const int im = i == 0 ? f.nx - 1 : i - 1, ip = i == f.nx - 1 ? 0 : i + 1;
                    const int jm = j == 0 ? f.ny - 1 : j - 1, jp = j == f.ny - 1 ? 0 : j + 1;
                    T cw, ce, cs, cn, cb, ct, diag;
                    s_coeffs(f, i, j, k, fc, ip, jp, cw, ce, cs, cn, cb, ct, diag);
                    const int row = fc - i;
                    T off = cw * f.x[row + im] + ce * f.x[row + ip] + cs * f.x[fc + (jm - j) * f.nx] + cn * f.x[fc + (jp - j) * f.nx];
                    if (k > 0) off += cb * f.x[fc - f.nxy];
                    if (k < f.nz - 1) off += ct * f.x[fc + f.nxy];
                    s += f.b[fc] - (diag * f.x[fc] - off);
                }
        c.b[cc] = s / T(rx * ry * rz);
        c.x[cc] = T(0);
    }
    __syncthreads();
}

template <typename T>
__device__ void s_prolong(const SV<T>& f, const SV<T>& c, int rx, int ry, int rz, const float* wx, const float* wy,
                          const float* wz) {
    for (int fc = threadIdx.x; fc < f.N; fc += blockDim.x) {
        const int i = fc % f.nx, j = (fc / f.nx) % f.ny, k = fc / f.nxy;
        int I[2], J[2], K[2];
        T wi[2], wj[2], wk[2];
        int ni = 1, nj = 1, nk = 1;
        I[0] = i / rx; wi[0] = T(1);
        if (rx == 2) { ni = 2; wi[1] = T(wx[fc]); wi[0] = T(1) - wi[1]; I[1] = (i & 1) ? I[0] + 1 : I[0] - 1; I[1] = (I[1] + c.nx) % c.nx; }
        J[0] = j / ry; wj[0] = T(1);
        if (ry == 2) { nj = 2; wj[1] = T(wy[fc]); wj[0] = T(1) - wj[1]; J[1] = (j & 1) ? J[0] + 1 : J[0] - 1; J[1] = (J[1] + c.ny) % c.ny; }
        K[0] = k / rz; wk[0] = T(1);
        if (rz == 2) {
            nk = 2; wk[1] = T(wz[fc]); wk[0] = T(1) - wk[1]; K[1] = (k & 1) ? K[0] + 1 : K[0] - 1;
            if (K[1] < 0 || K[1] >= c.nz) { K[1] = K[0]; wk[1] = T(0); }
        }
        T s = T(0);
        for (int a = 0; a < nk; ++a)
            for (int bb = 0; bb < nj; ++bb)
                for (int d = 0; d < ni; ++d) s += wk[a] * wj[bb] * wi[d] * c.x[I[d] + c.nx * (J[bb] + c.ny * K[a])];
        f.x[fc] += s;
    }
    __syncthreads();
}

// one element global -> shared without waiting (cp.async, 4 or 8 bytes)
template <typename E>
__device__ __forceinline__ void cp_async_el(E* dst, const E* src) {
    static_assert(sizeof(E) == 4 || sizeof(E) == 8, "cp.async element size");
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (sizeof(E) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

// The V-cycle of the shared-memory levels, run by one CTA on the shared
// memory smraw.
template <typename T>
__device__ void coarse_cta_cycle(const CoarseArgs& A, unsigned char* smraw) {
    __shared__ int s_valid;
    T* sm = reinterpret_cast<T*>(smraw);
    float* sw = reinterpret_cast<float*>(smraw + A.wbase);
    if (threadIdx.x == 0) s_valid = *(volatile int*)A.fvalid;
    __syncthreads();
    const bool valid = s_valid != 0;
    // load coefficients and the top right-hand side: every copy is issued
    // asynchronously (cp.async) before the block waits once, so the levels'
    // global reads overlap instead of costing one round trip each
    for (int l = 0; l < A.nlev; ++l) {
        const CoarseLevelDesc& d = A.L[l];
        const int nxy = d.nx * d.ny;
        const T* gbw = (const T*)d.gbw;
        const T* gbs = (const T*)d.gbs;
        const T* gbb = (const T*)d.gbb;
        const T* ga = (const T*)d.ga;
        for (int c = threadIdx.x; c < d.N; c += blockDim.x) {
            cp_async_el(sm + d.obw + c, gbw + c);
            cp_async_el(sm + d.obs + c, gbs + c);
            if (d.oa >= 0) cp_async_el(sm + d.oa + c, ga + c);
            sm[d.ox + c] = T(0);
        }
        for (int c = threadIdx.x; c < d.N + nxy; c += blockDim.x) cp_async_el(sm + d.obb + c, gbb + c);
        for (int q = 0; q < 3; ++q)
            if (d.gw[q])
                for (int c = threadIdx.x; c < d.N; c += blockDim.x) cp_async_el(sw + d.ow[q] + c, d.gw[q] + c);
        if (valid) {
            const long long fo[3] = {d.oq, d.oi, d.op};
            for (int q = 0; q < 3; ++q)
                if (fo[q] >= 0)
                    for (int c = threadIdx.x; c < d.N; c += blockDim.x) cp_async_el(sm + fo[q] + c, (const T*)d.gf[q] + c);
        }
    }
    {
        const T* b_in = (const T*)A.b_in;
        for (int c = threadIdx.x; c < A.L[0].N; c += blockDim.x) cp_async_el(sm + A.L[0].ob + c, b_in + c);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    if (!valid) {
        // first call since alpha changed: factor, and keep the factors for
        // the next calls (visible to them at the kernel boundary)
        for (int l = 0; l < A.nlev; ++l) s_factor(sview<T>(A.L[l], sm), A.L[l].line != 0);
        __syncthreads();
        for (int l = 0; l < A.nlev; ++l) {
            const CoarseLevelDesc& d = A.L[l];
            const long long fo[3] = {d.oq, d.oi, d.op};
            for (int q = 0; q < 3; ++q)
                if (fo[q] >= 0)
                    for (int c = threadIdx.x; c < d.N; c += blockDim.x) ((T*)d.gf[q])[c] = sm[fo[q] + c];
        }
        if (threadIdx.x == 0) *A.fvalid = 1;
    }
    // V-cycle over the shared-memory levels
    for (int l = 0; l < A.nlev - 1; ++l) {
        const SV<T> f = sview<T>(A.L[l], sm), c = sview<T>(A.L[l + 1], sm);
        s_smooth(f, A.L[l].line != 0, A.nu1);
        s_restrict(f, c, A.L[l].rx, A.L[l].ry, A.L[l].rz);
    }
    {
        const CoarseLevelDesc& d = A.L[A.nlev - 1];
        const SV<T> o = sview<T>(d, sm);
        const bool exact = d.line && d.nx * d.ny == 1;
        s_smooth(o, d.line != 0, exact ? 1 : A.nu_bottom);
    }
    for (int l = A.nlev - 2; l >= 0; --l) {
        const SV<T> f = sview<T>(A.L[l], sm), c = sview<T>(A.L[l + 1], sm);
        const CoarseLevelDesc& d = A.L[l];
        s_prolong(f, c, d.rx, d.ry, d.rz, d.gw[0] ? sw + d.ow[0] : nullptr, d.gw[1] ? sw + d.ow[1] : nullptr,
                  d.gw[2] ? sw + d.ow[2] : nullptr);
        s_smooth(f, d.line != 0, A.nu2);
    }
    T* x_out = (T*)A.x_out;
    for (int c = threadIdx.x; c < A.L[0].N; c += blockDim.x) x_out[c] = sm[A.L[0].ox + c];
}

template <typename T>
__global__ void __launch_bounds__(1024) k_coarse_vcycle(CoarseArgs A) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char smraw[];
    coarse_cta_cycle<T>(A, smraw);
}

template <typename Tin, typename T>
__global__ void __launch_bounds__(256) k_avg_alpha(const Tin* __restrict__ af, T* __restrict__ ac, int nx, int ny,
                                                   int ncx, int ncy, int ncz, int rx, int ry, int rz) {
    pdl_entry();
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    const int K = blockIdx.z;
    if (I >= ncx || J >= ncy) return;
    double s = 0.0;
    for (int dk = 0; dk < rz; ++dk)
        for (int dj = 0; dj < ry; ++dj)
            for (int di = 0; di < rx; ++di)
                s += (double)af[(size_t)(rx * I + di) + (size_t)nx * ((size_t)(ry * J + dj) + (size_t)ny * (rz * K + dk))];
    ac[(size_t)I + (size_t)ncx * ((size_t)J + (size_t)ncy * K)] = (T)(s / (rx * ry * rz));
}

// Every coarse alpha below level 1 in one launch.  Block b owns one cell of
// the tile level T and the cells of levels 2..T inside it (tile dims tl[l]),
// staged level by level in shared memory; the last block to finish forms the
// levels below T from the level-T arrays.  Each coarse cell is the same
// double sum in the same order as k_avg_alpha forms it (FP64 chain from the
// FP64 level above, FP32 chain from the FP32 level above), so the values are
// those of the per-level launches.
struct AlphaTiles {
    int* fvalid;                 // cleared: the one-CTA factors depend on alpha
    int nlev, T, cap;
    int n[MAXLEV][3], cr[MAXLEV][3], tl[MAXLEV][3];
    double* a64[MAXLEV];
    float* a32[MAXLEV];
    unsigned int* counter;
};

__global__ void __launch_bounds__(256) k_alpha_tiles(AlphaTiles A) {
    pdl_entry();
    extern __shared__ __align__(16) double atile[];
    __shared__ bool last;
    if (blockIdx.x == 0 && threadIdx.x < 2 && A.fvalid) A.fvalid[threadIdx.x] = 0;
    float* const f32 = reinterpret_cast<float*>(atile + 2 * A.cap);
    const bool has32 = A.a32[1] != nullptr;
    const int nT0 = A.n[A.T][0], nT1 = A.n[A.T][1];
    const int IT = blockIdx.x % nT0, JT = (blockIdx.x / nT0) % nT1, KT = blockIdx.x / (nT0 * nT1);
    int cur = 0;
    for (int l = 2; l <= A.T; ++l) {
        const double* src64 = atile + cur * A.cap;
        const float* src32 = f32 + cur * A.cap;
        double* dst64 = atile + (1 - cur) * A.cap;
        float* dst32 = f32 + (1 - cur) * A.cap;
        const int tx = A.tl[l][0], ty = A.tl[l][1], tz = A.tl[l][2];
        const int rx = A.cr[l][0], ry = A.cr[l][1], rz = A.cr[l][2];
        const int ox = IT * tx, oy = JT * ty, oz = KT * tz;
        const int ptx = A.tl[l - 1][0], pty = A.tl[l - 1][1];
        const int fnx = A.n[l - 1][0], fny = A.n[l - 1][1];
        for (int q = threadIdx.x; q < tx * ty * tz; q += blockDim.x) {
            const int i = q % tx, j = (q / tx) % ty, k = q / (tx * ty);
            double s = 0.0, s2 = 0.0;
            for (int dk = 0; dk < rz; ++dk)
                for (int dj = 0; dj < ry; ++dj)
                    for (int di = 0; di < rx; ++di) {
                        if (l == 2) {
                            const size_t g = (size_t)(rx * (ox + i) + di) +
                                             (size_t)fnx * ((size_t)(ry * (oy + j) + dj) + (size_t)fny * (size_t)(rz * (oz + k) + dk));
                            s += A.a64[1][g];
                            if (has32) s2 += (double)A.a32[1][g];
                        } else {
                            const int lq = (rx * i + di) + ptx * ((ry * j + dj) + pty * (rz * k + dk));
                            s += src64[lq];
                            if (has32) s2 += (double)src32[lq];
                        }
                    }
            const double v = s / (rx * ry * rz);
            const size_t gc = (size_t)(ox + i) + (size_t)A.n[l][0] * ((size_t)(oy + j) + (size_t)A.n[l][1] * (size_t)(oz + k));
            A.a64[l][gc] = v;
            dst64[q] = v;
            if (has32) {
                const float v2 = (float)(s2 / (rx * ry * rz));
                A.a32[l][gc] = v2;
                dst32[q] = v2;
            }
        }
        __syncthreads();
        cur = 1 - cur;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(A.counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int l = A.T + 1; l < A.nlev; ++l) {
        const int rx = A.cr[l][0], ry = A.cr[l][1], rz = A.cr[l][2];
        const int nx = A.n[l][0], ny = A.n[l][1], nz = A.n[l][2];
        const int fnx = A.n[l - 1][0], fny = A.n[l - 1][1];
        for (int q = threadIdx.x; q < nx * ny * nz; q += blockDim.x) {
            const int I = q % nx, J = (q / nx) % ny, K = q / (nx * ny);
            double s = 0.0, s2 = 0.0;
            for (int dk = 0; dk < rz; ++dk)
                for (int dj = 0; dj < ry; ++dj)
                    for (int di = 0; di < rx; ++di) {
                        const size_t g = (size_t)(rx * I + di) + (size_t)fnx * ((size_t)(ry * J + dj) + (size_t)fny * (rz * K + dk));
                        s += __ldcg(A.a64[l - 1] + g);
                        if (has32) s2 += (double)__ldcg(A.a32[l - 1] + g);
                    }
            A.a64[l][q] = s / (rx * ry * rz);
            if (has32) A.a32[l][q] = (float)(s2 / (rx * ry * rz));
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *A.counter = 0;
}


template <typename T>
T* dalloc(size_t n, size_t& bytes) {
    T* p = nullptr;
    if (n == 0) return nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    // zeroed: nothing may depend on what an earlier allocation left there
    if (cudaMemset(p, 0, n * sizeof(T)) != cudaSuccess) { cudaFree(p); return nullptr; }
    bytes += n * sizeof(T);
    return p;
}

template <typename T>
Op<T> make_op(const MGLevel& L, int l, const uint8_t* code, const double* eps, const T* a, bool inhom,
              const DevParams& p) {
    Op<T> o;
    o.nx = L.n[0]; o.ny = L.n[1]; o.nz = L.n[2];
    o.nxy = L.n[0] * L.n[1];
    o.ih2x = T(1.0 / (L.h[0] * L.h[0]));
    o.ih2y = T(1.0 / (L.h[1] * L.h[1]));
    o.ih2z = T(1.0 / (L.h[2] * L.h[2]));
    o.code = code;
    for (int q = 0; q < 8; ++q) o.eps[q] = T(eps[q]);
    if constexpr (sizeof(T) == 8) { o.bw = (const T*)L.bw64; o.bs = (const T*)L.bs64; o.bb = (const T*)L.bb64; }
    else { o.bw = (const T*)L.bw32; o.bs = (const T*)L.bs32; o.bb = (const T*)L.bb32; }
    o.a = a;
    if constexpr (sizeof(T) == 8) o.zc = (const T*)L.zc64;
    else o.zc = (const T*)L.zc32;
    o.vlo = inhom ? T(p.V_lo) : T(0);
    o.vhi = inhom ? T(p.V_hi) : T(0);
    o.bwh = o.bsh = o.bbh = nullptr;
    if constexpr (sizeof(T) == 4) {
        if (l > 0 && L.bwh && !o.zc) {
            // FP16 faces scaled by 1 / hscale: the couplings carry hscale
            o.bwh = L.bwh; o.bsh = L.bsh; o.bbh = L.bbh;
            o.ih2x = T(L.hscale / (L.h[0] * L.h[0]));
            o.ih2y = T(L.hscale / (L.h[1] * L.h[1]));
            o.ih2z = T(L.hscale / (L.h[2] * L.h[2]));
        }
    }
    return o;
}

template <typename T> T* lx(MGLevel& L);
template <> double* lx<double>(MGLevel& L) { return L.x64; }
template <> float* lx<float>(MGLevel& L) { return L.x32; }
template <typename T> T* lb(MGLevel& L);
template <> double* lb<double>(MGLevel& L) { return L.b64; }
template <> float* lb<float>(MGLevel& L) { return L.b32; }
template <typename T> T* la(MGLevel& L);
template <> double* la<double>(MGLevel& L) { return L.a64; }
template <> float* la<float>(MGLevel& L) { return L.a32; }
template <typename T> T* lq(MGLevel& L);
template <> double* lq<double>(MGLevel& L) { return L.cp64; }
template <> float* lq<float>(MGLevel& L) { return L.cp32; }

// ---- loop control of the device-controlled solves (fx_ctl.h); one thread each

// the max of the NORM_SLOTS slots, as the host takes it (std::max from 0)
__device__ __forceinline__ double ctl_slots_max(const double* __restrict__ slots) {
    double m = 0.0;
#pragma unroll 16
    for (int q = 0; q < NORM_SLOTS; ++q) {
        const double v = slots[q];
        m = m < v ? v : m;
    }
    return m;
}

// after a V-cycle: the level-0 norm after pre-smoothing bounds the residual
// after the cycle; the exact residual is formed (the next residual kernel,
// which otherwise returns at once) once it is within the target, or always
// with a single level
__global__ void k_mg_mid(double* __restrict__ slots, int single_level, int maxit, StepCtl* ctl,
                         cudaGraphConditionalHandle hw) {
    pdl_entry();
    ctl->nexec[KIND_MG_CYCLE] += 1;
    const double mid = ctl_slots_max(slots);
    for (int q = 0; q < NORM_SLOTS; ++q) slots[q] = 0.0;
    const int it = ctl->it + 1;
    ctl->it = it;
    // a non-finite norm (a NaN reaches the slots as +inf) ends the loop: the
    // exact residual then records the failure
    const bool need = single_level || mid <= ctl->target || !isfinite(mid);
    if (!need) ctl->rn = mid;
    ctl->need = need ? 1 : 0;
    cudaGraphSetConditional(hw, (!need && it < maxit) ? 1u : 0u);
}

// the iterate back into phi when the last refinement step wrote the second buffer
__global__ void __launch_bounds__(256) k_mx_copy(const double* __restrict__ src, double* __restrict__ dst, int n,
                                                 const StepCtl* __restrict__ ctl) {
    pdl_entry();
    if (!ctl->parity) return;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) dst[c] = src[c];
}

// the solve's statistics and, when it stopped short of the target, the failure
__global__ void k_mg_end(StepCtl* ctl) {
    pdl_entry();
    ctl_mg_end(ctl);
}

}  // namespace

double Multigrid::slots_max() const {
    double m = 0.0;
    for (int q = 0; q < NORM_SLOTS; ++q) m = std::max(m, h_norm_[q]);
    return m;
}

Multigrid::~Multigrid() {
    for (size_t l = 0; l < lev_.size(); ++l) {
        MGLevel& L = lev_[l];
        // level 0 borrows phi / rhs (FP64) and e32_ / r32_ (FP32), freed below
        if (l > 0) { cudaFree(L.x64); cudaFree(L.b64); cudaFree(L.x32); cudaFree(L.b32); }
        cudaFree(L.bw64); cudaFree(L.bs64); cudaFree(L.bb64); cudaFree(L.a64); cudaFree(L.cp64);
        cudaFree(L.bw32); cudaFree(L.bs32); cudaFree(L.bb32); cudaFree(L.a32); cudaFree(L.cp32);
        cudaFree(L.bwh); cudaFree(L.bsh); cudaFree(L.bbh);
        for (int d = 0; d < 3; ++d) { cudaFree(L.wf[d]); cudaFree(L.fac64[d]); cudaFree(L.fac32[d]); }
        cudaFree(L.zc64);
        cudaFree(L.zc32);
    }
    cudaFree(d_fvalid_);
    cudaFree(at_counter_);
    cudaFree(rc_counter_);
    if (g64_.exec) cudaGraphExecDestroy(g64_.exec);
    if (g32_.exec) cudaGraphExecDestroy(g32_.exec);
    if (g32b_.exec) cudaGraphExecDestroy(g32b_.exec);
    cudaFree(d_norm_);
    if (h_norm_) cudaFreeHost(h_norm_);
    cudaFree(dinv64_);
    cudaFree(dinv32_);
    dinv64_ = nullptr;
    dinv32_ = nullptr;
    cudaFree(e32_);
    cudaFree(alt64m_);
    cudaFree(r32_);
}

int Multigrid::setup(const DevParams& p, const std::vector<uint8_t>& code, bool want64, bool want32) {
    if ((long long)p.nx * p.ny * (p.nz + 2) >= (1LL << 31)) return -1;   // 32-bit cell indices in the kernels
    for (int q = 0; q < 8; ++q) eps_[q] = p.eps[q];
    lev_.clear();
    MGLevel L0{};
    L0.n[0] = p.nx; L0.n[1] = p.ny; L0.n[2] = p.nz;
    for (int d = 0; d < 3; ++d) { L0.h[d] = p.dx[d]; L0.cr[d] = 1; }
    L0.N = (size_t)p.N;
    L0.line = false;
    lev_.push_back(L0);
    auto coarsenable_xy = [](int n) { return n % 2 == 0 && (n / 2 == 1 || (n / 2) % 2 == 0); };
    while (true) {
        MGLevel& f = lev_.back();
        const double hmin = std::min(f.h[0], std::min(f.h[1], f.h[2]));
        const bool cz = f.n[2] % 2 == 0 && f.h[2] <= 1.5 * hmin;
        int cr[3] = {1, 1, 1};
        if (cz) {
            cr[2] = 2;
            for (int d = 0; d < 2; ++d)
                if (coarsenable_xy(f.n[d]) && f.h[d] <= 1.5 * hmin) cr[d] = 2;
            f.line = false;
        } else {
            for (int d = 0; d < 2; ++d)
                if (coarsenable_xy(f.n[d])) cr[d] = 2;
            // z-lines where z is the strongly coupled direction, and on the
            // bottom level (an exact solve when it is one column); a level
            // that keeps z only because nz is odd but is isotropic takes
            // point red-black sweeps
            f.line = (cr[0] == 1 && cr[1] == 1) || 1.5 * f.h[2] < std::min(f.h[0], f.h[1]);
            if (cr[0] == 1 && cr[1] == 1) break;   // bottom
        }
        MGLevel c{};
        for (int d = 0; d < 3; ++d) { c.n[d] = f.n[d] / cr[d]; c.h[d] = f.h[d] * cr[d]; c.cr[d] = cr[d]; }
        c.N = (size_t)c.n[0] * c.n[1] * c.n[2];
        c.line = true;
        lev_.push_back(c);
        if (lev_.size() > 64) return -1;
    }

    // level-0 face beta on the host, then face averages down the hierarchy
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const size_t nxy = (size_t)nx * ny;
    auto ecode = [&](int i, int j, int k) { return eps_[code[(size_t)i + nx * ((size_t)j + (size_t)ny * (k + 1))] & 7]; };
    std::vector<double> fw(L0.N), fs(L0.N), fb(L0.N + nxy);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t c = (size_t)i + nx * ((size_t)j + (size_t)ny * k);
                const double ec = ecode(i, j, k);
                fw[c] = 0.5 * (ec + ecode((i + nx - 1) % nx, j, k));
                fs[c] = 0.5 * (ec + ecode(i, (j + ny - 1) % ny, k));
                fb[c] = k == 0 ? ec : 0.5 * (ec + ecode(i, j, k - 1));
            }
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) fb[nz * nxy + (size_t)i + nx * (size_t)j] = ecode(i, j, nz - 1);

    bytes_ = 0;
    // face beta that depends on z only (a layered stack): keep it by plane
    auto try_planes = [&](MGLevel& L, const std::vector<double>& bw, const std::vector<double>& bs,
                          const std::vector<double>& bb) -> int {
        const size_t lnxy = (size_t)L.n[0] * L.n[1];
        std::vector<double> zc(3 * L.n[2] + 1);
        for (int k = 0; k < L.n[2]; ++k) {
            const size_t c0 = lnxy * k;
            zc[k] = bw[c0];
            zc[L.n[2] + k] = bs[c0];
            for (size_t q = 0; q < lnxy; ++q)
                if (bw[c0 + q] != bw[c0] || bs[c0 + q] != bs[c0]) return 0;
        }
        for (int k = 0; k <= L.n[2]; ++k) {
            const size_t c0 = lnxy * k;
            zc[2 * L.n[2] + k] = bb[c0];
            for (size_t q = 0; q < lnxy; ++q)
                if (bb[c0 + q] != bb[c0]) return 0;
        }
        const size_t nzc = zc.size();
        if (want64) {
            L.zc64 = dalloc<double>(nzc, bytes_);
            if (!L.zc64 || cudaMemcpy(L.zc64, zc.data(), nzc * 8, cudaMemcpyHostToDevice) != cudaSuccess) return -2;
        }
        if (want32) {
            std::vector<float> z32(zc.begin(), zc.end());
            L.zc32 = dalloc<float>(nzc, bytes_);
            if (!L.zc32 || cudaMemcpy(L.zc32, z32.data(), nzc * 4, cudaMemcpyHostToDevice) != cudaSuccess) return -2;
        }
        return 0;
    };
    for (size_t l = 0; l < lev_.size(); ++l) {
        MGLevel& L = lev_[l];
        const size_t N = L.N, lnxy = (size_t)L.n[0] * L.n[1];
        if (l == 0) {
            // level 0's face beta from the codes, as coeffs<T, CK_FINE> forms
            // it; bb[0] and bb[nz] are the electrode-layer cells' eps
            if (try_planes(L, fw, fs, fb)) return -2;
        }
        if (l > 0) {
            const MGLevel& F = lev_[l - 1];
            const int rx = L.cr[0], ry = L.cr[1], rz = L.cr[2];
            const int fnx = F.n[0], fny = F.n[1];
            // Face beta of the coarse level.  Along a coarsened direction the
            // coarse face joins the fine links between the two coarse centres
            // in series (half link, full link, half link: beta_c =
            // 4 / (1/b_{2I-1} + 2/b_{2I} + 1/b_{2I+1})), so thin low-eps layers
            // keep their resistance; across the transverse children the links
            // are in parallel (arithmetic mean).  At a Dirichlet face the path
            // runs from the coarse centre to the electrode: half of the first
            // interior link and the fine boundary link, beta_c = 2/(1/b_0 + 1/b_1).
            const int fnz = F.n[2];
            // prolongation weights: a fine cell between its parent's centre
            // (h/2 away) and the neighbouring coarse centre (3h/2 away) takes
            // the weights of a 1-D resistor chain built from the fine face
            // beta (3/4, 1/4 for uniform beta; the neighbour beyond an
            // electrode is the homogeneous Dirichlet value)
            for (int d = 0; d < 3; ++d) {
                if (L.cr[d] != 2) continue;
                std::vector<float> w(F.N);
                const double h = F.h[d];
                const int nd = F.n[d];
                for (int k = 0; k < fnz; ++k)
                    for (int j = 0; j < fny; ++j)
                        for (int i = 0; i < fnx; ++i) {
                            const int q = d == 0 ? i : d == 1 ? j : k;
                            auto B = [&](int t) {
                                if (d == 0) return fw[(size_t)(((t % nd) + nd) % nd) + fnx * ((size_t)j + (size_t)fny * k)];
                                if (d == 1) return fs[(size_t)i + fnx * ((size_t)(((t % nd) + nd) % nd) + (size_t)fny * k)];
                                return fb[(size_t)i + fnx * ((size_t)j + (size_t)fny * t)];
                            };
                            double gn, gf;
                            if ((q & 1) == 0) {
                                gn = 2.0 * B(q + 1) / h;
                                gf = (d == 2 && q == 0) ? 2.0 * B(0) / h : 1.0 / (h / B(q) + h / (2.0 * B(q - 1)));
                            } else {
                                gn = 2.0 * B(q) / h;
                                gf = (d == 2 && q == nd - 1) ? 2.0 * B(nd) / h : 1.0 / (h / B(q + 1) + h / (2.0 * B(q + 2)));
                            }
                            w[(size_t)i + fnx * ((size_t)j + (size_t)fny * k)] = (float)(gf / (gn + gf));
                        }
                L.wf[d] = dalloc<float>(F.N, bytes_);
                if (!L.wf[d]) return -2;
                if (cudaMemcpy(L.wf[d], w.data(), F.N * 4, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
            }
            auto FW = [&](int i, int j, int k) { return fw[(size_t)((i % fnx + fnx) % fnx) + fnx * ((size_t)j + (size_t)fny * k)]; };
            auto FS = [&](int i, int j, int k) { return fs[(size_t)i + fnx * ((size_t)((j % fny + fny) % fny) + (size_t)fny * k)]; };
            auto FB = [&](int i, int j, int k) { return fb[(size_t)i + fnx * ((size_t)j + (size_t)fny * k)]; };
            auto ser = [](double a, double b, double c) { return 4.0 / (1.0 / a + 2.0 / b + 1.0 / c); };
            std::vector<double> cw(N), cs(N), cb(N + lnxy);
            for (int k = 0; k < L.n[2]; ++k)
                for (int j = 0; j < L.n[1]; ++j)
                    for (int i = 0; i < L.n[0]; ++i) {
                        const size_t c = (size_t)i + L.n[0] * ((size_t)j + (size_t)L.n[1] * k);
                        double s = 0;
                        for (int dk = 0; dk < rz; ++dk)
                            for (int dj = 0; dj < ry; ++dj) {
                                const int fj = ry * j + dj, fk = rz * k + dk;
                                s += rx == 2 ? ser(FW(2 * i - 1, fj, fk), FW(2 * i, fj, fk), FW(2 * i + 1, fj, fk)) : FW(i, fj, fk);
                            }
                        cw[c] = s / (ry * rz);
                        s = 0;
                        for (int dk = 0; dk < rz; ++dk)
                            for (int di = 0; di < rx; ++di) {
                                const int fi = rx * i + di, fk = rz * k + dk;
                                s += ry == 2 ? ser(FS(fi, 2 * j - 1, fk), FS(fi, 2 * j, fk), FS(fi, 2 * j + 1, fk)) : FS(fi, j, fk);
                            }
                        cs[c] = s / (rx * rz);
                    }
            for (int k = 0; k <= L.n[2]; ++k)
                for (int j = 0; j < L.n[1]; ++j)
                    for (int i = 0; i < L.n[0]; ++i) {
                        double s = 0;
                        for (int dj = 0; dj < ry; ++dj)
                            for (int di = 0; di < rx; ++di) {
                                const int fi = rx * i + di, fj = ry * j + dj;
                                double v;
                                if (rz == 1) v = FB(fi, fj, k);
                                else if (k == 0) v = 2.0 / (1.0 / FB(fi, fj, 0) + 1.0 / FB(fi, fj, 1));
                                else if (k == L.n[2]) v = 2.0 / (1.0 / FB(fi, fj, fnz) + 1.0 / FB(fi, fj, fnz - 1));
                                else v = ser(FB(fi, fj, 2 * k - 1), FB(fi, fj, 2 * k), FB(fi, fj, 2 * k + 1));
                                s += v;
                            }
                        cb[(size_t)i + L.n[0] * ((size_t)j + (size_t)L.n[1] * k)] = s / (rx * ry);
                    }
            fw.swap(cw); fs.swap(cs); fb.swap(cb);
            if (try_planes(L, fw, fs, fb)) return -2;
            if (want64) {
                L.x64 = dalloc<double>(N, bytes_); L.b64 = dalloc<double>(N, bytes_); L.a64 = dalloc<double>(N, bytes_);
                L.bw64 = dalloc<double>(N, bytes_); L.bs64 = dalloc<double>(N, bytes_); L.bb64 = dalloc<double>(N + lnxy, bytes_);
                if (!L.x64 || !L.b64 || !L.a64 || !L.bw64 || !L.bs64 || !L.bb64) return -2;
                if (cudaMemcpy(L.bw64, fw.data(), N * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
                    cudaMemcpy(L.bs64, fs.data(), N * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
                    cudaMemcpy(L.bb64, fb.data(), (N + lnxy) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
                    cudaMemset(L.a64, 0, N * 8) != cudaSuccess)
                    return -1;
            }
            if (want32) {
                L.x32 = dalloc<float>(N, bytes_); L.b32 = dalloc<float>(N, bytes_); L.a32 = dalloc<float>(N, bytes_);
                L.bw32 = dalloc<float>(N, bytes_); L.bs32 = dalloc<float>(N, bytes_); L.bb32 = dalloc<float>(N + lnxy, bytes_);
                if (!L.x32 || !L.b32 || !L.a32 || !L.bw32 || !L.bs32 || !L.bb32) return -2;
                std::vector<float> t(N + lnxy);
                for (size_t q = 0; q < N; ++q) t[q] = (float)fw[q];
                if (cudaMemcpy(L.bw32, t.data(), N * 4, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
                for (size_t q = 0; q < N; ++q) t[q] = (float)fs[q];
                if (cudaMemcpy(L.bs32, t.data(), N * 4, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
                for (size_t q = 0; q < N + lnxy; ++q) t[q] = (float)fb[q];
                if (cudaMemcpy(L.bb32, t.data(), (N + lnxy) * 4, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
                if (cudaMemset(L.a32, 0, N * 4) != cudaSuccess) return -1;
                if (half_coarse && !L.zc32) {
                    // the FP32 cycle's launched kernels read the faces in FP16,
                    // scaled into (0, 1] by the level's largest face beta
                    double mx = 0.0;
                    for (size_t q = 0; q < N; ++q) mx = std::max(mx, std::max(fw[q], fs[q]));
                    for (size_t q = 0; q < N + lnxy; ++q) mx = std::max(mx, fb[q]);
                    if (mx > 0.0 && std::isfinite(mx)) {
                        L.hscale = mx;
                        L.bwh = dalloc<uint16_t>(N, bytes_); L.bsh = dalloc<uint16_t>(N, bytes_);
                        L.bbh = dalloc<uint16_t>(N + lnxy, bytes_);
                        if (!L.bwh || !L.bsh || !L.bbh) return -2;
                        std::vector<uint16_t> h(N + lnxy);
                        auto put = [&](const std::vector<double>& v, uint16_t* d, size_t n) {
                            for (size_t q = 0; q < n; ++q) h[q] = __half_as_ushort(__double2half(v[q] / mx));
                            return cudaMemcpy(d, h.data(), n * 2, cudaMemcpyHostToDevice) == cudaSuccess;
                        };
                        if (!put(fw, L.bwh, N) || !put(fs, L.bsh, N) || !put(fb, L.bbh, N + lnxy)) return -1;
                    }
                }
            }
        }
        if (L.line) {
            if (want64) { L.cp64 = dalloc<double>(N, bytes_); if (!L.cp64) return -2; }
            if (want32) { L.cp32 = dalloc<float>(N, bytes_); if (!L.cp32) return -2; }
        }
    }
    if (cudaMalloc(&d_norm_, NORM_SLOTS * 8) != cudaSuccess) return -2;
    if (cudaMemset(d_norm_, 0, NORM_SLOTS * 8) != cudaSuccess) return -1;   // zero between uses
    if (cudaMemset(d_norm_, 0, NORM_SLOTS * 8) != cudaSuccess) return -1;
    if (cudaMalloc(&rc_counter_, sizeof(unsigned int)) != cudaSuccess) return -2;
    if (cudaMemset(rc_counter_, 0, sizeof(unsigned int)) != cudaSuccess) return -1;
    if (cudaMallocHost(&h_norm_, NORM_SLOTS * 8) != cudaSuccess) return -2;
    if (want32) {
        e32_ = dalloc<float>(L0.N, bytes_);
        r32_ = dalloc<float>(L0.N, bytes_);
        alt64m_ = dalloc<double>(L0.N, bytes_);
        if (!e32_ || !r32_) return -2;
        lev_[0].x32 = e32_;
        lev_[0].b32 = r32_;
    }
    plan_coarse(want64, want32);
    build_dense(want64, want32);
    // the tile level of k_alpha_tiles: the deepest level whose cells cover at
    // most 4096 level-1 cells, with few cells left below it for the last block
    at_T_ = 0;
    if (lev_.size() >= 3 && lev_.size() <= (size_t)kMaxLev) {
        int best = 0;
        for (int T = 2; T < (int)lev_.size(); ++T) {
            long long f = 1;
            for (int m = 2; m <= T; ++m) f *= (long long)lev_[m].cr[0] * lev_[m].cr[1] * lev_[m].cr[2];
            if (f > 4096) break;
            long long below = 0;
            for (size_t m = T + 1; m < lev_.size(); ++m) below += (long long)lev_[m].N;
            if (below <= 16384) best = T;
        }
        if (best >= 2 && cudaMalloc(&at_counter_, sizeof(unsigned int)) == cudaSuccess &&
            cudaMemset(at_counter_, 0, sizeof(unsigned int)) == cudaSuccess) {
            at_T_ = best;
            for (int d = 0; d < 3; ++d) at_tl_[best][d] = 1;
            for (int l = best; l >= 2; --l)
                for (int d = 0; d < 3; ++d) at_tl_[l - 1][d] = at_tl_[l][d] * lev_[l].cr[d];
            at_cap_ = at_tl_[2][0] * at_tl_[2][1] * at_tl_[2][2];
        }
    }
    if (verbose) {
        printf("  one-CTA coarse cycle from level %d (FP64, %zu B smem), %d (FP32, %zu B smem)\n", coarse_top64_,
               coarse_smem64_, coarse_top32_, coarse_smem32_);
        for (size_t l = 0; l < lev_.size(); ++l)
            printf("  mg level %zu: %d x %d x %d  h = %.4g %.4g %.4g nm  %s\n", l, lev_[l].n[0], lev_[l].n[1], lev_[l].n[2],
                   lev_[l].h[0] * 1e9, lev_[l].h[1] * 1e9, lev_[l].h[2] * 1e9, lev_[l].line ? "z-line GS" : "point RB-GS");
    }
    return 0;
}

int Multigrid::set_alpha(const double* a64, const float* a32, bool has_alpha, cudaStream_t s) {
    // the one-CTA factors depend on alpha: recompute them at the next call
    // (the tile kernel below clears the flags itself)
    const bool tiles = has_alpha && at_T_ >= 2 && alpha_tiles;
    if ((has_alpha || has_alpha_) && d_fvalid_ && !tiles) cudaMemsetAsync(d_fvalid_, 0, 2 * sizeof(int), s);
    a0_64 = a64;
    a0_32 = a32;
    has_alpha_ = has_alpha;
    if (!has_alpha) return 0;
    const size_t lmax = tiles ? 2 : lev_.size();   // per-level launches below this level
    for (size_t l = 1; l < lmax; ++l) {
        MGLevel& L = lev_[l];
        const MGLevel& F = lev_[l - 1];
        dim3 b(32, 8), g((L.n[0] + 31) / 32, (L.n[1] + 7) / 8, L.n[2]);
        if (L.a64) {
            if (l == 1) { ++g_launches; launch_k(k_avg_alpha<double, double>, g, b, 0, s, a64, L.a64, F.n[0], F.n[1], L.n[0], L.n[1], L.n[2], L.cr[0], L.cr[1], L.cr[2]); }
            else { ++g_launches; launch_k(k_avg_alpha<double, double>, g, b, 0, s, F.a64, L.a64, F.n[0], F.n[1], L.n[0], L.n[1], L.n[2], L.cr[0], L.cr[1], L.cr[2]); }
        }
        if (L.a32) {
            if (l == 1) { ++g_launches; launch_k(k_avg_alpha<double, float>, g, b, 0, s, a64, L.a32, F.n[0], F.n[1], L.n[0], L.n[1], L.n[2], L.cr[0], L.cr[1], L.cr[2]); }
            else { ++g_launches; launch_k(k_avg_alpha<float, float>, g, b, 0, s, F.a32, L.a32, F.n[0], F.n[1], L.n[0], L.n[1], L.n[2], L.cr[0], L.cr[1], L.cr[2]); }
        }
    }
    if (tiles) {
        AlphaTiles A;
        std::memset(&A, 0, sizeof(A));
        A.nlev = (int)lev_.size();
        A.T = at_T_;
        A.cap = at_cap_;
        for (int l = 0; l < A.nlev; ++l) {
            for (int d = 0; d < 3; ++d) { A.n[l][d] = lev_[l].n[d]; A.cr[l][d] = lev_[l].cr[d]; A.tl[l][d] = at_tl_[l][d]; }
            A.a64[l] = l == 0 ? nullptr : lev_[l].a64;
            A.a32[l] = l == 0 ? nullptr : lev_[l].a32;
        }
        A.counter = at_counter_;
        A.fvalid = d_fvalid_;
        const MGLevel& LT = lev_[at_T_];
        ++g_launches;
        launch_k(k_alpha_tiles, (unsigned)LT.N, 256, (size_t)at_cap_ * 24, s, A);
    }
    return (int)cudaGetLastError();
}

// shared-memory bytes of levels top..last for element size es (alpha and the
// line scratch always reserved so the plan holds for any alpha)
static size_t coarse_bytes(const std::vector<MGLevel>& lev, int top, size_t es, size_t* wbase) {
    size_t t = 0, w = 0;
    for (size_t l = top; l < lev.size(); ++l) {
        const size_t N = lev[l].N, nxy = (size_t)lev[l].n[0] * lev[l].n[1];
        t += (7 * N + nxy) * es + (lev[l].line ? 2 * N * es : 0);
        if (l + 1 < lev.size())
            for (int d = 0; d < 3; ++d) if (lev[l + 1].cr[d] == 2) w += N;
    }
    t = (t + 15) / 16 * 16;
    if (wbase) *wbase = t;
    return t + w * 4;
}

void Multigrid::plan_coarse(bool want64, bool want32) {
    constexpr size_t budget = 227 * 1024;   // the sm_100 per-block maximum of dynamic shared memory
    coarse_top64_ = coarse_top32_ = -1;
    for (int top = 1; top < (int)lev_.size(); ++top) {
        if (want64 && coarse_top64_ < 0 && coarse_bytes(lev_, top, 8, nullptr) <= budget) {
            coarse_top64_ = top;
            coarse_smem64_ = coarse_bytes(lev_, top, 8, nullptr);
        }
        if (want32 && coarse_top32_ < 0 && coarse_bytes(lev_, top, 4, nullptr) <= budget) {
            coarse_top32_ = top;
            coarse_smem32_ = coarse_bytes(lev_, top, 4, nullptr);
        }
    }
    if (coarse_top64_ > 0)
        cudaFuncSetAttribute(k_coarse_vcycle<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_smem64_);
    if (coarse_top32_ > 0)
        cudaFuncSetAttribute(k_coarse_vcycle<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_smem32_);
    // global copies of the one-CTA levels' smoother factors (q and p only on
    // z-line levels), and the flags that say whether they are current
    for (int l = 0; l < (int)lev_.size(); ++l) {
        MGLevel& L = lev_[l];
        const size_t n[3] = {L.line ? L.N : 0, L.N, L.line ? L.N : 0};
        for (int k = 0; k < 3; ++k) {
            if (coarse_top64_ > 0 && l >= coarse_top64_ && n[k]) L.fac64[k] = dalloc<double>(n[k], bytes_);
            if (coarse_top32_ > 0 && l >= coarse_top32_ && n[k]) L.fac32[k] = dalloc<float>(n[k], bytes_);
        }
    }
    if (cudaMalloc(&d_fvalid_, 2 * sizeof(int)) == cudaSuccess) cudaMemset(d_fvalid_, 0, 2 * sizeof(int));
}

// ---- the exact coarse solve: dense inverse of the first one-CTA level
//
// In-place Gauss-Jordan inversion of the level's operator (symmetric positive
// definite: no pivoting), one column k per step in three launches: keep
// column k, scale row k by the pivot's inverse, eliminate column k from every
// other row.  Run once at setup.
__global__ void k_gj_col(const double* __restrict__ A, int n, int k, double* __restrict__ col) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) col[i] = A[(size_t)i * n + k];
}
__global__ void k_gj_row(double* __restrict__ A, int n, int k, const double* __restrict__ col) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double pinv = 1.0 / col[k];
    A[(size_t)k * n + j] = j == k ? pinv : A[(size_t)k * n + j] * pinv;
}
__global__ void k_gj_rest(double* __restrict__ A, int n, int k, const double* __restrict__ col) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= n || i == k) return;
    const double ci = col[i];
    if (j == k) A[(size_t)i * n + k] = -ci * (1.0 / col[k]);
    else A[(size_t)i * n + j] -= ci * A[(size_t)k * n + j];
}
__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

// x = Ainv b for the first one-CTA level (one warp per row)
template <typename T>
__global__ void __launch_bounds__(256) k_dense_solve(const T* __restrict__ Ainv, const T* __restrict__ b,
                                                     T* __restrict__ x, int n) {
    pdl_entry();
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const T* a = Ainv + (size_t)row * n;
    T s = T(0);
    constexpr int V = 16 / (int)sizeof(T);   // elements per 16-byte load
    if (n % (32 * V) == 0) {
        // 16-byte loads, the row in 32 V-element strides
        for (int c = lane * V; c < n; c += 32 * V) {
            T av[V], bv[V];
            ldg16(a + c, av);
            ldg16(b + c, bv);
#pragma unroll
            for (int q = 0; q < V; ++q) s += av[q] * bv[q];
        }
    } else {
        for (int c = lane; c < n; c += 32) s += __ldg(a + c) * __ldg(b + c);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) x[row] = s;
}

// the dense inverse of level top's operator (the one-CTA kernel's arrays and
// arithmetic: face beta times 1/h^2, Dirichlet z faces folded into the
// diagonal, no alpha), FP64 on the device; null when the level is too large
static double* dense_inverse(const MGLevel& L, size_t& bytes) {
    const int n = (int)L.N;
    if (n <= 0 || n > Multigrid::kDenseMax) return nullptr;
    const int nx = L.n[0], ny = L.n[1], nz = L.n[2], nxy = nx * ny;
    std::vector<double> bw(L.N), bs(L.N), bb(L.N + nxy);
    if (L.bw64) {
        if (cudaMemcpy(bw.data(), L.bw64, L.N * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(bs.data(), L.bs64, L.N * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(bb.data(), L.bb64, (L.N + nxy) * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
            return nullptr;
    } else if (L.bw32) {
        std::vector<float> t(L.N + nxy);
        if (cudaMemcpy(t.data(), L.bw32, L.N * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return nullptr;
        for (size_t q = 0; q < L.N; ++q) bw[q] = t[q];
        if (cudaMemcpy(t.data(), L.bs32, L.N * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return nullptr;
        for (size_t q = 0; q < L.N; ++q) bs[q] = t[q];
        if (cudaMemcpy(t.data(), L.bb32, (L.N + nxy) * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return nullptr;
        for (size_t q = 0; q < L.N + nxy; ++q) bb[q] = t[q];
    } else {
        return nullptr;
    }
    const double ihx = 1.0 / (L.h[0] * L.h[0]), ihy = 1.0 / (L.h[1] * L.h[1]), ihz = 1.0 / (L.h[2] * L.h[2]);
    std::vector<double> A((size_t)n * n, 0.0);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const int c = i + nx * (j + ny * k);
                const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
                const int jm = j == 0 ? ny - 1 : j - 1, jp = j == ny - 1 ? 0 : j + 1;
                const int row = c - i;
                double cw = bw[c] * ihx, ce = bw[row + ip] * ihx;
                double cs = bs[c] * ihy, cn = bs[c + (jp - j) * nx] * ihy;
                double cb = 0.0, ct = 0.0, extra = 0.0;
                if (k > 0) cb = bb[c] * ihz; else extra += 2.0 * bb[c] * ihz;
                if (k < nz - 1) ct = bb[c + nxy] * ihz; else extra += 2.0 * bb[c + nxy] * ihz;
                if (nx == 1) { cw = 0.0; ce = 0.0; }
                if (ny == 1) { cs = 0.0; cn = 0.0; }
                double* a = &A[(size_t)c * n];
                a[c] += cw + ce + cs + cn + cb + ct + extra;
                a[row + im] -= cw;
                a[row + ip] -= ce;
                a[c + (jm - j) * nx] -= cs;
                a[c + (jp - j) * nx] -= cn;
                if (k > 0) a[c - nxy] -= cb;
                if (k < nz - 1) a[c + nxy] -= ct;
            }
    double *dA = nullptr, *col = nullptr;
    if (cudaMalloc(&dA, A.size() * 8) != cudaSuccess) return nullptr;
    if (cudaMalloc(&col, (size_t)n * 8) != cudaSuccess) { cudaFree(dA); return nullptr; }
    bool ok = cudaMemcpy(dA, A.data(), A.size() * 8, cudaMemcpyHostToDevice) == cudaSuccess;
    const int tb = 256, gb = (n + tb - 1) / tb;
    for (int k = 0; ok && k < n; ++k) {
        k_gj_col<<<gb, tb>>>(dA, n, k, col);
        k_gj_row<<<gb, tb>>>(dA, n, k, col);
        k_gj_rest<<<dim3(gb, n), tb>>>(dA, n, k, col);
    }
    ok = ok && cudaDeviceSynchronize() == cudaSuccess;
    cudaFree(col);
    if (!ok) { cudaFree(dA); return nullptr; }
    bytes += A.size() * 8;
    return dA;
}

// the exact coarse solves, built once at setup (after plan_coarse)
int Multigrid::build_dense(bool want64, bool want32) {
    if (!dense_coarse) return 0;
    if (want64 && coarse_top64_ > 0) dinv64_ = dense_inverse(lev_[coarse_top64_], bytes_);
    if (want32 && coarse_top32_ > 0) {
        size_t scratch = 0;
        double* d = (want64 && coarse_top64_ == coarse_top32_ && dinv64_) ? dinv64_
                                                                          : dense_inverse(lev_[coarse_top32_], scratch);
        if (d) {
            const size_t n2 = lev_[coarse_top32_].N * lev_[coarse_top32_].N;
            if (cudaMalloc(&dinv32_, n2 * 4) == cudaSuccess) {
                k_to_f32<<<(unsigned)((n2 + 255) / 256), 256>>>(d, dinv32_, n2);
                if (cudaDeviceSynchronize() != cudaSuccess) { cudaFree(dinv32_); dinv32_ = nullptr; }
                else bytes_ += n2 * 4;
            }
            if (d != dinv64_) cudaFree(d);
        }
    }
    return 0;
}

template <> int Multigrid::coarse_top<double>() const { return coarse_top64_; }
template <> int Multigrid::coarse_top<float>() const { return coarse_top32_; }

// the arguments of the one-CTA cycle for levels top .. bottom
template <typename T>
static CoarseArgs make_coarse_args(const std::vector<MGLevel>& lev_, int top, int nu1, int nu2, int nu_bottom,
                                   bool has_alpha_, int* d_fvalid_) {
    CoarseArgs A;
    std::memset(&A, 0, sizeof(A));
    const size_t es = sizeof(T);
    size_t wbase = 0;
    coarse_bytes(lev_, top, es, &wbase);
    A.nlev = (int)lev_.size() - top;
    A.nu1 = nu1; A.nu2 = nu2; A.nu_bottom = nu_bottom;
    A.wbase = (long long)wbase;
    A.b_in = lb<T>(const_cast<MGLevel&>(lev_[top]));
    A.x_out = lx<T>(const_cast<MGLevel&>(lev_[top]));
    A.fvalid = d_fvalid_ + (sizeof(T) == 8 ? 0 : 1);
    long long off = 0, woff = 0;
    for (int q = 0; q < A.nlev; ++q) {
        const MGLevel& L = lev_[top + q];
        CoarseLevelDesc& d = A.L[q];
        const long long N = (long long)L.N, nxy = (long long)L.n[0] * L.n[1];
        d.nx = L.n[0]; d.ny = L.n[1]; d.nz = L.n[2]; d.N = (int)N; d.line = L.line;
        d.ihx = 1.0 / (L.h[0] * L.h[0]); d.ihy = 1.0 / (L.h[1] * L.h[1]); d.ihz = 1.0 / (L.h[2] * L.h[2]);
        d.ox = off; off += N;
        d.ob = off; off += N;
        d.obw = off; off += N;
        d.obs = off; off += N;
        d.obb = off; off += N + nxy;
        d.oa = has_alpha_ ? off : -1; off += N;
        d.oq = L.line ? off : -1; off += L.line ? N : 0;
        d.op = L.line ? off : -1; off += L.line ? N : 0;
        d.oi = off; off += N;
        for (int k = 0; k < 3; ++k) {
            if constexpr (sizeof(T) == 8) d.gf[k] = L.fac64[k];
            else d.gf[k] = L.fac32[k];
        }
        if constexpr (sizeof(T) == 8) { d.gbw = L.bw64; d.gbs = L.bs64; d.gbb = L.bb64; d.ga = has_alpha_ ? L.a64 : nullptr; }
        else { d.gbw = L.bw32; d.gbs = L.bs32; d.gbb = L.bb32; d.ga = has_alpha_ ? L.a32 : nullptr; }
        if (top + q + 1 < (int)lev_.size()) {
            const MGLevel& C = lev_[top + q + 1];
            d.rx = C.cr[0]; d.ry = C.cr[1]; d.rz = C.cr[2];
            for (int k = 0; k < 3; ++k) {
                d.gw[k] = C.cr[k] == 2 ? C.wf[k] : nullptr;
                d.ow[k] = C.cr[k] == 2 ? woff : -1;
                if (C.cr[k] == 2) woff += N;
            }
        } else {
            d.rx = d.ry = d.rz = 1;
        }
    }
    return A;
}

template <typename T>
void Multigrid::launch_coarse(int top, cudaStream_t s) {
    const T* dinv = nullptr;
    if constexpr (sizeof(T) == 8) dinv = dinv64_;
    else dinv = dinv32_;
    if (dinv && dense_coarse && !has_alpha_) {
        // the exact solve of the first one-CTA level: x = Ainv b
        const int n = (int)lev_[top].N;
        if (prof) prof->begin(PROF_COARSE_CTA, s);
        ++g_launches;
        launch_k(k_dense_solve<T>, (n * 32 + 255) / 256, 256, 0, s, dinv, (const T*)lb<T>(lev_[top]), lx<T>(lev_[top]), n);
        if (prof) prof->end(s);
        return;
    }
    const CoarseArgs A = make_coarse_args<T>(lev_, top, nu1c >= 0 ? nu1c : nu1, nu2c >= 0 ? nu2c : nu2, nu_bottom,
                                             has_alpha_, d_fvalid_);
    const size_t bytes = coarse_bytes(lev_, top, sizeof(T), nullptr);
    if (prof) prof->begin(PROF_COARSE_CTA, s);
    ++g_launches;
    launch_k(k_coarse_vcycle<T>, 1, 1024, bytes, s, A);
    if (prof) prof->end(s);
}

// a level the row-segment half sweep (k_rbgs_seg) can take with SB-byte
// segments: rows of whole segments, a segment count per row that divides 32
// or is a multiple of it, and every array it reads 16-byte aligned (segment
// starts are then SB-byte aligned, the codes' loads aligned to their width)
template <typename T, int SB>
static bool seg_shape(const MGLevel& L, int l, const Op<T>& o, const T* x, const T* b) {
    constexpr int SEG = SegW<T, SB>::n;
    if (L.line || SEG < 2 || L.n[0] % SEG != 0) return false;
    const int gx = L.n[0] / SEG;
    if (!(gx % 32 == 0 || 32 % gx == 0)) return false;
    auto al = [](const void* p, uintptr_t a) { return ((uintptr_t)p % a) == 0; };
    if (!al(x, 16) || !al(b, 16) || !al(o.a, 16)) return false;
    if (o.zc) return true;
    if (l == 0) return al(o.code + o.nxy, SEG);   // the codes past the ghost layer
    if (o.bwh) return al(o.bwh, 2 * SEG) && al(o.bsh, 2 * SEG) && al(o.bbh, 2 * SEG);
    return al(o.bw, 16) && al(o.bs, 16) && al(o.bb, 16);
}

// the half sweeps of one smoothing pass by SB-byte row segments
template <typename T, int SB>
static void seg_sweeps(const MGLevel& L, int l, const Op<T>& o, T* x, const T* b, int sweeps, bool zero, int cat,
                       Prof* prof, cudaStream_t s) {
    // bx segments of a row per block row, 256 / bx rows per block
    const int gx = L.n[0] / SegW<T, SB>::n, bx = gx < 32 ? gx : 32, by = 256 / bx;
    dim3 b2(bx, by), g2(gx / bx, (L.n[1] + by - 1) / by, L.n[2]);
    for (int it = 0; it < sweeps; ++it)
        for (int color = 0; color < 2; ++color) {
            if (prof) prof->begin(cat, s);
            const bool z = zero && it == 0 && color == 0;
            ++g_launches;
            if (l == 0 && !o.zc) {
                if (z) launch_k(k_rbgs_seg<T, SB, CK_FINE, true>, g2, b2, 0, s, o, x, b, color);
                else launch_k(k_rbgs_seg<T, SB, CK_FINE>, g2, b2, 0, s, o, x, b, color);
            } else if (o.zc) {
                if (z) launch_k(k_rbgs_seg<T, SB, CK_PLANES, true>, g2, b2, 0, s, o, x, b, color);
                else launch_k(k_rbgs_seg<T, SB, CK_PLANES>, g2, b2, 0, s, o, x, b, color);
            } else if (half_faces(o)) {
                if constexpr (sizeof(T) == 4) {
                    if (z) launch_k(k_rbgs_seg<T, SB, CK_HALF, true>, g2, b2, 0, s, o, x, b, color);
                    else launch_k(k_rbgs_seg<T, SB, CK_HALF>, g2, b2, 0, s, o, x, b, color);
                }
            } else {
                if (z) launch_k(k_rbgs_seg<T, SB, CK_ARRAYS, true>, g2, b2, 0, s, o, x, b, color);
                else launch_k(k_rbgs_seg<T, SB, CK_ARRAYS>, g2, b2, 0, s, o, x, b, color);
            }
            if (prof) prof->end(s);
        }
}

// level 0's FP32 arrays can take the split layout for a mixed solve: rows of
// 8-cell groups in whole warps or warp fractions, an even ny (the y wrap keeps
// the colouring), z-only coarsening into level 1 (the split restriction and
// prolongation), the FP64 residual by 32-byte segments, every array aligned
bool Multigrid::split0_ok(const uint8_t* code, std::initializer_list<const void*> p64) const {
    if (!split_mode || seg_bytes == 0 || lev_.size() < 2 || !e32_ || !r32_) return false;
    const MGLevel& L = lev_[0];
    const MGLevel& C = lev_[1];
    if (L.line || (long long)L.N < seg_min_cells || L.n[0] % 8 != 0 || L.n[1] % 2 != 0) return false;
    const int gx = L.n[0] / 8;
    if (!(gx % 32 == 0 || 32 % gx == 0)) return false;
    if (!(C.cr[0] == 1 && C.cr[1] == 1 && C.cr[2] == 2)) return false;
    auto al = [](const void* q, uintptr_t a) { return ((uintptr_t)q % a) == 0; };
    if (!al(e32_, 16) || !al(r32_, 16) || !al(a0_32, 16) || !al(a0_64, 16) || !al(C.wf[2], 16) ||
        !al(C.x32, 16) || !al(C.b32, 16) || !al(code + (size_t)L.n[0] * L.n[1], 8))
        return false;
    for (const void* q : p64)
        if (!al(q, 16)) return false;
    return res_seg() == 32;
}

// a level whose first half sweep can start from an uncleared x (point
// red-black with x / colour pairs)
static bool zero_first_ok(const MGLevel& L) { return !L.line && L.n[0] % 2 == 0; }

template <typename T>
void Multigrid::smooth(const DevParams& p, const uint8_t* code, int l, T* x, const T* b, bool inhom, int sweeps,
                       cudaStream_t s, bool zero) {
    MGLevel& L = lev_[l];
    if (zero && sweeps == 0) {
        // no sweep to start from zero (fx.mg_nu1 = 0): the correction is zero
        cudaMemsetAsync(x, 0, L.N * sizeof(T), s);
        return;
    }
    const T* a = nullptr;
    if (has_alpha_) {
        if (l == 0) { if constexpr (sizeof(T) == 8) a = (const T*)a0_64; else a = (const T*)a0_32; }
        else a = la<T>(L);
    }
    Op<T> o = make_op<T>(L, l, code, eps_, a, inhom, p);
    if constexpr (sizeof(T) == 4) {
        if (l == 0 && split_now_) {
            // level 0 in the split layout: 8 natural cells (4 of one colour) per thread
            const int gx = L.n[0] / 8, bx = gx < 32 ? gx : 32, by = 256 / bx;
            const int Nh = (int)(L.N / 2);
            dim3 b2(bx, by), g2(gx / bx, (L.n[1] + by - 1) / by, L.n[2]);
            for (int it = 0; it < sweeps; ++it)
                for (int color = 0; color < 2; ++color) {
                    if (prof) prof->begin(PROF_SMOOTH_L0, s);
                    const bool z = zero && it == 0 && color == 0;
                    ++g_launches;
                    if (o.zc) {
                        if (z) launch_k(k_rbgs_split<CK_PLANES, true>, g2, b2, 0, s, o, x, b, color, Nh);
                        else launch_k(k_rbgs_split<CK_PLANES>, g2, b2, 0, s, o, x, b, color, Nh);
                    } else {
                        if (z) launch_k(k_rbgs_split<CK_FINE, true>, g2, b2, 0, s, o, x, b, color, Nh);
                        else launch_k(k_rbgs_split<CK_FINE>, g2, b2, 0, s, o, x, b, color, Nh);
                    }
                    if (prof) prof->end(s);
                }
            return;
        }
    }
    if (L.line) {
        T* q = lq<T>(L);
        dim3 b2(32, 4), g2(((L.n[0] + 1) / 2 + 31) / 32, (L.n[1] + 3) / 4, 1);
        for (int it = 0; it < sweeps; ++it)
            for (int color = 0; color < 2; ++color) {
                if (prof) prof->begin(l == 0 ? PROF_SMOOTH_L0 : l == 1 ? PROF_MG_L1 : l == 2 ? PROF_MG_L2 : PROF_MG_COARSE, s);
                ++g_launches;
                if (o.zc) launch_k(k_line<T, CK_PLANES>, g2, b2, 0, s, o, x, b, q, color);
                else if (l == 0) launch_k(k_line<T, CK_FINE>, g2, b2, 0, s, o, x, b, q, color);
                else if (half_faces(o)) {
                    if constexpr (sizeof(T) == 4) launch_k(k_line<T, CK_HALF>, g2, b2, 0, s, o, x, b, q, color);
                } else launch_k(k_line<T, CK_ARRAYS>, g2, b2, 0, s, o, x, b, q, color);
                if (prof) prof->end(s);
            }
    } else if (seg_bytes == 32 && (long long)L.N >= seg_min_cells && seg_shape<T, 32>(L, l, o, x, b)) {
        seg_sweeps<T, 32>(L, l, o, x, b, sweeps, zero,
                          l == 0 ? PROF_SMOOTH_L0 : l == 1 ? PROF_MG_L1 : l == 2 ? PROF_MG_L2 : PROF_MG_COARSE, prof, s);
    } else if (seg_bytes == 16 && (long long)L.N >= seg_min_cells && seg_shape<T, 16>(L, l, o, x, b)) {
        seg_sweeps<T, 16>(L, l, o, x, b, sweeps, zero,
                          l == 0 ? PROF_SMOOTH_L0 : l == 1 ? PROF_MG_L1 : l == 2 ? PROF_MG_L2 : PROF_MG_COARSE, prof, s);
    } else {
        dim3 b2(32, 8), g2(((L.n[0] + 1) / 2 + 31) / 32, (L.n[1] + 7) / 8, L.n[2]);
        for (int it = 0; it < sweeps; ++it)
            for (int color = 0; color < 2; ++color) {
                if (prof) prof->begin(l == 0 ? PROF_SMOOTH_L0 : l == 1 ? PROF_MG_L1 : l == 2 ? PROF_MG_L2 : PROF_MG_COARSE, s);
                const bool z = zero && it == 0 && color == 0;
                ++g_launches;
                if (l == 0 && !o.zc) {
                    if (z) launch_k(k_rbgs<T, CK_FINE, true>, g2, b2, 0, s, o, x, b, color);
                    else launch_k(k_rbgs<T, CK_FINE>, g2, b2, 0, s, o, x, b, color);
                } else {
                    if (o.zc) {
                        if (z) launch_k(k_rbgs<T, CK_PLANES, true>, g2, b2, 0, s, o, x, b, color);
                        else launch_k(k_rbgs<T, CK_PLANES>, g2, b2, 0, s, o, x, b, color);
                    } else {
                        if (half_faces(o)) {
                            if constexpr (sizeof(T) == 4) {
                                if (z) launch_k(k_rbgs<T, CK_HALF, true>, g2, b2, 0, s, o, x, b, color);
                                else launch_k(k_rbgs<T, CK_HALF>, g2, b2, 0, s, o, x, b, color);
                            }
                        } else if (z) launch_k(k_rbgs<T, CK_ARRAYS, true>, g2, b2, 0, s, o, x, b, color);
                        else launch_k(k_rbgs<T, CK_ARRAYS>, g2, b2, 0, s, o, x, b, color);
                    }
                }
                if (prof) prof->end(s);
            }
    }
}

template <typename T>
void Multigrid::vcycle(const DevParams& p, const uint8_t* code, int l, T* x, const T* b, bool inhom, cudaStream_t s,
                       bool zero) {
    MGLevel& L = lev_[l];
    const int last = (int)lev_.size() - 1;
    if (l > 0 && l == coarse_top<T>()) {
        launch_coarse<T>(l, s);
        return;
    }
    if (l == last) {
        const bool exact = L.line && L.n[0] * L.n[1] == 1;
        if (zero && !zero_first_ok(L)) cudaMemsetAsync(x, 0, L.N * sizeof(T), s);
        smooth<T>(p, code, l, x, b, inhom, exact ? 1 : nu_bottom, s, zero && zero_first_ok(L));
        return;
    }
    if (zero && !zero_first_ok(L)) cudaMemsetAsync(x, 0, L.N * sizeof(T), s);
    smooth<T>(p, code, l, x, b, inhom, (l > 0 && nu1c >= 0) ? nu1c : nu1, s, zero && zero_first_ok(L));
    MGLevel& C = lev_[l + 1];
    const T* a = nullptr;
    if (has_alpha_) {
        if (l == 0) { if constexpr (sizeof(T) == 8) a = (const T*)a0_64; else a = (const T*)a0_32; }
        else a = la<T>(L);
    }
    Op<T> o = make_op<T>(L, l, code, eps_, a, inhom, p);
    dim3 b2(32, 8), g2((C.n[0] + 31) / 32, (C.n[1] + 7) / 8, C.n[2]);
    double* norm = (l == 0 && sizeof(T) == 8) ? d_norm_ : nullptr;
    if (prof) prof->begin(l == 0 ? PROF_RESTRICT_L0 : l == 1 ? PROF_MG_L1 : l == 2 ? PROF_MG_L2 : PROF_MG_COARSE, s);
    ++g_launches;
    {
        const int key = (C.cr[0] == 2) * 4 + (C.cr[1] == 2) * 2 + (C.cr[2] == 2);
        T* bc = lb<T>(C);
#define FX_RR(F, RX, RY, RZ) launch_k(k_resid_restrict<T, F, RX, RY, RZ>, g2, b2, 0, s, o, x, b, bc, C.n[0], C.n[1], C.n[2], norm)
#define FX_RR_ALL(F)                                  \
        switch (key) {                                \
        case 1: FX_RR(F, 1, 1, 2); break;             \
        case 2: FX_RR(F, 1, 2, 1); break;             \
        case 3: FX_RR(F, 1, 2, 2); break;             \
        case 4: FX_RR(F, 2, 1, 1); break;             \
        case 5: FX_RR(F, 2, 1, 2); break;             \
        case 6: FX_RR(F, 2, 2, 1); break;             \
        default: FX_RR(F, 2, 2, 2); break;            \
        }
        const int sb = key == 1 && (long long)L.N >= seg_min_cells && ((uintptr_t)bc % 16) == 0
                           ? (seg_bytes == 32 && seg_shape<T, 32>(L, l, o, x, b) ? 32
                              : seg_bytes == 16 && seg_shape<T, 16>(L, l, o, x, b) ? 16 : 0)
                           : 0;
        bool done = false;
        if constexpr (sizeof(T) == 4) {
            if (l == 0 && split_now_) {
                const int gx = L.n[0] / 4, bx = gx < 32 ? gx : 32, by = 256 / bx;
                dim3 bs(bx, by), gs(gx / bx, (L.n[1] + by - 1) / by, C.n[2]);
                const int Nh = (int)(L.N / 2);
                if (o.zc) launch_k(k_rr_z_split<CK_PLANES>, gs, bs, 0, s, o, x, b, bc, Nh);
                else launch_k(k_rr_z_split<CK_FINE>, gs, bs, 0, s, o, x, b, bc, Nh);
                done = true;
            }
        }
        if (done) {
        } else if (sb) {
            // z-semicoarsening by row segments
            const int gx = L.n[0] / (sb / (int)sizeof(T)), bx = gx < 32 ? gx : 32, by = 256 / bx;
            dim3 bs(bx, by), gs(gx / bx, (L.n[1] + by - 1) / by, C.n[2]);
#define FX_RRS(SB) \
            if (o.zc) launch_k(k_rr_z_seg<T, SB, CK_PLANES>, gs, bs, 0, s, o, x, b, bc, norm); \
            else if (l == 0) launch_k(k_rr_z_seg<T, SB, CK_FINE>, gs, bs, 0, s, o, x, b, bc, norm); \
            else if (half_faces(o)) { if constexpr (sizeof(T) == 4) launch_k(k_rr_z_seg<T, SB, CK_HALF>, gs, bs, 0, s, o, x, b, bc, norm); } \
            else launch_k(k_rr_z_seg<T, SB, CK_ARRAYS>, gs, bs, 0, s, o, x, b, bc, norm);
            if (sb == 32) { FX_RRS(32) } else { FX_RRS(16) }
#undef FX_RRS
        } else if (o.zc) { FX_RR_ALL(CK_PLANES) } else if (l == 0) { FX_RR_ALL(CK_FINE) }
        else if (half_faces(o)) { if constexpr (sizeof(T) == 4) { FX_RR_ALL(CK_HALF) } }
        else { FX_RR_ALL(CK_ARRAYS) }
#undef FX_RR_ALL
#undef FX_RR
    }
    if (prof) prof->end(s);
    vcycle<T>(p, code, l + 1, lx<T>(C), lb<T>(C), false, s, true);   // coarse correction from zero
    dim3 g3((L.n[0] + 31) / 32, (L.n[1] + 7) / 8, L.n[2]);
    if (prof) prof->begin(l == 0 ? PROF_PROLONG_L0 : l == 1 ? PROF_MG_L1 : l == 2 ? PROF_MG_L2 : PROF_MG_COARSE, s);
    ++g_launches;
    {
        const int key = (C.cr[0] == 2) * 4 + (C.cr[1] == 2) * 2 + (C.cr[2] == 2);
        T* xc = lx<T>(C);
#define FX_PR(RX, RY, RZ) launch_k(k_prolong<T, RX, RY, RZ>, g3, b2, 0, s, x, xc, C.wf[0], C.wf[1], C.wf[2], L.n[0], L.n[1], L.n[2], C.n[0], C.n[1], C.n[2])
        bool done = false;
        if constexpr (sizeof(T) == 4) {
            if (l == 0 && split_now_) {
                const int gx = L.n[0] / 8, bx = gx < 32 ? gx : 32, by = 256 / bx;
                dim3 bs(bx, by), gs(gx / bx, (L.n[1] + by - 1) / by, L.n[2]);
                launch_k(k_prolong_z_split, gs, bs, 0, s, x, xc, C.wf[2], L.n[0], L.n[1], C.n[2], (int)(L.N / 2));
                done = true;
            }
        }
        auto al16 = [](const void* q) { return ((uintptr_t)q % 16) == 0; };
        const int sb = !done && key == 1 && (long long)L.N >= seg_min_cells && al16(xc) && al16(C.wf[2])
                           ? (seg_bytes == 32 && seg_shape<T, 32>(L, l, o, x, b) ? 32
                              : seg_bytes == 16 && seg_shape<T, 16>(L, l, o, x, b) ? 16 : 0)
                           : 0;
        if (done) {
        } else if (sb) {
            const int gx = L.n[0] / (sb / (int)sizeof(T)), bx = gx < 32 ? gx : 32, by = 256 / bx;
            dim3 bs(bx, by), gs(gx / bx, (L.n[1] + by - 1) / by, L.n[2]);
            if (sb == 32) launch_k(k_prolong_z_seg<T, 32>, gs, bs, 0, s, x, xc, C.wf[2], L.n[0], L.n[1], C.n[2]);
            else launch_k(k_prolong_z_seg<T, 16>, gs, bs, 0, s, x, xc, C.wf[2], L.n[0], L.n[1], C.n[2]);
        } else
        switch (key) {
        case 1: FX_PR(1, 1, 2); break;
        case 2: FX_PR(1, 2, 1); break;
        case 3: FX_PR(1, 2, 2); break;
        case 4: FX_PR(2, 1, 1); break;
        case 5: FX_PR(2, 1, 2); break;
        case 6: FX_PR(2, 2, 1); break;
        default: FX_PR(2, 2, 2); break;
        }
#undef FX_PR
    }
    if (prof) prof->end(s);
    smooth<T>(p, code, l, x, b, inhom, (l > 0 && nu2c >= 0) ? nu2c : nu2, s, false);
}

int Multigrid::residual64(const DevParams& p, const uint8_t* code, const double* phi, const double* rhs, double* r,
                          cudaStream_t s, double* norm_out) {
    MGLevel& L = lev_[0];
    Op<double> o = make_op<double>(L, 0, code, eps_, has_alpha_ ? a0_64 : nullptr, true, p);
    cudaMemsetAsync(d_norm_, 0, NORM_SLOTS * 8, s);
    dim3 b2(32, 8), g2((L.n[0] + 31) / 32, (L.n[1] + 7) / 8, L.n[2]);
    (void)r;
    if (prof) prof->begin(PROF_RESID64, s);
    { ++g_launches; launch_resid64<false>(o, dim3(g2.x, g2.y, (L.n[2] + R64_ZP - 1) / R64_ZP), b2, s, phi, nullptr, rhs, nullptr, nullptr, d_norm_, ResidCtl{}, res_seg()); }
    if (prof) prof->end(s);
    cudaMemcpyAsync(h_norm_, d_norm_, NORM_SLOTS * 8, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (norm_out) *norm_out = slots_max();
    cudaMemsetAsync(d_norm_, 0, NORM_SLOTS * 8, s);   // the slots are zero between uses
    return (int)e;
}

template <typename F>
int Multigrid::replay(GraphCache& g, const void* x, const void* rhs, const DevParams& p, cudaStream_t s, F&& enqueue) {
    const bool profiling = prof && prof->on;
    if (!use_graphs_ || profiling) {
        enqueue();
        return (int)cudaGetLastError();
    }
    if (!g.exec || g.x != x || g.rhs != rhs || g.has_alpha != has_alpha_ || g.vlo != p.V_lo || g.vhi != p.V_hi ||
        g.nu1 != nu1 || g.nu2 != nu2 || g.nu1c != nu1c || g.nu2c != nu2c || g.pdl != g_pdl ||
        g.seg != seg_bytes || g.seg_min != seg_min_cells || g.split != split_now_ || g.dense != dense_coarse) {
        if (g.exec) { cudaGraphExecDestroy(g.exec); g.exec = nullptr; }
        cudaGraph_t graph;
        const long long l0 = g_launches.load();
        cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e) return (int)e;
        enqueue();
        e = cudaStreamEndCapture(s, &graph);
        if (e) return (int)e;
        g.launches = g_launches.load() - l0;
        g_launches -= g.launches;    // counted per replay below
        e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e) return (int)e;
        g.x = x; g.rhs = rhs; g.has_alpha = has_alpha_; g.vlo = p.V_lo; g.vhi = p.V_hi; g.nu1 = nu1; g.nu2 = nu2;
        g.nu1c = nu1c; g.nu2c = nu2c;
        g.pdl = g_pdl; g.seg = seg_bytes; g.seg_min = seg_min_cells; g.split = split_now_; g.dense = dense_coarse;
    }
    g_launches += g.launches;
    return (int)cudaGraphLaunch(g.exec, s);
}

int Multigrid::solve64(const DevParams& p, const uint8_t* code, double* phi, const double* rhs, double target,
                       int maxit, cudaStream_t s, MGStats* st) {
    int it = 0;
    double rn = 0.0;
    int e = residual64(p, code, phi, rhs, nullptr, s, &rn);
    if (e) return e;
    while (!(rn <= target) && std::isfinite(rn) && it < maxit) {
        // one V-cycle; the level-0 residual norm after pre-smoothing bounds
        // the residual after the cycle, so it is the loop test; the exact
        // final residual is checked before returning
        e = replay(g64_, phi, rhs, p, s, [&]() {
            cudaMemsetAsync(d_norm_, 0, NORM_SLOTS * 8, s);
            vcycle<double>(p, code, 0, phi, rhs, true, s, false);
            cudaMemcpyAsync(h_norm_, d_norm_, NORM_SLOTS * 8, cudaMemcpyDeviceToHost, s);
        });
        if (e) return e;
        e = (int)cudaStreamSynchronize(s);
        if (e) return e;
        ++it;
        const double mid = slots_max();
        if (verbose > 1) printf("  mg cycle %d: |r|/target after pre-smoothing = %.3e\n", it, mid / target);
        if (lev_.size() == 1) { e = residual64(p, code, phi, rhs, nullptr, s, &rn); if (e) return e; continue; }
        if (mid <= target || !std::isfinite(mid)) {
            e = residual64(p, code, phi, rhs, nullptr, s, &rn);
            if (e) return e;
        } else {
            rn = mid;
        }
    }
    if (st) { st->cycles = it; st->resid = rn; }
    cudaMemsetAsync(d_norm_, 0, NORM_SLOTS * 8, s);
    return (rn <= target && std::isfinite(rn)) ? 0 : -3;
}

int Multigrid::solve_mixed(const DevParams& p, const uint8_t* code, double* phi, const double* rhs, double target,
                           int maxit, cudaStream_t s, MGStats* st) {
    MGLevel& L = lev_[0];
    Op<double> o64 = make_op<double>(L, 0, code, eps_, has_alpha_ ? a0_64 : nullptr, true, p);
    dim3 b2(32, 8), g2((L.n[0] + 31) / 32, (L.n[1] + 7) / 8, (L.n[2] + R64_ZP - 1) / R64_ZP);
    // the FP64 iterate alternates between phi and alt64m_: each refinement
    // step adds the FP32 correction while it forms the next residual
    double* buf[2] = {phi, alt64m_};
    int cur = 0;
    split_now_ = split0_ok(code, {phi, rhs, alt64m_});
    cudaMemsetAsync(d_norm_, 0, NORM_SLOTS * 8, s);
    if (prof) prof->begin(PROF_RESID64, s);
    ++g_launches;
    launch_resid64<false>(o64, g2, b2, s, phi, nullptr, rhs, nullptr, r32_, d_norm_, ResidCtl{}, res_seg(), split_now_);
    if (prof) prof->end(s);
    cudaMemcpyAsync(h_norm_, d_norm_, NORM_SLOTS * 8, cudaMemcpyDeviceToHost, s);
    int e = (int)cudaStreamSynchronize(s);
    if (e) return e;
    double rn = slots_max();
    int it = 0, cycles = 0;
    const int inner = std::max(1, mixed_cycles);
    if (verbose > 1) printf("  refinement %d: |r|/target = %.3e\n", it, rn / target);
    while (!(rn <= target) && std::isfinite(rn) && cycles < maxit) {
        // FP32 correction cycles on the FP32 residual, then the FP64 update
        // fused with the FP64 residual of the updated iterate
        double* xin = buf[cur];
        double* xout = buf[1 - cur];
        e = replay(cur == 0 ? g32_ : g32b_, xin, rhs, p, s, [&]() {
            for (int q = 0; q < inner; ++q) vcycle<float>(p, code, 0, e32_, r32_, false, s, q == 0);
            cudaMemsetAsync(d_norm_, 0, NORM_SLOTS * 8, s);
            if (prof) prof->begin(PROF_RESID64, s);
            ++g_launches;
            launch_resid64<true>(o64, g2, b2, s, xin, e32_, rhs, xout, r32_, d_norm_, ResidCtl{}, res_seg(), split_now_);
            if (prof) prof->end(s);
            cudaMemcpyAsync(h_norm_, d_norm_, NORM_SLOTS * 8, cudaMemcpyDeviceToHost, s);
        });
        if (e) return e;
        e = (int)cudaStreamSynchronize(s);
        if (e) return e;
        cur = 1 - cur;
        ++it;
        cycles += inner;
        rn = slots_max();
        if (verbose > 1) printf("  refinement %d: |r|/target = %.3e\n", it, rn / target);
    }
    if (cur == 1) {
        e = (int)cudaMemcpyAsync(phi, buf[1], L.N * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (e) return e;
    }
    if (st) { st->cycles = cycles; st->resid = rn; }
    cudaMemsetAsync(d_norm_, 0, NORM_SLOTS * 8, s);
    return (rn <= target && std::isfinite(rn)) ? 0 : -3;
}

// The loop of solve64 with its tests on the device: a WHILE node runs one
// V-cycle per pass; k_mg_mid decides from the pre-smoothing norm whether the
// exact residual is needed (the residual kernel after it returns at once
// otherwise) and whether another cycle follows.  The residual kernel's last
// block runs the test on the exact residual (and the first test, on the
// initial residual).  The norm slots are left zeroed by whoever reads them.  end_in_next: the next kernel (the charge kernel of
// a Newton pass) closes the solve, else k_mg_end does.
void Multigrid::enqueue_solve64_ctl(const DevParams& p, const uint8_t* code, double* phi, const double* rhs,
                                    const double* nb, double rtol, int maxit, StepCtl* ctl, CondCapture& cap,
                                    cudaStream_t s, bool end_in_next) {
    MGLevel& L = lev_[0];
    Op<double> o = make_op<double>(L, 0, code, eps_, has_alpha_ ? a0_64 : nullptr, true, p);
    const dim3 b2(32, 8), g2((L.n[0] + 31) / 32, (L.n[1] + 7) / 8, (L.n[2] + R64_ZP - 1) / R64_ZP);
    const int single = lev_.size() == 1 ? 1 : 0;
    const cudaGraphConditionalHandle hw = cap.handle(s);
    // the norm slots are zero between uses
    ResidCtl rb = {ctl, RC_BEGIN, nb, rtol, maxit, 0, 0, 0, hw, hw, rc_counter_};
    ++g_launches;
    launch_resid64<false>(o, g2, b2, s, phi, nullptr, rhs, nullptr, nullptr, d_norm_, rb, res_seg());
    cap.node(s, cudaGraphCondTypeWhile, hw, KIND_MG_CYCLE, [&](cudaStream_t b) {
        vcycle<double>(p, code, 0, phi, rhs, true, b, false);
        ++g_launches;
        launch_k(k_mg_mid, 1, 1, 0, b, d_norm_, single, maxit, ctl, hw);
        ResidCtl rr = {ctl, RC_RN, nullptr, 0.0, maxit, 0, 0, 0, hw, hw, rc_counter_};
        ++g_launches;
        launch_resid64<false>(o, g2, b2, b, phi, nullptr, rhs, nullptr, nullptr, d_norm_, rr, res_seg());
    });
    if (!end_in_next) {
        ++g_launches;
        launch_k(k_mg_end, 1, 1, 0, s, ctl);
    }
}

// The loop of solve_mixed with its tests on the device.  The iterate
// alternates between phi and the second buffer, so one WHILE pass holds two
// refinement steps, the second inside an IF node; each step's FP64 residual
// kernel runs the test in its last block; k_mx_copy brings the iterate back
// into phi when it ends in the second buffer.
void Multigrid::enqueue_solve_mixed_ctl(const DevParams& p, const uint8_t* code, double* phi, const double* rhs,
                                        const double* nb, double rtol, int maxit, StepCtl* ctl, CondCapture& cap,
                                        cudaStream_t s, bool end_in_next) {
    MGLevel& L = lev_[0];
    Op<double> o64 = make_op<double>(L, 0, code, eps_, has_alpha_ ? a0_64 : nullptr, true, p);
    const dim3 b2(32, 8), g2((L.n[0] + 31) / 32, (L.n[1] + 7) / 8, (L.n[2] + R64_ZP - 1) / R64_ZP);
    const int inner = std::max(1, mixed_cycles);
    const cudaGraphConditionalHandle hw = cap.handle(s);
    ResidCtl rb = {ctl, RC_BEGIN, nb, rtol, maxit, 0, 0, 0, hw, hw, rc_counter_};
    split_now_ = split0_ok(code, {phi, rhs, alt64m_});
    ++g_launches;
    launch_resid64<false>(o64, g2, b2, s, phi, nullptr, rhs, nullptr, r32_, d_norm_, rb, res_seg(), split_now_);
    auto refine = [&](cudaStream_t q, const double* xin, double* xout, const ResidCtl& rc) {
        for (int k = 0; k < inner; ++k) vcycle<float>(p, code, 0, e32_, r32_, false, q, k == 0);
        ++g_launches;
        launch_resid64<true>(o64, g2, b2, q, xin, e32_, rhs, xout, r32_, d_norm_, rc, res_seg(), split_now_);
    };
    cap.node(s, cudaGraphCondTypeWhile, hw, KIND_MX_FIRST, [&](cudaStream_t b) {
        const cudaGraphConditionalHandle hif = cap.handle(b);
        refine(b, phi, alt64m_, ResidCtl{ctl, RC_MX, nullptr, 0.0, maxit, inner, 1, KIND_MX_FIRST, hif, hw, rc_counter_});
        cap.node(b, cudaGraphCondTypeIf, hif, KIND_MX_SECOND, [&](cudaStream_t q) {
            refine(q, alt64m_, phi, ResidCtl{ctl, RC_MX, nullptr, 0.0, maxit, inner, 0, KIND_MX_SECOND, hw, hw, rc_counter_});
        });
    });
    ++g_launches;
    launch_k(k_mx_copy, (int)std::min<size_t>((L.N + 255) / 256, 4 * 148), 256, 0, s, alt64m_, phi, (int)L.N, ctl);
    if (!end_in_next) {
        ++g_launches;
        launch_k(k_mg_end, 1, 1, 0, s, ctl);
    }
}

template void Multigrid::vcycle<double>(const DevParams&, const uint8_t*, int, double*, const double*, bool, cudaStream_t, bool);
template void Multigrid::vcycle<float>(const DevParams&, const uint8_t*, int, float*, const float*, bool, cudaStream_t, bool);

}  // namespace fx
