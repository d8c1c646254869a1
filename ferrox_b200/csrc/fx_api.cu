// fx_api.cu -- context, host-side setup and the C ABI (include/ferrox_b200.h).
//
// Host setup restates the reference's initialization (masks, permittivity,
// initial P, electrode values); the per-step work is the device kernels of
// fx_kernels.cu and the multigrid of fx_mg.cu, ordered on one stream.  There
// is no CPU compute path: every hot-path function launches device kernels
// and returns FX_ERR_CUDA when no device is usable.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ferrox_b200.h"
#include "fx_kernels.h"
#include "fx_mg.h"
#include "fx_params.h"
#include "plotfile.h"

namespace {
thread_local std::string t_create_error;
}

namespace fx {
std::atomic<long long> g_launches{0};
bool g_pdl = true;
bool g_rhs_seg = true;
// message of the last failed call that has no context (fx_create and the
// context-free entry points)
void set_free_error(const std::string& m) { t_create_error = m; }
}

using namespace fx;

namespace {

// Silicon constants, Source/FerroX.cpp:534-554
constexpr double kNc = 2.8e25, kNv = 1.83e25, kEg = 1.12, kChi = 4.05, kQ = 1.602e-19, kKb = 1.38e-23, kT = 300.0;
constexpr double kEa = 44.0e-3, kEd = 46.0e-3;

uint64_t splitmix_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
// n-th draw (n >= 1) of a splitmix64 stream seeded with `seed`, in [0, 1)
double uniform(uint64_t seed, uint64_t n) {
    return (double)(splitmix_mix(seed + n * 0x9E3779B97F4A7C15ULL) >> 11) * (1.0 / 9007199254740992.0);
}

// rotation from Euler angles in degrees, TotalEnergyDensity.cpp:167-195
void rotation(int use_euler, double a_deg, double b_deg, double t_deg, double R[9]) {
    double Pi = 3.14159265358979323846;
    double alpha_rad = Pi / 180. * a_deg, beta_rad = Pi / 180. * b_deg, theta_rad = Pi / 180. * t_deg;
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

struct FxError {
    int code;
    std::string msg;
};

}  // namespace

// highest order of the time extrapolation of a step's first solve
constexpr int kMaxExtrap = 6;

struct fx_ctx {
    Params par;
    Inputs in;
    DevParams dp{};
    // an embedded boundary covering the layers k >= eb_nz: the Poisson solve
    // runs on the fluid layers below it, their top face the embedded
    // Dirichlet surface at eb_V (read_embedded_boundary, poisson_params)
    int eb_nz = 0;                       // 0: no embedded boundary
    double eb_V = 0.0;
    int nx = 0, ny = 0, nz = 0;
    size_t N = 0, nxy = 0;
    double dx[3] = {0, 0, 0};
    std::string err;

    // host setup
    std::vector<uint8_t> code;           // (nz+2)*nxy, mask | tphase << 2
    std::vector<double> mask_ref;        // reference ghosted mask (nx+2)(ny+2)(nz+2)
    std::vector<double> tphase, ang[3];  // valid cells
    std::vector<uint8_t> var;            // per-cell variant id (empty: identity R everywhere)
    std::vector<Variant> variants;
    std::vector<double> P0[3];
    std::vector<uint8_t> gid;            // per-cell grain id (255: none) once grains are set
    std::vector<double> galpha;          // per-grain Landau alpha (empty: global alpha)
    bool scalarP = true;                 // Px = Py = 0 and is_polarization_scalar
    bool contains_sc = false;
    bool grains_set = false;
    int ngrains = 0;
    bool user_P = false;

    // loop state, main.cpp:238-242
    int step = 0;
    int steady_state_step = 1000000;
    int sign = 1;
    int num_Vapp = 0;
    int inc_step = -1;
    double time = 0.0;
    double Phi_Bc_hi = 0.0;
    bool finished = false;
    double phi_max_last = 0.0;

    // stats
    int newton_last = 0, mg_last = 0;
    long long newton_total = 0, mg_total = 0;
    double mg_resid_last = 0, mg_target_last = 0, phi_err_last = 0, steady_err_last = 0;

    // device
    bool dev = false;
    cudaStream_t s = nullptr;
    bool own_stream = true;
    Prof prof;
    uint8_t *d_code = nullptr, *d_var = nullptr;
    uint8_t* d_interior = nullptr;       // DevParams::interior flags
    bool use_interior = true;            // fx.interior
    bool adj_store_phi = true;           // fx.adjoint_store_phi
    bool adj_extrap = true;          // the adjoint solves start from psi extrapolated in reverse time
    double* adj_phi_store = nullptr;     // the record's phi of every step; kept between records
    size_t adj_phi_store_n = 0;          // its length in doubles
    Variant* d_vt = nullptr;
    double* d_P[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int cur = 0;
    double *d_phi = nullptr, *d_phi_old = nullptr, *d_phi_prev = nullptr, *d_rho = nullptr, *d_e = nullptr, *d_h = nullptr;
    double *d_alpha = nullptr, *d_rhs = nullptr, *d_rhsP = nullptr, *d_dphi = nullptr, *d_E[3] = {nullptr, nullptr, nullptr};
    double* d_f[3] = {nullptr, nullptr, nullptr};   // f^n of the Order-2 predictor
    float* d_alpha32 = nullptr;
    double* d_part = nullptr;
    unsigned int* d_counter = nullptr;
    double* d_out = nullptr;
    double* h_out = nullptr;
    bool E_valid = false;
    bool rhs_is_newton = false;
    // the Newton loop leaves the carrier densities unwritten: they are formed
    // from phi (which the last charge evaluation used) when read
    bool carriers_stale = false;
    // phi of the previous step's first solve, for the extrapolated initial
    // iterate; valid only while nothing but time steps changed the state
    double* d_phi_hist[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};   // phi of the last steps' first solves
    int hist_n = 0;                                // how many of them are current
    bool hist_valid = false;
    double hist_vlo = 0.0, hist_vhi = 0.0;
    size_t dev_bytes = 0;
    Multigrid mg;
    bool mg_ready = false;

    // the step as one CUDA graph with its loops controlled on the device
    // (fx_ctl.h); graphs are cached by everything their capture bakes in
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        std::vector<unsigned char> key;
        long long top = 0;                 // kernel launches outside conditional bodies
        long long own[KIND_N] = {};        // per execution of each body kind
    };
    std::vector<StepGraph> sgraphs;
    StepCtl* d_ctl = nullptr;
    StepCtl* h_ctl = nullptr;              // pinned
    CondCapture cap;
    bool sg_off = false;                   // capture failed once: the host-driven loop from then on
    bool sg_ran = false;                   // the last step ran as a graph

    // bumped by every call that changes the state or a parameter of the
    // math; fx_backward requires the value fx_forward_record saw
    long long gen = 0;
    std::vector<uint8_t> variant_global_alpha;   // per variant: alpha is the global alpha

    // gradient record (fx_forward_record / fx_backward)
    struct AdjRecord {
        bool valid = false;
        long long gen = -1;
        int T = 0, k = 0, nck = 0;
        long long nfe = 0;
        std::vector<double> V, shape, target, m;
        double loss = 0.0;
        std::vector<void*> allocs;                 // freed together
        size_t bytes = 0;
        std::vector<double*> ckP, ckPhi, ckRho;    // 3 per checkpoint (null for unused components), 1, 1
        double* finP[3] = {nullptr, nullptr, nullptr};
        double *finPhi = nullptr, *finRho = nullptr;
        std::vector<double*> segP, segPhi;         // 3 per segment step, 1 (semiconductor only)
        double* phiAll = nullptr;                  // phi^n of every recorded step (n = 1..T), when it fits
        double* lam[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
        int lcur = 0;
        double *mu = nullptr, *psi = nullptr, *drho = nullptr, *grad = nullptr, *dV = nullptr, *hist = nullptr;
        double* psiHist[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};   // psi of the last reverse steps
        int psi_n = 0;                             // reverse steps of psi history held
        double* nmu = nullptr;                     // max|mu| of the reverse step (device), and a zero
        cudaGraphExec_t solve_exec = nullptr;      // the reverse step's adjoint solve as a graph (this backward)
        float* drho32 = nullptr;
        uint8_t* gid = nullptr;
        bool have_P0 = false;
        long long mg_cycles = 0;
        double fwd_ms = 0.0, bwd_ms = 0.0;
    } adj;
};

namespace {

int set_err(fx_ctx* c, int code, const std::string& m) {
    if (c) c->err = m;
    return code;
}

#define FX_CUDA(ctx, call)                                                                         \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? FX_ERR_OUT_OF_MEMORY : FX_ERR_CUDA, \
                           std::string(#call) + ": " + cudaGetErrorString(e_));                    \
    } while (0)

double eps_of_code(const Params& p, int code) {
    // InitializePermittivity, ElectrostaticSolver.cpp:238-251
    const int m = code & 3, tph = (code >> 2) & 1;
    if (m == 0) return tph ? p.epsilonX_fe_tphase * p.epsilon_0 : p.epsilonX_fe * p.epsilon_0;
    if (m == 1) return p.epsilon_de * p.epsilon_0;
    return p.epsilon_si * p.epsilon_0;
}

double phi_ref() { return kChi + 0.5 * kEg + 0.5 * kKb * kT * log(kNc / kNv) / kQ; }

// Embedded boundaries (domain.embedded_boundary = 1; EmbeddedBoundaries.cpp:66-140
// reads the objects, ElectrostaticSolver.cpp:613-676 hands them to MLEBABecLap
// with setEBDirichlet) in the form the reference's FET decks give them: one
// `box` object with no fluid inside that spans the periodic x / y extent and
// covers z from a cell face up to the top of the domain (inputs_mfim_eb:
// z >= 9 nm of 10 nm; inputs_mfis_eb: z >= 16 nm of 17 nm).  The embedded
// surface is then the plane z = box_lo[2], a face of the grid: the cells
// below it are whole fluid cells whose top face carries the Dirichlet value
// surf_soln (ebgeom.specify_inhomo_dir = 1; 0 V otherwise), the cells above
// are covered.  A cut-cell geometry -- a surface through the cells, or one
// that does not span x / y -- needs AMReX's EB2 volume and area fractions and
// is refused, as are planes, parser and STL objects, EB2 input and unions.
void read_embedded_boundary(fx_ctx* c) {
    const auto& T = c->in.table;
    const auto& K = c->in.constants;
    auto first = [&](const std::string& key) -> const std::string* {
        auto it = T.find(key);
        return (it == T.end() || it->second.empty()) ? nullptr : &it->second[0];
    };
    auto num = [&](const std::string& key, double dflt) {
        const std::string* v = first(key);
        return v ? eval_number(*v, K) : dflt;
    };
    if (num("domain.embedded_boundary", 0.0) == 0.0) return;
    auto refuse = [](const std::string& why) {
        throw FxError{FX_ERR_UNSUPPORTED, "embedded boundary: " + why +
                                              " (only a box object spanning x / y from a cell face to the top of z, "
                                              "whose surface lies on grid faces, is supported; cut cells are not)"};
    };
    if (num("ebgeom.specify_input_using_eb2", 0.0) != 0.0) refuse("ebgeom.specify_input_using_eb2 = 1");
    auto it = T.find("ebgeom.objects");
    if (it == T.end() || it->second.empty()) refuse("no ebgeom.objects");
    if (it->second.size() != 1) refuse("a union of " + std::to_string(it->second.size()) + " objects");
    const std::string name = it->second[0];
    const std::string* type = first(name + ".geom_type");
    if (!type) throw FxError{FX_ERR_INPUTS, "inputs: " + name + ".geom_type is missing"};
    if (*type != "box") refuse("geom_type " + *type);
    auto arr3 = [&](const std::string& key, double out[3]) {
        auto a = T.find(key);
        if (a == T.end() || a->second.size() < 3) throw FxError{FX_ERR_INPUTS, "inputs: " + key + " needs 3 entries"};
        for (int d = 0; d < 3; ++d) out[d] = eval_number(a->second[d], K);
    };
    double lo[3], hi[3];
    arr3(name + ".box_lo", lo);
    arr3(name + ".box_hi", hi);
    const std::string* fluid = first(name + ".has_fluid_inside");
    if (!fluid) throw FxError{FX_ERR_INPUTS, "inputs: " + name + ".has_fluid_inside is missing"};
    if (*fluid == "1" || *fluid == "true") refuse(name + ".has_fluid_inside = 1");
    if (!(*fluid == "0" || *fluid == "false")) throw FxError{FX_ERR_INPUTS, "inputs: " + name + ".has_fluid_inside must be 0 or 1"};
    const Params& p = c->par;
    double dx[3];
    for (int d = 0; d < 3; ++d) dx[d] = (p.prob_hi[d] - p.prob_lo[d]) / p.n_cell[d];
    for (int d = 0; d < 2; ++d)
        if (lo[d] > p.prob_lo[d] + 1e-6 * dx[d] || hi[d] < p.prob_hi[d] - 1e-6 * dx[d])
            refuse(name + " does not span the domain in " + std::string(d ? "y" : "x"));
    if (hi[2] < p.prob_hi[2] - 1e-6 * dx[2]) refuse(name + " does not reach the top of the domain");
    const double f = (lo[2] - p.prob_lo[2]) / dx[2];
    const long kb = std::lround(f);
    if (std::fabs(f - (double)kb) > 1e-6) refuse(name + ".box_lo[2] is not on a cell face");
    if (kb < 1 || kb >= p.n_cell[2]) refuse(name + " leaves no fluid layer or covers no cell");
    c->eb_nz = (int)kb;
    c->eb_V = 0.0;
    if (num("ebgeom.specify_inhomo_dir", 0.0) != 0.0) {
        const std::string* v = first(name + ".surf_soln");
        if (!v) throw FxError{FX_ERR_INPUTS, "inputs: " + name + ".surf_soln is missing (ebgeom.specify_inhomo_dir = 1)"};
        c->eb_V = eval_number(*v, K);
    }
}

// SetPhiBC_z values, ElectrostaticSolver.cpp:512-519
void electrode_values(fx_ctx* c) {
    const double pr = phi_ref();
    const double phi_m = c->par.use_work_function ? c->par.metal_work_function : pr;
    c->dp.V_lo = c->par.Phi_Bc_lo;
    c->dp.V_hi = c->Phi_Bc_hi - (phi_m - pr);
    c->dp.Ns = c->eb_nz > 0 ? (long long)c->nxy * c->eb_nz : (long long)c->N;
    c->dp.Vs_hi = c->eb_nz > 0 ? c->eb_V : c->dp.V_hi;
}

// The grid as the Poisson solver sees it.  With an embedded boundary the
// solve covers the fluid layers k < eb_nz, a prefix of every cell array, and
// their top face is the embedded surface: a Dirichlet face at surf_soln
// (setEBDirichlet, ElectrostaticSolver.cpp:668-672, takes it as given, with
// the cut cell's own beta_cc), at half a cell from the layer's centres like
// an electrode.  The covered cells are not part of the solve; phi there keeps
// the 0 that every solve of ComputePhi_Rho_EB starts from
// (ElectrostaticSolver.cpp:787).
DevParams poisson_params(const fx_ctx* c) {
    DevParams d = c->dp;
    if (c->eb_nz > 0) {
        d.nz = c->eb_nz;
        d.N = d.nxy * c->eb_nz;
        d.ngrid_red = (int)std::min<long long>(std::max<long long>((d.N + 255) / 256, 1), 148 * 8);
        d.V_hi = c->eb_V;
    }
    return d;
}

// InitializeMaterialMask, Initialization.cpp:184-202 at one cell centre
double mask_at(const Params& p, double x, double y, double z) {
    if (x <= p.FE_hi[0] && x >= p.FE_lo[0] && y <= p.FE_hi[1] && y >= p.FE_lo[1] && z <= p.FE_hi[2] && z >= p.FE_lo[2]) return 0.;
    if (x <= p.DE_hi[0] && x >= p.DE_lo[0] && y <= p.DE_hi[1] && y >= p.DE_lo[1] && z <= p.DE_hi[2] && z >= p.DE_lo[2]) return 1.;
    if (x <= p.SC_hi[0] && x >= p.SC_lo[0] && y <= p.SC_hi[1] && y >= p.SC_lo[1] && z <= p.SC_hi[2] && z >= p.SC_lo[2]) {
        if (x <= p.Channel_hi[0] && x >= p.Channel_lo[0] && y <= p.Channel_hi[1] && y >= p.Channel_lo[1] && z <= p.Channel_hi[2] && z >= p.Channel_lo[2])
            return 3.;
        return 2.;
    }
    return 1.;
}

void build_codes(fx_ctx* c) {
    const Params& p = c->par;
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const size_t gx = nx + 2, gy = ny + 2;
    c->mask_ref.assign(gx * gy * (nz + 2), 0.0);
    auto G = [&](int i, int j, int k) -> double& { return c->mask_ref[(size_t)(i + 1) + gx * ((size_t)(j + 1) + gy * (size_t)(k + 1))]; };
    for (int k = -1; k <= nz; ++k)
        for (int j = -1; j <= ny; ++j)
            for (int i = -1; i <= nx; ++i)
                G(i, j, k) = mask_at(p, p.prob_lo[0] + (i + 0.5) * c->dx[0], p.prob_lo[1] + (j + 0.5) * c->dx[1],
                                     p.prob_lo[2] + (k + 0.5) * c->dx[2]);
    // FillBoundary with the x/y periodic images that are valid cells
    for (int k = -1; k <= nz; ++k)
        for (int j = -1; j <= ny; ++j)
            for (int i = -1; i <= nx; ++i) {
                const bool gxo = i < 0 || i >= nx, gyo = j < 0 || j >= ny, gzo = k < 0 || k >= nz;
                if ((gxo || gyo) && !gzo) G(i, j, k) = G((i + nx) % nx, (j + ny) % ny, k);
            }
    c->code.assign((size_t)nx * ny * (nz + 2), 0);
    for (int k = -1; k <= nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                int m = (int)G(i, j, k);
                int t = 0;
                if (k >= 0 && k < nz) t = c->tphase[(size_t)i + nx * ((size_t)j + (size_t)ny * k)] == 1.0 ? 1 : 0;
                c->code[(size_t)i + nx * ((size_t)j + (size_t)ny * (k + 1))] = (uint8_t)(m | (t << 2));
            }
    c->contains_sc = false;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                if (G(i, j, k) >= 2.0) c->contains_sc = true;
}

// the device reads the mask of a ghost cell through periodic wrapping; check
// that this equals the reference's ghosted mask wherever the stencils read it
std::string check_wrapped_mask(fx_ctx* c) {
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const size_t gx = nx + 2, gy = ny + 2;
    for (int k = -1; k <= nz; ++k)
        for (int j = -1; j <= ny; ++j)
            for (int i = -1; i <= nx; ++i) {
                const double ref = c->mask_ref[(size_t)(i + 1) + gx * ((size_t)(j + 1) + gy * (size_t)(k + 1))];
                const int w = c->code[(size_t)((i + nx) % nx) + nx * ((size_t)((j + ny) % ny) + (size_t)ny * (k + 1))] & 3;
                if (ref != (double)w) {
                    std::ostringstream o;
                    o << "material boxes distinguish a periodic ghost corner from its image at cell (" << i << "," << j << "," << k
                      << "): mask " << ref << " vs " << w << "; the device layout wraps x/y ghosts";
                    return o.str();
                }
            }
    return "";
}

void build_variants(fx_ctx* c, const std::vector<uint8_t>* gid, const std::vector<double>* galpha) {
    c->var.clear();
    c->variants.clear();
    c->variant_global_alpha.clear();
    const size_t N = c->N;
    bool any = false;
    if (gid) any = true;
    for (int d = 0; d < 3 && !any; ++d)
        for (size_t q = 0; q < N; ++q)
            if (c->ang[d][q] != 0.0) { any = true; break; }
    if (!any) return;
    std::map<std::tuple<double, double, double, int, double>, uint8_t> ids;
    c->var.assign(N, 0);
    for (size_t q = 0; q < N; ++q) {
        double al = c->par.alpha;
        const bool own = gid && galpha && (*gid)[q] != 255 && (*gid)[q] < galpha->size();
        if (own) al = (*galpha)[(*gid)[q]];
        // a grain alpha equal to the global one stays a separate variant, so
        // that changing the global alpha later leaves it alone
        auto key = std::make_tuple(c->ang[0][q], c->ang[1][q], c->ang[2][q], own ? 1 : 0, own ? al : 0.0);
        auto it = ids.find(key);
        if (it == ids.end()) {
            if (ids.size() >= 255) throw FxError{FX_ERR_UNSUPPORTED, "more than 255 distinct Euler-angle / alpha combinations"};
            Variant v{};
            rotation(c->par.use_Euler_angles, c->ang[0][q], c->ang[1][q], c->ang[2][q], v.R);
            v.alpha = al;
            const uint8_t id = (uint8_t)c->variants.size();
            c->variants.push_back(v);
            c->variant_global_alpha.push_back(own ? 0 : 1);
            it = ids.emplace(key, id).first;
        }
        c->var[q] = it->second;
    }
}

// InitializePandRho, Initialization.cpp:83-131 (random draws from the seeded
// splitmix64 stream: the n-th draw is cell 3*idx + component + 1)
void build_P0(fx_ctx* c) {
    const Params& p = c->par;
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    for (int d = 0; d < 3; ++d) c->P0[d].assign(c->N, 0.0);
    const uint64_t seed = (uint64_t)(int64_t)p.random_seed;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t idx = (size_t)i + nx * ((size_t)j + (size_t)ny * k);
                const int m = c->code[idx + c->nxy] & 3;
                double pp = 0, pq = 0, pr = 0;
                if (m == 0) {
                    const double x = p.prob_lo[0] + (i + 0.5) * c->dx[0];
                    const double y = p.prob_lo[1] + (j + 0.5) * c->dx[1];
                    const double z = p.prob_lo[2] + (k + 0.5) * c->dx[2];
                    if (p.prob_type == 1) {
                        const double u = uniform(seed, (uint64_t)i + (uint64_t)k * nz + 1);
                        pp = (-1.0 + 2.0 * u) * p.Remnant_P[0];
                        pq = (-1.0 + 2.0 * u) * p.Remnant_P[1];
                        pr = (-1.0 + 2.0 * u) * p.Remnant_P[2];
                    } else if (p.prob_type == 2) {
                        pp = (-1.0 + 2.0 * uniform(seed, 3 * idx + 1)) * p.Remnant_P[0];
                        pq = (-1.0 + 2.0 * uniform(seed, 3 * idx + 2)) * p.Remnant_P[1];
                        pr = (-1.0 + 2.0 * uniform(seed, 3 * idx + 3)) * p.Remnant_P[2];
                    } else {
                        const double DEz = p.DE_hi[2];
                        const double g = exp(-(x * x / (2.0 * 5.e-9 * 5.e-9) + y * y / (2.0 * 5.e-9 * 5.e-9) +
                                               (z - 1.5 * DEz) * (z - 1.5 * DEz) / (2.0 * 2.0e-9 * 2.0e-9)));
                        pp = p.Remnant_P[0] * g; pq = p.Remnant_P[1] * g; pr = p.Remnant_P[2] * g;
                    }
                    if (c->tphase[idx] == 1.0) pr = 0.0;
                }
                if (p.is_polarization_scalar == 1) { pp = 0.0; pq = 0.0; }
                c->P0[0][idx] = pp; c->P0[1][idx] = pq; c->P0[2][idx] = pr;
            }
    c->scalarP = p.is_polarization_scalar == 1;
}

void fill_devparams(fx_ctx* c) {
    const Params& p = c->par;
    DevParams& d = c->dp;
    d.nx = c->nx; d.ny = c->ny; d.nz = c->nz;
    d.nxy = (long long)c->nxy; d.N = (long long)c->N;
    long long blocks = ((long long)c->N + 255) / 256;
    d.ngrid_red = (int)std::min<long long>(std::max<long long>(blocks, 1), 148 * 8);
    for (int q = 0; q < 3; ++q) { d.dx[q] = c->dx[q]; d.ih2[q] = 1.0 / (c->dx[q] * c->dx[q]); }
    d.dt = p.dt;
    d.alpha = p.alpha; d.beta = p.beta; d.gamma = p.gamma; d.a12 = p.alpha_12; d.a112 = p.alpha_112; d.a123 = p.alpha_123;
    d.BigGamma = p.BigGamma; d.g11 = p.g11; d.g44 = p.g44; d.g44p = p.g44_p; d.g12 = p.g12; d.lambda = p.lambda;
    for (int q = 0; q < 3; ++q) { d.flo[q] = p.P_BC_flag_lo[q]; d.fhi[q] = p.P_BC_flag_hi[q]; }
    d.incl_L = p.include_Landau == 1; d.incl_G = p.include_Grad == 1; d.incl_E = p.include_Elec == 1;
    d.scalar = p.is_polarization_scalar == 1;
    for (int q = 0; q < 8; ++q) d.eps[q] = eps_of_code(p, q);
    d.q = kQ; d.kb = kKb; d.T = kT; d.Nc = kNc; d.Nv = kNv; d.Eg = kEg; d.Chi = kChi; d.Ea = kEa; d.Ed = kEd;
    d.NA = p.acceptor_doping; d.ND = p.donor_doping; d.phi_ref = phi_ref(); d.use_FD = p.use_Fermi_Dirac;
    // the constants of the product form of the Boltzmann charge (Ef = 0,
    // g_A = 4, g_D = 2, ChargeDensity.cpp:46-93)
    const double kbT = kKb * kT;
    d.sc_qkT = kQ / kbT;
    d.sc_Ce = kNc * std::exp(kQ * kChi / kbT);
    d.sc_Ch = kNv * std::exp(-(kQ * kChi + kQ * kEg) / kbT);
    d.sc_Ca = 4.0 * std::exp((kQ * kEa - kQ * kChi - kQ * kEg) / kbT);
    d.sc_Cd = 2.0 * std::exp((kQ * kEd + kQ * kChi) / kbT);
    d.delta = p.delta; d.inv_delta = 1. / p.delta; d.neg_inv_delta = -1. / p.delta;
    d.ghost_mode = p.phi_ghost_mode;
    d.interior = c->use_interior ? c->d_interior : nullptr;
    electrode_values(c);
}

template <typename T>
int dmalloc(fx_ctx* c, T** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return set_err(c, FX_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    // zeroed on the context's stream: nothing may depend on what an earlier
    // allocation left there
    e = c->s ? cudaMemsetAsync(*p, 0, std::max<size_t>(n, 1) * sizeof(T), c->s)
             : cudaMemset(*p, 0, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return set_err(c, FX_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    c->dev_bytes += n * sizeof(T);
    return 0;
}

// InitializePandRho's charge (Initialization.cpp:134-160): intrinsic carrier
// densities n = p = n_i in the semiconductor and rho = q (p - n - N_A + N_D)
int upload_initial_charge(fx_ctx* c) {
    const size_t N = c->N;
    std::vector<double> rho0(N, 0.0), e0(N, 0.0);
    const double ni = std::sqrt(kNc * kNv) * exp(-0.5 * kQ * kEg / (kKb * kT));
    for (size_t q = 0; q < N; ++q)
        if ((c->code[q + c->nxy] & 3) >= 2) {
            e0[q] = ni;
            rho0[q] = kQ * (ni - ni - c->par.acceptor_doping + c->par.donor_doping);
        }
    FX_CUDA(c, cudaMemcpy(c->d_rho, rho0.data(), N * 8, cudaMemcpyHostToDevice));
    FX_CUDA(c, cudaMemcpy(c->d_e, e0.data(), N * 8, cudaMemcpyHostToDevice));
    FX_CUDA(c, cudaMemcpy(c->d_h, e0.data(), N * 8, cudaMemcpyHostToDevice));
    return FX_OK;
}

int ensure_device(fx_ctx* c) {
    if (c->dev) return FX_OK;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_err(c, FX_ERR_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
    if (c->own_stream) FX_CUDA(c, cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking));
    c->mg.prof = &c->prof;
    const size_t N = c->N;
    int r = 0;
    r |= dmalloc(c, &c->d_code, c->code.size());
    for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 3; ++d) r |= dmalloc(c, &c->d_P[b][d], N);
    r |= dmalloc(c, &c->d_phi, N); r |= dmalloc(c, &c->d_phi_old, N); r |= dmalloc(c, &c->d_phi_prev, N);
    r |= dmalloc(c, &c->d_rho, N); r |= dmalloc(c, &c->d_e, N); r |= dmalloc(c, &c->d_h, N);
    r |= dmalloc(c, &c->d_alpha, N); r |= dmalloc(c, &c->d_alpha32, N); r |= dmalloc(c, &c->d_rhs, N);
    r |= dmalloc(c, &c->d_rhsP, N); r |= dmalloc(c, &c->d_dphi, N);
    r |= dmalloc(c, &c->d_part, 4 * 148 * 8 + 64);
    r |= dmalloc(c, &c->d_counter, 4);
    r |= dmalloc(c, &c->d_out, 8);
    if (r) return r;
    FX_CUDA(c, cudaMallocHost(&c->h_out, 8 * sizeof(double)));
    if (!c->var.empty()) {
        r |= dmalloc(c, &c->d_var, N);
        r |= dmalloc(c, &c->d_vt, c->variants.size());
        if (r) return r;
        FX_CUDA(c, cudaMemcpy(c->d_var, c->var.data(), N, cudaMemcpyHostToDevice));
        FX_CUDA(c, cudaMemcpy(c->d_vt, c->variants.data(), c->variants.size() * sizeof(Variant), cudaMemcpyHostToDevice));
    }
    FX_CUDA(c, cudaMemcpy(c->d_code, c->code.data(), c->code.size(), cudaMemcpyHostToDevice));
    {
        // interior cells: the cell and its 18 face and edge neighbours are
        // ferroelectric and 1 <= k <= nz - 2 (every P stencil takes its
        // central form there, and every z index it reads is in range)
        std::vector<uint8_t> in(N, 0);
        const int nx = c->nx, ny = c->ny, nz = c->nz;
        auto fe = [&](int i, int j, int k) {
            i = (i % nx + nx) % nx;
            j = (j % ny + ny) % ny;
            return (c->code[(size_t)i + nx * ((size_t)j + (size_t)ny * (k + 1))] & 3) == 0;
        };
        for (int k = 1; k + 1 < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    bool ok = true;
                    for (int dk = -1; dk <= 1 && ok; ++dk)
                        for (int dj = -1; dj <= 1 && ok; ++dj)
                            for (int di = -1; di <= 1 && ok; ++di)
                                if (std::abs(di) + std::abs(dj) + std::abs(dk) <= 2) ok = fe(i + di, j + dj, k + dk);
                    in[(size_t)i + nx * ((size_t)j + (size_t)ny * k)] = ok ? 1 : 0;
                }
        // the planes of the cells the TDGL update changes (one plane when
        // there are none: the launch then changes nothing)
        c->dp.fe_k0 = nz;
        c->dp.fe_k1 = -1;
        for (int k = 0; k < nz; ++k)
            for (size_t q = 0; q < c->nxy; ++q) {
                const uint8_t m = c->code[q + c->nxy * (size_t)(k + 1)];
                if ((m & 3) == 0 && (m & 4) == 0) {
                    c->dp.fe_k0 = std::min(c->dp.fe_k0, k);
                    c->dp.fe_k1 = std::max(c->dp.fe_k1, k);
                    break;
                }
            }
        if (c->dp.fe_k1 < 0) c->dp.fe_k0 = c->dp.fe_k1 = 0;
        r = dmalloc(c, &c->d_interior, N);
        if (r) return r;
        FX_CUDA(c, cudaMemcpy(c->d_interior, in.data(), N, cudaMemcpyHostToDevice));
        c->dp.interior = c->use_interior ? c->d_interior : nullptr;
    }
    for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 3; ++d) FX_CUDA(c, cudaMemcpy(c->d_P[b][d], c->P0[d].data(), N * 8, cudaMemcpyHostToDevice));
    // main.cpp:157-173 zero fields; InitializePandRho's intrinsic carriers in SC
    r = upload_initial_charge(c);
    if (r) return r;
    for (double* a : {c->d_phi, c->d_phi_old, c->d_phi_prev, c->d_alpha, c->d_rhs, c->d_rhsP, c->d_dphi})
        FX_CUDA(c, cudaMemset(a, 0, N * 8));
    FX_CUDA(c, cudaMemset(c->d_alpha32, 0, N * 4));
    FX_CUDA(c, cudaMemset(c->d_counter, 0, 4));
    const bool mixed = c->par.precision == 1;
    c->mg.verbose = c->par.verbose;
    int st = c->mg.setup(poisson_params(c), c->code, true, mixed);
    if (st == -2) return set_err(c, FX_ERR_OUT_OF_MEMORY, "multigrid allocation failed");
    if (st != 0) return set_err(c, FX_ERR_CUDA, "multigrid setup failed");
    c->dev_bytes += c->mg.bytes();
    c->mg_ready = true;
    c->dev = true;
    FX_CUDA(c, cudaDeviceSynchronize());
    return FX_OK;
}

const double* const* P_in(fx_ctx* c, const double* arr[3]) {
    arr[0] = c->scalarP ? nullptr : c->d_P[c->cur][0];
    arr[1] = c->scalarP ? nullptr : c->d_P[c->cur][1];
    arr[2] = c->d_P[c->cur][2];
    return arr;
}

int k_status(fx_ctx* c, int e) {
    if (e) return set_err(c, FX_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString((cudaError_t)e));
    return FX_OK;
}

int read_out(fx_ctx* c, int n) {
    FX_CUDA(c, cudaMemcpyAsync(c->h_out, c->d_out, n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    return FX_OK;
}

// the FE part of ComputePoissonRHS for P in buffer `buf`
int compute_rhs_p(fx_ctx* c, bool norms, int buf) {
    const double* P[3] = {c->scalarP ? nullptr : c->d_P[buf][0], c->scalarP ? nullptr : c->d_P[buf][1], c->d_P[buf][2]};
    if (norms) FX_CUDA(c, cudaMemsetAsync(c->d_out, 0, 2 * sizeof(double), c->s));
    ++g_launches;
    c->prof.begin(PROF_RHS_P, c->s);
    int e = launch_rhs_p(c->dp, c->d_code, c->d_var, c->d_vt, P, c->d_rhsP, norms ? c->d_out : nullptr, c->s);
    c->prof.end(c->s);
    return k_status(c, e);
}

int mg_solve(fx_ctx* c, const double* rhs, double nb, double nbp) {
    const double target = std::max(c->par.mg_rtol, 1e-16) * std::max(nb, nbp);
    if (!c->par.warm_start) FX_CUDA(c, cudaMemsetAsync(c->d_phi, 0, c->N * 8, c->s));
    MGStats st;
    int r = c->par.precision == 1
                ? c->mg.solve_mixed(poisson_params(c), c->d_code, c->d_phi, rhs, target, c->par.mg_max_iter, c->s, &st)
                : c->mg.solve64(poisson_params(c), c->d_code, c->d_phi, rhs, target, c->par.mg_max_iter, c->s, &st);
    c->mg_last += st.cycles;
    c->mg_total += st.cycles;
    c->mg_resid_last = st.resid;
    c->mg_target_last = target;
    if (r == -3) {
        std::ostringstream o;
        o << "Poisson multigrid did not reach |r| <= " << target << " in " << c->par.mg_max_iter << " cycles (|r| = " << st.resid << ")";
        return set_err(c, std::isfinite(st.resid) ? FX_ERR_NO_CONVERGENCE : FX_ERR_NONFINITE, o.str());
    }
    if (r) return set_err(c, FX_ERR_CUDA, std::string("multigrid: ") + cudaGetErrorString((cudaError_t)r));
    return FX_OK;
}

// ComputePhi_Rho, ElectrostaticSolver.cpp:678-747, for P in buffer `buf`
// the first solve of a time step starts from 2 phi^n - phi^(n-1) (the
// multigrid's initial iterate only: the Newton linearisation point stays
// phi^n); skipped after a voltage change or any other change of the state
int start_guess(fx_ctx* c) {
    const int order = std::min(kMaxExtrap, c->par.phi_extrapolate);
    if (order <= 0 || !c->par.warm_start) return FX_OK;
    for (int q = 0; q < order; ++q)
        if (!c->d_phi_hist[q]) {
            int r = dmalloc(c, &c->d_phi_hist[q], c->N);
            if (r) return r;
            c->hist_n = 0;
        }
    if (!c->hist_valid || c->hist_vlo != c->dp.V_lo || c->hist_vhi != c->dp.V_hi) c->hist_n = 0;
    const int use = std::min(order, c->hist_n);   // steps of history available
    if (use > 0) {
        // the histories kept are those of `order`; shift all of them
        double* h[6];
        for (int m = 0; m < 6; ++m) h[m] = m < order ? c->d_phi_hist[m] : nullptr;
        ++g_launches;
        int r = k_status(c, launch_phi_extrap(c->dp, use, c->d_phi, h, c->s));
        if (r) return r;
    } else {
        FX_CUDA(c, cudaMemcpyAsync(c->d_phi_hist[0], c->d_phi, c->N * 8, cudaMemcpyDeviceToDevice, c->s));
    }
    c->hist_n = std::min(order, c->hist_n + 1);
    c->hist_valid = true;
    c->hist_vlo = c->dp.V_lo;
    c->hist_vhi = c->dp.V_hi;
    return FX_OK;
}

int compute_phi_rho_P(fx_ctx* c, int buf, bool step_start) {
    int r = ensure_device(c);
    if (r) return r;
    c->E_valid = false;
    c->mg_last = 0;
    if (!c->contains_sc) {
        r = compute_rhs_p(c, true, buf);
        if (r) return r;
        r = read_out(c, 2);
        if (r) return r;
        const double nb = c->h_out[0], nbp = c->h_out[1];
        c->mg.set_alpha(nullptr, nullptr, false, c->s);
        if (step_start && (r = start_guess(c))) return r;
        r = mg_solve(c, c->d_rhsP, nb, nbp);
        if (r) return r;
        c->rhs_is_newton = false;
        c->newton_last = 1;
        c->newton_total += 1;
        c->phi_err_last = 0.0;
        return FX_OK;
    }
    r = compute_rhs_p(c, false, buf);
    if (r) return r;
    const double tol = c->par.newton_tol;   // 1e-5 in the reference
    double err = 1.0;
    int iter = 0, passes = 0;
    while (err > tol) {
        if (passes >= c->par.newton_max_iter) {
            std::ostringstream o;
            o << "Phi-rho Newton iteration did not reach " << tol << " in " << passes << " passes (err = " << err << ")";
            return set_err(c, std::isfinite(err) ? FX_ERR_NO_CONVERGENCE : FX_ERR_NONFINITE, o.str());
        }
        ++passes;
        FX_CUDA(c, cudaMemsetAsync(c->d_out, 0, 2 * sizeof(double), c->s));
        ++g_launches;
        c->prof.begin(PROF_NEWTON, c->s);
        r = k_status(c, launch_newton(c->dp, c->d_code, c->d_phi, c->d_rho, c->d_rhsP, c->d_alpha, c->d_alpha32,
                                      c->d_rhs, c->d_out, c->s));
        c->prof.end(c->s);
        if (r) return r;
        r = read_out(c, 2);
        if (r) return r;
        const double nb = c->h_out[0], nbp = c->h_out[1];
        c->mg.set_alpha(c->d_alpha, c->d_alpha32, true, c->s);
        if (step_start && passes == 1 && (r = start_guess(c))) return r;
        r = mg_solve(c, c->d_rhs, nb, nbp);
        if (r) return r;
        ++g_launches;
        c->prof.begin(PROF_RHO, c->s);
        r = k_status(c, launch_rho(c->dp, c->d_code, c->d_phi, c->d_phi_prev, c->d_rho, c->d_e, c->d_h, c->d_part,
                                   c->d_counter, c->d_out, 1, 0, c->s));
        c->carriers_stale = true;
        c->prof.end(c->s);
        if (r) return r;
        r = read_out(c, 2);
        if (r) return r;
        if (iter > 0) err = c->h_out[0] / c->h_out[1];
        if (!std::isfinite(err)) {
            std::ostringstream o;
            o << "Phi-rho Newton iteration: the change of phi is not finite after " << passes << " passes";
            return set_err(c, FX_ERR_NONFINITE, o.str());
        }
        iter = iter + 1;
        if (c->par.verbose) printf("%d iterations :: err = %g\n", iter, err);
    }
    c->rhs_is_newton = true;
    c->newton_last = passes;
    c->newton_total += passes;
    c->phi_err_last = err;
    return FX_OK;
}

int compute_phi_rho(fx_ctx* c) { return compute_phi_rho_P(c, c->cur, false); }

// main.cpp:280-348: Order 1 is one fused Euler pass; Order 2 is a predictor
// pass (f^n kept, P* into the other buffer), ComputePhi_Rho at P*, and a
// corrector pass P^{n+1} = P^n + dt (0.5 f^n + 0.5 f*) written over P^n
// one Order-1 Euler update of P with a given phi (the segment recompute of
// the gradient, from the recorded phi of that step)
int tdgl_euler_with_phi(fx_ctx* c, const double* phi) {
    const double* Pin[3];
    P_in(c, Pin);
    const int nb = 1 - c->cur;
    double* Pout[3] = {c->scalarP ? nullptr : c->d_P[nb][0], c->scalarP ? nullptr : c->d_P[nb][1], c->d_P[nb][2]};
    ++g_launches;
    int r = k_status(c, launch_tdgl(c->dp, c->par.precision == 1, 0, c->d_code, c->d_var, c->d_vt, Pin, Pout, phi,
                                    nullptr, nullptr, c->s));
    if (r) return r;
    c->cur = nb;
    return FX_OK;
}

int tdgl_update(fx_ctx* c) {
    int r = ensure_device(c);
    if (r) return r;
    const double* Pin[3];
    P_in(c, Pin);
    const int nb = 1 - c->cur;
    double* Pout[3] = {c->scalarP ? nullptr : c->d_P[nb][0], c->scalarP ? nullptr : c->d_P[nb][1], c->d_P[nb][2]};
    const int mixed = c->par.precision == 1;
    if (c->par.TimeIntegratorOrder == 1) {
        ++g_launches;
        c->prof.begin(PROF_TDGL, c->s);
        r = k_status(c, launch_tdgl(c->dp, mixed, 0, c->d_code, c->d_var, c->d_vt, Pin, Pout, c->d_phi, nullptr, nullptr, c->s));
        c->prof.end(c->s);
        if (r) return r;
        c->cur = nb;
        return FX_OK;
    }
    for (int d = 0; d < 3; ++d)
        if (!c->d_f[d]) { r = dmalloc(c, &c->d_f[d], c->N); if (r) return r; }
    double* fb[3] = {c->d_f[0], c->d_f[1], c->d_f[2]};
    ++g_launches;
    c->prof.begin(PROF_TDGL, c->s);
    r = k_status(c, launch_tdgl(c->dp, mixed, 1, c->d_code, c->d_var, c->d_vt, Pin, Pout, c->d_phi, fb, nullptr, c->s));
    c->prof.end(c->s);
    if (r) return r;
    r = compute_phi_rho_P(c, nb, false);
    if (r) return r;
    const double* Ppre[3] = {Pout[0], Pout[1], Pout[2]};
    double* Pnew[3] = {c->scalarP ? nullptr : c->d_P[c->cur][0], c->scalarP ? nullptr : c->d_P[c->cur][1], c->d_P[c->cur][2]};
    const double* Pold[3] = {Pnew[0], Pnew[1], Pnew[2]};
    ++g_launches;
    c->prof.begin(PROF_TDGL, c->s);
    r = k_status(c, launch_tdgl(c->dp, mixed, 2, c->d_code, c->d_var, c->d_vt, Ppre, Pnew, c->d_phi, fb, Pold, c->s));
    c->prof.end(c->s);
    return r;
}

void steady_update(fx_ctx* c, int step, double phi_max, double dmax);

int check_steady(fx_ctx* c, int step) {
    int r = ensure_device(c);
    if (r) return r;
    FX_CUDA(c, cudaMemsetAsync(c->d_out, 0, 2 * sizeof(double), c->s));
    ++g_launches;
    c->prof.begin(PROF_STEADY, c->s);
    r = k_status(c, launch_steady(c->dp, c->d_phi, c->d_phi_old, c->d_dphi, c->d_out, c->s));
    c->prof.end(c->s);
    if (r) return r;
    r = read_out(c, 2);
    if (r) return r;
    steady_update(c, step, c->h_out[0], c->h_out[1]);
    return FX_OK;
}

// the host side of CheckSteadyState from max|phi| and max|phi - phi_old|
void steady_update(fx_ctx* c, int step, double phi_max, double dmax) {
    double max_phi_err;
    if (phi_max > 0) max_phi_err = dmax / phi_max;
    else max_phi_err = dmax > 0 ? INFINITY : 0.0;   // all-NaN Phidiff passes norm0 as 0
    c->phi_max_last = phi_max;
    if (step > 1 && max_phi_err < c->par.phi_tolerance) {
        c->steady_state_step = step;
        c->inc_step = step;
    }
    c->steady_err_last = max_phi_err;
    if (c->par.verbose) printf("Steady state check : (phi(t) - phi(t-1)).norm0() = %g\n", max_phi_err);
}

// ---- one step as one CUDA graph (fx_ctl.h)
//
// The graph holds what step_once's host path runs before its voltage
// bookkeeping -- ComputePhi_Rho with the extrapolated start, the TDGL update,
// CheckSteadyState -- with the same kernels in the same order, so the results
// are bit-identical; the Newton and multigrid loop tests run on the device.
// A failure in ComputePhi_Rho closes the gates (IF nodes) in front of the
// TDGL update and the steady-state check, as the host path returns there.

int sg_hist_before(fx_ctx* c, int* use) {
    *use = 0;
    const int order = std::min(kMaxExtrap, c->par.phi_extrapolate);
    if (order <= 0 || !c->par.warm_start) return FX_OK;
    for (int q = 0; q < order; ++q)
        if (!c->d_phi_hist[q]) {
            int r = dmalloc(c, &c->d_phi_hist[q], c->N);
            if (r) return r;
            c->hist_n = 0;
        }
    if (!c->hist_valid || c->hist_vlo != c->dp.V_lo || c->hist_vhi != c->dp.V_hi) c->hist_n = 0;
    *use = std::min(order, c->hist_n);
    return FX_OK;
}

void sg_hist_after(fx_ctx* c) {
    const int order = std::min(kMaxExtrap, c->par.phi_extrapolate);
    if (order <= 0 || !c->par.warm_start) return;
    c->hist_n = std::min(order, c->hist_n + 1);
    c->hist_valid = true;
    c->hist_vlo = c->dp.V_lo;
    c->hist_vhi = c->dp.V_hi;
}

// start_guess's launches for `use` steps of history (bookkeeping on the host)
void sg_start_guess(fx_ctx* c, cudaStream_t q, int use) {
    const int order = std::min(kMaxExtrap, c->par.phi_extrapolate);
    if (order <= 0 || !c->par.warm_start) return;
    if (use > 0) {
        double* h[6];
        for (int m = 0; m < 6; ++m) h[m] = m < order ? c->d_phi_hist[m] : nullptr;
        ++g_launches;
        launch_phi_extrap(c->dp, use, c->d_phi, h, q);
    } else {
        cudaMemcpyAsync(c->d_phi_hist[0], c->d_phi, c->N * 8, cudaMemcpyDeviceToDevice, q);
    }
}

// mg_solve with the target formed on the device from the norms in d_out
void sg_mg_solve(fx_ctx* c, cudaStream_t q, const double* rhs, bool end_in_next) {
    if (!c->par.warm_start) cudaMemsetAsync(c->d_phi, 0, c->N * 8, q);
    if (c->par.precision == 1)
        c->mg.enqueue_solve_mixed_ctl(poisson_params(c), c->d_code, c->d_phi, rhs, c->d_out, c->par.mg_rtol, c->par.mg_max_iter,
                                      c->d_ctl, c->cap, q, end_in_next);
    else
        c->mg.enqueue_solve64_ctl(poisson_params(c), c->d_code, c->d_phi, rhs, c->d_out, c->par.mg_rtol, c->par.mg_max_iter,
                                  c->d_ctl, c->cap, q, end_in_next);
}

// one pass of the ComputePhi_Rho loop (compute_phi_rho_P's loop body); the
// charge kernel's last block closes the solve and runs the loop test, and
// leaves the norm accumulators of the next pass's linearisation zeroed
void sg_newton_pass(fx_ctx* c, cudaStream_t q, bool start, int use, cudaGraphConditionalHandle hn, int in_body) {
    ++g_launches;
    launch_newton(c->dp, c->d_code, c->d_phi, c->d_rho, c->d_rhsP, c->d_alpha, c->d_alpha32, c->d_rhs, c->d_out, q);
    c->mg.set_alpha(c->d_alpha, c->d_alpha32, true, q);
    if (start) sg_start_guess(c, q, use);
    sg_mg_solve(c, q, c->d_rhs, true);
    const RhoCtl rc = {c->d_ctl, c->par.newton_tol, c->par.newton_max_iter, in_body, 1, hn};
    ++g_launches;
    launch_rho(c->dp, c->d_code, c->d_phi, c->d_phi_prev, c->d_rho, c->d_e, c->d_h, c->d_part, c->d_counter, c->d_out,
               1, 0, q, &rc);
}

// ComputePhi_Rho for P in buffer `buf` on stream q; its last kernel opens the
// IF node `gate` (of body kind `kind`) while no failure is recorded.  The
// step's first ComputePhi_Rho is begun by the step's first kernel.
void sg_phirho(fx_ctx* c, cudaStream_t q, int buf, bool step_start, int use, cudaGraphConditionalHandle gate, int kind) {
    if (!step_start) {
        ++g_launches;
        launch_ctl_phirho_begin(c->d_ctl, c->d_out, q);
    }
    const double* P[3] = {c->scalarP ? nullptr : c->d_P[buf][0], c->scalarP ? nullptr : c->d_P[buf][1], c->d_P[buf][2]};
    if (!c->contains_sc) {
        // (out[] zeroed by the step's or this ComputePhi_Rho's first kernel)
        ++g_launches;
        launch_rhs_p(c->dp, c->d_code, c->d_var, c->d_vt, P, c->d_rhsP, c->d_out, q);
        c->mg.set_alpha(nullptr, nullptr, false, q);
        if (step_start) sg_start_guess(c, q, use);
        sg_mg_solve(c, q, c->d_rhsP, false);
    } else {
        ++g_launches;
        launch_rhs_p(c->dp, c->d_code, c->d_var, c->d_vt, P, c->d_rhsP, nullptr, q);
        const cudaGraphConditionalHandle hn = c->cap.handle(q);
        sg_newton_pass(c, q, step_start, use, hn, 0);
        c->cap.node(q, cudaGraphCondTypeWhile, hn, KIND_NEWTON_PASS,
                    [&](cudaStream_t b) { sg_newton_pass(c, b, false, 0, hn, 1); });
    }
    ++g_launches;
    launch_ctl_phirho_end(c->d_ctl, c->contains_sc ? 1 : 0, gate, kind, q);
}

// ComputePhi_Rho, then `body` inside an IF node that runs only while no
// failure is recorded
template <typename F>
void sg_phirho_gated(fx_ctx* c, cudaStream_t q, int buf, bool step_start, int use, int kind, F&& body) {
    const cudaGraphConditionalHandle h = c->cap.handle(q);
    sg_phirho(c, q, buf, step_start, use, h, kind);
    c->cap.node(q, cudaGraphCondTypeIf, h, kind, body);
}

// CheckSteadyState's norms into the control block (zeroed by the step's first
// kernel); skipped after a failure
void sg_steady(fx_ctx* c, cudaStream_t q) {
    ++g_launches;
    launch_steady(c->dp, c->d_phi, c->d_phi_old, c->d_dphi, c->d_ctl->steady, q, &c->d_ctl->status);
}

void sg_enqueue_step(fx_ctx* c, int use) {
    cudaStream_t s = c->s;
    const int cur = c->cur, nb = 1 - cur;
    const int mixed = c->par.precision == 1;
    ++g_launches;
    launch_ctl_step_begin(c->d_ctl, c->d_out, s);
    const double* Pin[3] = {c->scalarP ? nullptr : c->d_P[cur][0], c->scalarP ? nullptr : c->d_P[cur][1], c->d_P[cur][2]};
    double* Pout[3] = {c->scalarP ? nullptr : c->d_P[nb][0], c->scalarP ? nullptr : c->d_P[nb][1], c->d_P[nb][2]};
    if (c->par.TimeIntegratorOrder == 1) {
        // the update and the check return at once after a failure (a flag
        // test costs less than an IF node)
        sg_phirho(c, s, cur, true, use, 0, 0);
        ++g_launches;
        launch_tdgl(c->dp, mixed, 0, c->d_code, c->d_var, c->d_vt, Pin, Pout, c->d_phi, nullptr, nullptr, s,
                    &c->d_ctl->status);
        sg_steady(c, s);
    } else {
        double* fb[3] = {c->d_f[0], c->d_f[1], c->d_f[2]};
        sg_phirho_gated(c, s, cur, true, use, KIND_GATE_TDGL, [&](cudaStream_t q) {
            ++g_launches;
            launch_tdgl(c->dp, mixed, 1, c->d_code, c->d_var, c->d_vt, Pin, Pout, c->d_phi, fb, nullptr, q);
            sg_phirho_gated(c, q, nb, false, 0, KIND_GATE_CORRECTOR, [&](cudaStream_t b) {
                const double* Ppre[3] = {Pout[0], Pout[1], Pout[2]};
                double* Pnew[3] = {c->scalarP ? nullptr : c->d_P[cur][0], c->scalarP ? nullptr : c->d_P[cur][1], c->d_P[cur][2]};
                const double* Pold[3] = {Pnew[0], Pnew[1], Pnew[2]};
                ++g_launches;
                launch_tdgl(c->dp, mixed, 2, c->d_code, c->d_var, c->d_vt, Ppre, Pnew, c->d_phi, fb, Pold, b);
                sg_steady(c, b);
            });
        });
    }
    cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s);
}

// the captured launch parameters and graph shape of a step
std::vector<unsigned char> sg_key(const fx_ctx* c, int use) {
    std::vector<unsigned char> k;
    auto put = [&](const void* v, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(v);
        k.insert(k.end(), b, b + n);
    };
    put(&c->dp, sizeof(DevParams));
    const int iv[] = {c->cur, use, c->par.TimeIntegratorOrder, c->par.precision, c->par.warm_start,
                      c->par.phi_extrapolate, c->par.newton_max_iter, c->par.mg_max_iter, c->mg.nu1, c->mg.nu2,
                      c->mg.mixed_cycles, c->scalarP ? 1 : 0, c->contains_sc ? 1 : 0, g_pdl ? 1 : 0, g_rhs_seg ? 1 : 0,
                      c->mg.alpha_tiles ? 1 : 0, c->mg.nu1c, c->mg.nu2c, c->mg.seg_bytes, c->mg.dense_coarse ? 1 : 0, c->mg.split_mode ? 1 : 0,
                      (int)std::min<long long>(c->mg.seg_min_cells, 2147483647LL)};
    put(iv, sizeof(iv));
    const double dv[] = {c->par.mg_rtol, c->par.newton_tol};
    put(dv, sizeof(dv));
    const void* pv[] = {c->s, c->d_var, c->d_vt, c->d_f[0], c->d_f[1], c->d_f[2], c->d_phi_hist[0], c->d_phi_hist[1],
                        c->d_phi_hist[2], c->d_phi_hist[3], c->d_phi_hist[4], c->d_phi_hist[5]};
    put(pv, sizeof(pv));
    return k;
}

int sg_build(fx_ctx* c, int use, fx_ctx::StepGraph& g) {
    c->cap.reset();
    const long long l0 = g_launches.load();
    cudaError_t e = cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal);
    if (e) return (int)e;
    sg_enqueue_step(c, use);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(c->s, &graph);
    const long long total = g_launches.load() - l0;
    g_launches -= total;   // counted per execution
    if (!e) e = c->cap.err;
    if (!e) e = cudaGetLastError();
    if (!e) e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e) {
        if (g.exec) { cudaGraphExecDestroy(g.exec); g.exec = nullptr; }
        return (int)e;
    }
    g.top = total - c->cap.in_bodies;
    for (int q = 0; q < KIND_N; ++q) g.own[q] = c->cap.own[q];
    return 0;
}

// Runs ComputePhi_Rho, the TDGL update and CheckSteadyState of one step as a
// graph.  *ran = false leaves the step to the host-driven path (profiling on,
// the graph path switched off, or no capture possible on this setup).
int step_graph(fx_ctx* c, int step, bool* ran) {
    *ran = false;
    c->sg_ran = false;
    if (!c->par.step_graph || c->sg_off || c->prof.on || c->par.newton_max_iter < 1) return FX_OK;
    int r = ensure_device(c);
    if (r) return r;
    if (!c->d_ctl) {
        r = dmalloc(c, &c->d_ctl, 1);
        if (r) return r;
        FX_CUDA(c, cudaMallocHost(&c->h_ctl, sizeof(StepCtl)));
        FX_CUDA(c, c->cap.init());
    }
    if (c->par.TimeIntegratorOrder != 1)
        for (int d = 0; d < 3; ++d)
            if (!c->d_f[d]) { r = dmalloc(c, &c->d_f[d], c->N); if (r) return r; }
    int use = 0;
    r = sg_hist_before(c, &use);
    if (r) return r;
    std::vector<unsigned char> key = sg_key(c, use);
    fx_ctx::StepGraph* g = nullptr;
    for (auto& x : c->sgraphs)
        if (x.key == key) { g = &x; break; }
    if (!g) {
        // a changed parameter makes every cached step stale
        bool same_params = true;
        if (!c->sgraphs.empty()) {
            const size_t n = sizeof(DevParams);
            same_params = std::memcmp(c->sgraphs[0].key.data(), key.data(), n) == 0 &&
                          std::memcmp(c->sgraphs[0].key.data() + n + 2 * sizeof(int), key.data() + n + 2 * sizeof(int),
                                      key.size() - n - 2 * sizeof(int)) == 0;
        }
        if (!same_params || c->sgraphs.size() >= 8) {
            for (auto& x : c->sgraphs) if (x.exec) cudaGraphExecDestroy(x.exec);
            c->sgraphs.clear();
        }
        fx_ctx::StepGraph ng;
        ng.key = key;
        const int e = sg_build(c, use, ng);
        if (e) {
            // stream capture of conditional nodes is not available here:
            // the host-driven loop runs this and every later step
            cudaGetLastError();
            c->sg_off = true;
            return FX_OK;
        }
        c->sgraphs.push_back(ng);
        g = &c->sgraphs.back();
    }
    FX_CUDA(c, cudaGraphLaunch(g->exec, c->s));
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    *ran = true;
    c->sg_ran = true;
    const StepCtl& t = *c->h_ctl;
    long long launches = g->top;
    for (int q = 0; q < KIND_N; ++q) launches += g->own[q] * t.nexec[q];
    g_launches += launches;
    c->E_valid = false;
    c->mg_last = t.mg_cycles_phirho;
    c->mg_total += t.mg_cycles_step;
    c->mg_resid_last = t.mg_resid_last;
    c->mg_target_last = t.mg_target_last;
    c->newton_last = t.passes;
    c->newton_total += t.newton_passes_step;
    c->phi_err_last = t.err;
    c->rhs_is_newton = c->contains_sc;
    if (c->contains_sc) c->carriers_stale = true;
    if (t.status != CTL_OK) {
        c->hist_valid = false;
        std::ostringstream o;
        if (t.status == CTL_MG_NO_CONV || t.status == CTL_MG_NONFINITE) {
            o << "Poisson multigrid did not reach |r| <= " << t.status_target << " in " << c->par.mg_max_iter
              << " cycles (|r| = " << t.status_val << ")";
            return set_err(c, t.status == CTL_MG_NO_CONV ? FX_ERR_NO_CONVERGENCE : FX_ERR_NONFINITE, o.str());
        }
        o << "Phi-rho Newton iteration did not reach " << c->par.newton_tol << " in " << t.status_n
          << " passes (err = " << t.status_val << ")";
        return set_err(c, t.status == CTL_NEWTON_NO_CONV ? FX_ERR_NO_CONVERGENCE : FX_ERR_NONFINITE, o.str());
    }
    sg_hist_after(c);
    if (c->par.TimeIntegratorOrder == 1) c->cur = 1 - c->cur;
    steady_update(c, step, t.steady[0], t.steady[1]);
    return FX_OK;
}

// one pass of main.cpp:261-621; returns 1 when the loop breaks
int step_once_impl(fx_ctx* c) {
    const int step = c->step + 1;
    bool ran = false;
    int r = step_graph(c, step, &ran);
    if (r) return r;
    if (!ran) {
        r = compute_phi_rho_P(c, c->cur, true);
        if (r) return r;
        r = tdgl_update(c);
        if (r) return r;
        r = check_steady(c, step);
        if (r) return r;
    }
    c->E_valid = false;
    c->time = c->time + c->par.dt;
    c->step = step;
    const Params& p = c->par;
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
        if (c->par.verbose)
            printf("step = %d, Phi_Bc_hi = %g, num_Vapp = %d, sign = %d\n", step, c->Phi_Bc_hi, c->num_Vapp, c->sign);
        electrode_values(c);
        r = compute_phi_rho(c);
        if (r) return r;
    }
    bool brk = false;
    if (p.voltage_sweep == 0 && step == c->steady_state_step) brk = true;
    if (p.voltage_sweep == 1 && c->Phi_Bc_hi > 0. && c->Phi_Bc_hi - p.Phi_Bc_hi_max > tiny) brk = true;
    if (p.voltage_sweep == 1 && c->Phi_Bc_hi < 0. && -c->Phi_Bc_hi - p.Phi_Bc_hi_max > tiny) brk = true;
    if (p.voltage_sweep == 1 && c->num_Vapp == p.num_Vapp_max) brk = true;
    if (brk) c->finished = true;
    c->prof.collect();
    return brk ? 1 : 0;
}

// A step whose solve failed (a non-finite residual, or no convergence within
// the caps) has left P as it was (the TDGL update and the steady-state check
// did not run); phi and the charge density go back to their values at the
// end of the last completed step, so the caller can change the input and
// step again.  phi_old holds that phi: CheckSteadyState copies phi into it at
// the end of every step (before the first step both are zero).
int restore_after_failure(fx_ctx* c) {
    if (!c->dev) return FX_OK;
    FX_CUDA(c, cudaMemcpyAsync(c->d_phi, c->d_phi_old, c->N * 8, cudaMemcpyDeviceToDevice, c->s));
    if (c->contains_sc) {
        if (c->step == 0) {
            FX_CUDA(c, cudaStreamSynchronize(c->s));
            int r = upload_initial_charge(c);
            if (r) return r;
            c->carriers_stale = false;
        } else {
            ++g_launches;
            int r = k_status(c, launch_rho(c->dp, c->d_code, c->d_phi, c->d_phi_prev, c->d_rho, c->d_e, c->d_h,
                                           c->d_part, c->d_counter, c->d_out, 0, 0, c->s));
            if (r) return r;
            c->carriers_stale = true;
        }
    }
    c->E_valid = false;
    c->hist_valid = false;
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    return FX_OK;
}

int step_once(fx_ctx* c) {
    const int r = step_once_impl(c);
    if (r == FX_ERR_NONFINITE || r == FX_ERR_NO_CONVERGENCE) {
        const std::string msg = c->err;
        const int q = restore_after_failure(c);
        if (q) return q;
        c->err = msg;
    }
    return r;
}

int materialize_E(fx_ctx* c) {
    int r = ensure_device(c);
    if (r) return r;
    if (c->E_valid) return FX_OK;
    for (int d = 0; d < 3; ++d)
        if (!c->d_E[d]) { r = dmalloc(c, &c->d_E[d], c->N); if (r) return r; }
    ++g_launches;
    c->prof.begin(PROF_EFIELD, c->s);
    r = k_status(c, launch_efield(c->dp, c->d_var, c->d_vt, c->d_phi, c->d_E, c->s));
    c->prof.end(c->s);
    if (r) return r;
    c->E_valid = true;
    return FX_OK;
}

int host_field(fx_ctx* c, int f, std::vector<double>& out) {
    const size_t N = c->N;
    switch (f) {
    case FX_FIELD_EPSILON: case FX_FIELD_MASK: case FX_FIELD_GAMMA: out.assign(N, 0.0); break;
    case FX_FIELD_TPHASE: case FX_FIELD_ANGLE_ALPHA: case FX_FIELD_ANGLE_BETA: case FX_FIELD_ANGLE_THETA: break;
    default: return 0;   // a device field: nothing allocated here
    }
    switch (f) {
    case FX_FIELD_EPSILON:
        for (size_t q = 0; q < N; ++q) out[q] = eps_of_code(c->par, c->code[q + c->nxy]);
        return 1;
    case FX_FIELD_MASK:
        for (size_t q = 0; q < N; ++q) out[q] = (double)(c->code[q + c->nxy] & 3);
        return 1;
    case FX_FIELD_TPHASE: out = c->tphase; return 1;
    case FX_FIELD_ANGLE_ALPHA: out = c->ang[0]; return 1;
    case FX_FIELD_ANGLE_BETA: out = c->ang[1]; return 1;
    case FX_FIELD_ANGLE_THETA: out = c->ang[2]; return 1;
    case FX_FIELD_GAMMA:
        for (size_t q = 0; q < N; ++q) out[q] = (c->code[q + c->nxy] & 3) == 0 ? c->par.BigGamma : 0.0;
        return 1;
    }
    return 0;
}

// the carrier densities at the phi of the last charge evaluation (phi has not
// changed since: the Newton loop ends with it, and fx_set_field forms them
// before replacing phi)
int carriers_now(fx_ctx* c) {
    if (!c->carriers_stale) return FX_OK;
    ++g_launches;
    int r = k_status(c, launch_rho(c->dp, c->d_code, c->d_phi, c->d_phi_prev, c->d_rho, c->d_e, c->d_h, c->d_part,
                                   c->d_counter, c->d_out, 0, 1, c->s));
    if (r) return r;
    c->carriers_stale = false;
    return FX_OK;
}

int get_field(fx_ctx* c, int f, double* out) {
    std::vector<double> h;
    if (host_field(c, f, h)) {
        std::memcpy(out, h.data(), c->N * 8);
        return FX_OK;
    }
    if (!c->dev && (f == FX_FIELD_PX || f == FX_FIELD_PY || f == FX_FIELD_PZ)) {
        std::memcpy(out, c->P0[f].data(), c->N * 8);
        return FX_OK;
    }
    int r = ensure_device(c);
    if (r) return r;
    const double* src = nullptr;
    switch (f) {
    case FX_FIELD_PX: case FX_FIELD_PY: case FX_FIELD_PZ: src = c->d_P[c->cur][f]; break;
    case FX_FIELD_PHI: src = c->d_phi; break;
    case FX_FIELD_POISSON_RHS: src = c->rhs_is_newton ? c->d_rhs : c->d_rhsP; break;
    case FX_FIELD_EX: case FX_FIELD_EY: case FX_FIELD_EZ:
        r = materialize_E(c);
        if (r) return r;
        src = c->d_E[f - FX_FIELD_EX];
        break;
    case FX_FIELD_HOLES: { int r = carriers_now(c); if (r) return r; src = c->d_h; break; }
    case FX_FIELD_ELECTRONS: { int r = carriers_now(c); if (r) return r; src = c->d_e; break; }
    case FX_FIELD_CHARGE: src = c->d_rho; break;
    case FX_FIELD_PHIDIFF: src = c->d_dphi; break;
    case FX_FIELD_ALPHA_CC: src = c->d_alpha; break;
    default: return set_err(c, FX_ERR_INVALID_ARGUMENT, "unknown field id");
    }
    FX_CUDA(c, cudaMemcpyAsync(out, src, c->N * 8, cudaMemcpyDeviceToHost, c->s));
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    if (f == FX_FIELD_PHIDIFF) {
        // Phidiff = |phi - phi_old| / max|phi| (ElectrostaticSolver.cpp:542)
        const double m = c->phi_max_last;
        for (size_t q = 0; q < c->N; ++q) out[q] = out[q] / m;
    }
    return FX_OK;
}

// ---- gradient record: checkpoints, segment recompute, reverse sweep ----

void adj_free(fx_ctx* c) {
    auto& A = c->adj;
    if (!A.allocs.empty() && c->s) cudaStreamSynchronize(c->s);
    for (void* q : A.allocs) cudaFree(q);
    A = fx_ctx::AdjRecord();
}

template <typename T>
int adj_alloc(fx_ctx* c, T** q, size_t n) {
    cudaError_t e = cudaMalloc((void**)q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        *q = nullptr;
        return set_err(c, FX_ERR_OUT_OF_MEMORY, std::string("gradient record: cudaMalloc: ") + cudaGetErrorString(e));
    }
    c->adj.allocs.push_back(*q);
    c->adj.bytes += n * sizeof(T);
    return FX_OK;
}

// the P components the kernels read (z only with scalar polarization)
int ncomp_first(const fx_ctx* c) { return c->scalarP ? 2 : 0; }

int dcopy(fx_ctx* c, double* dst, const double* src) {
    FX_CUDA(c, cudaMemcpyAsync(dst, src, c->N * 8, cudaMemcpyDeviceToDevice, c->s));
    return FX_OK;
}

// save / restore the step state: P, phi (the solve's warm start) and, with a
// semiconductor, rho (the Newton loop's first right-hand side)
int adj_save(fx_ctx* c, double* const P[3], double* phi, double* rho) {
    int r = 0;
    for (int d = ncomp_first(c); d < 3 && !r; ++d) r = dcopy(c, P[d], c->d_P[c->cur][d]);
    if (!r) r = dcopy(c, phi, c->d_phi);
    if (!r && rho) r = dcopy(c, rho, c->d_rho);
    return r;
}

int adj_restore(fx_ctx* c, double* const P[3], const double* phi, const double* rho) {
    int r = 0;
    for (int d = ncomp_first(c); d < 3 && !r; ++d) r = dcopy(c, c->d_P[c->cur][d], P[d]);
    if (!r) r = dcopy(c, c->d_phi, phi);
    if (!r && rho) r = dcopy(c, c->d_rho, rho);
    c->E_valid = false;
    return r;
}

// one step of the recorded loop: electrode value, ComputePhi_Rho, TDGL update
int adj_step(fx_ctx* c, double V) {
    c->Phi_Bc_hi = V;
    electrode_values(c);
    int r = compute_phi_rho(c);
    if (r) return r;
    r = tdgl_update(c);
    c->E_valid = false;
    c->prof.collect();
    return r;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int forward_record(fx_ctx* c, const fx_loss_spec* sp, double* loss) {
    const auto t0 = std::chrono::steady_clock::now();
    const int T = sp->nsteps, k = sp->checkpoint_every;
    int r = ensure_device(c);
    if (r) return r;
    adj_free(c);
    auto& A = c->adj;
    A.T = T;
    A.k = k;
    A.nck = (T + k - 1) / k;
    A.V.resize(T);
    A.shape.assign(T, 1.0);
    if (sp->v_shape) A.shape.assign(sp->v_shape, sp->v_shape + T);
    A.target.assign(sp->target, sp->target + T);
    for (int n = 0; n < T; ++n) A.V[n] = sp->v_amp * A.shape[n];
    A.nfe = 0;
    for (size_t q = 0; q < c->N; ++q) A.nfe += (c->code[q + c->nxy] & 3) == 0;
    if (A.nfe == 0) return set_err(c, FX_ERR_INVALID_ARGUMENT, "the loss needs ferroelectric cells");
    const bool sc = c->contains_sc;
    A.ckP.assign(3 * A.nck, nullptr);
    A.ckPhi.assign(A.nck, nullptr);
    A.ckRho.assign(A.nck, nullptr);
    for (int q = 0; q < A.nck; ++q) {
        for (int d = ncomp_first(c); d < 3; ++d) if ((r = adj_alloc(c, &A.ckP[3 * q + d], c->N))) return r;
        if ((r = adj_alloc(c, &A.ckPhi[q], c->N))) return r;
        if (sc && (r = adj_alloc(c, &A.ckRho[q], c->N))) return r;
    }
    for (int d = ncomp_first(c); d < 3; ++d) if ((r = adj_alloc(c, &A.finP[d], c->N))) return r;
    if ((r = adj_alloc(c, &A.finPhi, c->N))) return r;
    if (sc && (r = adj_alloc(c, &A.finRho, c->N))) return r;
    if ((r = adj_alloc(c, &A.hist, 3 * (size_t)T))) return r;
    // phi of every step, when it fits in three quarters of the free device
    // memory: the backward's segment recompute is then the TDGL updates
    // alone, with no Poisson or Newton solve (else it repeats the solves)
    if (c->adj_store_phi) {
        const size_t need = (size_t)T * c->N;
        if (c->adj_phi_store && c->adj_phi_store_n < need) {
            cudaStreamSynchronize(c->s);
            cudaFree(c->adj_phi_store);
            c->adj_phi_store = nullptr;
            c->adj_phi_store_n = 0;
        }
        if (!c->adj_phi_store) {
            size_t freeb = 0, totalb = 0;
            if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess && need * sizeof(double) <= freeb / 4 * 3 &&
                cudaMalloc(&c->adj_phi_store, need * sizeof(double)) == cudaSuccess)
                c->adj_phi_store_n = need;
            else
                c->adj_phi_store = nullptr;
            cudaGetLastError();
        }
        A.phiAll = c->adj_phi_store;
        if (A.phiAll) A.bytes += need * sizeof(double);
    }

    if ((r = adj_save(c, &A.ckP[0], A.ckPhi[0], A.ckRho[0]))) return r;
    for (int n = 1; n <= T; ++n) {
        if ((r = adj_step(c, A.V[n - 1]))) return r;
        if (A.phiAll)
            FX_CUDA(c, cudaMemcpyAsync(A.phiAll + (size_t)(n - 1) * c->N, c->d_phi, c->N * 8, cudaMemcpyDeviceToDevice, c->s));
        const double* Pin[3];
        P_in(c, Pin);
        ++g_launches;
        r = k_status(c, launch_mean_p(c->dp, c->d_code, Pin, c->d_part, c->d_counter, A.hist + 3 * (n - 1), c->s));
        if (r) return r;
        if (n % k == 0 && n / k < A.nck) {
            const int q = n / k;
            if ((r = adj_save(c, &A.ckP[3 * q], A.ckPhi[q], A.ckRho[q]))) return r;
        }
    }
    if ((r = adj_save(c, A.finP, A.finPhi, A.finRho))) return r;
    std::vector<double> h(3 * (size_t)T);
    FX_CUDA(c, cudaMemcpyAsync(h.data(), A.hist, h.size() * 8, cudaMemcpyDeviceToHost, c->s));
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    A.m.resize(T);
    double L = 0.0;
    for (int n = 0; n < T; ++n) {
        A.m[n] = h[3 * n + 2];
        const double e = A.m[n] - A.target[n];
        L += e * e;
    }
    A.loss = L / T;
    *loss = A.loss;
    c->step += T;
    c->time += T * c->par.dt;
    A.valid = true;
    A.gen = c->gen;
    A.fwd_ms = ms_since(t0);
    return FX_OK;
}

// The adjoint Poisson solve of a reverse step as one graph: the coarse
// alphas of the step's linearisation (semiconductor), psi cleared when the
// source is zero, and the device-controlled multigrid loop with its target
// rtol max|mu| formed on the device from A.nmu.  The loop's statistics and a
// failure accumulate in the step control block, read once after the
// backward.  Returns false where conditional capture is unavailable.
bool adj_solve_graph(fx_ctx* c, const DevParams& dp0, bool sc, bool mixed) {
    auto& A = c->adj;
    if (!c->d_ctl) {
        if (dmalloc(c, &c->d_ctl, 1)) return false;
        if (cudaMallocHost(&c->h_ctl, sizeof(StepCtl)) != cudaSuccess) return false;
        if (c->cap.init() != cudaSuccess) return false;
    }
    c->cap.reset();
    const long long l0 = g_launches.load();
    if (cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
    if (sc) c->mg.set_alpha(A.drho, A.drho32, true, c->s);
    else c->mg.set_alpha(nullptr, nullptr, false, c->s);
    launch_zero_if_zero(A.psi, A.nmu, (long long)c->N, c->s);
    if (mixed)
        c->mg.enqueue_solve_mixed_ctl(dp0, c->d_code, A.psi, A.mu, A.nmu, c->par.mg_rtol, c->par.mg_max_iter, c->d_ctl,
                                      c->cap, c->s, false);
    else
        c->mg.enqueue_solve64_ctl(dp0, c->d_code, A.psi, A.mu, A.nmu, c->par.mg_rtol, c->par.mg_max_iter, c->d_ctl,
                                  c->cap, c->s, false);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->s, &graph);
    g_launches -= g_launches.load() - l0;   // counted per execution by the caller's estimate
    if (!e) e = c->cap.err;
    if (!e) e = cudaGetLastError();
    if (!e) e = cudaGraphInstantiate(&A.solve_exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e) {
        if (A.solve_exec) { cudaGraphExecDestroy(A.solve_exec); A.solve_exec = nullptr; }
        cudaGetLastError();
        return false;
    }
    return true;
}

int backward(fx_ctx* c, double* grads, int ngrads) {
    const auto t0 = std::chrono::steady_clock::now();
    auto& A = c->adj;
    const int T = A.T, k = A.k;
    const bool sc = c->contains_sc, vec = !c->scalarP;
    const int mixed = c->par.precision == 1;
    const int d0 = ncomp_first(c);
    int r = 0;
    if (A.segP.empty()) {
        A.segP.assign(3 * (size_t)k, nullptr);
        A.segPhi.assign(k, nullptr);
        for (int q = 0; q < k; ++q) {
            for (int d = d0; d < 3; ++d) if ((r = adj_alloc(c, &A.segP[3 * q + d], c->N))) return r;
            if (sc && !A.phiAll && (r = adj_alloc(c, &A.segPhi[q], c->N))) return r;
        }
        for (int b = 0; b < 2; ++b)
            for (int d = d0; d < 3; ++d) if ((r = adj_alloc(c, &A.lam[b][d], c->N))) return r;
        if ((r = adj_alloc(c, &A.mu, c->N))) return r;
        if ((r = adj_alloc(c, &A.psi, c->N))) return r;
        for (int q = 0; q < std::min(kMaxExtrap, c->par.phi_extrapolate); ++q)
            if ((r = adj_alloc(c, &A.psiHist[q], c->N))) return r;
        if ((r = adj_alloc(c, &A.nmu, 2))) return r;
        if (sc && ((r = adj_alloc(c, &A.drho, c->N)) || (r = adj_alloc(c, &A.drho32, c->N)))) return r;
        if ((r = adj_alloc(c, &A.grad, 8 + 256))) return r;
        if ((r = adj_alloc(c, &A.dV, (size_t)T))) return r;
        if (c->grains_set && !c->gid.empty()) {
            if ((r = adj_alloc(c, &A.gid, c->N))) return r;
            FX_CUDA(c, cudaMemcpyAsync(A.gid, c->gid.data(), c->N, cudaMemcpyHostToDevice, c->s));
        }
    }
    FX_CUDA(c, cudaMemsetAsync(A.grad, 0, (8 + 256) * 8, c->s));
    FX_CUDA(c, cudaMemsetAsync(A.dV, 0, (size_t)T * 8, c->s));
    FX_CUDA(c, cudaMemsetAsync(A.psi, 0, c->N * 8, c->s));
    A.psi_n = 0;
    // dL/d<Pz>^n spread over the FE cells
    std::vector<double> g(T + 1, 0.0);
    for (int n = 1; n <= T; ++n) g[n] = 2.0 / T * (A.m[n - 1] - A.target[n - 1]) / (double)A.nfe;
    int cur = 0;
    if ((r = k_status(c, launch_adj_init(c->dp, c->d_code, A.lam[cur], g[T], c->s)))) return r;
    ++g_launches;
    DevParams dp0 = poisson_params(c);   // the adjoint solve: homogeneous electrode values
    dp0.V_lo = 0.0;
    dp0.V_hi = 0.0;
    const int ngalpha = (int)c->galpha.size();
    // the reverse steps without a host round trip: the adjoint solve as a
    // device-controlled graph (fx.step_graph = 1, no per-kernel profiling)
    bool dev_solve = false;
    // the solve graph lives for this backward only, whatever path leaves it
    struct ExecGuard {
        cudaGraphExec_t* e;
        ~ExecGuard() { if (*e) { cudaGraphExecDestroy(*e); *e = nullptr; } }
    } guard{&A.solve_exec};
    if (c->par.include_Elec && c->par.step_graph && !c->prof.on) {
        dev_solve = adj_solve_graph(c, dp0, sc, mixed);
        if (dev_solve) {
            ++g_launches;
            if ((r = k_status(c, launch_ctl_step_begin(c->d_ctl, A.nmu, c->s)))) return r;
        }
    }
    for (int s = A.nck - 1; s >= 0; --s) {
        const int start = s * k, end = std::min(T, start + k);
        if ((r = adj_restore(c, &A.ckP[3 * s], A.ckPhi[s], A.ckRho[s]))) return r;
        for (int n = start + 1; n <= end; ++n) {
            const int idx = n - 1 - start;
            for (int d = d0; d < 3; ++d)
                if ((r = dcopy(c, A.segP[3 * idx + d], c->d_P[c->cur][d]))) return r;
            c->Phi_Bc_hi = A.V[n - 1];
            electrode_values(c);
            if (A.phiAll) {
                // the recorded phi^n: the same TDGL update as the forward's
                if ((r = tdgl_euler_with_phi(c, A.phiAll + (size_t)(n - 1) * c->N))) return r;
            } else {
                if ((r = compute_phi_rho(c))) return r;
                if (sc && (r = dcopy(c, A.segPhi[idx], c->d_phi))) return r;
                if ((r = tdgl_update(c))) return r;
            }
            c->prof.collect();
        }
        for (int n = end; n >= start + 1; --n) {
            const int idx = n - 1 - start;
            const double* psi = nullptr;
            if (dev_solve) {
                // no host round trip: the source norm, the linearisation, the
                // initial iterate and the graph of the solve, in stream order
                FX_CUDA(c, cudaMemsetAsync(A.nmu, 0, 2 * sizeof(double), c->s));
                ++g_launches;
                r = k_status(c, launch_adj_phi(c->dp, mixed, vec, c->d_code, c->d_var, c->d_vt, A.lam[cur], A.mu,
                                               A.nmu, A.dV + (n - 1), c->s));
                if (r) return r;
                if (sc) {
                    ++g_launches;
                    const double* phin = A.phiAll ? A.phiAll + (size_t)(n - 1) * c->N : A.segPhi[idx];
                    if ((r = k_status(c, launch_drho(c->dp, c->d_code, phin, A.drho, A.drho32, c->s)))) return r;
                }
                int order = 0;
                while (order < 6 && A.psiHist[order]) ++order;
                if (order > 0 && c->par.warm_start && c->adj_extrap) {
                    const int use = std::min(order, A.psi_n);
                    if (use > 0) {
                        ++g_launches;
                        if ((r = k_status(c, launch_phi_extrap(c->dp, use, A.psi, A.psiHist, c->s)))) return r;
                    } else {
                        FX_CUDA(c, cudaMemcpyAsync(A.psiHist[0], A.psi, c->N * 8, cudaMemcpyDeviceToDevice, c->s));
                    }
                    A.psi_n = std::min(order, A.psi_n + 1);
                }
                FX_CUDA(c, cudaGraphLaunch(A.solve_exec, c->s));
                psi = A.psi;   // zero where the source is zero
            } else if (c->par.include_Elec) {
                FX_CUDA(c, cudaMemsetAsync(c->d_out, 0, sizeof(double), c->s));
                ++g_launches;
                r = k_status(c, launch_adj_phi(c->dp, mixed, vec, c->d_code, c->d_var, c->d_vt, A.lam[cur], A.mu,
                                               c->d_out, A.dV + (n - 1), c->s));
                if (r) return r;
                if ((r = read_out(c, 1))) return r;
                const double nmu = c->h_out[0];
                if (!std::isfinite(nmu)) return set_err(c, FX_ERR_NONFINITE, "adjoint source is not finite");
                if (nmu > 0.0) {
                    if (sc) {
                        ++g_launches;
                        const double* phin = A.phiAll ? A.phiAll + (size_t)(n - 1) * c->N : A.segPhi[idx];
                        r = k_status(c, launch_drho(c->dp, c->d_code, phin, A.drho, A.drho32, c->s));
                        if (r) return r;
                        c->mg.set_alpha(A.drho, A.drho32, true, c->s);
                    } else {
                        c->mg.set_alpha(nullptr, nullptr, false, c->s);
                    }
                    // the initial iterate: psi extrapolated in reverse time through the
                    // solutions of the last reverse steps (the forward's phi rule); the
                    // solve still runs to the residual bound
                    int order = 0;
                    while (order < 6 && A.psiHist[order]) ++order;
                    if (order > 0 && c->par.warm_start && c->adj_extrap) {
                        const int use = std::min(order, A.psi_n);
                        if (use > 0) {
                            ++g_launches;
                            if ((r = k_status(c, launch_phi_extrap(c->dp, use, A.psi, A.psiHist, c->s)))) return r;
                        } else {
                            FX_CUDA(c, cudaMemcpyAsync(A.psiHist[0], A.psi, c->N * 8, cudaMemcpyDeviceToDevice, c->s));
                        }
                        A.psi_n = std::min(order, A.psi_n + 1);
                    }
                    const double target = std::max(c->par.mg_rtol, 1e-16) * nmu;
                    MGStats st;
                    int e = mixed ? c->mg.solve_mixed(dp0, c->d_code, A.psi, A.mu, target, c->par.mg_max_iter, c->s, &st)
                                  : c->mg.solve64(dp0, c->d_code, A.psi, A.mu, target, c->par.mg_max_iter, c->s, &st);
                    A.mg_cycles += st.cycles;
                    if (e == -3) {
                        std::ostringstream o;
                        o << "adjoint Poisson multigrid did not reach |r| <= " << target << " (|r| = " << st.resid << ")";
                        return set_err(c, std::isfinite(st.resid) ? FX_ERR_NO_CONVERGENCE : FX_ERR_NONFINITE, o.str());
                    }
                    if (e) return set_err(c, FX_ERR_CUDA, std::string("multigrid: ") + cudaGetErrorString((cudaError_t)e));
                    psi = A.psi;
                } else {
                    A.psi_n = 0;   // psi = 0 this step: the history starts again
                }
            }
            const double* Pn[3] = {A.segP[3 * idx], A.segP[3 * idx + 1], A.segP[3 * idx + 2]};
            ++g_launches;
            r = k_status(c, launch_adj_P(c->dp, mixed, vec, c->d_code, c->d_var, c->d_vt, A.gid, ngalpha, Pn,
                                         A.lam[cur], psi, g[n - 1], A.lam[1 - cur], A.grad, A.dV + (n - 1), c->s));
            if (r) return r;
            cur = 1 - cur;
        }
    }
    if (dev_solve) {
        FX_CUDA(c, cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, c->s));
        FX_CUDA(c, cudaStreamSynchronize(c->s));
        const StepCtl& t = *c->h_ctl;
        A.mg_cycles += t.mg_cycles_step;
        if (t.status != CTL_OK) {
            std::ostringstream o;
            o << "adjoint Poisson multigrid did not reach |r| <= " << t.status_target << " (|r| = " << t.status_val << ")";
            return set_err(c, t.status == CTL_MG_NO_CONV ? FX_ERR_NO_CONVERGENCE : FX_ERR_NONFINITE, o.str());
        }
    }
    A.lcur = cur;
    A.have_P0 = true;
    if ((r = adj_restore(c, A.finP, A.finPhi, A.finRho))) return r;
    c->Phi_Bc_hi = A.V[T - 1];
    electrode_values(c);
    std::vector<double> hg(8 + 256), hv(T);
    FX_CUDA(c, cudaMemcpyAsync(hg.data(), A.grad, hg.size() * 8, cudaMemcpyDeviceToHost, c->s));
    FX_CUDA(c, cudaMemcpyAsync(hv.data(), A.dV, hv.size() * 8, cudaMemcpyDeviceToHost, c->s));
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    for (int q = 0; q < 5; ++q) grads[q] = hg[q];
    double gv = 0.0;
    for (int n = 0; n < T; ++n) gv += A.shape[n] * hv[n];
    grads[FX_GRAD_V_AMP] = gv;
    const int ng = c->grains_set ? c->ngrains : 0;
    for (int q = FX_GRAD_GRAIN_ALPHA; q < ngrads; ++q) {
        const int gi = q - FX_GRAD_GRAIN_ALPHA;
        grads[q] = gi < ng ? hg[8 + gi] : 0.0;
    }
    A.bwd_ms = ms_since(t0);
    return FX_OK;
}

void read_inputs(const char* inputs, int is_text, std::string& text) {
    if (is_text) { text = inputs; return; }
    std::ifstream f(inputs);
    if (!f) throw FxError{FX_ERR_IO, std::string("cannot open inputs file ") + inputs};
    std::stringstream ss;
    ss << f.rdbuf();
    text = ss.str();
}

}  // namespace

extern "C" {

const char* fx_version(void) { return "ferrox_b200 0.1 (sm_100a)"; }

const char* fx_create_error(void) { return t_create_error.c_str(); }

// ---- input files named by fx.initial_P_file and fx.grain_file ----

static std::vector<char> read_binary(const std::string& path, const char* what) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw FxError{FX_ERR_IO, std::string("cannot open ") + what + " '" + path + "'"};
    return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

// fx.initial_P_file: raw little-endian FP64, x fastest; N values (Pz, with
// Px = Py = 0) or 3N values (the Px, Py and Pz blocks in that order)
static void load_P_file(fx_ctx* c, const std::string& path) {
    const std::vector<char> b = read_binary(path, "fx.initial_P_file");
    const size_t N = c->N;
    if (b.size() != N * 8 && b.size() != 3 * N * 8)
        throw FxError{FX_ERR_INPUTS, "fx.initial_P_file '" + path + "' holds " + std::to_string(b.size()) +
                                         " bytes; expected 8*N (Pz) or 24*N (Px, Py, Pz) for N = " + std::to_string(N)};
    std::vector<double> v(b.size() / 8);
    std::memcpy(v.data(), b.data(), b.size());
    const bool three = v.size() == 3 * N;
    const int r = fx_set_initial_P(c, three ? v.data() : nullptr, three ? v.data() + N : nullptr,
                                   v.data() + (three ? 2 * N : 0), N);
    if (r) throw FxError{r, c->err};
}

// fx.grain_file: "FXGRAIN1", int32 nx, ny, nz, ngrains (little-endian), then
// per grain four FP64 (Euler angles alpha, beta, theta in degrees, t-phase
// flag 0/1), then N uint8 grain ids, x fastest (255: no grain)
static void load_grain_file(fx_ctx* c, const std::string& path) {
    const std::vector<char> b = read_binary(path, "fx.grain_file");
    const std::string bad = "fx.grain_file '" + path + "': ";
    if (b.size() < 24 || std::memcmp(b.data(), "FXGRAIN1", 8) != 0) throw FxError{FX_ERR_INPUTS, bad + "not a grain file"};
    int32_t h[4];
    std::memcpy(h, b.data() + 8, 16);
    if (h[0] != c->nx || h[1] != c->ny || h[2] != c->nz)
        throw FxError{FX_ERR_INPUTS, bad + "grid " + std::to_string(h[0]) + "x" + std::to_string(h[1]) + "x" +
                                         std::to_string(h[2]) + " differs from domain.n_cell"};
    const int ng = h[3];
    if (ng < 1 || ng > 255) throw FxError{FX_ERR_INPUTS, bad + "ngrains must be 1..255"};
    const size_t need = 24 + (size_t)ng * 32 + c->N;
    if (b.size() != need) throw FxError{FX_ERR_INPUTS, bad + "size " + std::to_string(b.size()) + ", expected " + std::to_string(need)};
    std::vector<double> per((size_t)ng * 4);
    std::memcpy(per.data(), b.data() + 24, per.size() * 8);
    std::vector<double> ang((size_t)ng * 3);
    std::vector<uint8_t> tph(ng);
    for (int g = 0; g < ng; ++g) {
        for (int d = 0; d < 3; ++d) ang[3 * g + d] = per[4 * g + d];
        const double t = per[4 * g + 3];
        if (t != 0.0 && t != 1.0) throw FxError{FX_ERR_INPUTS, bad + "t-phase flags must be 0 or 1"};
        tph[g] = t == 1.0 ? 1 : 0;
    }
    const uint8_t* gid = reinterpret_cast<const uint8_t*>(b.data() + 24 + (size_t)ng * 32);
    const int r = fx_set_grains(c, gid, c->N, ang.data(), tph.data(), ng);
    if (r) throw FxError{r, c->err};
}

int fx_create(const char* inputs, int is_text, fx_ctx** out) {
    if (!out) return FX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    t_create_error.clear();
    if (!inputs) { t_create_error = "inputs is NULL"; return FX_ERR_INVALID_ARGUMENT; }
    std::unique_ptr<fx_ctx> c(new fx_ctx());
    try {
        std::string text;
        read_inputs(inputs, is_text, text);
        c->in = parse_inputs(text);
        c->par = make_params(c->in);
        Params& p = c->par;
        read_embedded_boundary(c.get());
        if (!p.is_periodic[0] || !p.is_periodic[1] || p.is_periodic[2])
            throw FxError{FX_ERR_UNSUPPORTED, "only domain.is_periodic = 1 1 0 (periodic x/y, electrodes in z) is supported"};
        for (int d = 0; d < 2; ++d)
            if ((!p.bc_lo[d].empty() && p.bc_lo[d].substr(0, 3) != "per") || (!p.bc_hi[d].empty() && p.bc_hi[d].substr(0, 3) != "per"))
                throw FxError{FX_ERR_INPUTS, "boundary.lo/hi must be 'per' in periodic directions (BoundaryConditions.cpp:196)"};
        // the top boundary lies inside the covered cells of an embedded
        // boundary, where its type (the reference's EB decks give neu) never enters
        const bool hi_covered = c->eb_nz > 0;
        if ((!p.bc_lo[2].empty() && p.bc_lo[2].substr(0, 3) != "dir") ||
            (!hi_covered && !p.bc_hi[2].empty() && p.bc_hi[2].substr(0, 3) != "dir") ||
            (hi_covered && !p.bc_hi[2].empty() && p.bc_hi[2].substr(0, 3) == "per"))
            throw FxError{FX_ERR_UNSUPPORTED, "z boundaries must be Dirichlet electrodes (dir)"};
        c->nx = p.n_cell[0]; c->ny = p.n_cell[1]; c->nz = p.n_cell[2];
        for (int d = 0; d < 2; ++d)
            if (p.n_cell[d] != 1 && p.n_cell[d] % 2 != 0)
                throw FxError{FX_ERR_UNSUPPORTED, "periodic x/y cell counts must be even (red-black ordering) or 1"};
        c->nxy = (size_t)c->nx * c->ny;
        c->N = c->nxy * c->nz;
        for (int d = 0; d < 3; ++d) c->dx[d] = (p.prob_hi[d] - p.prob_lo[d]) / p.n_cell[d];
        // DphiDz decides the electrode layers from cell-face positions
        // (ElectrostaticSolver.cpp:162-163); the device uses k == 0 / nz-1
        for (int k = 0; k < c->nz; ++k) {
            const double z_hi = p.prob_lo[2] + (k + 1.5) * c->dx[2];
            const double z_lo = p.prob_lo[2] + (k - 0.5) * c->dx[2];
            const bool bot = z_lo < p.prob_lo[2], top = !bot && z_hi > p.prob_hi[2];
            if (bot != (k == 0) || top != (k == c->nz - 1 && c->nz > 1))
                throw FxError{FX_ERR_UNSUPPORTED, "electrode-layer test of DphiDz does not select k = 0 / nz-1 for this grid"};
        }
        // t-phase mask and Euler angles (main.cpp:178-181)
        c->tphase.assign(c->N, 0.0);
        for (int d = 0; d < 3; ++d) c->ang[d].assign(c->N, 0.0);
        if (p.Coordinate_Transformation == 1) {
            const char* keys[4] = {"tphase_geom.tphase_geom_function(x,y,z)", "angle_alpha.alpha_function(x,y,z)",
                                   "angle_beta.beta_function(x,y,z)", "angle_theta.theta_function(x,y,z)"};
            std::vector<double>* dst[4] = {&c->tphase, &c->ang[0], &c->ang[1], &c->ang[2]};
            for (int f = 0; f < 4; ++f) {
                auto it = c->in.table.find(keys[f]);
                if (it == c->in.table.end() || it->second.empty()) continue;   // set later by fx_set_grains
                std::string ex;
                for (auto& s : it->second) ex += (ex.empty() ? "" : " ") + s;
                auto e = compile_expr(ex, c->in.constants);
                for (int k = 0; k < c->nz; ++k)
                    for (int j = 0; j < c->ny; ++j)
                        for (int i = 0; i < c->nx; ++i)
                            (*dst[f])[(size_t)i + c->nx * ((size_t)j + (size_t)c->ny * k)] =
                                e->eval(p.prob_lo[0] + (i + 0.5) * c->dx[0], p.prob_lo[1] + (j + 0.5) * c->dx[1],
                                        p.prob_lo[2] + (k + 0.5) * c->dx[2]);
            }
        }
        build_codes(c.get());
        std::string w = check_wrapped_mask(c.get());
        if (!w.empty()) throw FxError{FX_ERR_UNSUPPORTED, w};
        build_variants(c.get(), nullptr, nullptr);
        build_P0(c.get());
        c->Phi_Bc_hi = p.Phi_Bc_hi;
        c->inc_step = p.inc_step;
        if (!p.grain_file.empty()) {
            if (p.Coordinate_Transformation != 1)
                throw FxError{FX_ERR_INPUTS, "fx.grain_file needs Coordinate_Transformation = 1 (the grains carry "
                                             "the tphase mask and Euler angles)"};
            load_grain_file(c.get(), p.grain_file);
        }
        if (!p.initial_P_file.empty()) load_P_file(c.get(), p.initial_P_file);
        fill_devparams(c.get());
    } catch (FxError& e) {
        t_create_error = e.msg;
        return e.code;
    } catch (std::exception& e) {
        t_create_error = e.what();
        return FX_ERR_INPUTS;
    }
    *out = c.release();
    return FX_OK;
}

void fx_destroy(fx_ctx* c) {
    if (!c) return;
    if (c->dev) {
        cudaStreamSynchronize(c->s);
        adj_free(c);
        cudaFree(c->adj_phi_store);
        cudaFree(c->d_code); cudaFree(c->d_var); cudaFree(c->d_vt); cudaFree(c->d_interior);
        for (int b = 0; b < 2; ++b)
            for (int d = 0; d < 3; ++d) cudaFree(c->d_P[b][d]);
        for (double* a : {c->d_phi, c->d_phi_old, c->d_phi_prev, c->d_rho, c->d_e, c->d_h, c->d_alpha, c->d_rhs,
                          c->d_rhsP, c->d_dphi, c->d_E[0], c->d_E[1], c->d_E[2], c->d_f[0], c->d_f[1], c->d_f[2],
                          c->d_part, c->d_out, c->d_phi_hist[0], c->d_phi_hist[1], c->d_phi_hist[2], c->d_phi_hist[3],
                          c->d_phi_hist[4], c->d_phi_hist[5]})
            cudaFree(a);
        cudaFree(c->d_alpha32);
        cudaFree(c->d_counter);
        if (c->h_out) cudaFreeHost(c->h_out);
        for (auto& g : c->sgraphs) if (g.exec) cudaGraphExecDestroy(g.exec);
        c->sgraphs.clear();
        cudaFree(c->d_ctl);
        if (c->h_ctl) cudaFreeHost(c->h_ctl);
        c->cap.release();
        c->prof.collect();
        if (c->own_stream) cudaStreamDestroy(c->s);
    }
    delete c;
}

const char* fx_last_error(const fx_ctx* c) { return c ? c->err.c_str() : "null context"; }

int fx_get_dims(const fx_ctx* c, int n[3], double dx[3]) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    if (n) { n[0] = c->nx; n[1] = c->ny; n[2] = c->nz; }
    if (dx) for (int d = 0; d < 3; ++d) dx[d] = c->dx[d];
    return FX_OK;
}

int fx_get_param(const fx_ctx* c, const char* key, double* v) {
    if (!c || !key || !v) return FX_ERR_INVALID_ARGUMENT;
    const Params& p = c->par;
    const std::string k(key);
    static const char* arr3[] = {"FE_lo", "FE_hi", "DE_lo", "DE_hi", "SC_lo", "SC_hi", "Channel_lo", "Channel_hi", "Remnant_P",
                                 "domain.prob_lo", "domain.prob_hi"};
    const std::map<std::string, double> m = {
        {"dt", p.dt}, {"lambda", p.lambda}, {"epsilon_0", p.epsilon_0}, {"epsilonX_fe", p.epsilonX_fe},
        {"epsilonX_fe_tphase", p.epsilonX_fe_tphase}, {"epsilonZ_fe", p.epsilonZ_fe}, {"epsilon_de", p.epsilon_de},
        {"epsilon_si", p.epsilon_si}, {"alpha", p.alpha}, {"beta", p.beta}, {"gamma", p.gamma}, {"alpha_12", p.alpha_12},
        {"alpha_112", p.alpha_112}, {"alpha_123", p.alpha_123}, {"BigGamma", p.BigGamma}, {"g11", p.g11}, {"g44", p.g44},
        {"g12", p.g12}, {"g44_p", p.g44_p}, {"acceptor_doping", p.acceptor_doping}, {"donor_doping", p.donor_doping},
        {"use_Fermi_Dirac", p.use_Fermi_Dirac}, {"use_work_function", p.use_work_function},
        {"metal_work_function", p.metal_work_function}, {"is_polarization_scalar", p.is_polarization_scalar},
        {"delta", p.delta}, {"voltage_sweep", p.voltage_sweep}, {"inc_step", c->inc_step}, {"Phi_Bc_lo", p.Phi_Bc_lo},
        {"Phi_Bc_hi", c->Phi_Bc_hi}, {"Phi_Bc_inc", p.Phi_Bc_inc}, {"Phi_Bc_hi_max", p.Phi_Bc_hi_max},
        {"phi_tolerance", p.phi_tolerance}, {"num_Vapp_max", p.num_Vapp_max}, {"random_seed", p.random_seed},
        {"include_Landau", p.include_Landau}, {"include_Grad", p.include_Grad}, {"include_Elec", p.include_Elec},
        {"Coordinate_Transformation", p.Coordinate_Transformation}, {"use_Euler_angles", p.use_Euler_angles},
        {"prob_type", p.prob_type}, {"TimeIntegratorOrder", p.TimeIntegratorOrder}, {"nsteps", p.nsteps},
        {"plot_int", p.plot_int}, {"fx.mg_rtol", p.mg_rtol}, {"fx.phi_ghost_mode", p.phi_ghost_mode},
        {"fx.sweep_mode", p.sweep_mode}, {"fx.steps_per_voltage", p.steps_per_voltage},
        {"fx.newton_max_iter", p.newton_max_iter}, {"fx.mg_max_iter", p.mg_max_iter}, {"fx.precision", p.precision},
        {"fx.warm_start", p.warm_start}, {"fx.phi_extrapolate", p.phi_extrapolate}, {"fx.step_graph", p.step_graph},
        {"contains_sc", c->contains_sc ? 1.0 : 0.0},
        {"V_lo", c->dp.V_lo}, {"V_hi", c->dp.V_hi}, {"phi_ref", phi_ref()},
        {"intrinsic_carrier_concentration", std::sqrt(kNc * kNv) * exp(-0.5 * kQ * kEg / (kKb * kT))},
        {"num_variants", (double)c->variants.size()}, {"fx.newton_tol", p.newton_tol},
        {"adjoint_mg_cycles", (double)c->adj.mg_cycles}, {"adjoint_forward_ms", c->adj.fwd_ms},
        {"adjoint_backward_ms", c->adj.bwd_ms}, {"adjoint_bytes", (double)c->adj.bytes},
        {"adjoint_loss", c->adj.loss},
        {"fx.mg_nu1", (double)c->mg.nu1}, {"fx.mg_nu2", (double)c->mg.nu2},
        {"fx.mg_mixed_cycles", (double)c->mg.mixed_cycles}, {"fx.alpha_tiles", c->mg.alpha_tiles ? 1.0 : 0.0},
        {"fx.mg_seg", (double)c->mg.seg_bytes}, {"fx.mg_seg_min", (double)c->mg.seg_min_cells},
        {"fx.mg_split", c->mg.split_mode ? 1.0 : 0.0}, {"fx.mg_half", c->mg.half_coarse ? 1.0 : 0.0},
        {"fx.mg_dense", c->mg.dense_coarse ? 1.0 : 0.0}, {"mg_level0_split", c->mg.split_now_ ? 1.0 : 0.0},
        {"fx.mg_nu1_coarse", (double)c->mg.nu1c}, {"fx.mg_nu2_coarse", (double)c->mg.nu2c},
        {"fx.interior", c->use_interior ? 1.0 : 0.0}, {"fx.adjoint_store_phi", c->adj_store_phi ? 1.0 : 0.0},
        {"fx.adjoint_extrapolate", c->adj_extrap ? 1.0 : 0.0},
        {"adjoint_phi_stored", c->adj.phiAll ? 1.0 : 0.0},
        {"step_graph_ran", c->sg_ran ? 1.0 : 0.0}, {"fx.pdl", g_pdl ? 1.0 : 0.0},
        {"fx.rhs_seg", g_rhs_seg ? 1.0 : 0.0},
        // the embedded boundary: the Poisson solve's fluid layers (0: none)
        // and the Dirichlet value on their top face
        {"eb_fluid_layers", (double)c->eb_nz}, {"eb_surf_soln", c->eb_V},
        // 1 when level 0's face coefficients depend on z only and its smoother
        // reads them by plane instead of from the material codes
        {"mg_level0_planes",!c->mg.levels().empty() && (c->mg.levels()[0].zc64 || c->mg.levels()[0].zc32) ? 1.0 : 0.0}};
    auto it = m.find(k);
    if (it != m.end()) { *v = it->second; return FX_OK; }
    // "FE_lo[2]" style access to the 3-vectors
    for (const char* a : arr3) {
        const std::string s(a);
        if (k.size() == s.size() + 3 && k.compare(0, s.size(), s) == 0 && k[s.size()] == '[' && k.back() == ']') {
            const int d = k[s.size() + 1] - '0';
            if (d < 0 || d > 2) break;
            const double* arr = s == "FE_lo" ? p.FE_lo : s == "FE_hi" ? p.FE_hi : s == "DE_lo" ? p.DE_lo : s == "DE_hi" ? p.DE_hi
                              : s == "SC_lo" ? p.SC_lo : s == "SC_hi" ? p.SC_hi : s == "Channel_lo" ? p.Channel_lo
                              : s == "Channel_hi" ? p.Channel_hi : s == "Remnant_P" ? p.Remnant_P
                              : s == "domain.prob_lo" ? p.prob_lo : p.prob_hi;
            *v = arr[d];
            return FX_OK;
        }
    }
    for (const char* a : {"P_BC_flag_lo", "P_BC_flag_hi", "domain.n_cell", "domain.is_periodic"}) {
        const std::string s(a);
        if (k.size() == s.size() + 3 && k.compare(0, s.size(), s) == 0 && k[s.size()] == '[') {
            const int d = k[s.size() + 1] - '0';
            if (d < 0 || d > 2) break;
            const int* arr = s == "P_BC_flag_lo" ? p.P_BC_flag_lo : s == "P_BC_flag_hi" ? p.P_BC_flag_hi
                           : s == "domain.n_cell" ? p.n_cell : p.is_periodic;
            *v = arr[d];
            return FX_OK;
        }
    }
    return FX_ERR_INVALID_ARGUMENT;
}

int fx_set_param(fx_ctx* c, const char* key, double v) {
    if (!c || !key) return FX_ERR_INVALID_ARGUMENT;
    const std::string k(key);
    Params& p = c->par;
    // every refusal comes before any state changes: a refused call leaves the
    // context (the step graphs, the phi history, the adjoint record) as it was
    static const char* const known[] = {
        "Phi_Bc_hi", "Phi_Bc_lo", "fx.mg_rtol", "fx.mg_max_iter", "fx.newton_max_iter", "fx.warm_start",
        "fx.phi_extrapolate", "fx.step_graph", "fx.pdl", "fx.verbose", "fx.profile", "fx.mg_nu1", "fx.graphs",
        "fx.mg_nu2", "fx.alpha_tiles", "fx.interior", "fx.adjoint_store_phi", "fx.adjoint_extrapolate", "fx.mg_nu1_coarse", "fx.mg_nu2_coarse", "fx.mg_seg", "fx.mg_seg_min", "fx.mg_split", "fx.mg_half", "fx.mg_dense", "fx.rhs_seg", "fx.mg_mixed_cycles", "fx.phi_ghost_mode", "dt", "alpha", "fx.newton_tol",
        "beta", "gamma", "g11", "g44", "BigGamma", "inc_step"};
    bool is_known = false;
    for (const char* q : known) is_known = is_known || k == q;
    if (!is_known) return set_err(c, FX_ERR_INVALID_ARGUMENT, "parameter '" + k + "' cannot be set after creation");
    if (!std::isfinite(v)) return set_err(c, FX_ERR_INVALID_ARGUMENT, k + " must be finite");
    // the ranges the inputs reader applies to the same keys
    if (k == "fx.phi_extrapolate" && !(v >= 0 && v <= 6))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.phi_extrapolate must be 0..6");
    if (k == "fx.phi_ghost_mode" && !(v == 0 || v == 1 || v == 2))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.phi_ghost_mode must be 0 (extrap), 1 (face) or 2 (zero)");
    if ((k == "fx.mg_max_iter" || k == "fx.newton_max_iter") && !(v >= 1))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, k + " must be at least 1");
    if (k == "fx.mg_nu1_coarse" && !(v == -1 || v >= 1))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.mg_nu1_coarse must be -1 (as fx.mg_nu1) or at least 1");
    if (k == "fx.mg_nu2_coarse" && !(v >= -1))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.mg_nu2_coarse must be -1 (as fx.mg_nu2) or at least 0");
    if ((k == "fx.mg_nu1" || k == "fx.mg_nu2") && !(v >= 0))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, k + " must not be negative");
    if (k == "fx.mg_rtol" && !(v > 0))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.mg_rtol must be positive");
    if (k == "fx.mg_mixed_cycles" && !(v >= 1))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.mg_mixed_cycles must be at least 1");
    if (k == "fx.newton_tol" && !(v > 0.0))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.newton_tol must be positive");
    if (k == "fx.mg_seg" && !(v == 0 || v == 16 || v == 32))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.mg_seg must be 0 (one cell per thread), 16 or 32 (segment bytes)");
    if (k == "fx.mg_half" && c->dev)
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.mg_half must be set before the first device call");
    if (k == "fx.mg_seg_min" && !(v >= 0))
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx.mg_seg_min must not be negative");
    if (k != "fx.profile" && k != "fx.verbose" && k != "fx.graphs" && k != "fx.step_graph" && k != "fx.pdl" &&
        k != "fx.alpha_tiles" && k != "fx.interior" && k != "fx.adjoint_store_phi" && k != "fx.adjoint_extrapolate" &&
        k != "fx.mg_seg" &&
        k != "fx.mg_seg_min" && k != "fx.mg_split" && k != "fx.mg_half" && k != "fx.rhs_seg" && k != "fx.mg_dense")
        ++c->gen;
    // the time history of phi only seeds the next solve's initial iterate;
    // electrode values are compared on their own, solver settings leave the
    // trajectory alone, anything else starts the history afresh
    if (k != "Phi_Bc_hi" && k != "Phi_Bc_lo" && k.compare(0, 3, "fx.") != 0) c->hist_valid = false;
    if (k == "Phi_Bc_hi") { c->Phi_Bc_hi = v; electrode_values(c); c->E_valid = false; return FX_OK; }
    if (k == "Phi_Bc_lo") { p.Phi_Bc_lo = v; electrode_values(c); c->E_valid = false; return FX_OK; }
    if (k == "fx.mg_rtol") { p.mg_rtol = v; return FX_OK; }
    if (k == "fx.mg_max_iter") { p.mg_max_iter = (int)v; return FX_OK; }
    if (k == "fx.newton_max_iter") { p.newton_max_iter = (int)v; return FX_OK; }
    if (k == "fx.warm_start") { p.warm_start = (int)v; return FX_OK; }
    if (k == "fx.phi_extrapolate") { p.phi_extrapolate = (int)v; return FX_OK; }
    if (k == "fx.step_graph") { p.step_graph = (int)v; return FX_OK; }
    // process-wide: launches of every context
    if (k == "fx.pdl") { g_pdl = v != 0.0; return FX_OK; }
    if (k == "fx.verbose") { p.verbose = (int)v; c->mg.verbose = (int)v; return FX_OK; }
    if (k == "fx.profile") { c->prof.collect(); c->prof.on = v != 0.0; return FX_OK; }
    if (k == "fx.mg_nu1") { c->mg.nu1 = (int)v; return FX_OK; }
    if (k == "fx.graphs") { c->mg.set_graphs(v != 0.0); return FX_OK; }
    if (k == "fx.mg_nu2") { c->mg.nu2 = (int)v; return FX_OK; }
    if (k == "fx.alpha_tiles") { c->mg.alpha_tiles = v != 0.0; return FX_OK; }
    if (k == "fx.mg_seg") { c->mg.seg_bytes = (int)v; return FX_OK; }
    if (k == "fx.mg_split") { c->mg.split_mode = v != 0.0; return FX_OK; }
    if (k == "fx.mg_half") { c->mg.half_coarse = v != 0.0; return FX_OK; }
    if (k == "fx.rhs_seg") { g_rhs_seg = v != 0.0; return FX_OK; }
    if (k == "fx.mg_dense") { c->mg.dense_coarse = v != 0.0; return FX_OK; }
    if (k == "fx.mg_seg_min") { c->mg.seg_min_cells = (long long)std::min(v, 9.0e18); return FX_OK; }
    if (k == "fx.adjoint_store_phi") { c->adj_store_phi = v != 0.0; return FX_OK; }
    if (k == "fx.adjoint_extrapolate") { c->adj_extrap = v != 0.0; return FX_OK; }
    if (k == "fx.mg_nu1_coarse") { c->mg.nu1c = (int)v; return FX_OK; }
    if (k == "fx.mg_nu2_coarse") { c->mg.nu2c = (int)v; return FX_OK; }
    if (k == "fx.interior") {
        c->use_interior = v != 0.0;
        c->dp.interior = c->use_interior ? c->d_interior : nullptr;
        return FX_OK;
    }
    if (k == "fx.mg_mixed_cycles") { c->mg.mixed_cycles = (int)v; return FX_OK; }
    if (k == "fx.phi_ghost_mode") { p.phi_ghost_mode = (int)v; c->dp.ghost_mode = (int)v; c->E_valid = false; return FX_OK; }
    if (k == "dt") { p.dt = v; c->dp.dt = v; return FX_OK; }
    if (k == "alpha") {
        p.alpha = v;
        c->dp.alpha = v;
        // the rotation table carries alpha per variant: update the ones that
        // use the global value (grain alphas set by fx_set_grain_alpha stay)
        bool any = false;
        for (size_t q = 0; q < c->variants.size(); ++q)
            if (c->variant_global_alpha[q]) { c->variants[q].alpha = v; any = true; }
        if (any && c->dev && c->d_vt) {
            FX_CUDA(c, cudaMemcpyAsync(c->d_vt, c->variants.data(), c->variants.size() * sizeof(Variant),
                                       cudaMemcpyHostToDevice, c->s));
            FX_CUDA(c, cudaStreamSynchronize(c->s));
        }
        return FX_OK;
    }
    if (k == "fx.newton_tol") { p.newton_tol = v; return FX_OK; }
    if (k == "beta") { p.beta = v; c->dp.beta = v; return FX_OK; }
    if (k == "gamma") { p.gamma = v; c->dp.gamma = v; return FX_OK; }
    if (k == "g11") { p.g11 = v; c->dp.g11 = v; return FX_OK; }
    if (k == "g44") { p.g44 = v; c->dp.g44 = v; return FX_OK; }
    if (k == "BigGamma") { p.BigGamma = v; c->dp.BigGamma = v; return FX_OK; }
    if (k == "inc_step") { c->inc_step = (int)v; return FX_OK; }
    return set_err(c, FX_ERR_INVALID_ARGUMENT, "parameter '" + k + "' cannot be set after creation");
}

int fx_set_precision(fx_ctx* c, int mode) {
    if (!c || (mode != 0 && mode != 1)) return FX_ERR_INVALID_ARGUMENT;
    if (c->dev && mode != c->par.precision)
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "precision must be chosen before the first device call");
    ++c->gen;
    c->hist_valid = false;
    c->par.precision = mode;
    return FX_OK;
}

int fx_set_initial_P(fx_ctx* c, const double* Px, const double* Py, const double* Pz, size_t n) {
    if (!c || !Pz || n != c->N) return c ? set_err(c, FX_ERR_INVALID_ARGUMENT, "P arrays must hold nx*ny*nz values") : FX_ERR_INVALID_ARGUMENT;
    const double* src[3] = {Px, Py, Pz};
    bool zero_xy = true;
    for (int d = 0; d < 2 && zero_xy; ++d)
        if (src[d]) for (size_t q = 0; q < n; ++q) if (src[d][q] != 0.0) { zero_xy = false; break; }
    const bool scalar = c->par.is_polarization_scalar == 1 && zero_xy;
    ++c->gen;
    c->hist_valid = false;
    c->user_P = true;
    c->scalarP = scalar;
    if (!c->dev) {
        // kept on the host until the device state is made (ensure_device uploads it)
        for (int d = 0; d < 3; ++d) {
            if (src[d]) c->P0[d].assign(src[d], src[d] + n);
            else c->P0[d].assign(n, 0.0);
        }
        return FX_OK;
    }
    // on the device: each component crosses the bus once, straight from the
    // caller's buffer (a pinned buffer makes it a DMA transfer); the second
    // ping-pong buffer is filled on the device; missing components are zero
    const int other = 1 - c->cur;
    for (int d = 0; d < 3; ++d) {
        if (src[d]) FX_CUDA(c, cudaMemcpyAsync(c->d_P[c->cur][d], src[d], n * 8, cudaMemcpyHostToDevice, c->s));
        else FX_CUDA(c, cudaMemsetAsync(c->d_P[c->cur][d], 0, n * 8, c->s));
        FX_CUDA(c, cudaMemcpyAsync(c->d_P[other][d], c->d_P[c->cur][d], n * 8, cudaMemcpyDeviceToDevice, c->s));
    }
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    c->E_valid = false;
    return FX_OK;
}

int fx_set_grains(fx_ctx* c, const uint8_t* gid, size_t n, const double* ang, const uint8_t* gtph, int ng) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    if (!gid || !ang || !gtph || n != c->N || ng <= 0 || ng > 255)
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_set_grains: bad arguments");
    if (c->dev) return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_set_grains must precede the first device call");
    std::vector<uint8_t> g(gid, gid + n);
    for (size_t q = 0; q < n; ++q) {
        if (g[q] != 255 && g[q] >= ng) return set_err(c, FX_ERR_INVALID_ARGUMENT, "grain id out of range");
        const bool in = g[q] != 255;
        c->tphase[q] = in ? (gtph[g[q]] ? 1.0 : 0.0) : 0.0;
        for (int d = 0; d < 3; ++d) c->ang[d][q] = in ? ang[3 * g[q] + d] : 0.0;
    }
    try {
        build_codes(c);
        std::string w = check_wrapped_mask(c);
        if (!w.empty()) return set_err(c, FX_ERR_UNSUPPORTED, w);
        c->gid = g;
        build_variants(c, &c->gid, c->galpha.empty() ? nullptr : &c->galpha);
    } catch (FxError& e) {
        return set_err(c, e.code, e.msg);
    }
    c->grains_set = true;
    c->ngrains = ng;
    ++c->gen;
    if (!c->user_P) build_P0(c);
    else for (size_t q = 0; q < n; ++q) if (c->tphase[q] == 1.0) c->P0[2][q] = 0.0;
    return FX_OK;
}

int fx_set_grain_alpha(fx_ctx* c, const double* alpha, int ng) {
    if (!c || !alpha || ng <= 0) return FX_ERR_INVALID_ARGUMENT;
    if (!c->grains_set) return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_set_grains must come first");
    ++c->gen;
    c->hist_valid = false;
    c->galpha.assign(alpha, alpha + ng);
    try {
        build_variants(c, &c->gid, &c->galpha);
    } catch (FxError& e) {
        return set_err(c, e.code, e.msg);
    }
    if (c->dev) {
        cudaFree(c->d_vt);
        c->d_vt = nullptr;
        int r = dmalloc(c, &c->d_vt, c->variants.size());
        if (r) return r;
        FX_CUDA(c, cudaMemcpy(c->d_var, c->var.data(), c->N, cudaMemcpyHostToDevice));
        FX_CUDA(c, cudaMemcpy(c->d_vt, c->variants.data(), c->variants.size() * sizeof(Variant), cudaMemcpyHostToDevice));
    }
    return FX_OK;
}

int fx_get_field(fx_ctx* c, int f, double* out, size_t n) {
    if (!c || !out) return FX_ERR_INVALID_ARGUMENT;
    if (f < 0 || f >= FX_NFIELDS) return set_err(c, FX_ERR_INVALID_ARGUMENT, "unknown field id");
    if (n != c->N) return set_err(c, FX_ERR_INVALID_ARGUMENT, "field buffers hold nx*ny*nz values");
    return get_field(c, f, out);
}

int fx_set_field(fx_ctx* c, int f, const double* in, size_t n) {
    if (!c || !in) return FX_ERR_INVALID_ARGUMENT;
    if (n != c->N) return set_err(c, FX_ERR_INVALID_ARGUMENT, "field buffers hold nx*ny*nz values");
    if (f != FX_FIELD_PX && f != FX_FIELD_PY && f != FX_FIELD_PZ && f != FX_FIELD_PHI)
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "only Px, Py, Pz and Phi can be set");
    bool nonzero_xy = false;
    if ((f == FX_FIELD_PX || f == FX_FIELD_PY) && c->scalarP) {
        for (size_t q = 0; q < n; ++q) if (in[q] != 0.0) { nonzero_xy = true; break; }
        if (nonzero_xy && c->dev)
            return set_err(c, FX_ERR_INVALID_ARGUMENT, "nonzero Px/Py must be set before the first device call");
    }
    ++c->gen; c->hist_valid = false;
    if (f == FX_FIELD_PX || f == FX_FIELD_PY || f == FX_FIELD_PZ) {
        if (nonzero_xy) c->scalarP = false;
        if (!c->dev) { c->P0[f].assign(in, in + n); c->user_P = true; return FX_OK; }
        FX_CUDA(c, cudaMemcpyAsync(c->d_P[c->cur][f], in, n * 8, cudaMemcpyHostToDevice, c->s));
        // both ping-pong buffers: cells the TDGL update leaves alone are read
        // from either
        FX_CUDA(c, cudaMemcpyAsync(c->d_P[1 - c->cur][f], c->d_P[c->cur][f], n * 8, cudaMemcpyDeviceToDevice, c->s));
        FX_CUDA(c, cudaStreamSynchronize(c->s));
        c->E_valid = false;
        return FX_OK;
    }
    if (f == FX_FIELD_PHI) {
        if (c->dev) { int r = carriers_now(c); if (r) return r; }
        int r = ensure_device(c);
        if (r) return r;
        FX_CUDA(c, cudaMemcpyAsync(c->d_phi, in, n * 8, cudaMemcpyHostToDevice, c->s));
        if (c->eb_nz > 0) {
            // the cells covered by an embedded boundary are not unknowns of the
            // solve, which never writes them: they hold the 0 each solve of the
            // reference starts from (ElectrostaticSolver.cpp:787)
            const size_t n0 = c->nxy * (size_t)c->eb_nz;
            FX_CUDA(c, cudaMemsetAsync(c->d_phi + n0, 0, (c->N - n0) * 8, c->s));
        }
        FX_CUDA(c, cudaStreamSynchronize(c->s));
        c->E_valid = false;
        return FX_OK;
    }
    return set_err(c, FX_ERR_INVALID_ARGUMENT, "only Px, Py, Pz and Phi can be set");
}

int fx_compute_poisson_rhs(fx_ctx* c) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    ++c->gen; c->hist_valid = false;
    int r = ensure_device(c);
    if (r) return r;
    r = compute_rhs_p(c, false, c->cur);
    if (r) return r;
    if (c->contains_sc) {
        // SC cells take rho (ElectrostaticSolver.cpp:65-67): the Newton kernel
        // with alpha forced to zero is not the reference's RHS, so combine here
        FX_CUDA(c, cudaMemsetAsync(c->d_out, 0, 2 * sizeof(double), c->s));
        DevParams q = c->dp;
        q.delta = 0.0; q.inv_delta = 0.0; q.neg_inv_delta = 0.0;
        ++g_launches;
        r = k_status(c, launch_newton(q, c->d_code, c->d_phi, c->d_rho, c->d_rhsP, c->d_alpha, c->d_alpha32, c->d_rhs,
                                      c->d_out, c->s));
        if (r) return r;
        c->rhs_is_newton = true;
    } else {
        c->rhs_is_newton = false;
    }
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    return FX_OK;
}

int fx_compute_rho(fx_ctx* c) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    ++c->gen; c->hist_valid = false;
    int r = ensure_device(c);
    if (r) return r;
    ++g_launches;
    c->carriers_stale = false;
    r = k_status(c, launch_rho(c->dp, c->d_code, c->d_phi, c->d_phi_prev, c->d_rho, c->d_e, c->d_h, c->d_part,
                               c->d_counter, c->d_out, 0, 1, c->s));
    if (r) return r;
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    return FX_OK;
}

int fx_compute_phi_rho(fx_ctx* c) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    ++c->gen; c->hist_valid = false;
    return compute_phi_rho(c);
}

int fx_compute_E(fx_ctx* c) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    c->E_valid = false;
    int r = materialize_E(c);
    if (r) return r;
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    return FX_OK;
}

int fx_tdgl_euler(fx_ctx* c) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    ++c->gen; c->hist_valid = false;
    int r = tdgl_update(c);
    if (r) return r;
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    return FX_OK;
}

int fx_set_phi_bc(fx_ctx* c) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    ++c->gen; c->hist_valid = false;
    electrode_values(c);
    c->E_valid = false;
    return FX_OK;
}

int fx_check_steady_state(fx_ctx* c, int step) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    return check_steady(c, step);
}

int fx_step(fx_ctx* c, int nsteps, int* done) {
    if (!c || nsteps < 0) return FX_ERR_INVALID_ARGUMENT;
    ++c->gen;
    int k = 0;
    if (done) *done = 0;
    for (; k < nsteps && !c->finished; ++k) {
        int r = step_once(c);
        if (r < 0) { if (done) *done = k; return r; }
        if (done) *done = k + 1;
        if (r == 1) break;
    }
    return FX_OK;
}

int fx_write_plotfile(fx_ctx* c, int step, const char* dir) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    const Params& p = c->par;
    std::vector<std::string> names = {"Px", "Py", "Pz"};
    std::vector<int> ids = {FX_FIELD_PX, FX_FIELD_PY, FX_FIELD_PZ};
    auto add = [&](int flag, const char* nm, int id) { if (flag) { names.push_back(nm); ids.push_back(id); } };
    add(p.plot_Phi, "Phi", FX_FIELD_PHI);
    add(p.plot_PoissonRHS, "PoissonRHS", FX_FIELD_POISSON_RHS);
    if (p.plot_E) { names.insert(names.end(), {"Ex", "Ey", "Ez"}); ids.insert(ids.end(), {FX_FIELD_EX, FX_FIELD_EY, FX_FIELD_EZ}); }
    add(p.plot_holes, "holes", FX_FIELD_HOLES);
    add(p.plot_electrons, "electrons", FX_FIELD_ELECTRONS);
    add(p.plot_charge, "charge", FX_FIELD_CHARGE);
    add(p.plot_epsilon, "epsilon", FX_FIELD_EPSILON);
    add(p.plot_mask, "mask", FX_FIELD_MASK);
    add(p.plot_tphase, "tphase", FX_FIELD_TPHASE);
    add(p.plot_alpha, "alpha", FX_FIELD_ANGLE_ALPHA);
    add(p.plot_beta, "beta", FX_FIELD_ANGLE_BETA);
    add(p.plot_theta, "theta", FX_FIELD_ANGLE_THETA);
    add(p.plot_PhiDiff, "PhiDiff", FX_FIELD_PHIDIFF);
    std::vector<std::vector<double>> data(ids.size(), std::vector<double>(c->N));
    std::vector<const double*> ptr;
    for (size_t q = 0; q < ids.size(); ++q) {
        int r = get_field(c, ids[q], data[q].data());
        if (r) return r;
        ptr.push_back(data[q].data());
    }
    PlotGeom g;
    for (int d = 0; d < 3; ++d) { g.n[d] = p.n_cell[d]; g.prob_lo[d] = p.prob_lo[d]; g.prob_hi[d] = p.prob_hi[d]; g.dx[d] = c->dx[d]; }
    g.time = c->time;
    g.step = step;
    std::string base = dir ? dir : p.plot_dir;
    std::string e;
    if (write_plotfile(base + "/" + plotfile_name(step), g, names, ptr, &e)) return set_err(c, FX_ERR_IO, e);
    return FX_OK;
}

int fx_run(fx_ctx* c, int* done) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    ++c->gen;
    const Params& p = c->par;
    if (done) *done = 0;
    if (p.plot_int > 0 && c->step == 0) {
        int r = fx_write_plotfile(c, 0, nullptr);
        if (r) return r;
    }
    while (c->step < p.nsteps && !c->finished) {
        auto t0 = std::chrono::steady_clock::now();
        int r = step_once(c);
        if (r < 0) return r;
        if (p.verbose) {
            FX_CUDA(c, cudaStreamSynchronize(c->s));
            double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            printf("Advanced step %d in %g seconds\n \n", c->step, sec);
        }
        if (done) *done = c->step;
        if (p.plot_int > 0 && (c->step % p.plot_int == 0 || c->step == c->steady_state_step)) {
            int w = fx_write_plotfile(c, c->step, nullptr);
            if (w) return w;
        }
        if (r == 1) break;
    }
    return FX_OK;
}

int fx_get_stats(const fx_ctx* c, fx_stats* o) {
    if (!c || !o) return FX_ERR_INVALID_ARGUMENT;
    o->step = c->step;
    o->finished = c->finished;
    o->newton_iters_last = c->newton_last;
    o->mg_cycles_last = c->mg_last;
    o->newton_iters_total = c->newton_total;
    o->mg_cycles_total = c->mg_total;
    o->kernel_launches = g_launches.load();
    o->mg_resid_last = c->mg_resid_last;
    o->mg_target_last = c->mg_target_last;
    o->phi_err_last = c->phi_err_last;
    o->steady_err_last = c->steady_err_last;
    o->Phi_Bc_hi = c->Phi_Bc_hi;
    o->time = c->time;
    o->steady_state_step = c->steady_state_step;
    o->inc_step = c->inc_step;
    o->num_Vapp = c->num_Vapp;
    o->sign = c->sign;
    o->device_bytes = (double)c->dev_bytes;
    return FX_OK;
}

int fx_mean_P(fx_ctx* c, double out[3]) {
    if (!c || !out) return FX_ERR_INVALID_ARGUMENT;
    int r = ensure_device(c);
    if (r) return r;
    const double* P[3];
    P_in(c, P);
    ++g_launches;
    r = k_status(c, launch_mean_p(c->dp, c->d_code, P, c->d_part, c->d_counter, c->d_out, c->s));
    if (r) return r;
    r = read_out(c, 3);
    if (r) return r;
    for (int q = 0; q < 3; ++q) out[q] = c->h_out[q];
    return FX_OK;
}

int fx_set_stream(fx_ctx* c, void* stream) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    if (c->dev) {
        FX_CUDA(c, cudaStreamSynchronize(c->s));
        if (c->own_stream) cudaStreamDestroy(c->s);
    }
    c->s = (cudaStream_t)stream;
    c->own_stream = false;
    // stream capture is not permitted on the legacy default stream
    if (stream == nullptr || stream == (void*)cudaStreamLegacy) c->mg.set_graphs(false);
    return FX_OK;
}

int fx_get_kernel_times(fx_ctx* c, double* ms, long long* counts, int n) {
    if (!c || !ms || !counts || n <= 0) return FX_ERR_INVALID_ARGUMENT;
    if (c->dev) FX_CUDA(c, cudaStreamSynchronize(c->s));
    c->prof.collect();
    for (int q = 0; q < n && q < PROF_NCAT; ++q) { ms[q] = c->prof.ms[q]; counts[q] = c->prof.cnt[q]; }
    for (int q = PROF_NCAT; q < n; ++q) { ms[q] = 0; counts[q] = 0; }
    return PROF_NCAT;
}

int fx_reset_kernel_times(fx_ctx* c) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    if (c->dev) FX_CUDA(c, cudaStreamSynchronize(c->s));
    c->prof.collect();
    c->prof.reset();
    return FX_OK;
}

int fx_forward_record(fx_ctx* c, const fx_loss_spec* sp, double* loss) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    if (!sp || !loss || sp->nsteps < 1 || sp->checkpoint_every < 1 || !sp->target)
        return set_err(c, FX_ERR_INVALID_ARGUMENT,
                       "fx_forward_record: spec and loss are required, with nsteps >= 1, checkpoint_every >= 1 and a target");
    if (c->par.TimeIntegratorOrder != 1)
        return set_err(c, FX_ERR_UNSUPPORTED, "gradients are implemented for TimeIntegratorOrder = 1");
    if (c->nx < 6 || c->ny < 6)
        return set_err(c, FX_ERR_UNSUPPORTED, "gradients need at least 6 cells in x and y");
    for (int n = 0; n < sp->nsteps; ++n)
        if (!std::isfinite(sp->target[n]) || (sp->v_shape && !std::isfinite(sp->v_shape[n])))
            return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_forward_record: non-finite target or v_shape");
    if (!std::isfinite(sp->v_amp)) return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_forward_record: non-finite v_amp");
    ++c->gen;
    c->hist_valid = false;
    const int r = forward_record(c, sp, loss);
    if (r) c->adj.valid = false;
    return r;
}

int fx_backward(fx_ctx* c, double* grads, int ngrads) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    if (!grads || ngrads < FX_GRAD_GRAIN_ALPHA)
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_backward: grads needs at least 6 slots");
    if (!c->adj.valid) return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_backward: no fx_forward_record to differentiate");
    if (c->adj.gen != c->gen)
        return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_backward: the context changed since fx_forward_record");
    c->hist_valid = false;
    const int r = backward(c, grads, ngrads);
    if (r) {
        c->adj.valid = false;
        c->adj.have_P0 = false;
    }
    return r;
}

int fx_get_grad_P0(fx_ctx* c, double* dPx, double* dPy, double* dPz, size_t n) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    if (n != c->N) return set_err(c, FX_ERR_INVALID_ARGUMENT, "field buffers hold nx*ny*nz values");
    if (!c->adj.have_P0) return set_err(c, FX_ERR_INVALID_ARGUMENT, "fx_get_grad_P0: call fx_backward first");
    if (c->scalarP && (dPx || dPy))
        return set_err(c, FX_ERR_UNSUPPORTED, "scalar polarization: only dPz is available (pass NULL for dPx, dPy)");
    double* out[3] = {dPx, dPy, dPz};
    for (int d = 0; d < 3; ++d)
        if (out[d]) FX_CUDA(c, cudaMemcpyAsync(out[d], c->adj.lam[c->adj.lcur][d], n * 8, cudaMemcpyDeviceToHost, c->s));
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    return FX_OK;
}

int fx_sync(fx_ctx* c) {
    if (!c) return FX_ERR_INVALID_ARGUMENT;
    if (!c->dev) return FX_OK;
    FX_CUDA(c, cudaStreamSynchronize(c->s));
    return FX_OK;
}

}  // extern "C"
