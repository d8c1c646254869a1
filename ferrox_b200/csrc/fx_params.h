// fx_params.h -- host-side parameters of one FerroX run (inputs-file keys).
//
// The key names, meanings and defaults follow InitializeFerroXNamespace
// (Source/FerroX.cpp:273-572) and c_GeometryProperties::ParseBasicDomainInput
// (Source/Input/GeometryProperties/GeometryProperties.cpp:86-173); the fx.*
// keys are this library's extensions.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace fx {

struct Params {
    int n_cell[3] = {0, 0, 0};
    double prob_lo[3] = {0, 0, 0}, prob_hi[3] = {0, 0, 0};
    int is_periodic[3] = {0, 0, 0};
    std::string bc_lo[3], bc_hi[3];          // boundary.lo / boundary.hi tokens

    int prob_type = 2, TimeIntegratorOrder = 1, nsteps = 10, plot_int = -1;
    double dt = 0;
    int P_BC_flag_lo[3] = {0, 0, 0}, P_BC_flag_hi[3] = {0, 0, 0};
    double lambda = 0;

    double epsilon_0 = 0, epsilonX_fe = 0, epsilonX_fe_tphase = 0, epsilonZ_fe = 0, epsilon_de = 0, epsilon_si = 0;
    double alpha = 0, beta = 0, gamma = 0, alpha_12 = 0, alpha_112 = 0, alpha_123 = 0;
    double BigGamma = 0, g11 = 0, g44 = 0, g12 = 0, g44_p = 0;

    double FE_lo[3], FE_hi[3], DE_lo[3], DE_hi[3], SC_lo[3], SC_hi[3], Channel_lo[3], Channel_hi[3];
    double Remnant_P[3] = {0.0, 0.0, 0.002};

    double acceptor_doping = 0, donor_doping = 0;
    int use_Fermi_Dirac = 1, use_work_function = 0;
    double metal_work_function = 0;

    int is_polarization_scalar = 1;
    double delta = 1e-6;
    int voltage_sweep = 0, inc_step = -1;
    double Phi_Bc_lo = 0, Phi_Bc_hi = 0, Phi_Bc_inc = 0, Phi_Bc_hi_max = 0, phi_tolerance = 1e-7;
    int num_Vapp_max = 1, random_seed = 1;
    int include_Landau = 1, include_Grad = 1, include_Elec = 1;
    int Coordinate_Transformation = 0, use_Euler_angles = 0;
    int mlmg_verbosity = 1;
    int plot_Phi = 1, plot_PoissonRHS = 1, plot_E = 1, plot_holes = 1, plot_electrons = 1, plot_charge = 1,
        plot_epsilon = 1, plot_mask = 1, plot_tphase = 1, plot_alpha = 1, plot_beta = 1, plot_theta = 1,
        plot_PhiDiff = 1;

    // fx.* extensions
    double mg_rtol = 1e-10;
    int phi_ghost_mode = 0;      // 0 extrap, 1 face, 2 zero
    int sweep_mode = 0;          // 0 steady (reference), 1 fixed cadence
    int steps_per_voltage = 0;
    int newton_max_iter = 50;
    double newton_tol = 1.e-5;      // Newton stopping criterion (ElectrostaticSolver.cpp:697)
    int mg_max_iter = 200;
    int precision = 0;           // 0 fp64, 1 mixed
    int warm_start = 1;
    int phi_extrapolate = 4;       // first solve of a step starts from phi extrapolated in time (order 0-6)
    int step_graph = 1;            // a step runs as one CUDA graph with its loop tests on the device
    int verbose = 0;
    std::string plot_dir = ".";
    // input files (raw formats in include/ferrox_b200.h): the initial P, and
    // the grains of a polycrystal (per-cell grain id, per-grain Euler angles
    // and t-phase flag)
    std::string initial_P_file, grain_file;
};

// Expression over x, y, z (and my_constants) from a function-valued key.
class Expr {
public:
    virtual ~Expr() = default;
    virtual double eval(double x, double y, double z) const = 0;
};

struct Inputs {
    std::map<std::string, std::vector<std::string>> table;   // last definition wins
    std::map<std::string, double> constants;                 // my_constants.* and pi
};

// Parse inputs text; throws std::runtime_error with a message on bad input.
Inputs parse_inputs(const std::string& text);
Params make_params(const Inputs& in);
std::unique_ptr<Expr> compile_expr(const std::string& text, const std::map<std::string, double>& constants);
double eval_number(const std::string& tok, const std::map<std::string, double>& constants);

}  // namespace fx
