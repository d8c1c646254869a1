// inputs.cpp -- FerroX inputs-file reader (host, setup only).
//
// Restates the subset of AMReX ParmParse that FerroX decks use: "key = v1 v2"
// lines, '#' comments, double-quoted strings that may span lines, and the
// last definition of a key winning for get/query.  Defaults follow
// InitializeFerroXNamespace (Source/FerroX.cpp:273-572) and
// ParseBasicDomainInput (GeometryProperties.cpp:86-173).  Function-valued keys
// go through a small expression compiler covering the AMReX Parser grammar the
// example decks use (WarpXUtil.cpp:101-165 feeds my_constants into it).
#include "fx_params.h"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <stdexcept>

namespace fx {

namespace {

std::vector<std::string> tokenize(const std::string& t) {
    std::vector<std::string> toks;
    std::string cur;
    size_t i = 0, n = t.size();
    auto flush = [&]() { if (!cur.empty()) { toks.push_back(cur); cur.clear(); } };
    while (i < n) {
        char ch = t[i];
        if (ch == '"') {
            size_t j = t.find('"', i + 1);
            if (j == std::string::npos) throw std::runtime_error("inputs: unterminated string");
            flush();
            toks.push_back(t.substr(i, j - i + 1));
            i = j + 1;
        } else if (ch == '#') {
            while (i < n && t[i] != '\n') ++i;
        } else if (ch == '=') {
            flush();
            toks.push_back("=");
            ++i;
        } else if (std::isspace((unsigned char)ch)) {
            flush();
            ++i;
        } else {
            cur += ch;
            ++i;
        }
    }
    flush();
    return toks;
}

// ------------------------------------------------------------ expressions --
struct Node : Expr {
    enum K { NUM, VX, VY, VZ, ADD, SUB, MUL, DIV, POW, NEG, LT, GT, LE, GE, EQ, NE, AND, OR, CALL1, CALL2, IF } k;
    double v = 0;
    std::unique_ptr<Node> a, b, c;
    double (*f1)(double) = nullptr;
    double (*f2)(double, double) = nullptr;
    double eval(double x, double y, double z) const override {
        switch (k) {
        case NUM: return v;
        case VX: return x;
        case VY: return y;
        case VZ: return z;
        case ADD: return a->eval(x, y, z) + b->eval(x, y, z);
        case SUB: return a->eval(x, y, z) - b->eval(x, y, z);
        case MUL: return a->eval(x, y, z) * b->eval(x, y, z);
        case DIV: return a->eval(x, y, z) / b->eval(x, y, z);
        case POW: return std::pow(a->eval(x, y, z), b->eval(x, y, z));
        case NEG: return -a->eval(x, y, z);
        case LT: return a->eval(x, y, z) < b->eval(x, y, z) ? 1.0 : 0.0;
        case GT: return a->eval(x, y, z) > b->eval(x, y, z) ? 1.0 : 0.0;
        case LE: return a->eval(x, y, z) <= b->eval(x, y, z) ? 1.0 : 0.0;
        case GE: return a->eval(x, y, z) >= b->eval(x, y, z) ? 1.0 : 0.0;
        case EQ: return a->eval(x, y, z) == b->eval(x, y, z) ? 1.0 : 0.0;
        case NE: return a->eval(x, y, z) != b->eval(x, y, z) ? 1.0 : 0.0;
        case AND: return (a->eval(x, y, z) != 0.0 && b->eval(x, y, z) != 0.0) ? 1.0 : 0.0;
        case OR: return (a->eval(x, y, z) != 0.0 || b->eval(x, y, z) != 0.0) ? 1.0 : 0.0;
        case CALL1: return f1(a->eval(x, y, z));
        case CALL2: return f2(a->eval(x, y, z), b->eval(x, y, z));
        case IF: return a->eval(x, y, z) != 0.0 ? b->eval(x, y, z) : c->eval(x, y, z);
        }
        return 0.0;
    }
};

double f_abs(double a) { return std::fabs(a); }
double f_min(double a, double b) { return a < b ? a : b; }
double f_max(double a, double b) { return a > b ? a : b; }
double f_heav(double a, double h0) { return a > 0 ? 1.0 : (a < 0 ? 0.0 : h0); }

class ExprParser {
public:
    ExprParser(const std::string& s, const std::map<std::string, double>& c) : s_(s), c_(c) {}
    std::unique_ptr<Node> parse() {
        auto n = p_or();
        skip();
        if (pos_ != s_.size()) fail("unexpected '" + s_.substr(pos_, 8) + "'");
        return n;
    }

private:
    const std::string& s_;
    const std::map<std::string, double>& c_;
    size_t pos_ = 0;

    [[noreturn]] void fail(const std::string& m) { throw std::runtime_error("inputs: expression \"" + s_ + "\": " + m); }
    void skip() { while (pos_ < s_.size() && std::isspace((unsigned char)s_[pos_])) ++pos_; }
    bool eat(const char* t) {
        skip();
        size_t L = std::strlen(t);
        if (s_.compare(pos_, L, t) == 0) {
            // keywords must not be followed by an identifier character
            if (std::isalpha((unsigned char)t[0]) && pos_ + L < s_.size() && (std::isalnum((unsigned char)s_[pos_ + L]) || s_[pos_ + L] == '_'))
                return false;
            pos_ += L;
            return true;
        }
        return false;
    }
    static std::unique_ptr<Node> mk(Node::K k, std::unique_ptr<Node> a, std::unique_ptr<Node> b = nullptr) {
        auto n = std::make_unique<Node>();
        n->k = k; n->a = std::move(a); n->b = std::move(b);
        return n;
    }
    std::unique_ptr<Node> p_or() {
        auto l = p_and();
        while (eat("||") || eat("or")) l = mk(Node::OR, std::move(l), p_and());
        return l;
    }
    std::unique_ptr<Node> p_and() {
        auto l = p_cmp();
        while (eat("&&") || eat("and")) l = mk(Node::AND, std::move(l), p_cmp());
        return l;
    }
    std::unique_ptr<Node> p_cmp() {
        auto l = p_add();
        while (true) {
            if (eat("<=")) l = mk(Node::LE, std::move(l), p_add());
            else if (eat(">=")) l = mk(Node::GE, std::move(l), p_add());
            else if (eat("==")) l = mk(Node::EQ, std::move(l), p_add());
            else if (eat("!=")) l = mk(Node::NE, std::move(l), p_add());
            else if (eat("<")) l = mk(Node::LT, std::move(l), p_add());
            else if (eat(">")) l = mk(Node::GT, std::move(l), p_add());
            else return l;
        }
    }
    std::unique_ptr<Node> p_add() {
        auto l = p_mul();
        while (true) {
            if (eat("+")) l = mk(Node::ADD, std::move(l), p_mul());
            else if (eat("-")) l = mk(Node::SUB, std::move(l), p_mul());
            else return l;
        }
    }
    std::unique_ptr<Node> p_mul() {
        auto l = p_unary();
        while (true) {
            skip();
            if (s_.compare(pos_, 2, "**") == 0) return l;   // handled by p_pow
            if (eat("*")) l = mk(Node::MUL, std::move(l), p_unary());
            else if (eat("/")) l = mk(Node::DIV, std::move(l), p_unary());
            else return l;
        }
    }
    std::unique_ptr<Node> p_unary() {
        if (eat("-")) return mk(Node::NEG, p_unary());
        if (eat("+")) return p_unary();
        return p_pow();
    }
    std::unique_ptr<Node> p_pow() {
        auto b = p_primary();
        if (eat("**") || eat("^")) return mk(Node::POW, std::move(b), p_unary());
        return b;
    }
    std::unique_ptr<Node> p_primary() {
        skip();
        if (pos_ >= s_.size()) fail("unexpected end");
        char ch = s_[pos_];
        if (ch == '(') {
            ++pos_;
            auto e = p_or();
            if (!eat(")")) fail("missing ')'");
            return e;
        }
        if (std::isdigit((unsigned char)ch) || ch == '.') {
            const char* b = s_.c_str() + pos_;
            char* e = nullptr;
            double v = std::strtod(b, &e);
            if (e == b) fail("bad number");
            pos_ += (size_t)(e - b);
            auto n = std::make_unique<Node>();
            n->k = Node::NUM; n->v = v;
            return n;
        }
        if (std::isalpha((unsigned char)ch) || ch == '_') {
            size_t b = pos_;
            while (pos_ < s_.size() && (std::isalnum((unsigned char)s_[pos_]) || s_[pos_] == '_')) ++pos_;
            std::string id = s_.substr(b, pos_ - b);
            skip();
            if (pos_ < s_.size() && s_[pos_] == '(') {
                ++pos_;
                std::vector<std::unique_ptr<Node>> args;
                skip();
                if (!eat(")")) {
                    do { args.push_back(p_or()); } while (eat(","));
                    if (!eat(")")) fail("missing ')' after arguments of " + id);
                }
                return call(id, std::move(args));
            }
            auto n = std::make_unique<Node>();
            if (id == "x") n->k = Node::VX;
            else if (id == "y") n->k = Node::VY;
            else if (id == "z") n->k = Node::VZ;
            else {
                auto it = c_.find(id);
                if (it == c_.end()) fail("unknown symbol '" + id + "'");
                n->k = Node::NUM; n->v = it->second;
            }
            return n;
        }
        fail(std::string("unexpected character '") + ch + "'");
    }
    std::unique_ptr<Node> call(const std::string& id, std::vector<std::unique_ptr<Node>> args) {
        static const std::map<std::string, double (*)(double)> f1 = {
            {"sin", ::sin}, {"cos", ::cos}, {"tan", ::tan}, {"asin", ::asin}, {"acos", ::acos}, {"atan", ::atan},
            {"sinh", ::sinh}, {"cosh", ::cosh}, {"tanh", ::tanh}, {"exp", ::exp}, {"log", ::log}, {"log10", ::log10},
            {"sqrt", ::sqrt}, {"abs", f_abs}, {"fabs", f_abs}, {"floor", ::floor}, {"ceil", ::ceil}};
        static const std::map<std::string, double (*)(double, double)> f2 = {
            {"atan2", ::atan2}, {"pow", ::pow}, {"min", f_min}, {"max", f_max}, {"heaviside", f_heav}};
        auto n = std::make_unique<Node>();
        if (id == "if") {
            if (args.size() != 3) fail("if() takes 3 arguments");
            n->k = Node::IF; n->a = std::move(args[0]); n->b = std::move(args[1]); n->c = std::move(args[2]);
            return n;
        }
        auto i1 = f1.find(id);
        if (i1 != f1.end()) {
            if (args.size() != 1) fail(id + "() takes 1 argument");
            n->k = Node::CALL1; n->f1 = i1->second; n->a = std::move(args[0]);
            return n;
        }
        auto i2 = f2.find(id);
        if (i2 != f2.end()) {
            if (args.size() != 2) fail(id + "() takes 2 arguments");
            n->k = Node::CALL2; n->f2 = i2->second; n->a = std::move(args[0]); n->b = std::move(args[1]);
            return n;
        }
        fail("unknown function '" + id + "'");
    }
};

}  // namespace

std::unique_ptr<Expr> compile_expr(const std::string& text, const std::map<std::string, double>& constants) {
    ExprParser p(text, constants);
    return p.parse();
}

double eval_number(const std::string& tok, const std::map<std::string, double>& constants) {
    const char* b = tok.c_str();
    char* e = nullptr;
    double v = std::strtod(b, &e);
    if (e != b && *e == '\0') return v;
    return compile_expr(tok, constants)->eval(0, 0, 0);
}

Inputs parse_inputs(const std::string& text) {
    Inputs in;
    auto toks = tokenize(text);
    size_t i = 0;
    while (i < toks.size()) {
        if (i + 1 < toks.size() && toks[i + 1] == "=") {
            std::string key = toks[i];
            size_t j = i + 2;
            std::vector<std::string> vals;
            while (j < toks.size() && !(j + 1 < toks.size() && toks[j + 1] == "=")) {
                std::string v = toks[j];
                if (v.size() >= 2 && v.front() == '"' && v.back() == '"') v = v.substr(1, v.size() - 2);
                vals.push_back(v);
                ++j;
            }
            in.table[key] = vals;
            i = j;
        } else {
            throw std::runtime_error("inputs: unexpected token '" + toks[i] + "'");
        }
    }
    // my_constants.* may refer to each other; resolve in passes
    in.constants["pi"] = 3.14159265358979323846;
    std::map<std::string, std::string> pending;
    for (auto& kv : in.table)
        if (kv.first.rfind("my_constants.", 0) == 0 && !kv.second.empty()) {
            std::string all;
            for (auto& s : kv.second) all += (all.empty() ? "" : " ") + s;
            pending[kv.first.substr(13)] = all;
        }
    for (size_t pass = 0; pass <= pending.size() && !pending.empty(); ++pass) {
        for (auto it = pending.begin(); it != pending.end();) {
            try {
                in.constants[it->first] = eval_number(it->second, in.constants);
                it = pending.erase(it);
            } catch (std::runtime_error&) {
                ++it;
            }
        }
    }
    if (!pending.empty()) throw std::runtime_error("inputs: unresolved my_constants." + pending.begin()->first);
    return in;
}

namespace {

struct Reader {
    const Inputs& in;
    bool has(const std::string& k) const { return in.table.count(k) && !in.table.at(k).empty(); }
    const std::vector<std::string>& vals(const std::string& k) const { return in.table.at(k); }
    double num(const std::string& k) const {
        if (!has(k)) throw std::runtime_error("inputs: required key '" + k + "' missing");
        return eval_number(vals(k)[0], in.constants);
    }
    int inum(const std::string& k) const {
        double v = num(k);
        if (v != std::floor(v)) throw std::runtime_error("inputs: key '" + k + "' must be an integer");
        return (int)v;
    }
    void query(const std::string& k, double& v) const { if (has(k)) v = num(k); }
    void query(const std::string& k, int& v) const { if (has(k)) v = inum(k); }
    bool queryarr(const std::string& k, double* v) const {
        if (!has(k)) return false;
        if (vals(k).size() < 3) throw std::runtime_error("inputs: key '" + k + "' needs 3 values");
        for (int d = 0; d < 3; ++d) v[d] = eval_number(vals(k)[d], in.constants);
        return true;
    }
    bool queryarr(const std::string& k, int* v) const {
        if (!has(k)) return false;
        if (vals(k).size() < 3) throw std::runtime_error("inputs: key '" + k + "' needs 3 values");
        for (int d = 0; d < 3; ++d) {
            double x = eval_number(vals(k)[d], in.constants);
            if (x != std::floor(x)) throw std::runtime_error("inputs: key '" + k + "' must hold integers");
            v[d] = (int)x;
        }
        return true;
    }
    void getarr(const std::string& k, double* v) const {
        if (!queryarr(k, v)) throw std::runtime_error("inputs: required key '" + k + "' missing");
    }
};

}  // namespace

Params make_params(const Inputs& in) {
    Reader r{in};
    Params p;
    // domain (GeometryProperties.cpp:105-124)
    if (!r.queryarr("domain.n_cell", p.n_cell)) throw std::runtime_error("inputs: required key 'domain.n_cell' missing");
    r.getarr("domain.prob_lo", p.prob_lo);
    r.getarr("domain.prob_hi", p.prob_hi);
    r.queryarr("domain.is_periodic", p.is_periodic);
    for (int d = 0; d < 3; ++d) {
        if (p.n_cell[d] < 1) throw std::runtime_error("inputs: domain.n_cell must be positive");
        if (!(p.prob_hi[d] > p.prob_lo[d])) throw std::runtime_error("inputs: domain.prob_hi must exceed domain.prob_lo");
    }
    // boundary.lo / boundary.hi (BoundaryConditions.cpp:136-157)
    for (int side = 0; side < 2; ++side) {
        std::string key = side ? "boundary.hi" : "boundary.lo";
        if (r.has(key)) {
            auto& v = r.vals(key);
            if (v.size() < 3) throw std::runtime_error("inputs: " + key + " needs 3 entries");
            for (int d = 0; d < 3; ++d) {
                std::string t = v[d].substr(0, 3);
                if (t != "per" && t != "dir" && t != "neu") throw std::runtime_error("inputs: " + key + " entry '" + v[d] + "' is not per/dir/neu");
                (side ? p.bc_hi : p.bc_lo)[d] = v[d];
            }
        }
    }

    // InitializeFerroXNamespace, FerroX.cpp:285-571
    r.queryarr("P_BC_flag_lo", p.P_BC_flag_lo);
    r.queryarr("P_BC_flag_hi", p.P_BC_flag_hi);
    r.query("plot_Phi", p.plot_Phi); r.query("plot_PoissonRHS", p.plot_PoissonRHS); r.query("plot_E", p.plot_E);
    r.query("plot_holes", p.plot_holes); r.query("plot_electrons", p.plot_electrons); r.query("plot_charge", p.plot_charge);
    r.query("plot_epsilon", p.plot_epsilon); r.query("plot_mask", p.plot_mask); r.query("plot_tphase", p.plot_tphase);
    r.query("plot_alpha", p.plot_alpha); r.query("plot_beta", p.plot_beta); r.query("plot_theta", p.plot_theta);
    r.query("plot_PhiDiff", p.plot_PhiDiff);
    p.TimeIntegratorOrder = r.inum("TimeIntegratorOrder");
    int use_sundials = 0;
    r.query("use_sundials", use_sundials);
    if (use_sundials) throw std::runtime_error("inputs: use_sundials = 1 is not supported (forward Euler / order 2 only)");
    p.prob_type = r.inum("prob_type");
    r.query("is_polarization_scalar", p.is_polarization_scalar);
    r.query("mlmg_verbosity", p.mlmg_verbosity);
    p.epsilon_0 = r.num("epsilon_0");
    p.epsilonX_fe = r.num("epsilonX_fe");
    p.epsilonX_fe_tphase = p.epsilonX_fe;
    r.query("epsilonX_fe_tphase", p.epsilonX_fe_tphase);
    p.epsilonZ_fe = r.num("epsilonZ_fe");
    p.epsilon_de = r.num("epsilon_de");
    p.epsilon_si = r.num("epsilon_si");
    p.alpha = r.num("alpha"); p.beta = r.num("beta"); p.gamma = r.num("gamma");
    p.alpha_12 = r.num("alpha_12"); p.alpha_112 = r.num("alpha_112"); p.alpha_123 = r.num("alpha_123");
    p.BigGamma = r.num("BigGamma");
    p.g11 = r.num("g11"); p.g44 = r.num("g44"); p.g12 = r.num("g12"); p.g44_p = r.num("g44_p");
    p.lambda = r.num("lambda");
    r.query("nsteps", p.nsteps);
    r.query("plot_int", p.plot_int);
    p.dt = r.num("dt");
    r.query("delta", p.delta);
    r.query("inc_step", p.inc_step);
    r.query("random_seed", p.random_seed);
    r.query("voltage_sweep", p.voltage_sweep);
    r.query("Phi_Bc_hi", p.Phi_Bc_hi);
    r.query("Phi_Bc_lo", p.Phi_Bc_lo);
    r.query("Phi_Bc_inc", p.Phi_Bc_inc);
    r.query("Phi_Bc_hi_max", p.Phi_Bc_hi_max);
    r.query("phi_tolerance", p.phi_tolerance);
    r.query("num_Vapp_max", p.num_Vapp_max);
    r.query("include_Landau", p.include_Landau);
    r.query("include_Grad", p.include_Grad);
    r.query("include_Elec", p.include_Elec);
    for (int d = 0; d < 3; ++d) {
        p.DE_lo[d] = p.SC_lo[d] = p.Channel_lo[d] = p.prob_lo[d] - 1.0;
        p.DE_hi[d] = p.SC_hi[d] = p.Channel_hi[d] = p.prob_hi[d] + 1.0;
    }
    r.getarr("FE_lo", p.FE_lo);
    r.getarr("FE_hi", p.FE_hi);
    r.queryarr("DE_lo", p.DE_lo); r.queryarr("DE_hi", p.DE_hi);
    r.queryarr("SC_lo", p.SC_lo); r.queryarr("SC_hi", p.SC_hi);
    r.queryarr("Channel_lo", p.Channel_lo); r.queryarr("Channel_hi", p.Channel_hi);
    r.queryarr("Remnant_P", p.Remnant_P);
    r.query("acceptor_doping", p.acceptor_doping);
    r.query("donor_doping", p.donor_doping);
    r.query("use_Fermi_Dirac", p.use_Fermi_Dirac);
    r.query("use_work_function", p.use_work_function);
    if (p.use_work_function == 1) {
        p.metal_work_function = 4.85;
        r.query("metal_work_function", p.metal_work_function);
    }
    r.query("Coordinate_Transformation", p.Coordinate_Transformation);
    r.query("use_Euler_angles", p.use_Euler_angles);

    // fx.* extensions
    r.query("fx.mg_rtol", p.mg_rtol);
    if (r.has("fx.phi_ghost_mode")) {
        std::string m = r.vals("fx.phi_ghost_mode")[0];
        if (m == "extrap") p.phi_ghost_mode = 0;
        else if (m == "face") p.phi_ghost_mode = 1;
        else if (m == "zero") p.phi_ghost_mode = 2;
        else throw std::runtime_error("inputs: fx.phi_ghost_mode must be extrap, face or zero");
    }
    if (r.has("fx.sweep_mode")) {
        std::string m = r.vals("fx.sweep_mode")[0];
        if (m == "steady") p.sweep_mode = 0;
        else if (m == "fixed") p.sweep_mode = 1;
        else throw std::runtime_error("inputs: fx.sweep_mode must be steady or fixed");
    }
    r.query("fx.steps_per_voltage", p.steps_per_voltage);
    r.query("fx.newton_max_iter", p.newton_max_iter);
    r.query("fx.newton_tol", p.newton_tol);
    r.query("fx.mg_max_iter", p.mg_max_iter);
    if (r.has("fx.precision")) {
        std::string m = r.vals("fx.precision")[0];
        if (m == "fp64") p.precision = 0;
        else if (m == "mixed") p.precision = 1;
        else throw std::runtime_error("inputs: fx.precision must be fp64 or mixed");
    }
    r.query("fx.warm_start", p.warm_start);
    r.query("fx.phi_extrapolate", p.phi_extrapolate);
    r.query("fx.step_graph", p.step_graph);
    r.query("fx.verbose", p.verbose);
    if (r.has("fx.plot_dir")) p.plot_dir = r.vals("fx.plot_dir")[0];
    if (r.has("fx.initial_P_file")) p.initial_P_file = r.vals("fx.initial_P_file")[0];
    if (r.has("fx.grain_file")) p.grain_file = r.vals("fx.grain_file")[0];

    // validation the reference does by amrex::Abort / assertions
    for (int d = 0; d < 3; ++d)
        if (p.P_BC_flag_lo[d] < 0 || p.P_BC_flag_lo[d] > 4 || p.P_BC_flag_hi[d] < 0 || p.P_BC_flag_hi[d] > 4)
            throw std::runtime_error("inputs: P_BC_flag_lo/hi entries must be 0..4 (DerivativeAlgorithm.H:71-73)");
    if (p.prob_type < 1 || p.prob_type > 3) throw std::runtime_error("inputs: prob_type must be 1, 2 or 3 (Initialization.cpp:37-43)");
    if (p.TimeIntegratorOrder != 1 && p.TimeIntegratorOrder != 2) throw std::runtime_error("inputs: TimeIntegratorOrder must be 1 or 2");
    // the solver settings of this library (fx_set_param applies the same ranges)
    if (p.phi_extrapolate < 0 || p.phi_extrapolate > 6) throw std::runtime_error("inputs: fx.phi_extrapolate must be 0..6");
    if (p.mg_max_iter < 1) throw std::runtime_error("inputs: fx.mg_max_iter must be at least 1");
    if (p.newton_max_iter < 1) throw std::runtime_error("inputs: fx.newton_max_iter must be at least 1");
    if (!(p.mg_rtol > 0.0)) throw std::runtime_error("inputs: fx.mg_rtol must be positive");
    return p;
}

}  // namespace fx
