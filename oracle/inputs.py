"""FerroX inputs-file reader for the oracle (TEST INFRASTRUCTURE ONLY).

A Python restatement of the subset of AMReX ParmParse that FerroX's inputs
decks use (``key = v1 v2 ...``, ``#`` comments, double-quoted strings that may
span lines, the last definition of a key wins), and of the defaults that
``InitializeFerroXNamespace`` (Source/FerroX.cpp:273-572) and
``c_GeometryProperties::ParseBasicDomainInput``
(Source/Input/GeometryProperties/GeometryProperties.cpp:86-173) apply.

Function-valued keys (``tphase_geom.tphase_geom_function(x,y,z)``,
``angle_alpha.alpha_function(x,y,z)``, ...; Initialization.cpp:227-365) are
evaluated with numpy over cell centres.  The AMReX Parser itself is a
third-party component absent from the reference tree; this evaluator covers
the grammar the example decks use (arithmetic, ``^``, comparisons, ``and`` /
``or``, ``if``, ``heaviside``, the usual functions, ``my_constants.*``) with
AMReX Parser's C-like precedence.  With no AMReX Parser to run, it is pinned by
closed-form known answers, not by the parser's own outputs.

The product library has its own C++ reader; tests compare the two.
"""
from __future__ import annotations

import math
import re

import numpy as np

# --------------------------------------------------------------- ParmParse --


def tokenize(text: str) -> list[str]:
    toks: list[str] = []
    i, n = 0, len(text)
    cur = ""
    while i < n:
        ch = text[i]
        if ch == '"':
            j = text.index('"', i + 1)
            if cur:
                toks.append(cur)
                cur = ""
            toks.append(text[i:j + 1])
            i = j + 1
            continue
        if ch == "#":
            while i < n and text[i] != "\n":
                i += 1
            continue
        if ch == "=":
            if cur:
                toks.append(cur)
                cur = ""
            toks.append("=")
            i += 1
            continue
        if ch.isspace():
            if cur:
                toks.append(cur)
                cur = ""
            i += 1
            continue
        cur += ch
        i += 1
    if cur:
        toks.append(cur)
    return toks


def parse_table(text: str) -> dict[str, list[str]]:
    """key -> value tokens of its last definition (quotes stripped)."""
    toks = tokenize(text)
    table: dict[str, list[str]] = {}
    i = 0
    while i < len(toks):
        if i + 1 < len(toks) and toks[i + 1] == "=":
            key = toks[i]
            j = i + 2
            vals = []
            while j < len(toks) and not (j + 1 < len(toks) and toks[j + 1] == "="):
                vals.append(toks[j])
                j += 1
            table[key] = [v[1:-1] if v.startswith('"') else v for v in vals]
            i = j
        else:
            raise ValueError(f"inputs: unexpected token {toks[i]!r}")
    return table


# ---------------------------------------------------------- expressions ----

_FUNCS = {
    "sin": np.sin, "cos": np.cos, "tan": np.tan, "asin": np.arcsin, "acos": np.arccos,
    "atan": np.arctan, "atan2": np.arctan2, "sinh": np.sinh, "cosh": np.cosh, "tanh": np.tanh,
    "exp": np.exp, "log": np.log, "log10": np.log10, "sqrt": np.sqrt, "abs": np.abs,
    "fabs": np.abs, "floor": np.floor, "ceil": np.ceil, "pow": np.power,
    "min": np.minimum, "max": np.maximum,
    "_if": lambda c, a, b: np.where(np.asarray(c) != 0, a, b),
    "heaviside": lambda x, h0=0.0: np.where(np.asarray(x) > 0, 1.0, np.where(np.asarray(x) < 0, 0.0, h0)),
    "_f": lambda v: np.asarray(v, dtype=np.float64),
    "_pow": lambda a, b: np.power(np.asarray(a, dtype=np.float64), b),
    "_and": lambda a, b: np.asarray((np.asarray(a) != 0) & (np.asarray(b) != 0), dtype=np.float64),
    "_or": lambda a, b: np.asarray((np.asarray(a) != 0) | (np.asarray(b) != 0), dtype=np.float64),
}

_EXPR_TOKEN = re.compile(r"\s*(?:(\d+\.?\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?)|([A-Za-z_]\w*)"
                         r"|(\*\*|<=|>=|==|!=|&&|\|\||[-+*/^<>(),]))")


class _ExprToPython:
    """Rewrites an AMReX Parser expression as fully parenthesised numpy code.

    Precedence, loosest first, as in AMReX Parser's C-like grammar:
    ``or ||`` < ``and &&`` < comparisons < ``+ -`` < ``* /`` < unary ``- +``
    < ``^ **`` (right-associative, its exponent may carry a unary sign, so
    ``-2^2 = -4`` and ``2^-1 = 0.5``).  Comparisons and the logical operators
    give 0.0 / 1.0; ``if(c, a, b)`` selects per cell.
    """

    def __init__(self, expr: str):
        self.toks: list[str] = []
        s, pos = expr.strip(), 0
        while pos < len(s):
            m = _EXPR_TOKEN.match(s, pos)
            if m is None or m.end() == pos:
                raise SyntaxError(f"expression {expr!r}: unexpected {s[pos:pos + 8]!r}")
            self.toks.append(m.group(m.lastindex))
            pos = m.end()
        self.i = 0
        self.expr = expr

    def run(self) -> str:
        code = self.p_or()
        if self.i != len(self.toks):
            raise SyntaxError(f"expression {self.expr!r}: unexpected {self.toks[self.i]!r}")
        return code

    def peek(self):
        return self.toks[self.i] if self.i < len(self.toks) else None

    def eat(self, *ops) -> bool:
        if self.peek() in ops:
            self.i += 1
            return True
        return False

    def want(self, op: str) -> None:
        if not self.eat(op):
            raise SyntaxError(f"expression {self.expr!r}: missing {op!r}")

    def p_or(self) -> str:
        a = self.p_and()
        while self.eat("||", "or"):
            a = f"_or({a}, {self.p_and()})"
        return a

    def p_and(self) -> str:
        a = self.p_cmp()
        while self.eat("&&", "and"):
            a = f"_and({a}, {self.p_cmp()})"
        return a

    def p_cmp(self) -> str:
        a = self.p_add()
        while self.peek() in ("<", ">", "<=", ">=", "==", "!="):
            op = self.toks[self.i]
            self.i += 1
            a = f"_f({a} {op} {self.p_add()})"
        return a

    def p_add(self) -> str:
        a = self.p_mul()
        while self.peek() in ("+", "-"):
            op = self.toks[self.i]
            self.i += 1
            a = f"({a} {op} {self.p_mul()})"
        return a

    def p_mul(self) -> str:
        a = self.p_unary()
        while self.peek() in ("*", "/"):
            op = self.toks[self.i]
            self.i += 1
            a = f"({a} {op} {self.p_unary()})"
        return a

    def p_unary(self) -> str:
        if self.eat("-"):
            return f"(-{self.p_unary()})"
        if self.eat("+"):
            return self.p_unary()
        return self.p_pow()

    def p_pow(self) -> str:
        b = self.p_primary()
        if self.eat("^", "**"):
            return f"_pow({b}, {self.p_unary()})"
        return b

    def p_primary(self) -> str:
        t = self.peek()
        if t is None:
            raise SyntaxError(f"expression {self.expr!r}: unexpected end")
        self.i += 1
        if t == "(":
            e = self.p_or()
            self.want(")")
            return f"({e})"
        if t[0].isdigit() or t[0] == ".":
            return repr(float(t))
        if t[0].isalpha() or t[0] == "_":
            if self.eat("("):
                args = []
                if not self.eat(")"):
                    args.append(self.p_or())
                    while self.eat(","):
                        args.append(self.p_or())
                    self.want(")")
                return f"{'_if' if t == 'if' else t}({', '.join(args)})"
            return t
        raise SyntaxError(f"expression {self.expr!r}: unexpected {t!r}")


def _to_python(expr: str) -> str:
    return _ExprToPython(expr).run()


def constants(table: dict[str, list[str]]) -> dict[str, float]:
    out: dict[str, float] = {"pi": math.pi}
    pending = {k[len("my_constants."):]: " ".join(v) for k, v in table.items() if k.startswith("my_constants.")}
    for _ in range(len(pending) + 1):
        for name, ex in list(pending.items()):
            try:
                out[name] = float(eval_expr(ex, out))
                del pending[name]
            except NameError:
                pass
    if pending:
        raise ValueError(f"inputs: unresolved my_constants {sorted(pending)}")
    return out


def eval_expr(expr: str, consts: dict[str, float], x=None, y=None, z=None):
    env = dict(_FUNCS)
    env.update(consts)
    if x is not None:
        env.update(x=x, y=y, z=z)
    code = _to_python(" ".join(expr.split()))
    val = eval(code, {"__builtins__": {}}, env)  # noqa: S307 - trusted test decks
    return np.asarray(val, dtype=np.float64) * 1.0


# ------------------------------------------------------------- defaults -----

REQUIRED = ["TimeIntegratorOrder", "prob_type", "epsilon_0", "epsilonX_fe", "epsilonZ_fe", "epsilon_de",
            "epsilon_si", "alpha", "beta", "gamma", "alpha_12", "alpha_112", "alpha_123", "BigGamma",
            "g11", "g44", "g12", "g44_p", "lambda", "dt", "FE_lo", "FE_hi",
            "domain.prob_lo", "domain.prob_hi", "domain.n_cell"]

GHOST_MODES = {"extrap": 0, "face": 1, "zero": 2}


def ferrox_params(table: dict[str, list[str]]) -> dict:
    """Physics and domain parameters with the reference's defaults."""
    for k in REQUIRED:
        if k not in table:
            raise KeyError(f"inputs: required key {k!r} missing")
    consts = constants(table)

    def num(key, default=None, cast=float):
        if key not in table:
            if default is None:
                raise KeyError(key)
            return default
        v = table[key][0]
        try:
            return cast(v) if cast is int else float(v)
        except ValueError:
            return cast(float(eval_expr(v, consts)))

    def arr(key, default=None, cast=float):
        if key not in table:
            return list(default)
        out = []
        for v in table[key][:3]:
            try:
                out.append(cast(v) if cast is int else float(v))
            except ValueError:
                out.append(cast(float(eval_expr(v, consts))))
        return out

    p: dict = {}
    p["n_cell"] = arr("domain.n_cell", cast=int)
    p["prob_lo"] = arr("domain.prob_lo")
    p["prob_hi"] = arr("domain.prob_hi")
    p["is_periodic"] = arr("domain.is_periodic", [0, 0, 0], cast=int)
    lo, hi = p["prob_lo"], p["prob_hi"]

    p["P_BC_flag_lo"] = arr("P_BC_flag_lo", [0, 0, 0], cast=int)
    p["P_BC_flag_hi"] = arr("P_BC_flag_hi", [0, 0, 0], cast=int)
    p["TimeIntegratorOrder"] = num("TimeIntegratorOrder", cast=int)
    p["prob_type"] = num("prob_type", cast=int)
    p["is_polarization_scalar"] = num("is_polarization_scalar", 1, int)
    for k in ["epsilon_0", "epsilonX_fe", "epsilonZ_fe", "epsilon_de", "epsilon_si", "alpha", "beta", "gamma",
              "alpha_12", "alpha_112", "alpha_123", "BigGamma", "g11", "g44", "g12", "g44_p", "lambda", "dt"]:
        p[k] = num(k)
    p["epsilonX_fe_tphase"] = num("epsilonX_fe_tphase", p["epsilonX_fe"])
    p["nsteps"] = num("nsteps", 10, int)
    p["plot_int"] = num("plot_int", -1, int)
    p["delta"] = num("delta", 1.e-6)
    p["inc_step"] = num("inc_step", -1, int)
    p["random_seed"] = num("random_seed", 1, int)
    p["voltage_sweep"] = num("voltage_sweep", 0, int)
    p["Phi_Bc_hi"] = num("Phi_Bc_hi", 0.0)
    p["Phi_Bc_lo"] = num("Phi_Bc_lo", 0.0)
    p["Phi_Bc_inc"] = num("Phi_Bc_inc", 0.0)
    p["Phi_Bc_hi_max"] = num("Phi_Bc_hi_max", 0.0)
    p["phi_tolerance"] = num("phi_tolerance", 1.e-7)
    p["num_Vapp_max"] = num("num_Vapp_max", 1, int)
    p["include_Landau"] = num("include_Landau", 1, int)
    p["include_Grad"] = num("include_Grad", 1, int)
    p["include_Elec"] = num("include_Elec", 1, int)
    outside_lo = [lo[i] - 1.0 for i in range(3)]
    outside_hi = [hi[i] + 1.0 for i in range(3)]
    p["FE_lo"] = arr("FE_lo")
    p["FE_hi"] = arr("FE_hi")
    p["DE_lo"] = arr("DE_lo", outside_lo)
    p["DE_hi"] = arr("DE_hi", outside_hi)
    p["SC_lo"] = arr("SC_lo", outside_lo)
    p["SC_hi"] = arr("SC_hi", outside_hi)
    p["Channel_lo"] = arr("Channel_lo", outside_lo)
    p["Channel_hi"] = arr("Channel_hi", outside_hi)
    p["Remnant_P"] = arr("Remnant_P", [0.0, 0.0, 0.002])
    p["acceptor_doping"] = num("acceptor_doping", 0.0)
    p["donor_doping"] = num("donor_doping", 0.0)
    p["use_Fermi_Dirac"] = num("use_Fermi_Dirac", 1, int)
    p["use_work_function"] = num("use_work_function", 0, int)
    p["metal_work_function"] = num("metal_work_function", 4.85) if p["use_work_function"] == 1 else 0.0
    p["Coordinate_Transformation"] = num("Coordinate_Transformation", 0, int)
    p["use_Euler_angles"] = num("use_Euler_angles", 0, int)
    # fx.* extensions
    p["mg_rtol"] = num("fx.mg_rtol", 1.e-10)
    gm = table.get("fx.phi_ghost_mode", ["extrap"])[0]
    p["phi_ghost_mode"] = GHOST_MODES[gm]
    p["sweep_mode"] = 1 if table.get("fx.sweep_mode", ["steady"])[0] == "fixed" else 0
    p["steps_per_voltage"] = num("fx.steps_per_voltage", 0, int)
    p["newton_max_iter"] = num("fx.newton_max_iter", 50, int)
    p["mg_max_iter"] = num("fx.mg_max_iter", 200, int)
    p["verbose"] = 0
    return p


def embedded_boundary(table: dict[str, list[str]], p: dict):
    """(fluid layers, surface value) of a grid-aligned embedded boundary, or None.

    EmbeddedBoundaries.cpp:66-140 reads ``ebgeom.objects`` and each object's
    ``geom_type``, ``box_lo`` / ``box_hi``, ``has_fluid_inside`` and, with
    ``ebgeom.specify_inhomo_dir = 1``, ``surf_soln``.  The oracle takes the
    form the reference's FET decks use: one box with no fluid inside spanning
    x and y and covering z from a cell face to the top, so the embedded surface
    is the face below layer ``kb`` and the solve runs on layers ``k < kb``.
    Any other geometry raises ``ValueError``.
    """
    consts = constants(table)

    def first(key, default=None):
        return table[key][0] if key in table and table[key] else default

    if float(eval_expr(first("domain.embedded_boundary", "0"), consts)) == 0.0:
        return None
    if float(eval_expr(first("ebgeom.specify_input_using_eb2", "0"), consts)) != 0.0:
        raise ValueError("embedded boundary: EB2 input")
    names = table.get("ebgeom.objects", [])
    if len(names) != 1:
        raise ValueError("embedded boundary: exactly one object expected")
    name = names[0]
    if first(name + ".geom_type") != "box":
        raise ValueError("embedded boundary: only box objects")
    if first(name + ".has_fluid_inside") not in ("0", "false"):
        raise ValueError("embedded boundary: the box must have no fluid inside")
    lo = [float(eval_expr(v, consts)) for v in table[name + ".box_lo"][:3]]
    hi = [float(eval_expr(v, consts)) for v in table[name + ".box_hi"][:3]]
    plo, phi_, n = p["prob_lo"], p["prob_hi"], p["n_cell"]
    h = [(phi_[d] - plo[d]) / n[d] for d in range(3)]
    for d in range(2):
        if lo[d] > plo[d] + 1e-6 * h[d] or hi[d] < phi_[d] - 1e-6 * h[d]:
            raise ValueError("embedded boundary: the box must span x and y")
    if hi[2] < phi_[2] - 1e-6 * h[2]:
        raise ValueError("embedded boundary: the box must reach the top")
    f = (lo[2] - plo[2]) / h[2]
    kb = int(round(f))
    if abs(f - kb) > 1e-6 or not 1 <= kb < n[2]:
        raise ValueError("embedded boundary: the surface must be an interior cell face")
    V = 0.0
    if float(eval_expr(first("ebgeom.specify_inhomo_dir", "0"), consts)) != 0.0:
        V = float(eval_expr(first(name + ".surf_soln"), consts))
    return kb, V


def cell_centres(p: dict):
    n = p["n_cell"]
    dx = [(p["prob_hi"][d] - p["prob_lo"][d]) / n[d] for d in range(3)]
    x = p["prob_lo"][0] + (np.arange(n[0]) + 0.5) * dx[0]
    y = p["prob_lo"][1] + (np.arange(n[1]) + 0.5) * dx[1]
    z = p["prob_lo"][2] + (np.arange(n[2]) + 0.5) * dx[2]
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return X, Y, Z


def function_fields(table: dict[str, list[str]], p: dict):
    """tphase and Euler-angle fields (valid cells, shape (nz, ny, nx)) from the
    parser keys, as Initialize_tphase_Mask / Initialize_Euler_angles do when
    Coordinate_Transformation == 1 (Source/main.cpp:178-181)."""
    n = p["n_cell"]
    shape = (n[2], n[1], n[0])
    if "fx.grain_file" in table and p["Coordinate_Transformation"] == 1:
        # the polycrystal input file (format: ferrox_b200.decks.write_grain_file)
        from ferrox_b200 import decks
        g = decks.read_grain_file(table["fx.grain_file"][0])
        if g["id"].shape != shape:
            raise ValueError("inputs: fx.grain_file grid differs from domain.n_cell")
        tph, ang = decks.grain_fields(g)
        return (tph,) + tuple(ang)
    if p["Coordinate_Transformation"] != 1:
        z0 = np.zeros(shape)
        return z0, z0.copy(), z0.copy(), z0.copy()
    consts = constants(table)
    X, Y, Z = cell_centres(p)
    out = []
    for key in ["tphase_geom.tphase_geom_function(x,y,z)", "angle_alpha.alpha_function(x,y,z)",
                "angle_beta.beta_function(x,y,z)", "angle_theta.theta_function(x,y,z)"]:
        if key not in table:
            raise KeyError(f"inputs: {key!r} is required when Coordinate_Transformation = 1")
        out.append(np.broadcast_to(eval_expr(" ".join(table[key]), consts, X, Y, Z), shape).astype(np.float64))
    return tuple(out)
