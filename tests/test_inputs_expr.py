"""Known answers for the inputs-file expression grammar (csrc/inputs.cpp), no GPU needed.

FerroX evaluates the tphase and Euler-angle functions of the inputs file with
AMReX Parser (Initialize_tphase_Mask / Initialize_Euler_angles, called from
Source/main.cpp:178-181 when Coordinate_Transformation = 1).  The library has
its own compiler for the subset of that grammar these keys use.  Here each
expression goes in as `angle_alpha.alpha_function(x,y,z)` and the resulting
"alpha" field, which setup fills on the host, is compared with the value
worked out independently in Python: precedence and associativity, the
comparison and logical operators, if() and heaviside(), the one- and
two-argument functions, my_constants defined in terms of one another, and
x, y, z at cell centres.  Malformed expressions are rejected with a message.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from ferrox_b200 import api, decks

NX, NY, NZ = 8, 8, 12


def _deck(alpha_expr: str, extra: str = "") -> str:
    return (decks.mfim(NX, NY, NZ) + "\nCoordinate_Transformation = 1\nuse_Euler_angles = 0\n"
            "epsilonX_fe_tphase = 40.0\n"
            'tphase_geom.tphase_geom_function(x,y,z) = "0.0"\n'
            f'angle_alpha.alpha_function(x,y,z) = "{alpha_expr}"\n'
            'angle_beta.beta_function(x,y,z) = "0.0"\n'
            'angle_theta.theta_function(x,y,z) = "0.0"\n' + extra)


def _alpha(expr: str, extra: str = "") -> np.ndarray:
    f = api.FerroX(_deck(expr, extra))
    try:
        return f.field("alpha")
    finally:
        f.close()


CONSTANT_CASES = [
    ("-2^2 + 2^3^2 + 2**-1", -4.0 + 512.0 + 0.5),                 # unary minus below ^, ^ right-assoc
    ("2*3+4*5 - 6/3/2 - 2 - -1", 6 + 20 - 1 - 2 + 1),              # left-assoc / and -
    ("(3 > 2) + (2 >= 2)*10 + (1 < 1)*100 + (1 <= 1)*1000 + (1 == 1)*1e4 + (1 != 1)*1e5", 11011.0),
    ("(1 and 0) + (1 or 0)*2 + (1 && 1)*4 + (0 || 0)*8", 6.0),
    ("1 + 2 < 4 and 3 > 2", 1.0),                                  # arithmetic binds before comparison
    ("if(1 < 0, 100, 7) + heaviside(0, 0.25) + heaviside(-3, 0.25)*10 + heaviside(2, 0.25)*100", 107.25),
    ("abs(-1.5) + fabs(-2) + floor(2.7) + ceil(2.1) + min(4, max(1, 2)) + pow(2, 10) + log10(1000)", 1037.5),
    ("atan2(1, 1)*4/pi + exp(log(3)) + sqrt(16) + sin(pi/2) + cos(0) + tanh(0) + cosh(0) + sinh(0)",
     math.atan2(1, 1) * 4 / math.pi + math.exp(math.log(3)) + 4 + 1 + 1 + 0 + 1 + 0),
    ("tan(0.5) + asin(0.5) + acos(0.5) + atan(2)",
     math.tan(0.5) + math.asin(0.5) + math.acos(0.5) + math.atan(2)),
    ("1.5e1 + .25 + 3.", 18.25),
]


@pytest.mark.parametrize("expr,want", CONSTANT_CASES)
def test_constant_expression(expr, want):
    a = _alpha(expr)
    assert a.shape == (NZ, NY, NX)
    np.testing.assert_allclose(a, want, rtol=1e-15, atol=0)


def test_my_constants_chain():
    extra = "my_constants.c1 = 3\nmy_constants.c2 = c1^2\nmy_constants.c3 = -c2 + 1\n"
    np.testing.assert_array_equal(_alpha("c1*c2 + c3", extra), 27.0 - 8.0)


def test_position_dependent_expression_at_cell_centres():
    text = _deck("0")
    dom = {}
    for line in text.splitlines():
        key, _, val = line.partition("=")
        if key.strip() in ("domain.prob_lo", "domain.prob_hi"):
            dom[key.strip()] = [float(v) for v in val.split()]   # the last definition wins
    lo, hi, n = dom["domain.prob_lo"], dom["domain.prob_hi"], [NX, NY, NZ]
    c = [lo[d] + (np.arange(n[d]) + 0.5) * (hi[d] - lo[d]) / n[d] for d in range(3)]
    Z, Y, X = np.meshgrid(c[2], c[1], c[0], indexing="ij")
    got = _alpha("if(x > 0 and z < 4e-9, 1e9*x + (2e9*y)^2, -3*sin(1e9*z))")
    want = np.where((X > 0) & (Z < 4e-9), 1e9 * X + (2e9 * Y) ** 2, -3 * np.sin(1e9 * Z))
    assert ((X > 0) & (Z < 4e-9)).any() and not ((X > 0) & (Z < 4e-9)).all()
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("expr,want", CONSTANT_CASES)
def test_oracle_grammar_gives_the_same_known_answers(expr, want):
    """The oracle's restated grammar (the checker of setup parity) is pinned to the same answers."""
    from oracle import inputs as I
    np.testing.assert_allclose(I.eval_expr(expr, {"pi": math.pi}), want, rtol=1e-15, atol=0)


def test_oracle_my_constants_chain_and_syntax_error():
    from oracle import inputs as I
    table = I.parse_table("my_constants.c3 = -c2 + 1\nmy_constants.c1 = 3\nmy_constants.c2 = c1^2\n")
    c = I.constants(table)
    assert (c["c1"], c["c2"], c["c3"]) == (3.0, 9.0, -8.0)
    with pytest.raises(SyntaxError):
        I.eval_expr("(1 + 2", c)


@pytest.mark.parametrize("expr,words", [
    ("if(1, 2)", "3 arguments"),
    ("sin(1, 2)", "1 argument"),
    ("pow(2)", "2 arguments"),
    ("foo + 1", "unknown symbol"),
    ("(1 + 2", "missing ')'"),
    ("1 + ", "unexpected end"),
    ("2 $ 3", "unexpected"),
])
def test_malformed_expression_is_rejected(expr, words):
    with pytest.raises(api.FxError) as e:
        _alpha(expr)
    assert e.value.code == -2
    assert words in str(e.value), str(e.value)
