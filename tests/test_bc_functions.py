"""Prescribed-displacement functions of x, y, z, t (the reference's "Value"
strings, src/core/Peridigm_BoundaryCondition.cpp:68-84, 157-160, 217-220):
the compiler and the interpreter through pd_expr_eval, on the host (no
device). Each case is checked against the same formula written in Python
(IEEE double arithmetic and the C library's functions, as the interpreter's
host build uses).
"""
import math

import pytest

from peridigm_b200 import PDError, expr_eval


CASES = [
    # (body, variables, the same formula in Python)
    ("0.0", {}, lambda x, y, z, t: 0.0),
    ("-1.5", {}, lambda x, y, z, t: -1.5),
    ("0.002*x*t/2.0e-8", dict(x=0.31, t=3.0e-8), lambda x, y, z, t: 0.002 * x * t / 2.0e-8),
    ("z*0.02*t", dict(z=-0.2, t=7.0), lambda x, y, z, t: z * 0.02 * t),
    ("-0.3*t/0.0004", dict(t=1.0e-4), lambda x, y, z, t: -0.3 * t / 0.0004),
    ("-0.2 * 0.5*(cos(3.14159265359 + t*3.14159265359/2.0e-2) + 1.0)", dict(t=6.0e-3),
     lambda x, y, z, t: -0.2 * 0.5 * (math.cos(3.14159265359 + t * 3.14159265359 / 2.0e-2) + 1.0)),
    ("300.0+500.0*(t/1800.0)", dict(t=900.0), lambda x, y, z, t: 300.0 + 500.0 * (t / 1800.0)),
    ("x*exp(-0.05*t/1.0e-8)", dict(x=0.4, t=2.0e-8), lambda x, y, z, t: x * math.exp(-0.05 * t / 1.0e-8)),
    ("2E-4 * 12.5^2 * z", dict(z=0.9), lambda x, y, z, t: 2e-4 * 12.5 ** 2 * z),
    ("-500.0 * x / sqrt(x*x + z*z)", dict(x=0.6, z=-0.8), lambda x, y, z, t: -500.0 * x / math.sqrt(x * x + z * z)),
    ("if(t<=2){value=-z*3.0e-6*t;} else{value=-z*3.0e-6*2;}", dict(z=1.5, t=1.25),
     lambda x, y, z, t: -z * 3.0e-6 * t if t <= 2 else -z * 3.0e-6 * 2),
    ("if(t<=2){value=-z*3.0e-6*t;} else{value=-z*3.0e-6*2;}", dict(z=1.5, t=2.5),
     lambda x, y, z, t: -z * 3.0e-6 * t if t <= 2 else -z * 3.0e-6 * 2),
    ("double a = 2.0*t; value = a*a + y;", dict(y=0.25, t=0.75), lambda x, y, z, t: (2.0 * t) * (2.0 * t) + y),
    ("if (x > 0.5 && t < 1.0) value = 1.0; else if (x > 0.5) value = 2.0; else value = 3.0;",
     dict(x=0.7, t=1.5), lambda x, y, z, t: 1.0 if (x > 0.5 and t < 1.0) else (2.0 if x > 0.5 else 3.0)),
    ("pow(t, 1.5) + atan2(y, x) + fmod(t, 0.3) + min(x, y) - max(x, y) + abs(-t) + floor(t) + ceil(t)",
     dict(x=0.2, y=0.9, t=1.7), lambda x, y, z, t: (math.pow(t, 1.5) + math.atan2(y, x) + math.fmod(t, 0.3)
                                                     + min(x, y) - max(x, y) + abs(-t) + math.floor(t) + math.ceil(t))),
    ("sin(t) + tan(t) + asin(0.5) + acos(0.5) + atan(t) + sinh(t) + cosh(t) + tanh(t) + log(t) + log10(t)",
     dict(t=0.4), lambda x, y, z, t: (math.sin(t) + math.tan(t) + math.asin(0.5) + math.acos(0.5) + math.atan(t)
                                      + math.sinh(t) + math.cosh(t) + math.tanh(t) + math.log(t) + math.log10(t))),
]


@pytest.mark.parametrize("body,kw,ref", CASES)
def test_functions_match_python(body, kw, ref):
    vals = dict(x=0.0, y=0.0, z=0.0, t=0.0)
    vals.update(kw)
    got = expr_eval(body, **vals)
    want = ref(vals["x"], vals["y"], vals["z"], vals["t"])
    assert got == pytest.approx(want, rel=1e-15, abs=1e-300)


@pytest.mark.parametrize("body,want", [
    ("-2^2", -4.0), ("2^3^2", 512.0), ("1 + 2*3", 7.0), ("(1 + 2)*3", 9.0), ("10 - 4 - 3", 3.0),
    ("8/4/2", 1.0), ("7 % 4", 3.0), ("(1 < 2) + (2 >= 3) + (2 == 2) + (2 != 2)", 2.0), ("!0 + !3", 1.0),
    ("0 || 2", 1.0), ("0 && 2", 0.0), ("-(-3)", 3.0), ("+4", 4.0), (".5e1", 5.0),
    ("value = 1; value = value + 2;", 3.0), ("{ value = 4; } ;", 4.0), ("if (0) value = 1;", 0.0),
])
def test_operators_and_statements(body, want):
    assert expr_eval(body) == want


@pytest.mark.parametrize("body", [
    "value = foo(t)", "value = q + 1", "value = (t + 1", "value = t +", "value 1", "if (t) { value = 1;",
    "sin = 2; value = 1", "value = atan2(t)", "value = 1 $ 2", "else value = 1",
])
def test_errors_are_reported(body):
    with pytest.raises(PDError):
        expr_eval(body)


def test_deep_expression_is_refused_not_overflowed():
    """Operand stacks deeper than the interpreter's are refused at compile time."""
    deep = "value = " + "+".join(["(t" for _ in range(40)]) + ")" * 40
    with pytest.raises(PDError):
        expr_eval(deep)
    shallow = "value = " + "+".join(["(t" for _ in range(10)]) + ")" * 10
    assert expr_eval(shallow, t=1.0) == 10.0
