"""Initial-condition expressions on the CPU: the oracle against the reference's
own known answers, and the library's compiler against the oracle through the
compiled program text (no GPU needed).

Known answers: test/test_user_expression.cpp (UserExpression) and
test/initial_condition/test_prime_state_initializer.cpp (PrimeStateInitializer).
"""
import ctypes as C
import glob
import html
import os
import re

import numpy as np
import pytest

from alpaca_b200 import api
from alpaca_b200 import native as N
from oracle import ic_expr as X

# the reference checkout: $ALPACA_REFERENCE_DIR, else `reference` beside the repository
REF = os.environ.get("ALPACA_REFERENCE_DIR",
                     os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "reference"))

SOD = """if (x < 0.5)
{
    density : = 1.0;
    velocityX := 0.0;
    pressure := 1.0;
}
else
{
    density := 0.125;
    velocityX := 0.0;
    pressure := 0.1;
}"""

PROGRAMS = {
    "sod": SOD,
    "ternary": "density := z < 0.5 ? 1.0 : 2.0; pressure := y >= 0.25 ? x : -x;",
    "functions": """density := exp(-x); velocityX := tanh(x); velocityZ := abs(y*y);
                    pressure := 2.0 + sin(y * pi); velocityY := sqrt(pow(x, 2) + pow(y, 2))
                    / 0.4 * cos(atan(y / x));""",
    "chain": """// a chain of cases, comments and locals
        var r := sqrt((x - 0.3)^2 + (y - 0.3)^2 + (z - 0.3)^2);
        if ((x >= 0.2) & (x <= 0.4)) { density := (1 / 6) * (exp(-334.477 * (x - 0.3) * (x - 0.3)) + 4); }
        else if ((x >= 0.6) and (x <= 0.8)) density := 1.0;
        else if (r < 0.25 | x > 0.9) { density := 1 - abs(10 * (x - 1.1)); }
        else { density := sqrt(max(1 - 100 * (x - 1.5) * (x - 1.5), 0, 0.5)); }
        /* velocities */ velocityX := if (x > 0.5, 1, -1); velocityY := min(x, y, z);
        pressure := 1.0e4; pressure += 2x; pressure *= 1.5; pressure -= 3(y + 1);
        pressure /= 2; velocityZ := x % 0.3 + round(2.5) + sgn(-y) + floor(x) + (x == x);""",
    "implicit": "density := 2.000000(0.500000 * x + 1.000000 * y + 1.500000 * z); "
                "pressure := 5.0(x - y)(x + y); velocityX := -2^2 + 2^-1;",
    "logic": "density := not (x < 0.5) + !(y > 0.5) * 2 + (x <> y) * 4 + (x != x) * 8;"
             "pressure := (x < 0.5 and y < 0.5) + (x < 0.5 or y < 0.5) * 2;",
}


def points(n=97, seed=3):
    rng = np.random.default_rng(seed)
    return rng.uniform(-0.2, 1.3, n), rng.uniform(-0.2, 1.3, n), rng.uniform(-0.2, 1.3, n)


# ---- the oracle against the reference's own answers --------------------------

@pytest.mark.parametrize("x,f", [(0.0, 5.0), (-2.5, 0.0), (-2.625, -0.25)])
def test_linear_expression(x, f):
    """test_user_expression.cpp:100-123: f := 2 * x + 5."""
    v = X.evaluate("f := 2 * x + 5", {"x": np.array([x])}, outputs=("f",))
    assert v["f"][0] == pytest.approx(f)


@pytest.mark.parametrize("x,y,f,g", [(0.0, 0.0, 2.5, 0.0), (0.0, 2.125, 2.5, 0.0),
                                     (1.5, 0.0, 4.75, 0.0), (2.75, -1.25, 10.0625, -3.4375)])
def test_quadratic_expression(x, y, f, g):
    """test_user_expression.cpp:126-163: f := x * x + 2.5; g := x * y."""
    v = X.evaluate("f := x * x + 2.5; g := x * y;", {"x": np.array([x]), "y": np.array([y])},
                   outputs=("f", "g"))
    assert v["f"][0] == pytest.approx(f) and v["g"][0] == pytest.approx(g)


def test_spherical_expression():
    """test_user_expression.cpp:166-214: points at radii r1 < r2 < r3 on the
    same directions lie |r_a - r_b| apart and r from the origin."""
    prog = "x := r*sin(theta)*cos(phi); y := r*sin(theta)*sin(phi); z := r*cos(theta);"
    th, ph = np.meshgrid(np.arange(8) * 0.4, -3.1415926 + np.arange(16) * 0.4)
    pts = []
    for r in (0.5, 1.25, 2.0):
        v = X.evaluate(prog, {"r": np.full(th.size, r), "theta": th.ravel(), "phi": ph.ravel()},
                       outputs=("x", "y", "z"))
        pts.append(np.stack([v["x"], v["y"], v["z"]]))
    for a, b, d in ((0, 1, 0.75), (0, 2, 1.5), (1, 2, 0.75)):
        assert np.allclose(np.linalg.norm(pts[a] - pts[b], axis=0), d)
    for a, r in enumerate((0.5, 1.25, 2.0)):
        assert np.allclose(np.linalg.norm(pts[a], axis=0), r)


@pytest.mark.parametrize("bad", ["f := x* y", "f := 2 *", "f := (x", "g := x", "f := foo(x)",
                                 "x := 1", "f := x ^ 2 ^ 3", "f := 1 f := 2"])
def test_oracle_rejects(bad):
    """test_user_expression.cpp:77-95: UserExpression throws for unknown inputs
    and malformed programs."""
    with pytest.raises(X.ExprError):
        X.check_syntax(bad, inputs=("x",), outputs=("f",))


def _initializer_program(material: int, factors, dim: int):
    """CreateMaterialInitialConditions (test_prime_state_initializer.cpp:80-98):
    prime state p of material m := (m + 1)(p + 1)(f0 x + f1 y + f2 z), numbers
    written as std::to_string writes them."""
    names = ["density", "pressure", "velocityX", "velocityY", "velocityZ"][: dim + 2]
    s = ""
    for p, n in enumerate(names):
        k = float((material + 1) * (p + 1))
        s += (f"{n} := {k:f}({factors[0]:f} * x + {factors[1]:f} * y + "
              f"{factors[2]:f} * z);")
    return s


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_prime_state_initializer_relations(dim):
    """test_prime_state_initializer.cpp:99-170 on the level-0 node of size 1:
    material two's prime states are twice material one's, and within a
    material density = (1 / (p + 1)) times prime state p, none zero."""
    o = np.zeros((1, 3))
    h = 1.0 / 16
    a = X.initial_prime_states(_initializer_program(0, (0.5, 1.0, 1.5), dim), dim, o, h)
    b = X.initial_prime_states(_initializer_program(1, (0.5, 1.0, 1.5), dim), dim, o, h)
    assert np.array_equal(2.0 * a, b)
    for p in range(dim + 2):
        assert (a[:, p] != 0).all()
        assert np.allclose(a[:, 0], a[:, p] / (p + 1), rtol=2e-16, atol=0)


def test_units_scale_the_prime_states():
    """UnitHandler (unit_handler.cpp:45-46, 67-98): density / rho_ref,
    velocity / u_ref, pressure / (rho_ref u_ref^2); coordinates in length units."""
    prog = "density := 1000; velocityX := 20; pressure := 1e5 + x;"
    a = X.initial_prime_states(prog, 1, np.zeros((1, 3)), 0.5, units=(1000.0, 10.0, 2.0))
    assert np.allclose(a[0, 0], 1.0) and np.allclose(a[0, 2], 2.0)
    assert np.allclose(a[0, 1], (1e5 + (np.arange(16) + 0.5) * 0.5) / 1e5)


# ---- the library's compiler against the oracle -------------------------------

def same(got, ref, msg):
    """Equal up to the last bit of a transcendental function: numpy's scalar
    path (the listing interpreter) and its array path (the oracle) may round
    sin, exp, pow ... differently by one ulp."""
    np.testing.assert_allclose(got, ref, rtol=4.5e-16, atol=0, err_msg=msg)


def compiled(text):
    p = api.IcProgram(text)
    lines = p.listing()
    info = p.info()
    p.close()
    return lines, info


@pytest.mark.parametrize("name", list(PROGRAMS))
def test_compiled_program_matches_oracle(name):
    text = PROGRAMS[name]
    lines, info = compiled(text)
    assert lines[-1] == "END" and info["instructions"] == len(lines)
    assert 1 <= info["max_stack"] <= 32
    x, y, z = points()
    got = X.run_listing(lines, x, y, z)
    ref = X.evaluate(text, {"x": x, "y": y, "z": z})
    for n in X.PRIMES:
        same(got[n], ref[n], f"{name} {n}")


def test_jumps_only_go_forward():
    lines, _ = compiled(PROGRAMS["chain"])
    for pc, ln in enumerate(lines):
        op = ln.split()
        if op[0] in ("JZ", "JMP"):
            assert pc < int(op[1]) < len(lines)


@pytest.mark.parametrize("bad,why", [
    ("density := 2 *", "expected a value"),
    ("density := (x", "expected ')'"),
    ("phi := x", "unknown variable 'phi'"),
    ("density := foo(x)", "unknown symbol 'foo'"),
    ("x := 1", "cell centre"),
    ("density := x ^ 2 ^ 3", "chained"),
    ("density := 1 pressure := 2", "expected ';'"),
    ("density := atan2(x)", "two arguments"),
    ("density := max(x)", "at least two"),
    ("density := x $ 2", "unexpected character"),
    ("density := " + "(" * 40 + "x" + ")" * 40, None),
    ("density := " + "1 + (" * 40 + "x" + ")" * 40, "nested too deeply"),
    ("var density := 1;", "already defined"),
    ("/* open comment", "unterminated comment"),
])
def test_compiler_rejects(bad, why):
    lib = N.lib()
    h = C.c_void_p()
    rc = lib.alp_ic_program_create(bad.encode(), C.byref(h))
    if why is None:  # deep parentheses alone need no stack
        assert rc == N.ALP_OK
        lib.alp_ic_program_destroy(h)
        return
    assert rc == N.ALP_ERR_INVALID
    msg = lib.alp_last_error().decode()
    assert why in msg and "position" in msg, msg
    assert not h.value


def reference_programs():
    """Every material initial condition in the reference's input files."""
    out = []
    for f in sorted(glob.glob(os.path.join(REF, "**", "*.xml"), recursive=True)):
        s = open(f, errors="ignore").read()
        m = re.search(r"<initialConditions>(.*?)</initialConditions>", s, re.S)
        if not m:
            continue
        for mm in re.finditer(r"<(material\d)>(.*?)</\1>", m.group(1), re.S):
            out.append((os.path.relpath(f, REF) + ":" + mm.group(1), html.unescape(mm.group(2))))
    return out


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference input files not present")
def test_every_reference_initial_condition_compiles_and_agrees():
    progs = reference_programs()
    assert len(progs) >= 40
    x, y, z = points(31, seed=5)
    for where, text in progs:
        lines, _ = compiled(text)
        got = X.run_listing(lines, x, y, z)
        ref = X.evaluate(text, {"x": x, "y": y, "z": z})
        for n in X.PRIMES:
            same(got[n], ref[n], f"{where} {n}")
