"""Table files: the Python reader (mars_md_b200/tables.py) and the C++ mirror's
TableFile (mars_md_b200/host/b200_pairlist.hpp) against the reference's own
Table::read_file (src/Objects/Tables.h:27-120, host-compiled in oracle/_ref):
the same X, Y, start and step bit for bit, the same uniformity verdict, on the
reference's own table file (Unit_test/Compute/bond-19.190-3.800.dat, read from
the checkout when it is here) and on written files with comments, blank and
malformed lines, extra columns, degree abscissae, a non-uniform step and a
single row."""
import math
import os
import subprocess
import warnings
from decimal import Decimal, getcontext

import numpy as np
import pytest

import pyoracle
from mars_md_b200 import build as B
from mars_md_b200 import tables as T

KIND_CODE = {"pair": 0, "bond": 1, "angle": 2, "dihedral": 3}
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP_SRC = os.path.join(ROOT, "tests", "cpp", "table_reader_test.cpp")
CPP_BIN = os.path.join(ROOT, "tests", "cpp", "_build", "table_reader_test")


def _double_rounding_trap() -> str:
    """Decimal text of 1 + 2^-24 + 2^-60: through double it rounds to the tie
    1 + 2^-24 and then to 1.0; straight to float it is 1 + 2^-23."""
    getcontext().prec = 60
    return str(Decimal(1) + Decimal(2) ** -24 + Decimal(2) ** -60)


def _write(path, rows, header=""):
    with open(path, "w") as f:
        f.write(header)
        for r in rows:
            f.write(r + "\n")
    return str(path)


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    d = tmp_path_factory.mktemp("tables")
    out = []
    ref_bond = B.reference_checkout()
    if ref_bond:
        p = os.path.join(ref_bond, "Unit_test", "Compute", "bond-19.190-3.800.dat")
        if os.path.exists(p):
            out.append(("reference bond file", p, "bond"))
    ang = [f"{k} {0.5 * 5.0 * (math.radians(k) - math.pi) ** 2:.9e}" for k in range(181)]
    ang.insert(10, "")                       # blank line
    ang.insert(20, "not a row")              # malformed
    ang[30] = ang[30] + " 7 extra columns"   # ignored tail
    out.append(("angle, degrees", _write(d / "angle.dat", ang, "# harmonic angle\n#k 5\n"), "angle"))
    dih = [f"{x} {math.cos(math.radians(x)):.7f}" for x in range(-180, 181, 10)]
    out.append(("dihedral", _write(d / "dih.dat", dih), "dihedral"))
    pair = [f"{0.1 * k:.6f} {_double_rounding_trap() if k == 3 else 1.0 / (1 + k)}"
            for k in range(50)]
    out.append(("pair, direct float parsing", _write(d / "pair.dat", pair), "pair"))
    wide = [f"{x:.4f} {x * x:.4f}" for x in (0.0, 0.5, 1.0, 1.5, 2.01, 2.51)]
    out.append(("non-uniform", _write(d / "wide.dat", wide), "bond"))
    narrow = [f"{x:.4f} {x:.4f}" for x in (0.0, 0.5, 1.0, 1.4, 1.9)]
    out.append(("smaller step (one-sided test)", _write(d / "narrow.dat", narrow), "bond"))
    out.append(("one row", _write(d / "one.dat", ["3.0 1.0"]), "dihedral"))
    return out


@pytest.fixture(scope="module")
def cpp_reader():
    deps = [CPP_SRC, os.path.join(ROOT, "mars_md_b200", "host", "b200_pairlist.hpp")]
    if not os.path.exists(CPP_BIN) or any(os.path.getmtime(p) > os.path.getmtime(CPP_BIN)
                                          for p in deps):
        os.makedirs(os.path.dirname(CPP_BIN), exist_ok=True)
        cuda = os.path.dirname(os.path.dirname(B.NVCC))
        subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
                        "-I" + os.path.join(ROOT, "mars_md_b200", "host"),
                        "-I" + os.path.join(cuda, "include"), CPP_SRC, "-o", CPP_BIN], check=True)
    return CPP_BIN


def _read_cpp(binary, path, kind):
    out = subprocess.run([binary, path, str(KIND_CODE[kind])], capture_output=True, text=True,
                         check=True).stdout.split("\n")
    n, start, step, uniform, step_inv = out[0].split()
    rows = [ln.split() for ln in out[1:1 + int(n)]]
    f = np.float32
    return (np.array([float.fromhex(r[0]) for r in rows], np.float32),
            np.array([float.fromhex(r[1]) for r in rows], np.float32),
            f(float.fromhex(start)), f(float.fromhex(step)), uniform == "1",
            f(float.fromhex(step_inv)))


def _read_py(path, kind):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return T.read_table(path, kind)


def test_python_reader_matches_reference_table(cases, ref):
    for what, path, kind in cases:
        t = _read_py(path, kind)
        x, y, start, step, uniform = ref.read_table(path, KIND_CODE[kind])
        assert np.array_equal(t.x.view(np.uint32), x.view(np.uint32)), what
        assert np.array_equal(t.y.view(np.uint32), y.view(np.uint32)), what
        assert t.start.view(np.uint32) == start.view(np.uint32), what
        assert t.step.view(np.uint32) == step.view(np.uint32), what
        assert t.uniform == uniform, what


def test_cpp_mirror_reader_matches_python(cases, cpp_reader):
    for what, path, kind in cases:
        t = _read_py(path, kind)
        x, y, start, step, uniform, step_inv = _read_cpp(cpp_reader, path, kind)
        assert np.array_equal(t.x.view(np.uint32), x.view(np.uint32)), what
        assert np.array_equal(t.y.view(np.uint32), y.view(np.uint32)), what
        assert t.start == start and t.step == step and t.uniform == uniform, what
        if len(t.x) >= 2:
            assert np.float32(t.spec().step_inv) == step_inv, what


def test_reader_rules(cases):
    by = {what: (path, kind) for what, path, kind in cases}
    with pytest.warns(UserWarning, match="Failed to parse line"):
        t = T.read_table(*by["angle, degrees"])
    assert len(t.x) == 181 and len(t.skipped_lines) == 2
    assert t.uniform and t.spec().periodic
    assert t.step == np.float32(np.float32(1.0) * T.DEG_TO_RAD)
    t = _read_py(*by["pair, direct float parsing"])
    assert t.y[3] == np.float32(1.0 + 2.0 ** -23)      # not 1.0 (double rounding)
    assert np.float32(t.spec().step_inv) == np.float32(1.0) / np.float32(t.step)
    with pytest.warns(UserWarning, match="Step size is not the same"):
        t = T.read_table(*by["non-uniform"])
    assert not t.uniform and t.step == np.float32(0.5)
    with pytest.raises(ValueError, match="not uniformly spaced"), warnings.catch_warnings():
        warnings.simplefilter("ignore")
        T.read_table(*by["non-uniform"], strict=True)
    assert _read_py(*by["smaller step (one-sided test)"]).uniform
    t = _read_py(*by["one row"])
    assert not t.uniform and t.step == 0.0
    assert t.start == np.float32(np.float32(-np.pi) * T.DEG_TO_RAD)
    with pytest.raises(ValueError, match="kind must be one of"):
        T.read_table(by["one row"][0], "torsion")
