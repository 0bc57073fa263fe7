"""Tabulated potentials read from the reference's "x y" text files.

``read_table`` restates Table::read_file, check_same_step_size and
convert_angular_abscissa_to_radians (src/Objects/Tables.h:41-120), so a drop-in
user hands this library the same table files the reference loads:

* every line is read; a line whose first character is '#' is a comment; a line
  that does not start with two numbers (blank lines included) is skipped with
  a warning, as ``std::istringstream >> x >> y`` fails on it; anything after
  the second number is ignored;
* numbers are parsed straight to float32 (correctly rounded from the decimal
  text, as the C++ stream extraction into a float does), not through double;
* step = X[1] - X[0] and start = X[0], both in float32; the table is uniform
  unless some |X[i] - X[i-1]| - step exceeds 1e-4 (the reference's one-sided
  test), and, like the reference, a non-uniform table only warns: its Y values
  are then used with the first step (``strict=True`` raises ValueError
  instead); fewer than two rows also warn and leave step 0;
* angle and dihedral abscissae are degrees: X, start and step are each
  multiplied by float32(pi / 180) after the step check.

The result is a ``workloads.TableSpec``; its ``step_inv`` applies the
reference's non-bonded (1.0f / step) or bonded (float(1.0 / double(step)))
rule for the table's kind.
"""
from __future__ import annotations

import ctypes
import os
import re
import warnings
from dataclasses import dataclass

import numpy as np

from .workloads import DEG_TO_RAD, TableSpec

KINDS = ("pair", "bond", "angle", "dihedral")

# The prefix std::num_get accepts for a float: sign, digits with an optional
# fraction (or a bare fraction), an optional exponent.
_NUMBER = re.compile(rb"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")
_libc = ctypes.CDLL(None)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]


def _to_f32(token: bytes):
    """Decimal text -> the nearest float32 (one rounding); None on overflow,
    which the stream extraction reports as a failure."""
    v = np.float32(_libc.strtof(token, None))
    return None if np.isinf(v) else v


def _two_numbers(line: bytes):
    """(x, y) as ``iss >> x >> y`` reads them into floats, or None."""
    pos = 0
    out = []
    for _ in range(2):
        while pos < len(line) and line[pos:pos + 1].isspace():
            pos += 1
        m = _NUMBER.match(line, pos)
        v = _to_f32(m.group(0)) if m else None
        if v is None:
            return None
        out.append(v)
        pos = m.end()
    return out


@dataclass
class TableFile:
    """A table as Table::read_file leaves it (X converted for angular kinds)."""
    name: str
    kind: str
    x: np.ndarray           # float32
    y: np.ndarray           # float32
    start: np.float32
    step: np.float32
    uniform: bool
    skipped_lines: list     # 1-based numbers of the lines that did not parse

    def spec(self) -> TableSpec:
        """The table as this library's set-up calls take it; angle and dihedral
        tables wrap (DeviceBondedInteraction::link_tables)."""
        return TableSpec(values=self.y, start=float(self.start), step=float(self.step),
                         periodic=self.kind in ("angle", "dihedral"), kind=self.kind)


def _check_same_step_size(x: np.ndarray, name: str, kind: str):
    """(uniform, start, step) of Table::check_same_step_size (Tables.h:41-59);
    with fewer than two rows the constructor's values stay (start -pi for a
    dihedral table, Tables.h:35-39, else 0; step 0)."""
    if len(x) < 2:
        warnings.warn(f"Table {name}: Not enough values to check step size")
        start = np.float32(-np.pi) if kind == "dihedral" else np.float32(0.0)
        return False, start, np.float32(0.0)
    step = np.float32(x[1] - x[0])
    start = np.float32(x[0])
    for i in range(2, len(x)):
        # float arithmetic as in the reference; the comparison with 1e-4 in double
        if float(np.float32(np.abs(np.float32(x[i] - x[i - 1])) - step)) > 1e-4:
            warnings.warn(f"Table {name}: Step size is not the same for all values at index "
                          f"{i}: {x[i]}")
            return False, start, step
    return True, start, step


def read_table(path: str, kind: str, name: str | None = None, strict: bool = False) -> TableFile:
    """Read one "x y" table file as the reference does (see the module docstring).
    kind: "pair", "bond", "angle" or "dihedral"."""
    if kind not in KINDS:
        raise ValueError(f"read_table: kind must be one of {KINDS}, not {kind!r}")
    name = name or os.path.splitext(os.path.basename(path))[0]
    xs, ys, skipped = [], [], []
    with open(path, "rb") as f:
        for number, line in enumerate(f, start=1):
            if line[:1] == b"#":
                continue
            xy = _two_numbers(line)
            if xy is None:
                skipped.append(number)
                warnings.warn(f"Tables: Failed to parse line {number}: {line!r}")
                continue
            xs.append(xy[0])
            ys.append(xy[1])
    x = np.array(xs, np.float32)
    y = np.array(ys, np.float32)
    uniform, start, step = _check_same_step_size(x, name, kind)
    if strict and not uniform:
        raise ValueError(f"read_table: {path}: abscissa is not uniformly spaced "
                         f"(or fewer than two rows)")
    if kind in ("angle", "dihedral"):
        x = (x * DEG_TO_RAD).astype(np.float32)
        start = np.float32(start * DEG_TO_RAD)
        step = np.float32(step * DEG_TO_RAD)
    return TableFile(name=name, kind=kind, x=x, y=y, start=start, step=step, uniform=uniform,
                     skipped_lines=skipped)
