"""The pair kernels' squared-distance window (mb2_pair_distance_window)
against the reference's pair test restated in numpy float32: a pair is
skipped when dist = sqrt(d2) < 1e-6 or dist * dist > cutoff * cutoff
(PairNonbondedComputer, src/Interactions/Nonbonded/Pairwise.h:214-304), both
in IEEE float. Host only: no GPU needed."""
import ctypes as C

import numpy as np
import pytest

from mars_md_b200 import _lib as L

f32 = np.float32


def _skip(d2, cutoff):
    d2 = np.asarray(d2, f32)
    dist = np.sqrt(d2)
    cut2 = f32(cutoff) * f32(cutoff) if cutoff > 0 else f32(0)
    out = dist < f32(1e-6)
    if cutoff > 0:
        out |= (dist * dist) > cut2
    return out


def _window(cutoff):
    lib = L.load()
    lo, hi = C.c_float(0), C.c_float(0)
    assert lib.mb2_pair_distance_window(f32(cutoff), C.byref(lo), C.byref(hi)) == 0
    return f32(lo.value), f32(hi.value)


@pytest.mark.parametrize("cutoff", [30.0, 20.0, 35.0, 2.0 ** (1 / 6) * 4.0, 0.5, 1e-3,
                                    100.7, 1e4, 0.0])
def test_window_is_the_reference_test(cutoff):
    lo, hi = _window(cutoff)
    assert not _skip(lo, cutoff) and _skip(np.nextafter(lo, f32(0)), cutoff)
    if cutoff > 0:
        assert not _skip(hi, cutoff) and _skip(np.nextafter(hi, f32(np.inf)), cutoff)
    else:
        assert hi == np.inf
    # Every float within 4096 ulps of each bound, and a spread over the range.
    rng = np.random.default_rng(1)
    bits = [lo.view(np.uint32).astype(np.int64)]
    if np.isfinite(hi):
        bits.append(hi.view(np.uint32).astype(np.int64))
    cand = np.concatenate([np.arange(b - 4096, b + 4097) for b in bits] +
                          [rng.integers(0, 0x7F800000, size=200_000)])
    cand = cand[(cand >= 0) & (cand < 0x7F800000)].astype(np.uint32).view(f32)
    want = _skip(cand, cutoff)
    got = (cand < lo) | (cand > hi)
    assert np.array_equal(want, got), cand[want != got][:8]


def test_window_rejects_null_outputs():
    lib = L.load()
    assert lib.mb2_pair_distance_window(f32(30.0), None, None) == L.MB2_ERR_ARG


def _wrap_reference(x, l):
    """PeriodicBox::wrap_diff_scalar (src/System/PeriodicBox.h:453-461) in
    float32: image = floor(x * (1/l)); x -= image * l; x >= l/2 -> x - l."""
    f = np.float32
    inv, half = f(1) / l, f(0.5) * l
    img = np.floor((x * inv).astype(f)).astype(f)
    y = (x - (img * l).astype(f)).astype(f)
    return np.where(y >= half, (y - l).astype(f), y).astype(f)


@pytest.mark.parametrize("l", [1015.9, 127.0, 253.98427, 600.0, 33.3])
def test_inner_row_minimum_image(l):
    """The pair kernel's rows inside the box (every neighbour's difference in
    [-l/2, l/2)) take x, or RN(RN(x + l) - l) for a set sign bit, in place of
    the reference's floor sequence: the same float on every such x, signed
    zeros and tiny magnitudes included (+l/2 itself is outside the rows'
    bound and is the one value where the two differ)."""
    f = np.float32
    l = f(l)
    half = f(0.5) * l
    rng = np.random.default_rng(7)
    x = np.concatenate([
        rng.uniform(-half, half, 1_000_000).astype(f),
        (rng.uniform(-1, 1, 100_000) * 1e-3).astype(f),
        (rng.uniform(-1, 1, 100_000) * 1e-30).astype(f),
        np.array([0.0, -0.0, -half, np.nextafter(half, f(0)), -np.nextafter(half, f(0))], f)])
    w = ((x + l).astype(f) + (-l)).astype(f)
    inner = np.where(x.view(np.int32) < 0, w, x).astype(f)
    ref = _wrap_reference(x, l)
    assert np.array_equal(inner.view(np.uint32), ref.view(np.uint32))
    assert _wrap_reference(np.array([half], f), l)[0] != half  # the excluded end
