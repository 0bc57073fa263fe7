"""The FP64 CPU adjoint of the BD window (oracle/mb2_adjoint.c) against
central finite differences of the FP64 forward: gradients of a Gaussian-smoothed
pair-distance histogram loss with respect to pair-table entries, bond-table
entries and initial positions.

The forces are piecewise constant in distance (per table bin), so the loss is
only piecewise smooth: the initial chain is jittered off the bond table's bin
edges (a seeded chain has every bond exactly 5.0 A long, on an edge) and the
finite-difference steps are small enough that no pair changes bin.
"""
import numpy as np
import pytest

import pyoracle as po
from mars_md_b200 import workloads as W

NB, DR, RMAX, SIG = 100, 0.25, 25.0, 0.25
TOL = 1e-4


@pytest.fixture(scope="module")
def case(oracle):
    rng = np.random.default_rng(3)
    nch, beads, L = 4, 32, 52.0
    xyz = np.mod(W._chains(rng, nch, beads, L) + rng.normal(scale=0.02, size=(nch * beads, 3)), L)
    bonds, angles, excl = W._topology(nch, beads)
    wca, bt = W.wca_table(), W.harmonic_bond_table()
    at = W.harmonic_angle_table(theta0_deg=150.0)
    A = po.Adjoint64(oracle, len(xyz), (L, L, L), (150.0, 150.0, 150.0), W.DT_NS, W.kT(),
                     (wca.values, wca.start, wca.step_inv), 20.0, bonds,
                     (bt.values, bt.start, bt.step_inv), angles, (at.values, at.start, at.step_inv),
                     excl)
    noise = rng.normal(size=(8, len(xyz), 3))
    target = A.rdf(xyz, NB, DR, RMAX, SIG) * 0.9

    def loss(x0):
        tr = A.forward(x0, noise)
        h = A.rdf(tr[-1], NB, DR, RMAX, SIG)
        return float(np.sum((h - target) ** 2)), tr, h

    _, tr, h = loss(xyz)
    lam_n = A.rdf_grad(tr[-1], NB, DR, RMAX, SIG, 2.0 * (h - target))
    g0, gp, gb = A.backward(tr, lam_n)
    return dict(A=A, xyz=xyz, loss=loss, g0=g0, gp=gp, gb=gb)


def _close(ad, fd, scale):
    return abs(ad - fd) <= TOL * max(abs(fd), 1e-3 * scale)


def test_pair_and_bond_table_gradients_match_finite_differences(case):
    A, loss = case["A"], case["loss"]
    for vals, g in ((A.pair_values, case["gp"]), (A.bond_values, case["gb"])):
        assert np.count_nonzero(g) > 5
        for k in np.argsort(-np.abs(g))[:5]:
            h = 1e-7 * max(1.0, abs(vals[k]))
            old = vals[k]
            vals[k] = old + h
            lp = loss(case["xyz"])[0]
            vals[k] = old - h
            lm = loss(case["xyz"])[0]
            vals[k] = old
            fd = (lp - lm) / (2 * h)
            assert _close(g[k], fd, np.abs(g).max()), (k, g[k], fd)


def test_position_gradient_matches_finite_differences(case):
    loss, g0, xyz = case["loss"], case["g0"], case["xyz"]
    rng = np.random.default_rng(11)
    for i, a in zip(rng.integers(0, len(xyz), 6), rng.integers(0, 3, 6)):
        h = 1e-6
        x = xyz.copy()
        x[i, a] += h
        lp = loss(x)[0]
        x[i, a] -= 2 * h
        lm = loss(x)[0]
        fd = (lp - lm) / (2 * h)
        assert _close(g0[i, a], fd, np.abs(g0).max()), (i, a, g0[i, a], fd)


def test_histogram_gradient_alone(case):
    """Zero steps: the loss gradient of the histogram itself."""
    A, xyz = case["A"], case["xyz"]
    target = np.zeros(NB)
    h = A.rdf(xyz, NB, DR, RMAX, SIG)
    g = A.rdf_grad(xyz, NB, DR, RMAX, SIG, 2.0 * (h - target))
    for i, a in [(0, 0), (40, 2), (90, 1)]:
        x = xyz.copy()
        x[i, a] += 1e-6
        lp = np.sum((A.rdf(x, NB, DR, RMAX, SIG) - target) ** 2)
        x[i, a] -= 2e-6
        lm = np.sum((A.rdf(x, NB, DR, RMAX, SIG) - target) ** 2)
        assert _close(g[i, a], (lp - lm) / 2e-6, np.abs(g).max())
