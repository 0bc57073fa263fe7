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


@pytest.mark.slow
def test_c5_system_gradients_match_finite_differences(oracle):
    """The benchmark's adjoint system (16 chains x 1,024 beads, box 378 A, WCA
    pair table, harmonic bonds and angles, 1-2/1-3 exclusions, target from the
    pair table with sigma 4 -> 4.2 A, seeded normals as noise) over one
    checkpoint segment (20 steps). The 5 largest pair-table and bond-table
    components and 6 position components against central differences of the
    FP64 forward, each within 1e-4 of the difference quotient.

    The loss is piecewise smooth: a step large enough to move some pair across
    a table-bin edge between the + and - runs adds a jump, a step too small
    drowns in FP64 rounding of a loss summed over 16,384 particles. Each
    component is therefore tried at three steps (1e-7, 1e-8, 1e-9, relative
    for table values, in A for positions) and passes when one of them agrees.
    Over the full 200-step window the tangent dynamics grow by about 10^4 and
    no step from 1e-8 to 1e-11 gives a converged quotient (bin crossings at
    the larger steps, rounding at the smaller), so the difference check is
    made on one segment."""
    steps = 20
    w = W.adjoint()
    rng = np.random.default_rng(W.DEFAULT_SEED)
    xyz = np.mod(w.pos[:, :3].astype(np.float64) + rng.normal(scale=0.02, size=(w.n, 3)),
                 w.box_size[0])
    t, b, a = w.pair_tables[0], w.bond_tables[0], w.angle_tables[0]

    def system(pair_values):
        return po.Adjoint64(oracle, w.n, w.box_size, w.diffusion[0], w.dt, w.kT,
                            (pair_values, t.start, t.step_inv), w.cutoff, w.bonds,
                            (b.values, b.start, b.step_inv), w.angles,
                            (a.values, a.start, a.step_inv), w.exclusions)
    A, pert = system(t.values), system(W.wca_table(sigma=4.2).values)
    noise = rng.normal(size=(steps, w.n, 3))
    target = pert.rdf(pert.forward(xyz, noise)[-1], NB, DR, RMAX, SIG)

    def loss(x0):
        tr = A.forward(x0, noise)
        h = A.rdf(tr[-1], NB, DR, RMAX, SIG)
        return float(np.sum((h - target) ** 2)), tr, h

    _, tr, h = loss(xyz)
    lam = A.rdf_grad(tr[-1], NB, DR, RMAX, SIG, 2.0 * (h - target))
    g0, gp, gb = A.backward(tr, lam)

    def check(g, scale, at, unit):
        fds = []
        for h in (1e-7 * unit, 1e-8 * unit, 1e-9 * unit):
            fds.append((at(h) - at(-h)) / (2 * h))
            if _close(g, fds[-1], scale):
                return
        raise AssertionError((g, fds))

    checked = 0
    for vals, g in ((A.pair_values, gp), (A.bond_values, gb)):
        for k in np.argsort(-np.abs(g))[:5]:
            old = vals[k]

            def at(d, k=k, old=old, vals=vals):
                vals[k] = old + d
                v = loss(xyz)[0]
                vals[k] = old
                return v
            check(g[k], np.abs(g).max(), at, max(1.0, abs(old)))
            checked += 1
    order = np.argsort(-np.abs(g0).ravel())
    picks = list(order[:3]) + list(rng.choice(order[3:], 3, replace=False))
    for q in picks:
        i, ax = divmod(int(q), 3)

        def at(d, i=i, ax=ax):
            x = xyz.copy()
            x[i, ax] += d
            return loss(x)[0]
        check(g0[i, ax], np.abs(g0).max(), at, 1.0)
        checked += 1
    assert checked == 16


def test_float_bin_decisions_match_double_off_edges(oracle):
    """With float states away from table-bin edges, deciding bins in the
    reference's float arithmetic gives the double adjoint's gradients."""
    rng = np.random.default_rng(3)
    nch, beads, L = 4, 32, 52.0
    xyz = np.mod(W._chains(rng, nch, beads, L) + rng.normal(scale=0.02, size=(nch * beads, 3)),
                 L).astype(np.float32).astype(np.float64)
    bonds, angles, excl = W._topology(nch, beads)
    wca, bt = W.wca_table(), W.harmonic_bond_table()
    at = W.harmonic_angle_table(theta0_deg=150.0)
    grads = []
    for fb in (False, True):
        A = po.Adjoint64(oracle, len(xyz), (L, L, L), (150.0, 150.0, 150.0), W.DT_NS, W.kT(),
                         (wca.values, wca.start, wca.step_inv), 20.0, bonds,
                         (bt.values, bt.start, bt.step_inv), angles,
                         (at.values, at.start, at.step_inv), excl, float_bins=fb)
        noise = rng.normal(size=(3, len(xyz), 3)) if not grads else grads[0][3]
        tr = A.forward(xyz, noise)
        h = A.rdf(tr[-1], NB, DR, RMAX, SIG)
        g0, gp, gb = A.backward(tr, A.rdf_grad(tr[-1], NB, DR, RMAX, SIG, 2.0 * h))
        grads.append((g0, gp, gb, noise))
    for a, b in zip(grads[0][:3], grads[1][:3]):
        assert np.abs(a - b).max() <= 1e-6 * np.abs(a).max()


def test_pairlist_segments_match_fresh_pairs_when_rebuilt_every_step(oracle):
    """list_every = 1 (a list within the list radius built at every step) gives
    the all-pairs-within-the-cutoff forward and adjoint; with longer segments
    on a short window the pairs within the cutoff stay in the list too."""
    rng = np.random.default_rng(5)
    w = W.adjoint(seed=7, n_chains=4, beads=256)
    x0 = np.mod(w.pos[:, :3].astype(np.float64) + rng.normal(scale=0.02, size=(w.n, 3)),
                w.box_size[0])
    t, b, a = w.pair_tables[0], w.bond_tables[0], w.angle_tables[0]

    def system(every):
        return po.Adjoint64(oracle, w.n, w.box_size, w.diffusion[0], w.dt, w.kT,
                            (t.values, t.start, t.step_inv), w.cutoff, w.bonds,
                            (b.values, b.start, b.step_inv), w.angles,
                            (a.values, a.start, a.step_inv), w.exclusions, list_every=every,
                            list_radius=w.list_radius)
    noise = rng.normal(size=(10, w.n, 3))
    lam = rng.normal(size=(w.n, 3))
    ref_tr = system(0).forward(x0, noise)
    ref_g = system(0).backward(ref_tr, lam)
    for every in (1, 5):
        A = system(every)
        tr = A.forward(x0, noise)
        assert np.abs(tr - ref_tr).max() < 1e-10
        for g, h in zip(A.backward(ref_tr, lam), ref_g):
            assert np.abs(g - h).max() <= 1e-12 * np.abs(h).max()
