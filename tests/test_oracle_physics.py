"""Physics checks of the oracle, restating the reference's own test intent:
analytic tabulated pair energy (Unit_test/Interactions/NonbondedEnergy.cpp),
cutoff drop, angle finite differences (Unit_test/Interactions/TabulatedBonded.cpp),
Box-Muller moments and free-diffusion MSD (Unit_test/Compute/BDKernels.cpp),
seed decorrelation (Unit_test/Compute/StochasticIntegrators.cpp) and noise keyed
on the absolute step (Unit_test/System/RestartContinuation.cpp).
"""
import numpy as np
import pytest

import pyoracle as po
from mars_md_b200 import workloads as W


def _analytic_table():
    """U(r) = (r - 3)^2 - 1 sampled at 2048 bins over [0, 10) A."""
    x = (np.arange(2048, dtype=np.float64) * (10.0 / 2048)).astype(np.float32)
    u = ((x.astype(np.float64) - 3.0) ** 2 - 1.0).astype(np.float32)
    t = W.table_from_xy(x, u, "pair")
    return t, po.TableSet([(t.values, t.start, t.step_inv)])


def test_table_interpolates_analytic_force_and_energy(oracle):
    _, ts = _analytic_table()
    for r in np.linspace(0.5, 9.5, 37):
        f, e = oracle.table_lookup(ts, 0, float(r))
        assert f == pytest.approx(-2.0 * (r - 3.0), abs=1e-2)
        assert e == pytest.approx((r - 3.0) ** 2 - 1.0, abs=1e-2)


def _one_pair(oracle, r, cutoff=9.0):
    _, ts = _analytic_table()
    pos = np.zeros((2, 4), np.float32)
    pos[1, 0] = r
    box = po.Box.make((-50.0, -50.0, -50.0), (100.0, 100.0, 100.0))
    pairs = np.array([[0, 1]], np.int32)
    tags = np.array([(1 << 5) | (0 << 8)], np.uint32)
    fe, _, _ = oracle.pair_forces(pairs, pos, tags, ts, box, np.float32(cutoff) ** 2)
    return fe


def test_pair_energy_split_half_and_well_sign(oracle):
    fe = _one_pair(oracle, 2.0)  # repulsive side of the well at 3 A
    u = (2.0 - 3.0) ** 2 - 1.0
    assert fe[0, 3] == pytest.approx(u / 2, abs=1e-3) and fe[1, 3] == pytest.approx(u / 2, abs=1e-3)
    assert fe[1, 0] > 0 and fe[0, 0] == -fe[1, 0]   # pushes the pair apart
    fe = _one_pair(oracle, 4.0)  # attractive side
    assert fe[1, 0] < 0 and fe[0, 0] == -fe[1, 0]


def test_pair_beyond_cutoff_contributes_nothing(oracle):
    fe = _one_pair(oracle, 9.5, cutoff=9.0)
    assert not fe.any()


def test_angle_forces_are_energy_gradient(oracle):
    spec = W.harmonic_angle_table(k=5.0, theta0_deg=120.0)
    at = po.TableSet([(spec.values, spec.start, spec.step_inv)], periodic=True)
    box = po.Box.make((-50.0, -50.0, -50.0), (100.0, 100.0, 100.0), (0, 0, 0))
    rng = np.random.default_rng(5)
    pos = np.zeros((3, 4), np.float32)
    pos[:, :3] = np.array([[3.0, 0.2, 0.1], [0.0, 0.0, 0.0], [-1.0, 2.6, 0.3]], np.float32)
    ang = np.array([[0, 1, 2, 0]], np.int32)
    idx = np.zeros(1, np.int32)

    def energy(p):
        _, fe64, _ = oracle.angle_forces(ang, idx, p, at, box)
        return fe64[:, 3].sum()

    fe, _, _ = oracle.angle_forces(ang, idx, pos, at, box)
    h = 1e-3
    for b in range(3):
        for a in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[b, a] += h
            pm[b, a] -= h
            fd = -(energy(pp) - energy(pm)) / (2 * h)
            assert fe[b, a] == pytest.approx(fd, rel=2e-2, abs=2e-2)
    assert abs(fe[:, :3].astype(np.float64).sum(0)).max() < 1e-4


def _noise(oracle, n, seed, step):
    ty = po.TypeSet(np.zeros(1, np.float32), np.full((1, 3), 1.0, np.float32))
    box = po.Box.make((0, 0, 0), (1e4, 1e4, 1e4))
    pos = np.full((n, 4), 5e3, np.float32)
    pos[:, 3] = 0.0
    _, _, nz = oracle.bd_integrate(pos, np.zeros_like(pos), np.zeros(n, np.int32), None, ty, None,
                                   box, 1e-4, 1.0, step, oracle.bd_seed(seed, 0, step),
                                   want_noise=True)
    return nz[:, :3].astype(np.float64)


def test_box_muller_moments(oracle):
    z = _noise(oracle, 50_000, 12345, 1).ravel()
    assert abs(z.mean()) < 0.02
    assert abs(z.var() - 1.0) < 0.02
    assert abs((z ** 3).mean()) < 0.05
    assert abs((z ** 4).mean() - 3.0) < 0.1


def test_adjacent_seeds_decorrelated(oracle):
    a = _noise(oracle, 20_000, 1000, 4).ravel()
    b = _noise(oracle, 20_000, 1001, 4).ravel()
    assert abs(np.corrcoef(a, b)[0, 1]) < 0.15
    c = _noise(oracle, 20_000, 1000, 5).ravel()
    assert abs(np.corrcoef(a, c)[0, 1]) < 0.15


def test_free_diffusion_msd(oracle):
    """MSD = 6 D t for free particles (5 seeds x 200 particles x 100 steps, 10 %)."""
    D, dt, steps, n = 150.0, 1e-4, 100, 200
    ty = po.TypeSet(np.zeros(1, np.float32), np.full((1, 3), D, np.float32))
    L = 1e5
    box = po.Box.make((0, 0, 0), (L, L, L))
    msd = []
    for seed in range(5):
        pos0 = np.zeros((n, 4), np.float32)
        pos0[:, :3] = L / 2
        pos = pos0
        for s in range(1, steps + 1):
            pos, _, _ = oracle.bd_integrate(pos, np.zeros_like(pos), np.zeros(n, np.int32), None,
                                            ty, None, box, dt, W.kT(), s,
                                            oracle.bd_seed(seed, 0, s))
        msd.append(np.mean(np.sum((pos[:, :3] - pos0[:, :3]).astype(np.float64) ** 2, axis=1)))
    assert np.mean(msd) == pytest.approx(6.0 * D * dt * steps, rel=0.1)


def test_noise_keyed_on_absolute_step(oracle):
    """A run resumed at step k draws the same noise as an uninterrupted one."""
    assert np.array_equal(_noise(oracle, 64, 7, 6), _noise(oracle, 64, 7, 6))
    assert not np.array_equal(_noise(oracle, 64, 7, 6), _noise(oracle, 64, 7, 7))
    assert oracle.bd_seed(7, 0, 6) != oracle.bd_seed(7, 1, 6)


def test_baoab_momentum_reaches_equipartition(oracle):
    """Free particles under BAOAB: the momentum variance settles at kT m (in the
    reference's units, times SQRT_CAL_TO_JOULE^2), per axis, for each damping."""
    n, steps = 4000, 120
    mass = np.array([12.0], np.float32)
    damping = np.array([[50.0, 100.0, 200.0]], np.float32)
    ty = po.TypeSet(np.zeros(1, np.float32), np.full((1, 3), 150.0, np.float32))
    box = po.Box.make((0, 0, 0), (1e4, 1e4, 1e4))
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = 5e3
    mom = np.zeros((n, 4), np.float32)
    fe = np.zeros((n, 4), np.float32)
    dt, kT = 1e-3, W.kT()
    for s in range(1, steps + 1):
        pos, mom, fe = oracle.baoab_integrate(pos, mom, fe, np.zeros(n, np.int32), None, ty, None,
                                              mass, damping, box, dt, kT, s,
                                              oracle.bd_seed(3, 0, s), pending=0)
    want = kT * 12.0 * 2.046167337 ** 2
    var = mom[:, :3].astype(np.float64).var(axis=0)
    assert np.allclose(var, want, rtol=0.08), (var, want)
