"""Generate the golden fixtures in this directory from the reference itself.

Every output here comes from the reference's own functors, compiled for the
host from the reference sources by ``oracle/ref_harness/Makefile`` into
``oracle/_ref/libmars_ref.so`` (MortonEncodeKernel, the CUB-equivalent stable
sort, BuildCellRanges/Neighbors + ZOrderCellNeighborKernel,
PairForceKernel/TabulatedPotential, BondComputer, BDIntegrate, openrand
Philox, PeriodicBox). Inputs are seeded synthetic data generated here and
stored beside the outputs, so the tests need neither this script nor the
reference checkout.

Run from the repository root, where the reference checkout is available:

    make -C oracle/ref_harness REF=<reference checkout> && python tests/golden/make_golden.py [case ...]

The fixtures pin the C restatement in ``oracle/`` (tests/test_oracle_golden.py)
and, through it, the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle as po  # noqa: E402
from mars_md_b200 import workloads as W  # noqa: E402

SEED = 20261203
FLAG_RB_ATTACHED = 4   # ParticleFlags bit that freezes a particle in BDIntegrate


def _tables_arrays(specs):
    ts = po.TableSet([(t.values, t.start, t.step_inv) for t in specs])
    return dict(tab_values=ts.values, tab_sizes=ts.sizes, tab_starts=ts.starts,
                tab_step_invs=ts.step_invs), ts


def _box_arrays(origin, size, periodic):
    return dict(box_origin=np.asarray(origin, np.float32), box_size=np.asarray(size, np.float32),
                box_periodic=np.asarray(periodic, np.int32))


def _pair_walk(O, R, pos, box, rc_list, excl=None, rigid=None):
    """Reference pair set: Morton sort + cell ranges + neighbour table + walk."""
    s = O.sort_particles(box, pos)
    keys_r, idx_r = R.morton_encode(pos, s["bmin"], s["bmax"])
    keys_r, s2o_r = R.sort_pairs(keys_r, idx_r)
    sp = R.reorder_pos(pos, s2o_r)
    ext = s["bmax"] - s["bmin"]
    m, radii, slots = O.select_cell_grid(ext, rc_list, len(pos), 1 << 40)
    shift = 3 * (10 - m)
    b, e = R.cell_ranges(keys_r, shift, 1 << (3 * m))
    bl = np.array(list(box.size), np.float32)
    table = R.cell_neighbors(m, radii, slots, bl)
    pairs, cnt = R.neighbor_walk(sp, keys_r, s2o_r, b, e, table, np.float32(rc_list) ** 2, slots,
                                 shift, box, excl=excl, rigid_body_id=rigid,
                                 max_pairs=len(pos) * 512)
    pairs = np.sort(pairs, axis=1)
    pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]
    return dict(bmin=s["bmin"], bmax=s["bmax"], keys=keys_r, s2o=s2o_r,
                inverse=R.inverse(s2o_r), sorted_pos=sp), np.ascontiguousarray(pairs), cnt


def _row_counts(pairs, n):
    return np.bincount(pairs.ravel(), minlength=n).astype(np.int32)


def uniform(O, R):
    """4,096 beads in a 200 A periodic box, 4 types, Debye-Hueckel + soft-core
    tables (400 bins over 30 A), cutoff 20 A, list radius 25 A; one BD step."""
    rng = np.random.default_rng(SEED)
    n, L = 4096, 200.0
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-100.0, 100.0, size=(n, 3)).astype(np.float32)
    types = (np.arange(n) % 4).astype(np.int32)
    charges = [1.0, -1.0, 1.0, -1.0]
    pairs_tt = [(a, b) for a in range(4) for b in range(a, 4)]
    specs = [W.dh_softcore_table(charges[a], charges[b]) for a, b in pairs_tt]
    index = {p: k for k, p in enumerate(pairs_tt)}
    term = W._term_matrix(4, lambda a, b: index[(a, b)])
    tab, ts = _tables_arrays(specs)
    box = po.Box.make((-100.0, -100.0, -100.0), (L, L, L))
    rc_list, cutoff = 25.0, 20.0
    sort, pairs, cnt = _pair_walk(O, R, pos, box, rc_list)
    tags = R.resolve_tags(pairs, types, term, 4)
    cutoff_sq = np.float32(cutoff) ** 2
    fe = R.pair_forces(pairs, pos, types, tags, ts, box, cutoff_sq)
    ty = po.TypeSet(np.zeros(4, np.float32), np.full((4, 3), W.DIFFUSION, np.float32))
    step = 7
    seed = O.bd_seed(SEED, 0, step)
    pos1, fe1 = R.bd_integrate(pos, fe, types, None, ty, None, box, W.DT_NS, W.kT(), step, seed)
    return dict(pos=pos, type_ids=types, term_matrix=term, rc_list=np.float32(rc_list),
                cutoff=np.float32(cutoff), **tab, **_box_arrays(box.origin, box.size, box.periodic),
                **sort, num_pairs=np.int64(cnt), checksum=np.uint64(O.pair_hash_sum(pairs)),
                row_counts=_row_counts(pairs, n), pair_fe=fe, bd_step=np.int64(step),
                bd_seed=np.uint64(seed), dt=np.float32(W.DT_NS), kT=np.float32(W.kT()),
                diffusion=ty.diffusion4, pos_after=pos1, fe_after=fe1)


def lattice(O, R):
    """4 x 4 x 4 lattice, 1.5 A spacing, open box, list radius 2 A: the 144
    nearest-neighbour pairs (the reference's own lattice check)."""
    g = np.arange(4, dtype=np.float32) * np.float32(1.5)
    xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    pos = np.zeros((64, 4), np.float32)
    pos[:, :3] = xyz
    box = po.Box.make((0.0, 0.0, 0.0), (100.0, 100.0, 100.0), (0, 0, 0))
    sort, pairs, cnt = _pair_walk(O, R, pos, box, 2.0)
    return dict(pos=pos, rc_list=np.float32(2.0), **_box_arrays(box.origin, box.size, box.periodic),
                keys=sort["keys"], s2o=sort["s2o"], pairs=pairs.astype(np.int32),
                num_pairs=np.int64(cnt))


def polymer(O, R):
    """8 chains x 64 beads (bond 5 A) in a 120 A periodic box, two types,
    1-2 and 1-3 exclusions, harmonic bond and angle tables."""
    rng = np.random.default_rng(SEED + 1)
    nch, beads, L = 8, 64, 120.0
    xyz = W._chains(rng, nch, beads, L)
    pos = np.zeros((nch * beads, 4), np.float32)
    pos[:, :3] = xyz.astype(np.float32)
    n = len(pos)
    bonds, angles, excl = W._topology(nch, beads)
    off, nb, npart = O.exclusion_csr(excl)
    box = po.Box.make((0.0, 0.0, 0.0), (L, L, L))
    sort, pairs, cnt = _pair_walk(O, R, pos, box, 25.0, excl=(off, nb, npart))
    btab, bts = _tables_arrays([W.harmonic_bond_table()])
    atab_spec = [W.harmonic_angle_table(k=5.0, theta0_deg=120.0)]
    ats = po.TableSet([(t.values, t.start, t.step_inv) for t in atab_spec], periodic=True)
    bidx = np.zeros(len(bonds), np.int32)
    aidx = np.zeros(len(angles), np.int32)
    fb = R.bond_forces(bonds, bidx, pos, bts, box)
    fa = R.angle_forces(angles, aidx, pos, ats, box)
    return dict(pos=pos, rc_list=np.float32(25.0), **_box_arrays(box.origin, box.size, box.periodic),
                exclusions=excl, num_pairs=np.int64(cnt),
                checksum=np.uint64(O.pair_hash_sum(pairs)), row_counts=_row_counts(pairs, n),
                bonds=bonds, angles=angles, bond_values=bts.values,
                bond_start=np.float32(bts.starts[0]), bond_step_inv=np.float32(bts.step_invs[0]),
                angle_values=ats.values, angle_start=np.float32(ats.starts[0]),
                angle_step_inv=np.float32(ats.step_invs[0]), bond_fe=fb, angle_fe=fa)


def chain(O, R):
    """129-bead straight chain at 1.885 A spacing with a harmonic bond table
    (k = 19.19 kcal/mol/A^2, r0 = 3.8 A): end beads carry the table force with
    opposite signs, interior beads none."""
    n = 129
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = (np.arange(n) * 1.885).astype(np.float32)
    box = po.Box.make((-50.0, -50.0, -50.0), (400.0, 400.0, 400.0), (0, 0, 0))
    spec = W.harmonic_bond_table(k=19.19, r0=3.8, bins=200, dx=0.05)
    bts = po.TableSet([(spec.values, spec.start, spec.step_inv)])
    bonds = np.stack([np.arange(n - 1), np.arange(1, n)], axis=1).astype(np.int32)
    fb = R.bond_forces(bonds, np.zeros(n - 1, np.int32), pos, bts, box)
    return dict(pos=pos, **_box_arrays(box.origin, box.size, box.periodic), bonds=bonds,
                bond_values=bts.values, bond_start=np.float32(bts.starts[0]),
                bond_step_inv=np.float32(bts.step_invs[0]), bond_fe=fb)


def philox(O, R):
    """openrand Philox draws: integers and Box-Muller-ready floats."""
    cases = np.array([[123456789012345, 7, 3, 0x5324120], [0, 0, 0, 0],
                      [0xFFFFFFFFFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF],
                      [O.bd_seed(SEED, 2, 11), 1000, 0x5324120, 11]], dtype=np.uint64)
    ints = np.stack([R.philox_int4(int(s), int(c), int(g), int(c1), 4) for s, c, g, c1 in cases])
    floats = np.stack([R.philox_float4(int(s), int(c), int(g), int(c1), 4)
                       for s, c, g, c1 in cases])
    return dict(cases=cases, ints=ints, floats=floats)


def grid_bd(O, R):
    """2,048 beads in a 64 A periodic box, two types with a PMF from one
    32^3 grid (1 A spacing, centred), charges under an electric field, a few
    beads frozen by the rigid-body flag; one BD step."""
    rng = np.random.default_rng(SEED + 2)
    n, L = 2048, 64.0
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0.0, L, size=(n, 3)).astype(np.float32)
    types = rng.integers(0, 2, size=n).astype(np.int32)
    c = np.arange(32, dtype=np.float64)
    gx, gy, gz = np.meshgrid(c, c, c, indexing="ij")
    data = (2.0 * np.sin(gx / 5.0) * np.cos(gy / 7.0) + 0.05 * (gz - 16.0) ** 2).astype(np.float32)
    grids = [dict(data=data, origin=(16.0, 16.0, 16.0), basis=np.eye(3, dtype=np.float32),
                  boundary_condition=0)]
    gs = po.GridSet(grids)
    ty = po.TypeSet(np.array([0.5, -1.0], np.float32),
                    np.array([[150.0, 150.0, 150.0], [80.0, 90.0, 100.0]], np.float32),
                    [[(0, 1.0, 0.0, -1)], [(0, 1.5, 0.0, -1)]])
    fe = np.zeros((n, 4), np.float32)
    fe[:, :3] = rng.normal(0.0, 2.0, size=(n, 3)).astype(np.float32)
    flags = np.zeros(n, np.uint32)
    flags[::97] = FLAG_RB_ATTACHED
    box = po.Box.make((0.0, 0.0, 0.0), (L, L, L))
    efield = (0.0, 0.0, 0.1)
    step = 3
    seed = O.bd_seed(SEED, 1, step)
    pos1, fe1 = R.bd_integrate(pos, fe, types, flags, ty, gs, box, W.DT_NS, W.kT(), step, seed,
                               efield=efield)
    return dict(pos=pos, fe=fe, type_ids=types, flags=flags, grid=data,
                grid_origin=np.float32([16.0, 16.0, 16.0]), charge=ty.charge,
                diffusion=ty.diffusion4, pmf_scale=np.float32([1.0, 1.5]),
                efield=np.float32(efield), bd_step=np.int64(step), bd_seed=np.uint64(seed),
                dt=np.float32(W.DT_NS), kT=np.float32(W.kT()),
                **_box_arrays(box.origin, box.size, box.periodic), pos_after=pos1, fe_after=fe1)


def wrap_table(O, R):
    """PeriodicBox wrap/wrap_diff and TabulatedPotential lookups at edge cases."""
    rng = np.random.default_rng(SEED + 3)
    v = np.zeros((512, 4), np.float32)
    v[:, :3] = rng.uniform(-700.0, 700.0, size=(512, 3)).astype(np.float32)
    v[:8, :3] = np.float32([[100.0, -100.0, 50.0], [-50.0, 49.999996, 150.0], [0, 0, 0],
                            [300.0, -300.0, 1e-7], [99.99999, 100.00001, -100.0],
                            [450.0, -250.0, 250.0], [-0.0, 0.0, 200.0], [650.0, 0.25, -650.0]])
    out = {}
    for tag, per in (("p", (1, 1, 1)), ("m", (1, 0, 1))):
        box = po.Box.make((-30.0, 10.0, 5.0), (200.0, 150.0, 300.0), per)
        out[f"wrap_diff_{tag}"] = R.wrap_diff(box, v)
        out[f"wrap_{tag}"] = R.wrap(box, v)
    pair = W.dh_softcore_table(1.0, -1.0)
    ang = W.harmonic_angle_table(k=5.0, theta0_deg=120.0)
    xs_pair = np.float32(np.concatenate([[-1.0, 0.0, 1e-6, 0.0749, 0.075, 29.9, 29.925, 29.95,
                                          30.0, 45.0], rng.uniform(0.0, 30.0, 54)]))
    xs_ang = np.float32(np.concatenate([[-0.1, 0.0, math.pi - 1e-4, math.pi, 3.2, 2 * math.pi,
                                         7.0, -3.0], rng.uniform(-7.0, 7.0, 56)]))
    lib = R.lib
    lib.ref_table_lookup.argtypes = [C.c_float, C.c_void_p, C.c_uint32, C.c_float, C.c_float,
                                     C.c_int, C.c_void_p]

    def lookup(spec, xs, periodic):
        vals = np.ascontiguousarray(spec.values, np.float32)
        res = np.zeros((len(xs), 2), np.float32)
        for k, x in enumerate(xs):
            o = np.zeros(2, np.float32)
            lib.ref_table_lookup(C.c_float(float(x)), vals.ctypes.data, len(vals),
                                 C.c_float(spec.start), C.c_float(spec.step_inv), int(periodic),
                                 o.ctypes.data)
            res[k] = o
        return res

    return dict(vec=v, **out, pair_values=pair.values, pair_start=np.float32(pair.start),
                pair_step_inv=np.float32(pair.step_inv), pair_x=xs_pair,
                pair_lookup=lookup(pair, xs_pair, False), angle_values=ang.values,
                angle_start=np.float32(ang.start), angle_step_inv=np.float32(ang.step_inv),
                angle_x=xs_ang, angle_lookup=lookup(ang, xs_ang, True))


def baoab(O, R):
    """One Langevin BAOAB step (BAOABIntegrate, with the PMF pass and the
    deferred closing half-kick of Patch::integrate_motion) on 3,000 particles of
    two types with masses and per-axis damping, a 32^3 PMF grid, an electric
    field and frozen particles; once with and once without a pending kick."""
    rng = np.random.default_rng(SEED + 4)
    n, L = 3000, 64.0
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0.0, L, size=(n, 3)).astype(np.float32)
    mom = np.zeros((n, 4), np.float32)
    mom[:, :3] = rng.normal(0.0, 5.0, size=(n, 3)).astype(np.float32)
    fe = np.zeros((n, 4), np.float32)
    fe[:, :3] = rng.normal(0.0, 2.0, size=(n, 3)).astype(np.float32)
    types = rng.integers(0, 2, size=n).astype(np.int32)
    c = np.arange(32, dtype=np.float64)
    gx, gy, gz = np.meshgrid(c, c, c, indexing="ij")
    data = (2.0 * np.sin(gx / 5.0) * np.cos(gy / 7.0) + 0.05 * (gz - 16.0) ** 2).astype(np.float32)
    gs = po.GridSet([dict(data=data, origin=(16.0, 16.0, 16.0), basis=np.eye(3, dtype=np.float32),
                          boundary_condition=0)])
    ty = po.TypeSet(np.array([0.5, -1.0], np.float32),
                    np.array([[150.0, 150.0, 150.0], [80.0, 90.0, 100.0]], np.float32),
                    [[(0, 1.0, 0.0, -1)], [(0, 1.5, 0.0, -1)]])
    mass = np.array([12.0, 40.0], np.float32)
    damping = np.array([[50.0, 50.0, 50.0], [20.0, 30.0, 40.0]], np.float32)
    flags = np.zeros(n, np.uint32)
    flags[::97] = FLAG_RB_ATTACHED
    box = po.Box.make((0.0, 0.0, 0.0), (L, L, L))
    efield = (0.0, 0.0, 0.1)
    step = 5
    seed = O.bd_seed(SEED, 0, step)
    out = {}
    for pending in (0, 1):
        p1, m1, f1 = R.baoab_integrate(pos, mom, fe, types, flags, ty, gs, mass, damping, box,
                                       W.DT_NS, W.kT(), step, seed, efield=efield, pending=pending)
        out.update({f"pos_after_{pending}": p1, f"mom_after_{pending}": m1,
                    f"fe_after_{pending}": f1})
    return dict(pos=pos, mom=mom, fe=fe, type_ids=types, flags=flags, grid=data,
                grid_origin=np.float32([16.0, 16.0, 16.0]), charge=ty.charge,
                diffusion=ty.diffusion4, pmf_scale=np.float32([1.0, 1.5]), mass=mass,
                damping=damping, efield=np.float32(efield), step=np.int64(step),
                seed=np.uint64(seed), dt=np.float32(W.DT_NS), kT=np.float32(W.kT()),
                **_box_arrays(box.origin, box.size, box.periodic), **out)


def reorder(O, R):
    """Canonical Morton reorder of a bonded system (8 chains x 64 beads, two
    types, periodic 120 A box with origin -60 A): the permutation, the
    permuted positions and the remapped bond / angle indices from the
    reference's MortonEncodeKernel over the box, stable sort, InverseIndexKernel,
    ReorderDataKernel and RemapIndicesKernel. The index arrays carry -1 and
    out-of-range entries, which the remap leaves alone."""
    rng = np.random.default_rng(SEED + 7)
    nch, beads, L = 8, 64, 120.0
    xyz = W._chains(rng, nch, beads, L) - L / 2
    n = nch * beads
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = xyz.astype(np.float32)
    pos[:, 3] = rng.integers(0, 2, n).astype(np.float32)
    bonds, angles, excl = W._topology(nch, beads)
    extra = np.array([[-1, 3], [n, 5], [7, n + 100]], np.int32)
    idx_in = np.concatenate([bonds.reshape(-1), angles.reshape(-1), extra.reshape(-1)])
    origin, size = np.full(3, -L / 2, np.float32), np.full(3, L, np.float32)
    bmax = (origin + size).astype(np.float32)
    keys, idx = R.morton_encode(pos, origin, bmax)
    keys, s2o = R.sort_pairs(keys, idx)
    inv = R.inverse(s2o)
    return dict(pos=pos, **_box_arrays(origin, size, (1, 1, 1)), bonds=bonds, angles=angles,
                exclusions=excl, indices=idx_in, keys=keys, s2o=s2o, inverse=inv,
                pos_after=R.reorder_pos(pos, s2o), indices_after=R.remap_indices(idx_in, inv),
                rc_list=np.float32(25.0))


def _dihedral_table(k=2.0, mult=3, delta=0.3, bins=72):
    """Periodic cosine dihedral table on [-pi, pi): U = k (1 + cos(n phi - delta));
    step_inv as the bonded tables compute it, float(1 / double(step))."""
    step = 2.0 * math.pi / bins
    x = -math.pi + np.arange(bins) * step
    u = (k * (1.0 + np.cos(mult * x - delta))).astype(np.float32)
    return u, np.float32(-math.pi), np.float32(1.0 / step)


def terms(O, R):
    """Every remaining term on the path: analytical pair terms (Coulomb,
    Debye-Hueckel, Onck, Gaussian, softcore, alone and combined with each
    other and with tables), tabulated dihedrals (periodic tables, degenerate
    and wrapped quadruples, skipped rows), harmonic restraints (anchors across
    the boundary, skipped ids) and bonds / angles whose form is not tabulated.
    14^3 = 2,744 beads, 4 types, jittered lattice in a 60 A periodic box. The
    pair list (12 A) is the canonical sorted list, rebuilt by the tests."""
    rng = np.random.default_rng(SEED + 11)
    m, L = 14, 60.0
    a = L / m
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1)
    g = g.reshape(-1, 3)
    n = len(g)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = ((g + 0.5) * a + rng.uniform(-0.8, 0.8, size=(n, 3)) - L / 2).astype(np.float32)
    types = rng.integers(0, 4, n).astype(np.int32)
    charge = np.array([1.0, -1.0, 0.5, -0.25], np.float32)
    radius = np.array([2.0, 2.5, 3.0, 1.5], np.float32)
    eps = np.array([0.5, 0.3, 0.2, 0.4], np.float32)
    solvent = np.array([8.0, 78.5, 0.12, 78.0, 6.0], np.float32)
    gaussian = np.array([1.0, 1.0, 0.0], np.float32)
    # term bits: 1 Coulomb, 2 Debye-Hueckel, 4 Onck, 8 Gaussian, 16 softcore, 32 table
    tag = {(0, 0): 1, (0, 1): 2, (0, 2): 4, (0, 3): 8, (1, 1): 16, (1, 2): 32 | (0 << 8),
           (1, 3): 2 | 32 | (1 << 8), (2, 2): 1 | 8 | 16, (2, 3): 31 | 32 | (1 << 8), (3, 3): 0}
    term = np.zeros(16, np.uint32)
    for (x, y), t in tag.items():
        term[x * 4 + y] = term[y * 4 + x] = t
    tab, ts = _tables_arrays([W.wca_table(sigma=3.0), W.dh_softcore_table(1.0, -0.25, rmax=20.0)])
    box = po.Box.make((-L / 2,) * 3, (L, L, L))
    rc_list, cutoff = 12.0, 10.0
    _, pairs, _ = _pair_walk(O, R, pos, box, rc_list)
    tags = R.resolve_tags(pairs, types, term, 4)
    pts = po.PairTermSet(charge, radius, eps, solvent, gaussian)
    cutoff_sq = np.float32(cutoff) ** 2
    pair_fe = R.pair_forces_terms(pairs, pos, types, tags, ts, pts, box, cutoff_sq)
    pair_fe_noe = R.pair_forces_terms(pairs, pos, types, tags, ts, pts, box, cutoff_sq,
                                      get_energy=False)

    def idx(x, y, z):
        return ((x % m) * m + (y % m)) * m + (z % m)
    quads = []
    for x in range(m):
        for y in range(0, m, 2):
            for z in range(0, m, 3):
                quads.append((idx(x, y, z), idx(x + 1, y, z), idx(x + 1, y + 1, z),
                              idx(x + 1, y + 1, z + 1)))
    for x in range(0, m, 2):          # nearly collinear rows: the degenerate branch
        quads.append((idx(x, 0, 0), idx(x + 1, 0, 0), idx(x + 2, 0, 0), idx(x + 3, 0, 0)))
    dih = np.array(quads, np.int32)
    d_idx = (np.arange(len(dih)) % 2).astype(np.int32)
    d_idx[::17] = -1
    dtabs = [_dihedral_table(), _dihedral_table(k=1.0, mult=1, delta=-1.2, bins=36)]
    dts = po.TableSet(dtabs, periodic=True)
    dih_fe = R.dihedral_forces(dih, d_idx, pos, dts, box)

    nr = 400
    rid = rng.choice(n, nr, replace=False).astype(np.int32)
    rid[::23] = -1
    anchors = np.zeros((nr, 4), np.float32)
    anchors[:, :3] = (pos[np.maximum(rid, 0), :3] + rng.uniform(-3, 3, (nr, 3))).astype(np.float32)
    anchors[:10, :3] = (anchors[:10, :3] + L * 0.97).astype(np.float32)  # across the boundary
    rk = rng.uniform(0.5, 5.0, nr).astype(np.float32)
    rest_fe = R.restraint_forces(rid, anchors, rk, pos, box)

    bonds = np.array([(idx(x, y, z), idx(x, y, z + 1)) for x in range(m) for y in range(m)
                      for z in range(m - 1)], np.int32)
    b_idx = np.zeros(len(bonds), np.int32)
    b_idx[::5] = -1
    bspec = W.harmonic_bond_table(r0=4.3)
    bts = po.TableSet([(bspec.values, bspec.start, bspec.step_inv)])
    bond_fe = R.bond_forces(bonds, b_idx, pos, bts, box)
    angles = np.array([(idx(x, y, z), idx(x, y, z + 1), idx(x, y + 1, z + 1), 0)
                       for x in range(m) for y in range(m) for z in range(0, m, 2)], np.int32)
    a_idx = np.zeros(len(angles), np.int32)
    a_idx[::7] = -1
    aspec = W.harmonic_angle_table(k=5.0, theta0_deg=90.0)
    ats = po.TableSet([(aspec.values, aspec.start, aspec.step_inv)], periodic=True)
    angle_fe = R.angle_forces(angles, a_idx, pos, ats, box)
    return dict(pos=pos, type_ids=types, term_matrix=term, **tab, charge=charge, radius=radius,
                eps=eps, solvent=solvent, gaussian=gaussian,
                **_box_arrays(box.origin, box.size, box.periodic), rc_list=np.float32(rc_list),
                cutoff=np.float32(cutoff), num_pairs=np.int64(len(pairs)),
                checksum=np.uint64(O.pair_hash_sum(pairs)), pair_fe=pair_fe,
                pair_fe_noe=pair_fe_noe, dihedrals=dih, dihedral_idx=d_idx,
                dih_values=dts.values, dih_sizes=dts.sizes, dih_starts=dts.starts,
                dih_step_invs=dts.step_invs, dihedral_fe=dih_fe, restraint_ids=rid,
                restraint_anchors=anchors, restraint_k=rk, restraint_fe=rest_fe, bonds=bonds,
                bond_idx=b_idx, bond_values=bts.values, bond_start=np.float32(bts.starts[0]),
                bond_step_inv=np.float32(bts.step_invs[0]), bond_fe=bond_fe, angles=angles,
                angle_idx=a_idx, angle_values=ats.values, angle_start=np.float32(ats.starts[0]),
                angle_step_inv=np.float32(ats.step_invs[0]), angle_fe=angle_fe)


def dcd(O, R):
    """DCD files from the reference's own DcdWriter: 3 frames of 100 beads,
    output period 10, timestep 0.1, with the unit cell of a 60 x 70 x 80 A
    box; and 2 frames without a unit cell. The two title lines carry the
    file name and the date, which differ between writers."""
    import tempfile
    rng = np.random.default_rng(SEED + 13)
    frames = np.zeros((3, 100, 4), np.float32)
    frames[..., :3] = rng.uniform(-30, 30, (3, 100, 3)).astype(np.float32)
    out = dict(frames=frames, nsavc=np.int32(10), delta=np.float32(0.1),
               box=np.array([60.0, 70.0, 80.0], np.float32))
    with tempfile.TemporaryDirectory() as d:
        for tag, cell, nf in (("cell", 1, 3), ("nocell", 0, 2)):
            path = os.path.join(d, f"{tag}.dcd")
            R.dcd_write(path, frames[:nf], 10, 0.1, cell, out["box"])
            out[f"bytes_{tag}"] = np.frombuffer(open(path, "rb").read(), np.uint8)
    return out


CASES = {"uniform4096": uniform, "lattice_open": lattice, "polymer_excl": polymer,
         "chain129": chain, "philox": philox, "grid_bd": grid_bd, "wrap_table": wrap_table,
         "baoab": baoab, "reorder": reorder, "terms": terms,
         "dcd": dcd}


def main():
    if not po.ref_available():
        sys.exit("reference harness not built: make -C oracle/ref_harness REF=<reference checkout>")
    O, R = po.Oracle(), po.RefHarness()
    names = sys.argv[1:] or list(CASES)
    for name in names:
        fn = CASES[name]
        data = fn(O, R)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{name}: {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
