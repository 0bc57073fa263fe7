"""The CPU oracle (oracle/mb2_oracle.c) against the reference's own outputs.

The golden fixtures in tests/golden were produced by the reference's functors
compiled for the host (tests/golden/make_golden.py). Integer and index work
must match bit for bit; the float kernels were restated with the reference's
operation order, so they must too. These tests pin the oracle; the GPU tests
then hold the CUDA path to the oracle.
"""
import os

import numpy as np
import pytest

import pyoracle as po
from conftest import GOLDEN


def _load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def _box(d):
    return po.Box.make(d["box_origin"], d["box_size"], d["box_periodic"])


def _tables(d):
    vals, sizes = d["tab_values"], d["tab_sizes"]
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
    return po.TableSet([(vals[o:o + s], float(a), float(b)) for o, s, a, b in
                        zip(offs, sizes, d["tab_starts"], d["tab_step_invs"])])


def _canon(pairs):
    p = np.sort(np.asarray(pairs, np.int64), axis=1)
    return np.ascontiguousarray(p[np.lexsort((p[:, 1], p[:, 0]))].astype(np.int32))


# --- Z-order sort ----------------------------------------------------------------------

def test_reorder_matches_reference(oracle):
    """Canonical reorder: permutation over the box bounds, gathered positions
    and remapped indices (with -1 and out-of-range entries) bit-exact."""
    d = _load("reorder")
    s2o, inv = oracle.reorder(_box(d), d["pos"])
    assert np.array_equal(s2o, d["s2o"])
    assert np.array_equal(inv, d["inverse"])
    assert np.array_equal(oracle.gather4(d["pos"], s2o), d["pos_after"])
    assert np.array_equal(oracle.remap_indices(d["indices"], inv), d["indices_after"])


def test_host_exclusion_csr_matches_oracle(oracle):
    """The host layer's exclusion CSR (engine.exclusion_csr, rebuilt after a
    reorder) equals the oracle's restatement word for word."""
    from mars_md_b200.engine import exclusion_csr
    d = _load("reorder")
    excl = d["inverse"].astype(np.int64)[d["exclusions"].astype(np.int64)]
    _, off, nb, npart = exclusion_csr(excl)
    o_off, o_nb, o_n = oracle.exclusion_csr(excl.astype(np.int32))
    assert npart == o_n
    assert np.array_equal(off, o_off[:npart + 1])
    assert np.array_equal(nb, o_nb[:len(nb)]) and len(nb) == 2 * len(excl)
    e0, off0, nb0, n0 = exclusion_csr(np.zeros((0, 2), np.int32))
    assert n0 == 0 and len(nb0) == 0


def test_reorder_cadence_and_original_order():
    from mars_md_b200.engine import ReorderManager, to_original_order
    m = ReorderManager(0, rebuild_period=20)
    assert [s for s in range(60) if m.should_reorder(s)] == [1, 21, 41]
    assert not ReorderManager(5).should_reorder(6, bonded_prepared=False)
    assert not ReorderManager(0, 0).should_reorder(1)
    d = _load("reorder")
    out = to_original_order(d["pos_after"], d["s2o"])
    assert np.array_equal(out, d["pos"])
    with pytest.raises(ValueError):
        to_original_order(d["pos_after"][:2], np.array([0, 5]))


@pytest.mark.parametrize("name", ["uniform4096", "lattice_open"])
def test_morton_sort_matches_reference(oracle, name):
    d = _load(name)
    s = oracle.sort_particles(_box(d), d["pos"])
    assert np.array_equal(s["keys"], d["keys"])
    assert np.array_equal(s["sorted_to_orig"], d["s2o"])
    if "inverse" in d:
        assert np.array_equal(s["inverse"], d["inverse"])
        assert np.array_equal(s["sorted_pos"], d["sorted_pos"])
        assert np.array_equal(s["bmin"], d["bmin"]) and np.array_equal(s["bmax"], d["bmax"])


def test_sort_is_stable_on_ties(oracle):
    keys = np.array([5, 1, 5, 0, 1, 5, 0], np.uint32)
    k, v = oracle.sort_pairs(keys, np.arange(7, dtype=np.uint32))
    assert k.tolist() == [0, 0, 1, 1, 5, 5, 5]
    assert v.tolist() == [3, 6, 1, 4, 0, 2, 5]


# --- pair sets -------------------------------------------------------------------------

def test_pair_set_uniform_matches_reference(oracle):
    d = _load("uniform4096")
    pairs, cnt, cs = oracle.build_pairlist(d["pos"], _box(d), float(d["rc_list"]))
    assert cnt == int(d["num_pairs"])
    assert cs == int(d["checksum"])
    assert np.array_equal(np.bincount(pairs.ravel(), minlength=len(d["pos"])), d["row_counts"])


def test_pair_set_lattice_matches_reference(oracle):
    d = _load("lattice_open")
    pairs, cnt, _ = oracle.build_pairlist(d["pos"], _box(d), float(d["rc_list"]))
    assert cnt == int(d["num_pairs"]) == 144
    assert np.array_equal(_canon(pairs), d["pairs"])
    # every pair is a nearest-neighbour bond of the 1.5 A lattice
    p = d["pos"][:, :3].astype(np.float64)
    dist = np.linalg.norm(p[pairs[:, 0]] - p[pairs[:, 1]], axis=1)
    assert np.allclose(dist, 1.5)


def test_pair_set_with_exclusions_matches_reference(oracle):
    d = _load("polymer_excl")
    off, nb, npart = oracle.exclusion_csr(d["exclusions"])
    pairs, cnt, cs = oracle.build_pairlist(d["pos"], _box(d), float(d["rc_list"]),
                                           excl=(off, nb, npart))
    assert cnt == int(d["num_pairs"])
    assert cs == int(d["checksum"])
    assert np.array_equal(np.bincount(pairs.ravel(), minlength=len(d["pos"])), d["row_counts"])
    # no excluded pair survives, and without exclusions there are exactly that many more
    ex = {tuple(sorted(e)) for e in d["exclusions"].tolist()}
    assert not any(tuple(p) in ex for p in _canon(pairs).tolist())
    _, cnt_all, _ = oracle.build_pairlist(d["pos"], _box(d), float(d["rc_list"]), want_pairs=False)
    assert cnt_all - cnt == len(ex)


# --- forces ----------------------------------------------------------------------------

def test_pair_forces_match_reference_bit_exact(oracle):
    d = _load("uniform4096")
    box = _box(d)
    pairs, _, _ = oracle.build_pairlist(d["pos"], box, float(d["rc_list"]))
    pairs = _canon(pairs)
    tags = oracle.resolve_tags(pairs, d["type_ids"], d["term_matrix"], 4)
    fe, fe64, _ = oracle.pair_forces(pairs, d["pos"], tags, _tables(d), box,
                                     np.float32(d["cutoff"]) ** 2)
    assert np.array_equal(fe, d["pair_fe"])
    # FP64 restatement agrees with the float result to float accuracy
    assert np.allclose(fe64[:, :3], fe[:, :3], rtol=1e-4, atol=1e-4)


def test_bond_and_angle_forces_match_reference_bit_exact(oracle):
    d = _load("polymer_excl")
    box = _box(d)
    bt = po.TableSet([(d["bond_values"], float(d["bond_start"]), float(d["bond_step_inv"]))])
    at = po.TableSet([(d["angle_values"], float(d["angle_start"]), float(d["angle_step_inv"]))],
                     periodic=True)
    fb, _, _ = oracle.bond_forces(d["bonds"], np.zeros(len(d["bonds"]), np.int32), d["pos"], bt, box)
    fa, _, _ = oracle.angle_forces(d["angles"], np.zeros(len(d["angles"]), np.int32), d["pos"], at,
                                   box)
    assert np.array_equal(fb, d["bond_fe"])
    assert np.array_equal(fa, d["angle_fe"])
    # momentum conservation of the bonded terms
    assert abs(fb[:, :3].astype(np.float64).sum(0)).max() < 1e-3
    assert abs(fa[:, :3].astype(np.float64).sum(0)).max() < 1e-3


def test_chain_end_forces(oracle):
    """Straight chain: interior beads feel no net bond force, the two ends feel
    the table force with opposite signs (the reference's BDKernels chain check)."""
    d = _load("chain129")
    bt = po.TableSet([(d["bond_values"], float(d["bond_start"]), float(d["bond_step_inv"]))])
    fb, _, _ = oracle.bond_forces(d["bonds"], np.zeros(len(d["bonds"]), np.int32), d["pos"], bt,
                                  _box(d))
    assert np.array_equal(fb, d["bond_fe"])
    assert np.abs(fb[1:-1, :3]).max() == 0.0
    assert fb[0, 0] == -fb[-1, 0] and fb[0, 0] < 0.0
    f_table, _ = oracle.table_lookup(bt, 0, 1.885)
    assert fb[-1, 0] == pytest.approx(f_table, rel=1e-6)


# --- Philox and BD ---------------------------------------------------------------------

def test_philox_matches_openrand(oracle):
    d = _load("philox")
    for (seed, ctr, gseed, ctr1), ints, floats in zip(d["cases"], d["ints"], d["floats"]):
        for k in range(len(ints)):
            u = oracle.philox(int(seed), int(ctr), int(ctr1), int(gseed), k)
            assert np.array_equal(u, ints[k])
            f = np.array([oracle.lib.or_u01(int(x)) for x in u], np.float32)
            assert np.array_equal(f, floats[k])


def test_bd_step_matches_reference(oracle):
    d = _load("uniform4096")
    ty = po.TypeSet(np.zeros(4, np.float32), d["diffusion"][:, :3])
    pos, fe, _ = oracle.bd_integrate(d["pos"], d["pair_fe"], d["type_ids"], None, ty, None, _box(d),
                                     float(d["dt"]), float(d["kT"]), int(d["bd_step"]),
                                     int(d["bd_seed"]))
    assert np.array_equal(pos, d["pos_after"])
    assert np.array_equal(fe, d["fe_after"])


def test_bd_step_with_grid_field_and_flags_matches_reference(oracle):
    d = _load("grid_bd")
    grids = po.GridSet([dict(data=d["grid"], origin=tuple(d["grid_origin"]),
                             basis=np.eye(3, dtype=np.float32), boundary_condition=0)])
    ty = po.TypeSet(d["charge"], d["diffusion"][:, :3],
                    [[(0, float(s), 0.0, -1)] for s in d["pmf_scale"]])
    pos, fe, _ = oracle.bd_integrate(d["pos"], d["fe"], d["type_ids"], d["flags"], ty, grids,
                                     _box(d), float(d["dt"]), float(d["kT"]), int(d["bd_step"]),
                                     int(d["bd_seed"]), efield=tuple(d["efield"]))
    assert np.array_equal(pos, d["pos_after"])
    assert np.array_equal(fe, d["fe_after"])
    frozen = d["flags"] != 0
    assert np.array_equal(pos[frozen], d["pos"][frozen])


# --- periodic box and table lookup -----------------------------------------------------

@pytest.mark.parametrize("tag,periodic", [("p", (1, 1, 1)), ("m", (1, 0, 1))])
def test_wrap_matches_reference(oracle, tag, periodic):
    d = _load("wrap_table")
    box = po.Box.make((-30.0, 10.0, 5.0), (200.0, 150.0, 300.0), periodic)
    v = np.ascontiguousarray(d["vec"])
    for fn, key in ((oracle.lib.or_wrap_diff, f"wrap_diff_{tag}"), (oracle.lib.or_wrap, f"wrap_{tag}")):
        out = np.zeros_like(v)
        fn(po.C.byref(box), v.ctypes.data, out.ctypes.data, len(v))
        assert np.array_equal(out[:, :3], d[key][:, :3]), key


def test_table_lookup_matches_reference(oracle):
    d = _load("wrap_table")
    pair = po.TableSet([(d["pair_values"], float(d["pair_start"]), float(d["pair_step_inv"]))])
    ang = po.TableSet([(d["angle_values"], float(d["angle_start"]), float(d["angle_step_inv"]))],
                      periodic=True)
    for tabs, xs, want in ((pair, d["pair_x"], d["pair_lookup"]),
                           (ang, d["angle_x"], d["angle_lookup"])):
        got = np.array([oracle.table_lookup(tabs, 0, float(x)) for x in xs], np.float32)
        assert np.array_equal(got, want)


def test_baoab_step_matches_reference(oracle):
    """Langevin BAOAB with the PMF pass and the deferred closing half-kick."""
    d = _load("baoab")
    grids = po.GridSet([dict(data=d["grid"], origin=tuple(d["grid_origin"]),
                             basis=np.eye(3, dtype=np.float32), boundary_condition=0)])
    ty = po.TypeSet(d["charge"], d["diffusion"][:, :3],
                    [[(0, float(s), 0.0, -1)] for s in d["pmf_scale"]])
    for pending in (0, 1):
        pos, mom, fe = oracle.baoab_integrate(
            d["pos"], d["mom"], d["fe"], d["type_ids"], d["flags"], ty, grids, d["mass"],
            d["damping"], _box(d), float(d["dt"]), float(d["kT"]), int(d["step"]),
            int(d["seed"]), efield=tuple(d["efield"]), pending=pending)
        assert np.array_equal(pos, d[f"pos_after_{pending}"])
        assert np.array_equal(mom, d[f"mom_after_{pending}"])
        assert np.array_equal(fe, d[f"fe_after_{pending}"])


# --- analytical pair terms, dihedrals, restraints, skipped forms ------------------------

def _terms_setup(oracle):
    d = _load("terms")
    box = _box(d)
    pairs, cnt, _ = oracle.build_pairlist(d["pos"], box, float(d["rc_list"]))
    pairs = _canon(pairs)
    tags = oracle.resolve_tags(pairs, d["type_ids"], d["term_matrix"], 4)
    pts = po.PairTermSet(d["charge"], d["radius"], d["eps"], d["solvent"], d["gaussian"])
    return d, box, pairs, tags, pts


def test_analytical_pair_terms_match_reference_bit_exact(oracle):
    """Coulomb, Debye-Hueckel, Onck, Gaussian, softcore and tables, alone and
    summed in one pair, with and without energy."""
    d, box, pairs, tags, pts = _terms_setup(oracle)
    assert len(pairs) == int(d["num_pairs"])
    assert oracle.pair_hash_sum(pairs) == int(d["checksum"])
    present = {int(t) & 0xFF for t in np.unique(tags)}
    assert {1, 2, 4, 8, 16, 32, 34, 25, 63} <= present
    cut2 = np.float32(d["cutoff"]) ** 2
    fe, _, _ = oracle.pair_forces_terms(pairs, d["pos"], d["type_ids"], tags, _tables(d), pts,
                                        box, cut2)
    assert np.array_equal(fe, d["pair_fe"])
    fe0, _, _ = oracle.pair_forces_terms(pairs, d["pos"], d["type_ids"], tags, _tables(d), pts,
                                         box, cut2, get_energy=False)
    assert np.array_equal(fe0, d["pair_fe_noe"])


def test_dihedral_and_restraint_forces_match_reference_bit_exact(oracle):
    d = _load("terms")
    box = _box(d)
    vals, sizes = d["dih_values"], d["dih_sizes"]
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
    dts = po.TableSet([(vals[o:o + s], float(a), float(b)) for o, s, a, b in
                       zip(offs, sizes, d["dih_starts"], d["dih_step_invs"])], periodic=True)
    fd, _, _ = oracle.dihedral_forces(d["dihedrals"], d["dihedral_idx"], d["pos"], dts, box)
    assert np.array_equal(fd, d["dihedral_fe"])
    fr, _, _ = oracle.restraint_forces(d["restraint_ids"], d["restraint_anchors"],
                                       d["restraint_k"], d["pos"], box)
    assert np.array_equal(fr, d["restraint_fe"])
    skipped = d["restraint_ids"] < 0
    assert skipped.any() and (d["dihedral_idx"] < 0).any()


def test_bonded_rows_of_other_forms_are_skipped(oracle):
    """Bond / angle rows whose form is not tabulated (index < 0) add nothing,
    as TabulatedBondComputer / TabulatedAngleComputer skip them."""
    d = _load("terms")
    box = _box(d)
    bts = po.TableSet([(d["bond_values"], float(d["bond_start"]), float(d["bond_step_inv"]))])
    fb, _, _ = oracle.bond_forces(d["bonds"], d["bond_idx"], d["pos"], bts, box)
    assert np.array_equal(fb, d["bond_fe"])
    ats = po.TableSet([(d["angle_values"], float(d["angle_start"]), float(d["angle_step_inv"]))],
                      periodic=True)
    fa, _, _ = oracle.angle_forces(d["angles"], d["angle_idx"], d["pos"], ats, box)
    assert np.array_equal(fa, d["angle_fe"])


# --- output ---------------------------------------------------------------------------

def test_dcd_reader_reads_reference_fixture():
    """The oracle's DCD reader against the reference DcdWriter's bytes: header
    counters after three frames, unit cells, frames."""
    import dcd
    d = _load("dcd")
    r = dcd.read_dcd(d["bytes_cell"].tobytes())
    assert (r["nfile"], r["npriv"], r["nsavc"], r["nstep"]) == (3, 10, 10, 30)
    assert r["delta"] == np.float32(0.1) and r["unitcell"] == 1 and r["version"] == 24
    assert r["natoms"] == 100
    assert r["titles"][0].startswith("REMARKS FILENAME=") and r["titles"][1].startswith("REMARKS DATE: ")
    assert np.array_equal(r["frames"], d["frames"][..., :3])
    assert np.array_equal(r["cells"], np.tile([60.0, 0.0, 70.0, 0.0, 0.0, 80.0], (3, 1)))
    r2 = dcd.read_dcd(d["bytes_nocell"].tobytes())
    assert (r2["nfile"], r2["nstep"], r2["unitcell"]) == (2, 20, 0) and len(r2["cells"]) == 0
