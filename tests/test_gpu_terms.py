"""The remaining terms of the path through the C ABI, against the fixture made
from the reference's own functors (tests/golden/make_golden.py, case
"terms"): analytical pair terms (Coulomb, Debye-Hueckel, Onck, Gaussian,
softcore, alone and combined with tables), tabulated dihedrals, harmonic
restraints and bonded rows of other forms; and the fused step with all of
them equal to the separate calls."""
import os

import numpy as np
import pytest
import torch

import pyoracle as po
from conftest import GOLDEN
from mars_md_b200 import _lib as L
from mars_md_b200 import engine as E
from mars_md_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5   # per-particle |df| / sum of |pair forces| on the particle
ENERGY_TOL = 1e-6  # |E - E_fp64| / sum |E_pair|


def _load():
    return np.load(os.path.join(GOLDEN, "terms.npz"))


def _cuda(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t.to(dtype) if dtype is not None else t).cuda()


def _tables(d, prefix="tab"):
    vals, sizes = d[f"{prefix}_values"], d[f"{prefix}_sizes"]
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
    return [(vals[o:o + s], float(a), float(b)) for o, s, a, b in
            zip(offs, sizes, d[f"{prefix}_starts"], d[f"{prefix}_step_invs"])]


def _box(d):
    return po.Box.make(d["box_origin"], d["box_size"], d["box_periodic"])


def _setup_pairs(ctx, d):
    ctx.set_box(d["box_origin"], d["box_size"], d["box_periodic"])
    ctx.set_pair_tables(4, d["term_matrix"], _tables(d))
    sv, g = d["solvent"], d["gaussian"]
    ctx.set_pair_terms(d["charge"], d["radius"], d["eps"], *[float(x) for x in sv],
                       *[float(x) for x in g])


def _oracle_pairs(oracle, d):
    box = _box(d)
    pairs, _, _ = oracle.build_pairlist(d["pos"], box, float(d["rc_list"]))
    p = np.sort(pairs.astype(np.int64), axis=1)
    pairs = np.ascontiguousarray(p[np.lexsort((p[:, 1], p[:, 0]))].astype(np.int32))
    tags = oracle.resolve_tags(pairs, d["type_ids"], d["term_matrix"], 4)
    pts = po.PairTermSet(d["charge"], d["radius"], d["eps"], d["solvent"], d["gaussian"])
    ts = po.TableSet(_tables(d))
    return oracle.pair_forces_terms(pairs, d["pos"], d["type_ids"], tags, ts, pts, box,
                                    np.float32(d["cutoff"]) ** 2)


def _force_err(f_gpu, f_ref, scale):
    dd = np.linalg.norm(f_gpu[:, :3].astype(np.float64) - f_ref[:, :3].astype(np.float64), axis=1)
    return float(np.max(dd / np.maximum(scale, 1e-30), initial=0.0))


@pytest.mark.parametrize("get_energy", [1, 0])
def test_analytical_pair_terms_match_reference_fixture(ctx_factory, oracle, get_energy):
    d = _load()
    n = len(d["pos"])
    ctx = ctx_factory(n)
    _setup_pairs(ctx, d)
    pos, types = _cuda(d["pos"]), _cuda(d["type_ids"])
    assert ctx.build_pairlist(pos, types, float(d["rc_list"])) == int(d["num_pairs"])
    fe = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    ctx.reset_energies()
    ctx.pair_forces(pos, types, fe, float(d["cutoff"]), get_energy=bool(get_energy))
    got = fe.cpu().numpy()
    _, fe64, fabs = _oracle_pairs(oracle, d)
    ref = d["pair_fe"] if get_energy else d["pair_fe_noe"]
    assert _force_err(got, ref, fabs) <= FORCE_TOL
    if get_energy:
        assert np.allclose(got[:, 3], ref[:, 3], rtol=1e-5, atol=1e-5)
        e_gpu = ctx.energy_terms()[0]
        e_ref = float(fe64[:, 3].sum())
        assert abs(e_gpu - e_ref) <= ENERGY_TOL * float(np.abs(fe64[:, 3]).sum())
    else:
        assert not got[:, 3].any()


def test_analytical_terms_need_their_constants(ctx_factory):
    d = _load()
    n = len(d["pos"])
    ctx = ctx_factory(n)
    ctx.set_box(d["box_origin"], d["box_size"], d["box_periodic"])
    ctx.set_pair_tables(4, d["term_matrix"], _tables(d))
    pos, types = _cuda(d["pos"]), _cuda(d["type_ids"])
    ctx.build_pairlist(pos, types, float(d["rc_list"]))
    fe = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(L.MB2Error):
        ctx.pair_forces(pos, types, fe, float(d["cutoff"]))
    b = E.Batch([100, 100], [(50.0,) * 3, (50.0,) * 3])
    with pytest.raises(L.MB2Error):
        b.set_pair_tables(4, d["term_matrix"], _tables(d))


def test_dihedrals_restraints_and_skipped_forms_match_reference_fixture(ctx_factory):
    d = _load()
    n = len(d["pos"])
    ctx = ctx_factory(n)
    ctx.set_box(d["box_origin"], d["box_size"], d["box_periodic"])
    ctx.set_bonded_tables(0, [(d["bond_values"], float(d["bond_start"]), float(d["bond_step_inv"]))])
    ctx.set_bonded_tables(1, [(d["angle_values"], float(d["angle_start"]),
                               float(d["angle_step_inv"]))])
    ctx.set_bonded_tables(2, _tables(d, "dih"))
    pos = _cuda(d["pos"])
    ctx.reset_energies()

    def run(fn, *args):
        fe = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        fn(*args, pos, fe)
        return fe.cpu().numpy()

    fd = run(ctx.dihedral_forces, _cuda(d["dihedrals"]), _cuda(d["dihedral_idx"]))
    ref = d["dihedral_fe"]
    scale = np.abs(ref[:, :3]).max()
    assert np.abs(fd[:, :3] - ref[:, :3]).max() <= 1e-5 * scale
    assert np.allclose(fd[:, 3], ref[:, 3], rtol=1e-5, atol=1e-6)
    fr = run(ctx.restraint_forces, _cuda(d["restraint_ids"]), _cuda(d["restraint_anchors"]),
             _cuda(d["restraint_k"]))
    assert np.allclose(fr, d["restraint_fe"], rtol=1e-6, atol=1e-6)
    fb = run(ctx.bond_forces, _cuda(d["bonds"]), _cuda(d["bond_idx"]))
    assert np.abs(fb - d["bond_fe"]).max() <= 1e-5 * np.abs(d["bond_fe"]).max()
    fa = run(ctx.angle_forces, _cuda(d["angles"]), _cuda(d["angle_idx"]))
    assert np.abs(fa - d["angle_fe"]).max() <= 1e-5 * np.abs(d["angle_fe"]).max()
    e = ctx.energy_terms()
    assert abs(e[4] - float(ref[:, 3].astype(np.float64).sum())) <= 1e-5 * abs(e[4])
    assert abs(e[5] - float(d["restraint_fe"][:, 3].astype(np.float64).sum())) <= 1e-5 * abs(e[5])


def test_fused_step_with_every_term_equals_separate_calls(ctx_factory):
    """mb2_step with analytical pairs, bonds, angles, dihedrals and restraints
    moves every particle as the separate stage calls plus mb2_bd_integrate."""
    d = _load()
    n = len(d["pos"])
    dev = {k: _cuda(d[k]) for k in ("type_ids", "bonds", "bond_idx", "angles", "angle_idx",
                                    "dihedrals", "dihedral_idx", "restraint_ids",
                                    "restraint_anchors", "restraint_k")}
    diffusion = np.full((4, 3), 150.0, np.float32)
    kT, dt, seed, step = 0.5862, 1e-4, 12345, 3

    def make():
        ctx = ctx_factory(n)
        _setup_pairs(ctx, d)
        ctx.set_bonded_tables(0, [(d["bond_values"], float(d["bond_start"]),
                                   float(d["bond_step_inv"]))])
        ctx.set_bonded_tables(1, [(d["angle_values"], float(d["angle_start"]),
                                   float(d["angle_step_inv"]))])
        ctx.set_bonded_tables(2, _tables(d, "dih"))
        ctx.set_particle_types(np.zeros(4, np.float32), diffusion)
        return ctx

    a = make()
    pos_a = _cuda(d["pos"])
    fe_a = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    flags = torch.zeros(n, dtype=torch.int32, device="cuda")
    p = L.StepParams()
    p.pairlist_cutoff, p.cutoff, p.rebuild_period = float(d["rc_list"]), float(d["cutoff"]), 20
    p.dt, p.kT, p.seed, p.get_energy = dt, kT, seed, 1
    p.bonds2, p.bond_table_idx, p.num_bonds = (dev["bonds"].data_ptr(),
                                               dev["bond_idx"].data_ptr(), len(d["bonds"]))
    p.angles4, p.angle_table_idx, p.num_angles = (dev["angles"].data_ptr(),
                                                  dev["angle_idx"].data_ptr(), len(d["angles"]))
    p.dihedrals4, p.dihedral_table_idx = dev["dihedrals"].data_ptr(), dev["dihedral_idx"].data_ptr()
    p.num_dihedrals = len(d["dihedrals"])
    p.restraint_ids, p.restraint_anchors4 = (dev["restraint_ids"].data_ptr(),
                                             dev["restraint_anchors"].data_ptr())
    p.restraint_k, p.num_restraints = dev["restraint_k"].data_ptr(), len(d["restraint_ids"])
    a.step(pos_a, fe_a, dev["type_ids"], flags, step, p)

    b = make()
    pos_b = _cuda(d["pos"])
    fe_b = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    b.build_pairlist(pos_b, dev["type_ids"], float(d["rc_list"]))
    b.pair_forces(pos_b, dev["type_ids"], fe_b, float(d["cutoff"]))
    b.bond_forces(dev["bonds"], dev["bond_idx"], pos_b, fe_b)
    b.angle_forces(dev["angles"], dev["angle_idx"], pos_b, fe_b)
    b.dihedral_forces(dev["dihedrals"], dev["dihedral_idx"], pos_b, fe_b)
    b.restraint_forces(dev["restraint_ids"], dev["restraint_anchors"], dev["restraint_k"], pos_b,
                       fe_b)
    b.bd_integrate(pos_b, fe_b, dev["type_ids"], flags, dt, kT, step, b.bd_seed(seed, 0, step))
    torch.cuda.synchronize()
    dp = np.abs(pos_a.cpu().numpy()[:, :3] - pos_b.cpu().numpy()[:, :3])
    dp = np.minimum(dp, np.abs(dp - float(d["box_size"][0])))
    assert dp.max() <= 1e-4
    moved = np.abs(pos_a.cpu().numpy()[:, :3] - d["pos"][:, :3]).max()
    assert moved > 1e-3
    # The adjoint window covers tabulated pair, bond and angle terms only.
    rc = a.lib.mb2_window_forward(a.h, E._p(pos_a), E._p(fe_a), E._p(dev["type_ids"]), n, 21, 20,
                                  20, po.C.byref(p), None)
    assert rc != 0 and b"tabulated" in a.lib.mb2_last_error(a.h)


def test_fused_langevin_step_equals_separate_calls(ctx_factory):
    """mb2_step with integrator = 1 (pair and bonded forces gathered into the
    BAOAB kernel, grid PMF, deferred closing kick) moves particles and momenta
    as mb2_pair_forces + bonded calls + mb2_baoab_integrate do."""
    w = W.polymers(n_chains=8, beads=256, with_grid=True)
    n = w.n
    mass = np.array([120.0, 80.0], np.float32)[:w.num_types]
    damping = np.full((w.num_types, 3), 40.0, np.float32)
    rng = np.random.default_rng(4)
    mom0 = np.zeros((n, 4), np.float32)
    mom0[:, :3] = rng.normal(0, 20, (n, 3)).astype(np.float32)

    def make():
        ctx = ctx_factory(n)
        dev = E.setup_workload(ctx, w)
        ctx.set_langevin_types(mass, damping)
        return ctx, dev

    a, da = make()
    mom_a = torch.from_numpy(mom0.copy()).cuda()
    p = E.step_params(w, bonds=da["bonds"], bond_idx=da["bond_idx"], angles=da["angles"],
                      angle_idx=da["angle_idx"])
    p.integrator, p.mom4 = 1, mom_a.data_ptr()
    b, db = make()
    mom_b = torch.from_numpy(mom0.copy()).cuda()
    for s in (1, 2):
        p.deferred_kick_pending = int(s > 1)
        a.step(da["pos"], da["fe"], da["type"], None, s, p)
        db["fe"].zero_()
        b.build_pairlist(db["pos"], db["type"], w.list_radius)
        b.pair_forces(db["pos"], db["type"], db["fe"], w.cutoff, get_energy=False)
        b.bond_forces(db["bonds"], db["bond_idx"], db["pos"], db["fe"], get_energy=False)
        b.angle_forces(db["angles"], db["angle_idx"], db["pos"], db["fe"], get_energy=False)
        b.baoab_integrate(db["pos"], mom_b, db["fe"], db["type"], None, w.dt, w.kT, s,
                          b.bd_seed(w.seed, 0, s), pending=s > 1)
    torch.cuda.synchronize()
    L = float(w.box_size[0])
    dp = np.abs(da["pos"].cpu().numpy()[:, :3] - db["pos"].cpu().numpy()[:, :3])
    dp = np.minimum(dp, L - dp)
    assert dp.max() <= 1e-4
    ma, mb = mom_a.cpu().numpy()[:, :3], mom_b.cpu().numpy()[:, :3]
    assert np.abs(ma - mb).max() <= 1e-4 * np.abs(mb).max()
    assert np.abs(ma - mom0[:, :3]).max() > 1.0  # the momenta did move
