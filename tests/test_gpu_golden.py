"""The CUDA path against the golden fixtures made from the reference's own
host-compiled functors (tests/golden/make_golden.py), through the C ABI:
Morton keys and permutation bit-exact, pair sets identical (with exclusions,
on a periodic box and an open-box lattice), Philox words bit-exact, pair /
bond / angle forces and a BD step with a grid, a field and frozen particles
within the force and position tolerances of the other GPU tests."""
import os

import numpy as np
import pytest
import torch

import pyoracle as po
from conftest import GOLDEN, u32

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5   # per-particle |df| / sum of |pair forces| on the particle
POS_TOL = 1e-4     # A, after one BD step (device vs host libm transcendentals)


def _load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def _cuda(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t.to(dtype) if dtype is not None else t).cuda()


def _box(ctx, d):
    ctx.set_box(d["box_origin"], d["box_size"], d["box_periodic"])


def _pairs_of(ctx):
    p = ctx.export_pairs().cpu().numpy().astype(np.int64)
    p = np.sort(p, axis=1)
    return p[np.lexsort((p[:, 1], p[:, 0]))] if len(p) else p.reshape(0, 2)


def _tables(d):
    vals, sizes = d["tab_values"], d["tab_sizes"]
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
    return [(vals[o:o + s], float(a), float(b)) for o, s, a, b in
            zip(offs, sizes, d["tab_starts"], d["tab_step_invs"])]


def test_sort_matches_reference_fixture(ctx_factory):
    d = _load("uniform4096")
    ctx = ctx_factory(len(d["pos"]))
    keys, s2o, inv, sp = ctx.sort_morton(_cuda(d["pos"]), d["bmin"], d["bmax"])
    torch.cuda.synchronize()
    assert np.array_equal(u32(keys), d["keys"])
    assert np.array_equal(u32(s2o), d["s2o"])
    assert np.array_equal(u32(inv), d["inverse"])
    assert np.array_equal(sp.cpu().numpy(), d["sorted_pos"])


def test_pair_sets_match_reference_fixtures(ctx_factory, oracle):
    d = _load("uniform4096")
    ctx = ctx_factory(len(d["pos"]))
    _box(ctx, d)
    n = ctx.build_pairlist(_cuda(d["pos"]), _cuda(d["type_ids"]), float(d["rc_list"]))
    p = _pairs_of(ctx)
    assert n == int(d["num_pairs"])
    assert oracle.pair_hash_sum(p) == int(d["checksum"])
    assert np.array_equal(np.bincount(p.ravel(), minlength=len(d["pos"])), d["row_counts"])

    lat = _load("lattice_open")
    ctx2 = ctx_factory(64)
    _box(ctx2, lat)
    ctx2.build_pairlist(_cuda(lat["pos"]), _cuda(np.zeros(64, np.int32)), float(lat["rc_list"]))
    assert np.array_equal(_pairs_of(ctx2), lat["pairs"].astype(np.int64))

    poly = _load("polymer_excl")
    n3 = len(poly["pos"])
    off, nb, npart = oracle.exclusion_csr(poly["exclusions"])
    ctx3 = ctx_factory(n3)
    _box(ctx3, poly)
    doff, dnb = _cuda(off), _cuda(nb)
    ctx3.set_exclusions(doff, dnb, npart)
    m = ctx3.build_pairlist(_cuda(poly["pos"]), _cuda(np.zeros(n3, np.int32)),
                            float(poly["rc_list"]))
    p3 = _pairs_of(ctx3)
    assert m == int(poly["num_pairs"])
    assert oracle.pair_hash_sum(p3) == int(poly["checksum"])


def _force_err(f_gpu, f_ref, scale):
    d = np.linalg.norm(f_gpu[:, :3].astype(np.float64) - f_ref[:, :3].astype(np.float64), axis=1)
    return float(np.max(d / np.maximum(scale, 1e-30), initial=0.0))


def test_pair_forces_match_reference_fixture(ctx_factory, oracle):
    d = _load("uniform4096")
    n = len(d["pos"])
    ctx = ctx_factory(n)
    _box(ctx, d)
    ctx.set_pair_tables(4, d["term_matrix"], _tables(d))
    pos, types = _cuda(d["pos"]), _cuda(d["type_ids"])
    ctx.build_pairlist(pos, types, float(d["rc_list"]))
    fe = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    ctx.pair_forces(pos, types, fe, float(d["cutoff"]), get_energy=True)
    got = fe.cpu().numpy()
    # Scale: sum of |pair force| per particle (the oracle's FP64 restatement).
    pairs, _, _ = oracle.build_pairlist(d["pos"], po.Box.make(d["box_origin"], d["box_size"],
                                                              d["box_periodic"]),
                                        float(d["rc_list"]))
    ts = po.TableSet(_tables(d))
    tags = oracle.resolve_tags(pairs, d["type_ids"], d["term_matrix"], 4)
    _, _, fabs = oracle.pair_forces(pairs, d["pos"], tags, ts,
                                    po.Box.make(d["box_origin"], d["box_size"], d["box_periodic"]),
                                    np.float32(d["cutoff"]) ** 2)
    assert _force_err(got, d["pair_fe"], fabs) <= FORCE_TOL
    assert np.allclose(got[:, 3], d["pair_fe"][:, 3], rtol=1e-5, atol=1e-6)


def test_pair_forces_nonuniform_tables_match_oracle(ctx_factory, oracle):
    """The fixture's positions and tags with tables of different lengths,
    starts and bin widths (the kernel's general table path; uniform tables
    take a path that reads only each type pair's offset) against the FP64
    restatement, forces and energies."""
    d = _load("uniform4096")
    n = len(d["pos"])
    base = _tables(d)
    tabs = []
    for k, (vals, start, sinv) in enumerate(base):
        m = len(vals) - 23 * k                  # 400, 377, ... bins
        step = (1.0 / sinv) * (1.0 + 0.05 * k)  # wider bins for later tables
        r = start + 0.25 * k + step * np.arange(m)
        tabs.append((np.interp(r, start + np.arange(len(vals)) / sinv, vals).astype(np.float32),
                     float(np.float32(start + 0.25 * k)), float(np.float32(1.0 / step))))
    ctx = ctx_factory(n)
    _box(ctx, d)
    ctx.set_pair_tables(4, d["term_matrix"], tabs)
    pos, types = _cuda(d["pos"]), _cuda(d["type_ids"])
    ctx.build_pairlist(pos, types, float(d["rc_list"]))
    fe = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    ctx.pair_forces(pos, types, fe, float(d["cutoff"]), get_energy=True)
    got = fe.cpu().numpy()
    box = po.Box.make(d["box_origin"], d["box_size"], d["box_periodic"])
    pairs, _, _ = oracle.build_pairlist(d["pos"], box, float(d["rc_list"]))
    tags = oracle.resolve_tags(pairs, d["type_ids"], d["term_matrix"], 4)
    _, f64, fabs = oracle.pair_forces(pairs, d["pos"], tags, po.TableSet(tabs), box,
                                      np.float32(d["cutoff"]) ** 2)
    assert np.abs(f64[:, :3]).max() > 0.0
    assert _force_err(got, f64, fabs) <= FORCE_TOL
    assert np.allclose(got[:, 3], f64[:, 3], rtol=1e-5, atol=1e-6)


def test_bonded_forces_match_reference_fixture(ctx_factory):
    d = _load("polymer_excl")
    n = len(d["pos"])
    ctx = ctx_factory(n)
    _box(ctx, d)
    ctx.set_bonded_tables(0, [(d["bond_values"], float(d["bond_start"]), float(d["bond_step_inv"]))])
    ctx.set_bonded_tables(1, [(d["angle_values"], float(d["angle_start"]),
                               float(d["angle_step_inv"]))])
    pos = _cuda(d["pos"])
    for kind, key, idx in (("bond", "bonds", "bond_fe"), ("angle", "angles", "angle_fe")):
        fe = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        terms = _cuda(d[key])
        tidx = torch.zeros(len(d[key]), dtype=torch.int32, device="cuda")
        if kind == "bond":
            ctx.bond_forces(terms, tidx, pos, fe)
        else:
            ctx.angle_forces(terms, tidx, pos, fe)
        got = fe.cpu().numpy()
        ref = d[idx]
        scale = np.abs(ref[:, :3]).max()
        assert np.abs(got[:, :3] - ref[:, :3]).max() <= 1e-5 * scale, kind
        assert np.allclose(got[:, 3], ref[:, 3], rtol=1e-5, atol=1e-6), kind


def test_philox_matches_openrand_fixture(ctx_factory):
    """First draw of openrand::Philox(seed, ctr, global_seed, ctr1): counter words
    (ctr, ctr1, global_seed, 0)."""
    d = _load("philox")
    ctx = ctx_factory(16)
    for (seed, ctr, gseed, ctr1), ints in zip(d["cases"], d["ints"]):
        out = torch.empty((1, 4), dtype=torch.int32, device="cuda")
        ctx.check(ctx.lib.mb2_philox(ctx.h, int(seed), int(ctr), int(ctr1), int(gseed), 1,
                                     po.C.c_void_p(out.data_ptr()), None, None))
        assert np.array_equal(u32(out)[0], ints[0])


def test_bd_step_with_grid_matches_reference_fixture(ctx_factory):
    d = _load("grid_bd")
    n = len(d["pos"])
    ctx = ctx_factory(n)
    _box(ctx, d)
    grid = _cuda(d["grid"])
    ctx.set_grid(0, grid, tuple(d["grid_origin"]), np.eye(3, dtype=np.float32), 0)
    ctx.set_particle_types(d["charge"], d["diffusion"][:, :3],
                           [[(0, float(s), 0.0, -1)] for s in d["pmf_scale"]])
    pos, fe = _cuda(d["pos"]), _cuda(d["fe"])
    ctx.bd_integrate(pos, fe, _cuda(d["type_ids"]), _cuda(d["flags"].view(np.int32)),
                     float(d["dt"]), float(d["kT"]), int(d["bd_step"]), int(d["bd_seed"]),
                     efield=tuple(d["efield"]))
    got, gfe = pos.cpu().numpy(), fe.cpu().numpy()
    dp = np.abs(got[:, :3] - d["pos_after"][:, :3])
    dp = np.minimum(dp, np.abs(dp - d["box_size"][0]))
    assert dp.max() <= POS_TOL
    frozen = d["flags"] != 0
    assert np.array_equal(got[frozen], d["pos"][frozen])
    assert np.allclose(gfe[:, 3], d["fe_after"][:, 3], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("pending", [0, 1])
def test_baoab_step_matches_reference_fixture(ctx_factory, pending):
    """Langevin BAOAB with the PMF pass and, when pending, the closing kick."""
    d = _load("baoab")
    n = len(d["pos"])
    ctx = ctx_factory(n)
    _box(ctx, d)
    grid = _cuda(d["grid"])
    ctx.set_grid(0, grid, tuple(d["grid_origin"]), np.eye(3, dtype=np.float32), 0)
    ctx.set_particle_types(d["charge"], d["diffusion"][:, :3],
                           [[(0, float(s), 0.0, -1)] for s in d["pmf_scale"]])
    ctx.set_langevin_types(d["mass"], d["damping"])
    pos, mom, fe = _cuda(d["pos"]), _cuda(d["mom"]), _cuda(d["fe"])
    ctx.baoab_integrate(pos, mom, fe, _cuda(d["type_ids"]), _cuda(d["flags"].view(np.int32)),
                        float(d["dt"]), float(d["kT"]), int(d["step"]), int(d["seed"]),
                        efield=tuple(d["efield"]), pending=pending)
    got_p, got_m, got_f = pos.cpu().numpy(), mom.cpu().numpy(), fe.cpu().numpy()
    ref_p, ref_m = d[f"pos_after_{pending}"], d[f"mom_after_{pending}"]
    dp = np.abs(got_p[:, :3] - ref_p[:, :3])
    dp = np.minimum(dp, np.abs(dp - d["box_size"][0]))
    assert dp.max() <= POS_TOL
    assert np.abs(got_m[:, :3] - ref_m[:, :3]).max() <= 1e-5 * np.abs(ref_m[:, :3]).max()
    assert np.allclose(got_f, d[f"fe_after_{pending}"], rtol=1e-5, atol=1e-5)
    frozen = d["flags"] != 0
    assert np.array_equal(got_p[frozen], d["pos"][frozen])
    assert np.array_equal(got_m[frozen], d["mom"][frozen])
