"""Canonical Morton reorder through the C ABI (mb2_reorder_*): the permutation,
gathered arrays and remapped indices bit-exact against the fixture made from
the reference's own MortonEncode / InverseIndex / ReorderData / RemapIndices
functors, and a reordered bonded system that keeps its pair set (with the
exclusion CSR rebuilt on the host) and its forces."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, u32
from mars_md_b200 import _lib as L
from mars_md_b200 import engine as E
from mars_md_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def test_reorder_matches_reference_fixture(ctx_factory):
    d = _load("reorder")
    n = len(d["pos"])
    ctx = ctx_factory(n)
    ctx.set_box(d["box_origin"], d["box_size"], d["box_periodic"])
    pos = torch.from_numpy(d["pos"]).cuda()
    ctx.reorder_begin(pos)
    assert np.array_equal(u32(ctx.reorder_inverse()), d["inverse"])
    ctx.reorder_apply(pos)
    ids = torch.arange(n, dtype=torch.int32, device="cuda")
    ctx.reorder_apply(ids)
    idx = torch.from_numpy(d["indices"]).cuda()
    ctx.reorder_remap(idx)
    torch.cuda.synchronize()
    assert np.array_equal(pos.cpu().numpy(), d["pos_after"])
    assert np.array_equal(u32(ids), d["s2o"])
    assert np.array_equal(idx.cpu().numpy(), d["indices_after"])


def test_reorder_argument_errors(ctx_factory):
    d = _load("reorder")
    n = len(d["pos"])
    ctx = ctx_factory(n)
    ctx.set_box(d["box_origin"], d["box_size"], d["box_periodic"])
    pos = torch.from_numpy(d["pos"]).cuda()
    with pytest.raises(L.MB2Error):      # no permutation of this size yet
        ctx.reorder_apply(pos)
    ctx.reorder_begin(pos)
    with pytest.raises(L.MB2Error):      # n differs from the begin's
        ctx.reorder_apply(pos[: n // 2].contiguous())
    with pytest.raises(ValueError):      # 8-byte rows
        ctx.reorder_apply(torch.zeros((n, 2), dtype=torch.int32, device="cuda"))
    rc = ctx.lib.mb2_reorder_apply(ctx.h, E._p(pos), 8, n, None)
    assert rc != 0
    big = ctx_factory(8)
    big.set_box(d["box_origin"], d["box_size"], d["box_periodic"])
    with pytest.raises(L.MB2Error):      # above the context's capacity
        big.reorder_begin(pos)


def _canon(p):
    p = np.sort(np.asarray(p, np.int64), axis=1)
    return set(map(tuple, p))


def test_reordered_system_keeps_pairs_and_forces(ctx_factory):
    w = W.polymers(n_chains=16, beads=128, box=200.0, with_grid=False)
    ctx = ctx_factory(w.n)
    dev = E.setup_workload(ctx, w)
    _, off, nb, npart = E.exclusion_csr(w.exclusions)
    off_d, nb_d = torch.from_numpy(off).cuda(), torch.from_numpy(nb).cuda()
    ctx.set_exclusions(off_d, nb_d, npart)

    def forces():
        ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius)
        fe = torch.zeros((w.n, 4), dtype=torch.float32, device="cuda")
        ctx.pair_forces(dev["pos"], dev["type"], fe, w.cutoff, get_energy=True)
        ctx.bond_forces(dev["bonds"], dev["bond_idx"], dev["pos"], fe)
        ctx.angle_forces(dev["angles"], dev["angle_idx"], dev["pos"], fe)
        return fe.cpu().numpy().astype(np.float64), ctx.export_pairs().cpu().numpy()

    f0, p0 = forces()
    ids = torch.arange(w.n, dtype=torch.int32, device="cuda")
    out = E.reorder_particles(ctx, (w.box_origin, w.box_size),
                              {"pos": dev["pos"], "type_id": dev["type"], "flags": dev["flags"],
                               "id": ids},
                              indices=[dev["bonds"], dev["angles"]], exclusion_pairs=w.exclusions)
    assert out is not None and out["exclusions"] is not None
    f1, p1 = forces()
    s2o = ids.cpu().numpy().astype(np.int64)
    inv = out["inverse"].cpu().numpy().astype(np.int64)
    assert np.array_equal(inv[s2o], np.arange(w.n))
    assert not np.array_equal(s2o, np.arange(w.n))
    assert len(p0) == len(p1) and _canon(s2o[p1]) == _canon(p0)
    # Same physics, summed in another order.
    scale = np.abs(f0[:, :3]).max()
    assert np.abs(f1[inv, :3] - f0[:, :3]).max() <= 1e-5 * scale
    assert abs(f1[:, 3].sum() - f0[:, 3].sum()) <= 1e-5 * np.abs(f0[:, 3]).sum()
    assert np.array_equal(dev["type"].cpu().numpy(), w.type_ids[s2o])
    assert np.array_equal(dev["bonds"].cpu().numpy(), inv[w.bonds])
