"""Failure paths through the C ABI: bad inputs come back as a documented
status code with a message, the device keeps working, and the context can be
used again. No case here faults the GPU: every one is refused on the host, or
runs kernels whose indices stay in bounds whatever the coordinates.

The reference validates its box at build time (ZOrderPairlist.cpp:118-126) and
throws when the list overflows after one grow-and-retry (ZOrderPairlist.cpp:
292-335); it has no check for NaN coordinates or degenerate tables, which this
library adds.
"""
import numpy as np
import pytest
import torch

from conftest import box_of
from mars_md_b200 import _lib as L
from mars_md_b200 import workloads as W
from mars_md_b200.engine import setup_workload, step_params

pytestmark = pytest.mark.gpu


def _expect(code, fn, *args, match=None, **kw):
    with pytest.raises(L.MB2Error, match=match) as e:
        fn(*args, **kw)
    assert e.value.code == code, e.value


def _still_works(ctx, w, dev):
    """A clean build and a force call succeed after the failure."""
    n = ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius, w.cutoff)
    ctx.pair_forces(dev["pos"], dev["type"], dev["fe"], w.cutoff, get_energy=False)
    torch.cuda.synchronize()
    assert n > 0 and torch.isfinite(dev["fe"]).all()


@pytest.mark.parametrize("bad", [float("nan"), float("inf"), -float("inf")])
def test_nonfinite_position_refused_by_build(ctx_factory, bad):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    good = dev["pos"].clone()
    dev["pos"][123, 1] = bad
    _expect(L.MB2_ERR_ARG, ctx.build_pairlist, dev["pos"], dev["type"], w.list_radius,
            match="NaN or infinite")
    # No list is left behind by the failed build.
    _expect(L.MB2_ERR_STATE, ctx.pair_forces, dev["pos"], dev["type"], dev["fe"], w.cutoff,
            match="no pairlist")
    dev["pos"].copy_(good)
    _still_works(ctx, w, dev)


def test_nonfinite_position_on_open_axis(ctx_factory):
    w = W.plain_bd(n=512)
    w.periodic = (0, 1, 1)
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    good = dev["pos"].clone()
    dev["pos"][7, 0] = float("nan")
    _expect(L.MB2_ERR_ARG, ctx.build_pairlist, dev["pos"], dev["type"], w.list_radius,
            match="open axis")
    dev["pos"].copy_(good)
    _still_works(ctx, w, dev)


def test_step_with_nan_refused_at_rebuild(ctx_factory):
    """mb2_step: a NaN coordinate is caught at the next scheduled rebuild;
    between rebuilds it propagates as the reference's arithmetic does."""
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    prm = step_params(w)
    ctx.step(dev["pos"], dev["fe"], dev["type"], None, 1, prm)
    dev["pos"][5, 0] = float("nan")
    ctx.step(dev["pos"], dev["fe"], dev["type"], None, 2, prm)  # no rebuild at step 2
    prm.rebuild_period = 0  # rebuild at every step, no skin check (which a NaN would not trip)
    _expect(L.MB2_ERR_ARG, ctx.step, dev["pos"], dev["fe"], dev["type"], None, 3, prm,
            match="NaN or infinite")
    torch.cuda.synchronize()


def test_forces_with_nan_after_build_stay_in_bounds(ctx_factory):
    """A NaN coordinate after a clean build: the force kernels run (table
    bins are clamped, so no read leaves the tables) and the NaN reaches only
    the particles that interact with it."""
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius, w.cutoff)
    dev["pos"][42, 2] = float("nan")
    dev["fe"].zero_()
    ctx.pair_forces(dev["pos"], dev["type"], dev["fe"], w.cutoff, get_energy=True)
    torch.cuda.synchronize()
    bad = ~torch.isfinite(dev["fe"][:, :3]).all(dim=1)
    assert bad[42]
    assert int(bad.sum()) < w.n // 10
    assert torch.isfinite(dev["pos"][:42]).all()


def test_nan_interaction_cutoff_refused(ctx_factory):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    _expect(L.MB2_ERR_ARG, ctx.build_pairlist, dev["pos"], dev["type"], w.list_radius,
            float("nan"), match="interaction cutoff")
    _expect(L.MB2_ERR_ARG, ctx.build_pairlist, dev["pos"], dev["type"], float("inf"),
            match="positive and finite")
    _still_works(ctx, w, dev)


@pytest.mark.parametrize("values,start,step_inv,match", [
    (np.array([1.0], np.float32), 0.0, 10.0, "2 values"),
    (np.array([1.0, 0.5, 0.0], np.float32), 0.0, float("inf"), "finite"),
    (np.array([1.0, 0.5, 0.0], np.float32), 0.0, float("nan"), "finite"),
    (np.array([1.0, 0.5, 0.0], np.float32), 0.0, 0.0, "nonzero"),
    (np.array([1.0, 0.5, 0.0], np.float32), float("nan"), 10.0, "finite"),
])
def test_degenerate_tables_refused(ctx_factory, values, start, step_inv, match):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    _expect(L.MB2_ERR_ARG, ctx.set_pair_tables, 1, w.term_matrix, [(values, start, step_inv)],
            match=match)
    _expect(L.MB2_ERR_ARG, ctx.set_bonded_tables, 0, [(values, start, step_inv)], match=match)
    # The context still takes good tables and computes.
    dev = setup_workload(ctx, w)
    _still_works(ctx, w, dev)


def test_tag_naming_missing_table_refused(ctx_factory):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    bad = np.array([(1 << 5) | (3 << 8)], np.uint32)  # tabulated, table 3 of 1
    _expect(L.MB2_ERR_ARG, ctx.set_pair_tables, 1, bad,
            [(t.values, t.start, t.step_inv) for t in w.pair_tables], match="missing table")


def test_exclusion_csr_covering_fewer_particles(ctx_factory, oracle):
    """An exclusion CSR over the first half of the particles only: rows past
    num_particles hold no exclusions (ExclusionView::row_begin/row_end,
    DeviceExclusions.h:30-43); the pair set equals the oracle's with the same
    view."""
    w = W.polymers(n_chains=4, beads=1024, with_grid=False)
    off, nb, npart = oracle.exclusion_csr(w.exclusions)
    half = w.n // 2
    off_h = np.ascontiguousarray(off[:half + 1])
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    d_off, d_nb = torch.from_numpy(off_h).cuda(), torch.from_numpy(nb).cuda()
    ctx.set_exclusions(d_off, d_nb, half)
    ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius)
    got = ctx.export_pairs().cpu().numpy().astype(np.int64)
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    ref, cnt, _ = oracle.build_pairlist(w.pos, box_of(w), w.list_radius, excl=(off_h, nb, half))
    assert len(got) == cnt and np.array_equal(got, ref.astype(np.int64))
    full, cnt_full, _ = oracle.build_pairlist(w.pos, box_of(w), w.list_radius,
                                              excl=(off, nb, npart))
    assert cnt > cnt_full  # some exclusions were not applied


def test_capacity_refused_before_any_launch(ctx_factory):
    w = W.plain_bd(n=256)
    ctx = ctx_factory(w.n - 1)
    dev = setup_workload(ctx, w)
    _expect(L.MB2_ERR_CAPACITY, ctx.build_pairlist, dev["pos"], dev["type"], w.list_radius,
            match="more particles")
