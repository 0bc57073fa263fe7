"""Batched replicas (mb2_batch_*) against the oracle and against plain
per-system steps: the same pair set in every system, the same trajectories
(system s of a batch steps as a plain context with seed + s), graph replay
equal to eager steps, and tuning knobs that change speed but not results."""
import numpy as np
import pytest
import torch

from conftest import box_of
from mars_md_b200 import _lib, workloads as W
from mars_md_b200.engine import Context, setup_batch, setup_workload, step_params

pytestmark = pytest.mark.gpu

SEED = 4242


def _systems(k=10, nmax=3000):
    return W.batched(seed=SEED, systems=k, nmin=500, nmax=nmax)


def _canon(p):
    p = np.sort(np.asarray(p, np.int64), axis=1)
    return p[np.lexsort((p[:, 1], p[:, 0]))] if len(p) else p.reshape(0, 2)


def _split_pairs(pairs, offsets):
    sys_a = np.searchsorted(offsets, pairs[:, 0], side="right") - 1
    sys_b = np.searchsorted(offsets, pairs[:, 1], side="right") - 1
    assert np.array_equal(sys_a, sys_b), "a pair crosses systems"
    return [pairs[sys_a == s] - offsets[s] for s in range(len(offsets) - 1)]


def _check_pair_sets(oracle, b, ws):
    per = _split_pairs(b.export_pairs().cpu().numpy().astype(np.int64), b.offsets)
    for s, w in enumerate(ws):
        ref, cnt, _ = oracle.build_pairlist(w.pos, box_of(w), w.list_radius)
        assert len(per[s]) == cnt, f"system {s}"
        assert np.array_equal(_canon(per[s]), ref.astype(np.int64)), f"system {s}"


def test_batch_pair_sets_match_oracle_per_system(oracle):
    ws = _systems()
    b, dev = setup_batch(ws)
    try:
        n = b.build(dev["pos"], dev["type"], ws[0].list_radius)
        assert n == b.num_pairs()
        _check_pair_sets(oracle, b, ws)
    finally:
        b.close()


@pytest.mark.parametrize("level,lanes", [(1, 16), (-1, 4), (0, 32)])
def test_batch_tuning_knobs_keep_the_pair_set(oracle, level, lanes):
    ws = _systems(k=6)
    b, dev = setup_batch(ws)
    try:
        b.set_tuning(level, lanes)
        b.build(dev["pos"], dev["type"], ws[0].list_radius)
        assert b.tuning()[1] == lanes
        _check_pair_sets(oracle, b, ws)
    finally:
        b.close()


def _plain_trajectories(ws, prm_for, steps):
    out = []
    for s, w in enumerate(ws):
        ctx = Context(w.n)
        dev = setup_workload(ctx, w)
        prm = prm_for(w, s)
        for k in range(1, steps + 1):
            ctx.step(dev["pos"], dev["fe"], dev["type"], None, k, prm)
        torch.cuda.synchronize()
        out.append((dev["pos"].cpu().numpy(), dev["fe"].cpu().numpy()))
        ctx.close()
    return out


def _periodic_diff(a, b, box_len):
    d = np.abs(a - b)
    return np.minimum(d, np.abs(d - box_len))


def test_batch_run_equals_plain_steps_per_system():
    ws = _systems(k=8)
    steps, period = 7, 3

    def prm_for(w, s):
        p = step_params(w, seed=SEED + s)
        p.rebuild_period = period
        return p

    plain = _plain_trajectories(ws, prm_for, steps)
    b, dev = setup_batch(ws)
    try:
        prm = step_params(ws[0], seed=SEED)
        prm.rebuild_period = period
        b.run(dev["pos"], dev["fe"], dev["type"], 1, steps, prm)
        torch.cuda.synchronize()
        pos = dev["pos"].cpu().numpy()
        fe = dev["fe"].cpu().numpy()
        for s, w in enumerate(ws):
            lo, hi = b.offsets[s], b.offsets[s + 1]
            dp = _periodic_diff(pos[lo:hi, :3], plain[s][0][:, :3], w.box_size[0])
            assert dp.max() < 1e-4, f"system {s}: {dp.max()}"
            df = np.abs(fe[lo:hi, :3] - plain[s][1][:, :3]).max()
            scale = np.abs(plain[s][1][:, :3]).max() + 1e-30
            assert df / scale < 1e-5, f"system {s}: force {df / scale}"
        start = np.concatenate([w.pos for w in ws])[:, :3]
        assert np.abs(pos[:, :3] - start).max() > 0.1
    finally:
        b.close()


def test_batch_graph_replay_equals_eager_steps():
    ws = _systems(k=5)
    prm = step_params(ws[0], seed=SEED)
    prm.rebuild_period = 2
    b1, d1 = setup_batch(ws)
    b2, d2 = setup_batch(ws)
    try:
        for k in range(1, 6):
            b1.step(d1["pos"], d1["fe"], d1["type"], k, prm)
        b2.run(d2["pos"], d2["fe"], d2["type"], 1, 5, prm)
        torch.cuda.synchronize()
        box = np.repeat([w.box_size[0] for w in ws], [w.n for w in ws])[:, None]
        diff = _periodic_diff(d1["pos"].cpu().numpy()[:, :3], d2["pos"].cpu().numpy()[:, :3], box)
        assert diff.max() < 1e-5
    finally:
        b1.close()
        b2.close()


def test_batch_autotune_reports_and_keeps_results(oracle):
    ws = _systems(k=6)
    b, dev = setup_batch(ws)
    try:
        prm = step_params(ws[0], seed=SEED)
        before = dev["pos"].clone()
        r = b.autotune(dev["pos"], dev["type"], prm, trial_steps=2)
        torch.cuda.synchronize()
        assert torch.equal(before, dev["pos"])  # tuning runs on a copy
        assert r["lanes"] in (4, 8, 16) and r["level_offset"] in (-1, 0, 1)
        assert 1 <= r["safe_rebuild_period"] <= prm.rebuild_period
        assert r["step_ms"] > 0 and r["build_ms"] > 0
        b.build(dev["pos"], dev["type"], ws[0].list_radius)
        _check_pair_sets(oracle, b, ws)
    finally:
        b.close()


def test_batch_autotuned_cadence_in_force_and_list_stays_exact(oracle):
    """The tuner's cadence is the one the run uses (its rebuilds follow it),
    and a list built past the transient still holds every pair within the
    interaction cutoff after that many steps (checked per system against the
    oracle's pair set at the cutoff on the current positions)."""
    ws = _systems(k=6)
    b, dev = setup_batch(ws)
    try:
        prm = step_params(ws[0], seed=SEED)
        r = b.autotune(dev["pos"], dev["type"], prm, trial_steps=2)
        c = r["safe_rebuild_period"]
        assert b.rebuild_schedule()[0] == c
        # Past the transient of the fresh start: the first step builds, then one
        # scheduled check every c steps (a rebuild unless the skin still holds).
        steps = 2 * prm.rebuild_period
        b.run(dev["pos"], dev["fe"], dev["type"], 1, steps, prm)
        torch.cuda.synchronize()
        _, rebuilds = b.rebuild_schedule()
        assert 1 <= rebuilds <= (steps - 1) // c + 1
        # A fresh list, then c steps.
        b.build(dev["pos"], dev["type"], ws[0].list_radius)
        b.run(dev["pos"], dev["fe"], dev["type"], steps + 1, c, prm)
        torch.cuda.synchronize()
        listed = _split_pairs(b.export_pairs().cpu().numpy().astype(np.int64), b.offsets)
        pos = dev["pos"].cpu().numpy()
        for s, w in enumerate(ws):
            p = pos[b.offsets[s]:b.offsets[s + 1]]
            near, _, _ = oracle.build_pairlist(p, box_of(w), w.cutoff)
            have = {tuple(x) for x in _canon(listed[s]).tolist()}
            missing = [tuple(x) for x in near.tolist() if tuple(x) not in have]
            assert not missing, f"system {s}: {len(missing)} pairs within the cutoff not listed"
    finally:
        b.close()


def test_batch_rebuilds_only_the_systems_whose_skin_failed(oracle):
    """Each system is checked as a patch of its own: from a list built on the
    current positions, every other particle of system 0 is moved 3 A (beyond
    half the 5 A skin) and of system 1 by 0.8 A; the next step's check
    rebuilds system 0 alone. System
    0's rows then hold the pair set of the positions it was rebuilt from;
    system 1 keeps the set of the earlier build, which its current positions
    no longer give."""
    ws = _systems(k=4)
    b, dev = setup_batch(ws)
    try:
        prm = step_params(ws[0], seed=SEED)
        prm.rebuild_period = 1
        b.step(dev["pos"], dev["fe"], dev["type"], 1, prm)
        b.build(dev["pos"], dev["type"], ws[0].list_radius)
        torch.cuda.synchronize()
        built_at = dev["pos"].cpu().numpy().copy()
        builds, systems = b.rebuild_schedule()[1], b.system_rebuilds()
        pos = dev["pos"]
        for s, shift in ((0, 3.0), (1, 0.8)):  # every other particle, so pairs change
            lo, hi = b.offsets[s], b.offsets[s + 1]
            L = float(ws[s].box_size[0])
            pos[lo:hi:2, 0] = torch.remainder(pos[lo:hi:2, 0] + shift, L)
        at_rebuild = pos.cpu().numpy().copy()
        b.step(dev["pos"], dev["fe"], dev["type"], 2, prm)
        torch.cuda.synchronize()
        assert b.rebuild_schedule()[1] == builds + 1
        assert b.system_rebuilds() == systems + 1
        per = _split_pairs(b.export_pairs().cpu().numpy().astype(np.int64), b.offsets)
        for s, w in enumerate(ws):
            src = at_rebuild if s == 0 else built_at
            ref, _, _ = oracle.build_pairlist(src[b.offsets[s]:b.offsets[s + 1]], box_of(w),
                                              w.list_radius)
            assert np.array_equal(_canon(per[s]), ref.astype(np.int64)), f"system {s}"
        p1 = at_rebuild[b.offsets[1]:b.offsets[2]]
        now1, _, _ = oracle.build_pairlist(p1, box_of(ws[1]), ws[1].list_radius)
        ref1, _, _ = oracle.build_pairlist(built_at[b.offsets[1]:b.offsets[2]], box_of(ws[1]),
                                           ws[1].list_radius)
        assert not np.array_equal(now1, ref1)  # the kept list is the earlier one
    finally:
        b.close()


def test_batch_rejects_boxes_smaller_than_twice_the_list_radius():
    w = W.plain_bd(seed=1, n=600, box=40.0)
    b, dev = setup_batch([w])
    try:
        with pytest.raises(_lib.MB2Error):
            b.build(dev["pos"], dev["type"], 25.0)
    finally:
        b.close()
