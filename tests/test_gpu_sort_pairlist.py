"""CUDA Morton sort and pairlist against the CPU oracle (bit-exact).

Mirrors the reference's own checks: radix-sort sortedness at large N
(Unit_test/System/zorder_tests.cpp:84-229), pair sets on lattices and
distance checks (Unit_test/Compute/zorder_pairlist_tests.cpp,
Unit_test/Compute/Zorder_pairlist2.cpp), exclusions dropped at build time.
Here the pair SET must equal the oracle's exactly.
"""
import numpy as np
import pytest
import torch

from conftest import box_of, u32
from mars_md_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _sorted_pairs(t):
    p = t.cpu().numpy().astype(np.int64)
    if len(p) == 0:
        return p.reshape(0, 2)
    o = np.lexsort((p[:, 1], p[:, 0]))
    return p[o]


@pytest.mark.parametrize("n", [1, 7, 4096, 65536, 2_097_152])
def test_morton_sort_bit_exact(ctx_factory, oracle, n):
    rng = np.random.default_rng(n)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-50.0, 950.0, size=(n, 3)).astype(np.float32)
    bmin = np.array([0.0, 0.0, 0.0], np.float32)
    bmax = np.array([900.0, 900.0, 900.0], np.float32)
    ctx = ctx_factory(n)
    d = torch.from_numpy(pos).cuda()
    keys, s2o, inv, sp = ctx.sort_morton(d, bmin, bmax)
    torch.cuda.synchronize()
    ok, oi = oracle.morton_encode(pos, bmin, bmax)
    assert np.array_equal(u32(keys), oracle.sort_pairs(ok, oi)[0])
    ks, vs = oracle.sort_pairs(ok, oi)
    assert np.array_equal(u32(s2o), vs)
    assert np.array_equal(u32(inv), oracle.inverse(vs))
    assert np.array_equal(sp.cpu().numpy(), oracle.gather4(pos, vs))


def test_radix_sort_large_sortedness(ctx_factory):
    # The reference documents a missing large-N sort check (dev_notes); cover 2^25.
    n = 1 << 25
    g = torch.Generator(device="cuda").manual_seed(7)
    keys = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device="cuda", generator=g)
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ref_keys = keys.clone()
    ctx = ctx_factory(16)
    ctx.radix_sort_pairs(keys, vals)
    torch.cuda.synchronize()
    k = keys.cpu().numpy().view(np.uint32).astype(np.int64)
    v = vals.cpu().numpy().astype(np.int64)
    assert np.all(np.diff(k) >= 0)
    # stability: equal keys keep ascending payloads
    same = np.diff(k) == 0
    assert np.all(np.diff(v)[same] > 0)
    # permutation consistency
    assert np.array_equal(ref_keys.cpu().numpy().view(np.uint32)[v], k.astype(np.uint32))


@pytest.mark.parametrize("n", [2, 3, 1000, 4097, 8192, 8193, 20000])
def test_radix_sort_small_stable(ctx_factory, n):
    """Up to 8,192 pairs one CTA sorts (a bitonic network over key and
    position), above that the radix passes: both must give a host stable
    argsort's permutation, here with many equal keys (16 distinct values) and
    payloads that are not in ascending order, on both sides of the switch."""
    rng = np.random.default_rng(n)
    keys_np = rng.integers(0, 16, n).astype(np.uint32) * np.uint32(0x10001001)
    vals_np = rng.permutation(n).astype(np.uint32)
    keys = torch.from_numpy(keys_np.view(np.int32)).cuda()
    vals = torch.from_numpy(vals_np.view(np.int32)).cuda()
    ctx = ctx_factory(16)
    ctx.radix_sort_pairs(keys, vals)
    torch.cuda.synchronize()
    order = np.argsort(keys_np, kind="stable")
    assert np.array_equal(u32(keys), keys_np[order])
    assert np.array_equal(u32(vals), vals_np[order])


def _build_and_compare(ctx, oracle, w, rc_list, excl=None, excl_np=None):
    d = torch.from_numpy(w.pos).cuda()
    t = torch.from_numpy(w.type_ids).cuda()
    ctx.set_box(w.box_origin, w.box_size, w.periodic)
    if excl is not None:
        ctx.set_exclusions(*excl)
    npairs = ctx.build_pairlist(d, t, rc_list)
    gpu = _sorted_pairs(ctx.export_pairs())
    torch.cuda.synchronize()
    ref_pairs, cnt, cs = oracle.build_pairlist(w.pos, box_of(w), rc_list, excl=excl_np)
    assert npairs == cnt
    assert np.array_equal(gpu, ref_pairs.astype(np.int64))
    return npairs


def test_pairlist_plain_bd_exact(ctx_factory, oracle):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    assert _build_and_compare(ctx, oracle, w, w.list_radius) > 60000


def test_pairlist_polymers_with_exclusions(ctx_factory, oracle):
    w = W.polymers(n_chains=8, beads=1024, with_grid=False)
    off, nb, np_ = oracle.exclusion_csr(w.exclusions)
    ctx = ctx_factory(w.n)
    doff = torch.from_numpy(off).cuda()
    dnb = torch.from_numpy(nb).cuda()
    n_with = _build_and_compare(ctx, oracle, w, w.list_radius, excl=(doff, dnb, np_),
                                excl_np=(off, nb, np_))
    assert n_with > 0


def test_pairlist_open_lattice(ctx_factory, oracle):
    # 4x4x4 lattice, 1.5 A spacing, rc 2, open box (zorder_pairlist_tests.cpp:29-75)
    g = np.array([(i, j, k) for i in range(4) for j in range(4) for k in range(4)], np.float32) * 1.5
    pos = np.zeros((64, 4), np.float32)
    pos[:, :3] = g
    w = W.plain_bd(n=64)
    w.pos = pos
    w.box_origin, w.box_size, w.periodic = (-30, -30, -30), (60, 60, 60), (0, 0, 0)
    ctx = ctx_factory(64)
    n = _build_and_compare(ctx, oracle, w, 2.0)
    # nearest neighbours only at 1.5 A (diagonals are 2.12 A): 3 * 4 * 4 * 3
    assert n == 144


@pytest.mark.parametrize("rc,expect", [(1.1, 2), (2.5, 3)])
def test_pairlist_line_cutoffs(ctx_factory, oracle, rc, expect):
    # three particles on a line, 1 A apart (Zorder_pairlist2.cpp:365-404)
    pos = np.zeros((3, 4), np.float32)
    pos[:, 0] = [0.0, 1.0, 2.0]
    w = W.plain_bd(n=3)
    w.pos = pos
    w.box_origin, w.box_size, w.periodic = (-10, -10, -10), (20, 20, 20), (0, 0, 0)
    ctx = ctx_factory(3)
    assert _build_and_compare(ctx, oracle, w, rc) == expect


def test_pairlist_empty_and_single(ctx_factory):
    ctx = ctx_factory(4)
    ctx.set_box((0, 0, 0), (10, 10, 10), (1, 1, 1))
    t = torch.zeros(0, dtype=torch.int32, device="cuda")
    assert ctx.build_pairlist(torch.zeros((0, 4), device="cuda"), t, 3.0) == 0
    one = torch.tensor([[1.0, 2.0, 3.0, 0.0]], device="cuda")
    assert ctx.build_pairlist(one, torch.zeros(1, dtype=torch.int32, device="cuda"), 3.0) == 0
    assert ctx.export_pairs().shape[0] == 0


def test_pairlist_capacity_error(ctx_factory):
    ctx = ctx_factory(10)
    ctx.set_box((0, 0, 0), (10, 10, 10), (1, 1, 1))
    pos = torch.zeros((11, 4), device="cuda")
    with pytest.raises(Exception, match="more particles"):
        ctx.build_pairlist(pos, torch.zeros(11, dtype=torch.int32, device="cuda"), 3.0)


def test_needs_update_skin(ctx_factory, oracle):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    d = torch.from_numpy(w.pos).cuda()
    t = torch.from_numpy(w.type_ids).cuda()
    ctx.set_box(w.box_origin, w.box_size, w.periodic)
    ctx.build_pairlist(d, t, w.list_radius)
    moved = w.pos.copy()
    moved[17, 0] = np.float32((moved[17, 0] + 2.6) % 200.0)
    dm = torch.from_numpy(moved).cuda()
    disp, needs = ctx.needs_update(dm, 5.0)
    ref = oracle.max_displacement(moved, w.pos, np.array(w.box_size, np.float32))
    assert disp == ref
    assert needs
    disp0, needs0 = ctx.needs_update(d, 5.0)
    assert disp0 == 0.0 and not needs0


@pytest.mark.slow
def test_pairlist_large_plain_count_and_checksum(ctx_factory, oracle):
    """2,097,152 beads, 35 A list: count and order-independent checksum of the
    pair set equal the oracle's (size-independent set identity)."""
    w = W.large_plain()
    ctx = ctx_factory(w.n)
    d = torch.from_numpy(w.pos).cuda()
    t = torch.from_numpy(w.type_ids).cuda()
    ctx.set_box(w.box_origin, w.box_size, w.periodic)
    npairs = ctx.build_pairlist(d, t, w.list_radius)
    pairs = ctx.export_pairs()
    torch.cuda.synchronize()
    p = pairs.cpu().numpy()
    # Count-only oracle walk (threaded) at a finer cell level than the
    # reference's choice; the pair set does not depend on the level.
    _, cnt, cs = oracle.build_pairlist(w.pos, box_of(w), w.list_radius, want_pairs=False, m=6)
    assert npairs == cnt
    assert oracle.pair_hash_sum(p) == cs
