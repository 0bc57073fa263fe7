"""CUDA pair/bond/angle forces, Philox, grid force and BD step against the oracle.

Tolerances (float32 arithmetic):
* Per-particle forces: |F_gpu - F_64| / max(|F_64|, 1e-3 F_rms) <= 1e-5, with
  F_64 the FP64 oracle's sum and F_rms the RMS force over all particles. Each
  pair's float force is rounded exactly as the reference's, so the gap is the
  float summation order alone. The error relative to the sum of |pair force|
  on the particle is held to 1e-5 as well.
* Angles: the tabulated force is constant within a table bin, and the device
  acosf and the host's acos may differ by an ulp or two, so an angle within
  rounding of a bin edge can take the neighbouring bin's force on one side.
  The particles of such angles are counted and reported; every other particle
  is held to the bar above.
* Energies: FP64 device reduction vs the FP64 oracle, <= 1e-6 relative.
* Philox words: bit-exact. BD positions: the Box-Muller transcendentals are
  CUDA's logf/sinf/cosf vs host libm (a few ulp), so positions agree to
  1e-5 A absolute per step.
Mirrors Unit_test/Interactions/NonbondedEnergy.cpp (pair sums vs CPU),
Unit_test/Compute/BDKernels.cpp (bond chain, Box-Muller moments, free
diffusion), Unit_test/Interactions/TabulatedBonded.cpp (angles) and
Unit_test/Interactions/Pmf.cpp (grid forces).
"""
import numpy as np
import pytest
import torch

import pyoracle
from conftest import box_of, force_errors, tableset, u32
from mars_md_b200 import workloads as W
from mars_md_b200.engine import setup_workload, step_params

pytestmark = pytest.mark.gpu


def _pair_case(ctx, oracle, w, lanes=0, split=False):
    dev = setup_workload(ctx, w)
    if lanes:
        ctx.set_lanes_per_row(lanes)
    ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius, w.cutoff if split else 0.0)
    pairs = ctx.export_pairs().cpu().numpy()
    ctx.reset_energies()
    ctx.pair_forces(dev["pos"], dev["type"], dev["fe"], w.cutoff, get_energy=True)
    e = ctx.energies()
    fe = dev["fe"].cpu().numpy()
    tags = oracle.resolve_tags(pairs, w.type_ids, w.term_matrix, w.num_types)
    rc2 = np.float32(w.cutoff) ** 2
    f32, f64, fabs = oracle.pair_forces(pairs, w.pos, tags, tableset(w), box_of(w), rc2)
    e64 = oracle.pair_energy_f64(pairs, w.pos, tags, tableset(w), box_of(w), rc2)
    return fe, f64, fabs, e, e64


@pytest.mark.parametrize("lanes,split", [(0, False), (0, True), (4, False), (8, True),
                                         (16, False), (32, True)])
def test_pair_forces_plain_bd(ctx_factory, oracle, lanes, split):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    fe, f64, fabs, e, e64 = _pair_case(ctx, oracle, w, lanes, split)
    scaled, plain = force_errors(fe, f64, fabs)
    print(f"plain_bd lanes={lanes} split={split}: worst {plain:.3e} (scaled {scaled:.3e})")
    assert plain <= 1e-5, (plain, scaled)
    assert scaled <= 1e-5, (scaled, plain)
    # per-particle energy halves sum to the pair energy
    assert abs(fe[:, 3].astype(np.float64).sum() - f64[:, 3].sum()) <= 1e-5 * abs(f64[:, 3]).sum()
    assert abs(e[0] - e64) <= 1e-6 * abs(e64)
    # Newton's third law: total force vanishes
    assert np.abs(fe[:, :3].astype(np.float64).sum(0)).max() <= 1e-3 * fabs.sum() / len(fabs)


def test_pair_forces_without_cutoff(ctx_factory, oracle):
    """cutoff 0: the reference evaluates every listed pair (its test then has
    no upper bound), here the window's upper bound is +inf; pairs between
    the 20 A table end and the 25 A list radius take the last bin."""
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius)
    pairs = ctx.export_pairs().cpu().numpy()
    ctx.reset_energies()
    ctx.pair_forces(dev["pos"], dev["type"], dev["fe"], 0.0, get_energy=True)
    e = ctx.energies()
    fe = dev["fe"].cpu().numpy()
    tags = oracle.resolve_tags(pairs, w.type_ids, w.term_matrix, w.num_types)
    f32, f64, fabs = oracle.pair_forces(pairs, w.pos, tags, tableset(w), box_of(w),
                                        np.float32(0.0))
    e64 = oracle.pair_energy_f64(pairs, w.pos, tags, tableset(w), box_of(w), np.float32(0.0))
    scaled, plain = force_errors(fe, f64, fabs)
    assert plain <= 1e-5, (plain, scaled)
    assert abs(e[0] - e64) <= 1e-6 * abs(e64)


@pytest.mark.parametrize("split", [False, True])
def test_pair_forces_large_types(ctx_factory, oracle, split):
    # 4 types, 10 tables, Debye-Hueckel + soft core, at 1/64 of the full size
    w = W.large_plain(n=32768)
    ctx = ctx_factory(w.n)
    fe, f64, fabs, e, e64 = _pair_case(ctx, oracle, w, split=split)
    scaled, plain = force_errors(fe, f64, fabs)
    print(f"large_plain 32768 split={split}: worst {plain:.3e} (scaled {scaled:.3e})")
    assert plain <= 1e-5, (plain, scaled)
    assert scaled <= 1e-5, (scaled, plain)
    assert abs(e[0] - e64) <= 1e-6 * abs(e64)


@pytest.mark.slow
def test_pair_forces_large_plain_full_size_sample(ctx_factory, oracle):
    """All 2,097,152 forces of the benchmark workload from the GPU (rows split
    at the cutoff, as the fused step builds them); 65,536 strided particles
    checked against FP64 sums the oracle forms from the exported pairs that
    touch them (the pair set itself is checked at this size elsewhere)."""
    w = W.large_plain()
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius, w.cutoff)
    dev["fe"].zero_()
    ctx.pair_forces(dev["pos"], dev["type"], dev["fe"], w.cutoff, get_energy=False)
    fe = dev["fe"].cpu().numpy()
    sample = np.arange(0, w.n, 32)
    mask = torch.zeros(w.n, dtype=torch.bool, device="cuda")
    mask[torch.from_numpy(sample).cuda()] = True
    pairs = ctx.export_pairs()
    keep = mask[pairs[:, 0].long()] | mask[pairs[:, 1].long()]
    sub = pairs[keep].cpu().numpy()
    del pairs, keep
    torch.cuda.empty_cache()
    tags = oracle.resolve_tags(sub, w.type_ids, w.term_matrix, w.num_types)
    _, f64, fabs = oracle.pair_forces(sub, w.pos, tags, tableset(w), box_of(w),
                                      np.float32(w.cutoff) ** 2)
    # F_rms over the sample stands in for the RMS over all particles.
    scaled, plain = force_errors(fe[sample], f64[sample], fabs[sample])
    print(f"large_plain full size, {len(sample)} particles, {len(sub)} pairs: worst {plain:.3e} "
          f"(scaled {scaled:.3e})")
    assert plain <= 1e-5, (plain, scaled)
    assert scaled <= 1e-5, (scaled, plain)


def test_pair_forces_inner_rows_after_steps(ctx_factory, oracle):
    """Above 131,072 particles the packs track the largest displacement since
    the build, and rows deeper inside the box than the list radius plus twice
    that displacement take the shorter minimum image. After nine BD steps on
    the list of the first (no rebuild; the displacement is then a few
    angstrom), the forces on the current positions from that list must still
    be the oracle's: 16,384 strided particles at the bar above."""
    w = W.large_plain(n=262144)
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    prm = step_params(w)
    prm.rebuild_period = 1000  # step 1 builds; steps 2-10 keep its list
    for s in range(1, 11):
        ctx.step(dev["pos"], dev["fe"], dev["type"], None, s, prm)
    dev["fe"].zero_()
    ctx.pair_forces(dev["pos"], dev["type"], dev["fe"], w.cutoff, get_energy=False)
    fe = dev["fe"].cpu().numpy()
    pos = dev["pos"].cpu().numpy()
    pos[:, 3] = w.pos[:, 3]
    start = w.pos[:, :3].astype(np.float64)
    moved = np.abs(pos[:, :3] - start)
    moved = np.minimum(moved, np.array(w.box_size) - moved)
    dmax = float(np.sqrt((moved ** 2).sum(1)).max())
    assert dmax > 0.5, dmax
    sample = np.arange(0, w.n, 16)
    mask = torch.zeros(w.n, dtype=torch.bool, device="cuda")
    mask[torch.from_numpy(sample).cuda()] = True
    pairs = ctx.export_pairs()
    keep = mask[pairs[:, 0].long()] | mask[pairs[:, 1].long()]
    sub = pairs[keep].cpu().numpy()
    tags = oracle.resolve_tags(sub, w.type_ids, w.term_matrix, w.num_types)
    _, f64, fabs = oracle.pair_forces(sub, pos, tags, tableset(w), box_of(w),
                                      np.float32(w.cutoff) ** 2)
    scaled, plain = force_errors(fe[sample], f64[sample], fabs[sample])
    print(f"large_plain 262,144 after 9 steps (max displacement {dmax:.2f} A): "
          f"worst {plain:.3e} (scaled {scaled:.3e})")
    assert plain <= 1e-5, (plain, scaled)
    assert scaled <= 1e-5, (scaled, plain)


def test_pair_forces_match_reference_functor(ctx_factory, oracle, ref):
    """Against the reference's own host-compiled PairNonbondedComputer."""
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    fe, f64, fabs, e, e64 = _pair_case(ctx, oracle, w)
    pairs, _, _ = oracle.build_pairlist(w.pos, box_of(w), w.list_radius)
    tags = ref.resolve_tags(pairs, w.type_ids, w.term_matrix, w.num_types)
    fref = ref.pair_forces(pairs, w.pos, w.type_ids, tags, tableset(w), box_of(w),
                           np.float32(w.cutoff) ** 2)
    scaled, _ = force_errors(fe, fref.astype(np.float64), fabs)
    assert scaled <= 2e-5


def _bonded_setup(ctx, w):
    dev = setup_workload(ctx, w)
    return dev


def test_bond_and_angle_forces(ctx_factory, oracle):
    w = W.polymers(n_chains=4, beads=1024, with_grid=False)
    ctx = ctx_factory(w.n)
    dev = _bonded_setup(ctx, w)
    ctx.reset_energies()
    ctx.bond_forces(dev["bonds"], dev["bond_idx"], dev["pos"], dev["fe"])
    fb = dev["fe"].cpu().numpy().copy()
    dev["fe"].zero_()
    ctx.angle_forces(dev["angles"], dev["angle_idx"], dev["pos"], dev["fe"])
    fa = dev["fe"].cpu().numpy()
    e = ctx.energies()
    bt = pyoracle.TableSet([(t.values, t.start, t.step_inv) for t in w.bond_tables])
    at = pyoracle.TableSet([(t.values, t.start, t.step_inv) for t in w.angle_tables], periodic=True)
    _, b64, babs = oracle.bond_forces(w.bonds, w.bond_table_idx, w.pos, bt, box_of(w))
    _, a64, aabs = oracle.angle_forces(w.angles, w.angle_table_idx, w.pos, at, box_of(w))
    sb, pb = force_errors(fb, b64, babs)
    print(f"bonds: worst {pb:.3e} (scaled {sb:.3e})")
    assert pb <= 1e-5 and sb <= 1e-5, (pb, sb)
    # Angles within rounding of a table-bin edge may take the neighbouring
    # bin's force (device acosf vs host acos): their particles are reported.
    edge = _angles_near_bin_edge(w, tol=2e-5)
    touched = np.zeros(w.n, bool)
    touched[w.angles[edge, :3].ravel()] = True
    ok = ~touched
    sa, pa = force_errors(fa[ok], a64[ok], aabs[ok])
    print(f"angles: {int(edge.sum())} of {len(w.angles)} within 2e-5 rad of a bin edge "
          f"({int(touched.sum())} particles set aside); others worst {pa:.3e} (scaled {sa:.3e})")
    # Expected share of such angles: 2 * tol / bin width = 0.23 %.
    assert edge.sum() <= max(3, len(w.angles) // 100)
    assert pa <= 1e-5 and sa <= 1e-5, (pa, sa)
    # The set-aside particles: how many of them actually miss the bar.
    if touched.any():
        _, pt = force_errors(fa[touched], a64[touched], aabs[touched])
        d = np.linalg.norm(fa[touched, :3].astype(np.float64) - a64[touched, :3], axis=1)
        print(f"  set-aside particles: worst {pt:.3e}; {int((d > 1e-5 * np.abs(a64[touched, :3]).max()).sum())} "
              f"differ by more than 1e-5 of the largest angle force")
    assert abs(e[2] - b64[:, 3].sum()) <= 1e-6 * abs(b64[:, 3]).sum()
    assert abs(e[3] - a64[:, 3].sum()) <= 1e-5 * abs(a64[:, 3]).sum()


def _angles_near_bin_edge(w, tol):
    """Angles whose FP64 angle lies within tol radians of an edge of their
    (periodic, degree-abscissa) table's bins."""
    p = w.pos[:, :3].astype(np.float64)
    L = np.array(w.box_size, np.float64)
    a = w.angles[:, :3]

    def wrap(d):
        return d - L * np.floor(d / L + 0.5)
    ab = np.linalg.norm(wrap(p[a[:, 1]] - p[a[:, 0]]), axis=1)
    bc = np.linalg.norm(wrap(p[a[:, 2]] - p[a[:, 1]]), axis=1)
    ac = np.linalg.norm(wrap(p[a[:, 2]] - p[a[:, 0]]), axis=1)
    cos = np.clip((ab ** 2 + bc ** 2 - ac ** 2) / (2 * ab * bc), -1.0, 1.0)
    th = np.arccos(cos)
    t = w.angle_tables[0]
    step = 1.0 / float(t.step_inv)
    u = (th - float(t.start)) / step
    return np.abs(u - np.round(u)) * step < tol


def test_bond_chain_end_forces(ctx_factory, oracle):
    """129-bead straight chain at 1.885 A spacing: interior forces cancel, the
    ends feel -/+ the table force (Unit_test/Compute/BDKernels.cpp:222-305)."""
    n = 129
    pos = np.zeros((n, 4), np.float32)
    pos[:, 2] = 1.885 * np.arange(n, dtype=np.float32)
    bonds = np.stack([np.arange(n - 1), np.arange(1, n)], axis=1).astype(np.int32)
    tab = W.harmonic_bond_table(k=19.19, r0=3.8, bins=10001, dx=0.01)
    ctx = ctx_factory(n)
    ctx.set_box((0, 0, 0), (500, 500, 500), (1, 1, 1))
    ctx.set_bonded_tables(0, [(tab.values, tab.start, tab.step_inv)])
    d = torch.from_numpy(pos).cuda()
    fe = torch.zeros_like(d)
    ctx.bond_forces(torch.from_numpy(bonds).cuda(), torch.zeros(n - 1, dtype=torch.int32, device="cuda"),
                    d, fe)
    f = fe.cpu().numpy()
    ts = pyoracle.TableSet([(tab.values, tab.start, tab.step_inv)])
    fm, _ = oracle.table_lookup(ts, 0, 1.885)
    assert abs(f[0, 2] + fm) <= 1e-5 * abs(fm)
    assert abs(f[-1, 2] - fm) <= 1e-5 * abs(fm)
    assert np.abs(f[1:-1, :3]).max() <= 1e-5 * abs(fm)


def test_philox_bit_exact(ctx_factory, oracle):
    ctx = ctx_factory(1)
    seed = ctx.bd_seed(20261203, 0, 17)
    assert seed == oracle.bd_seed(20261203, 0, 17)
    words, normals = ctx.philox(seed, 0, 0x5324120, 17, 4096)
    w = u32(words).reshape(-1, 4)
    for i in (0, 1, 2, 1000, 4095):
        assert np.array_equal(w[i], oracle.philox(seed, i, 0x5324120, 17))
    nz = normals.cpu().numpy()[:, :3]
    # Box-Muller normals: unit variance (BDKernels.cpp:46-91)
    assert abs(nz.mean()) < 0.05 and abs(nz.var() - 1.0) < 0.05


def test_philox_reference_draws(ctx_factory, ref):
    ctx = ctx_factory(1)
    words, _ = ctx.philox(123456789012345, 7, 0x5324120, 3, 1)
    assert np.array_equal(u32(words)[0], ref.philox_int4(123456789012345, 7, 3, 0x5324120, 1)[0])


def _bd_compare(ctx, oracle, w, dev, fe_np, step, grids=None):
    types = pyoracle.TypeSet(w.charge, w.diffusion, w.pmf_terms)
    gs = pyoracle.GridSet(w.grids) if w.grids else None
    seed = oracle.bd_seed(w.seed, 0, step)
    flags = np.zeros(w.n, np.uint32)
    flags[5] = 4  # rigid-body attached: must not move
    dflags = torch.from_numpy(flags.view(np.int32)).cuda()
    dev["fe"].copy_(torch.from_numpy(fe_np))
    ctx.bd_integrate(dev["pos"], dev["fe"], dev["type"], dflags, w.dt, w.kT, step, seed)
    p_gpu = dev["pos"].cpu().numpy()
    f_gpu = dev["fe"].cpu().numpy()
    p_ref, f_ref, _ = oracle.bd_integrate(w.pos, fe_np, w.type_ids, flags, types, gs, box_of(w),
                                          w.dt, w.kT, step, seed)
    return p_gpu, f_gpu, p_ref, f_ref


def test_bd_step_plain(ctx_factory, oracle):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    rng = np.random.default_rng(3)
    fe = np.zeros((w.n, 4), np.float32)
    fe[:, :3] = rng.normal(0, 5, (w.n, 3)).astype(np.float32)
    p_gpu, f_gpu, p_ref, f_ref = _bd_compare(ctx, oracle, w, dev, fe, step=1)
    d = np.abs(p_gpu[:, :3] - p_ref[:, :3])
    d = np.minimum(d, 200.0 - d)  # periodic
    assert d.max() <= 1e-5
    assert np.array_equal(p_gpu[5], w.pos[5])


def test_bd_step_with_grid(ctx_factory, oracle):
    w = W.polymers(n_chains=8, beads=1024, with_grid=True)
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    fe = np.zeros((w.n, 4), np.float32)
    p_gpu, f_gpu, p_ref, f_ref = _bd_compare(ctx, oracle, w, dev, fe, step=3)
    d = np.abs(p_gpu[:, :3] - p_ref[:, :3])
    d = np.minimum(d, 600.0 - d)
    assert d.max() <= 1e-4
    # grid energy in .w is a pure float function of the position: bit-exact
    assert np.array_equal(f_gpu[:, 3], f_ref[:, 3])
    assert (f_ref[:, 3] != 0).sum() > 100


def test_free_diffusion_msd(ctx_factory):
    """Free particles: MSD after k steps = 6 D t within 10 % (BDKernels.cpp:92-220)."""
    n, steps = 20000, 50
    w = W.plain_bd(n=n, box=1e5)
    ctx = ctx_factory(n)
    dev = setup_workload(ctx, w)
    start = dev["pos"].clone()
    for s in range(1, steps + 1):
        dev["fe"].zero_()
        ctx.bd_integrate(dev["pos"], dev["fe"], dev["type"], None, w.dt, w.kT, s,
                         ctx.bd_seed(w.seed, 0, s))
    d = (dev["pos"] - start)[:, :3].double()
    d = d - 1e5 * torch.round(d / 1e5)  # minimum image across the periodic box
    msd = float((d * d).sum(1).mean())
    expect = 6.0 * W.DIFFUSION * w.dt * steps
    assert abs(msd - expect) <= 0.1 * expect


def test_fused_step_matches_composition(ctx_factory, oracle):
    """mb2_step over 25 steps (one rebuild at step 21) against the oracle's
    clear -> pairlist -> pair forces -> BD sequence, positions within 1e-4 A."""
    from mars_md_b200.engine import step_params
    w = W.plain_bd(n=2048, box=160.0)
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    prm = step_params(w)
    box = box_of(w)
    types = pyoracle.TypeSet(w.charge, w.diffusion)
    pos = w.pos.copy()
    rc2 = np.float32(w.cutoff) ** 2
    pairs = None
    ts = tableset(w)
    snap = None
    skin = w.list_radius - w.cutoff
    blen = np.array(w.box_size, np.float32)
    for s in range(1, 26):
        ctx.step(dev["pos"], dev["fe"], dev["type"], None, s, prm)
        # Patch.cpp:86-108: scheduled rebuild, skipped while the skin holds
        rebuild = pairs is None or ((s - 1) % w.rebuild_period == 0 and
                                    oracle.max_displacement(pos, snap, blen) > skin * 0.5)
        if rebuild:
            pairs, _, _ = oracle.build_pairlist(pos, box, w.list_radius)
            snap = pos.copy()
        tags = oracle.resolve_tags(pairs, w.type_ids, w.term_matrix, 1)
        f32, _, _ = oracle.pair_forces(pairs, pos, tags, ts, box, rc2)
        pos, _, _ = oracle.bd_integrate(pos, f32, w.type_ids, None, types, None, box, w.dt, w.kT,
                                        s, oracle.bd_seed(w.seed, 0, s))
    p = dev["pos"].cpu().numpy()
    d = np.abs(p[:, :3] - pos[:, :3])
    d = np.minimum(d, 160.0 - d)
    assert d.max() <= 1e-3, d.max()
    assert np.sqrt((d ** 2).mean()) <= 1e-5
