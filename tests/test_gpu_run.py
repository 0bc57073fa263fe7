"""mb2_run (Context.run): many steps, the ones between rebuild checks replayed
from a captured CUDA graph, against one mb2_step call per step: the plain
4,096-bead workload over three rebuild checks, a bonded polymer system with
exclusions and a grid, runs split across calls, a parameter change that forces
a new capture, and the Langevin branch (which runs step by step).

Two contexts stepping the same system agree to the last bits only up to the
order of the float atomics that add the pair forces (a few ulps of
ForceEnergy on some particles from the first step). Where that puts a pair
on the other side of a table-bin edge, the particle's path jumps by D dt / kT
times the bins' force difference (of order 1e-2 A) and follows its own
course from there. So the trajectories are held as the trajectory test holds
them: 99 % of the particles within 1e-4 A and every particle within 0.05 A
(a few such jumps). A wrong step number in the replayed graph (another
Philox stream) would move every particle by the noise, about 0.2 A a step."""
import numpy as np
import pytest
import torch

from mars_md_b200 import _lib as L
from mars_md_b200 import workloads as W
from mars_md_b200.engine import exclusion_csr, setup_workload, step_params

pytestmark = pytest.mark.gpu


def _two(ctx_factory, w):
    out = []
    for _ in range(2):
        ctx = ctx_factory(w.n)
        dev = setup_workload(ctx, w)
        if w.exclusions is not None:
            _, off, nb, npart = exclusion_csr(w.exclusions)
            dev["excl"] = (torch.from_numpy(off).cuda(), torch.from_numpy(nb).cuda())
            ctx.set_exclusions(dev["excl"][0], dev["excl"][1], npart)
        out.append((ctx, dev))
    return out


def _params(w, dev, **kw):
    return step_params(w, bonds=dev.get("bonds"), bond_idx=dev.get("bond_idx"),
                       angles=dev.get("angles"), angle_idx=dev.get("angle_idx"), **kw)


def _same(a, b, box=None):
    torch.cuda.synchronize()
    pa, pb = a["pos"].cpu().numpy()[:, :3], b["pos"].cpu().numpy()[:, :3]
    d = np.abs(pa - pb)
    if box is not None:
        d = np.minimum(d, np.asarray(box, np.float32) - d)
    d = d.max(axis=1)
    assert d.max() <= 0.05, float(d.max())
    assert (d <= 1e-4).mean() >= 0.99, int((d > 1e-4).sum())
    fa, fb = a["fe"].cpu().numpy()[:, :3], b["fe"].cpu().numpy()[:, :3]
    scale = np.abs(fb).max()
    assert (np.abs(fa - fb).max(axis=1) <= 1e-4 * scale).mean() >= 0.99


def test_run_matches_step_loop_plain(ctx_factory):
    w = W.plain_bd()
    (a, da), (b, db) = _two(ctx_factory, w)
    prm = _params(w, da)
    lib = L.load()
    l0 = lib.mb2_launch_count()
    a.run(da["pos"], da["fe"], da["type"], None, 1, 60, prm)
    launches = lib.mb2_launch_count() - l0
    for s in range(1, 61):
        b.step(db["pos"], db["fe"], db["type"], None, s, prm)
    _same(da, db, w.box_size)
    assert launches >= 3 * 60  # replayed kernels are counted too


def test_run_matches_step_loop_bonded_with_grid(ctx_factory):
    w = W.polymers(n_chains=8, beads=256, box=300.0, with_grid=True)
    (a, da), (b, db) = _two(ctx_factory, w)
    prm = _params(w, da, get_energy=True)
    a.run(da["pos"], da["fe"], da["type"], None, 1, 45, prm)
    for s in range(1, 46):
        b.step(db["pos"], db["fe"], db["type"], None, s, prm)
    _same(da, db, w.box_size)


def test_split_runs_and_recapture(ctx_factory):
    """Runs that start between rebuild checks, and a time step changed half
    way (the graph bakes it in and must be captured again)."""
    w = W.plain_bd()
    (a, da), (b, db) = _two(ctx_factory, w)
    prm = _params(w, da)
    prm2 = _params(w, da)
    prm2.dt = prm.dt * 0.5
    a.run(da["pos"], da["fe"], da["type"], None, 1, 7, prm)
    a.run(da["pos"], da["fe"], da["type"], None, 8, 23, prm)
    a.run(da["pos"], da["fe"], da["type"], None, 31, 30, prm2)
    for s in range(1, 31):
        b.step(db["pos"], db["fe"], db["type"], None, s, prm)
    for s in range(31, 61):
        b.step(db["pos"], db["fe"], db["type"], None, s, prm2)
    _same(da, db, w.box_size)


def test_run_langevin_matches_step_loop(ctx_factory):
    w = W.plain_bd()
    (a, da), (b, db) = _two(ctx_factory, w)
    mass = np.full(1, 100.0, np.float32)
    damping = np.full((1, 3), 5.0, np.float32)
    moms = []
    for ctx in (a, b):
        ctx.set_langevin_types(mass, damping)
        moms.append(torch.zeros((w.n, 4), dtype=torch.float32, device="cuda"))
    pa, pb = _params(w, da), _params(w, db)
    pa.integrator = pb.integrator = 1
    pa.mom4, pb.mom4 = moms[0].data_ptr(), moms[1].data_ptr()
    a.run(da["pos"], da["fe"], da["type"], None, 1, 25, pa)
    for s in range(1, 26):
        b.step(db["pos"], db["fe"], db["type"], None, s, pb)
    _same(da, db, w.box_size)
    ma, mb = moms[0].cpu().numpy()[:, :3], moms[1].cpu().numpy()[:, :3]
    assert (np.abs(ma - mb).max(axis=1) <= 1e-4 * np.abs(mb).max()).mean() >= 0.99


def test_run_argument_errors(ctx_factory):
    w = W.plain_bd()
    ctx = ctx_factory(w.n)
    dev = setup_workload(ctx, w)
    prm = _params(w, dev)
    prm.integrator = 3
    with pytest.raises(L.MB2Error):
        ctx.run(dev["pos"], dev["fe"], dev["type"], None, 1, 5, prm)
