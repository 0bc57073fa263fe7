"""The CUDA adjoint of a BD window against the FP64 CPU adjoint
(oracle/mb2_adjoint.c, itself checked against central finite differences in
tests/test_oracle_adjoint.py), on the same chains, tables and Philox noise:
gradients of the smoothed pair-distance-histogram loss with respect to the
pair table, the bond table and the initial positions, through the
torch.autograd.Function. Tolerances are relative to the largest component
of each FP64 gradient (FP32 forward and adjoint against FP64)."""
import numpy as np
import pytest
import torch

import pyoracle as po
from mars_md_b200 import workloads as W
from mars_md_b200.adjoint import BDWindowLoss, RdfSpec, Window

pytestmark = pytest.mark.gpu

STEPS = 6
TOL = 2e-4
BD_STREAM = 0x5324120


def _workload():
    w = W.adjoint(seed=7, n_chains=4, beads=32)
    rng = np.random.default_rng(5)
    # Off the bond table's bin edges: seeded chains have bonds exactly 5.0 A long.
    w.pos[:, :3] = np.mod(w.pos[:, :3] + rng.normal(scale=0.02, size=(w.n, 3)),
                          w.box_size[0]).astype(np.float32)
    return w


def _cpu_case(oracle, w):
    t, b, a = w.pair_tables[0], w.bond_tables[0], w.angle_tables[0]
    return po.Adjoint64(oracle, w.n, w.box_size, w.diffusion[0], w.dt, w.kT,
                        (t.values, t.start, t.step_inv), w.cutoff, w.bonds,
                        (b.values, b.start, b.step_inv), w.angles, (a.values, a.start, a.step_inv),
                        w.exclusions)


def _noise(win, steps):
    """The window's Philox normals, step by step (key mixed with the absolute step)."""
    out = []
    for k in range(1, steps + 1):
        seed = win.ctx.bd_seed(win.prm.seed, win.prm.patch_id, k)
        _, nrm = win.ctx.philox(seed, 0, BD_STREAM, k, win.w.n)
        out.append(nrm[:, :3].double().cpu().numpy())
    return np.stack(out)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("every", [1, 3])
def test_window_gradients_match_fp64_adjoint(oracle, every):
    w = _workload()
    rdf = RdfSpec()
    win = Window(w, STEPS, checkpoint_every=every, rdf=rdf)
    win.prm.rebuild_period = every
    try:
        pos0 = win.dev["pos"].clone()
        target = win.histogram(pos0) * win.norm * 0.9
        pv = win.pair_values().float().requires_grad_(True)
        bv = win.bond_values().float().requires_grad_(True)
        p0 = pos0.clone().requires_grad_(True)
        loss = BDWindowLoss.apply(pv, bv, p0, win, target)
        gp, gb, g0 = torch.autograd.grad(loss, [pv, bv, p0])
        torch.cuda.synchronize()

        A = _cpu_case(oracle, w)
        noise = _noise(win, STEPS)
        x0 = w.pos[:, :3].astype(np.float64)
        tr = A.forward(x0, noise)
        norm = rdf.norm(w.n, float(np.prod(w.box_size)))
        tgt = target.cpu().numpy()
        h = A.rdf(tr[-1], rdf.bins, rdf.bin_width, rdf.r_max, rdf.sigma)
        loss64 = float(np.sum((h * norm - tgt) ** 2))
        dldh = 2.0 * (h * norm - tgt) * norm
        lam = A.rdf_grad(tr[-1], rdf.bins, rdf.bin_width, rdf.r_max, rdf.sigma, dldh)
        c0, cp, cb = A.backward(tr, lam)

        assert abs(loss.item() - loss64) <= 1e-4 * abs(loss64)
        assert np.count_nonzero(cp) > 10 and np.count_nonzero(cb) > 5
        errs = (_rel(gp.double().cpu().numpy(), cp), _rel(gb.double().cpu().numpy(), cb),
                _rel(g0[:, :3].double().cpu().numpy(), c0))
        print("relative errors (pair table, bond table, positions):", errs)
        assert max(errs) < TOL, errs
        assert torch.all(g0[:, 3] == 0)
    finally:
        win.close()


def test_window_forward_keeps_x0_and_matches_plain_steps():
    """The checkpointed forward is the plain fused step sequence."""
    from mars_md_b200.engine import Context, setup_workload, step_params
    w = _workload()
    win = Window(w, STEPS, checkpoint_every=1)
    win.prm.rebuild_period = 1
    try:
        pos0 = win.dev["pos"].clone()
        xn = win.forward(pos0)
        assert torch.equal(pos0, win.dev["pos"])
        ctx = Context(w.n)
        dev = setup_workload(ctx, w)
        off, nb = win.dev["excl_off"], win.dev["excl_nb"]
        ctx.set_exclusions(off, nb, w.n)
        prm = step_params(w, seed=win.prm.seed, bonds=dev["bonds"], bond_idx=dev["bond_idx"],
                          angles=dev["angles"], angle_idx=dev["angle_idx"])
        prm.rebuild_period = 1
        for k in range(1, STEPS + 1):
            ctx.step(dev["pos"], dev["fe"], dev["type"], None, k, prm)
        torch.cuda.synchronize()
        d = (xn - dev["pos"]).abs()[:, :3].cpu().numpy()
        d = np.minimum(d, np.abs(d - w.box_size[0]))
        assert d.max() < 1e-4
        ctx.close()
    finally:
        win.close()
