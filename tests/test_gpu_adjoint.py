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


def _cpu_case(oracle, w, float_bins=False, list_every=0):
    t, b, a = w.pair_tables[0], w.bond_tables[0], w.angle_tables[0]
    return po.Adjoint64(oracle, w.n, w.box_size, w.diffusion[0], w.dt, w.kT,
                        (t.values, t.start, t.step_inv), w.cutoff, w.bonds,
                        (b.values, b.start, b.step_inv), w.angles, (a.values, a.start, a.step_inv),
                        w.exclusions, float_bins=float_bins, list_every=list_every,
                        list_radius=w.list_radius)


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


C5_STEPS = 200


def _c5_workload():
    w = W.adjoint()
    rng = np.random.default_rng(W.DEFAULT_SEED)
    # Off the bond table's bin edges: seeded chains have bonds exactly 5.0 A long.
    w.pos[:, :3] = np.mod(w.pos[:, :3] + rng.normal(scale=0.02, size=(w.n, 3)),
                          w.box_size[0]).astype(np.float32)
    return w


def _c5_device(w, steps, every, rdf):
    """Device gradients of the window loss against a target made with the pair
    table perturbed (sigma 4 -> 4.2 A), with the states the reverse sweep
    differentiated (recorded as it recomputes them) and the final state of the
    forward run."""
    win = Window(w, steps, checkpoint_every=every, rdf=rdf)
    states = torch.empty((steps, w.n, 4), dtype=torch.float32, device="cuda")
    win.record_states(states)
    try:
        pos0 = win.dev["pos"].clone()
        pv0, bv0 = win.pair_values().float(), win.bond_values().float()
        win.set_tables(torch.from_numpy(W.wca_table(sigma=4.2).values).cuda(), bv0)
        target = win.histogram(win.forward(pos0)) * win.norm
        win.set_tables(pv0, bv0)
        xn = win.forward(pos0)
        hist = win.histogram(xn)
        loss = float(win.loss_of(hist, target).item())
        dldh = 2.0 * (hist * win.norm - target) * win.norm
        g0, gp, gb = win.backward(win.histogram_backward(xn, dldh))
        ckpt = win.checkpoints()[:, :, :3].double().cpu().numpy()
        torch.cuda.synchronize()
        return dict(loss=loss, gp=gp.double().cpu().numpy(), gb=gb.double().cpu().numpy(),
                    g0=g0[:, :3].double().cpu().numpy(), ckpt=ckpt,
                    states=states[:, :, :3].double().cpu().numpy(),
                    xn=xn[:, :3].double().cpu().numpy(), noise=_noise(win, steps),
                    target=target.cpu().numpy(), seed=win.prm.seed)
    finally:
        win.close()


def _fp64_grads(A, tr, rdf, w, tgt):
    norm = rdf.norm(w.n, float(np.prod(w.box_size)))
    h = A.rdf(tr[-1], rdf.bins, rdf.bin_width, rdf.r_max, rdf.sigma)
    dldh = 2.0 * (h * norm - tgt) * norm
    lam = A.rdf_grad(tr[-1], rdf.bins, rdf.bin_width, rdf.r_max, rdf.sigma, dldh)
    c0, cp, cb = A.backward(tr, lam)
    return float(np.sum((h * norm - tgt) ** 2)), cp, cb, c0


@pytest.mark.slow
@pytest.mark.parametrize("every", [1, 20])
def test_window_gradients_c5_match_fp64_adjoint(oracle, every):
    """The benchmark's adjoint workload (16 chains x 1,024 beads, box 378 A,
    bonds, angles, 1-2/1-3 exclusions, WCA table), a 200-step window, the
    device's Philox noise, a target made with sigma 4 -> 4.2 A. Gradients with
    respect to the 200 pair-table entries, the 200 bond-table entries and the
    16,384 x 3 initial positions, each within 1e-4 of its largest component of
    the FP64 adjoint along the states the device's reverse sweep
    differentiated (recorded as it recomputed them from its checkpoints,
    every step or every 20), ending at the forward's x_N. The FP64 adjoint
    takes each table bin, cutoff and angle clamp as the float forward decided
    it, its pairs from a list built at each checkpoint as the window's is,
    and does everything else in double.

    The tangent dynamics of this model grow by about 10^4 over 200 steps
    (forces piecewise constant in distance, so no radial stiffness damps a
    perturbation) and a bond crossing a table-bin edge moves its beads by some
    0.03 A, so an FP64 forward from the same x_0 ends elsewhere, and so does
    any float recomputation whose sums run in another order; those are
    printed, not asserted."""
    w = _c5_workload()
    rdf = RdfSpec()
    d = _c5_device(w, C5_STEPS, every, rdf)
    if every == 1:
        # With a checkpoint at every step the recorded states are the stored ones.
        assert np.array_equal(d["states"], d["ckpt"])
    else:
        assert np.array_equal(d["states"][::every], d["ckpt"])
    tr = np.concatenate([d["states"], d["xn"][None]])
    A = _cpu_case(oracle, w, float_bins=True, list_every=every)
    loss64, cp, cb, c0 = _fp64_grads(A, tr, rdf, w, d["target"])
    errs = (_rel(d["gp"], cp), _rel(d["gb"], cb), _rel(d["g0"], c0))
    print(f"C5 200 steps, checkpoints every {every}: loss {d['loss']:.6e} / FP64 {loss64:.6e}; "
          f"relative errors pair table {errs[0]:.2e}, bond table {errs[1]:.2e}, positions "
          f"{errs[2]:.2e}")
    if every != 1:
        own = _fp64_grads(_cpu_case(oracle, w), A.forward(w.pos[:, :3].astype(np.float64),
                                                          d["noise"]), rdf, w, d["target"])
        print(f"  FP64 forward from x_0 instead (not asserted): loss {own[0]:.6e}; pair table "
              f"{_rel(d['gp'], own[1]):.2e}, bond table {_rel(d['gb'], own[2]):.2e}, positions "
              f"{_rel(d['g0'], own[3]):.2e}")
    assert abs(d["loss"] - loss64) <= 1e-4 * abs(loss64)
    assert max(errs) <= 1e-4, errs
