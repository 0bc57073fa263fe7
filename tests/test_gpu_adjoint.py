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


C5_STEPS, C5_EVERY = 200, 20


def _c5_workload():
    w = W.adjoint()
    rng = np.random.default_rng(W.DEFAULT_SEED)
    # Off the bond table's bin edges: seeded chains have bonds exactly 5.0 A long.
    w.pos[:, :3] = np.mod(w.pos[:, :3] + rng.normal(scale=0.02, size=(w.n, 3)),
                          w.box_size[0]).astype(np.float32)
    return w


def _c5_device(w, steps, rdf):
    """Device gradients of the window loss against a target made with the pair
    table perturbed (sigma 4 -> 4.2 A), the device's noise and checkpoints."""
    win = Window(w, steps, checkpoint_every=C5_EVERY, rdf=rdf)
    try:
        pos0 = win.dev["pos"].clone()
        pv0, bv0 = win.pair_values().float(), win.bond_values().float()
        win.set_tables(torch.from_numpy(W.wca_table(sigma=4.2).values).cuda(), bv0)
        target = win.histogram(win.forward(pos0)) * win.norm
        pv = pv0.clone().requires_grad_(True)
        bv = bv0.clone().requires_grad_(True)
        p0 = pos0.clone().requires_grad_(True)
        loss = BDWindowLoss.apply(pv, bv, p0, win, target)
        gp, gb, g0 = torch.autograd.grad(loss, [pv, bv, p0])
        ckpt = win.checkpoints()[:, :, :3].double().cpu().numpy()
        torch.cuda.synchronize()
        noise = _noise(win, steps)
        return dict(loss=loss.item(), gp=gp.double().cpu().numpy(), gb=gb.double().cpu().numpy(),
                    g0=g0[:, :3].double().cpu().numpy(), ckpt=ckpt, noise=noise,
                    target=target.cpu().numpy())
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
def test_window_gradients_c5_match_fp64_adjoint(oracle):
    """The benchmark's adjoint workload (16 chains x 1,024 beads, box 378 A,
    bonds, angles, 1-2/1-3 exclusions, WCA table), checkpoints every 20 steps,
    the device's Philox noise. Gradients with respect to the 200 pair-table
    entries, the 200 bond-table entries and the 16,384 x 3 initial positions,
    each within 1e-4 of its largest FP64 component:

    * the full 200-step window against the FP64 adjoint along the device's own
      checkpoints (each 20-step segment recomputed in FP64 from the device's
      checkpoint, as the device's reverse sweep recomputes it in FP32);
    * a 20-step window (one segment) against the FP64 adjoint of the FP64
      forward from the same x_0.

    The tangent dynamics of this model grow by about 10^4 over 200 steps (the
    forces are piecewise constant in distance, so no radial stiffness damps a
    perturbation), so an FP32 and an FP64 forward from the same x_0 drift apart
    over the full window; that comparison is printed, not asserted."""
    w = _c5_workload()
    rdf = RdfSpec()
    A = _cpu_case(oracle, w)

    d = _c5_device(w, C5_STEPS, rdf)
    # FP64 recompute of each segment from the device's checkpoint.
    segs = []
    for s in range(len(d["ckpt"])):
        seg = A.forward(d["ckpt"][s], d["noise"][s * C5_EVERY:(s + 1) * C5_EVERY])
        segs.append(seg if s == len(d["ckpt"]) - 1 else seg[:-1])
    tr = np.concatenate(segs)
    assert len(tr) == C5_STEPS + 1
    loss64, cp, cb, c0 = _fp64_grads(A, tr, rdf, w, d["target"])
    errs = (_rel(d["gp"], cp), _rel(d["gb"], cb), _rel(d["g0"], c0))
    print(f"C5 200 steps vs FP64 along the device checkpoints: loss {d['loss']:.6e} / "
          f"{loss64:.6e}; pair table {errs[0]:.2e}, bond table {errs[1]:.2e}, positions "
          f"{errs[2]:.2e}")
    own = _fp64_grads(A, A.forward(w.pos[:, :3].astype(np.float64), d["noise"]), rdf, w,
                      d["target"])
    print(f"C5 200 steps vs FP64 on its own trajectory (not asserted): loss {own[0]:.6e}; "
          f"pair table {_rel(d['gp'], own[1]):.2e}, bond table {_rel(d['gb'], own[2]):.2e}, "
          f"positions {_rel(d['g0'], own[3]):.2e}")
    assert abs(d["loss"] - loss64) <= 1e-4 * abs(loss64)
    assert max(errs) <= 1e-4, errs

    d20 = _c5_device(w, C5_EVERY, rdf)
    loss20, cp, cb, c0 = _fp64_grads(A, A.forward(w.pos[:, :3].astype(np.float64), d20["noise"]),
                                     rdf, w, d20["target"])
    errs20 = (_rel(d20["gp"], cp), _rel(d20["gb"], cb), _rel(d20["g0"], c0))
    print(f"C5 system, 20 steps vs FP64 forward and adjoint: loss {d20['loss']:.6e} / "
          f"{loss20:.6e}; pair table {errs20[0]:.2e}, bond table {errs20[1]:.2e}, positions "
          f"{errs20[2]:.2e}")
    assert abs(d20["loss"] - loss20) <= 1e-4 * abs(loss20)
    assert max(errs20) <= 1e-4, errs20
