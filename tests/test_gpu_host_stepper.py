"""engine.HostStepper: steps fed from pinned host memory, with their copies on
streams of their own (a host-owned trajectory whose read-back and next upload
overlap chunk by chunk; independent inputs on double buffers), give the
positions of the same steps on device buffers. Two contexts agree up to the
order of the float atomics that add the pair forces; where that puts a pair
across a table-bin edge the particle's path jumps by about 1e-2 A, so
trajectories are held to 1e-4 A for 99 % of the particles and 0.05 A for
every one; a single step from the same input is held the same way."""
import numpy as np
import pytest
import torch

from mars_md_b200 import workloads as W
from mars_md_b200.engine import HostStepper, setup_workload, step_params

pytestmark = pytest.mark.gpu


def _close(got, want, box):
    d = np.abs(np.asarray(got)[:, :3] - np.asarray(want)[:, :3])
    d = np.minimum(d, np.asarray(box, np.float32) - d).max(axis=1)
    assert d.max() <= 0.05, float(d.max())
    assert (d <= 1e-4).mean() >= 0.99, int((d > 1e-4).sum())


def _pair(ctx_factory):
    w = W.plain_bd()
    a, b = ctx_factory(w.n), ctx_factory(w.n)
    dev_a, dev_b = setup_workload(a, w), setup_workload(b, w)
    return w, a, dev_a, b, dev_b, step_params(w)


def test_host_owned_trajectory_matches_device_trajectory(ctx_factory):
    """advance(): 60 steps (three rebuild checks) with the positions living in
    pinned host memory, odd chunk sizes included."""
    w, a, dev_a, b, dev_b, prm = _pair(ctx_factory)
    stepper = HostStepper(a, dev_a["type"], prm, chunks=7)
    h_pos = torch.from_numpy(w.pos.copy()).pin_memory()
    for s in range(1, 61):
        stepper.advance(h_pos, s)
        b.step(dev_b["pos"], dev_b["fe"], dev_b["type"], None, s, prm)
    stepper.finish()
    torch.cuda.synchronize()
    _close(h_pos.numpy(), dev_b["pos"].cpu().numpy(), w.box_size)
    with pytest.raises(RuntimeError):  # one pattern per stepper
        stepper.submit(h_pos, h_pos, 61)
    with pytest.raises(ValueError):  # pageable host memory
        stepper.advance(torch.from_numpy(w.pos.copy()), 61)


def test_trajectory_through_host_matches_device_steps(ctx_factory):
    w, a, dev_a, b, dev_b, prm = _pair(ctx_factory)
    stepper = HostStepper(a, dev_a["type"], prm)
    h_in = torch.from_numpy(w.pos.copy()).pin_memory()
    h_out = [torch.empty_like(h_in).pin_memory() for _ in range(2)]
    for s in range(1, 61):
        ev = stepper.submit(h_in, h_out[s & 1], s)
        b.step(dev_b["pos"], dev_b["fe"], dev_b["type"], None, s, prm)
        ev.synchronize()
        h_in.copy_(h_out[s & 1])  # the next step starts from this one's result
    torch.cuda.synchronize()
    _close(h_in.numpy(), dev_b["pos"].cpu().numpy(), w.box_size)


def test_independent_inputs_overlap_and_match(ctx_factory):
    """Several submissions in flight from different host inputs: every read-back
    equals the in-line sequence's result for the same input and step."""
    w, a, dev_a, b, dev_b, prm = _pair(ctx_factory)
    stepper = HostStepper(a, dev_a["type"], prm)
    rng = np.random.default_rng(7)
    jitter = [w.pos + np.concatenate([rng.normal(0, 0.05, (w.n, 3)), np.zeros((w.n, 1))], 1)
              .astype(np.float32) for _ in range(6)]
    h_in = [torch.from_numpy(p).pin_memory() for p in jitter]
    h_out = [torch.empty_like(h_in[0]).pin_memory() for _ in range(6)]
    for k in range(6):
        stepper.submit(h_in[k], h_out[k], k + 1)
    stepper.finish()
    torch.cuda.synchronize()
    for k in range(6):
        dev_b["pos"].copy_(h_in[k])
        b.step(dev_b["pos"], dev_b["fe"], dev_b["type"], None, k + 1, prm)
        _close(h_out[k].numpy(), dev_b["pos"].cpu().numpy(), w.box_size)
