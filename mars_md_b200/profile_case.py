"""A small, self-contained case for kernel profiling (ncu) of the hot path.

    python -m mars_md_b200.profile_case [N] [--steps S]
    python -m mars_md_b200.profile_case --workload polymers [--steps S]

large_plain (default): the benchmark's workload at N beads (same density and
tables as the 2,097,152-bead benchmark; default 1,048,576 so the pairlist
still exceeds L2); one pairlist build, two pair-force launches (with
--split-rows one more build, whose rows put near pairs first as the fused
step's builds do, and two more launches) and S fused steps.

polymers: the 65,536-bead polymer workload with bonds, angles, 1-2/1-3
exclusions and the 256^3 grid potential; S fused steps (the integrate kernel
samples the grid for every bead each step).

batched: the 512 batched systems (500 to 20,000 beads each, 2,742,131 in
all) at the default tuning with a rebuild at every step (the cadence the
autotuner picks for them); S batched steps.

Few launches precede the kernels of interest, as ncu captures need.
"""
import argparse
import sys

import torch

from . import workloads as W
from .engine import Context, exclusion_csr, setup_workload, step_params


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("n", nargs="?", type=int, default=1_048_576)
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--split-rows", action="store_true",
                    help="rebuild once more with near/far rows at the interaction cutoff")
    ap.add_argument("--workload", choices=("large_plain", "polymers", "batched"),
                    default="large_plain")
    a = ap.parse_args(argv)
    if a.workload == "polymers":
        return polymers(a.steps)
    if a.workload == "batched":
        return batched(a.steps)
    w = W.large_plain(n=a.n)
    ctx = Context(w.n)
    dev = setup_workload(ctx, w)
    ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius)
    for _ in range(2):
        dev["fe"].zero_()
        ctx.pair_forces(dev["pos"], dev["type"], dev["fe"], w.cutoff, get_energy=False)
    if a.split_rows:
        # Rows split at the interaction cutoff (near pairs first), as the fused
        # step's builds are; two more launches.
        ctx.build_pairlist(dev["pos"], dev["type"], w.list_radius, w.cutoff)
        for _ in range(2):
            dev["fe"].zero_()
            ctx.pair_forces(dev["pos"], dev["type"], dev["fe"], w.cutoff, get_energy=False)
    prm = step_params(w)
    for s in range(1, a.steps + 1):
        ctx.step(dev["pos"], dev["fe"], dev["type"], None, s, prm)
    torch.cuda.synchronize()
    print("ok", w.n, ctx.num_pairs())
    ctx.close()


def polymers(steps):
    w = W.polymers()
    ctx = Context(w.n)
    dev = setup_workload(ctx, w)
    _, off, nb, npart = exclusion_csr(w.exclusions)
    d_off, d_nb = torch.from_numpy(off).cuda(), torch.from_numpy(nb).cuda()
    ctx.set_exclusions(d_off, d_nb, npart)
    prm = step_params(w, bonds=dev["bonds"], bond_idx=dev["bond_idx"], angles=dev["angles"],
                      angle_idx=dev["angle_idx"])
    for s in range(1, steps + 1):
        ctx.step(dev["pos"], dev["fe"], dev["type"], None, s, prm)
    torch.cuda.synchronize()
    print("ok", w.n, ctx.num_pairs())
    ctx.close()


def batched(steps):
    from .engine import setup_batch
    ws = W.batched(seed=W.DEFAULT_SEED)
    prm = step_params(ws[0], seed=W.DEFAULT_SEED)
    b, dev = setup_batch(ws)
    b.set_rebuild_period(1)
    b.run(dev["pos"], dev["fe"], dev["type"], 1, steps, prm)
    torch.cuda.synchronize()
    print("ok", sum(w.n for w in ws), b.num_pairs())
    b.close()


if __name__ == "__main__":
    main(sys.argv[1:])
