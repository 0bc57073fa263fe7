"""A small, self-contained case for kernel profiling (ncu) of the hot path.

    python -m mars_md_b200.profile_case [N] [--steps S]

Builds the large_plain workload at N beads (same density and tables as the
2,097,152-bead benchmark; default 1,048,576 so the pairlist still exceeds L2),
runs one pairlist build, two pair-force launches (with --split-rows one more
build, whose rows put near pairs first as the fused step's builds do, and two
more launches) and S fused steps, then exits.
Few launches precede the kernels of interest, as ncu captures need.
"""
import argparse
import sys

import torch

from . import workloads as W
from .engine import Context, setup_workload, step_params


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("n", nargs="?", type=int, default=1_048_576)
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--split-rows", action="store_true",
                    help="rebuild once more with near/far rows at the interaction cutoff")
    a = ap.parse_args(argv)
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


if __name__ == "__main__":
    main(sys.argv[1:])
