"""Benchmark: Brownian-dynamics particle-steps/s on the 2,097,152-bead workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full BD step of the hot path (clear forces, pairlist rebuild
every 20 steps, tabulated pair forces, BD integrate with Philox noise) on the
`large_plain` workload: 2,097,152 beads of 4 types at 0.002 A^-3 in a periodic
cube, 10 pair tables of 400 bins, cutoff 30 A, pairlist radius 35 A. Inputs
are seeded synthetic data (no dataset). The pairlist (~1.5 GB) is far larger
than L2, so every timed step streams it from HBM (no L2 flush needed).

Multi-GPU: the path does not shard; N GPUs run N independent replicas (one
process per GPU, weak scaling), and `value` counts all replicas' work over
the slowest rank's time.

`e2e` is the same trajectory with the positions owned by the host
(engine.HostStepper.advance: pinned upload, fused step, read-back every
step). At N=1 the line also carries `batched` (512 independent systems in one
batch against the same systems run one after another), `adjoint` (adjoint
window step against the forward step) and `small_plain` (a 4,096-bead system
through one mb2_step call per step and through mb2_run).

`--impl reference` times the reference's own CPU implementation of the path
(its functors host-compiled in oracle/_ref) on every host thread, on the whole
workload: each step computes every particle and pair, the wall clock times the
steps.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "particle-steps/s"
WORKLOAD = "large_plain"


def _config(w, extra=None):
    cfg = {"workload": f"{WORKLOAD}: {w.n} beads, 4 types, 10 pair tables x 400 bins, "
                       f"cutoff {w.cutoff} A, pairlist {w.list_radius} A, rebuild every "
                       f"{w.rebuild_period} steps, box {w.box_size[0]:.1f} A periodic",
           "beads": w.n, "rebuild_period": w.rebuild_period,
           "l2": "inputs larger than L2 (the ~1.5 GB pairlist is streamed every step)",
           "seed": w.seed}
    if extra:
        cfg.update(extra)
    return cfg


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML read every 5 ms from a thread (the timed region is tens of
    milliseconds), else nvidia-smi every 50 ms. Read-only; nothing is set."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.samples = []      # (time, sm MHz, set of reason names)
        self.max_mhz = None
        self.window = None
        self._stop = None
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"mb2_clocks_{os.getpid()}.csv")

    def _nvml_handle(self, nv):
        try:
            import torch
            p = torch.cuda.get_device_properties(self.dev)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            h = self._nvml_handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            self._stop = threading.Event()

            def poll():
                while not self._stop.is_set():
                    try:
                        sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((time.perf_counter(), sm,
                                             {n for n, b in zip(self.NAMES, bits) if r & b}))
                    except Exception:
                        pass
                    self._stop.wait(0.005)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self._stop = None
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                stderr=subprocess.DEVNULL)
            time.sleep(1.0)  # first sample before the timed region
        except Exception:
            self.proc = None

    def begin(self):
        self.window = [time.perf_counter(), None]
        self._lines0 = self._count_lines()

    def end(self):
        if self.window is not None:
            self.window[1] = time.perf_counter()

    def _count_lines(self):
        if self.proc is None:
            return 0
        try:
            self.f.flush()
            with open(self.path) as f:
                return sum(1 for _ in f)
        except Exception:
            return 0

    def stop(self):
        if self._stop is not None:
            self._stop.set()
            self.thread.join(timeout=2)
            t0, t1 = self.window if self.window else (0.0, float("inf"))
            inside = [x for x in self.samples if t0 <= x[0] <= (t1 or float("inf"))]
            if not inside:  # nearest sample after the region began
                inside = [x for x in self.samples if x[0] >= t0][:1]
            if not inside:
                return None
            return {"sm_mhz": float(np.median([x[1] for x in inside])), "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(set().union(*[x[2] for x in inside])),
                    "samples": len(inside), "source": "nvml, 5 ms"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        rows = rows[getattr(self, "_lines0", 0):] or rows[-1:]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for k, name in enumerate(self.NAMES):
                if r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows), "source": "nvidia-smi, 50 ms"}


def _traffic_from_profile():
    """Per-launch DRAM bytes of the pair-force kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "pair_force_large_plain.json")
    if not os.path.exists(path):
        return None
    try:
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    except Exception:
        return None


def _b_ps(p_half, period, bonded=0.0, grid=0.0):
    """Algorithmic bytes per particle-step of the step (float4 position read and
    write, one u32 per stored half pair, the rebuild's sort and list writes
    amortised over the rebuild period, bonded index tuples, grid taps)."""
    return 32.0 + 4.0 * p_half + (100.0 + 4.0 * p_half) / max(period, 1) + bonded + grid


def _roofline(value, b_ps, bw):
    roof = bw * 1e9 / b_ps
    return {"bytes_per_particle_step": b_ps, "roofline_particle_steps_per_s": roof,
            "frac": value / roof, "peak_gbs": bw}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from mars_md_b200 import _lib, workloads as W
    from mars_md_b200.engine import Context, HostStepper, setup_workload, step_params
    from mars_md_b200.replicas import job_throughput, max_over_ranks, rank_env, replica_seed

    world, rank, local = rank_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    w = W.large_plain(seed=replica_seed(W.DEFAULT_SEED, rank))
    ctx = Context(w.n, device=local)
    dev = setup_workload(ctx, w, device=f"cuda:{local}")
    if args.lanes:
        ctx.set_lanes_per_row(args.lanes)
    prm = step_params(w)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    s = 0
    for _ in range(args.warmup):
        s += 1
        ctx.step(dev["pos"], dev["fe"], dev["type"], None, s, prm)
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    L = _lib.load()
    launches0 = L.mb2_launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clocks.begin()
    start.record(stream)
    rebuilds = 0
    for _ in range(args.steps):
        s += 1
        if (s - 1) % w.rebuild_period == 0:
            rebuilds += 1
        ctx.step(dev["pos"], dev["fe"], dev["type"], None, s, prm)
    stop.record(stream)
    torch.cuda.synchronize()
    clocks.end()
    launches = int(L.mb2_launch_count() - launches0)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(start.elapsed_time(stop), device=f"cuda:{local}")
    value = job_throughput(w.n, args.steps, ms, world)

    # Per-kernel device time over one rebuild period, on the launching stream.
    ctx.set_profiling(True)
    for _ in range(w.rebuild_period):
        s += 1
        ctx.step(dev["pos"], dev["fe"], dev["type"], None, s, prm)
    torch.cuda.synchronize()
    prof = {name: ctx.profile_read(st) for name, st in
            (("step", _lib.STAGE_STEP), ("pairlist_build", _lib.STAGE_PAIRLIST),
             ("pair_force_kernel", _lib.STAGE_PAIR_FORCE), ("integrate_kernel", _lib.STAGE_INTEGRATE))}
    ctx.set_profiling(False)
    npairs = ctx.num_pairs()
    p_half = npairs / w.n

    # e2e: the same trajectory through the public API with the positions owned
    # by the host (engine.HostStepper.advance): every step uploads them from
    # pinned memory, runs the fused step and reads the integrated positions
    # back into the same pinned buffer, which the next step uploads. The
    # rebuild cadence is the timed loop's (the skin check sees the
    # trajectory's own displacements). Only the read-back of one step and the
    # upload of the next overlap, chunk by chunk.
    host_pos = torch.empty((w.n, 4), dtype=torch.float32).pin_memory()
    host_pos.copy_(dev["pos"])
    stepper = HostStepper(ctx, dev["type"], prm)
    for _ in range(2):  # first use of the stepper's streams and buffers
        s += 1
        stepper.advance(host_pos, s)
    stepper.finish()
    e_steps = args.steps
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e_rebuilds = 0
    for _ in range(e_steps):
        s += 1
        if (s - 1) % w.rebuild_period == 0:
            e_rebuilds += 1
        stepper.advance(host_pos, s)
    stepper.finish()
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = max_over_ranks(e0.elapsed_time(e1), device=f"cuda:{local}")
    e_value = job_throughput(w.n, e_steps, e_ms, world)

    bw, peak_kind = _peaks()
    pf_ms, pf_n = prof["pair_force_kernel"]
    pf_avg = pf_ms / max(pf_n, 1)
    # Algorithmic bytes of one pair-force launch: one u32 index per stored half
    # pair, plus one float4 position read and one float4 force write per bead.
    pf_bytes = w.n * (4.0 * p_half + 32.0)
    achieved = pf_bytes / (pf_avg / 1e3) / 1e9
    traffic = _traffic_from_profile()
    b_ps = 32.0 + 4.0 * p_half + (100.0 + 4.0 * p_half) / w.rebuild_period
    roof_ps = bw * 1e9 / b_ps
    # HBM GB/s per kernel from algorithmic bytes over the CUDA-event time: the
    # pair-force launch (above); the integrate (position read and write, the
    # pair force gathered through the inverse map with its index, type id,
    # ForceEnergy write: 72 B per bead); the rebuild (sort, cell ranges and
    # list writes: 100 B per bead plus 4 B per stored half pair).
    per_kernel_bytes = {"pair_force_kernel": pf_bytes, "integrate_kernel": w.n * 72.0,
                        "pairlist_build": w.n * (100.0 + 4.0 * p_half)}
    kernel_gbs = {}
    for k, nbytes in per_kernel_bytes.items():
        t_ms, cnt = prof[k]
        if cnt:
            gbs = nbytes / (t_ms / cnt / 1e3) / 1e9
            kernel_gbs[k] = {"gbs": gbs, "frac": gbs / bw, "bytes_per_launch": nbytes}

    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform beads, Debye-Hueckel + soft-core tables)",
        "config": _config(w, {"parallelism": f"replicas x{world}", "pairs": npairs,
                              "p_half": p_half, "rebuilds_in_timed_region": rebuilds,
                              "step_roofline_bytes_per_particle_step": b_ps,
                              "step_roofline_particle_steps_per_s": roof_ps,
                              "step_roofline_frac": (value / world) / roof_ps,
                              "kernel_ms": {k: (v[0] / max(v[1], 1)) for k, v in prof.items()},
                              "kernel_gbs": kernel_gbs,
                              "hbm_peak": peak_kind}),
        "roofline": {"bound": "hbm", "kernel": "pair_force", "achieved": achieved, "peak": bw,
                     "unit": "GB/s", "frac": achieved / bw, "traffic": traffic,
                     "algorithmic_bytes_per_launch": pf_bytes,
                     "launch_ms": pf_avg,
                     "peak_source": ("MEASURED_PEAKS.json (measured)" if peak_kind == "measured"
                                     else "fallback 6,650 GB/s (no MEASURED_PEAKS.json)")},
        "e2e": {"value": e_value, "unit": METRIC, "h2d_bytes_per_step": w.n * 16,
                "d2h_bytes_per_step": w.n * 16, "rebuilds_in_timed_region": e_rebuilds,
                "mode": "host-owned trajectory: each step uploads the positions read back "
                        "after the previous one (pinned; read-back and next upload overlap "
                        "in 8 chunks)"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    cpu = rank == 0 and world == 1 and not args.no_cpu_baseline
    if world == 1 and not (args.no_batched and args.no_adjoint):
        del dev
        ctx.close()
        torch.cuda.empty_cache()
        if not args.no_batched:
            out["batched"] = run_batched(local, bw)
            if cpu:
                out["batched"]["cpu_baseline"] = cpu_baseline_batched()
        if not args.no_adjoint:
            out["adjoint"] = run_adjoint(local, bw)
            if cpu:
                out["adjoint"]["cpu_baseline"] = cpu_baseline_adjoint(local)
        if not args.no_batched:
            out["small_plain"] = run_small(local)
            if cpu:
                out["small_plain"]["cpu_baseline"] = cpu_baseline_small()
            out["polymers_grid"] = run_polymers_grid(local, bw)
    if cpu:
        out["cpu_baseline"] = cpu_baseline(w)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_small(local, steps=400):
    """The 4,096-bead plain workload (one type, 200 A periodic box, WCA table,
    20 / 25 A radii, rebuild checks every 20 steps): device time per step with
    one mb2_step call per step and with mb2_run (steps between rebuild checks
    replayed from a CUDA graph)."""
    import torch
    from mars_md_b200 import workloads as W
    from mars_md_b200.engine import Context, setup_workload, step_params
    w = W.plain_bd()
    res = {"metric": "particle-steps/s, small plain system: step calls vs graph-replayed run",
           "beads": w.n, "steps": steps}
    for mode in ("step", "run"):
        ctx = Context(w.n, device=local)
        dev = setup_workload(ctx, w, device=f"cuda:{local}")
        prm = step_params(w)
        ctx.run(dev["pos"], dev["fe"], dev["type"], None, 1, 40, prm)  # warm-up and capture
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        if mode == "step":
            for s in range(41, 41 + steps):
                ctx.step(dev["pos"], dev["fe"], dev["type"], None, s, prm)
        else:
            ctx.run(dev["pos"], dev["fe"], dev["type"], None, 41, steps, prm)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        res[f"us_per_step_{mode}"] = 1e3 * ms / steps
        res[f"value_{mode}"] = w.n * steps / (ms / 1e3)
        ctx.close()
    res["ratio"] = res["value_run"] / res["value_step"]
    return res


def run_batched(local, bw, period_steps=20):
    """512 independent systems (sizes log-uniform in [500, 20000], own periodic boxes at
    0.002 A^-3, WCA table, cutoff 20 A, list 25 A). The autotuner picks the cell level,
    the lanes per row and the rebuild cadence (after its own equilibration, on a copy)
    and puts them in force; the systems then run two periods untimed, past the
    transient of the random start, and a window of two periods is timed. The same
    systems as 512 sequential plain runs through mb2_run, with the same cadence, the
    same equilibration and the same window, are the comparison."""
    import torch
    from mars_md_b200 import _lib, workloads as W
    from mars_md_b200.engine import Context, setup_batch, setup_workload, step_params

    device = f"cuda:{local}"
    stream = torch.cuda.current_stream()
    L = _lib.load()
    ws = W.batched(seed=W.DEFAULT_SEED)
    total = sum(w.n for w in ws)
    prm = step_params(ws[0], seed=W.DEFAULT_SEED)
    equil, window = 2 * period_steps, 2 * period_steps
    b, dev = setup_batch(ws, device=device)
    tune = b.autotune(dev["pos"], dev["type"], prm, trial_steps=4)
    cadence, _ = b.rebuild_schedule()
    b.run(dev["pos"], dev["fe"], dev["type"], 1, equil, prm)  # untimed: past the transient
    torch.cuda.synchronize()
    _, r0 = b.rebuild_schedule()
    sr0 = b.system_rebuilds()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = L.mb2_launch_count()
    e0.record(stream)
    b.run(dev["pos"], dev["fe"], dev["type"], equil + 1, window, prm)
    e1.record(stream)
    torch.cuda.synchronize()
    batched_launches = int(L.mb2_launch_count() - l0)
    batched_ms = e0.elapsed_time(e1)
    _, r1 = b.rebuild_schedule()
    sr1 = b.system_rebuilds()
    npairs = b.num_pairs()
    b.close()
    del dev
    torch.cuda.empty_cache()

    # The same systems as sequential plain runs: one context per system, each run
    # through the window (mb2_run, same cadence) before the next system starts.
    ctxs = []
    for s, w in enumerate(ws):
        c = Context(w.n, device=local)
        d = setup_workload(c, w, device=device)
        p = step_params(w, seed=W.DEFAULT_SEED + s)
        p.rebuild_period = cadence
        ctxs.append((c, d, p))
    for c, d, p in ctxs:
        c.run(d["pos"], d["fe"], d["type"], None, 1, equil, p)
    torch.cuda.synchronize()
    l0 = L.mb2_launch_count()
    e0.record(stream)
    for c, d, p in ctxs:
        c.run(d["pos"], d["fe"], d["type"], None, equil + 1, window, p)
    e1.record(stream)
    torch.cuda.synchronize()
    seq_launches = int(L.mb2_launch_count() - l0)
    seq_ms = e0.elapsed_time(e1)
    for c, _, _ in ctxs:
        c.close()
    bv = total * window / (batched_ms / 1e3)
    sv = total * window / (seq_ms / 1e3)
    return {"metric": "particle-steps/s, batched vs sequential plain runs (mb2_run)",
            "roofline": _roofline(bv, _b_ps(npairs / total, cadence), bw),
            "systems": len(ws), "beads": total, "steps": window, "equilibration_steps": equil,
            "rebuild_period_used": cadence, "rebuilds_in_window": int(r1 - r0),
            "system_rebuilds_in_window": int(sr1 - sr0),
            "pairs": npairs, "value": bv, "sequential_value": sv, "ratio": bv / sv,
            "ms": batched_ms, "sequential_ms": seq_ms, "gpu_launches": batched_launches,
            "sequential_gpu_launches": seq_launches,
            "tuning": {k: (float(v) if isinstance(v, float) else v) for k, v in tune.items()},
            "workload": "512 systems, sizes log-uniform in [500, 20000] beads, own periodic "
                        "boxes at 0.002 A^-3, WCA table, cutoff 20 A, list 25 A, rebuild "
                        "cadence autotuned (at most 20), each system rebuilt on its own skin "
                        "check, seeded synthetic"}


def run_adjoint(local, bw, steps=200, every=20):
    """16 chains x 1,024 beads (bonds, angles, exclusions, WCA table), a 200-step window
    with fixed Philox noise, checkpoints every 20 steps; loss = squared error of the
    smoothed pair-distance histogram (100 bins on [0, 25) A) against a target made with
    the pair table perturbed (sigma 4 -> 4.2 A). Times the forward window and the
    adjoint (histogram gradient + recompute + reverse sweep) with CUDA events."""
    import torch
    from mars_md_b200 import workloads as W
    from mars_md_b200.adjoint import Window

    device = f"cuda:{local}"
    stream = torch.cuda.current_stream()
    w = W.adjoint()
    rng = np.random.default_rng(W.DEFAULT_SEED)
    w.pos[:, :3] = np.mod(w.pos[:, :3] + rng.normal(scale=0.02, size=(w.n, 3)),
                          w.box_size[0]).astype(np.float32)
    win = Window(w, steps, checkpoint_every=every, device=device)
    pos0 = win.dev["pos"].clone()
    pv, bv = win.pair_values().float(), win.bond_values().float()
    # Target from the perturbed table.
    win.set_tables(torch.from_numpy(W.wca_table(sigma=4.2).values).to(device), bv)
    target = win.histogram(win.forward(pos0)) * win.norm
    win.set_tables(pv, bv)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for rep in range(2):  # the first repetition warms up
        e[0].record(stream)
        xn = win.forward(pos0)
        e[1].record(stream)
        hist = win.histogram(xn)
        dldh = 2.0 * (hist * win.norm - target) * win.norm
        e[2].record(stream)
        lam = win.histogram_backward(xn, dldh)
        g0, gp, gb = win.backward(lam)
        e[3].record(stream)
        torch.cuda.synchronize()
    fwd_ms, bwd_ms = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])
    loss = float(win.loss_of(hist, target).item())
    p_half = win.ctx.num_pairs() / w.n
    win.close()
    # B_adj = 2 B_ps + 32: the forward recompute and the reverse pass each read
    # the step's bytes, plus the float4 adjoint read and write. Bonded terms:
    # an (i, j) pair and a table index per bond, an int4 and an index per angle.
    bonded = (8 + 4) * len(w.bonds) / w.n + (16 + 4) * len(w.angles) / w.n
    b_adj = 2.0 * _b_ps(p_half, every, bonded) + 32.0
    adj_value = w.n * steps / (bwd_ms / 1e3)
    return {"metric": "adjoint step / forward step (device time)", "beads": w.n,
            "window_steps": steps, "checkpoint_every": every,
            "forward_ms_per_step": fwd_ms / steps, "adjoint_ms_per_step": bwd_ms / steps,
            "ratio": bwd_ms / fwd_ms,
            "forward_particle_steps_per_s": w.n * steps / (fwd_ms / 1e3),
            "adjoint_particle_steps_per_s": adj_value,
            "roofline": dict(_roofline(adj_value, b_adj, bw), p_half=p_half,
                             note="B_adj = 2 B_ps + 32 with B_ps of the window's step "
                                  "(list rebuilt at each of the 10 checkpoints, bonds, angles)"),
            "loss": loss, "grad_norms": {"positions": float(g0.norm().item()),
                                         "pair_table": float(gp.norm().item()),
                                         "bond_table": float(gb.norm().item())},
            "workload": "16 chains x 1,024 beads, one type, WCA table, harmonic bonds and "
                        "angles, 1-2/1-3 exclusions, box 378 A, seeded synthetic"}


def run_polymers_grid(local, bw, steps=200):
    """The 65,536-bead polymer workload (64 chains x 1,024 beads, two types,
    harmonic bond and angle tables, 1-2/1-3 exclusions, three WCA pair tables,
    the 256^3 cylindrical-pore grid potential on both types, 600 A periodic
    box): particle-steps/s through mb2_run over `steps` steps after a warm-up
    period, and the integrate kernel (grid sampling, Philox noise, pair-force
    gather) against its bytes."""
    import torch
    from mars_md_b200 import _lib, workloads as W
    from mars_md_b200.engine import Context, exclusion_csr, setup_workload, step_params
    w = W.polymers()
    ctx = Context(w.n, device=local)
    device = f"cuda:{local}"
    dev = setup_workload(ctx, w, device=device)
    _, off, nb, npart = exclusion_csr(w.exclusions)
    d_off, d_nb = torch.from_numpy(off).to(device), torch.from_numpy(nb).to(device)
    ctx.set_exclusions(d_off, d_nb, npart)
    prm = step_params(w, bonds=dev["bonds"], bond_idx=dev["bond_idx"], angles=dev["angles"],
                      angle_idx=dev["angle_idx"])
    ctx.run(dev["pos"], dev["fe"], dev["type"], None, 1, w.rebuild_period, prm)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    ctx.run(dev["pos"], dev["fe"], dev["type"], None, w.rebuild_period + 1, steps, prm)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    value = w.n * steps / (ms / 1e3)
    # Per-stage device time over one rebuild period (event timers on).
    ctx.set_profiling(True)
    first = w.rebuild_period + steps + 1
    for k in range(first, first + w.rebuild_period):
        ctx.step(dev["pos"], dev["fe"], dev["type"], None, k, prm)
    torch.cuda.synchronize()
    prof = {name: ctx.profile_read(st) for name, st in
            (("step", _lib.STAGE_STEP), ("pairlist_build", _lib.STAGE_PAIRLIST),
             ("pair_force_kernel", _lib.STAGE_PAIR_FORCE),
             ("integrate_kernel", _lib.STAGE_INTEGRATE))}
    ctx.set_profiling(False)
    p_half = ctx.num_pairs() / w.n
    ctx.close()
    bonded = (8 + 4) * len(w.bonds) / w.n + (16 + 4) * len(w.angles) / w.n
    b_ps = _b_ps(p_half, w.rebuild_period, bonded, 32.0)
    int_ms = prof["integrate_kernel"][0] / max(prof["integrate_kernel"][1], 1)
    # Integrate kernel, per bead: position read and write (32 B), the pair force
    # gathered through the inverse map (16 + 4 B), ForceEnergy read and write
    # (32 B, bonded terms in, energy out), type id (4 B), 8 grid taps (32 B).
    int_bytes = w.n * 120.0
    return {"metric": "particle-steps/s, polymers with bonds, angles, exclusions and grid",
            "beads": w.n, "steps": steps, "value": value, "ms_per_step": ms / steps,
            "p_half": p_half, "roofline": _roofline(value, b_ps, bw),
            "kernel_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
            "integrate_kernel": {"ms": int_ms, "bytes_per_launch": int_bytes,
                                 "achieved_gbs": int_bytes / (int_ms / 1e3) / 1e9,
                                 "frac": int_bytes / (int_ms / 1e3) / 1e9 / bw},
            "workload": "64 chains x 1,024 beads (65,536), 2 types, 600 A periodic box, "
                        "harmonic bond and angle tables, 1-2/1-3 exclusions, 3 WCA pair tables, "
                        "256^3 float32 cylindrical-pore grid (1 A), cutoff 20 A, list 25 A, "
                        "rebuild checks every 20 steps, seeded synthetic"}


def cpu_baseline_small(steps=1000):
    """The 4,096-bead plain workload on the host, every one of its 1,000 steps
    run in full (the reference's functors from oracle/_ref, else the oracle):
    wall-clock time of the whole loop, nothing extrapolated."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_step
    from mars_md_b200 import workloads as W
    w = W.plain_bd()
    c = cpu_step.SampledStep(w, walk_sample=w.n)
    t0 = time.perf_counter()
    parts = c.window(steps)
    wall = time.perf_counter() - t0
    return {"value": w.n * steps / wall, "unit": METRIC, "cores": c.nthreads, "kind": c.kind,
            "sample": f"plain_bd N={w.n}: all {steps} steps in full (rebuild every "
                      f"{w.rebuild_period} steps, every pair, every particle); wall clock of the "
                      f"loop ({wall:.1f} s; the functors alone {parts * steps:.1f} s)",
            "wall_s": wall}


def cpu_baseline_batched(every=64, steps=20):
    """The batched workload on the host: every `every`-th system run in full for
    one rebuild period (sort, walk, tag resolve, pair forces, BD integrate; the
    reference's functors), particle-steps/s over the sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_step
    from mars_md_b200 import workloads as W
    ws = W.batched(seed=W.DEFAULT_SEED)[::every]
    beads, wall, kind, cores = 0, 0.0, None, None
    for w in ws:
        c = cpu_step.SampledStep(w, walk_sample=w.n)
        t0 = time.perf_counter()
        c.window(steps)
        wall += time.perf_counter() - t0
        beads += w.n
        kind, cores = c.kind, c.nthreads
    return {"value": beads * steps / wall, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"{len(ws)} of the 512 systems (every {every}th, {beads} beads) run in "
                      f"full for {steps} steps, wall clock {wall:.1f} s"}


def cpu_baseline_adjoint(local, steps=200, every=20):
    """The adjoint workload on the host: the FP64 restatement of the window and
    its adjoint (oracle/mb2_adjoint.c, threaded pair loops) timed over the
    200-step window, particle-steps/s of the reverse sweep. Beside it, as the
    checker: the device's gradients of the benchmark's window (checkpoints
    every 20 steps) against the FP64 adjoint along the states the device's
    reverse sweep differentiated (recorded as it recomputed them; max-normalised
    relative errors)."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from mars_md_b200 import workloads as W
    from mars_md_b200.adjoint import Window
    device = f"cuda:{local}"
    w = W.adjoint()
    rng = np.random.default_rng(W.DEFAULT_SEED)
    w.pos[:, :3] = np.mod(w.pos[:, :3] + rng.normal(scale=0.02, size=(w.n, 3)),
                          w.box_size[0]).astype(np.float32)
    win = Window(w, steps, checkpoint_every=every, device=device)
    recorded = torch.empty((steps, w.n, 4), dtype=torch.float32, device=device)
    win.record_states(recorded)
    pos0 = win.dev["pos"].clone()
    pv, bv = win.pair_values().float(), win.bond_values().float()
    win.set_tables(torch.from_numpy(W.wca_table(sigma=4.2).values).to(device), bv)
    target = win.histogram(win.forward(pos0)) * win.norm
    win.set_tables(pv, bv)
    xn = win.forward(pos0)
    hist = win.histogram(xn)
    dldh = 2.0 * (hist * win.norm - target) * win.norm
    g0, gp, gb = win.backward(win.histogram_backward(xn, dldh))
    states = np.concatenate([recorded[:, :, :3].double().cpu().numpy(),
                             xn[None, :, :3].double().cpu().numpy()])
    noise = []
    for k in range(1, steps + 1):
        seed = win.ctx.bd_seed(win.prm.seed, win.prm.patch_id, k)
        noise.append(win.ctx.philox(seed, 0, 0x5324120, k, w.n)[1][:, :3].double().cpu().numpy())
    noise = np.stack(noise)
    tgt = target.cpu().numpy()
    norm = win.rdf.norm(w.n, float(np.prod(w.box_size)))
    r = win.rdf
    win.close()
    O = po.Oracle()
    t, bt, at = w.pair_tables[0], w.bond_tables[0], w.angle_tables[0]

    def system(float_bins):
        return po.Adjoint64(O, w.n, w.box_size, w.diffusion[0], w.dt, w.kT,
                            (t.values, t.start, t.step_inv), w.cutoff, w.bonds,
                            (bt.values, bt.start, bt.step_inv), w.angles,
                            (at.values, at.start, at.step_inv), w.exclusions,
                            float_bins=float_bins, list_every=every if float_bins else 0,
                            list_radius=w.list_radius)

    def grads(A, tr):
        h = A.rdf(tr[-1], r.bins, r.bin_width, r.r_max, r.sigma)
        lam = A.rdf_grad(tr[-1], r.bins, r.bin_width, r.r_max, r.sigma,
                         2.0 * (h * norm - tgt) * norm)
        return A.backward(tr, lam)

    A = system(False)
    t0 = time.perf_counter()
    tr = A.forward(w.pos[:, :3].astype(np.float64), noise)
    t1 = time.perf_counter()
    grads(A, tr)
    t2 = time.perf_counter()
    c0, cp, cb = grads(system(True), states)

    def rel(a, b):
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
    return {"value": w.n * steps / (t2 - t1), "unit": METRIC,
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)), "kind": "port",
            "sample": f"adjoint N={w.n}: the whole {steps}-step window in FP64 (forward "
                      f"{t1 - t0:.1f} s, histogram gradient and reverse sweep {t2 - t1:.1f} s)",
            "forward_value": w.n * steps / (t1 - t0),
            "gradient_errors_vs_fp64": {
                "pair_table": rel(gp.double().cpu().numpy(), cp),
                "bond_table": rel(gb.double().cpu().numpy(), cb),
                "positions": rel(g0[:, :3].double().cpu().numpy(), c0),
                "how": f"device window with checkpoints every {every} steps against the "
                       "FP64 adjoint along the states its reverse sweep differentiated "
                       "(table bins as the float forward decided them, pairs from a list "
                       "built at each checkpoint), max-normalised"}}


def cpu_baseline(w):
    """The reference's CPU path on the whole system: one pairlist rebuild and one
    force-and-integrate step of all 2,097,152 beads on every host thread, the
    rebuild amortised over its period (about 20-40 s of CPU work)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_step
    c = cpu_step.SampledStep(w, walk_sample=None)
    t0 = time.perf_counter()
    c.rebuild()
    t1 = time.perf_counter()
    c.forces_and_integrate(1)
    t2 = time.perf_counter()
    per_step = (t2 - t1) + (t1 - t0) / w.rebuild_period
    return {"value": w.n / per_step, "unit": METRIC, "cores": c.nthreads, "kind": c.kind,
            "sample": f"{w.name} N={w.n}, every particle and pair: one rebuild "
                      f"({t1 - t0:.1f} s, amortised over {w.rebuild_period} steps) and one "
                      f"force-and-integrate step ({t2 - t1:.1f} s), wall clock; the reference's "
                      f"functors on {c.nthreads} threads (scatter functors over per-thread "
                      f"outputs), sort on one",
            "components_s": dict(c.last)}


def run_reference(args):
    from mars_md_b200.replicas import rank_env
    world, rank, local = rank_env()
    if rank != 0:
        return
    from mars_md_b200 import workloads as W
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_step
    w = W.large_plain()
    # Every particle and pair of the workload each step (nothing sampled or
    # scaled), the rebuild at its period, timed by the wall clock.
    c = cpu_step.SampledStep(w, walk_sample=None)
    s = 0
    for _ in range(args.warmup):
        s += 1
        c.step(s)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s += 1
        c.step(s)
    total = time.perf_counter() - t0
    value = w.n * args.steps / total
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": _config(w, {"parallelism": "host CPU"}),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": c.nthreads, "kind": c.kind,
                         "sample": f"{w.name} N={w.n}: every particle and pair each step, "
                                   f"rebuild every {w.rebuild_period} steps; {args.steps} "
                                   f"steps timed by the wall clock ({total:.1f} s)"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-replicas measurement")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint-window measurement")
    ap.add_argument("--lanes", type=int, default=0,
                    help="lanes per pairlist row in the pair kernel (0 = automatic)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
