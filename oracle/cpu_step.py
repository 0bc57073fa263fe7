"""Brownian-dynamics steps on the host CPU, for the benchmark's CPU legs.

TEST/MEASUREMENT INFRASTRUCTURE ONLY: used by bench.py's ``cpu_baseline`` leg
and ``--impl reference`` arm, never by the product.

``kind="reference"`` runs the reference's own functors (oracle/_ref, built from
the reference checkout by oracle/ref_harness); ``kind="port"`` runs this
project's C restatement (oracle/liboracle.so) where the harness is absent.

Step order follows SimManager::execute_force_calculation / execute_integration
for one patch (src/SimManager.cpp:337-504, src/PatchOperation/Patch.cpp:43-352):
clear forces; every `rebuild_period` steps rebuild the pairlist (Morton
domain, encode, stable sort, inverse, gather, cell grid choice, cell ranges,
stencil table, neighbour walk, pair-tag resolve); tabulated pair forces; BD
integrate.

Threads: race-free functors (encode, tag resolve, BD integrate) are chunked
over `nthreads` host threads, following the reference's launch_cpu_kernel
(src/Backend/Kernels.h:204-238). The scatter functors (neighbour emit, pair
forces) cannot share outputs between threads, because the reference's host
atomics are plain `+=`: with the reference's functors each thread runs them
over its own range into its own outputs, joined in order (the harness's
``_mt`` calls); the port runs them on one thread. The sort runs on one thread.

``SampledStep`` bounds the work on a large system: the whole sort and the
whole BD integrate run on all N particles, while the neighbour walk runs for
a strided sample of particles and the pair forces for the pairs that sample
emits. Their times are scaled by N / sample and P / sample, and the rebuild
is amortised over `rebuild_period` steps. With ``walk_sample=None`` every
particle is walked and every pair computed: nothing is scaled.
"""
from __future__ import annotations

import os
import time

import numpy as np

import pyoracle as po


class SampledStep:
    def __init__(self, w, nthreads=None, kind=None, walk_sample=16384):
        self.w = w
        self.nthreads = nthreads or os.cpu_count() or 1
        if kind is None:
            kind = "reference" if po.ref_available() else "port"
        self.kind = kind
        self.O = po.Oracle()
        self.R = po.RefHarness() if kind == "reference" else None
        self.box = po.Box.make(w.box_origin, w.box_size, w.periodic)
        self.tables = po.TableSet([(t.values, t.start, t.step_inv) for t in w.pair_tables])
        self.types = po.TypeSet(w.charge, w.diffusion, w.pmf_terms)
        self.pos = w.pos.copy()
        self.flags = np.zeros(w.n, np.uint32)
        self.walk_sample = w.n if walk_sample is None else min(walk_sample, w.n)
        self.pairs = None
        self.total_pairs_est = 0.0
        self.last = {}

    @property
    def sample_desc(self) -> str:
        return (f"{self.w.name} N={self.w.n}: sort and BD integrate on all N; neighbour walk on "
                f"{self.walk_sample} strided particles and pair forces on the "
                f"{0 if self.pairs is None else len(self.pairs)} pairs they emit, scaled to N "
                f"and to all pairs; rebuild amortised over {self.w.rebuild_period} steps")

    def rebuild(self) -> float:
        """Sort + sampled walk + tag resolve; returns the full-system rebuild time (s)."""
        w, O = self.w, self.O
        R = self.R
        t0 = time.perf_counter()
        bmin, bmax = O.morton_domain(self.box, self.pos)
        if R is not None:
            keys, idx = R.morton_encode(self.pos, bmin, bmax, self.nthreads)
            keys, s2o = R.sort_pairs(keys, idx)
            R.inverse(s2o)
            spos = R.reorder_pos(self.pos, s2o)
        else:
            keys, idx = O.morton_encode(self.pos, bmin, bmax)
            keys, s2o = O.sort_pairs(keys, idx)
            O.inverse(s2o)
            spos = O.gather4(self.pos, s2o)
        m, radii, slots = O.select_cell_grid(bmax - bmin, w.list_radius, w.n, 1 << 40)
        shift = 3 * (10 - m)
        blen = np.array([w.box_size[a] if w.periodic[a] else 0.0 for a in range(3)], np.float32)
        if R is not None:
            begin, end = R.cell_ranges(keys, shift, 1 << (3 * m))
            table = R.cell_neighbors(m, radii, slots, blen)
        else:
            begin, end = O.cell_ranges(keys, shift, 1 << (3 * m))
            table = O.cell_neighbors(m, radii, slots, blen)
        t_sort = time.perf_counter() - t0

        items = (np.arange(self.walk_sample, dtype=np.int64) * w.n // self.walk_sample).astype(np.uint32)
        t0 = time.perf_counter()
        rc2 = np.float32(w.list_radius) ** 2
        if R is not None:
            # Room for 1.5x the half pairs a uniform density would give each item.
            vol = float(np.prod(bmax - bmin))
            per_item = w.n / max(vol, 1e-30) * (4.0 / 3.0) * np.pi * w.list_radius ** 3 / 2.0
            max_pairs = int(self.walk_sample * (1.5 * per_item + 8)) + 4096
            pairs, cnt = R.neighbor_walk_items_mt(spos, keys, s2o, begin, end, table, rc2, slots,
                                                  shift, self.box, items, max_pairs, self.nthreads)
            if pairs is None:
                pairs, cnt = R.neighbor_walk_items_mt(spos, keys, s2o, begin, end, table, rc2,
                                                      slots, shift, self.box, items, cnt,
                                                      self.nthreads)
        else:
            # the port walks the same items through the full-list restatement
            pairs, cnt, _ = O.build_pairlist(self.pos, self.box, w.list_radius)
            pairs = pairs[: self.walk_sample * 200]
            cnt = len(pairs)
        t_walk = time.perf_counter() - t0
        self.pairs = np.ascontiguousarray(pairs)
        scale_walk = w.n / self.walk_sample
        self.total_pairs_est = cnt * scale_walk
        t0 = time.perf_counter()
        if R is not None:
            self.tags = R.resolve_tags(self.pairs, w.type_ids, w.term_matrix, w.num_types,
                                       self.nthreads)
        else:
            self.tags = O.resolve_tags(self.pairs, w.type_ids, w.term_matrix, w.num_types)
        t_tags = time.perf_counter() - t0
        scale_pairs = self.total_pairs_est / max(len(self.pairs), 1)
        total = t_sort + t_walk * scale_walk + t_tags * scale_pairs
        self.last.update(sort_s=t_sort, walk_s=t_walk * scale_walk, tags_s=t_tags * scale_pairs)
        return total

    def forces_and_integrate(self, s: int) -> float:
        """Sampled pair forces (scaled to all pairs) + full BD integrate; seconds."""
        w = self.w
        rc2 = np.float32(w.cutoff) ** 2
        seed = self.O.bd_seed(w.seed, 0, s)
        t0 = time.perf_counter()
        if self.R is not None:
            fe = self.R.pair_forces_mt(self.pairs, self.pos, w.type_ids, self.tags, self.tables,
                                       self.box, rc2, self.nthreads, get_energy=False)
        else:
            fe, _, _ = self.O.pair_forces(self.pairs, self.pos, self.tags, self.tables, self.box,
                                          rc2, get_energy=False)
        t_force = (time.perf_counter() - t0) * self.total_pairs_est / max(len(self.pairs), 1)
        t0 = time.perf_counter()
        if self.R is not None:
            self.pos, _ = self.R.bd_integrate(self.pos, fe, w.type_ids, self.flags, self.types,
                                              None, self.box, w.dt, w.kT, s, seed,
                                              nthreads=self.nthreads)
        else:
            self.pos, _, _ = self.O.bd_integrate(self.pos, fe, w.type_ids, self.flags, self.types,
                                                 None, self.box, w.dt, w.kT, s, seed)
        t_bd = time.perf_counter() - t0
        self.last.update(force_s=t_force, integrate_s=t_bd)
        return t_force + t_bd

    def step(self, s: int) -> float:
        """One step's full-system time estimate (s): rebuild on schedule + forces + BD."""
        t = 0.0
        period = self.w.rebuild_period
        if self.pairs is None or period == 0 or (s - 1) % period == 0:
            t += self.rebuild()
        return t + self.forces_and_integrate(s)

    def window(self, steps: int, first: int = 1) -> float:
        """Per-step time averaged over a window of `steps` steps (rebuilds included)."""
        total = 0.0
        for s in range(first, first + steps):
            total += self.step(s)
        return total / steps
