"""Python host layer over the C ABI, with torch tensors as device memory.

``Context`` wraps one ``mb2_context``; its methods follow the reference's
call surface on the Brownian-dynamics path:

* ``set_box`` / ``set_exclusions`` / ``build_pairlist`` / ``needs_update`` /
  ``export_pairs`` (``get_neighbor_pairs``) / ``num_pairs`` -- the ``Pairlist``
  virtuals (src/PatchOperation/Pairlist.h:85-172);
* ``set_pair_tables`` / ``pair_forces`` -- DevicePairNonBondedInteractions and
  launch_pairwise_nonbonded (src/Interactions/NonBondedInteraction.h:205-296);
* ``set_bonded_tables`` / ``bond_forces`` / ``angle_forces`` --
  launch_tabulated_{bonds,angles} (src/Interactions/DeviceBondedInteraction.h:495-549);
* ``set_particle_types`` / ``set_grid`` / ``bd_integrate`` -- launch_BD
  (src/PatchOperation/Integrator.h:26-54);
* ``step`` -- one SimManager step for one patch (src/SimManager.cpp:337-504).

``Batch`` wraps one ``mb2_batch``: many independent periodic systems stepped
together (one launch per stage for all of them, CUDA-graph step replay, an
autotuner for cell level and lanes per row).

Device arrays are torch CUDA tensors (positions and forces float32 [N, 4]).
torch is only the allocator and stream provider here; every kernel is the
library's own.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L


def _p(t):
    """Device pointer of a tensor (or None)."""
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return C.c_void_p(t.data_ptr())


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Context:
    def __init__(self, max_particles: int, device: int = 0):
        self.lib = L.load()
        self.device = device
        self.max_particles = int(max_particles)
        h = C.c_void_p()
        rc = self.lib.mb2_create(int(device), self.max_particles, C.byref(h))
        if rc != 0:
            raise L.MB2Error(rc, "mb2_create failed (no CUDA device or out of memory)")
        self.h = h
        self._keep = {}

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.mb2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int):
        if rc != 0:
            raise L.MB2Error(rc, self.lib.mb2_last_error(self.h).decode())

    # -- set-up ------------------------------------------------------------
    def set_box(self, origin, size, periodic=(1, 1, 1)):
        self.check(self.lib.mb2_set_box(self.h, _f3(origin), _f3(size),
                                        (C.c_int * 3)(*[int(p) for p in periodic])))

    def set_exclusions(self, offsets=None, neighbors=None, num_particles=0, rigid_body_id=None):
        self._keep["excl"] = (offsets, neighbors, rigid_body_id)
        self.check(self.lib.mb2_set_exclusions(self.h, _p(offsets), _p(neighbors),
                                               int(num_particles), _p(rigid_body_id)))

    @staticmethod
    def _tables(tables):
        vals = np.concatenate([np.asarray(t[0], np.float32) for t in tables]).astype(np.float32)
        sizes = np.array([len(t[0]) for t in tables], np.uint32)
        starts = np.array([t[1] for t in tables], np.float32)
        sinv = np.array([t[2] for t in tables], np.float32)
        return vals, sizes, starts, sinv

    def set_pair_tables(self, num_types, term_matrix, tables):
        """tables: [(values, start, step_inv)]; term_matrix uint32 [T*T]."""
        vals, sizes, starts, sinv = self._tables(tables)
        tm = np.ascontiguousarray(term_matrix, np.uint32)
        self.check(self.lib.mb2_set_pair_tables(
            self.h, int(num_types), tm.ctypes.data_as(C.POINTER(C.c_uint32)), len(tables),
            vals.ctypes.data_as(C.POINTER(C.c_float)), sizes.ctypes.data_as(C.POINTER(C.c_uint32)),
            starts.ctypes.data_as(C.POINTER(C.c_float)), sinv.ctypes.data_as(C.POINTER(C.c_float))))

    def set_bonded_tables(self, kind, tables):
        vals, sizes, starts, sinv = self._tables(tables)
        self.check(self.lib.mb2_set_bonded_tables(
            self.h, int(kind), len(tables), vals.ctypes.data_as(C.POINTER(C.c_float)),
            sizes.ctypes.data_as(C.POINTER(C.c_uint32)), starts.ctypes.data_as(C.POINTER(C.c_float)),
            sinv.ctypes.data_as(C.POINTER(C.c_float))))

    def set_particle_types(self, charge, diffusion, pmf_terms_per_type=None, force_grid_id=None,
                           force_grid_scale=None):
        T = len(charge)
        ch = np.ascontiguousarray(charge, np.float32)
        dif = np.ascontiguousarray(np.asarray(diffusion, np.float32).reshape(T, 3))
        pmf_terms_per_type = pmf_terms_per_type or [[] for _ in range(T)]
        off = np.zeros(T, np.int32)
        cnt = np.zeros(T, np.int32)
        flat = []
        for k, terms in enumerate(pmf_terms_per_type):
            off[k], cnt[k] = len(flat), len(terms)
            flat.extend(terms)
        terms4 = np.array(flat, np.float32).reshape(-1, 4) if flat else np.zeros((1, 4), np.float32)
        fg = None if force_grid_id is None else np.ascontiguousarray(force_grid_id, np.int32).reshape(T, 3)
        fs = None if force_grid_scale is None else np.ascontiguousarray(force_grid_scale, np.float32).reshape(T, 3)
        fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int)
        self.check(self.lib.mb2_set_particle_types(
            self.h, T, ch.ctypes.data_as(fp), dif.ctypes.data_as(fp), off.ctypes.data_as(ip),
            cnt.ctypes.data_as(ip), len(flat), terms4.ctypes.data_as(fp),
            fg.ctypes.data_as(ip) if fg is not None else None,
            fs.ctypes.data_as(fp) if fs is not None else None))

    def set_grid(self, grid_id, data, origin, basis_inv, boundary_condition=0):
        """data: CUDA float32 tensor [nx, ny, nz]; basis_inv 3x3 (row-major numpy)."""
        self._keep[f"grid{grid_id}"] = data
        dims = (C.c_int64 * 3)(*data.shape)
        binv = np.asarray(basis_inv, np.float32)
        colmajor = (C.c_float * 9)(*[float(binv[r, c]) for c in range(3) for r in range(3)])
        self.check(self.lib.mb2_set_grid(self.h, int(grid_id), _p(data), dims, _f3(origin),
                                         colmajor, int(boundary_condition)))

    def set_profiling(self, on: bool):
        self.check(self.lib.mb2_set_profiling(self.h, int(on)))

    def profile_read(self, stage: int):
        """(total ms, launches) of one stage since the last read."""
        ms = C.c_double()
        cnt = C.c_uint32()
        self.check(self.lib.mb2_profile_read(self.h, int(stage), C.byref(ms), C.byref(cnt)))
        return float(ms.value), int(cnt.value)

    def set_lanes_per_row(self, lanes: int):
        self.check(self.lib.mb2_set_lanes_per_row(self.h, int(lanes)))

    # -- sort --------------------------------------------------------------
    def sort_morton(self, pos, bmin, bmax, stream=None):
        n = pos.shape[0]
        dev = pos.device
        keys = torch.empty(n, dtype=torch.int32, device=dev)
        s2o = torch.empty(n, dtype=torch.int32, device=dev)
        inv = torch.empty(n, dtype=torch.int32, device=dev)
        sp = torch.empty_like(pos)
        self.check(self.lib.mb2_sort_morton(self.h, _p(pos), n, _f3(bmin), _f3(bmax), _p(keys),
                                            _p(s2o), _p(inv), _p(sp), _stream(stream)))
        return keys, s2o, inv, sp

    def radix_sort_pairs(self, keys, vals, stream=None):
        self.check(self.lib.mb2_radix_sort_pairs(self.h, _p(keys), _p(vals), keys.shape[0],
                                                 _stream(stream)))

    def radix_sort_pairs_static(self, keys, vals, stream=None):
        """Same sort over the library's static scratch: allocates no device memory
        (n <= MB2_SORT_STATIC_MAX; concurrent calls on one device race)."""
        self.check(self.lib.mb2_radix_sort_pairs_static(self.h, _p(keys), _p(vals),
                                                        keys.shape[0], _stream(stream)))

    # -- pairlist ----------------------------------------------------------
    def build_pairlist(self, pos, type_ids, pairlist_cutoff, stream=None) -> int:
        npairs = C.c_uint64()
        self.check(self.lib.mb2_build_pairlist(self.h, _p(pos), _p(type_ids), pos.shape[0],
                                               float(pairlist_cutoff), _stream(stream),
                                               C.byref(npairs)))
        return int(npairs.value)

    def num_pairs(self) -> int:
        v = C.c_uint64()
        self.check(self.lib.mb2_num_pairs(self.h, C.byref(v)))
        return int(v.value)

    def export_pairs(self, stream=None):
        n = self.num_pairs()
        out = torch.empty((max(n, 1), 2), dtype=torch.int32, device=f"cuda:{self.device}")
        self.check(self.lib.mb2_export_pairs(self.h, _p(out), n, _stream(stream)))
        return out[:n]

    def needs_update(self, pos, skin, stream=None):
        d = C.c_float()
        needs = C.c_int()
        self.check(self.lib.mb2_needs_update(self.h, _p(pos), pos.shape[0], float(skin),
                                             _stream(stream), C.byref(d), C.byref(needs)))
        return float(d.value), bool(needs.value)

    # -- forces ------------------------------------------------------------
    def pair_forces(self, pos, type_ids, fe, cutoff, get_energy=True, stream=None):
        self.check(self.lib.mb2_pair_forces(self.h, _p(pos), _p(type_ids), _p(fe), pos.shape[0],
                                            float(cutoff), int(get_energy), _stream(stream)))

    def bond_forces(self, bonds, table_idx, pos, fe, get_energy=True, stream=None):
        self.check(self.lib.mb2_bond_forces(self.h, _p(bonds), _p(table_idx), bonds.shape[0],
                                            _p(pos), _p(fe), int(get_energy), _stream(stream)))

    def angle_forces(self, angles, table_idx, pos, fe, get_energy=True, stream=None):
        self.check(self.lib.mb2_angle_forces(self.h, _p(angles), _p(table_idx), angles.shape[0],
                                             _p(pos), _p(fe), int(get_energy), _stream(stream)))

    def energies(self, stream=None):
        out = (C.c_double * 4)()
        self.check(self.lib.mb2_energies(self.h, _stream(stream), out))
        return np.array(list(out))

    def reset_energies(self, stream=None):
        self.check(self.lib.mb2_reset_energies(self.h, _stream(stream)))

    # -- integrator --------------------------------------------------------
    def bd_integrate(self, pos, fe, type_ids, flags, dt, kT, step, base_seed, base_ctr=0,
                     efield=(0.0, 0.0, 0.0), stream=None):
        self.check(self.lib.mb2_bd_integrate(self.h, _p(pos), _p(fe), _p(type_ids), _p(flags),
                                             pos.shape[0], float(dt), float(kT), int(step),
                                             int(base_seed), int(base_ctr), _f3(efield),
                                             _stream(stream)))

    def set_langevin_types(self, mass, damping):
        """Per-type mass and damping (x, y, z) for the BAOAB integrator."""
        m = np.ascontiguousarray(mass, np.float32)
        d = np.ascontiguousarray(np.asarray(damping, np.float32).reshape(len(m), 3))
        fp = C.POINTER(C.c_float)
        self.check(self.lib.mb2_set_langevin_types(self.h, len(m), m.ctypes.data_as(fp),
                                                   d.ctypes.data_as(fp)))

    def baoab_integrate(self, pos, mom, fe, type_ids, flags, dt, kT, step, base_seed, base_ctr=0,
                        efield=(0.0, 0.0, 0.0), pending=False, stream=None):
        self.check(self.lib.mb2_baoab_integrate(
            self.h, _p(pos), _p(mom), _p(fe), _p(type_ids), _p(flags), pos.shape[0], float(dt),
            float(kT), int(step), int(base_seed), int(base_ctr), _f3(efield), int(bool(pending)),
            _stream(stream)))

    def baoab_last_update(self, mom, fe, flags, dt, stream=None):
        self.check(self.lib.mb2_baoab_last_update(self.h, _p(mom), _p(fe), _p(flags),
                                                  mom.shape[0], float(dt), _stream(stream)))

    def bd_seed(self, seed, patch_id, step) -> int:
        return int(self.lib.mb2_bd_seed(int(seed), int(patch_id), int(step)))

    def philox(self, seed, ctr0, ctr1, ctr2, n, stream=None):
        out = torch.empty((n, 4), dtype=torch.int32, device=f"cuda:{self.device}")
        nrm = torch.empty((n, 4), dtype=torch.float32, device=f"cuda:{self.device}")
        self.check(self.lib.mb2_philox(self.h, int(seed), int(ctr0), int(ctr1), int(ctr2), int(n),
                                       _p(out), _p(nrm), _stream(stream)))
        return out, nrm

    def step(self, pos, fe, type_ids, flags, step, params: "L.StepParams", stream=None):
        self.check(self.lib.mb2_step(self.h, _p(pos), _p(fe), _p(type_ids), _p(flags),
                                     pos.shape[0], int(step), C.byref(params), _stream(stream)))


def step_params(w, seed=None, patch_id=0, get_energy=False, bonds=None, bond_idx=None,
                angles=None, angle_idx=None) -> L.StepParams:
    """StepParams for a workload (see mars_md_b200.workloads)."""
    p = L.StepParams()
    p.pairlist_cutoff = float(w.list_radius)
    p.cutoff = float(w.cutoff)
    p.rebuild_period = int(w.rebuild_period)
    p.dt = float(w.dt)
    p.kT = float(w.kT)
    p.seed = int(w.seed if seed is None else seed)
    p.patch_id = int(patch_id)
    p.get_energy = int(get_energy)
    if bonds is not None:
        p.bonds2, p.bond_table_idx, p.num_bonds = bonds.data_ptr(), bond_idx.data_ptr(), bonds.shape[0]
    if angles is not None:
        p.angles4, p.angle_table_idx, p.num_angles = angles.data_ptr(), angle_idx.data_ptr(), angles.shape[0]
    return p


def setup_workload(ctx: Context, w, device="cuda:0"):
    """Upload a workload's box, tables, types and grids; returns device tensors."""
    ctx.set_box(w.box_origin, w.box_size, w.periodic)
    ctx.set_pair_tables(w.num_types, w.term_matrix,
                        [(t.values, t.start, t.step_inv) for t in w.pair_tables])
    dev = {}
    dev["pos"] = torch.from_numpy(w.pos).to(device)
    dev["type"] = torch.from_numpy(w.type_ids).to(device)
    dev["fe"] = torch.zeros((w.n, 4), dtype=torch.float32, device=device)
    dev["flags"] = torch.zeros(w.n, dtype=torch.int32, device=device)
    if w.bond_tables:
        ctx.set_bonded_tables(0, [(t.values, t.start, t.step_inv) for t in w.bond_tables])
        dev["bonds"] = torch.from_numpy(w.bonds).to(device)
        dev["bond_idx"] = torch.from_numpy(w.bond_table_idx).to(device)
    if w.angle_tables:
        ctx.set_bonded_tables(1, [(t.values, t.start, t.step_inv) for t in w.angle_tables])
        dev["angles"] = torch.from_numpy(w.angles).to(device)
        dev["angle_idx"] = torch.from_numpy(w.angle_table_idx).to(device)
    grids = []
    for g, spec in enumerate(w.grids):
        data = torch.from_numpy(np.ascontiguousarray(spec["data"], np.float32)).to(device)
        grids.append(data)
        binv = np.linalg.inv(np.asarray(spec["basis"], np.float64)).astype(np.float32)
        ctx.set_grid(g, data, spec["origin"], binv, spec.get("boundary_condition", 0))
    dev["grids"] = grids
    ctx.set_particle_types(w.charge, w.diffusion, w.pmf_terms)
    return dev


class Batch:
    """Batched replicas: systems concatenated in one set of arrays; system s
    steps as a plain context with seed (params.seed + s) would."""

    def __init__(self, counts, box_sizes, box_origins=None, device: int = 0):
        self.lib = L.load()
        self.device = device
        self.counts = np.ascontiguousarray(counts, np.uint32)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.n = int(self.offsets[-1])
        sizes = np.ascontiguousarray(box_sizes, np.float32).reshape(-1, 3)
        origins = None if box_origins is None else \
            np.ascontiguousarray(box_origins, np.float32).reshape(-1, 3)
        fp = C.POINTER(C.c_float)
        h = C.c_void_p()
        rc = self.lib.mb2_batch_create(
            int(device), len(self.counts), self.counts.ctypes.data_as(C.POINTER(C.c_uint32)),
            None if origins is None else origins.ctypes.data_as(fp), sizes.ctypes.data_as(fp),
            C.byref(h))
        if rc != 0:
            raise L.MB2Error(rc, "mb2_batch_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.mb2_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int):
        if rc != 0:
            raise L.MB2Error(rc, self.lib.mb2_batch_last_error(self.h).decode())

    def set_pair_tables(self, num_types, term_matrix, tables):
        vals, sizes, starts, sinv = Context._tables(tables)
        tm = np.ascontiguousarray(term_matrix, np.uint32)
        fp = C.POINTER(C.c_float)
        self.check(self.lib.mb2_batch_set_pair_tables(
            self.h, int(num_types), tm.ctypes.data_as(C.POINTER(C.c_uint32)), len(tables),
            vals.ctypes.data_as(fp), sizes.ctypes.data_as(C.POINTER(C.c_uint32)),
            starts.ctypes.data_as(fp), sinv.ctypes.data_as(fp)))

    def set_particle_types(self, charge, diffusion):
        q = np.ascontiguousarray(charge, np.float32)
        d = np.ascontiguousarray(diffusion, np.float32).reshape(-1, 3)
        fp = C.POINTER(C.c_float)
        self.check(self.lib.mb2_batch_set_particle_types(self.h, len(q), q.ctypes.data_as(fp),
                                                         d.ctypes.data_as(fp)))

    def build(self, pos, type_ids, pairlist_cutoff, stream=None) -> int:
        npairs = C.c_uint64()
        self.check(self.lib.mb2_batch_build(self.h, _p(pos), _p(type_ids), float(pairlist_cutoff),
                                            _stream(stream), C.byref(npairs)))
        return int(npairs.value)

    def num_pairs(self) -> int:
        v = C.c_uint64()
        self.check(self.lib.mb2_batch_num_pairs(self.h, C.byref(v)))
        return int(v.value)

    def export_pairs(self, stream=None):
        n = self.num_pairs()
        out = torch.empty((max(n, 1), 2), dtype=torch.int32, device=f"cuda:{self.device}")
        self.check(self.lib.mb2_batch_export_pairs(self.h, _p(out), n, _stream(stream)))
        return out[:n]

    def step(self, pos, fe, type_ids, step, params: "L.StepParams", stream=None):
        self.check(self.lib.mb2_batch_step(self.h, _p(pos), _p(fe), _p(type_ids), int(step),
                                           C.byref(params), _stream(stream)))

    def run(self, pos, fe, type_ids, first_step, num_steps, params: "L.StepParams", stream=None):
        self.check(self.lib.mb2_batch_run(self.h, _p(pos), _p(fe), _p(type_ids), int(first_step),
                                          int(num_steps), C.byref(params), _stream(stream)))

    def set_tuning(self, level_offset=0, lanes=0):
        self.check(self.lib.mb2_batch_set_tuning(self.h, int(level_offset), int(lanes)))

    def tuning(self):
        lvl, lanes, cells = C.c_int(), C.c_int(), C.c_uint32()
        self.check(self.lib.mb2_batch_tuning(self.h, C.byref(lvl), C.byref(lanes), C.byref(cells)))
        return lvl.value, lanes.value, cells.value

    def autotune(self, pos, type_ids, params: "L.StepParams", trial_steps=4, stream=None) -> dict:
        r = L.BatchTuning()
        self.check(self.lib.mb2_batch_autotune(self.h, _p(pos), _p(type_ids), C.byref(params),
                                               int(trial_steps), _stream(stream), C.byref(r)))
        return {k: getattr(r, k) for k, _ in L.BatchTuning._fields_}


def setup_batch(ws, device="cuda:0"):
    """A Batch over workloads that share tables and types (e.g. workloads.batched());
    returns (batch, device tensors of the concatenated systems)."""
    w0 = ws[0]
    b = Batch([w.n for w in ws], [w.box_size for w in ws], [w.box_origin for w in ws],
              device=torch.device(device).index or 0)
    b.set_pair_tables(w0.num_types, w0.term_matrix,
                      [(t.values, t.start, t.step_inv) for t in w0.pair_tables])
    b.set_particle_types(w0.charge, w0.diffusion)
    dev = {"pos": torch.from_numpy(np.concatenate([w.pos for w in ws])).to(device),
           "type": torch.from_numpy(np.concatenate([w.type_ids for w in ws])).to(device)}
    dev["fe"] = torch.zeros((b.n, 4), dtype=torch.float32, device=device)
    return b, dev
