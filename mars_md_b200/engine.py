"""Python host layer over the C ABI, with torch tensors as device memory.

``Context`` wraps one ``mb2_context``; its methods follow the reference's
call surface on the Brownian-dynamics path:

* ``set_box`` / ``set_exclusions`` / ``build_pairlist`` / ``needs_update`` /
  ``export_pairs`` (``get_neighbor_pairs``) / ``num_pairs`` -- the ``Pairlist``
  virtuals (src/PatchOperation/Pairlist.h:85-172);
* ``set_pair_tables`` / ``pair_forces`` -- DevicePairNonBondedInteractions and
  launch_pairwise_nonbonded (src/Interactions/NonBondedInteraction.h:205-296);
* ``set_pair_terms`` -- the analytical pair terms of PairNonbondedComputer
  (src/Interactions/Nonbonded/Pairwise.h:214-304, Columb.h);
* ``set_bonded_tables`` / ``bond_forces`` / ``angle_forces`` /
  ``dihedral_forces`` / ``restraint_forces`` -- launch_tabulated_{bonds,angles,
  dihedrals} and launch_harmonic_restraints
  (src/Interactions/DeviceBondedInteraction.h:495-620);
* ``set_particle_types`` / ``set_grid`` / ``bd_integrate`` -- launch_BD
  (src/PatchOperation/Integrator.h:26-54);
* ``step`` -- one SimManager step for one patch (src/SimManager.cpp:337-504);
  ``run`` -- many of them, the steps between rebuild checks replayed from a
  CUDA graph;
* ``reorder_*`` / ``reorder_particles`` / ``ReorderManager`` -- the canonical
  Morton reorder of a patch (src/PatchOperation/Patch.cpp:455-480);
* ``Output`` -- DCD frames, the energy file and restart files
  (src/SimManager.cpp:541-1135, src/IO/DcdWriter.h);
* ``HostStepper`` -- steps fed from and read back to pinned host memory, the
  copies of neighbouring steps overlapping the device work.

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

    def set_pair_terms(self, charge, radius, eps, debye_length=10.0, dielectric=80.0,
                       onck_kappa=0.1, onck_sz=80.0, onck_z=6.86, gaussian_amp=1.0,
                       gaussian_sigma=1.0, gaussian_cutoff_sq=0.0):
        """Analytical pair terms: per-type charge / softcore radius / eps plus
        the solvent and Gaussian constants (defaults: the reference's)."""
        T = len(charge)
        fp = C.POINTER(C.c_float)
        arrs = [np.ascontiguousarray(a, np.float32) for a in (charge, radius, eps)]
        prm = L.PairParams(debye_length, dielectric, onck_kappa, onck_sz, onck_z, gaussian_amp,
                           gaussian_sigma, gaussian_cutoff_sq)
        self.check(self.lib.mb2_set_pair_terms(self.h, T, *[a.ctypes.data_as(fp) for a in arrs],
                                               C.byref(prm)))

    def set_bonded_tables(self, kind, tables):
        """kind 0 bonds, 1 angles, 2 dihedrals."""
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

    def set_cell_level_offset(self, offset: int):
        self.check(self.lib.mb2_set_cell_level_offset(self.h, int(offset)))

    def cell_level(self) -> int:
        v = C.c_int()
        self.check(self.lib.mb2_cell_level(self.h, C.byref(v)))
        return int(v.value)

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

    # -- canonical reorder -------------------------------------------------
    def reorder_begin(self, pos, stream=None):
        """Morton permutation of the positions over the periodic box (the
        pairlist becomes stale)."""
        self.check(self.lib.mb2_reorder_begin(self.h, _p(pos), pos.shape[0], _stream(stream)))
        self._reorder_n = pos.shape[0]

    def reorder_apply(self, t, stream=None):
        """Permute one per-particle tensor in place: [n] of 4-byte or [n, 4] of
        4-byte elements."""
        n = t.shape[0]
        width = t.numel() // max(n, 1) * t.element_size()
        if width not in (4, 16):
            raise ValueError("reorder_apply: rows of 4 or 16 bytes")
        self.check(self.lib.mb2_reorder_apply(self.h, _p(t), width, n, _stream(stream)))

    def reorder_remap(self, indices, stream=None):
        """indices (int32, any shape) -> inverse[indices] where in [0, n)."""
        self.check(self.lib.mb2_reorder_remap(self.h, _p(indices), indices.numel(),
                                              _stream(stream)))

    def reorder_inverse(self, stream=None):
        n = getattr(self, "_reorder_n", 0)
        out = torch.empty(max(n, 1), dtype=torch.int32, device=f"cuda:{self.device}")
        self.check(self.lib.mb2_reorder_inverse(self.h, _p(out), n, _stream(stream)))
        return out[:n]

    # -- pairlist ----------------------------------------------------------
    def build_pairlist(self, pos, type_ids, pairlist_cutoff, interaction_cutoff=0.0,
                       stream=None) -> int:
        """Half pairlist within pairlist_cutoff. With an interaction_cutoff in
        (0, pairlist_cutoff) rows hold the pairs likely to interact first
        (same pair set, another summation order); 0 keeps candidate order."""
        npairs = C.c_uint64()
        self.check(self.lib.mb2_build_pairlist(self.h, _p(pos), _p(type_ids), pos.shape[0],
                                               float(pairlist_cutoff), float(interaction_cutoff),
                                               _stream(stream), C.byref(npairs)))
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

    def dihedral_forces(self, dihedrals, table_idx, pos, fe, get_energy=True, stream=None):
        self.check(self.lib.mb2_dihedral_forces(self.h, _p(dihedrals), _p(table_idx),
                                                dihedrals.shape[0], _p(pos), _p(fe),
                                                int(get_energy), _stream(stream)))

    def restraint_forces(self, ids, anchors, spring_k, pos, fe, get_energy=True, stream=None):
        self.check(self.lib.mb2_restraint_forces(self.h, _p(ids), _p(anchors), _p(spring_k),
                                                 ids.shape[0], _p(pos), _p(fe), int(get_energy),
                                                 _stream(stream)))

    def energy_terms(self, stream=None):
        """[pair, virial, bond, angle, dihedral, restraint] energies (FP64)."""
        out = (C.c_double * 6)()
        self.check(self.lib.mb2_energy_terms(self.h, _stream(stream), out, 6))
        return np.array(list(out))

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

    def selftest_sqrt(self) -> int:
        """Mismatches of the pair kernels' square root against __fsqrt_rn over
        every float in [2^-60, FLT_MAX] (0 expected)."""
        a = C.c_uint64(0)
        self.check(self.lib.mb2_selftest_sqrt(self.h, C.byref(a)))
        return a.value

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

    def run(self, pos, fe, type_ids, flags, first_step, num_steps, params: "L.StepParams",
            stream=None):
        """Steps first_step .. first_step + num_steps - 1 as ``step`` would, the
        steps between rebuild checks replayed from one captured CUDA graph."""
        self.check(self.lib.mb2_run(self.h, _p(pos), _p(fe), _p(type_ids), _p(flags),
                                    pos.shape[0], int(first_step), int(num_steps),
                                    C.byref(params), _stream(stream)))


def exclusion_csr(pairs):
    """Per-particle CSR of excluded pairs, as DeviceBondedInteractions builds it
    (rebuild_exclusions_after_reorder, src/Interactions/DeviceBondedInteraction.h:385-430):
    each pair canonicalised to (a < b), pairs sorted, then each particle's
    neighbours in sorted-pair order. Returns (pairs, offsets, neighbors,
    num_excl_particles); offsets has num_excl_particles + 1 entries."""
    e = np.asarray(pairs, np.int64).reshape(-1, 2)
    if len(e) == 0:
        return (np.zeros((0, 2), np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32), 0)
    e = np.sort(e, axis=1)
    e = e[np.lexsort((e[:, 1], e[:, 0]))]
    np_ = int(e[:, 1].max()) + 1
    owner = np.concatenate([e[:, 0], e[:, 1]])
    other = np.concatenate([e[:, 1], e[:, 0]])
    edge = np.concatenate([np.arange(len(e)), np.arange(len(e))])
    order = np.lexsort((edge, owner))
    offsets = np.zeros(np_ + 1, np.int64)
    np.add.at(offsets, owner + 1, 1)
    return (e.astype(np.int32), np.cumsum(offsets).astype(np.int32),
            other[order].astype(np.int32), np_)


def reorder_particles(ctx: Context, box, particles: dict, indices=(), exclusion_pairs=None,
                      stream=None):
    """Patch::reorder_particles (src/PatchOperation/Patch.cpp:455-480) for one
    patch: Morton order over the periodic box of particles["pos"], every tensor
    in ``particles`` permuted in place (pos, mom, orient, id, type_id, flags,
    attached_rigid_body_id as DeviceParticle::permute does; force/energy is
    cleared each step and is left alone), every int32 tensor in ``indices``
    (bonds, angles, dihedrals, restraint ids) remapped in place, and the
    exclusion pairs remapped and rebuilt into a CSR on the host, which is
    handed to the context (the returned dict keeps its device arrays alive).

    box: (origin, size); a degenerate box skips the reorder (returns None), as
    the reference does. Returns {"inverse", "exclusions"} otherwise."""
    origin, size = np.asarray(box[0], np.float32), np.asarray(box[1], np.float32)
    if not np.all(origin + size > origin):
        return None
    pos = particles["pos"]
    ctx.reorder_begin(pos, stream)
    for t in particles.values():
        if t is not None:
            ctx.reorder_apply(t, stream)
    for t in indices:
        if t is not None and t.numel():
            ctx.reorder_remap(t, stream)
    out = {"inverse": ctx.reorder_inverse(stream), "exclusions": None}
    if exclusion_pairs is not None and len(exclusion_pairs):
        inv = out["inverse"].cpu().numpy().astype(np.int64)
        e, off, nb, npart = exclusion_csr(inv[np.asarray(exclusion_pairs, np.int64)])
        dev = pos.device
        off_d, nb_d = torch.from_numpy(off).to(dev), torch.from_numpy(nb).to(dev)
        rb = particles.get("attached_rigid_body_id")
        ctx.set_exclusions(off_d, nb_d, npart, rb)
        out["exclusions"] = (e, off_d, nb_d, npart)
    return out


class ReorderManager:
    """ParticleReorderManager::maybe_reorder (src/PatchOperation/ReorderManager.cpp:8-25):
    reorder on steps 1, 1 + period, 1 + 2 period, ... once the bonded topology
    is on the device. The period defaults to the pairlist rebuild period
    (src/SimManager.cpp:345-349)."""

    def __init__(self, reorder_period: int, rebuild_period: int = 0):
        self.period = int(reorder_period) if reorder_period > 0 else int(rebuild_period)

    def should_reorder(self, step: int, bonded_prepared: bool = True) -> bool:
        if self.period <= 0 or step == 0:
            return False
        if (step - 1) % self.period:
            return False
        return bool(bonded_prepared)


class Output:
    """SimManager's output side for one system (src/SimManager.cpp:318-330,
    541-575, 596-633, 833-861, 999-1135) over mb2_output: DCD frames (and the
    Langevin momentum DCD), the energy file and restart files, rows in
    global-id order; frames and restarts are written by a background thread.

    ``handle_output(step, ...)`` applies the reference's cadence: a frame when
    step % output_period == 0, energies (then restart files) when
    step % energy_output_period == 0."""

    def __init__(self, output_name, num_particles, output_period=1, energy_output_period=0,
                 timestep=1.0, box=(0.0, 0.0, 0.0), periodic=(1, 1, 1), with_momentum=False,
                 device=0):
        self.lib = L.load()
        cfg = L.OutputConfig()
        cfg.output_name = str(output_name).encode()
        cfg.num_particles = int(num_particles)
        cfg.output_period = int(output_period)
        cfg.timestep = float(timestep)
        for a in range(3):
            cfg.box[a] = float(box[a])
            cfg.periodic[a] = int(periodic[a])
        cfg.with_momentum = int(with_momentum)
        cfg.device = int(device)
        h = C.c_void_p()
        rc = self.lib.mb2_output_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise L.MB2Error(rc, "mb2_output_create failed")
        self.h = h
        self.n = int(num_particles)
        self.output_period = int(output_period)
        self.energy_output_period = int(energy_output_period)
        self.with_momentum = bool(with_momentum)

    def check(self, rc):
        if rc != 0:
            raise L.MB2Error(rc, self.lib.mb2_output_last_error(self.h).decode())

    def frame(self, pos, mom=None, ids=None, stream=None):
        self.check(self.lib.mb2_output_frame(self.h, _p(pos), _p(mom), _p(ids), self.n,
                                             _stream(stream)))

    def restart(self, pos, type_ids, mom=None, ids=None, stream=None):
        self.check(self.lib.mb2_output_restart(self.h, _p(pos), _p(mom), _p(type_ids), _p(ids),
                                               self.n, _stream(stream)))

    def energy(self, fe, kT, mom=None, type_ids=None, mass=None, stream=None):
        """Appends to <name>.energy.dat; returns (kinetic in kT, potential in kcal/mol)."""
        out = (C.c_double * 2)()
        m = None if mass is None else np.ascontiguousarray(mass, np.float32)
        self.check(self.lib.mb2_output_energy(
            self.h, _p(fe), _p(mom), _p(type_ids),
            m.ctypes.data_as(C.POINTER(C.c_float)) if m is not None else None,
            0 if m is None else len(m), self.n, float(kT), _stream(stream), out))
        return float(out[0]), float(out[1])

    def handle_output(self, step, pos, fe, type_ids, kT, mom=None, mass=None, ids=None,
                      stream=None):
        """SimManager::handle_output's schedule for one step."""
        if self.output_period > 0 and step % self.output_period == 0:
            self.frame(pos, mom, ids, stream)
        if self.energy_output_period > 0 and step % self.energy_output_period == 0:
            self.energy(fe, kT, mom, type_ids, mass, stream)
            self.restart(pos, type_ids, mom, ids, stream)

    def flush(self):
        self.check(self.lib.mb2_output_flush(self.h))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.mb2_output_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostStepper:
    """Steps whose positions live in pinned host memory.

    Two patterns, both through ``Context.step`` on the compute stream with
    the copies on two copy streams of their own:

    * ``advance(host_pos, step)``: a trajectory owned by the host. The step
      uploads ``host_pos``, runs, and reads the integrated positions back
      into ``host_pos``, which the next ``advance`` uploads. The copies are
      split into chunks: chunk c of the next upload waits only for chunk c of
      the last read-back, so the two directions overlap each other.
    * ``submit(host_in, host_out, step)``: inputs that do not depend on the
      previous result. Two device position buffers alternate, so the upload
      of one submission and the read-back of another overlap the steps on
      the device. The submissions step one context, whose pairlist follows
      the rebuild schedule and skin check of ``Context.step``: the inputs
      must be nearby states of one system, as successive frames are.

    A stepper serves one of the two patterns. Both return the CUDA event that
    marks the host buffer as written: read it (or change ``host_in``) only
    after ``event.synchronize()``. ``finish()`` joins the copy streams into
    the compute stream, so that work queued there afterwards (an event, a
    synchronize) follows every copy."""

    def __init__(self, ctx: Context, type_ids, params: "L.StepParams", flags=None, n=None,
                 chunks: int = 8):
        self.ctx = ctx
        self.type_ids = type_ids
        self.flags = flags
        self.params = params
        self.n = int(type_ids.shape[0] if n is None else n)
        dev = type_ids.device
        self.pos = [torch.empty((self.n, 4), dtype=torch.float32, device=dev) for _ in range(2)]
        self.fe = torch.zeros((self.n, 4), dtype=torch.float32, device=dev)
        self.compute = torch.cuda.current_stream(dev)
        self.up = torch.cuda.Stream(dev)
        self.down = torch.cuda.Stream(dev)
        self._uploaded = [torch.cuda.Event() for _ in range(2)]
        self._stepped = [torch.cuda.Event() for _ in range(2)]
        self._read = [torch.cuda.Event() for _ in range(2)]
        self._used = [False, False]
        self.k = 0
        step = -(-self.n // max(int(chunks), 1))
        self._chunks = [(a, min(a + step, self.n)) for a in range(0, self.n, step)] or [(0, 0)]
        self._chunk_read = [torch.cuda.Event() for _ in self._chunks]
        self._traj_used = False
        self._mode = None

    def _use(self, mode):
        if self._mode not in (None, mode):
            raise RuntimeError("a HostStepper serves either advance() or submit(), not both")
        self._mode = mode

    def _check(self, *bufs):
        for b in bufs:
            if not b.is_pinned():
                raise ValueError("host buffers must be pinned")
            if tuple(b.shape) != (self.n, 4) or b.dtype != torch.float32:
                raise ValueError(f"host buffers must be float32 [{self.n}, 4]")

    def advance(self, host_pos, step: int):
        self._use("advance")
        self._check(host_pos)
        buf = self.pos[0]
        with torch.cuda.stream(self.up):
            for (a, b), ev in zip(self._chunks, self._chunk_read):
                if self._traj_used:
                    self.up.wait_event(ev)  # this chunk's last read-back
                buf[a:b].copy_(host_pos[a:b], non_blocking=True)
            self._uploaded[0].record(self.up)
        self.compute.wait_event(self._uploaded[0])
        self.ctx.step(buf, self.fe, self.type_ids, self.flags, step, self.params,
                      stream=self.compute)
        self._stepped[0].record(self.compute)
        self.down.wait_event(self._stepped[0])
        with torch.cuda.stream(self.down):
            for (a, b), ev in zip(self._chunks, self._chunk_read):
                host_pos[a:b].copy_(buf[a:b], non_blocking=True)
                ev.record(self.down)
        self._traj_used = True
        return self._chunk_read[-1]

    def submit(self, host_in, host_out, step: int):
        self._use("submit")
        self._check(host_in, host_out)
        b = self.k & 1
        self.k += 1
        buf = self.pos[b]
        if self._used[b]:
            self.up.wait_event(self._read[b])  # the previous read-back of this buffer
        with torch.cuda.stream(self.up):
            buf.copy_(host_in, non_blocking=True)
            self._uploaded[b].record(self.up)
        self.compute.wait_event(self._uploaded[b])
        self.ctx.step(buf, self.fe, self.type_ids, self.flags, step, self.params,
                      stream=self.compute)
        self._stepped[b].record(self.compute)
        self.down.wait_event(self._stepped[b])
        with torch.cuda.stream(self.down):
            host_out.copy_(buf, non_blocking=True)
            self._read[b].record(self.down)
        self._used[b] = True
        return self._read[b]

    def finish(self):
        """Make the compute stream wait for every copy submitted so far."""
        self.compute.wait_stream(self.up)
        self.compute.wait_stream(self.down)


def to_original_order(values, ids):
    """Rows of a reordered patch back in global-id order, as
    DeviceParticle::copy_to_host_unpermuted emits them
    (src/Objects/DeviceParticleManager.h:219-260): out[ids[i]] = values[i]; an id
    outside [0, n) is an error (dense single-patch ids)."""
    values, ids = np.asarray(values), np.asarray(ids, np.int64)
    n = len(ids)
    if n and (ids.min() < 0 or ids.max() >= n):
        raise ValueError("to_original_order: global id outside [0, n)")
    out = np.empty_like(values)
    out[ids] = values
    return out


def step_params(w, seed=None, patch_id=0, get_energy=False, bonds=None, bond_idx=None,
                angles=None, angle_idx=None, dihedrals=None, dihedral_idx=None,
                restraint_ids=None, restraint_anchors=None, restraint_k=None) -> L.StepParams:
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
    if dihedrals is not None:
        p.dihedrals4, p.dihedral_table_idx = dihedrals.data_ptr(), dihedral_idx.data_ptr()
        p.num_dihedrals = dihedrals.shape[0]
    if restraint_ids is not None:
        p.restraint_ids, p.restraint_anchors4 = restraint_ids.data_ptr(), restraint_anchors.data_ptr()
        p.restraint_k, p.num_restraints = restraint_k.data_ptr(), restraint_ids.shape[0]
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
        """Cell level, lanes per row and rebuild cadence chosen on a copy of the
        positions and put in force (see mb2_batch_autotune)."""
        r = L.BatchTuning()
        self.check(self.lib.mb2_batch_autotune(self.h, _p(pos), _p(type_ids), C.byref(params),
                                               int(trial_steps), _stream(stream), C.byref(r)))
        return {k: getattr(r, k) for k, _ in L.BatchTuning._fields_}

    def set_rebuild_period(self, period: int):
        """Rebuild cadence for step/run (0: the params' rebuild_period)."""
        self.check(self.lib.mb2_batch_set_rebuild_period(self.h, int(period)))

    def rebuild_schedule(self):
        """(cadence in force, 0 = the params'; list builds so far)."""
        p, r = C.c_uint32(), C.c_uint64()
        self.check(self.lib.mb2_batch_rebuild_schedule(self.h, C.byref(p), C.byref(r)))
        return int(p.value), int(r.value)

    def system_rebuilds(self) -> int:
        """System lists rebuilt so far, summed over the list builds (each
        build rebuilds only the systems whose own skin check failed)."""
        c = C.c_uint64()
        self.check(self.lib.mb2_batch_system_rebuilds(self.h, C.byref(c)))
        return int(c.value)


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
