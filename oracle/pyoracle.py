"""numpy front end for the CPU oracle (liboracle.so) and the reference harness.

TEST INFRASTRUCTURE ONLY. Imported by the test suite, the smoke check and the
benchmark's CPU-baseline leg, as the checker of the CUDA path; the product
never imports it.

Two libraries are wrapped:

* ``Oracle``: this project's C restatement of the reference algorithm
  (``oracle/mb2_oracle.c``), built by ``oracle/Makefile``.
* ``RefHarness``: the reference's own host-compiled functors
  (``oracle/_ref/libmars_ref.so``, built by ``oracle/ref_harness/Makefile``
  from the reference checkout). Present only where it was built.

Arrays are numpy, float4 rows for vectors, C-contiguous.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmars_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build_oracle() -> str:
    """Compile liboracle.so (gcc, seconds). Returns its path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


class Box(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("size", C.c_float * 3), ("periodic", C.c_int * 3)]

    @classmethod
    def make(cls, origin, size, periodic=(1, 1, 1)):
        b = cls()
        for a in range(3):
            b.origin[a] = float(origin[a])
            b.size[a] = float(size[a])
            b.periodic[a] = int(periodic[a])
        return b


class Table(C.Structure):
    _fields_ = [("pot", C.c_void_p), ("step_inv", C.c_float), ("size", C.c_uint32),
                ("start", C.c_float), ("is_periodic", C.c_int)]


class Grid(C.Structure):
    _fields_ = [("data", C.c_void_p), ("origin", C.c_float * 3), ("basis", C.c_float * 9),
                ("basis_inv", C.c_float * 9), ("dims", C.c_int64 * 3),
                ("boundary_condition", C.c_int)]


class GridTerm(C.Structure):
    _fields_ = [("grid_id", C.c_int), ("scale", C.c_float), ("scale_slope", C.c_float),
                ("boundary_condition", C.c_int)]


class Types(C.Structure):
    _fields_ = [("num_types", C.c_int), ("charge", C.c_void_p), ("diffusion4", C.c_void_p),
                ("pmf_offset", C.c_void_p), ("pmf_count", C.c_void_p), ("terms", C.c_void_p),
                ("force_grid_id4", C.c_void_p), ("force_grid_scale4", C.c_void_p)]


class PairTerms(C.Structure):
    _fields_ = [("charge", C.c_void_p), ("radius", C.c_void_p), ("eps", C.c_void_p),
                ("debye_length", C.c_float), ("dielectric", C.c_float),
                ("onck_kappa", C.c_float), ("onck_sz", C.c_float), ("onck_z", C.c_float),
                ("gaussian_amp", C.c_float), ("gaussian_sigma", C.c_float),
                ("gaussian_cutoff_sq", C.c_float), ("enabled_terms", C.c_uint32)]


# Solvent and Gaussian defaults of the reference (SolventParams,
# NonBondedInteraction.h:123-129; GaussianPotential, Pairwise.h:50-53).
SOLVENT_DEFAULTS = (10.0, 80.0, 0.1, 80.0, 6.86)
GAUSSIAN_DEFAULTS = (1.0, 1.0, 0.0)


class PairTermSet:
    """Per-type charge / radius / eps plus solvent and Gaussian constants."""

    def __init__(self, charge, radius, eps, solvent=SOLVENT_DEFAULTS, gaussian=GAUSSIAN_DEFAULTS,
                 enabled_terms=0xFF):
        self.charge = np.ascontiguousarray(charge, np.float32)
        self.radius = np.ascontiguousarray(radius, np.float32)
        self.eps = np.ascontiguousarray(eps, np.float32)
        self.solvent = np.asarray(solvent, np.float32)
        self.gaussian = np.asarray(gaussian, np.float32)
        self.s = PairTerms(_ptr(self.charge), _ptr(self.radius), _ptr(self.eps),
                           *[float(x) for x in self.solvent], *[float(x) for x in self.gaussian],
                           int(enabled_terms))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class TableSet:
    """Concatenated float tables plus per-table metadata, kept alive together."""

    def __init__(self, tables, periodic=False):
        # tables: list of (values float32[size], start, step_inv)
        vals = [np.ascontiguousarray(t[0], dtype=np.float32) for t in tables]
        self.values = np.concatenate(vals) if vals else np.zeros(1, np.float32)
        self.offsets = np.zeros(len(vals), np.uint32)
        off = 0
        for k, v in enumerate(vals):
            self.offsets[k] = off
            off += len(v)
        self.sizes = np.array([len(v) for v in vals], np.uint32)
        self.starts = np.array([t[1] for t in tables], np.float32)
        self.step_invs = np.array([t[2] for t in tables], np.float32)
        self.periodic = periodic
        self.structs = (Table * max(1, len(vals)))()
        for k in range(len(vals)):
            self.structs[k].pot = self.values.ctypes.data + 4 * int(self.offsets[k])
            self.structs[k].step_inv = float(self.step_invs[k])
            self.structs[k].size = int(self.sizes[k])
            self.structs[k].start = float(self.starts[k])
            self.structs[k].is_periodic = int(periodic)

    def __len__(self):
        return len(self.sizes)


class TypeSet:
    """Per-type BD data (charge, diffusion, PMF terms, force grids)."""

    def __init__(self, charge, diffusion, pmf_terms_per_type=None, force_grid_id=None,
                 force_grid_scale=None):
        t = len(charge)
        self.charge = np.ascontiguousarray(charge, np.float32)
        d = np.zeros((t, 4), np.float32)
        d[:, :3] = np.asarray(diffusion, np.float32).reshape(t, 3)
        self.diffusion4 = d
        pmf_terms_per_type = pmf_terms_per_type or [[] for _ in range(t)]
        self.pmf_offset = np.zeros(t, np.int32)
        self.pmf_count = np.zeros(t, np.int32)
        flat = []
        for k, terms in enumerate(pmf_terms_per_type):
            self.pmf_offset[k] = len(flat)
            self.pmf_count[k] = len(terms)
            flat.extend(terms)  # (grid_id, scale, scale_slope, bc)
        self.terms_flat = np.array(flat, np.float32).reshape(-1, 4) if flat else np.zeros((1, 4), np.float32)
        self.terms = (GridTerm * max(1, len(flat)))()
        for k, (gid, s, sl, bc) in enumerate(flat):
            self.terms[k].grid_id, self.terms[k].scale = int(gid), float(s)
            self.terms[k].scale_slope, self.terms[k].boundary_condition = float(sl), int(bc)
        self.n_terms = len(flat)
        fg = np.full((t, 4), -1, np.int32)
        if force_grid_id is not None:
            fg[:, :3] = np.asarray(force_grid_id, np.int32).reshape(t, 3)
        self.force_grid_id4 = fg
        fs = np.zeros((t, 4), np.float32)
        if force_grid_scale is not None:
            fs[:, :3] = np.asarray(force_grid_scale, np.float32).reshape(t, 3)
        self.force_grid_scale4 = fs
        self.struct = Types(t, _ptr(self.charge), _ptr(self.diffusion4), _ptr(self.pmf_offset),
                            _ptr(self.pmf_count), C.cast(self.terms, C.c_void_p),
                            _ptr(self.force_grid_id4), _ptr(self.force_grid_scale4))


class GridSet:
    """Dense grids: list of dicts with data (nx,ny,nz float32), origin, basis (3x3, columns
    are basis vectors), boundary_condition."""

    def __init__(self, grids):
        self.arrays = []
        self.structs = (Grid * max(1, len(grids)))()
        for k, g in enumerate(grids):
            data = np.ascontiguousarray(g["data"], np.float32)
            self.arrays.append(data)
            s = self.structs[k]
            s.data = data.ctypes.data
            basis = np.asarray(g["basis"], np.float32)
            binv = np.asarray(g.get("basis_inv", np.linalg.inv(basis.astype(np.float64))), np.float32)
            for a in range(3):
                s.origin[a] = float(g["origin"][a])
                s.dims[a] = int(data.shape[a])
            # column-major: element [3*c + r] = M[r, c]
            for c in range(3):
                for r in range(3):
                    s.basis[3 * c + r] = float(basis[r, c])
                    s.basis_inv[3 * c + r] = float(binv[r, c])
            s.boundary_condition = int(g.get("boundary_condition", 0))
        self.n = len(grids)

    def ptr(self):
        return C.cast(self.structs, C.c_void_p) if self.n else None


class Oracle:
    """C restatement of the reference algorithm."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        L = self.lib = C.CDLL(path)
        vp, sz, f, i, u32, u64 = C.c_void_p, C.c_size_t, C.c_float, C.c_int, C.c_uint32, C.c_uint64
        L.or_wrap_diff_scalar.restype = f
        L.or_wrap_diff_scalar.argtypes = [f, f]
        L.or_wrap_scalar.restype = f
        L.or_wrap_scalar.argtypes = [f, f, f]
        L.or_wrap_diff.argtypes = [vp, vp, vp, sz]
        L.or_wrap.argtypes = [vp, vp, vp, sz]
        L.or_morton_key.restype = u32
        L.or_morton_encode.argtypes = [vp, sz, vp, vp, vp, vp]
        L.or_sort_pairs.argtypes = [vp, vp, sz]
        L.or_inverse.argtypes = [vp, vp, sz]
        L.or_gather4.argtypes = [vp, vp, vp, sz]
        L.or_morton_domain.argtypes = [vp, vp, sz, vp, vp]
        L.or_select_cell_grid.argtypes = [vp, f, sz, sz, vp, vp, vp]
        L.or_cell_ranges.argtypes = [vp, sz, i, vp, vp]
        L.or_cell_neighbors.argtypes = [vp, i, vp, i, vp]
        L.or_neighbor_walk.restype = u64
        L.or_neighbor_walk.argtypes = [vp, vp, vp, vp, vp, vp, i, i, f, sz, vp, vp, vp, sz, vp,
                                       vp, u64, vp]
        L.or_build_pairlist.restype = u64
        L.or_build_pairlist.argtypes = [vp, sz, vp, f, vp, vp, sz, vp, vp, u64, vp]
        L.or_build_pairlist_m.restype = u64
        L.or_build_pairlist_m.argtypes = [vp, sz, vp, f, vp, vp, sz, vp, vp, u64, vp, i]
        L.or_pair_hash.restype = u64
        L.or_pair_hash.argtypes = [i, i]
        L.or_exclusion_csr.argtypes = [vp, sz, vp, vp, vp]
        L.or_max_displacement.restype = f
        L.or_max_displacement.argtypes = [vp, vp, sz, vp]
        L.or_table_lookup.argtypes = [vp, f, vp, vp]
        L.or_resolve_tags.argtypes = [vp, sz, vp, vp, i, vp]
        L.or_pair_forces.argtypes = [vp, sz, vp, vp, vp, vp, f, i, vp, vp, vp]
        L.or_bond_forces.argtypes = [vp, vp, sz, vp, vp, vp, i, vp, vp, vp]
        L.or_angle_forces.argtypes = [vp, vp, sz, vp, vp, vp, i, vp, vp, vp]
        L.or_pair_forces_terms.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp, f, i, vp, vp, vp]
        L.or_dihedral_forces.argtypes = [vp, vp, sz, vp, vp, vp, i, vp, vp, vp]
        L.or_restraint_forces.argtypes = [vp, vp, vp, sz, vp, vp, i, vp, vp, vp]
        L.or_pair_energy_f64.restype = C.c_double
        L.or_pair_energy_f64.argtypes = [vp, sz, vp, vp, vp, vp, f]
        L.or_grid_value.restype = f
        L.or_grid_value.argtypes = [vp, vp, i]
        L.or_grid_gradient.argtypes = [vp, vp, i, vp]
        L.or_position_force.argtypes = [vp, i, vp, vp, vp, vp]
        L.or_philox4x32_10.argtypes = [u64, u32, u32, u32, u32, vp]
        L.or_u01.restype = f
        L.or_u01.argtypes = [u32]
        L.or_bd_seed.restype = u64
        L.or_bd_seed.argtypes = [u64, u64, u64]
        L.or_bd_integrate.argtypes = [vp, vp, vp, vp, sz, vp, vp, vp, f, f, u64, u64, u32, vp, vp]

    # -- Morton sort ------------------------------------------------------
    def morton_domain(self, box: Box, pos4):
        bmin = np.zeros(3, np.float32)
        bmax = np.zeros(3, np.float32)
        self.lib.or_morton_domain(C.byref(box), _ptr(pos4), len(pos4), _ptr(bmin), _ptr(bmax))
        return bmin, bmax

    def morton_encode(self, pos4, bmin, bmax):
        n = len(pos4)
        keys = np.zeros(n, np.uint32)
        idx = np.zeros(n, np.uint32)
        self.lib.or_morton_encode(_ptr(pos4), n, _ptr(np.asarray(bmin, np.float32)),
                                  _ptr(np.asarray(bmax, np.float32)), _ptr(keys), _ptr(idx))
        return keys, idx

    def sort_pairs(self, keys, vals):
        k = np.array(keys, np.uint32)
        v = np.array(vals, np.uint32)
        self.lib.or_sort_pairs(_ptr(k), _ptr(v), len(k))
        return k, v

    def inverse(self, sorted_idx):
        inv = np.zeros(len(sorted_idx), np.uint32)
        self.lib.or_inverse(_ptr(np.ascontiguousarray(sorted_idx, np.uint32)), _ptr(inv), len(inv))
        return inv

    def gather4(self, pos4, sorted_idx):
        out = np.zeros_like(pos4)
        self.lib.or_gather4(_ptr(pos4), _ptr(out), _ptr(np.ascontiguousarray(sorted_idx, np.uint32)),
                            len(pos4))
        return out

    def sort_particles(self, box: Box, pos4):
        """Domain + encode + sort + inverse + gather (ZOrderSort::sort_particles)."""
        bmin, bmax = self.morton_domain(box, pos4)
        keys, idx = self.morton_encode(pos4, bmin, bmax)
        keys, s2o = self.sort_pairs(keys, idx)
        inv = self.inverse(s2o)
        return dict(bmin=bmin, bmax=bmax, keys=keys, sorted_to_orig=s2o, inverse=inv,
                    sorted_pos=self.gather4(pos4, s2o))

    def reorder(self, box: Box, pos4):
        """Patch::reorder_particles (src/PatchOperation/Patch.cpp:455-480): the
        Morton sort with the periodic box origin .. origin + size as bounds.
        Returns (sorted_to_orig, inverse)."""
        o = np.array(list(box.origin), np.float32)
        hi = (o + np.array(list(box.size), np.float32)).astype(np.float32)
        keys, idx = self.morton_encode(pos4, o, hi)
        _, s2o = self.sort_pairs(keys, idx)
        return s2o, self.inverse(s2o)

    @staticmethod
    def remap_indices(indices, inv):
        """RemapIndicesKernel (src/PatchOperation/ZOrderKernels/ZOrderKernels.h:87-101):
        values in [0, len(inv)) go through inv, others stay."""
        a = np.array(indices, np.int64)
        ok = (a >= 0) & (a < len(inv))
        a[ok] = np.asarray(inv, np.int64)[a[ok]]
        return a.astype(np.int32)

    # -- pairlist ---------------------------------------------------------
    def select_cell_grid(self, extent, cutoff, n, max_pairs):
        m = C.c_int()
        radii = np.zeros(3, np.int32)
        slots = C.c_int()
        self.lib.or_select_cell_grid(_ptr(np.asarray(extent, np.float32)), C.c_float(cutoff), n,
                                     max_pairs, C.byref(m), _ptr(radii), C.byref(slots))
        return m.value, radii, slots.value

    def cell_ranges(self, keys, shift, num_cells):
        b = np.zeros(num_cells, np.uint32)
        e = np.zeros(num_cells, np.uint32)
        self.lib.or_cell_ranges(_ptr(keys), len(keys), shift, _ptr(b), _ptr(e))
        return b, e

    def cell_neighbors(self, m, radii, npc, box_len):
        t = np.zeros((1 << (3 * m)) * npc, np.uint32)
        self.lib.or_cell_neighbors(_ptr(t), m, _ptr(np.asarray(radii, np.int32)), npc,
                                   _ptr(np.asarray(box_len, np.float32)))
        return t

    def build_pairlist(self, pos4, box: Box, rc_list, excl=None, rigid_body_id=None,
                       want_pairs=True, max_pairs=None, m=-1):
        """Pair set within rc_list: returns (pairs int32[P,2] sorted lexicographically
        or None, count, checksum). m >= 0 forces the cell level (speed only)."""
        n = len(pos4)
        off, nb, excl_n = (None, None, 0) if excl is None else excl
        if want_pairs and max_pairs is None:
            cnt = self.lib.or_build_pairlist_m(_ptr(pos4), n, C.byref(box), C.c_float(rc_list),
                                               _ptr(off), _ptr(nb), excl_n, _ptr(rigid_body_id),
                                               None, 0, None, m)
            max_pairs = int(cnt)
        buf = np.zeros((max_pairs if want_pairs else 0, 2), np.int32)
        cs = C.c_uint64()
        cnt = self.lib.or_build_pairlist_m(_ptr(pos4), n, C.byref(box), C.c_float(rc_list),
                                           _ptr(off), _ptr(nb), excl_n, _ptr(rigid_body_id),
                                           _ptr(buf) if want_pairs else None,
                                           max_pairs if want_pairs else 0, C.byref(cs), m)
        pairs = None
        if want_pairs:
            pairs = buf[: min(int(cnt), max_pairs)]
            order = np.lexsort((pairs[:, 1], pairs[:, 0]))
            pairs = np.ascontiguousarray(pairs[order])
        return pairs, int(cnt), int(cs.value)

    def pair_hash_sum(self, pairs):
        """Order-independent checksum of a pair set (same as build_pairlist's)."""
        a = np.minimum(pairs[:, 0], pairs[:, 1]).astype(np.uint64)
        b = np.maximum(pairs[:, 0], pairs[:, 1]).astype(np.uint64)
        z = (a << np.uint64(32)) | b
        with np.errstate(over="ignore"):
            z = z + np.uint64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
            return int(np.sum(z, dtype=np.uint64))

    def exclusion_csr(self, pairs):
        pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        mx = int(pairs.max()) if len(pairs) else 0
        off = np.zeros(mx + 2, np.int32)
        nb = np.zeros(max(1, 2 * len(pairs)), np.int32)
        npart = C.c_size_t()
        self.lib.or_exclusion_csr(_ptr(pairs), len(pairs), _ptr(off), _ptr(nb), C.byref(npart))
        return off, nb, npart.value

    def max_displacement(self, cur4, prev4, box_len):
        return self.lib.or_max_displacement(_ptr(cur4), _ptr(prev4), len(cur4),
                                            _ptr(np.asarray(box_len, np.float32)))

    # -- forces -----------------------------------------------------------
    def table_lookup(self, tables: TableSet, k, x):
        fo, en = C.c_float(), C.c_float()
        self.lib.or_table_lookup(C.byref(tables.structs[k]), C.c_float(x), C.byref(fo), C.byref(en))
        return fo.value, en.value

    def resolve_tags(self, pairs, type_ids, term_matrix, num_types):
        tags = np.zeros(len(pairs), np.uint32)
        self.lib.or_resolve_tags(_ptr(pairs), len(pairs), _ptr(type_ids), _ptr(term_matrix),
                                 num_types, _ptr(tags))
        return tags

    def pair_forces(self, pairs, pos4, tags, tables: TableSet, box: Box, cutoff_sq,
                    get_energy=True):
        n = len(pos4)
        fe4 = np.zeros((n, 4), np.float32)
        fe64 = np.zeros((n, 4), np.float64)
        fabs = np.zeros(n, np.float64)
        self.lib.or_pair_forces(_ptr(pairs), len(pairs), _ptr(pos4), _ptr(tags),
                                C.cast(tables.structs, C.c_void_p), C.byref(box),
                                C.c_float(cutoff_sq), int(get_energy), _ptr(fe4), _ptr(fe64),
                                _ptr(fabs))
        return fe4, fe64, fabs

    def pair_forces_terms(self, pairs, pos4, type_ids, tags, tables: TableSet,
                          terms: "PairTermSet", box: Box, cutoff_sq, get_energy=True):
        """Every pair term (analytical and tabulated); returns (fe4, fe64, fabs)."""
        n = len(pos4)
        fe4 = np.zeros((n, 4), np.float32)
        fe64 = np.zeros((n, 4), np.float64)
        fabs = np.zeros(n, np.float64)
        self.lib.or_pair_forces_terms(_ptr(np.ascontiguousarray(pairs, np.int32)), len(pairs),
                                      _ptr(pos4), _ptr(np.ascontiguousarray(type_ids, np.int32)),
                                      _ptr(np.ascontiguousarray(tags, np.uint32)),
                                      C.cast(tables.structs, C.c_void_p), C.byref(terms.s),
                                      C.byref(box), C.c_float(cutoff_sq), int(get_energy),
                                      _ptr(fe4), _ptr(fe64), _ptr(fabs))
        return fe4, fe64, fabs

    def dihedral_forces(self, dihedrals4, table_idx, pos4, tables: TableSet, box: Box,
                        get_energy=True):
        n = len(pos4)
        fe4 = np.zeros((n, 4), np.float32)
        fe64 = np.zeros((n, 4), np.float64)
        fabs = np.zeros(n, np.float64)
        self.lib.or_dihedral_forces(_ptr(np.ascontiguousarray(dihedrals4, np.int32)),
                                    _ptr(np.ascontiguousarray(table_idx, np.int32)),
                                    len(dihedrals4), _ptr(pos4), C.cast(tables.structs, C.c_void_p),
                                    C.byref(box), int(get_energy), _ptr(fe4), _ptr(fe64),
                                    _ptr(fabs))
        return fe4, fe64, fabs

    def restraint_forces(self, ids, anchors4, k_spring, pos4, box: Box, get_energy=True):
        n = len(pos4)
        fe4 = np.zeros((n, 4), np.float32)
        fe64 = np.zeros((n, 4), np.float64)
        fabs = np.zeros(n, np.float64)
        self.lib.or_restraint_forces(_ptr(np.ascontiguousarray(ids, np.int32)),
                                     _ptr(np.ascontiguousarray(anchors4, np.float32)),
                                     _ptr(np.ascontiguousarray(k_spring, np.float32)), len(ids),
                                     _ptr(pos4), C.byref(box), int(get_energy), _ptr(fe4),
                                     _ptr(fe64), _ptr(fabs))
        return fe4, fe64, fabs

    def pair_energy_f64(self, pairs, pos4, tags, tables: TableSet, box: Box, cutoff_sq):
        return self.lib.or_pair_energy_f64(_ptr(pairs), len(pairs), _ptr(pos4), _ptr(tags),
                                           C.cast(tables.structs, C.c_void_p), C.byref(box),
                                           C.c_float(cutoff_sq))

    def bond_forces(self, bonds, table_idx, pos4, tables: TableSet, box: Box, get_energy=True,
                    fe4=None, fe64=None, fabs=None):
        n = len(pos4)
        fe4 = np.zeros((n, 4), np.float32) if fe4 is None else fe4
        fe64 = np.zeros((n, 4), np.float64) if fe64 is None else fe64
        fabs = np.zeros(n, np.float64) if fabs is None else fabs
        self.lib.or_bond_forces(_ptr(bonds), _ptr(table_idx), len(bonds), _ptr(pos4),
                                C.cast(tables.structs, C.c_void_p), C.byref(box), int(get_energy),
                                _ptr(fe4), _ptr(fe64), _ptr(fabs))
        return fe4, fe64, fabs

    def angle_forces(self, angles4, table_idx, pos4, tables: TableSet, box: Box, get_energy=True,
                     fe4=None, fe64=None, fabs=None):
        n = len(pos4)
        fe4 = np.zeros((n, 4), np.float32) if fe4 is None else fe4
        fe64 = np.zeros((n, 4), np.float64) if fe64 is None else fe64
        fabs = np.zeros(n, np.float64) if fabs is None else fabs
        self.lib.or_angle_forces(_ptr(angles4), _ptr(table_idx), len(angles4), _ptr(pos4),
                                 C.cast(tables.structs, C.c_void_p), C.byref(box), int(get_energy),
                                 _ptr(fe4), _ptr(fe64), _ptr(fabs))
        return fe4, fe64, fabs

    # -- grid, Philox, BD -------------------------------------------------
    def philox(self, seed, ctr0, ctr1, ctr2, internal=0):
        out = np.zeros(4, np.uint32)
        self.lib.or_philox4x32_10(seed, ctr0, ctr1, ctr2, internal, _ptr(out))
        return out

    def bd_seed(self, seed, patch_id, step):
        return int(self.lib.or_bd_seed(seed, patch_id, step))

    def position_force(self, pos3, type_id, types: TypeSet, grids: GridSet, efield=(0, 0, 0)):
        out = np.zeros(4, np.float32)
        p = np.asarray(pos3, np.float32)
        self.lib.or_position_force(_ptr(p), int(type_id), C.byref(types.struct), grids.ptr(),
                                   _ptr(np.asarray(efield, np.float32)), _ptr(out))
        return out

    def bd_integrate(self, pos4, fe4, type_ids, flags, types: TypeSet, grids, box: Box, dt, kT,
                     step, base_seed, base_ctr=0, efield=(0, 0, 0), want_noise=False):
        """In-place on copies; returns (pos4, fe4, noise4 or None)."""
        pos = np.array(pos4, np.float32)
        fe = np.array(fe4, np.float32)
        noise = np.zeros_like(pos) if want_noise else None
        self.lib.or_bd_integrate(_ptr(pos), _ptr(fe), _ptr(np.ascontiguousarray(type_ids, np.int32)),
                                 _ptr(flags), len(pos), C.byref(types.struct),
                                 grids.ptr() if grids is not None else None, C.byref(box),
                                 C.c_float(dt), C.c_float(kT), step, base_seed, base_ctr,
                                 _ptr(np.asarray(efield, np.float32)), _ptr(noise))
        return pos, fe, noise


def _oracle_baoab(self, pos4, mom4, fe4, type_ids, flags, types: "TypeSet", grids, mass, damping,
                  box: Box, dt, kT, step, base_seed, base_ctr=0, efield=(0, 0, 0), pending=0):
    """Langevin BAOAB step on copies; returns (pos4, mom4, fe4)."""
    L = self.lib
    vp = C.c_void_p
    L.or_baoab_integrate.argtypes = [vp, vp, vp, vp, vp, C.c_size_t, vp, vp, vp, vp, vp, C.c_float,
                                     C.c_float, C.c_uint64, C.c_uint64, C.c_uint32, vp, C.c_int]
    pos, mom, fe = (np.array(a, np.float32) for a in (pos4, mom4, fe4))
    ms = np.ascontiguousarray(mass, np.float32)
    dmp = np.ascontiguousarray(damping, np.float32).reshape(-1, 3)
    L.or_baoab_integrate(_ptr(pos), _ptr(mom), _ptr(fe), _ptr(np.ascontiguousarray(type_ids, np.int32)),
                         _ptr(flags), len(pos), C.byref(types.struct),
                         grids.ptr() if grids is not None else None, _ptr(ms), _ptr(dmp),
                         C.byref(box), C.c_float(dt), C.c_float(kT), step, base_seed, base_ctr,
                         _ptr(np.asarray(efield, np.float32)), int(pending))
    return pos, mom, fe


Oracle.baoab_integrate = _oracle_baoab


class RefGrid(C.Structure):
    _fields_ = [("data", C.c_void_p), ("origin", C.c_float * 3), ("basis", C.c_float * 9),
                ("basis_inv", C.c_float * 9), ("dims", C.c_int64 * 3),
                ("boundary_condition", C.c_int)]


def ref_available(path: str = REF_SO) -> bool:
    return os.path.exists(path)


class RefHarness:
    """The reference's own functors, host-compiled (see oracle/ref_harness)."""

    def __init__(self, path: str = REF_SO):
        L = self.lib = C.CDLL(path)
        vp, sz, f, i, u32, u64 = C.c_void_p, C.c_size_t, C.c_float, C.c_int, C.c_uint32, C.c_uint64
        L.ref_morton_encode.argtypes = [vp, sz, vp, vp, vp, vp, i]
        L.ref_sort_pairs.argtypes = [vp, vp, sz]
        L.ref_inverse.argtypes = [vp, vp, sz]
        L.ref_reorder_pos.argtypes = [vp, vp, vp, sz]
        L.ref_remap_indices.argtypes = [vp, sz, vp, sz]
        L.ref_dcd_write.argtypes = [C.c_char_p, vp, i, i, i, f, i, vp]
        L.ref_pair_forces_terms.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp, vp, vp, vp, i, vp, vp,
                                            vp, i, f, u32, vp, vp, vp, vp, vp]
        L.ref_dihedral_forces.argtypes = [vp, vp, vp, sz, vp, vp, vp, vp, vp, vp, vp, i, vp, vp,
                                          vp, i]
        L.ref_restraint_forces.argtypes = [vp, vp, vp, sz, vp, vp, vp, vp, vp, i]
        L.ref_cell_ranges.argtypes = [vp, sz, i, vp, vp]
        L.ref_cell_neighbors.argtypes = [vp, sz, i, vp, i, vp]
        L.ref_neighbor_walk.restype = u32
        L.ref_neighbor_walk.argtypes = [vp, vp, vp, vp, vp, vp, vp, sz, f, sz, i, i, i, vp, vp, vp,
                                        vp, vp, sz, vp]
        L.ref_neighbor_walk_items.restype = u64
        L.ref_neighbor_walk_items.argtypes = [vp, vp, vp, vp, vp, vp, f, sz, i, i, vp, vp, vp,
                                              vp, sz, vp, sz]
        L.ref_resolve_tags.argtypes = [vp, sz, vp, vp, sz, vp, i]
        L.ref_read_table.argtypes = [C.c_char_p, i, vp, vp, sz, vp, vp, vp, vp]
        L.ref_neighbor_walk_items_mt.restype = u64
        L.ref_neighbor_walk_items_mt.argtypes = [vp, vp, vp, vp, vp, vp, f, sz, i, i, vp, vp, vp,
                                                 vp, sz, vp, sz, i]
        L.ref_pair_forces_mt.argtypes = [vp, sz, sz, vp, vp, vp, vp, vp, vp, vp, vp, vp, i, vp, vp,
                                         vp, i, f, u32, i]
        L.ref_pair_forces.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp, vp, vp, vp, i, vp, vp, vp,
                                      i, f, u32]
        L.ref_bond_forces.argtypes = [vp, vp, vp, sz, vp, vp, vp, vp, vp, vp, vp, i, vp, vp, vp, i]
        L.ref_angle_forces.argtypes = [vp, vp, vp, sz, vp, vp, vp, vp, vp, vp, vp, i, vp, vp, vp, i]
        L.ref_bd_integrate.argtypes = [vp, vp, vp, vp, sz, i, vp, vp, vp, vp, vp, i, vp, vp, vp, i,
                                       vp, vp, vp, f, f, u64, u64, u32, vp, i]
        L.ref_philox_int4.argtypes = [u64, u32, u32, u32, i, vp]
        L.ref_philox_float4.argtypes = [u64, u32, u32, u32, i, vp]
        L.ref_max_displacement.restype = f
        L.ref_max_displacement.argtypes = [vp, vp, sz, vp]
        L.ref_wrap_diff.argtypes = [vp, vp, vp, vp, vp, sz]
        L.ref_wrap.argtypes = [vp, vp, vp, vp, vp, sz]
        L.ref_table_lookup.argtypes = [f, vp, u32, f, f, i, vp]

    @staticmethod
    def _box(box: Box):
        o = np.array(list(box.origin), np.float32)
        s = np.array(list(box.size), np.float32)
        p = np.array(list(box.periodic), np.int32)
        return o, s, p

    def morton_encode(self, pos4, bmin, bmax, nthreads=1):
        n = len(pos4)
        keys = np.zeros(n, np.uint32)
        idx = np.zeros(n, np.uint32)
        self.lib.ref_morton_encode(_ptr(pos4), n, _ptr(np.asarray(bmin, np.float32)),
                                   _ptr(np.asarray(bmax, np.float32)), _ptr(keys), _ptr(idx),
                                   nthreads)
        return keys, idx

    def sort_pairs(self, keys, vals):
        k = np.array(keys, np.uint32)
        v = np.array(vals, np.uint32)
        self.lib.ref_sort_pairs(_ptr(k), _ptr(v), len(k))
        return k, v

    def inverse(self, s):
        inv = np.zeros(len(s), np.uint32)
        self.lib.ref_inverse(_ptr(s), _ptr(inv), len(s))
        return inv

    def reorder_pos(self, pos4, s):
        out = np.zeros_like(pos4)
        self.lib.ref_reorder_pos(_ptr(pos4), _ptr(out), _ptr(s), len(s))
        return out

    def dcd_write(self, path, frames4, nsavc, delta, with_unitcell, box):
        """The reference's DcdWriter driven as write_dcd_frame drives it."""
        fr = np.ascontiguousarray(frames4, np.float32)
        rc = self.lib.ref_dcd_write(str(path).encode(), _ptr(fr), fr.shape[0], fr.shape[1],
                                    int(nsavc), C.c_float(delta), int(with_unitcell),
                                    _ptr(np.asarray(box, np.float32)))
        if rc != 0:
            raise RuntimeError("reference DcdWriter failed")

    def remap_indices(self, indices, inv):
        out = np.ascontiguousarray(indices, np.int32).copy()
        self.lib.ref_remap_indices(_ptr(out), out.size, _ptr(np.asarray(inv, np.uint32)), len(inv))
        return out

    def cell_ranges(self, keys, shift, num_cells):
        b = np.zeros(num_cells, np.uint32)
        e = np.zeros(num_cells, np.uint32)
        self.lib.ref_cell_ranges(_ptr(keys), len(keys), shift, _ptr(b), _ptr(e))
        return b, e

    def cell_neighbors(self, m, radii, npc, box_len):
        t = np.zeros((1 << (3 * m)) * npc, np.uint32)
        self.lib.ref_cell_neighbors(_ptr(t), 1 << (3 * m), m, _ptr(np.asarray(radii, np.int32)),
                                    npc, _ptr(np.asarray(box_len, np.float32)))
        return t

    def neighbor_walk(self, sorted_pos, keys, s2o, begin, end, table, cutoff_sq, npc, shift,
                      box: Box, excl=None, rigid_body_id=None, tpp=4, max_pairs=None):
        n = len(keys)
        o, s, p = self._box(box)
        off, nb, excl_n = (None, None, 0) if excl is None else excl
        max_pairs = max_pairs if max_pairs is not None else n * 400
        buf = np.zeros((max_pairs + 1, 2), np.int32)
        cnt = self.lib.ref_neighbor_walk(_ptr(sorted_pos), _ptr(keys), _ptr(s2o), _ptr(begin),
                                         _ptr(end), _ptr(table), _ptr(buf), max_pairs,
                                         C.c_float(cutoff_sq), n, npc, min(tpp, npc), shift,
                                         _ptr(o), _ptr(s), _ptr(p), _ptr(off), _ptr(nb), excl_n,
                                         _ptr(rigid_body_id))
        return buf[1: cnt + 1], int(cnt)

    def neighbor_walk_items(self, sorted_pos, keys, s2o, begin, end, table, cutoff_sq, npc,
                            shift, box: Box, items, max_pairs=0):
        """Run the walk for the listed particles only. Returns (pairs or None, count)."""
        o, s, p = self._box(box)
        items = np.ascontiguousarray(items, np.uint32)
        buf = np.zeros((max_pairs + 1, 2), np.int32) if max_pairs else None
        cnt = int(self.lib.ref_neighbor_walk_items(
            _ptr(sorted_pos), _ptr(keys), _ptr(s2o), _ptr(begin), _ptr(end), _ptr(table),
            C.c_float(cutoff_sq), len(keys), npc, shift, _ptr(o), _ptr(s), _ptr(p), _ptr(items),
            len(items), _ptr(buf), max_pairs))
        pairs = None if buf is None else np.ascontiguousarray(buf[1: min(cnt, max_pairs) + 1])
        return pairs, cnt

    def neighbor_walk_items_mt(self, sorted_pos, keys, s2o, begin, end, table, cutoff_sq, npc,
                               shift, box: Box, items, max_pairs, nthreads):
        """neighbor_walk_items on host threads (per-thread outputs joined in
        order). Returns (pairs or None when they exceed max_pairs, count)."""
        o, s, p = self._box(box)
        items = np.ascontiguousarray(items, np.uint32)
        buf = np.zeros((max_pairs + 1, 2), np.int32)
        cnt = int(self.lib.ref_neighbor_walk_items_mt(
            _ptr(sorted_pos), _ptr(keys), _ptr(s2o), _ptr(begin), _ptr(end), _ptr(table),
            C.c_float(cutoff_sq), len(keys), npc, shift, _ptr(o), _ptr(s), _ptr(p), _ptr(items),
            len(items), _ptr(buf), max_pairs, int(nthreads)))
        return (np.ascontiguousarray(buf[1:cnt + 1]) if cnt <= max_pairs else None), cnt

    def read_table(self, path, kind):
        """Table::read_file of one text table; kind 0 pair, 1 bond, 2 angle,
        3 dihedral. Returns (X, Y, start, step, uniform) as float32."""
        cap = 1 << 20
        x = np.zeros(cap, np.float32)
        y = np.zeros(cap, np.float32)
        n = C.c_size_t()
        start, step, uniform = C.c_float(), C.c_float(), C.c_int()
        rc = self.lib.ref_read_table(str(path).encode(), int(kind), _ptr(x), _ptr(y), cap,
                                     C.byref(n), C.byref(start), C.byref(step), C.byref(uniform))
        assert rc == 0 and n.value <= cap
        return (x[:n.value].copy(), y[:n.value].copy(), np.float32(start.value),
                np.float32(step.value), bool(uniform.value))

    def resolve_tags(self, pairs, type_ids, term_matrix, num_types, nthreads=1):
        tags = np.zeros(len(pairs), np.uint32)
        self.lib.ref_resolve_tags(_ptr(pairs), len(pairs), _ptr(type_ids), _ptr(term_matrix),
                                  num_types, _ptr(tags), nthreads)
        return tags

    def pair_forces(self, pairs, pos4, type_ids, tags, tables: TableSet, box: Box, cutoff_sq,
                    get_energy=True, enabled_terms=0xFF):
        fe = np.zeros((len(pos4), 4), np.float32)
        o, s, p = self._box(box)
        self.lib.ref_pair_forces(_ptr(pairs), len(pairs), _ptr(pos4), _ptr(type_ids), _ptr(fe),
                                 _ptr(tags), _ptr(tables.values), _ptr(tables.offsets),
                                 _ptr(tables.sizes), _ptr(tables.starts), _ptr(tables.step_invs),
                                 len(tables), _ptr(o), _ptr(s), _ptr(p), int(get_energy),
                                 C.c_float(cutoff_sq), enabled_terms)
        return fe

    def pair_forces_mt(self, pairs, pos4, type_ids, tags, tables: TableSet, box: Box, cutoff_sq,
                       nthreads, get_energy=True, enabled_terms=0xFF):
        """pair_forces on host threads (per-thread ForceEnergy arrays added in order)."""
        fe = np.zeros((len(pos4), 4), np.float32)
        o, s, p = self._box(box)
        self.lib.ref_pair_forces_mt(_ptr(pairs), len(pairs), len(pos4), _ptr(pos4), _ptr(type_ids),
                                    _ptr(fe), _ptr(tags), _ptr(tables.values),
                                    _ptr(tables.offsets), _ptr(tables.sizes),
                                    _ptr(tables.starts), _ptr(tables.step_invs), len(tables),
                                    _ptr(o), _ptr(s), _ptr(p), int(get_energy),
                                    C.c_float(cutoff_sq), enabled_terms, int(nthreads))
        return fe

    def pair_forces_terms(self, pairs, pos4, type_ids, tags, tables: TableSet,
                          terms: "PairTermSet", box: Box, cutoff_sq, get_energy=True,
                          enabled_terms=0xFF):
        fe = np.zeros((len(pos4), 4), np.float32)
        o, s, p = self._box(box)
        tid = np.ascontiguousarray(type_ids, np.int32)
        self.lib.ref_pair_forces_terms(
            _ptr(np.ascontiguousarray(pairs, np.int32)), len(pairs), _ptr(pos4), _ptr(tid),
            _ptr(fe), _ptr(np.ascontiguousarray(tags, np.uint32)), _ptr(tables.values),
            _ptr(tables.offsets), _ptr(tables.sizes), _ptr(tables.starts),
            _ptr(tables.step_invs), len(tables), _ptr(o), _ptr(s), _ptr(p), int(get_energy),
            C.c_float(cutoff_sq), enabled_terms, _ptr(terms.charge), _ptr(terms.radius),
            _ptr(terms.eps), _ptr(terms.solvent), _ptr(terms.gaussian))
        return fe

    def dihedral_forces(self, dihedrals4, table_idx, pos4, tables: TableSet, box: Box,
                        get_energy=True):
        fe = np.zeros((len(pos4), 4), np.float32)
        tidx = np.ascontiguousarray(table_idx, np.int32)
        forms = np.where(tidx >= 0, 1, 2).astype(np.int32)  # Tabulated = 1, Analytical = 2
        tidx = np.maximum(tidx, 0).astype(np.int32)
        o, s, p = self._box(box)
        self.lib.ref_dihedral_forces(_ptr(np.ascontiguousarray(dihedrals4, np.int32)), _ptr(tidx),
                                     _ptr(forms), len(dihedrals4), _ptr(pos4), _ptr(fe),
                                     _ptr(tables.values), _ptr(tables.offsets),
                                     _ptr(tables.sizes), _ptr(tables.starts),
                                     _ptr(tables.step_invs), len(tables), _ptr(o), _ptr(s),
                                     _ptr(p), int(get_energy))
        return fe

    def restraint_forces(self, ids, anchors4, k_spring, pos4, box: Box, get_energy=True):
        fe = np.zeros((len(pos4), 4), np.float32)
        o, s, p = self._box(box)
        self.lib.ref_restraint_forces(_ptr(np.ascontiguousarray(ids, np.int32)),
                                      _ptr(np.ascontiguousarray(anchors4, np.float32)),
                                      _ptr(np.ascontiguousarray(k_spring, np.float32)), len(ids),
                                      _ptr(pos4), _ptr(fe), _ptr(o), _ptr(s), _ptr(p),
                                      int(get_energy))
        return fe

    def bond_forces(self, bonds, table_idx, pos4, tables: TableSet, box: Box, get_energy=True,
                    fe=None):
        fe = np.zeros((len(pos4), 4), np.float32) if fe is None else fe
        # InteractionForm (SimParam.h:174): Tabulated = 1; a negative index
        # stands for another form, which the tabulated functor skips.
        table_idx = np.ascontiguousarray(table_idx, np.int32)
        forms = np.where(table_idx >= 0, 1, 2).astype(np.int32)
        table_idx = np.maximum(table_idx, 0).astype(np.int32)
        o, s, p = self._box(box)
        self.lib.ref_bond_forces(_ptr(bonds), _ptr(table_idx), _ptr(forms), len(bonds), _ptr(pos4),
                                 _ptr(fe), _ptr(tables.values), _ptr(tables.offsets),
                                 _ptr(tables.sizes), _ptr(tables.starts), _ptr(tables.step_invs),
                                 len(tables), _ptr(o), _ptr(s), _ptr(p), int(get_energy))
        return fe

    def angle_forces(self, angles4, table_idx, pos4, tables: TableSet, box: Box, get_energy=True,
                     fe=None):
        fe = np.zeros((len(pos4), 4), np.float32) if fe is None else fe
        table_idx = np.ascontiguousarray(table_idx, np.int32)
        forms = np.where(table_idx >= 0, 1, 2).astype(np.int32)
        table_idx = np.maximum(table_idx, 0).astype(np.int32)
        o, s, p = self._box(box)
        self.lib.ref_angle_forces(_ptr(angles4), _ptr(table_idx), _ptr(forms), len(angles4),
                                  _ptr(pos4), _ptr(fe), _ptr(tables.values), _ptr(tables.offsets),
                                  _ptr(tables.sizes), _ptr(tables.starts), _ptr(tables.step_invs),
                                  len(tables), _ptr(o), _ptr(s), _ptr(p), int(get_energy))
        return fe

    def bd_integrate(self, pos4, fe4, type_ids, flags, types: TypeSet, grids, box: Box, dt, kT,
                     step, base_seed, base_ctr=0, efield=(0, 0, 0), nthreads=1):
        pos = np.array(pos4, np.float32)
        fe = np.array(fe4, np.float32)
        o, s, p = self._box(box)
        tid = np.ascontiguousarray(type_ids, np.int32)
        fl = np.zeros(len(pos), np.uint32) if flags is None else np.ascontiguousarray(flags, np.uint32)
        rg = None
        ng = 0
        if grids is not None and grids.n:
            rg = (RefGrid * grids.n)()
            for k in range(grids.n):
                C.memmove(C.byref(rg[k]), C.byref(grids.structs[k]), C.sizeof(RefGrid))
            ng = grids.n
        self.lib.ref_bd_integrate(_ptr(pos), _ptr(fe), _ptr(tid), _ptr(fl), len(pos),
                                  len(types.charge), _ptr(types.charge), _ptr(types.diffusion4),
                                  _ptr(types.pmf_offset), _ptr(types.pmf_count),
                                  _ptr(types.terms_flat), types.n_terms,
                                  _ptr(types.force_grid_id4), _ptr(types.force_grid_scale4),
                                  C.cast(rg, C.c_void_p) if rg is not None else None, ng,
                                  _ptr(o), _ptr(s), _ptr(p), C.c_float(dt), C.c_float(kT), step,
                                  base_seed, base_ctr, _ptr(np.asarray(efield, np.float32)),
                                  nthreads)
        return pos, fe

    def baoab_integrate(self, pos4, mom4, fe4, type_ids, flags, types: TypeSet, grids, mass,
                        damping, box: Box, dt, kT, step, base_seed, base_ctr=0, efield=(0, 0, 0),
                        pending=0):
        vp, f = C.c_void_p, C.c_float
        self.lib.ref_baoab_integrate.argtypes = [vp, vp, vp, vp, vp, C.c_size_t, C.c_int, vp, vp, vp,
                                                 vp, vp, vp, C.c_int, vp, vp, vp, C.c_int, vp, vp,
                                                 vp, f, f, C.c_uint64, C.c_uint64, C.c_uint32, vp,
                                                 C.c_int]
        pos, mom, fe = (np.array(a, np.float32) for a in (pos4, mom4, fe4))
        o, s, p = self._box(box)
        tid = np.ascontiguousarray(type_ids, np.int32)
        fl = np.zeros(len(pos), np.uint32) if flags is None else np.ascontiguousarray(flags, np.uint32)
        ms = np.ascontiguousarray(mass, np.float32)
        d4 = np.zeros((len(ms), 4), np.float32)
        d4[:, :3] = np.asarray(damping, np.float32).reshape(-1, 3)
        rg, ng = None, 0
        if grids is not None and grids.n:
            rg = (RefGrid * grids.n)()
            for k in range(grids.n):
                C.memmove(C.byref(rg[k]), C.byref(grids.structs[k]), C.sizeof(RefGrid))
            ng = grids.n
        self.lib.ref_baoab_integrate(
            _ptr(pos), _ptr(mom), _ptr(fe), _ptr(tid), _ptr(fl), len(pos), len(types.charge),
            _ptr(types.charge), _ptr(ms), _ptr(d4), _ptr(types.pmf_offset), _ptr(types.pmf_count),
            _ptr(types.terms_flat), types.n_terms, _ptr(types.force_grid_id4),
            _ptr(types.force_grid_scale4), C.cast(rg, C.c_void_p) if rg is not None else None, ng,
            _ptr(o), _ptr(s), _ptr(p), f(dt), f(kT), step, base_seed, base_ctr,
            _ptr(np.asarray(efield, np.float32)), int(pending))
        return pos, mom, fe

    def philox_int4(self, seed, ctr, global_seed, ctr1, ndraw=1):
        out = np.zeros((ndraw, 4), np.uint32)
        self.lib.ref_philox_int4(seed, ctr, global_seed, ctr1, ndraw, _ptr(out))
        return out

    def philox_float4(self, seed, ctr, global_seed, ctr1, ndraw=1):
        out = np.zeros((ndraw, 4), np.float32)
        self.lib.ref_philox_float4(seed, ctr, global_seed, ctr1, ndraw, _ptr(out))
        return out

    def max_displacement(self, cur4, prev4, box_len):
        return self.lib.ref_max_displacement(_ptr(cur4), _ptr(prev4), len(cur4),
                                             _ptr(np.asarray(box_len, np.float32)))

    def wrap_diff(self, box: Box, v4):
        o, s, p = self._box(box)
        out = np.zeros_like(v4)
        self.lib.ref_wrap_diff(_ptr(o), _ptr(s), _ptr(p), _ptr(v4), _ptr(out), len(v4))
        return out

    def wrap(self, box: Box, v4):
        o, s, p = self._box(box)
        out = np.zeros_like(v4)
        self.lib.ref_wrap(_ptr(o), _ptr(s), _ptr(p), _ptr(v4), _ptr(out), len(v4))
        return out


# -- FP64 BD window and adjoint (oracle/mb2_adjoint.c) ----------------------------

class AdjTable(C.Structure):
    _fields_ = [("v", C.c_void_p), ("size", C.c_int), ("start", C.c_double),
                ("step_inv", C.c_double), ("periodic", C.c_int)]


class AdjSys(C.Structure):
    _fields_ = [("n", C.c_int), ("L", C.c_double * 3), ("c", C.c_double * 3),
                ("s", C.c_double * 3), ("pair", AdjTable), ("cutoff", C.c_double),
                ("excl_off", C.c_void_p), ("excl_nb", C.c_void_p), ("excl_n", C.c_int),
                ("bonds", C.c_void_p), ("nb", C.c_int), ("bond", AdjTable),
                ("angles", C.c_void_p), ("na", C.c_int), ("angle", AdjTable),
                ("float_bins", C.c_int), ("list_every", C.c_int), ("list_radius", C.c_double)]


class Adjoint64:
    """FP64 forward window, RDF loss and adjoint of a BD system with one pair
    table, one bond table and one (periodic) angle table. Keeps the arrays the
    C structure points to alive."""

    def __init__(self, oracle: "Oracle", n, box_len, diffusion, dt, kT, pair, cutoff,
                 bonds=None, bond=None, angles=None, angle=None, exclusions=None,
                 float_bins=False, list_every=0, list_radius=0.0):
        """The box edges are taken as float32 values, as the library holds
        them. float_bins: decide table bins, cutoffs and angle clamps with the
        reference's float arithmetic (the derivative of a float forward along
        float states); otherwise in double."""
        L = self.lib = oracle.lib
        vp = C.c_void_p
        L.adj_forces64.argtypes = [vp, vp, vp]
        L.adj_forward64.argtypes = [vp, vp, vp, C.c_int, vp]
        L.adj_backward64.argtypes = [vp, vp, C.c_int, vp, vp, vp]
        L.adj_rdf64.argtypes = [vp, vp, C.c_int, C.c_double, C.c_double, C.c_double, vp]
        L.adj_rdf_grad64.argtypes = [vp, vp, C.c_int, C.c_double, C.c_double, C.c_double, vp, vp]
        self.keep = []
        s = self.sys = AdjSys()
        s.n = int(n)
        d = np.asarray(diffusion, np.float64).reshape(3)
        s.float_bins = int(bool(float_bins))
        # list_every > 0: pairs as the window's pairlist (built every list_every
        # steps within list_radius) instead of all pairs within the cutoff.
        s.list_every = int(list_every)
        s.list_radius = float(list_radius)
        for a in range(3):
            s.L[a] = float(np.float32(box_len[a]))
            s.c[a] = float(d[a] * dt / kT)
            s.s[a] = float(np.sqrt(2.0 * d[a] * dt))
        self.pair_values = self._table(s.pair, pair, False)
        s.cutoff = float(cutoff)
        if exclusions is not None and len(exclusions):
            off, nb, npart = oracle.exclusion_csr(exclusions)
            self.keep += [off, nb]
            s.excl_off, s.excl_nb, s.excl_n = off.ctypes.data, nb.ctypes.data, int(npart)
        if bonds is not None and len(bonds):
            b = np.ascontiguousarray(bonds, np.int32)
            self.keep.append(b)
            s.bonds, s.nb = b.ctypes.data, len(b)
            self.bond_values = self._table(s.bond, bond, False)
        if angles is not None and len(angles):
            a4 = np.ascontiguousarray(angles, np.int32)
            self.keep.append(a4)
            s.angles, s.na = a4.ctypes.data, len(a4)
            self._table(s.angle, angle, True)

    def _table(self, dst, spec, periodic):
        """spec: (values, start, step_inv); returns the float64 values array (mutable)."""
        v = np.ascontiguousarray(spec[0], np.float64).copy()
        self.keep.append(v)
        dst.v, dst.size, dst.start, dst.step_inv, dst.periodic = (
            v.ctypes.data, len(v), float(spec[1]), float(spec[2]), int(periodic))
        return v

    def forward(self, x0, noise):
        """x0 [n, 3] float64, noise [steps, n, 3]; returns trajectory [steps + 1, n, 3]."""
        steps = len(noise)
        traj = np.zeros((steps + 1, self.sys.n, 3), np.float64)
        x0 = np.ascontiguousarray(x0, np.float64)
        nz = np.ascontiguousarray(noise, np.float64)
        self.lib.adj_forward64(C.byref(self.sys), x0.ctypes.data, nz.ctypes.data, steps,
                               traj.ctypes.data)
        return traj

    def rdf(self, x, nbins, dr, rmax, sigma):
        h = np.zeros(nbins, np.float64)
        self.lib.adj_rdf64(C.byref(self.sys), np.ascontiguousarray(x, np.float64).ctypes.data,
                           nbins, dr, rmax, sigma, h.ctypes.data)
        return h

    def rdf_grad(self, x, nbins, dr, rmax, sigma, dLdh):
        g = np.zeros((self.sys.n, 3), np.float64)
        dl = np.ascontiguousarray(dLdh, np.float64)
        self.lib.adj_rdf_grad64(C.byref(self.sys), np.ascontiguousarray(x, np.float64).ctypes.data,
                                nbins, dr, rmax, sigma, dl.ctypes.data, g.ctypes.data)
        return g

    def backward(self, traj, lamN):
        """Returns (grad x0 [n, 3], grad pair table, grad bond table)."""
        lam = np.ascontiguousarray(lamN, np.float64).copy()
        gp = np.zeros(len(self.pair_values), np.float64)
        gb = np.zeros(len(getattr(self, "bond_values", [0.0])), np.float64)
        self.lib.adj_backward64(C.byref(self.sys), np.ascontiguousarray(traj).ctypes.data,
                                len(traj) - 1, lam.ctypes.data, gp.ctypes.data, gb.ctypes.data)
        return lam, gp, gb
