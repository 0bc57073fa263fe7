"""ctypes binding of libmarsb200.so (the C ABI in include/marsb200.h).

The library is loaded from this package directory. There is no fallback: if
it is missing, or no CUDA device is present, every call fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmarsb200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "marsb200.h")

MB2_OK, MB2_ERR_ARG, MB2_ERR_CUDA, MB2_ERR_CAPACITY, MB2_ERR_STATE = 0, 1, 2, 3, 4
MB2_SORT_STATIC_MAX = 1048576  # largest n of mb2_radix_sort_pairs_static
STAGE_STEP, STAGE_PAIRLIST, STAGE_PAIR_FORCE, STAGE_INTEGRATE = 0, 1, 2, 3


class MB2Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[mb2 error {code}] {msg}")
        self.code = code


class StepParams(C.Structure):
    _fields_ = [("pairlist_cutoff", C.c_float), ("cutoff", C.c_float),
                ("rebuild_period", C.c_uint32), ("dt", C.c_float), ("kT", C.c_float),
                ("seed", C.c_uint64), ("patch_id", C.c_uint64), ("efield", C.c_float * 3),
                ("get_energy", C.c_int), ("bonds2", C.c_void_p), ("bond_table_idx", C.c_void_p),
                ("num_bonds", C.c_uint32), ("angles4", C.c_void_p),
                ("angle_table_idx", C.c_void_p), ("num_angles", C.c_uint32),
                ("dihedrals4", C.c_void_p), ("dihedral_table_idx", C.c_void_p),
                ("num_dihedrals", C.c_uint32), ("restraint_ids", C.c_void_p),
                ("restraint_anchors4", C.c_void_p), ("restraint_k", C.c_void_p),
                ("num_restraints", C.c_uint32), ("integrator", C.c_int), ("mom4", C.c_void_p),
                ("deferred_kick_pending", C.c_int)]


class OutputConfig(C.Structure):
    """mb2_output_config."""
    _fields_ = [("output_name", C.c_char_p), ("num_particles", C.c_uint32),
                ("output_period", C.c_int), ("timestep", C.c_float), ("box", C.c_float * 3),
                ("periodic", C.c_int * 3), ("with_momentum", C.c_int), ("device", C.c_int)]


class PairParams(C.Structure):
    """mb2_pair_params (defaults: the reference's SolventParams and Gaussian)."""
    _fields_ = [("debye_length", C.c_float), ("dielectric", C.c_float),
                ("onck_kappa", C.c_float), ("onck_sz", C.c_float), ("onck_z", C.c_float),
                ("gaussian_amp", C.c_float), ("gaussian_sigma", C.c_float),
                ("gaussian_cutoff_sq", C.c_float)]


class BatchTuning(C.Structure):
    """mb2_batch_tuning_result."""
    _fields_ = [("level_offset", C.c_int), ("lanes", C.c_int), ("build_ms", C.c_float),
                ("step_ms", C.c_float), ("safe_rebuild_period", C.c_uint32),
                ("max_displacement_at_period", C.c_float), ("total_cells", C.c_uint32)]


_lib = None


def header_symbols() -> list:
    """Names of the functions include/marsb200.h declares."""
    txt = open(HEADER).read()
    return re.findall(r"^MB2_API\s+[\w\s\*]+?\b(mb2_\w+)\s*\(", txt, flags=re.M)


def load(path: str = LIB_PATH):
    """Load the library once. Raises if the CUDA extension was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libmarsb200.so not built at {path}; run `python -m mars_md_b200.build`")
    L = C.CDLL(path)
    vp, u32, u64, i, f = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_float
    fp, ip, u32p, u64p = C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
    L.mb2_version.restype = i
    L.mb2_create.argtypes = [i, u32, C.POINTER(vp)]
    L.mb2_destroy.argtypes = [vp]
    L.mb2_last_error.restype = C.c_char_p
    L.mb2_last_error.argtypes = [vp]
    L.mb2_set_box.argtypes = [vp, fp, fp, ip]
    L.mb2_sort_morton.argtypes = [vp, vp, u32, fp, fp, vp, vp, vp, vp, vp]
    L.mb2_radix_sort_pairs.argtypes = [vp, vp, vp, u32, vp]
    L.mb2_radix_sort_pairs_static.argtypes = [vp, vp, vp, u32, vp]
    L.mb2_set_exclusions.argtypes = [vp, vp, vp, u32, vp]
    L.mb2_build_pairlist.argtypes = [vp, vp, vp, u32, f, f, vp, u64p]
    L.mb2_num_pairs.argtypes = [vp, u64p]
    L.mb2_export_pairs.argtypes = [vp, vp, u64, vp]
    L.mb2_needs_update.argtypes = [vp, vp, u32, f, vp, fp, ip]
    L.mb2_set_pair_tables.argtypes = [vp, i, u32p, i, fp, u32p, fp, fp]
    L.mb2_pair_forces.argtypes = [vp, vp, vp, vp, u32, f, i, vp]
    L.mb2_energies.argtypes = [vp, vp, C.POINTER(C.c_double)]
    L.mb2_reset_energies.argtypes = [vp, vp]
    L.mb2_set_bonded_tables.argtypes = [vp, i, i, fp, u32p, fp, fp]
    L.mb2_bond_forces.argtypes = [vp, vp, vp, u32, vp, vp, i, vp]
    L.mb2_angle_forces.argtypes = [vp, vp, vp, u32, vp, vp, i, vp]
    L.mb2_set_particle_types.argtypes = [vp, i, fp, fp, ip, ip, i, fp, ip, fp]
    L.mb2_set_grid.argtypes = [vp, i, vp, C.POINTER(C.c_int64), fp, fp, i]
    L.mb2_bd_integrate.argtypes = [vp, vp, vp, vp, vp, u32, f, f, u64, u64, u32, fp, vp]
    L.mb2_bd_seed.restype = u64
    L.mb2_bd_seed.argtypes = [u64, u64, u64]
    L.mb2_philox.argtypes = [vp, u64, u32, u32, u32, u32, vp, vp, vp]
    L.mb2_step.argtypes = [vp, vp, vp, vp, vp, u32, u64, C.POINTER(StepParams), vp]
    L.mb2_run.argtypes = [vp, vp, vp, vp, vp, u32, u64, u32, C.POINTER(StepParams), vp]
    L.mb2_set_lanes_per_row.argtypes = [vp, i]
    L.mb2_set_cell_level_offset.argtypes = [vp, i]
    L.mb2_cell_level.argtypes = [vp, C.POINTER(C.c_int)]
    L.mb2_set_profiling.argtypes = [vp, i]
    L.mb2_profile_read.argtypes = [vp, i, C.POINTER(C.c_double), u32p]
    L.mb2_launch_count.restype = u64
    L.mb2_launch_count.argtypes = []
    L.mb2_output_create.argtypes = [C.POINTER(OutputConfig), C.POINTER(vp)]
    L.mb2_output_destroy.argtypes = [vp]
    L.mb2_output_last_error.restype = C.c_char_p
    L.mb2_output_last_error.argtypes = [vp]
    L.mb2_output_frame.argtypes = [vp, vp, vp, vp, u32, vp]
    L.mb2_output_restart.argtypes = [vp, vp, vp, vp, vp, u32, vp]
    L.mb2_output_energy.argtypes = [vp, vp, vp, vp, fp, i, u32, f, vp, C.POINTER(C.c_double)]
    L.mb2_output_flush.argtypes = [vp]
    L.mb2_set_pair_terms.argtypes = [vp, i, fp, fp, fp, C.POINTER(PairParams)]
    L.mb2_dihedral_forces.argtypes = [vp, vp, vp, u32, vp, vp, i, vp]
    L.mb2_restraint_forces.argtypes = [vp, vp, vp, vp, u32, vp, vp, i, vp]
    L.mb2_energy_terms.argtypes = [vp, vp, C.POINTER(C.c_double), i]
    L.mb2_reorder_begin.argtypes = [vp, vp, u32, vp]
    L.mb2_reorder_apply.argtypes = [vp, vp, u32, u32, vp]
    L.mb2_reorder_remap.argtypes = [vp, vp, u64, vp]
    L.mb2_reorder_inverse.argtypes = [vp, vp, u32, vp]
    L.mb2_set_langevin_types.argtypes = [vp, i, fp, fp]
    L.mb2_baoab_integrate.argtypes = [vp, vp, vp, vp, vp, vp, u32, f, f, u64, u64, u32, fp, i, vp]
    L.mb2_baoab_last_update.argtypes = [vp, vp, vp, vp, u32, f, vp]
    L.mb2_window_forward.argtypes = [vp, vp, vp, vp, u32, u64, u32, u32, C.POINTER(StepParams), vp]
    L.mb2_window_backward.argtypes = [vp, vp, vp, vp, vp, vp]
    L.mb2_window_checkpoints.argtypes = [vp, vp, u64, vp]
    L.mb2_window_record_states.argtypes = [vp, vp, u64]
    L.mb2_pair_distance_window.argtypes = [f, fp, fp]
    L.mb2_selftest_sqrt.argtypes = [vp, u64p]
    L.mb2_rdf_histogram.argtypes = [vp, vp, vp, u32, u32, f, f, f, vp, vp]
    L.mb2_rdf_backward.argtypes = [vp, vp, u32, u32, f, f, f, vp, vp, vp]
    L.mb2_batch_create.argtypes = [i, u32, u32p, fp, fp, C.POINTER(vp)]
    L.mb2_batch_destroy.argtypes = [vp]
    L.mb2_batch_last_error.restype = C.c_char_p
    L.mb2_batch_last_error.argtypes = [vp]
    L.mb2_batch_set_pair_tables.argtypes = [vp, i, u32p, i, fp, u32p, fp, fp]
    L.mb2_batch_set_particle_types.argtypes = [vp, i, fp, fp]
    L.mb2_batch_build.argtypes = [vp, vp, vp, f, vp, u64p]
    L.mb2_batch_num_pairs.argtypes = [vp, u64p]
    L.mb2_batch_export_pairs.argtypes = [vp, vp, u64, vp]
    L.mb2_batch_step.argtypes = [vp, vp, vp, vp, u64, C.POINTER(StepParams), vp]
    L.mb2_batch_run.argtypes = [vp, vp, vp, vp, u64, u32, C.POINTER(StepParams), vp]
    L.mb2_batch_set_tuning.argtypes = [vp, i, i]
    L.mb2_batch_set_rebuild_period.argtypes = [vp, u32]
    L.mb2_batch_rebuild_schedule.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.mb2_batch_system_rebuilds.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.mb2_batch_tuning.argtypes = [vp, ip, ip, u32p]
    L.mb2_batch_autotune.argtypes = [vp, vp, vp, C.POINTER(StepParams), u32, vp,
                                     C.POINTER(BatchTuning)]
    _lib = L
    return L
