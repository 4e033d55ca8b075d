"""ctypes binding of libmdx.so (include/mdx.h).

The library is the product: if it is missing or cannot be loaded this module
raises -- there is no CPU or PyTorch fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmdx.so")
_lib = None

c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_dbl = ctypes.c_double
c_flt = ctypes.c_float
c_char_p = ctypes.c_char_p
c_void_p = ctypes.c_void_p
P = ctypes.POINTER

# (name, restype, argtypes) for every entry point declared in include/mdx.h
SIGNATURES = [
    ("mdx_last_error", c_char_p, []),
    ("mdx_version", c_int, []),
    ("mdx_set_device", c_int, [c_int]),
    ("mdx_kernel_launch_count", c_u64, []),
    ("mdx_state_create", c_int, [P(c_void_p)]),
    ("mdx_state_destroy", c_int, [c_void_p]),
    ("mdx_state_set_units", c_int, [c_void_p, c_int]),
    ("mdx_state_set_bounds", c_int, [c_void_p, P(c_dbl), P(c_dbl)]),
    ("mdx_state_set_double", c_int, [c_void_p, c_char_p, c_dbl]),
    ("mdx_state_get_double", c_int, [c_void_p, c_char_p, P(c_dbl)]),
    ("mdx_state_set_int", c_int, [c_void_p, c_char_p, c_i64]),
    ("mdx_state_get_int", c_int, [c_void_p, c_char_p, P(c_i64)]),
    ("mdx_state_set_special_neighbor_coefs", c_int, [c_void_p, c_dbl, c_dbl, c_dbl]),
    ("mdx_state_add_species", c_int, [c_void_p, c_char_p, c_dbl, c_int, P(c_int)]),
    ("mdx_state_add_atoms", c_int, [c_void_p, c_int, P(c_char_p), P(c_dbl), P(c_dbl), P(c_int)]),
    ("mdx_state_n_atoms", c_int, [c_void_p, P(c_int)]),
    ("mdx_state_set_velocities", c_int, [c_void_p, c_int, P(c_int), P(c_dbl)]),
    ("mdx_state_get_atoms", c_int, [c_void_p, P(c_dbl), P(c_dbl), P(c_dbl)]),
    ("mdx_state_put_atoms", c_int, [c_void_p, P(c_dbl), P(c_dbl)]),
    ("mdx_state_activate_fix", c_int, [c_void_p, c_void_p]),
    ("mdx_state_deactivate_fix", c_int, [c_void_p, c_void_p]),
    ("mdx_state_status", c_int, [c_void_p, P(c_u32), P(c_u32), P(c_u64)]),
    ("mdx_state_set_stream", c_int, [c_void_p, c_void_p]),
    ("mdx_state_synchronize", c_int, [c_void_p]),
    ("mdx_fix_lj_cut_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_wca_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_lj_cut_fs_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_lj_charmm_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_ticg_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_charge_pair_dsf_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_charge_pair_dsf_set_parameters", c_int, [c_void_p, c_dbl, c_dbl]),
    ("mdx_fix_pair_set_parameter", c_int, [c_void_p, c_char_p, c_char_p, c_char_p, c_dbl]),
    ("mdx_fix_pair_get_parameter", c_int, [c_void_p, c_char_p, c_char_p, c_char_p, P(c_dbl)]),
    ("mdx_fix_charge_ewald_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_charge_ewald_set_parameters", c_int, [c_void_p, c_int, c_int, c_int, c_dbl, c_int]),
    ("mdx_fix_charge_ewald_set_alpha", c_int, [c_void_p, c_dbl]),
    ("mdx_fix_charge_ewald_get_alpha", c_int, [c_void_p, P(c_dbl)]),
    ("mdx_fix_e3b_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_e3b_add_molecule", c_int, [c_void_p, c_int, c_int, c_int, c_int]),
    ("mdx_fix_rigid_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_rigid_create_rigid", c_int, [c_void_p, c_int, c_int, c_int, c_int]),
    ("mdx_fix_nose_hoover_create", c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    ("mdx_fix_nose_hoover_set_temperature", c_int, [c_void_p, c_dbl, c_dbl]),
    ("mdx_fix_nose_hoover_set_pressure", c_int, [c_void_p, c_char_p, c_dbl, c_dbl]),
    ("mdx_fix_nose_hoover_get", c_int, [c_void_p, c_char_p, P(c_dbl)]),
    ("mdx_fix_destroy", c_int, [c_void_p]),
    ("mdx_integrator_verlet_create", c_int, [c_void_p, P(c_void_p)]),
    ("mdx_integrator_run", c_int, [c_void_p, c_int, P(c_dbl)]),
    ("mdx_integrator_set_mode", c_int, [c_void_p, c_int]),
    ("mdx_integrator_destroy", c_int, [c_void_p]),
    ("mdx_integrator_run_host", c_int, [c_void_p, c_int, P(c_dbl), P(c_dbl), P(c_dbl), P(c_dbl), P(c_dbl)]),
    ("mdx_integrator_run_timed", c_int, [c_void_p, c_int, c_int, ctypes.c_size_t, P(c_dbl)]),
    ("mdx_integrator_autotune", c_int, [c_void_p, c_int, P(c_int), c_int, P(c_int), P(c_dbl)]),
    ("mdx_time_stage", c_int, [c_void_p, c_int, c_int, ctypes.c_size_t, P(c_dbl)]),
    ("mdx_prepare", c_int, [c_void_p]),
    ("mdx_nlist_build", c_int, [c_void_p, c_int]),
    ("mdx_nlist_get", c_int, [c_void_p, c_int, P(c_int), P(c_int), P(c_int)]),
    ("mdx_compute_forces", c_int, [c_void_p, c_int]),
    ("mdx_potential_energy", c_int, [c_void_p, P(c_dbl)]),
    ("mdx_kinetic", c_int, [c_void_p, P(c_dbl), P(c_dbl)]),
    ("mdx_kinetic_noalloc", c_int, [c_void_p, P(c_dbl)]),
    ("mdx_get_virials", c_int, [c_void_p, P(c_dbl), P(c_dbl)]),
    ("mdx_pressure", c_int, [c_void_p, P(c_dbl), P(c_dbl)]),
    ("mdx_rigid_settle_positions", c_int, [c_void_p, c_void_p]),
    ("mdx_rigid_save_prev", c_int, [c_void_p, c_void_p]),
    ("mdx_rigid_settle_velocities", c_int, [c_void_p, c_void_p]),
    ("mdx_rigid_distribute_msite", c_int, [c_void_p, c_void_p]),
    ("mdx_verlet_first_half", c_int, [c_void_p]),
    ("mdx_verlet_second_half", c_int, [c_void_p]),
    ("mdx_pair_force_raw", c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                   c_void_p, c_int, P(c_dbl), P(c_dbl), P(c_flt), c_int, c_flt, c_flt, c_flt,
                                   c_void_p, c_int, c_void_p]),
    ("mdx_pair_force_gridgpu", c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                       c_void_p, c_int, P(c_dbl), P(c_dbl), c_flt, c_flt, c_flt, c_void_p, c_void_p,
                                       c_flt, c_int, c_int, c_int, c_int, c_flt, c_flt, c_void_p]),
    ("mdx_rigid_validate", c_int, [c_void_p, c_void_p, P(ctypes.c_uint32)]),
    ("mdx_e3b_surrogate_collect", c_int, [c_void_p, c_void_p]),
    ("mdx_e3b_surrogate_dataset_size", c_int, [c_void_p, P(ctypes.c_int64)]),
    ("mdx_e3b_surrogate_train", c_int, [c_void_p, c_void_p, c_int, c_int, c_flt, ctypes.c_uint64, P(c_dbl), P(c_dbl)]),
    ("mdx_e3b_surrogate_enable", c_int, [c_void_p, c_int]),
    ("mdx_e3b_surrogate_eval", c_int, [c_void_p, c_void_p, P(c_dbl), P(c_dbl)]),
    ("mdx_e3b_surrogate_get_params", c_int, [c_void_p, P(c_flt), P(c_flt), P(c_flt), P(c_flt)]),
    ("mdx_e3b_surrogate_set_params", c_int, [c_void_p, c_void_p, P(c_flt), P(c_flt), P(c_flt), c_flt]),
    ("mdx_e3b_surrogate_features", c_int, [c_void_p, c_void_p, P(c_flt), P(c_flt)]),
    ("mdx_e3b_surrogate_infer", c_int, [c_void_p, c_void_p, P(c_flt), c_int, P(c_flt)]),
    ("mdx_e3b_surrogate_grad", c_int, [c_void_p, c_void_p, P(c_flt), P(c_flt), c_int, P(c_flt), P(c_dbl)]),
    ("mdx_batch_create", c_int, [P(c_void_p)]),
    ("mdx_batch_add", c_int, [c_void_p, c_void_p]),
    ("mdx_batch_size", c_int, [c_void_p, P(c_int)]),
    ("mdx_batch_prepare", c_int, [c_void_p]),
    ("mdx_batch_run", c_int, [c_void_p, c_int, P(c_dbl)]),
    ("mdx_batch_run_timed", c_int, [c_void_p, c_int, c_int, ctypes.c_size_t, P(c_dbl)]),
    ("mdx_batch_autotune", c_int, [c_void_p, c_int, P(c_int), c_int, P(c_int), P(c_dbl)]),
    ("mdx_batch_destroy", c_int, [c_void_p]),
    ("mdx_fix_pressure_berendsen_create", c_int, [c_void_p, c_char_p, c_dbl, c_dbl, c_int, P(c_void_p)]),
    ("mdx_fix_pressure_berendsen_set", c_int, [c_void_p, c_char_p, c_dbl]),
    ("mdx_fix_pressure_berendsen_get", c_int, [c_void_p, c_char_p, P(c_dbl)]),
    ("mdx_state_scale_system", c_int, [c_void_p, c_dbl]),
    ("mdx_write_config_create", c_int, [c_void_p, c_char_p, c_char_p, c_char_p, c_int, c_char_p, c_int,
                                        P(c_void_p)]),
    ("mdx_write_config_set", c_int, [c_void_p, c_char_p, c_i64]),
    ("mdx_write_config_write", c_int, [c_void_p, c_i64]),
    ("mdx_write_config_destroy", c_int, [c_void_p]),
    ("mdx_state_activate_write_config", c_int, [c_void_p, c_void_p]),
    ("mdx_state_deactivate_write_config", c_int, [c_void_p, c_void_p]),
    ("mdx_write_output", c_int, [c_void_p]),
    ("mdx_read_config_load", c_int, [c_void_p, c_char_p]),
    ("mdx_read_config_move", c_int, [c_void_p, c_int, c_int, P(c_int)]),
    ("mdx_state_create_group", c_int, [c_void_p, c_char_p, c_int, P(c_int)]),
    ("mdx_state_group_tag", c_int, [c_void_p, c_char_p, P(c_u32)]),
    ("mdx_state_create_molecule", c_int, [c_void_p, c_int, P(c_int)]),
    ("mdx_state_get_bounds", c_int, [c_void_p, P(c_dbl), P(c_dbl)]),
    ("mdx_state_get_species", c_int, [c_void_p, c_int, c_char_p, c_int, P(c_dbl), P(c_int), P(c_int)]),
]


class MdxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mdx error {code}: {msg}")
        self.code = code


def lib():
    """Load libmdx.so (raises if it is missing: no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with md_engine_b200.build.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code):
    if code != 0:
        raise MdxError(code, lib().mdx_last_error().decode())
    return code
