"""ctypes binding of the C ABI declared in include/mjolnir_b200.h.

Loading fails loudly when ``libmjolnir_b200.so`` is missing: there is no CPU
fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmjolnir_b200.so")

OK, EINVAL, ECUDA, ESTATE, ENOMEM, EOVERFLOW, ENONFINITE = 0, -1, -2, -3, -4, -5, -6
PRECISION_FP64, PRECISION_MIXED = 0, 1
UNLIMITED, PERIODIC_CUBOID = 0, 1
TERM_BOND, TERM_ANGLE, TERM_DIHEDRAL, TERM_EXV, TERM_DH, TERM_LJ = range(6)
TERM_NAMES = ("bond", "angle", "dihedral", "exv", "dh", "lj")
IGNORE = {"Nothing": 0, "Self": 1, "Intra": 1, "Others": 2, "Inter": 2}
BAOAB, VELOCITY_VERLET, UNDERDAMPED_LANGEVIN, GJF_LANGEVIN, GBAOAB_LANGEVIN = 0, 1, 2, 3, 4

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_ctx = C.c_void_p

# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "mjg_context_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mjg_context_destroy": (None, [_ctx]),
    "mjg_last_error": (C.c_char_p, [_ctx]),
    "mjg_context_set_graphs": (C.c_int, [_ctx, C.c_int]),
    "mjg_context_set_rollback": (C.c_int, [_ctx, C.c_int]),
    "mjg_system_create": (C.c_int, [_ctx, C.c_int64, C.c_int, _f64p, _f64p, _f64p, _f64p, _f64p,
                                    C.POINTER(C.c_int)]),
    "mjg_system_set_attributes": (C.c_int, [_ctx, C.c_int, C.c_double, C.c_double]),
    "mjg_system_add_connections": (C.c_int, [_ctx, C.c_int, C.c_char_p, C.c_int64, _i64p]),
    "mjg_system_remove": (C.c_int, [_ctx, C.c_int]),
    "mjg_system_set_step": (C.c_int, [_ctx, C.c_int, C.c_uint64]),
    "mjg_system_set_temperature": (C.c_int, [_ctx, C.c_int, C.c_double]),
    "mjg_system_freeze": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "mjg_exv_set": (C.c_int, [_ctx, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int64, _i64p, _f64p]),
    "mjg_dh_set": (C.c_int, [_ctx, C.c_int, C.c_double, C.c_double, C.c_int64, _i64p, _f64p]),
    "mjg_exv_family_set": (C.c_int, [_ctx, C.c_int, C.c_char_p, C.c_double, C.c_double, C.c_int, C.c_double,
                                     C.c_int64, _i64p, _f64p, _f64p]),
    "mjg_pair_set": (C.c_int, [_ctx, C.c_int, C.c_char_p, C.c_double, C.c_double, C.c_int64, _i64p, _f64p, _f64p]),
    "mjg_lj_set": (C.c_int, [_ctx, C.c_int, C.c_double, C.c_double, C.c_int64, _i64p, _f64p, _f64p]),
    "mjg_ignore_set": (C.c_int, [_ctx, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_char_p), _i32p]),
    "mjg_bonds_set": (C.c_int, [_ctx, C.c_int, C.c_char_p, C.c_int64, _i64p, _f64p, _f64p]),
    "mjg_angles_set": (C.c_int, [_ctx, C.c_int, C.c_char_p, C.c_int64, _i64p, _f64p, _f64p]),
    "mjg_dihedrals_set": (C.c_int, [_ctx, C.c_int, C.c_char_p, C.c_int64, _i64p, _f64p, _i32p, _f64p]),
    "mjg_integrator_set": (C.c_int, [_ctx, C.c_int, C.c_int, C.c_double, _f64p, C.c_uint64]),
    "mjg_commit": (C.c_int, [_ctx]),
    "mjg_step": (C.c_int, [_ctx, C.c_int64]),
    "mjg_synchronize": (C.c_int, [_ctx]),
    "mjg_rebuild": (C.c_int, [_ctx]),
    "mjg_get_state": (C.c_int, [_ctx, C.c_int, _f64p, _f64p, _f64p]),
    "mjg_set_state": (C.c_int, [_ctx, C.c_int, _f64p, _f64p]),
    "mjg_get_state_all": (C.c_int, [_ctx, _f64p, _f64p]),
    "mjg_set_state_all": (C.c_int, [_ctx, _f64p, _f64p]),
    "mjg_energies": (C.c_int, [_ctx, C.c_int, _f64p]),
    "mjg_term_force": (C.c_int, [_ctx, C.c_int, C.c_int, _f64p, _f64p]),
    "mjg_neighbors": (C.c_int, [_ctx, C.c_int, C.c_int, _i64p, C.c_int64, _i64p]),
    "mjg_rebuild_count": (C.c_int, [_ctx, C.c_int, C.c_int, _i64p]),
    "mjg_step_count": (C.c_int, [_ctx, C.c_int, _i64p]),
    "mjg_context_reserve": (C.c_int, [_ctx, C.c_int64]),
    "mjg_molecule_count": (C.c_int, [_ctx, C.c_int, _i64p]),
    "mjg_particle_count": (C.c_int, [_ctx, C.c_int, _i64p]),
    "mjg_device_bytes": (C.c_int, [_ctx, _i64p]),
    "mjg_launch_count": (C.c_int, [_ctx, _i64p]),
    "mjg_pair_count": (C.c_int, [_ctx, C.c_int, C.c_int, _i64p]),
    "mjg_set_list_capacity": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "mjg_context_get_stream": (C.c_int, [_ctx, C.POINTER(C.c_void_p)]),
    "mjg_time_kernel": (C.c_int, [_ctx, C.c_int, C.c_int, _f64p]),
    "mjg_set_threads_per_particle": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "mjg_get_threads_per_particle": (C.c_int, [_ctx, C.c_int, C.POINTER(C.c_int)]),
    "mjg_set_pair_unroll": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "mjg_get_pair_unroll": (C.c_int, [_ctx, C.c_int, C.POINTER(C.c_int)]),
    "mjg_set_pair_schedule": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "mjg_get_pair_schedule": (C.c_int, [_ctx, C.c_int, C.POINTER(C.c_int)]),
    "mjg_set_half_lists": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "mjg_get_half_lists": (C.c_int, [_ctx, C.c_int, C.POINTER(C.c_int)]),
    "mjg_set_build_lanes": (C.c_int, [_ctx, C.c_int, C.c_int]),
    "mjg_get_build_lanes": (C.c_int, [_ctx, C.c_int, C.POINTER(C.c_int)]),
    "mjg_set_margin": (C.c_int, [_ctx, C.c_int, C.c_double]),
    "mjg_exv_force_noalloc": (C.c_int, [C.c_int64, C.c_int, _f64p, _f64p, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
}

# include/mjolnir_b200_synthetic.h (host-only builders)
SYNTH_SIGNATURES = {
    "mjg_synth_polymer_chains": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                                           C.c_uint64, _f64p]),
    "mjg_synth_uniform_fluid": (C.c_int, [C.c_int64, C.c_double, C.c_double, C.c_uint64, _f64p]),
}

_lib = None


class MjgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m mjolnir_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in {**SIGNATURES, **SYNTH_SIGNATURES}.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(ctx, code):
    if code != OK:
        msg = lib().mjg_last_error(ctx)
        raise MjgError(code, msg.decode() if msg else "")
    return code


def f64(a):
    return a.ctypes.data_as(_f64p) if a is not None else None


def i64(a):
    return a.ctypes.data_as(_i64p) if a is not None else None


def i32(a):
    return a.ctypes.data_as(_i32p) if a is not None else None
