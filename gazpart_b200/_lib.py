"""ctypes binding of ``libgazpart_b200.so`` (the C ABI in ``include/gazpart_gpu.h`` and
``include/gazpart_files.h``).

The shared library is built in-tree (``gazpart_b200/csrc/Makefile``).  Loading fails
loudly if it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgazpart_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
HEADERS = tuple(os.path.join(INCLUDE, h) for h in ("gazpart_gpu.h", "gazpart_files.h"))

GP_OK = 0
ERRORS = {
    1: "GP_ENAN_FORCE: NaN drag coefficient ('In Fluid force')",
    2: "GP_ENAN_TORQUE: NaN angular velocity in FLUID_TORQUE_ELLIPSOID",
    3: "GP_EENERGY: kinetic-energy balance violated in an impulse response",
    4: "GP_ESINGULAR: matrix is numerically singular",
    5: "GP_EPAIR_OVERFLOW: pair buffer full",
    6: "GP_EOUT_OF_GRID: particle outside the box grid or stencil range",
    7: "GP_ETIMEOUT: bounded loop or wait gave up",
    8: "GP_ECUDA: CUDA runtime error",
    9: "GP_EBADARG: invalid argument or unsupported configuration",
    10: "GP_ENOMEM: device allocation refused",
    11: "GP_EIO: file could not be opened, read or written, or is truncated",
    12: "GP_ERECORD: read past the end of a record, or inconsistent record markers",
    13: "GP_EEOF: end of file where a record was expected",
}
GP_EIO, GP_ERECORD, GP_EEOF = 11, 12, 13
PREC_FP64, PREC_MIXED = 0, 1
LAYOUT_INTERIOR, LAYOUT_REFERENCE = 0, 1
PHASES = ("gather", "integrate", "bin", "search", "contact", "response")   # GP_PHASE_*
TUNABLES = ("gather", "integrate", "bin", "search")   # GP_TUNE_*
COUNTERS = ("near", "candidates", "solves", "contacts", "colliding", "accepted", "evaluations", "max_evaluations")
NSTAT_PARTFLUID, NSTAT_COLLISION, STAT_MAX_GROUPS = 36, 8, 8   # GP_NSTAT_*, GP_STAT_MAX_GROUPS
# MEAN_PARTFLUID(1:36) in stat_partfluid.f90's order
STAT_PARTFLUID = ("rep", "cdrag", "clift", "fdrag_x", "fdrag_y", "fdrag_z", "flift_x", "flift_y", "flift_z",
                  "fdrag", "flift", "re_r", "ctpitch", "ctrotation", "tpitch_x", "tpitch_y", "tpitch_z",
                  "trot_x", "trot_y", "trot_z", "tpitch", "trot", "taupf", "gravity", "phi",
                  "axis_x", "axis_y", "axis_z", "invtaup", "up", "vp", "wp", "omegax", "omegay", "omegaz", "count")
# MEAN_PART_COL(1:8) in collision_interaction.f90's order
STAT_COLLISION = ("contacts", "collisions", "frequency", "depth", "depth_per_contact", "nvrel", "vrel", "angle")
GHOST_PERIODIC, GHOST_ZERO = 0, 1


class GPError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)}")


class GPParams(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("visc", C.c_double), ("rhof", C.c_double), ("dtime", C.c_double),
                ("gravity", C.c_double), ("ecp", C.c_double), ("mup", C.c_double),
                ("ecw", C.c_double), ("muw", C.c_double),
                ("periodicity", C.c_int32), ("wall_boundary", C.c_int32),
                ("interp_scheme", C.c_int32), ("frozen_flow", C.c_int32),
                ("precision", C.c_int32), ("store_fluid", C.c_int32),
                ("max_particles", C.c_int64)]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p
_ctx = C.c_void_p

# name -> argtypes (restype is int for all)
SIGNATURES = {
    "gp_ctx_create": [C.POINTER(GPParams), C.POINTER(_ctx)],
    "gp_ctx_destroy": [_ctx],
    "gp_status": [_ctx, _ip, _i64p],
    "gp_status_class": [_ctx, _ip],
    "gp_collision_counters": [_ctx, _i64p],
    "gp_set_class_groups": [_ctx, C.c_int32, C.c_int32, _ip],
    "gp_stat_partfluid": [_ctx, C.c_int32, _dp],
    "gp_collision_stats_enable": [_ctx, C.c_int32],
    "gp_collision_stats": [_ctx, C.c_int32, _dp, _i64p, C.c_int32],
    "gp_clear_status": [_ctx],
    "gp_sync": [_ctx],
    "gp_set_class": [_ctx, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double],
    "gp_set_field": [_ctx, C.c_int32, _vp, C.c_int32, C.c_int32, C.c_int32],
    "gp_upload_state": [_ctx, C.c_int64, C.POINTER(_vp), C.POINTER(_vp), C.c_int32],
    "gp_download_state": [_ctx, C.c_int64, C.POINTER(_vp), C.POINTER(_vp), C.c_int32],
    "gp_put_state": [_ctx, C.c_int64, C.POINTER(_vp), C.c_int32],
    "gp_step_host": [_ctx, C.c_int64, C.POINTER(_vp), C.POINTER(_vp)],
    "gp_upload_classes": [_ctx, C.c_int32, _i64p, C.POINTER(_vp), C.POINTER(_vp), C.c_int32],
    "gp_autotune": [_ctx, _ip],
    "gp_set_launch": [_ctx, _ip],
    "gp_set_pair_capacity": [_ctx, C.c_int64, C.c_int64],
    "gp_pair_capacity": [_ctx, _i64p, _i64p],
    "gp_add_field": [_ctx, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, _ip],
    "gp_set_field_slot": [_ctx, C.c_int32, C.c_int32, _vp, C.c_int32, C.c_int32, C.c_int32],
    "gp_add_class": [_ctx, C.c_int32, C.c_int64, C.POINTER(_vp), C.POINTER(_vp), C.c_int32, _ip],
    "gp_download_class": [_ctx, C.c_int32, C.POINTER(_vp), C.c_int32],
    "gp_remove_class": [_ctx, C.c_int32, C.POINTER(_vp), C.c_int32],
    "gp_class_count": [_ctx, C.c_int32, _i64p],
    "gp_serve": [_ctx, _vp, C.c_int32, C.c_double, C.c_double, _i64p],
    "gp_step_timed": [_ctx, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float), _ip],
    "gp_adv_particle_ellp": [_ctx, C.c_int32],
    "gp_collision": [_ctx, C.c_int32, C.c_double, _i64p, _i64p, _i64p],
    "gp_step": [_ctx, C.c_int32],
    "gp_collision_pairs": [_ctx, C.c_int64, _ip, _ip, _i64p],
    "gp_collision_box_connectivity": [_ctx, _ip, _ip, _ip, _ip, _dp],
    "gp_interp_lag3": [_ctx, C.c_int32, C.c_int64, _vp, _vp, _vp, _vp, C.c_int32],
    "gp_frozen_interp_lag3": [_ctx, _dp, _dp, _dp, C.c_int32, C.c_int32, C.c_int32, _dp, C.c_int64,
                              _dp, _dp, _dp, _dp],
    "gp_fluid_force_ellipsoid": [_ctx, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double, _dp, _dp, _dp],
    "gp_fluid_force_ellipsoid_batch": [_ctx, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int32],
    "gp_fluid_torque_ellipsoid": [_ctx, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, _dp,
                                  _dp, _dp, _dp, _dp, _dp],
    "gp_fluid_torque_ellipsoid_batch": [_ctx, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                        C.c_int32],
    "gp_quaternion_integration": [_ctx, _dp, C.c_double, C.c_double, C.c_double, C.c_double],
    "gp_quaternion_integration_batch": [_ctx, C.c_int64, _vp, _vp, C.c_double, C.c_int32],
    "gp_euler_integration": [_ctx, C.c_int32, C.c_int32, _dp, _dp, _dp],
    "gp_ellipsoid_contact_detection": [_ctx, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                       C.c_double, _dp, C.c_double, C.c_double, C.c_double, _dp, _ip,
                                       _dp, _dp, _dp],
    "gp_ellipsoid_contact_detection_batch": [_ctx, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                             C.c_int32],
    "gp_ellipsoid_contact_detection_batch_noalloc": [C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int32,
                                                     _vp],
    "gp_collision_response": [_ctx, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp, _dp],
    "gp_field_shape": [_ctx, C.c_int32, _ip],
    "gp_set_contact_tail": [_ctx, C.c_int32],
    "gp_get_contact_tail": [_ctx, _ip],
    "gp_set_contact_order": [_ctx, C.c_int32],
    "gp_get_contact_order": [_ctx, _ip],
    "gp_set_gather_staging": [_ctx, C.c_int32],
    "gp_get_gather_staging": [_ctx, _ip],
    "gp_dns_create": [C.POINTER(GPParams), C.c_int32, C.c_double, C.POINTER(_vp)],
    "gp_dns_destroy": [_vp],
    "gp_dns_set_velocity": [_vp, _vp, _vp, _vp, C.c_int32],
    "gp_dns_get_velocity": [_vp, _vp, _vp, _vp, C.c_int32],
    "gp_adv_fluid": [_vp, C.c_int32],
    "gp_dns_vorticity": [_vp, _vp, _vp, _vp, C.c_int32],
    "gp_dns_couple": [_vp, _ctx, C.c_int32, C.c_int32],
    # gazpart_files.h
    "gp_funf_open": [C.c_char_p, C.c_int32, C.POINTER(_vp)],
    "gp_funf_close": [_vp],
    "gp_funf_set_max_subrecord": [_vp, C.c_int64],
    "gp_funf_write": [_vp, _vp, C.c_int64],
    "gp_funf_record_size": [_vp, _i64p],
    "gp_funf_read": [_vp, _vp, C.c_int64],
    "gp_write_part_class": [C.c_char_p, C.c_int64, C.c_int32, _ip, _dp, _dp, C.c_double, C.POINTER(_vp)],
    "gp_read_part_class_header": [C.c_char_p, _i64p, _ip],
    "gp_read_part_class": [C.c_char_p, C.c_int64, C.c_int32, _ip, _dp, _dp, _dp, C.POINTER(_vp)],
    "gp_write_part_snapshot": [C.c_char_p, C.c_int64, C.POINTER(_vp)],
    "gp_read_part_snapshot": [C.c_char_p, C.c_int64, C.POINTER(_vp)],
    "gp_save_part_class": [_ctx, C.c_int32, C.c_char_p, C.c_int32, _ip, _dp, _dp, C.c_double, _ip],
    "gp_load_part_class": [_ctx, C.c_char_p, C.c_int32, _ip, _i64p],
}

_lib = None


def build(verbose: bool = False) -> None:
    """Compile the CUDA library in-tree for sm_100a."""
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), "-j4"]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with gazpart_b200._lib.build() "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        _lib = L
    return _lib


def check(rc: int, where: str) -> None:
    if rc != GP_OK:
        raise GPError(rc, where)


def exported_symbols():
    """Names declared in the C ABI headers (parsed from them)."""
    import re
    names = set()
    for h in HEADERS:
        names.update(re.findall(r"^int\s+(gp_\w+)\s*\(", open(h).read(), flags=re.M))
    return sorted(names)
