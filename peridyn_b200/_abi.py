"""ctypes binding of libperidyn_b200.so (include/peridyn_b200.h).

The library is required: there is no CPU fallback.  Importing this module
does not load it; the first call to :func:`lib` does, and raises
:class:`PDError` when the shared object is missing or no CUDA device is
usable for a compute call.
"""
import ctypes
import os
import re

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libperidyn_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "peridyn_b200.h")

PD_OK = 0
PD_ERR_ARG = 1
PD_ERR_OOM = 2
PD_ERR_FAMILY_OVERFLOW = 3
PD_ERR_NAN = 4
PD_ERR_CUDA = 5
PD_ERR_TIMEOUT = 6
PD_ERR_STATE = 7
PD_ERR_NO_DEVICE = 8
PD_ERR_UNSUPPORTED = 9

PD_MAT_BOND_BASED = 0
PD_MAT_ORDINARY_STATE_BASED = 1
PD_MAT_SKIP = 2
PD_MAT_ELASTO_PLASTIC = 3

PD_PREC_FP64_SERIAL = 0
PD_PREC_FP64 = 1
PD_PREC_FP32C = 2
PRECISIONS = {"fp64_serial": PD_PREC_FP64_SERIAL, "fp64": PD_PREC_FP64, "fp32c": PD_PREC_FP32C}

PD_BC_FIX = 0
PD_BC_TOFRO = 1
PD_BC_DELTA_SCALE = 2
PD_BC_SCALE_FIX_WAIT = 3
PD_BC_CONTAINER = 4

PD_CONTACT_12 = 0
PD_CONTACT_11 = 1
PD_CONTACT_11_ORDERED = 2

c_dp = ctypes.POINTER(ctypes.c_double)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_vp = ctypes.c_void_p


class PDError(RuntimeError):
    """A pd_status other than PD_OK, with the library's message."""

    def __init__(self, status, message):
        super().__init__(f"peridyn_b200 error {status}: {message}")
        self.status = status
        self.message = message


class MaterialDesc(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("ntypes", ctypes.c_int32),
        ("type_start", ctypes.c_int64),
        ("bond_stiffness", c_dp),
        ("bulk_modulus", c_dp),
        ("shear_modulus", c_dp),
        ("critical_stretch", c_dp),
        ("density", c_dp),
        ("horizon", ctypes.c_double),
        ("particle_size", ctypes.c_double),
        ("max_neigh", ctypes.c_int64),
        ("plastic_psi", c_dp),
    ]


class JobInfo(ctypes.Structure):
    _fields_ = [
        ("state", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("steps_done", ctypes.c_int64),
        ("particles", ctypes.c_int64),
        ("footprint_bytes", ctypes.c_int64),
        ("bond_updates", ctypes.c_int64),
        ("queue_ms", ctypes.c_double),
        ("latency_ms", ctypes.c_double),
    ]


JOB_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}

_SIGNATURES = {
    "pd_abi_version": (ctypes.c_int, []),
    "pd_status_string": (ctypes.c_char_p, [ctypes.c_int32]),
    "pd_last_error": (ctypes.c_char_p, []),
    "pd_device_count": (ctypes.c_int32, [c_i32p]),
    "pd_env_create": (ctypes.c_int32, [ctypes.POINTER(c_vp), ctypes.c_int32, ctypes.c_int32, ctypes.c_double]),
    "pd_env_destroy": (ctypes.c_int32, [c_vp]),
    "pd_env_add_block": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_dp, c_dp, c_dp, c_dp, c_i64p,
                                          ctypes.POINTER(MaterialDesc), c_i64p]),
    "pd_env_set_family": (ctypes.c_int32, [c_vp, ctypes.c_int64, ctypes.c_int64, c_i64p, c_u8p]),
    "pd_env_add_scaled_bc": (ctypes.c_int32, [c_vp, ctypes.c_int32, c_u8p, c_u8p, c_dp, c_dp, ctypes.c_int64, c_u8p,
                                              ctypes.c_int32, c_i64p]),
    "pd_env_add_container_bc": (ctypes.c_int32, [c_vp, c_u8p, c_u8p, c_dp, ctypes.c_int32, c_i64p]),
    "pd_env_add_contact": (ctypes.c_int32, [c_vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                            c_i64p]),
    "pd_env_add_bc": (ctypes.c_int32, [c_vp, ctypes.c_int32, c_u8p, c_u8p, c_dp, ctypes.c_double, ctypes.c_int64,
                                       ctypes.c_int32, c_i64p]),
    "pd_env_finalize": (ctypes.c_int32, [c_vp]),
    "pd_env_num_particles": (ctypes.c_int32, [c_vp, c_i64p]),
    "pd_env_num_bonds": (ctypes.c_int32, [c_vp, c_i64p]),
    "pd_env_family_rows": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_i64p]),
    "pd_env_get_family": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_i64p, c_u8p]),
    "pd_env_get_weighted_volume": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_dp]),
    "pd_env_get_theta": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_dp]),
    "pd_env_get_plastic_strain": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_dp]),
    "pd_env_get_state": (ctypes.c_int32, [c_vp, c_dp, c_dp, c_dp, c_dp]),
    "pd_env_set_state": (ctypes.c_int32, [c_vp, c_dp, c_dp, c_dp]),
    "pd_env_get_mass": (ctypes.c_int32, [c_vp, c_dp, c_dp, c_dp]),
    "pd_env_get_time_step": (ctypes.c_int32, [c_vp, c_i64p]),
    "pd_env_set_time_step": (ctypes.c_int32, [c_vp, ctypes.c_int64]),
    "pd_env_reset_bonds": (ctypes.c_int32, [c_vp]),
    "pd_env_reset_deformed": (ctypes.c_int32, [c_vp]),
    "pd_env_apply_bc_at0": (ctypes.c_int32, [c_vp]),
    "pd_env_update_acc": (ctypes.c_int32, [c_vp]),
    "pd_env_vv_steps": (ctypes.c_int32, [c_vp, ctypes.c_int64]),
    "pd_env_qsdrag": (ctypes.c_int32, [c_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_double,
                                       ctypes.c_double, c_i64p]),
    "pd_env_update_neighs": (ctypes.c_int32, [c_vp, ctypes.c_int64]),
    "pd_env_get_contact_neighs": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_i64p, c_i64p]),
    "pd_env_damage": (ctypes.c_int32, [c_vp, c_dp]),
    "pd_env_diagnostics": (ctypes.c_int32, [c_vp, c_dp]),
    "pd_env_deformed": (ctypes.c_int32, [c_vp, c_u8p]),
    "pd_env_check_finite": (ctypes.c_int32, [c_vp]),
    "pd_env_layout": (ctypes.c_int32, [c_vp, c_i64p]),
    "pd_env_layout_stats": (ctypes.c_int32, [c_vp, c_i64p, ctypes.c_int64]),
    "pd_env_pack_halo": (ctypes.c_int32, [c_vp, c_vp, ctypes.c_int64, c_vp]),
    "pd_env_set_deformed": (ctypes.c_int32, [c_vp, c_vp, ctypes.c_int32]),
    "pd_env_intact0": (ctypes.c_int32, [c_vp, c_i64p]),
    "pd_env_unpack_halo": (ctypes.c_int32, [c_vp, c_vp, ctypes.c_int64, c_vp]),
    "pd_force_density_device": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_vp, c_vp, c_vp]),
    "pd_force_density_device_static": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_vp, c_vp, c_vp]),
    "pd_env_stream": (ctypes.c_int32, [c_vp, ctypes.POINTER(c_vp)]),
    "pd_kernel_launches": (ctypes.c_int32, [c_i64p]),
    "pd_pipe_peaks": (ctypes.c_int32, [ctypes.c_int32, c_dp]),
    "pd_env_vv_steps_async": (ctypes.c_int32, [c_vp, ctypes.c_int64]),
    "pd_env_profile": (ctypes.c_int32, [c_vp, ctypes.c_int32]),
    "pd_env_profile_read": (ctypes.c_int32, [c_vp, c_dp, c_i64p]),
    "pd_env_stage_state": (ctypes.c_int32, [c_vp, ctypes.c_int32]),
    "pd_env_stage_read": (ctypes.c_int32, [c_vp, ctypes.c_int32, c_dp, c_dp, c_dp, c_dp, c_i64p]),
    "pd_env_set_kernel_shape": (ctypes.c_int32, [c_vp, ctypes.c_int32, ctypes.c_int32]),
    "pd_env_kernel_shape": (ctypes.c_int32, [c_vp, c_i32p, c_i32p]),
    "pd_env_set_record_staging": (ctypes.c_int32, [c_vp, ctypes.c_int32]),
    "pd_env_record_staging": (ctypes.c_int32, [c_vp, c_i32p, c_i64p, c_i64p]),
    "pd_server_create": (ctypes.c_int32, [ctypes.POINTER(c_vp), ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                          ctypes.c_int64]),
    "pd_server_submit": (ctypes.c_int32, [c_vp, c_vp, ctypes.c_int64, c_i64p]),
    "pd_server_poll": (ctypes.c_int32, [c_vp, ctypes.c_int64, ctypes.c_void_p]),
    "pd_server_wait": (ctypes.c_int32, [c_vp, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p]),
    "pd_server_result": (ctypes.c_int32, [c_vp, ctypes.c_int64, c_dp, c_dp, c_dp]),
    "pd_server_cancel": (ctypes.c_int32, [c_vp, ctypes.c_int64]),
    "pd_server_destroy": (ctypes.c_int32, [c_vp]),
}

_lib = None


def header_symbols(path=HEADER_PATH):
    """Names of every function the public header declares."""
    text = open(path).read()
    return sorted(set(re.findall(r"^PD_API\s+[\w\s\*]*?\b(pd_\w+)\s*\(", text, flags=re.M)))


def lib():
    """Load the shared library (once) and declare its signatures."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PDError(PD_ERR_NO_DEVICE, f"{LIB_PATH} is not built; run `python -m peridyn_b200.build`")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status):
    if status != PD_OK:
        msg = lib().pd_last_error()
        raise PDError(status, msg.decode() if msg else "")


def dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous)
    return a.ctypes.data_as(c_dp)


def i64ptr(a):
    if a is None:
        return None
    assert a.dtype == np.int64
    return a.ctypes.data_as(c_i64p)


def u8ptr(a):
    if a is None:
        return None
    assert a.dtype == np.uint8
    return a.ctypes.data_as(c_u8p)


def device_count():
    n = ctypes.c_int32(0)
    check(lib().pd_device_count(ctypes.byref(n)))
    return int(n.value)


def kernel_launches():
    n = ctypes.c_int64(0)
    check(lib().pd_kernel_launches(ctypes.byref(n)))
    return int(n.value)


PIPE_KEYS = ("ffma_lane_ops_per_s", "ffma2_lane_fmas_per_s", "sqrt_approx_lane_ops_per_s",
             "rcp_approx_lane_ops_per_s", "ffma_lop3_warp_instr_per_s")


def pipe_peaks(device=0):
    """Measured pipe rates of a GPU (pd_pipe_peaks) as a dict keyed by
    PIPE_KEYS."""
    out = np.zeros(5)
    check(lib().pd_pipe_peaks(int(device), dptr(out)))
    return dict(zip(PIPE_KEYS, (float(x) for x in out)))
