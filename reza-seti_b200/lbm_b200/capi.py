"""ctypes binding of the engine's C ABI (include/lbm_b200.h).

Loads the in-tree liblbm_b200.so built by ``make -C reza-seti_b200``. There is
no fallback: if the library is missing or cannot load, import fails loudly.
"""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "liblbm_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(PKG_DIR), "include", "lbm_b200.h")

LBM_OK = 0
LBM_ERR_ARGUMENT = -1
LBM_ERR_CUDA = -2
LBM_ERR_NO_DEVICE = -3
LBM_ERR_STATE = -4
LBM_ERR_NUMERIC = -5
FLUX_NOALLOC_MAX_NODES = 1048576  # LBM_FLUX_NOALLOC_MAX_NODES

STORAGE = {"f64": 0, "f32": 1, "f16": 2, "bf16": 3}
BC_REFERENCE, BC_PHYSICS = 0, 1
FLOW_CONSTANT, FLOW_PULSATILE, FLOW_HARMONIC = 0, 1, 2
FLAG_ZERO_SKIP, FLAG_NONFINITE = 1, 2
ADJOINT_OBJECTIVE = {"wss2": 0, "osi": 1}

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_f64p = ctypes.POINTER(ctypes.c_double)


class LbmDesc(ctypes.Structure):
    _fields_ = [
        ("lattice", ctypes.c_int32), ("storage", ctypes.c_int32), ("bc_mode", ctypes.c_int32),
        ("device", ctypes.c_int32), ("n_nodes", ctypes.c_int64), ("coords", _i32p),
        ("kind", _u8p), ("n_inlet", ctypes.c_int64), ("inlet", _i64p),
        ("inlet_normal", ctypes.c_double * 3), ("n_outlets", ctypes.c_int32),
        ("outlet_offsets", _i64p), ("outlet_nodes", _i64p), ("outlet_normals", _f64p),
        ("n_wall", ctypes.c_int64), ("wall", _i64p), ("n_nearwall", ctypes.c_int64),
        ("nearwall", _i64p), ("nearwall_normals", _f64p), ("tau", ctypes.c_double),
        ("dt", ctypes.c_double), ("spacing", ctypes.c_double),
    ]


class LbmAdjointDesc(ctypes.Structure):
    _fields_ = [
        ("n_steps", ctypes.c_int64), ("checkpoint_every", ctypes.c_int64), ("precision", ctypes.c_int32),
        ("n_target", ctypes.c_int32), ("target", _i64p), ("n_coeffs", ctypes.c_int32),
        ("basis", _f64p), ("coeffs", _f64p), ("objective", ctypes.c_int32),
    ]


class LbmAdjointResult(ctypes.Structure):
    _fields_ = [
        ("objective", ctypes.c_double), ("dJ_dtau", ctypes.c_double), ("grad_coeffs", _f64p),
        ("grad_inlet", _f64p), ("final_populations", _f64p), ("forward_ms", ctypes.c_double),
        ("reverse_ms", ctypes.c_double), ("steps_recomputed", ctypes.c_int64),
        ("device_bytes", ctypes.c_int64),
    ]


class LbmOpening(ctypes.Structure):
    _fields_ = [
        ("outlet", ctypes.c_int32), ("axis", ctypes.c_int32), ("coordinate", ctypes.c_double),
        ("normal", ctypes.c_double * 3), ("range", (ctypes.c_double * 2) * 3),
    ]


class LbmVoxelDesc(ctypes.Structure):
    _fields_ = [
        ("n_triangles", ctypes.c_int64), ("triangles", _f64p), ("grid_size", ctypes.c_double),
        ("n_openings", ctypes.c_int32), ("openings", ctypes.POINTER(LbmOpening)), ("device", ctypes.c_int32),
    ]


class LbmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("lbm error %d: %s" % (code, msg))
        self.code = code


_lib = None

# name -> (restype, argtypes); mirrors include/lbm_b200.h
PULSE_MAX_COEFFS = 16
CONFIG_MAX_OPENINGS = 64
CONFIG_MAX_EQUATIONS = 16
CONFIG_MAX_HARMONICS = 16


class LbmPulseDesc(ctypes.Structure):
    _fields_ = [
        ("period", ctypes.c_double), ("n_pieces", ctypes.c_int32), ("bounds", _f64p),
        ("n_coeffs", _i32p), ("coeffs", _f64p),
    ]


class LbmEquation(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 64), ("n_coeffs", ctypes.c_int32),
                ("coeffs", ctypes.c_double * PULSE_MAX_COEFFS)]


class LbmConfig(ctypes.Structure):
    _fields_ = [
        ("stl_file", ctypes.c_char * 1024), ("flow_type", ctypes.c_char * 64),
        ("dt", ctypes.c_double), ("rho", ctypes.c_double), ("nu_blood", ctypes.c_double), ("tau", ctypes.c_double),
        ("grid_size", ctypes.c_double), ("pressure", ctypes.c_double), ("cte_vel", ctypes.c_double),
        ("reynolds_number", ctypes.c_double), ("systole", ctypes.c_double), ("diastole", ctypes.c_double),
        ("number_of_outlets", ctypes.c_int32), ("max_iter", ctypes.c_int32), ("iter_to_write", ctypes.c_int32),
        ("num_cycle", ctypes.c_int32), ("n_inlets", ctypes.c_int32), ("n_outlets", ctypes.c_int32),
        ("openings", LbmOpening * CONFIG_MAX_OPENINGS), ("n_equations", ctypes.c_int32),
        ("equations", LbmEquation * CONFIG_MAX_EQUATIONS),
        ("flow", ctypes.c_int32), ("lattice", ctypes.c_int32), ("storage", ctypes.c_int32),
        ("bc_mode", ctypes.c_int32), ("device", ctypes.c_int32), ("period", ctypes.c_double),
        ("n_bounds", ctypes.c_int32), ("equation_bounds", ctypes.c_double * (CONFIG_MAX_EQUATIONS + 1)),
        ("outlet_density", ctypes.c_double), ("harmonic_period_steps", ctypes.c_double),
        ("n_harmonics", ctypes.c_int32), ("harmonic_amplitudes", ctypes.c_double * CONFIG_MAX_HARMONICS),
        ("harmonic_phases", ctypes.c_double * CONFIG_MAX_HARMONICS),
    ]


_E = ctypes.c_void_p
SIGNATURES = {
    "lbm_create": (ctypes.c_int, [ctypes.POINTER(LbmDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "lbm_destroy": (ctypes.c_int, [_E]),
    "lbm_set_stream": (ctypes.c_int, [_E, ctypes.c_void_p]),
    "lbm_set_flow": (ctypes.c_int, [_E, ctypes.c_int32, ctypes.c_double]),
    "lbm_set_inlet_profile": (ctypes.c_int, [_E, _f64p]),
    "lbm_set_waveform": (ctypes.c_int, [_E, ctypes.c_double, ctypes.c_int32, _f64p, _f64p]),
    "lbm_set_outlet_density": (ctypes.c_int, [_E, ctypes.c_double]),
    "lbm_step": (ctypes.c_int, [_E, ctypes.c_int64]),
    "lbm_set_observation": (ctypes.c_int, [_E, ctypes.c_int32]),
    "lbm_set_numeric_check": (ctypes.c_int, [_E, ctypes.c_int32]),
    "lbm_get_time": (ctypes.c_int, [_E, _i64p, _f64p]),
    "lbm_state_size": (ctypes.c_int, [_E, _i64p]),
    "lbm_get_state": (ctypes.c_int, [_E, ctypes.c_void_p, ctypes.c_int64]),
    "lbm_set_state": (ctypes.c_int, [_E, ctypes.c_void_p, ctypes.c_int64]),
    "lbm_get_populations": (ctypes.c_int, [_E, ctypes.c_void_p]),
    "lbm_set_populations": (ctypes.c_int, [_E, ctypes.c_void_p]),
    "lbm_get_macros": (ctypes.c_int, [_E, ctypes.c_void_p, ctypes.c_void_p]),
    "lbm_get_wss": (ctypes.c_int, [_E, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "lbm_get_osi_tawss": (ctypes.c_int, [_E, ctypes.c_void_p, ctypes.c_void_p]),
    "lbm_get_flux": (ctypes.c_int, [_E, ctypes.c_void_p, ctypes.c_void_p]),
    "lbm_flux_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p,
                                        ctypes.c_int64, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p,
                                        ctypes.c_void_p]),
    "lbm_get_flags": (ctypes.c_int, [_E, ctypes.POINTER(ctypes.c_uint32)]),
    "lbm_step_timed": (ctypes.c_int, [_E, ctypes.c_int64, _f64p, _f64p]),
    "lbm_get_info": (ctypes.c_int, [_E, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p]),
    "lbm_adjoint_run": (ctypes.c_int, [_E, ctypes.POINTER(LbmAdjointDesc), ctypes.c_int32,
                                       ctypes.POINTER(LbmAdjointResult)]),
    "lbm_stl_read_ascii": (ctypes.c_int, [ctypes.c_char_p, _i64p, ctypes.POINTER(_f64p)]),
    "lbm_free": (None, [ctypes.c_void_p]),
    "lbm_voxelise": (ctypes.c_int, [ctypes.POINTER(LbmVoxelDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "lbm_voxel_info": (ctypes.c_int, [_E, _i32p, _f64p, _f64p, _i64p, _i64p, _f64p]),
    "lbm_voxel_describe": (ctypes.c_int, [_E, ctypes.POINTER(LbmDesc)]),
    "lbm_voxel_destroy": (ctypes.c_int, [_E]),
    "lbm_write_surface_csv": (ctypes.c_int, [_E, ctypes.c_char_p, _f64p, ctypes.c_double, ctypes.c_int32]),
    "lbm_smooth_surface_csv": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_int32,
                                              ctypes.c_int32]),
    "lbm_write_vtu": (ctypes.c_int, [_E, ctypes.c_char_p, _i32p]),
    "lbm_set_pulsatile": (ctypes.c_int, [_E, ctypes.POINTER(LbmPulseDesc)]),
    "lbm_pulse_eval": (ctypes.c_int, [ctypes.POINTER(LbmPulseDesc), ctypes.c_double, _f64p]),
    "lbm_config_parse": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(LbmConfig)]),
    "lbm_halo_define": (ctypes.c_int, [_E, ctypes.c_int32, ctypes.c_int64, _i64p, _i32p]),
    "lbm_halo_pack": (ctypes.c_int, [_E, ctypes.c_int32, ctypes.c_void_p]),
    "lbm_halo_unpack": (ctypes.c_int, [_E, ctypes.c_int32, ctypes.c_void_p]),
    "lbm_get_phase": (ctypes.c_int, [_E, _i32p]),
    "lbm_last_error": (ctypes.c_char_p, [_E]),
}


def lib():
    """The loaded engine library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("liblbm_b200.so is not built: run `make -C reza-seti_b200`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code, handle=None):
    if code != LBM_OK:
        msg = lib().lbm_last_error(handle)
        raise LbmError(code, msg.decode() if msg else "")
    return code
