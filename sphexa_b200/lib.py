"""ctypes binding of libsphb200.so (the C ABI declared in include/sphb200.h).

The library is the only compute path: importing this module fails loudly if it has not been built
(python -m sphexa_b200.build), and every call checks its status code.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsphb200.so")

SPHB_OK = 0
SPHB_ERR_ARG, SPHB_ERR_CUDA, SPHB_ERR_CAPACITY, SPHB_ERR_NOT_CONVERGED, SPHB_ERR_STATE = 1, 2, 3, 4, 5
SPHB_ERR_TIMEOUT = 6
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "capacity exhausted", 4: "smoothing length not converged",
          5: "call out of order", 6: "bounded device wait gave up"}
SPHB_FP64 = 0
SPHB_MIXED = 1
SPHB_F32, SPHB_F64, SPHB_U32, SPHB_U64 = 1, 2, 3, 4


class SphbError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {ERRORS.get(code, code)} (status {code})")
        self.code = code


class Box(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3), ("periodic", C.c_int * 3)]


class Field(C.Structure):
    """sphb_field: one caller array of a particle field, by the reference's field name"""
    _fields_ = [("name", C.c_char_p), ("data", C.c_void_p), ("dtype", C.c_int)]


def dtype_code(a) -> int:
    """SPHB_F32 ... of a numpy array or torch tensor"""
    name = str(a.dtype).replace("torch.", "")
    codes = {"float32": SPHB_F32, "float64": SPHB_F64, "uint32": SPHB_U32, "int32": SPHB_U32,
             "uint64": SPHB_U64, "int64": SPHB_U64}
    if name not in codes:
        raise TypeError(f"no sphb element type for {a.dtype}")
    return codes[name]


def make_fields(arrays: dict):
    """A ctypes array of sphb_field from {name: numpy array or torch tensor}; the arrays must stay alive."""
    tbl = (Field * len(arrays))()
    for q, (name, a) in enumerate(arrays.items()):
        tbl[q].name = name.encode()
        tbl[q].data = ptr(a).value
        tbl[q].dtype = dtype_code(a)
    return tbl


class BdtTimestep(C.Structure):
    """sphb_bdt_timestep: sph::Timestep of the block time-step propagator"""
    _fields_ = [("next_dt", C.c_float), ("elapsed_dt", C.c_float), ("total_dt", C.c_float), ("num_rungs", C.c_int),
                ("substep", C.c_int), ("rung_ranges", C.c_uint32 * 5), ("dt_m1", C.c_float * 4),
                ("dt_drift", C.c_float * 4), ("num_active", C.c_uint32)]


class Params(C.Structure):
    _fields_ = [("ng0", C.c_uint32), ("ngmax", C.c_uint32), ("gamma", C.c_double), ("mui", C.c_double),
                ("Kcour", C.c_double), ("Krho", C.c_double), ("alphamin", C.c_double), ("alphamax", C.c_double),
                ("decay_constant", C.c_double), ("sinc_index", C.c_double), ("minDt", C.c_double),
                ("minDt_m1", C.c_double), ("precision", C.c_int), ("bucket_focus", C.c_uint32),
                ("av_clean", C.c_int), ("nb_skin", C.c_double)]


#: every extern "C" symbol of include/sphb200.h
EXPORTED = ("sphb_default_params", "sphb_version", "sphb_compute_sfc_keys", "sphb_sort_by_key_scratch_bytes",
            "sphb_sort_by_key", "sphb_gather8", "sphb_compute_octree", "sphb_sim_create", "sphb_sim_destroy",
            "sphb_sim_upload", "sphb_sim_initial_sync", "sphb_sim_compute_forces", "sphb_sim_integrate",
            "sphb_sim_step", "sphb_sim_bdt_enable", "sphb_sim_bdt_step", "sphb_sim_bdt_timestep", "sphb_sim_sync", "sphb_sim_find_neighbors", "sphb_sim_xmass",
            "sphb_sim_ve_def_gradh_eos", "sphb_sim_iad_divv_curlv", "sphb_sim_av_switches", "sphb_sim_momentum_energy",
            "sphb_sim_conserved", "sphb_sim_size", "sphb_sim_get_field", "sphb_sim_set_field", "sphb_sim_scalars",
            "sphb_sim_tree", "sphb_sim_neighbors", "sphb_sim_stage_times", "sphb_sim_kernel_launches",
            "sphb_sim_search_stats",
            "sphb_sim_stream", "sphb_sim_load_state", "sphb_sim_store_state", "sphb_probe_fma_peak",
            "sphb_sort_by_key_static", "sphb_sort_by_key_static_max", "sphb_sim_set_fixed_dt",
            "sphb_sim_set_params", "sphb_sim_step_vjp", "sphb_sort_by_key_nearly_sorted", "sphb_sim_tape_reserve", "sphb_sim_step_record",
            "sphb_sim_step_vjp_recorded", "sphb_ensemble_create", "sphb_ensemble_destroy",
            "sphb_ensemble_upload", "sphb_ensemble_initial_sync", "sphb_ensemble_rebuild_trees",
            "sphb_ensemble_set_threads", "sphb_ensemble_autotune", "sphb_ensemble_step", "sphb_ensemble_size", "sphb_ensemble_search_stats",
            "sphb_ensemble_stage_times",
            "sphb_ensemble_get_field", "sphb_ensemble_scalars", "sphb_ensemble_stream",
            "sphb_sim_upload_fields", "sphb_sim_load_fields", "sphb_sim_store_fields",
            "sphb_sim_step_fields", "sphb_sim_bind_fields",
            "sphb_dataset_xmass", "sphb_dataset_ve_def_gradh", "sphb_ideal_gas_eos",
            "sphb_dataset_iad_divv_curlv", "sphb_dataset_av_switches", "sphb_dataset_momentum_energy",
            "sphb_dataset_positions", "sphb_dataset_update_h", "sphb_compute_group_splits",
            "sphb_build_octree", "sphb_leaf_counts", "sphb_rebalance_tree", "sphb_find_halos")

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m sphexa_b200.build`")
    lib = C.CDLL(LIB_PATH)
    P, S = C.c_void_p, C.c_size_t
    sig = {
        "sphb_default_params": (None, [C.POINTER(Params)]),
        "sphb_version": (C.c_char_p, []),
        "sphb_compute_sfc_keys": (C.c_int, [P, P, P, P, S, C.POINTER(Box), P]),
        "sphb_sort_by_key_scratch_bytes": (S, [S]),
        "sphb_sort_by_key": (C.c_int, [P, P, S, C.c_int, P, S, P]),
        "sphb_gather8": (C.c_int, [P, S, C.c_int, P, P, P]),
        "sphb_compute_octree": (C.c_int, [P, S, C.c_uint, P, P, S, C.POINTER(S), P]),
        "sphb_sim_create": (C.c_int, [C.POINTER(P), S, C.POINTER(Box), C.POINTER(Params)]),
        "sphb_sim_destroy": (C.c_int, [P]),
        "sphb_sim_upload": (C.c_int, [P, P, P, C.c_int]),
        "sphb_sim_initial_sync": (C.c_int, [P]),
        "sphb_sim_compute_forces": (C.c_int, [P]),
        "sphb_sim_integrate": (C.c_int, [P]),
        "sphb_sim_step": (C.c_int, [P]),
        "sphb_sim_bdt_enable": (C.c_int, [P, C.c_double]),
        "sphb_sim_bdt_step": (C.c_int, [P]),
        "sphb_sim_bdt_timestep": (C.c_int, [P, C.POINTER(BdtTimestep)]),
        "sphb_sim_sync": (C.c_int, [P]),
        "sphb_sim_find_neighbors": (C.c_int, [P]),
        "sphb_sim_xmass": (C.c_int, [P]),
        "sphb_sim_ve_def_gradh_eos": (C.c_int, [P]),
        "sphb_sim_iad_divv_curlv": (C.c_int, [P]),
        "sphb_sim_av_switches": (C.c_int, [P]),
        "sphb_sim_momentum_energy": (C.c_int, [P, P]),
        "sphb_sim_conserved": (C.c_int, [P, P]),
        "sphb_sim_size": (S, [P]),
        "sphb_sim_get_field": (C.c_int, [P, C.c_char_p, P, C.c_int]),
        "sphb_sim_set_field": (C.c_int, [P, C.c_char_p, P, C.c_int]),
        "sphb_sim_scalars": (C.c_int, [P, P]),
        "sphb_sim_tree": (C.c_int, [P, C.POINTER(S), P, P, P]),
        "sphb_sim_neighbors": (C.c_int, [P, P]),
        "sphb_sim_stage_times": (C.c_int, [P, P]),
        "sphb_sim_kernel_launches": (C.c_uint64, [P]),
        "sphb_sim_search_stats": (C.c_int, [P, P]),
        "sphb_sim_stream": (C.c_void_p, [P]),
        "sphb_sim_load_state": (C.c_int, [P, P, P, C.c_int]),
        "sphb_sim_store_state": (C.c_int, [P, P, P, C.c_int]),
        "sphb_probe_fma_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
        "sphb_sort_by_key_static": (C.c_int, [P, P, S, C.c_int, P]),
        "sphb_sort_by_key_static_max": (S, []),
        "sphb_sim_set_fixed_dt": (C.c_int, [P, C.c_double]),
        "sphb_sim_set_params": (C.c_int, [P, C.POINTER(Params)]),
        "sphb_sim_step_vjp": (C.c_int, [P, P, P, C.POINTER(C.c_double)]),
        "sphb_sort_by_key_nearly_sorted": (C.c_int, [P, P, S, P, S, C.POINTER(C.c_int), P]),
        "sphb_sim_tape_reserve": (C.c_int, [P, C.c_int]),
        "sphb_sim_step_record": (C.c_int, [P, C.c_int]),
        "sphb_sim_step_vjp_recorded": (C.c_int, [P, C.c_int, P, P, C.POINTER(C.c_double)]),
        "sphb_ensemble_create": (C.c_int, [C.POINTER(P), C.c_int, P, C.POINTER(Box), P]),
        "sphb_ensemble_destroy": (C.c_int, [P]),
        "sphb_ensemble_upload": (C.c_int, [P, C.c_int, P, P, C.c_int]),
        "sphb_ensemble_initial_sync": (C.c_int, [P]),
        "sphb_ensemble_rebuild_trees": (C.c_int, [P]),
        "sphb_ensemble_set_threads": (C.c_int, [P, P]),
        "sphb_ensemble_autotune": (C.c_int, [P, P]),
        "sphb_ensemble_step": (C.c_int, [P, C.c_int, C.c_int]),
        "sphb_ensemble_size": (S, [P, C.c_int]),
        "sphb_ensemble_search_stats": (C.c_int, [P, P]),
        "sphb_ensemble_stage_times": (C.c_int, [P, P]),
        "sphb_ensemble_get_field": (C.c_int, [P, C.c_int, C.c_char_p, P]),
        "sphb_ensemble_scalars": (C.c_int, [P, C.c_int, P]),
        "sphb_ensemble_stream": (C.c_void_p, [P]),
        "sphb_sim_upload_fields": (C.c_int, [P, P, C.c_int, C.c_int]),
        "sphb_sim_load_fields": (C.c_int, [P, P, C.c_int, C.c_int]),
        "sphb_sim_store_fields": (C.c_int, [P, P, C.c_int, C.c_int]),
        "sphb_sim_step_fields": (C.c_int, [P, P, C.c_int, P, C.c_int]),
        "sphb_sim_bind_fields": (C.c_int, [P, P, C.c_int]),
        "sphb_dataset_xmass": (C.c_int, [P, S, S, C.POINTER(Box)]),
        "sphb_dataset_ve_def_gradh": (C.c_int, [P, S, S, C.POINTER(Box)]),
        "sphb_ideal_gas_eos": (C.c_int, [S, S, C.c_double, C.c_double, P, C.c_int, P]),
        "sphb_dataset_iad_divv_curlv": (C.c_int, [P, S, S, C.POINTER(Box)]),
        "sphb_dataset_av_switches": (C.c_int, [P, S, S, C.POINTER(Box), C.c_double]),
        "sphb_dataset_momentum_energy": (C.c_int, [P, S, S, C.POINTER(Box), C.POINTER(C.c_float)]),
        "sphb_dataset_positions": (C.c_int, [P, S, S, C.c_double, C.c_double, C.POINTER(Box)]),
        "sphb_dataset_update_h": (C.c_int, [P, S, S, C.c_uint]),
        "sphb_compute_group_splits": (C.c_int, [S, S, P, P, P, P, C.c_int, P, S, P, C.POINTER(Box), C.c_uint,
                                                C.c_float, P, S, C.POINTER(S), P]),
        "sphb_build_octree": (C.c_int, [P, S, P, P, P, P, P, P, P]),
        "sphb_leaf_counts": (C.c_int, [P, S, P, S, P, P]),
        "sphb_rebalance_tree": (C.c_int, [P, S, P, C.c_uint, P, S, C.POINTER(S), C.POINTER(C.c_int), P]),
        "sphb_find_halos": (C.c_int, [P, S, P, P, P, P, C.c_int, P, S, S, C.POINTER(Box), C.c_float, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str):
    if rc != SPHB_OK:
        raise SphbError(rc, what)


def ptr(a) -> C.c_void_p:
    """Address of a numpy array or torch tensor."""
    if isinstance(a, np.ndarray):
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())


def make_box(limits, periodic) -> Box:
    b = Box()
    for k in range(3):
        b.lo[k] = float(limits[2 * k])
        b.hi[k] = float(limits[2 * k + 1])
        b.periodic[k] = int(bool(periodic[k] if hasattr(periodic, "__len__") else periodic))
    return b


def make_params(p: dict, precision: int = SPHB_FP64, bucket: int = 64) -> Params:
    lib = load()
    prm = Params()
    lib.sphb_default_params(C.byref(prm))
    prm.ng0 = int(p["ng0"])
    prm.ngmax = int(p["ngmax"])
    prm.gamma = float(p["gamma"])
    prm.mui = float(p["mui"])
    prm.Kcour = float(p["Kcour"])
    prm.Krho = float(p["Krho"])
    prm.alphamin = float(p["alphamin"])
    prm.alphamax = float(p["alphamax"])
    prm.decay_constant = float(p["decay_constant"])
    prm.sinc_index = float(p.get("sincIndex", 6.0))
    prm.minDt = float(p["minDt"])
    prm.minDt_m1 = float(p["minDt_m1"])
    prm.precision = int(precision)
    prm.bucket_focus = int(bucket)
    prm.av_clean = int(bool(p.get("avClean", False)))
    if "nbSkin" in p:
        prm.nb_skin = float(p["nbSkin"])
    return prm
