"""TEST ORACLE ONLY: ctypes wrapper of oracle/liboracle.so, the plain-C restatement of the reference algorithm
(oracle/sph_oracle.c). Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU arm."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
KTABLE = 20000
_lib = None


class OrcBox(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3), ("periodic", C.c_int * 3)]


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise FileNotFoundError(f"{LIB} not built (make -C oracle)")
    lib = C.CDLL(LIB)
    P, S, U, D = C.c_void_p, C.c_size_t, C.c_uint, C.c_double
    B = C.POINTER(OrcBox)
    sig = {
        "orc_hilbert": (C.c_uint64, [U, U, U]),
        "orc_hilbert_decode": (None, [C.c_uint64, P, P, P]),
        "orc_sfc_keys": (None, [S, P, P, P, B, P]),
        "orc_sort_by_key": (None, [S, P, P]),
        "orc_compute_octree": (S, [S, P, U, P, P, S]),
        "orc_kernel_tables": (D, [D, P, P]),
        "orc_sphynx_3d_k": (D, [D]),
        "orc_find_neighbors": (None, [S, P, P, P, P, B, U, U, C.c_int, P, P]),
        "orc_xmass": (D, [U, D, B, P, U, P, P, P, P, P, P]),
        "orc_ve_def_gradh": (None, [U, D, B, P, U, P, P, P, P, P, P, P, P, P, P]),
        "orc_iad": (None, [U, D, B, P, U, P, P, P, P, P, P, P, P]),
        "orc_divv_curlv": (None, [U, D, B, P, U, P, P, P, P, P, P, P, P, P, P, P, P, P, P]),
        "orc_av_switches": (D, [U, D, B, P, U, P, P, P, P, P, P, P, P, P, P, P, P, P, D, D, D, D, D]),
        "orc_momentum_energy": (None, [U, C.c_int, D, B, P, U, P, P, P, P, P, P, P, P, P, P, P, D, D, D, P, P, P, P,
                                       P, P]),
        "orc_sim_create": (P, [S, P, P, P, C.c_int, P]),
        "orc_sim_destroy": (None, [P]),
        "orc_sim_sync": (None, [P]),
        "orc_sim_compute_forces": (C.c_int, [P]),
        "orc_sim_integrate": (C.c_int, [P]),
        "orc_sim_set_av_clean": (None, [P, C.c_int]),
        "orc_sim_size": (S, [P]),
        "orc_sim_get": (C.c_int, [P, C.c_char_p, P]),
        "orc_sim_keys": (None, [P, P]),
        "orc_sim_neighbors": (None, [P, P]),
        "orc_sim_scalars": (None, [P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def box(limits, periodic) -> OrcBox:
    b = OrcBox()
    for k in range(3):
        b.lo[k] = limits[2 * k]
        b.hi[k] = limits[2 * k + 1]
        b.periodic[k] = int(bool(periodic))
    return b


def sfc_keys(x, y, z, limits, periodic):
    lib = load()
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    keys = np.zeros(x.size, dtype=np.uint64)
    b = box(limits, periodic)
    lib.orc_sfc_keys(x.size, ptr(x), ptr(y), ptr(z), C.byref(b), ptr(keys))
    return keys


def sort_by_key(keys):
    lib = load()
    k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    perm = np.arange(k.size, dtype=np.uint32)
    lib.orc_sort_by_key(k.size, ptr(k), ptr(perm))
    return k, perm


def compute_octree(sorted_keys, bucket):
    lib = load()
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint64)
    cap = 8 * (k.size // max(bucket, 1) + 8) * 8 + 64
    leaves = np.empty(cap + 1, dtype=np.uint64)
    counts = np.empty(cap, dtype=np.uint32)
    nl = lib.orc_compute_octree(k.size, ptr(k), bucket, ptr(leaves), ptr(counts), cap)
    return leaves[:nl + 1].copy(), counts[:nl].copy()


def tables(sinc_index=6.0):
    lib = load()
    wh = np.empty(KTABLE)
    whd = np.empty(KTABLE)
    K = lib.orc_kernel_tables(sinc_index, ptr(wh), ptr(whd))
    return K, wh, whd


def find_neighbors(x, y, z, h, limits, periodic, ng0, ngmax, iterate):
    lib = load()
    n = x.size
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
    hh = np.ascontiguousarray(h, dtype=np.float64).copy()
    nbr = np.zeros((n, ngmax), dtype=np.uint32)
    nc = np.zeros(n, dtype=np.uint32)
    b = box(limits, periodic)
    lib.orc_find_neighbors(n, *[ptr(a) for a in arrs], ptr(hh), C.byref(b), ng0, ngmax, int(iterate), ptr(nbr),
                           ptr(nc))
    return nbr, nc, hh


SCALAR_NAMES = ("minDt", "minDt_m1", "minDtCourant", "minDtRho", "ttot", "etot", "ecin", "eint", "linmom", "angmom",
                "totalNeighbors", "iteration", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


class OracleSim:
    """Whole hydro step of the restated oracle (FP64, one rank)."""

    def __init__(self, ic: dict):
        from sphexa_b200.ic import CONSERVED_FIELDS
        self.lib = load()
        p = ic["params"]
        self._keep = [np.ascontiguousarray(ic[f], dtype=np.float64) for f in CONSERVED_FIELDS]
        tbl = (C.c_void_p * len(self._keep))(*[a.ctypes.data for a in self._keep])
        ids = np.ascontiguousarray(ic["id"], dtype=np.uint64)
        lim = np.array(ic["box"], dtype=np.float64)
        prm = np.array([p["ng0"], p["ngmax"], p["gamma"], p["mui"], p["minDt"], p["minDt_m1"], p["Kcour"], p["Krho"],
                        p["alphamin"], p["alphamax"], p["decay_constant"]], dtype=np.float64)
        self.ngmax = int(p["ngmax"])
        self.h = self.lib.orc_sim_create(ids.size, tbl, ptr(ids), ptr(lim), int(bool(ic["periodic"])), ptr(prm))
        self.n = ids.size
        # HydroVeProp<avClean = true>: IAD keeps the velocity gradients, MomentumEnergy corrects r.v with them
        self.lib.orc_sim_set_av_clean(self.h, int(bool(p.get("avClean", False))))
        self.lib.orc_sim_sync(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_sim_destroy(self.h)
            self.h = None

    def compute_forces(self):
        self.lib.orc_sim_compute_forces(self.h)

    def integrate(self):
        return self.lib.orc_sim_integrate(self.h)

    def step(self):
        self.compute_forces()
        return self.integrate()

    def get(self, name):
        out = np.empty(self.n)
        if self.lib.orc_sim_get(self.h, name.encode(), ptr(out)):
            raise KeyError(name)
        return out.view(np.uint64) if name == "id" else out

    def keys(self):
        out = np.empty(self.n, dtype=np.uint64)
        self.lib.orc_sim_keys(self.h, ptr(out))
        return out

    def neighbors(self):
        out = np.empty((self.n, self.ngmax), dtype=np.uint32)
        self.lib.orc_sim_neighbors(self.h, ptr(out))
        return out

    def scalars(self):
        out = np.empty(len(SCALAR_NAMES))
        self.lib.orc_sim_scalars(self.h, ptr(out))
        return dict(zip(SCALAR_NAMES, out.tolist()))
