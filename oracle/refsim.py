"""TEST ORACLE ONLY: ctypes wrapper of oracle/_ref/libsphref*.so (the reference's own CPU hydro step, built from the
reference sources by oracle/Makefile). Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU arms.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KTABLE = 20000

_LIBS = {}


#: x86-64 feature levels of the timed builds, widest first, with the CPU flags each needs
TIMED_ISAS = (("v4", ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl", "avx2", "fma", "bmi2")),
              ("v3", ("avx2", "fma", "bmi2", "movbe")))


def host_cpu() -> tuple[str, set]:
    """Model name and feature flags of this host's CPU (from /proc/cpuinfo)."""
    model, flags = "unknown", set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and model == "unknown":
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return model, flags


def timed_isa() -> str | None:
    """The widest x86-64 level whose timed build exists and that this host's CPU supports."""
    _, flags = host_cpu()
    for isa, need in TIMED_ISAS:
        if all(f in flags for f in need) and os.path.exists(os.path.join(HERE, "_ref", f"libsphref_timed_{isa}.so")):
            return isa
    return None


def ref_lib_path(mixed: bool | str = False) -> str:
    """mixed=False: the FP64 parity build; True: the reference-default-types parity build; "timed": the
    reference-default-types build with the compiler's default FP contraction for this host's widest ISA level (the
    build the CPU baselines time), else the parity build of the same types."""
    if mixed == "timed":
        isa = timed_isa()
        return os.path.join(HERE, "_ref", f"libsphref_timed_{isa}.so" if isa else "libsphref_mixed.so")
    return os.path.join(HERE, "_ref", "libsphref_mixed.so" if mixed else "libsphref.so")


def available(mixed: bool | str = False) -> bool:
    return os.path.exists(ref_lib_path(mixed))


def load(mixed: bool | str = False):
    if mixed in _LIBS:
        return _LIBS[mixed]
    path = ref_lib_path(mixed)
    if not os.path.exists(path):
        raise FileNotFoundError(f"reference oracle not built: {path} (run make -C oracle ref)")
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.ref_sim_create.restype = P
    lib.ref_sim_create.argtypes = [C.c_size_t, C.POINTER(C.c_void_p), P, P, C.c_int, P]
    for name in ("ref_sim_initial_sync", "ref_sim_compute_forces", "ref_sim_integrate", "ref_sim_step"):
        getattr(lib, name).argtypes = [P]
        getattr(lib, name).restype = C.c_int
    lib.ref_sim_destroy.argtypes = [P]
    lib.ref_sim_set_av_clean.argtypes = [P, C.c_int]
    lib.ref_sim_get.argtypes = [P, C.c_char_p, P]
    lib.ref_sim_set.argtypes = [P, C.c_char_p, P]
    lib.ref_sim_keys.argtypes = [P, P]
    lib.ref_sim_scalars.argtypes = [P, P]
    lib.ref_sim_timings.argtypes = [P, P]
    lib.ref_sim_range.argtypes = [P, P, P]
    lib.ref_sim_num_leaves.argtypes = [P]
    lib.ref_sim_num_leaves.restype = C.c_size_t
    lib.ref_sim_num_global_leaves.argtypes = [P]
    lib.ref_sim_num_global_leaves.restype = C.c_size_t
    lib.ref_sim_tree.argtypes = [P, P, P, P]
    lib.ref_sim_neighbors.argtypes = [P, P]
    lib.ref_sim_tables.argtypes = [P, P, P, P]
    lib.ref_tables_fp64.argtypes = [C.c_double, P, P, P]
    lib.ref_sphynx_3d_k.argtypes = [C.c_double]
    lib.ref_sphynx_3d_k.restype = C.c_double
    lib.ref_sfc_keys.argtypes = [C.c_size_t, P, P, P, P, C.c_int, P]
    lib.ref_compute_octree.argtypes = [C.c_size_t, P, C.c_uint, P, P, C.c_size_t]
    lib.ref_compute_octree.restype = C.c_size_t
    lib.ref_find_neighbors.argtypes = [C.c_size_t, P, P, P, P, P, P, C.c_int, C.c_uint, C.c_uint, P, P]
    lib.ref_hydro_bits.restype = C.c_int
    _LIBS[mixed] = lib
    return lib


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


SCALAR_NAMES = ("minDt", "minDt_m1", "minDtCourant", "minDtRho", "ttot", "etot", "ecin", "eint", "linmom", "angmom",
                "totalNeighbors", "iteration", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


class RefSim:
    """One simulation of the reference CPU hydro step (1 rank, OpenMP)."""

    def __init__(self, ic: dict, mixed: bool | str = False):
        """ic["params"].get("avClean") selects HydroVeProp<avClean = true>; mixed as in ref_lib_path."""
        from sphexa_b200.ic import CONSERVED_FIELDS
        self.lib = load(mixed)
        p = ic["params"]
        self._keep = [np.ascontiguousarray(ic[f], dtype=np.float64) for f in CONSERVED_FIELDS]
        arr = (C.c_void_p * len(self._keep))(*[a.ctypes.data for a in self._keep])
        self._id = np.ascontiguousarray(ic["id"], dtype=np.uint64)
        self._box = np.array(ic["box"], dtype=np.float64)
        prm = np.array([p["ng0"], p["ngmax"], p["gamma"], p["mui"], p["minDt"], p["minDt_m1"], p["Kcour"], p["Krho"],
                        p["alphamin"], p["alphamax"], p["decay_constant"]], dtype=np.float64)
        self.ngmax = int(p["ngmax"])
        self.n0 = self._id.size
        self.h = self.lib.ref_sim_create(self.n0, arr, ptr(self._id), ptr(self._box), int(bool(ic["periodic"])),
                                         ptr(prm))
        if p.get("avClean"):
            self.lib.ref_sim_set_av_clean(self.h, 1)
        rc = self.lib.ref_sim_initial_sync(self.h)
        if rc:
            raise RuntimeError("reference initial sync failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_sim_destroy(self.h)
            self.h = None

    def compute_forces(self):
        if self.lib.ref_sim_compute_forces(self.h):
            raise RuntimeError("reference computeForces failed")

    def integrate(self) -> int:
        return self.lib.ref_sim_integrate(self.h)

    def step(self) -> int:
        self.compute_forces()
        return self.integrate()

    @property
    def n(self) -> int:
        a, b = C.c_size_t(), C.c_size_t()
        self.lib.ref_sim_range(self.h, C.byref(a), C.byref(b))
        return b.value - a.value

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        rc = self.lib.ref_sim_get(self.h, name.encode(), ptr(out))
        if rc:
            raise KeyError(f"field {name} not available ({rc})")
        return out

    def set(self, name: str, val: np.ndarray):
        v = np.ascontiguousarray(val, dtype=np.float64)
        if self.lib.ref_sim_set(self.h, name.encode(), ptr(v)):
            raise KeyError(name)

    def keys(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.uint64)
        self.lib.ref_sim_keys(self.h, ptr(out))
        return out

    def scalars(self) -> dict:
        out = np.empty(len(SCALAR_NAMES), dtype=np.float64)
        self.lib.ref_sim_scalars(self.h, ptr(out))
        return dict(zip(SCALAR_NAMES, out.tolist()))

    def timings(self) -> np.ndarray:
        out = np.empty(4, dtype=np.float64)
        self.lib.ref_sim_timings(self.h, ptr(out))
        return out

    def tree(self):
        nl = self.lib.ref_sim_num_leaves(self.h)
        leaves = np.empty(nl + 1, dtype=np.uint64)
        counts = np.empty(nl, dtype=np.uint32)
        layout = np.empty(nl + 1, dtype=np.uint32)
        self.lib.ref_sim_tree(self.h, ptr(leaves), ptr(counts), ptr(layout))
        return leaves, counts, layout

    def neighbors(self) -> np.ndarray:
        out = np.empty((self.n, self.ngmax), dtype=np.uint32)
        if self.lib.ref_sim_neighbors(self.h, ptr(out)):
            raise RuntimeError("no neighbour lists stored")
        return out

    def tables(self):
        K = C.c_double()
        wh = np.empty(KTABLE)
        whd = np.empty(KTABLE)
        self.lib.ref_sim_tables(self.h, C.byref(K), ptr(wh), ptr(whd))
        return K.value, wh, whd


def tables_fp64(sinc_index: float = 6.0):
    lib = load(False)
    K = C.c_double()
    wh = np.empty(KTABLE)
    whd = np.empty(KTABLE)
    lib.ref_tables_fp64(sinc_index, C.byref(K), ptr(wh), ptr(whd))
    return K.value, wh, whd


def sfc_keys(x, y, z, box, periodic) -> np.ndarray:
    lib = load(False)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    keys = np.zeros(x.size, dtype=np.uint64)
    b = np.array(box, dtype=np.float64)
    lib.ref_sfc_keys(x.size, ptr(x), ptr(y), ptr(z), ptr(b), int(periodic), ptr(keys))
    return keys


def compute_octree(sorted_keys: np.ndarray, bucket: int):
    lib = load(False)
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint64)
    cap = 8 * (k.size // max(bucket, 1) + 8) * 8 + 64
    leaves = np.empty(cap + 1, dtype=np.uint64)
    counts = np.empty(cap, dtype=np.uint32)
    nl = lib.ref_compute_octree(k.size, ptr(k), bucket, ptr(leaves), ptr(counts), cap)
    if nl + 1 > cap:
        raise RuntimeError("octree capacity")
    return leaves[:nl + 1].copy(), counts[:nl].copy()


def build_octree(leaves: np.ndarray) -> dict:
    """The reference's internal octree of a cornerstone leaf array (buildOctreeCpu), OctreeData arrays."""
    lib = load(False)
    lib.ref_build_octree.restype = C.c_int
    lib.ref_build_octree.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 6
    lv = np.ascontiguousarray(leaves, dtype=np.uint64)
    nl = lv.size - 1
    nn = nl + (nl - 1) // 7
    out = {"prefixes": np.zeros(nn, dtype=np.uint64), "childOffsets": np.zeros(nn, dtype=np.int32),
           "parents": np.zeros(max(1, (nn - 1) // 8), dtype=np.int32), "levelRange": np.zeros(23, dtype=np.int32),
           "internalToLeaf": np.zeros(nn, dtype=np.int32), "leafToInternal": np.zeros(nn, dtype=np.int32)}
    got = lib.ref_build_octree(ptr(lv), nl, *[ptr(out[k]) for k in ("prefixes", "childOffsets", "parents",
                                                                     "levelRange", "internalToLeaf",
                                                                     "leafToInternal")])
    assert got == nn
    return out


def find_neighbors(sorted_keys, x, y, z, h, box, periodic, ngmax, bucket=64):
    """Reference neighbour lists (no h iteration) for particles already in SFC order."""
    lib = load(False)
    n = x.size
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, h)]
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint64)
    nbr = np.zeros((n, ngmax), dtype=np.uint32)
    cnt = np.zeros(n, dtype=np.uint32)
    b = np.array(box, dtype=np.float64)
    lib.ref_find_neighbors(n, ptr(k), *[ptr(a) for a in arrs], ptr(b), int(periodic), bucket, ngmax, ptr(nbr),
                           ptr(cnt))
    return nbr, cnt
