"""TEST ORACLE ONLY: the multi-rank domain's tree, assignment and halo-discovery steps, as the reference computes them
(ctypes wrappers of the reference's own functions compiled into oracle/_ref/libsphref.so by oracle/ref/ref_driver.cpp)
and restated in numpy; plus OracleEngine, the CPU stand-in for the device engine of sphexa_b200.domain.Domain that
the world_size-2 gloo tests run the domain's host logic with. Imported only by tests/.

Reference functions: computeNodeCounts (domain/include/cstone/tree/csarray.hpp:181-235), rebalanceDecision +
rebalanceTree (csarray.hpp:309-389) as updateOctreeGlobal applies them (tree/update_mpi.hpp:64-99),
makeSfcAssignment (domain/domaindecomp.hpp:112-127), computeBoundingBox + findHalos (focus/source_center.hpp:28-43,
traversal/collisions.hpp:69-104) as FocusedOctree::discoverHalos calls them (focus/octree_focus_mpi.hpp:556-569).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle import refsim

MAX_LEVEL = 21
ROOT_END = np.uint64(1) << np.uint64(63)


def _lib():
    lib = refsim.load(False)
    if not getattr(lib, "_domain_sigs", False):
        P, S = C.c_void_p, C.c_size_t
        lib.ref_leaf_counts.argtypes = [P, S, P, S, P]
        lib.ref_rebalance_tree.argtypes = [P, S, P, C.c_uint, P, S, C.POINTER(C.c_int)]
        lib.ref_rebalance_tree.restype = S
        lib.ref_find_halos.argtypes = [P, S, P, P, P, P, P, P, C.c_int, C.c_int, P, C.c_int, C.c_float, P]
        lib.ref_sfc_assignment.argtypes = [C.c_int, P, S, P, P, P, P]
        lib._domain_sigs = True
    return lib


def _p(a):
    return refsim.ptr(a)


# ------------------------------------------------------------------------------------------------------------------
# the reference's own functions
# ------------------------------------------------------------------------------------------------------------------

def ref_leaf_counts(leaves: np.ndarray, sorted_keys: np.ndarray) -> np.ndarray:
    lv = np.ascontiguousarray(leaves, dtype=np.uint64)
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint64)
    out = np.zeros(lv.size - 1, dtype=np.uint32)
    _lib().ref_leaf_counts(_p(lv), lv.size - 1, _p(k), k.size, _p(out))
    return out


def ref_rebalance_tree(leaves: np.ndarray, counts: np.ndarray, bucket: int):
    """(new leaves, converged) of one rebalance step"""
    lv = np.ascontiguousarray(leaves, dtype=np.uint64)
    c = np.ascontiguousarray(counts, dtype=np.uint32)
    cap = 4096 * lv.size + 8  # a leaf splits into at most 8^4 leaves per step
    out = np.zeros(cap + 1, dtype=np.uint64)
    conv = C.c_int()
    nl = _lib().ref_rebalance_tree(_p(lv), lv.size - 1, _p(c), bucket, _p(out), cap, C.byref(conv))
    if nl + 1 > cap:
        raise RuntimeError("rebalance capacity")
    return out[:nl + 1].copy(), bool(conv.value)


def ref_sfc_assignment(num_ranks: int, counts: np.ndarray, leaves: np.ndarray):
    """(boundary keys [num_ranks + 1], first leaf per rank [num_ranks + 1], particles per rank)"""
    c = np.ascontiguousarray(counts, dtype=np.uint32)
    lv = np.ascontiguousarray(leaves, dtype=np.uint64)
    b = np.zeros(num_ranks + 1, dtype=np.uint64)
    off = np.zeros(num_ranks + 1, dtype=np.int32)
    rc = np.zeros(num_ranks, dtype=np.uint32)
    _lib().ref_sfc_assignment(num_ranks, _p(c), c.size, _p(lv), _p(b), _p(off), _p(rc))
    return b, off, rc


def ref_find_halos(leaves, x, y, z, h, layout, first_leaf, last_leaf, box, periodic, search_ext=1.0):
    """halo flag (0/1) per leaf of the rank owning [first_leaf, last_leaf); x, y, z, h its particles in SFC order,
    layout (last_leaf - first_leaf + 1 offsets) their leaf ranges; h float32 uses the reference's float radius"""
    lv = np.ascontiguousarray(leaves, dtype=np.uint64)
    xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
    hf = h.dtype == np.float32
    hh = np.ascontiguousarray(h)
    lay = np.ascontiguousarray(layout, dtype=np.uint32)
    lim = np.array(box, dtype=np.float64)
    flags = np.zeros(lv.size - 1, dtype=np.uint8)
    _lib().ref_find_halos(_p(lv), lv.size - 1, *[_p(a) for a in xs], None if hf else _p(hh), _p(hh) if hf else None,
                          _p(lay), int(first_leaf), int(last_leaf), _p(lim), int(bool(periodic)), float(search_ext),
                          _p(flags))
    return flags


# ------------------------------------------------------------------------------------------------------------------
# restatements
# ------------------------------------------------------------------------------------------------------------------

def leaf_counts(leaves: np.ndarray, sorted_keys: np.ndarray) -> np.ndarray:
    """particles per leaf: keys in [leaves[i], leaves[i + 1])"""
    idx = np.searchsorted(sorted_keys.astype(np.uint64), leaves.astype(np.uint64), side="left")
    return np.diff(idx).astype(np.uint32)


def uniform_bins(counts: np.ndarray, num_ranks: int):
    """first leaf per rank (num_ranks + 1) and particles per rank: rank r starts at the first leaf whose count
    prefix reaches r * total / num_ranks (uniformBins, domaindecomp.hpp:32-56)"""
    scan = np.concatenate([[0], np.cumsum(counts.astype(np.uint64))])
    per = float(scan[-1]) / num_ranks
    bins = np.zeros(num_ranks + 1, dtype=np.int64)
    bins[-1] = counts.size
    for r in range(1, num_ranks):
        bins[r] = np.searchsorted(scan, np.uint64(int(r * per)), side="left")
    return bins, np.diff(scan[bins]).astype(np.uint32)


def global_tree(keys_per_rank: list, bucket: int):
    """the converged global cornerstone tree of the union of every rank's sorted keys, stepped as the multi-rank
    update does: summed leaf counts, one rebalance, until a rebalance changes nothing"""
    leaves = np.array([0, ROOT_END], dtype=np.uint64)
    while True:
        counts = sum(ref_leaf_counts(leaves, k) for k in keys_per_rank).astype(np.uint32)
        new, conv = ref_rebalance_tree(leaves, counts, bucket)
        if conv:
            return leaves, counts
        leaves = new


def _node_geometry(leaves: np.ndarray, box):
    """geometric centre and half size of every leaf cell (centerAndSize, sfc/box.hpp:317-334)"""
    lv = leaves.astype(np.uint64)
    rng = lv[1:] - lv[:-1]
    level = MAX_LEVEL - (np.floor(np.log2(rng.astype(np.float64))).astype(np.int64)) // 3
    start = lv[:-1]
    ix, iy, iz = _hilbert_decode(start)
    edge = (np.uint64(1) << np.uint64(MAX_LEVEL)) >> level.astype(np.uint64)
    lo = [a & ~(edge - np.uint64(1)) for a in (ix, iy, iz)]
    centers, sizes = np.zeros((lv.size - 1, 3)), np.zeros((lv.size - 1, 3))
    for k in range(3):
        L = box[2 * k + 1] - box[2 * k]
        half_unit = 0.5 * (1.0 / float(1 << MAX_LEVEL)) * L
        hi = lo[k] + edge
        centers[:, k] = box[2 * k] + (hi + lo[k]).astype(np.float64) * half_unit
        sizes[:, k] = (hi - lo[k]).astype(np.float64) * half_unit
    return centers, sizes


def _hilbert_decode(keys: np.ndarray):
    """3D Hilbert key to integer coordinates, by the oracle's C restatement (oracle/sph_oracle.c)"""
    from oracle import restated
    lib = restated.load()
    out = np.zeros((3, keys.size), dtype=np.uint64)
    cx, cy, cz = C.c_uint(), C.c_uint(), C.c_uint()
    for i, k in enumerate(keys):
        lib.orc_hilbert_decode(int(k), C.byref(cx), C.byref(cy), C.byref(cz))
        out[0, i], out[1, i], out[2, i] = cx.value, cy.value, cz.value
    return out[0], out[1], out[2]


def find_halos(leaves, x, y, z, h, layout, first_leaf, last_leaf, box, periodic, search_ext=1.0):
    """brute force: leaf l outside [first_leaf, last_leaf) is a halo if its cell overlaps the search box of any owned
    leaf (boxes as computeBoundingBox, overlap with the minimum image as traversal/boxoverlap.hpp:280-292)"""
    centers, sizes = _node_geometry(leaves, box)
    hf = h.dtype == np.float32
    scale = np.float32(2.0 * np.float32(search_ext)) if hf else np.float64(np.float32(2.0 * np.float32(search_ext)))
    n_own = last_leaf - first_leaf
    sc, ss = np.zeros((n_own, 3)), np.zeros((n_own, 3))
    for i in range(n_own):
        a, b = int(layout[i]), int(layout[i + 1])
        c0 = centers[first_leaf + i]
        mn, mx = c0.copy(), c0.copy()
        if b > a:
            r = (h[a:b] * scale).astype(np.float64)
            p = np.stack([x[a:b], y[a:b], z[a:b]], axis=1)
            mn = np.minimum(mn, (p - r[:, None]).min(axis=0))
            mx = np.maximum(mx, (p + r[:, None]).max(axis=0))
        sc[i], ss[i] = (mx + mn) * 0.5, (mx - mn) * 0.5
    L = np.array([box[1] - box[0], box[3] - box[2], box[5] - box[4]])
    flags = np.zeros(leaves.size - 1, dtype=np.uint8)
    for i in range(n_own):
        d = sc[i][None, :] - centers
        if periodic:
            d = d - L * np.rint(d * (1.0 / L))
        d = np.abs(d) - sizes - ss[i][None, :]
        hit = np.all(d < 0.0, axis=1)
        flags[hit] = 1
    flags[first_leaf:last_leaf] = 0
    return flags


# ------------------------------------------------------------------------------------------------------------------
# the CPU engine of the domain's host logic in the tests
# ------------------------------------------------------------------------------------------------------------------

class OracleEngine:
    """The per-particle and per-leaf operations of sphexa_b200.domain.Domain on CPU tensors, computed by the
    reference's own functions (keys, leaf counts, rebalance, halo discovery) and numpy (stable key sort)."""

    def __init__(self, periodic: bool = True):
        self.periodic = periodic

    @staticmethod
    def _np(t):
        return t.detach().cpu().numpy()

    def sfc_keys(self, x, y, z, box):
        import torch
        k = refsim.sfc_keys(self._np(x), self._np(y), self._np(z), box.limits, box.periodic[0])
        return torch.from_numpy(k.view(np.int64).copy())

    def sort_by_key(self, keys):
        import torch
        k = self._np(keys).view(np.uint64)
        order = np.argsort(k, kind="stable")
        return torch.from_numpy(k[order].view(np.int64).copy()), torch.from_numpy(order.astype(np.int64))

    def leaf_counts(self, leaves, sorted_keys):
        import torch
        c = ref_leaf_counts(self._np(leaves).view(np.uint64), self._np(sorted_keys).view(np.uint64))
        return torch.from_numpy(c.astype(np.int64))

    def rebalance(self, leaves, counts, bucket):
        import torch
        new, conv = ref_rebalance_tree(self._np(leaves).view(np.uint64), self._np(counts).astype(np.uint32), bucket)
        return torch.from_numpy(new.view(np.int64).copy()), conv

    def find_halos(self, leaves, x, y, z, h, layout, first_leaf, last_leaf, box, search_ext):
        import torch
        f = ref_find_halos(self._np(leaves).view(np.uint64), self._np(x), self._np(y), self._np(z), self._np(h),
                           self._np(layout).astype(np.uint32), first_leaf, last_leaf, box.limits, box.periodic[0],
                           search_ext)
        return torch.from_numpy(f)
