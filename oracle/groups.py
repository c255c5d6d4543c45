"""TEST ORACLE ONLY: restatement of the spatial target groups (cstone computeGroupSplits,
domain/include/cstone/traversal/groups_gpu.cu:58-137 and groups_gpu.cuh:37-216, as sph::computeSpatialGroups calls
it, sph/include/sph/groups.hpp:41-55) in numpy, and a ctypes wrapper of the reference's own kernels compiled in
oracle/_ref/libsphref_groups.so (oracle/ref/groups_driver.cu). Imported only by tests/."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_LEVEL = 21


def group_splits(x, y, z, h, leaves, layout, box, group_size=32, tol_factor=2.0, h_float=False):
    """Boundaries (numGroups + 1) of the spatial groups of all particles (first = 0), following groupSplitsKernel:
    fixed runs of group_size; split after lane i when |X_{i+1} - X_i|^2 > min(distCrit^2, (2 h_i / minExtent)^2)
    with X = x / L per axis and distCrit = tol_factor * cbrt(smallest leaf volume of the run in the unit box), the
    leaf of the run's first-segment particle standing for every segment (groups_gpu.cuh:188-193). The threshold is
    computed in the precision of h (float if h_float), as the reference's template type T."""
    n = x.size
    ft = np.float32 if h_float else np.float64
    lx, ly, lz = box[1] - box[0], box[3] - box[2], box[5] - box[4]
    ilx, ily, ilz = 1.0 / lx, 1.0 / ly, 1.0 / lz
    min_ext = min(min(lx, ly), lz)
    num_fixed = (n + group_size - 1) // group_size
    idx = np.minimum(np.arange(num_fixed * group_size), n - 1)
    px, py, pz = x[idx] * ilx, y[idx] * ily, z[idx] * ilz
    ph = (2.0 * h[idx].astype(np.float64) / min_ext) if h is not None else np.ones(idx.size)
    # leaf of every particle: upper_bound over layout[0, numLeaves) minus one
    num_leaves = leaves.size - 1
    leaf = np.searchsorted(layout[:num_leaves], idx, side="right") - 1
    rng = (leaves[leaf + 1] - leaves[leaf]).astype(np.uint64)
    level = MAX_LEVEL - (np.floor(np.log2(rng.astype(np.float64))).astype(np.int64)) // 3
    edge = np.ldexp(1.0, -level)                              # 8 * (edge / 2)^3 = edge^3, exact
    vol = (edge ** 3).astype(ft)
    nwt = group_size // 32
    # the smallest volume over the warp of the run, each lane taking its first-segment particle's leaf
    vol_first = vol.reshape(num_fixed, nwt, 32)[:, 0, :]
    node_vol = vol_first.min(axis=1)
    dist_crit = (np.cbrt(node_vol).astype(ft) * ft(tol_factor)).astype(np.float64)
    crit_sq = dist_crit * dist_crit
    # successor of every slot of a run; the run's last slot has none (distance zero)
    X = np.stack([px, py, pz], axis=1).reshape(num_fixed, group_size, 3)
    nxt = np.concatenate([X[:, 1:, :], X[:, -1:, :]], axis=1)
    d = nxt - X
    dist_sq = (d[:, :, 0] * d[:, :, 0] + d[:, :, 1] * d[:, :, 1]) + d[:, :, 2] * d[:, :, 2]
    phr = ph.reshape(num_fixed, group_size)
    split = dist_sq > np.minimum(crit_sq[:, None], phr * phr)
    starts = [0]
    for w in range(num_fixed):
        base = w * group_size
        for b in np.nonzero(split[w])[0]:
            starts.append(base + int(b) + 1)
        if w + 1 < num_fixed:
            starts.append(base + group_size)
    return np.array(starts + [n], dtype=np.uint32)


def reference_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libsphref_groups.so"))


def reference_group_splits(x, y, z, h, leaves, layout, box, periodic, group_size=32, tol_factor=2.0,
                           h_float=False):
    """The reference's own kernels on the GPU (host arrays in and out)."""
    lib = C.CDLL(os.path.join(HERE, "_ref", "libsphref_groups.so"))
    P = C.c_void_p
    lib.ref_group_splits.restype = C.c_int
    lib.ref_group_splits.argtypes = [C.c_size_t, C.c_size_t, P, P, P, P, C.c_int, P, C.c_int, P, P, C.c_int,
                                     C.c_uint, C.c_float, P, C.c_size_t, C.POINTER(C.c_size_t)]
    n = x.size
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
    hh = None if h is None else np.ascontiguousarray(h, dtype=np.float32 if h_float else np.float64)
    lv = np.ascontiguousarray(leaves, dtype=np.uint64)
    ly = np.ascontiguousarray(layout, dtype=np.uint32)
    b = np.ascontiguousarray(box, dtype=np.float64)
    cap = n + 2
    out = np.zeros(cap, dtype=np.uint32)
    num = C.c_size_t()
    ptr = (lambda a: None if a is None else a.ctypes.data_as(P))
    rc = lib.ref_group_splits(0, n, *[ptr(a) for a in arrs], ptr(hh), int(h_float), ptr(lv), lv.size - 1, ptr(ly),
                              ptr(b), int(periodic), group_size, tol_factor, ptr(out), cap, C.byref(num))
    if rc:
        raise RuntimeError(f"reference group kernels failed ({rc})")
    return out[:num.value + 1].copy()
