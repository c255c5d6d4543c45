"""TEST ORACLE ONLY: restatement of the block time-step propagator HydroVeBdtProp<avClean>
(main/src/propagator/ve_hydro_bdt.hpp:165-380) with the rung logic of sph/include/sph/ts_rungs.hpp:84-166 and the
group time steps of sph/include/sph/ts_groups.cu, over the plain-C oracle (oracle/sph_oracle.c) for the J-loops,
drifts and kick-drifts. Imported only by tests/.

Groups are the reference's spatial target groups (sph::computeSpatialGroups at every full sync,
ve_hydro_bdt.hpp:185), from the restated group splits of oracle/groups.py over a cornerstone focus tree: the tree
comes from a caller-supplied provider (the tests pass the CUDA path's focus tree, which other tests pin bit for bit
to the reference's), by default the converged tree of the current keys. Time-step arithmetic is float32, as in the
reference (sph::Timestep holds floats). The reference runs this propagator only on GPUs (its constructor refuses
CPUs, ve_hydro_bdt.hpp:119), so nothing of the reference itself can pin this restatement here: it is checked only
against the reading of the sources cited on each step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .groups import group_splits
from .restated import OracleSim, compute_octree, load, ptr

F32 = np.float32
MAX_RUNGS = 4   # Timestep::maxNumRungs (sph/include/sph/timestep.h:19)
GROUP = 32
FLT_MAX = np.finfo(np.float32).max


def butterfly(i: int) -> int:
    """cstone::butterfly (cstone/primitives/math.hpp:35-40): 0 for 0, else 1 + trailing zeros of i"""
    return 0 if i == 0 else (i & -i).bit_length()


def active_rung(substep: int, num_rungs: int) -> int:
    """HydroVeBdtProp::activeRung (ve_hydro_bdt.hpp:109-113)"""
    if substep == 0 or substep >= (1 << (num_rungs - 1)):
        return 0
    return butterfly(substep)


def lower_bound(sorted_dt: np.ndarray, value) -> int:
    return int(np.searchsorted(sorted_dt, F32(value), side="left"))


class Timestep:
    """sph::Timestep (sph/include/sph/timestep.h:17-31)"""

    def __init__(self):
        self.next_dt = F32(0)
        self.elapsed_dt = F32(0)
        self.tot_dt = F32(0)
        self.num_rungs = 1
        self.substep = 0
        self.rung_ranges = [0] * (MAX_RUNGS + 1)
        self.dt_m1 = np.zeros(MAX_RUNGS, dtype=np.float32)
        self.dt_drift = np.zeros(MAX_RUNGS, dtype=np.float32)

    def copy(self) -> "Timestep":
        t = Timestep()
        t.next_dt, t.elapsed_dt, t.tot_dt = self.next_dt, self.elapsed_dt, self.tot_dt
        t.num_rungs, t.substep = self.num_rungs, self.substep
        t.rung_ranges = list(self.rung_ranges)
        t.dt_m1, t.dt_drift = self.dt_m1.copy(), self.dt_drift.copy()
        return t

    def as_dict(self) -> dict:
        return {"next_dt": float(self.next_dt), "elapsed_dt": float(self.elapsed_dt), "total_dt": float(self.tot_dt),
                "num_rungs": self.num_rungs, "substep": self.substep, "rung_ranges": list(self.rung_ranges),
                "dt_m1": [float(v) for v in self.dt_m1], "dt_drift": [float(v) for v in self.dt_drift]}


class BdtOracle(OracleSim):
    """One substep per step(): computeForces then integrate of HydroVeBdtProp, one rank."""

    def __init__(self, ic: dict, eta_acc: float = 0.2, tree=None):
        """tree: callable returning (leaves, layout) of the focus tree for the particles in their current SFC order,
        called at every full sync; None: the converged cornerstone tree (bucket 64) of the current keys."""
        super().__init__(ic)
        self.tree = tree
        lib = load()
        lib.orc_sim_sync_perm.restype = None
        lib.orc_sim_sync_perm.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_sim_forces_active.restype = C.c_int
        lib.orc_sim_forces_active.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        lib.orc_drift.restype = None
        lib.orc_drift.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_float, C.c_float, C.c_void_p, C.c_void_p]
        lib.orc_rung_positions.restype = None
        lib.orc_rung_positions.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_float, C.c_void_p, C.c_void_p,
                                           C.c_int]
        lib.orc_update_h_subset.restype = C.c_int
        lib.orc_update_h_subset.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        p = ic["params"]
        self.eta_acc = F32(eta_acc)
        self.krho = F32(p["Krho"])
        self.bounds = np.array([0, self.n], dtype=np.uint32)  # set at every full sync
        self.num_groups = 1
        self.ts = Timestep()
        self.ts.dt_m1[0] = F32(p["minDt"])          # the constructor, ve_hydro_bdt.hpp:122
        self.prev = self.ts.copy()
        self.rung = np.zeros(self.n, dtype=np.uint8)
        self.groups = np.arange(self.num_groups, dtype=np.uint32)    # groups_ (SFC order)
        self.ts_groups = np.arange(self.num_groups, dtype=np.uint32)  # tsGroups_ (by time step)
        self.group_dt = np.full(self.num_groups, FLT_MAX, dtype=np.float32)
        self.group_idx = np.zeros(self.num_groups, dtype=np.uint32)
        self.min_dt = float(p["minDt"])           # d.minDt, the AV switches' time step
        self.active = self.groups.copy()

    # -- particles of a list of groups, in list order
    def particles(self, groups: np.ndarray) -> np.ndarray:
        if len(groups) == 0:
            return np.zeros(0, dtype=np.uint32)
        g = groups.astype(np.int64)
        return np.ascontiguousarray(np.concatenate([np.arange(self.bounds[k], self.bounds[k + 1]) for k in g]),
                                    dtype=np.uint32)

    def spatial_groups(self):
        """computeGroups -> computeSpatialGroups (sph/include/sph/groups.hpp:41-74): group boundaries of the current
        SFC order, tolFactor 2, groups of 32"""
        if self.tree is not None:
            leaves, layout = self.tree()
        else:
            leaves, counts = compute_octree(self.keys(), 64)
            layout = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
        sc = self.scalars()
        box = (sc["xmin"], sc["xmax"], sc["ymin"], sc["ymax"], sc["zmin"], sc["zmax"])
        x, y, z, h = (self.get(f) for f in ("x", "y", "z", "h"))
        return group_splits(x, y, z, h, np.asarray(leaves, dtype=np.uint64), np.asarray(layout, dtype=np.uint32),
                            box, GROUP, 2.0, False)

    def sync(self):
        """fullSync / partialSync (ve_hydro_bdt.hpp:165-215)"""
        ts = self.ts
        if active_rung(ts.substep, ts.num_rungs) == 0:
            perm = np.empty(self.n, dtype=np.uint32)
            self.lib.orc_sim_sync_perm(self.h, ptr(perm))
            self.rung = self.rung[perm]                  # rung is a conserved field
            self.bounds = self.spatial_groups()
            self.num_groups = self.bounds.size - 1
            self.groups = np.arange(self.num_groups, dtype=np.uint32)
            self.active = self.groups.copy()
            self.group_dt = np.full(self.num_groups, FLT_MAX, dtype=np.float32)
            self.group_idx = np.zeros(self.num_groups, dtype=np.uint32)
        else:
            highest = butterfly(ts.substep)
            self.active = self.ts_groups[ts.rung_ranges[0]:ts.rung_ranges[highest]].copy()

    def compute_forces(self):
        self.sync()
        mask = np.zeros(self.n, dtype=np.uint8)
        mask[self.particles(self.active)] = 1
        dt = np.empty(self.n)
        self.lib.orc_sim_forces_active(self.h, ptr(mask), self.min_dt, ptr(dt))
        starts = self.bounds[:-1].astype(np.int64)

        def per_group(a, fill, red):
            return (np.maximum if red is np.max else np.minimum).reduceat(a, starts)

        divv, h = self.get("divv"), self.get("h")
        ax, ay, az = self.get("ax"), self.get("ay"), self.get("az")
        # groupDivvTimestep (ts_groups.cu:17-45): float max of divv, Krho / |max| in float (inf for divv = 0)
        with np.errstate(divide="ignore"):
            gdivv = self.krho / np.abs(per_group(divv, -np.inf, np.max).astype(np.float32))
        # momentum_energy_gpu.cu:96-103: the group's Courant step (warp min of the per-particle doubles)
        gcour = per_group(dt, np.inf, np.min).astype(np.float32)
        # groupAccTimestep (ts_groups.cu:47-80): eta (min h^2 / |a|^2)^(1/4) in float
        with np.errstate(divide="ignore"):
            q = h * h / (ax * ax + ay * ay + az * az)
        gacc = self.eta_acc * np.sqrt(np.sqrt(per_group(q, np.inf, np.min).astype(np.float32)))
        g = self.active.astype(np.int64)
        w = np.arange(len(g))
        self.group_dt[w] = np.minimum(np.minimum(np.minimum(self.group_dt[w], gdivv[g]), gcour[g]), gacc[g])

    def _sort(self, num: int):
        """computeMinTimestep (ts_rungs.hpp:84-108) on group_dt[0, num): stable sort, permutation in group_idx"""
        order = np.argsort(self.group_dt[:num], kind="stable")
        self.group_dt[:num] = self.group_dt[:num][order]
        self.group_idx[:num] = order.astype(np.uint32)
        fast = self.group_dt[min(int(F32(0.4) * F32(num)), num - 1)]
        return self.group_dt[0], fast

    def compute_rungs(self):
        """computeRungs (ve_hydro_bdt.hpp:299-334)"""
        ts = self.ts
        high = active_rung(ts.substep, ts.num_rungs)
        G = self.num_groups
        if high == 0:
            # rungTimestep (ts_rungs.hpp:148-158)
            self.prev = ts.copy()
            max_dt = F32(float(ts.dt_m1[0]) * 1.1)
            min_dt, fast = self._sort(G)
            num_rungs = min(int(np.log2(F32(fast / min_dt))) + 1, MAX_RUNGS)
            ranges = [0] + [lower_bound(self.group_dt[:G], F32(1 << r) * min_dt) if r < num_rungs else G
                            for r in range(1, MAX_RUNGS)] + [G]
            min_dt = min(max_dt, min_dt)
            t = Timestep()
            t.next_dt, t.tot_dt, t.num_rungs, t.rung_ranges = min_dt, F32(min_dt * F32(1 << num_rungs)), num_rungs, ranges
            self.ts = ts = t
        else:
            # minimumGroupDt (ts_rungs.hpp:160-166)
            na, nt = ts.rung_ranges[high], ts.rung_ranges[MAX_RUNGS]
            min_dt, _ = self._sort(na)
            self.group_idx[na:nt] = np.arange(na, nt, dtype=np.uint32)
            lb = [0] + [lower_bound(self.group_dt[:na], F32(1 << r) * min_dt) for r in range(1, MAX_RUNGS)]
            time_left = F32(ts.tot_dt - ts.elapsed_dt)
            left = F32((1 << ts.num_rungs) - ts.substep)
            ts.next_dt = min(min_dt, F32(time_left / left))
            for r in range(1, high):
                ts.rung_ranges[r] = lb[r]
        if high == 0 or high > 1:
            if high > 1:
                self.groups, self.ts_groups = self.ts_groups, self.groups
            # extractGroupGpu (sph/include/sph/groups.hpp:77-93)
            self.ts_groups = self.groups[self.group_idx[:ts.rung_ranges[MAX_RUNGS]]]

    def integrate(self) -> int:
        """integrate (ve_hydro_bdt.hpp:336-380)"""
        self.compute_rungs()
        ts = self.ts
        lowest = butterfly(ts.substep + 1)
        last = active_rung(ts.substep + 1, ts.num_rungs) == 0
        for i in range(ts.num_rungs):
            use_rung = ts.substep == ts.substep % (1 << i)
            advance = i < lowest
            dt = ts.next_dt
            dtm1 = np.ascontiguousarray((self.prev if use_rung else ts).dt_m1, dtype=np.float32)
            idx = self.particles(self.ts_groups[ts.rung_ranges[i]:ts.rung_ranges[i + 1]])
            if advance:
                if ts.dt_drift[i] > 0:
                    self.lib.orc_drift(self.h, ptr(idx), idx.size, 0.0, float(ts.dt_drift[i]), ptr(dtm1),
                                       ptr(self.rung))
                step = F32(ts.dt_drift[i] + dt)
                self.lib.orc_rung_positions(self.h, ptr(idx), idx.size, float(step), ptr(dtm1), ptr(self.rung),
                                            int(last))
                ts.dt_m1[i] = step
                ts.dt_drift[i] = F32(0)
                self.rung[idx] = i
            else:
                self.lib.orc_drift(self.h, ptr(idx), idx.size, float(F32(ts.dt_drift[i] + dt)),
                                   float(ts.dt_drift[i]), ptr(dtm1), ptr(self.rung))
                ts.dt_drift[i] = F32(ts.dt_drift[i] + dt)
        act = self.particles(self.active)
        removed = self.lib.orc_update_h_subset(self.h, ptr(act), act.size)
        ts.substep += 1
        ts.elapsed_dt = F32(ts.elapsed_dt + ts.next_dt)
        self.min_dt = float(ts.next_dt)
        return removed

    def step(self) -> int:
        self.compute_forces()
        return self.integrate()
