"""Batched ensemble of independent VE hydro simulations (sphb_ensemble): all instances advance together, one launch
per stage over every instance, the step replayed as one captured CUDA graph.

Each instance evolves as a `Simulation` of the same initial conditions would; instances share the periodic box and the
kernel and neighbour settings, and may differ in size, gamma, mui and therefore their time steps.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as L
from .ic import CONSERVED_FIELDS

ENSEMBLE_SCALARS = ("minDt", "minDt_m1", "ttot", "etot", "ecin", "eint", "linmom", "angmom", "totalNeighbors")
JLOOPS = ("xmass", "ve_def_gradh_eos", "iad_divv_curlv", "av_switches", "momentum_energy")


class Ensemble:
    def __init__(self, ics: list[dict], precision: str = "mixed"):
        self.lib = L.load()
        self.num = len(ics)
        self.sizes = [int(ic["x"].size) for ic in ics]
        self.precision = precision
        prec = L.SPHB_MIXED if precision == "mixed" else L.SPHB_FP64
        box = L.make_box(ics[0]["box"], [ics[0]["periodic"]] * 3)
        params = (L.Params * self.num)(*[L.make_params(ic["params"], prec) for ic in ics])
        sizes = (C.c_size_t * self.num)(*self.sizes)
        h = C.c_void_p()
        L.check(self.lib.sphb_ensemble_create(C.byref(h), self.num, sizes, C.byref(box), params),
                "sphb_ensemble_create")
        self.h = h
        for k, ic in enumerate(ics):
            arrs = [np.ascontiguousarray(ic[f], dtype=np.float64) for f in CONSERVED_FIELDS]
            ids = np.ascontiguousarray(ic["id"], dtype=np.uint64)
            table = (C.c_void_p * len(arrs))(*[L.ptr(a).value for a in arrs])
            L.check(self.lib.sphb_ensemble_upload(self.h, k, table, L.ptr(ids), 0), "sphb_ensemble_upload")
        L.check(self.lib.sphb_ensemble_initial_sync(self.h), "sphb_ensemble_initial_sync")

    def step(self, steps: int = 1, graph: bool = True) -> int:
        rc = self.lib.sphb_ensemble_step(self.h, int(steps), int(graph))
        if rc not in (L.SPHB_OK, 4):
            L.check(rc, "sphb_ensemble_step")
        return rc

    def autotune(self) -> dict:
        out = (C.c_int * 5)()
        L.check(self.lib.sphb_ensemble_autotune(self.h, out), "sphb_ensemble_autotune")
        return dict(zip(JLOOPS, list(out)))

    def set_threads(self, threads):
        arr = (C.c_int * 5)(*threads)
        L.check(self.lib.sphb_ensemble_set_threads(self.h, arr), "sphb_ensemble_set_threads")

    def rebuild_trees(self):
        L.check(self.lib.sphb_ensemble_rebuild_trees(self.h), "sphb_ensemble_rebuild_trees")

    def get(self, k: int, name: str) -> np.ndarray:
        out = np.empty(self.sizes[k], dtype=np.float64)
        L.check(self.lib.sphb_ensemble_get_field(self.h, k, name.encode(), L.ptr(out)), f"get_field({name})")
        if name in ("keys", "id"):
            return out.view(np.uint64)
        return out

    def scalars(self, k: int) -> dict:
        out = np.empty(len(ENSEMBLE_SCALARS))
        L.check(self.lib.sphb_ensemble_scalars(self.h, k, L.ptr(out)), "sphb_ensemble_scalars")
        return dict(zip(ENSEMBLE_SCALARS, out.tolist()))

    def stream(self):
        return self.lib.sphb_ensemble_stream(self.h)

    def stage_times(self) -> dict:
        """Stage times in ms of the last step (CUDA events recorded inside the step)."""
        from .simulation import STAGE_NAMES
        out = np.empty(len(STAGE_NAMES), dtype=np.float32)
        L.check(self.lib.sphb_ensemble_stage_times(self.h, L.ptr(out)), "sphb_ensemble_stage_times")
        return dict(zip(STAGE_NAMES, out.tolist()))

    def search_stats(self) -> dict:
        """How the neighbour stage ran since the initial sync: tree searches of every group, skin-row builds, steps
        served from the skin rows, and groups those steps deferred to the tree search."""
        out = np.zeros(4, dtype=np.uint64)
        L.check(self.lib.sphb_ensemble_search_stats(self.h, L.ptr(out)), "sphb_ensemble_search_stats")
        return dict(zip(("tree_searches", "skin_builds", "skin_steps", "deferred_groups"), (int(v) for v in out)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.sphb_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
