"""Host-side mirror of the reference's propagator interface for the VE hydro step.

`Simulation` owns one sphb_sim (the particle dataset in HBM) and exposes the calls of HydroVeProp
(main/src/propagator/ve_hydro.hpp): sync, computeForces, integrate, plus field access by the reference's field names
(sph/include/sph/particles_data.hpp:262-266).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as L
from .ic import CONSERVED_FIELDS

SCALAR_NAMES = ("minDt", "minDt_m1", "minDtCourant", "minDtRho", "ttot", "etot", "ecin", "eint", "linmom", "angmom",
                "totalNeighbors", "iteration", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax")
STAGE_NAMES = ("sync", "neighbors", "xmass", "ve_def_gradh_eos", "iad_divv_curlv", "av_switches", "momentum_energy",
               "conserved", "integrate")


class Simulation:
    """One SPH-VE simulation on the current CUDA device.

    ic: dict from sphexa_b200.ic (fields, "box", "periodic", "params"); precision: "fp64" or "mixed".
    """

    def __init__(self, ic: dict, precision: str = "fp64", initial_sync: bool = True):
        self.lib = L.load()
        self.n = int(ic["x"].size)
        self.params = dict(ic["params"])
        self.precision = precision
        prec = L.SPHB_MIXED if precision == "mixed" else L.SPHB_FP64
        box = L.make_box(ic["box"], [ic["periodic"]] * 3)
        prm = L.make_params(self.params, prec)
        h = C.c_void_p()
        L.check(self.lib.sphb_sim_create(C.byref(h), self.n, C.byref(box), C.byref(prm)), "sphb_sim_create")
        self.h = h
        self.upload(ic)
        if initial_sync:
            self.initial_sync()

    def upload(self, ic: dict, on_device: bool = False):
        """Copy the 14 conserved fields and ids in (host numpy arrays, or device tensors with on_device)."""
        if on_device:
            arrs = [ic[f] for f in CONSERVED_FIELDS]
            ids = ic["id"]
        else:
            arrs = [np.ascontiguousarray(ic[f], dtype=np.float64) for f in CONSERVED_FIELDS]
            ids = np.ascontiguousarray(ic["id"], dtype=np.uint64)
        table = (C.c_void_p * len(arrs))(*[L.ptr(a).value for a in arrs])
        L.check(self.lib.sphb_sim_upload(self.h, table, L.ptr(ids), int(on_device)), "sphb_sim_upload")

    def initial_sync(self):
        L.check(self.lib.sphb_sim_initial_sync(self.h), "sphb_sim_initial_sync")

    def compute_forces(self):
        L.check(self.lib.sphb_sim_compute_forces(self.h), "sphb_sim_compute_forces")

    # the force computation one stage at a time (HydroVeProp::computeForces order)
    def sync(self):
        L.check(self.lib.sphb_sim_sync(self.h), "sphb_sim_sync")

    def find_neighbors(self):
        L.check(self.lib.sphb_sim_find_neighbors(self.h), "sphb_sim_find_neighbors")

    def xmass(self):
        L.check(self.lib.sphb_sim_xmass(self.h), "sphb_sim_xmass")

    def ve_def_gradh_eos(self):
        L.check(self.lib.sphb_sim_ve_def_gradh_eos(self.h), "sphb_sim_ve_def_gradh_eos")

    def iad_divv_curlv(self):
        L.check(self.lib.sphb_sim_iad_divv_curlv(self.h), "sphb_sim_iad_divv_curlv")

    def av_switches(self):
        L.check(self.lib.sphb_sim_av_switches(self.h), "sphb_sim_av_switches")

    def momentum_energy(self) -> float:
        """Returns the minimum Courant time step of the particles."""
        dt = C.c_double()
        L.check(self.lib.sphb_sim_momentum_energy(self.h, C.byref(dt)), "sphb_sim_momentum_energy")
        return dt.value

    def conserved(self) -> dict:
        out = np.empty(5)
        L.check(self.lib.sphb_sim_conserved(self.h, L.ptr(out)), "sphb_sim_conserved")
        return dict(zip(("ecin", "eint", "etot", "linmom", "angmom"), out.tolist()))

    def integrate(self) -> int:
        rc = self.lib.sphb_sim_integrate(self.h)
        if rc not in (L.SPHB_OK, 4):
            L.check(rc, "sphb_sim_integrate")
        return rc

    def step(self) -> int:
        self.compute_forces()
        return self.integrate()

    def enable_block_timesteps(self, eta_acc: float = 0.2):
        """Switch to the block time-step propagator (HydroVeBdtProp, main/src/propagator/ve_hydro_bdt.hpp)."""
        L.check(self.lib.sphb_sim_bdt_enable(self.h, float(eta_acc)), "bdt_enable")

    def bdt_step(self) -> int:
        """One substep of the block time-step propagator; returns 0 or 4 (particles with nc <= 1)."""
        rc = self.lib.sphb_sim_bdt_step(self.h)
        if rc not in (L.SPHB_OK, 4):
            L.check(rc, "bdt_step")
        return rc

    def bdt_timestep(self) -> dict:
        t = L.BdtTimestep()
        L.check(self.lib.sphb_sim_bdt_timestep(self.h, C.byref(t)), "bdt_timestep")
        return {"next_dt": t.next_dt, "elapsed_dt": t.elapsed_dt, "total_dt": t.total_dt, "num_rungs": t.num_rungs,
                "substep": t.substep, "rung_ranges": list(t.rung_ranges), "dt_m1": list(t.dt_m1),
                "dt_drift": list(t.dt_drift), "num_active": t.num_active}

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        L.check(self.lib.sphb_sim_get_field(self.h, name.encode(), L.ptr(out), 0), f"get_field({name})")
        if name in ("keys", "id", "rung"):
            return out.view(np.uint64)
        return out

    def get_device(self, name: str, out) -> None:
        """Copy a field as doubles into a device buffer (torch tensor)."""
        L.check(self.lib.sphb_sim_get_field(self.h, name.encode(), L.ptr(out), 1), f"get_field({name})")

    def set(self, name: str, values: np.ndarray):
        v = np.ascontiguousarray(values, dtype=np.float64)
        L.check(self.lib.sphb_sim_set_field(self.h, name.encode(), L.ptr(v), 0), f"set_field({name})")

    def keys(self) -> np.ndarray:
        return self.get("keys")

    def scalars(self) -> dict:
        out = np.empty(len(SCALAR_NAMES))
        L.check(self.lib.sphb_sim_scalars(self.h, L.ptr(out)), "scalars")
        return dict(zip(SCALAR_NAMES, out.tolist()))

    def tree(self):
        nl = C.c_size_t()
        L.check(self.lib.sphb_sim_tree(self.h, C.byref(nl), None, None, None), "tree")
        leaves = np.empty(nl.value + 1, dtype=np.uint64)
        counts = np.empty(nl.value, dtype=np.uint32)
        layout = np.empty(nl.value + 1, dtype=np.uint32)
        L.check(self.lib.sphb_sim_tree(self.h, C.byref(nl), L.ptr(leaves), L.ptr(counts), L.ptr(layout)), "tree")
        return leaves, counts, layout

    def neighbors(self) -> np.ndarray:
        out = np.empty((self.n, int(self.params["ngmax"])), dtype=np.uint32)
        L.check(self.lib.sphb_sim_neighbors(self.h, L.ptr(out)), "neighbors")
        return out

    def stage_times(self) -> dict:
        out = np.empty(len(STAGE_NAMES), dtype=np.float32)
        L.check(self.lib.sphb_sim_stage_times(self.h, L.ptr(out)), "stage_times")
        return dict(zip(STAGE_NAMES, out.tolist()))

    def search_stats(self) -> dict:
        """How the neighbour stage ran: tree searches of every group, skin-row builds, steps served from the skin
        rows, groups those steps deferred to the tree search, and syncs that moved particles while rows were kept."""
        out = np.zeros(5, dtype=np.uint64)
        L.check(self.lib.sphb_sim_search_stats(self.h, L.ptr(out)), "search_stats")
        return dict(zip(("tree_searches", "skin_builds", "skin_steps", "deferred_groups", "remapped_syncs"),
                        (int(v) for v in out)))

    def kernel_launches(self) -> int:
        return int(self.lib.sphb_sim_kernel_launches(self.h))

    def set_fixed_dt(self, dt: float):
        L.check(self.lib.sphb_sim_set_fixed_dt(self.h, float(dt)), "set_fixed_dt")

    def set_params(self, **over):
        """Change physics parameters between steps (gamma, mui, Kcour, Krho, alphamin, alphamax, decay_constant)."""
        self.params.update(over)
        prec = L.SPHB_MIXED if self.precision == "mixed" else L.SPHB_FP64
        prm = L.make_params(self.params, prec)
        L.check(self.lib.sphb_sim_set_params(self.h, C.byref(prm)), "set_params")

    def store_state(self, fields, ids, on_device: bool = True):
        """Copy the 14 conserved fields (CONSERVED_FIELDS order) and ids into the given buffers."""
        tbl = (C.c_void_p * len(fields))(*[L.ptr(f).value for f in fields])
        L.check(self.lib.sphb_sim_store_state(self.h, tbl, L.ptr(ids), int(on_device)), "store_state")

    def load_state(self, fields, ids, on_device: bool = True):
        tbl = (C.c_void_p * len(fields))(*[L.ptr(f).value for f in fields])
        L.check(self.lib.sphb_sim_load_state(self.h, tbl, L.ptr(ids), int(on_device)), "load_state")

    def step_vjp(self, adj_post, adj_pre) -> float:
        """Adjoint of one step from the current state (see sphb_sim_step_vjp); returns d/d alphamax."""
        post = (C.c_void_p * len(adj_post))(*[L.ptr(f).value for f in adj_post])
        pre = (C.c_void_p * len(adj_pre))(*[L.ptr(f).value for f in adj_pre])
        am = C.c_double(0.0)
        L.check(self.lib.sphb_sim_step_vjp(self.h, post, pre, C.byref(am)), "step_vjp")
        return am.value

    def tape_reserve(self, slots: int):
        L.check(self.lib.sphb_sim_tape_reserve(self.h, int(slots)), "tape_reserve")

    def step_record(self, slot: int) -> int:
        rc = self.lib.sphb_sim_step_record(self.h, int(slot))
        if rc not in (L.SPHB_OK, 4):
            L.check(rc, "step_record")
        return rc

    def step_vjp_recorded(self, slot: int, adj_post, adj_pre) -> float:
        post = (C.c_void_p * len(adj_post))(*[L.ptr(f).value for f in adj_post])
        pre = (C.c_void_p * len(adj_pre))(*[L.ptr(f).value for f in adj_pre])
        am = C.c_double(0.0)
        L.check(self.lib.sphb_sim_step_vjp_recorded(self.h, int(slot), post, pre, C.byref(am)), "step_vjp_recorded")
        return am.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.sphb_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
