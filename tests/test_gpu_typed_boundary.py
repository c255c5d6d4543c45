"""The typed boundary: particle fields in the caller's own element types, and the force stages run in place on a
caller's device arrays bound by the reference's field names (the drop-in for sph::gpu::computeXMass ...
computeMomentumEnergy, computePositionsGpu and updateSmoothingLengthGpu, sph/include/sph/sph_gpu.hpp:24-87).

* With every bound array in FP64, one whole step through the sphb_dataset_* entry points equals sphb_sim_step bit for
  bit: the same kernels run on the same values.
* With the reference's default types (sph/types.hpp:39-46: coordinates, temp and du double; hydro fields, mass,
  x_m1 and du_m1 float), the step agrees with sphb_sim_step on the same float-rounded state to float resolution, and
  the typed upload, load and store convert exactly as a cast would.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONSERVED = ("x", "y", "z", "h", "m", "temp", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha")
DERIVED = ("xm", "kx", "gradh", "prho", "c", "c11", "c12", "c13", "c22", "c23", "c33", "divv", "curlv", "ax", "ay",
           "az")
#: the reference's default SphTypes: which fields are double (the rest of the real fields are float)
DOUBLE_FIELDS = {"x", "y", "z", "temp", "du"}


@pytest.fixture(scope="module")
def lib(cuda_device):
    from sphexa_b200 import lib as L
    return L.load()


def _dataset(sim, torch, typed):
    """The caller's Dataset on the device: sim's current state and empty derived fields, in FP64 or in the
    reference's default types."""
    n = sim.n
    d = {}

    def real(name):
        return torch.float64 if (not typed or name in DOUBLE_FIELDS) else torch.float32

    for f in CONSERVED:
        d[f] = torch.from_numpy(sim.get(f)).to(device="cuda", dtype=real(f))
    d["id"] = torch.from_numpy(sim.get("id").view(np.int64)).cuda()
    for f in DERIVED + ("du",):
        d[f] = torch.zeros(n, dtype=real(f), device="cuda")
    d["nc"] = torch.zeros(n, dtype=torch.int32, device="cuda")
    d["keys"] = torch.zeros(n, dtype=torch.int64, device="cuda")
    d["rho"] = torch.zeros(n, dtype=real("rho"), device="cuda")
    d["p"] = torch.zeros(n, dtype=real("p"), device="cuda")
    return d


def _bound_step(lib, L, sim_b, d, box, params, min_dt, dt, dt_m1):
    n = sim_b.n
    h = sim_b.h
    L.check(lib.sphb_dataset_xmass(h, 0, n, C.byref(box)), "xmass")
    L.check(lib.sphb_dataset_ve_def_gradh(h, 0, n, C.byref(box)), "ve_def_gradh")
    eos = L.make_fields({f: d[f] for f in ("temp", "m", "kx", "xm", "gradh", "prho", "c", "rho", "p")})
    # on the simulation's stream, so that the next stage reads its outputs
    L.check(lib.sphb_ideal_gas_eos(0, n, params["mui"], params["gamma"], eos, len(eos), lib.sphb_sim_stream(h)),
            "eos")
    L.check(lib.sphb_dataset_iad_divv_curlv(h, 0, n, C.byref(box)), "iad")
    L.check(lib.sphb_dataset_av_switches(h, 0, n, C.byref(box), min_dt), "av")
    courant = C.c_float()
    L.check(lib.sphb_dataset_momentum_energy(h, 0, n, C.byref(box), C.byref(courant)), "momentum_energy")
    forces = {f: d[f].double().cpu().numpy().copy() for f in ("h", "nc", "xm", "kx", "gradh", "prho", "c", "c11",
                                                              "c33", "divv", "curlv", "alpha", "ax", "ay", "az",
                                                              "du", "rho", "p")}
    L.check(lib.sphb_dataset_positions(h, 0, n, dt, dt_m1, C.byref(box)), "positions")
    rc = lib.sphb_dataset_update_h(h, 0, n, int(params["ng0"]))
    assert rc == L.SPHB_OK
    return forces, courant.value


FORCE_FIELDS = ("h", "nc", "xm", "kx", "gradh", "prho", "c", "c11", "c33", "divv", "curlv", "alpha", "ax", "ay",
                "az", "du")


def test_fp64_dataset_step_equals_sim_step(lib):
    """Every bound array FP64: the forces of sphb_dataset_* and then the integrated state equal those of
    sphb_sim_compute_forces / sphb_sim_integrate bit for bit (Sedov 20^3, two steps)."""
    import torch
    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(20)
    a = Simulation(ic, "fp64")
    b = Simulation(ic, "fp64", initial_sync=False)
    box = L.make_box(ic["box"], [1, 1, 1])
    d = _dataset(a, torch, typed=False)
    tbl = L.make_fields(d)
    L.check(lib.sphb_sim_bind_fields(b.h, tbl, len(tbl)), "bind")
    for step in range(2):
        min_dt = a.scalars()["minDt"]
        a.compute_forces()
        fa = {f: a.get(f) for f in FORCE_FIELDS}
        sa = a.scalars()
        a.integrate()
        dt = a.scalars()["minDt"]
        forces, courant = _bound_step(lib, L, b, d, box, ic["params"], min_dt, dt, min_dt)
        for f in FORCE_FIELDS:
            assert np.array_equal(forces[f], fa[f]), (step, f)
        assert courant == np.float32(sa["minDtCourant"])
        rho = fa["kx"] * d["m"].cpu().numpy() / fa["xm"]
        assert np.allclose(forces["rho"], rho, rtol=1e-15, atol=0)
        for f in CONSERVED:
            assert np.array_equal(d[f].cpu().numpy(), a.get(f)), (step, f)


def test_reference_typed_dataset_step(lib):
    """The reference's default types (float hydro fields): one step through the bound entry points against
    sphb_sim on the same float-rounded state, uploaded through the typed upload. Neighbour counts are equal, h is
    the simulation's rounded to float, the other force outputs agree to 1e-5 of each field's largest magnitude (the
    stages read each other's outputs rounded to float), and the Courant step to 1e-6."""
    import torch
    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(20)
    seed = Simulation(ic, "fp64")
    for _ in range(3):
        seed.step()
    d = _dataset(seed, torch, typed=True)
    b = Simulation(ic, "fp64", initial_sync=False)
    a = Simulation(ic, "fp64", initial_sync=False)
    # the simulation object gets the same float-rounded state through the typed upload
    up = L.make_fields({f: d[f] for f in CONSERVED + ("id",)})
    L.check(lib.sphb_sim_upload_fields(a.h, up, len(up), 1), "upload_fields")
    a.initial_sync()
    box = L.make_box(ic["box"], [1, 1, 1])
    tbl = L.make_fields(d)
    L.check(lib.sphb_sim_bind_fields(b.h, tbl, len(tbl)), "bind")
    min_dt = seed.scalars()["minDt"]
    # give the simulation object the seed's previous time step (read by the AV switches), then the adaptive step again
    a.set_fixed_dt(min_dt)
    a.set_fixed_dt(0.0)
    a.compute_forces()
    sa = a.scalars()
    fa = {f: a.get(f) for f in FORCE_FIELDS}
    dt = min(sa["minDtCourant"], sa["minDtRho"], 1.1 * min_dt)
    forces, courant = _bound_step(lib, L, b, d, box, ic["params"], min_dt, dt, min_dt)
    assert np.array_equal(forces["nc"], fa["nc"])
    assert np.array_equal(forces["h"], np.float32(fa["h"]).astype(np.float64))
    for f in ("xm", "kx", "gradh", "prho", "c", "c11", "c33", "divv", "curlv", "alpha", "ax", "ay", "az", "du"):
        scale = float(np.max(np.abs(fa[f])))
        err = float(np.max(np.abs(forces[f] - fa[f]))) / scale
        assert err < 1e-5, (f, err)
    assert abs(courant - sa["minDtCourant"]) <= 1e-6 * sa["minDtCourant"]


def test_typed_store_and_load_round_trip(lib):
    """sphb_sim_store_fields converts as a cast; sphb_sim_load_fields of the stored typed state and a step give the
    same result as sphb_sim_load_state of the cast FP64 values."""
    import torch
    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(16)
    a = Simulation(ic, "mixed")
    a.step()
    n = a.n
    host = {}
    for f in CONSERVED:
        host[f] = np.zeros(n, dtype=np.float64 if f in DOUBLE_FIELDS else np.float32)
    host["id"] = np.zeros(n, dtype=np.uint64)
    host["nc"] = np.zeros(n, dtype=np.uint32)
    host["kx"] = np.zeros(n, dtype=np.float32)
    tbl = L.make_fields(host)
    L.check(lib.sphb_sim_store_fields(a.h, tbl, len(tbl), 0), "store_fields")
    for f in CONSERVED + ("kx",):
        assert np.array_equal(host[f], a.get(f).astype(host[f].dtype)), f
    assert np.array_equal(host["id"], a.get("id"))
    assert np.array_equal(host["nc"], a.get("nc").astype(np.uint32))
    # load the typed state back (host memory) and step; the same as loading the cast values as FP64
    b = Simulation(ic, "mixed")
    b.step()
    up = L.make_fields({f: host[f] for f in CONSERVED + ("id",)})
    L.check(lib.sphb_sim_load_fields(a.h, up, len(up), 0), "load_fields")
    fields = [torch.from_numpy(host[f].astype(np.float64)).cuda() for f in CONSERVED]
    ids = torch.from_numpy(host["id"].view(np.int64)).cuda()
    b.load_state(fields, ids)
    a.step()
    b.step()
    for f in CONSERVED:
        assert np.array_equal(a.get(f), b.get(f)), f


def _shuffle(bufs, seed):
    """the same random particle order for every array of every buffer set (host or device tensors)"""
    import torch
    n = next(iter(bufs[0].values())).numel()
    perm = torch.from_numpy(np.random.default_rng(seed).permutation(n))
    for d in bufs:
        for f, t in d.items():
            t.copy_(t[perm.to(t.device)].clone())


def test_host_load_overlapped_copies_equal_device_load(lib):
    """A typed load from host memory leaves h and the ids in flight beside the next step's sync, temp, v and alpha
    beside the search and XMass (VeDefGradh then leaves the velocities of its hydro record to a later kernel), and
    x_m1, y_m1, z_m1 and du_m1 beside the J-loops. Seven round trips (store to pinned host
    buffers in the reference's default types, load, step) give the same states, bit for bit, as the same round trips
    through device buffers, where every copy is ordered on the simulation's stream. Twice the stored particles are
    shuffled before the load: the sync then reorders all of them while the late fields are still in flight (they
    are gathered once they arrive), and the ids no longer match the skin rows, which both simulations drop alike."""
    import torch
    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(24)
    a = Simulation(ic, "mixed")
    b = Simulation(ic, "mixed")
    n = a.n

    def buffers(pinned):
        kw = {"pin_memory": True} if pinned else {"device": "cuda"}
        d = {f: torch.empty(n, dtype=torch.float64 if f in DOUBLE_FIELDS else torch.float32, **kw) for f in CONSERVED}
        d["id"] = torch.empty(n, dtype=torch.int64, **kw)
        return d

    ha, db = buffers(True), buffers(False)
    ta, tb = L.make_fields(ha), L.make_fields(db)
    for step in range(7):
        L.check(lib.sphb_sim_store_fields(a.h, ta, len(ta), 0), "store host")
        L.check(lib.sphb_sim_store_fields(b.h, tb, len(tb), 1), "store device")
        if step in (3, 5):
            torch.cuda.synchronize()
            _shuffle([ha, db], step)
            torch.cuda.synchronize()
        L.check(lib.sphb_sim_load_fields(a.h, ta, len(ta), 0), "load host")
        L.check(lib.sphb_sim_load_fields(b.h, tb, len(tb), 1), "load device")
        a.step()
        b.step()
        for f in CONSERVED:
            assert np.array_equal(a.get(f), b.get(f)), (step, f)
        assert np.array_equal(a.get("id"), b.get("id"))
    assert a.scalars()["minDt"] == b.scalars()["minDt"]
    assert a.search_stats() == b.search_stats()
    assert a.search_stats()["skin_builds"] >= 3, a.search_stats()


@pytest.mark.parametrize("types,precision", [("reference", "mixed"), ("double", "mixed"), ("float", "fp64")])
def test_step_fields_equals_load_step_store(lib, types, precision):
    """sphb_sim_step_fields (the load, the step and the store in one call, with m, id, alpha and h copied out while
    the later stages run) gives the same host state as the three calls one after another, over five round trips with
    the same pinned arrays as input and output. The caller's arrays have the reference's default types (a mix of
    float and double), or all double (no conversion on either side), or all float (every field converted)."""
    import torch
    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(24)
    a = Simulation(ic, precision)
    b = Simulation(ic, precision)
    n = a.n

    def dtype_of(f):
        if types == "double":
            return torch.float64
        if types == "float":
            return torch.float32
        return torch.float64 if f in DOUBLE_FIELDS else torch.float32

    def buffers():
        d = {f: torch.empty(n, dtype=dtype_of(f), pin_memory=True) for f in CONSERVED}
        d["id"] = torch.empty(n, dtype=torch.int64, pin_memory=True)
        return d

    ha, hb = buffers(), buffers()
    ta, tb = L.make_fields(ha), L.make_fields(hb)
    L.check(lib.sphb_sim_store_fields(a.h, ta, len(ta), 0), "store a")
    L.check(lib.sphb_sim_store_fields(b.h, tb, len(tb), 0), "store b")
    for step in range(5):
        if step == 2:
            _shuffle([ha, hb], step)
        L.check(lib.sphb_sim_step_fields(a.h, ta, len(ta), ta, len(ta)), "step_fields")
        L.check(lib.sphb_sim_load_fields(b.h, tb, len(tb), 0), "load")
        b.step()
        L.check(lib.sphb_sim_store_fields(b.h, tb, len(tb), 0), "store")
        for f in list(CONSERVED) + ["id"]:
            assert np.array_equal(ha[f].numpy(), hb[f].numpy()), (step, f)
    for f in CONSERVED:
        assert np.array_equal(a.get(f), b.get(f)), f
    assert a.scalars()["minDt"] == b.scalars()["minDt"]
    assert a.search_stats() == b.search_stats()
