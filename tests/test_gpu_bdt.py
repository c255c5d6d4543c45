"""GPU tests of the block time-step propagator (sphb_sim_bdt_*, main/src/propagator/ve_hydro_bdt.hpp) against its
restatement over the C oracle (oracle/bdt.py), substep by substep. The reference runs this propagator only on
GPUs, so the restatement is pinned through the oracle's J-loops (themselves pinned to the reference's CPU code), the
spatial groups (restated, and pinned to the reference's own group kernels in test_gpu_groups.py) and by reading the
cited sources. Integer state (rungs, rung ranges, particle order) must be equal; time steps are
float32 values that must agree to a few ulp; fields are compared by relative error with the tolerance in each test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(cuda_device):
    from sphexa_b200 import lib as L
    return L.load()


def _max_rel(a, b, floor=0.0):
    d = np.abs(a - b)
    s = np.maximum(np.abs(b), floor)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(s > 0, d / s, d)
    return float(np.max(r)) if r.size else 0.0


def _tree_of(g):
    """the focus tree of the CUDA path (pinned to the reference's by test_sedov_multi_step_fp64_vs_reference) for
    the restated propagator's spatial groups: after the GPU's substep, the tree of that substep's sync"""
    def tree():
        leaves, counts, layout = g.tree()
        return leaves, layout
    return tree


def _check_timestep(tg, to, where):
    assert tg["num_rungs"] == to["num_rungs"], where
    assert tg["substep"] == to["substep"], where
    assert tg["rung_ranges"] == to["rung_ranges"], (where, tg["rung_ranges"], to["rung_ranges"])
    for k in ("next_dt", "elapsed_dt", "total_dt"):
        assert abs(tg[k] - to[k]) <= 4e-7 * abs(to[k]), (where, k, tg[k], to[k])
    for k in ("dt_m1", "dt_drift"):
        assert np.allclose(tg[k], to[k], rtol=4e-7, atol=0), (where, k)


@pytest.mark.parametrize("skin", [0.0, 0.05])
def test_bdt_fp64_vs_oracle(lib, skin):
    """Twelve substeps of Sedov 20^3 (one block of 8 substeps over 4 rungs and the start of the next), with the tree
    searched every substep or skin rows refiltered."""
    from oracle.bdt import BdtOracle
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(20, seed=3)
    ic["params"] = dict(ic["params"], nbSkin=skin)
    g = Simulation(ic, "fp64")
    o = BdtOracle(ic, tree=_tree_of(g))
    g.enable_block_timesteps(0.2)
    rungs_seen = set()
    for k in range(12):
        assert g.bdt_step() == 0
        assert o.step() == 0
        tg, to = g.bdt_timestep(), o.ts.as_dict()
        _check_timestep(tg, to, k)
        rungs_seen.add(tg["num_rungs"])
        assert tg["num_active"] == len(o.active), k
        assert tg["rung_ranges"][4] == o.num_groups, k
        assert np.array_equal(g.get("id"), o.get("id")), k
        assert np.array_equal(g.get("rung"), o.rung.astype(np.uint64)), k
        assert np.array_equal(g.get("nc"), o.get("nc")), k
        for f in ("x", "y", "z", "temp"):
            assert _max_rel(g.get(f), o.get(f), floor=1e-3) < 1e-9, (k, f)
        assert _max_rel(g.get("h"), o.get("h")) < 1e-12, k
        for f in ("vx", "vy", "vz", "ax", "du", "alpha"):
            b = o.get(f)
            assert _max_rel(g.get(f), b, floor=1e-6 * np.max(np.abs(b))) < 1e-8, (k, f)
    assert max(rungs_seen) > 1
    if skin > 0:
        assert g.search_stats()["skin_steps"] >= 6


def test_bdt_first_substep_equals_global_forces(lib):
    """The first substep has every group active after a full sync: its forces are those of the global step."""
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(24, seed=5)
    a = Simulation(ic, "fp64")
    a.compute_forces()
    b = Simulation(ic, "fp64")
    b.enable_block_timesteps(0.2)
    b.bdt_step()
    for f in ("xm", "kx", "gradh", "prho", "c", "c11", "divv", "alpha", "ax", "ay", "az", "du", "nc"):
        assert np.array_equal(a.get(f), b.get(f)), f
    t = b.bdt_timestep()
    # every spatial group active (a uniform lattice has no gaps: its groups are the runs of 32)
    assert t["num_active"] == t["rung_ranges"][4] == (b.n + 31) // 32


def _with_gap(ic, lo=0.05, hi=0.2):
    """the lattice without the particles of the slab lo < x < hi: SFC runs that cross the gap split into several
    spatial groups"""
    keep = ~((ic["x"] > lo) & (ic["x"] < hi))
    out = dict(ic)
    for f, v in ic.items():
        if isinstance(v, np.ndarray) and v.shape == keep.shape:
            out[f] = v[keep]
    out["id"] = np.arange(int(keep.sum()), dtype=np.uint64)
    return out


def test_bdt_split_groups_vs_oracle(lib):
    """Spatial groups that really split (a slab of the Sedov lattice removed): ten substeps against the restated
    propagator, whose groups come from the restated group splits; the group counts, rung ranges, order and FP64
    fields agree."""
    from oracle.bdt import BdtOracle
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    ic = _with_gap(icm.sedov(20, seed=4))
    g = Simulation(ic, "fp64")
    o = BdtOracle(ic, tree=_tree_of(g))
    g.enable_block_timesteps(0.2)
    for k in range(10):
        assert g.bdt_step() == 0
        assert o.step() == 0
        tg, to = g.bdt_timestep(), o.ts.as_dict()
        _check_timestep(tg, to, k)
        assert tg["rung_ranges"][4] == o.num_groups, k
        assert tg["num_active"] == len(o.active), k
        assert np.array_equal(g.get("id"), o.get("id")), k
        assert np.array_equal(g.get("rung"), o.rung.astype(np.uint64)), k
        assert np.array_equal(g.get("nc"), o.get("nc")), k
        for f in ("x", "y", "z", "temp"):
            assert _max_rel(g.get(f), o.get(f), floor=1e-3) < 1e-9, (k, f)
        for f in ("vx", "ax", "du"):
            b = o.get(f)
            assert _max_rel(g.get(f), b, floor=1e-6 * np.max(np.abs(b))) < 1e-8, (k, f)
    assert o.num_groups > (g.n + 31) // 32 + 5  # the gap split runs
    assert g.bdt_timestep()["num_rungs"] > 1


def test_bdt_mixed_vs_oracle(lib):
    """Mixed precision through one block: the rung structure follows the FP64 restatement and the fields stay within
    the mixed form's tolerance."""
    from oracle.bdt import BdtOracle
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(20, seed=3)
    g = Simulation(ic, "mixed")
    o = BdtOracle(ic, tree=_tree_of(g))
    g.enable_block_timesteps(0.2)
    for k in range(8):
        assert g.bdt_step() == 0
        assert o.step() == 0
        tg, to = g.bdt_timestep(), o.ts.as_dict()
        assert tg["num_rungs"] == to["num_rungs"] and tg["rung_ranges"] == to["rung_ranges"], k
        assert abs(tg["next_dt"] - to["next_dt"]) <= 1e-5 * to["next_dt"], k
    for f in ("x", "y", "z"):
        assert _max_rel(g.get(f), o.get(f), floor=1e-3) < 1e-7, f
    for f in ("temp", "h"):
        assert _max_rel(g.get(f), o.get(f)) < 1e-5, f
    b = o.get("vx")
    assert _max_rel(g.get("vx"), b, floor=1e-3 * np.max(np.abs(b))) < 1e-4


@pytest.mark.parametrize("skin", [0.0, 0.05])
def test_bdt_periodic_drift_out_of_box(lib, skin):
    """A uniform flow across the periodic boundary: between full syncs particles drift past the box faces without
    folding and without a resort; the lists (and so nc and the forces) must still match the oracle's exact search,
    through the widened tree search and through the skin rows' wrapped displacement grid."""
    from oracle.bdt import BdtOracle
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(16, seed=9)
    ic["params"] = dict(ic["params"], nbSkin=skin)
    # a bulk flow of about one lattice spacing per block of substeps; Sedov's hot centre keeps several rungs
    ic["vx"] = ic["vx"] + 1.0e4
    ic["x_m1"] = ic["vx"] * ic["params"]["minDt"]
    g = Simulation(ic, "fp64")
    o = BdtOracle(ic, tree=_tree_of(g))
    g.enable_block_timesteps(0.2)
    outside = 0
    for k in range(10):
        assert g.bdt_step() == 0
        assert o.step() == 0
        _check_timestep(g.bdt_timestep(), o.ts.as_dict(), k)
        assert np.array_equal(g.get("nc"), o.get("nc")), k
        x = g.get("x")
        outside += int(np.sum((x > 0.5) | (x < -0.5)))
        assert _max_rel(x, o.get("x"), floor=1e-3) < 1e-9, k
        b = o.get("ax")
        assert _max_rel(g.get("ax"), b, floor=1e-6 * np.max(np.abs(b))) < 1e-8, k
    assert outside > 0  # the case this test is for happened


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bdt_open_box_vs_oracle(lib, precision):
    """Sedov in an open box with one face moving outward: the box follows the particles only at full syncs, so
    between them that face drifts past the box (fixed-point coordinates beyond the frame, clamped grid cells, the
    widened tree search). The moving face sits on the fastest rung, the interior on the slowest."""
    from oracle.bdt import BdtOracle
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(16, seed=2)
    ic["periodic"] = False
    face = ic["x"] > 0.44
    ic["vx"] = np.where(face, 2.0e4, 0.0)
    ic["x_m1"] = ic["vx"] * ic["params"]["minDt"]
    g = Simulation(ic, precision)
    o = BdtOracle(ic, tree=_tree_of(g))
    g.enable_block_timesteps(0.2)
    tight = precision == "fp64"
    xmax0 = float(np.max(ic["x"]))
    beyond = False
    for k in range(12):
        assert g.bdt_step() == 0
        assert o.step() == 0
        tg, to = g.bdt_timestep(), o.ts.as_dict()
        if tight:
            _check_timestep(tg, to, k)
        else:
            assert tg["num_rungs"] == to["num_rungs"] and tg["rung_ranges"] == to["rung_ranges"], k
        assert np.array_equal(g.get("nc"), o.get("nc")), k
        x = g.get("x")
        beyond = beyond or (tg["num_active"] < tg["rung_ranges"][4] and float(x.max()) > xmax0 + 0.005)
        for f in ("x", "y", "z"):
            assert _max_rel(g.get(f), o.get(f), floor=1e-3) < (1e-9 if tight else 1e-7), (k, f)
        b = o.get("ax")
        assert _max_rel(g.get("ax"), b, floor=1e-6 * np.max(np.abs(b))) < (1e-8 if tight else 1e-3), k
    assert g.bdt_timestep()["num_rungs"] > 1 and beyond


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bdt_av_clean_vs_oracle(lib, precision):
    """HydroVeBdtProp<avClean = true>: IAD keeps the symmetrised velocity gradients of the active groups and
    MomentumEnergy corrects r.v with them, inactive neighbours contributing their last gradients. One block over
    four rungs and the start of the next, against the restated propagator with AV cleaning."""
    from oracle.bdt import BdtOracle
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(20, seed=3)
    ic["params"] = dict(ic["params"], avClean=True)
    g = Simulation(ic, precision)
    o = BdtOracle(ic, tree=_tree_of(g))
    g.enable_block_timesteps(0.2)
    tight = precision == "fp64"
    for k in range(10):
        assert g.bdt_step() == 0
        assert o.step() == 0
        tg, to = g.bdt_timestep(), o.ts.as_dict()
        if tight:
            _check_timestep(tg, to, k)
        else:
            assert tg["num_rungs"] == to["num_rungs"] and tg["rung_ranges"] == to["rung_ranges"], k
        assert np.array_equal(g.get("nc"), o.get("nc")), k
        for f in ("x", "y", "z"):
            assert _max_rel(g.get(f), o.get(f), floor=1e-3) < (1e-9 if tight else 1e-7), (k, f)
        for f in ("dV11", "dV12", "dV23", "ax", "du"):
            # FP32 sums of velocity differences: normalised by the field's largest magnitude
            b = o.get(f)
            floor = (1e-6 if tight else 1e-3) * np.max(np.abs(b))
            assert _max_rel(g.get(f), b, floor=floor) < (1e-8 if tight else 1e-3), (k, f)
    assert g.bdt_timestep()["num_rungs"] > 1


def test_bdt_state_errors(lib):
    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(12)
    g = Simulation(ic, "fp64")
    with pytest.raises(L.SphbError) as e:
        g.bdt_timestep()
    assert e.value.code == L.SPHB_ERR_STATE
    with pytest.raises(L.SphbError):
        g.enable_block_timesteps(0.0)
    g.enable_block_timesteps(0.2)
    with pytest.raises(L.SphbError) as e:
        g.compute_forces()
    assert e.value.code == L.SPHB_ERR_STATE
    with pytest.raises(L.SphbError) as e:
        g.sync()
    assert e.value.code == L.SPHB_ERR_STATE
