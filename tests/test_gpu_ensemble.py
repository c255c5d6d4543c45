"""GPU tests of the batched ensemble (sphb_ensemble): every instance must evolve bit for bit as a single simulation
of the same initial conditions (same sort order, same neighbour lists, same arithmetic, same time steps), with the
step replayed from a captured CUDA graph or issued eagerly, and after the launch-shape autotuner ran."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "h", "temp", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha", "id", "nc")


def _ics():
    from sphexa_b200 import ic as icm
    return [icm.sedov(12, seed=3, energy=1.0, gamma=5.0 / 3.0),
            icm.sedov(17, seed=4, energy=0.7, gamma=1.4),
            icm.sedov(14, seed=5, energy=1.6, gamma=5.0 / 3.0)]


@pytest.mark.parametrize("precision,graph,av_clean", [("mixed", True, False), ("fp64", False, False),
                                                     ("mixed", True, True)])
def test_ensemble_matches_single_simulations(cuda_device, precision, graph, av_clean):
    from sphexa_b200.ensemble import Ensemble
    from sphexa_b200.simulation import Simulation
    ics = _ics()
    for ic in ics:
        ic["params"] = dict(ic["params"], avClean=av_clean)
    steps = 4
    ens = Ensemble(ics, precision)
    assert ens.step(steps, graph=graph) == 0
    for k, ic in enumerate(ics):
        sim = Simulation(ic, precision)
        for _ in range(steps):
            sim.step()
        for f in FIELDS:
            a, b = ens.get(k, f), sim.get(f)
            assert np.array_equal(a, b), (k, f)
        se, ss = ens.scalars(k), sim.scalars()
        for s in ("minDt", "minDt_m1", "ttot"):
            assert se[s] == ss[s], (k, s, se[s], ss[s])
        assert abs(se["etot"] - ss["etot"]) <= 1e-12 * abs(ss["etot"])
        sim.close()
    ens.close()


def test_autotune_then_graph_steps(cuda_device):
    from sphexa_b200.ensemble import Ensemble
    from sphexa_b200.simulation import Simulation
    ics = _ics()
    ens = Ensemble(ics, "mixed")
    choice = ens.autotune()
    assert all(t in (64, 128, 256) for t in choice.values())
    ens.step(2, graph=True)
    ens.rebuild_trees()
    ens.step(1, graph=True)
    for k, ic in enumerate(ics):
        sim = Simulation(ic, "mixed")
        for _ in range(3):
            sim.step()
        for f in FIELDS:
            assert np.array_equal(ens.get(k, f), sim.get(f)), (k, f)
        sim.close()
    ens.close()


def test_ensemble_skin_rows_match_tree_searches(cuda_device):
    """The ensemble's skin rows (mode chosen on the device every replay of the captured step) against single
    simulations that search the tree every step: identical states after 12 steps. One member has a stirred region,
    so that some of its groups are deferred (each member has its own displacement grid, so the others are not) and
    its particles change index between steps."""
    import copy
    from sphexa_b200.ensemble import Ensemble
    from sphexa_b200.simulation import Simulation
    ics = _ics()
    rng = np.random.default_rng(9)
    st = ics[1]
    inside = np.sqrt(st["x"] ** 2 + st["y"] ** 2 + st["z"] ** 2) < 0.08
    for k in ("vx", "vy", "vz"):
        v = np.zeros_like(st["x"])
        v[inside] = rng.uniform(-20.0, 20.0, inside.sum())
        st[k] = v
    st["params"] = dict(st["params"], minDt=1e-4, minDt_m1=1e-4)
    steps = 12
    ens = Ensemble(ics, "mixed")
    assert ens.step(steps, graph=True) == 0
    stats = ens.search_stats()
    assert stats["skin_steps"] >= 5 and stats["deferred_groups"] > 0, stats
    for k, ic in enumerate(ics):
        plain = copy.deepcopy(ic)
        plain["params"]["nbSkin"] = 0.0
        sim = Simulation(plain, "mixed")
        for _ in range(steps):
            sim.step()
        assert sim.search_stats()["skin_steps"] == 0
        for f in FIELDS:
            assert np.array_equal(ens.get(k, f), sim.get(f)), (k, f)
        sim.close()
    ens.close()
    print(stats)
