"""Skin lists: candidate rows found once within 2h(1 + skin) and refiltered exactly every step. Every step's
neighbour lists, counts and smoothing lengths must equal those of the tree search of every step bit for bit, so the
trajectories with and without the rows are identical. The cases cover rows served for many steps (Sedov), particles
that change index between steps and groups deferred to the tree search (a stirred region), and flows that move
everywhere, where the rows are dropped for plain tree searches (Noh)."""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(ic, precision, skin=0.05):
    from sphexa_b200.simulation import Simulation
    a_ic = copy.deepcopy(ic)
    a_ic["params"]["nbSkin"] = skin
    b_ic = copy.deepcopy(ic)
    b_ic["params"]["nbSkin"] = 0.0
    return Simulation(a_ic, precision), Simulation(b_ic, precision)


def _same_lists(a, b, step):
    nca = a.get("nc").astype(np.int64)
    assert np.array_equal(nca, b.get("nc").astype(np.int64)), step
    assert np.array_equal(a.get("h"), b.get("h")), step
    assert np.array_equal(a.get("id"), b.get("id")), step
    la, lb = a.neighbors(), b.neighbors()
    ngmax = la.shape[1]
    used = np.arange(ngmax)[None, :] < np.minimum(nca - 1, ngmax)[:, None]
    assert np.array_equal(la[used], lb[used]), step


def _run(a, b, steps):
    from sphexa_b200.ic import CONSERVED_FIELDS
    for step in range(steps):
        a.compute_forces()
        b.compute_forces()
        _same_lists(a, b, step)
        a.integrate()
        b.integrate()
    for f in CONSERVED_FIELDS:
        assert np.array_equal(a.get(f), b.get(f)), f
    assert a.scalars()["ttot"] == b.scalars()["ttot"]


def _stirred(side, seed=3, radius=0.15, speed=20.0, centre=(0.0, 0.0, 0.0)):
    """Sedov lattice with random velocities inside a sphere (minimum image around `centre`): particles there cross
    each other (indices change between steps) while the rest is at rest."""
    from sphexa_b200 import ic as icm
    ic = icm.sedov(side, seed=seed)
    rng = np.random.default_rng(seed)
    d = [ic[k] - c for k, c in zip(("x", "y", "z"), centre)]
    d = [v - np.round(v) for v in d]
    r = np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
    inside = r < radius
    for k in ("vx", "vy", "vz"):
        v = np.zeros_like(r)
        v[inside] = rng.uniform(-speed, speed, inside.sum())
        ic[k] = v
    ic["temp"] = np.full_like(r, ic["temp"].min())
    ic["params"]["minDt"] = ic["params"]["minDt_m1"] = 1e-4
    return ic


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_skin_sedov(cuda_device, precision):
    from sphexa_b200 import ic as icm
    a, b = _pair(icm.sedov(32), precision)
    _run(a, b, 25)
    st = a.search_stats()
    assert st["skin_steps"] >= 20, st
    assert b.search_stats()["skin_steps"] == 0


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_skin_stirred(cuda_device, precision):
    """A small stirred region: its groups are deferred every step while the rest is served from the rows, and the
    sort moves particles between steps (rows remapped)."""
    a, b = _pair(_stirred(40, radius=0.08), precision)
    _run(a, b, 16)
    st = a.search_stats()
    print(st)
    assert st["skin_steps"] >= 5 and st["deferred_groups"] > 0 and st["remapped_syncs"] > 0, st


def test_skin_stirred_across_the_periodic_boundary(cuda_device):
    """The stirred region sits on the corner of the periodic box: displacements, grid cells and the region of each
    group wrap around."""
    a, b = _pair(_stirred(40, radius=0.08, centre=(0.5, 0.5, 0.5)), "mixed")
    _run(a, b, 16)
    st = a.search_stats()
    print(st)
    assert st["skin_steps"] >= 5 and st["deferred_groups"] > 0, st


def test_skin_stirred_wide(cuda_device):
    """A stirred region too large for the rows: they are dropped for plain tree searches."""
    a, b = _pair(_stirred(28, radius=0.15), "mixed")
    _run(a, b, 16)
    st = a.search_stats()
    print(st)
    assert st["tree_searches"] > 8, st


def test_skin_noh(cuda_device):
    from sphexa_b200 import ic as icm
    a, b = _pair(icm.noh(24), "mixed")
    _run(a, b, 12)
    print(a.search_stats())


def test_skin_params(cuda_device):
    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    a, _ = _pair(icm.sedov(12), "mixed")
    a.step()
    a.step()
    with pytest.raises(RuntimeError):
        a.set_params(nbSkin=0.1)
