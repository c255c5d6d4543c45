"""CPU tests of the host-side logic: the synthetic initial conditions, the bench's roofline, error and ensemble
helpers, and the parameter/box packing of the C ABI structs (no GPU calls)."""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_sedov_initial_conditions():
    from sphexa_b200 import ic as icm
    from sphexa_b200.adjoint import ideal_gas_cv
    for side, energy, gamma in ((12, 1.0, 5.0 / 3.0), (20, 0.7, 1.4)):
        ic = icm.sedov(side, seed=3, energy=energy, gamma=gamma)
        n = side ** 3
        assert ic["x"].size == n and np.array_equal(ic["id"], np.arange(n, dtype=np.uint64))
        assert math.isclose(ic["m"].sum(), 1.0, rel_tol=1e-12)
        for c in ("x", "y", "z"):
            assert np.all(np.abs(ic[c]) <= 0.5)
        cv = ideal_gas_cv(ic["params"]["mui"], gamma)
        u = ic["temp"] * cv
        # internal energy: the floor everywhere plus the deposited blast energy
        assert math.isclose(np.sum(ic["m"] * (u - 1e-8)), energy, rel_tol=1e-9)
        assert np.all(ic["vx"] == 0) and np.all(ic["alpha"] == ic["params"]["alphamin"])
        h0 = 0.5 * np.cbrt(3.0 / (4.0 * np.pi) * ic["params"]["ng0"] / n)
        assert np.allclose(ic["h"], h0)
    # the generator is deterministic and depends on the seed
    a, b, c = icm.sedov(10, seed=1), icm.sedov(10, seed=1), icm.sedov(10, seed=2)
    assert np.array_equal(a["x"], b["x"]) and not np.array_equal(a["x"], c["x"])


def test_noh_initial_conditions():
    from sphexa_b200 import ic as icm
    ic = icm.noh(24)
    r = np.sqrt(ic["x"] ** 2 + ic["y"] ** 2 + ic["z"] ** 2)
    assert np.all(r <= 0.5) and not ic["periodic"]
    v = np.stack([ic["vx"], ic["vy"], ic["vz"]])
    assert np.allclose(np.sqrt(np.sum(v * v, axis=0)), 1.0)
    # inward radial velocity, x_m1 = v dt0
    assert np.all(np.sum(v * np.stack([ic["x"], ic["y"], ic["z"]]), axis=0) <= 1e-12)
    assert np.allclose(ic["x_m1"], ic["vx"] * ic["params"]["minDt"])


def test_stage_rooflines_and_errors():
    import bench
    stages = {"neighbors": 2.0, "momentum_energy": 1.0, "sync": 1.0}
    per, t_roof = bench.stage_rooflines(stages, n=1000, pairs=100_000, precision="mixed", fma_peak_tf=10.0,
                                        hbm_gbs=1000.0)
    me = per["momentum_energy"]
    assert me["flops"] == 140 * 100_000
    assert me["bytes"] == 128 * 1000 + 4 * 100_000
    assert me["bound"] == "fp32"  # 1.4e7 flop at 10 TF/s (1.4 us) outlasts 5.28e5 B at 1 TB/s (0.53 us)
    assert per["sync"]["bound"] == "hbm" and per["sync"]["flops"] == 0
    assert abs(t_roof - sum(v["roof_ms"] for v in per.values())) <= 5e-4  # per-stage values are rounded to 1e-4 ms
    snap = {"id": np.arange(4, dtype=np.uint64), "kx": np.ones(4), "xm": np.ones(4), "m": np.ones(4),
            "temp": np.array([1.0, 2.0, 3.0, 4.0]), "h": np.ones(4)}
    for f in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        snap[f] = np.linspace(-1, 1, 4)
    other = {k: v.copy() for k, v in snap.items()}
    other["temp"][2] *= 1 + 1e-6
    err = bench.field_errors(other, snap)
    assert err["rho"]["max"] == 0.0 and math.isclose(err["u"]["max"], 1e-6, rel_tol=1e-6)


def test_ensemble_config_deterministic():
    import bench
    s1, e1, g1 = bench.ensemble_config()
    s2, e2, g2 = bench.ensemble_config()
    assert s1 == s2 and e1 == e2 and g1 == g2
    assert len(s1) == 64 and min(s1) >= 20 and max(s1) <= 64
    assert all(0.5 <= e <= 2.0 for e in e1) and set(g1) <= {1.4, 5.0 / 3.0}


def test_param_and_box_packing():
    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    p = dict(icm.default_params(), avClean=True)
    prm = L.make_params(p, L.SPHB_MIXED, bucket=32)
    assert prm.ng0 == 100 and prm.ngmax == 150 and prm.precision == L.SPHB_MIXED and prm.bucket_focus == 32
    assert prm.av_clean == 1 and prm.gamma == pytest.approx(5.0 / 3.0)
    b = L.make_box((-1, 1, -2, 2, -3, 3), [1, 0, 1])
    assert list(b.lo) == [-1, -2, -3] and list(b.hi) == [1, 2, 3] and list(b.periodic) == [1, 0, 1]
