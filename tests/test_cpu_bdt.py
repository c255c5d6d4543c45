"""CPU checks of the restated block time-step propagator (oracle/bdt.py): the rung helpers against the sequences
their reference definitions give, and the invariants of a block of substeps on a small Sedov run."""
import numpy as np
import pytest


def test_butterfly_and_active_rung():
    from oracle.bdt import active_rung, butterfly
    # cstone/primitives/math.hpp:34: the 1 2 1 3 1 2 1 4 pattern
    assert [butterfly(i) for i in range(1, 17)] == [1, 2, 1, 3, 1, 2, 1, 4, 1, 2, 1, 3, 1, 2, 1, 5]
    assert butterfly(0) == 0
    # four rungs: a block of 8 substeps, rung 0 alone on odd substeps, all rungs at the block's first substep
    assert [active_rung(s, 4) for s in range(9)] == [0, 1, 2, 1, 3, 1, 2, 1, 0]
    assert [active_rung(s, 1) for s in range(3)] == [0, 0, 0]
    assert [active_rung(s, 2) for s in range(3)] == [0, 1, 0]


def test_bdt_block_invariants():
    from oracle import restated
    if not restated.available():
        pytest.skip("oracle not built")
    from oracle.bdt import MAX_RUNGS, BdtOracle
    from sphexa_b200 import ic as icm
    o = BdtOracle(icm.sedov(14, seed=1))
    blocks = 0
    elapsed = 0.0
    for k in range(20):
        starts_block = o.ts.substep == 0 or o.ts.substep >= (1 << (o.ts.num_rungs - 1))
        assert o.step() == 0
        ts = o.ts
        if starts_block:
            blocks += 1
            elapsed = 0.0
            r = ts.rung_ranges
            assert r[0] == 0 and r[MAX_RUNGS] == o.num_groups
            assert all(r[i] <= r[i + 1] for i in range(MAX_RUNGS))
            # after the sort every group of rung q >= 1 has a time step of at least 2^q times the smallest
            base = o.group_dt[0]
            for q in range(1, ts.num_rungs):
                assert np.all(o.group_dt[r[q]:r[q + 1]] >= np.float32(1 << q) * base)
        elapsed += float(ts.next_dt)
        assert abs(float(ts.elapsed_dt) - elapsed) <= 1e-6 * elapsed
        assert int(o.rung.max()) < ts.num_rungs
        if ts.substep == (1 << (ts.num_rungs - 1)):
            # the block is complete: every rung has caught up, nothing is left drifting
            assert np.all(ts.dt_drift == 0)
            assert len(o.active) == o.num_groups or ts.num_rungs > 1
    assert blocks >= 2
    assert np.all(np.isfinite(o.get("x"))) and np.all(np.isfinite(o.get("temp")))
