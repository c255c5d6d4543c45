"""Spatial target groups (row a7): sphb_compute_group_splits against the reference's own kernels
(groupSplitsKernel + makeSplitsKernel of cstone/traversal/groups_gpu.cuh, compiled in oracle/_ref) and against the
numpy restatement of the oracle, bit-exact group boundaries. The inputs are particles in SFC order with their
cornerstone tree: a Sedov lattice after a few steps, and clumped particles whose runs really split."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(cuda_device):
    from sphexa_b200 import lib as L
    return L.load()


@pytest.fixture(scope="module")
def ref_groups():
    from oracle import groups
    if not groups.reference_available():
        pytest.skip("reference group kernels not built")
    return groups


def _ours(lib, x, y, z, h, leaves, layout, box, periodic, group_size, h_float):
    import torch
    from sphexa_b200 import lib as L
    n = x.size
    dx, dy, dz = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (x, y, z))
    dh = None
    if h is not None:
        dh = torch.from_numpy(np.ascontiguousarray(h, dtype=np.float32 if h_float else np.float64)).cuda()
    dl = torch.from_numpy(leaves.view(np.int64).copy()).cuda()
    dy_ = torch.from_numpy(layout.astype(np.int32)).cuda()
    cap = n + 2
    out = torch.zeros(cap, dtype=torch.int32, device="cuda")
    num = C.c_size_t()
    b = L.make_box(box, [periodic] * 3)
    L.check(lib.sphb_compute_group_splits(0, n, L.ptr(dx), L.ptr(dy), L.ptr(dz), None if dh is None else L.ptr(dh),
                                          L.SPHB_F32 if h_float else L.SPHB_F64, L.ptr(dl), leaves.size - 1,
                                          L.ptr(dy_), C.byref(b), group_size, 2.0, L.ptr(out), cap, C.byref(num),
                                          None), "group splits")
    return out.cpu().numpy().view(np.uint32)[:num.value + 1].copy()


def _clumps(n, seed):
    """Gaussian clumps of different widths in the unit box, sorted by Hilbert key, with h from the local spacing."""
    from oracle import refsim
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-0.4, 0.4, (12, 3))
    widths = rng.uniform(0.005, 0.06, 12)
    which = rng.integers(0, 12, n)
    p = centers[which] + rng.normal(0, 1, (n, 3)) * widths[which, None]
    p = np.clip(p, -0.4999, 0.4999)
    box = (-0.5, 0.5, -0.5, 0.5, -0.5, 0.5)
    keys = refsim.sfc_keys(p[:, 0], p[:, 1], p[:, 2], box, True)
    order = np.argsort(keys, kind="stable")
    x, y, z = (np.ascontiguousarray(p[order, k]) for k in range(3))
    h = 0.5 * widths[which][order] * rng.uniform(0.5, 1.5, n)
    leaves, counts = refsim.compute_octree(keys[order], 64)
    layout = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    return x, y, z, h, leaves, layout, box


@pytest.mark.parametrize("group_size", [32, 64])
@pytest.mark.parametrize("h_float", [False, True])
def test_group_splits_clumps_bit_exact(lib, ref_groups, group_size, h_float):
    x, y, z, h, leaves, layout, box = _clumps(40_003, 7)
    hq = h.astype(np.float32) if h_float else h
    ref = ref_groups.reference_group_splits(x, y, z, hq, leaves, layout, box, True, group_size, 2.0, h_float)
    ours = _ours(lib, x, y, z, hq, leaves, layout, box, True, group_size, h_float)
    restated = ref_groups.group_splits(x, y, z, hq, leaves, layout, box, group_size, 2.0, h_float)
    num_fixed = (x.size + group_size - 1) // group_size
    assert ref.size - 1 > 1.05 * num_fixed  # the runs really split
    assert np.array_equal(ours, ref)
    assert np.array_equal(restated, ref)
    # without the smoothing-length criterion
    ref0 = ref_groups.reference_group_splits(x, y, z, None, leaves, layout, box, True, group_size, 2.0, h_float)
    assert np.array_equal(_ours(lib, x, y, z, None, leaves, layout, box, True, group_size, h_float), ref0)


@pytest.mark.parametrize("side", [20, 33])
def test_group_splits_sedov_bit_exact(lib, ref_groups, side):
    """The simulation's own state (SFC order, focus tree) after three steps; ragged last run at side 33."""
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(side)
    s = Simulation(ic, "fp64")
    for _ in range(3):
        s.step()
    x, y, z, h = (s.get(f) for f in ("x", "y", "z", "h"))
    leaves, counts, layout = s.tree()
    box = ic["box"]
    ref = ref_groups.reference_group_splits(x, y, z, h, leaves, layout, box, True, 32, 2.0, False)
    assert np.array_equal(_ours(lib, x, y, z, h, leaves, layout, box, True, 32, False), ref)
    assert np.array_equal(ref_groups.group_splits(x, y, z, h, leaves, layout, box, 32, 2.0, False), ref)
