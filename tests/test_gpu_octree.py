"""Row a5: the linked octree in the reference's own layout. sphb_build_octree against the reference's CPU build of
OctreeData (buildOctreeCpu, cstone/tree/octree.hpp:170-196, compiled in oracle/_ref): prefixes, childOffsets,
parents, levelRange, internalToLeaf and leafToInternal bit-exact, for shallow and deep trees."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(cuda_device):
    from sphexa_b200 import lib as L
    return L.load()


@pytest.fixture(scope="module")
def ref():
    from oracle import refsim
    if not refsim.available():
        pytest.skip("reference oracle not built")
    return refsim


def _ours(lib, leaves):
    import torch
    from sphexa_b200 import lib as L
    nl = leaves.size - 1
    nn = nl + (nl - 1) // 7
    dl = torch.from_numpy(leaves.view(np.int64).copy()).cuda()
    pre = torch.zeros(nn, dtype=torch.int64, device="cuda")
    co = torch.zeros(nn, dtype=torch.int32, device="cuda")
    par = torch.zeros(max(1, (nn - 1) // 8), dtype=torch.int32, device="cuda")
    i2l = torch.zeros(nn, dtype=torch.int32, device="cuda")
    l2i = torch.zeros(nn, dtype=torch.int32, device="cuda")
    lr = np.zeros(23, dtype=np.int32)
    L.check(lib.sphb_build_octree(L.ptr(dl), nl, L.ptr(pre), L.ptr(co), L.ptr(par), L.ptr(lr), L.ptr(i2l), L.ptr(l2i),
                                  None), "build_octree")
    return {"prefixes": pre.cpu().numpy().view(np.uint64), "childOffsets": co.cpu().numpy(),
            "parents": par.cpu().numpy(), "levelRange": lr, "internalToLeaf": i2l.cpu().numpy(),
            "leafToInternal": l2i.cpu().numpy()}


@pytest.mark.parametrize("dist,n,bucket", [("uniform", 100_000, 64), ("gauss", 300_000, 16), ("gauss", 20_000, 1),
                                           ("one", 1, 64)])
def test_octree_layout_bit_exact(lib, ref, dist, n, bucket):
    rng = np.random.default_rng(n + bucket)
    if dist == "uniform":
        p = rng.uniform(-0.5, 0.5, (n, 3))
    elif dist == "gauss":
        p = np.clip(rng.normal(0, 0.05, (n, 3)), -0.4999, 0.4999)
    else:
        p = np.zeros((n, 3))
    keys = np.sort(ref.sfc_keys(p[:, 0], p[:, 1], p[:, 2], (-0.5, 0.5, -0.5, 0.5, -0.5, 0.5), True))
    leaves, _ = ref.compute_octree(keys, bucket)
    want = ref.build_octree(leaves)
    got = _ours(lib, leaves)
    for k in ("prefixes", "childOffsets", "parents", "levelRange", "internalToLeaf", "leafToInternal"):
        assert np.array_equal(got[k], want[k]), k


def test_octree_layout_of_the_simulation_focus_tree(lib, ref):
    """the focus tree of a running simulation (Sedov 24^3 after two steps)"""
    from sphexa_b200 import ic as icm
    from sphexa_b200.simulation import Simulation
    s = Simulation(icm.sedov(24), "fp64")
    s.step()
    s.step()
    leaves, _, _ = s.tree()
    want = ref.build_octree(leaves)
    got = _ours(lib, leaves)
    for k in want:
        assert np.array_equal(got[k], want[k]), k
