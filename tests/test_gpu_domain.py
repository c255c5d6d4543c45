"""The multi-rank domain's device steps (sphb_leaf_counts, sphb_rebalance_tree, sphb_find_halos) against the
reference's own functions compiled in oracle/_ref, bit for bit; and the whole Domain.sync / exchange_halos with its
CUDA engine for two and three ranks on one GPU, the ranks being threads of this process that communicate through
host queues (no kernel of one rank waits for another rank), checked like the gloo CPU test against the single-rank
result."""
import ctypes as C
import os
import sys
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


@pytest.fixture(scope="module")
def lib(cuda_device):
    from oracle import refsim
    if not refsim.available():
        pytest.skip("reference oracle not built")
    from sphexa_b200 import lib as L
    return L.load()


def _clumps(n, seed, periodic):
    rng = np.random.default_rng(seed)
    centers = rng.uniform(0.1, 0.9, (8, 3))
    which = rng.integers(0, 8, n)
    p = centers[which] + rng.normal(0, 1, (n, 3)) * rng.uniform(0.02, 0.15, 8)[which, None]
    p = np.mod(p, 1.0) if periodic else np.clip(p, 0.001, 0.999)
    h = 0.5 * (40.0 / (n * 4.18879)) ** (1 / 3) * rng.uniform(0.6, 1.4, n)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), h


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_tree_steps_over_summed_counts(lib):
    """two ranks' keys: every step's leaf counts and rebalance equal the reference's; the converged tree is the
    single-rank tree of all keys"""
    import torch
    from oracle import domain as od
    from oracle import refsim
    from sphexa_b200 import lib as L
    x, y, z, _ = _clumps(60_000, 3, True)
    box = (0, 1, 0, 1, 0, 1)
    keys = refsim.sfc_keys(x, y, z, box, True)
    part = np.random.default_rng(4).integers(0, 2, keys.size)
    rank_keys = [np.sort(keys[part == r]) for r in range(2)]
    dkeys = [_dev(k.view(np.int64), torch) for k in rank_keys]
    leaves = np.array([0, 1 << 63], dtype=np.uint64)
    for step in range(64):
        dl = _dev(leaves.view(np.int64), torch)
        total = np.zeros(leaves.size - 1, dtype=np.uint32)
        for r in range(2):
            c = torch.zeros(leaves.size - 1, dtype=torch.int32, device="cuda")
            L.check(lib.sphb_leaf_counts(L.ptr(dl), leaves.size - 1, L.ptr(dkeys[r]), rank_keys[r].size, L.ptr(c),
                                         None), "leaf counts")
            torch.cuda.synchronize()
            got = c.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, od.ref_leaf_counts(leaves, rank_keys[r]))
            total += got
        cap = 8 * leaves.size + 8
        num, conv = C.c_size_t(), C.c_int()
        dc = _dev(total.view(np.int32), torch)
        while True:
            out = torch.zeros(cap + 1, dtype=torch.int64, device="cuda")
            rc = lib.sphb_rebalance_tree(L.ptr(dl), leaves.size - 1, L.ptr(dc), 16, L.ptr(out), cap, C.byref(num),
                                         C.byref(conv), None)
            if rc != L.SPHB_ERR_CAPACITY:
                break
            assert num.value + 1 > cap
            cap = num.value + 1
        L.check(rc, "rebalance")
        ref_new, ref_conv = od.ref_rebalance_tree(leaves, total, 16)
        new = out.cpu().numpy().view(np.uint64)[:num.value + 1]
        assert bool(conv.value) == ref_conv
        assert np.array_equal(new, ref_new)
        if ref_conv:
            break
        leaves = new
    ref_leaves, ref_counts = refsim.compute_octree(np.sort(keys), 16)
    assert np.array_equal(leaves, ref_leaves) and np.array_equal(total, ref_counts)
    assert step >= 2  # the tree grew over several steps


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("h_float", [False, True])
@pytest.mark.parametrize("world", [2, 3])
def test_find_halos_bit_exact(lib, periodic, h_float, world):
    """the halo flags of every rank of an SFC split equal the reference's findHalos (and the restatement's)"""
    import torch
    from oracle import domain as od
    from oracle import refsim
    from sphexa_b200 import lib as L
    x, y, z, h = _clumps(30_000, 5 + world, periodic)
    box = (0, 1, 0, 1, 0, 1)
    keys = refsim.sfc_keys(x, y, z, box, periodic)
    order = np.argsort(keys, kind="stable")
    x, y, z, h, keys = x[order], y[order], z[order], h[order], keys[order]
    if h_float:
        h = h.astype(np.float32)
    leaves, counts = refsim.compute_octree(keys, 32)
    _, off, _ = od.ref_sfc_assignment(world, counts, leaves)
    scan = np.concatenate([[0], np.cumsum(counts)])
    dl = _dev(leaves.view(np.int64), torch)
    b = L.make_box(box, [int(periodic)] * 3)
    halos = 0
    for r in range(world):
        first, last = int(off[r]), int(off[r + 1])
        s, e = int(scan[first]), int(scan[last])
        lay = (scan[first:last + 1] - s).astype(np.uint32)
        dx, dy, dz, dh = (_dev(a[s:e], torch) for a in (x, y, z, h))
        dlay = _dev(lay.view(np.int32), torch)
        flags = torch.full((leaves.size - 1,), 7, dtype=torch.uint8, device="cuda")
        L.check(lib.sphb_find_halos(L.ptr(dl), leaves.size - 1, L.ptr(dx), L.ptr(dy), L.ptr(dz), L.ptr(dh),
                                    L.SPHB_F32 if h_float else L.SPHB_F64, L.ptr(dlay), first, last, C.byref(b),
                                    1.0, L.ptr(flags), None), "find halos")
        got = flags.cpu().numpy()
        ref = od.ref_find_halos(leaves, x[s:e], y[s:e], z[s:e], h[s:e], lay, first, last, box, periodic)
        assert np.array_equal(got, ref), (r, int(np.sum(got != ref)))
        assert np.array_equal(od.find_halos(leaves, x[s:e], y[s:e], z[s:e], h[s:e], lay, first, last, box,
                                            periodic), ref)
        halos += int(ref.sum())
    assert halos > 0


class _Hub:
    def __init__(self, world):
        self.world = world
        self.barrier = threading.Barrier(world, timeout=120)
        self.slots = [None] * world
        self.mail = {}


class _ThreadComm:
    """the domain's communication between threads of one process (one per rank), through host-side slots"""

    def __init__(self, hub, rank):
        self.hub, self.rank = hub, rank

    def _publish(self, t):
        self.hub.slots[self.rank] = t.clone()
        self.hub.barrier.wait()
        vals = [v.clone() for v in self.hub.slots]
        self.hub.barrier.wait()
        return vals

    def all_reduce(self, t, op="sum"):
        import torch
        vals = self._publish(t)
        st = torch.stack(vals)
        res = st.sum(0) if op == "sum" else (st.min(0).values if op == "min" else st.max(0).values)
        t.copy_(res)
        return t

    def all_gather(self, t):
        return self._publish(t)

    def exchange(self, sends, recv_shapes, dtype, device):
        for p, t in sends.items():
            self.hub.mail[(self.rank, p)] = t.clone()
        self.hub.barrier.wait()
        out = {p: self.hub.mail.pop((p, self.rank)).reshape(shape) for p, shape in recv_shapes.items()}
        self.hub.barrier.wait()
        return out


class _LockedEngine:
    """one engine call at a time across the rank threads"""

    def __init__(self, engine, lock):
        self.engine, self.lock = engine, lock

    def __getattr__(self, name):
        fn = getattr(self.engine, name)

        def call(*a, **k):
            import torch
            with self.lock:
                r = fn(*a, **k)
                torch.cuda.synchronize()
                return r
        return call


@pytest.mark.parametrize("world,periodic", [(2, True), (3, True), (2, False)])
def test_domain_sync_cuda_engine_ranks_as_threads(lib, tmp_path, world, periodic):
    import torch
    import test_cpu_domain as T
    from sphexa_b200.domain import CudaEngine, Domain
    seed = 21 + world
    hub = _Hub(world)
    lock = threading.Lock()
    engine = CudaEngine()
    errors = []

    def rank_main(rank):
        try:
            torch.cuda.set_device(0)
            x, y, z, h, ids, m = T._particles(seed, periodic)
            mine = np.random.default_rng(seed + 1).permutation(T.N) % world == rank
            t = {k: torch.from_numpy(np.ascontiguousarray(v[mine])).cuda() for k, v in
                 dict(x=x, y=y, z=z, h=h, id=ids, m=m).items()}
            dom = Domain(rank, world, bucket_size=T.BUCKET, limits=(0, 1, 0, 1, 0, 1), periodic=periodic,
                         comm=_ThreadComm(hub, rank), engine=_LockedEngine(engine, lock))
            for rep in range(2):
                r = dom.sync(t["x"], t["y"], t["z"], t["h"], {"id": t["id"], "m": t["m"]})
                halo_id, halo_m = r["id"].clone(), r["m"].clone()
                dom.exchange_halos(halo_id, halo_m)
                c = {k: v.cpu().numpy() for k, v in r.items()}
                np.savez(os.path.join(str(tmp_path), f"rank{rank}_rep{rep}.npz"),
                         x=c["x"], y=c["y"], z=c["z"], h=c["h"], keys=c["keys"], id_owned=c["id"],
                         id=halo_id.cpu().numpy(), m=halo_m.cpu().numpy(), leaves=dom.leaves.cpu().numpy(),
                         counts=dom.counts, offsets=dom.tree_offsets, boundaries=dom.boundaries,
                         flags=dom.halo_flags[rank], start=dom.start_index, end=dom.end_index,
                         box=np.array(dom.box.limits))
                nx, ny, nz = T._moved(c["x"], c["y"], c["z"], c["id"], periodic, seed + 10)
                t = {"x": torch.from_numpy(nx).cuda(), "y": torch.from_numpy(ny).cuda(),
                     "z": torch.from_numpy(nz).cuda(), "h": r["h"], "id": r["id"], "m": r["m"]}
        except BaseException as exc:  # noqa: BLE001 - reported below, the other ranks see a broken barrier
            errors.append((rank, exc))
            hub.barrier.abort()

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    first = [e for e in errors if not isinstance(e[1], threading.BrokenBarrierError)]
    assert not errors, first or errors
    T._check(str(tmp_path), world, periodic, seed)
