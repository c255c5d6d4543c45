"""The multi-rank domain (sphexa_b200/domain.py) with two and three gloo ranks on the CPU, against the single-rank
result. The ranks start from a random split of one particle set; the domain's per-particle and per-leaf steps run
through the oracle's engine (the reference's own tree, assignment and halo functions compiled in oracle/_ref), so
these tests check the domain's host logic: the tree steps over summed counts, the assignment, the particle exchange,
the layout, the halo plan and the halo exchange.

* the global tree equals the single-rank cornerstone tree of all keys (computeOctree), the assignment the reference's
  makeSfcAssignment on it;
* the owned particles of the ranks, concatenated in rank order, are all particles in SFC order, bit for bit;
* the halo flags of every rank are the reference's findHalos flags for that rank's leaves, and the numpy
  restatement's;
* every particle within 2 h_i (minimum image) of an owned particle i is in the rank's arrays, every halo row holds its
  owner's values, and the local keys are in SFC order;
* exchange_halos fills the halo rows of further fields with the owners' values;
* a second sync after the particles moved repeats all of it.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUCKET = 16
N = 5000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _particles(seed, periodic, h32=False):
    """clumped particles in the unit box, h giving about 40 neighbours where the density is mean (float32 h with
    h32, the reference's default type for h)"""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(0.1, 0.9, (6, 3))
    which = rng.integers(0, 6, N)
    p = centers[which] + rng.normal(0, 1, (N, 3)) * rng.uniform(0.05, 0.2, 6)[which, None]
    p = np.mod(p, 1.0) if periodic else np.clip(p, 0.001, 0.999)
    h = 0.5 * (40.0 / (N * 4.18879)) ** (1 / 3) * rng.uniform(0.7, 1.3, N)
    ids = np.arange(N, dtype=np.int64)
    m = rng.uniform(0.5, 1.5, N).astype(np.float32)
    if h32:
        h = h.astype(np.float32)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), h, ids, m


def _moved(x, y, z, ids, periodic, seed):
    rng = np.random.default_rng(seed)
    d = rng.normal(0, 0.01, (3, x.size))
    out = []
    for a, da in zip((x, y, z), d):
        b = a + da
        out.append(np.mod(b, 1.0) if periodic else np.clip(b, 0.001, 0.999))
    return out


def _worker(rank, world, port, outdir, periodic, seed, h32=False):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from oracle.domain import OracleEngine
    from sphexa_b200.domain import Domain
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    x, y, z, h, ids, m = _particles(seed, periodic, h32)
    mine = np.random.default_rng(seed + 1).permutation(N) % world == rank
    t = {k: torch.from_numpy(np.ascontiguousarray(v[mine])) for k, v in
         dict(x=x, y=y, z=z, h=h, id=ids, m=m).items()}
    limits = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    dom = Domain(rank, world, bucket_size=BUCKET, limits=limits, periodic=periodic, engine=OracleEngine(periodic))
    for rep in range(2):
        r = dom.sync(t["x"], t["y"], t["z"], t["h"], {"id": t["id"], "m": t["m"]})
        halo_id, halo_m = r["id"].clone(), r["m"].clone()
        dom.exchange_halos(halo_id, halo_m)
        np.savez(os.path.join(outdir, f"rank{rank}_rep{rep}.npz"),
                 x=r["x"].numpy(), y=r["y"].numpy(), z=r["z"].numpy(), h=r["h"].numpy(), keys=r["keys"].numpy(),
                 id_owned=r["id"].numpy(), id=halo_id.numpy(), m=halo_m.numpy(),
                 leaves=dom.leaves.numpy(), counts=dom.counts, offsets=dom.tree_offsets,
                 boundaries=dom.boundaries, flags=dom.halo_flags[rank], start=dom.start_index, end=dom.end_index,
                 box=np.array(dom.box.limits))
        # the particles move; the next sync takes the arrays this one returned
        nx, ny, nz = _moved(r["x"].numpy(), r["y"].numpy(), r["z"].numpy(), r["id"].numpy(), periodic, seed + 10)
        t = {"x": torch.from_numpy(nx), "y": torch.from_numpy(ny), "z": torch.from_numpy(nz), "h": r["h"],
             "id": r["id"], "m": r["m"]}
    dist.barrier()
    dist.destroy_process_group()


def _check(outdir, world, periodic, seed, h32=False):
    from oracle import domain as od
    from oracle import refsim
    x, y, z, h, ids, m = _particles(seed, periodic, h32)
    for rep in range(2):
        res = [dict(np.load(os.path.join(outdir, f"rank{r}_rep{rep}.npz"))) for r in range(world)]
        box = tuple(res[0]["box"])
        for r in range(1, world):
            assert np.array_equal(res[r]["leaves"], res[0]["leaves"])
            assert np.array_equal(res[r]["counts"], res[0]["counts"])
            assert tuple(res[r]["box"]) == box
        # the single-rank order of all particles
        keys = refsim.sfc_keys(x, y, z, box, periodic)
        order = np.argsort(keys, kind="stable")
        skeys = keys[order]
        leaves = res[0]["leaves"].view(np.uint64)
        ref_leaves, ref_counts = refsim.compute_octree(skeys, BUCKET)
        assert np.array_equal(leaves, ref_leaves)
        assert np.array_equal(res[0]["counts"], ref_counts.astype(np.int64))
        b, off, rc = od.ref_sfc_assignment(world, ref_counts, ref_leaves)
        assert np.array_equal(res[0]["offsets"], off.astype(np.int64))
        assert np.array_equal(res[0]["boundaries"], b)
        bins, counts = od.uniform_bins(ref_counts, world)
        assert np.array_equal(bins, off) and np.array_equal(counts, rc)
        # owned particles, concatenated over the ranks: all particles in SFC order
        owned = {f: np.concatenate([q[f][q["start"]:q["end"]] for q in res]) for f in ("x", "y", "z", "h", "keys")}
        owned_id = np.concatenate([q["id_owned"][q["start"]:q["end"]] for q in res])
        assert np.array_equal(owned["keys"].view(np.uint64), skeys)
        assert np.array_equal(np.sort(owned_id), ids)
        for f, a in (("x", x), ("y", y), ("z", z), ("h", h)):
            assert np.array_equal(owned[f], a[owned_id]), f
        # halos
        L = np.array([box[1] - box[0], box[3] - box[2], box[5] - box[4]])
        P = np.stack([x, y, z], axis=1)
        for r, q in enumerate(res):
            first, last = int(q["offsets"][r]), int(q["offsets"][r + 1])
            s, e = int(q["start"]), int(q["end"])
            lay = np.concatenate([[0], np.cumsum(ref_counts[first:last])]).astype(np.uint32)
            ref_flags = od.ref_find_halos(ref_leaves, q["x"][s:e], q["y"][s:e], q["z"][s:e], q["h"][s:e], lay, first,
                                          last, box, periodic)
            assert np.array_equal(q["flags"], ref_flags)
            assert np.array_equal(od.find_halos(ref_leaves, q["x"][s:e], q["y"][s:e], q["z"][s:e], q["h"][s:e], lay,
                                                first, last, box, periodic), ref_flags)
            assert (ref_flags[:first].sum() + ref_flags[last:].sum()) > 0
            assert np.all(np.diff(q["keys"].view(np.uint64)) >= 0)
            local = q["id"]
            assert np.array_equal(np.sort(local), np.unique(local))
            for f, a in (("x", x), ("y", y), ("z", z), ("h", h)):
                assert np.array_equal(q[f], a[local]), (r, f)
            assert np.array_equal(q["m"], m[local])
            # neighbour completeness: every particle within 2 h_i of an owned particle i is present
            present = np.zeros(N, dtype=bool)
            present[local] = True
            for i in q["id_owned"][s:e]:
                d = P - P[i]
                if periodic:
                    d -= L * np.rint(d / L)
                near = np.einsum("ij,ij->i", d, d) < (2 * h[i]) ** 2
                assert present[near].all(), (r, int(i))
        # the second sync saw the moved particles
        x, y, z = _moved_all(res, world, periodic, seed, x, y, z)


def _moved_all(res, world, periodic, seed, x, y, z):
    """the global positions after the workers' move: each rank moved its whole returned arrays (halos too) with the
    same seeded displacement per local row; the owners' rows define the new positions"""
    nx, ny, nz = x.copy(), y.copy(), z.copy()
    for q in res:
        mx, my, mz = _moved(q["x"], q["y"], q["z"], q["id"], periodic, seed + 10)
        s, e = int(q["start"]), int(q["end"])
        own = q["id_owned"][s:e]
        nx[own], ny[own], nz[own] = mx[s:e], my[s:e], mz[s:e]
    return nx, ny, nz


@pytest.mark.parametrize("world,periodic,h32", [(2, True, False), (3, True, False), (2, False, False), (2, True, True)])
def test_domain_sync_and_halos_gloo(tmp_path, world, periodic, h32):
    from oracle import refsim
    if not refsim.available():
        pytest.skip("reference oracle not built")
    seed = 11 + world
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path), periodic, seed, h32), nprocs=world, join=True)
    _check(str(tmp_path), world, periodic, seed, h32)
