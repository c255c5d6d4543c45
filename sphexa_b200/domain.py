"""Multi-rank domain: the SFC split of the particles over the ranks and the halo exchange between them.

The counterpart of cstone::Domain::sync (domain/include/cstone/domain/domain.hpp:165-213) and
Domain::exchangeHalos / Halos::exchangeHalos (halos/halos.hpp:84-121) for the hydro propagator, one process per GPU:

* every rank holds the same global cornerstone tree; each tree step counts the rank's sorted keys per leaf on the
  device (sphb_leaf_counts), the counts are summed over the ranks (one all-reduce) and the rebalance runs on the
  device (sphb_rebalance_tree), until a rebalance changes nothing (cstone::updateOctreeGlobal,
  tree/update_mpi.hpp:64-99, as GlobalAssignment::assign loops over it, domain/assignment.hpp:95-140);
* the ranks get contiguous runs of leaves with equal particle counts (makeSfcAssignment,
  domain/domaindecomp.hpp:112-127) and exchange the particles outside their run point to point into local device
  memory (exchangeParticles, domain/exchange_domain.hpp), then SFC-sort what they own;
* halo discovery runs on the device on the shared tree (sphb_find_halos: the leaves of other ranks that overlap the
  2h search boxes of the owned leaves); the halo flags of all ranks are all-gathered, so every rank knows which of its
  leaves each peer receives (the reference exchanges request keys point to point instead, exchange_keys.hpp);
* the local arrays are laid out in leaf order: halos from lower ranks, the owned particles, halos from higher ranks
  (computeNodeLayout, domain/layout.hpp:151-177); exchange_halos sends each peer its leaves' particles, packed into
  one record buffer per peer and direction.

The per-particle and per-leaf work runs through an engine: CudaEngine (libsphb200 on the GPU) by default. The
communication runs through a comm object: TorchComm (torch.distributed point-to-point and collective calls on a
process group, NCCL between GPUs) by default; with one rank no call is made. Host arrays of the tree (leaf keys,
counts, layout) are O(leaves).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

ROOT_END = 1 << 63


@dataclass
class DomainBox:
    """coordinate box [lo, hi) per axis and its boundary kind (periodic or open) per axis"""
    limits: tuple
    periodic: tuple

    def __post_init__(self):
        self.limits = tuple(float(v) for v in self.limits)
        p = self.periodic
        self.periodic = tuple(int(bool(v)) for v in (p if hasattr(p, "__len__") else (p, p, p)))

    def sphb(self):
        from sphexa_b200 import lib as L
        return L.make_box(self.limits, self.periodic)


class CudaEngine:
    """The domain's per-particle and per-leaf operations on the GPU through the C ABI of libsphb200, on the current
    torch stream. Keys and leaf keys travel as int64 tensors holding the uint64 bit patterns."""

    def __init__(self):
        from sphexa_b200 import lib as L
        self.L = L
        self.lib = L.load()

    @staticmethod
    def _stream():
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def sfc_keys(self, x, y, z, box: DomainBox):
        L = self.L
        n = x.numel()
        keys = torch.zeros(n, dtype=torch.int64, device=x.device)
        if n:
            b = box.sphb()
            L.check(self.lib.sphb_compute_sfc_keys(L.ptr(x), L.ptr(y), L.ptr(z), L.ptr(keys), n, C.byref(b),
                                                   self._stream()), "sfc keys")
        return keys

    def sort_by_key(self, keys):
        L = self.L
        n = keys.numel()
        k = keys.clone()
        vals = torch.empty(n, dtype=torch.int32, device=keys.device)
        if n:
            nbytes = self.lib.sphb_sort_by_key_scratch_bytes(n)
            scratch = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=keys.device)
            L.check(self.lib.sphb_sort_by_key(L.ptr(k), L.ptr(vals), n, 1, L.ptr(scratch), nbytes, self._stream()),
                    "sort by key")
        return k, vals.long()

    def leaf_counts(self, leaves, sorted_keys):
        L = self.L
        nl = leaves.numel() - 1
        counts = torch.zeros(nl, dtype=torch.int32, device=leaves.device)
        L.check(self.lib.sphb_leaf_counts(L.ptr(leaves), nl, L.ptr(sorted_keys) if sorted_keys.numel() else None,
                                          sorted_keys.numel(), L.ptr(counts), self._stream()), "leaf counts")
        return counts.long()

    def rebalance(self, leaves, counts, bucket: int):
        L = self.L
        nl = leaves.numel() - 1
        c32 = counts.to(torch.int32).contiguous()
        cap = 8 * nl + 8
        while True:
            out = torch.empty(cap + 1, dtype=torch.int64, device=leaves.device)
            num = C.c_size_t()
            conv = C.c_int()
            rc = self.lib.sphb_rebalance_tree(L.ptr(leaves), nl, L.ptr(c32), bucket, L.ptr(out), cap, C.byref(num),
                                              C.byref(conv), self._stream())
            if rc == L.SPHB_ERR_CAPACITY:
                cap = int(num.value) + 1
                continue
            L.check(rc, "rebalance tree")
            return out[:num.value + 1].clone(), bool(conv.value)

    def find_halos(self, leaves, x, y, z, h, layout, first_leaf, last_leaf, box: DomainBox, search_ext: float):
        L = self.L
        nl = leaves.numel() - 1
        flags = torch.zeros(nl, dtype=torch.uint8, device=leaves.device)
        if last_leaf <= first_leaf:
            return flags
        lay = layout.to(torch.int32).contiguous()
        b = box.sphb()
        n = x.numel()
        L.check(self.lib.sphb_find_halos(L.ptr(leaves), nl, L.ptr(x) if n else None, L.ptr(y) if n else None,
                                         L.ptr(z) if n else None, L.ptr(h) if n else None, L.dtype_code(h),
                                         L.ptr(lay), int(first_leaf), int(last_leaf), C.byref(b), float(search_ext),
                                         L.ptr(flags), self._stream()), "find halos")
        return flags


def uniform_bins(counts: np.ndarray, num_ranks: int):
    """First leaf of every rank (num_ranks + 1 entries) and particles per rank: rank r starts at the first leaf where
    the running count reaches r * total / num_ranks, truncated to an integer (uniformBins,
    domain/domaindecomp.hpp:32-56)."""
    scan = np.zeros(counts.size + 1, dtype=np.uint64)
    np.cumsum(counts.astype(np.uint64), out=scan[1:])
    per = float(scan[-1]) / num_ranks
    bins = np.empty(num_ranks + 1, dtype=np.int64)
    bins[0], bins[-1] = 0, counts.size
    for r in range(1, num_ranks):
        bins[r] = np.searchsorted(scan, np.uint64(int(r * per)), side="left")
    return bins, np.diff(scan[bins]).astype(np.int64)


def _runs(mask: np.ndarray, lo: int, hi: int):
    """[a, b) runs of consecutive set entries of mask within [lo, hi)"""
    m = np.zeros(hi - lo + 2, dtype=np.int8)
    m[1:-1] = mask[lo:hi] != 0
    d = np.diff(m)
    starts = np.nonzero(d == 1)[0] + lo
    ends = np.nonzero(d == -1)[0] + lo
    return list(zip(starts.tolist(), ends.tolist()))


def _pack(arrays, index=None):
    """rows of several 1-D arrays as one (n, record bytes) uint8 buffer, each row the array elements' bytes"""
    cols = []
    for a in arrays:
        v = a if index is None else a.index_select(0, index)
        cols.append(v.contiguous().view(torch.uint8).view(v.numel(), a.element_size()))
    return torch.cat(cols, dim=1) if cols else None


def _unpack_into(record, arrays, lo: int):
    """write the record rows into arrays[k][lo:lo + rows]"""
    off = 0
    rows = record.shape[0]
    for a in arrays:
        w = a.element_size()
        a[lo:lo + rows] = record[:, off:off + w].contiguous().view(a.dtype).view(rows)
        off += w


def _unpack(record, like):
    out = []
    off = 0
    rows = record.shape[0]
    for a in like:
        w = a.element_size()
        out.append(record[:, off:off + w].contiguous().view(a.dtype).view(rows))
        off += w
    return out


class TorchComm:
    """The domain's communication over a torch.distributed process group (NCCL between GPUs): sum/min/max
    all-reduce, all-gather, and point-to-point exchange of one tensor per peer and direction."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def all_reduce(self, t, op="sum"):
        ops = {"sum": self.dist.ReduceOp.SUM, "min": self.dist.ReduceOp.MIN, "max": self.dist.ReduceOp.MAX}
        self.dist.all_reduce(t, op=ops[op], group=self.group)
        return t

    def all_gather(self, t):
        out = [torch.empty_like(t) for _ in range(self.dist.get_world_size(self.group))]
        self.dist.all_gather(out, t.contiguous(), group=self.group)
        return out

    def exchange(self, sends: dict, recv_shapes: dict, dtype, device):
        """sends {peer: tensor}, receives {peer: new tensor of recv_shapes[peer]}; both sides of every pair agree
        on the sizes beforehand, and empty messages are not sent"""
        recvs = {p: torch.empty(shape, dtype=dtype, device=device) for p, shape in recv_shapes.items()}
        ops = []
        for p in sorted(set(sends) | set(recvs)):
            if p in recvs:
                ops.append(self.dist.P2POp(self.dist.irecv, recvs[p], p, group=self.group))
            if p in sends:
                ops.append(self.dist.P2POp(self.dist.isend, sends[p].contiguous(), p, group=self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        return recvs


class Domain:
    """The domain of one rank.

    sync(x, y, z, h, properties) takes the rank's particle arrays (at the first call every element is the rank's;
    afterwards the arrays that the previous sync returned, owned particles in [start_index, end_index) and halos
    around them), redistributes and SFC-sorts the owned particles, discovers the halos and returns the new arrays:
    x, y, z, h with their halos filled, keys of every element, and the properties with their owned part filled
    (halo entries zero until exchange_halos fills them, as the reference leaves them to the propagator).
    """

    def __init__(self, rank: int, num_ranks: int, bucket_size: int = 64, limits=(0, 1, 0, 1, 0, 1), periodic=True,
                 halo_search_ext: float = 1.0, comm=None, engine=None, max_tree_steps: int = 64):
        if not (0 <= rank < num_ranks) or bucket_size < 1:
            raise ValueError("rank, num_ranks or bucket_size out of range")
        self.rank, self.num_ranks = rank, num_ranks
        self.bucket_size = int(bucket_size)
        self.box = DomainBox(limits, periodic)
        self.halo_search_ext = float(halo_search_ext)
        self.comm = comm if comm is not None or num_ranks == 1 else TorchComm()
        self.engine = engine if engine is not None else CudaEngine()
        self.max_tree_steps = max_tree_steps
        self.leaves = None           # device int64 bit patterns, num_leaves + 1
        self.counts = None           # host int64, global particles per leaf
        self.tree_offsets = None     # host, first leaf of every rank (num_ranks + 1)
        self.boundaries = None       # host uint64, first key of every rank (num_ranks + 1)
        self.rank_counts = None
        self.layout = None           # host int64, offset of every leaf in the local arrays (num_leaves + 1)
        self.halo_flags = None       # host uint8 [num_ranks, num_leaves]: which leaves each rank receives
        self.start_index = 0
        self.end_index = 0
        self.n_particles_with_halos = 0
        self._owned = None
        self._send = {}              # peer -> device index tensor of the local rows it receives
        self._recv = {}              # peer -> (lo, hi) of the local rows it sends
        self._first_call = True

    def _all_reduce(self, t, op="sum"):
        return t if self.num_ranks == 1 else self.comm.all_reduce(t, op)

    def _all_gather(self, t):
        return [t] if self.num_ranks == 1 else self.comm.all_gather(t)

    def _exchange(self, sends: dict, recv_shapes: dict, dtype, device):
        if self.num_ranks == 1:
            return {}
        return self.comm.exchange(sends, recv_shapes, dtype, device)

    # -------------------------------------------------------------------------------------------------------------
    # sync steps
    # -------------------------------------------------------------------------------------------------------------
    def _update_box(self, x, y, z):
        """open axes follow the global extent of the owned particles: the fitting box at the first call, afterwards
        shrinking by at most 5 % of the previous length per side (makeGlobalBox, sfc/box_mpi.hpp:69-108;
        limitBoxShrinking, sfc/box.hpp:397-416); periodic axes keep their limits"""
        if all(self.box.periodic):
            return
        lim = list(self.box.limits)
        ext = torch.empty(6, dtype=torch.float64, device=x.device)
        for k, a in enumerate((x, y, z)):
            if a.numel():
                ext[2 * k] = a.min()
                ext[2 * k + 1] = -a.max()
            else:
                ext[2 * k] = float("inf")
                ext[2 * k + 1] = float("inf")
        self._all_reduce(ext, "min")
        e = ext.cpu().numpy()
        for k in range(3):
            if self.box.periodic[k]:
                continue
            lo, hi = float(e[2 * k]), float(-e[2 * k + 1])
            if not self._first_call:
                length = lim[2 * k + 1] - lim[2 * k]
                lo = min(lo, lim[2 * k] + 0.05 * length)
                hi = max(hi, lim[2 * k + 1] - 0.05 * length)
            lim[2 * k], lim[2 * k + 1] = lo, hi
        self.box = DomainBox(lim, self.box.periodic)

    def _update_tree(self, sorted_keys):
        device = sorted_keys.device
        leaves = self.leaves
        if leaves is None:
            leaves = torch.tensor(np.array([0, ROOT_END], dtype=np.uint64).view(np.int64), device=device)
        for _ in range(self.max_tree_steps):
            counts = self.engine.leaf_counts(leaves, sorted_keys)
            self._all_reduce(counts, "sum")
            new, converged = self.engine.rebalance(leaves, counts, self.bucket_size)
            if converged:
                self.leaves = leaves
                self.counts = counts.cpu().numpy().astype(np.int64)
                return
            leaves = new
        raise RuntimeError("global tree did not converge")

    def sync(self, x, y, z, h, properties: dict | None = None) -> dict:
        props = dict(properties or {})
        n = x.numel()
        for a in [y, z, h] + list(props.values()):
            if a.numel() != n or a.device != x.device:
                raise ValueError("particle arrays differ in length or device")
        if self._owned is not None and n != self.n_particles_with_halos:
            raise ValueError(f"sync after the first takes the arrays the previous sync returned "
                             f"({self.n_particles_with_halos} rows), got {n}")
        s, e = self._owned if self._owned is not None else (0, n)
        own = [a[s:e] for a in (x, y, z, h)] + [a[s:e] for a in props.values()]
        self._update_box(*own[:3])

        # keys and SFC order of the owned particles, global tree, assignment
        keys = self.engine.sfc_keys(own[0].contiguous(), own[1].contiguous(), own[2].contiguous(), self.box)
        skeys, order = self.engine.sort_by_key(keys)
        self._update_tree(skeys)
        R = self.num_ranks
        self.tree_offsets, self.rank_counts = uniform_bins(self.counts, R)
        leaves_host = self.leaves.cpu().numpy().view(np.uint64)
        self.boundaries = leaves_host[self.tree_offsets]

        # particle exchange: the sorted owned particles of rank r's key range go to rank r
        inner = torch.tensor(self.boundaries[1:R].view(np.int64), device=x.device)
        cuts = torch.searchsorted(skeys, inner) if R > 1 else torch.empty(0, dtype=torch.int64, device=x.device)
        edges = [0] + cuts.cpu().tolist() + [skeys.numel()]
        send_counts = torch.tensor([edges[r + 1] - edges[r] for r in range(R)], dtype=torch.int64, device=x.device)
        all_counts = torch.stack(self._all_gather(send_counts)).cpu().numpy()
        record = _pack(own, order)
        width = record.shape[1] if record is not None else 0
        sends = {r: record[edges[r]:edges[r + 1]] for r in range(R) if r != self.rank and edges[r + 1] > edges[r]}
        recv_shapes = {p: (int(all_counts[p, self.rank]), width) for p in range(R)
                       if p != self.rank and all_counts[p, self.rank] > 0}
        recvs = self._exchange(sends, recv_shapes, torch.uint8, x.device)
        parts = [record[edges[self.rank]:edges[self.rank + 1]]] + [recvs[p] for p in sorted(recvs)]
        mine = _unpack(torch.cat(parts, dim=0), own)
        m = mine[0].numel()
        if m != int(self.rank_counts[self.rank]):
            raise RuntimeError(f"rank {self.rank} holds {m} particles after the exchange, its leaves count "
                               f"{int(self.rank_counts[self.rank])}")
        mkeys = self.engine.sfc_keys(mine[0], mine[1], mine[2], self.box)
        mkeys, morder = self.engine.sort_by_key(mkeys)
        mine = [a.index_select(0, morder) for a in mine]

        # halo discovery on the shared tree, everyone's flags, the local layout
        first, last = int(self.tree_offsets[self.rank]), int(self.tree_offsets[self.rank + 1])
        own_layout = np.zeros(last - first + 1, dtype=np.int64)
        np.cumsum(self.counts[first:last], out=own_layout[1:])
        flags = self.engine.find_halos(self.leaves, mine[0], mine[1], mine[2], mine[3],
                                       torch.tensor(own_layout, dtype=torch.int32, device=x.device), first, last,
                                       self.box, self.halo_search_ext)
        self.halo_flags = torch.stack(self._all_gather(flags)).cpu().numpy()
        present = self.halo_flags[self.rank].astype(bool)
        present[first:last] = True
        self.layout = np.zeros(self.counts.size + 1, dtype=np.int64)
        np.cumsum(np.where(present, self.counts, 0), out=self.layout[1:])
        self.start_index, self.end_index = int(self.layout[first]), int(self.layout[last])
        self.n_particles_with_halos = int(self.layout[-1])
        self._plan_halos(x.device)

        # the new arrays: owned rows at [start, end), halos exchanged for x, y, z, h
        nwh = self.n_particles_with_halos
        out = []
        for a, src in zip(own, mine):
            b = torch.zeros(nwh, dtype=a.dtype, device=a.device)
            b[self.start_index:self.end_index] = src
            out.append(b)
        self.exchange_halos(*out[:4])
        self._owned = (self.start_index, self.end_index)
        self._first_call = False
        keys_all = self.engine.sfc_keys(out[0], out[1], out[2], self.box)
        res = {"x": out[0], "y": out[1], "z": out[2], "h": out[3], "keys": keys_all}
        res.update(zip(props.keys(), out[4:]))
        return res

    def _plan_halos(self, device):
        """rows each peer receives from this rank (its flagged leaves inside this rank's run) and the rows this rank
        receives from each peer (the present leaves of the peer's run: one contiguous range)"""
        R = self.num_ranks
        off = self.tree_offsets
        first, last = int(off[self.rank]), int(off[self.rank + 1])
        self._send, self._recv = {}, {}
        for q in range(R):
            if q == self.rank:
                continue
            rows = [np.arange(self.layout[a], self.layout[b]) for a, b in _runs(self.halo_flags[q], first, last)]
            idx = np.concatenate(rows) if rows else np.zeros(0, dtype=np.int64)
            if idx.size:
                self._send[q] = torch.tensor(idx, dtype=torch.int64, device=device)
            lo, hi = int(self.layout[off[q]]), int(self.layout[off[q + 1]])
            if hi > lo:
                self._recv[q] = (lo, hi)

    def exchange_halos(self, *arrays):
        """fill the halo rows of arrays (each n_particles_with_halos long) from the ranks that own them, in place
        (Halos::exchangeHalos, halos/halos.hpp:84-121: one message per peer and direction, all arrays packed)"""
        if not arrays:
            return
        for a in arrays:
            if a.numel() != self.n_particles_with_halos:
                raise ValueError("halo exchange on an array of another layout")
        sends = {q: _pack(arrays, idx) for q, idx in self._send.items()}
        width = sum(a.element_size() for a in arrays)
        recv_shapes = {p: (hi - lo, width) for p, (lo, hi) in self._recv.items()}
        recvs = self._exchange(sends, recv_shapes, torch.uint8, arrays[0].device)
        for p, rec in recvs.items():
            _unpack_into(rec, arrays, self._recv[p][0])
