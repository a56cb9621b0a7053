"""One hierarchy divided among ranks, one engine (and one GPU) per rank.

The reference gives every MPI rank a share of each level's blocks
(Parallel::distribute, Parallel.C:504-827, block i of a patch to rank
i mod nprocs, :797-798) and moves ghost, restriction and prolongation
segments between ranks (Parallel::Sync, :3677-3776; Parallel::transfer,
:3508-3592); the error flag of a step is reduced over all ranks
(bssn_class.C:3164-3178), as are the constraint norms (Parallel::L2Norm,
:4214-4243).  Here:

* `partition` names the owner of every block (balanced by points per level,
  or the reference's round robin);
* `Engine.from_hierarchy(H, rank, nranks, owners)` builds one rank's engine:
  it allocates and steps its own blocks; its transfers compute the boxes
  whose source it owns and exchange the rest (include/amss_b200.h);
* `LocalGroup` runs all ranks in this process, one thread and one engine per
  rank (one GPU each, or several ranks on one GPU for checking), exchanging
  through device-to-device copies;
* `NcclRank` is one rank of a torch.distributed job (one process per GPU),
  exchanging with grouped NCCL send/receive;
* `Plan` is a rank's transfer plan without a device.
"""
import ctypes
import threading

import numpy as np

from ._lib import _DP, _IP, AmssError, check, last_error, lib
from .engine import Engine

XFER_KINDS = ("sync", "restrict", "prolong")


def partition(H, nranks, mode="balanced"):
    """Owner rank of every block of H.  `balanced`: per level, blocks by
    descending point count, each to the rank with the fewest points of that
    level so far (every level is stepped on its own, so each level is
    balanced); `round_robin`: the i-th block of each patch to rank i mod
    nranks, as Parallel::distribute deals its blocks."""
    if nranks < 1:
        raise AmssError("partition: nranks must be >= 1")
    owners = [0] * len(H.blocks)
    if mode == "round_robin":
        for patches in H.levels:
            for p in patches:
                for i, bi in enumerate(p.blocks):
                    owners[bi] = i % nranks
        return owners
    if mode != "balanced":
        raise AmssError("partition: mode is 'balanced' or 'round_robin'")
    for patches in H.levels:
        ids = [bi for p in patches for bi in p.blocks]
        ids.sort(key=lambda bi: (-int(np.prod(H.blocks[bi].ex)), bi))
        load = [0] * nranks
        for bi in ids:
            r = min(range(nranks), key=lambda q: (load[q], q))
            owners[bi] = r
            load[r] += int(np.prod(H.blocks[bi].ex))
    return owners


def _xfer_tables(h, nblocks):
    L = lib()
    out = []
    n = check(L.amss_engine_xfer_count(h), "amss_engine_xfer_count")
    for k in range(n):
        info = (ctypes.c_longlong * 8)()
        check(L.amss_engine_xfer_info(h, k, info), "amss_engine_xfer_info")
        kind, level, nall, ncross, nrun, nunp, ob, ib = list(info)
        lists = []
        for lst, cnt in ((0, nrun), (1, nunp)):
            buf = np.zeros(8 * max(cnt, 1), dtype=np.int32)
            check(L.amss_engine_xfer_boxes(h, k, lst, buf.ctypes.data_as(_IP), int(cnt)), "amss_engine_xfer_boxes")
            lists.append(buf[:8 * cnt].reshape(-1, 8))
        peers = []
        for d in (0, 1):
            m = check(L.amss_engine_xfer_peers(h, k, d, None, 0), "amss_engine_xfer_peers")
            buf = (ctypes.c_longlong * (3 * max(m, 1)))()
            check(L.amss_engine_xfer_peers(h, k, d, buf, m), "amss_engine_xfer_peers")
            peers.append([(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]) for i in range(m)])
        out.append(dict(kind=XFER_KINDS[kind], level=level, nall=nall, ncross=ncross, run=lists[0],
                        unpack=lists[1], out_bytes=ob, in_bytes=ib, send=peers[0], recv=peers[1]))
    return out


class Plan(Engine):
    """A rank's transfer plan over a hierarchy, built without a device
    (amss_plan_create / amss_plan_commit): which boxes its kernels compute,
    which it receives, and the staging regions exchanged with each peer."""
    _create = "amss_plan_create"

    def commit(self):
        check(lib().amss_plan_commit(self._h), "amss_plan_commit")

    @classmethod
    def of(cls, H, rank, nranks, owners, **kw):
        return cls.from_hierarchy(H, rank=rank, nranks=nranks, owners=owners, **kw)

    def xfers(self):
        """Per transfer: kind, level, nall, ncross, run / unpack boxes
        (rows dst, src, lo[3], n[3]), staging bytes, send / recv peers
        (rank, offset, bytes)."""
        return _xfer_tables(self._h, len(self.blocks))

    def staging_block(self, sid):
        """(org, ex, byte offset, arena 0 out / 1 in) of a staging block."""
        v = (ctypes.c_longlong * 8)()
        check(lib().amss_engine_staging_block(self._h, int(sid), v), "amss_engine_staging_block")
        v = list(v)
        return tuple(v[0:3]), tuple(v[3:6]), v[6], v[7]


def xfer_tables(engine):
    """The transfer plan of a committed rank engine (as Plan.xfers)."""
    return _xfer_tables(engine._h, len(engine.blocks))


class LocalGroup:
    """`nranks` engines in this process, one per rank, stepped concurrently by
    one host thread each.  devices: the CUDA device of each rank (default
    all on device 0 -- the exchange still crosses engines, which is how the
    partitioned path is checked on one GPU).  timeout: seconds a rank waits at
    an exchange for the others before every rank fails."""

    def __init__(self, H, owners, nranks, devices=None, timeout=60.0, **engine_kw):
        self.H = H
        self.owners = list(owners)
        self.nranks = nranks
        self.devices = list(devices) if devices is not None else [0] * nranks
        self._g = lib().amss_group_create(nranks, float(timeout))
        if not self._g:
            raise AmssError("amss_group_create failed: " + last_error())
        self.engines = []
        try:
            for r in range(nranks):
                self._device(r)
                e = Engine.from_hierarchy(H, rank=r, nranks=nranks, owners=self.owners, **engine_kw)
                check(lib().amss_group_join(e._h, self._g), "amss_group_join")
                self.engines.append(e)
        except Exception:
            self.close()
            raise

    def _device(self, r):
        import torch
        torch.cuda.set_device(self.devices[r])

    def close(self):
        for e in self.engines:
            e.close()
        self.engines = []
        if self._g:
            lib().amss_group_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def engine_of(self, block):
        return self.engines[self.owners[block]]

    def set_state(self, block, state):
        self.engine_of(block).set_state(block, state)

    def get_state(self, block):
        return self.engine_of(block).get_state(block)

    def _each(self, fn):
        errs = [None] * self.nranks

        def work(r):
            try:
                self._device(r)
                fn(r, self.engines[r])
            except Exception as ex:   # reported after every thread has ended
                errs[r] = ex

        ts = [threading.Thread(target=work, args=(r,)) for r in range(self.nranks)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        bad = [(r, ex) for r, ex in enumerate(errs) if ex is not None]
        if bad:
            raise AmssError("; ".join(f"rank {r}: {ex}" for r, ex in bad))

    def coarse_step(self, dt0, steps=1):
        def go(r, e):
            for _ in range(steps):
                e.coarse_step(dt0)
        self._each(go)

    def step(self, level, dt):
        self._each(lambda r, e: e.step(level, dt))

    def sync(self):
        """Waits for every rank; 1 if any rank saw a NaN (the reduction of
        bssn_class.C:3164-3178)."""
        flags = [0] * self.nranks

        def go(r, e):
            flags[r] = e.sync()
        self._each(go)
        return max(flags)

    def constraint_norms(self, level):
        parts = [None] * self.nranks

        def go(r, e):
            parts[r] = e.constraint_sums(level)
        self._each(go)
        return np.sqrt(np.sum(parts, axis=0))


class NcclRank:
    """This process's rank of a torch.distributed job over one hierarchy:
    its engine on the current CUDA device, exchanging with the other ranks by
    NCCL send/receive.  The process group (any backend) carries the NCCL
    unique id and the reductions of the error flag and constraint sums."""

    def __init__(self, H, owners, group=None, **engine_kw):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.nranks = dist.get_world_size(group)
        self.engine = Engine.from_hierarchy(H, rank=self.rank, nranks=self.nranks, owners=owners, **engine_kw)
        uid = [None]
        if self.rank == 0:
            buf = ctypes.create_string_buffer(128)
            check(lib().amss_nccl_unique_id(buf), "amss_nccl_unique_id")
            uid[0] = bytes(buf.raw)
        dist.broadcast_object_list(uid, src=0, group=group)
        check(lib().amss_engine_set_nccl(self.engine._h, uid[0]), "amss_engine_set_nccl")

    def coarse_step(self, dt0, steps=1):
        for _ in range(steps):
            self.engine.coarse_step(dt0)

    def sync(self):
        import torch
        flag = torch.tensor([self.engine.sync()], dtype=torch.int64)
        self.dist.all_reduce(flag, op=self.dist.ReduceOp.MAX, group=self.group)
        return int(flag.item())

    def constraint_norms(self, level):
        import torch
        s = torch.tensor(self.engine.constraint_sums(level), dtype=torch.float64)
        self.dist.all_reduce(s, group=self.group)
        return np.sqrt(s.numpy())

    def close(self):
        self.engine.close()
