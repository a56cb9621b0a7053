"""Blocks divided among ranks, checked without a GPU.

* partition: every level balanced, or the reference's round robin
  (Parallel::distribute, Parallel.C:797-798);
* the transfer plans of the ranks (amss_plan_create, no device) fit
  together: every box of a transfer is computed by exactly one rank (its
  source's owner), a box that crosses ranks lands in a staging region of the
  sender whose offset and size the receiver expects;
* two gloo ranks on CPU run the ghost sync, restriction and prolongation of a
  three-level hierarchy through those plans -- packing into the staging
  layout the plans give, exchanging the regions over gloo, unpacking -- and
  end with exactly the arrays of the oracle's single-process transfers
  (Parallel::Sync / Restrict / OutBdLow2Hi restated in oracle/amr.py);
* the in-process group's host barrier gives up after its timeout, and the
  group stays failed (a rank that never reaches an exchange).
"""
import ctypes
import os
import socket
import sys
import threading
import time

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _paths():
    for sub in ("nr-amssncku_b200", "oracle"):
        p = os.path.join(ROOT, sub)
        if p not in sys.path:
            sys.path.insert(0, p)


_paths()
from amss_b200 import dist as D   # noqa: E402
from amss_b200._lib import AmssError, lib   # noqa: E402
from amss_b200.hierarchy import box_in_box   # noqa: E402


def small_hierarchy():
    return box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)


def test_balanced_partition_levels():
    H = small_hierarchy()
    for n in (2, 3, 4):
        own = D.partition(H, n)
        for patches in H.levels:
            ids = [bi for p in patches for bi in p.blocks]
            load = np.zeros(n)
            for bi in ids:
                load[own[bi]] += np.prod(H.blocks[bi].ex)
            biggest = max(np.prod(H.blocks[bi].ex) for bi in ids)
            assert load.max() - load.min() <= biggest
            assert set(own[bi] for bi in ids) == set(range(min(n, len(ids))))


def test_round_robin_partition():
    H = small_hierarchy()
    own = D.partition(H, 3, "round_robin")
    for patches in H.levels:
        for p in patches:
            assert [own[bi] for bi in p.blocks] == [i % 3 for i in range(len(p.blocks))]


@pytest.mark.parametrize("nranks,mode", [(2, "balanced"), (3, "round_robin"), (4, "balanced")])
def test_plans_fit_together(nranks, mode):
    H = small_hierarchy()
    nb = len(H.blocks)
    own = D.partition(H, nranks, mode)
    whole = D.Plan.of(H, 0, 1, [0] * nb)
    ref = whole.xfers()
    plans = [D.Plan.of(H, r, nranks, own) for r in range(nranks)]
    xs = [p.xfers() for p in plans]

    def segment(peers, off):
        for q, o, nbytes in peers:
            if o <= off < o + nbytes:
                return q, off - o
        raise AssertionError(f"offset {off} in no peer region")

    for k, full in enumerate(ref):
        assert full["ncross"] == 0 and len(full["run"]) == full["nall"] and len(full["unpack"]) == 0
        sent, recvd, got = {}, {}, []
        for r in range(nranks):
            x = xs[r][k]
            assert (x["kind"], x["level"], x["nall"]) == (full["kind"], full["level"], full["nall"])
            for b in x["run"].tolist():
                assert own[b[1]] == r                       # computed by the source's owner
                if b[0] < nb:
                    assert own[b[0]] == r
                    got.append(tuple(b))
                    continue
                org, ex, off, arena = plans[r].staging_block(b[0])   # the box itself, in the out arena
                assert arena == 0 and org == tuple(b[2:5]) and ex == tuple(b[5:8])
                q, rel = segment(x["send"], off)
                sent.setdefault((r, q), []).append((rel, b[1], tuple(b[2:8])))
            for u in x["unpack"].tolist():
                assert own[u[0]] == r and u[1] >= nb
                org, ex, off, arena = plans[r].staging_block(u[1])
                assert arena == 1 and org == tuple(u[2:5]) and ex == tuple(u[5:8])
                p, rel = segment(x["recv"], off)
                recvd.setdefault((p, r), []).append((rel, u[0], tuple(u[2:8])))
        # what r sends q is, offset by offset, what q unpacks from r
        assert sorted(sent) == sorted(recvd)
        for key in sent:
            a, b = sorted(sent[key]), sorted(recvd[key])
            assert [(o, g) for o, _, g in a] == [(o, g) for o, _, g in b]
            got += [(dst, src) + g for (_, src, g), (_, dst, _) in zip(a, b)]
        assert sorted(got) == sorted(tuple(b) for b in full["run"].tolist())
        assert sum(len(v) for v in sent.values()) == xs[0][k]["ncross"]
        for a in range(nranks):
            for (q, off, nbytes) in xs[a][k]["send"]:
                rec = [v for v in xs[q][k]["recv"] if v[0] == a]
                assert len(rec) == 1 and rec[0][2] == nbytes
    for p in plans + [whole]:
        p.close()


# ---- the exchange itself, two gloo ranks -------------------------------------

def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _initial(H, nf, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((nf, b.ex[2], b.ex[1], b.ex[0])) for b in H.blocks]


def _apply(kind, dst, dorg, dex, src, sorg, sex, lo, n):
    import oracle as O
    lib_o = O.lib()
    I3 = ctypes.c_int * 3
    P = ctypes.POINTER(ctypes.c_double)
    hi = [lo[d] + n[d] for d in range(3)]
    if kind == "sync":
        ds = tuple(slice(lo[d] - dorg[d], hi[d] - dorg[d]) for d in (2, 1, 0))
        ss = tuple(slice(lo[d] - sorg[d], hi[d] - sorg[d]) for d in (2, 1, 0))
        dst[(slice(None),) + ds] = src[(slice(None),) + ss]
        return
    for f in range(dst.shape[0]):
        if kind == "restrict":
            lib_o.oracle_restrict3_box(I3(*dex), I3(*dorg), dst[f].ctypes.data_as(P), I3(*sex), I3(*sorg),
                                       src[f].ctypes.data_as(P), I3(*lo), I3(*hi))
        else:
            lib_o.oracle_prolong3_box(I3(*sex), I3(*sorg), src[f].ctypes.data_as(P), I3(*dex), I3(*dorg),
                                      dst[f].ctypes.data_as(P), I3(*lo), I3(*hi))


def _exchange_rank(rank, world, port, out):
    _paths()
    from amss_b200 import dist as Dm
    import amr as OA
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        H = small_hierarchy()
        nb, nf = len(H.blocks), 24
        own = Dm.partition(H, world)
        init = _initial(H, nf, 7)
        # the oracle's transfers over all blocks in one process
        oh = OA.OracleHierarchy(H)
        for i, st in enumerate(init):
            oh.set_state(i, st)
        nlev = len(H.levels)
        for lv in range(nlev):
            oh.sync(lv, "state")
        for lv in range(1, nlev):
            oh.restrict_prolong(lv, True)
        # this rank: its own blocks only, the transfers of its plan
        plan = Dm.Plan.of(H, rank, world, own)
        xs = plan.xfers()
        arr = {i: init[i].copy() for i in range(nb) if own[i] == rank}
        blk = H.blocks
        sob = max(x["out_bytes"] for x in xs)
        sib = max(x["in_bytes"] for x in xs)
        arena = [np.zeros(max(sob, 8) // 8), np.zeros(max(sib, 8) // 8)]
        stage = {}

        def staging(sid):
            if sid not in stage:
                org, ex, off, a = plan.staging_block(sid)
                n = ex[0] * ex[1] * ex[2]
                v = arena[a][off // 8: off // 8 + nf * n].reshape(nf, ex[2], ex[1], ex[0])
                stage[sid] = (v, org, ex)
            return stage[sid]

        def geom(i):
            if i >= nb:
                return staging(i)
            return arr[i], blk[i].org, blk[i].ex

        def run(k):
            x = xs[k]
            for b in x["run"].tolist():
                d, s = geom(b[0]), geom(b[1])
                _apply(x["kind"], d[0], d[1], d[2], s[0], s[1], s[2], b[2:5], b[5:8])
            if x["ncross"] == 0:
                return
            reqs = []
            for q, off, nbytes in x["send"]:
                reqs.append(dist.isend(torch.from_numpy(arena[0][off // 8:(off + nbytes) // 8].copy()), q))
            bufs = []
            for q, off, nbytes in x["recv"]:
                t = torch.empty(nbytes // 8, dtype=torch.float64)
                reqs.append(dist.irecv(t, q))
                bufs.append((off, t))
            for rq in reqs:
                rq.wait()
            for off, t in bufs:
                arena[1][off // 8: off // 8 + t.numel()] = t.numpy()
            for b in x["unpack"].tolist():
                d, s = geom(b[0]), geom(b[1])
                _apply("sync", d[0], d[1], d[2], s[0], s[1], s[2], b[2:5], b[5:8])

        by = {(x["kind"], x["level"]): k for k, x in enumerate(xs)}
        for lv in range(nlev):
            run(by[("sync", lv)])
        for lv in range(1, nlev):
            run(by[("restrict", lv)])
            run(by[("sync", lv - 1)])
            run(by[("prolong", lv)])
            run(by[("sync", lv)])
        bad = [i for i in arr if not np.array_equal(arr[i], oh.state(i))]
        ncross = sum(x["ncross"] for x in xs)
        out[rank] = (bad, len(arr), ncross)
        dist.barrier()
        plan.close()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_single_process_transfers():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_exchange_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0][0] == [] and res[1][0] == [], res
    assert res[0][1] + res[1][1] == len(small_hierarchy().blocks)
    assert res[0][2] > 0


# ---- the in-process group's barrier -------------------------------------------

def test_group_barrier_meets_and_times_out():
    L = lib()
    g = L.amss_group_create(2, 0.5)
    assert g
    try:
        rcs = [None, None]

        def arrive(r):
            rcs[r] = L.amss_group_barrier(g)

        ts = [threading.Thread(target=arrive, args=(r,)) for r in range(2)]
        for t in ts:
            t.start()
        for t in ts:
            t.join(10)
        assert rcs == [0, 0]
        # one rank never arrives: the other gives up after the timeout
        t0 = time.perf_counter()
        rc = L.amss_group_barrier(g)
        waited = time.perf_counter() - t0
        assert rc < 0 and 0.4 <= waited < 5.0
        assert "timeout" in L.amss_last_error().decode()
        # and the group stays failed
        assert L.amss_group_barrier(g) < 0
    finally:
        L.amss_group_destroy(g)


def test_plan_refuses_device_calls():
    H = small_hierarchy()
    p = D.Plan.of(H, 0, 2, D.partition(H, 2))
    with pytest.raises(AmssError):
        p.coarse_step(0.1)
    with pytest.raises(AmssError):
        p.sync()
    p.close()


def test_nccl_transport_resolves_without_a_gpu():
    """The NCCL transport opens the libnccl already in the process (PyTorch's)
    at run time; making the unique id rank 0 broadcasts needs no GPU.  Joining
    a communicator needs a committed engine: a plan is refused."""
    L = lib()
    buf = ctypes.create_string_buffer(128)
    assert L.amss_nccl_unique_id(buf) == 0
    assert any(buf.raw)
    H = small_hierarchy()
    p = D.Plan.of(H, 0, 2, D.partition(H, 2))
    try:
        assert L.amss_engine_set_nccl(p._h, buf) < 0
        assert "commit" in L.amss_last_error().decode()
    finally:
        p.close()
