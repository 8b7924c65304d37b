"""Slab decomposition (bbwadg_b200/decomp.py) on the CPU: the partition's
bookkeeping, and a two-rank gloo run in which each rank advances its slab
with the C restatement and refreshes its halo through DistExchange after
every stage; the owned elements must equal the single-mesh run bit for bit
(the per-element arithmetic does not depend on the cut)."""
import os
import socket

import numpy as np
import pytest

from bbwadg_b200 import make_problem
from bbwadg_b200.decomp import local_state, slab_partition


def _problem():
    return make_problem(3, 3, c2="sine", c2_jitter=0.3, seed=5)


def test_partition_bookkeeping():
    p = _problem()
    Np, NF = p.Np, 4 * (p.N + 1) * (p.N + 2) // 2
    parts = slab_partition(p, 3)
    owned = np.concatenate([q.owned for q in parts])
    assert np.array_equal(np.sort(owned), np.arange(p.K))
    vm = np.asarray(p.mesh["vmapP"]).reshape(p.K, NF)
    for q in parts:
        ids = q.ids
        lv = q.vmapP.reshape(q.K, NF)[:q.Kc]
        assert np.array_equal(ids[lv // (4 * Np)] * 4 * Np + lv % (4 * Np), vm[q.owned])
        nb = np.unique(vm[q.owned] // (4 * Np))
        assert np.array_equal(np.sort(q.halo), np.setdiff1d(nb, q.owned))
        for r, recv in q.recv.items():
            send = parts[r].send[q.index]
            assert np.array_equal(parts[r].ids[send], ids[recv])
            assert (recv >= q.Kc).all()
        assert sum(len(v) for v in q.recv.values()) == len(q.halo)


def _stage_loop(orc, Q, dt, nsteps, exchange):
    from oracle import RK4A, RK4B
    res = np.zeros_like(Q)
    rhs = np.zeros_like(Q)
    for _ in range(nsteps):
        for i in range(5):
            orc.rk_volume(Q, rhs)
            orc.rk_surface(Q, rhs)
            orc.rk_update_wadg(np.float32(RK4A[i]), np.float32(RK4B[i]), np.float32(dt), rhs, res, Q)
            exchange(Q)
    return Q


def _rank(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [here, os.path.join(here, ".."), os.path.join(here, "..", "oracle")]
    import torch
    import torch.distributed as dist
    from oracle import Oracle
    from bbwadg_b200.decomp import DistExchange
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    p = _problem()
    part = slab_partition(p, world)[rank]
    geo = dict(vgeo=part.vgeo, fgeo=part.fgeo, vmapP=part.vmapP, c2q=part.c2q,
               Jq=np.ones(part.c2q.size, np.float32))
    orc = Oracle(p.N, part.K, p.ops_dict(), geo)
    Q = np.ascontiguousarray(local_state(p, part, p.Q0), np.float32)
    rows = lambda: Q.reshape(part.K, -1)

    def gather(idx, buf):
        buf.copy_(torch.from_numpy(rows()[idx.numpy()].ravel()))

    def scatter(idx, buf):
        rows()[idx.numpy()] = buf.numpy().reshape(len(idx), -1)

    ex = DistExchange(part, gather, scatter, 4 * p.Np, torch.device("cpu"))
    _stage_loop(orc, Q, p.dt, 3, lambda _: ex())
    np.save(os.path.join(out, "q%d.npy" % rank), rows()[:part.Kc])
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_decomposed_run_equals_single_mesh(tmp_path):
    import torch.multiprocessing as mp
    from oracle import Oracle
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    p = _problem()
    Q = np.ascontiguousarray(p.Q0, np.float32).copy()
    _stage_loop(Oracle(p.N, p.K, p.ops_dict(), p.geo_dict()), Q, p.dt, 3, lambda _: None)
    full = Q.reshape(p.K, -1)
    for r, part in enumerate(slab_partition(p, 2)):
        assert np.array_equal(np.load(str(tmp_path / ("q%d.npy" % r))), full[part.owned])


def test_interface_first_partition():
    """Owned elements with a face neighbour in another part come first (Ki of
    them); the send lists name exactly those, and the maps still agree."""
    from bbwadg_b200 import make_problem
    p = make_problem(3, 4)
    parts = slab_partition(p, 3, interface_first=True)
    K, Np = p.K, p.Np
    nbr = np.asarray(p.mesh["vmapP"], np.int64).reshape(K, -1) // (4 * Np)
    part_of = np.empty(K, np.int64)
    for part in parts:
        part_of[part.owned] = part.index
    for part in parts:
        iface = (part_of[nbr[part.owned]] != part.index).any(1)
        assert iface[:part.Ki].all() and not iface[part.Ki:].any()
        sent = np.unique(np.concatenate(list(part.send.values())))
        assert np.array_equal(sent, np.arange(part.Ki))
        for q, idx in part.send.items():  # element sent to q is the one q receives
            g_sent = part.owned[idx]
            g_recv = parts[q].ids[parts[q].recv[part.index]]
            assert np.array_equal(g_sent, g_recv)

