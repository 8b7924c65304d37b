"""Shot sharding and the gradient all-reduce on two gloo ranks (CPU).  Each
rank computes the FP64 restatement's gradient for its own shots; the summed
result must equal the serial gradient over all shots."""
import os
import socket

import numpy as np
import pytest

from bbwadg_b200.shards import shot_range


def test_shot_ranges_cover_every_shot_once():
    for n in (0, 1, 7, 32, 33):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shot_range(n, r, world)
                seen.extend(range(lo, hi))
                assert hi - lo in (n // world, n // world + 1)
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        shot_range(4, 2, 2)


def _problem():
    from bbwadg_b200 import make_problem
    from bbwadg_b200.problem import gaussian_source, receiver_weights
    p = make_problem(2, 2, c2="sine", c2_jitter=0.3, seed=1)
    rec = receiver_weights(p, np.array([[0.1, 0.2, -0.3], [0.4, -0.2, 0.3]]))
    centres = [(0.0, 0.0, 0.1), (0.3, -0.2, -0.1), (-0.3, 0.3, 0.2)]
    srcs = [dict(fsrc=gaussian_source(p, c, a=3.0).astype(np.float64), f0=10.0, tR=0.1,
                 amp=1e2, stage_times=True) for c in centres]
    return p, rec, srcs


def _grad(p, rec, srcs, shots):
    from test_adjoint_oracle import adjoint_oracle
    ad = adjoint_oracle(p)
    g = np.zeros((p.K, p.Nq))
    for i in shots:
        _, tr, st = ad.forward(p.Q0.astype(np.float64), float(p.dt), 6, rec, srcs[i])
        g += ad.backward(float(p.dt), 6, st, tr, rec, srcs[i])[0]
    return g


def _rank(rank, world, port, out):
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [here, os.path.join(here, ".."), os.path.join(here, "..", "oracle")]
    from bbwadg_b200.shards import allreduce_gradient
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    p, rec, srcs = _problem()
    lo, hi = shot_range(len(srcs), rank, world)
    g = allreduce_gradient(_grad(p, rec, srcs, range(lo, hi)))
    np.save(os.path.join(out, "g%d.npy" % rank), g)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_gradient_equals_serial(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    p, rec, srcs = _problem()
    serial = _grad(p, rec, srcs, range(len(srcs)))
    for r in range(2):
        g = np.load(str(tmp_path / ("g%d.npy" % r)))
        assert np.allclose(g, serial, rtol=1e-12, atol=1e-14 * np.abs(serial).max())
