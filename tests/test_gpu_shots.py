"""Batched shots, Ricker sources and receivers of the fused FP32 stage
against the C restatement run one shot at a time.

The source term follows acous_elas_cpp (src/WaveOKL3d.cpp:176-186, 226-228,
765-781; okl/ElasKernelsWADG.okl:400-403): ricker(t) * Pq f added to the
projected rhs_p.  FP32 tolerance: 1e-5 relative L2 on the states, 1e-4 on
the traces (a handful of small values each)."""
import numpy as np
import pytest
from conftest import rel_l2

from bbwadg_b200 import WaveSolver, make_problem
from bbwadg_b200._lib import BBWError
from bbwadg_b200.problem import gaussian_source, receiver_weights, source_entries

pytestmark = pytest.mark.gpu
TOL = 1e-5


def oracle_for(p):
    from oracle import Oracle
    return Oracle(p.N, p.K, p.ops_dict(), p.geo_dict(), variant=p.variant)


@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("N", [3, 5])
def test_batched_shots_match_single_runs(cuda, variant, N):
    p = make_problem(N, 3, variant=variant, c2="sine", c2_jitter=0.5, seed=1)
    rng = np.random.default_rng(0)
    S = 3
    Q0 = np.stack([p.Q0 * (1.0 + 0.5 * s) + 0.01 * rng.standard_normal(p.Q0.size)
                   for s in range(S)]).astype(np.float32)
    s = WaveSolver(p)
    s.set_shots(S)
    s.set_data(Q0)
    s.steps(p.dt, 6)
    out = s.get_data().reshape(S, -1)
    s.close()
    orc = oracle_for(p)
    for i in range(S):
        q, _ = orc.run(Q0[i].copy(), p.dt, 30)
        assert rel_l2(out[i], q) < TOL, i


@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("stage_times", [False, True])
def test_sources_and_receivers_match_oracle(cuda, variant, stage_times):
    p = make_problem(3, 3, variant=variant, c2="sine", seed=2)
    centres = [(0.0, 0.0, 0.1), (0.3, -0.2, 0.0)]
    pts = np.array([[0.05, 0.0, 0.1], [0.2, 0.1, 0.0], [-0.3, 0.4, 0.5]])
    el, w = receiver_weights(p, pts)
    S, nsteps = 2, 40
    dense, ent = [], []
    for i, x0 in enumerate(centres):
        f = gaussian_source(p, x0, a=5.0)
        dense.append(f)
        ent.append(source_entries(f, shot=i))
    s = WaveSolver(p)
    s.set_shots(S)
    s.set_sources(*(np.concatenate(x) for x in zip(*ent)), f0=10.0, amplitude=1e4,
                  stage_times=stage_times)
    s.set_receivers(el, w, nsteps)
    s.set_time(0.0)
    s.steps(p.dt, nsteps)
    traces = s.get_traces()
    Q = s.get_data().reshape(S, -1)
    t, st = s.get_time()
    s.close()
    assert st == nsteps
    assert abs(t - nsteps * np.float64(np.float32(p.dt))) < 1e-12
    assert traces.shape == (S, len(el), nsteps)
    orc = oracle_for(p)
    for i in range(S):
        src = dict(fsrc=dense[i], f0=10.0, tR=0.1, amp=1e4, stage_times=stage_times)
        q, _, tr = orc.run(np.zeros(p.K * 4 * p.Np, np.float32), np.float32(p.dt), 5 * nsteps,
                           source=src, receivers=(el, w))
        assert np.linalg.norm(q) > 0
        assert rel_l2(Q[i], q) < TOL, i
        assert rel_l2(traces[i], tr) < 1e-4, i


def test_source_time_is_the_device_clock(cuda):
    """A later start time changes the injected wavelet: set_time(t0) must
    match the oracle started at t0."""
    p = make_problem(3, 2, c2="one")
    f = gaussian_source(p, (0.0, 0.0, 0.0), a=3.0)
    s = WaveSolver(p)
    s.set_sources(*source_entries(f), f0=10.0, amplitude=1e4)
    s.set_data(np.zeros(p.K * 4 * p.Np, np.float32))
    s.set_time(0.05)
    s.steps(p.dt, 10)
    q_gpu = s.get_data()
    s.close()
    src = dict(fsrc=f, f0=10.0, tR=0.1, amp=1e4)
    q, _ = oracle_for(p).run(np.zeros(p.K * 4 * p.Np, np.float32), np.float32(p.dt), 50,
                             source=src, t0=0.05)
    assert rel_l2(q_gpu, q) < TOL


def test_receivers_stop_at_capacity_and_reset(cuda):
    p = make_problem(3, 2)
    el, w = receiver_weights(p, np.array([[0.1, 0.1, 0.1]]))
    s = WaveSolver(p)
    s.set_data(p.Q0)
    s.set_receivers(el, w, 3)
    s.steps(p.dt, 5)
    assert s.get_traces().shape == (1, 1, 3)
    assert s.get_time()[1] == 5
    s.set_time(0.0)
    assert s.get_traces().shape == (1, 1, 0)
    s.close()


def test_bad_arguments_are_rejected(cuda):
    p = make_problem(3, 2)
    s = WaveSolver(p)
    with pytest.raises(BBWError):
        s.set_sources([0], [p.K], np.zeros((1, p.Np), np.float32))
    with pytest.raises(BBWError):
        s.set_sources([1], [0], np.zeros((1, p.Np), np.float32))  # only one shot
    with pytest.raises(BBWError):
        s.set_receivers([-1], np.zeros((1, p.Np), np.float32), 4)
    with pytest.raises(ValueError):
        s.set_data(np.zeros(3, np.float32))
    s.close()


@pytest.mark.parametrize("n_elems", [1, 2])
@pytest.mark.parametrize("N", [1, 2, 4])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_shots_on_one_and_two_elements(cuda, n_elems, N, variant):
    """Three shots of a one- or two-element mesh: every (shot, tile) work
    item is a partial tile; each shot against its own oracle run."""
    VX = np.array([0.0, 1.0, 0.0, 0.0, 0.3])
    VY = np.array([0.0, 0.0, 1.0, 0.0, 0.3])
    VZ = np.array([0.0, 0.0, 0.0, 1.0, -0.9])
    EToV = np.array([[0, 1, 2, 3], [0, 2, 1, 4]][:n_elems], np.int32)
    p = make_problem(N, mesh=(VX, VY, VZ, EToV), variant=variant, c2="sine", seed=4)
    rng = np.random.default_rng(N)
    S = 3
    Q0 = np.stack([p.Q0 * (1.0 - 0.3 * s) + 0.05 * rng.standard_normal(p.Q0.size)
                   for s in range(S)]).astype(np.float32)
    s = WaveSolver(p)
    s.set_shots(S)
    s.set_data(Q0)
    s.steps(p.dt, 3)
    out = s.get_data().reshape(S, -1)
    s.close()
    orc = oracle_for(p)
    for i in range(S):
        q, _ = orc.run(Q0[i].copy(), p.dt, 15)
        assert rel_l2(out[i], q) < TOL, i


@pytest.mark.parametrize("prec", ["f16x3", "bf16x3"])
@pytest.mark.parametrize("N", [3, 4])
def test_tensor_core_shots_sources_and_receivers_match_oracle(cuda, prec, N):
    """The split-precision tensor-core stage with batched shots, Ricker
    sources at the stage times and receivers, against the FP32 restatement
    run one shot at a time (N = 4: the reference's 57-point rule)."""
    from conftest import golden
    g = golden("ops_N%d.npz" % N)
    nfq = int(g["Nfq"][0])
    p = make_problem(N, 3, variant="nodal", c2="sine", c2_jitter=0.3, seed=2,
                     cubature=(g["rq"], g["sq"], g["tq"], g["wq"]),
                     tri_cubature=(g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))
    centres = [(0.0, 0.0, 0.1), (0.3, -0.2, 0.0), (-0.2, 0.4, -0.3)]
    pts = np.array([[0.05, 0.0, 0.1], [0.2, 0.1, 0.0], [-0.3, 0.4, 0.5]])
    el, w = receiver_weights(p, pts)
    S, nsteps = 3, 30
    dense = [gaussian_source(p, x0, a=5.0) for x0 in centres]
    ent = [source_entries(f, shot=i) for i, f in enumerate(dense)]
    s = WaveSolver(p, precision=prec)
    s.set_shots(S)
    s.set_grid_limit(2)  # every CTA walks shots and tiles
    s.set_sources(*(np.concatenate(x) for x in zip(*ent)), f0=10.0, amplitude=1e4,
                  stage_times=True)
    s.set_receivers(el, w, nsteps)
    s.set_time(0.0)
    s.steps(p.dt, nsteps)
    s.check()
    traces = s.get_traces()
    Q = s.get_data().reshape(S, -1)
    s.close()
    orc = oracle_for(p)
    for i in range(S):
        src = dict(fsrc=dense[i], f0=10.0, tR=0.1, amp=1e4, stage_times=True)
        q, _, tr = orc.run(np.zeros(p.K * 4 * p.Np, np.float32), np.float32(p.dt), 5 * nsteps,
                           source=src, receivers=(el, w))
        assert rel_l2(Q[i], q) < TOL, i
        assert rel_l2(traces[i], tr) < 1e-4, i
