"""GPU discrete adjoint (bbw_forward / bbw_backward) against the FP64
restatement (oracle/adjoint.py) and FP64 central finite differences.

Tolerances: gradient vs the FP64 discrete adjoint 1e-4 relative L2;
directional derivatives vs finite differences 1e-4 relative (5 seeded
directions)."""
import numpy as np
import pytest
from conftest import rel_l2
from test_adjoint_oracle import adjoint_oracle

from bbwadg_b200 import WaveSolver, make_problem
from bbwadg_b200._lib import BBWError
from bbwadg_b200.problem import gaussian_source, receiver_weights, source_entries

pytestmark = pytest.mark.gpu
TOL = 1e-4


def setup(variant, bc, S=2, N=3, n=2, seed=0, rules=(None, None)):
    p = make_problem(N, n, variant=variant, c2="sine", c2_jitter=0.3, seed=seed,
                     cubature=rules[0], tri_cubature=rules[1])
    pts = np.array([[0.1, 0.2, -0.3], [0.5, -0.5, 0.25], [-0.4, 0.0, 0.6], [0.0, 0.3, 0.0]])
    rec = receiver_weights(p, pts)
    centres = [(0.0, 0.0, 0.1), (0.3, -0.2, -0.1), (-0.3, 0.3, 0.2)][:S]
    dense = [gaussian_source(p, x0, a=3.0) for x0 in centres]
    return p, rec, dense


def gpu_gradient(p, rec, dense, bc, nsteps, every, Q0, stage_times=True, precision="fp32",
                 keep="cubature"):
    S = len(dense)
    s = WaveSolver(p, bc="rigid" if bc else "pressure_release", precision=precision)
    s.set_shots(S)
    ent = [source_entries(f, shot=i, rtol=0.0) for i, f in enumerate(dense)]
    s.set_sources(*(np.concatenate(x) for x in zip(*ent)), f0=10.0, amplitude=1e2,
                  stage_times=stage_times)
    s.set_receivers(*rec, nsteps)
    s.set_data(np.tile(Q0, S))
    s.set_time(0.0)
    tape = s.forward(p.dt, nsteps, every, keep=keep)
    assert tape.kind == keep  # small meshes: the cubature tape always fits
    tr = s.get_traces()
    grad, dq = s.backward(tape, tr, want_state=True)
    tape.free()
    s.close()
    return tr, grad, dq


def oracle_gradient(p, rec, dense, bc, nsteps, Q0, stage_times=True):
    ad = adjoint_oracle(p, bc)
    dt = float(np.float32(p.dt))
    total = np.zeros((p.K, p.Nq))
    trs = []
    for f in dense:
        src = dict(fsrc=f.astype(np.float64), f0=10.0, tR=0.1, amp=1e2, stage_times=stage_times)
        _, tr, states = ad.forward(Q0.astype(np.float64), dt, nsteps, rec, src)
        g, _ = ad.backward(dt, nsteps, states, tr, rec, src)
        total += g
        trs.append(tr)
    return np.array(trs), total, ad


@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("bc", [0, 1])
def test_gradient_matches_fp64_adjoint(cuda, variant, bc):
    p, rec, dense = setup(variant, bc)
    nsteps = 12
    tr, grad, _ = gpu_gradient(p, rec, dense, bc, nsteps, 5, p.Q0)
    tr64, grad64, _ = oracle_gradient(p, rec, dense, bc, nsteps, p.Q0)
    assert rel_l2(tr, tr64) < 1e-5
    assert rel_l2(grad, grad64) < TOL


@pytest.mark.parametrize("N", [5, 6, 7])
def test_gradient_matches_fp64_adjoint_higher_orders(cuda, N):
    """The reference's cubature rules (Nq = 95, 146, 214).  N = 5: the
    reverse-stage kernels stage their operators in shared memory; N = 7: too
    large to stage, they read them from global memory."""
    from conftest import golden
    g = golden("ops_N%d.npz" % N)
    nfq = int(np.asarray(g["Nfq"]).ravel()[0])
    rules = ((g["rq"], g["sq"], g["tq"], g["wq"]), (g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))
    p, rec, dense = setup("nodal", 0, S=1, N=N, rules=rules)
    nsteps = 4
    tr, grad, _ = gpu_gradient(p, rec, dense, 0, nsteps, 2, p.Q0)
    tr64, grad64, _ = oracle_gradient(p, rec, dense, 0, nsteps, p.Q0)
    assert rel_l2(tr, tr64) < 1e-5
    assert rel_l2(grad, grad64) < TOL


def test_directional_derivatives_match_finite_differences(cuda):
    p, rec, dense = setup("nodal", 0, S=1)
    nsteps = 12
    _, grad, _ = gpu_gradient(p, rec, dense, 0, nsteps, 4, p.Q0)
    ad = adjoint_oracle(p, 0)
    dt = float(np.float32(p.dt))
    src = dict(fsrc=dense[0].astype(np.float64), f0=10.0, tR=0.1, amp=1e2, stage_times=True)
    c2 = ad.c2q.copy()

    def loss(c):
        ad.c2q = c
        return 0.5 * float((ad.forward(p.Q0.astype(np.float64), dt, nsteps, rec, src)[1] ** 2).sum())

    rng = np.random.default_rng(11)
    for _ in range(5):
        d = rng.standard_normal(c2.shape)
        eps = 1e-4
        fd = (loss(c2 + eps * d) - loss(c2 - eps * d)) / (2 * eps)
        assert abs(float((grad * d).sum()) - fd) <= TOL * abs(fd)


def test_checkpoint_interval_does_not_change_the_gradient(cuda):
    p, rec, dense = setup("nodal", 0, S=1)
    ref = gpu_gradient(p, rec, dense, 0, 10, 1, p.Q0, keep="checkpoints")[1]
    for every in (3, 10, 64):
        assert np.array_equal(
            gpu_gradient(p, rec, dense, 0, 10, every, p.Q0, keep="checkpoints")[1], ref)


@pytest.mark.parametrize("precision", ["fp32", "f16x3"])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_cubature_tape_equals_checkpoint_tape(cuda, variant, precision):
    """A tape of every stage's cubature values (no recomputation in the
    backward pass) and a checkpoint tape (each segment recomputed) give the
    same traces, c^2 gradient and state gradient bit for bit: the forward
    stages are the same kernels on the same inputs."""
    p, rec, dense = setup(variant, 0, S=2)
    a = gpu_gradient(p, rec, dense, 0, 12, 5, p.Q0, precision=precision, keep="cubature")
    b = gpu_gradient(p, rec, dense, 0, 12, 5, p.Q0, precision=precision, keep="checkpoints")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_state_gradient_matches_fp64_adjoint(cuda):
    p, rec, dense = setup("nodal", 0, S=1)
    _, _, dq = gpu_gradient(p, rec, dense, 0, 8, 3, p.Q0)
    ad = adjoint_oracle(p, 0)
    dt = float(np.float32(p.dt))
    src = dict(fsrc=dense[0].astype(np.float64), f0=10.0, tR=0.1, amp=1e2, stage_times=True)
    _, tr, states = ad.forward(p.Q0.astype(np.float64), dt, 8, rec, src)
    _, gQ = ad.backward(dt, 8, states, tr, rec, src)
    assert rel_l2(dq, gQ.ravel()) < TOL


def test_autograd_function(cuda):
    import torch
    from bbwadg_b200.autograd import receiver_traces
    p, rec, dense = setup("nodal", 0, S=1)
    s = WaveSolver(p)
    s.set_sources(*source_entries(dense[0], rtol=0.0), f0=10.0, amplitude=1e2, stage_times=True)
    s.set_receivers(*rec, 16)
    c2 = torch.tensor(p.c2q, dtype=torch.float64, requires_grad=True)
    tr = receiver_traces(c2, s, p.Q0, p.dt, 10, 4)
    loss = 0.5 * (tr.double() ** 2).sum()
    loss.backward()
    _, g64, _ = oracle_gradient(p, rec, dense, 0, 10, p.Q0)
    assert rel_l2(c2.grad.numpy(), g64) < TOL
    s.close()


def test_adjoint_errors(cuda):
    p, rec, dense = setup("nodal", 0, S=1)
    s = WaveSolver(p)
    with pytest.raises(BBWError):  # no receivers
        s.forward(p.dt, 4, 2)
    s.set_receivers(*rec, 3)
    with pytest.raises(BBWError):  # capacity
        s.forward(p.dt, 4, 2)
    s.close()


@pytest.mark.parametrize("n_elems", [1, 2])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_gradient_on_one_and_two_elements(cuda, n_elems, variant):
    """Partial element tiles in every forward and reverse kernel: one
    element (all faces walls) or two sharing a face, two shots."""
    VX = np.array([0.0, 1.0, 0.0, 0.0, 0.3])
    VY = np.array([0.0, 0.0, 1.0, 0.0, 0.3])
    VZ = np.array([0.0, 0.0, 0.0, 1.0, -0.9])
    EToV = np.array([[0, 1, 2, 3], [0, 2, 1, 4]][:n_elems], np.int32)
    p = make_problem(3, mesh=(VX, VY, VZ, EToV), variant=variant, c2="sine", c2_jitter=0.3,
                     seed=6)
    pts = np.array([[0.2, 0.2, 0.2], [0.1, 0.3, 0.1], [0.3, 0.3, -0.2]][:2 + (n_elems - 1)])
    rec = receiver_weights(p, pts)
    dense = [gaussian_source(p, x0, a=3.0) for x0 in ((0.2, 0.2, 0.1), (0.1, 0.1, 0.3))]
    nsteps = 10
    tr, grad, _ = gpu_gradient(p, rec, dense, 0, nsteps, 4, p.Q0)
    tr64, grad64, _ = oracle_gradient(p, rec, dense, 0, nsteps, p.Q0)
    assert rel_l2(tr, tr64) < 1e-5
    assert rel_l2(grad, grad64) < TOL


def test_gradient_at_size_matches_fp64_adjoint_and_finite_differences(cuda):
    """A mid-size case: N = 4 with the reference's 57-point rule, 4^3 x 6
    tets (K = 384), 2 shots, 16 seeded receivers, 100 LSRK45 steps,
    checkpoints every 25.  The GPU gradient against the FP64 discrete
    adjoint, and its directional derivatives along 5 seeded directions
    against FP64 central finite differences of the misfit."""
    from conftest import golden
    g = golden("ops_N4.npz")
    nfq = int(np.asarray(g["Nfq"]).ravel()[0])
    rules = ((g["rq"], g["sq"], g["tq"], g["wq"]), (g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))
    p = make_problem(4, 4, variant="nodal", c2="sine", c2_jitter=0.3, seed=21, cubature=rules[0],
                     tri_cubature=rules[1])
    assert p.K == 384
    rng = np.random.default_rng(64)
    rec = receiver_weights(p, rng.uniform(-0.8, 0.8, (16, 3)))
    dense = [gaussian_source(p, x0, a=3.0) for x0 in rng.uniform(-0.5, 0.5, (2, 3))]
    nsteps, every = 100, 25
    Q0 = np.zeros_like(p.Q0)
    tr, grad, _ = gpu_gradient(p, rec, dense, 0, nsteps, every, Q0)
    tr64, grad64, ad = oracle_gradient(p, rec, dense, 0, nsteps, Q0)
    assert rel_l2(tr, tr64) < 1e-5
    assert rel_l2(grad, grad64) < TOL
    dt = float(np.float32(p.dt))
    srcs = [dict(fsrc=f.astype(np.float64), f0=10.0, tR=0.1, amp=1e2, stage_times=True)
            for f in dense]
    c2 = ad.c2q.copy()

    def loss(c):
        ad.c2q = c
        return sum(0.5 * float((ad.forward(Q0.astype(np.float64), dt, nsteps, rec, s)[1] ** 2).sum())
                   for s in srcs)

    for _ in range(5):
        d = rng.standard_normal(c2.shape)
        eps = 1e-4
        fd = (loss(c2 + eps * d) - loss(c2 - eps * d)) / (2 * eps)
        assert abs(float((grad * d).sum()) - fd) <= TOL * abs(fd)


@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("N", [3, 5])
def test_gradient_with_the_tensor_core_forward(cuda, variant, N):
    """The forward pass and its recomputation on the split-FP16 tensor-core
    stage (the reverse stages use the FP32 transposed operators): the
    gradient against the FP64 discrete adjoint, and a directional derivative
    against FP64 central finite differences; checkpoint intervals agree bit
    for bit."""
    from conftest import golden
    g = golden("ops_N%d.npz" % N)
    nfq = int(np.asarray(g["Nfq"]).ravel()[0])
    rules = ((g["rq"], g["sq"], g["tq"], g["wq"]), (g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))
    p, rec, dense = setup(variant, 0, S=2, N=N, rules=rules)
    nsteps = 10
    tr, grad, _ = gpu_gradient(p, rec, dense, 0, nsteps, 3, p.Q0, precision="f16x3")
    tr64, grad64, ad = oracle_gradient(p, rec, dense, 0, nsteps, p.Q0)
    assert rel_l2(tr, tr64) < 1e-5
    assert rel_l2(grad, grad64) < TOL
    assert np.array_equal(gpu_gradient(p, rec, dense, 0, nsteps, 10, p.Q0, precision="f16x3")[1],
                          grad)
    dt = float(np.float32(p.dt))
    srcs = [dict(fsrc=f.astype(np.float64), f0=10.0, tR=0.1, amp=1e2, stage_times=True)
            for f in dense]
    c2 = ad.c2q.copy()

    def loss(c):
        ad.c2q = c
        return sum(0.5 * float((ad.forward(p.Q0.astype(np.float64), dt, nsteps, rec, s)[1] ** 2)
                               .sum()) for s in srcs)

    d = np.random.default_rng(5).standard_normal(c2.shape)
    eps = 1e-4
    fd = (loss(c2 + eps * d) - loss(c2 - eps * d)) / (2 * eps)
    assert abs(float((grad * d).sum()) - fd) <= TOL * abs(fd)
