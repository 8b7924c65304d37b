"""CPU checks of the FP64 discrete-adjoint restatement (oracle/adjoint.py),
the checker of the GPU adjoint: its forward against the C restatement, its
gradient against central finite differences (FP64, 5 seeded directions)."""
import numpy as np
import pytest

from bbwadg_b200 import make_problem
from bbwadg_b200.problem import gaussian_source, receiver_weights


def cm(a, rows, cols):
    return np.asarray(a, np.float64).reshape(cols, rows).T


def colmajor(M):
    return np.ascontiguousarray(M.T).ravel()


def dense_ops(p):
    """FP64 dense operators of the problem's basis (column-major)."""
    o, Np = p.ops, p.Np
    if p.variant == "nodal":
        D = [o["Dr64"], o["Ds64"], o["Dt64"]]
        LIFT = o["LIFT64"]
    else:
        VB, iVB = cm(o["VB64"], Np, Np), cm(o["invVB64"], Np, Np)
        D = [colmajor(iVB @ cm(o[k + "64"], Np, Np) @ VB) for k in ("Dr", "Ds", "Dt")]
        LIFT = o["LIFTB64"]
    return D, LIFT, o["Vq_%s64" % p.variant], o["Pq_%s64" % p.variant]


def adjoint_oracle(p, bc=0, c2q=None):
    from adjoint import AdjointOracle
    D, LIFT, Vq, Pq = dense_ops(p)
    m = p.mesh
    return AdjointOracle(p.N, p.K, D, LIFT, Vq, Pq, p.ops["Fmask"], m["vgeo"], m["fgeo"],
                         m["vmapP"], p.c2q if c2q is None else c2q, bc=bc)


@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("bc", [0, 1])
def test_dense_forward_matches_c_restatement(variant, bc):
    from oracle import Oracle
    p = make_problem(3, 2, variant=variant, c2="sine", c2_jitter=0.3, seed=4)
    rng = np.random.default_rng(1)
    Q = rng.standard_normal(p.K * 4 * p.Np)
    orc = Oracle(3, p.K, p.ops_dict(), p.geo_dict(), variant=variant, bc=bc, dtype=np.float64)
    rhs = np.zeros_like(Q)
    orc.rk_volume(Q, rhs)
    orc.rk_surface(Q, rhs)
    ours = adjoint_oracle(p, bc).S(Q.reshape(p.K, 4, p.Np)).ravel()
    assert np.linalg.norm(ours - rhs) <= 1e-5 * np.linalg.norm(rhs)


def _setup(variant, bc, seed=0):
    p = make_problem(3, 2, variant=variant, c2="sine", c2_jitter=0.3, seed=seed)
    pts = np.array([[0.1, 0.2, -0.3], [0.5, -0.5, 0.25], [-0.4, 0.0, 0.6]])
    rec = receiver_weights(p, pts)
    src = dict(fsrc=gaussian_source(p, (0.0, 0.0, 0.1), a=3.0).astype(np.float64), f0=10.0,
               tR=0.1, amp=1e2, stage_times=True)
    return p, rec, src


@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("bc", [0, 1])
def test_adjoint_gradient_matches_finite_differences(variant, bc):
    p, rec, src = _setup(variant, bc)
    ad = adjoint_oracle(p, bc)
    dt, nsteps = float(p.dt), 12
    Q0 = p.Q0.astype(np.float64)

    def loss(c2q):
        ad.c2q = c2q
        _, tr, _ = ad.forward(Q0, dt, nsteps, rec, src)
        return 0.5 * float((tr ** 2).sum())

    c2 = ad.c2q.copy()
    _, tr, states = ad.forward(Q0, dt, nsteps, rec, src)
    grad, _ = ad.backward(dt, nsteps, states, tr, rec, src)
    rng = np.random.default_rng(7)
    for _ in range(5):
        d = rng.standard_normal(c2.shape)
        eps = 1e-4
        fd = (loss(c2 + eps * d) - loss(c2 - eps * d)) / (2 * eps)
        ad.c2q = c2
        an = float((grad * d).sum())
        assert abs(fd - an) <= 1e-7 * max(abs(fd), 1e-300), (fd, an)


def test_adjoint_state_gradient_matches_finite_differences():
    p, rec, src = _setup("nodal", 0, seed=2)
    ad = adjoint_oracle(p)
    dt, nsteps = float(p.dt), 8
    Q0 = p.Q0.astype(np.float64).reshape(p.K, 4, p.Np)
    _, tr, states = ad.forward(Q0, dt, nsteps, rec, src)
    _, gQ = ad.backward(dt, nsteps, states, tr, rec, src)
    d = np.random.default_rng(3).standard_normal(Q0.shape)
    eps = 1e-5

    def loss(Q):
        return 0.5 * float((ad.forward(Q, dt, nsteps, rec, src)[1] ** 2).sum())

    fd = (loss(Q0 + eps * d) - loss(Q0 - eps * d)) / (2 * eps)
    assert abs(fd - float((gQ * d).sum())) <= 1e-7 * abs(fd)
