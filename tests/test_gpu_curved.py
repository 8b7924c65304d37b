"""Curvilinear WADG path on the GPU against the reference's own kernels
and runs (tests/golden/curved_*_N*.npz: kuhn_ball(4) and the reference's
sphere48 / sphere385 meshes) and the FP64 restatement
(oracle/curved.py) at orders the reference's curving does not define.

FP32 tolerance: 1e-5 relative L2 on states and kernel outputs; 1e-3 on the
LSRK residual after 50 stages (a small difference of large terms)."""
import ctypes

import numpy as np
import pytest
from conftest import golden, rel_l2
from test_curved import oracle_of, problem_like_reference

from bbwadg_b200 import _lib
from bbwadg_b200._lib import BBWError
from bbwadg_b200.curved import CurvedSolver, make_curved_problem
from bbwadg_b200.mesh import kuhn_ball, kuhn_box
from bbwadg_b200.problem import c2_sine

pytestmark = pytest.mark.gpu
TOL = 1e-5
RK4A = (0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
        -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0)
RK4B = (1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
        1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
        2277821191437.0 / 14882151754819.0)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def stages(s, dt, n):
    for i in range(n):
        s.rk_stage(np.float32(RK4A[i % 5]), np.float32(RK4B[i % 5]), np.float32(dt))


@pytest.mark.parametrize("kernel", ["rk_volume_WADG_skew_combine", "rk_surface_WADG_skew_combine",
                                    "rk_volume_planar", "rk_surface_planar"])
def test_kernel_entries_match_reference(cuda, kernel):
    import torch
    p, g = problem_like_reference(3)
    a = {k: dev(v) for k, v in p.desc_arrays().items()}
    q, r = dev(g["q_in"]), dev(g["rhs_in"])
    P = _lib.ptr
    KC, KP = len(p.KlistCurved), len(p.KlistPlanar)
    if kernel == "rk_volume_WADG_skew_combine":
        _lib.call("bbw_rk_volume_wadg_skew_combine", p.N, p.Nq, KC, P(a["KlistCurved"]),
                  P(a["vgeoq"]), P(a["Jq"]), P(a["Vq"]), P(a["Vrq"]), P(a["Vsq"]), P(a["Vtq"]),
                  P(a["Pq"]), P(a["Prq"]), P(a["Psq"]), P(a["Ptq"]), None, None, P(q), P(r), None)
    elif kernel == "rk_surface_WADG_skew_combine":
        _lib.call("bbw_rk_surface_wadg_skew_combine", p.N, p.Nfq, KC, P(a["KlistCurved"]),
                  P(a["fgeo"]), P(a["fgeoq"]), P(a["VfqFace"]), P(a["Pfq"]), P(a["Fmask"]),
                  P(a["vmapP"]), P(q), P(r), None)
    elif kernel == "rk_volume_planar":
        _lib.call("bbw_rk_volume_planar", p.N, KP, P(a["KlistPlanar"]), P(a["vgeo"]),
                  P(a["Jplanar"]), P(a["Dr"]), P(a["Ds"]), P(a["Dt"]), P(q), P(r), None)
    else:
        _lib.call("bbw_rk_surface_planar", p.N, KP, P(a["KlistPlanar"]), P(a["fgeo"]),
                  P(a["Jplanar"]), P(a["Fmask"]), P(a["vmapP"]), P(a["LIFT"]), P(q), P(r), None)
    torch.cuda.synchronize()
    assert rel_l2(r.cpu().numpy(), g[kernel + ".rhsQ"]) < TOL


@pytest.mark.parametrize("mesh", ["ball4", "sphere48", "sphere385"])
@pytest.mark.parametrize("N", [2, 3])
def test_stages_match_reference(cuda, N, mesh):
    """50 stages on kuhn_ball(4) and on the reference's own sphere meshes
    (sphere48.msh: every element curved; sphere385.msh) against the
    reference's RK_step_WADG run on them."""
    p, g = problem_like_reference(N, mesh)
    s = CurvedSolver(p)
    s.set_data(p.Q0)
    stages(s, float(g["dt"][0]), int(g["stages"]))
    Q, res = s.get_data(), s.get_residual()
    s.close()
    assert rel_l2(Q, g["Q_run"]) < TOL
    assert rel_l2(res, g["res_run"]) < 1e-3


def test_graph_steps_equal_stage_loop(cuda):
    p = make_curved_problem(3, 4, c2=c2_sine)
    out = []
    for graph in (False, True):
        s = CurvedSolver(p)
        s.set_data(p.Q0)
        if graph:
            s.steps(p.dt, 4)
        else:
            stages(s, p.dt, 20)
        out.append(s.get_data())
        s.close()
    assert np.array_equal(out[0], out[1])


def reference_rules(N):
    """The reference's tabulated degree-2N+1 rules where a fixture holds them
    (the fused planar stage keeps a 32-element tile of Nq points in shared
    memory: N = 7 needs the reference's 214-point rule, not the 512-point
    Stroud rule)."""
    import os
    from conftest import GOLDEN
    if not os.path.exists(os.path.join(GOLDEN, "ops_N%d.npz" % N)):
        return None, None
    g = golden("ops_N%d.npz" % N)
    nfq = int(np.asarray(g["Nfq"]).ravel()[0])
    return (g["rq"], g["sq"], g["tq"], g["wq"]), (g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"])


@pytest.mark.parametrize("N", [1, 4, 5, 6, 7])
def test_matches_oracle_at_higher_orders(cuda, N):
    cub, tri = reference_rules(N)
    p = make_curved_problem(N, 4, c2=c2_sine, cubature=cub, tri_cubature=tri)
    s = CurvedSolver(p)
    s.set_data(p.Q0)
    stages(s, p.dt, 10)
    Q = s.get_data()
    s.close()
    Qo, _ = oracle_of(p).run(p.Q0, p.dt, 10)
    assert rel_l2(Q, Qo) < TOL


def test_all_curved_mesh(cuda):
    p = make_curved_problem(3, mesh=kuhn_ball(2), c2=c2_sine)
    assert len(p.KlistPlanar) == 0
    s = CurvedSolver(p)
    s.set_data(p.Q0)
    stages(s, p.dt, 10)
    Q = s.get_data()
    s.close()
    assert rel_l2(Q, oracle_of(p).run(p.Q0, p.dt, 10)[0]) < TOL


def test_all_planar_mesh_matches_affine_path(cuda):
    """No element touches the sphere: the J-weighted planar kernels plus the
    1/J update reproduce the affine path (C restatement, Jq = 1)."""
    from oracle import Oracle
    N = 3
    p = make_curved_problem(N, mesh=kuhn_box(2, -0.5, 0.5), c2=c2_sine)
    assert len(p.KlistCurved) == 0
    s = CurvedSolver(p)
    s.set_data(p.Q0)
    stages(s, p.dt, 25)
    Q = s.get_data()
    s.close()
    ops = dict(p.ops)
    ops["Vq"], ops["Pq"] = ops["Vq_nodal"], ops["Pq_nodal"]
    geo = dict(vgeo=p.mesh["vgeo"], fgeo=p.mesh["fgeo"], vmapP=p.mesh["vmapP"],
               c2q=p.c2q.ravel(), Jq=np.ones(p.K * p.Nq, np.float32))
    q, _ = Oracle(N, p.K, ops, geo, variant="nodal").run(p.Q0.copy(), np.float32(p.dt), 25)
    assert rel_l2(Q, q) < TOL


def test_bad_descriptions_are_rejected(cuda):
    p = make_curved_problem(2, 4)
    a = p.desc_arrays()

    def create(**over):
        arrs = dict(a, **over)
        d = _lib.CurvedDesc(N=p.N, K=p.K, Nq=p.Nq, Nfq=p.Nfq, Nq_reduced=p.Nq,
                            KCurved=len(arrs["KlistCurved"]), KPlanar=len(arrs["KlistPlanar"]))
        for k, v in arrs.items():
            setattr(d, k, _lib.ptr(v))
        h = ctypes.c_void_p()
        _lib.call("bbw_curved_create", ctypes.byref(d), 0, ctypes.byref(h))
        _lib.call("bbw_curved_destroy", h)

    create()
    dup = a["KlistCurved"].copy()
    dup[1] = dup[0]
    with pytest.raises(BBWError):
        create(KlistCurved=dup)
    bad = a["vmapP"].copy()
    bad[5] = p.K * 4 * p.Np
    with pytest.raises(BBWError):
        create(vmapP=bad)
    with pytest.raises(BBWError):
        _lib.call("bbw_rk_volume_planar", p.N, -1, None, None, None, None, None, None, None,
                  None, None)


def test_kernel_entries_accept_empty_lists(cuda):
    """K = 0 (an all-planar or all-curved mesh leaves one list empty): the
    entries return without touching rhsQ."""
    import torch
    p = make_curved_problem(2, 4)
    a = {k: dev(v) for k, v in p.desc_arrays().items()}
    r = torch.full((p.K * 4 * p.Np,), 7.0, device="cuda")
    P = _lib.ptr
    _lib.call("bbw_rk_volume_wadg_skew_combine", p.N, p.Nq, 0, None, None, None, None, None, None,
              None, None, None, None, None, None, None, None, P(r), None)
    _lib.call("bbw_rk_surface_wadg_skew_combine", p.N, p.Nfq, 0, None, None, None, None, None,
              None, None, None, P(r), None)
    _lib.call("bbw_rk_volume_planar", p.N, 0, None, None, None, None, None, None, None, P(r), None)
    _lib.call("bbw_rk_surface_planar", p.N, 0, None, None, None, None, None, None, None, P(r),
              None)
    torch.cuda.synchronize()
    assert bool((r == 7.0).all())
    del a


@pytest.mark.parametrize("n_elems", [1, 2])
@pytest.mark.parametrize("N", [2, 3])
def test_one_and_two_curved_elements(cuda, n_elems, N):
    """One curved tetrahedron (the centre and three points of the sphere:
    its outer face is a whole octant) or two sharing a face: a partial
    element block of the curved stage, no planar elements."""
    VX = np.array([0.0, 1.0, 0.0, 0.0, 0.0])
    VY = np.array([0.0, 0.0, 1.0, 0.0, 0.0])
    VZ = np.array([0.0, 0.0, 0.0, 1.0, -1.0])
    EToV = np.array([[0, 1, 2, 3], [0, 2, 1, 4]][:n_elems], np.int32)
    p = make_curved_problem(N, mesh=(VX, VY, VZ, EToV), c2=c2_sine)
    assert len(p.KlistCurved) == n_elems and len(p.KlistPlanar) == 0
    s = CurvedSolver(p)
    s.set_data(p.Q0)
    stages(s, p.dt, 10)
    Q = s.get_data()
    s.close()
    assert rel_l2(Q, oracle_of(p).run(p.Q0, p.dt, 10)[0]) < TOL


def test_one_planar_element(cuda):
    """A single element inside the ball (no vertex on the sphere): the
    fused affine stage over a one-element planar prefix."""
    VX = np.array([0.0, 0.5, 0.0, 0.0])
    VY = np.array([0.0, 0.0, 0.5, 0.0])
    VZ = np.array([0.0, 0.0, 0.0, 0.5])
    p = make_curved_problem(3, mesh=(VX, VY, VZ, np.array([[0, 1, 2, 3]], np.int32)), c2=c2_sine)
    assert len(p.KlistCurved) == 0 and len(p.KlistPlanar) == 1
    s = CurvedSolver(p)
    s.set_data(p.Q0)
    stages(s, p.dt, 10)
    Q = s.get_data()
    s.close()
    assert rel_l2(Q, oracle_of(p).run(p.Q0, p.dt, 10)[0]) < TOL


def test_autotune_restores_state_and_steps_match_oracle(cuda):
    """bbw_curved_autotune: the state and residual come back unchanged, the
    step graph captured before tuning is not reused (the variant's operator
    buffer changed), and the tuned steps equal the oracle's."""
    cub, tri = reference_rules(3)
    p = make_curved_problem(3, 4, c2=c2_sine, cubature=cub, tri_cubature=tri)
    s = CurvedSolver(p)
    s.set_data(p.Q0)
    s.steps(p.dt, 1)
    q, r = s.get_data(), s.get_residual()
    cfg = s.autotune(p.dt, 5)
    assert cfg & 255 in (8, 16)
    assert np.array_equal(s.get_data(), q)
    assert np.array_equal(s.get_residual(), r)
    s.steps(p.dt, 1)
    Q = s.get_data()
    s.close()
    assert rel_l2(Q, oracle_of(p).run(p.Q0, p.dt, 10)[0]) < TOL


def test_autotune_without_planar_elements(cuda):
    p = make_curved_problem(3, mesh=kuhn_ball(2), c2=c2_sine)
    assert len(p.KlistPlanar) == 0
    s = CurvedSolver(p)
    assert s.autotune(p.dt, 2) == 0
    s.close()
