"""Curvilinear WADG path on the CPU: the native setup (Gordon-Hall curving,
geometric factors at the cubature, curved operators) against the reference's
own setup, and the FP64 restatement of the curved stage (oracle/curved.py)
pinned to the reference's kernels (tests/golden/curved_*_N*.npz, from
oracle/_ref/ref_curved_N* on kuhn_ball(4): K = 384, 288 curved, and on the
reference's own sphere meshes sphere48.msh and sphere385.msh)."""
import numpy as np
import pytest
from conftest import golden, rel_l2

from bbwadg_b200.curved import make_curved_problem
from bbwadg_b200.mesh import kuhn_ball

OPS = ["Vrq", "Vsq", "Vtq", "Prq", "Psq", "Ptq", "VfqFace", "Pfq", "Vfq"]


def ref_rules(g):
    Nfq = len(g["wfqFace"])
    return ((g["rq"], g["sq"], g["tq"], g["wq"]), (g["rfq"][:Nfq], g["sfq"][:Nfq], g["wfqFace"]))


def problem_like_reference(N, mesh="ball4"):
    """The reference's curved setup on kuhn_ball(4) or on one of its own
    sphere meshes (sphere48 / sphere385, read as ReadGmsh3d reads them)."""
    g = golden("curved_%s_N%d.npz" % (mesh, N))
    cub, tri = ref_rules(g)
    if mesh == "ball4":
        p = make_curved_problem(N, 4, cubature=cub, tri_cubature=tri)
    else:
        m = golden("gmsh_%s.npz" % mesh)
        p = make_curved_problem(N, mesh=(m["VX"], m["VY"], m["VZ"], m["EToV"]), cubature=cub,
                                tri_cubature=tri)
    p.c2q = g["c2q_in"].reshape(p.K, p.Nq)
    return p, g


MESHES = ["ball4", "sphere48", "sphere385"]


def oracle_of(p):
    from curved import CurvedOracle
    return CurvedOracle(p.N, p.K, p.Nq, p.Nfq, p.desc_arrays())


@pytest.mark.parametrize("mesh", MESHES)
@pytest.mark.parametrize("N", [2, 3])
def test_gordon_hall_matches_reference(N, mesh):
    p, g = problem_like_reference(N, mesh)
    assert np.array_equal(p.KlistCurved, g["KlistCurved"])
    # the reference sizes its planar list max(1, KPlanar) (cpp/src/WaveOKL3d.cpp:1239):
    # with every element curved (sphere48) it holds one unused 0
    KP = p.K - len(g["KlistCurved"])
    assert np.array_equal(p.KlistPlanar, g["KlistPlanar"][:KP])
    for c in ("x", "y", "z"):
        assert np.abs(p.mesh[c] - g[c]).max() < 1e-13, c
    assert abs(p.dt - float(g["dt"][0])) <= 1e-7 * p.dt


@pytest.mark.parametrize("mesh", MESHES)
@pytest.mark.parametrize("N", [2, 3])
def test_curved_geometry_matches_reference(N, mesh):
    p, g = problem_like_reference(N, mesh)
    n = len(g["Jq_sub"])
    for ours, ref in ((p.vgeoq, g["vgeoq_sub"]), (p.Jq, g["Jq_sub"]), (p.fgeoq, g["fgeoq_sub"])):
        a = ours.reshape(p.K, -1)[:n]
        assert np.abs(a - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("mesh", MESHES)
@pytest.mark.parametrize("N", [2, 3])
def test_curved_operators_match_reference(N, mesh):
    p, g = problem_like_reference(N, mesh)
    for k in OPS:
        assert np.abs(p.ops[k] - g[k]).max() <= 1e-6 * np.abs(g[k]).max(), k


@pytest.mark.parametrize("mesh", MESHES)
@pytest.mark.parametrize("N", [2, 3])
def test_oracle_run_matches_reference(N, mesh):
    p, g = problem_like_reference(N, mesh)
    Q, res = oracle_of(p).run(p.Q0, float(g["dt"][0]), int(g["stages"]))
    assert rel_l2(Q, g["Q_run"]) < 1e-6
    assert rel_l2(res, g["res_run"]) < 1e-4  # small residual: FP32 noise of the reference


@pytest.mark.parametrize("kernel", ["rk_volume_WADG_skew_combine", "rk_surface_WADG_skew_combine",
                                    "rk_volume_planar", "rk_surface_planar"])
def test_oracle_kernels_match_reference(kernel):
    p, g = problem_like_reference(3)
    orc = oracle_of(p)
    fn = {"rk_volume_WADG_skew_combine": orc.volume_skew,
          "rk_surface_WADG_skew_combine": orc.surface_skew,
          "rk_volume_planar": orc.volume_planar, "rk_surface_planar": orc.surface_planar}[kernel]
    shape = (p.K, 4, p.Np)
    q = g["q_in"].astype(np.float64).reshape(shape)
    r = g["rhs_in"].astype(np.float64).reshape(shape).copy()
    fn(q, r)
    assert rel_l2(r, g[kernel + ".rhsQ"]) < 1e-6


@pytest.mark.parametrize("N", [3, 4, 5])
def test_curved_ball_geometry(N):
    """Volume of the curved ball, boundary nodes on the sphere, positive J,
    outward unit normals on the sphere close to radial."""
    p = make_curved_problem(N, 4)
    assert abs(p.volume() - 4 * np.pi / 3) < 2e-3
    assert p.geo64["Jq"].min() > 0
    Fm = p.ops["Fmask"].reshape(4, -1)
    EToE = p.mesh["EToE"]
    r = np.sqrt(p.mesh["x"] ** 2 + p.mesh["y"] ** 2 + p.mesh["z"] ** 2)
    nb = 0
    for f in range(4):
        bk = np.nonzero(EToE[:, f] == np.arange(p.K))[0]  # boundary faces map to themselves
        nb += len(bk)
        if not len(bk):
            continue
        assert np.abs(r[bk][:, Fm[f]] - 1.0).max() < 1e-12
        assert np.isin(bk, p.KlistCurved).all()
        n = p.geo64["fgeoq"][bk, f, :3]                     # [E][3][Nfq]
        assert np.abs(np.sqrt((n ** 2).sum(1)) - 1).max() < 1e-12
    assert nb == 6 * 4 * 4 * 2  # 2 triangles on each of the 16 cells of each cube face


def test_kuhn_ball_mesh():
    VX, VY, VZ, EToV = kuhn_ball(6)
    X = np.stack([VX, VY, VZ], 1)
    v = X[EToV]
    d = v[:, 1:] - v[:, :1]
    assert (np.einsum("ij,ij->i", d[:, 0], np.cross(d[:, 1], d[:, 2])) > 0).all()
    onS = np.abs(np.linalg.norm(X, axis=1) - 1) < 1e-12
    assert not (onS[EToV].sum(1) == 4).any()  # no chord with both ends on the sphere
    first_interior = np.argmin(onS)
    assert onS[:first_interior].all() and not onS[first_interior:].any()  # boundary first
    with pytest.raises(ValueError):
        kuhn_ball(3)
