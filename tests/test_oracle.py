"""The C restatement (oracle/wadg_oracle.c) against the reference's own
kernels and time loop (golden vectors produced by oracle/_ref from the
reference sources).  CPU only."""
import numpy as np
import pytest
from conftest import golden, ref_ops, rel_l2

from oracle import Oracle

TOL = 2e-6  # FP32, FMA vs non-FMA rounding only


@pytest.mark.parametrize("N", [3, 5])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_kernels_match_reference(N, variant):
    ops, geo, k = ref_ops(N, variant), golden("mesh_box2_N%d.npz" % N), golden("kernels_N%d_box2.npz" % N)
    o = Oracle(N, 48, ops, geo, variant=variant)
    tag = "" if variant == "nodal" else "_bern"
    Q = k["Q_in"].copy()
    rhs = np.zeros_like(Q)
    o.rk_volume(Q, rhs)
    assert rel_l2(rhs, k["rk_volume%s.rhsQ" % tag]) < TOL
    rhs = k["rhs_in"].copy()
    o.rk_surface(Q, rhs)
    assert rel_l2(rhs, k["rk_surface%s.rhsQ" % tag]) < TOL
    rhs, res, Q = k["rhs_in"].copy(), k["res_in"].copy(), k["Q_in"].copy()
    o.rk_update_wadg(k["fa"], k["fb"], np.float32(k["dt"][0]), rhs, res, Q)
    t = "rk_update_WADG" + ("_bb" if variant == "bb" else "")
    assert rel_l2(res, k[t + ".resQ"]) < TOL
    assert rel_l2(Q, k[t + ".Q"]) < TOL


def test_update_matches_reference():
    ops, geo, k = ref_ops(3, "nodal"), golden("mesh_box2_N3.npz"), golden("kernels_N3_box2.npz")
    o = Oracle(3, 48, ops, geo)
    rhs, res, Q = k["rhs_in"].copy(), k["res_in"].copy(), k["Q_in"].copy()
    o.rk_update(k["fa"], k["fb"], np.float32(k["dt"][0]), rhs, res, Q)
    assert rel_l2(res, k["rk_update.resQ"]) < TOL
    assert rel_l2(Q, k["rk_update.Q"]) < TOL


def test_slice_lift_equals_sparse_lift():
    """The reference's two BB lift kernels agree (golden self-consistency)."""
    for N in (3, 5):
        k = golden("kernels_N%d_box2.npz" % N)
        assert rel_l2(k["rk_surface_bern_slice.rhsQ"], k["rk_surface_bern.rhsQ"]) < 1e-6


@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_time_loop_matches_reference(variant, box4_geo):
    """1 stage and 100 LSRK45 steps of the reference's Wave_RK loop."""
    r = golden("run_N3_box4.npz")
    o = Oracle(3, 384, ref_ops(3, variant), box4_geo, variant=variant)
    dt = float(r["dt"][0])
    Q, res = o.run(r["Q0_" + variant].copy(), dt, 1)
    assert rel_l2(Q, r["Q1stage_" + variant]) < 1e-6
    assert rel_l2(res, r["res1stage_" + variant]) < 1e-6
    Q, _ = o.run(r["Q0_" + variant].copy(), dt, 500)
    assert rel_l2(Q, r["Q100_" + variant]) < 1e-5


@pytest.fixture(scope="module")
def box4_geo():
    """Geometry of the 4^3 x 6 box from the product setup (checked bit-exact
    against the reference on the 2^3 box in test_setup.py); c2q from the
    reference run."""
    from bbwadg_b200.problem import build_operators, connect_and_geometry
    from bbwadg_b200.mesh import kuhn_box
    ops = build_operators(3)
    m = connect_and_geometry(3, *kuhn_box(4), ops)
    r = golden("run_N3_box4.npz")
    return dict(vgeo=m["vgeo"], fgeo=m["fgeo"], vmapP=m["vmapP"], c2q=r["c2q"],
                Jq=np.ones_like(r["c2q"]))


def test_fp64_oracle_is_closer_to_truth():
    """FP64 and FP32 restatements agree to FP32 accuracy on one stage."""
    ops, geo = ref_ops(5, "nodal"), golden("mesh_box2_N5.npz")
    o32 = Oracle(5, 48, ops, geo)
    o64 = Oracle(5, 48, ops, geo, dtype=np.float64)
    Q0 = geo["Q0_nodal"]
    q32, _ = o32.run(Q0.copy(), float(geo["dt"][0]), 5)
    q64, _ = o64.run(Q0.astype(np.float64), float(np.float32(geo["dt"][0])), 5)
    assert rel_l2(q32, q64) < 1e-6


def test_c1_restatement_matches_reference_cpu_path(tmp_path):
    """N=3 at full workload size (8^3 x 6 tets, CFL 0.5, 100 steps): the C
    restatement against the reference's own CPU path on the same mesh file,
    c^2, initial state and dt."""
    import os
    import subprocess

    import bbwa
    from conftest import ROOT, golden
    from bbwadg_b200 import make_problem
    from bbwadg_b200.mesh import kuhn_box, write_gmsh22
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_N3_B0")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref not built")
    msh = str(tmp_path / "box8.msh")
    write_gmsh22(msh, *kuhn_box(8))
    g = golden("ops_N3.npz")
    nfq = int(g["Nfq"][0])
    p = make_problem(3, mesh=msh, c2="sine", ic="gauss", cubature=(g["rq"], g["sq"], g["tq"], g["wq"]),
                     tri_cubature=(g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]), cfl=0.5)
    np.ascontiguousarray(p.Q0, np.float32).tofile(tmp_path / "q0")
    np.ascontiguousarray(p.c2q, np.float32).tofile(tmp_path / "c2")
    subprocess.run([exe, "run", msh, str(tmp_path / "out"), "--stages", "500", "--q0",
                    str(tmp_path / "q0"), "--c2q", str(tmp_path / "c2"), "--dt",
                    "%.9g" % np.float32(p.dt), "--c2", "sine"], check=True,
                   stdout=subprocess.DEVNULL, timeout=600)
    q_ref = bbwa.read(str(tmp_path / "out"))["Q"]
    q, _ = Oracle(3, p.K, p.ops_dict(), p.geo_dict()).run(p.Q0.copy(), p.dt, 500)
    assert np.linalg.norm(q - q_ref) <= 1e-6 * np.linalg.norm(q_ref)


@pytest.mark.parametrize("N", [3, 5, 7])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_wadg_projection_is_identity_on_polynomials(N, variant):
    """Pq Vq = I (cpp/src/WaveOKL3d.cpp:895-896) for the reference's FP32
    operators: the degree-2N+1 rule integrates the mass matrix exactly, which
    the fused stage relies on when it skips the velocity rows of the WADG
    update (J = 1)."""
    g = golden("ops_N%d.npz" % N)
    Np = (N + 1) * (N + 2) * (N + 3) // 6
    Nq = int(g["Nq"][0])
    Vq = np.asarray(g["Vq_" + variant], np.float64).reshape(Np, Nq).T
    Pq = np.asarray(g["Pq_" + variant], np.float64).reshape(Nq, Np).T
    assert np.abs(Pq @ Vq - np.eye(Np)).max() < 1e-5


def test_oracle_refuses_sizes_beyond_its_arrays():
    """The restatement's per-element work arrays have fixed sizes; a rule
    with more points is refused instead of overrunning them, and the
    729-point rule of N = 8 fits."""
    from oracle import lib
    from bbwadg_b200 import make_problem
    assert lib().ora_maxnq() >= 729
    p = make_problem(3, 2)
    ops = dict(p.ops_dict())
    ops["Vq"] = np.zeros(p.Np * (lib().ora_maxnq() + 1), np.float32)
    with pytest.raises(ValueError, match="compiled limits"):
        Oracle(3, p.K, ops, p.geo_dict())
