"""Fused one-kernel-per-stage path (bbw_create / bbw_stage / bbw_steps /
bbw_run) against the reference's own time loop (golden) and the C
restatement.  FP32 tolerance: 1e-5 relative L2."""
import numpy as np
import pytest
from conftest import golden, ref_ops, rel_l2

from bbwadg_b200 import RK4A, RK4B, WaveSolver, make_problem
from bbwadg_b200.mesh import kuhn_box
from bbwadg_b200.problem import build_operators, connect_and_geometry, cavity_mode

pytestmark = pytest.mark.gpu
TOL = 1e-5


def ref_box4_solver(variant):
    r = golden("run_N3_box4.npz")
    ops = ref_ops(3, variant)
    m = connect_and_geometry(3, *kuhn_box(4), build_operators(3))
    s = WaveSolver(N=3, K=384, Nq=int(ops["Nq"][0]), variant=variant, ops=ops, vgeo=m["vgeo"],
                   fgeo=m["fgeo"], vmapP=m["vmapP"], c2q=r["c2q"])
    return s, r


@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_one_stage_matches_reference(cuda, variant):
    s, r = ref_box4_solver(variant)
    s.set_data(r["Q0_" + variant])
    dt = float(r["dt"][0])
    s.rk_step(np.float32(RK4A[0]), np.float32(RK4B[0]), dt)
    assert rel_l2(s.get_data(), r["Q1stage_" + variant]) < TOL
    assert rel_l2(s.get_residual(), r["res1stage_" + variant]) < TOL
    s.close()


@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_100_steps_match_reference(cuda, variant):
    """C1-shaped run (N=3, Gaussian pulse, sine c^2, p=0 walls) on 4^3 x 6
    tets: 100 LSRK45 steps through the CUDA-graph path vs the reference."""
    s, r = ref_box4_solver(variant)
    s.set_data(r["Q0_" + variant])
    s.steps(float(r["dt"][0]), 100)
    assert rel_l2(s.get_data(), r["Q100_" + variant]) < TOL
    s.close()


@pytest.mark.parametrize("N", [4, 5])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("bc", ["pressure_release", "rigid"])
def test_fused_matches_oracle(cuda, N, variant, bc):
    from oracle import Oracle
    p = make_problem(N, 4, variant=variant, c2="sine", c2_jitter=0.5, seed=3)
    orc = Oracle(N, p.K, p.ops_dict(), p.geo_dict(), variant=variant, bc=1 if bc == "rigid" else 0)
    q_ref, _ = orc.run(p.Q0.copy(), p.dt, 50)
    s = WaveSolver(p, bc=bc)
    s.set_data(p.Q0)
    s.steps(p.dt, 10)
    assert rel_l2(s.get_data(), q_ref) < TOL
    s.close()


def test_graph_steps_equal_stage_loop(cuda):
    p = make_problem(3, 3, variant="nodal")
    a = WaveSolver(p)
    b = WaveSolver(p)
    a.set_data(p.Q0)
    b.set_data(p.Q0)
    a.steps(p.dt, 3)
    for _ in range(3):
        for i in range(5):
            b.rk_step(np.float32(RK4A[i]), np.float32(RK4B[i]), p.dt)
    assert np.array_equal(a.get_data(), b.get_data())
    assert np.array_equal(a.get_residual(), b.get_residual())


def test_wave_rk_lands_on_final_time(cuda):
    p = make_problem(3, 2, variant="nodal")
    a, b = WaveSolver(p), WaveSolver(p)
    a.set_data(p.Q0)
    b.set_data(p.Q0)
    T = 2.5 * p.dt
    a.wave_rk(T, p.dt)
    b.steps(p.dt, 2)
    last = np.float32(T - 2 * np.float64(np.float32(p.dt)))
    b.steps(float(last), 1)
    assert rel_l2(a.get_data(), b.get_data()) < 1e-7


def test_cavity_mode_converges_at_order_N_plus_1(cuda):
    """Standing mode cos(pi x)cos(pi y)cos(pi z)cos(sqrt3 pi t), exact for the
    p = 0 wall on [-0.5,0.5]^3 (cpp/main_subelem.cpp:3-5), c^2 = 1."""
    N, T = 3, 0.1
    errs = []
    for n in (2, 4):
        p = make_problem(N, n, variant="nodal", c2="one", ic="cavity", lo=-0.5, hi=0.5)
        s = WaveSolver(p)
        s.set_data(p.Q0)
        s.wave_rk(T, p.dt)
        errs.append(p.l2_error(s.get_data(), T, cavity_mode)[0])
        s.close()
    rate = np.log2(errs[0] / errs[1])
    assert rate > N + 0.5, (errs, rate)


def test_nodal_and_bb_agree(cuda):
    """Same polynomial space: after 5 steps the BB run, mapped to nodal
    values, matches the nodal run to round-off times cond(VB)."""
    pn = make_problem(4, 3, variant="nodal")
    pb = make_problem(4, 3, variant="bb")
    sn, sb = WaveSolver(pn), WaveSolver(pb)
    sn.set_data(pn.Q0)
    sb.set_data(pb.Q0)
    sn.steps(pn.dt, 5)
    sb.steps(pb.dt, 5)
    assert rel_l2(pb.to_nodal(sb.get_data()), sn.get_data()) < 1e-4


@pytest.mark.parametrize("N", [3, 5])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_every_stage_configuration_matches_oracle(cuda, N, variant):
    """All element-tile / warps-per-CTA / operator-placement / pipelining
    variants the autotuner chooses from give the restatement's result; the
    autotuner keeps one of them and leaves the state untouched."""
    from oracle import Oracle
    from bbwadg_b200._lib import BBWError
    p = make_problem(N, 3, variant=variant, c2="sine", c2_jitter=0.5, seed=3)
    q_ref, _ = Oracle(N, p.K, p.ops_dict(), p.geo_dict(), variant=variant).run(p.Q0.copy(), p.dt, 10)
    ran = 0
    for tile in (32, 16):
      for warps in (8, 16):
        for ops in (True, False):
            for pipe in (True, False):
                s = WaveSolver(p)
                try:
                    s.set_config(warps, ops, pipe, tile)
                except BBWError:
                    s.close()
                    continue
                s.set_data(p.Q0)
                s.steps(p.dt, 2)
                assert rel_l2(s.get_data(), q_ref) < TOL, (warps, ops, pipe, tile)
                s.close()
                ran += 1
    assert ran >= 8
    s = WaveSolver(p)
    s.set_data(p.Q0)
    cfg = s.autotune(p.dt, 5)
    assert cfg["warps"] in (8, 16) and cfg["tile"] in (16, 32)
    assert np.array_equal(s.get_data(), p.Q0.astype(np.float32))
    s.steps(p.dt, 2)
    assert rel_l2(s.get_data(), q_ref) < TOL
    s.close()


@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_fused_n7_matches_oracle(cuda, variant):
    """N = 7 (Np = 120, reference rule Nq = 214): operators, and for BB the
    lift tables, read through the cache (they do not fit in shared memory
    next to the tiles)."""
    from oracle import Oracle
    g = golden("ops_N7.npz")
    nfq = int(g["Nfq"][0])
    p = make_problem(7, 2, variant=variant, c2="sine", c2_jitter=0.5, seed=8,
                     cubature=(g["rq"], g["sq"], g["tq"], g["wq"]),
                     tri_cubature=(g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))
    q_ref, _ = Oracle(7, p.K, p.ops_dict(), p.geo_dict(), variant=variant).run(p.Q0.copy(), p.dt, 15)
    s = WaveSolver(p)
    s.set_data(p.Q0)
    s.steps(p.dt, 3)
    assert rel_l2(s.get_data(), q_ref) < TOL
    cfg = s.autotune(p.dt, 3)
    s.set_data(p.Q0)
    s.set_residual(np.zeros(p.K * 4 * p.Np, np.float32))
    s.steps(p.dt, 3)
    assert rel_l2(s.get_data(), q_ref) < TOL, cfg
    s.close()


def test_get_data_into_caller_buffer(cuda):
    """WaveGetData3d into a caller's (pinned) buffer: same values as a fresh
    array; wrong dtype or size is rejected."""
    import torch
    p = make_problem(3, 2)
    s = WaveSolver(p)
    s.set_data(p.Q0)
    s.steps(p.dt, 2)
    ref = s.get_data()
    out = torch.empty(ref.size, dtype=torch.float32).pin_memory()
    got = s.get_data(out=out.numpy())
    assert got is not None and np.array_equal(out.numpy(), ref)
    with pytest.raises(ValueError):
        s.get_data(out=np.empty(ref.size, np.float64))
    with pytest.raises(ValueError):
        s.get_data(out=np.empty(ref.size - 1, np.float32))
    s.close()



def _tets(n_elems):
    """One positively oriented tetrahedron, or two sharing the face (0,1,2)."""
    VX = np.array([0.0, 1.0, 0.0, 0.0, 0.3])
    VY = np.array([0.0, 0.0, 1.0, 0.0, 0.3])
    VZ = np.array([0.0, 0.0, 0.0, 1.0, -0.9])
    EToV = np.array([[0, 1, 2, 3], [0, 2, 1, 4]][:n_elems], np.int32)
    return VX, VY, VZ, EToV


@pytest.mark.parametrize("n_elems", [1, 2])
@pytest.mark.parametrize("N", [3, 5])
@pytest.mark.parametrize("form", ["nodal", "bb", "nodal-f16x3", "bb-f16x3"])
def test_one_and_two_element_meshes_match_oracle(cuda, n_elems, N, form):
    """A tile holding one or two elements, every face but the shared one a
    wall: the stage (FP32 fused, or the split-FP16 tensor-core form) against
    the oracle over two steps."""
    from oracle import Oracle
    variant = form.split("-")[0]
    g = golden("ops_N%d.npz" % N)  # the reference's rules (Nq = 31 / 95)
    nfq = int(g["Nfq"][0])
    p = make_problem(N, mesh=_tets(n_elems), variant=variant, c2="sine", seed=2,
                     cubature=(g["rq"], g["sq"], g["tq"], g["wq"]),
                     tri_cubature=(g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))
    assert p.K == n_elems
    if n_elems == 2:
        assert (p.mesh["EToE"].reshape(2, 4) != np.arange(2)[:, None]).sum() == 2
    orc = Oracle(N, p.K, p.ops_dict(), p.geo_dict(), variant=variant)
    q_ref, _ = orc.run(p.Q0.copy(), p.dt, 10)
    s = WaveSolver(p, precision="f16x3" if form.endswith("f16x3") else "fp32")
    s.set_data(p.Q0)
    s.steps(p.dt, 2)
    assert rel_l2(s.get_data(), q_ref) < TOL
    s.close()


@pytest.mark.parametrize("rule", ["reference", "stroud"])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_fused_n6_matches_oracle(cuda, variant, rule):
    """N = 6 (Np = 84) with the reference's 146-point rule or the 343-point
    Stroud rule: operators read through the cache, the cubature arrays of
    the tile in shared memory."""
    from oracle import Oracle
    cub = tri = None
    if rule == "reference":
        g = golden("ops_N6.npz")
        nfq = int(g["Nfq"][0])
        cub = (g["rq"], g["sq"], g["tq"], g["wq"])
        tri = (g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"])
    p = make_problem(6, 2, variant=variant, c2="sine", c2_jitter=0.5, seed=3, cubature=cub,
                     tri_cubature=tri)
    assert p.Nq == (146 if rule == "reference" else 343)
    s = WaveSolver(p)
    s.set_data(p.Q0)
    s.steps(p.dt, 2)
    q = s.get_data()
    s.close()
    q_ref, _ = Oracle(6, p.K, p.ops_dict(), p.geo_dict(), variant=variant).run(p.Q0.copy(), p.dt, 10)
    assert rel_l2(q, q_ref) < TOL


@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_fused_n8_on_16_element_tiles(cuda, variant):
    """N = 8 with the 729-point Stroud rule: a 32-element tile's cubature
    arrays alone exceed one SM's shared memory, so the context runs 16-element
    tiles (operators read through the cache).  2^3 x 6 tets = 3 tiles, on the
    full grid and on one CTA walking all three; the 32-element variants are
    refused rather than run out of bounds, and the autotuner keeps a
    16-element one."""
    from oracle import Oracle
    from bbwadg_b200._lib import BBWError
    p = make_problem(8, 2, variant=variant, c2="sine", c2_jitter=0.5, seed=3)
    assert p.Nq == 729 and p.K == 48
    q_ref, _ = Oracle(8, p.K, p.ops_dict(), p.geo_dict(), variant=variant).run(p.Q0.copy(), p.dt, 10)
    s = WaveSolver(p)
    for limit in (0, 1):
        s.set_grid_limit(limit)
        s.set_data(p.Q0)
        s.steps(p.dt, 2)
        assert rel_l2(s.get_data(), q_ref) < TOL, limit
    for warps in (8, 16):
        with pytest.raises(BBWError, match="shared memory"):
            s.set_config(warps, False, False, 32)
    s.set_data(p.Q0)
    cfg = s.autotune(p.dt, 3)
    assert cfg["tile"] == 16
    s.steps(p.dt, 2)
    assert rel_l2(s.get_data(), q_ref) < TOL
    s.close()


@pytest.mark.parametrize("form", ["fp32", "f16x3"])
def test_contexts_on_different_meshes_do_not_undercut_each_other(cuda, form):
    """Two contexts of the same order on meshes with different numbers of
    face permutations (hence different shared-memory footprints): creating
    the second must not break the first one's launches."""
    from oracle import Oracle
    g = golden("ops_N3.npz")
    nfq = int(g["Nfq"][0])
    rule = dict(cubature=(g["rq"], g["sq"], g["tq"], g["wq"]),
                tri_cubature=(g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))
    a = make_problem(3, 3, variant="nodal", c2="sine", seed=2, **rule)
    b = make_problem(3, mesh=_tets(2), variant="nodal", c2="sine", seed=2, **rule)
    sa = WaveSolver(a, precision=form)
    sb = WaveSolver(b, precision=form)
    for s, p in ((sa, a), (sb, b)):
        s.set_data(p.Q0)
        s.steps(p.dt, 2)
        q_ref, _ = Oracle(3, p.K, p.ops_dict(), p.geo_dict()).run(p.Q0.copy(), p.dt, 10)
        assert rel_l2(s.get_data(), q_ref) < TOL
    sa.close()
    sb.close()
