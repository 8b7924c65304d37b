"""Tensor-core (tcgen05) stage, split-FP16 three-product form, against the
reference's time loop (golden) and the FP32 C restatement.  Tolerance:
1e-5 relative L2, the same bar as the FP32 path.  The split-BF16 form is
checked against the restatement at its own bar (BF16X3_TOL)."""
import numpy as np
import pytest
from conftest import golden, ref_ops, rel_l2

from bbwadg_b200 import RK4A, RK4B, WaveSolver, make_problem
from bbwadg_b200.mesh import kuhn_box
from bbwadg_b200.problem import build_operators, connect_and_geometry

pytestmark = pytest.mark.gpu
TOL = 1e-5


def ref_rule(N):
    g = golden("ops_N%d.npz" % N)
    nfq = int(g["Nfq"][0])
    return (g["rq"], g["sq"], g["tq"], g["wq"]), (g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"])


def test_tc_100_steps_match_reference(cuda):
    r = golden("run_N3_box4.npz")
    ops = ref_ops(3, "nodal")
    m = connect_and_geometry(3, *kuhn_box(4), build_operators(3))
    s = WaveSolver(N=3, K=384, Nq=int(ops["Nq"][0]), variant="nodal", ops=ops, vgeo=m["vgeo"],
                   fgeo=m["fgeo"], vmapP=m["vmapP"], c2q=r["c2q"], precision="f16x3")
    s.set_data(r["Q0_nodal"])
    s.rk_step(np.float32(RK4A[0]), np.float32(RK4B[0]), float(r["dt"][0]))
    assert rel_l2(s.get_data(), r["Q1stage_nodal"]) < TOL
    s.close()
    s = WaveSolver(N=3, K=384, Nq=int(ops["Nq"][0]), variant="nodal", ops=ops, vgeo=m["vgeo"],
                   fgeo=m["fgeo"], vmapP=m["vmapP"], c2q=r["c2q"], precision="f16x3")
    s.set_data(r["Q0_nodal"])
    s.steps(float(r["dt"][0]), 100)
    s.check()
    assert rel_l2(s.get_data(), r["Q100_nodal"]) < TOL


@pytest.mark.parametrize("bc", ["pressure_release", "rigid"])
@pytest.mark.parametrize("n", [3, 4])
def test_tc_n5_matches_oracle(cuda, bc, n):
    """N=5 with the reference's 95-point rule; 4^3 x 6 (K=384, tiles full)
    and 3^3 x 6 (K=162, a partial last tile)."""
    from oracle import Oracle
    cub, tri = ref_rule(5)
    p = make_problem(5, n, variant="nodal", c2="sine", c2_jitter=0.5, seed=5, cubature=cub,
                     tri_cubature=tri)
    orc = Oracle(5, p.K, p.ops_dict(), p.geo_dict(), variant="nodal",
                 bc=1 if bc == "rigid" else 0)
    q_ref, r_ref = orc.run(p.Q0.copy(), p.dt, 25)
    s = WaveSolver(p, bc=bc, precision="f16x3")
    s.set_data(p.Q0)
    s.steps(p.dt, 5)
    s.check()
    assert rel_l2(s.get_data(), q_ref) < TOL
    assert rel_l2(s.get_residual(), r_ref) < 1e-4


def test_tc_agrees_with_fp32_stage_over_many_steps(cuda):
    cub, tri = ref_rule(5)
    p = make_problem(5, 4, variant="nodal", c2="sine", c2_jitter=0.5, seed=9, cubature=cub,
                     tri_cubature=tri, cfl=0.25)
    a = WaveSolver(p, precision="fp32")
    b = WaveSolver(p, precision="f16x3")
    a.set_data(p.Q0)
    b.set_data(p.Q0)
    a.steps(p.dt, 50)
    b.steps(p.dt, 50)
    b.check()
    assert rel_l2(b.get_data(), a.get_data()) < TOL


def test_tc_many_tiles_per_cta_and_tiny_tiles(cuda):
    """10^3 x 6 tets (K=6000, 188 tiles: CTAs loop over several tiles) with
    one tile scaled to ~1e-39 (below 2^-127, where a per-tile power-of-two
    scale must stay finite) and one tile exactly zero."""
    from oracle import Oracle
    cub, tri = ref_rule(5)
    p = make_problem(5, 10, variant="nodal", c2="sine", c2_jitter=0.5, seed=11, cubature=cub,
                     tri_cubature=tri, cfl=0.25)
    Q0 = p.Q0.reshape(p.K, 4, p.Np).copy()
    Q0[:, 0, :] += 0.1  # every tile carries signal
    Q0[32 * 40:32 * 41] = 1e-39 * np.sign(Q0[32 * 40:32 * 41] + 0.5)
    Q0[32 * 90:32 * 91] = 0.0
    Q0 = Q0.ravel()
    q_ref, _ = Oracle(5, p.K, p.ops_dict(), p.geo_dict(), variant="nodal").run(Q0.copy(), p.dt, 10)
    s = WaveSolver(p, precision="f16x3")
    s.set_data(Q0)
    s.steps(p.dt, 2)
    s.check()
    q = s.get_data()
    assert np.isfinite(q).all()
    assert rel_l2(q, q_ref) < TOL
    s.close()


def test_tc_other_orders_take_the_gemm_form(cuda):
    """N >= 6 (Np > 64: operators beyond one M = 64 MMA and one SM's shared
    memory) and N = 1 do not fit the fused tensor-core stage; a split-FP16
    context there runs the GEMM form instead (one shot only, so set_shots(2)
    is refused), for both bases, within the FP32 bar of the FP64
    restatement after 2 LSRK45 steps."""
    from bbwadg_b200._lib import BBWError
    from oracle import Oracle
    for N, n in ((6, 1), (1, 2)):
        for variant in ("nodal", "bb"):
            p = make_problem(N, n, variant=variant, c2="sine")
            q64, _ = Oracle(N, p.K, p.ops_dict(), p.geo_dict(), variant=variant,
                            dtype=np.float64).run(p.Q0.astype(np.float64), p.dt, 10)
            s = WaveSolver(p, precision="f16x3")
            with pytest.raises(BBWError):
                s.set_shots(2)
            s.set_data(p.Q0)
            s.steps(p.dt, 2)
            err = rel_l2(s.get_data(), q64)
            s.close()
            assert err < TOL, (N, variant, err)


@pytest.mark.parametrize("prec", ["f16x3", "bf16x3"])
@pytest.mark.parametrize("N,rule", [(2, "stroud"), (4, "reference"), (4, "stroud")])
@pytest.mark.parametrize("bc", ["pressure_release", "rigid"])
def test_tc_other_orders_match_oracle(cuda, prec, N, rule, bc):
    """N = 2 (Np = 10) and N = 4 (Np = 35: field rows not 16-byte aligned in
    the state tile) with the reference's rule or the Stroud rule, both walls,
    a ragged last tile (3^3 x 6 = 162 elements)."""
    from oracle import Oracle
    cub, tri = ref_rule(N) if rule == "reference" else (None, None)
    p = make_problem(N, 3, variant="nodal", c2="sine", c2_jitter=0.5, seed=7, cubature=cub,
                     tri_cubature=tri)
    q_ref, _ = Oracle(N, p.K, p.ops_dict(), p.geo_dict(), variant="nodal",
                      bc=1 if bc == "rigid" else 0).run(p.Q0.copy(), p.dt, 25)
    s = WaveSolver(p, bc=bc, precision=prec)
    s.set_data(p.Q0)
    s.steps(p.dt, 5)
    s.check()
    assert rel_l2(s.get_data(), q_ref) < TOL
    s.close()


# split-BF16: 16 significant bits per hi/lo pair, so each contraction is good
# to about 2^-16 of its tile maximum; after 25 stages the state is within
# 1e-6 of the FP32 restatement on these cases (split-FP16: 1e-7); the bar
# keeps a factor of ten.
BF16X3_TOL = 1e-5


@pytest.mark.parametrize("N,n", [(3, 4), (5, 3)])
def test_bf16x3_matches_oracle(cuda, N, n):
    from oracle import Oracle
    cub, tri = ref_rule(N)
    p = make_problem(N, n, variant="nodal", c2="sine", c2_jitter=0.5, seed=6, cubature=cub,
                     tri_cubature=tri)
    q_ref, _ = Oracle(N, p.K, p.ops_dict(), p.geo_dict(), variant="nodal").run(
        p.Q0.copy(), p.dt, 25)
    errs = {}
    for prec in ("f16x3", "bf16x3"):
        s = WaveSolver(p, precision=prec)
        s.set_data(p.Q0)
        s.steps(p.dt, 5)
        s.check()
        errs[prec] = rel_l2(s.get_data(), q_ref)
        s.close()
    print("relative L2 vs FP32 restatement:", errs)
    assert errs["f16x3"] < TOL
    assert errs["bf16x3"] < BF16X3_TOL


@pytest.mark.parametrize("prec", ["f16x3", "bf16x3"])
@pytest.mark.parametrize("N", [3, 4, 5])
@pytest.mark.parametrize("bc", ["pressure_release", "rigid"])
def test_tc_bb_matches_oracle(cuda, prec, N, bc):
    """The Bernstein-Bezier variant on the tensor cores: the dense
    equivalents of the sparse BB derivative and of the L0 + degree-elevation
    lift, applied to BB coefficients, against the restatement of the
    reference's sparse BB kernels (cpp/okl/WaveKernels.okl:344-647); the
    reference's rules, a ragged last tile."""
    from oracle import Oracle
    cub, tri = ref_rule(N)
    p = make_problem(N, 3, variant="bb", c2="sine", c2_jitter=0.5, seed=17, cubature=cub,
                     tri_cubature=tri)
    q_ref, _ = Oracle(N, p.K, p.ops_dict(), p.geo_dict(), variant="bb",
                      bc=1 if bc == "rigid" else 0).run(p.Q0.copy(), p.dt, 25)
    s = WaveSolver(p, bc=bc, precision=prec)
    s.set_data(p.Q0)
    s.steps(p.dt, 5)
    s.check()
    assert rel_l2(s.get_data(), q_ref) < TOL
    s.close()


def test_tc_bb_over_many_tiles_matches_the_bb_reference_run(cuda):
    """The BB tensor-core stage through the 100-step run of the reference's
    own BB path (4^3 x 6, Gaussian pulse, sine c^2, p = 0 walls)."""
    r = golden("run_N3_box4.npz")
    ops = ref_ops(3, "bb")
    m = connect_and_geometry(3, *kuhn_box(4), build_operators(3))
    s = WaveSolver(N=3, K=384, Nq=int(ops["Nq"][0]), variant="bb", ops=ops, vgeo=m["vgeo"],
                   fgeo=m["fgeo"], vmapP=m["vmapP"], c2q=r["c2q"], precision="f16x3")
    s.set_grid_limit(2)
    s.set_data(r["Q0_bb"])
    s.steps(float(r["dt"][0]), 100)
    s.check()
    assert rel_l2(s.get_data(), r["Q100_bb"]) < TOL
    s.close()
