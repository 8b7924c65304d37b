"""Precision-study GEMM form of the stage (csrc/gemm_stage.cu): split FP16,
split BF16 and TF32 contractions as cuBLAS GEMMs over all elements at the
orders the fused tensor-core stage does not take (N = 6, 7 with the
reference's rules), and TF32 at a low order.  Each run is compared with the
FP64 C restatement over 3 LSRK45 steps (15 stages of
cpp/src/WaveOKL3d.cpp:2084-2109).

Bars (relative L2 against FP64): split FP16 keeps 22 significant bits per
pair, so it meets the FP32 bar 1e-5; split BF16 keeps 16 bits per pair
(bar 1e-4); TF32 inputs keep 11 bits (bar 5e-3)."""
import numpy as np
import pytest
from conftest import golden, rel_l2

from bbwadg_b200 import WaveSolver, make_problem
from bbwadg_b200._lib import BBWError

pytestmark = pytest.mark.gpu
BARS = {"f16x3": 1e-5, "bf16x3": 1e-4, "tf32": 5e-3}


def ref_problem(N, nh, variant, seed=8):
    g = golden("ops_N%d.npz" % N)
    nfq = int(g["Nfq"][0])
    return make_problem(N, nh, variant=variant, c2="sine", c2_jitter=0.5, seed=seed,
                        cubature=(g["rq"], g["sq"], g["tq"], g["wq"]),
                        tri_cubature=(g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))


def fp64_reference(p, stages):
    from oracle import Oracle
    q, _ = Oracle(p.N, p.K, p.ops_dict(), p.geo_dict(), variant=p.variant,
                  dtype=np.float64).run(p.Q0.astype(np.float64), p.dt, stages)
    return q


@pytest.mark.parametrize("prec", ["f16x3", "bf16x3", "tf32"])
@pytest.mark.parametrize("N,variant", [(7, "nodal"), (7, "bb"), (6, "nodal")])
def test_gemm_form_against_fp64(cuda, N, variant, prec):
    p = ref_problem(N, 2, variant)
    q64 = fp64_reference(p, 15)
    s = WaveSolver(p, precision=prec)
    s.set_data(p.Q0)
    s.steps(p.dt, 3)
    err = rel_l2(s.get_data(), q64)
    s.close()
    assert err < BARS[prec], (N, variant, prec, err)


def test_tf32_at_a_low_order(cuda):
    """TF32 runs on the GEMM form at every order: N = 3 on 3^3 x 6 tets."""
    p = ref_problem(3, 3, "nodal", seed=2)
    q64 = fp64_reference(p, 15)
    s = WaveSolver(p, precision="tf32")
    s.set_data(p.Q0)
    s.steps(p.dt, 3)
    err = rel_l2(s.get_data(), q64)
    s.close()
    assert err < BARS["tf32"], err


def test_gemm_form_is_deterministic_and_stage_level(cuda):
    """Graph-replayed steps and single stages give the same state bit for
    bit, and two runs agree bit for bit."""
    from bbwadg_b200 import RK4A, RK4B
    p = ref_problem(7, 2, "nodal")
    a, b = WaveSolver(p, precision="f16x3"), WaveSolver(p, precision="f16x3")
    a.set_data(p.Q0)
    a.steps(p.dt, 2)
    b.set_data(p.Q0)
    for _ in range(2):
        for i in range(5):
            b.rk_stage(np.float32(RK4A[i]), np.float32(RK4B[i]), p.dt, 0.0)
    assert np.array_equal(a.get_data(), b.get_data())
    a.close(), b.close()


def test_gemm_form_refuses_shots_sources_and_adjoint(cuda):
    p = ref_problem(7, 2, "nodal")
    s = WaveSolver(p, precision="bf16x3")
    with pytest.raises(BBWError):
        s.set_shots(2)
    with pytest.raises(BBWError):
        s.set_sources(np.array([0], np.int32), np.array([0], np.int32),
                      np.ones((1, p.Np), np.float32), f0=4.0)
    s.close()
