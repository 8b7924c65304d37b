"""bbw_rk_stage_noalloc (static-scratch stage) against the kernel-level
entry points it composes, called with a caller-allocated rhs buffer.  The
file sorts last so that the check also runs after every other GPU test."""
import numpy as np
import pytest
from conftest import golden, ref_ops

from bbwadg_b200 import RK4A, RK4B, _lib
from bbwadg_b200._lib import BBWError

pytestmark = pytest.mark.gpu


def _case(N):
    import torch
    o, g, k = ref_ops(N, "nodal"), golden("mesh_box2_N%d.npz" % N), golden("kernels_N%d_box2.npz" % N)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).copy()).cuda()
    arrs = dict(vgeo=d(g["vgeo"]), Dr=d(o["Dr"]), Ds=d(o["Ds"]), Dt=d(o["Dt"]), fgeo=d(g["fgeo"]),
                Fmask=d(o["Fmask"]), vmapP=d(g["vmapP"]), LIFT=d(o["LIFT"]), Vq=d(o["Vq"]),
                Pq=d(o["Pq"]), Jq=d(np.ones(g["c2q"].size, np.float32)), c2q=d(g["c2q"]))
    return arrs, k["Q_in"], k["res_in"], int(o["Nq"][0])


def _three_kernels(N, K, Nq, a, Q, res, rhs, fa, fb, dt):
    p = lambda t: t.data_ptr()
    _lib.call("bbw_rk_volume", N, K, p(a["vgeo"]), p(a["Dr"]), p(a["Ds"]), p(a["Dt"]), p(Q), p(rhs),
              None)
    _lib.call("bbw_rk_surface", N, K, 0, p(a["fgeo"]), p(a["Fmask"]), p(a["vmapP"]), p(a["LIFT"]),
              p(Q), p(rhs), None)
    _lib.call("bbw_rk_update_wadg", N, K, Nq, p(a["Vq"]), p(a["Pq"]), p(a["Jq"]), p(a["c2q"]),
              fa, fb, dt, p(rhs), p(res), p(Q), None)


def _noalloc(N, K, Nq, a, Q, res, fa, fb, dt, k_override=None):
    p = lambda t: t.data_ptr()
    _lib.call("bbw_rk_stage_noalloc", N, K if k_override is None else k_override, Nq, 0,
              p(a["vgeo"]), p(a["Dr"]), p(a["Ds"]), p(a["Dt"]), p(a["fgeo"]), p(a["Fmask"]),
              p(a["vmapP"]), p(a["LIFT"]), p(a["Vq"]), p(a["Pq"]), p(a["Jq"]), p(a["c2q"]),
              fa, fb, dt, p(res), p(Q), None)


@pytest.mark.parametrize("N", [3, 5])
def test_noalloc_stage_equals_kernel_level_stage(cuda, N):
    import torch
    a, Q0, R0, Nq = _case(N)
    K = 48
    Qa, Ra = torch.from_numpy(Q0.copy()).cuda(), torch.from_numpy(R0.copy()).cuda()
    Qb, Rb = Qa.clone(), Ra.clone()
    rhs = torch.empty_like(Qa)
    dt = 1e-3
    for i in range(2):  # two calls in a row
        fa, fb = float(np.float32(RK4A[i])), float(np.float32(RK4B[i]))
        _three_kernels(N, K, Nq, a, Qa, Ra, rhs, fa, fb, dt)
        _noalloc(N, K, Nq, a, Qb, Rb, fa, fb, dt)
    torch.cuda.synchronize()
    assert torch.equal(Qa, Qb) and torch.equal(Ra, Rb)
    assert not torch.equal(Qa, torch.from_numpy(Q0).cuda())


def test_noalloc_rejects_meshes_beyond_the_scratch(cuda):
    a, Q0, R0, Nq = _case(5)
    import torch
    Q, R = torch.from_numpy(Q0.copy()).cuda(), torch.from_numpy(R0.copy()).cuda()
    with pytest.raises(BBWError) as e:
        _noalloc(5, 48, Nq, a, Q, R, 0.0, 0.1, 1e-3, k_override=18725)  # 18725 * 224 > 4 Mi
    assert e.value.status == 7
    torch.cuda.synchronize()
    assert torch.equal(Q, torch.from_numpy(Q0).cuda())
