"""Kernel-level entry points (bbw_rk_*) on the GPU against the reference's
own kernels (golden vectors from oracle/_ref) and, at larger sizes, against
the C restatement.  Tolerance: 1e-5 relative L2 (FP32)."""
import numpy as np
import pytest
from conftest import golden, ref_ops, rel_l2

from bbwadg_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-5


_KEEP = []  # device buffers must outlive the asynchronous launches that use them


def dev(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a).copy()).cuda()
    _KEEP.append(t)
    return t


@pytest.fixture(autouse=True)
def _release_buffers():
    yield
    import torch
    torch.cuda.synchronize()
    _KEEP.clear()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def P(t):
    return t.data_ptr()


@pytest.mark.parametrize("N", [3, 5])
def test_rk_volume_and_surface_nodal(cuda, N):
    o, g, k = ref_ops(N, "nodal"), golden("mesh_box2_N%d.npz" % N), golden("kernels_N%d_box2.npz" % N)
    Q = dev(k["Q_in"])
    rhs = dev(np.zeros_like(k["Q_in"]))
    _lib.call("bbw_rk_volume", N, 48, P(dev(g["vgeo"])), P(dev(o["Dr"])), P(dev(o["Ds"])),
              P(dev(o["Dt"])), P(Q), P(rhs), None)
    assert rel_l2(host(rhs), k["rk_volume.rhsQ"]) < TOL
    rhs = dev(k["rhs_in"])
    _lib.call("bbw_rk_surface", N, 48, 0, P(dev(g["fgeo"])), P(dev(o["Fmask"])), P(dev(g["vmapP"])),
              P(dev(o["LIFT"])), P(Q), P(rhs), None)
    assert rel_l2(host(rhs), k["rk_surface.rhsQ"]) < TOL


@pytest.mark.parametrize("N", [3, 5])
def test_rk_volume_and_surface_bern(cuda, N):
    o, g, k = ref_ops(N, "bb"), golden("mesh_box2_N%d.npz" % N), golden("kernels_N%d_box2.npz" % N)
    Q = dev(k["Q_in"])
    rhs = dev(np.zeros_like(k["Q_in"]))
    _lib.call("bbw_rk_volume_bern", N, 48, P(dev(g["vgeo"])), P(dev(o["D_ids1"])),
              P(dev(o["D_ids2"])), P(dev(o["D_ids3"])), P(dev(o["D_ids4"])), P(dev(o["Dvals4"])),
              P(Q), P(rhs), None)
    assert rel_l2(host(rhs), k["rk_volume_bern.rhsQ"]) < TOL
    rhs = dev(k["rhs_in"])
    Np, Nfp = (N + 1) * (N + 2) * (N + 3) // 6, (N + 1) * (N + 2) // 2
    _lib.call("bbw_rk_surface_bern", N, 48, 0, P(dev(g["fgeo"])), P(dev(o["Fmask"])),
              P(dev(g["vmapP"])), P(dev(o["slice_ids"])), o["EEL_ids"].size // Np,
              P(dev(o["EEL_ids"])), P(dev(o["EEL_vals"])), o["L0_ids"].size // Nfp,
              P(dev(o["L0_ids"])), P(dev(o["L0_vals"])), P(dev(o["cEL"])), P(Q), P(rhs), None)
    assert rel_l2(host(rhs), k["rk_surface_bern.rhsQ"]) < TOL


@pytest.mark.parametrize("N", [3, 5])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_rk_update_wadg(cuda, N, variant):
    o, g, k = ref_ops(N, variant), golden("mesh_box2_N%d.npz" % N), golden("kernels_N%d_box2.npz" % N)
    rhs, res, Q = dev(k["rhs_in"]), dev(k["res_in"]), dev(k["Q_in"])
    Nq = int(o["Nq"][0])
    _lib.call("bbw_rk_update_wadg", N, 48, Nq, P(dev(o["Vq"])), P(dev(o["Pq"])), P(dev(g["Jq"])),
              P(dev(g["c2q"])), float(k["fa"]), float(k["fb"]), float(k["dt"][0]), P(rhs), P(res),
              P(Q), None)
    t = "rk_update_WADG" + ("_bb" if variant == "bb" else "")
    assert rel_l2(host(res), k[t + ".resQ"]) < TOL
    assert rel_l2(host(Q), k[t + ".Q"]) < TOL


def test_rk_update(cuda):
    k = golden("kernels_N3_box2.npz")
    rhs, res, Q = dev(k["rhs_in"]), dev(k["res_in"]), dev(k["Q_in"])
    _lib.call("bbw_rk_update", 3, 48, float(k["fa"]), float(k["fb"]), float(k["dt"][0]), P(rhs),
              P(res), P(Q), None)
    assert rel_l2(host(res), k["rk_update.resQ"]) < TOL
    assert rel_l2(host(Q), k["rk_update.Q"]) < TOL


def test_kernels_against_oracle_larger_mesh(cuda):
    """N=4 on 6^3 x 6 tets with the product setup: every kernel vs the C
    restatement (FP32, same summation order)."""
    from oracle import Oracle
    from bbwadg_b200 import make_problem
    for variant in ("nodal", "bb"):
        p = make_problem(4, 6, variant=variant)
        ops, geo = p.ops_dict(), p.geo_dict()
        orc = Oracle(4, p.K, ops, geo, variant=variant)
        rng = np.random.default_rng(7)
        q = rng.standard_normal(p.K * 4 * p.Np).astype(np.float32)
        r0 = np.zeros_like(q)
        orc.rk_volume(q, r0)
        orc.rk_surface(q, r0)
        Q, rhs = dev(q), dev(np.zeros_like(q))
        if variant == "nodal":
            _lib.call("bbw_rk_volume", 4, p.K, P(dev(geo["vgeo"])), P(dev(ops["Dr"])),
                      P(dev(ops["Ds"])), P(dev(ops["Dt"])), P(Q), P(rhs), None)
            _lib.call("bbw_rk_surface", 4, p.K, 0, P(dev(geo["fgeo"])), P(dev(ops["Fmask"])),
                      P(dev(geo["vmapP"])), P(dev(ops["LIFT"])), P(Q), P(rhs), None)
        else:
            _lib.call("bbw_rk_volume_bern", 4, p.K, P(dev(geo["vgeo"])), P(dev(ops["D_ids1"])),
                      P(dev(ops["D_ids2"])), P(dev(ops["D_ids3"])), P(dev(ops["D_ids4"])),
                      P(dev(ops["Dvals4"])), P(Q), P(rhs), None)
            _lib.call("bbw_rk_surface_bern", 4, p.K, 0, P(dev(geo["fgeo"])), P(dev(ops["Fmask"])),
                      P(dev(geo["vmapP"])), P(dev(ops["slice_ids"])), ops["EEL_nnz"],
                      P(dev(ops["EEL_ids"])), P(dev(ops["EEL_vals"])), ops["L0_nnz"],
                      P(dev(ops["L0_ids"])), P(dev(ops["L0_vals"])), P(dev(ops["cEL"])), P(Q),
                      P(rhs), None)
        assert rel_l2(host(rhs), r0) < TOL, variant


def test_empty_and_bad_arguments(cuda):
    assert _lib.lib().bbw_rk_volume(5, 0, None, None, None, None, None, None, None) == 0
    with pytest.raises(_lib.BBWError):
        _lib.call("bbw_rk_volume", 11, 4, 1, 1, 1, 1, 1, 1, None)


def _slice_args(o, N):
    Nfp = (N + 1) * (N + 2) // 2
    return [P(dev(o["slice_ids"])), P(dev(np.asarray(o["EEL_id_vec"], np.int32))),
            P(dev(np.asarray(o["EEL_val_vec"], np.float32))), o["L0_ids"].size // Nfp,
            P(dev(o["L0_ids"])), P(dev(o["L0_vals"])), P(dev(o["cEL"]))]


@pytest.mark.parametrize("N", [3, 5])
def test_rk_surface_bern_slice_matches_reference(cuda, N):
    """The slice-by-slice BB lift against the reference's own
    rk_surface_bern_slice (cpp/okl/WaveKernels.okl:652-939) on the same inputs."""
    o, g, k = ref_ops(N, "bb"), golden("mesh_box2_N%d.npz" % N), golden("kernels_N%d_box2.npz" % N)
    Q, rhs = dev(k["Q_in"]), dev(k["rhs_in"])
    _lib.call("bbw_rk_surface_bern_slice", N, 48, 0, P(dev(g["fgeo"])), P(dev(o["Fmask"])),
              P(dev(g["vmapP"])), *_slice_args(o, N), P(Q), P(rhs), None)
    assert rel_l2(host(rhs), k["rk_surface_bern_slice.rhsQ"]) < TOL


@pytest.mark.parametrize("bc", [0, 1])
def test_slice_lift_equals_sparse_lift_at_n7(cuda, bc):
    """N = 7, where the reference switches to the slice lift: both BB lifts
    agree (both boundary conditions)."""
    N = 7
    o, g = ref_ops(N, "bb"), golden("mesh_box2_N%d.npz" % N)
    Np, Nfp = (N + 1) * (N + 2) * (N + 3) // 6, (N + 1) * (N + 2) // 2
    rng = np.random.default_rng(3)
    Qh = rng.standard_normal(48 * 4 * Np).astype(np.float32)
    r0 = rng.standard_normal(48 * 4 * Np).astype(np.float32)
    Q, a, b = dev(Qh), dev(r0), dev(r0)
    common = [P(dev(g["fgeo"])), P(dev(o["Fmask"])), P(dev(g["vmapP"]))]
    _lib.call("bbw_rk_surface_bern_slice", N, 48, bc, *common, *_slice_args(o, N), P(Q), P(a), None)
    _lib.call("bbw_rk_surface_bern", N, 48, bc, *common, P(dev(o["slice_ids"])),
              o["EEL_ids"].size // Np, P(dev(o["EEL_ids"])), P(dev(o["EEL_vals"])),
              o["L0_ids"].size // Nfp, P(dev(o["L0_ids"])), P(dev(o["L0_vals"])),
              P(dev(o["cEL"])), P(Q), P(b), None)
    assert rel_l2(host(a) - r0, host(b) - r0) < 1e-5


@pytest.mark.parametrize("n_elems", [1, 2])
@pytest.mark.parametrize("N", [3, 5])
@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_kernels_on_one_and_two_elements(cuda, n_elems, N, variant):
    """Volume, surface and WADG update on one element (all faces walls) and
    on two sharing a face: partial element blocks against the restatement."""
    from oracle import Oracle
    from bbwadg_b200 import make_problem
    VX = np.array([0.0, 1.0, 0.0, 0.0, 0.3])
    VY = np.array([0.0, 0.0, 1.0, 0.0, 0.3])
    VZ = np.array([0.0, 0.0, 0.0, 1.0, -0.9])
    EToV = np.array([[0, 1, 2, 3], [0, 2, 1, 4]][:n_elems], np.int32)
    p = make_problem(N, mesh=(VX, VY, VZ, EToV), variant=variant, c2="sine", seed=3)
    ops, geo = p.ops_dict(), p.geo_dict()
    orc = Oracle(N, p.K, ops, geo, variant=variant)
    rng = np.random.default_rng(11)
    q = rng.standard_normal(p.K * 4 * p.Np).astype(np.float32)
    res0 = rng.standard_normal(q.size).astype(np.float32)
    r0 = np.zeros_like(q)
    orc.rk_volume(q, r0)
    orc.rk_surface(q, r0)
    rhs_ref = r0.copy()
    res_ref, q_ref = res0.copy(), q.copy()
    fa, fb, fdt = np.float32(-0.4), np.float32(0.37), np.float32(p.dt)
    orc.rk_update_wadg(fa, fb, fdt, r0, res_ref, q_ref)
    Q, rhs, res = dev(q), dev(np.zeros_like(q)), dev(res0)
    if variant == "nodal":
        _lib.call("bbw_rk_volume", N, p.K, P(dev(geo["vgeo"])), P(dev(ops["Dr"])),
                  P(dev(ops["Ds"])), P(dev(ops["Dt"])), P(Q), P(rhs), None)
        _lib.call("bbw_rk_surface", N, p.K, 0, P(dev(geo["fgeo"])), P(dev(ops["Fmask"])),
                  P(dev(geo["vmapP"])), P(dev(ops["LIFT"])), P(Q), P(rhs), None)
    else:
        _lib.call("bbw_rk_volume_bern", N, p.K, P(dev(geo["vgeo"])), P(dev(ops["D_ids1"])),
                  P(dev(ops["D_ids2"])), P(dev(ops["D_ids3"])), P(dev(ops["D_ids4"])),
                  P(dev(ops["Dvals4"])), P(Q), P(rhs), None)
        _lib.call("bbw_rk_surface_bern", N, p.K, 0, P(dev(geo["fgeo"])), P(dev(ops["Fmask"])),
                  P(dev(geo["vmapP"])), P(dev(ops["slice_ids"])), ops["EEL_nnz"],
                  P(dev(ops["EEL_ids"])), P(dev(ops["EEL_vals"])), ops["L0_nnz"],
                  P(dev(ops["L0_ids"])), P(dev(ops["L0_vals"])), P(dev(ops["cEL"])), P(Q),
                  P(rhs), None)
    assert rel_l2(host(rhs), rhs_ref) < TOL
    _lib.call("bbw_rk_update_wadg", N, p.K, p.Nq, P(dev(ops["Vq"])), P(dev(ops["Pq"])),
              P(dev(geo["Jq"])), P(dev(geo["c2q"])), float(fa), float(fb), float(fdt), P(rhs),
              P(res), P(Q), None)
    assert rel_l2(host(res), res_ref) < TOL
    assert rel_l2(host(Q), q_ref) < TOL


@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_kernels_at_n8(cuda, variant):
    """The highest order (N = 8, Np = 165, Nq = 729): volume, surface and WADG
    update against the restatement."""
    from oracle import Oracle
    from bbwadg_b200 import make_problem
    N = 8
    p = make_problem(N, 2, variant=variant, c2="sine", seed=3)
    ops, geo = p.ops_dict(), p.geo_dict()
    orc = Oracle(N, p.K, ops, geo, variant=variant)
    rng = np.random.default_rng(8)
    q = rng.standard_normal(p.K * 4 * p.Np).astype(np.float32)
    res0 = rng.standard_normal(q.size).astype(np.float32)
    r0 = np.zeros_like(q)
    orc.rk_volume(q, r0)
    orc.rk_surface(q, r0)
    rhs_ref = r0.copy()
    res_ref, q_ref = res0.copy(), q.copy()
    fa, fb, fdt = np.float32(-0.4), np.float32(0.37), np.float32(p.dt)
    orc.rk_update_wadg(fa, fb, fdt, r0, res_ref, q_ref)
    Q, rhs, res = dev(q), dev(np.zeros_like(q)), dev(res0)
    if variant == "nodal":
        _lib.call("bbw_rk_volume", N, p.K, P(dev(geo["vgeo"])), P(dev(ops["Dr"])),
                  P(dev(ops["Ds"])), P(dev(ops["Dt"])), P(Q), P(rhs), None)
        _lib.call("bbw_rk_surface", N, p.K, 0, P(dev(geo["fgeo"])), P(dev(ops["Fmask"])),
                  P(dev(geo["vmapP"])), P(dev(ops["LIFT"])), P(Q), P(rhs), None)
    else:
        _lib.call("bbw_rk_volume_bern", N, p.K, P(dev(geo["vgeo"])), P(dev(ops["D_ids1"])),
                  P(dev(ops["D_ids2"])), P(dev(ops["D_ids3"])), P(dev(ops["D_ids4"])),
                  P(dev(ops["Dvals4"])), P(Q), P(rhs), None)
        _lib.call("bbw_rk_surface_bern", N, p.K, 0, P(dev(geo["fgeo"])), P(dev(ops["Fmask"])),
                  P(dev(geo["vmapP"])), P(dev(ops["slice_ids"])), ops["EEL_nnz"],
                  P(dev(ops["EEL_ids"])), P(dev(ops["EEL_vals"])), ops["L0_nnz"],
                  P(dev(ops["L0_ids"])), P(dev(ops["L0_vals"])), P(dev(ops["cEL"])), P(Q),
                  P(rhs), None)
    assert rel_l2(host(rhs), rhs_ref) < TOL
    _lib.call("bbw_rk_update_wadg", N, p.K, p.Nq, P(dev(ops["Vq"])), P(dev(ops["Pq"])),
              P(dev(geo["Jq"])), P(dev(geo["c2q"])), float(fa), float(fb), float(fdt), P(rhs),
              P(res), P(Q), None)
    assert rel_l2(host(res), res_ref) < TOL
    assert rel_l2(host(Q), q_ref) < TOL
