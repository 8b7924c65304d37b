"""Host setup (C++, bbw_ops_build / bbw_mesh_*) against the reference's own
setup output (tests/golden, from StartUp3d / BuildMaps3d / WaveInitOCCA3d /
InitWADG_subelem run here).  CPU only."""
import numpy as np
import pytest
from conftest import golden

from bbwadg_b200.mesh import kuhn_box, read_gmsh22, write_gmsh22
from bbwadg_b200.problem import build_operators, connect_and_geometry


def ref_rule_ops(N):
    g = golden("ops_N%d.npz" % N)
    nfq = int(g["Nfq"][0])
    o = build_operators(N, cubature=(g["rq"], g["sq"], g["tq"], g["wq"]),
                        tri_cubature=(g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"]))
    return o, g


def maxrel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("N", [3, 4, 5, 6, 7])
def test_integer_maps_bit_exact(N):
    o, g = ref_rule_ops(N)
    for k in ["Fmask", "D_ids1", "D_ids2", "D_ids3", "D_ids4", "EEL_ids", "L0_ids", "slice_ids",
              "EEL_id_vec"]:
        assert np.array_equal(o[k], g[k].ravel()), k
    # faceVolPerm: reference stores an Eigen (Np x 3) column-major matrix
    assert np.array_equal(o["faceVolPerm"], g["faceVolPerm"].reshape(3, -1).T.ravel())


@pytest.mark.parametrize("N", [3, 4, 5, 6, 7])
def test_operators_match_reference(N):
    o, g = ref_rule_ops(N)
    for k in ["r", "s", "t"]:
        assert np.abs(o[k + "64"] - g[k]).max() < 1e-14, k
    # BB operators are rational; the reference's FP32 copies are reproduced exactly
    for k in ["Dvals4", "EEL_vals", "L0_vals", "cEL"]:
        assert np.array_equal(o[k], g[k]), k
    assert np.abs(o["EEL_val_vec64"] - g["EEL_val_vec"]).max() < 1e-12
    # nodal operators within 2 FP32 ulp (the reference evaluates its Jacobi
    # normalisation with single-precision tgamma)
    for k in ["Dr", "Ds", "Dt", "LIFT"]:
        assert maxrel(o[k], g[k]) < 2.5e-7, k
    for k in ["Vq_nodal", "Pq_nodal", "Vq_bb", "Pq_bb"]:
        assert maxrel(o[k], g[k]) < 2.5e-7, k


@pytest.mark.parametrize("N", [3, 5])
def test_fp64_operators_match_reference(N):
    o, g = ref_rule_ops(N)
    for k in ["V", "VB", "invVB"]:
        assert maxrel(o[k + "64"], g[k + "64"]) < 1e-6, k


@pytest.mark.parametrize("N", [3, 4, 5, 6, 7])
def test_connectivity_and_geometry_bit_exact(N):
    o, _ = ref_rule_ops(N)
    m = golden("mesh_box2_N%d.npz" % N)
    mm = connect_and_geometry(N, *kuhn_box(2), o)
    assert np.array_equal(mm["EToE"].ravel(), m["EToE"])
    assert np.array_equal(mm["EToF"].ravel(), m["EToF"])
    assert np.array_equal(mm["vmapP"], m["vmapP"])
    assert np.array_equal(mm["vgeo"], m["vgeo"])
    assert np.array_equal(mm["fgeo"], m["fgeo"])
    assert np.float32(mm["dt_ref"]) == np.float32(m["dt"][0])


def test_stroud_rule_gives_same_rule_independent_operators():
    for N in (3, 5):
        o, g = ref_rule_ops(N)
        s = build_operators(N)
        assert s["Nq"] == (N + 1) ** 3
        for k in ["Dr", "LIFT", "EEL_vals", "L0_vals", "Dvals4"]:
            assert maxrel(s[k], o[k]) < 1e-6, k
        for k in ["EEL_ids", "L0_ids", "D_ids1"]:
            assert np.array_equal(s[k], o[k]), k
        # both rules integrate degree 2N exactly: Pq Vq = I
        for v in ("nodal", "bb"):
            Np, Nq = s["Np"], s["Nq"]
            P = s["Pq_%s64" % v].reshape(Nq, Np).T
            V = s["Vq_%s64" % v].reshape(Np, Nq).T
            assert np.abs(P @ V - np.eye(Np)).max() < 1e-10


def test_vmapP_is_an_involution():
    N = 4
    o = build_operators(N)
    m = connect_and_geometry(N, *kuhn_box(3), o)
    Np, Nfp = o["Np"], o["Nfp"]
    vm = m["vmapP"].reshape(-1, 4 * Nfp)
    K = vm.shape[0]
    fm = o["Fmask"]
    # map (element, local volume node) of the + trace back through its own face
    for k in range(0, K, 7):
        for j in range(4 * Nfp):
            k2, v2 = divmod(int(vm[k, j]), 4 * Np)
            assert v2 < Np
            if k2 == k:
                assert v2 == fm[j]
                continue
            f2 = int(m["EToF"][k, j // Nfp])
            back = vm[k2, f2 * Nfp:(f2 + 1) * Nfp]
            assert k * 4 * Np + fm[j] in back


def test_gmsh_roundtrip(tmp_path):
    VX, VY, VZ, E = kuhn_box(3, -0.5, 0.5)
    p = str(tmp_path / "box.msh")
    write_gmsh22(p, VX, VY, VZ, E)
    VX2, VY2, VZ2, E2 = read_gmsh22(p)
    assert np.array_equal(VX, VX2) and np.array_equal(VY, VY2) and np.array_equal(VZ, VZ2)
    assert np.array_equal(E, E2)


def test_kuhn_box_is_conforming_and_positive():
    VX, VY, VZ, E = kuhn_box(4)
    o = build_operators(2)
    m = connect_and_geometry(2, VX, VY, VZ, E, o)
    bnd = (m["EToE"] == np.arange(len(E))[:, None]).sum()
    assert bnd == 6 * 4 * 4 * 2  # 2 triangles per boundary square
    assert m["dt_ref"] > 0


def test_mesh_errors_are_reported():
    from bbwadg_b200._lib import BBWError
    VX, VY, VZ, E = kuhn_box(1)
    E = E.copy()
    E[0, 2], E[0, 3] = E[0, 3], E[0, 2]  # negative orientation
    o = build_operators(2)
    with pytest.raises(BBWError):
        connect_and_geometry(2, VX, VY, VZ, E, o)
