"""The fused stage on the reference's own unstructured meshes
(cpp/meshes/{cube1-4,sphere48,sphere385}.msh: Gmsh-generated tetrahedra of
the unit cube and of the unit ball with flat faces) against the reference's
own CPU path run on the same file: Gaussian pulse, sine c^2 at the
reference's 31-point rule, p = 0 walls, the reference's dt, 20 LSRK45 steps
(tests/golden/gmsh_*.npz).  The single-tetrahedron mesh is left out: the
reference mis-pairs its faces (see tests/test_gmsh.py).  FP32 tolerance
1e-5 relative L2."""
import numpy as np
import pytest
from conftest import golden, rel_l2

from bbwadg_b200 import WaveSolver, make_problem

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.mark.parametrize("name", ["cube1", "cube2", "cube3", "cube4", "sphere48", "sphere385"])
@pytest.mark.parametrize("form", ["fp32", "f16x3"])
def test_unstructured_mesh_matches_reference_run(cuda, name, form):
    g = golden("gmsh_%s.npz" % name)
    o = golden("ops_N3.npz")
    nfq = int(o["Nfq"][0])
    p = make_problem(3, mesh=(g["VX"], g["VY"], g["VZ"], g["EToV"]), variant="nodal",
                     cubature=(o["rq"], o["sq"], o["tq"], o["wq"]),
                     tri_cubature=(o["rfq"][:nfq], o["sfq"][:nfq], o["wfqFace"]))
    assert np.float32(p.dt) == np.float32(g["dt"][0])
    # the reference's own c^2 at the cubature points and initial state
    assert rel_l2(p.c2q.ravel(), g["c2q"]) < 1e-6 and rel_l2(p.Q0, g["Q0"]) < 1e-6
    p.c2q = g["c2q"].reshape(p.K, -1).copy()
    p.Q0 = g["Q0"].copy()
    s = WaveSolver(p, precision=form)
    s.set_data(p.Q0)
    s.steps(float(g["dt"][0]), int(g["steps"]))
    s.check()
    q = s.get_data()
    s.close()
    assert np.isfinite(q).all()
    assert rel_l2(q, g["Q_run"]) < TOL
