"""The N=3 workload at full size (8^3 x 6 tets, K = 3072; sine c^2,
Gaussian pulse, p = 0 walls, CFL 0.5, 100 LSRK45 steps) on the GPU against
the reference's own CPU path (its host code and OKL kernels, built in
oracle/_ref) run here on the same mesh file, c^2, initial state and dt.
FP32 tolerance 1e-5 relative L2."""
import os
import subprocess

import numpy as np
import pytest
from conftest import ROOT, golden, rel_l2

from bbwadg_b200 import WaveSolver, make_problem
from bbwadg_b200.mesh import kuhn_box, write_gmsh22

pytestmark = pytest.mark.gpu


def ref_rule(N):
    g = golden("ops_N%d.npz" % N)
    nfq = int(g["Nfq"][0])
    return (g["rq"], g["sq"], g["tq"], g["wq"]), (g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"])


@pytest.mark.parametrize("variant", ["nodal", "bb"])
def test_c1_100_steps_match_the_reference_cpu_path(cuda, tmp_path, variant):
    import bbwa
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_N3_B%d" % (variant == "bb"))
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref not built")
    msh = str(tmp_path / "box8.msh")
    write_gmsh22(msh, *kuhn_box(8))
    cub, tri = ref_rule(3)
    p = make_problem(3, mesh=msh, variant=variant, c2="sine", ic="gauss", cubature=cub,
                     tri_cubature=tri, cfl=0.5)
    assert p.K == 3072
    q0, c2q, out = tmp_path / "q0.bin", tmp_path / "c2q.bin", str(tmp_path / "out.bin")
    np.ascontiguousarray(p.Q0, np.float32).tofile(q0)
    np.ascontiguousarray(p.c2q, np.float32).tofile(c2q)
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    subprocess.run([exe, "run", msh, out, "--stages", "500", "--q0", str(q0), "--c2q", str(c2q),
                    "--dt", "%.9g" % np.float32(p.dt), "--c2", "sine"], check=True, env=env,
                   stdout=subprocess.DEVNULL, timeout=600)
    q_ref = bbwa.read(out)["Q"]
    s = WaveSolver(p)
    s.set_data(p.Q0)
    s.steps(p.dt, 100)
    q = s.get_data()
    s.close()
    assert np.isfinite(q).all()
    assert rel_l2(q, q_ref) < 1e-5
