#!/usr/bin/env python3
"""Generate the curvilinear-path golden fixtures from the reference itself.

Runs the reference's own curved setup and kernels (cpp/main.cpp:58-99 with
GORDON_HALL=1, RK_step_WADG), built by ``make -C oracle curved`` into
oracle/_ref/ref_curved_N{2,3}, on the unit ball kuhn_ball(4) (K = 384,
288 curved), and stores:

  curved_ball4_N{N}.npz
    cubature rules (rq sq tq wq, face rule rfq sfq wfqFace), dt,
    KlistCurved / KlistPlanar, Gordon-Hall node coordinates x y z (FP64,
    [K][Np]) and vgeoq / Jq / fgeoq of the first 64 elements (FP32),
    the curved operators (FP32), c2q_in (seeded, [K][Nq]) and the state and
    residual after 50 stages of RK_step_WADG from the Bessel initial state;
    for N = 3 also each of the four curved-path kernels on seeded random
    inputs (q_in, rhs_in -> <kernel>.rhsQ).

With the reference's mesh directory as argument, the same fixtures (without
the kernel cases) are also written for its Gmsh sphere meshes
sphere48.msh and sphere385.msh (the inputs of cpp/main.cpp:58-99):
curved_sphere48_N{N}.npz, curved_sphere385_N{N}.npz (the mesh itself, as
the reference reads it, is in gmsh_sphere*.npz).

Usage: python tests/golden/make_curved_golden.py [<reference>/cpp/meshes]
(needs oracle/_ref built from the reference checkout)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import bbwa  # noqa: E402
from bbwadg_b200.mesh import kuhn_ball, write_gmsh22  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OPS = ["Vrq", "Vsq", "Vtq", "Prq", "Psq", "Ptq", "VfqFace", "Pfq", "Vfq"]
KERNELS = ["rk_volume_WADG_skew_combine", "rk_surface_WADG_skew_combine", "rk_volume_planar",
           "rk_surface_planar"]
NSUB = 64
STAGES = 50


def run(N, *args):
    exe = os.path.join(REF, "ref_curved_N%d" % N)
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    subprocess.run([exe] + [str(a) for a in args], check=True, env=env, stdout=subprocess.PIPE)


def main(mesh_dir=None):
    tmp = tempfile.mkdtemp()
    ball = os.path.join(tmp, "ball4.msh")
    write_gmsh22(ball, *kuhn_ball(4))
    cases = [("ball4", ball)]
    if mesh_dir:
        cases += [(m, os.path.join(mesh_dir, m + ".msh")) for m in ("sphere48", "sphere385")]
    for name, msh in cases:
        for N in (2, 3):
            fixture(tmp, name, msh, N)
    print("fixtures written to", HERE)


def fixture(tmp, name, ball, N):
    """One fixture file: the reference's curved setup and run on mesh `ball`."""
    out = os.path.join(tmp, "dump_%s_%d.bin" % (name, N))
    run(N, "dump", ball, out)
    d = bbwa.read(out)
    K, Nq = int(d["K"][0]), int(d["Nq"][0])
    Np, Nfq = (N + 1) * (N + 2) * (N + 3) // 6, int(d["Nfq"][0])
    g = {k: d[k] for k in ("rq", "sq", "tq", "wq", "rfq", "sfq", "wfqFace", "dt")}
    g["KlistCurved"] = d["KlistCurved"].astype(np.int32)
    g["KlistPlanar"] = d["KlistPlanar"].astype(np.int32)
    for c in ("x", "y", "z"):  # column-major [Np x K] -> [K][Np]
        g[c] = d[c].reshape(K, Np)
    g["vgeoq_sub"] = d["vgeoq"].reshape(K, 9 * Nq)[:NSUB]
    g["Jq_sub"] = d["Jq"].reshape(K, Nq)[:NSUB]
    g["fgeoq_sub"] = d["fgeoq"].reshape(K, 16 * Nfq)[:NSUB]
    for k in OPS:
        g[k] = d[k]
    rng = np.random.default_rng(3000 + N)
    c2q = (1.0 + 0.5 * rng.random(K * Nq)).astype(np.float32)
    g["c2q_in"] = c2q
    fc2 = os.path.join(tmp, "c2q_%s_%d.bin" % (name, N))
    c2q.tofile(fc2)
    out = os.path.join(tmp, "run_%s_%d.bin" % (name, N))
    run(N, "run", ball, out, "--stages", STAGES, "--c2q", fc2)
    o = bbwa.read(out)
    g["Q_run"], g["res_run"] = o["Q"], o["resQ"]
    g["stages"] = np.int32(STAGES)
    if N == 3 and name == "ball4":
        q = rng.standard_normal(K * 4 * Np).astype(np.float32)
        rhs = rng.standard_normal(K * 4 * Np).astype(np.float32)
        fq, fr = os.path.join(tmp, "q.bin"), os.path.join(tmp, "rhs.bin")
        q.tofile(fq)
        rhs.tofile(fr)
        g["q_in"], g["rhs_in"] = q, rhs
        for which in KERNELS:
            out = os.path.join(tmp, "k_%s.bin" % which)
            run(N, "kernel", ball, out, "--which", which, "--q0", fq, "--rhs", fr)
            g[which + ".rhsQ"] = bbwa.read(out)["rhsQ"]
    np.savez_compressed(os.path.join(HERE, "curved_%s_N%d.npz" % (name, N)), **g)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
