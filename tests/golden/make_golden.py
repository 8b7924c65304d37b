#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden from the reference itself.

Runs the reference's own setup code and OKL kernels, built by
``make -C oracle`` into oracle/_ref (the reference sources are compiled
where they lie; see oracle/Makefile), and stores their outputs as .npz:

  ops_N{N}.npz            operators exactly as uploaded by WaveInitOCCA3d /
                          InitWADG_subelem (FP32), the nodes and cubature,
                          FP64 operators for N <= 5, LSRK45 coefficients
  mesh_box2_N{N}.npz      2^3 x 6 tets on [-1,1]^3: vgeo, fgeo, vmapP,
                          EToE/EToF, c2q (sine field), dt, initial states
  kernels_N{N}_box2.npz   each hot-path kernel on seeded random inputs
  run_N3_box4.npz         4^3 x 6 tets, Gaussian pulse, sine c^2, 100 LSRK45
                          steps (nodal and BB): initial and final state

Usage: python tests/golden/make_golden.py [N ...]   (needs the reference
checkout; default orders 3 4 5 6 7; run_N3_box4 is written when 3 is among
them)
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
from bbwadg_b200.mesh import kuhn_box, write_gmsh22  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
F32_OPS = ["Dr", "Ds", "Dt", "LIFT", "Fmask", "D_ids1", "D_ids2", "D_ids3", "D_ids4", "Dvals4",
           "EEL_ids", "EEL_vals", "L0_ids", "L0_vals", "cEL", "slice_ids"]
NODE_OPS = ["r", "s", "t", "rq", "sq", "tq", "wq", "wfqFace", "rfq", "sfq", "EEL_val_vec", "EEL_id_vec",
            "faceVolPerm", "rk"]
F64_OPS = ["V64", "Dr64", "Ds64", "Dt64", "LIFT64", "VB64", "invVB64", "Vq64"]


def run(N, B, *args):
    exe = os.path.join(REF, "ref_N%d_B%d" % (N, B))
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    subprocess.run([exe] + [str(a) for a in args], check=True, env=env,
                   stdout=subprocess.PIPE)


def main(orders=(3, 4, 5, 6, 7)):
    tmp = tempfile.mkdtemp()
    box2 = os.path.join(tmp, "box2.msh")
    write_gmsh22(box2, *kuhn_box(2))
    box4 = os.path.join(tmp, "box4.msh")
    write_gmsh22(box4, *kuhn_box(4))

    for N in orders:
        d = {}
        for B in (0, 1):
            out = os.path.join(tmp, "dump_%d_%d.bin" % (N, B))
            run(N, B, "dump", box2, out, "--c2", "sine", "--ic", "gauss")
            d[B] = bbwa.read(out)
        a = d[0]
        ops = {k: a[k] for k in F32_OPS + NODE_OPS}
        for k in ("Nq", "Nfq", "EEL_nnz", "L0_nnz"):
            ops[k] = a[k]
        ops["Vq_nodal"], ops["Pq_nodal"] = d[0]["Vq"], d[0]["Pq"]
        ops["Vq_bb"], ops["Pq_bb"] = d[1]["Vq"], d[1]["Pq"]
        if N <= 5:
            for k in F64_OPS:
                ops[k] = a[k]
        np.savez_compressed(os.path.join(HERE, "ops_N%d.npz" % N), **ops)

        mesh = {k: a[k] for k in ("vgeo", "fgeo", "vmapP", "EToE", "EToF", "c2q", "Jq", "dt",
                                  "vmapM_raw", "vmapP_raw")}
        mesh["Q0_nodal"], mesh["Q0_bb"] = d[0]["Q0"], d[1]["Q0"]
        if N == 3:
            for k in ("x", "y", "z"):
                mesh[k] = a[k]
        np.savez_compressed(os.path.join(HERE, "mesh_box2_N%d.npz" % N), **mesh)

        if N in (3, 5):
            K, Np = 48, (N + 1) * (N + 2) * (N + 3) // 6
            rng = np.random.default_rng(1000 + N)
            q = rng.standard_normal(K * 4 * Np).astype(np.float32)
            rhs = rng.standard_normal(K * 4 * Np).astype(np.float32)
            res = rng.standard_normal(K * 4 * Np).astype(np.float32)
            fa, fb = -0.41789047, 0.37921031
            files = {}
            for nm, arr in (("q", q), ("rhs", rhs), ("res", res)):
                files[nm] = os.path.join(tmp, "%s_%d.bin" % (nm, N))
                arr.tofile(files[nm])
            kern = {"Q_in": q, "rhs_in": rhs, "res_in": res, "fa": np.float32(fa),
                    "fb": np.float32(fb)}
            jobs = [(0, "rk_volume"), (0, "rk_surface"), (0, "rk_update"), (0, "rk_update_WADG"),
                    (1, "rk_volume_bern"), (1, "rk_surface_bern"), (1, "rk_surface_bern_slice"),
                    (1, "rk_update_WADG")]
            for B, which in jobs:
                out = os.path.join(tmp, "k_%d_%s_%d.bin" % (N, which, B))
                run(N, B, "kernel", box2, out, "--which", which, "--c2", "sine",
                    "--q0", files["q"], "--rhs", files["rhs"], "--res", files["res"],
                    "--fa", repr(fa), "--fb", repr(fb))
                o = bbwa.read(out)
                tag = which + ("_bb" if (which == "rk_update_WADG" and B) else "")
                if which.startswith("rk_update"):
                    kern[tag + ".resQ"], kern[tag + ".Q"] = o["resQ"], o["Q"]
                    kern["dt"] = o["dt"]
                else:
                    kern[tag + ".rhsQ"] = o["rhsQ"]
            np.savez_compressed(os.path.join(HERE, "kernels_N%d_box2.npz" % N), **kern)

    if 3 not in orders:
        print("fixtures written to", HERE)
        return
    N = 3
    runs = {}
    for B, tag in ((0, "nodal"), (1, "bb")):
        out = os.path.join(tmp, "d4_%d.bin" % B)
        run(N, B, "dump", box4, out, "--c2", "sine", "--ic", "gauss")
        dd = bbwa.read(out)
        runs["Q0_" + tag] = dd["Q0"]
        runs["c2q"], runs["dt"] = dd["c2q"], dd["dt"]
        out = os.path.join(tmp, "r4_%d.bin" % B)
        run(N, B, "run", box4, out, "--c2", "sine", "--ic", "gauss", "--stages", 500)
        runs["Q100_" + tag] = bbwa.read(out)["Q"]
        out = os.path.join(tmp, "r4s_%d.bin" % B)
        run(N, B, "run", box4, out, "--c2", "sine", "--ic", "gauss", "--stages", 1)
        o = bbwa.read(out)
        runs["Q1stage_" + tag], runs["res1stage_" + tag] = o["Q"], o["resQ"]
    np.savez_compressed(os.path.join(HERE, "run_N3_box4.npz"), **runs)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main(tuple(int(a) for a in sys.argv[1:]) or (3, 4, 5, 6, 7))
