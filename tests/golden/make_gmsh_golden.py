#!/usr/bin/env python3
"""Generate the unstructured-mesh fixtures from the reference itself.

Runs the reference's own Gmsh reader and connectivity (ReadGmsh3d,
FacePair3d, StartUp3d / BuildMaps3d: cpp/src/Mesh3d.cpp:9-200, 335-410,
cpp/src/StartUp3d.cpp:643-741), built into oracle/_ref (``make -C oracle
REF=<reference>/cpp``), on the Gmsh 2.2 meshes shipped with the reference
(cpp/meshes/*.msh), and stores per mesh

  gmsh_<name>.npz   VX VY VZ (FP64) and EToV (after the reference's
                    orientation fix) as read by ReadGmsh3d; EToE, EToF
                    (FacePair3d); vmapM / vmapP (BuildMaps3d, node ids
                    k*Np + n) at N = 3; the element list as written in the
                    file (EToV_file); the state after 20 LSRK45 steps of the
                    reference's affine path at N = 3 (Gaussian pulse, sine
                    c^2, p = 0 walls, the reference's own dt) on the same
                    mesh, and the c^2 / initial state it started from.

Usage: python tests/golden/make_gmsh_golden.py <reference>/cpp/meshes
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

REF = os.path.join(ROOT, "oracle", "_ref")
MESHES = ["tet", "cube1", "cube2", "cube3", "cube4", "sphere48", "sphere385"]
STEPS = 20


def run(*args):
    exe = os.path.join(REF, "ref_N3_B0")
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    subprocess.run([exe] + [str(a) for a in args], check=True, env=env, stdout=subprocess.PIPE)


def file_elements(path):
    """The tetrahedra of a Gmsh 2.2 file as listed (1-based ids -> 0-based),
    before any orientation fix."""
    with open(path) as f:
        lines = f.read().split("\n")
    i = lines.index("$Elements")
    tets = []
    for ln in lines[i + 2:i + 2 + int(lines[i + 1])]:
        tok = ln.split()
        if int(tok[1]) == 4:
            nt = int(tok[2])
            tets.append([int(v) - 1 for v in tok[3 + nt:7 + nt]])
    return np.array(tets, np.int32)


def main(mesh_dir):
    tmp = tempfile.mkdtemp()
    for name in MESHES:
        msh = os.path.join(mesh_dir, name + ".msh")
        out = os.path.join(tmp, name + ".bin")
        run("mesh", msh, out)
        d = bbwa.read(out)
        K = int(d["K"][0])
        g = {"VX": d["VX"], "VY": d["VY"], "VZ": d["VZ"],
             "EToV": d["EToV"].reshape(K, 4), "EToE": d["EToE"].reshape(K, 4),
             "EToF": d["EToF"].reshape(K, 4), "vmapM": d["vmapM_raw"], "vmapP": d["vmapP_raw"],
             "EToV_file": file_elements(msh)}
        # the reference's affine path on the same mesh (its own dt and c^2)
        out = os.path.join(tmp, name + "_dump.bin")
        run("dump", msh, out, "--c2", "sine", "--ic", "gauss")
        dd = bbwa.read(out)
        g["c2q"], g["Q0"], g["dt"] = dd["c2q"], dd["Q0"], dd["dt"]
        out = os.path.join(tmp, name + "_run.bin")
        run("run", msh, out, "--stages", 5 * STEPS, "--c2", "sine", "--ic", "gauss")
        o = bbwa.read(out)
        g["Q_run"] = o["Q"]
        g["steps"] = np.int32(STEPS)
        np.savez_compressed(os.path.join(HERE, "gmsh_%s.npz" % name), **g)
        print(name, "K =", K)


if __name__ == "__main__":
    main(sys.argv[1])
