"""Structured tetrahedral meshes and Gmsh 2.2 I/O.

The reference reads meshes with ``ReadGmsh3d`` (cpp/src/Mesh3d.cpp:9-200):
Gmsh 2.2 ASCII, tetrahedra are element type 4 with exactly two tags, vertex
ids are 1-based.  The workloads here are the unit box [lo,hi]^3 split into
n^3 hexahedra and each hexahedron into 6 Kuhn (Freudenthal) tetrahedra, so
K = 6 n^3.

Two properties are enforced so that the reference's own connectivity code
produces a correct mesh from the same file:

* every tetrahedron is positively oriented, because ``ReadGmsh3d`` fills the
  vertex coordinates before it swaps vertices of negatively oriented
  elements (cpp/src/Mesh3d.cpp:117-160), which would leave geometry and
  connectivity inconsistent;
* boundary vertices are numbered before interior ones, because
  ``FacePair3d`` (cpp/src/Mesh3d.cpp:383-405) compares only two of the three
  sorted face vertices and never visits the last sorted face; with the
  largest vertex ids interior, the last face is interior and no two
  consecutive sorted faces share their two smallest vertices.
"""
import itertools

import numpy as np


def kuhn_box(n, lo=-1.0, hi=1.0):
    """Return (VX, VY, VZ, EToV) for [lo,hi]^3 split into n^3 x 6 tets.

    EToV is int32 [K][4], 0-based.  Elements are ordered hex by hex with
    x fastest, the 6 tets of a hex contiguous.
    """
    n = int(n)
    g = np.linspace(lo, hi, n + 1)
    # grid index (i,j,k) -> vertex id, boundary vertices first
    ii, jj, kk = np.meshgrid(np.arange(n + 1), np.arange(n + 1), np.arange(n + 1), indexing="ij")
    ii, jj, kk = ii.ravel(order="F"), jj.ravel(order="F"), kk.ravel(order="F")
    on_bnd = (ii == 0) | (ii == n) | (jj == 0) | (jj == n) | (kk == 0) | (kk == n)
    order = np.concatenate([np.nonzero(on_bnd)[0], np.nonzero(~on_bnd)[0]])
    vid = np.empty((n + 1) ** 3, dtype=np.int64)
    vid[order] = np.arange((n + 1) ** 3)
    VX = g[ii[order]].copy()
    VY = g[jj[order]].copy()
    VZ = g[kk[order]].copy()

    def gid(i, j, k):
        return vid[i + (n + 1) * (j + (n + 1) * k)]

    tets = []
    for perm in itertools.permutations(range(3)):
        path = [(0, 0, 0)]
        cur = [0, 0, 0]
        for ax in perm:
            cur[ax] = 1
            path.append(tuple(cur))
        tets.append(path)
    hk, hj, hi_ = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    hi_, hj, hk = hi_.ravel(), hj.ravel(), hk.ravel()
    EToV = np.empty((n ** 3, 6, 4), dtype=np.int64)
    for t, path in enumerate(tets):
        for v, (a, b, c) in enumerate(path):
            EToV[:, t, v] = gid(hi_ + a, hj + b, hk + c)
    EToV = EToV.reshape(-1, 4)
    # force positive orientation (swap the last two vertices)
    x = VX[EToV]
    y = VY[EToV]
    z = VZ[EToV]
    d1 = np.stack([x[:, 1] - x[:, 0], y[:, 1] - y[:, 0], z[:, 1] - z[:, 0]], 1)
    d2 = np.stack([x[:, 2] - x[:, 0], y[:, 2] - y[:, 0], z[:, 2] - z[:, 0]], 1)
    d3 = np.stack([x[:, 3] - x[:, 0], y[:, 3] - y[:, 0], z[:, 3] - z[:, 0]], 1)
    J = np.einsum("ij,ij->i", d1, np.cross(d2, d3))
    neg = J < 0
    EToV[neg, 2], EToV[neg, 3] = EToV[neg, 3].copy(), EToV[neg, 2].copy()
    return VX, VY, VZ, EToV.astype(np.int32)


def kuhn_ball(n):
    """Return (VX, VY, VZ, EToV) for the unit ball, n even.

    The box [-1,1]^3 is cut into n^3 hexahedra and each into 6 Kuhn
    tetrahedra around the hexahedron's diagonal that points away from the
    centre (the Kuhn pattern mirrored into each octant, which keeps shared
    faces conforming).  Every vertex then moves radially, x -> x |x|_inf /
    |x|_2, so the cube surface lands on the unit sphere.  With the diagonal
    pointing outward, two vertices of one tetrahedron that both lie on the
    sphere always share a boundary face, so no chord through the interior
    has both ends on the sphere: the Gordon-Hall curving, which snaps every
    edge whose end points lie on the sphere (cpp/src/WaveOKL3d.cpp:1071-1100),
    only moves true boundary edges.  Stands in for the reference's Gmsh
    sphere meshes (cpp/meshes/sphere*.msh)."""
    n = int(n)
    if n < 2 or n % 2:
        raise ValueError("kuhn_ball: n must be even and >= 2")
    VX, VY, VZ, _ = kuhn_box(n)
    # vertex id of grid point (i,j,k), from the coordinates kuhn_box assigned
    idx = np.rint((np.stack([VX, VY, VZ], 1) + 1.0) * n / 2.0).astype(np.int64)
    vid = np.empty((n + 1) ** 3, np.int64)
    vid[idx[:, 0] + (n + 1) * (idx[:, 1] + (n + 1) * idx[:, 2])] = np.arange(len(VX))
    hk, hj, hi_ = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    h = np.stack([hi_.ravel(), hj.ravel(), hk.ravel()], 1)          # hex lower corner
    sgn = np.where(h >= n // 2, 1, -1)                                # outward per axis
    start = np.where(sgn > 0, h, h + 1)                               # corner nearest the centre
    EToV = np.empty((len(h), 6, 4), np.int64)
    for t, perm in enumerate(itertools.permutations(range(3))):
        cur = start.copy()
        for v in range(4):
            if v:
                ax = perm[v - 1]
                cur[:, ax] += sgn[:, ax]
            EToV[:, t, v] = vid[cur[:, 0] + (n + 1) * (cur[:, 1] + (n + 1) * cur[:, 2])]
    EToV = EToV.reshape(-1, 4)
    X = np.stack([VX, VY, VZ], 1)
    n2 = np.linalg.norm(X, axis=1)
    s = np.where(n2 > 0, np.abs(X).max(1) / np.where(n2 > 0, n2, 1.0), 1.0)
    X = X * s[:, None]
    v = X[EToV]
    d = v[:, 1:] - v[:, :1]
    J = np.einsum("ij,ij->i", d[:, 0], np.cross(d[:, 1], d[:, 2]))
    neg = J < 0
    EToV[neg, 2], EToV[neg, 3] = EToV[neg, 3].copy(), EToV[neg, 2].copy()
    if (np.abs(J) <= 1e-14).any():
        raise RuntimeError("kuhn_ball: degenerate element")
    return X[:, 0].copy(), X[:, 1].copy(), X[:, 2].copy(), EToV.astype(np.int32)


def write_gmsh22(path, VX, VY, VZ, EToV):
    """Write a Gmsh 2.2 ASCII file with coordinates in round-trip precision."""
    Nv = len(VX)
    K = len(EToV)
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % Nv)
        f.write("".join("%d %.17g %.17g %.17g\n" % (i + 1, VX[i], VY[i], VZ[i]) for i in range(Nv)))
        f.write("$EndNodes\n$Elements\n%d\n" % K)
        e = EToV.astype(np.int64) + 1
        f.write("".join("%d 4 2 0 1 %d %d %d %d\n" % (k + 1, e[k, 0], e[k, 1], e[k, 2], e[k, 3])
                        for k in range(K)))
        f.write("$EndElements\n")


def read_gmsh22(path):
    """Read tetrahedra from a Gmsh 2.2 ASCII file (the subset ReadGmsh3d reads).

    Negatively oriented tets get vertices 2 and 3 swapped, as in
    cpp/src/Mesh3d.cpp:142-160; unlike the reference, coordinates are taken
    after the swap, so geometry and connectivity always agree.
    """
    with open(path) as f:
        lines = f.read().split("\n")
    i = 0
    VX = VY = VZ = None
    tets = []
    while i < len(lines):
        ln = lines[i].strip()
        if ln == "$Nodes":
            nv = int(lines[i + 1])
            arr = np.array([lines[i + 2 + v].split() for v in range(nv)], dtype=np.float64)
            VX, VY, VZ = arr[:, 1].copy(), arr[:, 2].copy(), arr[:, 3].copy()
            i += 2 + nv
            continue
        if ln == "$Elements":
            ne = int(lines[i + 1])
            for e in range(ne):
                tok = lines[i + 2 + e].split()
                if int(tok[1]) == 4:
                    ntag = int(tok[2])
                    tets.append([int(v) - 1 for v in tok[3 + ntag:7 + ntag]])
            i += 2 + ne
            continue
        i += 1
    if VX is None:
        raise ValueError("%s: no $Nodes section" % path)
    EToV = np.array(tets, dtype=np.int64).reshape(-1, 4)
    x, y, z = VX[EToV], VY[EToV], VZ[EToV]
    d = [np.stack([x[:, m] - x[:, 0], y[:, m] - y[:, 0], z[:, m] - z[:, 0]], 1) for m in (1, 2, 3)]
    J = np.einsum("ij,ij->i", d[0], np.cross(d[1], d[2]))
    neg = J < 0
    EToV[neg, 2], EToV[neg, 3] = EToV[neg, 3].copy(), EToV[neg, 2].copy()
    return VX, VY, VZ, EToV.astype(np.int32)
