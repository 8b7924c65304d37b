"""Problem setup: operators, mesh arrays, wave-speed field and initial state.

Thin Python front end over the native setup entry points (include/bbwadg.h:
bbw_ops_build, bbw_mesh_connect, bbw_mesh_geometry, bbw_mesh_vmapP).  It
plays the role of the reference's host setup sequence
(cpp/main_subelem.cpp:27-69: ReadGmsh3d, FacePair3d, StartUp3d,
WaveInitOCCA3d, InitWADG_subelem, WaveSetU0) and returns plain numpy arrays
in the reference's layouts.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .mesh import kuhn_box, read_gmsh22

_F32, _F64, _I32 = 0, 1, 2
_CURVED_OPS = ["Vrq", "Vsq", "Vtq", "Prq", "Psq", "Ptq", "Vfq", "Pfq", "VfqFace"]
_OPS_F32 = ["Dr", "Ds", "Dt", "LIFT", "Vq_nodal", "Pq_nodal", "Vq_bb", "Pq_bb", "cEL", "Dvals4",
            "EEL_vals", "L0_vals"] + _CURVED_OPS
_OPS_F64 = ["V", "VB", "invVB", "LIFTB", "EEL", "r", "s", "t", "rq", "sq", "tq", "wq", "rfq", "sfq",
            "wfq", "EEL_val_vec", "Dr", "Ds", "Dt", "LIFT", "Vq_nodal", "Pq_nodal", "Vq_bb",
            "Pq_bb", "cEL", "Dvals4", "EEL_vals", "L0_vals"] + _CURVED_OPS
_OPS_I32 = ["Fmask", "D_ids1", "D_ids2", "D_ids3", "D_ids4", "EEL_ids", "L0_ids", "slice_ids",
            "EEL_id_vec", "faceVolPerm", "sizes"]


def np_of(N):
    return (N + 1) * (N + 2) * (N + 3) // 6


def nfp_of(N):
    return (N + 1) * (N + 2) // 2


def build_operators(N, cubature=None, tri_cubature=None):
    """Reference-element operators of degree N.

    ``cubature`` = (rq, sq, tq, wq) and ``tri_cubature`` = (rfq, sfq, wfq)
    select the volume / face rules; None builds Stroud rules of degree 2N+1.
    Returns a dict: FP32 arrays in kernel layouts under their names, FP64
    arrays under ``name + '64'``, int32 arrays under their names.
    """
    cub = tri = None
    nq = nfq = 0
    if cubature is not None:
        cub = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64) for a in cubature]))
        nq = len(cubature[0])
    if tri_cubature is not None:
        tri = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64) for a in tri_cubature]))
        nfq = len(tri_cubature[0])
    h = ctypes.c_void_p()
    _lib.call("bbw_ops_build", N, _lib.ptr(cub), nq, _lib.ptr(tri), nfq, ctypes.byref(h))
    out = {}
    try:
        for names, dt, np_dt, suffix in ((_OPS_F32, _F32, np.float32, ""),
                                         (_OPS_F64, _F64, np.float64, "64"),
                                         (_OPS_I32, _I32, np.int32, "")):
            for nm in names:
                cnt = ctypes.c_longlong(0)
                _lib.call("bbw_ops_get", h, nm.encode(), dt, None, ctypes.byref(cnt))
                a = np.empty(cnt.value, dtype=np_dt)
                _lib.call("bbw_ops_get", h, nm.encode(), dt, _lib.ptr(a), ctypes.byref(cnt))
                out[nm + suffix] = a
    finally:
        _lib.lib().bbw_ops_free(h)
    sz = out["sizes"]
    out.update(N=int(sz[0]), Np=int(sz[1]), Nfp=int(sz[2]), Nq=int(sz[3]), Nfq=int(sz[4]),
               EEL_nnz=int(sz[5]), L0_nnz=int(sz[6]))
    return out


def connect_and_geometry(N, VX, VY, VZ, EToV, ops):
    """EToE/EToF, vgeo/fgeo, node coordinates, vmapP and dt for one mesh."""
    K, Np = len(EToV), np_of(N)
    EToV = np.ascontiguousarray(EToV, np.int32)
    VX, VY, VZ = (np.ascontiguousarray(a, np.float64) for a in (VX, VY, VZ))
    EToE = np.empty((K, 4), np.int32)
    EToF = np.empty((K, 4), np.int32)
    _lib.call("bbw_mesh_connect", len(VX), K, _lib.ptr(EToV), _lib.ptr(EToE), _lib.ptr(EToF))
    vgeo = np.empty(K * 9, np.float32)
    fgeo = np.empty(K * 16, np.float32)
    x, y, z = (np.empty(K * Np, np.float64) for _ in range(3))
    dt = np.zeros(1, np.float32)
    r, s, t = ops["r64"], ops["s64"], ops["t64"]
    _lib.call("bbw_mesh_geometry", N, K, _lib.ptr(VX), _lib.ptr(VY), _lib.ptr(VZ), _lib.ptr(EToV),
              _lib.ptr(r), _lib.ptr(s), _lib.ptr(t), _lib.ptr(vgeo), _lib.ptr(fgeo), _lib.ptr(x),
              _lib.ptr(y), _lib.ptr(z), _lib.ptr(dt))
    vmapP = np.empty(K * 4 * nfp_of(N), np.int32)
    _lib.call("bbw_mesh_vmapP", N, K, _lib.ptr(EToE), _lib.ptr(EToF), _lib.ptr(ops["Fmask"]),
              _lib.ptr(x), _lib.ptr(y), _lib.ptr(z), _lib.ptr(vmapP))
    return dict(EToE=EToE, EToF=EToF, vgeo=vgeo, fgeo=fgeo, x=x.reshape(K, Np),
                y=y.reshape(K, Np), z=z.reshape(K, Np), vmapP=vmapP, dt_ref=float(dt[0]))


# ---------------------------------------------------------------- fields
def c2_sine(x, y, z):
    """1 + 0.5 sin(pi x) sin(pi y) sin(pi z)."""
    return 1.0 + 0.5 * np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)


def c2_one(x, y, z):
    return np.ones_like(x)


def gaussian_pulse(x, y, z, t=0.0, a=50.0):
    return np.exp(-a * (x * x + y * y + z * z))


def cavity_mode(x, y, z, t=0.0):
    """cos(pi x) cos(pi y) cos(pi z) cos(sqrt(3) pi t): exact for the p = 0
    wall on [-0.5, 0.5]^3 (cpp/main_subelem.cpp:3-5)."""
    return np.cos(np.pi * x) * np.cos(np.pi * y) * np.cos(np.pi * z) * np.cos(np.sqrt(3) * np.pi * t)


@dataclass
class Problem:
    """Everything the time step consumes, in the reference's layouts."""
    N: int
    K: int
    variant: str
    ops: dict
    mesh: dict
    c2q: np.ndarray          # [K][Nq] float32
    Q0: np.ndarray           # [K][4][Np] float32 (nodal values or BB coefficients)
    dt: float
    extra: dict = field(default_factory=dict)

    @property
    def Np(self):
        return np_of(self.N)

    @property
    def Nq(self):
        return self.ops["Nq"]

    def Vq(self):
        return self.ops["Vq_" + self.variant]

    def Pq(self):
        return self.ops["Pq_" + self.variant]

    def cubature_xyz(self):
        """Cubature point coordinates [K][Nq] (FP64): nodal interpolation of
        x, y, z, as InitWADG_subelem does (cpp/src/WaveOKL3d.cpp:465-476)."""
        Vq = self.ops["Vq_nodal64"].reshape(self.Np, self.Nq).T  # column-major -> [Nq][Np]
        m = self.mesh
        return m["x"] @ Vq.T, m["y"] @ Vq.T, m["z"] @ Vq.T

    def to_nodal(self, Q):
        """BB coefficients -> nodal values (WaveGetData3d, cpp/src/WaveOKL3d.cpp:2538-2556)."""
        if self.variant == "nodal":
            return Q
        VB = self.ops["VB64"].reshape(self.Np, self.Np).T
        Qr = np.asarray(Q, np.float64).reshape(self.K, 4, self.Np)
        return np.einsum("ij,kfj->kfi", VB, Qr).astype(Q.dtype).ravel()

    def from_nodal(self, Qn):
        if self.variant == "nodal":
            return Qn
        iVB = self.ops["invVB64"].reshape(self.Np, self.Np).T
        Qr = np.asarray(Qn, np.float64).reshape(self.K, 4, self.Np)
        return np.einsum("ij,kfj->kfi", iVB, Qr).astype(np.float32).ravel()

    def geo_dict(self):
        """Arrays the oracle / kernel-level entry points take."""
        return dict(vgeo=self.mesh["vgeo"], fgeo=self.mesh["fgeo"], vmapP=self.mesh["vmapP"],
                    c2q=self.c2q.ravel(), Jq=np.ones(self.K * self.Nq, np.float32))

    def ops_dict(self):
        o = dict(self.ops)
        o["Vq"], o["Pq"] = self.Vq(), self.Pq()
        return o

    def l2_error(self, Q, t, exact):
        """FP64 L2 error of p at the volume cubature points against exact(x,y,z,t),
        as compute_error (cpp/src/WaveOKL3d.cpp:1683-1726) with the relative
        error taken as |e| / |u| (the reference's :1722 takes a second root)."""
        Qn = np.asarray(self.to_nodal(np.asarray(Q)), np.float64).reshape(self.K, 4, self.Np)
        Vq = self.ops["Vq_nodal64"].reshape(self.Np, self.Nq).T
        pq = Qn[:, 0, :] @ Vq.T
        xq, yq, zq = self.cubature_xyz()
        uex = exact(xq, yq, zq, t)
        J = self.extra["J"]
        w = self.ops["wq64"][None, :] * J[:, None]
        err = np.sqrt(np.sum((pq - uex) ** 2 * w))
        nrm = np.sqrt(np.sum(uex ** 2 * w))
        return err, err / nrm


def gaussian_source(prob, x0, a=100.0, xyz=None):
    """Smoothed point source of acous_elas_cpp/src/WaveOKL3d.cpp:176-186 and
    :226-228: exp(-a^2 |x - x0|^2) at the cubature points, normalised to max 1
    over the mesh, projected with Pq (L2 projection onto the element basis).
    Returns the dense [K][Np] float32 array the reference uploads (c_fsrc)."""
    xq, yq, zq = prob.cubature_xyz() if xyz is None else xyz
    r2 = (xq - x0[0]) ** 2 + (yq - x0[1]) ** 2 + (zq - x0[2]) ** 2
    f = np.exp(-a * a * r2)
    f *= 1.0 / np.abs(f).max()
    Pq = prob.ops["Pq_%s64" % prob.variant].reshape(prob.Nq, prob.Np).T  # [Np][Nq]
    return np.ascontiguousarray(f @ Pq.T, np.float32)


def source_entries(fsrc, shot=0, rtol=1e-9):
    """Sparse (shot, elem, vec) entries of a dense [K][Np] source: the
    elements whose coefficients reach rtol * max|fsrc| (the rest are below
    FP32 resolution of the step and contribute nothing)."""
    f = np.asarray(fsrc, np.float32)
    m = np.abs(f).max(axis=1)
    elem = np.nonzero(m >= rtol * m.max())[0].astype(np.int32)
    return np.full(len(elem), shot, np.int32), elem, np.ascontiguousarray(f[elem])


def locate_points(prob, pts):
    """Element and reference coordinates (r, s, t) of each physical point
    (first containing element; tolerance 1e-10 in barycentric coordinates).
    The affine map is x = -(1+r+s+t)/2 v1 + (1+r)/2 v2 + (1+s)/2 v3 + (1+t)/2 v4
    (cpp/src/StartUp3d.cpp:556-559, vertex order of EToV)."""
    (VX, VY, VZ), EToV = prob.extra["VX"], np.asarray(prob.extra["EToV"])
    V = np.stack([np.asarray(VX)[EToV], np.asarray(VY)[EToV], np.asarray(VZ)[EToV]], -1)
    A = np.stack([V[:, 1] - V[:, 0], V[:, 2] - V[:, 0], V[:, 3] - V[:, 0]], -1)  # [K][3][3]
    Ainv = np.linalg.inv(A)
    pts = np.atleast_2d(np.asarray(pts, np.float64))
    elem = np.empty(len(pts), np.int32)
    rst = np.empty((len(pts), 3))
    for i, x in enumerate(pts):
        lam = np.einsum("kij,kj->ki", Ainv, x[None, :] - V[:, 0])  # barycentric 1..3
        ok = (lam >= -1e-10).all(1) & (lam.sum(1) <= 1 + 1e-10)
        hit = np.nonzero(ok)[0]
        if len(hit) == 0:
            raise ValueError("point %r is outside the mesh" % (tuple(x),))
        k = hit[0]
        elem[i] = k
        rst[i] = 2.0 * lam[k] - 1.0
    return elem, rst


def basis_eval(N, variant, rst):
    """phi_n at reference points: [npts][Np] FP64 (nodal Lagrange or Bernstein)."""
    rst = np.ascontiguousarray(np.atleast_2d(rst), np.float64)
    r, s, t = (np.ascontiguousarray(rst[:, i]) for i in range(3))
    out = np.empty((len(rst), np_of(N)), np.float64)
    _lib.call("bbw_basis_eval", N, 0 if variant == "nodal" else 1, len(rst), _lib.ptr(r),
              _lib.ptr(s), _lib.ptr(t), _lib.ptr(out))
    return out


def receiver_weights(prob, pts):
    """Receivers at physical points: (elem[R], w[R][Np]) with
    p(x) = sum_n w[n] Q[elem][p][n] for the problem's basis."""
    elem, rst = locate_points(prob, pts)
    return elem, np.ascontiguousarray(basis_eval(prob.N, prob.variant, rst), np.float32)


def _jacobians(VX, VY, VZ, EToV):
    x, y, z = VX[EToV], VY[EToV], VZ[EToV]
    d = [np.stack([x[:, m] - x[:, 0], y[:, m] - y[:, 0], z[:, m] - z[:, 0]], 1) / 2 for m in (1, 2, 3)]
    return np.einsum("ij,ij->i", d[0], np.cross(d[1], d[2]))


def make_problem(N, n=None, variant="nodal", c2="sine", ic="gauss", lo=-1.0, hi=1.0, mesh=None,
                 cubature=None, tri_cubature=None, ops=None, cfl=None, seed=0, c2_jitter=0.0):
    """Build a problem on the n^3 x 6 Kuhn box [lo,hi]^3 (or ``mesh`` =
    (VX,VY,VZ,EToV) / a Gmsh 2.2 path).

    c2: 'sine' | 'one' | callable(x,y,z); c2_jitter adds a per-element
    c2_jitter * U(0,1) drawn with ``seed``.  ic: 'gauss' | 'cavity' |
    callable(x,y,z,t).  dt is the reference's 0.25/((N+1)^2 max Fscale) or,
    with ``cfl``, cfl/((N+1)^2 max Fscale sqrt(max c2)).
    """
    if ops is None:
        ops = build_operators(N, cubature, tri_cubature)
    if mesh is None:
        VX, VY, VZ, EToV = kuhn_box(n, lo, hi)
    elif isinstance(mesh, str):
        VX, VY, VZ, EToV = read_gmsh22(mesh)
    else:
        VX, VY, VZ, EToV = mesh
    K = len(EToV)
    m = connect_and_geometry(N, VX, VY, VZ, EToV, ops)
    prob = Problem(N=N, K=K, variant=variant, ops=ops, mesh=m, c2q=None, Q0=None, dt=m["dt_ref"])
    prob.extra["J"] = _jacobians(np.asarray(VX), np.asarray(VY), np.asarray(VZ), np.asarray(EToV))
    prob.extra["VX"], prob.extra["EToV"] = (VX, VY, VZ), EToV
    xq, yq, zq = prob.cubature_xyz()
    f = {"sine": c2_sine, "one": c2_one}.get(c2, c2) if isinstance(c2, str) else c2
    c2v = f(xq, yq, zq)
    if c2_jitter:
        rng = np.random.default_rng(seed)
        c2v = c2v + c2_jitter * rng.random(K)[:, None]
    prob.c2q = np.ascontiguousarray(c2v, np.float32)
    g = {"gauss": gaussian_pulse, "cavity": cavity_mode}.get(ic, ic) if isinstance(ic, str) else ic
    Np = np_of(N)
    Qn = np.zeros((K, 4, Np), np.float32)
    Qn[:, 0, :] = g(m["x"], m["y"], m["z"], 0.0)
    prob.Q0 = prob.from_nodal(Qn.ravel()) if variant == "bb" else Qn.ravel()
    if cfl is not None:
        fmax = float(m["fgeo"].reshape(K, 4, 4)[:, :, 0].max())
        prob.dt = float(np.float32(cfl / ((N + 1) ** 2 * fmax * np.sqrt(float(prob.c2q.max())))))
    return prob
