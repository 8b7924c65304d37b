"""Curvilinear WADG path: setup and solver.

``make_curved_problem`` plays the role of the reference's curved setup
sequence (cpp/main.cpp:58-99 with GORDON_HALL=1): connectivity and affine
geometry (FacePair3d, StartUp3d, WaveInitOCCA3d), Gordon-Hall curving of the
elements that touch the unit sphere (GordonHallSphere), geometric factors at
the cubature points (InitQuadratureArrays) and the arrays InitWADG_curved
uploads (cpp/src/WaveOKL3d.cpp:164-417), in the reference's layouts.
``CurvedSolver`` owns a native ``bbw_curved`` handle and runs the
reference's stage RK_step_WADG (cpp/src/WaveOKL3d.cpp:2111-2185) on the GPU.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .mesh import kuhn_ball, read_gmsh22
from .problem import build_operators, connect_and_geometry, np_of, nfp_of


def bessel_mode(x, y, z, t=0.0):
    """sin(pi r)/(pi r) cos(pi t): the reference's exact solution on the
    unit ball with a pressure-release wall (cpp/main.cpp:10-15)."""
    r = np.sqrt(x * x + y * y + z * z)
    with np.errstate(invalid="ignore", divide="ignore"):
        v = np.where(r < 1e-10, 1.0, np.sin(np.pi * r) / (np.pi * np.where(r < 1e-10, 1, r)))
    return v * np.cos(np.pi * t)


@dataclass
class CurvedProblem:
    """Arrays of the curvilinear path (FP32 in kernel layouts unless noted)."""
    N: int
    K: int
    Nq: int
    Nfq: int
    ops: dict
    mesh: dict                 # affine: vgeo fgeo vmapP EToE EToF; FP64 x y z (curved)
    curved: np.ndarray         # [K] 1 = curved element
    KlistCurved: np.ndarray
    KlistPlanar: np.ndarray
    vgeoq: np.ndarray          # [K][9][Nq]
    Jq: np.ndarray             # [K][Nq]
    fgeoq: np.ndarray          # [K][4][4][Nfq]
    Jplanar: np.ndarray        # [K]
    c2q: np.ndarray            # [K][Nq]
    Q0: np.ndarray             # [K][4][Np]
    dt: float
    geo64: dict = field(default_factory=dict)  # FP64 vgeoq, Jq, fgeoq

    @property
    def Np(self):
        return np_of(self.N)

    @property
    def Nfp(self):
        return nfp_of(self.N)

    def cubature_xyz(self):
        """Volume cubature point coordinates [K][Nq] of the curved map (FP64)."""
        Vq = self.ops["Vq_nodal64"].reshape(self.Np, self.Nq).T
        m = self.mesh
        return m["x"] @ Vq.T, m["y"] @ Vq.T, m["z"] @ Vq.T

    def volume(self):
        """Integral of 1 over the mesh (4 pi / 3 for the curved unit ball)."""
        return float((self.geo64["Jq"] @ self.ops["wq64"]).sum())

    def desc_arrays(self):
        """The arrays bbw_curved_desc points to, keyed by field name."""
        o = self.ops
        d = dict(KlistCurved=self.KlistCurved, KlistPlanar=self.KlistPlanar,
                 vgeo=self.mesh["vgeo"], fgeo=self.mesh["fgeo"], Jplanar=self.Jplanar,
                 Fmask=o["Fmask"], vmapP=self.mesh["vmapP"], vgeoq=self.vgeoq, Jq=self.Jq,
                 fgeoq=self.fgeoq, Jq_reduced=self.Jq, c2q=self.c2q, Dr=o["Dr"], Ds=o["Ds"],
                 Dt=o["Dt"], LIFT=o["LIFT"], Vq=o["Vq_nodal"], Vrq=o["Vrq"], Vsq=o["Vsq"],
                 Vtq=o["Vtq"], Pq=o["Pq_nodal"], Prq=o["Prq"], Psq=o["Psq"], Ptq=o["Ptq"],
                 VfqFace=o["VfqFace"], Pfq=o["Pfq"], Vq_reduced=o["Vq_nodal"],
                 Pq_reduced=o["Pq_nodal"])
        return {k: np.ascontiguousarray(v) for k, v in d.items()}


def curve_mesh(N, K, EToF, x, y, z):
    """Gordon-Hall curving in place (bbw_gordon_hall_sphere); returns the
    per-element curved flags."""
    curved = np.zeros(K, np.int32)
    E = np.ascontiguousarray(EToF, np.int32)
    _lib.call("bbw_gordon_hall_sphere", N, K, _lib.ptr(E), _lib.ptr(x), _lib.ptr(y), _lib.ptr(z),
              _lib.ptr(curved))
    return curved


def curved_geometry(N, K, x, y, z, ops):
    """FP64 vgeoq [K][9][Nq], Jq [K][Nq], fgeoq [K][4][4][Nfq] (bbw_curved_geometry)."""
    Nq, Nfq = ops["Nq"], ops["Nfq"]
    cub = np.ascontiguousarray(np.concatenate([ops["rq64"], ops["sq64"], ops["tq64"]]))
    tri = np.ascontiguousarray(np.concatenate([ops["rfq64"], ops["sfq64"]]))
    vgeoq = np.empty(K * 9 * Nq)
    Jq = np.empty(K * Nq)
    fgeoq = np.empty(K * 16 * Nfq)
    _lib.call("bbw_curved_geometry", N, K, _lib.ptr(x), _lib.ptr(y), _lib.ptr(z), Nq,
              _lib.ptr(cub), Nfq, _lib.ptr(tri), _lib.ptr(vgeoq), _lib.ptr(Jq), _lib.ptr(fgeoq))
    return vgeoq, Jq, fgeoq


def make_curved_problem(N, n=None, mesh=None, cubature=None, tri_cubature=None, ops=None,
                        c2=None, ic="bessel", cfl=None):
    """Curved unit-ball problem on kuhn_ball(n) (or ``mesh`` = (VX,VY,VZ,EToV)
    / a Gmsh 2.2 path).  c2: None (c^2 = 1, as InitWADG_curved sets) or
    callable(x,y,z) at the cubature points.  ic: 'bessel' | callable(x,y,z,t)
    for p at the (curved) nodes; velocities start at zero.  dt is the
    reference's 0.25/((N+1)^2 max Fscale) on the affine mesh or, with cfl,
    cfl/((N+1)^2 max Fscale sqrt(max c^2))."""
    if ops is None:
        ops = build_operators(N, cubature, tri_cubature)
    if mesh is None:
        VX, VY, VZ, EToV = kuhn_ball(n)
    elif isinstance(mesh, str):
        VX, VY, VZ, EToV = read_gmsh22(mesh)
    else:
        VX, VY, VZ, EToV = mesh
    K, Np, Nq, Nfq = len(EToV), np_of(N), ops["Nq"], ops["Nfq"]
    m = connect_and_geometry(N, VX, VY, VZ, EToV, ops)
    x, y, z = (np.ascontiguousarray(m[c], np.float64).ravel() for c in ("x", "y", "z"))
    curved = curve_mesh(N, K, m["EToF"], x, y, z)
    vgeoq, Jq, fgeoq = curved_geometry(N, K, x, y, z, ops)
    m["x"], m["y"], m["z"] = x.reshape(K, Np), y.reshape(K, Np), z.reshape(K, Np)
    Jaff = Jq.reshape(K, Nq)[:, 0]  # Jplanar(e) = Jq(0,e), cpp/src/WaveOKL3d.cpp:315-318
    prob = CurvedProblem(
        N=N, K=K, Nq=Nq, Nfq=Nfq, ops=ops, mesh=m, curved=curved,
        KlistCurved=np.nonzero(curved)[0].astype(np.int32),
        KlistPlanar=np.nonzero(curved == 0)[0].astype(np.int32),
        vgeoq=vgeoq.astype(np.float32), Jq=Jq.astype(np.float32), fgeoq=fgeoq.astype(np.float32),
        Jplanar=Jaff.astype(np.float32), c2q=None, Q0=None, dt=m["dt_ref"],
        geo64=dict(vgeoq=vgeoq.reshape(K, 9, Nq), Jq=Jq.reshape(K, Nq),
                   fgeoq=fgeoq.reshape(K, 4, 4, Nfq)))
    xq, yq, zq = prob.cubature_xyz()
    c2v = np.ones_like(xq) if c2 is None else c2(xq, yq, zq)
    prob.c2q = np.ascontiguousarray(c2v, np.float32)
    g = bessel_mode if ic == "bessel" else ic
    Q = np.zeros((K, 4, Np), np.float32)
    Q[:, 0, :] = g(m["x"], m["y"], m["z"], 0.0)
    prob.Q0 = Q.ravel()
    if cfl is not None:
        fmax = float(m["fgeo"].reshape(K, 4, 4)[:, :, 0].max())
        prob.dt = float(np.float32(cfl / ((N + 1) ** 2 * fmax * np.sqrt(float(prob.c2q.max())))))
    return prob


class CurvedSolver:
    """GPU solver of the curvilinear WADG path (native bbw_curved handle)."""

    def __init__(self, prob, device=0):
        self.prob = prob
        self.N, self.K, self.Np = prob.N, prob.K, prob.Np
        self._arrays = prob.desc_arrays()  # keep the host arrays alive for the call
        d = _lib.CurvedDesc(N=prob.N, K=prob.K, Nq=prob.Nq, Nfq=prob.Nfq, Nq_reduced=prob.Nq,
                            KCurved=len(prob.KlistCurved), KPlanar=len(prob.KlistPlanar))
        for k, v in self._arrays.items():
            setattr(d, k, _lib.ptr(v) if v.size else None)
        h = ctypes.c_void_p()
        _lib.call("bbw_curved_create", ctypes.byref(d), device, ctypes.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.call("bbw_curved_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_data(self, Q):
        Q = np.ascontiguousarray(Q, np.float32).ravel()
        if Q.size != self.K * 4 * self.Np:
            raise ValueError("state has %d entries, expected %d" % (Q.size, self.K * 4 * self.Np))
        _lib.call("bbw_curved_set_state", self._h, _lib.ptr(Q))

    def get_data(self):
        Q = np.empty(self.K * 4 * self.Np, np.float32)
        _lib.call("bbw_curved_get_state", self._h, _lib.ptr(Q))
        return Q

    def get_residual(self):
        r = np.empty(self.K * 4 * self.Np, np.float32)
        _lib.call("bbw_curved_get_residual", self._h, _lib.ptr(r))
        return r

    def rk_stage(self, fa, fb, fdt):
        _lib.call("bbw_curved_stage", self._h, float(fa), float(fb), float(fdt))

    def steps(self, dt, nsteps):
        _lib.call("bbw_curved_steps", self._h, float(dt), int(nsteps))

    def sync(self):
        _lib.call("bbw_curved_sync", self._h)

    def autotune(self, dt, stages=10):
        """Pick the fastest fused variant for the planar elements, timed
        inside whole curved stages (bbw_curved_autotune); returns its
        configuration code (0: no planar element)."""
        cfg = ctypes.c_int(0)
        _lib.call("bbw_curved_autotune", self._h, float(dt), int(stages), ctypes.byref(cfg))
        return cfg.value

    @property
    def stream(self):
        return _lib.lib().bbw_curved_stream(self._h)


__all__ = ["CurvedProblem", "CurvedSolver", "make_curved_problem", "curve_mesh",
           "curved_geometry", "bessel_mode"]
