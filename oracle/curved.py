"""FP64 restatement of the reference's curvilinear WADG stage (numpy).

ORACLE - TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the
GPU curvilinear path (bbw_rk_*_wadg_skew_combine, bbw_rk_*_planar,
bbw_curved_*); never by the product path.  It is pinned to the reference's
own kernels through the golden fixtures tests/golden/curved_ball4_N*.npz
(made by tests/golden/make_golden.py from oracle/_ref/ref_curved_N*).

Stage (cpp/src/WaveOKL3d.cpp:2111-2185, RK_step_WADG):
  curved elements: rk_volume_WADG_skew_combine (cpp/okl/WaveKernelsWADG.okl:
                   514-682) then rk_surface_WADG_skew_combine (:3024-3195)
  planar elements: rk_volume_planar (:2203-2318), rk_surface_planar
                   (:2320-2441)
  all elements:    rk_update_WADG (:1760-1887) with Jq and c2q
Operators are column-major flat arrays as uploaded by InitWADG_curved.
"""
import numpy as np

RK4A = (0.0,
        -567301805773.0 / 1357537059087.0,
        -2404267990393.0 / 2016746695238.0,
        -3550918686646.0 / 2091501179385.0,
        -1275806237668.0 / 842570457699.0)
RK4B = (1432997174477.0 / 9575080441755.0,
        5161836677717.0 / 13612068292357.0,
        1720146321549.0 / 2090206949498.0,
        3134564353537.0 / 4481467310338.0,
        2277821191437.0 / 14882151754819.0)


def _cm(a, rows, cols):
    return np.asarray(a, np.float64).reshape(cols, rows).T


class CurvedOracle:
    """arrays: the bbw_curved_desc fields (see CurvedProblem.desc_arrays)."""

    def __init__(self, N, K, Nq, Nfq, a):
        self.N, self.K, self.Nq, self.Nfq = N, K, Nq, Nfq
        self.Np = Np = (N + 1) * (N + 2) * (N + 3) // 6
        self.Nfp = Nfp = (N + 1) * (N + 2) // 2
        NF = 4 * Nfp
        f64 = lambda k: np.asarray(a[k], np.float64)  # noqa: E731
        self.KC = np.asarray(a["KlistCurved"], np.int64)
        self.KP = np.asarray(a["KlistPlanar"], np.int64)
        self.vgeo = f64("vgeo").reshape(K, 9)
        self.fgeo = f64("fgeo").reshape(K, 4, 4)
        self.Jpl = f64("Jplanar")
        self.Fmask = np.asarray(a["Fmask"], np.int64)
        self.vmapP = np.asarray(a["vmapP"], np.int64).reshape(K, NF)
        self.vgeoq = f64("vgeoq").reshape(K, 9, Nq)
        self.Jq = f64("Jq").reshape(K, Nq)
        self.fgeoq = f64("fgeoq").reshape(K, 4, 4, Nfq)
        Nr = np.asarray(a["Vq_reduced"]).size // Np
        self.Nr = Nr
        self.Jr = f64("Jq_reduced").reshape(K, Nr)
        self.c2q = f64("c2q").reshape(K, Nr)
        self.D = [_cm(a[k], Np, Np) for k in ("Dr", "Ds", "Dt")]
        self.LIFT = _cm(a["LIFT"], Np, NF)
        self.Vq, self.Vr, self.Vs, self.Vt = (_cm(a[k], Nq, Np) for k in ("Vq", "Vrq", "Vsq", "Vtq"))
        self.Pq, self.Pr, self.Ps, self.Pt = (_cm(a[k], Np, Nq) for k in ("Pq", "Prq", "Psq", "Ptq"))
        self.VfqFace = _cm(a["VfqFace"], Nfq, Nfp)
        self.Pfq = _cm(a["Pfq"], Np, 4 * Nfq)
        self.Vqr = _cm(a["Vq_reduced"], Nr, Np)
        self.Pqr = _cm(a["Pq_reduced"], Np, Nr)

    # Q, rhs: [K][4][Np] FP64
    def volume_skew(self, Q, rhs):
        L = self.KC
        if not len(L):
            return
        q = Q[L]
        p, U = q[:, 0], q[:, 1:4]
        uq = U @ self.Vq.T                                      # [E][3][Nq]
        dr, ds, dt = p @ self.Vr.T, p @ self.Vs.T, p @ self.Vt.T
        g, J = self.vgeoq[L], self.Jq[L]
        rx, sx, tx, ry, sy, ty, rz, sz, tz = (g[:, c] for c in range(9))
        gx = (rx * dr + sx * ds + tx * dt) * J
        gy = (ry * dr + sy * ds + ty * dt) * J
        gz = (rz * dr + sz * ds + tz * dt) * J
        Ur = (uq[:, 0] * rx + uq[:, 1] * ry + uq[:, 2] * rz) * J
        Us = (uq[:, 0] * sx + uq[:, 1] * sy + uq[:, 2] * sz) * J
        Ut = (uq[:, 0] * tx + uq[:, 1] * ty + uq[:, 2] * tz) * J
        divU = (-Ur) @ self.Pr.T + (-Us) @ self.Ps.T + (-Ut) @ self.Pt.T
        rhs[L, 0] = -divU
        rhs[L, 1] = -(gx @ self.Pq.T)
        rhs[L, 2] = -(gy @ self.Pq.T)
        rhs[L, 3] = -(gz @ self.Pq.T)

    def _traces(self, Q, L):
        Np, NF = self.Np, 4 * self.Nfp
        flat = Q.reshape(-1)
        idM = L[:, None] * 4 * Np + self.Fmask[None, :]
        idP = self.vmapP[L]
        M = np.stack([flat[idM + c * Np] for c in range(4)], 1)  # [E][4][NF]
        P = np.stack([flat[idP + c * Np] for c in range(4)], 1)
        return M, P, idM == idP

    def surface_skew(self, Q, rhs):
        L = self.KC
        if not len(L):
            return
        Nfp, Nfq = self.Nfp, self.Nfq
        M, P, bnd = self._traces(Q, L)
        dp = np.where(bnd, -2 * M[:, 0], P[:, 0] - M[:, 0])
        du = [np.where(bnd, 0.0, P[:, c] - M[:, c]) for c in (1, 2, 3)]
        av = [np.where(bnd, M[:, c], .5 * (P[:, c] + M[:, c])) for c in (1, 2)]
        av.append(np.where(bnd, P[:, 3], .5 * (P[:, 3] + M[:, 3])))
        E = len(L)

        def toq(v):  # [E][4Nfp] -> [E][4][Nfq]
            return v.reshape(E, 4, Nfp) @ self.VfqFace.T

        dpq, duq, avq = toq(dp), [toq(v) for v in du], [toq(v) for v in av]
        g = self.fgeoq[L]
        nx, ny, nz, sJ = g[:, :, 0], g[:, :, 1], g[:, :, 2], g[:, :, 3]
        Unjump = duq[0] * nx + duq[1] * ny + duq[2] * nz
        Unavg = avq[0] * nx + avq[1] * ny + avq[2] * nz
        pflux = -(Unavg - .5 * dpq) * sJ
        Uflux = -.5 * (dpq - Unjump) * sJ
        fl = [pflux, Uflux * nx, Uflux * ny, Uflux * nz]
        for c in range(4):
            rhs[L, c] += fl[c].reshape(E, 4 * Nfq) @ self.Pfq.T

    def volume_planar(self, Q, rhs):
        L = self.KP
        if not len(L):
            return
        G, J = self.vgeo[L], self.Jpl[L][:, None]
        q = Q[L]
        p, u, v, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
        Us = [u * G[:, 3 * d, None] + v * G[:, 3 * d + 1, None] + w * G[:, 3 * d + 2, None]
              for d in range(3)]
        dp = [p @ self.D[d].T for d in range(3)]
        divU = Us[0] @ self.D[0].T + Us[1] @ self.D[1].T + Us[2] @ self.D[2].T
        rhs[L, 0] = -divU * J
        for c in range(3):
            rhs[L, 1 + c] = -(G[:, c, None] * dp[0] + G[:, 3 + c, None] * dp[1] +
                              G[:, 6 + c, None] * dp[2]) * J

    def surface_planar(self, Q, rhs):
        L = self.KP
        if not len(L):
            return
        Nfp = self.Nfp
        M, P, bnd = self._traces(Q, L)
        f_of_m = np.arange(4 * Nfp) // Nfp
        fg = self.fgeo[L][:, f_of_m]                            # [E][NF][4]
        Fs = fg[..., 0] * self.Jpl[L][:, None]
        n = fg[..., 1:4]
        pjump = np.where(bnd, -2 * M[:, 0], P[:, 0] - M[:, 0])
        Unjump = np.where(bnd, 0.0, ((P[:, 1:4] - M[:, 1:4]) * n.transpose(0, 2, 1)).sum(1))
        pflux = .5 * (pjump - Unjump) * Fs
        Uflux = .5 * (Unjump - pjump) * Fs
        rhs[L, 0] += pflux @ self.LIFT.T
        for c in range(3):
            rhs[L, 1 + c] += (Uflux * n[..., c]) @ self.LIFT.T

    def update(self, rhs, res, Q, fa, fb, fdt):
        rq = rhs @ self.Vqr.T                                   # [K][4][Nr]
        rq = rq / self.Jr[:, None, :]
        rq[:, 0] *= self.c2q
        r = rq @ self.Pqr.T
        res *= fa
        res += fdt * r
        Q += fb * res

    def rhs(self, Q):
        rhs = np.zeros_like(Q)
        self.volume_skew(Q, rhs)
        self.surface_skew(Q, rhs)
        self.volume_planar(Q, rhs)
        self.surface_planar(Q, rhs)
        return rhs

    def run(self, Q0, dt, stages, res=None):
        """`stages` stages of RK_step_WADG from Q0; returns (Q, res)."""
        Q = np.asarray(Q0, np.float64).reshape(self.K, 4, self.Np).copy()
        res = np.zeros_like(Q) if res is None else np.asarray(res, np.float64).reshape(Q.shape).copy()
        for s in range(stages):
            i = s % 5
            self.update(self.rhs(Q), res, Q, float(np.float32(RK4A[i])),
                        float(np.float32(RK4B[i])), float(np.float32(dt)))
        return Q.ravel(), res.ravel()
