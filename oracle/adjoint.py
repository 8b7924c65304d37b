"""FP64 restatement of the forward step and its discrete adjoint (numpy).

ORACLE - TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the
GPU adjoint (bbw_forward / bbw_backward); never by the product path.

Forward (per LSRK45 stage, cpp/src/WaveOKL3d.cpp:2050-2106):
    rhs  = S(Q)                   rk_volume + rk_surface
                                  (cpp/okl/WaveKernels.okl:44-153, 156-260)
    rhs_p <- Pq diag(c2q) Vq rhs_p  (+ ftime fsrc)   rk_update_WADG
                                  (cpp/okl/WaveKernelsWADG.okl:1760-1887;
                                  J = 1, velocity rows unchanged; source as
                                  acous_elas_cpp/okl/ElasKernelsWADG.okl:400-403)
    res  = a res + dt rhs;  Q = Q + b res
and receivers trace[r][n] = w_r . Q_p(elem_r) after step n.  The adjoint
reverses each stage exactly (see bbwadg_b200/csrc/kernels_adj.cu for the
formulas); the loss is any function of the traces, given its gradient.

Operators are dense FP64 in the reference's column-major layouts.
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
RK4C = (0.0,
        1432997174477.0 / 9575080441755.0,
        2526269341429.0 / 6820363962896.0,
        2006345519317.0 / 3224310063776.0,
        2802321613138.0 / 2924317926251.0)


def _cm(a, rows, cols):
    """Column-major flat array -> [rows][cols] matrix."""
    return np.asarray(a, np.float64).reshape(cols, rows).T


def face_pairs(K, Np, Nfp, Fmask, vmapP):
    """mapP[k][m] = k2*4Nfp + m2 (matching face node), -1 on the boundary."""
    NF = 4 * Nfp
    vm = np.asarray(vmapP).reshape(K, NF)
    Fm = np.asarray(Fmask)
    k2 = vm // (4 * Np)
    node = vm % (4 * Np)
    mapP = -np.ones((K, NF), np.int64)
    for k in range(K):
        for f in range(4):
            sl = slice(f * Nfp, (f + 1) * Nfp)
            kk = k2[k, sl][0]
            if kk == k and (node[k, sl] == Fm[sl]).all():
                continue
            f2 = [g for g in range(4) if k2[kk, g * Nfp] == k][0]
            inv = {int(Fm[f2 * Nfp + j]): j for j in range(Nfp)}
            for i in range(Nfp):
                j = inv[int(node[k, f * Nfp + i])]
                assert vm[kk, f2 * Nfp + j] == k * 4 * Np + Fm[f * Nfp + i]
                mapP[k, f * Nfp + i] = kk * NF + f2 * Nfp + j
    return mapP


class AdjointOracle:
    """Dense FP64 forward / adjoint for small meshes.

    ops: D = (Dr, Ds, Dt) [Np x Np] column-major, LIFT [Np x 4Nfp], Vq
    [Nq x Np], Pq [Np x Nq] (column-major, the basis of the state), Fmask.
    geo: vgeo [K][9], fgeo [K][4][4], vmapP [K][4Nfp], c2q [K][Nq]."""

    def __init__(self, N, K, D, LIFT, Vq, Pq, Fmask, vgeo, fgeo, vmapP, c2q, bc=0):
        self.N, self.K, self.bc = N, K, bc
        self.Np = Np = (N + 1) * (N + 2) * (N + 3) // 6
        self.Nfp = Nfp = (N + 1) * (N + 2) // 2
        NF = 4 * Nfp
        self.Nq = Nq = np.asarray(Vq).size // Np
        self.D = [_cm(d, Np, Np) for d in D]
        self.LIFT = _cm(LIFT, Np, NF)
        self.Vq, self.Pq = _cm(Vq, Nq, Np), _cm(Pq, Np, Nq)
        self.Fmask = np.asarray(Fmask, np.int64)
        self.G = np.asarray(vgeo, np.float64).reshape(K, 9)
        fg = np.asarray(fgeo, np.float64).reshape(K, 4, 4)
        f_of_m = np.arange(NF) // Nfp
        self.Fs, self.nrm = fg[:, f_of_m, 0], fg[:, f_of_m, 1:4]  # [K][NF], [K][NF][3]
        self.vmapP = np.asarray(vmapP, np.int64).reshape(K, NF)
        own = np.arange(K)[:, None] * 4 * Np + self.Fmask[None, :]
        self.bnd = self.vmapP == own
        self.mapP = face_pairs(K, Np, Nfp, self.Fmask, self.vmapP)
        self.c2q = np.asarray(c2q, np.float64).reshape(K, Nq)

    # ---- forward pieces
    def _vol(self, Q, D):
        G = self.G
        p, u, v, w = Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3]
        U = [u * G[:, 3 * d, None] + v * G[:, 3 * d + 1, None] + w * G[:, 3 * d + 2, None]
             for d in range(3)]
        dp = [p @ D[d].T for d in range(3)]
        out = np.empty_like(Q)
        out[:, 0] = -(U[0] @ D[0].T + U[1] @ D[1].T + U[2] @ D[2].T)
        for c in range(3):
            out[:, 1 + c] = -(G[:, c, None] * dp[0] + G[:, 3 + c, None] * dp[1] +
                              G[:, 6 + c, None] * dp[2])
        return out

    def S(self, Q):
        """rk_volume + rk_surface (raw rhs)."""
        K, Np = self.K, self.Np
        out = self._vol(Q, self.D)
        flat = Q.reshape(-1)
        Fm = self.Fmask
        pM, UM = Q[:, 0, Fm], np.stack([Q[:, c, Fm] for c in (1, 2, 3)], -1)
        pP = flat[self.vmapP]
        UP = np.stack([flat[self.vmapP + c * Np] for c in (1, 2, 3)], -1)
        n = self.nrm
        pjump = pP - pM
        Unjump = ((UP - UM) * n).sum(-1)
        if self.bc == 0:
            pjump = np.where(self.bnd, -2 * pM, pjump)
            Unjump = np.where(self.bnd, 0.0, Unjump)
        else:
            pjump = np.where(self.bnd, 0.0, pjump)
            Unjump = np.where(self.bnd, -2 * (UM * n).sum(-1), Unjump)
        pflux = .5 * (pjump - Unjump) * self.Fs
        out[:, 0] += pflux @ self.LIFT.T
        for c in range(3):
            out[:, 1 + c] -= (pflux * n[..., c]) @ self.LIFT.T
        return out

    def A(self, Q):
        r = self.S(Q)
        r[:, 0] = ((r[:, 0] @ self.Vq.T) * self.c2q) @ self.Pq.T
        return r

    def forward(self, Q0, dt, nsteps, rec=None, src=None, t0=0.0):
        """Returns (Q_final, traces [R][nsteps], step-start states)."""
        Q = np.asarray(Q0, np.float64).reshape(self.K, 4, self.Np).copy()
        res = np.zeros_like(Q)
        states, traces = [], []
        t = t0
        for n in range(nsteps):
            states.append(Q.copy())
            for i in range(5):
                rhs = self.A(Q)
                if src is not None:
                    ts = t + (RK4C[i] * dt if src.get("stage_times") else 0.0)
                    a = np.pi * src["f0"] * (ts - src["tR"])
                    rhs[:, 0] += src["amp"] * (1 - 2 * a * a) * np.exp(-a * a) * src["fsrc"]
                res = RK4A[i] * res + dt * rhs
                Q = Q + RK4B[i] * res
            t += dt
            if rec is not None:
                el, w = rec
                traces.append((np.asarray(w, np.float64) * Q[np.asarray(el), 0]).sum(-1))
        tr = np.array(traces).T if rec is not None else None
        return Q, tr, states

    # ---- adjoint pieces
    def S_T(self, z):
        K, Np, Nfp = self.K, self.Np, self.Nfp
        out = self._vol(z, [d.T for d in self.D])
        n = self.nrm
        Wf = z[:, 0][:, None, :] - np.einsum("kmc,kcn->kmn", n, z[:, 1:4])  # [K][NF][Np]
        sig = .5 * self.Fs * np.einsum("kmn,nm->km", Wf, self.LIFT)
        sflat = sig.reshape(-1)
        s2 = np.where(self.mapP >= 0, sflat[np.maximum(self.mapP, 0)], 0.0)
        k2 = np.maximum(self.mapP, 0) // (4 * Nfp)
        m2 = np.maximum(self.mapP, 0) % (4 * Nfp)
        n2 = n[k2, m2]
        if self.bc == 0:
            dp = np.where(self.bnd, -2 * sig, s2 - sig)
            dU = np.where(self.bnd[..., None], 0.0, n * sig[..., None] - n2 * s2[..., None])
        else:
            dp = np.where(self.bnd, 0.0, s2 - sig)
            dU = np.where(self.bnd[..., None], 2 * n * sig[..., None],
                          n * sig[..., None] - n2 * s2[..., None])
        kk = np.repeat(np.arange(K), 4 * Nfp)
        nodes = np.tile(self.Fmask, K)
        np.add.at(out[:, 0], (kk, nodes), dp.reshape(-1))
        for c in range(3):
            np.add.at(out[:, 1 + c], (kk, nodes), dU[..., c].reshape(-1))
        return out

    def backward(self, dt, nsteps, states, g, rec, src=None, t0=0.0):
        """g = dL/dtraces [R][nsteps]; returns (dL/dc2q [K][Nq], dL/dQ0)."""
        K, Np = self.K, self.Np
        el, w = np.asarray(rec[0]), np.asarray(rec[1], np.float64)
        lamQ = np.zeros((K, 4, Np))
        lamR = np.zeros_like(lamQ)
        grad = np.zeros((K, self.Nq))
        for n in range(nsteps - 1, -1, -1):
            for r in range(len(el)):
                lamQ[el[r], 0] += g[r, n] * w[r]
            # stage inputs of step n
            Q = states[n].copy()
            res = np.zeros_like(Q)
            ins = []
            t = t0 + n * dt
            for i in range(5):
                ins.append(Q.copy())
                rhs = self.A(Q)
                if src is not None:
                    ts = t + (RK4C[i] * dt if src.get("stage_times") else 0.0)
                    a = np.pi * src["f0"] * (ts - src["tR"])
                    rhs[:, 0] += src["amp"] * (1 - 2 * a * a) * np.exp(-a * a) * src["fsrc"]
                res = RK4A[i] * res + dt * rhs
                Q = Q + RK4B[i] * res
            for i in range(4, -1, -1):
                mu = lamR + RK4B[i] * lamQ
                tq = mu[:, 0] @ self.Pq                       # Pq^T mu_p
                rp = self.S(ins[i])[:, 0]
                grad += dt * tq * (rp @ self.Vq.T)
                z = mu.copy()
                z[:, 0] = (self.c2q * tq) @ self.Vq
                lamQ = lamQ + dt * self.S_T(z)
                lamR = RK4A[i] * mu
        return grad, lamQ
