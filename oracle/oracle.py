"""ctypes front end of the C restatement in oracle/wadg_oracle.c.

ORACLE - TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the
CPU-baseline leg of bench.py as the checker; never by the product path.

Arrays use the reference's layouts (see wadg_oracle_body.h).  ``dtype``
selects the FP32 restatement (reference arithmetic) or the FP64 one.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

# LSRK45 coefficients, cpp/src/StartUp3d.cpp:517-537
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


def ricker(t, f0, tR, amp):
    """acous_elas_cpp/src/WaveOKL3d.cpp:767-770: amp (1 - 2 a^2) exp(-a^2),
    a = pi f0 (t - tR)."""
    a = np.pi * f0 * (t - tR)
    return amp * (1.0 - 2.0 * a * a) * np.exp(-a * a)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)
        _LIB = ctypes.CDLL(path)
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _sfx(dtype):
    return "_f32" if np.dtype(dtype) == np.float32 else "_f64"


def _R(dtype, x):
    return (ctypes.c_float if np.dtype(dtype) == np.float32 else ctypes.c_double)(x)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Oracle:
    """Holds one operator set (nodal or BB) and advances states on the CPU."""

    def __init__(self, N, K, ops, geo, variant="nodal", bc=0, dtype=np.float32):
        self.N, self.K, self.variant, self.bc = N, K, variant, bc
        self.dtype = np.dtype(dtype)
        self.Np = (N + 1) * (N + 2) * (N + 3) // 6
        self.Nfp = (N + 1) * (N + 2) // 2
        d = self.dtype
        self.vgeo, self.fgeo = _c(geo["vgeo"], d), _c(geo["fgeo"], d)
        self.vmapP, self.Fmask = _i(geo["vmapP"]), _i(ops["Fmask"])
        self.c2q, self.Jq = _c(geo["c2q"], d), _c(geo["Jq"], d)
        self.Vq, self.Pq = _c(ops["Vq"], d), _c(ops["Pq"], d)
        self.Nq = self.Vq.size // self.Np
        # the restatement keeps per-element work arrays of fixed size
        if self.Np > lib().ora_maxnp() or self.Nq > lib().ora_maxnq():
            raise ValueError("oracle: Np = %d, Nq = %d exceed the compiled limits (%d, %d)"
                             % (self.Np, self.Nq, lib().ora_maxnp(), lib().ora_maxnq()))
        if variant == "nodal":
            self.Dr, self.Ds, self.Dt = (_c(ops[k], d) for k in ("Dr", "Ds", "Dt"))
            self.LIFT = _c(ops["LIFT"], d)
        else:
            self.D = [_i(ops["D_ids%d" % j]) for j in (1, 2, 3, 4)]
            self.Dvals4 = _c(ops["Dvals4"], d)
            self.EEL_ids, self.EEL_vals = _i(ops["EEL_ids"]), _c(ops["EEL_vals"], d)
            self.L0_ids, self.L0_vals = _i(ops["L0_ids"]), _c(ops["L0_vals"], d)
            self.EEL_nnz = self.EEL_ids.size // self.Np
            self.L0_nnz = self.L0_ids.size // self.Nfp

    # ---- single kernels (reference names) ----
    def rk_volume(self, Q, rhs):
        s = _sfx(self.dtype)
        if self.variant == "nodal":
            getattr(lib(), "ora_rk_volume" + s)(self.K, self.Np, _p(self.vgeo), _p(self.Dr),
                                                _p(self.Ds), _p(self.Dt), _p(Q), _p(rhs))
        else:
            getattr(lib(), "ora_rk_volume_bern" + s)(self.K, self.Np, _p(self.vgeo),
                                                     *[_p(x) for x in self.D], _p(self.Dvals4),
                                                     _p(Q), _p(rhs))

    def rk_surface(self, Q, rhs):
        s = _sfx(self.dtype)
        if self.variant == "nodal":
            getattr(lib(), "ora_rk_surface" + s)(self.K, self.Np, self.Nfp, self.bc, _p(self.fgeo),
                                                 _p(self.Fmask), _p(self.vmapP), _p(self.LIFT),
                                                 _p(Q), _p(rhs))
        else:
            getattr(lib(), "ora_rk_surface_bern" + s)(
                self.K, self.Np, self.Nfp, self.bc, _p(self.fgeo), _p(self.Fmask),
                _p(self.vmapP), self.EEL_nnz, _p(self.EEL_ids), _p(self.EEL_vals), self.L0_nnz,
                _p(self.L0_ids), _p(self.L0_vals), _p(Q), _p(rhs))

    def rk_update_wadg(self, fa, fb, fdt, rhs, res, Q):
        getattr(lib(), "ora_rk_update_wadg" + _sfx(self.dtype))(
            self.K, self.Np, self.Nq, _p(self.Vq), _p(self.Pq), _p(self.Jq), _p(self.c2q),
            _R(self.dtype, fa), _R(self.dtype, fb), _R(self.dtype, fdt), _p(rhs), _p(res), _p(Q))

    def rk_update_wadg_src(self, fa, fb, fdt, ftime, fsrc, rhs, res, Q):
        getattr(lib(), "ora_rk_update_wadg_src" + _sfx(self.dtype))(
            self.K, self.Np, self.Nq, _p(self.Vq), _p(self.Pq), _p(self.Jq), _p(self.c2q),
            _R(self.dtype, fa), _R(self.dtype, fb), _R(self.dtype, fdt), _R(self.dtype, ftime),
            _p(fsrc), _p(rhs), _p(res), _p(Q))

    def rk_update(self, fa, fb, fdt, rhs, res, Q):
        getattr(lib(), "ora_rk_update" + _sfx(self.dtype))(
            self.K, self.Np, _R(self.dtype, fa), _R(self.dtype, fb), _R(self.dtype, fdt),
            _p(rhs), _p(res), _p(Q))

    # ---- stage / step driver: RK_step_WADG_subelem + Wave_RK ----
    def run(self, Q, dt, nstages, res=None, source=None, receivers=None, t0=0.0):
        """Advance Q in place by ``nstages`` LSRK45 stages (stage s uses
        coefficient s % 5), as cpp/src/WaveOKL3d.cpp:2050-2106 does.  The
        FP32 family casts the coefficients to float like the reference.

        source = dict(fsrc=[K][Np] array, f0, tR, amp, stage_times): the
        acous_elas_cpp source term (WaveOKL3d.cpp:765-781), evaluated at the
        step start time (stage_times False, as the reference) or at the stage
        times.  receivers = (elem[R], w[R][Np]): p interpolated after every
        full step; returned as traces [R][nsteps] when given."""
        Q = np.ascontiguousarray(Q, dtype=self.dtype)
        res = np.zeros_like(Q) if res is None else res
        rhs = np.zeros_like(Q)
        fsrc = None if source is None else _c(source["fsrc"], self.dtype)
        traces = []
        t = t0
        for s in range(nstages):
            i = s % 5
            fa, fb = RK4A[i], RK4B[i]
            if self.dtype == np.float32:
                fa, fb, fdt = np.float32(fa), np.float32(fb), np.float32(dt)
            else:
                fdt = dt
            self.rk_volume(Q, rhs)
            self.rk_surface(Q, rhs)
            if fsrc is None:
                self.rk_update_wadg(fa, fb, fdt, rhs, res, Q)
            else:
                ts = t + (RK4C[i] * dt if source.get("stage_times") else 0.0)
                ftime = ricker(ts, source["f0"], source["tR"], source["amp"])
                self.rk_update_wadg_src(fa, fb, fdt, ftime, fsrc, rhs, res, Q)
            if i == 4:
                t += float(dt)
                if receivers is not None:
                    el, w = receivers
                    Qr = Q.reshape(self.K, 4, self.Np)
                    traces.append(np.einsum("rn,rn->r", np.asarray(w, np.float64),
                                            Qr[np.asarray(el), 0, :].astype(np.float64)))
        if receivers is not None:
            return Q, res, np.array(traces).T
        return Q, res
