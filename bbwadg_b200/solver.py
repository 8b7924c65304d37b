"""Host API mirroring the reference's solver entry points (cpp/include/fem.h:49-70).

    reference                                 here
    WaveInitOCCA3d + InitWADG_subelem         WaveSolver(problem)
    WaveSetData3d(Q)                          solver.set_data(Q)
    RK_step_WADG_subelem(mesh, rka, rkb, dt)  solver.rk_step(rka, rkb, dt)
    Wave_RK(mesh, FinalTime, dt, 1)           solver.wave_rk(final_time, dt)
    WaveGetData3d(mesh, Q)                    solver.get_data()   (raw coefficients)

All work runs in the native library on the GPU (one fused kernel per LSRK
stage); there is no CPU path.
"""
import ctypes

import numpy as np

from . import _lib
from .problem import np_of

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
        2802321613138.0 / 2924317926251.0,
        1.0)

VARIANTS = {"nodal": 0, "bb": 1}
PRECISIONS = {"fp32": 0, "f16x3": 1, "bf16x3": 2, "tf32": 3}
BCS = {"pressure_release": 0, "rigid": 1}


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def encode_config(warps, ops_in_smem, pipelined, tile=32):
    """Configuration code of a fused-stage variant (bbw_set_config)."""
    if tile not in (16, 32):
        raise ValueError("tile must be 16 or 32")
    return (int(warps) | (int(bool(ops_in_smem)) << 8) | (int(bool(pipelined)) << 9)
            | (int(tile == 16) << 10))


def decode_config(code):
    """Fields of a configuration code as bbw_autotune returns it."""
    return dict(warps=code & 255, ops_in_smem=bool(code >> 8 & 1),
                pipelined=bool(code >> 9 & 1), tile=16 if code >> 10 & 1 else 32, code=code)


class WaveSolver:
    """Fused-stage solver context for one mesh / operator set on the current GPU."""

    def __init__(self, problem=None, *, N=None, K=None, Nq=None, variant=None, ops=None,
                 vgeo=None, fgeo=None, vmapP=None, c2q=None, Jq=None, bc="pressure_release",
                 precision="fp32"):
        if problem is not None:
            N, K, Nq = problem.N, problem.K, problem.Nq
            variant = variant or problem.variant
            ops = problem.ops_dict() if ops is None else ops
            vgeo, fgeo = problem.mesh["vgeo"], problem.mesh["fgeo"]
            vmapP, c2q = problem.mesh["vmapP"], problem.c2q
        self.N, self.K, self.Nq, self.variant = N, K, Nq, variant
        self.Np = np_of(N)
        keep = {}

        def f(a):
            keep[id(a)] = a = _f32(a)
            return a.ctypes.data

        def i(a):
            keep[id(a)] = a = _i32(a)
            return a.ctypes.data

        md = _lib.MeshDesc(N=N, K=K, Nq=Nq, vgeo=f(vgeo), fgeo=f(fgeo), Fmask=i(ops["Fmask"]),
                           vmapP=i(vmapP), c2q=f(c2q), Jq=f(Jq) if Jq is not None else None)
        od = _lib.OpsDesc(Vq=f(ops["Vq"]), Pq=f(ops["Pq"]))
        if variant == "nodal":
            od.Dr, od.Ds, od.Dt, od.LIFT = f(ops["Dr"]), f(ops["Ds"]), f(ops["Dt"]), f(ops["LIFT"])
        else:
            od.D_ids1, od.D_ids2 = i(ops["D_ids1"]), i(ops["D_ids2"])
            od.D_ids3, od.D_ids4 = i(ops["D_ids3"]), i(ops["D_ids4"])
            od.Dvals4 = f(ops["Dvals4"])
            od.EEL_nnz = int(np.asarray(ops["EEL_ids"]).size // self.Np)
            od.L0_nnz = int(np.asarray(ops["L0_ids"]).size // ((N + 1) * (N + 2) // 2))
            od.EEL_ids, od.EEL_vals = i(ops["EEL_ids"]), f(ops["EEL_vals"])
            od.L0_ids, od.L0_vals = i(ops["L0_ids"]), f(ops["L0_vals"])
        h = ctypes.c_void_p()
        _lib.call("bbw_create_ex", ctypes.byref(md), ctypes.byref(od), VARIANTS[variant], BCS[bc],
                  PRECISIONS[precision], ctypes.byref(h))
        self.precision = precision
        self.S, self.R, self.max_steps = 1, 0, 0
        self._h = h
        del keep

    # ---- reference-named entry points
    @property
    def state_size(self):
        return self.S * self.K * 4 * self.Np

    def set_data(self, Q):
        """WaveSetData3d: host state [S][K][4][Np] -> device."""
        Q = _f32(Q)
        if Q.size != self.state_size:
            raise ValueError("state has %d values, expected %d" % (Q.size, self.state_size))
        _lib.call("bbw_set_state", self._h, Q.ctypes.data)

    def get_data(self, out=None):
        """WaveGetData3d (raw coefficients; BB -> nodal is Problem.to_nodal).
        ``out``: a contiguous float32 host array of the state's size to copy
        into (pinned memory makes the device-to-host copy direct)."""
        if out is None:
            out = np.empty(self.state_size, np.float32)
        elif (out.dtype != np.float32 or out.size != self.state_size
              or not out.flags["C_CONTIGUOUS"]):
            raise ValueError("out must be a contiguous float32 array of %d values"
                             % self.state_size)
        _lib.call("bbw_get_state", self._h, out.ctypes.data)
        return out

    def set_residual(self, r):
        r = _f32(r)
        if r.size != self.state_size:
            raise ValueError("residual has %d values, expected %d" % (r.size, self.state_size))
        _lib.call("bbw_set_residual", self._h, r.ctypes.data)

    def get_residual(self):
        r = np.empty(self.state_size, np.float32)
        _lib.call("bbw_get_residual", self._h, r.ctypes.data)
        return r

    def rk_step(self, rka, rkb, fdt):
        """RK_step_WADG_subelem: one fused LSRK stage (asynchronous)."""
        _lib.call("bbw_stage", self._h, float(rka), float(rkb), float(fdt))

    def steps(self, dt, nsteps):
        """nsteps LSRK45 steps of size dt (CUDA-graph replay; asynchronous)."""
        _lib.call("bbw_steps", self._h, float(dt), int(nsteps))

    def wave_rk(self, final_time, dt):
        """Wave_RK: steps of dt until final_time, last step shortened."""
        _lib.call("bbw_run", self._h, float(final_time), float(dt))

    def rk_stage(self, rka, rkb, fdt, c):
        """One fused stage with stage-time offset c (source time = clock + c fdt)."""
        _lib.call("bbw_stage_ex", self._h, float(rka), float(rkb), float(fdt), float(c))

    # ---- element decomposition (see decomp.py)
    def set_compute_range(self, Kc):
        """Advance elements [0, Kc) only; [Kc, K) are halo copies."""
        _lib.call("bbw_set_compute_range", self._h, int(Kc))

    def gather_elements(self, idx, buf):
        """buf[s][j] = state of element idx[j] in shot s (device int32 idx,
        device float32 buf of S * len(idx) * 4 * Np floats)."""
        _lib.call("bbw_gather_elements", self._h, int(idx.numel()), _lib.ptr(idx), _lib.ptr(buf))

    def scatter_elements(self, idx, buf):
        """State of element idx[j] in shot s = buf[s][j]."""
        _lib.call("bbw_scatter_elements", self._h, int(idx.numel()), _lib.ptr(idx), _lib.ptr(buf))

    def stage_part(self, fa, fb, dt, K0, K1):
        """Advance elements [K0, K1) into the next state (bbw_stage_part)."""
        _lib.call("bbw_stage_part", self._h, float(fa), float(fb), float(dt), int(K0), int(K1))

    def stage_commit(self):
        """Make the next state current (bbw_stage_commit)."""
        _lib.call("bbw_stage_commit", self._h)

    def move_elements(self, which, dir, idx, buf, stream=None):
        """Gather (dir 0) / scatter (dir 1) listed elements of the current
        (which 0) or next (which 1) state on a CUDA stream handle."""
        _lib.call("bbw_move_elements", self._h, int(which), int(dir), int(idx.numel()),
                  _lib.ptr(idx), _lib.ptr(buf), stream)

    def autotune(self, dt, stages=10):
        """Pick the fastest fused-stage variant for this mesh and batch;
        returns dict(warps, ops_in_smem, pipelined, tile, code)."""
        cfg = ctypes.c_int(0)
        _lib.call("bbw_autotune", self._h, float(dt), int(stages), ctypes.byref(cfg))
        return decode_config(cfg.value)

    def set_config(self, warps, ops_in_smem, pipelined, tile=32):
        """Pin a fused-stage variant (as returned by autotune); tile is the
        elements per tile, 32 or 16."""
        _lib.call("bbw_set_config", self._h, encode_config(warps, ops_in_smem, pipelined, tile))

    def set_grid_limit(self, max_ctas):
        """Cap the persistent stage kernels at max_ctas CTAs (0: one per SM)."""
        _lib.call("bbw_set_grid_limit", self._h, int(max_ctas))

    # ---- batched shots, sources, receivers
    def set_shots(self, S):
        """S independent shots per launch (state [S][K][4][Np], zeroed)."""
        _lib.call("bbw_set_shots", self._h, int(S))
        self.S = int(S)

    def set_sources(self, shot, elem, vec, f0=10.0, t_delay=None, amplitude=1e4,
                    stage_times=False):
        """Ricker sources (acous_elas_cpp/src/WaveOKL3d.cpp:765-781): entry j adds
        ricker(t) * vec[j] to the projected rhs_p of element elem[j] in shot
        shot[j].  Defaults are the reference's f0 = 10, tR = 1/f0, 1e4."""
        shot, elem = _i32(shot).ravel(), _i32(elem).ravel()
        vec = _f32(vec)
        if vec.size != len(elem) * self.Np or len(shot) != len(elem):
            raise ValueError("source entries: shot, elem and vec[n][Np] disagree")
        tR = 1.0 / f0 if t_delay is None else t_delay
        _lib.call("bbw_set_sources", self._h, len(elem), shot.ctypes.data, elem.ctypes.data,
                  vec.ctypes.data, float(f0), float(tR), float(amplitude), int(bool(stage_times)))

    def clear_sources(self):
        _lib.call("bbw_set_sources", self._h, 0, None, None, None, 0.0, 0.0, 0.0, 0)

    def set_receivers(self, elem, w, max_steps):
        """Receivers p(x_r) = w[r] . Q[elem[r]][p], recorded after every step."""
        elem, w = _i32(elem).ravel(), _f32(w)
        if w.size != len(elem) * self.Np:
            raise ValueError("receiver weights must be [R][Np]")
        _lib.call("bbw_set_receivers", self._h, len(elem), elem.ctypes.data, w.ctypes.data,
                  int(max_steps))
        self.R, self.max_steps = len(elem), int(max_steps)

    def get_traces(self):
        """Recorded traces [S][R][nsteps]."""
        out = np.zeros((self.S, self.R, max(self.max_steps, 1)), np.float32)
        n = ctypes.c_int(0)
        _lib.call("bbw_get_traces", self._h, out.ctypes.data, ctypes.byref(n))
        return out[:, :, :n.value]

    def set_time(self, t=0.0):
        """Device clock (time of the next step's start); resets the step count."""
        _lib.call("bbw_set_time", self._h, float(t))

    def get_time(self):
        t, st = ctypes.c_double(0), ctypes.c_int(0)
        _lib.call("bbw_get_time", self._h, ctypes.byref(t), ctypes.byref(st))
        return t.value, st.value

    # ---- discrete adjoint
    def set_c2q(self, c2q):
        """Replace c^2/J at the cubature points ([K][Nq])."""
        c2q = _f32(c2q)
        if c2q.size != self.K * self.Nq:
            raise ValueError("c2q must have K*Nq values")
        _lib.call("bbw_set_c2q", self._h, c2q.ctypes.data)

    def forward(self, dt, nsteps, checkpoint_every=50, keep="cubature"):
        """nsteps steps as steps() does; returns a Tape.  keep="cubature"
        stores every stage's cubature values when the device has room (the
        backward pass then recomputes nothing), else checkpoints every
        checkpoint_every steps; keep="checkpoints" always checkpoints."""
        modes = {"checkpoints": 0, "cubature": 1}
        if keep not in modes:
            raise ValueError("keep must be 'checkpoints' or 'cubature'")
        t = ctypes.c_void_p()
        _lib.call("bbw_forward_ex", self._h, float(dt), int(nsteps), int(checkpoint_every),
                  modes[keep], ctypes.byref(t))
        return Tape(t, int(nsteps))

    def backward(self, tape, dL_dtraces, want_state=False):
        """dL/dtraces [S][R][nsteps] -> dL/dc2q [K][Nq] (FP64, summed over
        shots) and, with want_state, dL/d(initial state) [S*K*4*Np]."""
        g = _f32(dL_dtraces)
        if g.size != self.S * self.R * tape.nsteps:
            raise ValueError("dL/dtraces must be [S][R][nsteps]")
        grad = np.zeros((self.K, self.Nq), np.float64)
        dq = np.zeros(self.state_size, np.float32) if want_state else None
        _lib.call("bbw_backward", self._h, tape.handle, g.ctypes.data, grad.ctypes.data,
                  dq.ctypes.data if want_state else None)
        return (grad, dq) if want_state else grad

    def sync(self):
        _lib.call("bbw_sync", self._h)

    def check(self):
        """Raise if a bounded device-side wait gave up (state invalid)."""
        _lib.call("bbw_check", self._h)

    def device_state(self):
        q, r, s = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _lib.call("bbw_device_state", self._h, ctypes.byref(q), ctypes.byref(r), ctypes.byref(s))
        return q.value, r.value, s.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.call("bbw_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Tape:
    """What one bbw_forward call kept (freed with the object): every stage's
    cubature values (kind "cubature") or checkpoints ("checkpoints")."""

    def __init__(self, handle, nsteps):
        self.handle, self.nsteps = handle, nsteps
        self.kind = "cubature" if _lib.lib().bbw_tape_kind(handle) else "checkpoints"

    def free(self):
        if getattr(self, "handle", None):
            _lib.call("bbw_tape_free", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
