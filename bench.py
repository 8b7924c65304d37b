#!/usr/bin/env python3
"""Benchmark: acoustic WADG LSRK45 step, N=5, 32^3 x 6 affine tets (K=196608).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Metric: DOF-stage updates per second,
K * Np * 4 fields * 5 stages * steps / seconds, the reference's own per-DOF
normalisation (cpp/src/WaveOKL3d.cpp:1763).  Workload (the configuration the
metric is quoted on): N=5 (Np=56, Nq=95 from the reference's degree-11 tet
rule), [-1,1]^3 split into 32^3 hexes x 6 tets, c^2 = 1 + 0.5 sin sin sin +
0.5 U(0,1) per element (seeded), Gaussian pulse, p = 0 walls, FP32 state.
The state (3 x 176 MB) exceeds the 126 MB L2, so no flush is needed between
steps.

The headline form is the tensor-core stage (nodal-f16x3): FP32 state, the
dense contractions on tcgen05 as three FP16 products per split pair with
FP32 accumulation.  Its error against the FP64 restatement is the FP32
stage's (the line's `precision` object gives both, measured in the same
run); the FP32 CUDA-core stage and the BB stage run beside it
(`side_by_side`).

* value      device-timed throughput of the fused stage kernels, inputs
             resident in HBM (CUDA events on the solver's stream, max over
             ranks, weak scaling: each rank advances its own copy of the
             workload, one shot per GPU);
* e2e        the same run through the public API with host buffers: the
             initial state is copied in from pinned host memory and the final
             state read back inside the timed region;
* roofline   the fused stage kernel against the measured HBM copy bandwidth;
             algorithmic bytes per element-stage 64 Np + 4 Nq + 132;
* cpu_baseline  the reference's own OKL kernels (oracle/_ref, built from the
             reference sources, OpenMP over elements) on all of this host's
             cores, on the same 32^3 x 6 mesh, N and operators, one LSRK45
             step (a bounded sample of the run).

--impl reference runs only that CPU path on the same workload (rank 0;
other ranks exit 0): --warmup untimed steps (at most 2) then --steps timed
steps (at most 30), each a full LSRK45 step of the 32^3 x 6 mesh.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

N_ORDER, N_HEX = 5, 32
REF_MAX_STEPS, REF_MAX_WARMUP = 30, 2  # bound on the reference arm's CPU time


def algorithmic_bytes_per_element(Np, Nq):
    # Q read + write, res read + write (4 fields, FP32), c2 at cubature
    # points, vgeo (9) + fgeo (16) floats, neighbour + permutation codes
    return 64 * Np + 4 * Nq + 132


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def reference_rule(N):
    """The reference's tabulated degree-2N+1 tet rule (from the golden
    fixture produced by running the reference), so Nq matches its cost."""
    p = os.path.join(ROOT, "tests", "golden", "ops_N%d.npz" % N)
    if not os.path.exists(p):
        return None, None
    g = np.load(p)
    nfq = int(g["Nfq"][0])
    return (g["rq"], g["sq"], g["tq"], g["wq"]), (g["rfq"][:nfq], g["sfq"][:nfq], g["wfqFace"])


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def reference_cpu(steps, warmup, nhex=N_HEX, N=N_ORDER, bern=0, timeout=900):
    """The reference's own CPU path: oracle/_ref driver (reference host code +
    OKL kernels translated and JIT-compiled with OpenMP), all host threads."""
    from bbwadg_b200.mesh import kuhn_box, write_gmsh22
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_N%d_B%d" % (N, bern))
    if not os.path.exists(exe):
        return None, "oracle/_ref/ref_N%d_B%d not built" % (N, bern)
    d = tempfile.mkdtemp()
    msh = os.path.join(d, "box.msh")
    write_gmsh22(msh, *kuhn_box(nhex))
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    p = subprocess.run([exe, "bench", msh, "--steps", str(steps), "--warmup", str(warmup),
                        "--c2", "sine"], capture_output=True, text=True, env=env, timeout=timeout)
    if p.returncode != 0:
        return None, "reference run failed: " + p.stderr[-200:]
    r = json.loads(p.stdout.strip().splitlines()[-1])
    r["cores"] = cores
    r["cpu_model"] = cpu_model()
    return r, None


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    steps = min(max(args.steps, 1), REF_MAX_STEPS)
    warm = min(max(args.warmup, 0), REF_MAX_WARMUP)
    r, err = reference_cpu(steps, warm)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    v = r["dof_stage_per_s"]
    sample = ("N=%d, %d^3 x 6 tets (K=%d, the full workload), %d LSRK45 steps timed after %d "
              "warm-up (steps capped at %d)" % (N_ORDER, N_HEX, r["K"], r["steps"], warm,
                                                REF_MAX_STEPS))
    print(json.dumps({
        "metric": "DOF-stage updates/s (acoustic WADG, affine tets, N=5)", "impl": "reference",
        "value": v, "unit": "DOF-stage/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": warm, "ms_per_step": 1e3 * r["seconds"] / r["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": workload_config(args, "nodal"),
        "cpu_baseline": {"value": v, "unit": "DOF-stage/s", "cores": r["cores"],
                         "cpu_model": r["cpu_model"], "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))
    return 0


def workload_config(args, variant):
    nh = getattr(args, "hex", N_HEX)
    return {"workload": "acoustic WADG LSRK45 step, N=%d, %d^3x6 affine tets, %s" % (
                N_ORDER, nh, variant),
            "N": N_ORDER, "K": 6 * nh ** 3, "Np": 56, "Nq": 95, "variant": variant,
            "global_batch": args.gpus, "parallelism": "replicas (one shot per GPU)",
            "l2_flush": "state 3x176 MB > L2", "bc": "pressure_release"}


def c2_inclusions(seed, n=10, lo=-0.8, hi=0.8):
    """c^2 in [1, 2): 1 + s/(1+s), s a sum of n seeded Gaussian inclusions."""
    rng = np.random.default_rng(seed)
    cen = rng.uniform(lo, hi, (n, 3))
    rad = rng.uniform(0.1, 0.3, n)
    amp = rng.uniform(0.5, 2.0, n)

    def f(x, y, z):
        s = np.zeros_like(x)
        for c, r, a in zip(cen, rad, amp):
            s += a * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / r ** 2)
        return 1.0 + s / (1.0 + s)
    return f


def anomalies(base, seed, n=5, amp=0.3):
    """base + n seeded Gaussian anomalies of amplitude +-amp."""
    rng = np.random.default_rng(seed)
    cen = rng.uniform(-0.6, 0.6, (n, 3))
    rad = rng.uniform(0.15, 0.3, n)
    sgn = rng.choice([-1.0, 1.0], n)

    def f(x, y, z):
        v = base(x, y, z)
        for c, r, sg in zip(cen, rad, sgn):
            v = v + sg * amp * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / r ** 2)
        return v
    return f


def shot_sources(prob, S, seed, a=20.0, first=0):
    """Seeded point-like sources in [-0.8, 0.8]^3 for global shots
    first..first+S-1 (local shots 0..S-1): (shot, elem, vec) entries."""
    from bbwadg_b200.problem import gaussian_source, source_entries
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.8, 0.8, (first + S, 3))[first:]
    xyz = prob.cubature_xyz()
    ent = [source_entries(gaussian_source(prob, c, a=a, xyz=xyz), shot=i)
           for i, c in enumerate(centres)]
    return [np.concatenate(x) for x in zip(*ent)]


def shots_workload(args, torch, dist, world):
    """Batched multi-shot: N=4, 24^3 x 6 tets (K=82944), 32 shots in one
    launch per stage (graph-captured steps), Ricker f0 = 4 point sources at
    seeded locations, c^2 in [1, 2] with 10 seeded Gaussian inclusions."""
    from bbwadg_b200 import WaveSolver, make_problem
    N, nh, S = 4, args.shots_hex, args.shots
    cub, tri = reference_rule(N)
    prob = make_problem(N, nh, c2=c2_inclusions(77), cubature=cub, tri_cubature=tri, cfl=0.25)
    out = {"workload": "batched shots, N=4, %d^3x6 tets (K=%d), %d shots, Ricker f0=4, "
                       "c2 in [1,2] with 10 inclusions" % (nh, prob.K, S),
           "N": N, "K": prob.K, "shots": S}
    finals = {}
    for label, nshot, prec in (("batched", S, "fp32"), ("one_shot", 1, "fp32"),
                               ("batched_f16x3", S, "f16x3"), ("one_shot_f16x3", 1, "f16x3")):
        s = WaveSolver(prob, precision=prec)
        s.set_shots(nshot)
        s.set_sources(*shot_sources(prob, nshot, 99), f0=4.0, amplitude=1e4, stage_times=True)
        s.set_time(0.0)
        tuned = s.autotune(prob.dt, 5) if prec == "fp32" else None
        _, _, sp = s.device_state()
        stream = torch.cuda.ExternalStream(sp)
        s.steps(prob.dt, args.warmup)
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        s.steps(prob.dt, args.shots_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        dofs = prob.K * prob.Np * 4 * 5 * args.shots_steps * nshot
        q = s.get_data()
        out[label] = {"value": world * dofs / (ms / 1e3), "unit": "DOF-stage/s",
                      "ms_per_step": ms / args.shots_steps, "steps": args.shots_steps,
                      "precision": prec,
                      "config": tuned["code"] if tuned else None,  # autotuned FP32 variant
                      "finite": bool(np.isfinite(q).all())}
        finals[label] = q
        s.close()
    # the split-FP16 run against the FP32 run of the same shots (same inputs,
    # warm-up + timed steps): relative L2 over all shots
    a, b = finals["batched_f16x3"].astype(np.float64), finals["batched"].astype(np.float64)
    out["batched_f16x3"]["rel_l2_vs_fp32"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return out


def adjoint_workload(args, torch, dist, rank, world):
    """Forward + adjoint gradient: N=4, 16^3 x 6 tets (K=24576), 8 seeded
    Ricker shots per GPU, 64 seeded receivers, 400 steps, checkpoints every
    50, L2 trace misfit against a target with 5 seeded +-0.3 Gaussian
    anomalies.  With several ranks the shots are sharded (8 per rank) and the
    FP64 gradient is summed with one all-reduce, inside the timed region."""
    from bbwadg_b200 import WaveSolver, make_problem
    from bbwadg_b200.problem import c2_sine, receiver_weights
    from bbwadg_b200.shards import allreduce_gradient, shot_range
    N, nh, R, steps, every = 4, 16, 64, args.adj_steps, 50
    lo, hi = shot_range(8 * world, rank, world)
    S = hi - lo
    cub, tri = reference_rule(N)
    base = c2_sine
    prob = make_problem(N, nh, c2=anomalies(base, 5), cubature=cub, tri_cubature=tri, cfl=0.25)
    xq, yq, zq = prob.cubature_xyz()
    c2_target = prob.c2q.copy()
    c2_back = np.ascontiguousarray(base(xq, yq, zq), np.float32)
    rng = np.random.default_rng(64)
    el, w = receiver_weights(prob, rng.uniform(-0.8, 0.8, (R, 3)))
    def one(prec):
        """Forward + backward with the stage form `prec`; times, misfit, gradient."""
        s = WaveSolver(prob, precision=prec)
        s.set_shots(S)
        s.set_sources(*shot_sources(prob, S, 8, first=lo), f0=4.0, amplitude=1e4,
                      stage_times=True)
        s.set_receivers(el, w, steps)
        zero = np.zeros(s.state_size, np.float32)

        def run(c2, tape):
            s.set_c2q(c2)
            s.set_data(zero)
            s.set_residual(zero)
            s.set_time(0.0)
            if tape:
                return s.forward(prob.dt, steps, every)
            s.steps(prob.dt, steps)
            s.sync()
            return None

        run(c2_target, False)
        obs = s.get_traces().copy()
        s.sync()
        t0 = time.perf_counter()
        tape = run(c2_back, True)
        s.sync()
        t1 = time.perf_counter()
        kind = tape.kind
        tr = s.get_traces()
        misfit = 0.5 * float(((tr - obs).astype(np.float64) ** 2).sum())
        t2 = time.perf_counter()
        grad = s.backward(tape, tr - obs)
        if world > 1:
            grad = allreduce_gradient(grad, device="cuda")
            misfit = allreduce_gradient(np.array([misfit]), device="cuda")[0]
        t3 = time.perf_counter()
        tape.free()
        s.close()
        tf, tb = t1 - t0, t3 - t2
        if world > 1:
            t = torch.tensor([tf, tb], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tf, tb = float(t[0]), float(t[1])
        return tf, tb, misfit, grad, kind

    tf, tb, misfit, grad, kind = one("fp32")
    tf2, tb2, misfit2, grad2, kind2 = one("f16x3")
    return {"workload": "forward + adjoint c2 gradient, N=4, 16^3x6 tets (K=%d), %d shots per "
                        "GPU, %d receivers, %d steps; tape: every stage's cubature values, or "
                        "checkpoints every %d where they do not fit" % (prob.K, S, R, steps, every),
            "tape": kind,  # cubature: every stage's Vq S(Q)_p kept, no recomputation
            "forward_s": tf, "backward_s": tb, "total_s": tf + tb, "shots_total": 8 * world,
            "misfit": misfit, "grad_norm": float(np.linalg.norm(grad)),
            "grad_finite": bool(np.isfinite(grad).all()),
            "f16x3": {"tape": kind2, "forward_s": tf2, "backward_s": tb2, "total_s": tf2 + tb2,
                      "misfit": misfit2,
                      "grad_rel_l2_vs_fp32": float(np.linalg.norm(grad2 - grad) /
                                                   np.linalg.norm(grad)),
                      "note": "forward (and any recomputation) on the split-FP16 tensor-core "
                              "stage"}}


def precision_workload(args, torch):
    """Error study on the standing mode p = cos(pi x)cos(pi y)cos(pi z)
    cos(sqrt(3) pi t), c^2 = 1, p = 0 walls on [-1/2, 1/2]^3 (exact for the
    reference's boundary condition), h-refinement 8/16/24: at N = 7 the FP32
    fused stage against the GEMM precision form (split FP16, split BF16, TF32
    contractions as cuBLAS GEMMs; the fused tensor-core stage needs
    Np <= 64), at N = 5 the FP32 stage against the split-FP16 and split-BF16
    tensor-core stage and TF32 on the GEMM form.  Errors: relative L2
    against the exact solution at T (FP64 quadrature), and against the FP64
    C restatement over the first 10 steps on the 8^3 mesh."""
    import math
    from oracle import Oracle
    from bbwadg_b200 import WaveSolver, make_problem
    from bbwadg_b200.problem import cavity_mode
    T = args.prec_time
    rows = []
    for N, precs in ((7, ("fp32", "f16x3", "bf16x3", "tf32")),
                     (5, ("fp32", "f16x3", "bf16x3", "tf32"))):
        cub, tri = reference_rule(N)
        for nh in (8, 16, 24):
            p = make_problem(N, nh, c2="one", ic="cavity", lo=-0.5, hi=0.5, cubature=cub,
                             tri_cubature=tri, cfl=0.25)
            nsteps = int(math.ceil(T / p.dt))
            dt = float(np.float32(T / nsteps))
            zero = np.zeros(p.K * 4 * p.Np, np.float32)
            q64 = None
            for prec in precs:
                s = WaveSolver(p, precision=prec)
                s.set_data(p.Q0)
                s.steps(dt, 2)  # warm-up (graph capture)
                s.set_data(p.Q0)
                s.set_residual(zero)
                s.sync()
                t0 = time.perf_counter()
                s.steps(dt, nsteps)
                s.sync()
                el = time.perf_counter() - t0
                Q = s.get_data()
                err, rel = p.l2_error(Q, nsteps * dt, cavity_mode)
                row = {"N": N, "n": nh, "K": p.K, "precision": prec, "steps": nsteps,
                       "form": ("fused FP32" if prec == "fp32" else
                                "tensor-core stage" if (N <= 5 and prec != "tf32") else
                                "GEMM precision form"),
                       "rel_l2_vs_exact": rel, "ms_per_step": 1e3 * el / nsteps}
                if nh == 8:
                    s.set_data(p.Q0)
                    s.set_residual(zero)
                    s.steps(dt, 10)
                    q10 = s.get_data()
                    if q64 is None:  # once per mesh
                        q64, _ = Oracle(N, p.K, p.ops_dict(), p.geo_dict(),
                                        dtype=np.float64).run(p.Q0.astype(np.float64), dt, 50)
                    row["rel_l2_vs_fp64_10_steps"] = float(
                        np.linalg.norm(q10 - q64) / np.linalg.norm(q64))
                rows.append(row)
                s.close()
    return {"workload": "standing mode, c2=1, p=0 walls on [-1/2,1/2]^3, T=%g, CFL 0.25" % T,
            "rows": rows}


def headline_precision(variant, prec_rows):
    """Arithmetic of the headline form, with its error against the FP64
    restatement and the FP32 stage's, from the precision study of the same
    run (N = 5, 8^3 x 6, standing mode, 10 steps)."""
    tc = variant.endswith("f16x3")
    out = {"state": "fp32", "update": "fp32",
           "contractions": "split-FP16, 3 products per pair on tcgen05, FP32 accumulation"
           if tc else "FP32 CUDA cores"}
    if prec_rows:
        for r in prec_rows["rows"]:
            if r["N"] == 5 and "rel_l2_vs_fp64_10_steps" in r:
                key = {"f16x3": "f16x3", "fp32": "fp32"}.get(r["precision"])
                if key:
                    out["rel_l2_vs_fp64_%s" % key] = r["rel_l2_vs_fp64_10_steps"]
    return out


def curved_bytes_per_element(Np, Nq, Nfq, Nfp, curved):
    """Algorithmic bytes of one curvilinear stage per element: state and
    residual read + write (4 fields, FP32), J and c^2 at the update's
    cubature, the trace map; curved elements add vgeoq + Jq at the volume
    cubature and nx ny nz sJ at the face cubature, planar ones vgeo, fgeo, J."""
    base = 64 * Np + 8 * Nq + 16 * Nfp
    return base + (40 * Nq + 64 * Nfq if curved else 4 * (9 + 16 + 1))


def reference_curved_cpu(steps, warmup, nhex, timeout=900):
    """The reference's curvilinear path on the host cores (oracle/_ref/ref_curved_N3)."""
    from bbwadg_b200.mesh import kuhn_ball, write_gmsh22
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_curved_N3")
    if not os.path.exists(exe):
        return None, "oracle/_ref/ref_curved_N3 not built"
    d = tempfile.mkdtemp()
    msh = os.path.join(d, "ball.msh")
    write_gmsh22(msh, *kuhn_ball(nhex))
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    p = subprocess.run([exe, "bench", msh, "--steps", str(steps), "--warmup", str(warmup)],
                       capture_output=True, text=True, env=env, timeout=timeout)
    if p.returncode != 0:
        return None, "reference run failed: " + p.stderr[-200:]
    r = json.loads(p.stdout.strip().splitlines()[-1])
    r["cores"] = cores
    return r, None


def curved_workload(args, torch):
    """Curvilinear WADG step (RK_step_WADG) on the Gordon-Hall curved unit
    ball kuhn_ball(n), N = 3 (the reference's tabulated degree-7 rules),
    c^2 = 1 as InitWADG_curved sets, Bessel initial state: device-timed
    DOF-stage/s, HBM fraction of the whole stage, and the reference's curved
    path on the host cores on kuhn_ball(16)."""
    from bbwadg_b200.curved import CurvedSolver, make_curved_problem
    N, nh = 3, args.curved_hex
    cub, tri = reference_rule(N)
    p = make_curved_problem(N, nh, cubature=cub, tri_cubature=tri)
    s = CurvedSolver(p)
    s.set_data(p.Q0)
    tuned = s.autotune(p.dt, 10)  # planar variant, timed inside whole stages
    stream = torch.cuda.ExternalStream(s.stream)
    s.steps(p.dt, args.warmup)
    s.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = args.curved_steps
    torch.cuda.synchronize()
    e0.record(stream)
    s.steps(p.dt, steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    Q = s.get_data()
    s.close()
    KC, KP = len(p.KlistCurved), len(p.KlistPlanar)
    nfp = (N + 1) * (N + 2) // 2
    alg = (KC * curved_bytes_per_element(p.Np, p.Nq, p.Nfq, nfp, True) +
           KP * curved_bytes_per_element(p.Np, p.Nq, p.Nfq, nfp, False))
    stage_s = ms / 1e3 / (5 * steps)
    peak, kind = measured_peak()
    dofs = p.K * p.Np * 4 * 5 * steps
    out = {"workload": "curvilinear WADG step (RK_step_WADG), N=3, kuhn_ball(%d): K=%d, %d curved"
                       % (nh, p.K, KC),
           "value": dofs / (ms / 1e3), "unit": "DOF-stage/s", "ms_per_step": ms / steps,
           "steps": steps, "hbm_frac_of_stage": alg / stage_s / 1e9 / peak, "peak_kind": kind,
           "alg_bytes_per_stage": alg,
           "gpu_launches": 5 * steps * ((KP > 0) + (KC > 0)),  # planar + curved stage kernels
           "planar_config": tuned, "finite": bool(np.isfinite(Q).all())}
    # the reference's curved timing runs span N = 2..5 (cpp/runCurvedBlkTimings)
    out["by_order"] = []
    for No in (2, 4, 5):
        cb, tr = reference_rule(No)
        po = make_curved_problem(No, nh, cubature=cb, tri_cubature=tr)
        so = CurvedSolver(po)
        so.set_data(po.Q0)
        tuned_o = so.autotune(po.dt, 10)
        so.steps(po.dt, args.warmup)
        so.sync()
        st = torch.cuda.ExternalStream(so.stream)
        torch.cuda.synchronize()
        e0.record(st)
        so.steps(po.dt, 10)
        e1.record(st)
        torch.cuda.synchronize()
        mso = e0.elapsed_time(e1)
        out["by_order"].append({"N": No, "Nq": po.Nq, "value": po.K * po.Np * 4 * 50 / (mso / 1e3),
                                "ms_per_step": mso / 10, "planar_config": tuned_o,
                                "finite": bool(np.isfinite(so.get_data()).all())})
        so.close()
    if not args.no_cpu_baseline:
        r, err = reference_curved_cpu(5, 1, 16)
        out["cpu_baseline"] = ({"value": r["dof_stage_per_s"], "unit": "DOF-stage/s",
                                "cores": r["cores"], "kind": "reference",
                                "sample": "N=3, kuhn_ball(16) (K=%d, %d curved), 5 LSRK45 steps, "
                                          "reference kernels via oracle/_ref" % (r["K"], r["KCurved"])}
                               if r else {"value": None, "unavailable": err})
    return out


def kernel_level_workload(args, torch):
    """The headline workload through the kernel-level entry points, the
    reference's three launches per stage (rk_volume, rk_surface,
    rk_update_WADG; cpp/src/WaveOKL3d.cpp:2084-2109) with an rhs array in
    HBM: what a kernel-for-kernel integration gets, beside the fused stage."""
    from bbwadg_b200 import RK4A, RK4B, _lib, make_problem
    cub, tri = reference_rule(N_ORDER)
    p = make_problem(N_ORDER, args.hex, c2="sine", c2_jitter=0.5, seed=1234, cubature=cub,
                     tri_cubature=tri, cfl=0.25)
    o = p.ops_dict()

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()
    vgeo, fgeo, vmapP = dev(p.mesh["vgeo"]), dev(p.mesh["fgeo"]), dev(p.mesh["vmapP"])
    Dr, Ds, Dt, LIFT = dev(o["Dr"]), dev(o["Ds"]), dev(o["Dt"]), dev(o["LIFT"])
    Fmask, Vq, Pq, c2q = dev(o["Fmask"]), dev(o["Vq"]), dev(o["Pq"]), dev(p.c2q.ravel())
    Jq = torch.ones(p.K * p.Nq, device="cuda")
    Q = dev(p.Q0)
    res = torch.zeros(p.Q0.size, device="cuda")
    rhs = torch.empty(p.Q0.size, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    P = _lib.ptr
    dt = float(np.float32(p.dt))

    def step():
        for i in range(5):
            _lib.call("bbw_rk_volume", p.N, p.K, P(vgeo), P(Dr), P(Ds), P(Dt), P(Q), P(rhs), st)
            _lib.call("bbw_rk_surface", p.N, p.K, 0, P(fgeo), P(Fmask), P(vmapP), P(LIFT), P(Q),
                      P(rhs), st)
            _lib.call("bbw_rk_update_wadg", p.N, p.K, p.Nq, P(Vq), P(Pq), P(Jq), P(c2q),
                      float(np.float32(RK4A[i])), float(np.float32(RK4B[i])), dt, P(rhs), P(res),
                      P(Q), st)
    for _ in range(args.warmup):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(args.steps // 4, 5)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"workload": "same as the headline, kernel-level entry points (3 launches per stage)",
            "value": p.K * p.Np * 4 * 5 * steps / (ms / 1e3), "unit": "DOF-stage/s",
            "ms_per_step": ms / steps, "steps": steps, "gpu_launches": 15 * steps,
            "finite": bool(torch.isfinite(Q).all().item())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variant", default="nodal-f16x3",
                    choices=["nodal", "bb", "nodal-f16x3", "bb-f16x3"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--hex", type=int, default=N_HEX, help="hexes per direction (profiling cases)")
    ap.add_argument("--variants", default="nodal-f16x3,nodal,bb,bb-f16x3",
                    help="variants to run, comma separated (nodal, bb, nodal-f16x3, bb-f16x3)")
    ap.add_argument("--extra", default="shots,adjoint,precision,curved,kernel_level",
                    help="extra workloads reported beside the headline: shots, adjoint, "
                         "precision, curved, kernel_level")
    ap.add_argument("--prec-time", type=float, default=0.02)
    ap.add_argument("--config", type=int, default=0,
                    help="pin the fused-stage configuration code instead of autotuning")
    ap.add_argument("--shots", type=int, default=32)
    ap.add_argument("--shots-hex", type=int, default=24)
    ap.add_argument("--shots-steps", type=int, default=10)
    ap.add_argument("--adj-steps", type=int, default=400)
    ap.add_argument("--curved-hex", type=int, default=24)
    ap.add_argument("--curved-steps", type=int, default=50)
    ap.add_argument("--curved-only", action="store_true",
                    help="run only the curvilinear workload and print its object")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    args.warmup = max(args.warmup, 3)
    if args.curved_only:  # the curvilinear workload alone (profiling runs)
        import torch
        torch.cuda.set_device(dist_env()[2])
        print(json.dumps({"curved": curved_workload(args, torch)}))
        return 0

    import torch
    import torch.distributed as dist
    from bbwadg_b200 import WaveSolver, make_problem
    from bbwadg_b200.solver import decode_config

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    cub, tri = reference_rule(N_ORDER)

    results = {}
    variants = [v for v in args.variants.split(",") if v]
    if args.variant not in variants:
        variants.insert(0, args.variant)
    for variant in variants:
        basis, prec = (variant.split("-") + ["fp32"])[:2]
        prob = make_problem(N_ORDER, args.hex, variant=basis, c2="sine", c2_jitter=0.5,
                            seed=1234 + rank, cubature=cub, tri_cubature=tri, cfl=0.25)
        K, Np, Nq = prob.K, prob.Np, prob.Nq
        s = WaveSolver(prob, precision=prec)
        s.set_data(prob.Q0)
        tuned = None
        if prec == "fp32" and args.config:  # a pinned configuration (profiling runs)
            tuned = dict(decode_config(args.config), pinned=True)
            s.set_config(tuned["warps"], tuned["ops_in_smem"], tuned["pipelined"], tuned["tile"])
        elif prec == "fp32":
            tuned = s.autotune(prob.dt, 10)
        qptr, rptr, stream_ptr = s.device_state()
        stream = torch.cuda.ExternalStream(stream_ptr)
        # clocks are sampled every 100 ms from the warm-up through the timed
        # and end-to-end regions (a timed region alone can be shorter than
        # one sample)
        clk = ClockSampler(local).__enter__()
        s.steps(prob.dt, args.warmup)
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        s.steps(prob.dt, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        dofs = K * Np * 4 * 5 * args.steps
        launches = 6 * args.steps  # five fused stages + the clock/receiver kernel per step
        # e2e: WaveSetData3d (pinned host -> device), steps, WaveGetData3d
        pinned = torch.from_numpy(prob.Q0.copy()).pin_memory()
        out = torch.empty_like(pinned).pin_memory()
        # one untimed round trip through both host buffers: the first DMA
        # into a freshly pinned buffer costs about 3 ms more than later ones
        # (a caller reuses its host state buffers)
        s.get_data(out=out.numpy())
        s.set_data(pinned.numpy())
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.set_data(pinned.numpy())
        s.steps(prob.dt, args.steps)
        s.get_data(out=out.numpy())
        t_e2e = time.perf_counter() - t0
        clk.__exit__(None, None, None)
        if world > 1:
            t = torch.tensor([t_e2e], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        state_bytes = K * 4 * Np * 4
        results[variant] = dict(ms=ms, K=K, Np=Np, Nq=Nq, dofs=dofs, launches=launches, tuned=tuned,
                                clocks=clk.summary(), e2e_s=t_e2e, state_bytes=state_bytes,
                                finite=bool(np.isfinite(out.numpy()).all()))
        s.close()

    extra = [x for x in args.extra.split(",") if x]
    shots = shots_workload(args, torch, dist, world) if "shots" in extra else None
    adj = adjoint_workload(args, torch, dist, rank, world) if "adjoint" in extra else None
    prec = precision_workload(args, torch) if ("precision" in extra and rank == 0) else None
    curv = curved_workload(args, torch) if ("curved" in extra and rank == 0) else None
    klev = kernel_level_workload(args, torch) if ("kernel_level" in extra and rank == 0) else None
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    peak, peak_kind = measured_peak()
    head = results[args.variant]
    K, Np, Nq = head["K"], head["Np"], head["Nq"]
    value = world * head["dofs"] / (head["ms"] / 1e3)
    per_launch_s = head["ms"] / 1e3 / (5 * args.steps)  # per stage launch
    alg_bytes = K * algorithmic_bytes_per_element(Np, Nq)
    achieved = alg_bytes / per_launch_s / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "fused_stage_N5_dram.json")
    if os.path.exists(tp):
        with open(tp) as f:
            t = json.load(f).get("%s_bytes_per_element" % args.variant)
        traffic = None if t is None else t * K
    line = {
        "metric": "DOF-stage updates/s (acoustic WADG, affine tets, N=5)",
        "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": dict(workload_config(args, args.variant),
                                            autotuned=head["tuned"]),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": ("k_tc_stage<%d>" % N_ORDER) if args.variant.endswith("f16x3")
                     else "k_fused_stage<%d,%s>" % (N_ORDER, args.variant == "bb"),
                     "peak_kind": peak_kind},
        "e2e": {"value": world * head["dofs"] / head["e2e_s"], "unit": "DOF-stage/s",
                "h2d_bytes_per_step": head["state_bytes"] / args.steps,
                "d2h_bytes_per_step": head["state_bytes"] / args.steps,
                "copies": "per run, as the reference's WaveSetData3d -> Wave_RK -> "
                          "WaveGetData3d: the state in from pinned host memory once, the "
                          "timed steps, the state out once; bytes per step = state bytes / "
                          "steps; both host buffers warmed by one untimed round trip"},
        "gpu_launches": head["launches"],
        "clocks": head["clocks"],
        "precision": headline_precision(args.variant, prec),
        "side_by_side": {v: {"value": world * r["dofs"] / (r["ms"] / 1e3),
                             "ms_per_step": r["ms"] / args.steps,
                             "hbm_frac": K * algorithmic_bytes_per_element(Np, Nq) /
                             (r["ms"] / 1e3 / (5 * args.steps)) / 1e9 / peak,
                             "finite": r["finite"]} for v, r in results.items()},
    }
    if not args.no_cpu_baseline and world == 1:
        r, err = reference_cpu(1, 0)
        if r is not None:
            line["cpu_baseline"] = {
                "value": r["dof_stage_per_s"], "unit": "DOF-stage/s", "cores": r["cores"],
                "cpu_model": r["cpu_model"], "kind": "reference",
                "sample": "N=5, %d^3 x 6 tets (K=%d, the full workload), %d LSRK45 step, "
                          "reference OKL kernels via oracle/_ref" % (N_HEX, r["K"], r["steps"])}
        else:
            line["cpu_baseline"] = {"value": None, "unavailable": err}
    if shots is not None:
        line["shots"] = shots
    if adj is not None:
        line["adjoint"] = adj
    if prec is not None:
        line["precision"] = prec
    if curv is not None:
        line["curved"] = curv
    if klev is not None:
        line["kernel_level"] = klev
    # the most compared objects at the end of the line, where a reader of
    # the output's last lines finds them: the stage forms side by side and
    # the batched shots
    for k in ("curved", "kernel_level", "adjoint", "shots", "side_by_side"):
        if k in line:
            line[k] = line.pop(k)
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
