"""Element (slab) decomposition of one mesh across devices.

The mesh is cut into slabs of equal element count along one axis (element
centroids sorted along it).  Each part owns its slab's elements and keeps
halo copies of the neighbouring elements owned by other parts; a part's
context advances only its owned elements (bbw_set_compute_range) and reads
the halo copies for their face traces.  After every stage each part sends the
new state of its owned elements that appear in other parts' halos, and
writes what it receives into its halo slots (bbw_gather_elements /
bbw_scatter_elements), so the next stage sees current neighbour traces.

One exchange per stage carries 4 Np floats per halo element and shot.  The
reference runs on one device (cpp/src/WaveOKL3d.cpp:1415); the per-element
arithmetic is unchanged by the cut, so the decomposed run reproduces the
single-device run.

Overlap (``slab_partition(..., interface_first=True)`` and
``run_decomposed(..., overlap=True)``): each part's owned elements are
ordered interface first (those with a face neighbour in another part); a
stage advances the interface elements, then the interior ones, while on a
side stream the interface elements' new states are packed, copied and
written into the other parts' halo slots of their next state; every part
commits the stage once its incoming halos have landed.
"""
from dataclasses import dataclass, field

import numpy as np

from .problem import np_of, nfp_of
from .solver import RK4A, RK4B


@dataclass
class Part:
    """One slab: local element order = owned (global order) then halo."""
    index: int
    owned: np.ndarray            # global ids of owned elements
    halo: np.ndarray             # global ids of halo elements
    vgeo: np.ndarray             # [K][9]
    fgeo: np.ndarray             # [K][16]
    vmapP: np.ndarray            # [K][4Nfp] local trace indices; halo faces are boundary faces
    c2q: np.ndarray              # [K][Nq]
    send: dict = field(default_factory=dict)   # part q -> local ids sent to q
    recv: dict = field(default_factory=dict)   # part q -> local halo ids received from q
    Ki: int = 0                  # interface elements [0, Ki) of the owned ones (interface_first)

    @property
    def K(self):
        return len(self.owned) + len(self.halo)

    @property
    def Kc(self):
        return len(self.owned)

    @property
    def ids(self):
        return np.concatenate([self.owned, self.halo])


def slab_partition(prob, nparts, axis=2, interface_first=False):
    """Cut prob's mesh into nparts slabs along `axis` (0, 1, 2 = x, y, z).
    interface_first: order each part's owned elements with those that have a
    face neighbour in another part first (Part.Ki of them)."""
    N, K = prob.N, prob.K
    Np, NF = np_of(N), 4 * nfp_of(N)
    if not 1 <= nparts <= K:
        raise ValueError("nparts must be in [1, K]")
    V = np.stack(prob.extra["VX"], -1)[np.asarray(prob.extra["EToV"])]  # [K][4][3]
    cen = V.mean(1)[:, axis]
    order = np.argsort(cen, kind="stable")
    part_of = np.empty(K, np.int64)
    for p, chunk in enumerate(np.array_split(order, nparts)):
        part_of[chunk] = p
    vm = np.asarray(prob.mesh["vmapP"], np.int64).reshape(K, NF)
    nbr = vm // (4 * Np)
    Fmask = np.asarray(prob.ops["Fmask"], np.int64)
    vgeo = np.asarray(prob.mesh["vgeo"]).reshape(K, 9)
    fgeo = np.asarray(prob.mesh["fgeo"]).reshape(K, 16)
    c2q = np.asarray(prob.c2q).reshape(K, -1)
    parts = []
    for p in range(nparts):
        owned = np.nonzero(part_of == p)[0]
        ki = 0
        if interface_first:
            iface = (part_of[nbr[owned]] != p).any(1)
            owned = np.concatenate([owned[iface], owned[~iface]])
            ki = int(iface.sum())
        cand = np.unique(nbr[owned])
        halo = cand[part_of[cand] != p]
        ids = np.concatenate([owned, halo])
        g2l = np.full(K, -1, np.int64)
        g2l[ids] = np.arange(len(ids))
        lv = np.empty((len(ids), NF), np.int64)
        lv[:len(owned)] = g2l[nbr[owned]] * 4 * Np + vm[owned] % (4 * Np)
        hl = np.arange(len(owned), len(ids))
        lv[len(owned):] = hl[:, None] * 4 * Np + Fmask[None, :]  # halo faces: boundary
        parts.append(Part(p, owned, halo, np.ascontiguousarray(vgeo[ids]),
                          np.ascontiguousarray(fgeo[ids]), np.ascontiguousarray(lv, np.int32),
                          np.ascontiguousarray(c2q[ids]), Ki=ki))
    for q in parts:  # q's halo elements owned by p
        for p in parts:
            if p is q:
                continue
            g = q.halo[part_of[q.halo] == p.index]
            if len(g):
                pos = np.full(K, -1, np.int64)  # global id -> position among p's owned
                pos[p.owned] = np.arange(len(p.owned))
                p.send[q.index] = pos[g].astype(np.int32)
                q.recv[p.index] = (len(q.owned) + np.searchsorted(q.halo, g)).astype(np.int32)
    return parts


def local_solver(prob, part, **kw):
    """WaveSolver for one part (halo included, only owned elements advanced)."""
    from .solver import WaveSolver
    s = WaveSolver(N=prob.N, K=part.K, Nq=prob.Nq, variant=prob.variant, ops=prob.ops_dict(),
                   vgeo=part.vgeo, fgeo=part.fgeo, vmapP=part.vmapP, c2q=part.c2q, **kw)
    s.set_compute_range(part.Kc)
    return s


def local_state(prob, part, Q):
    """Rows of a global state [K][4][Np] for the part's local elements."""
    return np.ascontiguousarray(np.asarray(Q).reshape(prob.K, -1)[part.ids]).ravel()


class LocalExchange:
    """Halo exchange between parts whose contexts live in this process (on
    one or several devices): gather into a device buffer, copy, scatter."""

    def __init__(self, parts, solvers, devices=None):
        import torch
        self.parts, self.solvers = parts, solvers
        devices = devices or [0] * len(parts)
        self.devices = devices
        self.links = []
        for p in parts:
            dp = torch.device("cuda", devices[p.index])
            for q, send in p.send.items():
                dq = torch.device("cuda", devices[q])
                recv = parts[q].recv[p.index]
                n = len(send) * solvers[p.index].S * 4 * solvers[p.index].Np
                self.links.append((p.index, q, torch.from_numpy(send).to(dp),
                                   torch.from_numpy(recv).to(dq),
                                   torch.empty(n, dtype=torch.float32, device=dp),
                                   torch.empty(n, dtype=torch.float32, device=dq)))

    def stage_overlapped(self, fa, fb, dt):
        """One stage with the halo exchange overlapping the interior elements
        (parts from slab_partition(..., interface_first=True))."""
        import torch
        if not hasattr(self, "_side"):
            self._main = [torch.cuda.ExternalStream(s.device_state()[2],
                                                    device=torch.device("cuda", d))
                          for s, d in zip(self.solvers, self.devices)]
            self._side = [torch.cuda.Stream(device=st.device) for st in self._main]
        done = []
        for part, s, main in zip(self.parts, self.solvers, self._main):
            if part.Ki > 0:
                s.stage_part(fa, fb, dt, 0, part.Ki)
            ev = torch.cuda.Event()
            ev.record(main)  # interface elements advanced
            done.append(ev)
            if part.Ki < part.Kc:
                s.stage_part(fa, fb, dt, part.Ki, part.Kc)
        touched = [[] for _ in self.solvers]
        for p, q, si, ri, bp, bq in self.links:
            side = self._side[p]
            side.wait_event(done[p])
            self.solvers[p].move_elements(1, 0, si, bp, side.cuda_stream)  # next state of p
            with torch.cuda.stream(side):
                bq.copy_(bp, non_blocking=True)
            copied = torch.cuda.Event()
            copied.record(side)
            # the scatter is a launch on q's device: on one of q's streams
            side_q = self._side[q] if self.devices[q] != self.devices[p] else side
            if side_q is not side:
                side_q.wait_event(copied)
            self.solvers[q].move_elements(1, 1, ri, bq, side_q.cuda_stream)  # q's next-state halo
            ev = torch.cuda.Event()
            ev.record(side_q)
            touched[p].append(copied)
            touched[q].append(ev)
        for s, main, evs in zip(self.solvers, self._main, touched):
            for ev in evs:  # halos in place; own buffers free again
                main.wait_event(ev)
            s.stage_commit()

    def __call__(self):
        for s in self.solvers:
            s.sync()
        for p, q, si, ri, bp, bq in self.links:
            self.solvers[p].gather_elements(si, bp)
            self.solvers[p].sync()
            bq.copy_(bp)
            self.solvers[q].scatter_elements(ri, bq)
        for s in self.solvers:
            s.sync()


class DistExchange:
    """Halo exchange of this rank's part with the parts of the other ranks
    (torch.distributed point-to-point: NCCL over NVLink with device buffers,
    gloo with host buffers).  gather(idx, buf) / scatter(idx, buf) move the
    listed elements' states; for a WaveSolver they are its
    gather_elements / scatter_elements, with sync its sync."""

    def __init__(self, part, gather, scatter, floats_per_element, device, sync=None,
                 group=None, solver=None):
        import torch
        if torch.device(device).type == "cuda" and sync is None:
            # the gather kernels run on the solver's stream, NCCL reads the
            # buffers on another: without sync the send could read them early
            raise ValueError("DistExchange: device buffers need sync (the solver's sync)")
        self.gather, self.scatter, self.sync, self.group = gather, scatter, sync, group
        self.part, self.solver = part, solver  # solver: for stage_overlapped (device buffers)
        n = floats_per_element
        self.sends = [(q, torch.from_numpy(i).to(device),
                       torch.empty(len(i) * n, dtype=torch.float32, device=device))
                      for q, i in sorted(part.send.items())]
        self.recvs = [(q, torch.from_numpy(i).to(device),
                       torch.empty(len(i) * n, dtype=torch.float32, device=device))
                      for q, i in sorted(part.recv.items())]

    def stage_overlapped(self, fa, fb, dt):
        """One stage of this rank's part (cut interface first) with the
        exchange on a side stream beside the interior elements: pack the
        interface elements' next state, NCCL send / receive, write the
        received halos into the next state, then commit.  Device buffers
        (NCCL) only; not run here on several GPUs."""
        import torch
        import torch.distributed as dist
        s, part = self.solver, self.part
        if not hasattr(self, "_side"):
            self._main = torch.cuda.ExternalStream(s.device_state()[2])
            self._side = torch.cuda.Stream()
        if part.Ki > 0:
            s.stage_part(fa, fb, dt, 0, part.Ki)
        ev = torch.cuda.Event()
        ev.record(self._main)
        if part.Ki < part.Kc:
            s.stage_part(fa, fb, dt, part.Ki, part.Kc)
        side = self._side
        side.wait_event(ev)
        with torch.cuda.stream(side):
            for q, idx, buf in self.sends:
                s.move_elements(1, 0, idx, buf, side.cuda_stream)
            ops = [dist.P2POp(dist.isend, buf, q, self.group) for q, _, buf in self.sends]
            ops += [dist.P2POp(dist.irecv, buf, q, self.group) for q, _, buf in self.recvs]
            if ops:
                for r in dist.batch_isend_irecv(ops):
                    r.wait()  # the side stream waits for the transfers
            for q, idx, buf in self.recvs:
                s.move_elements(1, 1, idx, buf, side.cuda_stream)
        done = torch.cuda.Event()
        done.record(side)
        self._main.wait_event(done)
        s.stage_commit()

    def __call__(self):
        import torch.distributed as dist
        for q, idx, buf in self.sends:
            self.gather(idx, buf)
        if self.sync:
            self.sync()
        ops = [dist.P2POp(dist.isend, buf, q, self.group) for q, _, buf in self.sends]
        ops += [dist.P2POp(dist.irecv, buf, q, self.group) for q, _, buf in self.recvs]
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        if self.recvs and self.recvs[0][2].is_cuda:  # received data visible to the scatter stream
            import torch
            torch.cuda.current_stream(self.recvs[0][2].device).synchronize()
        for q, idx, buf in self.recvs:
            self.scatter(idx, buf)


def run_decomposed(solvers, exchange, dt, nsteps, overlap=False):
    """nsteps LSRK45 steps of every part, the halo refreshed after each stage
    (overlap: the exchange's stage_overlapped, parts cut interface first)."""
    for _ in range(nsteps):
        for i in range(5):
            if overlap:
                exchange.stage_overlapped(np.float32(RK4A[i]), np.float32(RK4B[i]), dt)
                continue
            for s in solvers:
                s.rk_stage(np.float32(RK4A[i]), np.float32(RK4B[i]), dt, 0.0)
            exchange()
    if overlap:
        for s in solvers:
            s.sync()
    return solvers
