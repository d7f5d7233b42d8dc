"""Domain-decomposed runs of the fused engine: contiguous element ranges per
rank (DomainDecomp, src/SELF_Mesh.f90:2159-2177) and one face-trace exchange
per RK stage (MPIExchangeAsync + ApplyFlip, src/SELF_MappedData.f90:3323-3443).

A rank's off-rank neighbours are halo elements appended to its trace caches;
its sideInfo points those sides at the halo element, so the fused kernels
(flip included) run unchanged.  Between stages each rank packs the trace
blocks its peers need into one buffer per peer, moves them (NCCL / gloo
send-recv through ``torch.distributed``, or the in-process transport used to
emulate ranks on one GPU), and unpacks what it receives into its halo blocks.
ShallowWater's stage-lagged velocity traces are exchanged the same way.
"""
import ctypes

import numpy as np
import torch

from . import api as A
from ._lib import check, lib


def domain_decomp(nElems, nDomains):
    """offsetElem (nDomains + 1,): first element (0-based) of each rank."""
    off = np.zeros(nDomains + 1, dtype=np.int32)
    check(lib().selfgpu_domain_decomp(int(nElems), int(nDomains), off.ctypes.data_as(ctypes.c_void_p)))
    return off


def elem_to_rank(offsetElem, elemID):
    """Rank holding the 1-based element elemID (ElemToRank)."""
    off = np.ascontiguousarray(offsetElem, dtype=np.int32)
    d = ctypes.c_int()
    check(lib().selfgpu_elem_to_rank(len(off) - 1, off.ctypes.data_as(ctypes.c_void_p), int(elemID), ctypes.byref(d)))
    return d.value


class HaloPlan:
    """One rank's share of a global Mesh2D: local sideInfo with halo
    neighbours, and per peer the trace blocks to send and to receive."""

    def __init__(self, mesh, nDomains, rank):
        self.nDomains, self.rank = nDomains, rank
        self.offsets = domain_decomp(mesh.nElem, nDomains)
        self.first = int(self.offsets[rank])
        self.nLocal = int(self.offsets[rank + 1] - self.offsets[rank])
        si = np.asfortranarray(mesh.sideInfo, dtype=np.int32)
        self.sideInfo = np.zeros((5, 4, self.nLocal), dtype=np.int32, order="F")
        nHalo = ctypes.c_int()
        counts = np.zeros(nDomains, dtype=np.int32)
        send = np.zeros(4 * self.nLocal, dtype=np.int32)
        recv = np.zeros(4 * self.nLocal, dtype=np.int32)
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        check(lib().selfgpu_halo_plan(vp(si), mesh.nElem, nDomains, vp(self.offsets), rank, vp(self.sideInfo),
                                      ctypes.byref(nHalo), vp(counts), vp(send), vp(recv)))
        self.nHalo = nHalo.value
        self.peers = []  # (peer, send block indices, receive block indices)
        o = 0
        for p in range(nDomains):
            c = int(counts[p])
            if c:
                self.peers.append((p, send[o:o + c].copy(), recv[o:o + c].copy()))
            o += c

    def local_mesh(self, mesh):
        """The rank's Mesh2D: its elements' corner coordinates and the local sideInfo."""
        m = A.Mesh2D.from_arrays(mesh.nodeCoords[..., self.first:self.first + self.nLocal], self.sideInfo)
        m.nHalo = self.nHalo
        return m

    def local_slice(self):
        return slice(self.first, self.first + self.nLocal)


class DecomposedModel:
    """One rank's engine handle plus its halo exchange."""

    def __init__(self, model, plan):
        if model.nHalo != plan.nHalo:
            raise ValueError("the model must be built on plan.local_mesh(...)")
        self.model, self.plan = model, plan
        self._blocks = {p: (torch.from_numpy(s).cuda(), torch.from_numpy(r).cuda()) for p, s, r in plan.peers}
        self.primed = False

    def _caches(self):
        tr, vel = ctypes.c_void_p(), ctypes.c_void_p()
        tb, vb = ctypes.c_int(), ctypes.c_int()
        check(lib().selfgpu_model2d_caches(self.model._h, ctypes.byref(tr), ctypes.byref(tb), ctypes.byref(vel),
                                           ctypes.byref(vb)))
        out = [(tr.value, tb.value)]
        if vel.value:
            out.append((vel.value, vb.value))
        return out

    def post(self):
        """Packed outgoing blocks per peer (device uint8 tensors)."""
        self.model.Sync()
        out = {}
        for p, (send, _) in self._blocks.items():
            parts = []
            for ptr, bb in self._caches():
                buf = torch.empty(send.numel() * bb, device="cuda", dtype=torch.uint8)
                check(lib().selfgpu_pack_blocks(ctypes.c_void_p(ptr), send.data_ptr(), send.numel(), bb,
                                                buf.data_ptr(), None))
                parts.append(buf)
            out[p] = torch.cat(parts) if len(parts) > 1 else parts[0]
        torch.cuda.synchronize()
        return out

    def incoming_sizes(self):
        caches = self._caches()
        return {p: recv.numel() * sum(bb for _, bb in caches) for p, (_, recv) in self._blocks.items()}

    def deliver(self, incoming):
        """Unpack each peer's buffer into this rank's halo blocks."""
        for p, (_, recv) in self._blocks.items():
            buf, o = incoming[p], 0
            for ptr, bb in self._caches():
                n = recv.numel() * bb
                check(lib().selfgpu_unpack_blocks(buf[o:o + n].data_ptr(), recv.data_ptr(), recv.numel(), bb,
                                                  ctypes.c_void_p(ptr), None))
                o += n
        torch.cuda.synchronize()

    def SetSolution(self, values):
        self.model.SetSolution(values)
        self.primed = False

    def prologue(self):
        check(lib().selfgpu_model2d_prologue(self.model._h))
        self.primed = True

    def stage(self, dt, m):
        check(lib().selfgpu_model2d_stage(self.model._h, float(dt), int(m)))


def exchange_buffers(outgoing, sizes):
    """Send outgoing[p] (uint8 tensor) to each peer p and receive sizes[p]
    bytes from it, all as one batch of point-to-point operations over
    torch.distributed; returns {p: uint8 tensor} on the backend's device
    (CUDA for NCCL, host for gloo)."""
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    incoming = {p: torch.empty(n, dtype=torch.uint8, device=dev) for p, n in sizes.items()}
    ops = []
    for p in sorted(set(outgoing) | set(sizes)):
        if p in outgoing:
            ops.append(dist.P2POp(dist.isend, outgoing[p].to(dev), p))
        if p in sizes:
            ops.append(dist.P2POp(dist.irecv, incoming[p], p))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()
    return incoming


class TorchDistTransport:
    """Point-to-point exchange over torch.distributed (NCCL on GPUs, gloo on CPU)."""

    def exchange(self, dm, outgoing):
        incoming = exchange_buffers(outgoing, dm.incoming_sizes())
        return {p: t.cuda() for p, t in incoming.items()}

    def step(self, ranks, dt, nSteps):
        """nSteps RK3 steps of this process's rank (ranks = [DecomposedModel])."""
        (dm,) = ranks
        if not dm.primed:
            dm.prologue()
            dm.deliver(self.exchange(dm, dm.post()))
        for _ in range(nSteps):
            for m in range(3):
                dm.stage(dt, m)
                dm.deliver(self.exchange(dm, dm.post()))
        dm.model.t += nSteps * dt


class LocalTransport:
    """All ranks in one process (one GPU): stages are issued rank by rank from
    the host and the buffers moved between them in between; no kernel waits on
    another rank's kernel."""

    def exchange_all(self, ranks):
        out = {dm.plan.rank: dm.post() for dm in ranks}
        for dm in ranks:
            dm.deliver({p: out[p][dm.plan.rank] for p in dm._blocks})

    def step(self, ranks, dt, nSteps):
        if not all(dm.primed for dm in ranks):
            for dm in ranks:
                dm.prologue()
            self.exchange_all(ranks)
        for _ in range(nSteps):
            for m in range(3):
                for dm in ranks:
                    dm.stage(dt, m)
                self.exchange_all(ranks)
        for dm in ranks:
            dm.model.t += nSteps * dt
