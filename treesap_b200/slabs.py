"""A domain shared by several processes, one z slab each (one GPU per process).

The reference distributes its boxes over MPI ranks and AMReX's FillPatch exchanges their ghost
cells (SingleLevelIntegrator.hpp:153-163). Here process r of W owns planes
[bounds[r], bounds[r+1]) of the domain (near-equal depths, `slab_bounds`) as one slab
integrator of the C ABI (ts_integrator_create_slab). A step takes every RK4 stage in lockstep:

    prepare(s); exchange(s); fill(s); launch(s)      for s in stages;   finish()

`exchange(s)` sends the slab's ngrow lowest valid planes to the lower neighbour and its ngrow
highest to the upper one, and receives theirs into its ghost planes (ranks r - 1 and r + 1;
in a domain periodic in z the first and last ranks are neighbours). The messages go through a
`comm` object; `TorchComm` wraps torch.distributed: over NCCL the planes move between GPUs as
device tensors (NVLink), over gloo as host tensors. The exchange is the same for any slab
backend: `GpuSlab` (the C ABI) or any object with the same six methods (the CPU tests use a
numpy slab), which is how the partition and exchange logic is tested on CPU ranks.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import TSError, WaveDesc, lib


def slab_bounds(nz: int, parts: int) -> list[int]:
    """First plane of each of `parts` near-equal slabs of nz planes, and nz at the end (the same
    split as ZSlabDomain.hpp's zslab_bounds)."""
    if parts < 1 or parts > nz:
        raise ValueError("need 1 <= parts <= nz")
    return [nz * k // parts for k in range(parts + 1)]


def neighbours(rank: int, world: int, periodic_z: bool) -> tuple[int | None, int | None]:
    """(lower, upper) neighbour ranks of `rank`; None where the slab touches a non-periodic face."""
    if world == 1:
        return None, None
    lo = rank - 1 if rank > 0 else (world - 1 if periodic_z else None)
    hi = rank + 1 if rank < world - 1 else (0 if periodic_z else None)
    return lo, hi


class _DevicePlanes:
    """A device-memory span exposed through __cuda_array_interface__ (zero-copy torch view)."""

    def __init__(self, ptr: int, elems: int, esize: int = 8):
        self.__cuda_array_interface__ = {"shape": (elems,), "typestr": f"<f{esize}", "data": (ptr, False),
                                         "version": 3, "strides": None}


class GpuSlab:
    """One slab through the C ABI (ts_integrator_create_slab and ts_slab_*)."""

    def __init__(self, ctx, desc: WaveDesc, zlo: int, nz: int, lo_ex: bool, hi_ex: bool):
        self.ctx = ctx
        self.handle = C.c_void_p()
        L = lib()
        st = L.ts_integrator_create_slab(ctx.handle, C.byref(desc), zlo, nz, int(lo_ex), int(hi_ex),
                                         C.byref(self.handle))
        if st != 0:
            raise TSError(st, "ts_integrator_create_slab", (L.ts_context_last_error(ctx.handle) or b"").decode())
        ctx._adopt(self)  # destroyed before the context
        self.ncomp = desc.ncomp()
        self.shape = (self.ncomp, nz, desc.n[1], desc.n[0])
        self.stages = L.ts_slab_stages(self.handle)

    def _ok(self, st: int, what: str) -> None:
        if st != 0:
            raise TSError(st, what, (lib().ts_context_last_error(self.ctx.handle) or b"").decode())

    def initialise(self, kind: int, items: np.ndarray) -> None:
        items = np.ascontiguousarray(items, dtype=np.float64).reshape(-1, 6)
        self._ok(lib().ts_integrator_initialise(self.handle, kind, len(items), items.ctypes.data), "initialise")

    def set_state(self, state: np.ndarray) -> None:
        a = np.ascontiguousarray(state, dtype=np.float64)
        assert a.shape == self.shape
        self._ok(lib().ts_integrator_set_state(self.handle, a.ctypes.data, 0), "set_state")
        self.ctx.sync()

    def get_state(self) -> np.ndarray:
        out = np.empty(self.shape)
        self._ok(lib().ts_integrator_get_state(self.handle, out.ctypes.data, 0), "get_state")
        return out

    def prepare(self, s: int) -> None:
        self._ok(lib().ts_slab_prepare(self.handle, s), "ts_slab_prepare")

    def _planes(self, s: int, face: int):
        p, elems, cs, es = C.c_void_p(), C.c_longlong(), C.c_longlong(), C.c_int()
        self._ok(lib().ts_slab_send_planes(self.handle, s, face, C.byref(p), C.byref(elems), C.byref(cs),
                                           C.byref(es)), "ts_slab_send_planes")
        return p.value, elems.value, cs.value, es.value

    def send_planes(self, s: int, face: int) -> list:
        """Per component, a device tensor viewing the planes to send across `face`."""
        import torch

        base, elems, cs, es = self._planes(s, face)
        return [torch.as_tensor(_DevicePlanes(base + es * c * cs, elems, es), device="cuda")
                for c in range(self.ncomp)]

    def receive_buffers(self, s: int, face: int) -> list:
        """Per component, a device tensor to receive the neighbour's planes into (one staging
        buffer of ncomp blocks per face and element type)."""
        import torch

        _, elems, _, es = self._planes(s, face)
        key = (face, elems, es)
        bufs = getattr(self, "_recv", {})
        if key not in bufs:
            dt = torch.float64 if es == 8 else torch.float32
            bufs[key] = torch.empty(self.ncomp * elems, dtype=dt, device="cuda")
            self._recv = bufs
        return list(bufs[key].view(self.ncomp, elems).unbind(0))

    def receive_planes(self, s: int, face: int, bufs: list) -> None:
        base = bufs[0].data_ptr()
        self._ok(lib().ts_slab_receive_planes(self.handle, s, face, C.c_void_p(base)), "ts_slab_receive_planes")

    def fill(self, s: int) -> None:
        self._ok(lib().ts_slab_fill(self.handle, s), "ts_slab_fill")

    def launch(self, s: int) -> None:
        self._ok(lib().ts_slab_launch(self.handle, s), "ts_slab_launch")

    def finish(self) -> None:
        self._ok(lib().ts_slab_finish(self.handle), "ts_slab_finish")

    def close(self) -> None:
        if self.handle:
            lib().ts_integrator_destroy(self.handle)
            self.handle = C.c_void_p()


class TorchComm:
    """Point-to-point plane exchange over torch.distributed (NCCL: device tensors; gloo: host
    tensors). `stream`: the CUDA stream the slab's kernels run on (the library's context
    stream), so that the transfers are ordered after the kernels that wrote the planes and
    before the ones that read them."""

    def __init__(self, stream: int | None = None):
        import torch.distributed as dist

        self.dist = dist
        self.stream = stream

    def exchange(self, sends: list[tuple[int, list]], recvs: list[tuple[int, list]]) -> None:
        """Posts every send (peer, tensors) and receive (peer, tensors) together and waits."""
        import contextlib

        import torch

        ctx = contextlib.nullcontext()
        if self.stream is not None and torch.cuda.is_available():
            ctx = torch.cuda.stream(torch.cuda.ExternalStream(self.stream))
        with ctx:
            ops = []
            for peer, ts in sends:
                ops += [self.dist.P2POp(self.dist.isend, t, peer) for t in ts]
            for peer, ts in recvs:
                ops += [self.dist.P2POp(self.dist.irecv, t, peer) for t in ts]
            if ops:
                for w in self.dist.batch_isend_irecv(ops):
                    w.wait()


class SlabDomain:
    """This process's slab of a domain split along z over `world` processes, and the lockstep
    stage loop with the halo exchange. `slab`: the slab backend built for planes
    [zlo, zlo + nz) (default: a GpuSlab on ctx)."""

    def __init__(self, desc: WaveDesc, rank: int, world: int, comm, ctx=None, slab=None):
        self.rank, self.world, self.comm = rank, world, comm
        self.bounds = slab_bounds(desc.n[2], world)
        self.zlo, self.zhi = self.bounds[rank], self.bounds[rank + 1]
        if self.zhi - self.zlo < desc.ngrow:
            raise ValueError("slabs thinner than the ghost width")
        self.lo, self.hi = neighbours(rank, world, bool(desc.periodic[2]))
        if slab is None:
            slab = GpuSlab(ctx, desc, self.zlo, self.zhi - self.zlo, self.lo is not None, self.hi is not None)
        self.slab = slab

    def exchange(self, s: int) -> None:
        """My lower planes go to the lower neighbour's upper ghosts and vice versa. Messages between
        one pair of ranks match in posting order, so when both faces talk to the same peer (two
        ranks, periodic in z) the receives are posted upper face first: my first send (lower
        planes) then meets the peer's first receive (its upper ghosts)."""
        sends, recvs, faces = [], [], []
        for face, peer in ((0, self.lo), (1, self.hi)):
            if peer is None:
                continue
            sends.append((peer, self.slab.send_planes(s, face)))
            bufs = self.slab.receive_buffers(s, face)
            recvs.append((peer, bufs))
            faces.append((face, bufs))
        if self.lo is not None and self.lo == self.hi:
            recvs.reverse()
        self.comm.exchange(sends, recvs)
        for face, bufs in faces:
            self.slab.receive_planes(s, face, bufs)

    def step(self, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            for s in range(self.slab.stages):
                self.slab.prepare(s)
                self.exchange(s)
                self.slab.fill(s)
                self.slab.launch(s)
            self.slab.finish()


def step_lockstep(domains: list[SlabDomain], nsteps: int = 1, stream: int | None = None) -> None:
    """Steps the slabs of several SlabDomains held by ONE process (e.g. on one GPU, or several
    GPUs driven by one process) in lockstep: per stage every slab's register step, then the halo
    exchange as device-to-device copies of the send planes into the peers' receive buffers, then
    every slab's ghost fill and stage kernel. `domains[r]` must be rank r of the same
    decomposition; `stream`: the CUDA stream of the slabs' kernels (the copies run on it)."""
    import contextlib

    import torch

    ctx = contextlib.nullcontext()
    if stream is not None:
        ctx = torch.cuda.stream(torch.cuda.ExternalStream(stream))
    stages = domains[0].slab.stages
    with ctx:
        for _ in range(nsteps):
            for s in range(stages):
                for d in domains:
                    d.slab.prepare(s)
                recv = {}
                for d in domains:
                    for face, peer in ((0, d.lo), (1, d.hi)):
                        if peer is not None:
                            recv[(d.rank, face)] = d.slab.receive_buffers(s, face)
                for d in domains:
                    for face, peer in ((0, d.lo), (1, d.hi)):
                        if peer is None:
                            continue
                        # my lower planes fill the lower neighbour's upper ghosts, and vice versa
                        for dst, src in zip(recv[(peer, 1 - face)], d.slab.send_planes(s, face)):
                            dst.copy_(src)
                for d in domains:
                    for face, peer in ((0, d.lo), (1, d.hi)):
                        if peer is not None:
                            d.slab.receive_planes(s, face, recv[(d.rank, face)])
                for d in domains:
                    d.slab.fill(s)
                    d.slab.launch(s)
            for d in domains:
                d.slab.finish()
