"""The multi-process z-slab exchange (treesap_b200/slabs.py) on CPU ranks over gloo.

SlabDomain drives any slab backend with the six stage calls of ts_slab_* (prepare, send_planes,
receive_buffers, receive_planes, fill, launch, finish). Here the backend is a numpy slab of the
same protocol: the scalar wave (phi, pi), 4th-order centred D2 in x, y (periodic, by rolling)
and z (ghost planes), RK4 with the reference's register scheme, z ghosts Dirichlet 0 or
periodic. Two and three gloo ranks each own a slab; the gathered result must be bitwise the
single-process run of the same backend over the whole domain, for non-periodic and periodic z
(with two ranks periodic in z both faces talk to the same peer, which checks the message order).
The GPU side of the protocol (the C ABI slab integrator) is the same code path as
tests/test_gpu_slab_ranks.py, which runs the domain's slabs in one process on one GPU.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
G = 2
W2 = (4.0 / 3.0, -1.0 / 12.0)  # D2 weights of half-width 2
W0 = -2.5


class NumpySlab:
    """Planes [zlo, zlo + nz) of an n^3-cell wave problem, z ghost planes of width G."""

    stages = 4

    def __init__(self, n, zlo, nz, lo_ex, hi_ex, periodic_z, dt):
        self.n, self.zlo, self.nz, self.lo_ex, self.hi_ex, self.per = n, zlo, nz, lo_ex, hi_ex, periodic_z
        self.dt, self.dx = dt, 1.0 / n
        shape = (2, nz + 2 * G, n, n)
        self.old, self.new, self.arg, self.argn = (np.zeros(shape) for _ in range(4))
        self.t = 0.0

    def set_state(self, s):
        self.old[:, G:G + self.nz] = s

    def get_state(self):
        return self.old[:, G:G + self.nz].copy()

    def _input(self, s):
        return self.old if s == 0 else self.arg

    def prepare(self, s):
        if s > 0:
            self.arg, self.argn = self.argn, self.arg

    def send_planes(self, s, face):
        f = self._input(s)
        sl = slice(G, 2 * G) if face == 0 else slice(self.nz, self.nz + G)
        return [torch.from_numpy(np.ascontiguousarray(f[c, sl]).ravel()) for c in range(2)]

    def receive_buffers(self, s, face):
        return [torch.zeros(G * self.n * self.n, dtype=torch.float64) for _ in range(2)]

    def receive_planes(self, s, face, bufs):
        f = self._input(s)
        sl = slice(0, G) if face == 0 else slice(self.nz + G, self.nz + 2 * G)
        for c in range(2):
            f[c, sl] = bufs[c].numpy().reshape(G, self.n, self.n)

    def fill(self, s):
        f = self._input(s)
        if not self.lo_ex:
            f[:, :G] = f[:, self.nz:self.nz + G] if self.per else 0.0
        if not self.hi_ex:
            f[:, self.nz + G:] = f[:, G:2 * G] if self.per else 0.0

    def _rhs(self, f):
        phi = f[0]
        c = phi[G:G + self.nz]
        lap = np.zeros_like(c)
        for ax in (1, 2):  # y, x: periodic
            acc = W0 * c
            for s, w in enumerate(W2, start=1):
                acc = acc + w * (np.roll(c, s, axis=ax) + np.roll(c, -s, axis=ax))
            lap = lap + acc / self.dx**2
        acc = W0 * c
        for s, w in enumerate(W2, start=1):
            acc = acc + w * (phi[G + s:G + s + self.nz] + phi[G - s:G - s + self.nz])
        lap = lap + acc / self.dx**2
        return np.stack([f[1, G:G + self.nz], lap])

    def launch(self, s):
        a = (0.0, 0.5, 0.5, 1.0)
        b = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)
        k = self._rhs(self._input(s))
        v = slice(G, G + self.nz)
        init = self.old[:, v]
        if s == 0:
            self.new[:, v] = init + self.dt * b[0] * k
        else:
            self.new[:, v] = self.new[:, v] + self.dt * b[s] * k
        if s < 3:
            self.argn[:, v] = init + self.dt * a[s + 1] * k

    def finish(self):
        self.old, self.new = self.new, self.old
        self.t += self.dt


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _initial(n):
    x = (np.arange(n) + 0.5) / n
    z, y, xx = np.meshgrid(x, x, x, indexing="ij")
    phi = np.exp(-((xx - 0.5) ** 2 + (y - 0.45) ** 2 + (z - 0.55) ** 2) / 0.15**2)
    return np.stack([phi, np.zeros_like(phi)])


class _Desc:
    """The descriptor fields SlabDomain reads."""

    def __init__(self, n, periodic_z):
        self.n = (n, n, n)
        self.ngrow = G
        self.periodic = (1, 1, int(periodic_z))


def _worker(rank, world, port, n, periodic_z, steps, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    from treesap_b200.slabs import SlabDomain, TorchComm, neighbours, slab_bounds

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b = slab_bounds(n, world)
    lo, hi = neighbours(rank, world, periodic_z)
    slab = NumpySlab(n, b[rank], b[rank + 1] - b[rank], lo is not None, hi is not None, periodic_z, 0.25 / n)
    slab.set_state(_initial(n)[:, b[rank]:b[rank + 1]])
    dom = SlabDomain(_Desc(n, periodic_z), rank, world, TorchComm(), slab=slab)
    dom.step(steps)
    q.put((rank, slab.get_state()))
    dist.barrier()
    dist.destroy_process_group()


def _run_ranks(world, n, periodic_z, steps):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, n, periodic_z, steps, q)) for r in range(world)]
    for p in ps:
        p.start()
    parts = dict(q.get(timeout=180) for _ in range(world))
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    return np.concatenate([parts[r] for r in range(world)], axis=1)


@pytest.mark.parametrize("world,periodic_z", [(2, False), (2, True), (3, True), (3, False)])
def test_ranks_reproduce_the_single_slab_run(world, periodic_z):
    n, steps = 12, 5
    whole = NumpySlab(n, 0, n, False, False, periodic_z, 0.25 / n)
    whole.set_state(_initial(n))
    for _ in range(steps):
        for s in range(4):
            whole.prepare(s)
            whole.fill(s)
            whole.launch(s)
        whole.finish()
    got = _run_ranks(world, n, periodic_z, steps)
    assert np.abs(whole.get_state()).max() > 0.1
    assert np.array_equal(got, whole.get_state())


def test_partition_and_neighbours():
    from treesap_b200.slabs import neighbours, slab_bounds

    assert slab_bounds(256, 4) == [0, 64, 128, 192, 256]
    assert slab_bounds(10, 3) == [0, 3, 6, 10]
    assert neighbours(0, 1, True) == (None, None)
    assert neighbours(0, 3, False) == (None, 1) and neighbours(2, 3, False) == (1, None)
    assert neighbours(0, 3, True) == (2, 1) and neighbours(2, 3, True) == (1, 0)
    assert neighbours(0, 2, True) == (1, 1)
    with pytest.raises(ValueError):
        slab_bounds(3, 4)
