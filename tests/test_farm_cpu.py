"""The multi-GPU sweep farm's host logic on CPU: dealing of systems by
predicted cost, and a world-size-2 gloo run in which each rank "solves" its
share (a stand-in solver that returns recognisable vectors) and rank 0
gathers every system exactly once, in system order."""
import os
import socket

import numpy as np
import pytest

from aphid_git_b200 import farm


def test_assign_balances_and_covers():
    freqs = np.logspace(-3, 5, 24)
    c = farm.predicted_cost(freqs)
    for world in (1, 2, 3, 4, 8):
        parts = farm.assign(c, world)
        flat = sorted(s for p in parts for s in p)
        assert flat == list(range(24))
        loads = [c[p].sum() for p in parts]
        assert max(loads) - min(loads) <= c.max() + 1e-12  # LPT bound
    assert farm.assign([5, 1, 1, 1, 1, 1], 2) == [[0], [1, 2, 3, 4, 5]]


def test_low_frequencies_cost_more():
    c = farm.predicted_cost([1e-3, 1e-1, 1e1, 1e3])
    assert np.all(np.diff(c) < 0)


class FakeSolver:
    def __init__(self, n):
        self.n = n

    def sweep(self, omegas, sources, sos, **kw):
        X = np.array([np.full(self.n, w + 10 * q) for w, q in zip(omegas, sos)], np.complex128)
        return X, [{"status_name": "converged", "omega": w} for w in omegas]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    om = [2 * np.pi * f for f in np.logspace(-3, 5, 10)]
    sos = [s % 3 for s in range(10)]
    X, infos = farm.sweep(FakeSolver(5), om, [[], [], []], sos, rank=rank, world=world, dist=dist)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put((X, [i["omega"] for i in infos]))


def test_gloo_world2_gathers_every_system_once():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    X, oms = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    om = [2 * np.pi * f for f in np.logspace(-3, 5, 10)]
    assert np.allclose(oms, om)
    for s in range(10):
        assert np.allclose(X[s], om[s] + 10 * (s % 3))
