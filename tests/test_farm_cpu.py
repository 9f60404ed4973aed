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


def test_read_sweep_orders_systems_as_the_reference_farm(tmp_path):
    """aphid_mpi.* files: MT gives the x- then the y-polarised source at every
    frequency, CS one dipole list per array at every frequency, frequencies
    fastest (src/aphid_parallel.f90:75-103)"""
    from aphid_git_b200 import model
    xn, yn, zn, sig, _ = model.serial_mt_model(5)
    model.write_mesh(str(tmp_path / "aphid.mesh"), xn, yn, zn, sig_re=sig)
    model.write_mpi_freq(str(tmp_path / "aphid_mpi.freq"), [0.01, 0.1, 1.0])
    model.write_mpi_input(str(tmp_path / "aphid_mpi.input"), "MT", 1e-10, 3000, "R")
    job = farm.read_sweep(str(tmp_path))
    assert job["sources"] == [2, 3] and job["source_of_system"] == [0, 0, 0, 1, 1, 1]
    assert np.allclose(np.array(job["omegas"]) / (2 * np.pi), [0.01, 0.1, 1.0] * 2)
    assert job["qmr_target"] == 1e-10 and job["qmr_max_it"] == 3000 and job["csig_flag"] == "R"
    assert np.allclose(job["mesh"]["zn"], zn, rtol=1e-5) and job["mesh"]["sig_re"].shape == (np.prod(sig.shape),)
    arrays = [[("+X", 2, 2, 3)], [("+X", 2, 2, 3), ("-Y", 3, 3, 3)]]
    model.write_mpi_source(str(tmp_path / "aphid_mpi.source"), arrays)
    model.write_mpi_input(str(tmp_path / "aphid_mpi.input"), "CS", 1e-8, 500, "R")
    job = farm.read_sweep(str(tmp_path))
    assert job["sources"] == [list(a) for a in arrays]
    assert job["source_of_system"] == [0, 0, 0, 1, 1, 1]


class FakeSolver:
    """stands in for Solver.sweep: x = omega + 10 source (+ x0 when given);
    fails when asked to solve the system with omega == fail_at"""

    def __init__(self, n, fail_at=None):
        self.n = n
        self.fail_at = fail_at

    def sweep(self, omegas, sources, sos, x0=None, **kw):
        if self.fail_at is not None and any(abs(w - self.fail_at) < 1e-12 for w in omegas):
            raise RuntimeError("device allocation failed")
        X = np.array([np.full(self.n, w + 10 * q) for w, q in zip(omegas, sos)], np.complex128)
        if x0 is not None:
            assert x0.shape == (len(omegas), self.n)
            X = X + x0
        self.last = X
        return X, [{"status_name": "converged", "omega": w} for w in omegas]

    def sweep_receivers(self, rec):
        rec = np.asarray(rec)
        E = self.last[:, None, :3] * rec.sum(axis=1)[None, :, None]
        return E, 2 * E


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
    # per-system initial guesses: each rank passes on its own rows
    x0 = np.arange(10)[:, None] * np.ones((10, 5))
    X0, _ = farm.sweep(FakeSolver(5), om, [[], [], []], sos, rank=rank, world=world, dist=dist, x0=x0)
    # receivers only: each rank ships E and H at the receivers, not solutions
    R, _ = farm.sweep(FakeSolver(5), om, [[], [], []], sos, rank=rank, world=world, dist=dist,
                      receivers=[[2, 2, 2], [3, 2, 2]])
    if rank == 0:
        q.put(("rec", R["E"], R["H"]))
    # a failing share raises on every rank (none waits in the gather)
    failed = None
    try:
        farm.sweep(FakeSolver(5, fail_at=om[0]), om, [[], [], []], sos, rank=rank, world=world, dist=dist)
    except farm.FarmError as e:
        failed = str(e)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, failed))
    if rank == 0:
        q.put((X, [i["omega"] for i in infos], X0))


def test_gloo_world2_gathers_every_system_once():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = [q.get(timeout=120) for _ in range(4)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    fails = {g[0]: g[1] for g in got if len(g) == 2 and not isinstance(g[0], str)}
    isrec = lambda g: isinstance(g[0], str)
    X, oms, X0 = [g for g in got if len(g) == 3 and not isrec(g)][0]
    _, RE, RH = [g for g in got if isrec(g)][0]
    assert RE.shape == (10, 2, 3) and np.allclose(RH, 2 * RE)
    om_ = [2 * np.pi * f for f in np.logspace(-3, 5, 10)]
    for s in range(10):
        assert np.allclose(RE[s, 1], 7 * (om_[s] + 10 * (s % 3)))
    assert set(fails) == {0, 1} and all(f and "device allocation failed" in f for f in fails.values())
    om = [2 * np.pi * f for f in np.logspace(-3, 5, 10)]
    assert np.allclose(oms, om)
    for s in range(10):
        assert np.allclose(X[s], om[s] + 10 * (s % 3))
        assert np.allclose(X0[s], om[s] + 10 * (s % 3) + s)


def test_farm_refuses_out():
    with pytest.raises(ValueError):
        farm.sweep(FakeSolver(5), [1.0], [[]], [0], out=np.zeros((1, 5), np.complex128))
