"""Multi-GPU sweep farm: the systems (frequency x source) of one sweep dealt
to one process per GPU, each solving its share with one batched sweep.  This
replaces the MPI farm of the reference (src/aphid_parallel.f90:179-201),
which gives each rank whole systems in turn; there is no collective in the
solve, only the results travel (gathered to rank 0 over torch.distributed:
NCCL between GPUs, gloo on CPUs).

Balance: low frequencies need the most iterations (diffusion over many
cells), so the systems are dealt by predicted cost, largest first, each to
the rank with the least work so far (longest-processing-time first).
"""
import numpy as np


def predicted_cost(freqs):
    """relative cost of a system at frequency f: iterations of the
    complex128 QMR to 1e-8 fall with frequency up to about 1e3 Hz (eval160,
    seed 901: 2135 at 1e-2 Hz, 1458 at 1 Hz, 968 at 1e2 Hz) and rise again
    above it towards the iteration cap (sweep128: the top decade does not
    converge)"""
    lf = np.log10(np.asarray(freqs, np.float64))
    return np.where(lf <= 3.0, 1.0 - 0.11 * (lf + 3.0), 0.34 + 0.3 * (lf - 3.0))


def assign(costs, nranks):
    """list of system indices per rank (LPT: largest first to the least
    loaded rank; ties to the lower rank)"""
    costs = np.asarray(costs, np.float64)
    load = np.zeros(nranks)
    parts = [[] for _ in range(nranks)]
    for s in sorted(range(len(costs)), key=lambda q: (-costs[q], q)):
        r = int(np.argmin(load))
        parts[r].append(s)
        load[r] += costs[s]
    return [sorted(p) for p in parts]


def gather(local, part, nsys, rank, world, dist=None):
    """rank 0 gets the per-system results of every rank in system order.
    local: list of per-system results (numpy arrays or dicts) of this rank's
    systems, in the order of `part`.  Other ranks get None."""
    if world == 1:
        return list(local)
    obj = list(zip(part, local))
    bucket = [None] * world if rank == 0 else None
    dist.gather_object(obj, bucket, dst=0)
    if rank != 0:
        return None
    out = [None] * nsys
    for lst in bucket:
        for s, v in lst:
            out[s] = v
    return out


class FarmError(RuntimeError):
    """A rank's share of the sweep failed; raised on every rank."""


def sweep(solver, omegas, sources, source_of_system, rank=0, world=1, dist=None, x0=None, receivers=None,
          **kw):
    """One sweep over `world` ranks (this process solves its share with
    solver.sweep).  Returns (X, infos) on rank 0, (None, None) elsewhere.

    x0 (optional): initial guesses of all systems, (nsys, nunk); each rank
    passes on the rows of its own systems.  The solutions come back through
    the gather, so solver.sweep's `out` array does not apply and is refused.
    receivers (optional): (nrec, 3) 1-based interior nodes; the solutions
    then stay on each rank's device and only E and H at the receivers
    (Solver.sweep_receivers) travel: the result is ({"E": (nsys, nrec, 3),
    "H": ...}, infos) on rank 0.
    If any rank's solve raises, every rank raises FarmError after the
    collective that shares the outcome, so no rank is left waiting in the
    gather."""
    if "out" in kw:
        raise ValueError("farm.sweep gathers the solutions to rank 0: `out` is not supported")
    nsys = len(omegas)
    freqs = np.asarray(omegas, np.float64) / (2 * np.pi)
    parts = assign(predicted_cost(freqs), world)
    mine = parts[rank]
    local, err = [], None
    try:
        if mine:
            if x0 is not None:
                kw["x0"] = np.asarray(x0).reshape(nsys, -1)[mine]
            if receivers is not None:
                kw["fetch"] = False
            X, infos = solver.sweep([omegas[s] for s in mine], sources, [source_of_system[s] for s in mine], **kw)
            if receivers is not None:
                E, H = solver.sweep_receivers(receivers)
                local = [((E[q], H[q]), infos[q]) for q in range(len(mine))]
            else:
                local = [(X[q] if X is not None else None, infos[q]) for q in range(len(mine))]
    except Exception as e:  # shared below, raised on every rank
        err = "rank %d: %s: %s" % (rank, type(e).__name__, e)
    if world > 1:
        errs = [None] * world
        dist.all_gather_object(errs, err)
        errs = [e for e in errs if e]
    else:
        errs = [err] if err else []
    if errs:
        raise FarmError("; ".join(errs))
    res = gather(local, mine, nsys, rank, world, dist)
    if res is None:
        return None, None
    if receivers is not None:
        return ({"E": np.stack([r[0][0] for r in res]), "H": np.stack([r[0][1] for r in res])},
                [r[1] for r in res])
    X = None if any(r[0] is None for r in res) else np.stack([r[0] for r in res])
    return X, [r[1] for r in res]


def read_sweep(directory):
    """The reference's farm inputs in `directory` (src/aphid_parallel.f90:45-103,
    formats of man/aphid.1): aphid_mpi.freq (frequencies), aphid_mpi.input
    (MT or CS, QMR target, iteration cap, conductivity model), aphid_mpi.source
    (CS only: the dipole arrays) and aphid.mesh.  The systems are ordered as
    the farm deals them to its ranks, frequencies fastest: MT is the x- and
    then the y-polarised sheet source (oper_mode 2, 3) at every frequency, CS
    one oper_mode-5 dipole list per array at every frequency.  Returns a dict
    with the mesh (xn, yn, zn, cell arrays), csig_flag, qmr_target,
    qmr_max_it, sources (as Solver.sweep takes them), omegas and
    source_of_system."""
    import os
    from . import model
    freqs = model.read_mpi_freq(os.path.join(directory, "aphid_mpi.freq"))
    inp = model.read_mpi_input(os.path.join(directory, "aphid_mpi.input"))
    mesh = model.read_mesh(os.path.join(directory, "aphid.mesh"), inp["csig_flag"])
    if inp["source_type"] == "MT":
        sources = [2, 3]
    elif inp["source_type"] == "CS":
        sources = [list(a) for a in model.read_mpi_source(os.path.join(directory, "aphid_mpi.source"))]
    else:
        raise ValueError("aphid_mpi.input: source type must be MT or CS, got %r" % inp["source_type"])
    omegas, sos = [], []
    for q in range(len(sources)):
        for f in freqs:
            omegas.append(2.0 * model.PI * float(f))
            sos.append(q)
    out = dict(mesh=mesh, sources=sources, omegas=omegas, source_of_system=sos, freqs=freqs)
    out.update(inp)
    return out


def sweep_files(solver, directory, rank=0, world=1, dist=None, precision="auto", receivers=None, **kw):
    """One farm sweep of the problem described by the reference's farm files
    in `directory` (read_sweep): every rank reads the files, binds the mesh
    and conductivity model, and solves its share of the systems.  Models R, C
    and I run as one batched sweep per rank.  Returns (results, infos, job)
    on rank 0 (results as in sweep()), (None, None, job) elsewhere."""
    job = read_sweep(directory)
    m = job["mesh"]
    solver.set_nodes(m["xn"], m["yn"], m["zn"])
    solver.set_model(job["csig_flag"], m.get("sig_re"), m.get("eps_rel"))
    res, infos = sweep(solver, job["omegas"], job["sources"], job["source_of_system"], rank=rank, world=world,
                       dist=dist, receivers=receivers, precision=precision, target=job["qmr_target"],
                       max_it=job["qmr_max_it"], **kw)
    return res, infos, job
