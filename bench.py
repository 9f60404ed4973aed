"""Benchmark: time-to-residual-1e-8 of a whole frequency sweep of APhiD's
frequency-domain solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload seafloor256] [--precision auto]

Workload (default): seafloor256, the full-scale configuration -- 256 x 256 x
192 cells (50.8 M unknowns per system), 10 air layers over 15 layers of
3.3 S/m seawater over a heterogeneous earth, one +X dipole on the sea floor,
24 frequencies log-spaced 1e-3..1e5 Hz.  One step is one sweep: all 24
systems solved from a zero start to a true FP64 relative residual of 1e-8,
batched in one persistent solve (aphid_gpu_sweep), AUTO precision (complex64
inner QMR in FP64 defect correction; systems whose Lanczos form collapses in
complex64 finish in complex128).

  value   sweeps/s with the model resident on the device (Solver.sweep, the
          solutions left on the device), K timed sweeps between CUDA events;
          the working set (about 120 GB) is far larger than L2, no flush.
  e2e     the same call with host buffers: the real(4) conductivity uploaded
          from pinned host memory and all solutions copied into a pinned host
          array inside the timed region (--e2e-steps sweeps, default 2).
  plain_fp64_sweep / fused64_sweep
          the same 24 systems through the reference's own complex128
          recurrence one system at a time (aphid_gpu_qmr path) and through the
          batched complex128 pass, timed once each; the speed-ups are their
          times over ours.
  field_err
          E and H at sea-floor receivers of the AUTO solutions against
          complex128 solves to 1e-12 (low, middle and high frequency).
  roofline
          the fused complex64 pass (k_sw_pass), timed with CUDA events on the
          sweep's stream over timing launches on the resident batch; plus the
          pass's effective bandwidth over a whole sweep.
  cpu_baseline / --impl reference
          the oracle's 4-thread component split (the reference's qmr_mthread
          parallelism, OMP_NUM_THREADS=4) on 4 pinned host cores, timed over a
          bounded sample of QMR iterations of the workload and extrapolated
          with the per-system complex128 iteration counts (measured in this
          run by the plain sweep; the reference arm, which runs no GPU code,
          uses the counts recorded by `bench.py --record-fp64-iters` in
          profiles/fp64_iters.json).

Multi-GPU: one process per GPU; the systems of the sweep are dealt to the
ranks by predicted cost (aphid_git_b200.farm, the reference's MPI farm split
over frequencies x sources), no collective in the solve, receiver values
gathered to rank 0; value = sweeps / max-over-ranks time ("strong": the total
work is one sweep at every N).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-residual-1e-8 per frequency sweep (reported as sweeps/s) and QMR iters/s"
TARGET = 1e-8
MAX_IT = 20000
ITERS_FILE = os.path.join(ROOT, "profiles", "fp64_iters.json")
CPU_THREADS = 4


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                t = [x.strip() for x in line.split(",")]
                if len(t) >= 9:
                    rows.append(t)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------------ workload
def systems_of(m):
    """(omega, source index) of every system, frequencies fastest, as the
    reference's MPI farm orders them (src/aphid_parallel.f90:97-101)."""
    om, sos = [], []
    for q in range(len(m.sources)):
        for f in m.freqs:
            om.append(2 * np.pi * float(f))
            sos.append(q)
    return om, sos


def receivers_of(m):
    """sea-floor (or surface) receivers: the nodes on the source's node layer
    along x through the source, every 4th node of the interior"""
    nx, ny, nz = m.dims
    _, _, jc, ks = m.sources[0][0]
    return np.array([[i, jc, ks] for i in range(2, nx, 4)], np.int32)


# ------------------------------------------------------------ CPU arms
def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def pin_cores(n=CPU_THREADS):
    """pin this process to its first n allowed cores (the OpenMP threads the
    oracle starts afterwards inherit the mask); returns (cores, old mask)"""
    old = sorted(os.sched_getaffinity(0))
    cores = old[:n]
    os.sched_setaffinity(0, cores)
    return cores, old


def cpu_sample(m, iters, threads=CPU_THREADS):
    """seconds per QMR iteration of the oracle's 4-thread component split
    (the reference's qmr_mthread parallelism, src/aphid_qmr.f90:744-928) on
    the first system of the workload, on pinned cores: two runs of a and
    a + iters iterations, s/iter = (t(a + iters) - t(a)) / iters, so that the
    fixed start-up of a solve (thread spin-up, first touch of the work
    vectors, the initial residual) is not charged to the iterations.  (A
    plain short run over-states the steady rate: 6 iterations on hetero96
    gave 0.149 s/iter against 0.061 s/iter over a full 1082-iteration
    solve.)  Returns (s/iter, iterations timed, cores)."""
    from aphid_git_b200 import model
    from oracle import oracle as O
    cores, old = pin_cores(threads)
    try:
        w = 2 * np.pi * float(m.freqs[0])
        sig = model.sigma_hat("R", w, m.sig_re.ravel(order="F"))
        b, _ = model.gen_rhs(m.xn, m.yn, m.zn, 5, m.sources[0])
        g = O.Grid(m.xn, m.yn, m.zn)
        k2 = O.gen_k2(g, sig, w)
        diag = O.gen_diag(g, k2)
        a = 3
        ra = O.qmr(g, k2, diag, b, 1e-30, a, nthreads=threads)
        # on small meshes the difference of two short runs is within the
        # timer's noise: lengthen the sample until it spans half a second
        while True:
            rb = O.qmr(g, k2, diag, b, 1e-30, a + iters, nthreads=threads)
            done = len(rb["hist"]) - len(ra["hist"])
            dt = rb["seconds"] - ra["seconds"]
            if dt >= 0.5 or iters >= 4096 or done < iters:
                break
            iters *= 4
        return max(dt, 1e-9) / max(1, done), done, cores
    finally:
        os.sched_setaffinity(0, old)


def recorded_iters(workload):
    try:
        with open(ITERS_FILE) as f:
            d = json.load(f)[workload]
        return [int(v) for v in d["iters"]], d.get("source", "")
    except Exception:
        return None, None


def cpu_baseline_obj(spi, done, cores, iters, iters_src, nsys_per_sweep):
    total = int(sum(iters))
    return {"value": 1.0 / (spi * total), "unit": "sweeps/s", "cores": len(cores), "kind": "port",
            "cpu": cpu_model(), "pinned_cores": cores, "s_per_iter": spi,
            "sample": "%d QMR iterations of the first system (difference of a 3- and a longer run), "
                      "oracle 4-thread component split on %d pinned cores; time-to-tolerance "
                      "extrapolated = %.3f s/iter x %d complex128 "
                      "iterations summed over the %d systems (%s)"
                      % (done, len(cores), spi, total, nsys_per_sweep, iters_src)}


def run_reference(args):
    """--impl reference: the CPU restatement of the reference's path (the
    reference is Fortran + MPI; no Fortran compiler exists here, so no
    oracle/_ref), timed on this host's cores.  Rank 0 only."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from aphid_git_b200 import model
    m = model.make_model(args.workload)
    om, _ = systems_of(m)
    iters, src = recorded_iters(args.workload)
    if iters is None or len(iters) != len(om):
        print(json.dumps({"impl": "reference", "unavailable":
                          "no recorded complex128 iteration counts for %s in profiles/fp64_iters.json "
                          "(run bench.py --record-fp64-iters on a GPU)" % args.workload}))
        return 0
    times, done, cores = [], 0, []
    for step in range(args.warmup + args.steps):
        spi, done, cores = cpu_sample(m, args.cpu_sample_iters)
        if step >= args.warmup:
            times.append(spi)
    spi = float(np.mean(times))
    cb = cpu_baseline_obj(spi, done, cores, iters, "recorded on B200 in " + os.path.basename(ITERS_FILE)
                          + ": " + src, len(om))
    value = cb["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "sweeps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": args.workload, "precision": "complex128 (the reference's algorithm, CPU)",
                   "unknowns": int(m.n), "systems": len(om), "target": TARGET,
                   "parallelism": "one process, 4 threads (qmr_mthread component split)"},
        "s_per_iter": spi, "iters_to_tol": iters, "extrapolated": True,
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------ GPU arm
def pass_bytes(nsys, n):
    """Algorithmic bytes of one fused complex64 QMR pass over a batch: per
    unknown and system read q^, v^, p^ and write q^, v^, p^ (6 x 8 B; the
    Jacobi diagonal is formed on chip), plus the shared FP32 sigma-bar once
    (4 B).  The solution update runs outside the pass, once per R passes
    (update_bytes)."""
    return nsys * n * 48 + n * 4


def update_bytes(nsys, n, ring):
    """Algorithmic bytes of one flush of the pending solution updates
    (k_sw_dxupd): per unknown and system read R p^ slots and d^ (complex64)
    and x (complex128), write d^ and x"""
    return nsys * n * ((ring + 2) * 8 + 32)


def timed(stream, dev, fn, steps, barrier, world):
    """Run fn() `steps` times between CUDA events on `stream`, barrier and
    synchronize on both sides; returns (ms max over ranks, results)."""
    import torch
    import torch.distributed as dist
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = [fn() for _ in range(steps)]
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, out


def field_error(s, m, om, sos, rec, Ea, Ha, Xa, idx):
    """E and H of systems idx of a finished sweep (receiver values Ea, Ha;
    solutions Xa[q] fetched right after it) against complex128 solves of the
    reference's recurrence to 1e-12, beside the error of that recurrence
    itself stopped at the same 1e-8 target.

    Two measures per system: the relative error over the whole mesh (E on
    the edges, B on the faces, from gen_fields) and at the receivers.  A
    1e-8 residual resolves a field only down to about 1e-8 of the largest
    one, so the receiver bound has a floor: where the receivers see a field
    that is a fraction f of the mesh-wide one (at 1e5 Hz in seawater the
    receivers 2 km from the source see rounding noise of the source region's
    field), no solve to 1e-8 fixes it better than 1e-8 / f.  Bounds:
    mesh-wide max(1e-6, 2 x the reference's own error); receivers the same
    or 1e-8 / f, whichever is larger."""
    sub = ([om[q] for q in idx], m.sources, [sos[q] for q in idx])
    err = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    oms = [om[q] for q in idx]
    s.sweep(*sub, precision="fp64", target=1e-12, max_it=4 * MAX_IT, fetch=False)
    Er, Hr = s.sweep_receivers(rec)
    Xr = [s.sweep_fetch(r) for r in range(len(idx))]
    s.sweep(*sub, precision="fp64", target=TARGET, max_it=4 * MAX_IT, fetch=False)
    E8, H8 = s.sweep_receivers(rec)
    X8 = [s.sweep_fetch(r) for r in range(len(idx))]
    out = {"freq_hz": [w / (2 * np.pi) for w in oms]}
    for key in ("E", "H"):
        out[key] = {k: [] for k in ("mesh", "mesh_reference_at_1e-8", "mesh_bound", "receivers",
                                    "receivers_reference_at_1e-8", "receiver_field_fraction", "receivers_bound")}
    ok = True
    for r, q in enumerate(idx):  # one system at a time: three mesh-wide (B, E) pairs in host memory
        Fa, Fr, F8 = (s.gen_fields(oms[r], x) for x in (Xa[q], Xr[r], X8[r]))
        for key, ra, rr, r8, fi in (("E", Ea, Er, E8, 1), ("H", Ha, Hr, H8, 0)):
            mesh, mesh8 = err(Fa[fi], Fr[fi]), err(F8[fi], Fr[fi])
            recv, recv8 = err(ra[q], rr[r]), err(r8[r], rr[r])
            # the receivers' share of the field: their rms against the
            # largest field on the mesh (H = B / mu0 at the receivers; B on
            # the mesh), the scale a 1e-8 residual resolves to
            scale = 1.0 if key == "E" else 4e-7 * np.pi
            rec_rms = np.linalg.norm(rr[r]) * scale / np.sqrt(rr[r].size)
            mesh_max = float(np.max(np.abs(Fr[fi])))
            frac = float(rec_rms / max(mesh_max, 1e-300))
            b_mesh = max(1e-6, 2 * mesh8)
            b_recv = max(1e-6, 2 * recv8, 1e-8 / max(frac, 1e-300))
            ok = ok and mesh <= b_mesh and recv <= b_recv
            o = out[key]
            for k, v in (("mesh", mesh), ("mesh_reference_at_1e-8", mesh8), ("mesh_bound", b_mesh),
                         ("receivers", recv), ("receivers_reference_at_1e-8", recv8),
                         ("receiver_field_fraction", frac), ("receivers_bound", b_recv)):
                o[k].append(v)
        del Fa, Fr, F8
    return {"E": max(out["E"]["mesh"]), "H": max(out["H"]["mesh"]),
            "E_receivers": max(out["E"]["receivers"]), "H_receivers": max(out["H"]["receivers"]),
            "within_bound": ok, "per_system": out,
            "reference": "complex128 Jacobi-QMR (reference recurrence) to 1e-12",
            "bound": "mesh-wide: max(1e-6, 2 x the reference recurrence's own error at 1e-8); receivers: "
                     "the same or 1e-8 / (receiver rms field / largest mesh field), whichever is larger",
            "receivers": int(len(rec))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="seafloor256")
    ap.add_argument("--precision", default="auto", choices=["mixed", "auto", "fused64"])
    ap.add_argument("--inner-tol", type=float, default=0.0)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain complex128 sweep")
    ap.add_argument("--no-fused64", action="store_true", help="skip the batched complex128 sweep")
    ap.add_argument("--no-field-err", action="store_true")
    ap.add_argument("--cpu-sample-iters", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--record-fp64-iters", action="store_true",
                    help="write the plain sweep's per-system iteration counts to profiles/fp64_iters.json")
    ap.add_argument("--one-sweep", action="store_true",
                    help="run one sweep of the workload and exit (profiling target)")
    ap.add_argument("--only-apply", action="store_true",
                    help="set up the workload and time only the fused pass (profiling)")
    ap.add_argument("--freqs", default="",
                    help="comma-separated frequencies (Hz) in place of the workload's own (profiling batches)")
    ap.add_argument("--verbose", action="store_true",
                    help="the library reports its tuning and sweep phases on stderr")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from aphid_git_b200 import Solver, farm, model

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    # a real stream shared by the library and the CUDA events
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)

    def barrier():
        if world > 1:
            dist.barrier()

    m = model.make_model(args.workload)
    if args.freqs:
        m.freqs = np.array([float(f) for f in args.freqs.split(",")])
    s = Solver(device=local, stream=stream.cuda_stream, verbose=args.verbose)
    s.set_nodes(m.xn, m.yn, m.zn)
    n = s.n
    om, sos = systems_of(m)
    nsys = len(om)
    rec = receivers_of(m)
    parts = farm.assign(farm.predicted_cost(np.array(om) / (2 * np.pi)), world)
    mine = parts[rank]
    my_om, my_sos = [om[q] for q in mine], [sos[q] for q in mine]
    peak, peak_kind = peaks()
    s.set_model("R", m.sig_re)

    def sweep(prec=args.precision, out=None):
        if not mine:
            return []
        return s.sweep(my_om, m.sources, my_sos, precision=prec, target=TARGET, max_it=MAX_IT,
                       inner_tol=args.inner_tol, fetch=False if out is None else True, out=out)[1]

    if args.one_sweep:
        inf = sweep()
        print(json.dumps({"workload": args.workload, "precision": args.precision, "systems": len(mine),
                          "plane_kz_last_pass": s.sweep_plane_kz(),
                          "inner_iters": [i["inner_iters"] for i in inf],
                          "inner64_iters": [i["inner64_iters"] for i in inf],
                          "status": [i["status_name"] for i in inf],
                          "true_rel_resid": [i["true_rel_resid"] for i in inf],
                          "seconds": inf[0]["seconds"], "launches": inf[0]["kernel_launches"]}))
        return 0
    if args.only_apply:
        sweep("mixed" if args.precision == "auto" else args.precision)
        ms_a, _ = timed(stream, dev, lambda: s.sweep_time_apply(10), 1, lambda: None, 1)
        t = ms_a * 1e-3 / 10
        print(json.dumps({"apply_us": t * 1e6, "unknowns": n, "systems": len(mine),
                          "alg_GBps": pass_bytes(len(mine), n) / t / 1e9}))
        return 0

    # ---- the timed region: K sweeps, inputs resident
    for _ in range(args.warmup):
        sweep()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    def farm_sweep():
        # N > 1: the farm deals the systems by predicted cost, each rank solves
        # its share in one batched sweep, and E, H at the receivers are
        # gathered to rank 0 (the solutions stay on the ranks' devices)
        _, inf = farm.sweep(s, om, m.sources, sos, rank=rank, world=world, dist=dist, receivers=rec,
                            precision=args.precision, target=TARGET, max_it=MAX_IT, inner_tol=args.inner_tol)
        return [inf[q] for q in mine] if inf is not None else []

    ms, infs = timed(stream, dev, farm_sweep if world > 1 else sweep, args.steps, barrier, world)
    clk = clocks.stop()
    last = infs[-1]
    launches = int(sum(i[0]["kernel_launches"] for i in infs if i))
    value = args.steps / (ms * 1e-3)
    Ea, Ha = s.sweep_receivers(rec) if mine else (None, None)
    # the solutions of the field check's systems (lowest, middle, highest
    # frequency of this rank), before the comparison legs overwrite them
    idx_f = sorted({0, len(mine) // 2, len(mine) - 1}) if mine else []
    Xa = {q: s.sweep_fetch(q) for q in idx_f} if not args.no_field_err else {}

    # ---- e2e: host buffers, copies inside the timed region
    sig_host = torch.empty(m.sig_re.shape[::-1], dtype=torch.float32, pin_memory=True).numpy().T
    sig_host[...] = m.sig_re
    x_host = torch.empty((max(1, len(mine)), n), dtype=torch.complex128, pin_memory=True).numpy()

    def run_e2e():
        s.set_model("R", sig_host)
        return sweep(out=x_host[:len(mine)])

    e2e_steps = max(1, args.e2e_steps)
    ms_e, _ = timed(stream, dev, run_e2e, e2e_steps, barrier, world)
    e2e = {"value": e2e_steps / (ms_e * 1e-3), "unit": "sweeps/s", "steps": e2e_steps,
           "h2d_bytes_per_step": 4 * m.ncell, "d2h_bytes_per_step": 16 * n * len(mine),
           "note": "real(4) conductivity host->device and every solution device->host (pinned) "
                   "inside the timed region"}
    del x_host

    it_in = [i["inner_iters"] for i in last]
    extra = {"time_to_tol_s": ms / args.steps * 1e-3, "systems": nsys, "systems_this_rank": len(mine),
             "inner_iters": it_in, "inner_iters_total": int(sum(it_in)),
             "inner64_iters_total": int(sum(i["inner64_iters"] for i in last)),
             "outer_iters_max": max(i["outer_iters"] for i in last) if last else 0,
             "qmr_iters_per_s": world * sum(it_in) / (ms / args.steps * 1e-3),
             "cell_updates_per_s": world * sum(it_in) * m.ncell / (ms / args.steps * 1e-3),
             "true_rel_resid_max": max(i["true_rel_resid"] for i in last) if last else None,
             "status": sorted({i["status_name"] for i in last}), "plane_kz_last_pass": s.sweep_plane_kz()}

    # ---- the dominant kernel: the fused complex64 pass
    reps = 10
    if mine:  # the complex64 state of the whole batch (AUTO releases it after escalation)
        s.sweep(my_om, m.sources, my_sos, precision="mixed", target=TARGET, max_it=8, fetch=False)
        s.sweep_time_apply(2)
    ms_a, _ = timed(stream, dev, lambda: s.sweep_time_apply(reps) if mine else None, 1, lambda: None, 1)
    t_apply = max(ms_a, 1e-9) * 1e-3 / reps
    alg = pass_bytes(len(mine), n)
    achieved = alg / t_apply / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get("sw_pass_" + args.workload)
    roofline = {"bound": "hbm", "kernel": "k_sw_pass (fused complex64 QMR iteration: v^, p^ update, "
                "q^ = D^-1 K p^, 12 inner products)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, burst)",
                "traffic": traffic, "alg_bytes_per_launch": alg, "launch_us": t_apply * 1e6,
                "systems_per_launch": len(mine),
                "units": "48 B per unknown and system + 4 B sigma-bar per unknown"}

    # ---- comparisons on the same GPU (rank 0's share at N > 1)
    if not args.no_plain:  # every rank takes the same collective steps
        ms_p, inf_p = timed(stream, dev, lambda: sweep("fp64"), 1, barrier, world)
        pi = inf_p[-1] or [{"iters": 0, "status_name": "none"}]
        extra["plain_fp64_sweep"] = {
            "time_s": ms_p * 1e-3, "iters": [i["iters"] for i in pi],
            "status": sorted({i["status_name"] for i in pi}),
            "note": "complex128 Jacobi-QMR, the reference's recurrence and stop test, one system at a "
                    "time on the same GPU (k_apply64 + streaming kernels, graph-captured)"}
        extra["speedup_vs_plain_fp64_sweep"] = ms_p / (ms / args.steps)
        if args.record_fp64_iters and world == 1:
            d = {}
            if os.path.exists(ITERS_FILE):
                with open(ITERS_FILE) as f:
                    d = json.load(f)
            d[args.workload] = {"iters": [i["iters"] for i in pi], "freq_hz": [w / (2 * np.pi) for w in om],
                                "source": "bench.py --workload %s --record-fp64-iters, plain complex128 sweep "
                                          "on %s" % (args.workload, torch.cuda.get_device_name(dev))}
            with open(ITERS_FILE, "w") as f:
                json.dump(d, f, indent=1)
    if not args.no_fused64:
        try:
            # the first FUSED64 sweep of a batch size tunes the complex128
            # pass (24 timed configurations, about 3 s on seafloor256): one
            # untimed sweep runs first, so that the leg times the solve alone
            sweep("fused64")
            ms_f, inf_f = timed(stream, dev, lambda: sweep("fused64"), 1, barrier, world)
            fi = inf_f[-1] or [{"inner_iters": 0, "status_name": "none"}]
            extra["fused64_sweep"] = {"time_s": ms_f * 1e-3, "iters": [i["inner_iters"] for i in fi],
                                      "status": sorted({i["status_name"] for i in fi}),
                                      "note": "batched complex128 pass (k_sw_pass64) for every system, in "
                                              "as many chunks as device memory holds",
                                      "tuned_before_timing": True}
            extra["speedup_vs_fused64_sweep"] = ms_f / (ms / args.steps)
        except Exception as e:  # a comparison leg: report, keep the line
            extra["fused64_sweep"] = {"error": str(e)}
    if not args.no_field_err and mine:
        try:
            extra["field_err"] = field_error(s, m, my_om, my_sos, rec, Ea, Ha, Xa, idx_f)
        except Exception as e:
            extra["field_err"] = {"error": str(e)}
    # effective bandwidth of the inner iterations over a whole sweep (all
    # kernels' time): 48 B per pass and unknown, plus the updates at R = 4
    extra["sweep_effective_GBps"] = (sum(it_in) * (48.0 + 64.0 / 4) * n) / (ms / args.steps * 1e-3) / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": {"mixed": "c64 inner / f64 outer", "fused64": "c128 inner / f64 outer",
                  "auto": "c64 inner (c128 after escalation) / f64 outer"}[args.precision],
        "data": "synthetic (seeded generator, no public dataset)",
        "config": {"workload": args.workload, "precision": args.precision, "unknowns": n,
                   "systems": nsys, "target": TARGET, "max_it": MAX_IT,
                   "l2": "working set > L2 (126 MB), no flush",
                   "parallelism": "systems dealt to ranks (farm), one batched sweep per rank"},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk, "roofline": roofline,
    }
    line.update(extra)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        iters = extra.get("plain_fp64_sweep", {}).get("iters")
        src = "measured by the plain sweep in this run"
        if iters is None:
            iters, src = recorded_iters(args.workload)
            src = "recorded: %s" % src
        if iters:
            try:
                spi, done, cores = cpu_sample(m, args.cpu_sample_iters)
                line["cpu_baseline"] = cpu_baseline_obj(spi, done, cores, iters, src, nsys)
                line["cpu_baseline"]["extrapolated"] = True
            except Exception as e:
                line["cpu_baseline"] = {"error": str(e)}
    s.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
