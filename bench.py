"""Benchmark: time-to-residual-1e-8 of APhiD's frequency-domain solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload hetero96] [--precision fp64]

One step = one full solve of the workload to relative residual 1e-8 from a
zero start.  `value` = sweeps per second over all ranks, measured on device
with CUDA events, inputs resident in HBM (aphid_gpu_qmr_run); `e2e` = the same
through the public host-buffer call (aphid_gpu_qmr: host->device copies of
k^2, the Jacobi diagonal and b, device->host copy of the solution, inside the
timed region).  The working set (10 complex128 vectors of 3.6 M unknowns,
580 MB) is larger than L2, so no explicit flush is needed.

Multi-GPU: one process per GPU, each solving its own sweep (the reference's
MPI farm is an embarrassingly parallel split over frequencies x sources), no
collective in the solve; value = sweeps of all ranks / max-over-ranks time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-residual-1e-8 per frequency sweep (reported as sweeps/s) and QMR iters/s"
TARGET = 1e-8
MAX_IT = 20000
# Iterations to relative residual 1e-8 of the complex128 Jacobi-QMR (the
# reference's own recurrence and stop test) on each workload, measured on the
# B200 complex128 path, which reproduces the reference's iteration count.  The
# CPU arms time a bounded number of iterations and extrapolate with it.
FP64_ITERS = {"halfspace32": 360, "hetero96": 1088}


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


def setup_problem(workload):
    from aphid_git_b200 import model
    m = model.make_model(workload)
    w = 2 * np.pi * float(m.freqs[0])
    sig = model.sigma_hat("R", w, m.sig_re.ravel(order="F"))
    b, _ = model.gen_rhs(m.xn, m.yn, m.zn, 5, m.sources[0])
    return m, w, sig, b


def cpu_port_sample(workload, iters, threads=4):
    """The oracle's 4-thread component split (the reference's qmr_mthread
    parallelism, src/aphid_qmr.f90:744-928) for `iters` iterations.
    Returns seconds per iteration."""
    from oracle import oracle as O
    m, w, sig, b = setup_problem(workload)
    g = O.Grid(m.xn, m.yn, m.zn)
    k2 = O.gen_k2(g, sig, w)
    diag = O.gen_diag(g, k2)
    r = O.qmr(g, k2, diag, b, 1e-30, iters, nthreads=threads)
    return r["seconds"] / max(1, len(r["hist"])), len(r["hist"])


def run_reference(args):
    """--impl reference: the CPU port of the reference's path (no Fortran
    compiler exists here, so oracle/_ref cannot be built)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    iters = FP64_ITERS.get(args.workload)
    from aphid_git_b200 import model
    m = model.make_model(args.workload)
    sample_it = args.cpu_sample_iters
    times = []
    for step in range(args.warmup + args.steps):
        spi, done = cpu_port_sample(args.workload, sample_it)
        if step >= args.warmup:
            times.append(spi)
    spi = float(np.mean(times))
    value = 1.0 / (spi * iters) if iters else None
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "sweeps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": spi * iters * 1e3 if iters else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": args.workload, "precision": "complex128 (the reference's algorithm, CPU)",
                   "unknowns": int(m.n), "systems": len(systems_of(m)[0]), "target": TARGET,
                   "parallelism": "one process, 4 threads (qmr_mthread component split)"},
        "s_per_iter": spi, "iters_to_tol": iters,
        "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": 4, "kind": "port",
                         "sample": "%d QMR iterations per step, 4-thread component split; "
                                   "time-to-tolerance = s/iter x %s iterations" % (sample_it, iters)},
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def pass_bytes(nsys, n):
    """Algorithmic bytes of one fused complex64 QMR pass over a batch: per
    unknown and system read q^, v^, p^, d^, x^ and write q^, v^, p^, d^, x^
    (10 x 8 B; the Jacobi diagonal is formed on chip), plus the shared FP32
    sigma-bar once (4 B)."""
    return nsys * n * 80 + n * 4


def time_apply(s, k2, n, dev, stream, reps=50):
    """Seconds per launch of the QMR-step operator apply (q = K p and
    epsilon = p^T q in one pass) on the library's stream, CUDA events."""
    import torch
    kt = torch.from_numpy(k2.view(np.float64)).to(dev)
    pt = torch.randn(2 * n, dtype=torch.float64, device=dev)
    qt = torch.empty(2 * n, dtype=torch.float64, device=dev)
    et = torch.empty(2, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    for _ in range(5):
        s.inprod_dev(kt.data_ptr(), pt.data_ptr(), qt.data_ptr(), et.data_ptr())
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        s.inprod_dev(kt.data_ptr(), pt.data_ptr(), qt.data_ptr(), et.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) * 1e-3 / reps


def only_apply(s, k2, n, dev, stream):
    t = time_apply(s, k2, n, dev, stream, reps=10)
    print(json.dumps({"apply_us": t * 1e6, "unknowns": n, "alg_GBps": 48 * n / t / 1e9}))
    return 0


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


def systems_of(m):
    """(omega, source index) of every system, frequencies fastest, as the
    reference's MPI farm orders them (src/aphid_parallel.f90:97-101)."""
    om, sos = [], []
    for q in range(len(m.sources)):
        for f in m.freqs:
            om.append(2 * np.pi * float(f))
            sos.append(q)
    return om, sos


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hetero96")
    ap.add_argument("--precision", default="auto", choices=["mixed", "auto", "fused64", "fp64"])
    ap.add_argument("--plain-sweep", action="store_true",
                    help="also time the plain complex128 path over every system of the workload "
                         "(one solve each, the reference's algorithm) and report the ratio")
    ap.add_argument("--inner-tol", type=float, default=0.0)
    ap.add_argument("--plain-steps", type=int, default=2,
                    help="timed complex128 solves for the speed-up comparison (0: skip)")
    ap.add_argument("--cpu-sample-iters", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--one-sweep", action="store_true",
                    help="run one mixed sweep of the workload and exit (profiling target)")
    ap.add_argument("--only-apply", action="store_true",
                    help="set up the workload and time only the operator apply (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from aphid_git_b200 import Solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    # a real stream (not the NULL stream) shared by the library and the
    # CUDA events, so the events bracket the library's kernels
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)

    def barrier():
        if world > 1:
            dist.barrier()

    m, w, sig, b = setup_problem(args.workload)
    s = Solver(device=local, stream=stream.cuda_stream)
    s.set_nodes(m.xn, m.yn, m.zn)
    n = s.n
    om, sos = systems_of(m)
    nsys = len(om)
    peak, peak_kind = peaks()
    clocks = ClockSampler(local)

    if args.one_sweep:
        # one mixed sweep of the workload, nothing timed (profiling target)
        s.set_model("R", m.sig_re)
        prec = "mixed" if args.precision == "fp64" else args.precision
        _, inf = s.sweep(om, m.sources, sos, precision=prec, target=TARGET, max_it=MAX_IT, fetch=False)
        print(json.dumps({"workload": args.workload, "precision": prec, "systems": nsys, "plane_kz": s.sweep_plane_kz(),
                          "inner_iters": [i["inner_iters"] for i in inf][:8],
                          "outer_iters": [i["outer_iters"] for i in inf][:8],
                          "inner64_iters": [i["inner64_iters"] for i in inf][:8],
                          "seconds": inf[0]["seconds"], "launches": inf[0]["kernel_launches"]}))
        return 0

    if args.only_apply and args.precision == "mixed":
        # resident complex64 state from a short sweep, then the operator pass
        s.set_model("R", m.sig_re)
        s.sweep(om, m.sources, sos, precision="mixed", target=TARGET, max_it=8, fetch=False)
        ms_a, _ = timed(stream, dev, lambda: s.sweep_time_apply(10), 1, lambda: None, 1)
        t = ms_a * 1e-3 / 10
        print(json.dumps({"apply_us": t * 1e6, "unknowns": n, "systems": nsys,
                          "alg_GBps": pass_bytes(nsys, n) / t / 1e9}))
        return 0

    plain = None
    if args.precision == "fp64" or args.only_apply or args.plain_steps > 0:
        # the plain complex128 path: the reference's algorithm, one system at
        # a time, inputs resident (k^2, Jacobi diagonal and b on the device)
        k2 = s.gen_k2(sig, w)
        diag = s.gen_diag(k2)
        if args.only_apply:
            return only_apply(s, k2, n, dev, stream)
        s.qmr_load(k2, diag, b)
        s.qmr_run(TARGET, MAX_IT)
        steps = args.steps if args.precision == "fp64" else args.plain_steps
        if args.precision == "fp64":
            for _ in range(args.warmup - 1):
                s.qmr_run(TARGET, MAX_IT)
            clocks.start()
            time.sleep(0.3)
        ms_p, inf_p = timed(stream, dev, lambda: s.qmr_run(TARGET, MAX_IT)[0], steps, barrier, world)
        plain = {"time_to_tol_s": ms_p / steps * 1e-3, "iters_to_tol": inf_p[-1]["iters"],
                 "true_rel_resid": inf_p[-1]["true_rel_resid"],
                 "launches": int(sum(i["kernel_launches"] for i in inf_p)), "ms": ms_p,
                 "steps": steps, "note": "complex128 Jacobi-QMR, reference recurrence, "
                 "first system of the workload"}

    if args.precision == "fp64":
        clk = clocks.stop()
        ms, launches = plain["ms"], plain["launches"]
        iters = plain["iters_to_tol"]
        value = world * args.steps / (ms * 1e-3)
        ms_e, _ = timed(stream, dev, lambda: s.qmr(k2, diag, b, TARGET, MAX_IT, hist=False)[1],
                        args.steps, barrier, world)
        e2e = {"value": world * args.steps / (ms_e * 1e-3), "unit": "sweeps/s",
               "h2d_bytes_per_step": 3 * 16 * n, "d2h_bytes_per_step": 16 * n}
        t_apply = time_apply(s, k2, n, dev, stream)
        alg = 3 * 16 * n
        kernel = "k_apply64 (complex128 QMR step: q = K p, epsilon)"
        extra = {"time_to_tol_s": ms / args.steps * 1e-3, "iters_to_tol": iters,
                 "qmr_iters_per_s": world * args.steps * iters / (ms * 1e-3),
                 "true_rel_resid": plain["true_rel_resid"]}
        dtype = "c128"
        traffic_key = "apply64_qmr_" + args.workload
    else:
        # the product path: batched mixed-precision sweep of all systems
        s.set_model("R", m.sig_re)

        def run_sweep():
            return s.sweep(om, m.sources, sos, precision=args.precision, target=TARGET, max_it=MAX_IT,
                           inner_tol=args.inner_tol, fetch=False)[1]

        for _ in range(args.warmup):
            run_sweep()
        clocks.start()
        time.sleep(0.3)
        ms, infs = timed(stream, dev, run_sweep, args.steps, barrier, world)
        clk = clocks.stop()
        last = infs[-1]
        launches = int(sum(i[0]["kernel_launches"] for i in infs))
        value = world * args.steps / (ms * 1e-3)

        # host buffers in pinned memory, as a caller streaming many models would keep them
        sig_host = torch.empty(m.sig_re.shape[::-1], dtype=torch.float32, pin_memory=True).numpy().T
        sig_host[...] = m.sig_re
        x_host = torch.empty((nsys, n), dtype=torch.complex128, pin_memory=True).numpy()

        def run_e2e():
            s.set_model("R", sig_host)
            return s.sweep(om, m.sources, sos, precision=args.precision, target=TARGET, max_it=MAX_IT,
                           inner_tol=args.inner_tol, out=x_host)[1]

        ms_e, _ = timed(stream, dev, run_e2e, args.steps, barrier, world)
        e2e = {"value": world * args.steps / (ms_e * 1e-3), "unit": "sweeps/s",
               "h2d_bytes_per_step": 4 * m.ncell, "d2h_bytes_per_step": 16 * n * nsys}
        # dominant kernel: the fused complex64 QMR iteration (one launch per
        # inner iteration); algorithmic bytes per launch in pass_bytes().
        reps = 20
        if args.precision == "auto":
            # escalation releases the complex64 state: rebuild it for the timing launches
            s.sweep(om, m.sources, sos, precision="mixed", target=TARGET, max_it=8, fetch=False)
        s.sweep_time_apply(3)
        ms_a, _ = timed(stream, dev, lambda: s.sweep_time_apply(reps), 1, lambda: None, 1)
        t_apply = ms_a * 1e-3 / reps
        f64 = args.precision == "fused64"
        alg = pass_bytes(nsys, n) * (2 if f64 else 1)
        kernel = ("k_sw_pass64 (fused complex128 QMR iteration" if f64 else
                  "k_sw_pass (fused complex64 QMR iteration") + (
                  ": p^ update, q^ = D^-1 K p^, lagged d^/x^ update, 12 inner products)")
        it_in = [i["inner_iters"] for i in last]
        extra = {"time_to_tol_s": ms / args.steps * 1e-3, "systems": nsys,
                 "inner_iters_max": max(it_in), "inner_iters_total": int(sum(it_in)),
                 "outer_iters_max": max(i["outer_iters"] for i in last),
                 "qmr_iters_per_s": world * args.steps * sum(it_in) / (ms * 1e-3),
                 "inner64_iters_total": int(sum(i["inner64_iters"] for i in last)),
                 "true_rel_resid_max": max(i["true_rel_resid"] for i in last),
                 "status": sorted({i["status_name"] for i in last})}
        if args.plain_sweep:
            # the plain complex128 path over every system, once
            ms_p, inf_p = timed(stream, dev, lambda: s.sweep(om, m.sources, sos, precision="fp64", target=TARGET,
                                                              max_it=MAX_IT, fetch=False)[1], 1, barrier, world)
            pi = inf_p[-1]
            extra["plain_fp64_sweep"] = {
                "time_s": ms_p * 1e-3, "iters": [i["iters"] for i in pi],
                "status": sorted({i["status_name"] for i in pi}),
                "note": "complex128 Jacobi-QMR, the reference's recurrence and stop test, one system "
                        "at a time on the same GPU"}
            extra["speedup_vs_plain_fp64_sweep"] = ms_p * 1e-3 / (ms / args.steps * 1e-3)
            extra["inner_iters"] = it_in
        if plain is not None:
            extra["plain_fp64"] = plain
            extra["speedup_vs_plain_fp64"] = plain["time_to_tol_s"] * nsys / (ms / args.steps * 1e-3)
        dtype = {"mixed": "c64 inner / f64 outer", "fused64": "c128 inner / f64 outer",
                 "auto": "c64 inner (c128 after escalation) / f64 outer"}[args.precision]
        traffic_key = ("sw_pass64_" if f64 else "sw_pass_") + args.workload

    achieved = alg / t_apply / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(traffic_key)
    line = {
        "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded generator, no public dataset)",
        "config": {"workload": args.workload, "precision": args.precision, "unknowns": n,
                   "systems": nsys, "target": TARGET,
                   "l2": "working set > L2 (126 MB), no flush",
                   "parallelism": "independent sweep per GPU"},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk,
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, burst)",
                     "traffic": traffic, "alg_bytes_per_launch": alg,
                     "launch_us": t_apply * 1e6},
    }
    line.update(extra)
    iters_ref = FP64_ITERS.get(args.workload)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and iters_ref:
        spi, done = cpu_port_sample(args.workload, args.cpu_sample_iters)
        line["cpu_baseline"] = {
            "value": 1.0 / (spi * iters_ref * nsys), "unit": "sweeps/s", "cores": 4,
            "kind": "port",
            "sample": "%d QMR iterations of the workload, oracle 4-thread component split; "
                      "time-to-tolerance = %.3f s/iter x %d iterations (complex128 count, same "
                      "recurrence) x %d systems" % (done, spi, iters_ref, nsys),
            "s_per_iter": spi}
    s.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
