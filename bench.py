"""Benchmark of the PaScaL_POISSON_FFT solve path on B200 (libppf).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--slab]

Workload: the 512^3 solve (periodic x,y on [0,2pi)^2, Neumann z on [0,1]
with tanh stretching beta=1.5), right-hand side of seeded random Fourier
modes with a |k|^-2 spectrum plus white noise.  A step is one solve of that
problem.  `value` is the mixed-precision solve (FP32 transforms and bulk
tridiagonal solves, FP64 low-|k| rows, FP64 7-point residual refinement) in
whole-job solves/s with the inputs resident in HBM; its rel-L2 against the
plain FP64 solve of the same input is checked before timing and reported.
The plain FP64 solve (the reference's precision) is timed beside it.  `e2e`
times the host-array C-ABI call (ppf_solve_host_async: H2D of f, solve, D2H
of P, two plans alternating on two streams).
With N > 1 (torchrun) every rank solves its own 512^3 problem (independent
problems: weak scaling, no collective on the data path).

--slab instead splits one problem in z slabs over the torchrun ranks
(dist.SlabPoisson, the reference's np3 > 1 decomposition) and reports the
whole problem's solves/s (strong scaling).

--impl reference times the CPU restatement of the reference's solve (the
reference's own CPU build needs Fortran/MPI/FFTW, absent here) on the
host's cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "512³ solves/s: mixed-prec+refine vs FP64 plain, 1 B200, ≤1e-10 rel-L2; HBM %"
TOL = 1e-10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, nargs=3, default=[512, 512, 512], help="n1m n2m n3m")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end run and the 768x768x384 FP32 run (profiling runs)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--slab", action="store_true",
                    help="one problem split in z slabs over the torchrun ranks (strong scaling)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, lrank


def max_over_ranks(value: float, ws: int, device=None) -> float:
    """The job's time of a step: the slowest rank's (all ranks call this)."""
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms while running
    (start() returns once the first sample is in, so the timed region is covered)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.gpu)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()
        t0 = time.time()
        while not self.rows and time.time() - t0 < 3.0:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.06)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def stage_bytes(p, prec_bytes, sweeps):
    """Algorithmic bytes per stage, summed over one solve.

    Every pass reads and writes one spectral field per y and z stage; the x
    forward reads f (FP64) and writes the x spectrum A, the x inverse reads A
    and writes the iterate.  A is (n1m/2+1) complex values per (y, z) line for
    periodic x and n1m reals for a DCT in x; the y spectrum B is complex for
    periodic x or y and real for DCT in both.  With refinement sweeps the first
    iterate is an FP32 ghosted field (4 bytes a cell, written by the first
    pass, read by the first sweep's residual and accumulate); later sweeps
    read and write the FP64 iterate (8 bytes a cell)."""
    n1, n2, n3 = p.n1m, p.n2m, p.n3m
    N = n1 * n2 * n3
    px, py = bool(p.pbc[0]), bool(p.pbc[1])
    spec_a = (n1 // 2 + 1) * n2 * n3 * 2 * prec_bytes if px else N * prec_bytes
    if px:
        spec_b = spec_a
    elif py:
        spec_b = n1 * (n2 // 2 + 1) * n3 * 2 * prec_bytes
    else:
        spec_b = N * prec_bytes
    runs = 1 + sweeps
    if sweeps == 0 or prec_bytes == 8:
        u_read, u_rw = 0, 8 * N
    else:
        u_read = 4 * N + (sweeps - 1) * 8 * N           # residual reads of the iterate
        u_rw = 4 * N + (4 * N + 8 * N) + (sweeps - 1) * 16 * N   # x-inverse writes + accumulate reads
    return {
        "x-forward": runs * (8 * N + spec_a) + u_read,
        "y-forward": runs * (spec_a + spec_b),
        "tdma-z": runs * 2 * spec_b,
        "y-inverse": runs * (spec_a + spec_b),
        "x-inverse": runs * spec_a + u_rw,
    }


def stage_report(stages, sb, k, peak):
    """Per-stage ms per solve, achieved GB/s and fraction of the HBM peak."""
    out = {}
    for name, nbytes in sb.items():
        ms = stages[name][0] / k
        gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else None
        out[name] = {"ms": ms, "gbs": gbs, "frac": gbs / peak if gbs else None}
    return out


def load_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return d.get(kernel)
    except (OSError, ValueError):
        return None


def cpu_baseline(p, threads, keep=False):
    """Seconds of one oracle solve of p (and its output when keep)."""
    from oracle import oracle as O
    m = p.metrics
    t0 = time.perf_counter()
    out = O.poisson_solve(p.f, p.L1, p.L2, p.pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"], nthreads=threads)
    sec = time.perf_counter() - t0
    return (sec, out) if keep else sec


def cpu_stage_seconds():
    """The last oracle solve's stages under the reference's timer labels
    (01_Fortran/examples/main.f90:65-78)."""
    from oracle import oracle as O
    st = O.last_stage_seconds()
    if st is None:
        return None
    return {"build TDMA + FFT forward": st["setup"] + st["fft-forward"], "TDMA": st["tdma-z"],
            "FFT backward": st["fft-inverse"], "update solution": st["update-solution"]}


def scipy_fft_stage(f, workers):
    """Seconds of the x/y transform stages of one periodic solve with
    scipy.fft (pocketfft): real FFT along x, complex FFT along y, and back."""
    import scipy.fft as sf
    t0 = time.perf_counter()
    c = sf.rfft(f, axis=2, workers=workers)
    c = sf.fft(c, axis=1, workers=workers, overwrite_x=True)
    t1 = time.perf_counter()
    c = sf.ifft(c, axis=1, workers=workers, overwrite_x=True)
    sf.irfft(c, n=f.shape[2], axis=2, workers=workers)
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from pascal_poisson_fft_b200 import workloads as W
    threads = os.cpu_count() or 1
    n1, n2, n3 = args.n
    # full-size problem if (steps+warmup) solves fit the budget, else a
    # z-slab sample of it scaled to whole solves
    p = W.config3(n1m=n1, n2m=n2, n3m=n3)
    t1 = cpu_baseline(p, threads)
    budget = 150.0
    nz_s, sample = n3, f"full {n1}x{n2}x{n3} FP64 solve per step"
    if (args.steps + args.warmup) * t1 > budget:
        nz_s = max(16, int(n3 * budget / ((args.steps + args.warmup) * t1)) // 16 * 16)
        p = W.config3(n1m=n1, n2m=n2, n3m=nz_s)
        sample = f"{n1}x{n2}x{nz_s} FP64 solve per step (z-slab sample), time scaled by {n3}/{nz_s}"
    for _ in range(args.warmup):
        cpu_baseline(p, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_baseline(p, threads)
    sec = (time.perf_counter() - t0) / args.steps * (n3 / nz_s)
    value = 1.0 / sec
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, PCG64)", "impl": "reference",
            "config": {"workload": f"{n1}x{n2}x{n3} periodic-x,y Neumann-z tanh(beta=1.5) FP64 solve, CPU",
                       "grid": [n1, n2, n3]},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _device_time(fn, k, warm, stream):
    """ms per call of fn (CUDA events on `stream`, after `warm` calls)."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / k


def other_configs(args, dev, peak):
    """The other workloads of the configuration set, one GPU each, each timed
    with CUDA events and checked against its reference answer:
    c1 64^3 FP64 (periodic x,y), c2 256^3 FP64 DCT x,y with tanh z (beta 2),
    c4 96 uneven problems in one graph launch (FP64 and mixed), c5 the
    256x256x128 adjoint (FP64 and mixed)."""
    import torch
    import pascal_poisson_fft_b200 as ppf
    from oracle import oracle as O
    from pascal_poisson_fft_b200 import workloads as W
    st = torch.cuda.current_stream()
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    k = max(5, min(args.steps, 20))
    out = {}

    def plain(p, name):
        m = p.metrics
        mm = [t(m[q]) for q in ("dmx1", "dmx2", "dmx3", "dx3")]
        fd = t(p.f)
        P = torch.zeros(p.n3m + 2, p.n2m + 2, p.n1m + 2, dtype=torch.float64, device=dev)
        plan = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc, precision=ppf.PPF_FP64)
        ms = _device_time(lambda: plan.solve(fd, P, *mm), k, 3, st)
        plan.stage_timing(True)
        for _ in range(3):
            plan.solve(fd, P, *mm)
        stg = plan.stage_times()
        plan.stage_timing(False)
        R = O.poisson_solve(p.f, p.L1, p.L2, p.pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])
        rel = float(np.linalg.norm(P.cpu().numpy() - R) / np.linalg.norm(R))
        sb = stage_bytes(p, 8, 0)
        tot = sum(sb.values())
        plan.close()
        return {"workload": name, "value": 1000.0 / ms, "unit": "solves/s", "ms_per_step": ms,
                "mcells_s": p.n1m * p.n2m * p.n3m / ms / 1e3, "gbs_alg": tot / (ms * 1e-3) / 1e9,
                "hbm_frac": tot / (ms * 1e-3) / 1e9 / peak, "rel_l2_vs_oracle": rel,
                "stages": stage_report(stg, sb, 3, peak)}

    out["c1"] = plain(W.config1(), "64^3 FP64, periodic x,y, Neumann z, uniform")
    out["c2"] = plain(W.config2(), "256^3 FP64, DCT x,y, Neumann z, tanh z beta=2")

    # c4: 96 uneven problems, one graph launch per batch solve
    probs = W.config4(device=dev)
    cells = sum(p.n1m * p.n2m * p.n3m for p in probs)
    fs = [p.f for p in probs]
    ms_ = [[t(p.metrics[q]) for p in probs] for q in ("dmx1", "dmx2", "dmx3", "dx3")]
    res = {}
    outs = {}
    for prec, name, sw in ((ppf.PPF_FP64, "fp64", 0), (ppf.PPF_MIXED, "mixed", 2)):
        t0 = time.perf_counter()
        b = ppf.Batch([dict(n1m=p.n1m, n2m=p.n2m, n3m=p.n3m, L1=p.L1, L2=p.L2, pbc=p.pbc, precision=prec,
                            max_sweeps=sw) for p in probs], autotune=True)
        t_create = time.perf_counter() - t0
        Ps = [torch.zeros(p.n3m + 2, p.n2m + 2, p.n1m + 2, dtype=torch.float64, device=dev) for p in probs]
        ms = _device_time(lambda: b.solve(fs, Ps, *ms_), k, 3, st)
        res[name] = {"ms_per_batch": ms, "gcells_s": cells / ms / 1e6, "create_s": t_create}
        outs[name] = Ps
        b.close()
    worst = max(float(torch.linalg.vector_norm(a - c) / torch.linalg.vector_norm(c))
                for a, c in zip(outs["mixed"], outs["fp64"]))
    res["mixed"]["max_rel_l2_vs_fp64"] = worst
    # the same batch as one persistent work-queue kernel (one graph launch)
    for prec, name, sw in ((ppf.PPF_FP64, "fp64", 0), (ppf.PPF_MIXED, "mixed", 2)):
        b = ppf.Batch([dict(n1m=p.n1m, n2m=p.n2m, n3m=p.n3m, L1=p.L1, L2=p.L2, pbc=p.pbc, precision=prec,
                            max_sweeps=sw) for p in probs], persistent=True)
        Ps = [torch.zeros(p.n3m + 2, p.n2m + 2, p.n1m + 2, dtype=torch.float64, device=dev) for p in probs]
        ms = _device_time(lambda: b.solve(fs, Ps, *ms_), k, 3, st)
        rel = max(float(torch.linalg.vector_norm(a - c) / torch.linalg.vector_norm(c))
                  for a, c in zip(Ps, outs[name]))
        res[name]["persistent"] = {"ms_per_batch": ms, "gcells_s": cells / ms / 1e6, "max_rel_l2_vs_graph": rel}
        b.close()
        del Ps
    out["c4"] = {"workload": f"96 uneven problems ({cells / 1e6:.0f} Mcells), one graph launch", **res}
    del outs, fs, probs

    # c5: adjoint at 256x256x128 (transpose solve + z-metric gradient)
    p, _ = W.config5()
    m = p.metrics
    mm = [t(m[q]) for q in ("dmx1", "dmx2", "dmx3", "dx3")]
    fd = t(p.f)
    res = {}
    for prec, name in ((ppf.PPF_FP64, "fp64"), (ppf.PPF_MIXED, "mixed")):
        plan = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc, precision=prec, max_sweeps=3)
        u = torch.zeros(plan.gshape, dtype=torch.float64, device=dev)
        plan.solve(fd, u, *mm)
        df = torch.empty(plan.shape, dtype=torch.float64, device=dev)
        gx = torch.empty(p.n3m + 2, dtype=torch.float64, device=dev)
        gm = torch.empty(p.n3m + 2, dtype=torch.float64, device=dev)
        ms_f = _device_time(lambda: plan.solve(fd, u, *mm), k, 3, st)
        ms_a = _device_time(lambda: plan.solve_adjoint(fd, df, *mm, u=u, ddx3=gx, ddmx3=gm), k, 3, st)
        res[name] = {"forward_ms": ms_f, "adjoint_ms": ms_a}
        plan.close()
    n1, n2, n3 = p.n1m, p.n2m, p.n3m
    res["recompute_bytes"] = (n1 + 2) * (n2 + 2) * (n3 + 2) * 8
    res["store_bytes"] = (n1 // 2 + 1) * n2 * n3 * 16
    out["c5"] = {"workload": "256x256x128 adjoint (dJ/df and dJ/d dx3, dmx3), periodic x,y, tanh z beta=2", **res}
    return out


def run_ours(args, ws, rank, lrank):
    import torch
    import pascal_poisson_fft_b200 as ppf
    from pascal_poisson_fft_b200 import workloads as W

    dev = torch.device("cuda", lrank)
    torch.cuda.set_device(dev)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    n1, n2, n3 = args.n
    p = W.config3(n1m=n1, n2m=n2, n3m=n3, generate=False)
    f = W.config3_field(p, seed=3 + rank, device=dev)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    m = p.metrics
    dmx1, dmx2, dmx3, dx3 = t(m["dmx1"]), t(m["dmx2"]), t(m["dmx3"]), t(m["dx3"])
    P = torch.zeros(p.n3m + 2, p.n2m + 2, p.n1m + 2, dtype=torch.float64, device=dev)
    P64 = torch.zeros_like(P)
    st = torch.cuda.current_stream()

    plan64 = ppf.Plan(n1, n2, n3, p.L1, p.L2, *p.pbc, precision=ppf.PPF_FP64)
    plan64.solve(f, P64, dmx1, dmx2, dmx3, dx3)

    # fewest refinement sweeps that meet the tolerance against the FP64 solve
    sweeps, rel = None, None
    for s in (1, 2, 3, 4):
        planm = ppf.Plan(n1, n2, n3, p.L1, p.L2, *p.pbc, precision=ppf.PPF_MIXED, max_sweeps=s)
        planm.solve(f, P, dmx1, dmx2, dmx3, dx3)
        torch.cuda.synchronize()
        rel = float(torch.linalg.vector_norm(P - P64) / torch.linalg.vector_norm(P64))
        if rel <= TOL:
            sweeps = s
            break
        planm.close()
    if sweeps is None:
        sweeps = 4

    def timed(plan, out, k, inputs=None):
        fi, d1, d2, d3, x3 = inputs if inputs is not None else (f, dmx1, dmx2, dmx3, dx3)
        for _ in range(args.warmup):
            plan.solve(fi, out, d1, d2, d3, x3)
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(k):
            plan.solve(fi, out, d1, d2, d3, x3)
        e1.record(st)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / k, ws, dev)

    clocks = ClockSampler(dev.index if "CUDA_VISIBLE_DEVICES" not in os.environ else lrank)
    clocks.start()
    ms_mixed = timed(planm, P, args.steps)
    ms_fp64 = timed(plan64, P64, args.steps)
    clk = clocks.stop()

    # per-stage device times of the mixed solve (CUDA events on the solve's stream)
    planm.stage_timing(True)
    kst = max(3, min(args.steps, 10))
    for _ in range(kst):
        planm.solve(f, P, dmx1, dmx2, dmx3, dx3)
    stages = planm.stage_times()
    planm.stage_timing(False)
    launches_per_solve = sum(v[1] for v in stages.values()) / kst
    plan64.stage_timing(True)
    for _ in range(kst):
        plan64.solve(f, P64, dmx1, dmx2, dmx3, dx3)
    stages64 = plan64.stage_times()
    plan64.stage_timing(False)
    sb = stage_bytes(p, 4, sweeps)
    dom = max(sb, key=lambda s: stages[s][0])
    dom_ms_per_launch = stages[dom][0] / stages[dom][1]
    dom_bytes_per_launch = sb[dom] / (stages[dom][1] / kst)
    peak, peak_kind = measured_hbm_peak()
    achieved = dom_bytes_per_launch / (dom_ms_per_launch * 1e-3) / 1e9

    # end to end through the host-array C ABI: every step copies f in from
    # page-locked host memory, solves and copies P out (ppf_solve_host_async).
    # Three plans take turns on three streams, so the copy engines stay busy:
    # one step's copy-out overlaps the next steps' copy-in (separate engines),
    # and a stream's next copy-in does not wait behind its own copy-out.  The
    # timed region spans all K steps and every copy.
    e2e = None
    if not args.no_e2e:
        NP = 3
        plans = [planm] + [ppf.Plan(n1, n2, n3, p.L1, p.L2, *p.pbc, precision=ppf.PPF_MIXED, max_sweeps=sweeps)
                           for _ in range(NP - 1)]
        streams = [torch.cuda.Stream(device=dev) for _ in range(NP)]
        fh = torch.empty(f.shape, dtype=torch.float64, pin_memory=True)
        fh.copy_(f)
        Ph = [torch.empty(P.shape, dtype=torch.float64, pin_memory=True) for _ in range(NP)]
        mh = [torch.as_tensor(np.ascontiguousarray(m[k])).pin_memory() for k in ("dmx1", "dmx2", "dmx3", "dx3")]

        def e2e_steps(k, e_start=None, e_ends=None):
            if e_start is not None:
                e_start.record(streams[0])
                for sm in streams[1:]:
                    sm.wait_event(e_start)
            for i in range(k):
                plans[i % NP].solve_host_async(fh, Ph[i % NP], *mh, stream=streams[i % NP])
            if e_ends is not None:
                for ev, sm in zip(e_ends, streams):
                    ev.record(sm)

        e2e_steps(max(NP, min(args.warmup, 6)))
        torch.cuda.synchronize()
        k2 = max(2 * NP, min(args.steps, 12))
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(NP)]
        e2e_steps(k2, e0, ends)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(max(e0.elapsed_time(ev) for ev in ends) / k2, ws, dev)
        # the last step's result matches the device solve of the same input
        e2e_rel = float(torch.linalg.vector_norm(Ph[(k2 - 1) % NP].to(dev) - P64) / torch.linalg.vector_norm(P64))
        h2d = fh.nbytes + sum(a.nbytes for a in mh)
        e2e = {"value": ws * 1000.0 / ms_e2e, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(Ph[0].nbytes), "ms_per_step": ms_e2e,
               "api": f"ppf_solve_host_async, {NP} plans on {NP} streams", "rel_l2_vs_fp64": e2e_rel}
        for q in plans[1:]:
            q.close()

    # the FP32 single-solve throughput run of the same configuration family at
    # mixed radix 3*2^k (768 = 3*256): 768x768x384, no refinement, its error
    # against the FP64 solve of the same input reported beside it
    fp32_run = None
    if not args.no_e2e and tuple(args.n) == (512, 512, 512):
        q = W.config3(n1m=768, n2m=768, n3m=384, generate=False)
        fq = W.config3_field(q, seed=3 + rank, device=dev)
        qin = (fq, *[t(q.metrics[k]) for k in ("dmx1", "dmx2", "dmx3", "dx3")])
        Pq = torch.zeros(q.n3m + 2, q.n2m + 2, q.n1m + 2, dtype=torch.float64, device=dev)
        Rq = torch.zeros_like(Pq)
        pq64 = ppf.Plan(768, 768, 384, q.L1, q.L2, *q.pbc, precision=ppf.PPF_FP64)
        pq64.solve(*qin[:1], Rq, *qin[1:])
        pq64.close()
        pq32 = ppf.Plan(768, 768, 384, q.L1, q.L2, *q.pbc, precision=ppf.PPF_FP32)
        ms32 = timed(pq32, Pq, args.steps, qin)
        rel32 = float(torch.linalg.vector_norm(Pq - Rq) / torch.linalg.vector_norm(Rq))
        pq32.close()
        fp32_run = {"workload": "768x768x384 Poisson, periodic x,y / Neumann z, tanh z beta=1.5, FP32 single solve "
                                "(radix 3*2^k, no refinement)",
                    "value": ws * 1000.0 / ms32, "unit": "solves/s", "ms_per_step": ms32,
                    "rel_l2_vs_fp64": rel32}
        del Pq, Rq, qin, fq

    # the CPU baseline (the oracle on all host cores) on the same right-hand
    # side; its output also pins the headline results: rel-L2 of the FP64 and
    # of the mixed 512^3 solve against the FP64 oracle
    cpu, vs_oracle = None, {}
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            pc = W.config3(n1m=n1, n2m=n2, n3m=n3, generate=False)
            pc.f = f.cpu().numpy()
            threads = os.cpu_count() or 1
            sec, R = cpu_baseline(pc, threads, keep=True)
            stages_cpu = cpu_stage_seconds()
            nrm = float(np.linalg.norm(R))
            vs_oracle = {"mixed": float(np.linalg.norm(P.cpu().numpy() - R) / nrm),
                         "fp64": float(np.linalg.norm(P64.cpu().numpy() - R) / nrm)}
            del R
            # one host thread, on a z-slab sample of the same workload (the
            # solve's cost is linear in the z rows), scaled to a whole solve
            nz1 = min(n3, 64)
            p1 = W.config3(n1m=n1, n2m=n2, n3m=nz1, generate=False)
            p1.f = np.ascontiguousarray(pc.f[:nz1])
            sec1 = cpu_baseline(p1, 1) * (n3 / nz1)
            fwd, inv = scipy_fft_stage(pc.f, threads)
            best = None
            if stages_cpu:
                # the oracle's own stages with the faster of its transforms
                # and scipy.fft's (an estimate of a CPU solve on an optimised
                # FFT library, as the reference's FFTW/MKL build would be)
                best = 1.0 / (stages_cpu["TDMA"] + stages_cpu["update solution"] +
                              min(stages_cpu["build TDMA + FFT forward"], fwd) + min(stages_cpu["FFT backward"], inv))
            cpu = {"value": 1.0 / sec, "unit": "solves/s", "cores": threads, "kind": "port",
                   "fast_fft_estimate": best,
                   "sample": f"one full {n1}x{n2}x{n3} FP64 solve of the same right-hand side",
                   "stage_s": stages_cpu,
                   "single_thread": {"value": 1.0 / sec1, "unit": "solves/s", "cores": 1,
                                     "sample": f"{n1}x{n2}x{nz1} z-slab of the workload, time scaled by {n3}/{nz1}"},
                   "scipy_fft_stage_s": {"forward x+y": fwd, "inverse y+x": inv, "workers": threads,
                                         "oracle_forward": stages_cpu["build TDMA + FFT forward"] if stages_cpu else None,
                                         "oracle_inverse": stages_cpu["FFT backward"] if stages_cpu else None}}
            del pc
        except Exception as exc:  # the baseline is reported, never the product
            cpu = {"value": None, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {exc}"}

    configs = None
    if rank == 0 and ws == 1 and not args.no_e2e and tuple(args.n) == (512, 512, 512):
        configs = other_configs(args, dev, peak)

    if rank == 0:
        line = {
            "metric": METRIC, "value": ws * 1000.0 / ms_mixed, "unit": "solves/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64-refine",
            "data": "synthetic (seeded PCG64 Fourier modes, |k|^-2 spectrum + white noise)",
            "config": {"workload": f"{n1}x{n2}x{n3} Poisson, periodic x,y / Neumann z, tanh z beta=1.5, "
                                   f"mixed FP32+FP64 refine ({sweeps} sweeps)",
                       "grid": [n1, n2, n3], "sweeps": sweeps, "rel_l2_vs_fp64": rel,
                       "rel_l2_vs_oracle": vs_oracle.get("mixed"),
                       "l2_policy": "inputs larger than L2 (1 GiB FP64 field per step)",
                       "problems_per_gpu": 1},
            "fp64_plain": {"value": ws * 1000.0 / ms_fp64, "unit": "solves/s", "ms_per_step": ms_fp64,
                           "rel_l2_vs_oracle": vs_oracle.get("fp64"),
                           "stage_ms_per_solve": {k: v[0] / kst for k, v in stages64.items()},
                           "stages": stage_report(stages64, stage_bytes(p, 8, 0), kst, peak)},
            "mixed_over_fp64": ms_fp64 / ms_mixed,
            "stage_ms_per_solve": {k: v[0] / kst for k, v in stages.items()},
            "stages": stage_report(stages, sb, kst, peak),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": dom_bytes_per_launch, "traffic": load_traffic(dom)},
            "gpu_launches": int(round(launches_per_solve * args.steps)),
            "clocks": clk,
            "e2e": e2e,
            "fp32_768x768x384": fp32_run,
            "cpu_baseline": cpu,
            "configs": configs,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_slab(args, ws, rank, lrank):
    """One n1m x n2m x n3m FP64 problem split in z slabs over the ranks (the
    reference's np3 = ranks decomposition, dist.SlabPoisson: rank-local x/y
    transforms, PaScaL's multi-rank TDMA with all-to-all exchanges of the
    reduced systems, global mean, ghost planes), NCCL between GPUs.  value:
    solves/s of the whole problem, timed with CUDA events as the slowest
    rank's time (strong scaling).  Checked against the single-GPU FP64 solve
    on rank 0 for N = 1."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import pascal_poisson_fft_b200 as ppf
    from pascal_poisson_fft_b200 import dist as D
    from pascal_poisson_fft_b200 import workloads as W

    dev = torch.device("cuda", lrank)
    torch.cuda.set_device(dev)
    if not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29512")
        dist.init_process_group("nccl", rank=rank, world_size=ws, timeout=timedelta(seconds=300),
                                device_id=dev)
    n1, n2, n3 = args.n
    p = W.config3(n1m=n1, n2m=n2, n3m=n3, generate=False)
    f = W.config3_field(p, seed=3, device=dev)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    m = p.metrics
    dmx1, dmx2, dmx3, dx3 = t(m["dmx1"]), t(m["dmx2"]), t(m["dmx3"]), t(m["dx3"])
    slab = D.SlabPoisson(n1, n2, n3, p.L1, p.L2, p.pbc, rank, ws, dev)
    fl = f[slab.z0:slab.z0 + slab.rows].contiguous()
    P = torch.zeros(slab.ghost_shape(), dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream()
    for _ in range(args.warmup):
        slab.solve(fl, P, dmx1, dmx2, dmx3, dx3)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        slab.solve(fl, P, dmx1, dmx2, dmx3, dx3)
    e1.record(st)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, ws, dev)
    rel = None
    if ws == 1:
        plan = ppf.Plan(n1, n2, n3, p.L1, p.L2, *p.pbc, precision=ppf.PPF_FP64)
        R = torch.zeros_like(P)
        plan.solve(f, R, dmx1, dmx2, dmx3, dx3)
        torch.cuda.synchronize()
        rel = float(torch.linalg.vector_norm(P - R) / torch.linalg.vector_norm(R))
        plan.close()
    if rank == 0:
        print(json.dumps({
            "metric": f"{n1}x{n2}x{n3} z-slab solves/s (one problem over the ranks), FP64",
            "value": 1000.0 / ms, "unit": "solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64 Fourier modes, |k|^-2 spectrum + white noise)",
            "config": {"workload": f"{n1}x{n2}x{n3} Poisson split in {ws} z slabs, periodic x,y / Neumann z, "
                                   "tanh z beta=1.5", "grid": [n1, n2, n3], "slab_rows": slab.rows,
                       "rel_l2_vs_single_gpu_fp64": rel}}), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def main():
    args = parse()
    ws, rank, lrank = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    elif args.slab:
        run_slab(args, ws, rank, lrank)
    else:
        run_ours(args, ws, rank, lrank)


if __name__ == "__main__":
    main()
