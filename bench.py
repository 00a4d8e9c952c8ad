"""Benchmark: LPs solved per second at 1e-8 relative gap on one B200.

Workload (a "step"): 4096 transportation LPs of uneven size (ns, nt ~ U{10..60}, up to 3600
variables each; costs U[1,100], integer supplies/demands as in the 50x50 single-LP workload),
seeded synthetic data, solved to the reference's tolerances (1e-9 on the scaled problem, which
keeps every objective within 1e-8 of the reference's) by the batched persistent kernel.

  value   device time only: the batch is resident in HBM (sov_batch_create once), each step is
          one sov_batch_solve (all bucket launches) timed with CUDA events on the launching
          stream. Per step the kernels read ~0.6 GB of per-LP data, several times the 126 MB L2.
  e2e     the public C-ABI call sov_lp_solve_batch with host buffers: host standard form,
          host->device copy, solve, device->host copy and publishing, per step.
  plain_fp64_gpu   the same 4096 LPs through the single-problem FP64 engine (sov_lp_solve), 16
          concurrent solves on separate CUDA streams, for the batched vs plain-FP64 comparison.
  cpu_baseline     the reference's own CPU IPM (oracle/_ref, compiled from the reference sources)
          on a bounded sample of the same LPs with all host threads.

python bench.py [--gpus N --steps K --warmup W] [--impl reference]
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

METRIC = "LPs solved/sec at 1e-8 rel gap on 1 B200: mixed+batched+warm-start vs plain FP64"
UNIT = "LPs/s"
WORKLOAD = "4096 uneven transportation LPs (ns, nt ~ U{10..60}), batched persistent launch"
COUNT = 4096
PLAIN_WORKERS = 16  # concurrent single-problem solves of the plain FP64 baseline


def traffic_per_step(count: int, chosen: dict):
    """DRAM bytes (read + write) of one step of the default batch workload, summed over its bucket
    launches, from the ncu capture in profiles/traffic.json (taken with the bucket widths pinned to an
    autotuned run's choice). Buckets that ran another width in this run may differ; if they carry less
    than 1 % of the captured bytes the sum is kept with a note, otherwise the traffic is unknown."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            t = json.load(fh)["k_batch_ipm"]
        per = t["dram_bytes_per_bucket"]
        widths = t["threads_per_bucket"]
    except (OSError, KeyError, ValueError):
        return None, "no capture"
    if count != t.get("lps", COUNT) or set(per) != set(chosen):
        return None, "capture of another workload"
    total = float(sum(per.values()))
    other = [k for k in per if widths.get(k) != chosen.get(k)]
    if sum(per[k] for k in other) > 0.01 * total:
        return None, f"buckets {other} ran other widths than the capture"
    note = "capture with this run's widths"
    if other:
        note += f"; {other} ran another width (under 1 % of the captured bytes)"
    return total, note


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return dict(hbm_gbs=d["hbm_gbs"], bf16_tflops=d["bf16_tflops"], source="measured")
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, source="fallback")


class ClockSampler:
    """SM clock, its maximum and the throttle reasons sampled during the timed region: NVML polled
    every 10 ms from a thread (read-only queries), or nvidia-smi every 200 ms where NVML cannot be
    loaded (then the region starts only once its first sample has arrived)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.rows: list[tuple[float, float, list[str]]] = []  # (sm MHz, max sm MHz, active reasons)
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:  # the CUDA device's own GPU (CUDA_VISIBLE_DEVICES may renumber), by its PCI address
            import torch
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            N, h = self._nvml_handle()
            bits = [N.nvmlClocksEventReasonHwSlowdown, N.nvmlClocksEventReasonHwThermalSlowdown,
                    N.nvmlClocksEventReasonSwThermalSlowdown, N.nvmlClocksEventReasonSwPowerCap]
            mx = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))

            def sample():
                sm = float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM))
                r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((sm, mx, [nm for nm, b in zip(self.NAMES, bits) if r & b]))

            sample()
            self.nvml = N

            def loop():
                while not self.stop.wait(0.01):
                    try:
                        sample()
                    except Exception:
                        return
            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
            self.rows = []
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            r = [v.strip() for v in line.split(",")]
            if len(r) > 8 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                self.rows.append((float(r[1]), float(r[2]),
                                  [self.NAMES[k] for k in range(4) if r[5 + k] == "Active"]))

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml is not None:
            self.thread.join(timeout=1.0)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["unsampled"], samples=0)
        reasons = sorted({nm for _, _, rs in self.rows for nm in rs})
        return dict(sm_mhz=statistics.median(r[0] for r in self.rows), sm_max_mhz=max(r[1] for r in self.rows),
                    reasons=reasons, samples=len(self.rows), source="nvml" if self.nvml is not None else "nvidia-smi")


def dist_setup(n_gpus: int):
    from sovereign_b200.shard import world as world_env
    rank, world, local = world_env()
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        return rank, world, local, dist
    return 0, 1, 0, None


def barrier(dist, local):
    if dist is not None:
        import torch
        dist.barrier(device_ids=[local])
        torch.cuda.synchronize()


def max_over_ranks(dist, v: float, local: int) -> float:
    from sovereign_b200.shard import max_over_ranks as mor
    return mor(v, dist, device=f"cuda:{local}")


def per_lp_bytes(mdl) -> float:
    # algorithmic HBM bytes of one IPM iteration: 6 SpMVs (3 A, 3 A') + ~15 n-vector and ~10
    # m-vector passes (standard form of a transport LP has no slacks: n_ipm = n, nnz = 2n)
    n, m, nnz = mdl.n, mdl.m, mdl.nnz
    return 6.0 * (12.0 * nnz + 8.0 * (m + n)) + 15.0 * 8.0 * n + 10.0 * 8.0 * m


def per_lp_flops(mdl) -> float:
    # FP64 flops of one IPM iteration of the batched kernel: the dense L D L' of the m x m normal
    # matrix, two right-hand sides forward and backward, and the assembly (2 k_j^2 per column)
    m = mdl.m
    k = np.diff(mdl.col_ptr).astype(np.float64)
    return (2.0 / 3.0) * m ** 3 + 8.0 * m * m + 2.0 * float(np.sum(k * k))


def cpu_reference_sample(models, seconds_target: float = 15.0) -> dict:
    import oracle
    threads = oracle.reference().ref_hardware_threads()
    # calibrate on a small slice, then size the sample to ~seconds_target of work
    probe = models[:max(threads, 16)]
    secs, _, _, _ = oracle.solve_many_reference(probe, threads=threads)
    rate = len(probe) / max(secs, 1e-9)
    k = int(min(len(models), max(len(probe), rate * seconds_target)))
    sample = models[:k]
    secs, obj, its, st = oracle.solve_many_reference(sample, threads=threads)
    return dict(value=len(sample) / secs, unit=UNIT, cores=threads, kind="reference",
                sample=f"first {len(sample)} of the {COUNT} LPs, InteriorPointSolver on {threads} host threads, "
                       f"{secs:.1f} s", seconds=secs, objectives=obj, statuses=st)


def run_reference(args, rank: int, world: int):
    """--impl reference: the reference's own CPU IPM on the same workload, rank 0 only."""
    if rank != 0:
        return
    from sovereign_b200 import problems as P
    import oracle
    models = P.transport_batch(COUNT, seed=2026)
    threads = oracle.reference().ref_hardware_threads()
    # each step solves a bounded sample (about 4 s of CPU time) drawn round-robin from the batch
    probe = models[:threads]
    secs, *_ = oracle.solve_many_reference(probe, threads=threads)
    per_step = int(max(threads, min(COUNT, 4.0 * len(probe) / max(secs, 1e-9))))
    for w in range(args.warmup):
        oracle.solve_many_reference(models[:threads], threads=threads)
    times = []
    solved = 0
    for k in range(args.steps):
        start = (k * per_step) % COUNT
        sample = (models + models)[start:start + per_step]
        t, obj, its, st = oracle.solve_many_reference(sample, threads=threads)
        times.append(t)
        solved += len(sample)
    total = sum(times)
    value = solved / total
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=1e3 * total / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic", impl="reference",
                config=dict(workload=WORKLOAD, sample_per_step=per_step, l2="inputs on host"),
                cpu_baseline=dict(value=value, unit=UNIT, cores=threads, kind="reference",
                                  sample=f"{per_step} of the {COUNT} LPs per step on {threads} host threads"),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line))


def _line(metric, value, unit, args, ms, dtype, config, **extra):
    d = dict(metric=metric, value=value, unit=unit, n_gpus=1, steps=args.steps, warmup=args.warmup, ms_per_step=ms,
             higher_is_better=True, scaling="weak", vs_baseline=None, dtype=dtype, data="synthetic", config=config)
    d.update(extra)
    print(json.dumps(d))


def run_single_workload(args):
    """Single-problem workloads of the other configurations (one JSON line each)."""
    import torch
    from sovereign_b200 import abi, problems as P
    from sovereign_b200.ipm import InteriorPointOptions, InteriorPointSolver, QpInteriorPointSolver
    import oracle
    torch.cuda.init()

    def timed(solver, mdl, **kw):
        for _ in range(args.warmup):
            solver.solve(mdl, **kw)
        rs, ts = [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            r = solver.solve(mdl, with_diag=True, **kw)
            ts.append(time.perf_counter() - t0)
            rs.append(r)
        return rs[-1], float(np.median(ts)), float(np.median([r.solve_seconds for r in rs]))

    if args.workload in ("c0", "c1"):
        rows = args.rows
        mdl = P.transport(50, 50, 0) if args.workload == "c0" else P.random_sparse_lp(rows, 5 * rows, 8, 1)
        lines = {}
        for name, prec in (("fp64", abi.PRECISION_FP64), ("mixed", abi.PRECISION_MIXED)):
            r, wall, dev = timed(InteriorPointSolver(InteriorPointOptions(precision=prec)), mdl)
            lines[name] = dict(status=r.status_name, iterations=r.iterations, objective=r.objective_value,
                               wall_s=wall, device_s=dev, pcg_iterations=r.diagnostics["pcg_iterations"],
                               fp64_refactorizations=r.diagnostics["fp64_fallbacks"])
        ref = None
        if args.workload == "c0":
            rr = oracle.solve(mdl, kind="reference")
            ref = dict(objective=rr.objective_value, seconds=rr.solve_seconds, iterations=rr.iterations)
        elif rows == 2000:  # the reference's solve takes ~10 minutes of CPU: its result is a committed fixture
            g = np.load(os.path.join(ROOT, "tests", "golden", "c1_reference.npz"))
            ref = dict(objective=float(g["objective"]), seconds=float(g["seconds"]), iterations=int(g["iterations"]),
                       source="tests/golden/c1_reference.npz (reference InteriorPointSolver, dense LU, one CPU thread)")
        for v in lines.values():
            v["rel_obj_err_vs_reference"] = (abs(v["objective"] - ref["objective"]) / max(1.0, abs(ref["objective"]))
                                             if ref else None)
        # larger orders have no reference run (its dense LU would take hours): FP64 against mixed only
        o64, omx = lines["fp64"]["objective"], lines["mixed"]["objective"]
        best = min(lines.values(), key=lambda v: v["wall_s"])
        _line(METRIC, 1.0 / best["wall_s"], UNIT, args, 1e3 * best["wall_s"], "f64",
              dict(workload="transport 50x50 (single LP)" if args.workload == "c0" else
                   f"random sparse LP m={rows} n={5 * rows}, 8 nnz/column (single LP)"),
              variants=lines, cpu_reference=ref,
              rel_obj_diff_mixed_vs_fp64=abs(omx - o64) / max(1.0, abs(o64)),
              max_rel_obj_err_vs_reference=(max(v["rel_obj_err_vs_reference"] for v in lines.values())
                                            if ref else None))
        return
    if args.workload == "kkt":
        # a QP whose Hessian couples neighbours, at n = 200000 (KKT order 650001): the sparse
        # quasi-definite KKT path; the reference's answer and its CPU time are a committed fixture
        key = "coupled_chain_qp(200000,5)"
        g = json.load(open(os.path.join(ROOT, "tests", "golden", "kkt_reference.json")))[key]
        mdl = P.coupled_chain_qp(200000, 5)
        r, wall, dev = timed(QpInteriorPointSolver(), mdl)
        _line(METRIC, 1.0 / wall, UNIT, args, 1e3 * wall, "f64",
              dict(workload="coupled chain QP n=200000 (tridiagonal Hessian, KKT order 650001), single QP"),
              status=r.status_name, iterations=r.iterations, objective=r.objective_value, device_s=dev,
              message=r.message[-160:],
              max_rel_obj_err_vs_reference=abs(r.objective_value - g["objective"]) / max(1.0, abs(g["objective"])),
              cpu_reference=dict(objective=g["objective"], seconds=g["seconds"], iterations=g["iterations"],
                                 source="tests/golden/kkt_reference.json (reference QpInteriorPointSolver, sparse "
                                        "quasi-definite KKT, one CPU thread)"))
        return
    if args.workload == "wide":
        # an LP far wider than L2 (16M nonzeros): the single engine's HBM-bound passes
        mdl = P.wide_lp(2000, 2_000_000, 8, 1)
        r, wall, dev = timed(InteriorPointSolver(), mdl)
        _line(METRIC, 1.0 / wall, UNIT, args, 1e3 * wall, "f64",
              dict(workload="wide LP m=2000 n=2000000, 8 nnz/column (single LP)"),
              status=r.status_name, iterations=r.iterations, objective=r.objective_value, device_s=dev,
              message=r.message[-120:])
        return
    if args.workload == "c2":
        mdl = P.convex_sequence_qp(20002, 2)
        r, wall, dev = timed(QpInteriorPointSolver(), mdl)
        # the reference's structured LISWET path takes ~3 minutes of CPU: its answer is a fixture
        g = np.load(os.path.join(ROOT, "tests", "golden", "c2_reference.npz"))
        ref_obj = float(g["objective"])
        _line(METRIC, 1.0 / wall, UNIT, args, 1e3 * wall, "dd (double-double) + f64",
              dict(workload="convex-sequence QP n=20002, m=20000 (single QP)"),
              status=r.status_name, iterations=r.iterations, objective=r.objective_value, device_s=dev,
              duality_gap=r.duality_gap, primal_residual=r.primal_residual, dual_residual=r.dual_residual,
              message=r.message[:200],
              max_rel_obj_err_vs_reference=abs(r.objective_value - ref_obj) / max(1.0, abs(ref_obj)),
              max_abs_primal_diff_vs_reference=float(np.max(np.abs(r.primal - g["primal"]))),
              cpu_reference=dict(objective=ref_obj, seconds=float(g["seconds"]),
                                 status="ERROR (its certifier: dual residual 1.2e-7)",
                                 source="tests/golden/c2_reference.npz (reference structured LISWET path, one CPU "
                                        "thread)"))
        return
    if args.workload == "c3w":
        run_batched_warm_start(args)
        return
    # c4: learned warm start on the multicommodity family
    from sovereign_b200.ipm import solve_family
    from sovereign_b200.warmstart import WarmStart, solve_many
    fam = P.MulticommodityFamily()
    train = [fam.instance_from_seed(100000 + k) for k in range(args.train)]
    test = [fam.instance_from_seed(900000 + k) for k in range(args.eval)]
    opts = InteriorPointOptions()
    t0 = time.perf_counter()
    # training targets: the iterate at the start of iteration 6 (early central-path stretch), made
    # in chunks so that a 50k-instance set keeps only its float32 targets in host memory
    xs, ts, ws = [], [], None
    for c0 in range(0, len(train), 2048):
        chunk = train[c0:c0 + 2048]
        # the family path: the instances share A (one symbolic analysis, 64 per launch)
        res = solve_family([m for m, _ in chunk], InteriorPointOptions(ipm_iterate_at=6), with_ipm=True)
        if ws is None:
            ws = WarmStart(fam.param_dim, res[0].n_ipm, res[0].m_ipm, hidden=512, layers=3, seed=0)
        ok, t = ws.targets(res)
        xs.append(np.stack([p for _, p in chunk])[ok])
        ts.append(t.astype(np.float32))
        del res
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = ws.fit_arrays(np.concatenate(xs), np.concatenate(ts), epochs=args.epochs, batch=128,
                         lr=1e-3)
    t_train = time.perf_counter() - t0
    cold, t_cold = solve_many([m for m, _ in test], opts, workers=args.workers)
    t0 = time.perf_counter()
    starts = ws.predict(np.stack([p for _, p in test]))
    t_pred = time.perf_counter() - t0
    warm, t_warm = solve_many([m for m, _ in test], opts, warm=starts, workers=args.workers)
    ok = [k for k in range(len(test)) if cold[k].status_name == "OPTIMAL" and warm[k].status_name == "OPTIMAL"]
    err = max(abs(cold[k].objective_value - warm[k].objective_value) / max(1.0, abs(cold[k].objective_value))
              for k in ok) if ok else None
    # the family path: every eval instance shares A, so they are solved 64 per launch with one
    # symbolic analysis (sov_lp_solve_family), cold and from the same predicted starts
    test_models = [m for m, _ in test]
    solve_family(test_models[:64])  # module load, device pools
    t0 = time.perf_counter()
    fcold = solve_family(test_models, opts)
    t_fcold = time.perf_counter() - t0
    t0 = time.perf_counter()
    fwarm = solve_family(test_models, opts, warm_starts=starts, with_diag=True)
    t_fwarm = time.perf_counter() - t0
    fok = [k for k in range(len(test)) if fcold[k].status_name == "OPTIMAL" and fwarm[k].status_name == "OPTIMAL"]
    ferr = max(abs(fwarm[k].objective_value - cold[k].objective_value) / max(1.0, abs(cold[k].objective_value))
               for k in fok) if fok else None
    value = len(test) / (t_fwarm + t_pred)
    _line(METRIC, value, UNIT, args, 1e3 * (t_fwarm + t_pred) / len(test), "f64",
          dict(workload=f"multicommodity 200 nodes / 1000 arcs / 4 commodities, {args.eval} eval instances, "
                        f"MLP 4040-512x3-11800 trained on {args.train} IPM solutions ({args.epochs} epochs); "
                        "value: the family path (64 LPs per launch, shared symbolic factor) from the predicted "
                        "starts, prediction included, wall clock"),
          cold=dict(lps_per_s=len(test) / t_cold, mean_iterations=float(np.mean([r.iterations for r in cold])),
                    sample=f"single-problem engine, {args.workers} concurrent solves"),
          warm=dict(lps_per_s=len(test) / (t_warm + t_pred), mean_iterations=float(np.mean([r.iterations for r in warm])),
                    used=int(sum(r.diagnostics["warm_start_used"] for r in warm)),
                    sample=f"single-problem engine, {args.workers} concurrent solves, prediction included"),
          family_cold=dict(lps_per_s=len(test) / t_fcold, mean_iterations=float(np.mean([r.iterations for r in fcold])),
                           optimal=f"{sum(r.status_name == 'OPTIMAL' for r in fcold)}/{len(test)}"),
          family_warm=dict(lps_per_s=value, mean_iterations=float(np.mean([r.iterations for r in fwarm])),
                           used=int(sum(r.diagnostics["warm_start_used"] for r in fwarm)),
                           optimal=f"{sum(r.status_name == 'OPTIMAL' for r in fwarm)}/{len(test)}",
                           max_rel_obj_diff_vs_single_cold=ferr),
          speedup_family_warm_vs_single_cold=value / (len(test) / t_cold),
          optimal=f"{len(ok)}/{len(test)}", max_rel_obj_diff_warm_vs_cold=err, train_loss=loss,
          seconds=dict(generate=t_gen, train=t_train, predict=t_pred, family_cold=t_fcold, family_warm=t_fwarm))


def run_batched_warm_start(args):
    """Batched + learned warm start: a parametric 40 x 40 transportation family, `--eval` instances
    solved in one sov_lp_solve_batch call cold (Mehrotra start in every CTA) and warm (one predicted
    start per LP, passed as per-LP option blocks), both through the C ABI with caller-owned host
    buffers, after training the MLP on `--train` instances' early iterates."""
    import ctypes as C

    from sovereign_b200 import _lib, abi as A, problems as P
    from sovereign_b200.ipm import InteriorPointOptions
    from sovereign_b200.model import ResultBuffers
    from sovereign_b200.warmstart import WarmStart, solve_many
    lib = _lib.load(build_if_missing=False)
    fam = P.TransportFamily()
    train = [fam.instance_from_seed(200000 + k) for k in range(args.train)]
    count = args.count
    test = [fam.instance_from_seed(700000 + k) for k in range(count)]
    t0 = time.perf_counter()
    early, _ = solve_many([m for m, _ in train], InteriorPointOptions(ipm_iterate_at=5), workers=args.workers)
    t_gen = time.perf_counter() - t0
    ws = WarmStart(fam.param_dim, early[0].n_ipm, early[0].m_ipm, hidden=512, layers=3, seed=0)
    t0 = time.perf_counter()
    loss = ws.fit(np.stack([p for _, p in train]), early, epochs=60, batch=128, lr=1e-3)
    t_train = time.perf_counter() - t0
    models = [m for m, _ in test]
    arr = (A.SovModel * count)(*[m.to_abi() for m in models])
    bufs = [ResultBuffers(m, with_diag=True) for m in models]
    res = (A.SovResult * count)(*[b.raw for b in bufs])
    base = A.default_options()

    def run(opts, stride, steps):
        best = float("inf")
        for _ in range(steps):
            t = time.perf_counter()
            _lib.check(lib.sov_lp_solve_batch(count, arr, opts, stride, res))
            best = min(best, time.perf_counter() - t)
        return best, [(r.status, r.iterations, r.objective_value, r.diagnostics.contents.warm_start_used) for r in res]

    run(C.byref(base), 0, 1)  # warm-up
    t_cold, cold = run(C.byref(base), 0, max(1, args.steps))
    params = np.stack([p for _, p in test])
    ws.predict(params)  # untimed: sizes the network's work buffers for this batch
    t0 = time.perf_counter()
    starts = ws.predict(params)
    t_pred = time.perf_counter() - t0
    opts = (A.SovOptions * count)()
    keep = []
    for k, (x, y, s_) in enumerate(starts):
        C.memmove(C.byref(opts[k]), C.byref(base), C.sizeof(A.SovOptions))
        a = [np.ascontiguousarray(v) for v in (x, y, s_)]
        keep.append(a)
        opts[k].warm_x, opts[k].warm_y, opts[k].warm_s = (A.dptr(v) for v in a)
    t_warm, warm = run(opts, C.sizeof(A.SovOptions), max(1, args.steps))
    # the same starts handed over on the device (sov_lp_solve_batch_predicted): prediction and solve
    # in one call, the starts never in host memory
    norms = [np.ascontiguousarray(v, dtype=np.float64) for v in (ws.fin.mean, ws.fin.std, ws.fout.mean, ws.fout.std)]
    params_c = np.ascontiguousarray(params, dtype=np.float64)

    def run_pred(steps):
        best = float("inf")
        for _ in range(steps):
            t = time.perf_counter()
            _lib.check(lib.sov_lp_solve_batch_predicted(ws.mlp.h, params_c.ctypes.data, *(v.ctypes.data for v in norms),
                                                        ws.n_ipm, ws.m_ipm, 1e-6, count, arr, C.byref(base), res))
            best = min(best, time.perf_counter() - t)
        return best, [(r.status, r.iterations, r.objective_value, r.diagnostics.contents.warm_start_used) for r in res]

    run_pred(1)  # warm-up
    t_pred_dev, warm_dev = run_pred(max(1, args.steps))
    same_dev = all(a == b for a, b in zip(warm, warm_dev))
    ok = [k for k in range(count) if cold[k][0] == A.OPTIMAL and warm[k][0] == A.OPTIMAL]
    err = max(abs(cold[k][2] - warm[k][2]) / max(1.0, abs(cold[k][2])) for k in ok) if ok else None
    del keep
    # device time with the batch resident (the headline's measure), cold and warm
    from sovereign_b200.ipm import DeviceBatch

    def device_ms(batch):
        batch.solve()
        times = []
        for _ in range(max(3, args.steps)):
            batch.solve()
            times.append(batch.stats()["kernel_ms"])
        return float(np.mean(times))

    # the plain FP64 GPU IPM on the same instances: the single-problem engine, PLAIN_WORKERS solves
    # in flight on separate streams (the composition's baseline: batched cold, then batched warm)
    import concurrent.futures as cf
    from sovereign_b200.ipm import InteriorPointSolver
    solver = InteriorPointSolver()
    with cf.ThreadPoolExecutor(max_workers=PLAIN_WORKERS) as ex:
        list(ex.map(solver.solve, models[:2 * PLAIN_WORKERS]))
        t0 = time.perf_counter()
        plain_res = list(ex.map(solver.solve, models))
        t_plain = time.perf_counter() - t0
    plain_err = max(abs(p.objective_value - c[2]) / max(1.0, abs(c[2])) for p, c in zip(plain_res, cold)
                    if p.status_name == "OPTIMAL" and c[0] == A.OPTIMAL)
    with DeviceBatch(models) as b:
        ms_cold = device_ms(b)
    with DeviceBatch(models, warm_starts=starts) as b:
        ms_warm = device_ms(b)
    value = count / (ms_warm * 1e-3)
    _line(METRIC, value, UNIT, args, ms_warm, "f64",
          dict(workload=f"parametric transportation family 40x40 (m=80, n=1600), {count} LPs per batch, "
                        f"MLP 1680-512x3-3280 trained on {args.train} early IPM iterates",
               parallelism="one batched launch set per step; value = device time with the batch resident"),
          cold=dict(lps_per_s=count / (ms_cold * 1e-3), mean_iterations=float(np.mean([c[1] for c in cold])),
                    e2e_lps_per_s=count / t_cold),
          warm=dict(lps_per_s=value, mean_iterations=float(np.mean([w[1] for w in warm])),
                    used=int(sum(w[3] for w in warm)), e2e_lps_per_s=count / (t_warm + t_pred), predict_s=t_pred,
                    e2e_device_starts_lps_per_s=count / t_pred_dev, device_starts_identical=same_dev),
          speedup_warm_vs_cold=ms_cold / ms_warm, optimal=f"{len(ok)}/{count}",
          plain_fp64_gpu=dict(lps_per_s=count / t_plain, workers=PLAIN_WORKERS,
                              max_rel_obj_diff_vs_batched=plain_err,
                              sample=f"the same {count} LPs through sov_lp_solve (FP64), {PLAIN_WORKERS} concurrent "
                                     "solves, wall clock"),
          composition=dict(batched_cold_vs_plain=(count / (ms_cold * 1e-3)) / (count / t_plain),
                           batched_warm_vs_plain=value / (count / t_plain),
                           e2e_batched_warm_device_starts_vs_plain=(count / t_pred_dev) / (count / t_plain)),
          max_rel_obj_diff_warm_vs_cold=err, train_loss=loss, seconds=dict(generate=t_gen, train=t_train),
          e2e=dict(value=count / (t_warm + t_pred), unit=UNIT,
                   note="sov_lp_solve_batch with per-LP warm starts from host buffers, plus the MLP prediction"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sovereign_b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain FP64 single-engine arm (profiler captures of the batched kernel)")
    ap.add_argument("--count", type=int, default=COUNT, help="LPs per step (profiling runs use fewer)")
    ap.add_argument("--workload", default="batch", choices=["batch", "c0", "c1", "c2", "c3w", "c4", "kkt", "wide"],
                    help="batch (default, headline): 4096 uneven transportation LPs; c0: one 50x50 transportation "
                         "LP; c1: random LP m=2000 n=10000 (FP64 and mixed); c2: convex-sequence QP n=20002; "
                         "c3w: parametric 40x40 transportation family, batched, learned warm start vs cold; "
                         "c4: multicommodity family, learned warm start vs Mehrotra start")
    ap.add_argument("--rows", type=int, default=2000,
                    help="c1: rows m of the random LP (n = 5m); only m = 2000 has the reference's answer")
    ap.add_argument("--train", type=int, default=1024, help="c4: training instances")
    ap.add_argument("--workers", type=int, default=16, help="c4: concurrent single-LP solves (one stream each)")
    ap.add_argument("--eval", type=int, default=128, help="c4: evaluation instances")
    ap.add_argument("--epochs", type=int, default=40, help="c4: training epochs")
    args = ap.parse_args()
    if args.workload != "batch":
        run_single_workload(args)
        return
    rank, world, local, dist = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist is not None:
            dist.destroy_process_group()
        return

    import ctypes as C

    from sovereign_b200 import _lib, problems as P
    from sovereign_b200.ipm import DeviceBatch, InteriorPointSolver, autotune, solve_batch

    lib = _lib.load(build_if_missing=False)
    # weak scaling: every rank solves its own 4096 LPs (seed offset by rank)
    count = args.count
    from sovereign_b200.shard import shard_seed
    models = P.transport_batch(count, seed=shard_seed(2026, rank))
    bytes_iter = np.array([per_lp_bytes(m) for m in models])
    flops_iter = np.array([per_lp_flops(m) for m in models])

    import torch
    torch.cuda.set_device(local)
    plain = single = None
    if rank == 0 and not args.no_plain:
        # the plain FP64 GPU IPM: the same LPs through the single-problem engine (sov_lp_solve, FP64),
        # PLAIN_WORKERS solves in flight at a time, each on its own CUDA stream, measured first
        # (after an untimed pass over a slice) so that it runs in a clean process state
        import concurrent.futures as cf
        solver = InteriorPointSolver()
        with cf.ThreadPoolExecutor(max_workers=PLAIN_WORKERS) as ex:
            list(ex.map(solver.solve, models[:2 * PLAIN_WORKERS]))
            t0 = time.perf_counter()
            single = list(ex.map(solver.solve, models))
            t_plain = time.perf_counter() - t0
        plain = dict(value=len(models) / t_plain, unit=UNIT,
                     sample=f"all {len(models)} LPs through sov_lp_solve (FP64 single-problem engine), "
                            f"{PLAIN_WORKERS} concurrent solves on separate streams, wall clock",
                     optimal=f"{sum(r.status_name == 'OPTIMAL' for r in single)}/{len(models)}")
    # untimed: threads per CTA for each size bucket, picked by timing the bucket alone
    tuning = json.loads(autotune(models))
    batch = DeviceBatch(models)
    ts = torch.cuda.Stream()
    for _ in range(args.warmup):
        batch.solve(ts.cuda_stream)
    torch.cuda.synchronize()
    res = batch.results()
    iters = np.array([r.iterations for r in res])
    status_ok = int(sum(r.status_name == "OPTIMAL" for r in res))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, local)
    with ClockSampler(local) as clk:
        ev0.record(ts)
        for _ in range(args.steps):
            batch.solve(ts.cuda_stream)
        ev1.record(ts)
        torch.cuda.synchronize()
    barrier(dist, local)
    dev_ms = ev0.elapsed_time(ev1)
    dev_ms = max_over_ranks(dist, dev_ms, local)
    stats = batch.stats()
    value = world * count * args.steps / (dev_ms * 1e-3)

    # roofline of the (only) kernel: algorithmic bytes of all IPM iterations / device time per step
    # (the same CUDA-event timing as ms_per_step: all bucket launches of a step, concurrent)
    alg_bytes = float(np.sum(bytes_iter * (iters + 1)))
    alg_flops = float(np.sum(flops_iter * (iters + 1)))
    step_s = dev_ms * 1e-3 / args.steps
    pk = peaks()
    achieved = alg_bytes / step_s / 1e9
    chosen = {k: v["chosen"] for k, v in tuning.items()}
    traffic, traffic_note = traffic_per_step(count, chosen)
    roofline = dict(bound="hbm", achieved=achieved, peak=pk["hbm_gbs"], unit="GB/s",
                    frac=achieved / pk["hbm_gbs"], traffic=traffic, traffic_note=traffic_note,
                    algorithmic_bytes_per_step=alg_bytes, kernel="k_batch_ipm", peak_source=pk["source"],
                    note="algorithmic bytes = sum over LPs of (iterations + 1) x [6 SpMV x (12 nnz + 8(m+n)) + "
                         "15 x 8n + 10 x 8m] / device time per step. traffic = DRAM bytes of one step's bucket "
                         "launches from an ncu capture run with this run's threads per bucket "
                         "(profiles/traffic.json), null when a bucket that carries traffic ran another width",
                    binding=dict(limit="latency: global-load chains of the row and column passes through L2 "
                                       "(66-75 % sector hit rate) and CTA barriers behind the one-warp phases "
                                       "(panel diagonal blocks, triangular solves); issue active 24-28 %, FP64 "
                                       "pipe 9-11 % (ncu, profiles/k_batch_ipm_transport4096.md)",
                                 fp64_tflops=alg_flops / step_s / 1e12,
                                 fp64_flops_per_step=alg_flops,
                                 note="FP64 flops = sum over LPs of (iterations + 1) x [(2/3) m^3 + 8 m^2 + "
                                      "2 sum_j k_j^2]; against the B200's nominal FP64 rate (about 37 TFLOP/s) "
                                      "this is the chain-latency bound, not a throughput one"))

    # end to end through the C ABI, sov_lp_solve_batch, with caller-owned host buffers (the models'
    # CSC arrays in, primal/dual arrays out), as a C or C++ caller holds them: host standard form,
    # H2D, solve, D2H and publishing are all inside the timed region
    from sovereign_b200 import abi as A
    from sovereign_b200.model import ResultBuffers
    arr = (A.SovModel * count)(*[m.to_abi() for m in models])
    bufs = [ResultBuffers(m) for m in models]
    res_arr = (A.SovResult * count)(*[b.raw for b in bufs])
    opt = A.default_options()
    e2e_steps = max(1, min(args.steps, 20))  # as many calls as device steps (at most 20)
    for _ in range(max(1, min(args.warmup, 2))):  # untimed, like the device steps' warm-up
        _lib.check(lib.sov_lp_solve_batch(count, arr, C.byref(opt), 0, res_arr))
    barrier(dist, local)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        _lib.check(lib.sov_lp_solve_batch(count, arr, C.byref(opt), 0, res_arr))
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(dist, e2e_s, local)
    e2e_obj_diff = max(abs(r.objective_value - q.objective_value) / max(1.0, abs(q.objective_value))
                       for r, q in zip(res_arr, res))
    h2d, d2h = C.c_double(), C.c_double()
    lib.sov_batch_transfer_bytes(batch.handle, C.byref(h2d), C.byref(d2h))
    e2e = dict(value=world * count * e2e_steps / e2e_s, unit=UNIT, h2d_bytes_per_step=int(h2d.value),
               d2h_bytes_per_step=int(d2h.value), max_rel_obj_diff_vs_device_batch=e2e_obj_diff,
               note="sov_lp_solve_batch with caller-owned host buffers: host standard form + H2D + solve + "
                    "D2H + publish, wall clock")
    # the Python wrapper adds marshalling of the model and result objects on top
    t0 = time.perf_counter()
    solve_batch(models)
    e2e["python_api_lps_per_s"] = world * count / max_over_ranks(dist, time.perf_counter() - t0, local)

    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=dev_ms / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic",
                config=dict(workload=WORKLOAD if count == COUNT else f"{count} uneven transportation LPs (profiling size)",
                            lps_per_gpu=count, precision="fp64 batched",
                            l2="per-step working set ~0.6 GB > 126 MB L2 (no flush needed)",
                            parallelism=f"independent LPs sharded per rank (dp{world})",
                            threads_per_bucket={k: v["chosen"] for k, v in tuning.items()},
                            grid_per_bucket={k: v.get("grid") for k, v in tuning.items()}),
                gpu_launches=int(stats["launches"] * args.steps), roofline=roofline, e2e=e2e,
                optimal=f"{status_ok}/{count}", mean_iterations=float(iters.mean()))
    if rank == 0:
        line["clocks"] = clk.summary()
        if plain is not None:
            line["plain_fp64_gpu"] = plain
            line["speedup_vs_plain_fp64"] = value / plain["value"]
            err = max(abs(a.objective_value - b.objective_value) / max(1.0, abs(b.objective_value))
                      for a, b in zip(res, single) if b.status_name == "OPTIMAL")
            line["max_rel_obj_diff_batched_vs_plain"] = err
        if not args.no_cpu_baseline and world == 1:
            try:
                cb = cpu_reference_sample(models)
                k = len(cb["objectives"])
                ref_obj = np.array(cb["objectives"], dtype=np.float64)
                ref_st = np.array(cb["statuses"])
                # where the reference's dense LU stops short of OPTIMAL (a pivot under its 1e-14 floor
                # on a dependent row), its own sparse L D L' path gives the comparison (untimed)
                import oracle
                os.environ["SOVEREIGN_IPM_NORMAL_EQUATIONS"] = "sparse"
                try:
                    for i in np.flatnonzero(ref_st != 0):
                        rr = oracle.solve(models[i], kind="reference")
                        ref_obj[i], ref_st[i] = rr.objective_value, rr.status
                finally:
                    del os.environ["SOVEREIGN_IPM_NORMAL_EQUATIONS"]
                both = [i for i in range(k) if ref_st[i] == 0 and res[i].status_name == "OPTIMAL"]
                line["max_rel_obj_err_vs_reference"] = float(max(
                    abs(res[i].objective_value - ref_obj[i]) / max(1.0, abs(ref_obj[i])) for i in both))
                line["reference_compared"] = len(both)
                line["reference_dense_lu_non_optimal"] = int(sum(1 for i in range(k) if cb["statuses"][i] != 0))
                for key in ("objectives", "statuses", "seconds"):
                    cb.pop(key)
                line["cpu_baseline"] = cb
            except Exception as e:  # the reference library may be missing on a fresh checkout
                line["cpu_baseline"] = dict(value=None, unit=UNIT, cores=0, kind="reference",
                                            sample=f"unavailable: {e}")
        print(json.dumps(line))
    batch.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
