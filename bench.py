"""Benchmark: accepted DOP853 steps per second on the uneven Bovy-composite
workload at rtol = atol = 1e-10, against the plain one-thread-per-particle
launch.

Default workload (one "step" = one pass of the integration path over one
batch): 4,194,304 test particles in the Bovy-style composite (power-law bulge
with cutoff, Miyamoto-Nagai disk, NFW halo; natural units), R log-uniform on
[0.05, 20], z ~ N(0, 0.1 R), near-circular velocities with 10 % dispersion,
per-particle end times t_end ~ U[10, 1000] with 101 outputs each, DOP853 at
rtol = atol = 1e-10 in float64: a (101, 2^22, 6) trajectory (20.3 GB) per
pass, step counts per particle spanning three decades.

* ``value``        -- device path: inputs resident in HBM, one
  ``drift_integrate`` call per pass (ordered longest-first persistent
  schedule), timed with CUDA events on the launching stream.
* ``plain_launch`` -- one pass of the same particles under the plain schedule
  (one thread per particle for the life of the launch, the reference's
  launch, kernels/src/lib.rs:175-216); ``vs_plain_launch`` is the ratio.
* ``e2e``          -- the same metric through ``drift_integrate_host`` with
  pinned host buffers: host->device copy of the initial states and end times
  and device->host copy of every trajectory sample inside the timed region.
* ``cpu_baseline`` -- the CPU oracle (a line-faithful C restatement of the
  reference's CPU integrator) on a bounded seeded subsample, all host threads
  and one thread.
* ``serving``      -- a short pass of the request server on the mixed-request
  workload: p50/p99 latency of an open-loop Poisson stream and the saturated
  throughput against serial plain launches (``--workload serving`` runs the
  full sweep).
* ``--impl reference`` times the CPU oracle alone on the chosen workload (the
  reference's own CPU path is Rust and cannot be built here).

Other workloads: ``--workload plummer`` (2^20 Plummer particles, DOP853
1e-12), ``kepler`` (1,024 Kepler particles, DOPR54 1e-10), ``serving`` (the
Poisson request stream swept over arrival rates) and ``stream-gradient``
(forward + discrete-adjoint gradient of a stream-track loss).

Multi-GPU (torchrun): every rank integrates its own seeded particles of the
same size (weak scaling, no data-path collective); time is the max over
ranks and ``value`` the accepted steps of all ranks over that time.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

COUNTS = json.loads((ROOT / "astrodrift_b200" / "roofline_counts.json").read_text())

# The single-GPU workloads timed as device passes.
#   counts: key of astrodrift_b200/roofline_counts.json (exact operation
#           counts of the reference algorithm per accepted step, rejected
#           step, emitted sample and particle);
#   traffic_per_particle: DRAM bytes (read + write) per particle of one
#           ordered-schedule launch, from the ncu capture named in
#           traffic_source (a slice of the workload; traffic grows with the
#           particles processed, so a full launch is this times n).
WORKLOADS = {
    "bovy": dict(
        name="bovy-uneven-dop853", particles=1 << 22, nt=101, tol=1e-10, method="DOP853",
        potential="bovy composite (bulge alpha 1.8, rc 0.2375, F_r(1) -0.05; MN 0.7574802019, a 0.375, "
                  "b 0.035; NFW 4.852230533528, a 2)",
        grid="per-particle t0 = 0 .. t_end ~ U[10, 1000], 101 outputs", counts="dop853_bovy",
        traffic_per_particle=(0.965953280e9 + 1.748899072e9) / 262144,
        traffic_source="ncu dram__bytes_read+write of the first 262,144 particles "
                       "(profiles/dop853_bovy_uneven_slices.txt, section 7), times particles",
        data="synthetic (seeded Bovy disc: R log-uniform [0.05, 20], z ~ N(0, 0.1 R), 10 % dispersion)"),
    "plummer": dict(
        name="plummer-dop853", particles=1 << 20, nt=201, tol=1e-12, method="DOP853",
        potential="plummer(amp=1, b=1)", grid="ts = (0, 100, 201)", counts="dop853_plummer",
        traffic_per_particle=(1.696054272e9 + 3.397321984e9) / 262144,
        traffic_source="ncu dram__bytes_read+write of 262,144 particles (profiles/dop853_plummer_c2.txt, "
                       "section 5), times particles",
        data="synthetic (seeded isotropic Plummer DF, amp=1, b=1)"),
    "kepler": dict(
        name="kepler-dopr54", particles=1024, nt=1001, tol=1e-10, method="DOPR54",
        potential="kepler galpy cylindrical (amp=1)", grid="ts = (0, 20 pi, 1001)", counts="dopr54_kepler",
        traffic_per_particle=None, traffic_source=None,
        data="synthetic (seeded Kepler disc: r ~ U[0.5, 2], isotropic planes)"),
}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def log(msg: str) -> None:
    print(f"bench: {msg}", file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_id}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_uuid(torch, dev) -> str:
    u = str(torch.cuda.get_device_properties(dev).uuid)
    return u if u.startswith("GPU-") else f"GPU-{u}"


def fp64_peak_tflops(torch) -> float:
    """Measured FP64 peak: cuBLAS DGEMM (torch.matmul, float64, 8192^3), best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def measured_hbm_gbs() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "profiling-recipe fallback 6.65 TB/s"


# ---------------------------------------------------------------------------
# Workload inputs (host numpy, identical in every arm)
# ---------------------------------------------------------------------------

def make_inputs(workload: str, n: int, seed_offset: int = 0):
    """(y0 (n, 6), ts or None, t_end or None, nt) of a workload's first n
    particles; rank r of a multi-GPU run draws with its own seed."""
    from astrodrift_b200.workloads import bovy_disc, kepler_disc, plummer_sphere

    wl = WORKLOADS[workload]
    if workload == "bovy":
        y0, t_end = bovy_disc(wl["particles"], seed=3 + seed_offset)
        return np.ascontiguousarray(y0[:n]), None, np.ascontiguousarray(t_end[:n]), wl["nt"]
    if workload == "plummer":
        return plummer_sphere(wl["particles"], seed=2 + seed_offset)[:n], np.linspace(0.0, 100.0, 201), None, 201
    return kepler_disc(n, seed=1 + seed_offset), np.linspace(0.0, 20.0 * np.pi, 1001), None, 1001


def _oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.build()
    return oracle


def cpu_oracle_rate(workload: str, y0, ts, t_end, nt, sample: int, threads: int, seed: int = 12345) -> dict:
    """The CPU oracle on a seeded subsample of the workload; accepted steps/s."""
    oracle = _oracle()
    wl = WORKLOADS[workload]
    idx = np.sort(np.random.default_rng(seed).choice(len(y0), min(sample, len(y0)), replace=False))
    opot = {"bovy": oracle.bovy(), "plummer": oracle.plummer(1.0, 1.0), "kepler": oracle.kepler(1.0)}[workload]
    method = oracle.DOP853 if wl["method"] == "DOP853" else oracle.DOPR54
    kw = dict(ts=ts) if ts is not None else dict(t_end=t_end[idx], nt=nt)
    t0 = time.perf_counter()
    res = oracle.integrate_batch(method, opot, y0[idx], rtol=wl["tol"], atol=wl["tol"], threads=threads,
                                 want_output=True, **kw)
    dt = time.perf_counter() - t0
    acc = int(res["accepted"].astype(np.int64).sum())
    return {"value": acc / dt, "seconds": dt, "accepted": acc, "particles": int(len(idx))}


def accuracy_vs_oracle(workload: str, y0, ts, t_end, nt, out_sample, accepted_sample, idx) -> dict:
    """Max relative error per sample and accepted-step agreement of a seeded
    particle sample against the CPU oracle (run after timing).
    out_sample: (nt, len(idx), 6) of the benchmarked build."""
    oracle = _oracle()
    wl = WORKLOADS[workload]
    opot = {"bovy": oracle.bovy(), "plummer": oracle.plummer(1.0, 1.0), "kepler": oracle.kepler(1.0)}[workload]
    method = oracle.DOP853 if wl["method"] == "DOP853" else oracle.DOPR54
    kw = dict(ts=ts) if ts is not None else dict(t_end=t_end[idx], nt=nt)
    ref = oracle.integrate_batch(method, opot, y0[idx], rtol=wl["tol"], atol=wl["tol"],
                                 threads=os.cpu_count() or 1, **kw)
    scale = np.maximum(np.abs(ref["out"]).max(axis=2), 1e-300)
    err = np.abs(out_sample - ref["out"]).max(axis=2) / scale
    return {"particles": int(len(idx)), "max_rel_err": float(err.max()), "median_rel_err": float(np.median(err)),
            "accepted_step_agreement": float((accepted_sample.astype(np.int64) == ref["accepted"]).mean())}


# ---------------------------------------------------------------------------
# Reference arm: the CPU oracle alone
# ---------------------------------------------------------------------------

def run_reference(args) -> None:
    world, rank, _ = _dist()
    if rank != 0:
        return  # rank 0 alone times the CPU path
    workload = args.workload if args.workload in WORKLOADS else "bovy"
    wl = WORKLOADS[workload]
    n = args.particles or wl["particles"]
    y0, ts, t_end, nt = make_inputs(workload, n)
    threads = os.cpu_count() or 1
    sample = args.cpu_sample or {"bovy": 4096, "plummer": 65536, "kepler": 1024}[workload]
    for _ in range(args.warmup):
        cpu_oracle_rate(workload, y0, ts, t_end, nt, max(64, sample // 16), threads, seed=99)
    vals, secs = [], []
    for k in range(args.steps):
        r = cpu_oracle_rate(workload, y0, ts, t_end, nt, sample, threads, seed=12345 + k)
        vals.append(r["value"])
        secs.append(r["seconds"])
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "accepted steps/s", "value": value,
        "unit": "accepted steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": wl["data"],
        "config": {"workload": wl["name"], "particles": n, "nt": nt, "grid": wl["grid"], "rtol": wl["tol"],
                   "atol": wl["tol"], "method": wl["method"], "potential": wl["potential"]},
        "cpu_baseline": {"value": value, "unit": "accepted steps/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} seeded particles of the {n} per step (a new seed each step), "
                                   "full time spans and output grids"},
        "e2e": {"value": value, "unit": "accepted steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference's CPU path is Rust and cannot be built here; this times the oracle, a "
                "line-faithful C restatement of src/integrators/galpy/dop853.rs and dopr54.rs",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Device workloads (configurations 1 to 3)
# ---------------------------------------------------------------------------

def run_device(args) -> None:
    import torch

    from astrodrift_b200 import capi

    workload = args.workload
    wl = WORKLOADS[workload]
    world, rank, local = _dist()
    if workload == "kepler" and world > 1 and rank != 0:
        return  # one small batch: rank 0 alone
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    dist = None
    if world > 1 and workload != "kepler":
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900), device_id=dev)

    n = args.particles or wl["particles"]
    y0, ts, t_end, nt = make_inputs(workload, n, seed_offset=rank)
    pot = {"bovy": capi.bovy(), "plummer": capi.plummer(1.0, 1.0), "kepler": capi.kepler(1.0)}[workload]
    method = capi.DOP853 if wl["method"] == "DOP853" else capi.DOPR54
    tol = wl["tol"]
    precision = capi.EXACT if args.precision == "exact" else capi.FMA
    schedule = {"plain": capi.PLAIN, "persistent": capi.PERSISTENT, "ordered": capi.ORDERED}[args.schedule]
    log(f"{wl['name']}: {n} particles, nt {nt}, rank {rank}/{world}")

    y0_d = torch.from_numpy(y0).to(dev)
    grid_d = torch.from_numpy(ts if ts is not None else t_end).to(dev)
    out_d = torch.empty((nt, n, 6), dtype=torch.float64, device=dev)
    acc_d = torch.zeros(n, dtype=torch.int32, device=dev)
    rej_d = torch.zeros(n, dtype=torch.int32, device=dev)
    st_d = torch.zeros(n, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def make(sched):
        L = capi.make_launch(method, pot, n, nt, rtol=tol, atol=tol, precision=precision, schedule=sched,
                             block_size=args.block)
        L.y0, L.out = y0_d.data_ptr(), out_d.data_ptr()
        if ts is not None:
            L.ts = grid_d.data_ptr()
        else:
            L.t_end = grid_d.data_ptr()
        L.n_accepted, L.n_rejected, L.status = acc_d.data_ptr(), rej_d.data_ptr(), st_d.data_ptr()
        ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
        L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
        return L, ws

    def passes(L, count):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(count)]
        for a_, b_ in ev:
            a_.record(stream)
            capi.integrate_device(L, stream.cuda_stream)
            b_.record(stream)
        torch.cuda.synchronize()
        return [a_.elapsed_time(b_) / 1e3 for a_, b_ in ev]

    L, ws = make(schedule)
    warm = max(args.warmup, 3)
    passes(L, warm)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_uuid(torch, dev)) as clocks:
        t_start = torch.cuda.Event(enable_timing=True)
        t_stop = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        launch_s = passes(L, args.steps)
        t_stop.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    elapsed = t_start.elapsed_time(t_stop) / 1e3
    mean_launch = statistics.mean(launch_s)
    status = st_d.cpu().numpy()
    acc_h = acc_d.cpu().numpy().astype(np.int64)
    accepted = int(acc_h.sum())
    rejected = int(rej_d.cpu().numpy().astype(np.int64).sum())
    not_ok = int((status != 0).sum())
    if not_ok:
        raise RuntimeError(f"{not_ok} particles did not finish (status {np.unique(status)})")
    log(f"device: {mean_launch * 1e3:.1f} ms per pass, {accepted} accepted steps")

    from astrodrift_b200.energy import angular_momentum_drift, drift_summary

    first_h, last_h = out_d[0].cpu().numpy(), out_d[nt - 1].cpu().numpy()
    e_drift = drift_summary(pot, first_h, last_h)
    l_drift = angular_momentum_drift(pot, first_h, last_h)
    out_last_ordered = last_h

    # the plain launch of the same particles (one pass, after the timed region)
    plain = None
    if schedule != capi.PLAIN and not args.no_plain:
        Lp, wsp = make(capi.PLAIN)
        psecs = passes(Lp, 1)
        same = bool(np.array_equal(out_d[nt - 1].cpu().numpy(), out_last_ordered))
        plain = {"value": accepted / psecs[0], "seconds": psecs[0], "speedup": psecs[0] / mean_launch,
                 "bitwise_equal_final_samples": same}
        log(f"plain launch: {psecs[0] * 1e3:.1f} ms per pass ({psecs[0] / mean_launch:.2f}x slower)")
        del wsp

    # accuracy of a seeded sample against the oracle (checker, after timing)
    acc_sample = None
    if rank == 0 and not args.no_cpu:
        idx = np.sort(np.random.default_rng(777).choice(n, min(256, n), replace=False))
        sub = out_d[:, torch.from_numpy(idx).to(dev)].cpu().numpy()
        acc_sample = accuracy_vs_oracle(workload, y0, ts, t_end, nt, sub, acc_h[idx], idx)
        log(f"accuracy: {acc_sample}")

    value_local = accepted / mean_launch
    accepted_all = float(accepted)
    elapsed_max = elapsed
    if dist:
        from astrodrift_b200.sharding import reduce_max, reduce_sum

        elapsed_max = reduce_max(elapsed, dist, dev)
        accepted_all = reduce_sum(accepted, dist, dev)
    value = accepted_all * args.steps / elapsed_max

    # --- end to end through the host entry point with pinned buffers -------
    e2e = None
    if args.e2e_steps > 0:
        del out_d
        torch.cuda.empty_cache()
        e2e = e2e_leg(args, capi, torch, method, pot, y0, ts, t_end, nt, tol, precision, schedule,
                      accepted_all, dist, dev, out_last_ordered)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return

    fp64_peak = float("nan") if args.no_peak else fp64_peak_tflops(torch)
    hbm_peak, hbm_src = measured_hbm_gbs()
    counts = COUNTS[wl["counts"]]
    fl = counts["flops"]
    samples = n * (nt - 1)
    per_sample = fl["per_sample"] or 0
    flops = accepted * fl["per_accepted"] + rejected * fl["per_rejected"] + samples * per_sample + n * fl["per_particle"]
    calls = {k: accepted * counts[k]["per_accepted"] + rejected * counts[k]["per_rejected"] + n * counts[k]["per_particle"]
             for k in ("pow", "exp", "log", "gamma") if k in counts}
    achieved = flops / mean_launch / 1e12
    bytes_alg = 48 * n * (nt + 1) + (8 * nt if ts is not None else 8 * n) + 13 * n
    traffic = wl["traffic_per_particle"] * n if wl["traffic_per_particle"] else None

    cpu = None
    if world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        sample = args.cpu_sample or {"bovy": 4096, "plummer": 65536, "kepler": 1024}[workload]
        r = cpu_oracle_rate(workload, y0, ts, t_end, nt, sample, threads)
        one_n = max(64, sample // 32)
        one = cpu_oracle_rate(workload, y0, ts, t_end, nt, one_n, 1, seed=4321)
        cpu = {"value": r["value"], "unit": "accepted steps/s", "cores": threads, "kind": "port",
               "sample": f"{r['particles']} seeded particles of the {n}, full spans and grids ({r['seconds']:.1f} s)",
               "one_core": {"value": one["value"], "cores": 1,
                            "sample": f"{one['particles']} particles ({one['seconds']:.1f} s), the reference's "
                                      "serial per-particle loop"}}

    serving = None
    if world == 1 and workload == "bovy" and args.serving_seconds > 0 and not args.no_serving:
        serving = serving_short_pass(args)

    line = {
        "metric": "accepted steps/s",
        "value": value,
        "unit": "accepted steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": warm,
        "ms_per_step": 1e3 * elapsed_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": wl["data"],
        "config": {"workload": wl["name"] if n == wl["particles"] else f"{wl['name']} (first {n} of {wl['particles']})",
                   "particles_per_gpu": n, "nt": nt, "grid": wl["grid"], "rtol": tol, "atol": tol,
                   "method": wl["method"], "potential": wl["potential"], "precision": args.precision,
                   "schedule": args.schedule,
                   "l2": f"inputs+outputs ({48 * n * (nt + 1) / 1e9:.2f} GB per pass) exceed the 126 MB L2; "
                         "no flush" if 48 * n * (nt + 1) > (1 << 28) else "small working set; no flush"},
        "accepted_steps_per_pass": accepted_all,
        "rejected_steps_per_pass": rejected,
        "steps_per_particle": {"median": float(np.median(acc_h)), "max": int(acc_h.max()), "min": int(acc_h.min())},
        "gpu_launches": args.steps * (4 if schedule == capi.ORDERED else 1),
        "gpu_launches_note": "per pass: the integration kernel, plus the rank, scan and scatter kernels of the "
                             "longest-first queue under the ordered schedule",
        "vs_plain_launch": plain["speedup"] if plain else None,
        "plain_launch": plain,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp64_peak, "traffic": traffic,
                     "traffic_source": wl["traffic_source"],
                     "peak_source": "FP64 DGEMM (torch.matmul float64 8192^3, best of 5) measured in this run; "
                                    "MEASURED_PEAKS.json has no FP64 figure",
                     "flops_per_launch": flops,
                     "units": f"{accepted} accepted x {fl['per_accepted']} + {rejected} rejected x "
                              f"{fl['per_rejected']} + {samples} samples x {per_sample} + {n} particles x "
                              f"{fl['per_particle']}",
                     "special_calls_per_s": {k: v / mean_launch for k, v in calls.items() if v},
                     "counts_source": "astrodrift_b200/roofline_counts.json (exact operation counts of the "
                                      "reference algorithm; pow/exp/log and the bulge's incomplete gamma are "
                                      "calls, not flops)"},
        "roofline_hbm": {"bound": "hbm", "achieved": bytes_alg / mean_launch / 1e9, "peak": hbm_peak,
                         "unit": "GB/s", "frac": bytes_alg / mean_launch / 1e9 / hbm_peak, "peak_source": hbm_src,
                         "algorithmic_bytes": bytes_alg},
        "kernel_ms_mean": 1e3 * mean_launch,
        "rank0_value": value_local,
        "energy_drift": e_drift,
        "angular_momentum_drift": l_drift,
        "accuracy": acc_sample,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "serving": serving,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def e2e_leg(args, capi, torch, method, pot, y0, ts, t_end, nt, tol, precision, schedule, accepted_all, dist,
            dev, out_last_device) -> dict:
    """The metric through drift_integrate_host (the C ABI's host-buffer entry
    point) with page-locked host buffers: every pass copies the initial
    states and grid in and the whole trajectory out inside the timed region."""
    import ctypes

    n = len(y0)
    lib = capi.lib()
    grid = ts if ts is not None else t_end
    bufs = {}

    def pinned(name, shape, dtype=np.float64):
        ptr = ctypes.c_void_p()
        nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        capi.check(lib.drift_host_alloc(nbytes, ctypes.byref(ptr)), "drift_host_alloc")
        bufs[name] = ptr
        arr = np.ctypeslib.as_array((ctypes.c_char * nbytes).from_address(ptr.value))
        return arr.view(dtype).reshape(shape)

    y0_p = pinned("y0", (n, 6))
    y0_p[:] = y0
    grid_p = pinned("grid", grid.shape)
    grid_p[:] = grid
    out_p = pinned("out", (nt, n, 6))
    per = dict(y_final=pinned("yf", (n, 6)), status=pinned("st", (n,), np.uint8),
               acc=pinned("acc", (n,), np.uint32), rej=pinned("rej", (n,), np.uint32))

    L = capi.make_launch(method, pot, n, nt, rtol=tol, atol=tol, precision=precision, schedule=schedule,
                         block_size=args.block)
    L.y0 = y0_p.ctypes.data
    if ts is not None:
        L.ts = grid_p.ctypes.data
    else:
        L.t_end = grid_p.ctypes.data
    L.out, L.y_final = out_p.ctypes.data, per["y_final"].ctypes.data
    L.status, L.n_accepted, L.n_rejected = per["status"].ctypes.data, per["acc"].ctypes.data, per["rej"].ctypes.data

    def one():
        capi.check(lib.drift_integrate_host(ctypes.byref(L)), "drift_integrate_host")

    one()  # warm: grows the context's buffers
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        one()
    elapsed = time.perf_counter() - t0
    if dist:
        from astrodrift_b200.sharding import reduce_max

        elapsed = reduce_max(elapsed, dist, dev)
    ok = bool(np.array_equal(out_p[nt - 1], out_last_device))
    # the copy roofline of this leg: pinned device->host bandwidth (1 GiB copies)
    probe_n = min(1 << 27, out_p.size)
    probe = torch.empty(probe_n, dtype=torch.float64, device=dev)
    host_probe = torch.from_numpy(out_p.reshape(-1)[:probe_n])
    d2h = []
    for _ in range(3):
        a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a_.record()
        host_probe.copy_(probe, non_blocking=True)
        b_.record()
        torch.cuda.synchronize()
        d2h.append(probe.numel() * 8 / (a_.elapsed_time(b_) * 1e-3) / 1e9)
    del probe, host_probe
    d2h_gbs = max(d2h)
    out_bytes = nt * n * 48
    res = {"value": accepted_all * args.e2e_steps / elapsed, "unit": "accepted steps/s",
           "h2d_bytes_per_step": int(y0.nbytes + grid.nbytes),
           "d2h_bytes_per_step": int(out_bytes + n * (48 + 1 + 4 + 4)),
           "ms_per_step": 1e3 * elapsed / args.e2e_steps, "steps": args.e2e_steps,
           "matches_device_path": ok,
           "copy_roofline": {"bound": "pcie_d2h", "peak_gbs": d2h_gbs,
                             "achieved_gbs": out_bytes * args.e2e_steps / elapsed / 1e9,
                             "frac": out_bytes * args.e2e_steps / elapsed / 1e9 / d2h_gbs,
                             "peak_source": f"pinned {probe_n * 8 / 2**30:.3g} GiB device->host copies measured "
                                            "in this run"}}
    del y0_p, grid_p, out_p, per
    for ptr in bufs.values():
        lib.drift_host_free(ptr)
    log(f"e2e: {res['ms_per_step']:.1f} ms per pass")
    return res


# ---------------------------------------------------------------------------
# Serving (configuration 4)
# ---------------------------------------------------------------------------

def serving_requests(count, seed, capi, arrival_rate=None):
    """The seeded mixed-request workload.  Each request: N = floor(2^U[0,20])
    particles; potential uniform in {Kepler(1), Plummer(1,1), Bovy}; method
    uniform in {DOPR54, DOP853}; nt = floor(exp(U[ln 2, ln 10001])) outputs on
    (0, t_end), t_end ~ U[10, 100]; rtol = atol uniform in {1e-8, 1e-10,
    1e-12}; initial conditions from that potential's generator.  With
    ``arrival_rate``, arrival times of a Poisson stream (seconds)."""
    from astrodrift_b200.workloads import bovy_disc, kepler_disc, plummer_sphere

    rng = np.random.default_rng(seed)
    pools = [capi.kepler(1.0), capi.plummer(1.0, 1.0), capi.bovy()]
    reqs, t = [], 0.0
    for _ in range(count):
        if arrival_rate:
            t += rng.exponential(1.0 / arrival_rate)
        n = int(2 ** rng.uniform(0, 20))
        kind = int(rng.integers(3))
        method = int(rng.integers(2))
        nt = int(np.exp(rng.uniform(np.log(2), np.log(10001))))
        rtol = float([1e-8, 1e-10, 1e-12][int(rng.integers(3))])
        t_end = float(rng.uniform(10.0, 100.0))
        s = int(rng.integers(1 << 31))
        if kind == 0:
            y0 = kepler_disc(n, seed=s)
        elif kind == 1:
            y0 = plummer_sphere(n, seed=s)
        else:
            y0, _ = bovy_disc(n, seed=s)
        reqs.append(dict(at=t, method=method, pot=pools[kind], kind=kind, y0=y0, nt=nt, t_end=t_end, rtol=rtol))
    return reqs


class ResultSlots:
    """Page-locked result buffers of cap_bytes each (drift_host_alloc), reused
    across requests, as a serving client keeps them: results then copy at the
    device-to-host rate instead of through the CUDA driver's pageable staging and
    first-touch page faults."""

    def __init__(self, count: int, cap_bytes: int):
        from astrodrift_b200.serving import PinnedArray

        self.bufs = [PinnedArray((cap_bytes // 8,)) for _ in range(count)]
        self.free = list(range(count))

    def view(self, slot: int, nt: int, n: int) -> np.ndarray:
        return self.bufs[slot].array[: nt * n * 6].reshape(nt, n, 6)

    def close(self) -> None:
        for b in self.bufs:
            b.free()


def _serve(srv, reqs, cap_bytes, precision, open_loop: bool, slots: ResultSlots):
    """Submit every request (at its arrival time when open_loop, else all at
    once); returns (seconds, accepted steps, latencies s, capped count, client
    waits s).  Results come back into the page-locked slots; when all are in
    use the client first waits for whichever request in flight finishes first
    (drift_server_wait_any; the wait is recorded, the request's own latency
    runs from its submission).  A request whose trajectory exceeds cap_bytes
    returns its final states only (its integration, dense output included, is
    unchanged; the samples are not stored)."""
    inflight, lat, waits, capped, acc = [], [], [], 0, 0

    def retire():
        nonlocal acc
        i, res = srv.wait_any([h for h, _ in inflight], timeout=3600.0)
        _, slot = inflight.pop(i)
        lat.append(res["latency_s"])
        acc += int(res["accepted"].astype(np.int64).sum())
        if slot is not None:
            slots.free.append(slot)

    t_begin = time.perf_counter()
    for r in reqs:
        if open_loop:
            delay = r["at"] - (time.perf_counter() - t_begin)
            if delay > 0:
                time.sleep(delay)
        n, nt = len(r["y0"]), r["nt"]
        want = nt * n * 48 <= cap_bytes
        capped += not want
        slot = None
        if want:
            t_want = time.perf_counter()
            while not slots.free:
                retire()
            waits.append(time.perf_counter() - t_want)
            slot = slots.free.pop()
        h = srv.submit(r["method"], r["pot"], r["y0"], ts=np.linspace(0.0, r["t_end"], nt), rtol=r["rtol"],
                       atol=r["rtol"], precision=precision, want_out=want,
                       out=slots.view(slot, nt, n) if want else None)
        inflight.append((h, slot))
    while inflight:
        retire()
    return time.perf_counter() - t_begin, acc, lat, capped, waits


def _serial(capi, reqs, cap_bytes, precision, slots: ResultSlots):
    """One drift_integrate_host call per request, plain schedule, one after
    another, results into a page-locked slot: the serial plain-launch
    baseline (and each request's time alone)."""
    alone, acc = [], 0
    t0 = time.perf_counter()
    for r in reqs:
        n, nt = len(r["y0"]), r["nt"]
        want = nt * n * 48 <= cap_bytes
        ti = time.perf_counter()
        res = capi.integrate_host(r["method"], r["pot"], r["y0"], ts=np.linspace(0.0, r["t_end"], nt),
                                  rtol=r["rtol"], atol=r["rtol"], precision=precision, schedule=capi.PLAIN,
                                  want_out=want, out=slots.view(0, nt, n) if want else None)
        alone.append(time.perf_counter() - ti)
        acc += int(res["accepted"].astype(np.int64).sum())
    return time.perf_counter() - t0, acc, alone


def _warm_server_kernels(capi, precision):
    y = np.array([[1.0, 0.0, 0.1, 0.0, 1.0, 0.0]])
    for pot in (capi.kepler(1.0), capi.plummer(1.0, 1.0), capi.bovy()):
        for method in (capi.DOPR54, capi.DOP853):
            for sched in (capi.PLAIN, capi.PERSISTENT, capi.ORDERED):
                capi.integrate_host(method, pot, y, ts=np.linspace(0, 1, 3), rtol=1e-8, atol=1e-8,
                                    precision=precision, schedule=sched)


def _pct(lat_s) -> dict:
    ms = np.asarray(lat_s) * 1e3
    return {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99)),
            "mean": float(ms.mean()), "max": float(ms.max())}


def serving_short_pass(args) -> dict:
    """Serving keys for the default line: the saturated throughput of a
    seeded set of requests against their serial plain launches, and the
    p50/p99 latency of a short open-loop Poisson stream at half the
    saturated capacity.  The saturated time is the median of three passes
    after one untimed warm-up pass, as in the full serving sweep."""
    from astrodrift_b200 import capi
    from astrodrift_b200.serving import Server

    precision = capi.EXACT if args.precision == "exact" else capi.FMA
    cap = args.trajectory_cap_mib << 20
    _warm_server_kernels(capi, precision)
    calib = serving_requests(args.serving_requests, args.seed, capi)
    slots = ResultSlots(args.result_buffers, cap)
    try:
        _serial(capi, calib, cap, precision, slots)  # warm, as the server's pool is warmed
        t_serial, acc_serial, _ = _serial(capi, calib, cap, precision, slots)
        with Server(memory_fraction=0.6, streams=args.streams) as srv:
            _serve(srv, calib, cap, precision, False, slots)  # warms the pool
            # median of three: the server admits in arrival order, so a pass
            # runs long when one of the largest requests happens to start late
            sat = sorted((_serve(srv, calib, cap, precision, False, slots) for _ in range(3)), key=lambda p: p[0])
            t_sat, acc_sat = sat[1][0], sat[1][1]
            rate = 0.5 * len(calib) / t_sat
            stream = serving_requests(max(8, int(rate * args.serving_seconds)), args.seed + 1, capi,
                                      arrival_rate=rate)
            t_run, acc_run, lat, capped, waits = _serve(srv, stream, cap, precision, True, slots)
    finally:
        slots.close()
    pct = _pct(lat)
    res = {"p50_ms": pct["p50"], "p99_ms": pct["p99"], "vs_serial": (acc_sat / t_sat) / (acc_serial / t_serial),
           "saturated_value": acc_sat / t_sat, "serial_value": acc_serial / t_serial,
           "saturated_passes_seconds": [p[0] for p in sat],
           "open_loop": {"rate_per_s": rate, "offered_load": 0.5, "requests": len(stream), "seconds": t_run,
                         "accepted_steps_per_s": acc_run / t_run, "latency_ms": pct, "capped_requests": capped,
                         "client_buffer_wait_ms_p99": float(np.percentile(np.array(waits) * 1e3, 99)) if waits else 0.0},
           "calibration_requests": len(calib),
           "note": "short pass; --workload serving sweeps three rates for 60 s each"}
    log(f"serving: p50 {pct['p50']:.1f} ms p99 {pct['p99']:.1f} ms, {res['vs_serial']:.2f}x serial")
    return res


def run_serving(args) -> None:
    """Configuration 4: Poisson request streams through the resident request
    server, swept over arrival rates.

    A seeded calibration set of --serving-requests requests is run (i) one
    drift_integrate_host call at a time under the plain schedule (the serial
    plain-launch baseline; one untimed pass first grows the host path's
    buffers) and (ii) all submitted at once to the server
    (saturated, continuous batching; median of three passes after a warm-up
    pass), which gives the capacity in requests/s.  Then, for each offered
    load in --loads, a fresh seeded Poisson stream at that fraction of the
    capacity arrives for --stream-seconds seconds; every request's latency
    (submission to results in host memory) is recorded.  Results go to
    --result-buffers page-locked buffers reused across requests, as a serving
    client keeps them (a client whose buffers are all in use waits for its
    oldest request; the line reports that wait).  Requests whose trajectory
    exceeds --trajectory-cap-mib return final states only: their integration
    (dense output included) is unchanged, the samples are not stored, and the
    line reports how many requests that touched.
    """
    import torch

    from astrodrift_b200 import capi
    from astrodrift_b200.serving import Server

    world, rank, local = _dist()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    precision = capi.EXACT if args.precision == "exact" else capi.FMA
    cap = args.trajectory_cap_mib << 20
    _warm_server_kernels(capi, precision)
    calib = serving_requests(args.serving_requests, args.seed, capi)
    log(f"serving: {len(calib)} calibration requests, {sum(len(r['y0']) for r in calib)} particles")
    slots = ResultSlots(args.result_buffers, cap)
    _serial(capi, calib, cap, precision, slots)  # warm, as the server's pool is warmed
    t_serial, acc_serial, alone = _serial(capi, calib, cap, precision, slots)
    log(f"serving: serial {t_serial:.2f} s")
    gpu = gpu_uuid(torch, torch.device(f"cuda:{local}"))
    with Server(memory_fraction=0.6, streams=args.streams, sm_reserve_percent=args.sm_reserve) as srv:
        _serve(srv, calib, cap, precision, False, slots)
        sat = sorted((_serve(srv, calib, cap, precision, False, slots) for _ in range(3)), key=lambda p: p[0])
        t_sat, acc_sat = sat[1][0], sat[1][1]
        capacity = len(calib) / t_sat
        log(f"serving: saturated {t_sat:.2f} s ({capacity:.2f} requests/s)")
        sweeps = []
        with ClockSampler(gpu) as clocks:
            for k, load in enumerate(float(x) for x in args.loads.split(",") if x):
                rate = load * capacity
                count = max(8, int(round(rate * args.stream_seconds)))
                stream = serving_requests(count, args.seed + 100 + k, capi, arrival_rate=rate)
                t_run, acc_run, lat, capped, waits = _serve(srv, stream, cap, precision, True, slots)
                pct = _pct(lat)
                sweeps.append({"offered_load": load, "rate_per_s": rate, "requests": count,
                               "particles": int(sum(len(r["y0"]) for r in stream)),
                               "arrival_window_s": float(stream[-1]["at"]), "seconds": t_run,
                               "accepted_steps_per_s": acc_run / t_run, "latency_ms": pct,
                               "capped_requests": capped, "capped_fraction": capped / count,
                               "client_buffer_wait_ms_p99": float(np.percentile(np.array(waits) * 1e3, 99))
                               if waits else 0.0})
                log(f"serving: load {load} ({rate:.2f}/s, {count} requests) p50 {pct['p50']:.1f} ms "
                    f"p99 {pct['p99']:.1f} ms")
        st = srv.stats()
    slots.close()
    alone_ms = np.array(alone) * 1e3
    line = {
        "metric": "accepted steps/s (served request stream)",
        "value": acc_sat / t_sat,
        "unit": "accepted steps/s",
        "n_gpus": 1,
        "steps": len(calib),
        "warmup": 1,
        "ms_per_step": 1e3 * t_sat / len(calib),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded request streams)",
        "config": {"workload": "serving", "calibration_requests": len(calib), "streams": args.streams,
                   "sm_reserve_percent": args.sm_reserve, "precision": args.precision,
                   "trajectory_cap_bytes": cap, "result_buffers": args.result_buffers,
                   "stream_seconds": args.stream_seconds, "seed": args.seed},
        "vs_serial": (acc_sat / t_sat) / (acc_serial / t_serial),
        "serial_plain": {"value": acc_serial / t_serial, "seconds": t_serial,
                         "latency_alone_ms": {"p50": float(np.percentile(alone_ms, 50)),
                                              "p99": float(np.percentile(alone_ms, 99))}},
        "saturated": {"seconds": t_sat, "capacity_requests_per_s": capacity,
                      "passes_seconds": [p[0] for p in sat],
                      "timing": "median of three passes after one untimed warm-up pass"},
        "sweep": sweeps,
        "server": {k: int(v) for k, v in st.items()},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Differentiation (configuration 5)
# ---------------------------------------------------------------------------

def run_gradient(args) -> None:
    """Stream-fitting gradient: 65,536 particles sprayed around a progenitor in
    the Bovy composite, DOP853 at rtol = atol = 1e-10 to t = 50; loss
    sum_i |x_i(50) - track(s_i)|^2 against a cubic-spline track through 32
    seeded points (s_i: the closest point of a dense sampling of the track to
    the particle's first-pass position, then held fixed).  One step = the
    taped forward integration, the loss and the adjoint pass, giving the
    gradient with respect to all 6-D initial conditions and the potential's
    parameters (MN amp, MN a and NFW a among them).  The metric counts the
    forward pass's accepted steps per second of the whole step.
    """
    import torch
    from scipy.interpolate import CubicSpline

    from astrodrift_b200 import adjoint, capi
    from astrodrift_b200.workloads import bovy_radial_force, stream_progenitor

    world, rank, local = _dist()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    n = args.particles or 65536
    pot = capi.bovy()
    vc = float(np.sqrt(1.5 * abs(float(bovy_radial_force(np.array([1.5]))[0]))))
    prog, y0 = stream_progenitor(n, vc, seed=5)
    ts = np.array([0.0, 50.0])
    rtol = 1e-10
    # target track: the progenitor's positions at 32 times in [45, 55] plus
    # seeded N(0, 0.01) offsets
    rng = np.random.default_rng(6)
    grid = np.concatenate([[0.0], np.linspace(45.0, 55.0, 32)])
    pts = capi.integrate_host(capi.DOP853, pot, prog[None, :], ts=grid, rtol=rtol, atol=rtol)["out"][1:, 0, :3]
    pts = pts + rng.normal(0.0, 0.01, pts.shape)
    spline = CubicSpline(np.linspace(0.0, 1.0, 32), pts)
    dense = spline(np.linspace(0.0, 1.0, 4096))
    y0_d = torch.tensor(y0, device=dev)
    params0 = adjoint.params_of(pot)
    first = adjoint.trajectory(y0_d, pot, ts=ts, rtol=rtol, atol=rtol)
    x50 = first[-1, :, :3].cpu().numpy()
    target = np.empty_like(x50)
    for i in range(0, n, 4096):
        d = ((x50[i:i + 4096, None, :] - dense[None, :, :]) ** 2).sum(-1)
        target[i:i + 4096] = dense[d.argmin(axis=1)]
    target_d = torch.tensor(target, device=dev)
    acc_d = torch.zeros(n, dtype=torch.int32, device=dev)
    L = capi.make_launch(capi.DOP853, pot, n, 2, rtol=rtol, atol=rtol, precision=capi.FMA,
                         schedule=capi.ORDERED)
    ts_d = torch.tensor(ts, device=dev)
    L.y0, L.ts, L.n_accepted = y0_d.data_ptr(), ts_d.data_ptr(), acc_d.data_ptr()
    ws = torch.zeros(capi.query_workspace(L), dtype=torch.uint8, device=dev)
    L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
    capi.integrate_device(L, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    steps_acc = int(acc_d.to(torch.int64).sum())
    tape_steps = int(acc_d.max())

    def step():
        y = y0_d.clone().requires_grad_(True)
        p = torch.tensor(params0, dtype=torch.float64, requires_grad=True)
        out = adjoint.trajectory(y, pot, params=p, ts=ts, rtol=rtol, atol=rtol, tape_steps=tape_steps,
                                 checkpoint_stride=args.checkpoint_stride)
        loss = ((out[-1, :, :3] - target_d) ** 2).sum()
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        loss.backward()
        return loss, y, p, ev

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    back_ms = []
    with ClockSampler(gpu_uuid(torch, dev)) as clocks:
        s.record()
        for _ in range(args.steps):
            loss, y, p, ev = step()
            ev_end = torch.cuda.Event(enable_timing=True)
            ev_end.record()
            back_ms.append((ev, ev_end))
        e.record()
        torch.cuda.synchronize()
    ms = s.elapsed_time(e) / args.steps
    back = statistics.median(a.elapsed_time(b) for a, b in back_ms)
    names = adjoint.PARAM_NAMES[pot.kind]
    line = {
        "metric": "accepted steps/s (forward + adjoint gradient)",
        "value": steps_acc / (ms * 1e-3),
        "unit": "accepted steps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": max(args.warmup, 3),
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded progenitor spray, seeded track)",
        "config": {"workload": "stream-gradient", "particles": n, "potential": "bovy", "method": "DOP853",
                   "rtol": rtol, "t_end": 50.0, "accepted_steps": steps_acc, "tape_rows": tape_steps,
                   "checkpoint_stride": args.checkpoint_stride,
                   "tape_bytes": n * capi.tape_doubles(tape_steps, args.checkpoint_stride) * 8,
                   "l2": "inputs reused; trajectory is 2 samples"},
        "backward_ms": back,
        "forward_ms": ms - back,
        "loss": float(loss.detach()),
        "grad_norm_y0": float(y.grad.norm()),
        "grad_params": {k: float(v) for k, v in zip(names, p.grad.tolist())},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="bovy", choices=["bovy", "plummer", "kepler", "serving", "stream-gradient"],
                    help="bovy (default): the uneven Bovy workload at 1e-10 against the plain launch; plummer: "
                         "2^20 Plummer particles at 1e-12; kepler: 1,024 Kepler particles with DOPR54; serving: "
                         "Poisson request streams; stream-gradient: forward + adjoint gradient")
    ap.add_argument("--precision", default="fma", choices=["exact", "fma"])
    ap.add_argument("--schedule", default="ordered", choices=["plain", "persistent", "ordered"])
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--particles", type=int, default=0,
                    help="particles per GPU (default: the workload's own size; smaller for ncu captures)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-sample", type=int, default=0, help="particles in the CPU oracle's sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-peak", action="store_true", help="skip the FP64 peak probe (profiling runs)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-launch pass")
    ap.add_argument("--no-serving", action="store_true", help="skip the short serving pass")
    ap.add_argument("--checkpoint-stride", type=int, default=1,
                    help="stream-gradient: adjoint tape checkpoint every m steps (1 = every step)")
    ap.add_argument("--serving-requests", type=int, default=32, help="serving: calibration requests")
    ap.add_argument("--serving-seconds", type=float, default=15.0,
                    help="default workload: seconds of the short open-loop serving stream (0: none)")
    ap.add_argument("--stream-seconds", type=float, default=60.0, help="serving: seconds of each Poisson stream")
    ap.add_argument("--loads", default="0.25,0.5,0.8",
                    help="serving: offered loads (fractions of the saturated capacity) of the streams")
    ap.add_argument("--streams", type=int, default=4, help="serving: batches in flight")
    ap.add_argument("--sm-reserve", type=int, default=0,
                    help="serving: percent of SMs large batches leave to small ones (default none)")
    ap.add_argument("--trajectory-cap-mib", type=int, default=2048,
                    help="serving: largest trajectory returned to host memory; larger requests return final "
                         "states only")
    ap.add_argument("--result-buffers", type=int, default=12,
                    help="serving: page-locked result buffers of --trajectory-cap-mib each, reused across requests")
    ap.add_argument("--seed", type=int, default=4)
    args = ap.parse_args()
    if args.no_e2e:
        args.e2e_steps = 0
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.workload == "stream-gradient":
        run_gradient(args)
    else:
        run_device(args)


if __name__ == "__main__":
    main()
