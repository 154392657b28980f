"""Benchmark: accepted DOP853 steps per second on the Plummer-sphere workload.

Workload (one "step" = one pass of the integration path over one batch):
1,048,576 particles drawn from the isotropic Plummer distribution function
(amp = 1, b = 1, seeded), DOP853 at rtol = atol = 1e-12, dense output on
ts = (0, 100, 201): a (201, 2^20, 6) float64 trajectory (10.1 GB) per step.

* ``value``  -- device path: inputs resident in HBM, one ``drift_integrate``
  launch per step, timed with CUDA events on the launching stream.
* ``e2e``    -- the same metric through ``drift_integrate_host`` with pinned
  host buffers: host->device copy of the initial states and device->host copy
  of every trajectory sample inside the timed region.
* ``cpu_baseline`` -- the CPU oracle (a line-faithful C restatement of the
  reference's CPU integrator) on a bounded seeded subsample, all host threads.
* ``--impl reference`` times only that CPU implementation (the reference's
  own CPU path cannot be built here: it is Rust and no Rust toolchain exists).

Multi-GPU (torchrun): every rank integrates its own 2^20-particle shard
(weak scaling, no data-path collective); time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
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

N_PARTICLES = 1 << 20
TS = (0.0, 100.0, 201)
RTOL = ATOL = 1e-12
WORKLOAD = "plummer-dop853"

# Algorithmic work per unit, counted exactly from the reference algorithm's
# arithmetic (+, -, *, /, sqrt = 1 flop; pow-type calls are transcendental
# calls, not flops): astrodrift_b200/roofline_counts.json, fitted without
# residual over seeded runs of the restatement compiled with a counting
# scalar.  DOP853 with the Plummer force: per accepted step, per rejected
# step, per emitted sample and per particle (set-up).
_COUNTS = json.loads((Path(__file__).resolve().parent / "astrodrift_b200" /
                      "roofline_counts.json").read_text())["dop853_plummer"]["flops"]
FLOPS_PER_ACCEPTED = _COUNTS["per_accepted"]  # 2066
FLOPS_PER_REJECTED = _COUNTS["per_rejected"]  # 1099
FLOPS_PER_SAMPLE = _COUNTS["per_sample"]  # 89
FLOPS_PER_PARTICLE = _COUNTS["per_particle"]  # 128
# DRAM bytes (read + write) per particle of one launch of this workload,
# from the ncu capture of 262,144 particles with the ordered schedule
# (profiles/dop853_plummer_c2.txt, section 5: 1.696 GB read + 3.397 GB
# written); traffic grows in proportion to the particles processed, so a
# full launch is this times n.
DRAM_BYTES_PER_PARTICLE = (1.696054272e9 + 3.397321984e9) / 262144


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


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


def cpu_reference(y0: np.ndarray, ts: np.ndarray, sample: int, threads: int) -> dict:
    """The CPU oracle on a seeded subsample; accepted steps/s."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.build()
    idx = np.random.default_rng(12345).choice(len(y0), sample, replace=False)
    t0 = time.perf_counter()
    res = oracle.integrate_batch(oracle.DOP853, oracle.plummer(1.0, 1.0), y0[idx], ts=ts,
                                 rtol=RTOL, atol=ATOL, threads=threads, want_output=True)
    dt = time.perf_counter() - t0
    return {"value": float(res["accepted"].sum()) / dt, "seconds": dt,
            "accepted": int(res["accepted"].sum())}


def accuracy_vs_oracle(method: int, pot_name: str, y0: np.ndarray, out: np.ndarray, accepted: np.ndarray,
                       rtol: float, *, ts=None, t_end=None, nt=None, sample: int = 256) -> dict:
    """Max relative error per sample and accepted-step agreement of a seeded
    particle sample against the CPU oracle (the checker; run after timing)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.build()
    idx = np.sort(np.random.default_rng(777).choice(len(y0), min(sample, len(y0)), replace=False))
    opot = {"plummer": oracle.plummer(1.0, 1.0), "kepler": oracle.kepler(1.0), "bovy": oracle.bovy()}[pot_name]
    kw = dict(ts=ts) if ts is not None else dict(t_end=t_end[idx], nt=nt)
    ref = oracle.integrate_batch(method, opot, y0[idx], rtol=rtol, atol=rtol, threads=os.cpu_count() or 1, **kw)
    got = out[:, idx]
    scale = np.maximum(np.abs(ref["out"]).max(axis=2), 1e-300)
    err = np.abs(got - ref["out"]).max(axis=2) / scale
    return {"particles": int(len(idx)), "max_rel_err": float(err.max()), "median_rel_err": float(np.median(err)),
            "accepted_step_agreement": float((accepted[idx].astype(np.int64) == ref["accepted"]).mean())}


def run_reference(args) -> None:
    world, rank, _ = _dist()
    if rank != 0:
        return
    from astrodrift_b200.workloads import plummer_sphere

    y0 = plummer_sphere(N_PARTICLES)
    ts = np.linspace(*TS[:2], TS[2])
    threads = os.cpu_count() or 1
    sample = args.cpu_sample
    for _ in range(args.warmup):
        cpu_reference(y0, ts, max(256, sample // 8), threads)
    vals, secs = [], []
    for _ in range(args.steps):
        r = cpu_reference(y0, ts, sample, threads)
        vals.append(r["value"])
        secs.append(r["seconds"])
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "accepted steps/s", "value": value,
        "unit": "accepted steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded isotropic Plummer DF)",
        "config": {"workload": WORKLOAD, "particles": N_PARTICLES, "ts": list(TS),
                   "rtol": RTOL, "atol": ATOL, "method": "DOP853", "potential": "plummer(1,1)"},
        "cpu_baseline": {"value": value, "unit": "accepted steps/s", "cores": threads,
                         "kind": "port",
                         "sample": f"{sample} of the {N_PARTICLES} seeded particles per step, "
                                   "full time span and output grid"},
        "e2e": {"value": value, "unit": "accepted steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference's CPU path is Rust and cannot be built here; this times the "
                "oracle, a line-faithful C restatement of src/integrators/galpy/dop853.rs",
    }
    print(json.dumps(line), flush=True)


def _serving_requests(args, capi, cap_bytes):
    """The seeded request mix of the serving workload (arrival times in units
    of the mean inter-arrival gap)."""
    import torch

    from astrodrift_b200.workloads import bovy_disc, kepler_disc, plummer_sphere

    rng = np.random.default_rng(args.seed)
    pools = [capi.kepler(1.0), capi.plummer(1.0, 1.0), capi.bovy()]
    fr_pot = capi.bovy()

    def bovy_fr(R):
        xyz = torch.zeros((len(R), 3), dtype=torch.float64, device="cuda")
        xyz[:, 0] = torch.from_numpy(np.asarray(R, dtype=np.float64))
        acc = torch.empty_like(xyz)
        capi.force_device(fr_pot, len(R), xyz.data_ptr(), acc.data_ptr())
        torch.cuda.synchronize()
        return acc[:, 0].cpu().numpy()

    reqs, t = [], 0.0
    for _ in range(args.requests):
        t += rng.exponential(1.0)
        n = int(2 ** rng.uniform(0, 20))
        kind = int(rng.integers(3))
        method = int(rng.integers(2))
        nt = int(np.exp(rng.uniform(np.log(2), np.log(10001))))
        nt = max(2, min(nt, cap_bytes // (48 * n)))
        rtol = float([1e-8, 1e-10, 1e-12][int(rng.integers(3))])
        t_end = float(rng.uniform(10.0, 100.0))
        seed = int(rng.integers(1 << 31))
        if kind == 0:
            y0 = kepler_disc(n, seed=seed)
        elif kind == 1:
            y0 = plummer_sphere(n, seed=seed)
        else:
            y0, _ = bovy_disc(n, seed=seed, radial_force=bovy_fr)
        reqs.append(dict(at=t, method=method, pot=pools[kind], kind=kind, y0=y0,
                         ts=np.linspace(0.0, t_end, nt), rtol=rtol))
    return reqs


def run_serving(args) -> None:
    """Serving workload: a request stream through the resident request server.

    Each request: N = floor(2^U[0,20]) particles; potential uniform in
    {Kepler(1), Plummer(1,1), Bovy}; method uniform in {DOPR54, DOP853};
    nt = floor(exp(U[ln 2, ln 10001])) outputs on (0, t_end), t_end ~ U[10, 100];
    rtol = atol uniform in {1e-8, 1e-10, 1e-12}.  One request's trajectory is
    capped at --trajectory-cap-mib (nt reduced) so every result can be
    returned to host memory.

    Three passes over the same requests:
      serial     -- one drift_integrate_host call per request, plain schedule,
                    one after another (the serial plain-launch baseline; its
                    per-request times are each request's latency alone);
      saturated  -- every request submitted to the server at once: aggregate
                    throughput under continuous batching (median of three
                    passes after an untimed warm-up pass);
      open loop  -- Poisson arrivals at each offered load in --loads, as a
                    fraction of the saturated capacity: p50/p99 latency
                    (submission to results in host memory).
    """
    import torch

    from astrodrift_b200 import capi
    from astrodrift_b200.serving import PinnedArray, Server

    world, rank, local = _dist()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    cap_bytes = args.trajectory_cap_mib << 20
    precision = capi.EXACT if args.precision == "exact" else capi.FMA
    reqs = _serving_requests(args, capi, cap_bytes)
    n_particles = sum(len(r["y0"]) for r in reqs)
    print(f"serving: {len(reqs)} requests, {n_particles} particles", file=sys.stderr, flush=True)
    # page-locked result buffers, reused across requests
    slots = [PinnedArray((cap_bytes // 8,)) for _ in range(args.result_buffers)]

    def out_view(slot, r):
        nt, n = len(r["ts"]), len(r["y0"])
        return slots[slot].array[: nt * n * 6].reshape(nt, n, 6)

    # warm-up: load every kernel instance once
    for pot in (capi.kepler(1.0), capi.plummer(1.0, 1.0), capi.bovy()):
        for method in (capi.DOPR54, capi.DOP853):
            capi.integrate_host(method, pot, reqs[0]["y0"][:1], ts=np.linspace(0, 1, 3), rtol=1e-8,
                                atol=1e-8, precision=precision, schedule=capi.PLAIN)
            capi.integrate_host(method, pot, reqs[0]["y0"][:1], ts=np.linspace(0, 1, 3), rtol=1e-8,
                                atol=1e-8, precision=precision, schedule=capi.PERSISTENT)

    # serial plain launches
    alone, serial_acc = [], 0
    t0 = time.perf_counter()
    for r in reqs:
        ti = time.perf_counter()
        res = capi.integrate_host(r["method"], r["pot"], r["y0"], ts=r["ts"], rtol=r["rtol"],
                                  atol=r["rtol"], precision=precision, schedule=capi.PLAIN,
                                  out=out_view(0, r))
        alone.append(time.perf_counter() - ti)
        serial_acc += int(res["accepted"].astype(np.int64).sum())
    t_serial = time.perf_counter() - t0
    print(f"serving: serial {t_serial:.2f} s", file=sys.stderr, flush=True)

    def stream(srv, gap_s):
        """Submit every request at its arrival time (gap_s = 0: all at once);
        returns (seconds, accepted steps, latencies, client buffer waits)."""
        free_slots = list(range(len(slots)))
        inflight, lat, waits, acc = [], {}, [], 0

        def retire():
            nonlocal acc
            h, slot, i = inflight.pop(0)
            res = h.wait()
            lat[i] = res["latency_s"]
            acc += int(res["accepted"].astype(np.int64).sum())
            free_slots.append(slot)

        t_begin = time.perf_counter()
        for i, r in enumerate(reqs):
            while time.perf_counter() - t_begin < r["at"] * gap_s:
                time.sleep(0.0002)
            t_want = time.perf_counter()
            while not free_slots:
                retire()
            waits.append(time.perf_counter() - t_want)
            slot = free_slots.pop()
            h = srv.submit(r["method"], r["pot"], r["y0"], ts=r["ts"], rtol=r["rtol"], atol=r["rtol"],
                           precision=precision, out=out_view(slot, r))
            inflight.append((h, slot, i))
        while inflight:
            retire()
        return time.perf_counter() - t_begin, acc, [lat[i] for i in range(len(reqs))], waits

    with Server(memory_fraction=0.6, streams=args.streams, sm_reserve_percent=args.sm_reserve) as srv:
        # Batches form from whatever is pending when a stream frees up, so a
        # saturated pass varies with submission timing: one untimed pass warms
        # the server's memory pool, then the median of three timed passes.
        stream(srv, 0.0)
        sat_passes = [stream(srv, 0.0) for _ in range(3)]
        sat_passes.sort(key=lambda p: p[0])
        t_sat, sat_acc, sat_lat, _ = sat_passes[1]
        print(f"serving: saturated {t_sat:.2f} s (passes {[round(p[0], 3) for p in sat_passes]})",
              file=sys.stderr, flush=True)
        loads = []
        for load in [float(x) for x in args.loads.split(",") if x]:
            rate = load * len(reqs) / t_sat
            t_run, acc, lat, waits = stream(srv, 1.0 / rate)
            lat_ms = np.array(lat) * 1e3
            slow = np.array(lat) / np.maximum(np.array(alone), 1e-9)
            loads.append({
                "offered_load": load, "rate_per_s": rate, "seconds": t_run,
                "accepted_steps_per_s": acc / t_run,
                "latency_ms": {"p50": float(np.percentile(lat_ms, 50)),
                               "p99": float(np.percentile(lat_ms, 99)),
                               "mean": float(lat_ms.mean()), "max": float(lat_ms.max())},
                "slowdown_vs_alone": {"p50": float(np.percentile(slow, 50)),
                                      "p99": float(np.percentile(slow, 99))},
                "client_buffer_wait_ms_p99": float(np.percentile(np.array(waits) * 1e3, 99)),
            })
            print(f"serving: load {load} rate {rate:.2f}/s p50 {loads[-1]['latency_ms']['p50']:.1f} ms "
                  f"p99 {loads[-1]['latency_ms']['p99']:.1f} ms", file=sys.stderr, flush=True)
        st = srv.stats()
    alone_ms = np.array(alone) * 1e3
    head = loads[0] if loads else None
    line = {
        "metric": "accepted steps/s (served request stream)",
        "value": sat_acc / t_sat,
        "unit": "accepted steps/s",
        "n_gpus": 1,
        "steps": len(reqs),
        "warmup": 1,
        "ms_per_step": 1e3 * t_sat / len(reqs),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded request stream)",
        "config": {"workload": "serving", "requests": len(reqs), "particles": n_particles,
                   "streams": args.streams, "sm_reserve_percent": args.sm_reserve, "precision": args.precision,
                   "trajectory_cap_bytes": cap_bytes, "result_buffers": args.result_buffers,
                   "seed": args.seed},
        "serial_plain": {"value": serial_acc / t_serial, "seconds": t_serial,
                         "latency_alone_ms": {"p50": float(np.percentile(alone_ms, 50)),
                                              "p99": float(np.percentile(alone_ms, 99))}},
        "saturated": {"seconds": t_sat, "speedup_vs_serial": t_serial / t_sat,
                      "passes_seconds": [p[0] for p in sat_passes],
                      "timing": "median of three passes after one untimed warm-up pass"},
        "latency_ms": head["latency_ms"] if head else None,
        "open_loop": loads,
        "server": {k: int(v) for k, v in st.items()},
    }
    print(json.dumps(line), flush=True)
    for s_ in slots:
        s_.free()


def run_config(args) -> None:
    """The other two single-GPU configurations.

    kepler -- configuration 1: 1,024 particles in the galpy-cylindrical Kepler
              force (amp 1), DOPR54 at rtol = atol = 1e-10, ts = (0, 20 pi, 1001).
    bovy   -- configuration 3: Bovy composite, R log-uniform on [0.05, 20],
              per-particle t_end ~ U[10, 1000] with 101 outputs each, DOP853 at
              1e-10.  The full configuration has 2^22 particles; the default
              is its first 2^18 (--particles 4194304 runs it whole).  The
              chosen schedule is timed beside one plain-schedule pass of the
              same particles (the plain-launch baseline).
    The line reports accepted steps/s, the energy drift |E(end)/E(0) - 1|
    over all particles, and the plain-launch ratio.
    """
    import torch

    from astrodrift_b200 import capi
    from astrodrift_b200.energy import angular_momentum_drift, drift_summary
    from astrodrift_b200.workloads import bovy_disc, kepler_disc

    world, rank, local = _dist()
    if args.workload == "kepler" and rank != 0:
        return  # configuration 1 is one small batch: rank 0 alone
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    dist = None
    if args.workload == "bovy" and world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    precision = capi.EXACT if args.precision == "exact" else capi.FMA
    schedule = {"plain": capi.PLAIN, "persistent": capi.PERSISTENT, "ordered": capi.ORDERED}[args.schedule]
    shard = None
    if args.workload == "kepler":
        pot, method, tol = capi.kepler(1.0), capi.DOPR54, 1e-10
        n = 1024 if args.particles == N_PARTICLES else args.particles
        y0 = kepler_disc(n, seed=1)
        ts, t_end, nt = np.linspace(0.0, 20.0 * np.pi, 1001), None, 1001
        name, full = "kepler-dopr54", 1024
    else:
        pot, method, tol = capi.bovy(), capi.DOP853, 1e-10
        full = 1 << 22
        n = (1 << 18) if args.particles == N_PARTICLES else args.particles
        fr_pot = capi.bovy()

        def radial_force(R):
            xyz = torch.zeros((len(R), 3), dtype=torch.float64, device=dev)
            xyz[:, 0] = torch.from_numpy(np.asarray(R, dtype=np.float64))
            acc = torch.empty_like(xyz)
            capi.force_device(fr_pot, len(R), xyz.data_ptr(), acc.data_ptr())
            torch.cuda.synchronize()
            return acc[:, 0].cpu().numpy()

        y0_all, te_all = bovy_disc(full, seed=3, radial_force=radial_force)
        y0, t_end = y0_all[:n], te_all[:n]
        if dist:
            # strong scaling: cost-balanced contiguous shards of the same particles
            from astrodrift_b200.sharding import balanced_ranges, orbit_cost

            xyz = torch.from_numpy(np.ascontiguousarray(y0[:, :3])).to(dev)
            acc = torch.empty_like(xyz)
            capi.force_device(fr_pot, n, xyz.data_ptr(), acc.data_ptr())
            torch.cuda.synchronize()
            lo, hi = balanced_ranges(orbit_cost(y0, t_end, acc.cpu().numpy()), world)[rank]
            y0, t_end, shard = y0[lo:hi], t_end[lo:hi], (lo, hi)
        ts, nt = None, 101
        name = "bovy-uneven-dop853"
    y0_d = torch.from_numpy(np.ascontiguousarray(y0)).to(dev)
    grid_d = torch.from_numpy(ts if ts is not None else np.ascontiguousarray(t_end)).to(dev)
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

    def timed(L, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a_, b_ in ev:
            a_.record(stream)
            capi.integrate_device(L, stream.cuda_stream)
            b_.record(stream)
        torch.cuda.synchronize()
        return [a_.elapsed_time(b_) / 1e3 for a_, b_ in ev]

    n_all = n
    n = len(y0)
    L, ws = make(schedule)
    timed(L, max(args.warmup, 3))
    gpu_id = str(torch.cuda.get_device_properties(dev).uuid)
    gpu_id = gpu_id if gpu_id.startswith("GPU-") else f"GPU-{gpu_id}"
    if dist:
        dist.barrier()
    with ClockSampler(gpu_id) as clocks:
        secs = timed(L, args.steps)
    status = st_d.cpu().numpy()
    accepted = int(acc_d.cpu().numpy().astype(np.int64).sum())
    rejected = int(rej_d.cpu().numpy().astype(np.int64).sum())
    acc_per = acc_d.cpu().numpy()
    out_first = out_d[0].cpu().numpy()
    last_idx = nt - 1
    out_last = out_d[last_idx].cpu().numpy()
    mean_s = statistics.mean(secs)
    if dist:
        from astrodrift_b200.sharding import reduce_max, reduce_sum

        mean_s = reduce_max(mean_s, dist, dev)
        accepted = int(reduce_sum(accepted, dist, dev))
        rejected = int(reduce_sum(rejected, dist, dev))
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return
    value = accepted / mean_s
    acc_sample = None
    if not args.no_cpu and rank == 0:
        out_host = out_d.cpu().numpy() if nt * n * 48 < (4 << 30) else None
        if out_host is not None:
            acc_sample = accuracy_vs_oracle(method, "kepler" if args.workload == "kepler" else "bovy", y0,
                                            out_host, acc_per, tol, ts=ts, t_end=t_end, nt=nt)
    plain = None
    if schedule != capi.PLAIN and not args.no_plain and not dist:
        Lp, wsp = make(capi.PLAIN)
        psecs = timed(Lp, 1)
        plain = {"value": accepted / psecs[0], "seconds": psecs[0], "speedup": psecs[0] / statistics.mean(secs),
                 "bitwise_equal_trajectory": bool(np.array_equal(out_d[last_idx].cpu().numpy(), out_last))}
    line = {
        "metric": "accepted steps/s",
        "value": value,
        "unit": "accepted steps/s",
        "n_gpus": world if dist else 1,
        "steps": args.steps,
        "warmup": max(args.warmup, 3),
        "ms_per_step": 1e3 * mean_s,
        "higher_is_better": True,
        "scaling": "strong" if dist else "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded, configuration generator)",
        "config": {"workload": name if n_all == full else f"{name} (first {n_all} of {full})",
                   "particles": n_all, "rank0_shard": shard,
                   "nt": nt, "rtol": tol, "method": "DOP853" if method == capi.DOP853 else "DOPR54",
                   "precision": args.precision, "schedule": args.schedule,
                   "l2": "outputs written once per pass; inputs re-read each pass"},
        "accepted_steps_per_pass": accepted,
        "rejected_steps_per_pass": rejected,
        "steps_per_particle": {"median": float(np.median(acc_per)), "max": int(acc_per.max()),
                               "min": int(acc_per.min())},
        "particles_not_ok": int((status != 0).sum()),
        "energy_drift": drift_summary(pot, out_first, out_last),  # rank 0's particles
        "angular_momentum_drift": angular_momentum_drift(pot, out_first, out_last),
        "accuracy": acc_sample,
        "plain_launch": plain,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


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
    from astrodrift_b200.workloads import stream_progenitor

    world, rank, local = _dist()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    n = 65536 if args.particles == N_PARTICLES else args.particles
    pot = capi.bovy()
    # circular speed at R = 1.5 from the composite's force
    xyz = torch.tensor([[1.5, 0.0, 0.0]], dtype=torch.float64, device=dev)
    acc = torch.empty_like(xyz)
    capi.force_device(pot, 1, xyz.data_ptr(), acc.data_ptr())
    torch.cuda.synchronize()
    vc = float(np.sqrt(1.5 * abs(float(acc[0, 0]))))
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
    # closest dense-track point of each particle (chunked to bound memory)
    target = np.empty_like(x50)
    for i in range(0, n, 4096):
        d = ((x50[i:i + 4096, None, :] - dense[None, :, :]) ** 2).sum(-1)
        target[i:i + 4096] = dense[d.argmin(axis=1)]
    target_d = torch.tensor(target, device=dev)
    # tape sized once from an untaped pass
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

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    back_ms = []
    with ClockSampler(str(local)) as clocks:
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
        "warmup": args.warmup,
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
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fma", choices=["exact", "fma"])
    ap.add_argument("--schedule", default="ordered", choices=["plain", "persistent", "ordered"])
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample", type=int, default=262144)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-peak", action="store_true", help="skip the FP64 peak probe (profiling runs)")
    ap.add_argument("--particles", type=int, default=N_PARTICLES,
                    help="particles per GPU (default: the workload's 2^20; smaller for ncu captures)")
    ap.add_argument("--workload", default="plummer",
                    choices=["plummer", "kepler", "bovy", "serving", "stream-gradient"],
                    help="plummer: the benchmark configuration; kepler / bovy: the other single-GPU "
                         "configurations; serving: a Poisson request stream; stream-gradient: forward + "
                         "adjoint gradient of a stream-track loss")
    ap.add_argument("--no-plain", action="store_true", help="kepler/bovy: skip the plain-launch pass")
    ap.add_argument("--checkpoint-stride", type=int, default=1,
                    help="stream-gradient: adjoint tape checkpoint every m steps (1 = every step)")
    ap.add_argument("--requests", type=int, default=32, help="serving: requests in the stream")
    ap.add_argument("--loads", default="0.5,0.8",
                    help="serving: offered loads (fractions of the saturated capacity) for latency")
    ap.add_argument("--streams", type=int, default=4, help="serving: batches in flight")
    ap.add_argument("--sm-reserve", type=int, default=0,
                    help="serving: percent of SMs large batches leave to small ones (default none)")
    ap.add_argument("--trajectory-cap-mib", type=int, default=256,
                    help="serving: largest trajectory of one request")
    ap.add_argument("--result-buffers", type=int, default=16, help="serving: pinned result buffers")
    ap.add_argument("--seed", type=int, default=4)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "stream-gradient":
        run_gradient(args)
        return
    if args.workload in ("kepler", "bovy"):
        run_config(args)
        return

    import torch

    from astrodrift_b200 import capi
    from astrodrift_b200.workloads import plummer_sphere

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{local}"))
    dev = torch.device(f"cuda:{local}")

    y0 = plummer_sphere(N_PARTICLES, seed=2 + rank)[: args.particles]
    ts = np.linspace(*TS[:2], TS[2])
    n, nt = len(y0), len(ts)
    precision = capi.EXACT if args.precision == "exact" else capi.FMA
    schedule = {"plain": capi.PLAIN, "persistent": capi.PERSISTENT, "ordered": capi.ORDERED}[args.schedule]

    y0_d = torch.from_numpy(y0).to(dev)
    ts_d = torch.from_numpy(ts).to(dev)
    out_d = torch.empty((nt, n, 6), dtype=torch.float64, device=dev)
    acc_d = torch.zeros(n, dtype=torch.int32, device=dev)
    rej_d = torch.zeros(n, dtype=torch.int32, device=dev)
    st_d = torch.zeros(n, dtype=torch.uint8, device=dev)
    L = capi.make_launch(capi.DOP853, capi.plummer(1.0, 1.0), n, nt, rtol=RTOL, atol=ATOL,
                         precision=precision, schedule=schedule, block_size=args.block)
    ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
    L.y0, L.ts, L.out = y0_d.data_ptr(), ts_d.data_ptr(), out_d.data_ptr()
    L.n_accepted, L.n_rejected, L.status = acc_d.data_ptr(), rej_d.data_ptr(), st_d.data_ptr()
    L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
    stream = torch.cuda.current_stream(dev)

    def launch():
        capi.integrate_device(L, stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        launch()
    torch.cuda.synchronize()

    gpu_id = str(torch.cuda.get_device_properties(dev).uuid)
    gpu_id = gpu_id if gpu_id.startswith("GPU-") else f"GPU-{gpu_id}"
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_id) as clocks:
        t_start = torch.cuda.Event(enable_timing=True)
        t_stop = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for s, e in events:
            s.record(stream)
            launch()
            e.record(stream)
        t_stop.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    elapsed = t_start.elapsed_time(t_stop) / 1e3
    launch_s = [s.elapsed_time(e) / 1e3 for s, e in events]

    status = st_d.cpu().numpy()
    accepted = int(acc_d.cpu().numpy().astype(np.int64).sum())
    rejected = int(rej_d.cpu().numpy().astype(np.int64).sum())
    if (status != 0).any():
        raise RuntimeError(f"{int((status != 0).sum())} particles did not finish")
    from astrodrift_b200.energy import angular_momentum_drift, drift_summary

    first_h, last_h = out_d[0].cpu().numpy(), out_d[-1].cpu().numpy()
    e_drift = drift_summary(capi.plummer(1.0, 1.0), first_h, last_h)
    l_drift = angular_momentum_drift(capi.plummer(1.0, 1.0), first_h, last_h)
    del first_h, last_h
    acc_c2 = None
    if rank == 0 and not args.no_cpu:
        pick = np.sort(np.random.default_rng(777).choice(n, min(256, n), replace=False))
        sub_out = out_d[:, torch.from_numpy(pick).to(dev)].cpu().numpy()
        sub_acc = acc_d.cpu().numpy()[pick]
        acc_c2 = accuracy_vs_oracle(capi.DOP853, "plummer", y0[pick], sub_out, sub_acc, RTOL, ts=ts)

    if dist:
        from astrodrift_b200.sharding import reduce_max, reduce_sum

        elapsed = reduce_max(elapsed, dist, dev)
        accepted_all = reduce_sum(accepted, dist, dev)
    else:
        accepted_all = float(accepted)
    value = accepted_all * args.steps / elapsed

    # --- end to end through the host entry point with pinned buffers --------
    import ctypes

    if args.no_e2e:
        args.e2e_steps = 0

    out_bytes = nt * n * 6 * 8
    e2e_value, e2e_elapsed, e2e_ok, d2h_gbs = None, 0.0, None, None
    if args.e2e_steps > 0:
        lib = capi.lib()
        h_y0, h_out = ctypes.c_void_p(), ctypes.c_void_p()
        capi.check(lib.drift_host_alloc(y0.nbytes, ctypes.byref(h_y0)), "drift_host_alloc")
        capi.check(lib.drift_host_alloc(out_bytes, ctypes.byref(h_out)), "drift_host_alloc")
        y0_pinned = np.ctypeslib.as_array(
            (ctypes.c_double * (n * 6)).from_address(h_y0.value)).reshape(n, 6)
        y0_pinned[:] = y0
        out_pinned = np.ctypeslib.as_array(
            (ctypes.c_double * (nt * n * 6)).from_address(h_out.value)).reshape(nt, n, 6)

        def e2e_step():
            capi.integrate_host(capi.DOP853, capi.plummer(1.0, 1.0), y0_pinned, ts=ts, rtol=RTOL,
                                atol=ATOL, precision=precision, schedule=schedule,
                                block_size=args.block, out=out_pinned)

        e2e_step()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        e2e_elapsed = time.perf_counter() - t0
        if dist:
            e2e_elapsed = reduce_max(e2e_elapsed, dist, dev)
        e2e_value = accepted_all * args.e2e_steps / e2e_elapsed
        e2e_ok = bool(np.array_equal(out_pinned[-1], out_d[-1].cpu().numpy()))
        # the copy roofline of this leg: pinned device->host bandwidth of 1 GiB
        # copies on this box (best of 3, CUDA events)
        probe = out_d.view(-1)[: (1 << 27)]
        host_probe = torch.from_numpy(out_pinned.reshape(-1)[: (1 << 27)])
        d2h = []
        for _ in range(3):
            a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a_.record()
            host_probe.copy_(probe, non_blocking=True)
            b_.record()
            torch.cuda.synchronize()
            d2h.append(probe.numel() * 8 / (a_.elapsed_time(b_) * 1e-3) / 1e9)
        d2h_gbs = max(d2h)
        del y0_pinned, out_pinned, host_probe
        lib.drift_host_free(h_y0)
        lib.drift_host_free(h_out)

    if rank == 0:
        fp64_peak = float("nan") if args.no_peak else fp64_peak_tflops(torch)
        hbm_peak, hbm_src = measured_hbm_gbs()
        mean_launch = statistics.mean(launch_s)
        samples = n * (nt - 1)
        flops = (accepted * FLOPS_PER_ACCEPTED + rejected * FLOPS_PER_REJECTED + samples * FLOPS_PER_SAMPLE
                 + n * FLOPS_PER_PARTICLE)
        achieved_tflops = flops / mean_launch / 1e12
        bytes_alg = 48 * n * (nt + 1) + 8 * nt + 12 * n
        cpu = None
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            r = cpu_reference(y0, ts, args.cpu_sample, threads)
            one = cpu_reference(y0, ts, max(256, args.cpu_sample // 32), 1)
            cpu = {"value": r["value"], "unit": "accepted steps/s", "cores": threads, "kind": "port",
                   "sample": f"{args.cpu_sample} of the {n} seeded particles, full span and grid "
                             f"({r['seconds']:.1f} s)",
                   "one_core": {"value": one["value"], "cores": 1,
                                "sample": f"{max(256, args.cpu_sample // 32)} particles ({one['seconds']:.1f} s), "
                                          "the reference's serial per-particle loop"}}
        line = {
            "metric": "accepted steps/s",
            "value": value,
            "unit": "accepted steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded isotropic Plummer DF, amp=1, b=1)",
            "config": {"workload": WORKLOAD if n == N_PARTICLES else f"{WORKLOAD} (subset of {n})",
                       "particles_per_gpu": n, "ts": list(TS),
                       "rtol": RTOL, "atol": ATOL, "method": "DOP853",
                       "potential": "plummer(amp=1, b=1)", "precision": args.precision,
                       "schedule": args.schedule,
                       "l2": "inputs+outputs (10.1 GB/step) far exceed the 126 MB L2; no flush"},
            "accepted_steps_per_pass": accepted_all,
            "rejected_steps_per_pass": rejected,
            "gpu_launches": args.steps,
            "roofline": {"bound": "fp64", "achieved": achieved_tflops, "peak": fp64_peak,
                         "unit": "TFLOP/s", "frac": achieved_tflops / fp64_peak,
                         "traffic": DRAM_BYTES_PER_PARTICLE * n,
                         "traffic_source": "ncu dram__bytes_read+write at 262,144 particles, scaled by "
                                           "particles (profiles/dop853_plummer_c2.txt, section 5)",
                         "peak_source": "FP64 DGEMM (torch.matmul float64 8192^3, best of 5) "
                                        "measured in this run; MEASURED_PEAKS.json has no FP64 figure",
                         "flops_per_launch": flops,
                         "units": f"{accepted} accepted x {FLOPS_PER_ACCEPTED} + {rejected} "
                                  f"rejected x {FLOPS_PER_REJECTED} + {samples} samples x "
                                  f"{FLOPS_PER_SAMPLE} + {n} particles x {FLOPS_PER_PARTICLE}",
                         "counts_source": "astrodrift_b200/roofline_counts.json (exact operation counts "
                                          "of the reference algorithm)"},
            "roofline_hbm": {"bound": "hbm", "achieved": bytes_alg / mean_launch / 1e9,
                             "peak": hbm_peak, "unit": "GB/s",
                             "frac": bytes_alg / mean_launch / 1e9 / hbm_peak, "peak_source": hbm_src},
            "kernel_ms_mean": 1e3 * mean_launch,
            "energy_drift": e_drift,
            "angular_momentum_drift": l_drift,
            "accuracy": acc_c2,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "accepted steps/s",
                    "h2d_bytes_per_step": int(y0.nbytes + ts.nbytes),
                    "d2h_bytes_per_step": int(out_bytes + n * (48 + 1 + 4 + 4 + 4)),
                    "ms_per_step": 1e3 * e2e_elapsed / max(args.e2e_steps, 1),
                    "matches_device_path": e2e_ok,
                    "copy_roofline": None if d2h_gbs is None else {
                        "bound": "pcie_d2h", "peak_gbs": d2h_gbs,
                        "achieved_gbs": out_bytes * args.e2e_steps / e2e_elapsed / 1e9,
                        "frac": out_bytes * args.e2e_steps / e2e_elapsed / 1e9 / d2h_gbs,
                        "peak_source": "pinned 1 GiB device->host copies measured in this run"}},
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
