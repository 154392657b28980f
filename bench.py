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

# Algorithmic work per unit (one accepted step of one particle), counted from
# the integrator's arithmetic: +, -, *, /, sqrt = 1 flop; pow-type calls are
# transcendental calls, not flops.  DOP853 stage/solution/error arithmetic is
# 948 flops per attempt, the accept branch adds 918 (rcont, three dense
# stages); Plummer's force is 10 flops + 1 pow per evaluation; 11 force
# evaluations per attempt plus 4 on accept; dense output is 87 flops/sample.
FLOPS_ATTEMPT = 948
FLOPS_ACCEPT_EXTRA = 918
FORCE_FLOPS = 10
FLOPS_PER_ACCEPTED = FLOPS_ATTEMPT + FLOPS_ACCEPT_EXTRA + 15 * FORCE_FLOPS  # 2016
FLOPS_PER_REJECTED = FLOPS_ATTEMPT + 11 * FORCE_FLOPS  # 1058
FLOPS_PER_SAMPLE = 87


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
                    throughput under continuous batching;
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

    with Server(memory_fraction=0.6, streams=args.streams) as srv:
        t_sat, sat_acc, sat_lat, _ = stream(srv, 0.0)
        print(f"serving: saturated {t_sat:.2f} s", file=sys.stderr, flush=True)
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
                   "streams": args.streams, "precision": args.precision,
                   "trajectory_cap_bytes": cap_bytes, "result_buffers": args.result_buffers,
                   "seed": args.seed},
        "serial_plain": {"value": serial_acc / t_serial, "seconds": t_serial,
                         "latency_alone_ms": {"p50": float(np.percentile(alone_ms, 50)),
                                              "p99": float(np.percentile(alone_ms, 99))}},
        "saturated": {"seconds": t_sat, "speedup_vs_serial": t_serial / t_sat},
        "latency_ms": head["latency_ms"] if head else None,
        "open_loop": loads,
        "server": {k: int(v) for k, v in st.items()},
    }
    print(json.dumps(line), flush=True)
    for s_ in slots:
        s_.free()


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
    ap.add_argument("--workload", default="plummer", choices=["plummer", "serving"],
                    help="plummer: the benchmark configuration; serving: a Poisson request stream")
    ap.add_argument("--requests", type=int, default=32, help="serving: requests in the stream")
    ap.add_argument("--loads", default="0.5,0.8",
                    help="serving: offered loads (fractions of the saturated capacity) for latency")
    ap.add_argument("--streams", type=int, default=4, help="serving: batches in flight")
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

    if dist:
        t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
        a = torch.tensor([accepted], dtype=torch.float64, device=dev)
        dist.all_reduce(a, op=dist.ReduceOp.SUM)
        accepted_all = float(a.item())
    else:
        accepted_all = float(accepted)
    value = accepted_all * args.steps / elapsed

    # --- end to end through the host entry point with pinned buffers --------
    import ctypes

    if args.no_e2e:
        args.e2e_steps = 0

    out_bytes = nt * n * 6 * 8
    e2e_value, e2e_elapsed, e2e_ok = None, 0.0, None
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
            t = torch.tensor([e2e_elapsed], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_elapsed = float(t.item())
        e2e_value = accepted_all * args.e2e_steps / e2e_elapsed
        e2e_ok = bool(np.array_equal(out_pinned[-1], out_d[-1].cpu().numpy()))
        del y0_pinned, out_pinned
        lib.drift_host_free(h_y0)
        lib.drift_host_free(h_out)

    if rank == 0:
        fp64_peak = float("nan") if args.no_peak else fp64_peak_tflops(torch)
        hbm_peak, hbm_src = measured_hbm_gbs()
        mean_launch = statistics.mean(launch_s)
        samples = n * (nt - 1)
        flops = accepted * FLOPS_PER_ACCEPTED + rejected * FLOPS_PER_REJECTED + samples * FLOPS_PER_SAMPLE
        achieved_tflops = flops / mean_launch / 1e12
        bytes_alg = 48 * n * (nt + 1) + 8 * nt + 12 * n
        cpu = None
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            r = cpu_reference(y0, ts, args.cpu_sample, threads)
            cpu = {"value": r["value"], "unit": "accepted steps/s", "cores": threads, "kind": "port",
                   "sample": f"{args.cpu_sample} of the {n} seeded particles, full span and grid "
                             f"({r['seconds']:.1f} s)"}
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
                         "unit": "TFLOP/s", "frac": achieved_tflops / fp64_peak, "traffic": None,
                         "peak_source": "FP64 DGEMM (torch.matmul float64 8192^3, best of 5) "
                                        "measured in this run; MEASURED_PEAKS.json has no FP64 figure",
                         "flops_per_launch": flops,
                         "units": f"{accepted} accepted x {FLOPS_PER_ACCEPTED} + {rejected} "
                                  f"rejected x {FLOPS_PER_REJECTED} + {samples} samples x "
                                  f"{FLOPS_PER_SAMPLE}"},
            "roofline_hbm": {"bound": "hbm", "achieved": bytes_alg / mean_launch / 1e9,
                             "peak": hbm_peak, "unit": "GB/s",
                             "frac": bytes_alg / mean_launch / 1e9 / hbm_peak, "peak_source": hbm_src},
            "kernel_ms_mean": 1e3 * mean_launch,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "accepted steps/s",
                    "h2d_bytes_per_step": int(y0.nbytes + ts.nbytes),
                    "d2h_bytes_per_step": int(out_bytes + n * (48 + 1 + 4 + 4 + 4)),
                    "ms_per_step": 1e3 * e2e_elapsed / max(args.e2e_steps, 1),
                    "matches_device_path": e2e_ok},
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
