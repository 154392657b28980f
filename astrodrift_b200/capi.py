"""ctypes binding of the C ABI in ``include/drift_b200.h`` (``libdrift_b200.so``).

This is the boundary a foreign-language host binds; the parity tests, the
smoke check and the benchmark call the kernels through it.
Functions here raise ``RuntimeError`` with the library's message when a call
fails; nothing falls back to a CPU implementation.
"""

from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libdrift_b200.so"

DOPR54, DOP853 = 0, 1
POT_KEPLER, POT_PLUMMER, POT_BOVY, POT_KEPLER_CARTESIAN, POT_MODEL = 0, 1, 2, 3, 4
MAX_COMPONENTS = 11
MAX_BATCH = 64  # DRIFT_MAX_BATCH: requests one batched launch carries
EXACT, FMA = 0, 1
Y0_ROWS, Y0_COLUMNS = 0, 1
PLAIN, PERSISTENT, ORDERED = 0, 1, 2
INITIAL_STEP_SENTINEL = -9999.99
(PARTICLE_OK, PARTICLE_MIN_STEP, PARTICLE_MAX_STEPS, PARTICLE_NONFINITE, PARTICLE_TIMEOUT,
 PARTICLE_TAPE_FULL) = range(6)
ADJOINT_MAX_PARAMS = 6
MAX_TAPE_STRIDE = 16


def tape_doubles(tape_steps: int, tape_stride: int) -> int:
    """Doubles of step tape per particle (drift_tape_doubles)."""
    if tape_stride <= 1:
        return tape_steps * 8
    return (tape_steps + tape_stride - 1) // tape_stride * 8 + ((tape_steps + 1) & ~1)

# Every symbol the header declares.
EXPORTED = (
    "drift_abi_version",
    "drift_result_string",
    "drift_last_error",
    "drift_host_alloc",
    "drift_host_free",
    "drift_potential_bovy",
    "drift_query_workspace",
    "drift_integrate",
    "drift_integrate_host",
    "drift_context_create",
    "drift_context_integrate_host",
    "drift_context_memory",
    "drift_context_destroy",
    "drift_galpy_dopr54",
    "drift_galpy_dop853",
    "drift_force",
    "drift_force_precision",
    "drift_integrate_noalloc",
    "drift_integrate_batch",
    "drift_server_create",
    "drift_server_submit",
    "drift_server_wait",
    "drift_server_wait_any",
    "drift_server_stats_get",
    "drift_server_cancel",
    "drift_server_destroy",
    "drift_integrate_adjoint",
    "drift_origin_table",
    "drift_origin_table_host",
    "drift_force_model_eval",
    "drift_graph_create",
    "drift_graph_launch",
    "drift_graph_destroy",
    "drift_autotune",
)


class DriftTuning(ctypes.Structure):
    _fields_ = [
        ("block_size", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("seconds", ctypes.c_double),
        ("candidates", ctypes.c_double * 12),
        ("sample", ctypes.c_int64),
        ("cached", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class DriftPotential(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("amp", ctypes.c_double),
        ("b", ctypes.c_double),
        ("mn_amp", ctypes.c_double),
        ("mn_a", ctypes.c_double),
        ("mn_b", ctypes.c_double),
        ("nfw_amp", ctypes.c_double),
        ("nfw_a", ctypes.c_double),
        ("bulge_alpha", ctypes.c_double),
        ("bulge_rc", ctypes.c_double),
        ("bulge_k", ctypes.c_double),
        ("bulge_gamma_s", ctypes.c_double),
    ]


class DriftSourceGroup(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("amp", ctypes.c_double),
        ("b", ctypes.c_double),
        ("first", ctypes.c_int64),
        ("count", ctypes.c_int64),
    ]


class DriftForceModel(ctypes.Structure):
    _fields_ = [
        ("n_static", ctypes.c_int32),
        ("n_groups", ctypes.c_int32),
        ("statics", DriftPotential * MAX_COMPONENTS),
        ("groups", DriftSourceGroup * MAX_COMPONENTS),
        ("n_sources", ctypes.c_int64),
        ("n_segments", ctypes.c_int64),
        ("t0", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("origins", ctypes.c_void_p),
    ]


class DriftLaunch(ctypes.Structure):
    _fields_ = [
        ("method", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("block_size", ctypes.c_int32),
        ("potential", DriftPotential),
        ("n", ctypes.c_int64),
        ("y0", ctypes.c_void_p),
        ("nt", ctypes.c_int64),
        ("ts", ctypes.c_void_p),
        ("t0", ctypes.c_double),
        ("t_end", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("y_final", ctypes.c_void_p),
        ("rtol_ln", ctypes.c_double),
        ("atol_ln", ctypes.c_double),
        ("dt_one", ctypes.c_double),
        ("max_steps", ctypes.c_int64),
        ("timeout_s", ctypes.c_double),
        ("status", ctypes.c_void_p),
        ("err_code", ctypes.c_void_p),
        ("n_accepted", ctypes.c_void_p),
        ("n_rejected", ctypes.c_void_p),
        ("workspace", ctypes.c_void_p),
        ("workspace_bytes", ctypes.c_size_t),
        ("tape", ctypes.c_void_p),
        ("tape_steps", ctypes.c_int64),
        ("force_model", ctypes.POINTER(DriftForceModel)),
        ("arbitrary_times", ctypes.c_int32),
        ("tape_stride", ctypes.c_int32),
        ("y0_layout", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("y0_stride", ctypes.c_int64),
    ]


class DriftAdjointLaunch(ctypes.Structure):
    _fields_ = [
        ("method", ctypes.c_int32),
        ("block_size", ctypes.c_int32),
        ("potential", DriftPotential),
        ("n", ctypes.c_int64),
        ("nt", ctypes.c_int64),
        ("ts", ctypes.c_void_p),
        ("t0", ctypes.c_double),
        ("t_end", ctypes.c_void_p),
        ("tape", ctypes.c_void_p),
        ("tape_steps", ctypes.c_int64),
        ("n_accepted", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("grad_out", ctypes.c_void_p),
        ("grad_y0", ctypes.c_void_p),
        ("grad_params", ctypes.c_void_p),
        ("tape_stride", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libdrift_b200.so (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is not built; run __graft_entry__.build()")
        L = ctypes.CDLL(str(LIB_PATH))
        L.drift_abi_version.restype = ctypes.c_int
        L.drift_result_string.restype = ctypes.c_char_p
        L.drift_result_string.argtypes = [ctypes.c_int]
        L.drift_last_error.restype = ctypes.c_char_p
        L.drift_host_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]
        L.drift_host_free.argtypes = [ctypes.c_void_p]
        L.drift_potential_bovy.argtypes = [ctypes.POINTER(DriftPotential)] + [ctypes.c_double] * 8
        L.drift_query_workspace.argtypes = [ctypes.POINTER(DriftLaunch), ctypes.POINTER(ctypes.c_size_t)]
        L.drift_integrate.argtypes = [ctypes.POINTER(DriftLaunch), ctypes.c_void_p]
        L.drift_integrate_host.argtypes = [ctypes.POINTER(DriftLaunch)]
        L.drift_context_create.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
        L.drift_context_integrate_host.argtypes = [ctypes.c_void_p, ctypes.POINTER(DriftLaunch)]
        L.drift_context_memory.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                           ctypes.POINTER(ctypes.c_size_t)]
        L.drift_context_destroy.argtypes = [ctypes.c_void_p]
        L.drift_galpy_dopr54.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64] * 2 + [ctypes.c_double] * 3 + [ctypes.c_void_p]
        L.drift_galpy_dop853.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64] * 2 + [ctypes.c_double] * 2 + [ctypes.c_void_p]
        L.drift_force.argtypes = [ctypes.POINTER(DriftPotential), ctypes.c_int64, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p]
        L.drift_force_precision.argtypes = [ctypes.POINTER(DriftPotential), ctypes.c_int32, ctypes.c_int64,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.drift_integrate_noalloc.argtypes = [ctypes.POINTER(DriftLaunch), ctypes.c_void_p]
        L.drift_integrate_batch.argtypes = [ctypes.POINTER(DriftLaunch), ctypes.c_int32, ctypes.c_void_p]
        L.drift_integrate_adjoint.argtypes = [ctypes.POINTER(DriftAdjointLaunch), ctypes.c_void_p]
        L.drift_origin_table.argtypes = [ctypes.POINTER(DriftForceModel), ctypes.c_int64, ctypes.c_int64,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]
        L.drift_origin_table_host.argtypes = [ctypes.POINTER(DriftForceModel), ctypes.c_int64, ctypes.c_int64,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                              ctypes.c_void_p]
        L.drift_graph_create.argtypes = [ctypes.POINTER(DriftLaunch), ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_void_p)]
        L.drift_graph_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.drift_graph_destroy.argtypes = [ctypes.c_void_p]
        L.drift_autotune.argtypes = [ctypes.POINTER(DriftLaunch), ctypes.c_int64, ctypes.POINTER(DriftTuning)]
        L.drift_force_model_eval.argtypes = [ctypes.POINTER(DriftForceModel), ctypes.c_int64, ctypes.c_double,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def check(rc: int, what: str = "drift call") -> None:
    if rc != 0:
        L = lib()
        raise RuntimeError(f"{what} failed: {L.drift_result_string(rc).decode()} "
                           f"({L.drift_last_error().decode()})")


# Reference constants of the Bovy composite (shared/src/potential.rs:103-112)
# and the cutoff power-law bulge (alpha = 1.8, rc = 1.9/8, F_r(1) = -0.05).
BOVY_DEFAULTS = dict(alpha=1.8, rc=1.9 / 8.0, bulge_force=0.05, mn_amp=0.7574802019,
                     mn_a=3.0 / 8.0, mn_b=0.28 / 8.0, nfw_amp=4.852230533528, nfw_a=16.0 / 8.0)


def kepler(amp: float = 1.0) -> DriftPotential:
    return DriftPotential(kind=POT_KEPLER, amp=amp)


def kepler_cartesian(amp: float = 1.0) -> DriftPotential:
    return DriftPotential(kind=POT_KEPLER_CARTESIAN, amp=amp)


def plummer(amp: float = 1.0, b: float = 1.0) -> DriftPotential:
    return DriftPotential(kind=POT_PLUMMER, amp=amp, b=b)


def bovy(**overrides) -> DriftPotential:
    p = dict(BOVY_DEFAULTS)
    p.update(overrides)
    pot = DriftPotential()
    check(lib().drift_potential_bovy(ctypes.byref(pot), p["alpha"], p["rc"], p["bulge_force"],
                                     p["mn_amp"], p["mn_a"], p["mn_b"], p["nfw_amp"], p["nfw_a"]),
          "drift_potential_bovy")
    return pot


def force_model(statics=(), groups=(), *, origins=None, n_sources=0, n_segments=0, t0=0.0,
                dt=1.0) -> DriftForceModel:
    """A summed force: `statics` (DriftPotentials, kinds 0..3) then `groups`,
    each (kind, amp, b, first, count) with kind POT_KEPLER_CARTESIAN or
    POT_PLUMMER; `origins` is the address of the (n_segments, n_sources, 18)
    origin table (device for device entry points, host for integrate_host)."""
    m = DriftForceModel()
    if len(statics) > MAX_COMPONENTS or len(groups) > MAX_COMPONENTS:
        raise ValueError(f"at most {MAX_COMPONENTS} stationary parts and source groups")
    m.n_static = len(statics)
    for i, p in enumerate(statics):
        m.statics[i] = p
    m.n_groups = len(groups)
    for i, (kind, amp, b, first, count) in enumerate(groups):
        m.groups[i] = DriftSourceGroup(kind=kind, amp=amp, b=b, first=first, count=count)
    m.origins = origins
    m.n_sources, m.n_segments, m.t0, m.dt = n_sources, n_segments, t0, dt
    return m


def model_potential() -> DriftPotential:
    """The potential descriptor that selects drift_launch.force_model."""
    return DriftPotential(kind=POT_MODEL)


def origin_table_device(source_model: DriftForceModel, n_sources: int, nt: int, t0: float, dt: float,
                        traj_ptr: int, origins_ptr: int, stream: int = 0) -> None:
    check(lib().drift_origin_table(ctypes.byref(source_model), n_sources, nt, t0, dt,
                                   ctypes.c_void_p(traj_ptr), ctypes.c_void_p(origins_ptr),
                                   ctypes.c_void_p(stream)), "drift_origin_table")


def force_model_eval_device(model: DriftForceModel, n: int, t: float, xyz_ptr: int, acc_ptr: int,
                            stream: int = 0) -> None:
    check(lib().drift_force_model_eval(ctypes.byref(model), n, t, ctypes.c_void_p(xyz_ptr),
                                       ctypes.c_void_p(acc_ptr), ctypes.c_void_p(stream)),
          "drift_force_model_eval")


def _ptr(a) -> int | None:
    return None if a is None else a.ctypes.data


def make_launch(method: int, pot: DriftPotential, n: int, nt: int, *, rtol: float, atol: float,
                precision: int = EXACT, schedule: int = PERSISTENT, block_size: int = 0,
                dt_one: float = INITIAL_STEP_SENTINEL, max_steps: int = 0,
                timeout_s: float = 0.0, t0: float = 0.0) -> DriftLaunch:
    L = DriftLaunch()
    L.method, L.precision, L.schedule, L.block_size = method, precision, schedule, block_size
    L.potential = pot
    L.n, L.nt, L.t0 = n, nt, t0
    # LogTolerance::from_linear: the reference hands its kernels ln(tolerance).
    L.rtol_ln, L.atol_ln = math.log(rtol), math.log(atol)
    L.dt_one, L.max_steps, L.timeout_s = dt_one, max_steps, timeout_s
    return L


def integrate_host(method: int, pot: DriftPotential, y0, *, ts=None, t_end=None, nt=None,
                   t0: float = 0.0, rtol: float = 1e-12, atol: float = 1e-12,
                   precision: int = EXACT, schedule: int = PERSISTENT, block_size: int = 0,
                   dt_one: float = INITIAL_STEP_SENTINEL, max_steps: int = 0,
                   timeout_s: float = 0.0, want_out: bool = True, out=None,
                   model: DriftForceModel | None = None, arbitrary_times: bool = False,
                   context: "Context | None" = None, columns: bool = False) -> dict:
    """drift_integrate_host: host arrays in, host arrays out.  With `model`
    (whose origin table is a host array), `pot` is ignored and the stage
    integrates in the summed force.  With `context`, the call runs on that
    explicit context (drift_context_integrate_host) instead of the device's
    implicit one.  ``columns``: y0 is given as (6, n) columns
    (DRIFT_Y0_COLUMNS) instead of (n, 6) rows."""
    if columns:
        y0 = np.ascontiguousarray(y0, dtype=np.float64).reshape(6, -1)
        n = y0.shape[1]
    else:
        y0 = np.ascontiguousarray(y0, dtype=np.float64).reshape(-1, 6)
        n = y0.shape[0]
    if ts is not None:
        ts = np.ascontiguousarray(ts, dtype=np.float64)
        nt = len(ts)
    else:
        t_end = np.ascontiguousarray(t_end, dtype=np.float64)
        assert nt is not None and t_end.shape == (n,)
    L = make_launch(method, pot, n, nt, rtol=rtol, atol=atol, precision=precision,
                    schedule=schedule, block_size=block_size, dt_one=dt_one,
                    max_steps=max_steps, timeout_s=timeout_s, t0=t0)
    if model is not None:
        L.potential = model_potential()
        L.force_model = ctypes.pointer(model)
    L.arbitrary_times = int(arbitrary_times)
    if columns:
        L.y0_layout, L.y0_stride = Y0_COLUMNS, n
    if want_out and out is None:
        out = np.empty((nt, n, 6))
    res = dict(
        out=out if want_out else None,
        y_final=np.empty((n, 6)),
        status=np.empty(n, np.uint8),
        err=np.empty(n, np.int32),
        accepted=np.empty(n, np.uint32),
        rejected=np.empty(n, np.uint32),
    )
    L.y0 = _ptr(y0)
    L.ts = _ptr(ts)
    L.t_end = _ptr(t_end)
    L.out = _ptr(res["out"])
    L.y_final = _ptr(res["y_final"])
    L.status = _ptr(res["status"])
    L.err_code = _ptr(res["err"])
    L.n_accepted = _ptr(res["accepted"])
    L.n_rejected = _ptr(res["rejected"])
    if context is not None:
        check(lib().drift_context_integrate_host(context.handle(), ctypes.byref(L)),
              "drift_context_integrate_host")
    else:
        check(lib().drift_integrate_host(ctypes.byref(L)), "drift_integrate_host")
    return res


class Context:
    """An explicit host-path context (drift_context_*): its own streams and
    grow-only buffers on one device, freed by close().

        with capi.Context(device=0) as ctx:
            res = capi.integrate_host(capi.DOP853, pot, y0, ts=ts, context=ctx)
            ctx.memory()       # (device bytes, page-locked host bytes) held
    """

    def __init__(self, device: int | None = None):
        self._ptr = ctypes.c_void_p()
        check(lib().drift_context_create(-1 if device is None else int(device), ctypes.byref(self._ptr)),
              "drift_context_create")

    def handle(self) -> ctypes.c_void_p:
        if not self._ptr:
            raise RuntimeError("the context is closed")
        return self._ptr

    def memory(self) -> tuple[int, int]:
        dev, pinned = ctypes.c_size_t(0), ctypes.c_size_t(0)
        check(lib().drift_context_memory(self.handle(), ctypes.byref(dev), ctypes.byref(pinned)),
              "drift_context_memory")
        return dev.value, pinned.value

    def close(self) -> None:
        if self._ptr:
            lib().drift_context_destroy(self._ptr)
            self._ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def query_workspace(L: DriftLaunch) -> int:
    b = ctypes.c_size_t(0)
    check(lib().drift_query_workspace(ctypes.byref(L), ctypes.byref(b)), "drift_query_workspace")
    return b.value


def integrate_device(L: DriftLaunch, stream: int = 0) -> None:
    """drift_integrate on device pointers already stored in ``L``."""
    check(lib().drift_integrate(ctypes.byref(L), ctypes.c_void_p(stream)), "drift_integrate")


def integrate_device_noalloc(L: DriftLaunch, stream: int = 0) -> None:
    """drift_integrate_noalloc on device pointers already stored in ``L`` (no workspace)."""
    check(lib().drift_integrate_noalloc(ctypes.byref(L), ctypes.c_void_p(stream)),
          "drift_integrate_noalloc")


def integrate_batch_device(launches: list, stream: int = 0) -> None:
    """drift_integrate_batch on device pointers already stored in each launch."""
    arr = (DriftLaunch * len(launches))(*launches)
    check(lib().drift_integrate_batch(arr, len(launches), ctypes.c_void_p(stream)),
          "drift_integrate_batch")


def force_device(pot: DriftPotential, n: int, xyz_ptr: int, acc_ptr: int, stream: int = 0,
                 precision: int = EXACT) -> None:
    """drift_force_precision on device pointers."""
    check(lib().drift_force_precision(ctypes.byref(pot), precision, n, ctypes.c_void_p(xyz_ptr),
                                      ctypes.c_void_p(acc_ptr), ctypes.c_void_p(stream)),
          "drift_force_precision")


def exported_symbols() -> dict[str, bool]:
    L = lib()
    return {name: hasattr(L, name) for name in EXPORTED}


def integrate_adjoint_device(A: DriftAdjointLaunch, stream: int = 0) -> None:
    """drift_integrate_adjoint on device pointers already stored in ``A``."""
    check(lib().drift_integrate_adjoint(ctypes.byref(A), ctypes.c_void_p(stream)),
          "drift_integrate_adjoint")


class Graph:
    """A captured integration (drift_graph_*): replay() re-runs the launch's
    whole stream sequence with one call."""

    def __init__(self, L: DriftLaunch, stream: int):
        self._L = L  # the launch (and what it points to) must outlive the graph
        self._ptr = ctypes.c_void_p()
        check(lib().drift_graph_create(ctypes.byref(L), ctypes.c_void_p(stream), ctypes.byref(self._ptr)),
              "drift_graph_create")

    def replay(self, stream: int) -> None:
        check(lib().drift_graph_launch(self._ptr, ctypes.c_void_p(stream)), "drift_graph_launch")

    def close(self) -> None:
        if self._ptr:
            lib().drift_graph_destroy(self._ptr)
            self._ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _device_name() -> str:
    try:
        import torch

        return torch.cuda.get_device_name(torch.cuda.current_device())
    except Exception:
        return "unknown"


def _ceil_log2(v: int) -> int:
    return max(int(v) - 1, 0).bit_length()


def tuning_key(L: DriftLaunch) -> str:
    """The workload class drift_autotune caches a choice under (method,
    precision, potential, grid kind, ceil log2 of nt and n, arbitrary
    times), prefixed with the GPU's name."""
    return "|".join(str(v) for v in (_device_name(), L.method, L.precision, L.potential.kind,
                                      int(bool(L.ts)), _ceil_log2(L.nt), _ceil_log2(L.n),
                                      int(L.arbitrary_times)))


def autotune(L: DriftLaunch, sample: int = 0, cache_path=None) -> DriftTuning:
    """drift_autotune: the fastest block size and schedule for launch L.

    The library caches choices for the life of the process.  With
    ``cache_path`` (a JSON file) they also persist across processes: a
    workload class found there is returned without timing (``cached`` = 2),
    and a new choice is added to the file."""
    import json
    import os

    key = tuning_key(L) if cache_path is not None else None
    if cache_path is not None and os.path.exists(cache_path):
        with open(cache_path) as f:
            entry = json.load(f).get(key)
        if entry is not None:
            t = DriftTuning()
            t.block_size, t.schedule = int(entry["block_size"]), int(entry["schedule"])
            t.seconds, t.sample, t.cached = float(entry["seconds"]), int(entry["sample"]), 2
            return t
    t = DriftTuning()
    check(lib().drift_autotune(ctypes.byref(L), sample, ctypes.byref(t)), "drift_autotune")
    if cache_path is not None:
        table = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                table = json.load(f)
        table[key] = {"block_size": t.block_size, "schedule": t.schedule, "seconds": t.seconds,
                      "sample": t.sample}
        tmp = f"{cache_path}.tmp{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, cache_path)
    return t
