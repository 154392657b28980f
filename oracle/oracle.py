"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C restatement of the reference's CPU integrators
(lbparticles/astrodrift ``src/integrators/galpy/dopr54.rs`` and
``src/integrators/galpy/dop853.rs``).  Only the test-suite, the smoke check and
the CPU-baseline leg of ``bench.py`` load it; the product never does.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

POT_KEPLER, POT_PLUMMER, POT_BOVY = 0, 1, 2
DOPR54, DOP853 = 0, 1
INITIAL_STEP_SENTINEL = -9999.99

# Reference constants of the Bovy composite (shared/src/potential.rs:103-112)
# plus the cutoff power-law bulge (alpha = 1.8, rc = 1.9/8, F_r(1) = -0.05).
BOVY_MN_AMP = 0.7574802019
BOVY_MN_A = 3.0 / 8.0
BOVY_MN_B = 0.28 / 8.0
BOVY_NFW_AMP = 4.852230533528
BOVY_NFW_A = 16.0 / 8.0
BOVY_BULGE_ALPHA = 1.8
BOVY_BULGE_RC = 1.9 / 8.0
BOVY_BULGE_FORCE_AT_1 = 0.05


class Potential(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
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
        ("model", ctypes.c_void_p),
    ]


POT_KEPLER_CARTESIAN, POT_MODEL = 3, 4


class SourceGroup(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("pad_", ctypes.c_int32), ("amp", ctypes.c_double),
                ("b", ctypes.c_double), ("first", ctypes.c_int64), ("count", ctypes.c_int64)]


class Model(ctypes.Structure):
    _fields_ = [
        ("n_static", ctypes.c_int32),
        ("n_groups", ctypes.c_int32),
        ("statics", Potential * 11),
        ("groups", SourceGroup * 11),
        ("n_sources", ctypes.c_int64),
        ("n_segments", ctypes.c_int64),
        ("t0", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("origins", ctypes.c_void_p),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("accepted", ctypes.c_int64),
        ("rejected", ctypes.c_int64),
        ("rhs", ctypes.c_int64),
    ]


def build() -> Path:
    """Compile ``liboracle.so`` with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.oracle_force.argtypes = [ctypes.POINTER(Potential)] + [ctypes.c_double] * 3 + [dp] * 3
        _lib.oracle_lower_gamma.restype = ctypes.c_double
        _lib.oracle_lower_gamma.argtypes = [ctypes.c_double] * 3
        _lib.oracle_bovy_setup.argtypes = [ctypes.POINTER(Potential)] + [ctypes.c_double] * 8
        _lib.oracle_dopr54.restype = ctypes.c_int
        _lib.oracle_dopr54.argtypes = [
            ctypes.POINTER(Potential), dp, ctypes.c_int, ctypes.c_double, dp,
            ctypes.c_double, ctypes.c_double, ctypes.c_int64, dp,
            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(Stats),
        ]
        _lib.oracle_dop853.restype = ctypes.c_int
        _lib.oracle_dop853.argtypes = [
            ctypes.POINTER(Potential), dp, ctypes.c_int, dp, ctypes.c_double,
            ctypes.c_double, ctypes.c_int64, dp, ctypes.POINTER(Stats),
        ]
        _lib.oracle_dop853_tape.restype = ctypes.c_int
        _lib.oracle_dop853_tape.argtypes = [
            ctypes.POINTER(Potential), dp, ctypes.c_int, dp, ctypes.c_double,
            ctypes.c_double, ctypes.c_int64, dp, ctypes.POINTER(Stats), dp, ctypes.c_int64,
        ]
        _lib.oracle_integrate_batch.restype = ctypes.c_int64
        _lib.oracle_integrate_batch.argtypes = [
            ctypes.c_int, ctypes.POINTER(Potential), ctypes.c_int64, dp, ctypes.c_int, dp,
            ctypes.c_double, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_int64, dp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
        ]
        _lib.oracle_force_t.argtypes = [ctypes.POINTER(Potential)] + [ctypes.c_double] * 4 + [dp] * 3
        _lib.oracle_origin_table.argtypes = [ctypes.POINTER(Potential), ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_double, ctypes.c_double, dp, dp]
        _lib.oracle_grid_sample.restype = ctypes.c_double
        _lib.oracle_grid_sample.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_int64]
    return _lib


def kepler(amp: float = 1.0) -> Potential:
    return Potential(kind=POT_KEPLER, amp=amp)


def plummer(amp: float = 1.0, b: float = 1.0) -> Potential:
    return Potential(kind=POT_PLUMMER, amp=amp, b=b)


def bovy(mn_amp: float = BOVY_MN_AMP, mn_a: float = BOVY_MN_A, mn_b: float = BOVY_MN_B,
         nfw_amp: float = BOVY_NFW_AMP, nfw_a: float = BOVY_NFW_A) -> Potential:
    p = Potential()
    lib().oracle_bovy_setup(ctypes.byref(p), BOVY_BULGE_ALPHA, BOVY_BULGE_RC, BOVY_BULGE_FORCE_AT_1,
                            mn_amp, mn_a, mn_b, nfw_amp, nfw_a)
    return p


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def model(statics=(), groups=(), *, origins=None, t0=0.0, dt=1.0, n_sources=0) -> Potential:
    """A summed force: `statics` (Potentials) then `groups`, each
    (kind, amp, b, first, count) with kind POT_KEPLER_CARTESIAN or POT_PLUMMER,
    placed by `origins` (n_segments, n_sources, 18).  The returned Potential
    keeps the model and table alive."""
    m = Model()
    m.n_static = len(statics)
    for i, p in enumerate(statics):
        m.statics[i] = p
    m.n_groups = len(groups)
    for i, (kind, amp, b, first, count) in enumerate(groups):
        m.groups[i] = SourceGroup(kind=kind, amp=amp, b=b, first=first, count=count)
    keep = None
    if origins is not None:
        keep = np.ascontiguousarray(origins, dtype=np.float64)
        m.origins = keep.ctypes.data
        m.n_segments = keep.shape[0]
        m.n_sources = keep.shape[1]
    else:
        m.n_sources = n_sources
    m.t0, m.dt = t0, dt
    pot = Potential(kind=POT_MODEL)
    pot.model = ctypes.addressof(m)
    pot._keep = (m, keep)
    return pot


def origin_table(source_pot: Potential, trajectory: np.ndarray, t0: float, dt: float) -> np.ndarray:
    """Quintic Hermite origin table (nt-1, n_sources, 18) of a source trajectory (nt, n_sources, 6)."""
    traj = np.ascontiguousarray(trajectory, dtype=np.float64)
    nt, ns = traj.shape[0], traj.shape[1]
    out = np.zeros((nt - 1, ns, 18))
    lib().oracle_origin_table(ctypes.byref(source_pot), ns, nt, t0, dt, _dptr(traj), _dptr(out))
    return out


def force_t(pot: Potential, t: float, x: float, y: float, z: float) -> tuple[float, float, float]:
    out = (ctypes.c_double(), ctypes.c_double(), ctypes.c_double())
    lib().oracle_force_t(ctypes.byref(pot), t, x, y, z, *(ctypes.byref(o) for o in out))
    return tuple(o.value for o in out)  # type: ignore[return-value]


def force(pot: Potential, x: float, y: float, z: float) -> tuple[float, float, float]:
    out = (ctypes.c_double(), ctypes.c_double(), ctypes.c_double())
    lib().oracle_force(ctypes.byref(pot), x, y, z, *(ctypes.byref(o) for o in out))
    return tuple(o.value for o in out)  # type: ignore[return-value]


def dopr54(pot: Potential, yo, t, rtol_ln: float, atol_ln: float,
           dt_one: float = INITIAL_STEP_SENTINEL, max_steps: int = 0):
    """One particle through the DOPR54 restatement; returns (result, err, status, stats)."""
    yo = np.ascontiguousarray(yo, dtype=np.float64)
    t = np.ascontiguousarray(t, dtype=np.float64)
    res = np.zeros((len(t), 6))
    err = ctypes.c_int(0)
    st = Stats()
    status = lib().oracle_dopr54(ctypes.byref(pot), _dptr(yo), len(t), dt_one, _dptr(t),
                                 rtol_ln, atol_ln, max_steps, _dptr(res), ctypes.byref(err),
                                 ctypes.byref(st))
    return res, err.value, status, st


def dop853(pot: Potential, y0, t, rtol_ln: float, atol_ln: float, max_steps: int = 0):
    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    t = np.ascontiguousarray(t, dtype=np.float64)
    res = np.zeros((len(t), 6))
    st = Stats()
    status = lib().oracle_dop853(ctypes.byref(pot), _dptr(y0), len(t), _dptr(t), rtol_ln,
                                 atol_ln, max_steps, _dptr(res), ctypes.byref(st))
    return res, status, st


def dop853_tape(pot: Potential, y0, t, rtol_ln: float, atol_ln: float, tape_steps: int = 100000):
    """DOP853 with its accepted steps recorded: returns (result, status, stats,
    tape (accepted, 8) of (t_old, h, y_old[6]))."""
    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    t = np.ascontiguousarray(t, dtype=np.float64)
    res = np.zeros((len(t), 6))
    tape = np.zeros((tape_steps, 8))
    st = Stats()
    status = lib().oracle_dop853_tape(ctypes.byref(pot), _dptr(y0), len(t), _dptr(t), rtol_ln,
                                      atol_ln, 0, _dptr(res), ctypes.byref(st), _dptr(tape),
                                      tape_steps)
    return res, status, st, tape[: min(st.accepted, tape_steps)].copy()


def integrate_batch(method: int, pot: Potential, y0: np.ndarray, *, ts=None, t0: float = 0.0,
                    t_end=None, nt: int | None = None, rtol: float = 1e-12, atol: float = 1e-12,
                    dt_one: float = INITIAL_STEP_SENTINEL, max_steps: int = 0,
                    threads: int | None = None, want_output: bool = True,
                    arbitrary_times: bool = False) -> dict:
    """Batch integration restating src/dispatch/cpu.rs:53-89.

    Tolerances are linear; they are converted to natural logarithms with the
    host libm, as ``LogTolerance::from_linear`` does (src/integrators/galpy/mod.rs:19-24).
    """
    y0 = np.ascontiguousarray(y0, dtype=np.float64).reshape(-1, 6)
    n = y0.shape[0]
    if ts is not None:
        ts = np.ascontiguousarray(ts, dtype=np.float64)
        nt = len(ts)
        te = None
    else:
        te = np.ascontiguousarray(t_end, dtype=np.float64)
        assert nt is not None
    out = np.zeros((nt, n, 6)) if want_output else None
    status = np.zeros(n, np.int32)
    err = np.zeros(n, np.int32)
    acc = np.zeros(n, np.int64)
    rej = np.zeros(n, np.int64)
    rhs = np.zeros(n, np.int64)
    if threads is None:
        threads = os.cpu_count() or 1
    fails = lib().oracle_integrate_batch(
        method, ctypes.byref(pot), n, _dptr(y0), nt,
        _dptr(ts) if ts is not None else None, t0,
        _dptr(te) if te is not None else None,
        math.log(rtol), math.log(atol), dt_one, max_steps,
        _dptr(out) if out is not None else None,
        status.ctypes.data, err.ctypes.data, acc.ctypes.data, rej.ctypes.data, rhs.ctypes.data,
        threads, int(arbitrary_times))
    return dict(out=out, status=status, err=err, accepted=acc, rejected=rej, rhs=rhs,
                failures=int(fails))


def grid_sample(start: float, end: float, steps: int, index: int) -> float:
    return lib().oracle_grid_sample(start, end, steps, index)
