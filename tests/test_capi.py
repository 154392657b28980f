"""The C ABI library loads, exports every declared symbol and validates its
arguments on the host (no device work)."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from astrodrift_b200 import capi, serving

HEADER = Path(__file__).resolve().parent.parent / "include" / "drift_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(drift_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 11
    lib = capi.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    assert set(names) == set(capi.EXPORTED)


def test_abi_version_and_messages():
    lib = capi.lib()
    assert lib.drift_abi_version() == 5
    assert lib.drift_result_string(0) == b"success"
    assert lib.drift_result_string(1) == b"invalid argument"


def test_struct_layout_matches_header(tmp_path):
    # Compile the header with the C compiler and compare every field offset
    # with the ctypes mirror used by the tests and the benchmark.
    import subprocess

    lines = []
    structs = (("drift_potential", capi.DriftPotential), ("drift_launch", capi.DriftLaunch),
               ("drift_adjoint_launch", capi.DriftAdjointLaunch), ("drift_source_group", capi.DriftSourceGroup),
               ("drift_force_model", capi.DriftForceModel), ("drift_server_options", serving.ServerOptions),
               ("drift_server_stats", serving.ServerStats))
    for struct_name, cls in structs:
        lines.append(f'printf("{struct_name} %zu\\n", sizeof({struct_name}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{struct_name}.{field} %zu\\n", offsetof({struct_name}, {field}));')
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "drift_b200.h"\nint main(void){\n'
                   + "\n".join(lines) + "\nreturn 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    for struct_name, cls in structs:
        assert int(got[struct_name]) == ctypes.sizeof(cls)
        for field, _ in cls._fields_:
            assert int(got[f"{struct_name}.{field}"]) == getattr(cls, field).offset, field


@pytest.mark.parametrize(
    "mutate, message",
    [
        (lambda L: setattr(L, "n", 0), "n must be >= 1"),
        (lambda L: setattr(L, "nt", 1), "nt must be"),
        (lambda L: setattr(L, "method", 7), "unknown method"),
        (lambda L: setattr(L, "precision", 9), "unknown precision"),
        (lambda L: setattr(L, "schedule", 9), "unknown schedule"),
        (lambda L: setattr(L, "block_size", 48), "block_size"),
        (lambda L: setattr(L.potential, "kind", 11), "unknown potential"),
        (lambda L: setattr(L, "rtol_ln", float("nan")), "tolerances"),
        (lambda L: setattr(L, "ts", None), "either ts or t_end"),
        (lambda L: setattr(L, "y0", None), "y0 is NULL"),
        (lambda L: (setattr(L, "tape", 4096), setattr(L, "tape_steps", 8), setattr(L, "method", 0)),
         "recorded by DOP853 only"),
        (lambda L: (setattr(L, "tape", 4096), setattr(L, "tape_steps", 0)), "tape_steps"),
        (lambda L: (setattr(L, "tape", 4104), setattr(L, "tape_steps", 8)), "16-byte aligned"),
        (lambda L: setattr(L, "y0_layout", 7), "unknown y0_layout"),
        (lambda L: (setattr(L, "y0_layout", 1), setattr(L, "y0_stride", 3)), "y0_stride must be 0 or at least n"),
    ],
)
def test_invalid_launches_are_rejected_before_any_device_work(mutate, message):
    y0 = np.zeros((4, 6))
    ts = np.linspace(0.0, 1.0, 3)
    L = capi.make_launch(capi.DOP853, capi.plummer(), 4, 3, rtol=1e-10, atol=1e-10)
    L.y0 = y0.ctypes.data
    L.ts = ts.ctypes.data
    mutate(L)
    rc = capi.lib().drift_integrate(ctypes.byref(L), None)
    assert rc == 1
    assert message in capi.lib().drift_last_error().decode()


def test_persistent_schedule_requires_workspace():
    L = capi.make_launch(capi.DOP853, capi.plummer(), 4, 3, rtol=1e-10, atol=1e-10,
                         schedule=capi.PERSISTENT)
    assert capi.query_workspace(L) >= 8
    L2 = capi.make_launch(capi.DOP853, capi.plummer(), 4, 3, rtol=1e-10, atol=1e-10,
                          schedule=capi.PLAIN)
    assert capi.query_workspace(L2) == 0


def test_bovy_descriptor_normalises_bulge():
    from scipy.special import gamma, gammainc

    p = capi.bovy()
    assert p.kind == capi.POT_BOVY
    s = 1.5 - 0.5 * 1.8
    gs = gamma(s)
    assert abs(p.bulge_gamma_s - gs) < 1e-15 * gs
    # F_r(1) = -k gamma(s, 1/rc^2) = -0.05
    assert abs(p.bulge_k * gammainc(s, 1.0 / (1.9 / 8.0) ** 2) * gs - 0.05) < 1e-15


def test_host_entry_point_rejects_a_step_tape():
    y0 = np.zeros((4, 6))
    ts = np.linspace(0.0, 1.0, 3)
    L = capi.make_launch(capi.DOP853, capi.plummer(), 4, 3, rtol=1e-10, atol=1e-10)
    L.y0, L.ts = y0.ctypes.data, ts.ctypes.data
    L.tape, L.tape_steps = 4096, 8
    assert capi.lib().drift_integrate_host(ctypes.byref(L)) == 1
    assert "device" in capi.lib().drift_last_error().decode()


@pytest.mark.parametrize(
    "mutate, message",
    [
        (lambda A: setattr(A, "method", 0), "supports DOP853"),
        (lambda A: setattr(A, "tape", None), "required"),
        (lambda A: setattr(A, "grad_out", None), "required"),
        (lambda A: setattr(A, "nt", 1), "nt in"),
        (lambda A: setattr(A.potential, "kind", 9), "unknown potential"),
        (lambda A: setattr(A, "block_size", 256), "block_size"),
    ],
)
def test_invalid_adjoint_launches_are_rejected(mutate, message):
    A = capi.DriftAdjointLaunch(method=capi.DOP853, potential=capi.plummer(), n=4, nt=3, ts=4096,
                                tape=4096, tape_steps=8, n_accepted=4096, grad_out=4096, grad_y0=4096)
    mutate(A)
    assert capi.lib().drift_integrate_adjoint(ctypes.byref(A), None) == 1
    assert message in capi.lib().drift_last_error().decode()


def _model_launch(model):
    y0 = np.zeros((4, 6))
    ts = np.linspace(0.0, 1.0, 3)
    L = capi.make_launch(capi.DOP853, capi.model_potential(), 4, 3, rtol=1e-10, atol=1e-10)
    L.y0, L.ts = y0.ctypes.data, ts.ctypes.data
    if model is not None:
        L.force_model = ctypes.pointer(model)
    return L, (y0, ts, model)


@pytest.mark.parametrize(
    "make, message",
    [
        (lambda: None, "needs force_model"),
        (lambda: capi.force_model([capi.plummer()] * 3, [(capi.POT_BOVY, 1.0, 0.0, 0, 1)], origins=8,
                                  n_sources=1, n_segments=1), "only Kepler and Plummer"),
        (lambda: capi.force_model([], [(capi.POT_PLUMMER, 1.0, 0.1, 0, 2)], origins=8, n_sources=1,
                                  n_segments=1), "exceed n_sources"),
        (lambda: capi.force_model([], [(capi.POT_PLUMMER, 1.0, 0.1, 0, 1)], origins=None, n_sources=1,
                                  n_segments=1), "origin table"),
        (lambda: capi.force_model([], [(capi.POT_PLUMMER, 1.0, 0.1, 0, 1)], origins=8, n_sources=1,
                                  n_segments=1, dt=0.0), "nonzero dt"),
        (lambda: capi.force_model([capi.bovy(), capi.bovy(alpha=1.5)]), "share bulge_alpha"),
    ],
)
def test_invalid_force_models_are_rejected_before_any_device_work(make, message):
    L, keep = _model_launch(make())
    assert capi.lib().drift_integrate(ctypes.byref(L), None) == 1
    assert message in capi.lib().drift_last_error().decode()


def test_force_model_with_too_many_parts_is_rejected():
    m = capi.force_model([capi.plummer()] * 5)
    m.n_static = 12
    L, keep = _model_launch(m)
    assert capi.lib().drift_integrate(ctypes.byref(L), None) == 1
    assert "at most 11" in capi.lib().drift_last_error().decode()


INVALID_ARGUMENT = 1  # DRIFT_ERROR_INVALID_ARGUMENT


def test_context_entry_points_validate_their_arguments():
    lib = capi.lib()
    assert lib.drift_context_create(0, None) == INVALID_ARGUMENT
    L = capi.make_launch(capi.DOP853, capi.plummer(), 1, 2, rtol=1e-10, atol=1e-10)
    assert lib.drift_context_integrate_host(None, ctypes.byref(L)) == INVALID_ARGUMENT
    assert lib.drift_context_memory(None, None, None) == INVALID_ARGUMENT
    assert lib.drift_context_destroy(None) == 0


def test_server_entry_points_validate_their_arguments():
    lib = serving._lib()
    tickets = (ctypes.c_uint64 * 1)(1)
    index = ctypes.c_int32(-1)
    assert lib.drift_server_wait_any(None, tickets, 1, 0.0, ctypes.byref(index), None, None) == INVALID_ARGUMENT
    assert "empty ticket list" in lib.drift_last_error().decode()
    assert lib.drift_server_wait(None, 1, 0.0, None, None) == INVALID_ARGUMENT
    assert lib.drift_server_cancel(None, 1) == INVALID_ARGUMENT
    assert lib.drift_server_destroy(None) == 0


def test_tuning_choices_persist_in_a_json_file(tmp_path, monkeypatch):
    import json

    monkeypatch.setattr(capi, "_device_name", lambda: "NVIDIA B200")
    L = capi.make_launch(capi.DOP853, capi.plummer(), 150000, 201, rtol=1e-12, atol=1e-12)
    L.ts = 4096  # a shared grid (the key only looks at its presence)
    key = capi.tuning_key(L)
    assert key == "NVIDIA B200|1|0|1|1|8|18|0"  # DOP853, exact, Plummer, shared grid, nt<=2^8, n<=2^18
    path = tmp_path / "tuning.json"
    path.write_text(json.dumps({key: {"block_size": 96, "schedule": 2, "seconds": 0.25, "sample": 16384}}))

    def no_timing():
        raise AssertionError("a cached class must not be timed again")

    monkeypatch.setattr(capi, "lib", no_timing)
    t = capi.autotune(L, cache_path=str(path))
    assert (t.block_size, t.schedule, t.cached, t.sample) == (96, 2, 2, 16384)
