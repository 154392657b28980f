"""The C ABI from a C host: a program compiled against include/drift_b200.h
and linked to libdrift_b200.so, as a foreign-language binding would use it.
Runs without a GPU: the ABI version, argument validation with its message,
the workspace query, and the no-device error of an entry point that needs a
GPU (skipped when one is present)."""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIBDIR = ROOT / "astrodrift_b200" / "_lib"

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "drift_b200.h"

int main(void)
{
    printf("abi %d\n", drift_abi_version());
    drift_launch L;
    memset(&L, 0, sizeof(L));
    L.method = DRIFT_DOP853;
    L.potential.kind = DRIFT_POT_PLUMMER;
    L.potential.amp = 1.0;
    L.potential.b = 1.0;
    L.n = 4;
    L.nt = 1; /* invalid */
    double y0[24] = {0}, ts[3] = {0.0, 0.5, 1.0};
    L.y0 = y0;
    L.ts = ts;
    int rc = drift_integrate(&L, 0);
    printf("invalid rc %d msg %s\n", rc, drift_last_error());
    L.nt = 3;
    L.schedule = DRIFT_SCHEDULE_ORDERED;
    size_t ws = 0;
    rc = drift_query_workspace(&L, &ws);
    printf("workspace rc %d bytes %zu\n", rc, ws);
    drift_context *ctx = NULL;
    rc = drift_context_create(-1, &ctx);
    printf("context rc %d %s\n", rc, drift_result_string(rc));
    drift_context_destroy(ctx);
    return 0;
}
"""


def test_a_c_program_uses_the_abi(tmp_path):
    src = tmp_path / "host.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "host"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src),
                    "-L", str(LIBDIR), "-ldrift_b200", "-o", str(exe)], check=True)
    env = dict(os.environ, LD_LIBRARY_PATH=f"{LIBDIR}:{os.environ.get('LD_LIBRARY_PATH', '')}")
    out = subprocess.run([str(exe)], capture_output=True, text=True, env=env, check=True).stdout
    lines = dict(line.split(" ", 1) for line in out.strip().splitlines())
    assert lines["abi"] == "5"
    assert lines["invalid"].startswith("rc 1 ") and "nt must be" in lines["invalid"]
    rc, size = lines["workspace"].split()[1], int(lines["workspace"].split()[3])
    assert rc == "0" and size >= 256 + 1024 + 5 * 4  # cursor, bucket counts, queue and keys
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present: the no-device path does not apply")
    assert lines["context"] == "rc 4 no CUDA device"  # DRIFT_ERROR_NO_DEVICE
