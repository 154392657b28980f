"""drift_integrate_host's streamed copy-out.

A large persistent or ordered request whose trajectory goes to page-locked
memory runs as one launch whose queue completes particle chunks in order,
each chunk copied out while the launch continues.  Its results must equal,
bit for bit, those of the chunked path the same request takes when its
destination is pageable memory (separate launches per particle chunk), for
uneven per-particle spans and for a shared grid."""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi
from astrodrift_b200.serving import PinnedArray
from astrodrift_b200.workloads import bovy_disc, plummer_sphere

pytestmark = pytest.mark.gpu


def _both(method, pot, y0, **kw):
    n = len(y0)
    nt = len(kw["ts"]) if "ts" in kw else kw["nt"]
    pinned = PinnedArray((nt, n, 6))
    a = capi.integrate_host(method, pot, y0, out=pinned.array, **kw)  # streamed
    b = capi.integrate_host(method, pot, y0, **kw)                    # pageable: chunked
    return a, b, pinned


@pytest.mark.parametrize("schedule", [capi.ORDERED, capi.PERSISTENT])
def test_streamed_equals_chunked_uneven_bovy(cuda_device, schedule):
    y0, t_end = bovy_disc(150_000, seed=21)
    t_end = 10.0 + (t_end - 10.0) * 0.1  # spans 10 .. 109
    a, b, pinned = _both(capi.DOP853, capi.bovy(), y0, t_end=t_end, nt=41, rtol=1e-10, atol=1e-10,
                         precision=capi.FMA, schedule=schedule)
    assert (a["status"] == 0).all()
    np.testing.assert_array_equal(a["out"], b["out"])
    np.testing.assert_array_equal(a["accepted"], b["accepted"])
    np.testing.assert_array_equal(a["y_final"], b["y_final"])
    assert np.isfinite(a["out"]).all()
    pinned.free()


def test_streamed_equals_chunked_shared_grid_plummer(cuda_device):
    y0 = plummer_sphere(100_003, seed=22)  # not a multiple of the chunk length
    a, b, pinned = _both(capi.DOP853, capi.plummer(1.0, 1.0), y0, ts=np.linspace(0.0, 20.0, 33), rtol=1e-11,
                         atol=1e-11, precision=capi.EXACT, schedule=capi.ORDERED)
    np.testing.assert_array_equal(a["out"], b["out"])
    np.testing.assert_array_equal(a["rejected"], b["rejected"])
    pinned.free()
