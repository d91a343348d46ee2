"""Aperture windows of batched uneven-aperture surveys (host rule, no GPU).

The windows are an extension without a reference counterpart; the engine's
C++ rule (fwi_util_window) is checked against the oracle's restatement
(oracle.window) over seeded random geometries, edges included."""
import numpy as np

from fwi2d_b200 import api
from oracle import oracle as O


def test_window_rule_matches_oracle():
    rng = np.random.default_rng(11)
    for _ in range(2000):
        nx = int(rng.integers(9, 3000))
        dh = np.float32(rng.choice([2.5, 5.0, 10.0, 12.5]))
        xs = np.float32(rng.uniform(0, (nx - 1) * dh))
        off = np.float32(rng.uniform(1.0, 1.2 * nx * dh))
        got = api.util_window(float(xs), float(off), nx, float(dh))
        want = O.window(float(xs), float(off), nx, float(dh))
        assert got == want, (nx, dh, xs, off, got, want)
        c0, w = got
        assert 0 <= c0 and c0 + w <= nx and w >= 9
        assert c0 * dh <= xs + 1e-3 and xs <= (c0 + w - 1) * dh + 1e-3


def test_window_edges_and_small_offsets():
    # tiny offsets widen to 9 columns about the source; at the edges the window is clamped
    assert api.util_window(0.0, 1.0, 100, 10.0) == (0, 9)
    assert api.util_window(990.0, 1.0, 100, 10.0) == (91, 9)
    assert api.util_window(500.0, 1.0, 100, 10.0) == O.window(500.0, 1.0, 100, 10.0)
    assert api.util_window(500.0, 1e6, 100, 10.0) == (0, 100)
    c0, w = api.util_window(505.0, 100.0, 100, 10.0)
    assert (c0, w) == (40, 22)
